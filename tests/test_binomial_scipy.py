"""The binomial distribution behind BINOMIAL scoring (calcMinCount,
calcProbMatches: Common/SeqEval.h:199-216) and the miBF minimum counts
(MIBFClassifier::getMinCount, BioBloomCategorizer/MIBFClassifier.hpp:930-939)
comes from Boost, which is absent here.  The reference is compiled against a
stand-in (oracle/shim/boost/math/distributions/binomial.hpp) and the product
carries its own quantile; both are checked here against scipy.stats.binom, an
independent implementation (regularised incomplete beta), on a grid that
covers the call sites: n up to 20000 frames, p from 1e-6 to 0.5, q down to
1e-13.

Boost's quantile(complement(binomial(n, p), q)) under integer_round_up is the
smallest integer x with P(X > x) <= q (scipy: the first x whose sf is <= q).
Where P(X > x) lies within 1e-9 (relative) of q, the two sides of the
comparison may round either way, and either neighbour is accepted."""
import ctypes
import os

import numpy as np
import pytest

scipy_stats = pytest.importorskip("scipy.stats")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NS = [1, 2, 5, 24, 126, 150, 276, 1000, 4951, 9976, 20000]
PS = [1e-6, 1e-4, 0.003, 0.075, 0.2, 0.4217, 0.5]
QS = [0.5, 0.1, 1e-2, 1e-4, 1e-6, 1e-9, 1e-11, 1e-13]
REL = 1e-9


@pytest.fixture(scope="module")
def shim():
    path = os.path.join(ROOT, "oracle", "_build", "libshimbinom.so")
    if not os.path.exists(path):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       capture_output=True)
    L = ctypes.CDLL(path)
    L.shim_binom_sf.restype = ctypes.c_double
    L.shim_binom_sf.argtypes = [ctypes.c_uint, ctypes.c_double, ctypes.c_uint]
    L.shim_binom_quantile.restype = ctypes.c_uint
    L.shim_binom_quantile.argtypes = [ctypes.c_uint, ctypes.c_double, ctypes.c_double]
    return L


def _want_quantile(n, p, q):
    """(x, tie): the smallest x with scipy's P(X > x) <= q, and whether the
    neighbour x - 1 or x is within rounding of q."""
    sf = scipy_stats.binom.sf(np.arange(n + 1), n, p)
    x = int(np.argmax(sf <= q)) if (sf <= q).any() else n
    tie = abs(sf[x] - q) <= REL * q or (x > 0 and abs(sf[x - 1] - q) <= REL * q)
    return x, tie


def _check_quantile(got, n, p, q):
    want, tie = _want_quantile(n, p, q)
    if tie:
        assert got in (want - 1, want, want + 1), (n, p, q, got, want)
    else:
        assert got == want, (n, p, q, got, want)


@pytest.mark.parametrize("n", NS)
def test_shim_quantile_matches_scipy(shim, n):
    for p in PS:
        for q in QS:
            _check_quantile(shim.shim_binom_quantile(n, p, q), n, p, q)


@pytest.mark.parametrize("n", NS)
def test_shim_upper_tail_matches_scipy(shim, n):
    for p in PS:
        xs = sorted(set([0, 1, n // 10, int(n * p), int(n * p) + 3, n // 2, n - 1]))
        for x in xs:
            if x < 0 or x > n:
                continue
            got = shim.shim_binom_sf(n, p, x)
            want = scipy_stats.binom.sf(x, n, p)
            if want < 1e-280:
                assert got < 1e-270, (n, p, x, got, want)
            else:
                assert abs(got - want) <= 1e-9 * want + 1e-300, (n, p, x, got, want)


@pytest.mark.parametrize("n", NS)
def test_product_min_count_matches_scipy(n):
    """The product's host-side quantile (bbt_mibf_min_count; the BINOMIAL
    threshold table uses the same routine): max(1, quantile) with
    q = score / (ids - 1)."""
    from biobloom_b200 import _lib as L
    lib = L.lib()
    for p in PS:
        for q in QS:
            got = lib.bbt_mibf_min_count(n, p, q, 2)
            want, tie = _want_quantile(n, p, q)
            want = max(1, want)
            if tie:
                assert got in (want - 1, want, want + 1) or (got == 1 and want <= 2), (n, p, q)
            else:
                assert got == want, (n, p, q, got, want)
