"""miBF path on the CPU: the oracle against the reference MI categorizer's own
output (tests/golden/mibf/, made by tests/golden/make_golden_mibf.py), and the
product's host-side pieces (names, frame probabilities, minCount, record and
summary text) against the oracle and the golden files.  No GPU needed."""
import os

import numpy as np
import pytest

from tests import mibf_util as mu
from tests import oracle_lib

CASES = sorted(mu.CASES)


def _expected(case):
    with open(mu.g(f"mi_{case}.tsv")) as f:
        return f.read()


@pytest.mark.parametrize("case", CASES)
def test_oracle_records_match_reference(case):
    results, names, o, recs = mu.oracle_results(case)
    paired = mu.CASES[case][2]
    text = []
    for i, (res, sat) in enumerate(results):
        if o["hit_only"] and not res:
            continue
        for m in range(2 if paired else 1):
            name, comment, seq, qual = recs[m][i]
            text.append(mu.format_record(names, o["out"], name, comment, seq, qual, res, sat))
    assert "".join(text) == _expected(case)


@pytest.mark.parametrize("case", [c for c in CASES if mu.CASES[c][2] is not None])
def test_oracle_summary_matches_reference(case):
    results, names, o, _ = mu.oracle_results(case)
    with open(mu.g(f"mi_{case}_summary.tsv")) as f:
        want = f.read()
    assert mu.summary_text(names, results, bool(mu.CASES[case][2]), o["hit_only"]) == want


def test_golden_cases_exercise_the_semantics():
    """The fixtures hold multi-matches, saturated frames, empty results and
    best-hit disagreement, so the cases above test those branches."""
    ss, _, _, _ = mu.oracle_results("ss_se")
    assert any(len(r) > 1 for r, _ in ss)
    assert any(s > 0 for _, s in ss)
    assert any(not r for r, _ in ss)
    m2, _, _, _ = mu.oracle_results("ss_se_s50_m2")
    assert sum(len(r) > 1 for r, _ in m2) > sum(len(r) > 1 for r, _ in ss)
    b, _, _, _ = mu.oracle_results("ss_se_a3_b")
    a3 = oracle_lib.MIBF.load(mu.g("ss.bf"))
    assert a3.f.nseeds == 3 and len(b) == len(ss)


def _host(case_prefix, **kw):
    from biobloom_b200.mibf import MIBFClassifier
    return MIBFClassifier(mu.g(f"{case_prefix}.bf"), host_only=True, **kw)


@pytest.mark.parametrize("prefix", ["ss", "km"])
@pytest.mark.parametrize("fm", [1, 2, 3, 4])
def test_product_frame_probs_equal_oracle(prefix, fm):
    mc = _host(prefix, frame_matches=fm)
    f = oracle_lib.MIBF.load(mu.g(f"{prefix}.bf"))
    allowed = 0 if (fm > f.f.h or f.f.nseeds == 0) else f.f.h - fm
    want, sat = f.frame_probs(mc.num_ids, allowed)
    got, rate = mc.frame_probs()
    assert got.tobytes() == want.tobytes()
    assert rate == sat
    assert mc.names == mu.names_of(prefix)


def test_product_min_count_equals_oracle_grid():
    """bbt_mibf_min_count skips the pmf terms that are exactly 0.0; the result
    must equal the oracle's full top-down sum everywhere."""
    from biobloom_b200 import _lib as L
    lib = L.lib()
    rng = np.random.default_rng(7)
    ns = [1, 2, 5, 25, 64, 65, 126, 150, 276, 500, 1000, 2976, 5000, 9976, 20000]
    ps = [0.0, 1e-9, 1e-6, 1e-4, 1e-3, 3e-3, 0.01, 0.05, 0.2, 0.5, 0.9, 0.999, 1.0]
    ps += list(rng.uniform(0, 0.02, 8))
    for n in ns:
        for p in ps:
            for nids in (2, 9, 501):
                for score in (1e-10, 1e-5, 0.5):
                    want = max(1, oracle_lib.binom_upper_quantile(n, float(p), score / (nids - 1)))
                    got = lib.bbt_mibf_min_count(n, float(p), score, nids)
                    assert got == want, (n, p, nids, score)


@pytest.mark.parametrize("case", CASES)
def test_product_record_text_matches_reference(case):
    """The product's record formatter over the oracle's results reproduces the
    reference CLI's stdout byte for byte."""
    from biobloom_b200 import _lib as L
    results, names, o, recs = mu.oracle_results(case)
    prefix = mu.CASES[case][0]
    paired = mu.CASES[case][2]
    mc = _host(prefix)
    out_type = {"tsv": L.MIBF_OUT_TSV, "fa": L.MIBF_OUT_FASTA, "fq": L.MIBF_OUT_FASTQ}[o["out"]]
    text = []
    for i, (res, sat) in enumerate(results):
        if o["hit_only"] and not res:
            continue
        for m in range(2 if paired else 1):
            name, comment, seq, qual = recs[m][i]
            text.append(mc.format_record(name, comment, seq, qual, res, sat, out_type))
    assert "".join(text) == _expected(case)


@pytest.mark.parametrize("case", ["ss_se", "ss_pe", "km_se"])
def test_product_min_counts_for_fixture_reads(case):
    results, names, o, recs = mu.oracle_results(case)
    prefix, _, paired = mu.CASES[case]
    mc = _host(prefix)
    f = oracle_lib.MIBF.load(mu.g(f"{prefix}.bf"))
    probs, _ = f.frame_probs(len(names), 0 if f.f.nseeds == 0 else f.f.h - 1)
    fcs = {mu.frame_count(len(recs[0][i][2]), len(recs[1][i][2]) if paired else 0, f.f.k,
                          bool(paired)) for i in range(len(recs[0]))}
    for fc in sorted(x for x in fcs if x):
        assert mc.min_counts(fc) == mu.min_counts(fc, probs, 1e-10)


def test_names_file_drops_unterminated_last_line(tmp_path):
    """MIBFClassifier.hpp:67-76 keeps a line only if the stream is still good
    after it, so a last line without a newline is not read."""
    import shutil
    for ext in (".bf", ".sdsl"):
        shutil.copy(mu.g("ss" + ext), tmp_path / ("x" + ext))
    with open(tmp_path / "x_ids.txt", "w") as fh:
        fh.write("1\ta\n2\tb\n3\tc")
    from biobloom_b200.mibf import MIBFClassifier
    mc = MIBFClassifier(str(tmp_path / "x.bf"), host_only=True)
    assert mc.names == ["repeat", "a", "b"]


def test_missing_ids_file_is_an_error(tmp_path):
    import shutil
    from biobloom_b200 import BBTError
    from biobloom_b200.mibf import MIBFClassifier
    for ext in (".bf", ".sdsl"):
        shutil.copy(mu.g("ss" + ext), tmp_path / ("y" + ext))
    with pytest.raises(BBTError, match="id file is needed"):
        MIBFClassifier(str(tmp_path / "y.bf"), host_only=True)


def test_st_hash_symmetry_and_oracle_reference_binary():
    """The spaced-seed restatement has the symmetry Tests/ntHashTests.cpp
    asserts: hash(seed, x) == hash(reverse(seed), revcomp(x))."""
    rng = np.random.default_rng(3)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    oracle_lib._mibf_lib()
    for _ in range(200):
        k = int(rng.integers(5, 33))
        seed = "".join(rng.choice(["0", "1"], k))
        x = bytes(rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), k))
        rc = x.translate(comp)[::-1]
        a = oracle_lib.lib().oracle_st_hash(seed.encode(), k, x)
        b = oracle_lib.lib().oracle_st_hash(seed[::-1].encode(), k, rc)
        assert a == b
    ref = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                       "_ref", "ntHashTests")
    if os.path.exists(ref):
        import subprocess
        assert subprocess.run([ref], capture_output=True).returncode == 0
