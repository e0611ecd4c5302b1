"""bbt_pack_bases (host code, no device needed): the BBT_BASES_2BIT layout of
random byte strings against a numpy model -- base g at bits 2 (g % 16) of word
g / 16 (A/a = 0, C/c = 1, G/g = 2, T/t = 3), validity bit g % 32 of word g / 32
set exactly for ACGTacgt, the count of other bytes -- for every length from 0
to a few words past a word boundary and for long strings split over the
library's host threads."""
import ctypes

import numpy as np
import pytest

CODES = {ord(c): i for i, c in enumerate("ACGT")}
CODES.update({ord(c): i for i, c in enumerate("acgt")})


@pytest.fixture(scope="module")
def lib():
    from biobloom_b200 import _lib
    return _lib


def _pack(L, seq):
    n = len(seq)
    words = np.full((n + 15) // 16 + 1, 0xFFFFFFFF, dtype=np.uint32)
    valid = np.full((n + 31) // 32 + 1, 0xFFFFFFFF, dtype=np.uint32)
    bad = ctypes.c_uint64()
    buf = np.frombuffer(seq or b"\0", dtype=np.uint8)
    L.check(L.lib().bbt_pack_bases(buf.ctypes.data, n, words.ctypes.data, valid.ctypes.data,
                                   ctypes.byref(bad)))
    return words, valid, bad.value


def _model(seq):
    a = np.frombuffer(seq, dtype=np.uint8)
    ok = np.isin(a, np.array(sorted(CODES), dtype=np.uint8))
    code = np.array([CODES.get(int(c), 0) for c in a], dtype=np.uint32)
    return code, ok


def _check(L, seq):
    words, valid, bad = _pack(L, seq)
    code, ok = _model(seq)
    n = len(seq)
    g = np.arange(n)
    got_code = (words[g // 16] >> (2 * (g % 16)).astype(np.uint32)) & 3
    got_ok = (valid[g // 32] >> (g % 32).astype(np.uint32)) & 1
    assert np.array_equal(got_ok.astype(bool), ok)
    assert np.array_equal(got_code[ok], code[ok])
    assert bad == int((~ok).sum())
    # the words past the last base are not written
    assert words[(n + 15) // 16] == 0xFFFFFFFF and valid[(n + 31) // 32] == 0xFFFFFFFF


def test_every_length_around_word_boundaries(lib):
    rng = np.random.default_rng(3)
    alphabet = np.frombuffer(b"ACGTacgtNnRYx-", dtype=np.uint8)
    for n in range(0, 100):
        _check(lib, rng.choice(alphabet, n).tobytes())


def test_long_strings_and_any_byte(lib):
    rng = np.random.default_rng(4)
    for n in (1 << 20, (1 << 22) + 37):
        s = rng.choice(np.frombuffer(b"ACGTACGTACGTacgtN", dtype=np.uint8), n)
        s[rng.integers(0, n, 1000)] = rng.integers(0, 256, 1000, dtype=np.uint8)
        _check(lib, s.tobytes())
