"""The C ABI library: it loads without a GPU, exports every function that
include/*.h declare, and its host-only entry points (synthetic workloads)
work on the CPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    inc = os.path.join(ROOT, "include")
    names = set()
    for h in sorted(os.listdir(inc)):
        if h.endswith(".h"):
            txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(inc, h)).read(), flags=re.S)
            names.update(re.findall(r"\b(bbt_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from biobloom_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from biobloom_b200 import build_native
        build_native.build()
    return _lib.lib()


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("bbt_open", "bbt_classify_batch", "bbt_summary", "bbt_close", "bbt_last_error",
              "bbt_make_filter", "bbt_filter_files", "bbt_filter_pair_files", "bbt_mibf_open",
              "bbt_mibf_classify_batch", "bbt_mibf_make", "bbt_mibf_filter_files"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    from biobloom_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert getattr(lib, n) is not None


def test_open_without_device_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from biobloom_b200 import _lib
    p = _lib.Params()
    lib.bbt_default_params(ctypes.byref(p))
    assert abs(p.score - 0.15) < 1e-12 and p.streak_threshold == 3
    ctx = ctypes.c_void_p()
    path = os.path.join(ROOT, "tests", "golden", "bbt", "f0.bf").encode()
    arr = (ctypes.c_char_p * 1)(path)
    rc = lib.bbt_open(arr, 1, ctypes.byref(p), ctypes.byref(ctx))
    assert rc == -8  # BBT_ERR_NODEVICE
    assert b"no CUDA device" in lib.bbt_last_error(None)


def test_synthetic_generators_are_deterministic(lib):
    from biobloom_b200 import synth
    g1 = synth.genome(5, 200000, gc=0.41, repeat_frac=0.2, rep_min=300, rep_max=600,
                      div_min=0.1, div_max=0.2)
    g2 = synth.genome(5, 200000, gc=0.41, repeat_frac=0.2, rep_min=300, rep_max=600,
                      div_min=0.1, div_max=0.2)
    assert np.array_equal(g1, g2)
    assert set(np.unique(g1).tolist()) <= set(b"ACGT")
    gc = np.isin(g1, np.frombuffer(b"GC", dtype=np.uint8)).mean()
    assert abs(gc - 0.41) < 0.01
    p = synth.read_params(50, 300, long_frac=0.05, long_min=300, long_max=10000, sub_rate=0.01)
    s, off, _, src = synth.reads(9, [g1], [0.7], 5000, p)
    lens = np.diff(off)
    assert lens.min() >= 50 and lens.max() <= 10000
    assert abs((src == 0).mean() - 0.7) < 0.03
    s2, off2, _, _ = synth.reads(9, [g1], [0.7], 5000, p)
    assert np.array_equal(s[:off[-1]], s2[:off2[-1]])
    # a read from the genome (no errors) occurs in it, on one strand
    p0 = synth.read_params(100, 100)
    s, off, _, src = synth.reads(3, [g1], [1.0], 20, p0)
    gb = g1.tobytes()
    rc = gb.translate(bytes.maketrans(b"ACGT", b"TGCA"))[::-1]
    for i in range(20):
        r = s[off[i]:off[i + 1]].tobytes()
        assert r in gb or r in rc
