"""Failures on the host, without a GPU: every unusable input file is refused
with its BBT_ERR_* code and a message before any device work, where the
reference prints a message and exits (BioBloomClassifier.cpp:54-57 for an
input it cannot open, the BloomFilter / BloomFilterInfo constructors for
filter files, MIBFClassifier.hpp:56-60 for a missing _ids.txt)."""
import ctypes
import os
import shutil

import pytest

from tests.fixtures import golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MIBF = os.path.join(ROOT, "tests", "golden", "mibf")


@pytest.fixture(scope="module")
def L():
    from biobloom_b200 import _lib
    _lib.lib()
    return _lib


def _copy_filter(tmp_path, name="f0"):
    shutil.copy(golden(f"{name}.bf"), tmp_path / "x.bf")
    shutil.copy(golden(f"{name}.txt"), tmp_path / "x.txt")
    return str(tmp_path / "x.bf")


def _open(L, path):
    ctx = ctypes.c_void_p()
    arr = (ctypes.c_char_p * 1)(path.encode())
    rc = L.lib().bbt_open(arr, 1, None, ctypes.byref(ctx))
    msg = L.lib().bbt_last_error(None).decode()
    if rc == 0:
        L.lib().bbt_close(ctx)
    return rc, msg


def test_missing_info_file(L, tmp_path):
    p = _copy_filter(tmp_path)
    os.unlink(tmp_path / "x.txt")
    rc, msg = _open(L, p)
    assert rc == -2 and "x.txt cannot be opened" in msg


def test_info_file_without_filter_id(L, tmp_path):
    p = _copy_filter(tmp_path)
    txt = (tmp_path / "x.txt").read_text().replace("filter_id=f0\n", "")
    (tmp_path / "x.txt").write_text(txt)
    rc, msg = _open(L, p)
    assert rc == -3 and "filter_id" in msg


def test_missing_filter_file(L, tmp_path):
    p = _copy_filter(tmp_path)
    os.unlink(p)
    rc, msg = _open(L, p)
    assert rc == -2 and "cannot be opened" in msg


@pytest.mark.parametrize("bad", [b"[NotAFilter]\n", b"[BTLBloomFilter]\nFormat = 1\n"
                                 b"BloomFilterSize = 12345\nHashNum = 3\nKmerSize = 25\n"
                                 b"[HeaderEnd]\n", b""])
def test_bad_header(L, tmp_path, bad):
    p = _copy_filter(tmp_path)
    with open(p, "wb") as f:
        f.write(bad)
    rc, msg = _open(L, p)
    assert rc == -3 and "x.bf" in msg


def test_short_payload(L, tmp_path):
    p = _copy_filter(tmp_path)
    data = open(p, "rb").read()
    with open(p, "wb") as f:
        f.write(data[:-100])
    rc, msg = _open(L, p)
    assert rc == -3 and "shorter" in msg


def test_later_filter_is_checked_too(L, tmp_path):
    """Every path is checked before any is loaded (the reference loads the
    filters in -f order and exits at the first bad one)."""
    good = _copy_filter(tmp_path)
    ctx = ctypes.c_void_p()
    arr = (ctypes.c_char_p * 2)(good.encode(), str(tmp_path / "none.bf").encode())
    rc = L.lib().bbt_open(arr, 2, None, ctypes.byref(ctx))
    assert rc == -2 and "none" in L.lib().bbt_last_error(None).decode()


def _mibf_copy(tmp_path):
    for ext in (".bf", ".sdsl", "_ids.txt"):
        shutil.copy(os.path.join(MIBF, "km" + ext), tmp_path / ("m" + ext))
    return str(tmp_path / "m.bf")


def _mibf_open(L, path):
    p = L.MibfParams()
    L.lib().bbt_mibf_default_params(ctypes.byref(p))
    ctx = ctypes.c_void_p()
    rc = L.lib().bbt_mibf_open_host(path.encode(), ctypes.byref(p), ctypes.byref(ctx))
    msg = L.lib().bbt_mibf_last_error(None).decode()
    if rc == 0:
        L.lib().bbt_mibf_close(ctx)
    return rc, msg


def test_mibf_opens(L, tmp_path):
    rc, msg = _mibf_open(L, _mibf_copy(tmp_path))
    assert rc == 0, msg


def test_mibf_missing_ids_file(L, tmp_path):
    p = _mibf_copy(tmp_path)
    os.unlink(tmp_path / "m_ids.txt")
    rc, msg = _mibf_open(L, p)
    assert rc == -2 and "A corresponding id file is needed" in msg


def test_mibf_bad_header(L, tmp_path):
    p = _mibf_copy(tmp_path)
    with open(p, "wb") as f:
        f.write(b"[BTLMIBloomFilter]\nFormat = 9\n[HeaderEnd]\n")
    rc, msg = _mibf_open(L, p)
    assert rc == -3


def test_mibf_short_id_array(L, tmp_path):
    p = _mibf_copy(tmp_path)
    data = open(p, "rb").read()
    with open(p, "wb") as f:
        f.write(data[:-1000])
    rc, msg = _mibf_open(L, p)
    assert rc in (-2, -3) and msg


def test_mibf_missing_filter(L, tmp_path):
    rc, msg = _mibf_open(L, str(tmp_path / "none.bf"))
    assert rc == -2 and "cannot be opened" in msg


def test_open_devices_arguments(L, tmp_path):
    """bbt_open_devices checks its filters on the host first, like bbt_open,
    and refuses an empty device list."""
    p = _copy_filter(tmp_path)
    arr = (ctypes.c_char_p * 1)(p.encode())
    ctx = ctypes.c_void_p()
    devs = (ctypes.c_int * 2)(0, 0)
    assert L.lib().bbt_open_devices(arr, 1, None, devs, 0, ctypes.byref(ctx)) == -1
    os.unlink(tmp_path / "x.txt")
    assert L.lib().bbt_open_devices(arr, 1, None, devs, 2, ctypes.byref(ctx)) == -2
