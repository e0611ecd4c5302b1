"""Python face of the serving engine (include/bbt_server.h): a request loop
with a Bloom-filter context and a miBF context resident on one GPU.

    srv = Server(bloom=BioBloomClassifier([...]), mibf=MIBFClassifier("t.bf"))
    req = srv.submit_bloom(seq, off)          # returns at once
    stats = srv.wait(req)                     # req.hits, req.category filled
    req = srv.submit_mibf(seq, off, max_hits=4)
    stats = srv.wait(req)                     # req.hits, req.n_hits, req.sat filled
    srv.close()

Host inputs may be numpy arrays or pinned torch tensors (pinned memory is
copied to the device without staging).  Results land in numpy arrays (pinned
when torch is available) that belong to the request object.
"""
import ctypes

import numpy as np

from . import _lib as L
from .classifier import pack


def _pinned(shape, dtype):
    try:
        import torch
        tdt = {np.uint64: torch.int64, np.uint32: torch.int32, np.int32: torch.int32}[dtype]
        t = torch.empty(shape, dtype=tdt).pin_memory()
        return t, t.numpy().view(dtype)
    except Exception:
        a = np.empty(shape, dtype=dtype)
        return a, a


def _host(x, dtype):
    """(keep-alive object, address) of a host array / pinned tensor."""
    if hasattr(x, "data_ptr"):
        return x, x.data_ptr()
    a = np.ascontiguousarray(x, dtype=dtype)
    return a, a.ctypes.data


class ServedRequest:
    def __init__(self, kind, n):
        self.kind = kind
        self.n = n
        self.ticket = None
        self._keep = []
        self.stats = None


class Server:
    def __init__(self, bloom=None, mibf=None, *, slots=4, mem_budget=0, chunk_reads=0,
                 max_frames=0):
        p = L.ServerParams()
        p.mem_budget, p.slots, p.chunk_reads, p.max_frames = (int(mem_budget), int(slots),
                                                              int(chunk_reads), int(max_frames))
        self._bloom, self._mibf = bloom, mibf
        srv = ctypes.c_void_p()
        L.check(L.lib().bbt_server_create(bloom._ctx if bloom else None,
                                          mibf._ctx if mibf else None, ctypes.byref(p),
                                          ctypes.byref(srv)))
        self._srv = srv
        self.words = bloom.words if bloom else 0

    def _submit(self, req, r):
        t = ctypes.c_uint64()
        rc = L.lib().bbt_server_submit(self._srv, ctypes.byref(r), ctypes.byref(t))
        if rc:
            msg = L.lib().bbt_server_last_error(self._srv)
            raise L.BBTError(rc, msg.decode() if msg else "")
        req.ticket = t.value
        return req

    def _reads(self, req, r, seq, off, seq2, off2):
        if isinstance(seq, list):
            seq, off = pack(seq)
        ks, ps = _host(seq, np.uint8)
        ko, po = _host(off, np.uint64)
        req._keep += [ks, ko]
        r.seq, r.offsets = ps, po
        n = (off.numel() if hasattr(off, "numel") else len(off)) - 1
        if seq2 is not None:
            if isinstance(seq2, list):
                seq2, off2 = pack(seq2)
            ks2, ps2 = _host(seq2, np.uint8)
            ko2, po2 = _host(off2, np.uint64)
            req._keep += [ks2, ko2]
            r.seq2, r.offsets2 = ps2, po2
        r.n_reads = n
        return n

    def submit_prepared(self, req):
        """Queue a request made with submit=False (its buffers already exist)."""
        return self._submit(req, req._req)

    def submit_bloom(self, seq, off=None, seq2=None, off2=None, submit=True):
        """Queue a Bloom-filter request (reads as a list of bytes, or
        (uint8 array, uint64 offsets)); submit=False only prepares it."""
        r = L.Request()
        r.kind = L.REQ_BLOOM
        req = ServedRequest(L.REQ_BLOOM, 0)
        n = self._reads(req, r, seq, off, seq2, off2)
        req.n = n
        k1, req.hits = _pinned((max(n, 1), self.words), np.uint64)
        kc, req.category = _pinned(max(n, 1), np.uint32)
        req._keep += [k1, kc]
        r.hits, r.category = req.hits.ctypes.data, req.category.ctypes.data
        if seq2 is not None:
            k2, req.hits2 = _pinned((max(n, 1), self.words), np.uint64)
            req._keep.append(k2)
            r.hits2 = req.hits2.ctypes.data
        req._req = r
        return self._submit(req, r) if submit else req

    def submit_mibf(self, seq, off=None, seq2=None, off2=None, max_hits=4, submit=True):
        """Queue a miBF request; results are (id, nonSatFrameCount, solidCount,
        count, nonSatCount, totalNonSatCount, totalCount) rows."""
        r = L.Request()
        r.kind = L.REQ_MIBF
        req = ServedRequest(L.REQ_MIBF, 0)
        n = self._reads(req, r, seq, off, seq2, off2)
        req.n = n
        kh, hv = _pinned((max(n, 1), max_hits * 7), np.uint32)
        req.hits = hv.reshape(max(n, 1), max_hits, 7)
        kn, req.n_hits = _pinned(max(n, 1), np.uint32)
        ks, req.sat = _pinned(max(n, 1), np.uint32)
        req._keep += [kh, hv, kn, ks]
        r.mi_hits, r.mi_max_hits = hv.ctypes.data, int(max_hits)
        r.mi_n_hits, r.mi_sat = req.n_hits.ctypes.data, req.sat.ctypes.data
        req._req = r
        return self._submit(req, r) if submit else req

    def wait(self, req, timeout=-1.0):
        """Wait for a request; returns its stats (raises on a failed request)."""
        st = L.RequestStats()
        rc = L.lib().bbt_server_wait(self._srv, req.ticket, float(timeout), ctypes.byref(st))
        if rc:
            raise L.BBTError(rc, "bbt_server_wait")
        req.stats = {"status": st.status, "t_submit": st.t_submit, "t_admit": st.t_admit,
                     "t_done": st.t_done, "device_bytes": st.device_bytes, "slot": st.slot}
        if st.status:
            msg = L.lib().bbt_server_last_error(self._srv)
            raise L.BBTError(st.status, msg.decode() if msg else "")
        return req.stats

    def mibf_results(self, req):
        return [[tuple(int(x) for x in req.hits[i, j]) for j in range(int(req.n_hits[i]))]
                for i in range(req.n)]

    def load(self):
        q, f, b = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        L.lib().bbt_server_load(self._srv, ctypes.byref(q), ctypes.byref(f), ctypes.byref(b))
        return q.value, f.value, b.value

    def close(self):
        if getattr(self, "_srv", None):
            L.lib().bbt_server_destroy(self._srv)
            self._srv = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
