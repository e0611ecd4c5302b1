"""The serving engine (include/bbt_server.h) on the GPU: requests of different
sizes, kinds and read lengths submitted together (so that they are admitted as
slots and memory free up and overlap on the device) give, bit for bit, the
results each gives alone and the results of the batch entry points; a small
memory budget forces queueing and in-request chunking without changing
anything."""
import numpy as np
import pytest

from tests import oracle_lib as ol

pytestmark = pytest.mark.gpu

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)


def _genome(rng, n):
    return BASES[rng.integers(0, 4, n)]


def _reads(rng, genomes, n, long_frac=0.1):
    out = []
    for _ in range(n):
        L = int(rng.integers(20, 300))
        if rng.random() < long_frac:
            L = int(rng.integers(1000, 6000))
        g = genomes[int(rng.integers(0, len(genomes)))]
        if rng.random() < 0.7 and L < len(g):
            st = int(rng.integers(0, len(g) - L))
            r = g[st:st + L].copy()
            m = rng.random(L) < 0.05
            r[m] = BASES[rng.integers(0, 4, int(m.sum()))]
        else:
            r = BASES[rng.integers(0, 4, L)]
        out.append(r.tobytes())
    return out


@pytest.fixture(scope="module")
def contexts(tmp_path_factory):
    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200.mibf import MIBFClassifier
    d = tmp_path_factory.mktemp("serve")
    rng = np.random.default_rng(31)
    genomes = [_genome(rng, 40000) for _ in range(3)]
    paths = []
    for i, g in enumerate(genomes):
        f = ol.Filter.make([g.tobytes()], k=25, fpr=0.075)
        stem = str(d / f"f{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"f{i}", 25, 0.075, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    seeds = ["1111011101110010111011111", "1101111101001011111011011",
             "1111101011100111010111111"]
    m = ol.MIBF.build([g.tobytes() for g in genomes], [1, 2, 3], seeds=seeds, occupancy=0.5)
    m.store(str(d / "mi"))
    with open(d / "mi_ids.txt", "w") as fh:
        fh.write("1\ta\n2\tb\n3\tc\n")
    bbc = BioBloomClassifier(paths, 0.15)
    mc = MIBFClassifier(str(d / "mi.bf"))
    yield bbc, mc, genomes
    bbc.close()
    mc.close()


def _requests(rng, genomes, count):
    reqs = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1), np.log(3000))))
        kind = ("bloom", "bloom_pe", "mibf")[i % 3]
        r1 = _reads(rng, genomes, n)
        r2 = _reads(rng, genomes, n) if kind == "bloom_pe" else None
        reqs.append((kind, r1, r2))
    return reqs


def _submit(srv, kind, r1, r2):
    if kind == "mibf":
        return srv.submit_mibf(r1, max_hits=3)
    return srv.submit_bloom(r1, None, r2, None)


def _result(srv, req, kind):
    if kind == "mibf":
        return srv.mibf_results(req), req.sat[:req.n].tolist()
    h2 = req.hits2[:req.n].tolist() if kind == "bloom_pe" else None
    return req.hits[:req.n].tolist(), h2, req.category[:req.n].tolist()


@pytest.mark.parametrize("budget,chunk,slots", [(0, 0, 4), (6 << 20, 300, 3)])
def test_mixed_requests_equal_alone_and_batch_entry_points(contexts, budget, chunk, slots):
    from biobloom_b200.server import Server
    bbc, mc, genomes = contexts
    rng = np.random.default_rng(budget + chunk)
    reqs = _requests(rng, genomes, 18)
    bbc.reset_summary()
    mc.reset_summary()
    with Server(bbc, mc, slots=slots, mem_budget=budget, chunk_reads=chunk) as srv:
        handles = [_submit(srv, *r) for r in reqs]       # all in flight together
        stats = [srv.wait(h) for h in handles]
        mixed = [_result(srv, h, r[0]) for h, r in zip(handles, reqs)]
        alone = []
        for r in reqs:                                   # one at a time
            h = _submit(srv, *r)
            srv.wait(h)
            alone.append(_result(srv, h, r[0]))
    assert mixed == alone
    assert all(s["t_submit"] <= s["t_admit"] <= s["t_done"] for s in stats)
    assert len({s["slot"] for s in stats}) > 1
    # the batch entry points on the same reads
    for (kind, r1, r2), res in zip(reqs, mixed):
        if kind == "mibf":
            want, sat = mc.classify(r1, max_hits=mc.num_ids)
            assert res == (want, sat.tolist())
        else:
            h1, h2, cat = bbc.classify(r1, r2)
            assert res[0] == h1.tolist() and res[2] == cat.tolist()
            if r2 is not None:
                assert res[1] == h2.tolist()


def test_bloom_results_match_oracle_in_the_mix(contexts, tmp_path):
    from biobloom_b200.server import Server
    bbc, mc, genomes = contexts
    rng = np.random.default_rng(77)
    filters = [ol.Filter.make([g.tobytes()], k=25, fpr=0.075) for g in genomes]
    reqs = [_reads(rng, genomes, n) for n in (5, 700, 40, 2500, 1)]
    with Server(bbc, mc, slots=4) as srv:
        hs = [srv.submit_bloom(r) for r in reqs] + [srv.submit_mibf(r) for r in reqs]
        for h in hs:
            srv.wait(h)
        for r, h in zip(reqs, hs):
            seq, off = ol.pack_reads(r)
            want, _ = ol.classify(seq, off, filters, 0.15, 3)
            assert np.array_equal(h.hits[:h.n], want)


def test_overflow_is_reported_per_request(contexts):
    from biobloom_b200 import BBTError
    from biobloom_b200.server import Server
    bbc, mc, genomes = contexts
    rng = np.random.default_rng(5)
    reads = _reads(rng, genomes, 300)
    want, _ = mc.classify(reads, max_hits=mc.num_ids)
    if not any(len(w) > 0 for w in want):
        pytest.skip("no read with a result")
    with Server(None, mc, slots=2) as srv:
        h = srv.submit_mibf(reads, max_hits=0)
        with pytest.raises(BBTError):
            srv.wait(h)
        assert [int(x) for x in h.n_hits[:h.n]] == [len(w) for w in want]
        ok = srv.submit_mibf(reads, max_hits=mc.num_ids)
        srv.wait(ok)
        assert srv.mibf_results(ok) == want


@pytest.mark.parametrize("mode", ["ordered", "besthit"])
def test_bloom_requests_follow_the_filtering_mode(contexts, mode):
    """ORDERED and BESTHIT requests give the hit words and categories of the
    batch entry point in the same mode."""
    from biobloom_b200 import MODE_BESTHIT, MODE_STD
    from biobloom_b200.server import Server
    bbc, mc, genomes = contexts
    rng = np.random.default_rng(5 if mode == "ordered" else 6)
    reqs = [(_reads(rng, genomes, n), _reads(rng, genomes, n)) for n in (3, 900, 60)]
    if mode == "ordered":
        bbc.setOrderedFilter()
    else:
        bbc.set_mode(MODE_BESTHIT)
    try:
        with Server(bbc, None, slots=2) as srv:
            hs = [srv.submit_bloom(r1, None, r2, None) for r1, r2 in reqs]
            for h in hs:
                srv.wait(h)
        for (r1, r2), h in zip(reqs, hs):
            w1, w2, wc = bbc.classify(r1, r2)
            assert np.array_equal(h.hits[:h.n], w1) and np.array_equal(h.hits2[:h.n], w2)
            assert np.array_equal(h.category[:h.n], wc)
    finally:
        bbc.set_mode(MODE_STD)


def test_server_refuses_a_dust_context(contexts):
    from biobloom_b200 import BBTError
    from biobloom_b200.server import Server
    bbc, mc, genomes = contexts
    bbc.set_dust(True)
    try:
        with pytest.raises(BBTError):
            Server(bbc, None, slots=1)
    finally:
        bbc.set_dust(False)
