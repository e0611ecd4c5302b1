"""Replica sharding (biobloom_b200/replicas.py) with two gloo ranks on the CPU:
the shards cover every read once, each rank classifies its shard (here with
the CPU oracle, standing in for the GPU kernel), and the reduced summary
counters equal those of one process classifying everything."""
import os
import socket

import numpy as np
import pytest

from biobloom_b200.replicas import shard_range


def test_shard_range_covers_every_read_once():
    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            got = [shard_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            for (a, b), (c, d) in zip(got, got[1:]):
                assert b == c
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from biobloom_b200.replicas import max_over_ranks, reduce_counts
    from tests import oracle_lib as ol
    from tests.fixtures import filter_paths, golden, read_fastx
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        recs = read_fastx(golden("reads_se.fa.gz"))
        lo, hi = shard_range(len(recs), rank, world)
        filters = [ol.Filter.load(p) for p in filter_paths()]
        seq, off = ol.pack_reads([s for _, s in recs[lo:hi]])
        hits, _ = ol.classify(seq, off, filters, 0.15, 3)
        counts, _ = ol.summary_counts(hits, len(filters))
        total = reduce_counts(counts)
        slowest = max_over_ranks(float(rank + 1))
        q.put((rank, total.tolist(), slowest, hi - lo))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_to_the_single_process_summary():
    import torch.multiprocessing as mp

    from tests import oracle_lib as ol
    from tests.fixtures import filter_paths, golden, read_fastx
    recs = read_fastx(golden("reads_se.fa.gz"))
    filters = [ol.Filter.load(p) for p in filter_paths()]
    seq, off = ol.pack_reads([s for _, s in recs])
    hits, _ = ol.classify(seq, off, filters, 0.15, 3)
    want, _ = ol.summary_counts(hits, len(filters))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, total, slowest, n in out:
        assert np.array_equal(np.array(total, dtype=np.uint64), want)
        assert slowest == 2.0
    assert sum(n for *_, n in out) == len(recs)
