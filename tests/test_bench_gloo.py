"""The bench's multi-rank set-up with two gloo ranks on the CPU: cached input
files that every rank reads are written by rank 0 alone, and no rank reads
them before they are complete (bench.build_once)."""
import os
import socket

CHUNKS = 64
CHUNK = 1 << 16


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, path, q):
    import datetime
    import time

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    built = []
    try:
        def build():
            built.append(rank)
            with open(path, "wb") as f:      # slowly, so that a reader would see it partial
                for _ in range(CHUNKS):
                    f.write(b"\x5a" * CHUNK)
                    f.flush()
                    time.sleep(0.005)
        bench.build_once(rank, dist, build)
        size = os.path.getsize(path)
        with open(path, "rb") as f:
            ok = f.read() == b"\x5a" * (CHUNKS * CHUNK)
        q.put((rank, built, size, ok))
    finally:
        dist.destroy_process_group()


def test_rank_zero_alone_writes_shared_inputs(tmp_path):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    path = str(tmp_path / "shared.bin")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, path, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == [0] and out[1][1] == []          # only rank 0 built
    for _, _, size, ok in out:
        assert size == CHUNKS * CHUNK and ok             # every rank saw the whole file
