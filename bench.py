#!/usr/bin/env python3
"""Benchmark of the read-classification path on B200.

Workload (default, --workload varlen): one Bloom filter (k=25, FPR 0.075,
hash count auto = 3, 2.12 GB by the reference's sizing formula) from a seeded
3.1 Gbp reference (41% GC, 45% of bases in repeat families of 300 bp - 6 kb at
10-20% divergence); 50M single-end reads, 95% of lengths log-uniform over
50-300 bp and 5% log-uniform over 300 bp - 10 kb, 70% drawn from the
reference with 1% substitutions and 30% uniform random; score 0.15.
Synthetic data: the reads and references are generated from fixed seeds.

A step classifies all reads once (13.5 G bases and the 2.12 GB filter resident
in HBM, far above the 126 MB L2, so no L2 flush is needed between steps).
`value` is reads/s of the batched path (autotuned, launches captured in one
CUDA graph) over the timed steps (device time, CUDA events); `plain` is the
one-warp-per-read, one-launch-per-batch kernel on the same data; `e2e` is the
same metric through the C ABI with pinned host buffers (host->device copies of
the reads and device->host copies of the per-read results inside the timed
region).  `--impl reference` times the reference's own classifier
(BioBloomClassifier::filter compiled from the reference sources,
oracle/_ref/ref_harness) on the host's cores, on inputs made by the CPU
oracle's copy of the generator and filter build (no product library loaded).

With --workload bf: 10 Bloom filters (k=25, FPR 0.075, h=3), each built from
an independent seeded 100 Mbp reference (41% GC, 5% of each reference in
300 bp repeat copies); 10M read pairs 2x150 bp, 10% drawn from each reference
with 0.5% substitutions and 0.01% N.  3 GB of bases and 685 MB of filters.

With --workload mibf: the multi-index workload -- a miBF over 500 targets,
each a seeded 2 Mbp reference at 35-65% GC (uniform per target) with 20% of
its sequence copied from another random target; 3 spaced seeds of span 25 and
weight 19 drawn from the seed; 20M single-end 150 bp reads, 90% from the
targets with 1% substitutions, 10% uniform random.  A step classifies all
reads once (reads and the 5 GB filter resident in HBM, far above L2).

With --workload small: one filter from a seeded 5 Mbp uniform reference,
1M single-end 150 bp reads, 50% from the reference with 1% substitutions
(the filter, 3.4 MB, is L2-resident).

With --workload serve: the serving engine with the 3.1 Gbp filter and the
500-target miBF resident.  Requests of 1k to 1M reads (log-uniform), half
Bloom and half miBF, read lengths 75-300 bp with 10% of 1-10 kb reads and 5%
substitutions, arrive as a seeded Poisson process at a fixed offered load
(a fraction of the capacity measured by submitting the same requests all at
once, the offline batched run); reports p50/p99 request latency and reads/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload varlen|bf|mibf|small|serve|modes]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_FILTERS = 10
REF_LEN = 100_000_000
READ_LEN = 150
K = 25
FPR = 0.075
SUB = 0.005
NRATE = 0.0001
SCORE = 0.15
STREAK = 3
METRIC = "reads/s & Bloom probes/s on 1 B200: batched vs plain kernel, % HBM sector peak"
WORKLOAD = ("10 filters x 100 Mbp (k=25, FPR 0.075, h=3), paired 2x150 bp reads, "
            "0.5% substitutions, 0.01% N, score 0.15")


STEP_FORMS = {"decision": 0, "full": 1, "wide": 2, "wide-full": 3}  # BBT_STEPS_*

def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="bbt_clocks_", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.out.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.out.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def workdir():
    d = os.environ.get("BBT_BENCH_DIR", os.path.join(tempfile.gettempdir(), "bbt_bench_c2"))
    os.makedirs(d, exist_ok=True)
    return d


def build_once(rank, pg, build):
    """Input files cached on this host, which every rank reads, are written by
    rank 0 alone while the other ranks wait at a barrier: ranks share the cache
    directory, and a rank that rewrote a file another rank was already reading
    would cut that read short."""
    if rank == 0:
        build()
    if pg:
        pg.barrier()


def build_filters(d, device, rank=0, pg=None):
    """Generate the 10 references and build their filters (cached in d)."""
    from biobloom_b200 import synth
    paths = [os.path.join(d, f"ref{j}.bf") for j in range(N_FILTERS)]
    genomes = []
    t0 = time.time()
    for j in range(N_FILTERS):
        genomes.append(synth.genome(1002 * 1000 + j, REF_LEN, gc=0.41, repeat_frac=0.05,
                                    rep_min=300, rep_max=300))

    def build():
        for j, g in enumerate(genomes):
            if not (os.path.exists(paths[j]) and os.path.exists(paths[j][:-2] + "txt")):
                synth.make_filter([g], paths[j][:-3], f"ref{j}", k=K, fpr=FPR, device=device,
                                  sources=f"ref{j}.fa")
    build_once(rank, pg, build)
    log(f"references + filters: {time.time() - t0:.1f} s")
    return paths, genomes


def make_reads(genomes, n_pairs, seed):
    from biobloom_b200 import synth
    p = synth.read_params(READ_LEN, READ_LEN, sub_rate=SUB, n_rate=NRATE, frag_min=300,
                          frag_max=500)
    t0 = time.time()
    s1, off, s2, src = synth.reads(seed, genomes, [1.0 / N_FILTERS] * N_FILTERS, n_pairs, p,
                                   paired=True)
    log(f"reads: {n_pairs} pairs in {time.time() - t0:.1f} s")
    return s1, s2, off


def write_fastq(path, seq, off, lo, hi):
    with open(path, "wb") as f:
        qual = b"I" * READ_LEN
        buf = []
        for i in range(lo, hi):
            s = seq[off[i]:off[i + 1]].tobytes()
            buf.append(b"@p%d\n%s\n+\n%s\n" % (i, s, qual[:len(s)]))
        f.write(b"".join(buf))


def cpu_reference_run(d, paths, s1, s2, off, n_pairs, threads, score=None, env=None):
    """Time the reference's own classifier (oracle/_ref/ref_harness, compiled
    from the reference sources) on n_pairs pairs with `threads` threads; env
    selects a scoring method (BBT_SCORING), filtering mode (BBT_MODE) or DUST
    (BBT_DUST) for the harness."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return None, "oracle/_ref/ref_harness is not built"
    f1 = os.path.join(d, f"sample_{n_pairs}_1.fq")
    f2 = os.path.join(d, f"sample_{n_pairs}_2.fq")
    if not os.path.exists(f2):
        write_fastq(f1, s1, off, 0, n_pairs)
        write_fastq(f2, s2, off, 0, n_pairs)
    p = subprocess.run([harness, "time", str(SCORE if score is None else score), str(STREAK),
                        str(threads), "0", os.path.join(d, "refcpu"), ",".join(paths), f1, f2],
                       capture_output=True, text=True,
                       env=dict(os.environ, **(env or {})))
    if p.returncode:
        return None, "ref_harness failed: " + p.stderr[-300:]
    line = [x for x in p.stdout.splitlines() if x.startswith("{")][-1]
    r = json.loads(line)
    return r, None


def cpu_baseline(d, paths, s1, s2, off, budget_s=15.0):
    threads = os.cpu_count() or 1
    probe = 2000
    r, err = cpu_reference_run(d, paths, s1, s2, off, probe, threads)
    if r is None:
        return None, err
    rate = probe / max(r["seconds"], 1e-6)
    n = int(min(len(off) - 1, max(probe, rate * budget_s)))
    n = max(probe, (n // 1000) * 1000)
    r, err = cpu_reference_run(d, paths, s1, s2, off, n, threads)
    if r is None:
        return None, err
    return {"value": 2 * r["records"] / r["seconds"], "unit": "reads/s", "cores": r["threads"],
            "kind": "reference",
            "sample": f"first {r['records']} pairs of the workload (2x150 bp, 10 filters), "
                      f"BioBloomClassifier::filterPair from the reference sources, "
                      f"{r['threads']} OpenMP threads, filter load excluded",
            "seconds": r["seconds"]}, None


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def native_libs():
    """Shared libraries of this repository mapped into this process."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 6 and parts[-1].startswith(ROOT + os.sep) and ".so" in parts[-1]:
                    out.add(os.path.relpath(parts[-1], ROOT))
    except OSError:
        pass
    return sorted(out)


def bf_config(args):
    """The 10-filter workload's config, the same on the GPU arm and on the
    reference arm (figures of the run sit beside it in the line)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"workload": WORKLOAD, "pairs_per_gpu": args.pairs, "reads_per_gpu": 2 * args.pairs,
            "filters": N_FILTERS, "l2": "inputs larger than L2 (3 GB reads + 685 MB filters)",
            "parallelism": f"replicas x{world} (reads sharded, filters replicated)"}


def ref_rank_zero():
    """The reference arm runs on rank 0 only; the other ranks exit without work."""
    return int(os.environ.get("RANK", "0")) == 0


def ref_store_filter(f, path, fid, source):
    """Write an oracle-built filter as <stem>.bf + <stem>.txt."""
    from tests import oracle_lib as ol
    f.store(path)
    n = f.bf.n_entry
    approx = (1.0 - np.exp(-float(f.h) * n / float(f.m))) ** f.h
    ol.write_info(path[:-2] + "txt", fid, f.k, FPR, f.h, f.expected_entries, source, f.m, n,
                  approx, f.redundant, approx)


def ref_step_budget(args):
    """Seconds of CPU classification per reference step: the whole run stays
    within about three minutes."""
    return max(3.0, min(10.0, 150.0 / max(1, args.warmup + args.steps)))


def ref_line(args, metric, value, sec, workload, sample, threads, extra=None):
    line = {"impl": "reference", "metric": metric, "value": value, "unit": "reads/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": workload},
            "cpu_baseline": {"value": value, "unit": "reads/s", "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "reads/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "inputs": "made by the CPU oracle's generator and threaded filter build "
                      "(oracle/synth_oracle.c), the same bytes as the GPU arm's",
            "native_so_loaded": native_libs()}
    line.update(extra or {})
    return line


def run_reference(args):
    """The 10-filter workload's CPU arm: the reference's own
    BioBloomClassifier::filterPair on a bounded sample of the same pairs."""
    if not ref_rank_zero():
        return
    from tests import oracle_lib as ol
    d = os.path.join(tempfile.gettempdir(), "bbt_ref_c2")
    os.makedirs(d, exist_ok=True)
    t0 = time.time()
    paths, genomes = [], []
    for j in range(N_FILTERS):
        g = ol.synth_genome(1002 * 1000 + j, REF_LEN, gc=0.41, repeat_frac=0.05, rep_min=300,
                            rep_max=300)
        genomes.append(g)
        p = os.path.join(d, f"ref{j}.bf")
        if not (os.path.exists(p) and os.path.exists(p[:-2] + "txt")):
            ref_store_filter(ol.make_filter_par([g], k=K, fpr=FPR), p, f"ref{j}", f"ref{j}.fa")
        paths.append(p)
    log(f"reference arm: references + filters {time.time() - t0:.1f} s")
    n_sample = 400_000
    rp = ol.read_params(READ_LEN, READ_LEN, sub_rate=SUB, n_rate=NRATE, frag_min=300,
                        frag_max=500)
    s1, off, s2, _ = ol.synth_reads(5000, genomes, [1.0 / N_FILTERS] * N_FILTERS, n_sample, rp,
                                    paired=True)
    threads = os.cpu_count() or 1
    r, err = cpu_reference_run(d, paths, s1, s2, off, 2000, threads)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    rate = 2000 / max(r["seconds"], 1e-6)
    n = int(min(n_sample, max(2000, rate * ref_step_budget(args))))
    n = (n // 1000) * 1000
    times = []
    for i in range(args.warmup + args.steps):
        r, err = cpu_reference_run(d, paths, s1, s2, off, n, threads)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return
        if i >= args.warmup:
            times.append(r["seconds"])
    sec = sum(times) / len(times)
    value = 2 * n / sec
    print(json.dumps(ref_line(args, METRIC, value, sec, WORKLOAD,
                              f"first {n} pairs of the workload per step, "
                              "BioBloomClassifier::filterPair compiled from the reference "
                              f"sources, {threads} OpenMP threads, filter load excluded",
                              threads, {"config": bf_config(args), "pairs_per_step": n})),
          flush=True)


def traffic_per_read(name="classify_c2_dram.json"):
    """DRAM bytes per read of a classify kernel from a committed ncu summary
    (profiles/<name>), or None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f).get("dram_bytes_per_read")


def run_gpu(args):
    import torch

    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200 import _lib as L

    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    d = workdir()
    paths, genomes = build_filters(d, local, rank, pg)
    n_pairs = args.pairs
    s1, s2, off = make_reads(genomes, n_pairs, 5000 + rank)
    n_reads = 2 * n_pairs
    bases = int(off[-1])

    # pinned host copies (e2e) and device copies (kernel value)
    h1 = torch.from_numpy(s1[:bases]).pin_memory()
    h2 = torch.from_numpy(s2[:bases]).pin_memory()
    hoff = torch.from_numpy(off.view(np.int64)).pin_memory()
    d1, d2, doff = h1.to(dev), h2.to(dev), hoff.to(dev)
    torch.cuda.synchronize()

    bbc = BioBloomClassifier(paths, SCORE, streak_threshold=STREAK, device=local,
                             path=L.PATH_AUTO, l2_fetch_bytes=args.l2_fetch)
    words = bbc.words
    hits1 = torch.empty((n_pairs, words), dtype=torch.int64, device=dev)
    hits2 = torch.empty((n_pairs, words), dtype=torch.int64, device=dev)
    cat = torch.empty(n_pairs, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    def step():
        bbc.classify_device(d1, doff, d2, doff, hits1, hits2, cat, stream=stream)

    # counters pass (outside the timed region): probes the sequential algorithm
    # makes, probes issued, frames hashed
    bbc.set_counting(True)
    step()
    stream.synchronize()
    st = bbc.last_stats()
    bbc.set_counting(False)
    alg_probes = st["probes_algorithmic"]
    issued = st["probes_issued"]
    frames = st["frames"]
    bbc.reset_summary()

    def timed(path):
        bbc.set_launch(path=path)
        for _ in range(args.warmup):
            step()
        stream.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        kms = []
        launches = 0
        e0.record(stream)
        for _ in range(args.steps):
            step()
            stream.synchronize()
            st_ = bbc.last_stats()
            kms.append(st_["classify_ms"])
            launches += st_["kernels"]
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        if pg:
            t = torch.tensor([ms], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = float(t.item())
        return ms, sum(kms) / len(kms), launches

    # the batched path: persistent kernel in the work order the tuner picks
    # (filter-major when the filters are probed from L2), timed with clocks
    paths_timed = {}
    for pth in (L.PATH_FILTER_MAJOR, L.PATH_PERSISTENT):
        paths_timed[pth] = timed(pth)
    best = min(paths_timed, key=lambda x: paths_timed[x][0])
    clocks = ClockSampler(local)
    clocks.start()
    ms_persistent, k_persistent, launches_best = timed(best)
    clk = clocks.stop()
    keep1, keep2 = hits1.clone(), hits2.clone()
    ms_plain, k_plain, _ = timed(L.PATH_PLAIN)
    plain_same = bool(torch.equal(keep1, hits1) and torch.equal(keep2, hits2))
    del keep1, keep2
    bbc.set_launch(path=best)

    g1_np = hits1.cpu().numpy().view(np.uint64)
    g2_np = hits2.cpu().numpy().view(np.uint64)

    # e2e through the C ABI with pinned host buffers
    hb1 = np.empty((n_pairs, words), dtype=np.uint64)
    hb2 = np.empty((n_pairs, words), dtype=np.uint64)
    hcat = np.empty(n_pairs, dtype=np.uint32)
    a1, a2, ao = h1.numpy(), h2.numpy(), hoff.numpy().view(np.uint64)

    def e2e_step():
        b = L.Batch()
        b.seq, b.offsets, b.seq2, b.offsets2 = (a1.ctypes.data, ao.ctypes.data, a2.ctypes.data,
                                                ao.ctypes.data)
        b.n_reads, b.location = n_pairs, L.HOST
        r = L.Result()
        r.hits, r.hits2, r.category, r.location = (hb1.ctypes.data, hb2.ctypes.data,
                                                   hcat.ctypes.data, L.HOST)
        import ctypes
        L.check(L.lib().bbt_classify_batch(bbc._ctx, ctypes.byref(b), ctypes.byref(r), None),
                bbc._ctx)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if pg:
        t = torch.tensor([e2e_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_ok = bool(np.array_equal(hb1, hits1.cpu().numpy().view(np.uint64)) and
                  np.array_equal(hb2, hits2.cpu().numpy().view(np.uint64)))

    # the same over the packed boundary form (BBT_BASES_2BIT), packed before timing
    import ctypes
    packed, bad = [], []
    for arr in (a1, a2):
        pw = torch.empty(((bases + 15) // 16 + 1,), dtype=torch.int32).pin_memory()
        pv = torch.empty(((bases + 31) // 32 + 1,), dtype=torch.int32).pin_memory()
        nb = ctypes.c_uint64()
        L.check(L.lib().bbt_pack_bases(arr.ctypes.data, bases, pw.data_ptr(), pv.data_ptr(),
                                       ctypes.byref(nb)))
        packed.append((pw, pv))
        bad.append(nb.value)
    hb1[:] = 0
    hb2[:] = 0

    def e2e_packed_step():
        b = L.Batch()
        b.seq, b.offsets, b.seq2, b.offsets2 = (packed[0][0].data_ptr(), ao.ctypes.data,
                                                packed[1][0].data_ptr(), ao.ctypes.data)
        b.n_reads, b.location, b.encoding = n_pairs, L.HOST, L.BASES_2BIT
        b.valid = packed[0][1].data_ptr() if bad[0] else None
        b.valid2 = packed[1][1].data_ptr() if bad[1] else None
        r = L.Result()
        r.hits, r.hits2, r.category, r.location = (hb1.ctypes.data, hb2.ctypes.data,
                                                   hcat.ctypes.data, L.HOST)
        L.check(L.lib().bbt_classify_batch(bbc._ctx, ctypes.byref(b), ctypes.byref(r), None),
                bbc._ctx)

    for _ in range(max(1, args.warmup)):
        e2e_packed_step()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_packed_step()
    e2e_p_s = (time.perf_counter() - t0) / args.steps
    if pg:
        t = torch.tensor([e2e_p_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_p_s = float(t.item())
    e2e_p_ok = bool(np.array_equal(hb1, hits1.cpu().numpy().view(np.uint64)) and
                    np.array_equal(hb2, hits2.cpu().numpy().view(np.uint64)))
    packed_h2d = int(2 * ((bases + 15) // 16) * 4 +
                     sum(((bases + 31) // 32) * 4 for x in bad if x) + 2 * (n_pairs + 1) * 8)
    del packed

    if rank != 0:
        bbc.close()
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return

    cpu = None
    cpu_err = None
    parity = None
    if world == 1 and not args.no_cpu:
        cpu, cpu_err = cpu_baseline(d, paths, s1, s2, off)
    if world == 1 and not args.no_check:
        parity = pair_parity(d, paths, s1, s2, off, g1_np, g2_np, min(n_pairs, PARITY_READS))

    peak, peak_kind = measured_peaks()
    read_bytes = bases * 2 / 4.0  # 2-bit packed read bytes (both mates)
    result_bytes = n_pairs * (2 * words * 8 + 4)
    alg_bytes = 32.0 * alg_probes + read_bytes + result_bytes
    achieved = alg_bytes / (k_persistent * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "kernel": "classify path (scan + hash pass + filter pass)",
                "classify_ms": k_persistent, "algorithmic_bytes_per_launch": alg_bytes}
    if best == L.PATH_FILTER_MAJOR:
        # each 68.5 MB filter is probed out of L2: the ceiling is the random
        # 4-byte gather rate into a table of that size, measured here
        import ctypes
        fbytes = max(os.path.getsize(p) for p in paths)
        rate = ctypes.c_double()
        L.check(L.lib().bbt_measure_gather(local, (fbytes + 4095) // 4096 * 4096, 1 << 29, 0, 5,
                                           ctypes.byref(rate)))
        l2_peak = rate.value * 32.0 / 1e9
        roofline.update({"bound": "l2", "peak": l2_peak, "frac": achieved / l2_peak,
                         "peak_kind": f"measured in this run: {rate.value / 1e9:.1f} G random "
                                      f"4-byte gathers/s into a {fbytes >> 20} MB table "
                                      "(bbt_measure_gather) x 32 B per probe",
                         "hbm_peak": peak, "hbm_frac": achieved / peak,
                         "hbm_peak_kind": peak_kind})
    tpr = traffic_per_read()
    roofline.update({"traffic": (tpr * n_reads if tpr else None),
                     "traffic_note": "filter pass DRAM read+write per read from the committed "
                                     "ncu capture, scaled to the step's reads"})
    value = world * n_reads / (ms_persistent * 1e-3)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "reads/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_persistent,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": bf_config(args),
        "filter_bytes_total": int(sum(os.path.getsize(p) for p in paths)),
        "path": {L.PATH_FILTER_MAJOR: "persistent, filter-major",
                 L.PATH_PERSISTENT: "persistent, read-major"}[best],
        "batched_paths_ms": {"filter_major": paths_timed[L.PATH_FILTER_MAJOR][0],
                             "read_major": paths_timed[L.PATH_PERSISTENT][0]},
        "probes_per_s": world * alg_probes / (ms_persistent * 1e-3),
        "probes_algorithmic_per_step": alg_probes,
        "probes_issued_per_step": issued,
        "frames_hashed_per_step": frames,
        "plain": {"value": world * n_reads / (ms_plain * 1e-3), "unit": "reads/s",
                  "ms_per_step": ms_plain, "classify_ms": k_plain},
        "batched_over_plain": ms_plain / ms_persistent,
        "plain_equals_batched": plain_same,
        "roofline": roofline,
        "cpu_baseline": cpu if cpu else {"value": None, "unavailable": cpu_err},
        "e2e": {"value": world * n_reads / e2e_p_s, "unit": "reads/s",
                "h2d_bytes_per_step": packed_h2d,
                "d2h_bytes_per_step": int(n_pairs * (2 * words * 8 + 4)),
                "matches_device_results": e2e_p_ok,
                "input": "bbt_classify_batch on pinned host buffers, bases 2-bit packed "
                         "with validity bits (BBT_BASES_2BIT), packed before timing",
                "ascii": {"value": world * n_reads / e2e_s, "unit": "reads/s",
                          "h2d_bytes_per_step": int(2 * bases + 2 * (n_pairs + 1) * 8),
                          "d2h_bytes_per_step": int(n_pairs * (2 * words * 8 + 4)),
                          "matches_device_results": e2e_ok}},
        "gpu_launches": launches_best,
        "clocks": clk,
        "parity_sample": parity,
    }
    print(json.dumps(line), flush=True)
    bbc.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def pair_parity(d, paths, s1, s2, off, g1, g2, m):
    """The first m pairs' hits of the timed path against the reference's own
    classifier code on the same pairs (outside the timed region)."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return {"checked_pairs": 0, "error": "oracle/_ref/ref_harness is not built"}
    f1 = os.path.join(d, f"sample_{m}_1.fq")
    f2 = os.path.join(d, f"sample_{m}_2.fq")
    if not os.path.exists(f2):
        write_fastq(f1, s1, off, 0, m)
        write_fastq(f2, s2, off, 0, m)
    t0 = time.time()
    try:
        rows = harness_hits(harness, paths, f1, f2)
    except RuntimeError as e:
        return {"checked_pairs": 0, "error": str(e)}
    w1 = np.array([r[0] for r in rows], dtype=np.uint64)
    w2 = np.array([r[1] for r in rows], dtype=np.uint64)
    n = len(rows)
    bad = int((w1 != g1[:n, 0]).sum() + (w2 != g2[:n, 0]).sum())
    return {"checked_pairs": n, "mismatched_reads": bad,
            "against": "SeqEval::evalRead of the reference sources (ref_harness hits)",
            "kind": "sample: the first pairs of the step", "seconds": time.time() - t0}


# ------------------------------------------------- filtering modes / scoring methods

MODE_VARIANTS = [
    # name, constructor keywords, mode, with scores, dust
    ("std_simple", dict(score_threshold=SCORE), "std", False, False),
    ("ordered", dict(score_threshold=SCORE), "ordered", False, False),
    ("besthit", dict(score_threshold=SCORE), "besthit", False, False),
    ("with_scores", dict(score_threshold=SCORE), "scores", True, False),
    ("harmonic", dict(score_threshold=SCORE, score_type="harmonic"), "std", False, False),
    ("binomial", dict(score_threshold=100, score_type="binomial"), "std", False, False),
    ("length_40", dict(score_threshold=40), "std", False, False),
    ("dust", dict(score_threshold=SCORE), "std", False, True),
]


def mode_oracle(ol, filters, name, kw, mode, dust, s, off):
    """The oracle's hits of one variant for the reads s[off[i]:off[i+1]]."""
    st = kw.get("score_type", "simple")
    thr = kw["score_threshold"]
    if st == "binomial":
        thr, scoring = 10.0 ** (-(thr / 10.0)), ol.BINOMIAL
    elif st == "harmonic":
        scoring = ol.HARMONIC
    elif thr > 1:
        scoring = ol.LENGTH
    else:
        scoring = ol.SIMPLE
    seq = s[:off[-1]].tobytes()
    if dust:
        with ol.dust():
            return ol.classify(seq, off, filters, thr, STREAK, scoring)[0]
    if mode == "besthit":
        return ol.best_hit(ol.classify_scores(seq, off, filters, scoring, STREAK))[0]
    return ol.classify(seq, off, filters, thr, STREAK, scoring)[0]


def mode_cpu(d, paths, s1, s2, off, kw, mode, dust, budget_s=8.0):
    """The reference's BioBloomClassifier::filterPair in one variant's mode and
    scoring method, on a bounded sample of the same pairs, all host threads."""
    env = {}
    st = kw.get("score_type", "simple")
    if st != "simple":
        env["BBT_SCORING"] = st
    if mode in ("ordered", "besthit", "scores"):
        env["BBT_MODE"] = mode
    if dust:
        env["BBT_DUST"] = "20,64"
    threads = os.cpu_count() or 1
    probe = 2000
    r, err = cpu_reference_run(d, paths, s1, s2, off, probe, threads, kw["score_threshold"], env)
    if r is None:
        return {"unavailable": err}
    rate = probe / max(r["seconds"], 1e-6)
    n = max(probe, (int(min(len(off) - 1, rate * budget_s)) // 1000) * 1000)
    r, err = cpu_reference_run(d, paths, s1, s2, off, n, threads, kw["score_threshold"], env)
    if r is None:
        return {"unavailable": err}
    return {"reads_per_s": 2 * r["records"] / r["seconds"], "cores": r["threads"],
            "sample_pairs": r["records"], "kind": "reference"}


def run_modes(args):
    """Every filtering mode and scoring method on the 10-filter workload's
    data (device-resident reads, CUDA-event timing per step), each checked
    against the oracle on a sample of pairs."""
    import torch

    from biobloom_b200 import MODE_BESTHIT, MODE_SCORES, BioBloomClassifier
    dev = torch.device("cuda", 0)
    d = workdir()
    paths, genomes = build_filters(d, 0)
    n_pairs = args.pairs
    s1, s2, off = make_reads(genomes, n_pairs, 5000)
    bases = int(off[-1])
    d1 = torch.from_numpy(s1[:bases]).to(dev)
    d2 = torch.from_numpy(s2[:bases]).to(dev)
    doff = torch.from_numpy(off.view(np.int64)).to(dev)
    stream = torch.cuda.Stream(device=dev)
    ol = None
    filters = None
    if not args.no_check:
        try:
            from tests import oracle_lib as ol
            filters = [ol.Filter.load(p) for p in paths]
        except Exception:
            ol = None
    n_check = 500
    out = {}
    for name, kw, mode, with_scores, dust in MODE_VARIANTS:
        bbc = BioBloomClassifier(paths, streak_threshold=STREAK, device=0, **kw)
        if mode == "ordered":
            bbc.setOrderedFilter()
        elif mode == "besthit":
            bbc.set_mode(MODE_BESTHIT)
        elif mode == "scores":
            bbc.set_mode(MODE_SCORES)
        if dust:
            bbc.set_dust(True)
        h1 = torch.empty((n_pairs, bbc.words), dtype=torch.int64, device=dev)
        h2 = torch.empty((n_pairs, bbc.words), dtype=torch.int64, device=dev)
        cat = torch.empty(n_pairs, dtype=torch.int32, device=dev)
        sc1 = sc2 = None
        if with_scores:
            sc1 = torch.empty((n_pairs, bbc.n_filters), dtype=torch.float64, device=dev)
            sc2 = torch.empty((n_pairs, bbc.n_filters), dtype=torch.float64, device=dev)

        def step():
            bbc.classify_device(d1, doff, d2, doff, h1, h2, cat, stream=stream, scores=sc1,
                                scores2=sc2)

        for _ in range(args.warmup):
            step()
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        res = {"reads_per_s": 2 * n_pairs / (ms * 1e-3), "ms_per_step": ms}
        if ol is not None:
            o = off[:n_check + 1]
            w1 = mode_oracle(ol, filters, name, kw, mode, dust, s1, o)
            w2 = mode_oracle(ol, filters, name, kw, mode, dust, s2, o)
            g1 = h1[:n_check].cpu().numpy().view(np.uint64).copy()
            g2 = h2[:n_check].cpu().numpy().view(np.uint64).copy()
            if mode == "ordered":
                w1, w2 = ol.ordered(w1, len(filters), w2, False)
            res["checked_pairs"] = n_check
            res["mismatched_reads"] = int((g1 != w1).any(1).sum() + (g2 != w2).any(1).sum())
        if not args.no_cpu:
            res["cpu_reference"] = mode_cpu(d, paths, s1, s2, off, kw, mode, dust)
            if kw.get("score_type") == "binomial":
                res["cpu_reference"]["note"] = (
                    "Boost is not installed here: the reference's binomial quantile runs on "
                    "the oracle shim's stand-in for boost::math::binomial (oracle/shim)")
            if res["cpu_reference"].get("reads_per_s"):
                res["vs_cpu_reference"] = res["reads_per_s"] / res["cpu_reference"]["reads_per_s"]
        out[name] = res
        bbc.close()
        log(name, json.dumps(res))
    base = out["std_simple"]["reads_per_s"]
    line = {
        "metric": "reads/s per filtering mode and scoring method on 1 B200",
        "value": base, "unit": "reads/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "dtype": "u8", "data": "synthetic",
        "config": {"workload": WORKLOAD.replace("10M pairs", f"{n_pairs} pairs"),
                   "pairs": n_pairs, "timed": "device-resident reads; every kernel of a call "
                   "(DUST masking, classification, scores, summary)"},
        "variants": {k: dict(v, relative_to_std=v["reads_per_s"] / base) for k, v in out.items()},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------- single-filter workloads

SINGLE = {
    "varlen": dict(name="3.1 Gbp", glen=3_100_000_000, gc=0.41, repeat_frac=0.45, rep_min=300,
                   rep_max=6000, div_min=0.10, div_max=0.20, reads=50_000_000, len_min=50,
                   len_max=300, long_frac=0.05, long_min=300, long_max=10_000, ref_frac=0.7,
                   sub=0.01, seed=3003, l2_note="inputs larger than L2",
                   workload="1 filter from a 3.1 Gbp reference (41% GC, 45% repeats 300 bp-6 kb "
                            "at 10-20% divergence; k=25, FPR 0.075, 2.12 GB), 50M single-end "
                            "reads 50-300 bp log-uniform with 5% 300 bp-10 kb, 70% from the "
                            "reference with 1% substitutions, score 0.15"),
    "small": dict(name="5 Mbp", glen=5_000_000, gc=0.5, repeat_frac=0.0, rep_min=0, rep_max=0,
                  div_min=0.0, div_max=0.0, reads=1_000_000, len_min=150, len_max=150,
                  long_frac=0.0, long_min=0, long_max=0, ref_frac=0.5, sub=0.01, seed=1001,
                  l2_note="filter L2-resident (3.4 MB); reads larger than L2",
                  workload="1 filter from a 5 Mbp uniform reference (k=25, FPR 0.075, 3.4 MB), "
                           "1M single-end 150 bp reads, 50% from the reference with 1% "
                           "substitutions, score 0.15"),
}
PLAIN_BATCH = 1 << 18   # reads per launch of the plain path (the CLI's batch)
SINGLE_METRIC = "reads/s & Bloom probes/s on 1 B200: batched vs plain kernel, % HBM sector peak"


def single_config(cfg, args):
    """The line's config for a single-filter workload: what the workload is,
    the same on the GPU arm and on the reference arm (figures of the run, such
    as the tuned launch configuration, sit beside it in the line)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"workload": cfg["workload"],
            "reads_per_gpu": args.reads if args.reads_set else cfg["reads"],
            "l2": cfg["l2_note"],
            "parallelism": f"replicas x{world} (reads sharded, filter replicated)"}


def single_setup(cfg, device, n_reads, rank=0, pg=None):
    from biobloom_b200 import synth
    d = os.path.join(tempfile.gettempdir(), f"bbt_bench_{cfg['seed']}")
    os.makedirs(d, exist_ok=True)
    t0 = time.time()
    g = synth.genome(cfg["seed"], cfg["glen"], gc=cfg["gc"], repeat_frac=cfg["repeat_frac"],
                     rep_min=cfg["rep_min"], rep_max=cfg["rep_max"], div_min=cfg["div_min"],
                     div_max=cfg["div_max"])
    path = os.path.join(d, "genome.bf")

    def build():
        if not (os.path.exists(path) and os.path.exists(path[:-2] + "txt")):
            synth.make_filter([g], path[:-3], "genome", k=K, fpr=FPR, device=device,
                              sources="genome.fa")
    build_once(rank, pg, build)
    log(f"reference + filter: {time.time() - t0:.1f} s")
    t0 = time.time()
    p = synth.read_params(cfg["len_min"], cfg["len_max"], long_frac=cfg["long_frac"],
                          long_min=cfg["long_min"], long_max=cfg["long_max"], sub_rate=cfg["sub"])
    s1, off, _, _ = synth.reads(cfg["seed"] + 17 + rank, [g], [cfg["ref_frac"]], n_reads, p)
    log(f"reads: {n_reads} in {time.time() - t0:.1f} s, {int(off[-1])} bases")
    return d, path, s1, off


def single_cpu(d, path, s1, off, budget_s=15.0):
    """The reference's BioBloomClassifier::filter (oracle/_ref/ref_harness) on a
    bounded sample of the workload's reads, all host threads."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return None, "oracle/_ref/ref_harness is not built"
    threads = os.cpu_count() or 1

    def run(n):
        fq = os.path.join(d, f"sample_{n}.fq")
        if not os.path.exists(fq):
            write_single_fastq(fq, s1, off, n)
        pr = subprocess.run([harness, "time", str(SCORE), str(STREAK), str(threads), "0",
                             os.path.join(d, "refcpu"), path, fq], capture_output=True, text=True)
        if pr.returncode:
            return None, "ref_harness failed: " + pr.stderr[-300:]
        return json.loads([x for x in pr.stdout.splitlines() if x.startswith("{")][-1]), None

    probe = 20000
    r, err = run(probe)
    if r is None:
        return None, err
    n = int(min(len(off) - 1, max(probe, probe / max(r["seconds"], 1e-6) * budget_s)))
    n = max(probe, (n // 10000) * 10000)
    r, err = run(n)
    if r is None:
        return None, err
    return {"value": r["records"] / r["seconds"], "unit": "reads/s", "cores": r["threads"],
            "kind": "reference",
            "sample": f"first {r['records']} reads of the workload, BioBloomClassifier::filter "
                      f"from the reference sources, {r['threads']} OpenMP threads, filter load "
                      f"excluded", "seconds": r["seconds"]}, None


PARITY_READS = 200_000


def harness_hits(harness, paths, fq1, fq2=None, score=SCORE, streak=STREAK):
    """Per-read hit lists from the reference's own SeqEval::evalRead
    (ref_harness hits), in file order: one list (or pair of lists) per read."""
    cmd = [harness, "hits", str(score), str(streak), ",".join(paths), fq1] + ([fq2] if fq2 else [])
    pr = subprocess.run(cmd, capture_output=True, text=True)
    if pr.returncode:
        raise RuntimeError("ref_harness hits failed: " + pr.stderr[-300:])
    rows = []
    for line in pr.stdout.splitlines():
        if line.startswith("#SUMMARY"):
            break
        ids = line.split("\t", 1)[1]

        def bits(x):
            w = 0
            for t in x.split(","):
                if t:
                    w |= 1 << int(t)
            return w
        rows.append(tuple(bits(x) for x in ids.split("|")))
    return rows


def harness_parity(d, path, s1, off, gpu_hits, m):
    """The first m reads' hits of the timed path against the reference's own
    classifier code on the same reads (outside the timed region)."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return {"checked_reads": 0, "error": "oracle/_ref/ref_harness is not built"}
    fq = os.path.join(d, f"sample_{m}.fq")
    if not os.path.exists(fq):
        write_single_fastq(fq, s1, off, m)
    t0 = time.time()
    try:
        rows = harness_hits(harness, [path], fq)
    except RuntimeError as e:
        return {"checked_reads": 0, "error": str(e)}
    want = np.array([r[0] for r in rows], dtype=np.uint64)
    got = gpu_hits[:len(want), 0]
    return {"checked_reads": len(want), "mismatched_reads": int((want != got).sum()),
            "against": "SeqEval::evalRead of the reference sources (ref_harness hits)",
            "kind": "sample: the first reads of the step", "seconds": time.time() - t0}


def run_single(args):
    import ctypes

    import torch

    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200 import _lib as L

    cfg = SINGLE[args.workload]
    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.reads if args.reads_set else cfg["reads"]
    d, path, s1, off = single_setup(cfg, local, n, rank, pg)
    bases = int(off[-1])
    h1 = torch.from_numpy(s1[:max(bases, 1)]).pin_memory()
    hoff = torch.from_numpy(off.view(np.int64)).pin_memory()
    d1, doff = h1.to(dev), hoff.to(dev)
    torch.cuda.synchronize()
    bbc = BioBloomClassifier([path], SCORE, streak_threshold=STREAK, device=local)
    hits = torch.zeros((n, 1), dtype=torch.int64, device=dev)
    cat = torch.zeros(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    def timed(step):
        for _ in range(args.warmup):
            step()
        stream.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        if pg:
            t = torch.tensor([ms], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # algorithmic probes of the workload (counting pass, outside the timed region)
    bbc.set_launch(path=L.PATH_PERSISTENT)
    bbc.set_counting(True)
    bbc.classify_device(d1, doff, hits=hits, category=cat, stream=stream)
    stream.synchronize()
    st = bbc.last_stats()
    bbc.set_counting(False)
    alg_probes, issued, frames = st["probes_algorithmic"], st["probes_issued"], st["frames"]
    want_hits = hits.clone()

    # plain: one warp per read, one launch per batch of PLAIN_BATCH reads
    bbc.set_launch(path=L.PATH_PLAIN, warps_per_block=8, frames_per_lane=4)
    bbc.set_schedule(0)

    def plain_step():
        for i in range(0, n, PLAIN_BATCH):
            j = min(n, i + PLAIN_BATCH)
            bbc.classify_device(d1, doff[i:j + 1], hits=hits[i:j], category=cat[i:j],
                                stream=stream)

    ms_plain = timed(plain_step)
    plain_launches = 2 * ((n + PLAIN_BATCH - 1) // PLAIN_BATCH)
    plain_ok = bool(torch.equal(hits, want_hits))

    # batched: autotuned configuration; the plain and persistent paths run
    # as one CUDA graph, the bucketed path (which plans its sub-batches on the
    # host) as direct launches
    sample = min(n, 2_000_000)
    if args.path == "auto":
        tune = bbc.autotune(d1, doff[:sample + 1])
    else:  # a pinned path (the tuner's other choices at their defaults)
        pinned = {"persistent": L.PATH_PERSISTENT, "bucketed": L.PATH_BUCKETED}[args.path]
        form = STEP_FORMS[args.step_form]
        bbc.set_launch(path=pinned, warps_per_block=8, frames_per_lane=4)
        bbc.set_schedule(1024 if pinned == L.PATH_PERSISTENT else 0)
        bbc.set_steps(form)
        tune = {"path": pinned, "warps_per_block": 8, "frames_per_lane": 4,
                "long_bases": 1024 if pinned == L.PATH_PERSISTENT else 0,
                "reads_per_launch": 0, "reads_per_s": None, "steps": form, "pinned": True}
        if args.bucketing:
            kv = {x.split("=")[0].strip(): int(x.split("=")[1]) for x in args.bucketing.split(",")}
            bbc.set_bucketing(**kv)
            tune["bucketing"] = kv
    log(f"autotune: {tune}")
    if tune["path"] == L.PATH_FILTER_MAJOR:  # one filter never picks it
        bbc.set_launch(path=L.PATH_PERSISTENT)
    bbc.classify_device(d1, doff, hits=hits, category=cat, stream=stream)  # warm-up, same sizes
    stream.synchronize()
    hits.zero_()
    graph = None
    if tune["path"] == L.PATH_BUCKETED:
        def batched_step():
            bbc.classify_device(d1, doff, hits=hits, category=cat, stream=stream)
    else:
        graph = bbc.graph(d1, doff, hits, category=cat,
                          reads_per_launch=tune["reads_per_launch"])

        def batched_step():
            graph.launch(stream)
    clocks = ClockSampler(local)
    clocks.start()
    ms_batched = timed(batched_step)
    clk = clocks.stop()
    batched_ok = bool(torch.equal(hits, want_hits))
    if graph is not None:
        kernels_per_launch = 3 if (tune["long_bases"] and tune["path"] != L.PATH_PLAIN) else 2
        batched_launches = graph.launches * kernels_per_launch
    else:
        batched_step()
        stream.synchronize()
        batched_launches = bbc.last_stats()["kernels"]

    # kernel time of one launch of the whole batch in the tuned configuration
    bbc.classify_device(d1, doff, hits=hits, category=cat, stream=stream)
    stream.synchronize()
    k_ms = bbc.last_stats()["classify_ms"]
    if tune["path"] != L.PATH_BUCKETED:
        # filter words the tuned configuration reads (its steps decide how
        # many frames it probes past a read's decision): counting pass, untimed
        bbc.set_counting(True)
        bbc.classify_device(d1, doff, hits=hits, category=cat, stream=stream)
        stream.synchronize()
        issued = bbc.last_stats()["probes_issued"]
        bbc.set_counting(False)

    gpu_np = hits.cpu().numpy().view(np.uint64)

    # e2e: the C ABI with pinned host buffers (staged, pipelined copies)
    hh = torch.empty((n, 1), dtype=torch.int64).pin_memory()
    hc = torch.empty(n, dtype=torch.int32).pin_memory()

    def e2e_step():
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = h1.data_ptr(), hoff.data_ptr(), n, L.HOST
        r = L.Result()
        r.hits, r.category, r.location = hh.data_ptr(), hc.data_ptr(), L.HOST
        L.check(L.lib().bbt_classify_batch(bbc._ctx, ctypes.byref(b), ctypes.byref(r), None),
                bbc._ctx)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if pg:
        t = torch.tensor([e2e_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_ok = bool(torch.equal(hh, want_hits.cpu()))

    # e2e over the packed boundary form (bbt_batch BBT_BASES_2BIT: 2-bit codes
    # + validity bits, as a parser that packs while it parses hands them
    # over); packed on the host before timing
    pw = torch.empty(((bases + 15) // 16 + 1,), dtype=torch.int32).pin_memory()
    pv = torch.empty(((bases + 31) // 32 + 1,), dtype=torch.int32).pin_memory()
    n_bad = ctypes.c_uint64()
    L.check(L.lib().bbt_pack_bases(h1.data_ptr(), bases, pw.data_ptr(), pv.data_ptr(),
                                   ctypes.byref(n_bad)))
    valid_ptr = pv.data_ptr() if n_bad.value else None
    hh.zero_()

    def e2e_packed_step():
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = pw.data_ptr(), hoff.data_ptr(), n, L.HOST
        b.encoding, b.valid = L.BASES_2BIT, valid_ptr
        r = L.Result()
        r.hits, r.category, r.location = hh.data_ptr(), hc.data_ptr(), L.HOST
        L.check(L.lib().bbt_classify_batch(bbc._ctx, ctypes.byref(b), ctypes.byref(r), None),
                bbc._ctx)

    for _ in range(max(1, args.warmup)):
        e2e_packed_step()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_packed_step()
    e2e_p_s = (time.perf_counter() - t0) / args.steps
    if pg:
        t = torch.tensor([e2e_p_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_p_s = float(t.item())
    e2e_p_ok = bool(torch.equal(hh, want_hits.cpu()))
    packed_h2d = int(((bases + 15) // 16) * 4 + (((bases + 31) // 32) * 4 if n_bad.value else 0)
                     + (n + 1) * 8)
    del pw, pv
    if rank != 0:
        if graph is not None:
            graph.close()
        bbc.close()
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    cpu, cpu_err = (None, "skipped (--no-cpu)")
    parity = None
    if world == 1 and not args.no_cpu:
        cpu, cpu_err = single_cpu(d, path, s1, off)
    if world == 1 and not args.no_check:
        parity = harness_parity(d, path, s1, off, gpu_np, min(n, PARITY_READS))
    peak, peak_kind = measured_peaks()
    alg_bytes = 32.0 * alg_probes + bases / 4.0 + n * (8 + 4)
    achieved = alg_bytes / (k_ms * 1e-3) / 1e9
    fbytes = os.path.getsize(path)
    l2_resident = fbytes < 96 << 20
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                "kernel": {L.PATH_BUCKETED: "bucketed path (sweeps, resolve, walk)"}.get(
                    tune["path"], "classify_kernel (tuned configuration)"),
                "classify_ms": k_ms, "algorithmic_bytes_per_launch": alg_bytes}
    if l2_resident:
        # the filter is probed out of L2: the ceiling is the random 4-byte
        # gather rate into a table of its size, measured here
        rate = ctypes.c_double()
        L.check(L.lib().bbt_measure_gather(local, max(fbytes, 1 << 20) // 4096 * 4096, 1 << 29, 0,
                                           5, ctypes.byref(rate)))
        l2_peak = rate.value * 32.0 / 1e9
        roofline.update({"bound": "l2", "peak": l2_peak, "frac": achieved / l2_peak,
                         "peak_kind": f"measured in this run: {rate.value / 1e9:.1f} G random "
                                      f"4-byte gathers/s into a table of the filter's size "
                                      "(bbt_measure_gather) x 32 B per probe",
                         "hbm_peak": peak, "hbm_frac": achieved / peak,
                         "hbm_peak_kind": peak_kind})
    else:
        # beside the sector roofline: the rate this GPU serves isolated random
        # 4-byte reads from a table of the filter's size (each a DRAM line
        # fill), measured here, against the probes the batched path issues
        rate = ctypes.c_double()
        L.check(L.lib().bbt_measure_gather(local, fbytes // 4096 * 4096, 1 << 29, 0, 5,
                                           ctypes.byref(rate)))
        issued_rate = issued / (k_ms * 1e-3)
        tpr = traffic_per_read("classify_varlen_dram.json")
        if tpr and tune["path"] != L.PATH_BUCKETED:
            roofline["traffic"] = tpr * n
            roofline["traffic_note"] = ("persistent kernel DRAM read+write per read from the "
                                        "committed ncu capture of 400k reads of this workload, "
                                        "scaled to the step's reads")
        roofline["random_gather"] = {
            "ceiling_per_s": rate.value, "issued_probes_per_s": issued_rate,
            "frac": issued_rate / rate.value if rate.value else None,
            "kind": "measured in this run: random 4-byte gathers/s into a table of the "
                    "filter's size, positions generated in the kernel (bbt_measure_gather)"}
    line = {
        "metric": SINGLE_METRIC, "value": world * n / (ms_batched * 1e-3), "unit": "reads/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_batched,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic",
        "config": single_config(cfg, args),
        "bases_per_gpu": bases, "filter_bytes": fbytes, "tuned": tune,
        "probes_per_s": world * alg_probes / (ms_batched * 1e-3),
        "probes_algorithmic_per_step": alg_probes, "probes_issued_per_step": issued,
        "frames_hashed_per_step": frames,
        "plain": {"value": world * n / (ms_plain * 1e-3), "unit": "reads/s",
                  "ms_per_step": ms_plain, "launches_per_step": plain_launches,
                  "reads_per_launch": PLAIN_BATCH, "equals_batched": plain_ok},
        "batched_over_plain": ms_plain / ms_batched,
        "batched_equals_counting_pass": batched_ok,
        "roofline": roofline,
        "cpu_baseline": cpu if cpu else {"value": None, "unavailable": cpu_err},
        "e2e": {"value": world * n / e2e_p_s, "unit": "reads/s",
                "h2d_bytes_per_step": packed_h2d,
                "d2h_bytes_per_step": int(n * (8 + 4)), "matches_device_results": e2e_p_ok,
                "input": "bbt_classify_batch on pinned host buffers, bases 2-bit packed "
                         "with validity bits (BBT_BASES_2BIT), packed before timing",
                "ascii": {"value": world * n / e2e_s, "unit": "reads/s",
                          "h2d_bytes_per_step": int(bases + (n + 1) * 8),
                          "d2h_bytes_per_step": int(n * (8 + 4)),
                          "matches_device_results": e2e_ok}},
        "gpu_launches": batched_launches * args.steps,
        "graph_launches_per_step": 1 if graph is not None else 0,
        "batched_path": {L.PATH_PLAIN: "plain", L.PATH_PERSISTENT: "persistent",
                         L.PATH_BUCKETED: "bucketed"}.get(tune["path"], str(tune["path"])),
        "clocks": clk,
        "parity_sample": parity,
        "batched_equals_reference_sample": (parity or {}).get("mismatched_reads") == 0,
    }
    print(json.dumps(line), flush=True)
    if graph is not None:
        graph.close()
    bbc.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def ref_single_setup(cfg, n_reads):
    """The single-filter workload built by the CPU oracle (generator restated
    in oracle/synth_oracle.c, threaded filter build): the same reference, bit
    array and first n_reads reads as single_setup, without the product
    library."""
    from tests import oracle_lib as ol
    d = os.path.join(tempfile.gettempdir(), f"bbt_ref_{cfg['seed']}")
    os.makedirs(d, exist_ok=True)
    t0 = time.time()
    g = ol.synth_genome(cfg["seed"], cfg["glen"], gc=cfg["gc"], repeat_frac=cfg["repeat_frac"],
                        rep_min=cfg["rep_min"], rep_max=cfg["rep_max"], div_min=cfg["div_min"],
                        div_max=cfg["div_max"])
    path = os.path.join(d, "genome.bf")
    if not (os.path.exists(path) and os.path.exists(path[:-2] + "txt")):
        ref_store_filter(ol.make_filter_par([g], k=K, fpr=FPR), path, "genome", "genome.fa")
    log(f"reference arm: reference + filter {time.time() - t0:.1f} s")
    p = ol.read_params(cfg["len_min"], cfg["len_max"], long_frac=cfg["long_frac"],
                       long_min=cfg["long_min"], long_max=cfg["long_max"], sub_rate=cfg["sub"])
    s1, off, _, _ = ol.synth_reads(cfg["seed"] + 17, [g], [cfg["ref_frac"]], n_reads, p)
    del g
    return d, path, s1, off


def run_single_reference(args):
    """CPU arm of a single-filter workload: the reference's own
    BioBloomClassifier::filter on a bounded sample of the workload's reads,
    each step one run on the same sample, all host threads."""
    if not ref_rank_zero():
        return
    cfg = SINGLE[args.workload]
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/ref_harness is not built"}))
        return
    d, path, s1, off = ref_single_setup(cfg, min(cfg["reads"], 4_000_000))
    threads = os.cpu_count() or 1

    def run(n):
        fq = os.path.join(d, f"sample_{n}.fq")
        if not os.path.exists(fq):
            write_single_fastq(fq, s1, off, n)
        pr = subprocess.run([harness, "time", str(SCORE), str(STREAK), str(threads), "0",
                             os.path.join(d, "refcpu"), path, fq], capture_output=True, text=True)
        if pr.returncode:
            return None, "ref_harness failed: " + pr.stderr[-300:]
        return json.loads([x for x in pr.stdout.splitlines() if x.startswith("{")][-1]), None

    probe = 20000
    r, err = run(probe)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    n = int(min(len(off) - 1, max(probe, probe / max(r["seconds"], 1e-6) * ref_step_budget(args))))
    n = max(probe, (n // 10000) * 10000)
    times = []
    for i in range(args.warmup + args.steps):
        r, err = run(n)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return
        if i >= args.warmup:
            times.append(r["seconds"])
    sec = sum(times) / len(times)
    value = n / sec
    print(json.dumps(ref_line(
        args, SINGLE_METRIC, value, sec, cfg["workload"],
        f"first {n} reads of the workload per step ({int(off[n])} bases), "
        f"BioBloomClassifier::filter compiled from the reference sources, {threads} OpenMP "
        "threads, filter load excluded", threads,
        {"config": single_config(cfg, args), "reads_per_step": n,
         "bases_per_step": int(off[n])})), flush=True)


def write_single_fastq(path, s1, off, n):
    with open(path, "wb") as f:
        f.write(b"".join(b"@r%d\n%s\n+\n%s\n" % (i, s1[off[i]:off[i + 1]].tobytes(),
                                                b"I" * int(off[i + 1] - off[i]))
                         for i in range(n)))


# ---------------------------------------------------------------- serving workload

SERVE_METRIC = "p50/p99 request latency and reads/s at fixed offered load, 1 B200"


def serve_pool(refs, frac, n, seed):
    from biobloom_b200 import synth
    p = synth.read_params(75, 300, long_frac=0.10, long_min=1000, long_max=10_000,
                          sub_rate=0.05)
    s1, off, _, _ = synth.reads(seed, refs, frac, n, p)
    return s1, off


def run_serve(args):
    import threading

    import torch

    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200.mibf import MIBFClassifier
    from biobloom_b200.server import Server

    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    cfg = SINGLE["varlen"]
    from biobloom_b200 import synth
    t0 = time.time()
    d = os.path.join(tempfile.gettempdir(), f"bbt_bench_{cfg['seed']}")
    os.makedirs(d, exist_ok=True)
    g = synth.genome(cfg["seed"], cfg["glen"], gc=cfg["gc"], repeat_frac=cfg["repeat_frac"],
                     rep_min=cfg["rep_min"], rep_max=cfg["rep_max"], div_min=cfg["div_min"],
                     div_max=cfg["div_max"])
    bf_path = os.path.join(d, "genome.bf")

    def build():
        if not (os.path.exists(bf_path) and os.path.exists(bf_path[:-2] + "txt")):
            synth.make_filter([g], bf_path[:-3], "genome", k=K, fpr=FPR, device=local,
                              sources="genome.fa")
    build_once(rank, pg, build)
    md = os.path.join(tempfile.gettempdir(), f"bbt_bench_mibf_{args.targets}")
    os.makedirs(md, exist_ok=True)
    mi_path, targets, _ = mi_build(md, args.targets, local, rank, pg)
    pool_n = 2_000_000
    bs, boff = serve_pool([g], [0.8], pool_n, 5151 + rank)
    ms, moff = serve_pool(targets, [0.9 / len(targets)] * len(targets), pool_n, 5252 + rank)
    del g, targets
    pools = {}
    for kind, (sq, of) in (("bloom", (bs, boff)), ("mibf", (ms, moff))):
        pools[kind] = (torch.from_numpy(sq[:int(of[-1])]).pin_memory(),
                       torch.from_numpy(of.view(np.int64)).pin_memory())
    log(f"serving setup: {time.time() - t0:.1f} s")
    bbc = BioBloomClassifier([bf_path], SCORE, streak_threshold=STREAK, device=local)
    bbc.set_launch(path=2, warps_per_block=8, frames_per_lane=8)
    bbc.set_schedule(1024)
    mc = MIBFClassifier(mi_path, device=local)
    rng = np.random.default_rng(555 + rank)
    n_req = args.requests
    sizes = np.exp(rng.uniform(np.log(1e3), np.log(1e6), n_req)).astype(np.int64)
    kinds = ["bloom" if k else "mibf" for k in rng.integers(0, 2, n_req)]
    starts = [int(rng.integers(0, pool_n - n)) for n in sizes]

    def prepare(srv):
        reqs = []
        for kind, n, st in zip(kinds, sizes, starts):
            sq, of = pools[kind]
            o = of[st:st + n + 1]
            if kind == "bloom":
                reqs.append(srv.submit_bloom(sq, o, submit=False))
            else:
                reqs.append(srv.submit_mibf(sq, o, max_hits=4, submit=False))
        return reqs

    total_reads = int(sizes.sum())
    total_bases = 0
    for kind, n, st in zip(kinds, sizes, starts):
        of = pools[kind][1]
        total_bases += int(of[st + n] - of[st])
    with Server(bbc, mc, slots=args.slots) as srv:
        reqs = prepare(srv)
        # warm-up and offline capacity: everything submitted at once
        offline = []
        for rep in range(2):
            t_start = time.perf_counter()
            for q in reqs:
                srv.submit_prepared(q)
            st = [srv.wait(q) for q in reqs]
            wall = time.perf_counter() - t_start
            offline.append(wall)
        off_s = min(offline)
        capacity = total_reads / off_s
        # online: Poisson arrivals at load x the offline request rate
        lam = args.load * n_req / off_s
        gaps = np.random.default_rng(777).exponential(1.0 / lam, n_req)
        arrivals = np.cumsum(gaps)
        clocks = ClockSampler(local)
        clocks.start()
        t_start = time.perf_counter()

        def submitter():
            for q, a in zip(reqs, arrivals):
                delay = t_start + a - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                srv.submit_prepared(q)

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        stats = [srv.wait(q) for q in reqs]
        wall = time.perf_counter() - t_start
        clk = clocks.stop()
    lat = np.array([s["t_done"] - s["t_submit"] for s in stats])
    queue = np.array([s["t_admit"] - s["t_submit"] for s in stats])
    span = max(s["t_done"] for s in stats) - min(s["t_submit"] for s in stats)
    small = lat[sizes < 10_000]
    line = {
        "metric": SERVE_METRIC, "value": total_reads / span, "unit": "reads/s",
        "n_gpus": world, "steps": 1, "warmup": 2, "ms_per_step": span * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic",
        "config": {"workload": ("serving: 3.1 Gbp filter + 500-target miBF resident; "
                                f"{n_req} requests of 1k-1M reads (log-uniform), half Bloom "
                                "half miBF, 75-300 bp with 10% 1-10 kb reads, 5% "
                                "substitutions, Poisson arrivals"),
                   "requests": n_req, "reads": total_reads, "bases": total_bases,
                   "offered_load": args.load, "slots": args.slots,
                   "arrival_rate_per_s": lam},
        "latency_ms": {"p50": float(np.percentile(lat, 50) * 1e3),
                       "p99": float(np.percentile(lat, 99) * 1e3),
                       "max": float(lat.max() * 1e3),
                       "p50_small_requests": (float(np.percentile(small, 50) * 1e3)
                                              if len(small) else None),
                       "queue_p50": float(np.percentile(queue, 50) * 1e3),
                       "queue_p99": float(np.percentile(queue, 99) * 1e3)},
        "offline": {"value": capacity, "unit": "reads/s", "seconds": off_s,
                    "note": "the same requests submitted all at once"},
        "e2e": {"value": total_reads / span, "unit": "reads/s",
                "h2d_bytes_per_step": int(total_bases + 8 * (total_reads + n_req)),
                "d2h_bytes_per_step": int(sum(n * (12 if k == "bloom" else 4 * 28 + 8)
                                              for k, n in zip(kinds, sizes)))},
        "cpu_baseline": {"value": None, "unavailable": "serving has no reference counterpart"},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    bbc.close()
    mc.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


# ---------------------------------------------------------------- miBF workload

MI_TARGET_LEN = 2_000_000
MI_SHARED = 0.20
MI_SUB = 0.01
MI_METRIC = "reads/s on 1 B200, miBF classification, % HBM sector peak"


def mi_workload(n_targets, n_reads):
    return (f"miBF over {n_targets} targets x 2 Mbp (35-65% GC, 20% shared between random "
            f"target pairs), 3 spaced seeds span 25 weight 19, {n_reads} single-end 150 bp "
            f"reads (90% from targets with 1% substitutions, 10% random)")


def mi_config(args):
    """The miBF workload's config, the same on the GPU arm and on the reference
    arm (figures of the run sit beside it in the line)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"workload": mi_workload(args.targets, args.reads), "reads_per_gpu": args.reads,
            "targets": args.targets, "l2": "inputs larger than L2 (3 GB reads + 5 GB miBF)",
            "parallelism": f"replicas x{world} (reads sharded, miBF replicated)"}


def mi_seeds(rng):
    out = []
    for _ in range(3):
        zeros = set(int(x) for x in rng.choice(np.arange(1, 24), 6, replace=False))
        out.append("".join("0" if i in zeros else "1" for i in range(25)))
    return out


def mi_targets(n_targets, genome=None):
    """The targets and spaced seeds; genome makes one seeded sequence (default:
    the product generator; the reference arm passes the oracle's copy, which
    makes the same bytes)."""
    if genome is None:
        from biobloom_b200 import synth
        genome = synth.genome
    rng = np.random.default_rng(4004)
    gcs = rng.uniform(0.35, 0.65, n_targets)
    pristine = [genome(4_000_000 + i, MI_TARGET_LEN, gc=float(gcs[i]))
                for i in range(n_targets)]
    out = [g.copy() for g in pristine]
    blk = int(MI_SHARED * MI_TARGET_LEN)
    for i in range(n_targets):
        j = int(rng.integers(0, n_targets - 1))
        j += j >= i
        a = int(rng.integers(0, MI_TARGET_LEN - blk))
        b = int(rng.integers(0, MI_TARGET_LEN - blk))
        out[i][b:b + blk] = pristine[j][a:a + blk]
    return out, mi_seeds(rng)


def mi_build(d, n_targets, device, rank=0, pg=None):
    from biobloom_b200.mibf import make_mibf
    t0 = time.time()
    targets, seeds = mi_targets(n_targets)
    path = os.path.join(d, "targets.bf")

    def build():
        if not all(os.path.exists(path[:-3] + e) for e in (".bf", ".sdsl", "_ids.txt")):
            make_mibf(path[:-3], [t.tobytes() for t in targets], list(range(1, n_targets + 1)),
                      [f"target{i + 1}" for i in range(n_targets)], seeds=seeds, occupancy=0.5,
                      device=device)
    build_once(rank, pg, build)
    log(f"targets + miBF: {time.time() - t0:.1f} s")
    return path, targets, seeds


def mi_reads(targets, n_reads, seed, oracle=False):
    """Reads of the miBF workload, by the product generator or (oracle=True)
    by the oracle's copy of it: the same bytes."""
    if oracle:
        from tests import oracle_lib as gen
        params, reads = gen.read_params, gen.synth_reads
    else:
        from biobloom_b200 import synth as gen
        params, reads = gen.read_params, gen.reads
    p = params(READ_LEN, READ_LEN, sub_rate=MI_SUB)
    frac = [0.9 / len(targets)] * len(targets)
    s1, off, _, _ = reads(seed, targets, frac, n_reads, p)
    return s1, off


def ref_mi_build(d, n_targets, threads):
    """The miBF workload's filter made without the product library: targets
    from the oracle's copy of the generator, written as one FASTA file (record
    i + 1 named target<i+1>, so IDs follow the target order), and the miBF from
    the reference's own maker (oracle/_ref/biobloommimaker, IDs by FASTA
    header, occupancy 0.5, the workload's spaced seeds).  Returns (path,
    targets, error)."""
    from tests import oracle_lib as ol
    t0 = time.time()
    targets, seeds = mi_targets(n_targets, genome=ol.synth_genome)
    path = os.path.join(d, "targets.bf")
    if not all(os.path.exists(path[:-3] + e) for e in (".bf", ".sdsl", "_ids.txt")):
        maker = os.path.join(ROOT, "oracle", "_ref", "biobloommimaker")
        if not os.path.exists(maker):
            return None, None, "oracle/_ref/biobloommimaker is not built"
        fa = os.path.join(d, "targets.fa")
        with open(fa, "wb") as f:
            for i, t in enumerate(targets):
                f.write(b">target%d\n" % (i + 1))
                f.write(t.tobytes())
                f.write(b"\n")
        pr = subprocess.run([maker, "-t", str(threads), "-p", "targets", "-b", "0.5",
                             "-S", " ".join(seeds), fa], cwd=d, capture_output=True, text=True)
        os.unlink(fa)
        if pr.returncode:
            return None, None, "reference MI maker failed: " + pr.stderr[-300:]
    log(f"reference arm: targets + miBF (reference maker) {time.time() - t0:.1f} s")
    return path, targets, None


def mi_cpu_run(d, path, s1, off, n, threads):
    """The reference's MI categorizer (oracle/_ref/biobloommicategorizer) on the
    first n reads; returns (seconds of its own classification timer, None)."""
    cli = os.path.join(ROOT, "oracle", "_ref", "biobloommicategorizer")
    if not os.path.exists(cli):
        return None, "oracle/_ref/biobloommicategorizer is not built"
    fa = os.path.join(d, f"sample_{n}.fa")
    if not os.path.exists(fa):
        with open(fa, "wb") as f:
            f.write(b"".join(b">r%d\n%s\n" % (i, s1[off[i]:off[i + 1]].tobytes())
                             for i in range(n)))
    p = subprocess.run([cli, "-t", str(threads), "-p", os.path.join(d, "refcpu"), "-f", path, fa],
                       stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True)
    if p.returncode:
        return None, "reference MI categorizer failed: " + p.stderr[-300:]
    for line in p.stderr.splitlines():
        if line.startswith("Classification time (s):"):
            return float(line.split(":")[1]), None
    return None, "no classification time in the reference's output"


def mi_cpu_baseline(d, path, s1, off, budget_s=15.0):
    threads = os.cpu_count() or 1
    probe = 20000
    sec, err = mi_cpu_run(d, path, s1, off, probe, threads)
    if sec is None:
        return None, err
    n = int(min(len(off) - 1, max(probe, probe / max(sec, 1e-6) * budget_s)))
    n = max(probe, (n // 10000) * 10000)
    sec, err = mi_cpu_run(d, path, s1, off, n, threads)
    if sec is None:
        return None, err
    return {"value": n / sec, "unit": "reads/s", "cores": threads, "kind": "reference",
            "sample": f"first {n} reads of the workload; the reference's MIBFClassifier::filter "
                      f"(BioBloomCategorizer sources) over the oracle's miBF structures, "
                      f"{threads} OpenMP threads, its own classification timer (filter load "
                      f"excluded)", "seconds": sec}, None


def mi_check_sample(path, s1, off, hits, nh, sat, n):
    try:
        from tests import mibf_util as mu
        from tests import oracle_lib as ol
    except Exception as e:
        return {"checked": 0, "error": str(e)}
    f = ol.MIBF.load(path)
    nids = 1
    with open(path[:-3] + "_ids.txt") as fh:
        nids += sum(1 for _ in fh)
    probs, _ = f.frame_probs(nids, f.f.h - 1)
    mc = mu.min_counts(READ_LEN - f.f.k + 1, probs, 1e-10)
    hits = hits[:n].cpu().numpy()
    nh = nh[:n].cpu().numpy()
    sat = sat[:n].cpu().numpy()
    bad = 0
    for i in range(n):
        s = s1[off[i]:off[i + 1]].tobytes()
        fc = len(s) - f.f.k + 1
        mcount = mc if fc == READ_LEN - f.f.k + 1 else mu.min_counts(fc, probs, 1e-10)
        want, wsat = f.query(s, mcount, allowed_miss=f.f.h - 1)
        got = [tuple(int(x) for x in hits[i, j]) for j in range(min(int(nh[i]), hits.shape[1]))]
        bad += (got != want) or int(sat[i]) != wsat or int(nh[i]) != len(want)
    return {"checked_reads": n, "mismatched_reads": int(bad)}


def run_mibf(args):
    import ctypes

    import torch

    from biobloom_b200 import _lib as L
    from biobloom_b200.mibf import MIBFClassifier

    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    d = os.path.join(tempfile.gettempdir(), f"bbt_bench_mibf_{args.targets}")
    os.makedirs(d, exist_ok=True)
    path, targets, _ = mi_build(d, args.targets, local, rank, pg)
    n = args.reads
    s1, off = mi_reads(targets, n, 6000 + rank)
    del targets
    bases = int(off[-1])
    h1 = torch.from_numpy(s1[:bases]).pin_memory()
    hoff = torch.from_numpy(off.view(np.int64)).pin_memory()
    d1, doff = h1.to(dev), hoff.to(dev)
    t0 = time.time()
    mc = MIBFClassifier(path, device=local, layout=args.layout)
    if args.mibf_bucketing >= 0:
        mc.set_bucketing(mode=args.mibf_bucketing)
    log(f"miBF load: {time.time() - t0:.1f} s")
    MH = 4
    hits = torch.empty((n, MH, 7), dtype=torch.int32, device=dev)
    nh = torch.empty(n, dtype=torch.int32, device=dev)
    sat = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    def step():
        mc.classify_device(d1, doff, stream=stream, out=(hits, nh, sat))

    for _ in range(args.warmup):
        step()
        mc.sync()
    counts = mc.last_counts()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kms = []
    e0.record(stream)
    for _ in range(args.steps):
        step()
        mc.sync()
        kms.append(mc.last_kernel_ms())
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    kernel_ms = sum(kms) / len(kms)
    if pg:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())

    parity = None
    if rank == 0 and not args.no_check:
        parity = mi_check_sample(path, s1, off, hits, nh, sat, 2000)

    # e2e: the C ABI with pinned host buffers (reads in, results out)
    hh = torch.empty((n, MH, 7), dtype=torch.int32).pin_memory()
    hn = torch.empty(n, dtype=torch.int32).pin_memory()
    hs = torch.empty(n, dtype=torch.int32).pin_memory()

    def e2e_step():
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = h1.data_ptr(), hoff.data_ptr(), n, L.HOST
        r = L.MibfResult()
        r.hits, r.max_hits, r.n_hits, r.sat_count, r.location = (
            hh.data_ptr(), MH, hn.data_ptr(), hs.data_ptr(), L.HOST)
        L.check_mibf(L.lib().bbt_mibf_classify_batch(mc._ctx, ctypes.byref(b), ctypes.byref(r),
                                                     None), mc._ctx)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if pg:
        t = torch.tensor([e2e_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_ok = bool(torch.equal(hn, nh.cpu()) and torch.equal(hs, sat.cpu()))

    # the same over the packed boundary form (BBT_BASES_2BIT), packed before timing
    pw = torch.empty(((bases + 15) // 16 + 1,), dtype=torch.int32).pin_memory()
    pv = torch.empty(((bases + 31) // 32 + 1,), dtype=torch.int32).pin_memory()
    n_bad = ctypes.c_uint64()
    L.check(L.lib().bbt_pack_bases(h1.data_ptr(), bases, pw.data_ptr(), pv.data_ptr(),
                                   ctypes.byref(n_bad)))
    hn.zero_()
    hs.zero_()

    def e2e_packed_step():
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = pw.data_ptr(), hoff.data_ptr(), n, L.HOST
        b.encoding, b.valid = L.BASES_2BIT, (pv.data_ptr() if n_bad.value else None)
        r = L.MibfResult()
        r.hits, r.max_hits, r.n_hits, r.sat_count, r.location = (
            hh.data_ptr(), MH, hn.data_ptr(), hs.data_ptr(), L.HOST)
        L.check_mibf(L.lib().bbt_mibf_classify_batch(mc._ctx, ctypes.byref(b), ctypes.byref(r),
                                                     None), mc._ctx)

    for _ in range(max(1, args.warmup)):
        e2e_packed_step()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_packed_step()
    e2e_p_s = (time.perf_counter() - t0) / args.steps
    if pg:
        t = torch.tensor([e2e_p_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_p_s = float(t.item())
    e2e_p_ok = bool(torch.equal(hn, nh.cpu()) and torch.equal(hs, sat.cpu()))
    packed_h2d = int(((bases + 15) // 16) * 4 + (((bases + 31) // 32) * 4 if n_bad.value else 0)
                     + (n + 1) * 8)
    del pw, pv

    if rank != 0:
        mc.close()
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    cpu, cpu_err = (None, "skipped (--no-cpu)")
    if world == 1 and not args.no_cpu:
        cpu, cpu_err = mi_cpu_baseline(d, path, s1, off)
    frames, probes, phits = counts
    peak, peak_kind = measured_peaks()
    dense = mc.layout == L.MIBF_LAYOUT_DENSE
    # one 32-byte sector per random read: dense = one read per probe; rank
    # layout = a block read per probe and an ID read per hit
    alg_bytes = 32.0 * probes + (0.0 if dense else 32.0 * phits) + bases / 4.0 + 8.0 * n
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    tpr = None
    tp = os.path.join(ROOT, "profiles", "mibf_query_dram.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tpr = json.load(f).get("dram_bytes_per_read")
    line = {
        "metric": MI_METRIC, "value": world * n / (ms * 1e-3), "unit": "reads/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic",
        "config": mi_config(args),
        "layout": "dense ID map" if dense else "rank blocks + ID array",
        "bucketed_query": {-1: "off (default)", 0: "off", 1: "on", 2: "auto"}[args.mibf_bucketing],
        "filter_bytes": int(os.path.getsize(path) + os.path.getsize(path[:-3] + ".sdsl")),
        "frames_per_step": frames, "probes_per_step": probes, "probe_hits_per_step": phits,
        "probes_per_s": world * probes / (ms * 1e-3),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": (tpr * n if tpr else None),
                     "kernel": "mibf_query_kernel", "kernel_ms": kernel_ms,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "algorithmic_bytes_note": ("32 B sector per probe (dense ID map)" if dense else
                                                "32 B block sector per probe + 32 B ID sector "
                                                "per hit") + " + 2-bit bases + 8 B results per "
                                                             "read"},
        "cpu_baseline": cpu if cpu else {"value": None, "unavailable": cpu_err},
        "e2e": {"value": world * n / e2e_p_s, "unit": "reads/s",
                "h2d_bytes_per_step": packed_h2d,
                "d2h_bytes_per_step": int(n * (MH * 28 + 8)),
                "matches_device_results": e2e_p_ok,
                "input": "bbt_mibf_classify_batch on pinned host buffers, bases 2-bit packed "
                         "with validity bits (BBT_BASES_2BIT), packed before timing",
                "ascii": {"value": world * n / e2e_s, "unit": "reads/s",
                          "h2d_bytes_per_step": int(bases + (n + 1) * 8),
                          "d2h_bytes_per_step": int(n * (MH * 28 + 8)),
                          "matches_device_results": e2e_ok}},
        "gpu_launches": 3 * args.steps,
        "clocks": clk,
        "parity_sample": parity,
    }
    print(json.dumps(line), flush=True)
    mc.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def run_mibf_reference(args):
    """The miBF workload's CPU arm: the reference's own MI categorizer on a
    bounded sample of the workload's reads, all host threads, over inputs made
    without the product library (ref_mi_build)."""
    if not ref_rank_zero():
        return
    d = os.path.join(tempfile.gettempdir(), f"bbt_ref_mibf_{args.targets}")
    os.makedirs(d, exist_ok=True)
    threads = os.cpu_count() or 1
    path, targets, err = ref_mi_build(d, args.targets, threads)
    if path is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    s1, off = mi_reads(targets, 400_000, 6000, oracle=True)
    sec, err = mi_cpu_run(d, path, s1, off, 20000, threads)
    if sec is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    n = int(min(400_000, max(20000, 20000 / max(sec, 1e-6) * 10.0)))
    n = (n // 10000) * 10000
    times = []
    for i in range(args.warmup + args.steps):
        sec, err = mi_cpu_run(d, path, s1, off, n, threads)
        if sec is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return
        if i >= args.warmup:
            times.append(sec)
    sec = sum(times) / len(times)
    value = n / sec
    print(json.dumps(ref_line(
        args, MI_METRIC, value, sec, mi_workload(args.targets, args.reads),
        f"first {n} reads of the workload per step, MIBFClassifier::filter from the reference "
        f"sources over the shim's miBF structures, {threads} OpenMP threads, filter load "
        "excluded", threads,
        {"config": mi_config(args), "reads_per_step": n,
         "inputs": "targets and reads made by the CPU oracle's generator (oracle/synth_oracle.c, "
                   "the same bytes as the GPU arm's), the miBF by the reference's own maker "
                   "(oracle/_ref/biobloommimaker)"})), flush=True)


# ---------------------------------------------------------------- gather ceilings

def run_gather(args):
    """Random 4-byte gather rates of this GPU (bbt_measure_gather): positions
    streamed from HBM into tables that fit L2, and positions generated in the
    kernel into tables from L2 size to several GB.  Prints one JSON line."""
    import ctypes

    from biobloom_b200 import _lib as L
    lib = L.lib()
    out = {"workload": "random 4-byte gathers (bbt_measure_gather)", "unit": "gathers/s",
           "n_gathers": 1 << 29, "reps": 5, "streamed": {}, "generated": {}}
    rate = ctypes.c_double()
    for mb in (4, 8, 16, 24, 32, 48, 64, 80, 96, 128, 192, 256, 512):
        L.check(lib.bbt_measure_gather(0, mb << 20, 1 << 29, 1, 5, ctypes.byref(rate)))
        out["streamed"][f"{mb}MB"] = rate.value
        log(f"streamed {mb} MB: {rate.value / 1e9:.1f} G/s")
    for mb in (16, 32, 64, 96, 128, 1024, 2048, 4096, 8192):
        L.check(lib.bbt_measure_gather(0, mb << 20, 1 << 29, 0, 5, ctypes.byref(rate)))
        out["generated"][f"{mb}MB"] = rate.value
        log(f"generated {mb} MB: {rate.value / 1e9:.1f} G/s")
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pairs", type=int, default=10_000_000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--l2-fetch", type=int, default=0, help="L2 fetch granularity (bytes)")
    ap.add_argument("--workload", default="varlen",
                    choices=["varlen", "bf", "mibf", "small", "serve", "modes", "gather"])
    ap.add_argument("--requests", type=int, default=200, help="requests (--workload serve)")
    ap.add_argument("--load", type=float, default=0.7,
                    help="offered load, fraction of offline capacity (--workload serve)")
    ap.add_argument("--slots", type=int, default=4, help="server slots (--workload serve)")
    ap.add_argument("--targets", type=int, default=500, help="miBF targets (--workload mibf)")
    ap.add_argument("--reads", type=int, default=None,
                    help="reads (--workload mibf / varlen / small; default: the workload's)")
    ap.add_argument("--layout", type=int, default=0, help="miBF layout: 0 auto, 1 rank, 2 dense")
    ap.add_argument("--mibf-bucketing", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="miBF bucketed query (bbt_mibf_set_bucketing mode; -1: the default)")
    ap.add_argument("--step-form", default="decision", choices=sorted(STEP_FORMS),
                    help="steps of a pinned persistent path (bbt_set_steps)")
    ap.add_argument("--path", default="auto", choices=["auto", "persistent", "bucketed"],
                    help="batched path of the single-filter workloads (default: autotuned)")
    ap.add_argument("--bucketing", default="",
                    help="settings of the bucketed path, e.g. 'bucket_shift=27,phase_split=4,"
                         "levels_per_round=1' (bbt_set_bucketing; --path bucketed)")
    args = ap.parse_args()
    args.reads_set = args.reads is not None
    if args.reads is None:
        args.reads = 20_000_000
    if args.warmup < 3:
        log("warning: fewer than 3 warm-up steps")
    if args.workload == "gather":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "a property of the GPU; the reference has no GPU path"}))
        else:
            run_gather(args)
    elif args.workload == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the serving engine has no counterpart in the reference"}))
        else:
            run_serve(args)
    elif args.workload == "mibf":
        (run_mibf_reference if args.impl == "reference" else run_mibf)(args)
    elif args.workload == "modes":
        if args.impl == "reference":
            run_reference(args)
        else:
            run_modes(args)
    elif args.workload in SINGLE:
        (run_single_reference if args.impl == "reference" else run_single)(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
