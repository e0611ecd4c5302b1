"""The miBF oracle against the reference MI categorizer, live, on seeded random
cases: a miBF made by the reference's own maker (oracle/_ref/biobloommimaker)
from six targets that share segments, single-end reads and pairs classified by the
reference CLI (oracle/_ref/biobloommicategorizer) and by the oracle's query,
the latter formatted as the CLI's TSV records (MIBFClassifier.hpp:652-736):
the texts must be equal; and the reference maker's files against the oracle's
build, byte for byte.  Host only; skipped where the reference has not been
built (make -C oracle ref)."""
import os
import subprocess

import numpy as np
import pytest

from tests import mibf_util as mu
from tests import oracle_lib as ol

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAKER = os.path.join(ROOT, "oracle", "_ref", "biobloommimaker")
CAT = os.path.join(ROOT, "oracle", "_ref", "biobloommicategorizer")


def _seeds(rng):
    out = []
    for _ in range(3):
        zeros = set(int(x) for x in rng.choice(np.arange(1, 24), 6, replace=False))
        out.append("".join("0" if i in zeros else "1" for i in range(25)))
    return out


def _reads(rng, targets, n):
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    reads = []
    for _ in range(n):
        length = int(rng.integers(20, 300))
        if rng.random() < 0.8:
            t = targets[int(rng.integers(0, 6))]
            st = int(rng.integers(0, len(t) - length))
            r = t[st:st + length].copy()
            m = rng.random(length) < 0.02
            r[m] = rng.choice(acgt, int(m.sum()))
        else:
            r = rng.choice(acgt, length)
        if rng.random() < 0.1:
            r[int(rng.integers(0, length))] = ord("N")
        reads.append(r.tobytes())
    return reads


def _write(path, reads):
    with open(path, "wb") as f:
        for i, r in enumerate(reads):
            f.write(b">r%d\n%s\n" % (i, r))


def _case(rng, tmp_path, paired):
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    targets = [rng.choice(acgt, 30000) for _ in range(6)]
    for i in range(6):                       # shared segments between targets
        j = (i + 1 + int(rng.integers(0, 5))) % 6
        a, b = int(rng.integers(0, 27000)), int(rng.integers(0, 27000))
        targets[i][b:b + 3000] = targets[j][a:a + 3000]
    with open(tmp_path / "targets.fa", "wb") as f:
        for i, t in enumerate(targets):
            f.write(b">t%d\n%s\n" % (i + 1, t.tobytes()))
    mates = [_reads(rng, targets, 400) for _ in range(2 if paired else 1)]
    for m, reads in enumerate(mates):
        _write(tmp_path / f"reads_{m + 1}.fa", reads)
    return mates


@pytest.mark.parametrize("seed,args,paired", [
    (1, [], False), (2, ["-s", "50"], False), (3, ["-a", "2", "-c", "1"], False),
    (4, ["-b", "-m", "2"], False), (5, ["-i"], False), (6, [], True), (7, ["-i", "-b"], True)])
def test_oracle_records_equal_reference_cli(seed, args, paired, tmp_path):
    if not (os.path.exists(MAKER) and os.path.exists(CAT)):
        pytest.skip("the reference's miBF maker / categorizer are not built (make -C oracle ref)")
    rng = np.random.default_rng(seed)
    seeds = _seeds(rng)
    mates = _case(rng, tmp_path, paired)
    subprocess.run([MAKER, "-t", "2", "-p", "x", "-S", " ".join(seeds), "targets.fa"],
                   cwd=tmp_path, check=True, capture_output=True)
    # one thread: the reference CLI then writes the records in input order
    files = ["-e", "reads_1.fa", "reads_2.fa"] if paired else ["reads_1.fa"]
    p = subprocess.run([CAT, "-t", "1", "-p", "out", "-f", "x.bf"] + args + files,
                       cwd=tmp_path, check=True, capture_output=True)
    want = p.stdout.decode()

    f = ol.MIBF.load(str(tmp_path / "x.bf"))
    names = ["repeat"]
    with open(tmp_path / "x_ids.txt") as fh:
        names += [line.split()[1] for line in fh]
    o = mu.options(args)
    h = f.f.h
    allowed = 0 if (o["frame_matches"] > h or f.f.nseeds == 0) else h - o["frame_matches"]
    probs, _ = f.frame_probs(len(names), allowed)
    cache, text, hits = {}, [], 0
    for i, s in enumerate(mates[0]):
        s2 = mates[1][i] if paired else None
        fc = mu.frame_count(len(s), len(s2) if paired else 0, f.f.k, paired)
        res, sat = [], 0
        if fc:
            if fc not in cache:
                cache[fc] = mu.min_counts(fc, probs, o["score"])
            res, sat = f.query(s, cache[fc], seq2=s2, multi=o["multi"], allowed_miss=allowed,
                               min_nonsat=o["min_nonsat"], best_agree=o["best"])
        hits += bool(res)
        if o["hit_only"] and not res:
            continue
        for m in range(len(mates)):
            text.append(mu.format_record(names, o["out"], f"r{i}", "", mates[m][i], b"", res,
                                         sat))
    assert hits > 0                          # the case exercises matches
    assert "".join(text) == want


@pytest.mark.parametrize("seed,mode", [(21, "seeds"), (22, "kmers"), (23, "seeds")])
def test_oracle_build_equals_reference_maker(seed, mode, tmp_path):
    """The reference's own miBF maker (BioBloomMIMaker.cpp / MIBFGen.hpp over the
    shim's MIBFConstructSupport) and the oracle's build write the same .bf and
    .sdsl bytes, for spaced seeds and for k-mers with 3 hashes, IDs by FASTA
    header."""
    import filecmp
    if not os.path.exists(MAKER):
        pytest.skip("oracle/_ref/biobloommimaker is not built (make -C oracle ref)")
    rng = np.random.default_rng(seed)
    seeds = _seeds(rng)
    _case(rng, tmp_path, False)
    targets = []
    with open(tmp_path / "targets.fa", "rb") as fh:
        for line in fh.read().split(b"\n"):
            if line and not line.startswith(b">"):
                targets.append(line)
    opts = ["-S", " ".join(seeds)] if mode == "seeds" else ["-k", "25", "-g", "3"]
    subprocess.run([MAKER, "-t", "2", "-p", "x"] + opts + ["targets.fa"], cwd=tmp_path,
                   check=True, capture_output=True)
    m = ol.MIBF.build(targets, list(range(1, len(targets) + 1)),
                      seeds=seeds if mode == "seeds" else None, k=25, h=3, occupancy=0.5)
    m.store(str(tmp_path / "o"))
    for ext in (".bf", ".sdsl"):
        assert filecmp.cmp(tmp_path / ("o" + ext), tmp_path / ("x" + ext), shallow=False), ext
