"""The miBF oracle against the reference MI categorizer, live, on seeded random
cases: a miBF made by the reference's own maker (oracle/_ref/biobloommimaker)
from six targets that share segments, single-end reads classified by the
reference CLI (oracle/_ref/biobloommicategorizer) and by the oracle's query,
the latter formatted as the CLI's TSV records (MIBFClassifier.hpp:652-736):
the texts must be equal.  Host only; skipped where the reference has not been
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


def _case(rng, tmp_path):
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    targets = [rng.choice(acgt, 30000) for _ in range(6)]
    for i in range(6):                       # shared segments between targets
        j = (i + 1 + int(rng.integers(0, 5))) % 6
        a, b = int(rng.integers(0, 27000)), int(rng.integers(0, 27000))
        targets[i][b:b + 3000] = targets[j][a:a + 3000]
    with open(tmp_path / "targets.fa", "wb") as f:
        for i, t in enumerate(targets):
            f.write(b">t%d\n%s\n" % (i + 1, t.tobytes()))
    reads = []
    for _ in range(400):
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
    with open(tmp_path / "reads.fa", "wb") as f:
        for i, r in enumerate(reads):
            f.write(b">r%d\n%s\n" % (i, r))
    return reads


@pytest.mark.parametrize("seed,args", [(1, []), (2, ["-s", "50"]), (3, ["-a", "2", "-c", "1"]),
                                       (4, ["-b", "-m", "2"]), (5, ["-i"])])
def test_oracle_records_equal_reference_cli(seed, args, tmp_path):
    if not (os.path.exists(MAKER) and os.path.exists(CAT)):
        pytest.skip("the reference's miBF maker / categorizer are not built (make -C oracle ref)")
    rng = np.random.default_rng(seed)
    seeds = _seeds(rng)
    reads = _case(rng, tmp_path)
    subprocess.run([MAKER, "-t", "2", "-p", "x", "-S", " ".join(seeds), "targets.fa"],
                   cwd=tmp_path, check=True, capture_output=True)
    # one thread: the reference CLI then writes the records in input order
    p = subprocess.run([CAT, "-t", "1", "-p", "out", "-f", "x.bf"] + args + ["reads.fa"],
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
    for i, s in enumerate(reads):
        fc = mu.frame_count(len(s), 0, f.f.k, False)
        res, sat = [], 0
        if fc:
            if fc not in cache:
                cache[fc] = mu.min_counts(fc, probs, o["score"])
            res, sat = f.query(s, cache[fc], multi=o["multi"], allowed_miss=allowed,
                               min_nonsat=o["min_nonsat"], best_agree=o["best"])
        hits += bool(res)
        if o["hit_only"] and not res:
            continue
        text.append(mu.format_record(names, o["out"], f"r{i}", "", s, b"", res, sat))
    assert hits > 0                          # the case exercises matches
    assert "".join(text) == want
