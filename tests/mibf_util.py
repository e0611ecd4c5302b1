"""Shared pieces of the miBF tests: the golden cases of tests/golden/mibf/ and
the oracle's records / summaries for them (restating MIBFClassifier's
record and summary output in Python)."""
import math
import os

from tests import oracle_lib
from tests.fixtures import read_fastx

MIBF_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mibf")

# name: (filter prefix, CLI args, paired; None = the edge-case file)
CASES = {
    "ss_se": ("ss", [], False),
    "ss_se_s50_m2": ("ss", ["-s", "50", "-m", "2"], False),
    "ss_se_a2_c2": ("ss", ["-a", "2", "-c", "2"], False),
    "ss_se_a3_b": ("ss", ["-a", "3", "-b"], False),
    "ss_se_hit": ("ss", ["-i"], False),
    "ss_se_fa": ("ss", ["--fa"], False),
    "ss_pe": ("ss", [], True),
    "ss_pe_hit_b": ("ss", ["-i", "-b", "-m", "3"], True),
    "ss_pe_fq": ("ss", ["--fq"], True),
    "ss_edge": ("ss", [], None),
    "km_se": ("km", [], False),
    "km_pe": ("km", [], True),
}


def g(name):
    return os.path.join(MIBF_GOLDEN, name)


def options(args):
    o = {"score": 1e-10, "multi": 1.0, "frame_matches": 1, "min_nonsat": 0, "best": False,
         "hit_only": False, "out": "tsv"}
    i = 0
    while i < len(args):
        a = args[i]
        if a == "-s":
            o["score"] = math.pow(10.0, -(float(args[i + 1]) / 10.0))
            i += 1
        elif a == "-m":
            o["multi"] = float(args[i + 1])
            i += 1
        elif a == "-a":
            o["frame_matches"] = int(args[i + 1])
            i += 1
        elif a == "-c":
            o["min_nonsat"] = int(args[i + 1])
            i += 1
        elif a == "-b":
            o["best"] = True
        elif a == "-i":
            o["hit_only"] = True
        elif a == "--fa":
            o["out"] = "fa"
        elif a == "--fq":
            o["out"] = "fq"
        i += 1
    return o


def read_records(path):
    """[(name, comment, seq, qual)] with kseq's name / comment split."""
    import gzip
    op = gzip.open if path.endswith(".gz") else open
    with op(path, "rb") as f:
        lines = f.read().split(b"\n")
    out = []
    i = 0
    while i < len(lines):
        line = lines[i]
        if line.startswith(b">") or line.startswith(b"@"):
            head = line[1:].decode()
            parts = head.split(None, 1)
            name = parts[0] if parts else ""
            comment = parts[1] if len(parts) > 1 else ""
            if line.startswith(b">"):
                seq = lines[i + 1] if i + 1 < len(lines) and not lines[i + 1].startswith(b">") \
                    else b""
                out.append((name, comment, seq, b""))
                i += 2 if seq else 1
            else:
                out.append((name, comment, lines[i + 1], lines[i + 3]))
                i += 4
        else:
            i += 1
    return out


def inputs(paired):
    if paired is None:
        return [read_records(g("reads_edge.fa.gz"))]
    if paired:
        return [read_records(g("reads_1.fq.gz")), read_records(g("reads_2.fq.gz"))]
    return [read_records(g("reads_se.fa.gz"))]


def names_of(prefix):
    names = ["repeat"]
    with open(g(f"{prefix}_ids.txt")) as f:
        for line in f:
            names.append(line.split()[1])
    return names


def min_counts(fc, probs, score):
    n = len(probs)
    return [0] + [max(1, oracle_lib.binom_upper_quantile(fc, float(probs[i]), score / (n - 1)))
                  for i in range(1, n)]


def frame_count(len1, len2, k, paired):
    if not paired:
        return len1 - k + 1 if len1 >= k else 0
    return len1 - k + 1 if len1 >= k else (len2 - k + 1 if len2 >= k else 0)


def oracle_results(case):
    """Per read (pair): (results, sat_count) from the oracle."""
    prefix, args, paired = CASES[case]
    o = options(args)
    f = oracle_lib.MIBF.load(g(f"{prefix}.bf"))
    names = names_of(prefix)
    h = f.f.h
    allowed = 0 if (o["frame_matches"] > h or f.f.nseeds == 0) else h - o["frame_matches"]
    probs, _ = f.frame_probs(len(names), allowed)
    recs = inputs(paired)
    cache = {}
    out = []
    for i in range(len(recs[0])):
        s1 = recs[0][i][2]
        s2 = recs[1][i][2] if paired else None
        fc = frame_count(len(s1), len(s2) if s2 is not None else 0, f.f.k, bool(paired))
        if fc == 0:
            out.append(([], 0))
            continue
        if fc not in cache:
            cache[fc] = min_counts(fc, probs, o["score"])
        res, sat = f.query(s1, cache[fc], seq2=s2, multi=o["multi"], allowed_miss=allowed,
                           min_nonsat=o["min_nonsat"], best_agree=o["best"])
        out.append((res, sat))
    return out, names, o, recs


def format_record(names, out, name, comment, seq, qual, res, sat):
    """formatOutStr (MIBFClassifier.hpp:652-736) in Python."""
    def results():
        return "\t" + ";".join(
            names[r[0]] + "," + ",".join(str(x) for x in r[1:]) for r in res)
    nc = name + (" " + comment if comment else "")
    if out in ("fa", "fq"):
        s = (">" if out == "fa" else "@") + nc
        if res:
            s += "\t" + names[res[0][0]] + results()
        s += "\n" + seq.decode()
        if out == "fq":
            s += "\n+\n" + qual.decode()
        return s + "\n"
    if not res:
        return f"*\t{nc}\t{sat}\t*\n"
    return f"{names[res[0][0]]}\t{nc}\t{sat}" + results() + "\n"


def summary_text(names, results, paired, hit_only):
    """ResultsManager<ID>::updateSummaryData + getResultsSummary."""
    nf = len(names)
    above = [0] * (nf + 2)
    unique = [0] * (nf + 2)
    multi = nomatch = 0
    for res, _ in results:
        if paired and hit_only and not res:
            continue
        for r in res:
            above[r[0]] += 1
        if not res:
            nomatch += 1
        elif len(res) == 1:
            unique[res[0][0]] += 1
        else:
            multi += 1
    n = len(results)

    def fmt(x):
        return "%g" % x
    lines = ["filter_id\thits\tmisses\tshared\trate_hit\trate_miss\trate_shared"]
    for i in range(nf):
        lines.append("\t".join([names[i], str(above[i]), str(n - above[i]),
                                str(above[i] - unique[i]), fmt(above[i] / n),
                                fmt((n - above[i]) / n), fmt((above[i] - unique[i]) / n)]))
    lines.append("\t".join(["multiMatch", str(multi), str(n - multi), "0", fmt(multi / n),
                            fmt((n - multi) / n), "0"]))
    lines.append("\t".join(["noMatch", str(nomatch), str(n - nomatch), "0", fmt(nomatch / n),
                            fmt((n - nomatch) / n), "0"]))
    return "\n".join(lines) + "\n"
