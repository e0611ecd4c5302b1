"""Command-line errors of biobloomcategorizer and biobloommicategorizer against
the reference CLIs built from their own sources (oracle/_ref/): for each
invalid invocation both exit with the same status and print the same
messages, in the same order (BioBloomCategorizer.cpp and
BioBloomMICategorizer.cpp option checks; an invalid option's message names the
program path, which is normalised).  Every case stops before any filter is
loaded, so no device is needed."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "biobloomcategorizer")
OURS = os.path.join(ROOT, "biobloom_b200", "bin", "biobloomcategorizer")
MI_REF = os.path.join(ROOT, "oracle", "_ref", "biobloommicategorizer")
MI_OURS = os.path.join(ROOT, "biobloom_b200", "bin", "biobloommicategorizer")

CASES = {
    "nothing": [],
    "no_input": ["-f", "x.bf"],
    "no_filter": ["r.fq"],
    "fa_and_fq": ["-f", "x.bf", "--fa", "--fq", "r.fq"],
    "fa_and_fq_no_input": ["-f", "x.bf", "--fa", "--fq"],
    "negative_score": ["-f", "x.bf", "-s", "-3", "r.fq"],
    "three_paired_files": ["-f", "x.bf", "-e", "a.fq", "b.fq", "c.fq"],
    "unknown_scoring": ["-f", "x.bf", "-S", "foo", "r.fq"],
    "scores_without_output": ["-f", "x.bf", "-w", "r.fq"],
    "list_and_files": ["-f", "x.bf", "-l", "list.txt", "r.fq"],
    "missing_filter_file": ["-f", "x.bf", "r.fq"],
    "missing_folder": ["-f", "x.bf", "-p", "nodir/pre", "r.fq"],
    "folder_is_a_file": ["-f", "x.bf", "-p", "afile/pre", "r.fq"],
    "bad_streak": ["-f", "x.bf", "-r", "abc", "r.fq"],
    "besthit_and_scores": ["-f", "x.bf", "-b", "-w", "r.fq"],
    "scoring_and_besthit": ["-f", "x.bf", "-S", "harmonic", "-b", "r.fq"],
    "unknown_option": ["-f", "x.bf", "-z", "r.fq"],
    "bad_threads": ["-f", "x.bf", "-t", "abc", "r.fq"],
    "bad_interval": ["-f", "x.bf", "-I", "abc", "r.fq"],
    "bad_dust_threshold": ["-f", "x.bf", "-T", "abc", "r.fq"],
    "bad_dust_window": ["-f", "x.bf", "-W", "abc", "r.fq"],
    "score_above_one": ["-f", "x.bf", "-s", "1.5", "r.fq"],
    "bad_binomial_score": ["-f", "x.bf", "-S", "binomial", "-s", "abc", "r.fq"],
    "ordered_and_besthit": ["-f", "x.bf", "-c", "-b", "r.fq"],
}

# -r is left out: this implementation warns that it has no effect (the rule it feeds
# lives in a submodule absent from the reference tree)
MI_CASES = {
    "nothing": [],
    "no_input": ["-f", "x.bf"],
    "no_filter": ["r.fq"],
    "missing_filter_file": ["-f", "x.bf", "r.fq"],
    "one_paired_file": ["-f", "x.bf", "-e", "a.fq"],
    "three_paired_files": ["-f", "x.bf", "-e", "a.fq", "b.fq", "c.fq"],
    "missing_folder": ["-f", "x.bf", "-p", "nodir/pre", "r.fq"],
    "folder_is_a_file": ["-f", "x.bf", "-p", "afile/pre", "r.fq"],
    "fa_and_fq": ["-f", "x.bf", "--fa", "--fq", "r.fq"],
    "bad_score": ["-f", "x.bf", "-s", "abc", "r.fq"],
    "bad_frame_matches": ["-f", "x.bf", "-a", "-1", "r.fq"],
    "multi_above_one": ["-f", "x.bf", "-m", "2", "r.fq"],
    "bad_threads": ["-f", "x.bf", "-t", "abc", "r.fq"],
    "bad_interval": ["-f", "x.bf", "-I", "abc", "r.fq"],
    "unknown_option": ["-f", "x.bf", "-z", "r.fq"],
}


def _binaries(ref, ours):
    if not os.path.exists(ref):
        pytest.skip(f"{os.path.relpath(ref, ROOT)} is not built (make -C oracle ref)")
    if not os.path.exists(ours):
        pytest.fail(f"{os.path.relpath(ours, ROOT)} is not built")
    return ref, ours


def _compare(binaries, args, tmp_path):
    (tmp_path / "afile").write_text("x")
    out = []
    for exe in binaries:
        p = subprocess.run([exe] + args, cwd=tmp_path, capture_output=True, text=True,
                           timeout=60)
        out.append((p.returncode, p.stderr.replace(exe, "PROGRAM"), p.stdout))
    assert out[1] == out[0]
    return out[0][0]


@pytest.mark.parametrize("case", sorted(CASES))
def test_argument_errors_match_reference_cli(case, tmp_path):
    rc = _compare(_binaries(REF, OURS), CASES[case], tmp_path)
    assert rc != 0 or case == "bad_interval"   # the reference returns 0 on a bad -I


@pytest.mark.parametrize("case", sorted(MI_CASES))
def test_mi_argument_errors_match_reference_cli(case, tmp_path):
    rc = _compare(_binaries(MI_REF, MI_OURS), MI_CASES[case], tmp_path)
    assert rc != 0 or case == "bad_interval"   # the reference returns 0 on a bad -I
