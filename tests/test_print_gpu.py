"""Categorized read outputs of the biobloomcategorizer CLI (--fa / --fq, -g,
-e, -i, -d, -n) against the reference CLI's files on the same fixtures
(tests/golden/make_golden_print.py), byte for byte after decompression."""
import gzip
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CLI = os.path.join(ROOT, "biobloom_b200", "bin", "biobloomcategorizer")
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden_print as mgp  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", sorted(mgp.CASES))
def test_categorized_outputs_match_reference(case, tmp_path):
    args, paired = mgp.CASES[case]
    filters = " ".join(os.path.join(mgp.BBT, f"f{i}.bf") for i in range(3))
    p = subprocess.run([CLI, "-p", str(tmp_path / "out"), "-f", filters] + args +
                       mgp.inputs(paired), capture_output=True)
    assert p.returncode == 0, p.stderr.decode()
    got = mgp.collect(str(tmp_path), p.stdout)
    with gzip.open(os.path.join(mgp.BBT, f"print_{case}.txt.gz"), "rb") as f:
        want = f.read()
    assert got == want
