"""The GPU miBF maker (bbt_mibf_make) writes, byte for byte, the files of the
reference's own miBF maker driver (BioBloomMIMaker.cpp / MIBFGen.hpp compiled
from the reference sources over the shim's restated construction support;
tests/golden/make_golden_mimaker.py): IDs by file (-F) or by FASTA name with
a repeated name, k-mer mode and spaced seeds, several contigs per ID, an N run
and a record shorter than k.  The IDs are assigned here the way MIBFGen's
constructor assigns them (BioBloomMaker/MIBFGen.hpp:45-111)."""
import gzip
import os

import pytest

from tests.golden.make_golden_mimaker import CASES, OUT, SEEDS, inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from biobloom_b200 import _lib
    _lib.lib()


def reference_ids(by_file):
    """(sequences, their IDs, names by ID) as MIBFGen's constructor assigns
    them: one ID per file name, or one per FASTA record in file order with a
    repeated name mapped to its last ID."""
    files = inputs()
    order = sorted(files)
    names, name_to_id = [], {}
    if by_file:
        for fn in order:
            names.append(fn)
            name_to_id[fn] = len(names)
    else:
        for fn in order:
            for n, _ in files[fn]:
                names.append(n)
                name_to_id[n] = len(names)
    seqs, ids = [], []
    for fn in order:
        for n, s in files[fn]:
            seqs.append(s)
            ids.append(name_to_id[fn if by_file else n])
    return seqs, ids, names


@pytest.mark.parametrize("case", sorted(CASES))
def test_gpu_maker_matches_the_reference_maker(case, tmp_path):
    from biobloom_b200.mibf import make_mibf
    seqs, ids, names = reference_ids(case.startswith("file"))
    prefix = str(tmp_path / case)
    if case.endswith("seeds"):
        make_mibf(prefix, seqs, ids, names, seeds=SEEDS, k=len(SEEDS[0]), occupancy=0.5)
    else:
        make_mibf(prefix, seqs, ids, names, k=25, hash_num=3, occupancy=0.5)
    for ext in (".bf", ".sdsl", "_ids.txt"):
        with gzip.open(os.path.join(OUT, case + ext + ".gz"), "rb") as want, \
                open(prefix + ext, "rb") as got:
            assert got.read() == want.read(), ext
