"""Failures on the file and serving paths, on a GPU, caused on the host: a
FASTQ file that ends in a truncated record is read up to that record and the
next input follows, as the reference's kseq loop does
(BioBloomClassifier.cpp:64,87-88; the summary is the reference CLI's on the
same files, tests/golden/make_golden_failures.py); an input that cannot be
opened is an error with a message after which the context still classifies;
a serving request whose read cannot fit the memory budget is refused at
submit and the server keeps serving."""
import numpy as np
import pytest

from tests.fixtures import filter_paths, golden, read_fastx

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from biobloom_b200 import _lib
    _lib.lib()


def test_truncated_fastq_ends_that_file(tmp_path):
    from biobloom_b200 import BioBloomClassifier
    prefix = str(tmp_path / "t")
    with BioBloomClassifier(filter_paths(), 0.15, prefix=prefix) as bbc:
        bbc.filter([golden("truncated.fq"), golden("after.fq")])
    with open(prefix + "_summary.tsv") as f:
        got = f.read()
    with open(golden("expected_summary_truncated.tsv")) as f:
        assert got == f.read()


def test_unopenable_input_then_the_context_still_works(tmp_path):
    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200._lib import BBTError
    prefix = str(tmp_path / "u")
    with BioBloomClassifier(filter_paths(), 0.15, prefix=prefix) as bbc:
        with pytest.raises(BBTError) as e:
            bbc.filter([str(tmp_path / "missing.fq")])
        assert e.value.code == -2 and "cannot be opened" in str(e.value)
        recs = read_fastx(golden("after.fq"))
        hits, _, _ = bbc.classify([s for _, s in recs])
        bbc.reset_summary()
        bbc.filter([golden("after.fq")])
    with BioBloomClassifier(filter_paths(), 0.15) as fresh:
        want, _, _ = fresh.classify([s for _, s in recs])
    assert np.array_equal(hits, want)


def test_server_refuses_a_read_larger_than_its_budget():
    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200._lib import BBTError
    from biobloom_b200.server import Server
    recs = [s for _, s in read_fastx(golden("after.fq"))]
    huge = b"ACGT" * (3 << 20)  # 12 Mbp: one read larger than a 4 MB budget
    with BioBloomClassifier(filter_paths(), 0.15) as bbc:
        want, _, _ = bbc.classify(recs)
        with Server(bbc, None, slots=2, mem_budget=4 << 20) as srv:
            with pytest.raises(BBTError) as e:
                srv.submit_bloom([huge])
            assert e.value.code == -5 and "budget" in str(e.value)
            req = srv.submit_bloom(recs)
            srv.wait(req)
            assert np.array_equal(req.hits[:len(recs)], want)
