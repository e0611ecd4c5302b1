"""The CPU oracle's copy of the workload generator (oracle/synth_oracle.c),
which the benchmark's reference arm uses so that it loads no product library,
makes the same bytes as the product's bbt_synth_* entry points; its threaded
filter build makes the same bit array as the sequential maker.  Host only."""
import numpy as np
import pytest

from biobloom_b200 import synth
from tests import oracle_lib as ol


@pytest.mark.parametrize("kw", [
    dict(seed=3003, length=400_000, gc=0.41, repeat_frac=0.45, rep_min=300, rep_max=6000,
         div_min=0.10, div_max=0.20),
    dict(seed=1001, length=150_000, gc=0.5),
    dict(seed=1002007, length=300_000, gc=0.41, repeat_frac=0.05, rep_min=300, rep_max=300),
])
def test_genome_same_bytes(kw):
    seed, length = kw.pop("seed"), kw.pop("length")
    a = synth.genome(seed, length, **kw)
    b = ol.synth_genome(seed, length, **kw)
    assert np.array_equal(a, b)


def test_reads_same_bytes_single_varlen():
    g = synth.genome(7, 200_000, gc=0.41)
    pp = dict(len_min=50, len_max=300, long_frac=0.05, long_min=300, long_max=10_000,
              sub_rate=0.01)
    a1, aoff, _, asrc = synth.reads(3020, [g], [0.7], 5000, synth.read_params(**pp))
    b1, boff, _, bsrc = ol.synth_reads(3020, [g], [0.7], 5000, ol.read_params(**pp))
    assert np.array_equal(aoff, boff)
    assert np.array_equal(a1, b1)
    assert np.array_equal(asrc, bsrc)


def test_reads_same_bytes_paired_with_n():
    gs = [synth.genome(100 + j, 50_000, gc=0.41) for j in range(3)]
    pp = dict(len_min=150, len_max=150, sub_rate=0.005, n_rate=0.0001, frag_min=300,
              frag_max=500)
    a1, aoff, a2, _ = synth.reads(5000, gs, [1 / 3] * 3, 3000, synth.read_params(**pp),
                                  paired=True)
    b1, boff, b2, _ = ol.synth_reads(5000, gs, [1 / 3] * 3, 3000, ol.read_params(**pp),
                                     paired=True)
    assert np.array_equal(aoff, boff)
    assert np.array_equal(a1, b1)
    assert np.array_equal(a2, b2)


def test_threaded_build_equals_sequential_build():
    g = ol.synth_genome(11, 3_000_000, gc=0.45, repeat_frac=0.2, rep_min=300, rep_max=2000,
                        div_min=0.1, div_max=0.2)
    g[1000:1040] = ord("N")
    seq = ol.Filter.make([g.tobytes()], k=25, fpr=0.075)
    par = ol.make_filter_par([g], k=25, fpr=0.075)
    assert (par.m, par.h, par.k) == (seq.m, seq.h, seq.k)
    assert par.expected_entries == seq.expected_entries
    assert np.array_equal(par.bits(), seq.bits())
    assert par.bf.n_entry + par.redundant == seq.bf.n_entry + seq.redundant
