"""biobloom_b200: BioBloom Tools' read-classification path on B200 GPUs.

The product is libbbt.so (CUDA kernels for sm_100a behind the C ABI in
include/bbt.h and include/bbt_mibf.h) and the biobloomcategorizer /
biobloommicategorizer CLIs over it; this package holds the Python mirrors of
the reference's BioBloomClassifier and MIBFClassifier interfaces and the
workload generators used by tests and the benchmark.
"""
from ._lib import (MODE_BESTHIT, MODE_ORDERED, MODE_SCORES, MODE_STD, BBTError,  # noqa: F401
                   LibraryMissing, lib)
from .classifier import BioBloomClassifier, pack  # noqa: F401
from .mibf import MIBFClassifier, make_mibf  # noqa: F401

__all__ = ["BioBloomClassifier", "MIBFClassifier", "BBTError", "LibraryMissing", "lib", "pack",
           "make_mibf", "MODE_STD", "MODE_ORDERED", "MODE_BESTHIT", "MODE_SCORES"]
