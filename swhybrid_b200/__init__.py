"""B200-native Smith-Waterman protein DB search (drop-in for SWhybrid's GPU worker).

The compute path is libswb200.so (hand-written sm_100a CUDA behind the C ABI
in include/swb200.h); this package holds its Python binding, the parameter and
encoding mirror of the reference's ``Param``, and the seeded workload
generators used by the benchmark.
"""
from .param import Param, blosum62, encode, decode  # noqa: F401
