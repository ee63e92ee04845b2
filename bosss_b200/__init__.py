"""bosss_b200 -- B200-native (sm_100a) implementation of the BoSSS linear-solver hot path.

The compute path is the C-ABI CUDA library ``lib/libbsgpu.so`` (sources in ``csrc/``, header in
``include/bsgpu.h``); this package holds its Python binding (``native``), the host-side mirror of the reference
solver API (``solvers``) and the workload generator that assembles SIP DG systems (``assembly``).
"""
__version__ = "0.1.0"
