"""B200-native drop-in for OpenFPM pdata's single-GPU vector_dist particle path.

The compute path is libpdgpu.so (hand-written CUDA for sm_100a behind a C ABI,
declared in include/pdgpu.h).  This package holds the ctypes binding used by
tests and bench.py (``openfpm_pdata_b200.pd``) and the synthetic workload
generators (``openfpm_pdata_b200.workloads``).
"""
