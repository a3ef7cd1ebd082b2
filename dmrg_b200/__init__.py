"""dmrg_b200: B200-native effective-Hamiltonian path of symmetry-blocked DMRG.

The compute lives in libdmrgx.so (CUDA for sm_100a behind the C ABI of
include/dmrgx.h); ``dmrg_b200.native`` binds it with ctypes.
"""
__all__ = ["native", "workloads"]
