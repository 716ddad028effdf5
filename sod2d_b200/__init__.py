"""sod2d_b200 -- B200-native spectral-element RHS hot path of SOD2D.

The product is the C-ABI library ``_lib/libsod2d_gpu.so`` (CUDA, sm_100a)
declared in ``include/sod2d_gpu.h``; ``host`` holds the set-up routines and
``gpu`` the Python view of the C-ABI used by the tests and the benchmark.
"""
__all__ = ["host", "build"]
