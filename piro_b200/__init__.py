"""piro_b200: PIRO's sparse finite-difference time-stepping path on B200.

The compute path is libpiro_b200.so (CUDA, sm_100a) behind the C ABI in
include/piro.h; piro_b200.ops wraps it for torch tensors.
"""
__version__ = "0.1.0"
