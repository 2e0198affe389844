"""B200-native rmblastn search core.

The compiled library (rmblast_b200/lib/librmb_b200.so, built by `python -m rmblast_b200.build`)
holds the sm_100a kernels and the host steps of the search; `rmblast_b200.api` is the Python
host over its C ABI (include/rmb_gpu.h).
"""
__all__ = ["api", "build", "synth"]
