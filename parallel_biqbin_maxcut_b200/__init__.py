"""B200-native implementation of BiqBin's per-node SDP bounding path.

The compute lives in ``lib/libbqb_gpu.so`` (hand-written sm_100a CUDA behind
a C ABI declared in ``include/bqb_gpu.h``); this package holds its build
script, a ctypes binding and the synthetic instance generators.
"""
__version__ = "0.1.0"
