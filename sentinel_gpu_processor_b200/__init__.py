"""B200-native (sm_100a) implementation of the s1proc per-burst interferogram
chain: geo2rdr (TOPS deramp, FP64 zero-Doppler geocoding, bilinear
resampling, reramp), crossmul with multilooking, coherence and the
Goldstein filter.

Compute runs only in ``libs1b.so`` (hand-written CUDA behind the C ABI of
``include/s1b.h``); PyTorch provides device memory and streams.
"""
__version__ = "0.1.0"
