"""B200-native rebuild of ReactiveFoam's per-cell hot path.

HLL face flux with the SSPRK2 conserved update, the WALE stress and the
Peng-Robinson HEM UV flash, as hand-written sm_100a CUDA behind the reference's
reactive_transport_* / reactive_gpu_hem_* C ABI (libreactive_b200.so), driven
from Python through ctypes and PyTorch device tensors.
"""
