"""B200-native backend for Prima's restarted-PDHG LP path (oluies/noaidi).

``noaidi_b200.prima`` mirrors prima-core's public interface (LpProblem,
LpBuilder, PdhgParams, Pdhg, MixedPrecision, the Kernels seam); the numerics
run in ``libprima_cuda.so`` (``noaidi_b200/csrc``), hand-written sm_100a CUDA
behind a C ABI declared in ``include/prima_cuda.h``.
"""
