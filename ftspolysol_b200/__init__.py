"""B200-native complex-Langevin engine for charged polymer solutions.

Drop-in for the step loop of FTSPolySol: the same input files, deviceState
field names and observable definitions, computed by hand-written sm_100a
kernels behind the C ABI in include/ftsp.h (libftsp.so).
"""
from .engine import Engine, FtspError, NonFinite, FP32, FP64, SCHEME_PC, SCHEME_SI  # noqa: F401
