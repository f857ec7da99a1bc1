"""B200-native (sm_100a) hot path of 2D_NNF_LBM.

The package name starts with a digit, so load it with
``importlib.import_module("2d_nnf_lbm_b200")``.  The compute path is the CUDA
library ``liblbm2d.so`` built next to this file (see ``build.py``); the
Python layer here only mirrors the reference driver's set-up (parameters,
particle input file, output time series) and binds the C ABI with ctypes.
Nothing here falls back to a CPU implementation: if the library is missing
or no CUDA device is present, the calls raise.
"""

from .lbm2d import (  # noqa: F401
    Batch,
    LbmError,
    LbmObjective,
    LbmParams,
    Simulation,
    library_path,
    load_library,
    r4,
)
from . import cases  # noqa: F401
