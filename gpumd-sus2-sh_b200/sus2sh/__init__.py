"""sus2sh: B200 SUS2-SH energy/force/virial engine (Python side).

The compute path is libsus2sh.so (hand-written sm_100a kernels behind the C-ABI
of include/sus2sh.h); this package binds it with ctypes and mirrors the
reference's GPUMD plugin interface.
"""
from ._lib import EXPORTS, LIB_PATH, EngineError, load  # noqa: F401
from .potential import SUS2_SH, Box, is_sus2_sh_potential_file, standard_graph_counts  # noqa: F401
