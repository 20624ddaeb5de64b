"""Python binding of the B200 statevector engine (C ABI in include/bk_engine.h).

The compute path is the in-tree CUDA library ``lib/libbk_b200.so``; this package
only marshals arguments. There is no CPU fallback: every device call raises
``BkError`` when the library or a CUDA device is missing.
"""
from ._lib import (BK_C64, BK_C128, BK_FUSED, BK_OBJ_D_H, BK_OBJ_P_LESS, BK_ORDER_REFERENCE, BK_ORDER_STRANG,
                   BK_PLAIN, BkError, Engine, labs_energy, library_path, load_library, random_states, select_trap,
                   steepest_descent)

__all__ = ["BK_C64", "BK_C128", "BK_FUSED", "BK_OBJ_D_H", "BK_OBJ_P_LESS", "BK_ORDER_REFERENCE", "BK_ORDER_STRANG",
           "BK_PLAIN", "BkError", "Engine", "labs_energy", "library_path", "load_library", "random_states",
           "select_trap", "steepest_descent"]
