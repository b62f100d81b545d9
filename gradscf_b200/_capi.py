"""ctypes binding of the C ABI in include/b200jk.h (libb200jk.so, built in-tree).

The library is the product: there is no CPU fallback.  If it is missing the
import of an operator fails loudly with instructions to build it.
"""
from __future__ import annotations

import ctypes
from functools import lru_cache
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libb200jk.so"

OK, INVALID_ARGUMENT, INTERNAL, UNSUPPORTED = 0, 1, 2, 3
FP64, SPLIT = 0, 1

EXPORTS = (
    "b200jk_last_error", "b200jk_plan_create", "b200jk_plan_destroy", "b200jk_plan_nao",
    "b200jk_plan_quartets", "b200jk_plan_block_offsets", "b200jk_direct_jk",
    "b200jk_check_status", "b200jk_direct_jk_tables", "b200jk_direct_jk_geom_vjp",
    "b200jk_int1e", "b200jk_int1e_grad", "b200jk_plan_class_stats", "b200jk_plan_split_stats",
    "b200jk_plan_border_stats", "b200jk_direct_jk_geom_vjp_precision",
    "b200jk_plan_set_profiling", "b200jk_plan_profile", "b200jk_measure_fma_peak",
    "b200jk_direct_jk_noalloc", "b200jk_graph_create", "b200jk_graph_launch", "b200jk_graph_destroy",
    "b200jk_partition_items", "b200jk_plan_set_shard", "b200jk_plan_autotune",
    "b200jk_packed_eri", "b200jk_packed_jk", "b200jk_plan_launches",
    "b200jk_direct_jk_geom_jvp", "b200jk_direct_jk_geom_hvp", "b200jk_measure_bra_transfer",
)
NOALLOC_SCRATCH_BYTES = 16 * 1024 * 1024
NCLASS = 55
PAIR_CLASSES = ((0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (3, 2), (3, 3))
QUARTET_CLASSES = tuple(PAIR_CLASSES[x] + PAIR_CLASSES[y] for x in range(10) for y in range(x + 1))


class B200JKError(RuntimeError):
    """A nonzero status from the C ABI."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class InvalidArgument(B200JKError, ValueError):
    pass


class Unsupported(B200JKError, NotImplementedError):
    pass


class Molecule(ctypes.Structure):
    _fields_ = [("atm", ctypes.c_void_p), ("natm", ctypes.c_int32),
                ("bas", ctypes.c_void_p), ("nbas", ctypes.c_int32),
                ("env", ctypes.c_void_p), ("nenv", ctypes.c_int32)]


@lru_cache(maxsize=1)
def lib():
    if not LIB_PATH.is_file():
        raise RuntimeError(
            f"The B200 J/K library is not built ({LIB_PATH} missing). "
            "Run `python -m gradscf_b200.build` (nvcc, sm_100a).")
    h = ctypes.CDLL(str(LIB_PATH))
    vp, i32, i64, f64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    h.b200jk_last_error.restype = ctypes.c_char_p
    h.b200jk_plan_create.argtypes = [ctypes.POINTER(Molecule), i32, i32, f64, i32, ctypes.POINTER(vp)]
    h.b200jk_plan_destroy.argtypes = [vp]
    h.b200jk_plan_destroy.restype = None
    h.b200jk_plan_nao.argtypes = [vp, i32, ctypes.POINTER(i32)]
    h.b200jk_plan_quartets.argtypes = [vp, ctypes.POINTER(i64)]
    h.b200jk_plan_block_offsets.argtypes = [vp, ctypes.POINTER(i64)]
    h.b200jk_direct_jk.argtypes = [vp, vp, i32, vp, i32, i32, i32, i32, f64, vp]
    h.b200jk_check_status.argtypes = [vp, vp]
    h.b200jk_direct_jk_tables.argtypes = [vp, i32, vp, i32, vp, i32, vp, i32, i32, vp, i32, f64,
                                          i32, i32, i32, vp]
    h.b200jk_direct_jk_geom_vjp.argtypes = [vp, vp, i32, vp, i32, i32, vp, vp]
    h.b200jk_direct_jk_geom_vjp_precision.argtypes = [vp, vp, i32, vp, i32, i32, i32, ctypes.c_double, vp, vp]
    h.b200jk_direct_jk_geom_jvp.argtypes = [vp, vp, i32, i32, vp, vp, i32, i32, vp, vp]
    h.b200jk_direct_jk_geom_hvp.argtypes = [vp, vp, i32, vp, vp, i32, i32, vp, vp]
    h.b200jk_int1e.argtypes = [vp, i32, vp, vp]
    h.b200jk_int1e_grad.argtypes = [vp, vp, vp, vp, vp]
    p64 = ctypes.POINTER(i64)
    h.b200jk_plan_class_stats.argtypes = [vp, p64, p64]
    h.b200jk_plan_split_stats.argtypes = [vp, vp, p64, p64, p64, p64]
    h.b200jk_plan_border_stats.argtypes = [vp, vp, p64, p64]
    h.b200jk_plan_set_profiling.argtypes = [vp, i32]
    h.b200jk_partition_items.argtypes = [vp, i64, i32, vp]
    h.b200jk_plan_set_shard.argtypes = [vp, i32, i32]
    h.b200jk_plan_autotune.argtypes = [vp, vp, i32, i32, i32, f64, i32, vp, vp]
    h.b200jk_packed_eri.argtypes = [vp, i32, vp, i64, vp]
    h.b200jk_plan_launches.argtypes = [vp, i32, p64]
    h.b200jk_packed_jk.argtypes = [vp, i32, i64, i32, vp, i32, vp, i32, i32, vp]
    h.b200jk_plan_profile.argtypes = [vp, ctypes.POINTER(f64), ctypes.POINTER(f64), ctypes.POINTER(i32)]
    h.b200jk_measure_fma_peak.argtypes = [i32, ctypes.POINTER(f64), vp]
    h.b200jk_measure_bra_transfer.argtypes = [i32, i32, ctypes.POINTER(f64), ctypes.POINTER(f64), vp]
    h.b200jk_direct_jk_noalloc.argtypes = [vp, vp, i32, vp, i32, i32, i32, i32, f64, vp]
    h.b200jk_graph_create.argtypes = [vp, vp, i32, vp, i32, i32, i32, i32, f64, ctypes.POINTER(vp)]
    h.b200jk_graph_launch.argtypes = [vp, vp]
    h.b200jk_graph_destroy.argtypes = [vp]
    h.b200jk_graph_destroy.restype = None
    return h


def check(rc):
    if rc == OK:
        return
    msg = lib().b200jk_last_error().decode()
    if rc == INVALID_ARGUMENT:
        raise InvalidArgument(rc, msg)
    if rc == UNSUPPORTED:
        raise Unsupported(rc, msg)
    raise B200JKError(rc, msg)


def partition_items(cost, world):
    """Owner rank of each work item: contiguous, cost-balanced blocks
    (b200jk_partition_items; host-only, no GPU needed)."""
    import numpy as np
    c = np.ascontiguousarray(cost, dtype=np.int64)
    owner = np.empty(c.shape[0], dtype=np.int32)
    check(lib().b200jk_partition_items(c.ctypes.data_as(ctypes.c_void_p), c.shape[0], int(world),
                                       owner.ctypes.data_as(ctypes.c_void_p)))
    return owner
