"""The tcgen05 tensor-core complex GEMMs of include/wqc_cuda.h, the
product of the two-site merge (src/tn/mps.rs:812-831) on its own:
``wqc_tc_zgemm`` (3xTF32 split products, FP32 accumulation: the
tensor-core form's merge) and ``wqc_tc_zgemm_int8`` (int8 digit slices,
exact int32 accumulation, FP64-level: WQC_MERGE_TC_INT8)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import Context, _check, lib


def _bind(L):
    if getattr(L, "_tc_bound", False):
        return L
    P, U32 = ctypes.c_void_p, ctypes.c_uint32
    L.wqc_tc_zgemm.argtypes = [P, U32, U32, U32, P, P, P, U32, ctypes.POINTER(ctypes.c_double)]
    L.wqc_tc_zgemm_int8.argtypes = [P, U32, U32, U32, P, P, P, U32, ctypes.POINTER(ctypes.c_double)]
    L._tc_bound = True
    return L


def zgemm(a, b, reps: int = 1, ctx: Context | None = None, form: str = "tf32x3"):
    """(C, kernel_ms): C = a @ b for complex matrices a (m x k) and b (k x n)
    on the tensor cores -- form "tf32x3" (3xTF32 split products, FP32
    accumulation: wqc_tc_zgemm) or "int8" (int8 digit slices, exact int32
    accumulation, FP64-level: wqc_tc_zgemm_int8); kernel_ms is the mean
    device time of one GEMM launch over `reps` launches."""
    ctx = ctx or Context.shared()
    L = _bind(lib())
    a = np.ascontiguousarray(a, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    if a.ndim != 2 or b.ndim != 2 or a.shape[1] != b.shape[0]:
        raise ValueError(f"shapes {a.shape} and {b.shape} do not multiply")
    m, k = a.shape
    n = b.shape[1]
    c = np.zeros((m, n), dtype=np.complex128)
    ms = ctypes.c_double(0.0)
    if form not in ("tf32x3", "int8"):
        raise ValueError(f"unknown tensor-core form {form!r}")
    fn = L.wqc_tc_zgemm if form == "tf32x3" else L.wqc_tc_zgemm_int8
    _check(fn(ctx._h, m, n, k, a.ctypes.data, b.ctypes.data, c.ctypes.data, int(reps), ctypes.byref(ms)))
    return c, ms.value
