"""ctypes binding of include/sac_fno.h (libsacfno.so)."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
FNO_LIB = os.path.join(HERE, "libsacfno.so")

VP = ctypes.c_void_p
FP = ctypes.POINTER(ctypes.c_float)


class GemmDesc(ctypes.Structure):
    _fields_ = [
        ("M", ctypes.c_int), ("N", ctypes.c_int), ("K", ctypes.c_int), ("batch", ctypes.c_int),
        ("ksplit", ctypes.c_int),
        ("a", VP), ("a_m0", ctypes.c_long), ("a_m1", ctypes.c_long), ("a_k", ctypes.c_long),
        ("a_b", ctypes.c_long), ("a_msplit", ctypes.c_int), ("a_mn_major", ctypes.c_int),
        ("b", VP), ("b_n", ctypes.c_long), ("b_k", ctypes.c_long), ("b_b", ctypes.c_long),
        ("b_mn_major", ctypes.c_int),
        ("c", VP), ("c_m0", ctypes.c_long), ("c_m1", ctypes.c_long), ("c_n", ctypes.c_long),
        ("c_b", ctypes.c_long), ("c_msplit", ctypes.c_int), ("c_bf16", ctypes.c_int), ("c_mode", ctypes.c_int),
        ("alpha", ctypes.c_float), ("bias_n", VP), ("add", VP), ("act", ctypes.c_int), ("pre", VP),
        ("err", VP),
    ]


class FnoError(RuntimeError):
    pass


_LIB = None


def load(path: str = FNO_LIB):
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run sac_b200.build.build_fno())")
    lib = ctypes.CDLL(path)
    lib.sac_fno_gemm.argtypes = [ctypes.POINTER(GemmDesc), VP]
    lib.sac_fno_gemm.restype = ctypes.c_int
    lib.sac_fno_last_error.argtypes = []
    lib.sac_fno_last_error.restype = ctypes.c_char_p
    _LIB = lib
    return lib


def check(rc, lib=None):
    if rc != 0:
        lib = lib or load()
        raise FnoError(f"status {rc}: {lib.sac_fno_last_error().decode(errors='replace')}")


def gemm(M, N, K, a, b, c, *, batch=1, ksplit=1, a_m0=None, a_m1=0, a_k=1, a_b=0, a_msplit=None,
         a_mn_major=False, b_n=None, b_k=1, b_b=0, b_mn_major=False, c_m0=None, c_m1=0, c_n=1, c_b=0,
         c_msplit=None, c_bf16=False, c_mode=0, alpha=1.0, bias_n=0, add=0, act=0, pre=0, err=0, stream=0):
    """Thin call of sac_fno_gemm with integer device pointers (0 = none)."""
    lib = load()
    d = GemmDesc()
    d.M, d.N, d.K, d.batch, d.ksplit = M, N, K, batch, ksplit
    d.a = a
    d.a_m0 = (K if not a_mn_major else 1) if a_m0 is None else a_m0
    d.a_m1, d.a_k, d.a_b = a_m1, a_k, a_b
    d.a_msplit = (1 << 30) if a_msplit is None else a_msplit
    d.a_mn_major = int(bool(a_mn_major))
    d.b = b
    d.b_n = (K if not b_mn_major else 1) if b_n is None else b_n
    d.b_k, d.b_b, d.b_mn_major = b_k, b_b, int(bool(b_mn_major))
    d.c = c
    d.c_m0 = N if c_m0 is None else c_m0
    d.c_m1, d.c_n, d.c_b = c_m1, c_n, c_b
    d.c_msplit = (1 << 30) if c_msplit is None else c_msplit
    d.c_bf16, d.c_mode, d.alpha = int(bool(c_bf16)), c_mode, alpha
    d.bias_n, d.add, d.act, d.pre, d.err = bias_n or None, add or None, act, pre or None, err or None
    check(lib.sac_fno_gemm(ctypes.byref(d), VP(stream) if stream else None), lib)
