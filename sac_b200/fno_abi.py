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
        ("err", VP), ("b_n1", ctypes.c_long), ("b_nsplit", ctypes.c_int), ("wait_tries", ctypes.c_int),
        ("K2", ctypes.c_int), ("a2_msplit", ctypes.c_int), ("a2_mn_major", ctypes.c_int),
        ("a2", VP), ("a2_m0", ctypes.c_long), ("a2_m1", ctypes.c_long), ("a2_k", ctypes.c_long),
        ("a2_b", ctypes.c_long),
        ("b2", VP), ("b2_n", ctypes.c_long), ("b2_k", ctypes.c_long), ("b2_b", ctypes.c_long),
        ("b2_m", ctypes.c_long), ("b2_mn_major", ctypes.c_int), ("b2_mdiv", ctypes.c_int),
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
         a_mn_major=False, b_n=None, b_k=1, b_b=0, b_mn_major=False, b_n1=0, b_nsplit=None,
         c_m0=None, c_m1=0, c_n=1, c_b=0,
         c_msplit=None, c_bf16=False, c_mode=0, alpha=1.0, bias_n=0, add=0, act=0, pre=0, err=0, stream=0,
         wait_tries=0, second=None):
    """Thin call of sac_fno_gemm with integer device pointers (0 = none).  second:
    a dict of the second product's fields (K2, a2, b2, a2_m0, ... b2_mdiv)."""
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
    d.b_n1 = b_n1
    d.b_nsplit = (1 << 30) if b_nsplit is None else b_nsplit
    d.c = c
    d.c_m0 = N if c_m0 is None else c_m0
    d.c_m1, d.c_n, d.c_b = c_m1, c_n, c_b
    d.c_msplit = (1 << 30) if c_msplit is None else c_msplit
    d.c_bf16, d.c_mode, d.alpha = int(bool(c_bf16)), c_mode, alpha
    d.bias_n, d.add, d.act, d.pre, d.err = bias_n or None, add or None, act, pre or None, err or None
    d.wait_tries = wait_tries
    if second:
        d.a2_msplit = 1 << 30
        for k, v in second.items():
            setattr(d, k, int(v))
    check(lib.sac_fno_gemm(ctypes.byref(d), VP(stream) if stream else None), lib)


class FnoConfig(ctypes.Structure):
    _fields_ = [("S", ctypes.c_int), ("F", ctypes.c_int), ("width", ctypes.c_int), ("layers", ctypes.c_int),
                ("modes1", ctypes.c_int), ("modes2", ctypes.c_int), ("hidden", ctypes.c_int),
                ("cin", ctypes.c_int), ("cout", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("device", ctypes.c_int)]


def _bind_net(lib):
    if getattr(lib, "_net_bound", False):
        return lib
    lib.sac_fno_default_config.argtypes = [ctypes.POINTER(FnoConfig)]
    lib.sac_fno_default_config.restype = None
    lib.sac_fno_create.argtypes = [ctypes.POINTER(FnoConfig), ctypes.POINTER(VP)]
    lib.sac_fno_destroy.argtypes = [VP]
    lib.sac_fno_destroy.restype = None
    lib.sac_fno_error.argtypes = [VP]
    lib.sac_fno_error.restype = ctypes.c_char_p
    lib.sac_fno_stream.argtypes = [VP]
    lib.sac_fno_stream.restype = VP
    lib.sac_fno_num_params.argtypes = [VP]
    lib.sac_fno_num_params.restype = ctypes.c_long
    lib.sac_fno_param_layout.argtypes = [VP, ctypes.POINTER(ctypes.c_long)]
    lib.sac_fno_init.argtypes = [VP, ctypes.c_ulonglong]
    lib.sac_fno_set_params.argtypes = [VP, FP]
    lib.sac_fno_get_params.argtypes = [VP, FP]
    lib.sac_fno_get_grads.argtypes = [VP, FP]
    lib.sac_fno_zero_grad.argtypes = [VP]
    lib.sac_fno_forward.argtypes = [VP, VP, VP, ctypes.c_int]
    lib.sac_fno_infer.argtypes = [VP, VP, VP, ctypes.c_int]
    lib.sac_fno_backward.argtypes = [VP, VP]
    lib.sac_fno_mse.argtypes = [VP, VP, VP, VP, VP, ctypes.c_int]
    lib.sac_fno_adam.argtypes = [VP, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                 ctypes.c_float, ctypes.c_int, ctypes.c_float]
    lib.sac_fno_features.argtypes = [VP, VP, ctypes.c_int, VP, VP, ctypes.c_int, VP, ctypes.c_int, ctypes.c_int]
    lib.sac_fno_apply.argtypes = [VP, VP, VP, VP, ctypes.c_int, ctypes.c_int]
    lib.sac_fno_check.argtypes = [VP, ctypes.c_int]
    lib.sac_fno_set_wait_tries.argtypes = [VP, ctypes.c_int]
    for f in ("sac_fno_create", "sac_fno_param_layout", "sac_fno_init", "sac_fno_set_params", "sac_fno_get_params",
              "sac_fno_get_grads", "sac_fno_zero_grad", "sac_fno_forward", "sac_fno_infer", "sac_fno_backward", "sac_fno_mse",
              "sac_fno_adam", "sac_fno_features", "sac_fno_apply", "sac_fno_check", "sac_fno_set_wait_tries"):
        getattr(lib, f).restype = ctypes.c_int
    lib._net_bound = True
    return lib


class Net:
    """The FNO of libsacfno.so.  Tensors are passed as integer device pointers
    (e.g. torch's data_ptr()); every call is enqueued on the network's stream."""

    def __init__(self, S=256, F=256, width=32, layers=4, hidden=128, cin=16, cout=6, max_batch=16, device=0,
                 seed=0):
        self.lib = _bind_net(load())
        c = FnoConfig()
        self.lib.sac_fno_default_config(ctypes.byref(c))
        c.S, c.F, c.width, c.layers, c.hidden = S, F, width, layers, hidden
        c.cin, c.cout, c.max_batch, c.device = cin, cout, max_batch, device
        self.cfg = c
        self.h = VP()
        rc = self.lib.sac_fno_create(ctypes.byref(c), ctypes.byref(self.h))
        if rc != 0:
            raise FnoError(f"sac_fno_create: {self.lib.sac_fno_last_error().decode()}")
        self.cpad = (cout + 7) // 8 * 8
        self.nparam = int(self.lib.sac_fno_num_params(self.h))
        if seed is not None:
            self._c(self.lib.sac_fno_init(self.h, seed))

    def _c(self, rc):
        if rc != 0:
            raise FnoError(f"status {rc}: {self.lib.sac_fno_error(self.h).decode(errors='replace')}")

    @property
    def stream(self):
        return self.lib.sac_fno_stream(self.h)

    def layout(self):
        import numpy as np
        n = 2 * (6 + 4 * self.cfg.layers)
        out = np.zeros(n, dtype=np.int64)
        self._c(self.lib.sac_fno_param_layout(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_long))))
        return out.reshape(-1, 2)

    def get_params(self):
        import numpy as np
        a = np.zeros(self.nparam, dtype=np.float32)
        self._c(self.lib.sac_fno_get_params(self.h, a.ctypes.data_as(FP)))
        return a

    def set_params(self, a):
        import numpy as np
        a = np.ascontiguousarray(a, dtype=np.float32)
        assert a.size == self.nparam
        self._c(self.lib.sac_fno_set_params(self.h, a.ctypes.data_as(FP)))

    def get_grads(self):
        import numpy as np
        a = np.zeros(self.nparam, dtype=np.float32)
        self._c(self.lib.sac_fno_get_grads(self.h, a.ctypes.data_as(FP)))
        return a

    def zero_grad(self):
        self._c(self.lib.sac_fno_zero_grad(self.h))

    def forward(self, x_ptr, y_ptr, B):
        self._c(self.lib.sac_fno_forward(self.h, VP(x_ptr), VP(y_ptr), B))

    def infer(self, x_ptr, y_ptr, B):
        """forward() without the stores the backward pass needs."""
        self._c(self.lib.sac_fno_infer(self.h, VP(x_ptr), VP(y_ptr), B))

    def backward(self, dy_ptr):
        self._c(self.lib.sac_fno_backward(self.h, VP(dy_ptr)))

    def mse(self, y_ptr, t_ptr, dy_ptr, loss_ptr, B):
        self._c(self.lib.sac_fno_mse(self.h, VP(y_ptr), VP(t_ptr), VP(dy_ptr), VP(loss_ptr), B))

    def adam(self, lr, step, b1=0.9, b2=0.999, eps=1e-8, wd=1e-4, clip=0.0):
        self._c(self.lib.sac_fno_adam(self.h, lr, b1, b2, eps, wd, step, clip))

    def features(self, state_ptr, state_bf16, scale_ptr, feat_ptr, nfeat, x_ptr, B, nst):
        self._c(self.lib.sac_fno_features(self.h, VP(state_ptr), int(bool(state_bf16)), VP(scale_ptr or None),
                                          VP(feat_ptr or None), nfeat, VP(x_ptr), B, nst))

    def apply(self, state_ptr, y_ptr, scale_ptr, B, nst):
        self._c(self.lib.sac_fno_apply(self.h, VP(state_ptr), VP(y_ptr), VP(scale_ptr), B, nst))

    def check(self, reset=True):
        self._c(self.lib.sac_fno_check(self.h, int(bool(reset))))

    def set_wait_tries(self, tries):
        """Bound of the tensor-core waits of every GEMM (0: default; -1: give up at once)."""
        self._c(self.lib.sac_fno_set_wait_tries(self.h, int(tries)))

    def close(self):
        if self.h:
            self.lib.sac_fno_destroy(self.h)
            self.h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
