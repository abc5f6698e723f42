"""ctypes handle on the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py.  The oracle has the same call shape as the product
C-ABI (include/sac_gpu.h) under the prefix ``oracle_``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

from sac_b200.abi import Context

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build(force=False):
    src = os.path.join(HERE, "sac_oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB


class Oracle(Context):
    def __init__(self, params):
        build()
        super().__init__(params, path=LIB, prefix="oracle_")


def set_threads(n: int):
    build()
    lib = ctypes.CDLL(LIB)
    lib.oracle_set_threads(ctypes.c_int(n))


def max_threads() -> int:
    build()
    lib = ctypes.CDLL(LIB)
    return int(lib.oracle_max_threads())
