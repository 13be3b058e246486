"""CPU oracle for the parity tests -- TEST INFRASTRUCTURE ONLY.

ctypes binding of oracle/_build/liboracle.so, the C restatement of
slitvinov/dns main.c's RK4 step (oracle/dns_oracle.c) on a project-written
FFTW-subset FFT (oracle/fftw_shim).  Only tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py use it, always as the checker; the product
(dns_b200) never imports it.

Parity pin: the oracle and oracle/_ref/dns (the reference main.c compiled
unchanged against the same shim) reproduce the reference's own golden
histories 0128/* and 0256/* (tests/golden); see tests/test_oracle.py.  A
second restatement on numpy's FFT (oracle/numpy_restatement.py) agrees with
the C one step by step, which pins the shim FFT independently.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_DNS = os.path.join(HERE, "_ref", "dns")

_lib = None
_P = ctypes.c_void_p


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    lib.oracle_create.restype = _P
    lib.oracle_create.argtypes = [ctypes.c_long]
    lib.oracle_destroy.argtypes = [_P]
    lib.oracle_set_velocity.argtypes = [_P, _P, _P, _P]
    lib.oracle_diagnostics.argtypes = [_P, _P, _P]
    lib.oracle_step.argtypes = [_P, ctypes.c_double, ctypes.c_double, ctypes.c_long]
    for name in ("oracle_get_spectral", "oracle_set_spectral", "oracle_get_stale",
                 "oracle_set_stale", "oracle_get_pressure", "oracle_dump_fields"):
        getattr(lib, name).argtypes = [_P, _P]
    for name in ("oracle_r2c_3d", "oracle_c2r_3d"):
        getattr(lib, name).argtypes = [ctypes.c_int] * 3 + [_P, _P]
    lib.oracle_max_threads.restype = ctypes.c_int
    lib.oracle_set_threads.argtypes = [ctypes.c_int]
    _lib = lib
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def set_threads(n: int) -> None:
    load().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(load().oracle_max_threads())


class Oracle:
    """State of one run of the restated main.c loop (spectral velocity plus
    the stale real-space velocity)."""

    def __init__(self, n: int):
        self.lib = load()
        self.n = int(n)
        self.nf = self.n // 2 + 1
        self.h = self.lib.oracle_create(self.n)
        if not self.h:
            raise ValueError(f"oracle: bad n={n}")

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_velocity(self, U, V, W):
        U, V, W = (np.ascontiguousarray(a, dtype=np.float64) for a in (U, V, W))
        self.lib.oracle_set_velocity(self.h, _p(U), _p(V), _p(W))

    def step(self, nu: float, dt: float, nsteps: int = 1):
        self.lib.oracle_step(self.h, nu, dt, nsteps)

    def diagnostics(self):
        # numpy buffers keep all 64 mantissa bits (ctypes' c_longdouble.value
        # would round to a Python float)
        e, o = np.zeros(1, dtype=np.longdouble), np.zeros(1, dtype=np.longdouble)
        self.lib.oracle_diagnostics(self.h, _p(e), _p(o))
        return e[0], o[0]

    def get_spectral(self):
        out = np.empty((3, self.n, self.n, self.nf), dtype=np.complex128)
        self.lib.oracle_get_spectral(self.h, _p(out))
        return out

    def set_spectral(self, uh):
        uh = np.ascontiguousarray(uh, dtype=np.complex128)
        self.lib.oracle_set_spectral(self.h, _p(uh))

    def get_stale(self):
        out = np.empty((3, self.n, self.n, self.n))
        self.lib.oracle_get_stale(self.h, _p(out))
        return out

    def set_stale(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.lib.oracle_set_stale(self.h, _p(u))

    def get_pressure(self):
        out = np.empty((self.n, self.n, self.nf), dtype=np.complex128)
        self.lib.oracle_get_pressure(self.h, _p(out))
        return out

    def dump_fields(self):
        out = np.empty((4, self.n, self.n, self.n))
        self.lib.oracle_dump_fields(self.h, _p(out))
        return out


def r2c_3d(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    n0, n1, n2 = x.shape
    out = np.empty((n0, n1, n2 // 2 + 1), dtype=np.complex128)
    load().oracle_r2c_3d(n0, n1, n2, _p(x), _p(out))
    return out


def c2r_3d(X: np.ndarray, n2: int) -> np.ndarray:
    X = np.ascontiguousarray(X, dtype=np.complex128)
    n0, n1, _ = X.shape
    out = np.empty((n0, n1, n2))
    load().oracle_c2r_3d(n0, n1, n2, _p(X), _p(out))
    return out
