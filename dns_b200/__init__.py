"""dns_b200 -- B200 (sm_100a) pseudo-spectral RK4 stepper, a drop-in for the
time-stepping path of slitvinov/dns main.c.

This module is the Python mirror of the C ABI in include/dns_b200.h (ctypes
over dns_b200/lib/libdns_b200.so).  The same library backs the C command-line
drop-in dns_b200/bin/dns.  There is no CPU fallback: every call runs the CUDA
kernels, and importing the bindings fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes
import math
import os
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libdns_b200.so")
CLI_PATH = os.path.join(HERE, "bin", "dns")

DNS_OK = 0
DNS_ERR_ARG = 1
DNS_ERR_UNSUPPORTED = 2
DNS_ERR_CUDA = 3
DNS_ERR_NOMEM = 4
DNS_ERR_NONFINITE = 5
DNS_ERR_STATE = 6
DNS_PREC_FP64 = 0
DNS_PREC_MIXED = 1
DNS_FLAG_PRESSURE = 1
DNS_FLAG_ENS_BATCHED = 2
DNS_FLAG_ENS_PERSISTENT = 4

SUPPORTED_N = (8, 16, 32, 64, 128, 256, 512)
KERNELS_PER_STAGE = 6
KERNELS_PER_STEP = 4 * KERNELS_PER_STAGE
PASS_NAMES = ("A:x-inverse", "B:y-inverse", "C:z-fused", "D:y-forward", "E1:x-forward", "E2:update")


class DNSError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


class _Info(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_long),
        ("precision", ctypes.c_int),
        ("flags", ctypes.c_uint),
        ("device_bytes", ctypes.c_size_t),
        ("slot_bytes", ctypes.c_size_t),
        ("kernels_per_step", ctypes.c_int),
    ]


_lib: Optional[ctypes.CDLL] = None

_P = ctypes.c_void_p
_D = ctypes.c_double
_SIGS = {
    "dns_create": (ctypes.c_int, [ctypes.c_long, ctypes.c_int, ctypes.c_uint, ctypes.POINTER(_P)]),
    "dns_destroy": (ctypes.c_int, [_P]),
    "dns_set_velocity": (ctypes.c_int, [_P, _P, _P, _P]),
    "dns_step": (ctypes.c_int, [_P, _D, _D, ctypes.c_long]),
    "dns_diagnostics": (ctypes.c_int, [_P] + [ctypes.POINTER(_D)] * 4),
    "dns_get_fields": (ctypes.c_int, [_P, _P, _P, _P, _P]),
    "dns_strerror": (ctypes.c_char_p, [ctypes.c_int]),
    "dns_last_error": (ctypes.c_char_p, []),
    "dns_get_spectral": (ctypes.c_int, [_P, _P]),
    "dns_set_spectral": (ctypes.c_int, [_P, _P]),
    "dns_get_stale": (ctypes.c_int, [_P, _P]),
    "dns_set_stale": (ctypes.c_int, [_P, _P]),
    "dns_get_info": (ctypes.c_int, [_P, ctypes.POINTER(_Info)]),
    "dns_get_stream": (_P, [_P]),
    "dns_get_schedule": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_long]),
    "dns_synchronize": (ctypes.c_int, [_P]),
    "dns_time_kernels": (ctypes.c_int, [_P, _D, _D, ctypes.c_long, ctypes.POINTER(_D)]),
    "dns_diagnostics_noalloc": (ctypes.c_int, [ctypes.c_long, _P, _P, _P]),
    "dns_set_tgv": (ctypes.c_int, [_P]),
    "dns_set_perturbed_tgv": (ctypes.c_int, [_P, ctypes.c_ulonglong, _D]),
    "dns_ens_set_tgv": (ctypes.c_int, [_P, ctypes.c_int]),
    "dns_ens_set_perturbed_tgv": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_ulonglong, _D]),
    "dns_ens_create": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_int, ctypes.c_uint, ctypes.POINTER(_P)]),
    "dns_ens_destroy": (ctypes.c_int, [_P]),
    "dns_ens_set_velocity": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P]),
    "dns_ens_set_params": (ctypes.c_int, [_P, _P, _P]),
    "dns_ens_step": (ctypes.c_int, [_P, ctypes.c_long]),
    "dns_ens_diagnostics": (ctypes.c_int, [_P, _P]),
    "dns_ens_get_spectral": (ctypes.c_int, [_P, ctypes.c_int, _P]),
    "dns_ens_get_stream": (_P, [_P]),
    "dns_ens_synchronize": (ctypes.c_int, [_P]),
    "dns_ens_get_schedule": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_long]),
    "dns_selftest_barrier_timeout": (ctypes.c_int, [_D, ctypes.POINTER(ctypes.c_int)]),
    "dns_adjoint_energy": (ctypes.c_int, [ctypes.c_long, _P, _P, _P, _D, _D, ctypes.c_long,
                                          ctypes.c_int, _P, _P, _P, _P, _P]),
    "dns_adjoint_energy_prec": (ctypes.c_int, [ctypes.c_long, ctypes.c_int, _P, _P, _P, _D, _D,
                                               ctypes.c_long, ctypes.c_int, _P, _P, _P, _P, _P]),
    "dns_adjoint_schedule": (ctypes.c_int, [ctypes.c_long, ctypes.c_int, _P, _P, _P]),
}


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libdns_b200.so and declare the C ABI.  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m dns_b200.build` "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(st: int) -> None:
    if st != DNS_OK:
        lib = load_library()
        raise DNSError(st, f"{lib.dns_strerror(st).decode()}: {lib.dns_last_error().decode()}")


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One simulation on one GPU (mirror of dns_ctx in include/dns_b200.h)."""

    def __init__(self, n: int, precision: int = DNS_PREC_FP64, flags: int = 0):
        self._lib = load_library()
        h = ctypes.c_void_p()
        _check(self._lib.dns_create(n, precision, flags, ctypes.byref(h)))
        self._h = h
        self.n = int(n)
        self.nf = self.n // 2 + 1
        self.flags = flags

    # -- lifetime --
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dns_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the path --
    def set_velocity(self, U, V, W) -> None:
        U, V, W = _f64(U), _f64(V), _f64(W)
        for a in (U, V, W):
            if a.size != self.n ** 3:
                raise ValueError("velocity component must have n^3 values")
        _check(self._lib.dns_set_velocity(self._h, _ptr(U), _ptr(V), _ptr(W)))

    def set_tgv(self) -> None:
        """Taylor-Green of tgv.py generated on the device (dns_set_tgv)."""
        _check(self._lib.dns_set_tgv(self._h))

    def set_perturbed_tgv(self, seed: int, amplitude: float = 1e-3) -> None:
        """Taylor-Green plus the seeded solenoidal perturbation of
        perturbed_tgv(..., rng="counter"), generated on the device."""
        _check(self._lib.dns_set_perturbed_tgv(self._h, seed, amplitude))

    def step(self, nu: float, dt: float, nsteps: int = 1) -> None:
        _check(self._lib.dns_step(self._h, nu, dt, nsteps))

    def diagnostics_dd(self, allow_nonfinite: bool = False) -> Tuple[float, float, float, float]:
        """Double-double sums (e_hi, e_lo, om_hi, om_lo) of dns_diagnostics.
        A NaN or Inf raises DNSError (DNS_ERR_NONFINITE), as main.c stops on
        the first non-finite value (main.c:49-50); allow_nonfinite=True
        returns the raw values instead."""
        v = [ctypes.c_double() for _ in range(4)]
        st = self._lib.dns_diagnostics(self._h, *[ctypes.byref(x) for x in v])
        if st != DNS_OK and not (allow_nonfinite and st == DNS_ERR_NONFINITE):
            _check(st)
        return tuple(x.value for x in v)

    def diagnostics(self, allow_nonfinite: bool = False) -> Tuple[np.longdouble, np.longdouble]:
        """Energy and enstrophy exactly as main.c:257-266 prints them."""
        eh, el, oh, ol = self.diagnostics_dd(allow_nonfinite)
        return scale_diagnostics(eh, el, oh, ol, self.n)

    def get_fields(self, pressure: bool = False):
        n3 = self.n ** 3
        out = [np.empty(n3) for _ in range(4 if pressure else 3)]
        ptrs = [_ptr(a) for a in out] + [None] * (4 - len(out))
        _check(self._lib.dns_get_fields(self._h, *ptrs))
        return [a.reshape(self.n, self.n, self.n) for a in out]

    def get_spectral(self) -> np.ndarray:
        out = np.empty((3, self.n, self.n, self.nf), dtype=np.complex128)
        _check(self._lib.dns_get_spectral(self._h, _ptr(out)))
        return out

    def set_spectral(self, uh) -> None:
        uh = np.ascontiguousarray(uh, dtype=np.complex128)
        if uh.shape != (3, self.n, self.n, self.nf):
            raise ValueError("spectral state must be (3, n, n, n/2+1)")
        _check(self._lib.dns_set_spectral(self._h, _ptr(uh)))

    def get_stale(self) -> np.ndarray:
        out = np.empty((3, self.n, self.n, self.n))
        _check(self._lib.dns_get_stale(self._h, _ptr(out)))
        return out

    def set_stale(self, u) -> None:
        u = _f64(u)
        if u.size != 3 * self.n ** 3:
            raise ValueError("stale velocity must have 3 n^3 values")
        _check(self._lib.dns_set_stale(self._h, _ptr(u)))

    # -- measurement --
    @property
    def stream(self) -> int:
        return int(self._lib.dns_get_stream(self._h) or 0)

    def synchronize(self) -> None:
        _check(self._lib.dns_synchronize(self._h))

    def info(self) -> dict:
        i = _Info()
        _check(self._lib.dns_get_info(self._h, ctypes.byref(i)))
        return {f: getattr(i, f) for f, _ in _Info._fields_}

    def schedule(self) -> str:
        """The autotuner's kernel schedule for this grid size (dns_get_schedule)."""
        buf = ctypes.create_string_buffer(4096)
        _check(self._lib.dns_get_schedule(self._h, buf, len(buf)))
        return buf.value.decode()

    def time_kernels(self, nu: float, dt: float, nsteps: int) -> np.ndarray:
        ms = (ctypes.c_double * KERNELS_PER_STEP)()
        _check(self._lib.dns_time_kernels(self._h, nu, dt, nsteps, ms))
        return np.array(list(ms))


class Ensemble:
    """Many independent runs stepped together (mirror of dns_ens)."""

    def __init__(self, sizes, precision: int = DNS_PREC_FP64, flags: int = 0):
        self._lib = load_library()
        self.sizes = [int(n) for n in sizes]
        arr = (ctypes.c_long * len(self.sizes))(*self.sizes)
        h = ctypes.c_void_p()
        _check(self._lib.dns_ens_create(len(self.sizes), arr, precision, flags, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dns_ens_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_velocity(self, run: int, U, V, W) -> None:
        U, V, W = _f64(U), _f64(V), _f64(W)
        _check(self._lib.dns_ens_set_velocity(self._h, run, _ptr(U), _ptr(V), _ptr(W)))

    def set_tgv(self, run: int) -> None:
        _check(self._lib.dns_ens_set_tgv(self._h, run))

    def set_perturbed_tgv(self, run: int, seed: int, amplitude: float = 1e-3) -> None:
        _check(self._lib.dns_ens_set_perturbed_tgv(self._h, run, seed, amplitude))

    def set_params(self, nu, dt) -> None:
        nu = _f64(np.broadcast_to(np.asarray(nu, dtype=np.float64), (len(self.sizes),)))
        dt = _f64(np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(self.sizes),)))
        _check(self._lib.dns_ens_set_params(self._h, _ptr(nu), _ptr(dt)))

    def step(self, nsteps: int = 1) -> None:
        _check(self._lib.dns_ens_step(self._h, nsteps))

    def diagnostics(self, allow_nonfinite: bool = False):
        """Per run (E, Omega) as main.c prints them.  A NaN or Inf in any run
        raises DNSError unless allow_nonfinite=True."""
        out = np.empty(4 * len(self.sizes))
        st = self._lib.dns_ens_diagnostics(self._h, _ptr(out))
        if st != DNS_OK and not (allow_nonfinite and st == DNS_ERR_NONFINITE):
            _check(st)
        return [scale_diagnostics(*out[4 * r:4 * r + 4], n) for r, n in enumerate(self.sizes)]

    def get_spectral(self, run: int) -> np.ndarray:
        n = self.sizes[run]
        out = np.empty((3, n, n, n // 2 + 1), dtype=np.complex128)
        _check(self._lib.dns_ens_get_spectral(self._h, run, _ptr(out)))
        return out

    @property
    def stream(self) -> int:
        return int(self._lib.dns_ens_get_stream(self._h) or 0)

    def synchronize(self) -> None:
        _check(self._lib.dns_ens_synchronize(self._h))

    def schedule(self) -> str:
        """The schedule the ensemble runs and the timings that chose it."""
        buf = ctypes.create_string_buffer(8192)
        _check(self._lib.dns_ens_get_schedule(self._h, buf, len(buf)))
        return buf.value.decode()


_M64 = (1 << 64) - 1
_GOLDEN64 = 0x9E3779B97F4A7C15


def _mix64(z):
    """SplitMix64 output function on uint64 arrays (wrapping arithmetic)."""
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def counter_normals(seed: int, field: int, count: int) -> np.ndarray:
    """Standard normal numbers 0..count-1 of stream `field` of `seed`, from the
    counter-based generator the device uses (dns_b200/csrc/init.cuh):
    SplitMix64's output function of key + (i + 1) * golden, two 53-bit
    uniforms per number, Box-Muller (cosine branch)."""
    key = int(_mix64(np.array([((seed * _GOLDEN64) + field + 1) & _M64], dtype=np.uint64))[0])
    out = np.empty(count)
    chunk = 1 << 22
    for a0 in range(0, count, chunk):
        i = np.arange(a0, min(count, a0 + chunk), dtype=np.uint64)
        with np.errstate(over="ignore"):
            a = _mix64(np.uint64(key) + (np.uint64(2) * i + np.uint64(1)) * np.uint64(_GOLDEN64))
            b = _mix64(np.uint64(key) + (np.uint64(2) * i + np.uint64(2)) * np.uint64(_GOLDEN64))
        u1 = ((a >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * 2.0 ** -53
        u2 = (b >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
        out[a0:a0 + len(i)] = np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)
    return out


def solenoidal_perturbation(n: int, seed: int, k0: float = 4.0, rng: str = "pcg64"):
    """Seeded random divergence-free velocity with energy spectrum
    E(k) ~ k^4 exp(-2 (k/k0)^2): white Gaussian noise, forward transform,
    amplitude sqrt(E(k)) / k per mode, projection onto k-perpendicular, back
    transform.  Returned with unit rms.  rng="pcg64": the noise of numpy's
    PCG64(seed); rng="counter": the device's counter-based generator
    (counter_normals), the stream dns_set_perturbed_tgv draws with k0 = 4."""
    if rng == "pcg64":
        gen = np.random.Generator(np.random.PCG64(seed))
        noise = [gen.standard_normal((n, n, n)) for _ in range(3)]
    elif rng == "counter":
        noise = [counter_normals(seed, f, n ** 3).reshape(n, n, n) for f in range(3)]
    else:
        raise ValueError(f"unknown rng {rng!r}")
    k1 = np.fft.fftfreq(n, 1.0 / n)
    kz = np.arange(n // 2 + 1, dtype=np.float64)
    KX, KY, KZ = np.meshgrid(k1, k1, kz, indexing="ij")
    kk = KX ** 2 + KY ** 2 + KZ ** 2
    kmag = np.sqrt(kk)
    amp = np.where(kmag > 0, kmag * np.exp(-((kmag / k0) ** 2)), 0.0)  # sqrt(E)/k
    # no Nyquist content (its derivative is ambiguous on the half spectrum)
    nyq = (np.abs(KX) == n // 2) | (np.abs(KY) == n // 2) | (KZ == n // 2)
    amp[nyq] = 0.0
    hats = [np.fft.rfftn(x) * amp for x in noise]
    div = (KX * hats[0] + KY * hats[1] + KZ * hats[2]) / np.where(kk > 0, kk, 1.0)
    hats = [hats[0] - KX * div, hats[1] - KY * div, hats[2] - KZ * div]
    u = [np.fft.irfftn(h, s=(n, n, n), axes=(0, 1, 2)) for h in hats]
    rms = np.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2))
    return [c / rms for c in u]


def perturbed_tgv(n: int, seed: int, amplitude: float = 1e-3, rng: str = "pcg64"):
    """Taylor-Green plus a seeded solenoidal perturbation whose rms is
    `amplitude` times the rms of the Taylor-Green field (the ensemble
    configuration's initial fields; rng as in solenoidal_perturbation)."""
    U, V, W, _ = tgv_fields(n)
    rms_tgv = np.sqrt(np.mean(U ** 2 + V ** 2 + W ** 2))
    d = solenoidal_perturbation(n, seed, rng=rng)
    s = amplitude * rms_tgv
    return U + s * d[0], V + s * d[1], W + s * d[2]


def adjoint_energy(U, V, W, nu: float, dt: float, nsteps: int, snapshots: int = 20,
                   precision: int = DNS_PREC_FP64):
    """Final energy J = E(T) (main.c's definition) after `nsteps` RK4 steps
    from (U, V, W), and its gradient: (J, (dJ/dU, dJ/dV, dJ/dW), dJ/dnu).
    The adjoint runs on the GPU (dns_adjoint_energy_prec) in the given
    precision (DNS_PREC_FP64 or DNS_PREC_MIXED)."""
    lib = load_library()
    U, V, W = _f64(U), _f64(V), _f64(W)
    n = round(U.size ** (1.0 / 3))
    g = [np.empty_like(U), np.empty_like(V), np.empty_like(W)]
    J, gnu = ctypes.c_double(), ctypes.c_double()
    _check(lib.dns_adjoint_energy_prec(n, precision, _ptr(U), _ptr(V), _ptr(W), nu, dt, nsteps,
                                       snapshots, ctypes.byref(J), _ptr(g[0]), _ptr(g[1]),
                                       _ptr(g[2]), ctypes.byref(gnu)))
    return J.value, tuple(a.reshape(U.shape) for a in g), gnu.value


def adjoint_schedule(nsteps: int, snapshots: int):
    """(forward_steps, recomputed_steps, snapshots_used) of the adjoint's
    checkpoint schedule (dns_adjoint_schedule; host only)."""
    lib = load_library()
    f, rc, used = ctypes.c_long(), ctypes.c_long(), ctypes.c_int()
    _check(lib.dns_adjoint_schedule(nsteps, snapshots, ctypes.byref(f), ctypes.byref(rc),
                                    ctypes.byref(used)))
    return f.value, rc.value, used.value


def final_energy(U, V, W, nu: float, dt: float, nsteps: int,
                 precision: int = DNS_PREC_FP64) -> float:
    """J = E(T) of adjoint_energy without its gradient: the forward sweep of
    dns_adjoint_energy_prec alone (all gradient pointers NULL), same
    arithmetic, so J is the value adjoint_energy returns."""
    lib = load_library()
    U, V, W = _f64(U), _f64(V), _f64(W)
    n = round(U.size ** (1.0 / 3))
    J = ctypes.c_double()
    _check(lib.dns_adjoint_energy_prec(n, precision, _ptr(U), _ptr(V), _ptr(W), nu, dt, nsteps, 1,
                                       ctypes.byref(J), None, None, None, None))
    return J.value


def selftest_barrier_timeout(limit_s: float = 0.05) -> bool:
    """Run the persistent kernel's barrier-wait self-test
    (dns_selftest_barrier_timeout): True when a barrier wait that can never
    complete gave up after limit_s and was reported."""
    lib = load_library()
    out = ctypes.c_int(0)
    _check(lib.dns_selftest_barrier_timeout(limit_s, ctypes.byref(out)))
    return bool(out.value)


def scale_diagnostics(eh, el, oh, ol, n):
    """main.c:265-266: long double sums times (double) invn3 * invn3."""
    invn3 = 1.0 / (n * n * n)
    s = np.longdouble(invn3 * invn3)
    return (np.longdouble(eh) + np.longdouble(el)) * s, (np.longdouble(oh) + np.longdouble(ol)) * s


def format_line(tstep: int, t: float, E, Om) -> str:
    """The stdout line of main.c:267: "% 10ld % .16e % .16Le % .16Le"."""
    def le(x):
        s = np.format_float_scientific(np.longdouble(x), precision=16, unique=False,
                                       exp_digits=2)
        return s if s.startswith("-") else " " + s
    return "% 10d % .16e %s %s" % (tstep, t, le(E), le(Om))


def step_schedule(T: float, dt: float):
    """(tstep, t) of every printed line of a run: the loop of main.c:256-423
    (print every 10 steps, stop when the accumulated t exceeds T)."""
    out = []
    t, tstep = 0.0, 0
    while True:
        if tstep % 10 == 0:
            out.append((tstep, t))
        if t > T:
            return out, tstep
        t += dt
        tstep += 1


def tgv_fields(n: int):
    """Taylor-Green initial condition as tgv.py writes it (tgv.py:14-27):
    U = sin x cos y cos z, V = -cos x sin y cos z, W = P = 0 on x_i = i 2pi/n."""
    dx = 2 * math.pi / n
    i = np.arange(n)
    s, c = np.sin(dx * i), np.cos(dx * i)
    U = np.einsum("i,j,k", s, c, c)
    V = np.einsum("i,j,k", -c, s, c)
    W = np.zeros((n, n, n))
    P = np.zeros((n, n, n))
    return U, V, W, P


def write_raw(path: str, fields) -> None:
    """Write a .raw file: 4 x n^3 float64, U V W P (tgv.py:19-27)."""
    with open(path, "wb") as f:
        for a in fields:
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())


def read_raw(path: str):
    """Read a .raw file; n from the size as main.c:163-171 does."""
    a = np.fromfile(path, dtype=np.float64)
    n = round(float(np.float32(len(a) // 4)) ** (1.0 / 3))
    if 4 * n ** 3 != len(a):
        raise ValueError(f"wrong file '{path}'")
    return n, a.reshape(4, n, n, n)
