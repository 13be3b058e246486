"""CPU tests of the oracle (the parity checker) -- no GPU.

1. Its FFT against a naive DFT, the pattern of the reference's
   poc/one.c:35-51 and poc/three.c:46-70 (e^{-i} forward, no normalisation),
   and against numpy's pocketfft.
2. The restated RK4 loop against the reference main.c compiled unchanged on
   the same FFT (oracle/_ref/dns): identical stdout, identical dumps.
3. Both against the reference's own shipped golden histories (0128/*,
   0256/*), which pins the oracle to FFTW-built runs of main.c.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, random_field, read_history, run_ref_dns


def naive_dft3(x, sign=-1):
    out = x.astype(np.complex128)
    for ax in range(x.ndim):
        n = x.shape[ax]
        j = np.arange(n)
        M = np.exp(sign * 2j * np.pi * np.outer(j, j) / n)
        out = np.moveaxis(np.tensordot(M, np.moveaxis(out, ax, 0), axes=(1, 0)), 0, ax)
    return out


@pytest.mark.parametrize("shape", [(2, 2, 2), (4, 4, 4), (8, 4, 16), (3, 5, 6), (1, 1, 10), (8, 8, 8)])
def test_r2c_matches_naive_dft(oracle_lib, shape):
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape)
    X = oracle_lib.r2c_3d(x)
    ref = naive_dft3(x)[..., : shape[2] // 2 + 1]
    assert np.abs(X - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("n", [8, 16, 32, 64])
def test_r2c_c2r_vs_pocketfft(oracle_lib, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n))
    X = oracle_lib.r2c_3d(x)
    ref = np.fft.rfftn(x)
    assert np.abs(X - ref).max() <= 1e-14 * np.abs(ref).max()
    y = oracle_lib.c2r_3d(X, n)
    assert np.abs(y / n ** 3 - x).max() <= 1e-14 * np.abs(x).max()


def test_c2r_ignores_imag_of_dc_and_nyquist(oracle_lib):
    """FFTW's c2r ignores Im of the kz = 0 and kz = n/2 inputs after the
    complex transforms of the leading axes (Hermitian part only)."""
    n = 8
    rng = np.random.default_rng(3)
    X = rng.standard_normal((n, n, n // 2 + 1)) + 1j * rng.standard_normal((n, n, n // 2 + 1))
    y = oracle_lib.c2r_3d(X, n)
    # explicit definition: complex inverse over x, y; then per z line take
    # the Hermitian extension with real DC / Nyquist
    Z = np.fft.ifft(np.fft.ifft(X, axis=0), axis=1) * n * n
    Z[..., 0] = Z[..., 0].real
    Z[..., n // 2] = Z[..., n // 2].real
    full = np.concatenate([Z, np.conj(Z[..., 1 : n // 2][..., ::-1])], axis=-1)
    ref = np.fft.ifft(full, axis=-1).real * n
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()


def test_twiddles_exact_symmetries(oracle_lib):
    import ctypes

    lib = oracle_lib.load()
    lib.shim_sincos2pi.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]
    c, s = ctypes.c_double(), ctypes.c_double()
    for n in (8, 64, 256):
        for k, (ce, se) in {0: (1, 0), n // 4: (0, 1), n // 2: (-1, 0), 3 * n // 4: (0, -1)}.items():
            lib.shim_sincos2pi(k, n, ctypes.byref(c), ctypes.byref(s))
            assert (c.value, s.value) == (ce, se)
        lib.shim_sincos2pi(n // 8, n, ctypes.byref(c), ctypes.byref(s))
        assert c.value == s.value == np.sqrt(0.5)


def test_restatement_equals_reference_main(oracle_lib, tmp_path):
    """The C restatement and main.c itself, on the same FFT, print the same
    bytes (Taylor-Green 32^3, 21 steps)."""
    import dns_b200

    n, nu, dt, T = 32, 0.01, 0.01, 0.2
    raw = str(tmp_path / "tgv.raw")
    dns_b200.write_raw(raw, dns_b200.tgv_fields(n))
    ref_out = run_ref_dns(raw, nu, dt, T).stdout.splitlines()
    o = oracle_lib.Oracle(n)
    U, V, W, _ = dns_b200.tgv_fields(n)
    o.set_velocity(U, V, W)
    sched, _ = dns_b200.step_schedule(T, dt)
    lines, done = [], 0
    for tstep, t in sched:
        o.step(nu, dt, tstep - done)
        done = tstep
        lines.append(dns_b200.format_line(tstep, t, *o.diagnostics()))
    assert lines == ref_out


def test_restatement_random_field_equals_reference_main(oracle_lib, tmp_path):
    """A general (non-Taylor-Green) field, with dumps: the -d output of
    main.c equals the restatement's fields bit for bit."""
    import dns_b200

    n, nu, dt, T = 16, 0.02, 0.005, 0.05
    U, V, W = random_field(n, 11)
    raw = str(tmp_path / "in.raw")
    dns_b200.write_raw(raw, [U, V, W, np.zeros_like(U)])
    r = run_ref_dns(raw, nu, dt, T, extra=("-d",), cwd=str(tmp_path))
    assert r.returncode == 0
    o = oracle_lib.Oracle(n)
    o.set_velocity(U, V, W)
    sched, _ = dns_b200.step_schedule(T, dt)
    lines, done = [], 0
    for tstep, t in sched:
        o.step(nu, dt, tstep - done)
        done = tstep
        lines.append(dns_b200.format_line(tstep, t, *o.diagnostics()))
        if tstep > 0:
            ref = np.fromfile(str(tmp_path / f"{tstep:08d}.raw")).reshape(4, n, n, n)
            mine = o.dump_fields()
            assert np.array_equal(ref, mine)
    assert lines == r.stdout.splitlines()


def _oracle_history(oracle_lib, n, nu, dt, nlines):
    import dns_b200

    o = oracle_lib.Oracle(n)
    U, V, W, _ = dns_b200.tgv_fields(n)
    o.set_velocity(U, V, W)
    E, Om = [], []
    for q in range(nlines):
        if q:
            o.step(nu, dt, 10)
        e, w = o.diagnostics()
        E.append(e)
        Om.append(w)
    return np.array(E, dtype=np.longdouble), np.array(Om, dtype=np.longdouble)


@pytest.mark.parametrize("re_", ["1600", "0100"])
def test_oracle_matches_golden_0128(oracle_lib, re_):
    """The oracle reproduces the reference's FFTW-built 128^3 history
    (dt = 0.0025, nu = 1/Re) over the first 20 steps to 1e-15."""
    steps, ts, Eg, Og = read_history(os.path.join(GOLDEN, f"ref_0128_{re_}.txt"))
    nu = float("%.16e" % (1.0 / int(re_)))  # run.sh:1 formats nu with %.16e
    E, Om = _oracle_history(oracle_lib, 128, nu, 0.0025, 3)
    assert np.all(np.abs(E - Eg[:3]) <= 1e-15 * Eg[:3])
    assert np.all(np.abs(Om - Og[:3]) <= 1e-15 * Og[:3])


def test_tgv_generator_matches_reference_bytes(tmp_path):
    """dns_b200.tgv writes the same bytes as the reference tgv.py."""
    import hashlib

    import dns_b200

    for level in (3, 4, 5, 6):
        raw = str(tmp_path / f"t{level}.raw")
        dns_b200.write_raw(raw, dns_b200.tgv_fields(1 << level))
        want = open(os.path.join(GOLDEN, f"tgv_l{level}.sha256")).read().strip()
        assert hashlib.sha256(open(raw, "rb").read()).hexdigest() == want


@pytest.mark.parametrize("n", [16, 32])
def test_numpy_restatement_agrees_with_c_oracle(oracle_lib, n):
    """The numpy restatement of main.c's step (pocketfft, not the shim FFT)
    against the C oracle: a Taylor-Green field plus a seeded solenoidal
    perturbation (so that every term of the step is exercised), 6 steps,
    energy and enstrophy at every step to 1e-13, final spectra to 1e-12
    (relative L2)."""
    import dns_b200
    from oracle import Oracle
    from oracle.numpy_restatement import NumpyDNS

    U, V, W, _ = dns_b200.tgv_fields(n)
    d = dns_b200.solenoidal_perturbation(n, seed=3)
    U, V, W = U + 0.1 * d[0], V + 0.1 * d[1], W + 0.1 * d[2]
    o = Oracle(n)
    m = NumpyDNS(n)
    try:
        o.set_velocity(U, V, W)
        m.set_velocity(U, V, W)
        for _ in range(6):
            Eo, Oo = o.diagnostics()
            Em, Om = m.diagnostics()
            assert abs(Eo - Em) <= 1e-13 * abs(Eo), (Eo, Em)
            assert abs(Oo - Om) <= 1e-13 * abs(Oo), (Oo, Om)
            o.step(0.01, 0.01, 1)
            m.step(0.01, 0.01, 1)
        uo = o.get_spectral()
        um = np.stack(m.uh)
        assert np.linalg.norm(uo - um) <= 1e-12 * np.linalg.norm(uo)
    finally:
        o.close()
