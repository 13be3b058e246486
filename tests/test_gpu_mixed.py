"""GPU tests of the mixed-precision path (DNS_PREC_MIXED): float32 fields,
FFTs and nonlinear term; float64 reductions and update coefficients.

Tolerances are float32 ones: transforms and single steps 1e-5 relative;
the energy history of the 128^3 Taylor-Green run over t in [0, 10]
(nu = 1/1600, dt = 0.005, 2000 steps) within 1e-5 relative of the FP64 path.
"""
import numpy as np
import pytest

from conftest import random_field

pytestmark = pytest.mark.gpu

F32_TOL = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b)))


@pytest.fixture(scope="module")
def dns(dns_lib):
    import dns_b200

    return dns_b200


@pytest.mark.parametrize("n", [16, 64, 256])
def test_mixed_r2c_c2r(dns, oracle_lib, n):
    rng = np.random.default_rng(n)
    U, V, W = (rng.standard_normal((n, n, n)) for _ in range(3))
    with dns.Context(n, dns.DNS_PREC_MIXED) as ctx:
        ctx.set_velocity(U, V, W)
        uh = ctx.get_spectral()
        back = ctx.get_fields()
    for c, x in enumerate((U, V, W)):
        ref = oracle_lib.r2c_3d(x)
        assert rel_l2(uh[c], ref) <= F32_TOL
        assert rel_l2(back[c], x) <= F32_TOL


@pytest.mark.parametrize("n,steps", [(32, 1), (64, 3)])
def test_mixed_steps_match_oracle(dns, oracle_lib, n, steps):
    nu, dt = 0.02, 0.004
    U, V, W = random_field(n, 3 + n)
    o = oracle_lib.Oracle(n)
    o.set_velocity(U, V, W)
    o.step(nu, dt, steps)
    with dns.Context(n, dns.DNS_PREC_MIXED) as ctx:
        ctx.set_velocity(U, V, W)
        ctx.step(nu, dt, steps)
        uh, stale = ctx.get_spectral(), ctx.get_stale()
        E, Om = ctx.diagnostics()
    Eo, Oo = o.diagnostics()
    assert rel_l2(uh, o.get_spectral()) <= F32_TOL
    assert rel_l2(stale, o.get_stale()) <= F32_TOL
    assert abs(E - Eo) <= F32_TOL * Eo and abs(Om - Oo) <= F32_TOL * Oo


def history(dns, n, prec, nu, dt, nsteps):
    U, V, W, _ = dns.tgv_fields(n)
    E, Om = [], []
    with dns.Context(n, prec) as ctx:
        ctx.set_velocity(U, V, W)
        for q in range(nsteps // 10 + 1):
            if q:
                ctx.step(nu, dt, 10)
            e, w = ctx.diagnostics()
            E.append(float(e))
            Om.append(float(w))
    return np.array(E), np.array(Om)


def test_mixed_tgv128_energy_error_over_t10(dns):
    """Config: 128^3 Taylor-Green, nu = 1/1600, dt = 0.005, t in [0, 10]
    (2000 steps).  Energy of the mixed path within 1e-5 of the FP64 path at
    every printed step; the enstrophy error is reported."""
    n, nu, dt = 128, 1.0 / 1600, 0.005
    E64, O64 = history(dns, n, dns.DNS_PREC_FP64, nu, dt, 2000)
    E32, O32 = history(dns, n, dns.DNS_PREC_MIXED, nu, dt, 2000)
    de = np.abs(E32 - E64) / E64
    do = np.abs(O32 - O64) / O64
    print(f"\nmixed vs fp64, 128^3 Re=1600 dt=0.005 t<=10: max rel err E {de.max():.3e}, "
          f"Omega {do.max():.3e}")
    assert de.max() <= 1e-5, de.max()
    assert do.max() <= 1e-3, do.max()
