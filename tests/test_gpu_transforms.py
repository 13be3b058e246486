"""Properties of the GPU real transforms, through the public API.

The library's r2c is main.c's `fftw_plan_dft_r2c_3d` (main.c:221, 249-251):
unnormalised, e^{-ik.x}, on the half spectrum kz = 0..n/2.  Its c2r follows
FFTW's semantics for the z (real) axis (main.c:23-30): c2r(X)(x) =
sum over the half spectrum of w_z Re(X_k e^{ik.x}), w_z = 1 on the kz = 0 and
kz = n/2 planes and 2 elsewhere.  `set_velocity` applies r2c, `get_spectral`
returns the result, `set_spectral` stores a half spectrum and `get_fields`
returns c2r / n^3.  These tests check, at every grid size the library takes:
  * the round trip c2r(r2c(u)) / n^3 = u,
  * Parseval: n^3 sum_x |u|^2 = sum_k w_z |U_k|^2,
  * the transpose identity sum_x c2r(X) y = Re sum_k w_z X_k conj(r2c(y)_k)
    that the discrete adjoint is built on (c2r^T = w_z r2c).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [8, 16, 32, 64, 128, 256]


@pytest.fixture(scope="module")
def dns(dns_lib):
    import dns_b200

    return dns_b200


def wz(n):
    w = np.full(n // 2 + 1, 2.0)
    w[0] = w[n // 2] = 1.0
    return w


def fields(n, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((n, n, n)) for _ in range(3)]


@pytest.mark.parametrize("n", SIZES)
def test_round_trip(dns, n):
    u = fields(n, 1)
    with dns.Context(n) as ctx:
        ctx.set_velocity(*u)
        back = ctx.get_fields()
    err = max(float(np.abs(b.reshape(n, n, n) - a).max()) for a, b in zip(u, back))
    scale = max(float(np.abs(a).max()) for a in u)
    assert err <= 1e-13 * scale, err / scale


@pytest.mark.parametrize("n", [16, 64, 256])
def test_round_trip_mixed(dns, n):
    """FP32 storage: the round trip holds to single-precision rounding."""
    u = fields(n, 2)
    with dns.Context(n, precision=dns.DNS_PREC_MIXED) as ctx:
        ctx.set_velocity(*u)
        back = ctx.get_fields()
    err = max(float(np.abs(b.reshape(n, n, n) - a).max()) for a, b in zip(u, back))
    scale = max(float(np.abs(a).max()) for a in u)
    assert err <= 1e-5 * scale, err / scale


@pytest.mark.parametrize("n", SIZES)
def test_parseval(dns, n):
    u = fields(n, 3)
    with dns.Context(n) as ctx:
        ctx.set_velocity(*u)
        uh = ctx.get_spectral()
    w = wz(n)
    for f in range(3):
        lhs = n ** 3 * float(np.sum(u[f] ** 2))
        rhs = float(np.sum(w * np.abs(uh[f]) ** 2))
        assert abs(lhs - rhs) <= 1e-13 * lhs, (f, lhs, rhs)


@pytest.mark.parametrize("n", [8, 16, 64, 128])
def test_c2r_transpose_is_weighted_r2c(dns, n):
    """<c2r X, y> = Re <w_z r2c(y), X> for a general (non-Hermitian) half
    spectrum X, whose imaginary parts on the kz = 0 and n/2 planes c2r
    ignores."""
    rng = np.random.default_rng(4)
    nf = n // 2 + 1
    X = rng.standard_normal((3, n, n, nf)) + 1j * rng.standard_normal((3, n, n, nf))
    y = fields(n, 5)
    with dns.Context(n) as ctx:
        ctx.set_spectral(X)
        cx = ctx.get_fields()          # c2r(X) / n^3
        ctx.set_velocity(*y)
        Y = ctx.get_spectral()         # r2c(y)
    w = wz(n)
    for f in range(3):
        lhs = n ** 3 * float(np.sum(cx[f].reshape(n, n, n) * y[f]))
        rhs = float(np.sum(w * (X[f] * np.conj(Y[f])).real))
        scale = float(np.sum(w * np.abs(X[f]) * np.abs(Y[f])))
        assert abs(lhs - rhs) <= 1e-13 * scale, (f, lhs, rhs, scale)
