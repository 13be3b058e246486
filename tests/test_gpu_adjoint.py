"""GPU tests of the discrete adjoint (dns_adjoint_energy): the gradient of
the final energy with respect to the initial velocity and nu, against
central finite differences of FP64 forward runs, along seeded directions.
Tolerance 1e-6 relative (the target); the FD truncation and roundoff are
~1e-9 here."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dns(dns_lib):
    import dns_b200

    return dns_b200


def energy(dns, n, U, V, W, nu, dt, nsteps):
    with dns.Context(n) as ctx:
        ctx.set_velocity(U, V, W)
        ctx.step(nu, dt, nsteps)
        E, _ = ctx.diagnostics()
    return E  # numpy longdouble


def fd_check(dns, n, u0, nu, dt, nsteps, g, gnu, directions, eps=1e-6, tol=1e-6):
    worst = 0.0
    for d in directions:
        Jp = energy(dns, n, *(u0[c] + eps * d[c] for c in range(3)), nu, dt, nsteps)
        Jm = energy(dns, n, *(u0[c] - eps * d[c] for c in range(3)), nu, dt, nsteps)
        fd = float((Jp - Jm) / (2 * eps))
        ad = float(sum(np.sum(g[c] * d[c]) for c in range(3)))
        assert abs(fd - ad) <= tol * abs(ad), (fd, ad)
        worst = max(worst, abs(fd - ad) / abs(ad))
    e = eps * nu
    Jp = energy(dns, n, *u0, nu + e, dt, nsteps)
    Jm = energy(dns, n, *u0, nu - e, dt, nsteps)
    fd = float((Jp - Jm) / (2 * e))
    assert abs(fd - gnu) <= tol * abs(gnu), (fd, gnu)
    print(f"\nadjoint vs central FD, n={n} steps={nsteps}: worst direction rel err {worst:.2e}, "
          f"nu rel err {abs(fd - gnu) / abs(gnu):.2e}")


@pytest.mark.parametrize("n", [16, 32])
def test_adjoint_matches_finite_differences_small(dns, n):
    """n = 16: the transposed stage takes the velocity and vorticity the
    forward z pass kept; n = 32 (FP64 with 8 values per thread): it
    transforms them again."""
    nu, dt, nsteps = 0.02, 0.01, 12
    u0 = dns.perturbed_tgv(n, seed=5, amplitude=0.3)
    J, g, gnu = dns.adjoint_energy(*u0, nu, dt, nsteps, snapshots=4)
    assert J == pytest.approx(float(energy(dns, n, *u0, nu, dt, nsteps)), rel=1e-14)
    rng = np.random.default_rng(1)
    dirs = [dns.solenoidal_perturbation(n, seed=s) for s in (11, 12)]
    dirs.append([rng.standard_normal((n, n, n)) for _ in range(3)])  # not solenoidal
    fd_check(dns, n, u0, nu, dt, nsteps, g, gnu, dirs)


@pytest.mark.parametrize("n", [16, 32])
def test_adjoint_independent_of_checkpointing(dns, n):
    nu, dt, nsteps = 0.01, 0.01, 9
    u0 = dns.perturbed_tgv(n, seed=2, amplitude=0.2)
    ref = dns.adjoint_energy(*u0, nu, dt, nsteps, snapshots=20)
    for snaps in (1, 2, 3):
        J, g, gnu = dns.adjoint_energy(*u0, nu, dt, nsteps, snapshots=snaps)
        assert J == ref[0] and gnu == ref[2]
        for c in range(3):
            assert np.array_equal(g[c], ref[1][c])


def test_adjoint_torch_autograd(dns):
    import torch

    from dns_b200.autograd import FinalEnergy

    n, nu, dt, nsteps = 16, 0.02, 0.01, 5
    u0 = torch.tensor(np.stack(dns.perturbed_tgv(n, seed=3, amplitude=0.3)), requires_grad=True)
    nut = torch.tensor(nu, dtype=torch.float64, requires_grad=True)
    J = FinalEnergy.apply(u0, nut, dt, nsteps, 3)
    (3.0 * J).backward()
    Ja, g, gnu = dns.adjoint_energy(*u0.detach().numpy(), nu, dt, nsteps, 3)
    # the forward call ran the forward sweep alone, with the same arithmetic
    assert J.item() == Ja == dns.final_energy(*u0.detach().numpy(), nu, dt, nsteps)
    assert np.allclose(u0.grad.numpy(), 3.0 * np.stack(g), rtol=0, atol=0)
    assert nut.grad.item() == 3.0 * gnu


@pytest.mark.parametrize("n", [128, 256])
def test_adjoint_config(dns, n):
    """Config: random isotropic solenoidal field, E(k) ~ k^4 exp(-2 (k/4)^2),
    unit energy (main.c's half-spectrum E), 128^3 and 256^3, nu = 0.005,
    dt = 0.005, T = 2 (401 steps by main.c's loop), 20 snapshots, 8 seeded
    directions."""
    nu, dt = 0.005, 0.005
    _, nsteps = dns.step_schedule(2.0, dt)
    assert nsteps == 401
    u0 = dns.solenoidal_perturbation(n, seed=0)
    with dns.Context(n) as ctx:
        ctx.set_velocity(*u0)
        E0, _ = ctx.diagnostics()
    s = float(1.0 / np.sqrt(E0))
    u0 = [c * s for c in u0]
    J, g, gnu = dns.adjoint_energy(*u0, nu, dt, nsteps, snapshots=20)
    dirs = [dns.solenoidal_perturbation(n, seed=k) for k in range(1, 9)]
    fd_check(dns, n, u0, nu, dt, nsteps, g, gnu, dirs)


def _rel(a, b):
    return float(np.sqrt(sum(np.sum((a[c] - b[c]) ** 2) for c in range(3)) /
                         sum(np.sum(b[c] ** 2) for c in range(3))))


def test_mixed_adjoint_against_fp64_adjoint(dns):
    """The mixed-precision adjoint (FP32 storage and transforms) against the
    FP64 adjoint, itself pinned to finite differences above: J equals the
    mixed forward run's energy exactly, and J, the velocity gradient (L2 over
    all points) and the nu gradient agree with FP64 to 1e-4 relative (FP32
    transform error, ~1e-6 per transform, accumulated over the steps)."""
    n, nu, dt, nsteps = 32, 0.02, 0.01, 12
    u0 = dns.perturbed_tgv(n, seed=5, amplitude=0.3)
    J64, g64, gnu64 = dns.adjoint_energy(*u0, nu, dt, nsteps, snapshots=4)
    J32, g32, gnu32 = dns.adjoint_energy(*u0, nu, dt, nsteps, snapshots=4,
                                         precision=dns.DNS_PREC_MIXED)
    with dns.Context(n, dns.DNS_PREC_MIXED) as ctx:
        ctx.set_velocity(*u0)
        ctx.step(nu, dt, nsteps)
        E, _ = ctx.diagnostics()
    assert J32 == pytest.approx(float(E), rel=1e-14)
    assert J32 == dns.final_energy(*u0, nu, dt, nsteps, precision=dns.DNS_PREC_MIXED)
    eg, enu = _rel(g32, g64), abs(gnu32 - gnu64) / abs(gnu64)
    print(f"\nmixed vs FP64 adjoint, n={n} steps={nsteps}: J rel {abs(J32 - J64) / J64:.2e}, "
          f"gradient rel L2 {eg:.2e}, nu gradient rel {enu:.2e}")
    assert abs(J32 - J64) <= 1e-4 * J64
    assert eg <= 1e-4 and enu <= 1e-4
    # checkpointing leaves the mixed gradient bit-identical too
    J, g, gnu = dns.adjoint_energy(*u0, nu, dt, nsteps, snapshots=1,
                                   precision=dns.DNS_PREC_MIXED)
    assert J == J32 and gnu == gnu32
    for c in range(3):
        assert np.array_equal(g[c], g32[c])


def test_mixed_adjoint_config_128(dns):
    """The adjoint configuration (random isotropic field of unit energy,
    128^3, nu = dt = 0.005, 401 steps, 20 snapshots) in mixed precision
    against FP64: gradient rel L2 and nu gradient within 1e-3 (the 401-step
    mixed forward itself differs from FP64 by ~1e-5 in energy)."""
    n, nu, dt = 128, 0.005, 0.005
    _, nsteps = dns.step_schedule(2.0, dt)
    u0 = dns.solenoidal_perturbation(n, seed=0)
    with dns.Context(n) as ctx:
        ctx.set_velocity(*u0)
        E0, _ = ctx.diagnostics()
    u0 = [c * float(1.0 / np.sqrt(E0)) for c in u0]
    J64, g64, gnu64 = dns.adjoint_energy(*u0, nu, dt, nsteps, snapshots=20)
    J32, g32, gnu32 = dns.adjoint_energy(*u0, nu, dt, nsteps, snapshots=20,
                                         precision=dns.DNS_PREC_MIXED)
    eg, enu = _rel(g32, g64), abs(gnu32 - gnu64) / abs(gnu64)
    print(f"\nmixed vs FP64 adjoint, n={n} steps={nsteps}: J rel {abs(J32 - J64) / J64:.2e}, "
          f"gradient rel L2 {eg:.2e}, nu gradient rel {enu:.2e}")
    assert abs(J32 - J64) <= 1e-4 * J64
    assert eg <= 1e-3 and enu <= 1e-3
