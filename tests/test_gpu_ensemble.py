"""GPU tests of the ensemble API (dns_ens_*): runs of mixed grid sizes and
viscosities stepped by batched kernels in one graph must give exactly the
states of the same runs stepped one at a time."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dns(dns_lib):
    import dns_b200

    return dns_b200


@pytest.mark.parametrize("prec", [0, 1])
def test_ensemble_equals_single_runs(dns, prec):
    sizes = [16, 32, 16, 64, 32, 16]
    nus = [1e-2, 3e-3, 5e-3, 2e-3, 1e-3, 2e-2]
    dts = [0.004, 0.003, 0.004, 0.002, 0.003, 0.005]
    steps = 7
    fields = [dns.perturbed_tgv(n, seed=r, amplitude=1e-2) for r, n in enumerate(sizes)]
    with dns.Ensemble(sizes, prec) as ens:
        for r, f in enumerate(fields):
            ens.set_velocity(r, *f)
        ens.set_params(nus, dts)
        ens.step(steps)
        got = [ens.get_spectral(r) for r in range(len(sizes))]
        diags = ens.diagnostics()
    for r, n in enumerate(sizes):
        with dns.Context(n, prec) as ctx:
            ctx.set_velocity(*fields[r])
            ctx.step(nus[r], dts[r], steps)
            want = ctx.get_spectral()
            E, Om = ctx.diagnostics()
        assert np.array_equal(got[r], want), r
        assert diags[r][0] == E and diags[r][1] == Om


def test_ensemble_needs_params(dns):
    with dns.Ensemble([16, 16]) as ens:
        for r in range(2):
            ens.set_velocity(r, *dns.perturbed_tgv(16, r))
        with pytest.raises(dns.DNSError) as e:
            ens.step(1)
        assert e.value.status == dns.DNS_ERR_STATE


def test_perturbation_is_solenoidal_with_unit_rms(dns):
    n = 32
    u = dns.solenoidal_perturbation(n, seed=3)
    k = np.fft.fftfreq(n, 1.0 / n)
    kz = np.arange(n // 2 + 1)
    hats = [np.fft.rfftn(c) for c in u]
    div = k[:, None, None] * hats[0] + k[None, :, None] * hats[1] + kz[None, None, :] * hats[2]
    assert np.abs(div).max() <= 1e-9 * max(np.abs(h).max() for h in hats)
    assert abs(np.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2)) - 1.0) < 1e-12
