"""GPU tests of the ensemble API (dns_ens_*): runs of mixed grid sizes and
viscosities stepped together, by batched kernels in one graph or by one
persistent cooperative kernel per step, must give exactly the states of the
same runs stepped one at a time."""
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


def _ens_states(dns, sizes, prec, flags, nus, dt, steps, seeds):
    with dns.Ensemble(sizes, prec, flags) as ens:
        for r in range(len(sizes)):
            ens.set_perturbed_tgv(r, seeds[r], 1e-2)
        ens.set_params(nus, dt)
        ens.step(steps)
        ens.synchronize()
        sched = ens.schedule()
        return [ens.get_spectral(r) for r in range(len(sizes))], ens.diagnostics(), sched


@pytest.mark.parametrize("prec", [0, 1])
def test_persistent_schedule_equals_batched_and_single_runs(dns, prec):
    """One cooperative launch per step (DNS_FLAG_ENS_PERSISTENT) against the
    batched graph (DNS_FLAG_ENS_BATCHED) and against each run alone: states
    and diagnostics bit-identical after 5 steps (sizes 64 and 128 mixed)."""
    sizes = [64, 128, 64, 128, 64]
    nus = [1e-2, 3e-3, 5e-3, 2e-3, 1e-3]
    dt, steps, seeds = 0.004, 5, [3, 4, 5, 6, 7]
    p, pd, ps = _ens_states(dns, sizes, prec, dns.DNS_FLAG_ENS_PERSISTENT, nus, dt, steps, seeds)
    b, bd, bs = _ens_states(dns, sizes, prec, dns.DNS_FLAG_ENS_BATCHED, nus, dt, steps, seeds)
    assert ps.startswith("persistent") and bs.startswith("batched"), (ps, bs)
    for r in range(len(sizes)):
        assert np.array_equal(p[r].view(np.float64), b[r].view(np.float64)), r
        assert pd[r] == bd[r]
    for r in (0, 1):
        with dns.Context(sizes[r], prec) as c:
            c.set_perturbed_tgv(seeds[r], 1e-2)
            c.step(nus[r], dt, steps)
            assert np.array_equal(c.get_spectral().view(np.float64), p[r].view(np.float64)), r


def test_benchmark_ensemble_both_schedules_equal_single_runs(dns):
    """The benchmark configuration (32 runs at 64^3 and 16 at 128^3, mixed
    precision, nu log-uniform in [1/3000, 1/100]) for 5 steps: the
    persistent and the batched schedules give the states of the runs
    stepped alone (checked on one run of each size and on all diagnostics)."""
    sizes = [64] * 32 + [128] * 16
    rng = np.random.Generator(np.random.PCG64(2024))
    nus = np.exp(rng.uniform(np.log(1 / 3000), np.log(1 / 100), len(sizes)))
    dt, steps, seeds = 0.005, 5, list(range(len(sizes)))
    prec = dns.DNS_PREC_MIXED
    p, pd, _ = _ens_states(dns, sizes, prec, dns.DNS_FLAG_ENS_PERSISTENT, nus, dt, steps, seeds)
    b, bd, _ = _ens_states(dns, sizes, prec, dns.DNS_FLAG_ENS_BATCHED, nus, dt, steps, seeds)
    assert pd == bd
    for r in range(len(sizes)):
        assert np.array_equal(p[r].view(np.float64), b[r].view(np.float64)), r
    for r in (5, 40):
        with dns.Context(sizes[r], prec) as c:
            c.set_perturbed_tgv(seeds[r], 1e-2)
            c.step(float(nus[r]), dt, steps)
            assert np.array_equal(c.get_spectral().view(np.float64), p[r].view(np.float64)), r


def test_ensemble_autotuner_reports_its_choice(dns):
    with dns.Ensemble([64, 128], dns.DNS_PREC_MIXED) as ens:
        s = ens.schedule()
    # "<mode> (ms per step: batched <tb>, persistent <tp>, ..."
    mode = s.split(" ")[0]
    times = s.split("ms per step: ")[1]
    tb = float(times.split("batched ")[1].split(",")[0])
    tp = float(times.split("persistent ")[1].split(",")[0])
    assert tb > 0 and tp > 0
    assert mode == ("persistent" if tp < tb else "batched"), s


def test_persistent_schedule_rejects_unsupported_sizes(dns):
    with pytest.raises(dns.DNSError) as e:
        dns.Ensemble([32, 64], dns.DNS_PREC_MIXED, dns.DNS_FLAG_ENS_PERSISTENT)
    assert e.value.status == dns.DNS_ERR_UNSUPPORTED
    with dns.Ensemble([32, 64], dns.DNS_PREC_MIXED) as ens:  # batched only
        assert ens.schedule().startswith("batched")


def test_grid_barrier_wait_limit_reports_instead_of_hanging(dns):
    """A grid barrier that can never complete gives up after its limit
    (50 ms here) and reports it; the device stays usable."""
    assert dns.selftest_barrier_timeout(0.05)
    with dns.Context(16) as c:
        c.set_tgv()
        c.step(0.01, 0.01, 1)
        E, _ = c.diagnostics()
    assert 0.12 < float(E) < 0.125
