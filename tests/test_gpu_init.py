"""Initial fields generated on the device (dns_set_tgv, dns_set_perturbed_tgv
and their ensemble forms) against the host generators:

* Taylor-Green must be bit-identical to tgv.py's field (tgv_fields, whose
  bytes the CPU tests pin against the reference tgv.py) and its transform
  bit-identical to dns_set_velocity of that field;
* the perturbation must match the numpy generator driven by the same
  counter-based random stream (perturbed_tgv(..., rng="counter")) within
  1e-14 relative to the perturbation itself in FP64 (the two differ only by
  the rounding of their FFTs and of log/cos);
* a mixed-precision context holds that field in float32, its perturbation
  made with FP32 transforms.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dns(dns_lib):
    import dns_b200

    return dns_b200


@pytest.mark.parametrize("n", [16, 64, 256])
def test_set_tgv_is_tgv_py_bit_for_bit(dns, n):
    U, V, W, _ = dns.tgv_fields(n)
    with dns.Context(n) as a:
        a.set_tgv()
        stale, uh = a.get_stale(), a.get_spectral()
        E, Om = a.diagnostics()
    assert np.array_equal(stale[0], U) and np.array_equal(stale[1], V) and np.array_equal(stale[2], W)
    with dns.Context(n) as b:
        b.set_velocity(U, V, W)
        assert np.array_equal(b.get_spectral().view(np.float64), uh.view(np.float64))
    assert abs(float(E) - 0.125) <= 1e-15 and abs(float(Om) - 0.375) <= 1e-15


@pytest.mark.parametrize("n,seed", [(32, 3), (64, 11)])
def test_set_perturbed_tgv_matches_numpy_counter_stream(dns, n, seed):
    amp = 1e-3
    want = np.stack(dns.perturbed_tgv(n, seed, amplitude=amp, rng="counter"))
    tgv = np.stack(dns.tgv_fields(n)[:3])
    with dns.Context(n) as a:
        a.set_perturbed_tgv(seed, amp)
        got, uh = a.get_stale(), a.get_spectral()
    err = np.linalg.norm(got - want) / np.linalg.norm(want - tgv)
    assert err <= 1e-14, err
    # the perturbation has the requested size and is divergence-free
    d = got - tgv
    rms = np.sqrt(np.mean(np.sum(d ** 2, axis=0)))
    assert abs(rms / (amp * np.sqrt(np.mean(np.sum(tgv ** 2, axis=0)))) - 1) <= 1e-12
    k = np.fft.fftfreq(n, 1.0 / n)
    D = [np.fft.rfftn(d[c]) for c in range(3)]
    div = k[:, None, None] * D[0] + k[None, :, None] * D[1] + np.arange(n // 2 + 1)[None, None, :] * D[2]
    assert np.abs(div).max() <= 1e-12 * n * np.abs(D[0]).max()
    # the state is that field's forward transform, exactly as dns_set_velocity makes it
    with dns.Context(n) as b:
        b.set_velocity(*got)
        assert np.array_equal(b.get_spectral().view(np.float64), uh.view(np.float64))


def test_set_perturbed_tgv_mixed_is_float32(dns):
    """A mixed-precision context builds the perturbation with its own FP32
    transforms (noise, r2c, shaping in FP64 registers, c2r), adds it to
    Taylor-Green in FP64 and rounds the sum to float32: the perturbation
    carries FP32 transform error (~1e-7 of itself), the Taylor-Green part
    only the final rounding."""
    n, seed, amp = 32, 5, 1e-3
    want = np.stack(dns.perturbed_tgv(n, seed, amplitude=amp, rng="counter"))
    tgv = np.stack(dns.tgv_fields(n)[:3])
    with dns.Context(n, dns.DNS_PREC_MIXED) as a:
        a.set_perturbed_tgv(seed, amp)
        got = a.get_stale()
    assert np.array_equal(got, got.astype(np.float32).astype(np.float64))  # float32 values
    # float32 storage of the whole field: 2^-24 relative per value
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err <= 1e-7, err
    # per value: the storage rounding (a rounding boundary may flip: one
    # ulp) plus the FP32 transforms' error on the perturbation
    ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
    pert = np.abs(want - tgv).max()
    assert np.all(np.abs(got - want) <= ulp + 1e-5 * pert)


def test_ensemble_generators_equal_single_runs(dns):
    sizes = [16, 32, 16]
    seeds = [4, 9, 13]
    with dns.Ensemble(sizes) as ens:
        ens.set_perturbed_tgv(0, seeds[0], 1e-2)
        ens.set_tgv(1)
        ens.set_perturbed_tgv(2, seeds[2], 3e-3)
        got = [ens.get_spectral(r) for r in range(3)]
    for r, n in enumerate(sizes):
        with dns.Context(n) as c:
            if r == 1:
                c.set_tgv()
            else:
                c.set_perturbed_tgv(seeds[r], 1e-2 if r == 0 else 3e-3)
            assert np.array_equal(c.get_spectral().view(np.float64), got[r].view(np.float64))
