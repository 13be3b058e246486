"""Restart from a saved state.

Two ways to stop a run and continue it later:

* the exact checkpoint of the C ABI: the spectral velocity plus the stale
  real-space velocity that main.c's first RK stage reads (main.c:344 skips
  the back transform at rk == 0, so that field is part of the step state).
  Stopping after k steps, saving both, restoring them into a fresh context
  and stepping m more must equal k + m unbroken steps bit for bit;
* the reference's own restart: a -d dump (main.c:269-279) fed back with -i
  (main.c:163-185).  The dump holds c2r(U_hat) / n^3 only, so on restart the
  stale velocity becomes that field instead of the one the unbroken run
  carried: the reference's restart is not bit-identical to its unbroken run,
  and the drop-in must reproduce exactly that behaviour.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import random_field, read_history

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dns(dns_lib):
    import dns_b200

    return dns_b200


@pytest.mark.parametrize("n,prec", [(32, 0), (64, 0), (64, 1)])
def test_checkpoint_restore_is_bit_identical(dns, n, prec):
    nu, dt, k, m = 0.01, 0.004, 7, 5
    U, V, W = random_field(n, 300 + n)
    with dns.Context(n, prec) as a:
        a.set_velocity(U, V, W)
        a.step(nu, dt, k)
        uh, stale = a.get_spectral(), a.get_stale()
        a.step(nu, dt, m)
        want_uh, want_stale = a.get_spectral(), a.get_stale()
        want_diag = a.diagnostics_dd()
    with dns.Context(n, prec) as b:
        b.set_spectral(uh)
        b.set_stale(stale)
        b.step(nu, dt, m)
        got_uh, got_stale = b.get_spectral(), b.get_stale()
        got_diag = b.diagnostics_dd()
    assert np.array_equal(got_uh.view(np.float64), want_uh.view(np.float64))
    assert np.array_equal(got_stale, want_stale)
    assert got_diag == want_diag


def test_checkpoint_without_stale_is_not_exact(dns):
    """Restoring the spectral state alone (the stale velocity left as the
    context's default) changes the next step: the stale field is state."""
    n, nu, dt = 32, 0.01, 0.004
    U, V, W = random_field(n, 333)
    with dns.Context(n) as a:
        a.set_velocity(U, V, W)
        a.step(nu, dt, 4)
        uh = a.get_spectral()
        a.step(nu, dt, 1)
        want = a.get_spectral()
    with dns.Context(n) as b:
        b.set_spectral(uh)
        b.step(nu, dt, 1)
        got = b.get_spectral()
    assert np.linalg.norm(got - want) > 1e-8 * np.linalg.norm(want)


def _run(cli, raw, cwd, nu, dt, T, dump=False):
    args = [cli] + (["-d"] if dump else []) + ["-i", raw, "-n", nu, "-s", dt, "-t", T]
    r = subprocess.run(args, capture_output=True, text=True, cwd=cwd)
    assert r.returncode == 0, r.stderr
    return r.stdout


def _lines(text):
    return [l for l in text.splitlines() if l.strip()]


def test_cli_restart_from_dump_matches_reference(dns, oracle_lib, tmp_path):
    """Run 20 steps with -d, restart from the step-10 dump for 10 more steps:
    the drop-in and the reference main.c (oracle/_ref) print the same
    restart history (1e-12), and both differ from their own unbroken run by
    far more than rounding, because the restart's stale velocity is
    c2r(U_hat) (main.c:344, main.c:270-279)."""
    n, nu, dt = 16, "0.02", "0.005"
    # velocity up to 3, so that the nonlinear term (where the stale field
    # enters) moves the restart visibly: ~4e-10 relative after 10 steps
    U, V, W = (3.0 * a for a in random_field(n, 44))
    raw = str(tmp_path / "in.raw")
    dns.write_raw(raw, [U, V, W, np.zeros_like(U)])
    hist = {}
    for who, exe in (("mine", dns.CLI_PATH), ("ref", oracle_lib.REF_DNS)):
        d = tmp_path / who
        d.mkdir()
        full = _run(exe, raw, d, nu, dt, "0.0999", dump=True)  # 20 steps, dumps at 0, 10, 20
        assert os.path.exists(d / "00000010.raw")
        restart = _run(exe, str(d / "00000010.raw"), d, nu, dt, "0.0499")  # 10 steps
        hist[who] = (_lines(full), _lines(restart))
    for a, b in zip(hist["mine"][1], hist["ref"][1]):
        xa, xb = a.split(), b.split()
        assert a[:10] == b[:10] and xa[:2] == xb[:2] and len(a) == len(b)
        for x, y in zip(xa[2:], xb[2:]):
            assert abs(float(x) - float(y)) <= 1e-12 * abs(float(y)), (a, b)
    assert len(hist["mine"][1]) == len(hist["ref"][1]) == 2
    for who in ("mine", "ref"):
        full, restart = hist[who]
        e_full = float(full[2].split()[2])      # unbroken run, step 20
        e_rst = float(restart[1].split()[2])    # restarted at 10, +10 steps
        assert abs(e_rst - e_full) > 1e-11 * e_full, (who, e_rst, e_full)
