"""CPU tests of the host side: the C ABI exports, the CLI's argument and
input handling (compared with the reference main.c's own behaviour), the
step schedule and the print format.  No GPU: every CLI case here exits
before the first CUDA call."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def declared_functions():
    hdr = open(os.path.join(ROOT, "include", "dns_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(dns_[a-z_0-9]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol(dns_lib):
    names = declared_functions()
    assert "dns_step" in names and "dns_create" in names
    for name in names:
        assert hasattr(dns_lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", dns_lib._name], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (dns_\w+)", out))
    assert set(names) <= exported


def test_strerror_without_gpu(dns_lib):
    import dns_b200

    assert dns_lib.dns_strerror(dns_b200.DNS_OK) == b"success"
    assert b"unsupported" in dns_lib.dns_strerror(dns_b200.DNS_ERR_UNSUPPORTED)


CLI_CASES = [
    [],
    ["-x"],
    ["-i"],
    ["-n"],
    ["-s"],
    ["-t"],
    ["-n", "0.1x"],
    ["-t", "1", "-n", "0.01", "-s", "0.01"],
    ["-t", "1", "-n", "0.01", "-i", "in.raw"],
    ["-t", "1", "-s", "0.01", "-i", "in.raw"],
    ["-n", "0.01", "-s", "0.01", "-i", "in.raw"],
    ["-t", "0", "-n", "0.01", "-s", "0.01", "-i", "in.raw"],
    ["-t", "1", "-n", "0.01", "-s", "0.01", "-i", "missing.raw"],
    ["-t", "1", "-n", "0.01", "-s", "0.01", "-i", "bad.raw"],
]


@pytest.mark.parametrize("args", CLI_CASES, ids=[" ".join(a) or "noargs" for a in CLI_CASES])
def test_cli_errors_match_reference(dns_lib, oracle_lib, tmp_path, args):
    import dns_b200

    (tmp_path / "bad.raw").write_bytes(b"\0" * (8 * 4 * 8 + 8))  # not 4 n^3 doubles
    (tmp_path / "in.raw").write_bytes(b"\0" * (8 * 4 * 8))
    mine = subprocess.run([dns_b200.CLI_PATH, *args], capture_output=True, text=True, cwd=tmp_path)
    ref = subprocess.run([oracle_lib.REF_DNS, *args], capture_output=True, text=True, cwd=tmp_path)
    assert mine.returncode == ref.returncode == 1
    assert mine.stdout == ref.stdout == ""
    assert mine.stderr == ref.stderr


def test_cli_help_text(dns_lib, oracle_lib):
    import dns_b200

    mine = subprocess.run([dns_b200.CLI_PATH, "-h"], capture_output=True, text=True)
    ref = subprocess.run([oracle_lib.REF_DNS, "-h"], capture_output=True, text=True)
    assert mine.returncode == ref.returncode == 1
    # identical usage; only the build-info line names the backend
    assert mine.stderr.split("\nBuild Info:")[0] == ref.stderr.split("\nBuild Info:")[0]


@pytest.mark.parametrize("T,dt,steps", [(1.0, 0.01, 100), (10.0, 0.005, 2000), (10.0, 0.0025, 4000),
                                        (0.5, 0.0025, 200), (2.0, 0.005, 401)])
def test_step_schedule(T, dt, steps):
    """main.c:332-333, 421: stop when the accumulated t exceeds T."""
    import dns_b200

    sched, total = dns_b200.step_schedule(T, dt)
    assert total == steps
    assert sched[0] == (0, 0.0)
    assert all(s % 10 == 0 for s, _ in sched)


def test_format_line_matches_reference_output():
    import dns_b200

    from conftest import read_history

    for name in ("ref_0128_1600.txt", "ref_0256_3000.txt", "refrun_tgv64_nu0.01_dt0.01_T1.txt"):
        path = os.path.join(GOLDEN, name)
        steps, ts, E, Om = read_history(path)
        lines = open(path).read().splitlines()
        for q in range(len(lines)):
            assert dns_b200.format_line(int(steps[q]), float(ts[q]), E[q], Om[q]) == lines[q]


def test_raw_roundtrip(tmp_path):
    import dns_b200

    f = dns_b200.tgv_fields(8)
    p = str(tmp_path / "a.raw")
    dns_b200.write_raw(p, f)
    n, a = dns_b200.read_raw(p)
    assert n == 8 and np.array_equal(a[0], f[0]) and np.array_equal(a[1], f[1])


def test_product_does_not_import_oracle():
    """The product package has no path into the oracle (no CPU fallback)."""
    pkg = os.path.join(ROOT, "dns_b200")
    for dirpath, _, files in os.walk(pkg):
        for fn in files:
            if fn.endswith((".py", ".c", ".cu", ".cuh", ".h")):
                text = open(os.path.join(dirpath, fn)).read()
                assert "import oracle" not in text and "liboracle" not in text, fn


@pytest.mark.parametrize("n", [8, 16, 32, 64, 128, 256, 512])
def test_bench_mask_fractions_follow_the_two_thirds_rule(n):
    """bench.py counts the N traffic of the masked forward passes with the
    mode counts of main.c's mask (|k| < 2/3 (n/2 + 1), main.c:231-238)."""
    import bench

    kmax = 2.0 / 3.0 * (n // 2 + 1)
    kz = [k for k in range(n // 2 + 1) if abs(k) < kmax]
    kxy = [i if i < n // 2 else i - n for i in range(n)]
    kxy = [k for k in kxy if abs(k) < kmax]
    fz, fxy = bench.mask_fractions(n)
    assert fz == len(kz) / (n // 2 + 1)
    assert fxy == len(kxy) / n


def test_bench_step_bytes_256():
    """Algorithmic bytes of one 256^3 FP64 step (the figure the roofline
    fields are built on): 25.13 GB with the masked forward passes."""
    import bench

    total = sum(map(sum, bench.pass_bytes(256)))
    assert abs(total / 1e9 - 25.13) < 0.01, total


def _scalar_counter_normal(seed, field, i):
    """Pure-Python restatement of the counter-based generator (SplitMix64
    output function, Box-Muller), one number at a time."""
    import math

    m = (1 << 64) - 1
    g = 0x9E3779B97F4A7C15

    def mix(z):
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
        return z ^ (z >> 31)

    key = mix((seed * g + field + 1) & m)
    a = mix((key + (2 * i + 1) * g) & m)
    b = mix((key + (2 * i + 2) * g) & m)
    u1 = ((a >> 11) + 1) * 2.0 ** -53
    u2 = (b >> 11) * 2.0 ** -53
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586 * u2)


def test_counter_normals_match_scalar_restatement_and_are_normal():
    """The numpy form of the device's noise generator (used as the host
    reference of dns_set_perturbed_tgv) against a scalar restatement, and
    its first two moments."""
    import dns_b200

    for seed, field in ((0, 0), (12345, 2), (2 ** 63 + 7, 1)):
        x = dns_b200.counter_normals(seed, field, 1 << 12)
        for i in (0, 1, 2, 1000, 4095):
            assert x[i] == pytest.approx(_scalar_counter_normal(seed, field, i), rel=1e-15, abs=1e-15)
    x = dns_b200.counter_normals(3, 0, 1 << 20)
    assert abs(x.mean()) < 5e-3 and abs(x.std() - 1) < 5e-3
    assert np.array_equal(x[:100], dns_b200.counter_normals(3, 0, 100))  # a counter, not a state
    assert not np.allclose(x[:100], dns_b200.counter_normals(3, 1, 100))


def _schedule_restated(nsteps, snapshots):
    """The binomial checkpoint schedule restated: (forward, recomputed)."""
    from math import comb

    cnt = {"adv": 0}

    def split(a, b, free):
        l, rr = b - a, 0
        while comb(free + rr, free) < l:
            rr += 1
        return b - max(min(comb(free - 1 + rr, free - 1), l - 1), 1)

    def rev(a, b, free, stored):
        if b - a == 1:
            return
        if free == 0:
            cnt["adv"] += sum(t - a for t in range(a, b))
            return
        m = split(a, b, free)
        if not stored:
            cnt["adv"] += m - a
        rev(m, b, free - 1, stored)
        rev(a, m, free, False)

    rev(0, nsteps, snapshots - 1, True)
    return nsteps + cnt["adv"], cnt["adv"]


@pytest.mark.parametrize("nsteps,snapshots", [(401, 20), (401, 1), (401, 2), (401, 401),
                                              (12, 4), (9, 3), (1, 1), (1000, 7)])
def test_adjoint_schedule_counts(dns_lib, nsteps, snapshots):
    """dns_adjoint_schedule (host only) counts the schedule the adjoint
    runs: against a restatement, the known cases (one snapshot recomputes
    every step from the start; enough snapshots recompute nothing), and
    never more snapshots than given."""
    import dns_b200

    fwd, rec, used = dns_b200.adjoint_schedule(nsteps, snapshots)
    assert (fwd, rec) == _schedule_restated(nsteps, snapshots)
    assert fwd == nsteps + rec and 1 <= used <= snapshots
    if snapshots == 1:
        assert rec == nsteps * (nsteps - 1) // 2
    if snapshots >= nsteps:
        assert rec == 0
    if (nsteps, snapshots) == (401, 20):
        assert rec == 684


def test_adjoint_schedule_more_snapshots_recompute_less(dns_lib):
    import dns_b200

    recs = [dns_b200.adjoint_schedule(401, s)[1] for s in range(1, 40)]
    assert all(a >= b for a, b in zip(recs, recs[1:]))
    with pytest.raises(dns_b200.DNSError):
        dns_b200.adjoint_schedule(0, 3)
