"""The column-pass autotuner: every register schedule it may pick computes
bit-identical results (candidates differ only in register allocation), and
the schedule it reports is the fastest one it timed.  Each candidate is
forced in a fresh process (the tuner decides once per process, size and
batch shape)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, random_field

pytestmark = pytest.mark.gpu

CHILD = r"""
import sys, json
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import dns_b200
from conftest import random_field
n, prec, out = int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
with dns_b200.Context(n, prec) as c:
    c.set_velocity(*random_field(n, 77))
    c.step(0.01, 0.004, 2)
    np.save(out, c.get_spectral())
    print(json.dumps({"schedule": c.schedule()}))
"""


def _run(tmp_path, n, prec, tune):
    out = str(tmp_path / f"s_{n}_{prec}_{tune}.npy")
    env = dict(os.environ, DNS_B200_TUNE=tune)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(n), str(prec), out],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out), json.loads(r.stdout.strip().splitlines()[-1])["schedule"]


@pytest.mark.parametrize("n,prec,ncand", [(64, 0, 5), (64, 1, 6), (256, 0, 5), (256, 1, 4)])
def test_every_schedule_is_bit_identical(dns_lib, tmp_path, n, prec, ncand):
    ref, _ = _run(tmp_path, n, prec, "0")
    for k in range(ncand):
        got, sched = _run(tmp_path, n, prec, f"f{k}")
        assert np.array_equal(got.view(np.float64), ref.view(np.float64)), (k, sched)


def test_tuned_schedule_is_the_fastest_timed(dns_lib, tmp_path):
    _, sched = _run(tmp_path, 256, 0, "1")
    # "column pass <name>: min blocks/SM <m> of {<m0>: <t0> ms, ...}" per pass
    for part in sched.split("; "):
        chosen = int(part.split("min blocks/SM ")[1].split(" ")[0])
        cands = part.split("{")[1].rstrip("}").split(", ")
        times = {int(c.split(":")[0]): float(c.split(": ")[1].split(" ")[0]) for c in cands}
        assert times[chosen] == min(times.values()), part


def test_batch_is_tuned_on_its_run_count(dns_lib):
    """An ensemble group is tuned on its own batch (up to the volume of two
    256^3 runs): the schedule names the run count, and each pick is the
    fastest candidate timed on it."""
    import dns_b200

    with dns_b200.Ensemble([64] * 4 + [128] * 2, dns_b200.DNS_PREC_MIXED) as ens:
        s = ens.schedule()
    for n, runs in ((64, 4), (128, 2)):
        part = s.split(f"; n={n}: ")[1].split("; n=")[0]
        assert part.startswith(f"timed on {runs} runs: "), s
        for p in part[len(f"timed on {runs} runs: "):].split("; "):
            chosen = int(p.split("min blocks/SM ")[1].split(" ")[0])
            cands = p.split("{")[1].rstrip("}").split(", ")
            times = {int(c.split(":")[0]): float(c.split(": ")[1].split(" ")[0]) for c in cands}
            assert times[chosen] == min(times.values()), p
