"""Failure paths under injected allocation failures.

DNS_B200_FAIL_ALLOC=<k> makes the k-th device allocation of a process fail
as an out-of-memory would, before cudaMalloc is called: a host-side fault
injection (nothing faults on the GPU).  Each case runs in a fresh process,
since the count is per process.  The failing call must return its status
(DNS_ERR_NOMEM or DNS_ERR_CUDA, with a message), leave nothing allocated
behind that a later call trips over, and the library must stay usable: the
same call repeated (the next allocation succeeds) computes the same
result as a run without injection."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import sys, json
sys.path.insert(0, sys.argv[1])
import numpy as np
import dns_b200
what = sys.argv[2]
out = {}

def attempt(fn):
    try:
        return "ok", fn()
    except dns_b200.DNSError as e:
        return e.status, str(e)

def ctx_energy():
    with dns_b200.Context(32) as c:
        c.set_tgv()
        c.step(0.01, 0.01, 3)
        E, _ = c.diagnostics()
        return float(E)

def ens_energy():
    with dns_b200.Ensemble([32, 32, 64], dns_b200.DNS_PREC_MIXED,
                           dns_b200.DNS_FLAG_ENS_BATCHED) as e:
        for r in range(3):
            e.set_tgv(r)
        e.set_params(np.full(3, 0.01), np.full(3, 0.01))
        e.step(3)
        return [float(a) for a, _ in e.diagnostics()]

def adjoint_gnu():
    u = dns_b200.perturbed_tgv(16, seed=1, amplitude=0.2)
    J, g, gnu = dns_b200.adjoint_energy(*u, 0.02, 0.01, 4, snapshots=2)
    return [J, gnu]

fn = {"ctx": ctx_energy, "ens": ens_energy, "adjoint": adjoint_gnu}[what]
out["first"] = attempt(fn)
out["second"] = attempt(fn)
print(json.dumps(out))
"""


def _child(what, fail_at):
    env = dict(os.environ)
    env.pop("DNS_B200_FAIL_ALLOC", None)
    if fail_at:
        env["DNS_B200_FAIL_ALLOC"] = str(fail_at)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, what], capture_output=True, text=True,
                       env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("what,fail_at", [
    ("ctx", 1),       # the context's arena
    ("ens", 1),       # the first size group's arena
    ("ens", 2),       # the second size group's arena (the first is freed again)
    ("adjoint", 1),   # the adjoint's group arena
    ("adjoint", 2),   # its work and snapshot arena
])
def test_injected_allocation_failure_is_reported_and_recovered(dns_lib, what, fail_at):
    clean = _child(what, 0)
    assert clean["first"][0] == "ok" and clean["second"] == clean["first"]
    got = _child(what, fail_at)
    status, message = got["first"]
    import dns_b200

    assert status == dns_b200.DNS_ERR_NOMEM, got
    assert "out of memory" in message.lower() or "memory" in message.lower(), message
    # the library is usable afterwards and computes the same result
    assert got["second"] == clean["first"], got
