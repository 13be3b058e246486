import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.load()
    # the host may be shared: a few threads are faster than oversubscription
    oracle.set_threads(min(4, os.cpu_count() or 1))
    return oracle


@pytest.fixture(scope="session")
def dns_lib():
    """The CUDA library; built in-tree if it is missing (nvcc present)."""
    import dns_b200

    if not os.path.exists(dns_b200.LIB_PATH) or not os.path.exists(dns_b200.CLI_PATH):
        from dns_b200 import build

        build.build_library()
        build.build_cli()
    return dns_b200.load_library()


def read_history(path):
    """Parse `tstep t E Om` lines (main.c:267) into arrays; E/Om as longdouble."""
    steps, ts, es, os_ = [], [], [], []
    with open(path) as f:
        for line in f:
            a = line.split()
            if len(a) != 4:
                continue
            steps.append(int(a[0]))
            ts.append(float(a[1]))
            es.append(np.longdouble(a[2]))
            os_.append(np.longdouble(a[3]))
    return np.array(steps), np.array(ts), np.array(es, dtype=np.longdouble), np.array(os_, dtype=np.longdouble)


def random_field(n, seed, kmax=None):
    """Seeded real random velocity with a decaying spectrum (smooth enough for
    a few explicit steps), returned as three n^3 float64 arrays."""
    rng = np.random.default_rng(seed)
    out = []
    k = np.fft.fftfreq(n, 1.0 / n)
    kz = np.arange(n // 2 + 1)
    kk = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    amp = np.exp(-kk / (2.0 * (n / 8) ** 2))
    for _ in range(3):
        x = rng.standard_normal((n, n, n))
        X = np.fft.rfftn(x) * amp
        out.append(np.fft.irfftn(X, s=(n, n, n), axes=(0, 1, 2)))
    s = max(np.abs(a).max() for a in out)
    return [a / s for a in out]


def run_ref_dns(raw, nu, dt, T, extra=(), cwd=None):
    import oracle

    r = subprocess.run([oracle.REF_DNS, *extra, "-i", raw, "-n", str(nu), "-s", str(dt), "-t", str(T)],
                       capture_output=True, text=True, cwd=cwd)
    return r
