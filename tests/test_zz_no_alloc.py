"""dns_diagnostics_noalloc: the diagnostics reduction for callers that cannot
allocate device memory at the point of the call (graph capture, a memory pool
that owns the device, latency-critical loops).  The input and the output live
in memory the caller already owns -- here torch tensors allocated by the test
itself -- and the entry point's own scratch is a fixed array inside the
library.  Checked against dns_diagnostics on the same state, twice in a row
with different states, so that a stale scratch array would show.

Collected last (file name) so that a run stopping at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROUND_TOL = 1e-13


def _noalloc(lib, n, uh_dev, out_dev, stream):
    return lib.dns_diagnostics_noalloc(n, ctypes.c_void_p(uh_dev.data_ptr()),
                                       ctypes.c_void_p(out_dev.data_ptr()), ctypes.c_void_p(stream))


@pytest.mark.parametrize("n", [32, 128])
def test_noalloc_matches_dns_diagnostics_twice(dns_lib, n):
    import torch

    import dns_b200
    from conftest import random_field

    U, V, W = random_field(n, 40 + n)
    torch.cuda.init()
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    with dns_b200.Context(n) as ctx:
        ctx.set_velocity(U, V, W)
        for call in range(2):
            if call:
                ctx.step(0.01, 0.004, 3)  # a different state for the second call
            want = ctx.diagnostics()
            uh = ctx.get_spectral()
            uh_dev = torch.from_numpy(uh.view(np.float64).copy()).to("cuda")
            out.fill_(np.nan)
            st = _noalloc(dns_lib, n, uh_dev, out, stream)
            assert st == dns_b200.DNS_OK, dns_lib.dns_last_error()
            torch.cuda.synchronize()
            eh, el, oh, ol = out.cpu().numpy().tolist()
            got = dns_b200.scale_diagnostics(eh, el, oh, ol, n)
            for g, w in zip(got, want):
                assert abs(g - w) <= ROUND_TOL * abs(w), (call, g, w)


def test_noalloc_rejects_sizes_beyond_its_scratch(dns_lib):
    import dns_b200

    for n in (1024, 2048, 12, 4):
        st = dns_lib.dns_diagnostics_noalloc(n, None, None, None)
        assert st == dns_b200.DNS_ERR_UNSUPPORTED
        assert b"n" in dns_lib.dns_last_error()
