"""Second CPU restatement of main.c's RK4 step, in numpy -- TEST
INFRASTRUCTURE ONLY (a cross-check of the C oracle, never the product).

The C oracle (oracle/dns_oracle.c) and the reference main.c compiled on the
project's FFTW-subset shim share that shim's FFT.  This restatement runs on
numpy's pocketfft instead, so agreement between the two pins the shim FFT
and the C restatement independently.  FFTW's conventions are kept:
unnormalised transforms, e^{-i} forward, and a c2r that takes complex
backward transforms over x and y, then a 1D c2r along z that ignores the
imaginary parts of the kz = 0 and kz = n/2 inputs (numpy's irfftn does the
same); numpy's 1/n^3 scaling is undone by an exact power-of-two factor.
Small n only (the tests use 16 and 32).
"""
from __future__ import annotations

import numpy as np

# main.c:15-16
RK_A = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)
RK_B = (0.5, 0.5, 1.0)


class NumpyDNS:
    def __init__(self, n: int):
        self.n = n
        nf = n // 2 + 1
        # main.c:224-230: kx[i] = i below n/2, i - n from n/2 (kx[n/2] = -n/2)
        k = np.arange(n, dtype=np.float64)
        kx = np.where(k < n // 2, k, k - n)
        kz = np.arange(nf, dtype=np.float64)
        self.KX = kx[:, None, None]
        self.KY = kx[None, :, None]
        self.KZ = kz[None, None, :]
        # main.c:231-239: the 2/3 rule with kmax = 2/3 (n/2 + 1)
        kmax = 2.0 / 3.0 * (n // 2 + 1)
        self.mask = ((np.abs(self.KX) < kmax) & (np.abs(self.KY) < kmax)
                     & (np.abs(self.KZ) < kmax)).astype(np.float64)
        # main.c:241-247
        self.kk = self.KX * self.KX + self.KY * self.KY + self.KZ * self.KZ
        self.invn3 = 1.0 / float(n) ** 3
        self.uh = None
        self.u = None

    def c2r(self, X: np.ndarray) -> np.ndarray:
        """main.c:23-30: unnormalised c2r (FFTW's semantics)."""
        n = self.n
        return np.fft.irfftn(X, s=(n, n, n), axes=(0, 1, 2)) * float(n) ** 3

    def set_velocity(self, U, V, W) -> None:
        """main.c:249-251; the real velocity doubles as the stale one that
        the first stage of the first step reads (main.c:344)."""
        self.u = [np.array(a, dtype=np.float64) for a in (U, V, W)]
        self.uh = [np.fft.rfftn(a) for a in self.u]

    def diagnostics(self):
        """main.c:257-266: E and Omega over the half spectrum (no Hermitian
        weighting), long double sums scaled by invn3^2."""
        e = sum((x.real * x.real + x.imag * x.imag) for x in self.uh)
        E = np.sum(e.astype(np.longdouble))
        O = np.sum((self.kk * e).astype(np.longdouble))
        s = np.longdouble(self.invn3) * np.longdouble(self.invn3)
        return E * s, O * s

    def step(self, nu: float, dt: float, nsteps: int = 1) -> None:
        KX, KY, KZ, kk = self.KX, self.KY, self.KZ, self.kk
        for _ in range(nsteps):
            u0h = [x.copy() for x in self.uh]  # main.c:334-342
            u1h = [x.copy() for x in self.uh]
            for rk in range(4):
                if rk > 0:  # main.c:344-353 (stage 0 keeps the stale velocity)
                    self.u = [self.c2r(x) * self.invn3 for x in self.uh]
                Uh, Vh, Wh = self.uh
                # main.c:354-362
                oxh = 1j * (KY * Wh - KZ * Vh)
                oyh = 1j * (KZ * Uh - KX * Wh)
                ozh = 1j * (KX * Vh - KY * Uh)
                cu, cv, cw = (self.c2r(x) * self.invn3 for x in (oxh, oyh, ozh))  # :363-371
                U, V, W = self.u
                N = (V * cw - W * cv, W * cu - U * cw, U * cv - V * cu)  # :372-377
                dU, dV, dW = (np.fft.rfftn(x) for x in N)  # :378-380
                md = self.mask * dt  # :381-386
                dU, dV, dW = dU * md, dV * md, dW * md
                with np.errstate(invalid="ignore", divide="ignore"):  # :387-399
                    P = np.where(kk > 0, (dU * KX + dV * KY + dW * KZ) / kk, 0.0)
                dU = dU - (P * KX + nu * dt * kk * Uh)
                dV = dV - (P * KY + nu * dt * kk * Vh)
                dW = dW - (P * KZ + nu * dt * kk * Wh)
                d = (dU, dV, dW)
                if rk < 3:  # :400-407
                    self.uh = [u0h[f] + RK_B[rk] * d[f] for f in range(3)]
                u1h = [u1h[f] + RK_A[rk] * d[f] for f in range(3)]  # :408-413
            self.uh = u1h  # :415-422
