"""Independent numpy restatement of the reference's quantitative Karma model
(test infrastructure).

Written from karma/karma3d.f90 a second time, in array-section form over
ghost-padded arrays of shape (nz+2, ny+2, nx+2) (memory order = Fortran, i
fastest), to cross-check the C oracle in oracle/karma_oracle.c bit for bit.
Fortran evaluation order: left to right, x**2 = x*x, x**3 = (x*x)*x,
x**4 = (x*x)*(x*x); numpy applies each binary operation once per element with
IEEE rounding, so the result matches a C loop compiled without contraction.

Sources followed: karma3d.f90:37-49 (fluxn), :52-67 (ruido), :118 (D),
:160-207 (phase equation), :209-276 (U equation), :279-287 (advance),
:290-296 (tip), :318-339 (espelho).
"""
from __future__ import annotations

import numpy as np

A2 = 0.6267
AT = 0.35355339059327373
M64 = (1 << 64) - 1


def ruido_grid(nx, ny, nz, it):
    """ruido(i, j, k, it) for every interior cell, shape (nz, ny, nx)."""
    k, j, i = np.meshgrid(np.arange(1, nz + 1, dtype=np.uint64), np.arange(1, ny + 1, dtype=np.uint64),
                          np.arange(1, nx + 1, dtype=np.uint64), indexing="ij")
    with np.errstate(over="ignore"):
        h = (i * np.uint64(2654435761) + j * np.uint64(2246822519) + k * np.uint64(3266489917)
             + np.uint64(it) * np.uint64(668265263) + np.uint64(1))
        h ^= h >> np.uint64(33)
        h *= np.uint64(0xFF51AFD7ED558CCD)
        h ^= h >> np.uint64(33)
        h *= np.uint64(0xC4CEB9FE1A85EC53)
        h ^= h >> np.uint64(33)
    m = (h & np.uint64(0x7FFFFFFFFFFFFFFF)).astype(np.int64).astype(np.float64)
    return 2.0 * m / 9223372036854775808.0 - 1.0


def espelho(f):
    f[:, :, 0] = f[:, :, 1]
    f[:, :, -1] = f[:, :, -2]
    f[:, 0, :] = f[:, 1, :]
    f[:, -1, :] = f[:, -2, :]
    f[0, :, :] = f[1, :, :]
    f[-1, :, :] = f[-2, :, :]


def fluxn(g1, g2, g3, eps4):
    g2s = g1 * g1 + g2 * g2 + g3 * g3
    small = g2s < 1.0e-20
    safe = np.where(small, 1.0, g2s)
    a, b, c = g1 * g1, g2 * g2, g3 * g3
    s4 = a * a + b * b + c * c
    as_ = 1.0 - 3.0 * eps4 + 4.0 * eps4 * s4 / (safe * safe)
    jn = as_ * (as_ * g1 + 16.0 * eps4 * ((g1 * g1) * g1 - g1 * s4 / safe) / safe)
    t = 1.0 - 3.0 * eps4
    return np.where(small, (t * t) * g1, jn)


class Karma:
    """Ghost-padded state and the time loop of karma3d.f90."""

    def __init__(self, nx, ny, nz, lambda_, eps4, dx, dt, Fnoise, k):
        self.n = (nx, ny, nz)
        self.lam, self.eps4, self.dx, self.dt, self.Fn, self.k = lambda_, eps4, dx, dt, Fnoise, k
        self.D = A2 * lambda_
        shp = (nz + 2, ny + 2, nx + 2)
        self.phi = np.zeros(shp)
        self.U = np.zeros(shp)
        self.dphi = np.zeros(shp)
        self.it = 0

    def set(self, phi, U):
        self.phi[1:-1, 1:-1, 1:-1] = phi
        self.U[1:-1, 1:-1, 1:-1] = U

    def get(self):
        s = (slice(1, -1),) * 3
        return self.phi[s].copy(), self.U[s].copy(), self.dphi[s].copy()

    def step(self, n=1):
        for _ in range(n):
            self._one()

    def _one(self):
        self.it += 1
        nx, ny, nz = self.n
        idx = 1.0 / self.dx
        eps4, lam, dt, k, D = self.eps4, self.lam, self.dt, self.k, self.D
        phi, U, dphi = self.phi, self.U, self.dphi
        espelho(phi)
        espelho(U)

        def P(di, dj, dk):   # phi(i+di, j+dj, kk+dk) over the interior
            return phi[1 + dk:nz + 1 + dk, 1 + dj:ny + 1 + dj, 1 + di:nx + 1 + di]

        def Uo(di, dj, dk):
            return U[1 + dk:nz + 1 + dk, 1 + dj:ny + 1 + dj, 1 + di:nx + 1 + di]

        def Do(di, dj, dk):
            return dphi[1 + dk:nz + 1 + dk, 1 + dj:ny + 1 + dj, 1 + di:nx + 1 + di]

        q = 0.25 * idx
        pp = P(0, 0, 0)
        Jxp = fluxn((P(1, 0, 0) - pp) * idx, q * (P(0, 1, 0) + P(1, 1, 0) - P(0, -1, 0) - P(1, -1, 0)),
                    q * (P(0, 0, 1) + P(1, 0, 1) - P(0, 0, -1) - P(1, 0, -1)), eps4)
        Jxm = fluxn((pp - P(-1, 0, 0)) * idx, q * (P(0, 1, 0) + P(-1, 1, 0) - P(0, -1, 0) - P(-1, -1, 0)),
                    q * (P(0, 0, 1) + P(-1, 0, 1) - P(0, 0, -1) - P(-1, 0, -1)), eps4)
        Jyp = fluxn((P(0, 1, 0) - pp) * idx, q * (P(1, 0, 0) + P(1, 1, 0) - P(-1, 0, 0) - P(-1, 1, 0)),
                    q * (P(0, 0, 1) + P(0, 1, 1) - P(0, 0, -1) - P(0, 1, -1)), eps4)
        Jym = fluxn((pp - P(0, -1, 0)) * idx, q * (P(1, 0, 0) + P(1, -1, 0) - P(-1, 0, 0) - P(-1, -1, 0)),
                    q * (P(0, 0, 1) + P(0, -1, 1) - P(0, 0, -1) - P(0, -1, -1)), eps4)
        Jzp = fluxn((P(0, 0, 1) - pp) * idx, q * (P(1, 0, 0) + P(1, 0, 1) - P(-1, 0, 0) - P(-1, 0, 1)),
                    q * (P(0, 1, 0) + P(0, 1, 1) - P(0, -1, 0) - P(0, -1, 1)), eps4)
        Jzm = fluxn((pp - P(0, 0, -1)) * idx, q * (P(1, 0, 0) + P(1, 0, -1) - P(-1, 0, 0) - P(-1, 0, -1)),
                    q * (P(0, 1, 0) + P(0, 1, -1) - P(0, -1, 0) - P(0, -1, -1)), eps4)
        divJ = (Jxp - Jxm + Jyp - Jym + Jzp - Jzm) * idx
        h = 0.5 * idx
        g1 = h * (P(1, 0, 0) - P(-1, 0, 0))
        g2 = h * (P(0, 1, 0) - P(0, -1, 0))
        g3 = h * (P(0, 0, 1) - P(0, 0, -1))
        gm = g1 * g1 + g2 * g2 + g3 * g3
        big = gm > 1.0e-20
        safe = np.where(big, gm, 1.0)
        a, b, c = g1 * g1, g2 * g2, g3 * g3
        s4 = (a * a + b * b + c * c) / (safe * safe)
        t = 1.0 - 3.0 * eps4 + 4.0 * eps4 * s4
        t0 = 1.0 - 3.0 * eps4
        as2 = np.where(big, t * t, t0 * t0)
        om = 1.0 - pp * pp
        d = ((divJ + pp - (pp * pp) * pp - lam * (om * om) * Uo(0, 0, 0)) / as2
             + self.Fn * ruido_grid(nx, ny, nz, self.it) * (1.0 - pp * pp) / np.sqrt(dt))
        dphi[1:-1, 1:-1, 1:-1] = d
        phin = pp + dt * d
        espelho(dphi)

        uc, dc = Uo(0, 0, 0), Do(0, 0, 0)

        def face(sign, axis):
            """flux through the face of the interior cells in direction sign * axis"""
            e = [0, 0, 0]
            e[axis] = sign
            nb = P(*e)
            normal = (nb - pp) * idx if sign > 0 else (pp - nb) * idx
            tang = []
            for ax in range(3):
                if ax == axis:
                    continue
                up = [0, 0, 0]
                up[ax] = 1
                dn = [0, 0, 0]
                dn[ax] = -1
                upn = list(up)
                upn[axis] = sign
                dnn = list(dn)
                dnn[axis] = sign
                tang.append(q * (P(*up) + P(*upn) - P(*dn) - P(*dnn)))
            g = [None, None, None]
            g[axis] = normal
            others = [ax for ax in range(3) if ax != axis]
            g[others[0]], g[others[1]] = tang
            gmag = np.sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2])
            qf = 0.25 * (2.0 - pp - nb)
            cf = 0.5 * ((1.0 + (1.0 - k) * uc) * dc + (1.0 + (1.0 - k) * Uo(*e)) * Do(*e))
            du = (Uo(*e) - uc) if sign > 0 else (uc - Uo(*e))
            F = D * qf * du * idx
            safe_g = np.where(gmag > 1.0e-10, gmag, 1.0)
            return np.where(gmag > 1.0e-10, F + AT * cf * g[axis] / safe_g, F)

        Fxp, Fxm = face(1, 0), face(-1, 0)
        Fyp, Fym = face(1, 1), face(-1, 1)
        Fzp, Fzm = face(1, 2), face(-1, 2)
        Au = 0.5 * (1.0 + k) - 0.5 * (1.0 - k) * pp
        rhsU = (Fxp - Fxm + Fyp - Fym + Fzp - Fzm) * idx + 0.5 * (1.0 + (1.0 - k) * uc) * dc
        Un = uc + dt * rhsU / Au
        phi[1:-1, 1:-1, 1:-1] = np.maximum(-1.0, np.minimum(1.0, phin))
        U[1:-1, 1:-1, 1:-1] = Un

    def tip(self):
        nx, ny, nz = self.n
        tx = max([i for i in range(1, nx + 1) if self.phi[1, 1, i] > 0.0], default=0)
        nd = min(nx, ny, nz)
        td = max([i for i in range(1, nd + 1) if self.phi[i, i, i] > 0.0], default=0)
        return tx, td


def seed_state(nx, ny, nz, dx, R0, Omega):
    """karma3d.f90:130-144: an eighth of a sphere at the corner, phi =
    -tanh((r - R0)/sqrt(2)) at the cell centres (i - 1/2) dx, U = -Omega
    (interior cells, shape (nz, ny, nx))."""
    k, j, i = np.meshgrid(np.arange(1, nz + 1), np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
    x, y, z = (i - 0.5) * dx, (j - 0.5) * dx, (k - 0.5) * dx
    r = np.sqrt(x * x + y * y + z * z)
    return -np.tanh((r - R0) / np.sqrt(2.0)), np.full(r.shape, -Omega)
