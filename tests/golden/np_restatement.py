"""Independent numpy restatement of the reference's hot path (test infrastructure).

Written from the Fortran a second time, in array-slice form (whole-array
expressions over the interior, like Fortran array sections), to cross-check
the C oracle in oracle/pf_oracle.c bit for bit on small grids.  Logs go
through math.log (glibc), the same libm the C oracle calls, so the two agree
exactly.  Arrays have shape (nz, ny, nx): memory order = Fortran (i fastest).

Sources followed: variaveis.f90:73-111 (noise), W0_E0.f90:10-31,
auxiliar.f90:12-42, entrada.f90:159-185, temp_body.inc:11-45,
phase_body.inc:14-198, equacao_campo_fase.f90:105-167, conc_body.inc:11-149,
concentracao_soluto.f90:78-124, diag_body.inc:8-22, principal.f90:93-226.
"""
from __future__ import annotations

import math

import numpy as np

M64 = (1 << 64) - 1


def pseudo_random_int(i: int, j: int, k: int, it: int, salt: int) -> int:
    h = (i * 2654435761 + j * 2246822519 + k * 3266489917 + it * 668265263 + salt * 374761393 + 1) & M64
    h ^= h >> 33
    h = (h * 0xFF51AFD7ED558CCD) & M64
    h ^= h >> 33
    h = (h * 0xC4CEB9FE1A85EC53) & M64
    h ^= h >> 33
    return h & 0x7FFFFFFFFFFFFFFF


def pseudo_random(i, j, k, it, salt) -> float:
    # int -> double is round-to-nearest (Python float() of an int rounds to nearest even)
    return float(pseudo_random_int(i, j, k, it, salt)) / float(0x7FFFFFFFFFFFFFFF)


def hash_grid(nx, ny, nz, it, salt) -> np.ndarray:
    """63-bit hashes of all 1-based cells, vectorised in uint64 (wrapping)."""
    k = np.arange(1, nz + 1, dtype=np.uint64)[:, None, None]
    j = np.arange(1, ny + 1, dtype=np.uint64)[None, :, None]
    i = np.arange(1, nx + 1, dtype=np.uint64)[None, None, :]
    with np.errstate(over="ignore"):
        h = (i * np.uint64(2654435761) + j * np.uint64(2246822519) + k * np.uint64(3266489917)
             + np.uint64(it) * np.uint64(668265263) + np.uint64(salt) * np.uint64(374761393) + np.uint64(1))
        h ^= h >> np.uint64(33)
        h *= np.uint64(0xFF51AFD7ED558CCD)
        h ^= h >> np.uint64(33)
        h *= np.uint64(0xC4CEB9FE1A85EC53)
        h ^= h >> np.uint64(33)
    return h & np.uint64(0x7FFFFFFFFFFFFFFF)


def ran_grid(nx, ny, nz, it) -> np.ndarray:
    """REAL(4) ran of phase_body.inc:184 for every cell."""
    h = hash_grid(nx, ny, nz, it, 1)
    r = h.astype(np.float64) / np.float64(9223372036854775808.0)
    return r.astype(np.float32)


def ruido_suave(i, j, k, it) -> float:
    LR, TR = 6, 20
    i0, j0, k0, tb = i // LR, j // LR, k // LR, it // TR
    fx, fy, fz = (i % LR) / float(LR), (j % LR) / float(LR), (k % LR) / float(LR)
    P = lambda a, b, c: pseudo_random(a, b, c, tb, 3)
    return ((1.0 - fz) * ((1.0 - fy) * ((1.0 - fx) * P(i0, j0, k0) + fx * P(i0 + 1, j0, k0))
                          + fy * ((1.0 - fx) * P(i0, j0 + 1, k0) + fx * P(i0 + 1, j0 + 1, k0)))
            + fz * ((1.0 - fy) * ((1.0 - fx) * P(i0, j0, k0 + 1) + fx * P(i0 + 1, j0, k0 + 1))
                    + fy * ((1.0 - fx) * P(i0, j0 + 1, k0 + 1) + fx * P(i0 + 1, j0 + 1, k0 + 1))))


def w0_e0(Lambda: float, ajuste: float, Sigma: float):
    step = float(np.float32(0.0000001))
    count = int((1.0 - 0.0 + step) / step)
    a_s = float(np.float32(ajuste) * np.float32(Sigma))
    eps = 0.0
    for n in range(count):
        W0 = ((1.5556349186104 / Lambda) * eps) * ((1.5556349186104 / Lambda) * eps)
        with np.errstate(divide="ignore"):
            E0 = float(np.float64(a_s * 4.24264068711929) / np.sqrt(np.float64(W0)))
        if abs(E0 - eps) < 1e-5:
            return W0, E0, n + 1
        eps = eps + step
    return W0, E0, count


def auxiliar(p, TP, Cs_eq, Cl_eq, E0, W0) -> float:
    F = 0.0
    phi = 0.11
    while True:
        h = phi * phi * (3.0 - 2.0 * phi)
        f1 = phi * (1.0 - phi)
        F = F + (h * (1.0 - h)) / (((1.0 - h) * Cl_eq * (1.0 - Cl_eq) + h * Cs_eq * (1.0 - Cs_eq)) * f1)
        phi = phi + 0.01
        if not phi <= 0.8999:
            break
    I = (float(np.float32(0.01)) / 2.0) * (float(np.float32(54.39180136)) + 2.0 * F + 234.073053)
    Qsi = p.R * TP * (1.0 / p.Vm) * (Cl_eq - Cs_eq) * (Cl_eq - Cs_eq) * I
    omk = float(np.float32(1.0) - np.float32(p.Ke))
    Inv = (E0 * E0 / float(np.float32(p.Sigma))) * ((float(np.float32(p.Beta)) * p.R * TP * omk / (p.Vm * p.Me))
                                                    + (E0 * Qsi / (p.D_liq * math.sqrt(2.0 * W0))))
    return float(np.float32(p.ajuste)) * 1.0 / Inv


_vlog = np.vectorize(math.log, otypes=[np.float64])


class NpRef:
    def __init__(self, g, p):
        self.nx, self.ny, self.nz = g.nx, g.ny, g.nz
        self.dx, self.dy, self.dz = g.dx, g.dy, g.dz
        self.p = p
        self.Ke = float(np.float32(p.Ke))
        dx = g.dx
        self.dt = (dx * dx) / (7.5 * p.D_liq)
        r = self.dt / ((dx * dx) / (5.0 * p.D_liq))
        self.AAA = p.AAA * r if p.ruido_tipo == 0 else p.AAA * math.sqrt(r)
        self.W0, self.E0, _ = w0_e0(p.Thin_Interface * dx, p.ajuste, p.Sigma)
        self.TP = p.T0 if p.taxa_resfr > 0.0 else p.TP
        self.M0 = p.M0
        self.it = 0
        shp = (g.nz, g.ny, g.nx)
        self.phi_old = np.zeros(shp); self.phi_new = np.zeros(shp)
        self.c_old = np.zeros(shp); self.c_new = np.zeros(shp)
        self.T_old = np.zeros(shp); self.T_new = np.zeros(shp)
        self.dpp = np.zeros(shp)

    def load_state(self, st):
        self.phi_old = st["phi"].copy()
        self.c_old = st["c"].copy()
        self.T_old = st["T"].copy()
        self.dpp = st.get("dpp", np.zeros_like(st["phi"])).copy()

    # -- temperatura --
    def temperatura(self):
        p = self.p
        T, phi = self.T_old, self.phi_old
        self.T_new = T.copy()
        s = (slice(1, -1),) * 3
        sh = lambda dk, dj, di: (slice(1 + dk, self.nz - 1 + dk), slice(1 + dj, self.ny - 1 + dj),
                                 slice(1 + di, self.nx - 1 + di))
        TE, TW = T[sh(0, 0, 1)], T[sh(0, 0, -1)]
        TN, TS = T[sh(0, 1, 0)], T[sh(0, -1, 0)]
        TT, TB = T[sh(1, 0, 0)], T[sh(-1, 0, 0)]
        PP = phi[s]
        if p.h_quintico == 1:
            hl = 30.0 * PP * PP * (1.0 - PP) * (1.0 - PP)
        else:
            hl = 2.0 * PP * (3.0 - 2.0 * PP) - 2.0 * PP * PP
        FONTE = (p.delta_H / p.Cp_s) * hl * self.dpp[s]
        TP = self.TP
        dx, dy, dz = self.dx, self.dy, self.dz
        self.T_new[s] = p.D * self.dt * (((TE - 2.0 * TP + TW) / (dx * dx)) + ((TN - 2.0 * TP + TS) / (dy * dy))
                                         + ((TT - 2.0 * TP + TB) / (dz * dz))) + FONTE + TP

    # -- equacao_campo_fase --
    def equacao_campo_fase(self):
        p, Ke = self.p, self.Ke
        E0, DE, w0 = self.E0, p.DELTA_EPSLON, self.W0
        dx, dy, dz = self.dx, self.dy, self.dz
        TP = self.TP
        self.Cs_eq = ((p.Tm - TP) * Ke) / p.Me
        self.Cl_eq = (p.Tm - TP) / p.Me
        po = self.phi_old
        pn = po.copy()
        nz, ny, nx = po.shape

        def P(di, dj, dk):
            return po[2 + dk:nz - 2 + dk, 2 + dj:ny - 2 + dj, 2 + di:nx - 2 + di]

        PP = P(0, 0, 0)
        PN, PS, PE, PW, PT, PB = P(0, 1, 0), P(0, -1, 0), P(1, 0, 0), P(-1, 0, 0), P(0, 0, 1), P(0, 0, -1)
        PNE, PSE, PNW, PSW = P(1, 1, 0), P(1, -1, 0), P(-1, 1, 0), P(-1, -1, 0)
        PNT, PNB, PST, PSB = P(0, 1, 1), P(0, 1, -1), P(0, -1, 1), P(0, -1, -1)
        PET, PEB, PWT, PWB = P(1, 0, 1), P(1, 0, -1), P(-1, 0, 1), P(-1, 0, -1)
        small = 1e-23
        K = 16.0 * E0 * DE

        def node(gx, gy, gz):
            Q = gx ** 2 + gy ** 2 + gz ** 2 + small
            S4 = (gx * gx) * (gx * gx) + (gy * gy) * (gy * gy) + (gz * gz) * (gz * gz)
            eps = E0 * (1.0 + DE * (4.0 * S4 / (Q * Q) - 3.0))
            exy = K * eps * gx * gy * (gx * gx - gy * gy) / (Q * Q)
            eyz = K * eps * gy * gz * (gy * gy - gz * gz) / (Q * Q)
            ezx = K * eps * gz * gx * (gz * gz - gx * gx) / (Q * Q)
            return eps, exy, eyz, ezx

        epsE, exyE, _, ezxE = node((P(2, 0, 0) - PP) * 0.5 / dx, (P(1, 1, 0) - P(1, -1, 0)) * 0.5 / dy,
                                   (P(1, 0, 1) - P(1, 0, -1)) * 0.5 / dz)
        epsW, exyW, _, ezxW = node((PP - P(-2, 0, 0)) * 0.5 / dx, (P(-1, 1, 0) - P(-1, -1, 0)) * 0.5 / dy,
                                   (P(-1, 0, 1) - P(-1, 0, -1)) * 0.5 / dz)
        epsN, exyN, eyzN, _ = node((P(1, 1, 0) - P(-1, 1, 0)) * 0.5 / dx, (P(0, 2, 0) - PP) * 0.5 / dy,
                                   (P(0, 1, 1) - P(0, 1, -1)) * 0.5 / dz)
        epsS, exyS, eyzS, _ = node((P(1, -1, 0) - P(-1, -1, 0)) * 0.5 / dx, (PP - P(0, -2, 0)) * 0.5 / dy,
                                   (P(0, -1, 1) - P(0, -1, -1)) * 0.5 / dz)
        epsT, _, eyzT, ezxT = node((P(1, 0, 1) - P(-1, 0, 1)) * 0.5 / dx, (P(0, 1, 1) - P(0, -1, 1)) * 0.5 / dy,
                                   (P(0, 0, 2) - PP) * 0.5 / dz)
        epsB, _, eyzB, ezxB = node((P(1, 0, -1) - P(-1, 0, -1)) * 0.5 / dx, (P(0, 1, -1) - P(0, -1, -1)) * 0.5 / dy,
                                   (PP - P(0, 0, -2)) * 0.5 / dz)
        AA = ((epsE * epsE * (PE - PP) + epsW * epsW * (PW - PP)) / (dx * dx)
              + (epsN * epsN * (PN - PP) + epsS * epsS * (PS - PP)) / (dy * dy)
              + (epsT * epsT * (PT - PP) + epsB * epsB * (PB - PP)) / (dz * dz))
        cxy, cyz, czx = 0.25 / (dx * dy), 0.25 / (dy * dz), 0.25 / (dz * dx)
        Cxy = (cxy * (PNE * (-exyN - (-exyE)) + PSE * (-exyE - (-exyS)) + PNW * (-exyW - (-exyN)) + PSW * (-exyS - (-exyW)))
               + PN * cxy * (-exyW - (-exyE)) + PS * cxy * (-exyE - (-exyW))
               + PE * cxy * (-exyN - (-exyS)) + PW * cxy * (-exyS - (-exyN)))
        Cyz = (cyz * (PNT * (-eyzT - (-eyzN)) + PNB * (-eyzN - (-eyzB)) + PST * (-eyzS - (-eyzT)) + PSB * (-eyzB - (-eyzS)))
               + PT * cyz * (-eyzS - (-eyzN)) + PB * cyz * (-eyzN - (-eyzS))
               + PN * cyz * (-eyzT - (-eyzB)) + PS * cyz * (-eyzB - (-eyzT)))
        Czx = (czx * (PET * (-ezxE - (-ezxT)) + PWT * (-ezxT - (-ezxW)) + PEB * (-ezxB - (-ezxE)) + PWB * (-ezxW - (-ezxB)))
               + PE * czx * (-ezxB - (-ezxT)) + PW * czx * (-ezxT - (-ezxB))
               + PT * czx * (-ezxE - (-ezxW)) + PB * czx * (-ezxW - (-ezxE)))
        AA = AA + Cxy + Cyz + Czx
        g_l = 2.0 * PP * (1.0 - PP) * (1.0 - PP) - 2.0 * PP * PP * (1.0 - PP)
        CPP = self.c_old[2:nz - 2, 2:ny - 2, 2:nx - 2]
        if p.h_quintico == 1:
            h_l = 30.0 * PP * PP * (1.0 - PP) * (1.0 - PP)
            h = PP * PP * PP * (10.0 - 15.0 * PP + 6.0 * PP * PP)
        else:
            h_l = 2.0 * PP * (3.0 - 2.0 * PP) - 2.0 * PP * PP
            h = PP * PP * (3.0 - 2.0 * PP)
        CLP = CPP / (Ke * h + (1.0 - h))
        CSP = Ke * CPP / (Ke * h + (1.0 - h))
        arg = np.abs(((1.0 - self.Cs_eq) * (1.0 - CLP)) / ((1.0 - self.Cl_eq) * (1.0 - CSP)))
        GG = (-(w0 * g_l)) + (p.R * TP / p.Vm) * h_l * _vlog(arg)
        if p.ruido_tipo == 2:
            ran = np.empty(PP.shape, dtype=np.float32)
            for kk in range(PP.shape[0]):
                for jj in range(PP.shape[1]):
                    for ii in range(PP.shape[2]):
                        ran[kk, jj, ii] = np.float32(ruido_suave(ii + 3, jj + 3, kk + 3, self.it))
        else:
            ran = ran_grid(nx, ny, nz, self.it)[2:nz - 2, 2:ny - 2, 2:nx - 2]
        ran = ran.astype(np.float64)
        if p.ruido_tipo == 0:
            ruidos = ran * self.AAA * 16.0 * (PP * PP) * ((1.0 - PP) * (1.0 - PP))
        else:
            ruidos = (2.0 * ran - 1.0) * self.AAA * 16.0 * (PP * PP) * ((1.0 - PP) * (1.0 - PP))
        PPNEW = PP + (self.M0 * self.dt) * (AA + GG) + ruidos
        self.dpp[2:nz - 2, 2:ny - 2, 2:nx - 2] = PPNEW - PP
        t = np.where(PPNEW < 1.0, PPNEW, 1.0)
        pn[2:nz - 2, 2:ny - 2, 2:nx - 2] = np.where(t > 0.0, t, 0.0)
        # boundary decoration, array sections in order (equacao_campo_fase.f90:151-167)
        pn[:, 0, :] = pn[:, 1, :]
        pn[:, 1, :] = pn[:, 2, :]
        pn[:, ny - 1, :] = pn[:, ny - 2, :]
        pn[:, ny - 2, :] = pn[:, ny - 3, :]
        pn[:, :, 0] = pn[:, :, 1]
        pn[:, :, 1] = pn[:, :, 2]
        pn[:, :, nx - 1] = pn[:, :, nx - 2]
        pn[:, :, nx - 2] = pn[:, :, nx - 3]
        pn[0, :, :] = pn[1, :, :]
        pn[1, :, :] = pn[2, :, :]
        pn[nz - 1, :, :] = pn[nz - 2, :, :]
        pn[nz - 2, :, :] = pn[nz - 3, :, :]
        self.phi_new = pn

    # -- concentracao_soluto --
    def concentracao_soluto(self):
        p, Ke = self.p, self.Ke
        po, co = self.phi_old, self.c_old
        nz, ny, nx = po.shape
        cn = co.copy()

        def S(a, dk, dj, di):
            return a[1 + dk:nz - 1 + dk, 1 + dj:ny - 1 + dj, 1 + di:nx - 1 + di]

        pts = {"P": (0, 0, 0), "S": (0, -1, 0), "N": (0, 1, 0), "W": (0, 0, -1), "E": (0, 0, 1),
               "T": (1, 0, 0), "B": (-1, 0, 0)}
        CS, CL, H = {}, {}, {}
        for n, (dk, dj, di) in pts.items():
            PX, CX = S(po, dk, dj, di), S(co, dk, dj, di)
            if p.h_quintico == 1:
                hX = (PX * PX * PX) * (10.0 - (15.0 * PX) + (6.0 * (PX * PX)))
            else:
                hX = PX * PX * (3.0 - 2.0 * PX)
            H[n] = hX
            CS[n] = (Ke * CX) / ((Ke * hX) + (1.0 - hX))
            CL[n] = CX / (Ke * hX + (1.0 - hX))
        PP = S(po, 0, 0, 0)
        Dc = np.where(PP <= 0.95, p.D_liq, p.D_sol)
        G = {n: Dc * ((1.0 - H[n]) * CL[n] * (1.0 - CL[n]) + H[n] * CS[n] * (1.0 - CS[n])) for n in pts}
        Gs = 2.0 / ((1.0 / G["P"]) + (1.0 / G["S"]))
        Gn = 2.0 / ((1.0 / G["N"]) + (1.0 / G["P"]))
        Gw = 2.0 / ((1.0 / G["P"]) + (1.0 / G["W"]))
        Ge = 2.0 / ((1.0 / G["E"]) + (1.0 / G["P"]))
        Gt = 2.0 / ((1.0 / G["T"]) + (1.0 / G["P"]))
        Gb = 2.0 / ((1.0 / G["P"]) + (1.0 / G["B"]))
        mu = {n: _vlog(CL[n] / (1.0 - CL[n])) for n in pts}
        iX, iY, iZ = 1.0 / (self.dx * self.dx), 1.0 / (self.dy * self.dy), 1.0 / (self.dz * self.dz)
        cnew = (Ge * iX * (mu["E"] - mu["P"]) - Gw * iX * (mu["P"] - mu["W"]) + Gn * iY * (mu["N"] - mu["P"])
                - Gs * iY * (mu["P"] - mu["S"]) + Gt * iZ * (mu["T"] - mu["P"]) - Gb * iZ * (mu["P"] - mu["B"])) \
            * self.dt + S(co, 0, 0, 0)
        cn[1:nz - 1, 1:ny - 1, 1:nx - 1] = cnew
        self.c_old = cn.copy()
        co2 = self.c_old
        cn[:, 0, :] = co2[:, 1, :]
        cn[:, ny - 1, :] = co2[:, ny - 2, :]
        cn[:, :, 0] = co2[:, :, 1]
        cn[:, :, nx - 1] = co2[:, :, nx - 2]
        cn[0, :, :] = co2[1, :, :]
        cn[nz - 1, :, :] = co2[nz - 2, :, :]
        self.c_new = cn

    def step(self, n=1):
        p = self.p
        for _ in range(n):
            self.it += 1
            self.temperatura()
            if p.taxa_resfr > 0.0:
                self.TP = p.T0 - p.taxa_resfr * self.dt * self.it
            for sw in range(1, max(1, p.n_varreduras) + 1):
                if sw > 1:
                    self.phi_old = self.phi_new.copy()
                self.equacao_campo_fase()
            self.concentracao_soluto()
            self.M0 = auxiliar(p, self.TP, self.Cs_eq, self.Cl_eq, self.E0, self.W0)
            self.phi_old = self.phi_new.copy()
            self.T_old = self.T_new.copy()
            self.c_old = self.c_new.copy()

    def fields(self):
        return {"phi": self.phi_old, "c": self.c_old, "T": self.T_old, "dpp": self.dpp}
