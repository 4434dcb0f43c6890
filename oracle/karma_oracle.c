/*
 * karma_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) of the quantitative
 * Karma model of the reference (karma/karma3d.f90): phase field phi in [-1,1]
 * and dimensionless supersaturation U, cubic anisotropy, anti-trapping
 * current, mirror ghost cells on every face.  Imported only by tests/ and the
 * CPU leg of the benchmark, never by the product.
 *
 * Restated statement by statement from karma3d.f90 with Fortran's
 * left-to-right evaluation: x**2 = x*x, x**3 = (x*x)*x, x**4 = (x*x)*(x*x),
 * divisions and square roots kept, no FMA contraction (-ffp-contract=off).
 * Arrays carry the reference's ghost layer: index 0..n+1 per axis, i fastest.
 * Pinned against the reference's own output: no Fortran compiler exists
 * here, but the reference's run log records the tip of its run3 (200^3,
 * Fnoise = 0.01) every 5000 steps to 45 000 (registro_runs.md:99-107), and
 * this restatement, stepped from the program's seed, prints all nine
 * recorded pairs of ponta_eixo / ponta_diag (oracle/karma_record_check.py;
 * about 100 minutes on 8 host threads).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "karma_oracle.h"

#define KA1 0.8839
#define KA2 0.6267
#define KAT 0.35355339059327373   /* 1/(2 sqrt 2), karma3d.f90:99 */

static inline size_t at3(const orc_karma* s, int i, int j, int k)
{
    return (size_t)i + (size_t)(s->nx + 2) * ((size_t)j + (size_t)(s->ny + 2) * (size_t)k);
}

/* karma3d.f90:37-49 (fluxn) */
static double fluxn(double g1, double g2, double g3, double eps4)
{
    double g2s = g1 * g1 + g2 * g2 + g3 * g3;
    if (g2s < 1.e-20) {
        double t = 1.0 - 3.0 * eps4;
        return (t * t) * g1;
    }
    double q1 = g1 * g1, q2 = g2 * g2, q3 = g3 * g3;
    double s4 = q1 * q1 + q2 * q2 + q3 * q3;
    double as = 1.0 - 3.0 * eps4 + 4.0 * eps4 * s4 / (g2s * g2s);
    return as * (as * g1 + 16.0 * eps4 * ((g1 * g1) * g1 - g1 * s4 / g2s) / g2s);
}

/* karma3d.f90:52-67 (ruido): the hash of variaveis.f90 without a salt term,
   mapped to [-1, 1) */
double orc_karma_ruido(int i, int j, int k, int it)
{
    uint64_t h = (uint64_t)(int64_t)i * 2654435761ull + (uint64_t)(int64_t)j * 2246822519ull +
                 (uint64_t)(int64_t)k * 3266489917ull + (uint64_t)(int64_t)it * 668265263ull + 1ull;
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    const double m = (double)(int64_t)(h & 0x7fffffffffffffffull);
    return 2.0 * m / 9223372036854775808.0 - 1.0;   /* real(MASK63,8) rounds to 2^63 */
}

orc_karma* orc_karma_create(int nx, int ny, int nz, double lambda, double eps4, double dx, double dt, double Fnoise,
                            double k)
{
    orc_karma* s = (orc_karma*)calloc(1, sizeof(orc_karma));
    s->nx = nx;
    s->ny = ny;
    s->nz = nz;
    s->lambda = lambda;
    s->eps4 = eps4;
    s->dx = dx;
    s->dt = dt;
    s->Fnoise = Fnoise;
    s->k = k;
    s->D = KA2 * lambda;   /* karma3d.f90:118 */
    size_t n = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    s->phi = (double*)calloc(n, sizeof(double));
    s->phin = (double*)calloc(n, sizeof(double));
    s->U = (double*)calloc(n, sizeof(double));
    s->Un = (double*)calloc(n, sizeof(double));
    s->dphi = (double*)calloc(n, sizeof(double));
    return s;
}

void orc_karma_destroy(orc_karma* s)
{
    if (!s) return;
    free(s->phi);
    free(s->phin);
    free(s->U);
    free(s->Un);
    free(s->dphi);
    free(s);
}

/* interior values (nx*ny*nz, i fastest) in / out */
void orc_karma_set(orc_karma* s, const double* phi, const double* U)
{
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                size_t q = (size_t)(i - 1) + (size_t)s->nx * ((size_t)(j - 1) + (size_t)s->ny * (size_t)(k - 1));
                s->phi[at3(s, i, j, k)] = phi[q];
                s->U[at3(s, i, j, k)] = U[q];
            }
}

void orc_karma_get(const orc_karma* s, double* phi, double* U, double* dphi)
{
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                size_t q = (size_t)(i - 1) + (size_t)s->nx * ((size_t)(j - 1) + (size_t)s->ny * (size_t)(k - 1));
                if (phi) phi[q] = s->phi[at3(s, i, j, k)];
                if (U) U[q] = s->U[at3(s, i, j, k)];
                if (dphi) dphi[q] = s->dphi[at3(s, i, j, k)];
            }
}

/* karma3d.f90:318-339 (espelho): x faces, then y, then z, over the full
   ghost-extended ranges */
static void espelho(orc_karma* s, double* f)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    for (int b = 0; b <= nz + 1; ++b)
        for (int a = 0; a <= ny + 1; ++a) {
            f[at3(s, 0, a, b)] = f[at3(s, 1, a, b)];
            f[at3(s, nx + 1, a, b)] = f[at3(s, nx, a, b)];
        }
    for (int b = 0; b <= nz + 1; ++b)
        for (int a = 0; a <= nx + 1; ++a) {
            f[at3(s, a, 0, b)] = f[at3(s, a, 1, b)];
            f[at3(s, a, ny + 1, b)] = f[at3(s, a, ny, b)];
        }
    for (int b = 0; b <= ny + 1; ++b)
        for (int a = 0; a <= nx + 1; ++a) {
            f[at3(s, a, b, 0)] = f[at3(s, a, b, 1)];
            f[at3(s, a, b, nz + 1)] = f[at3(s, a, b, nz)];
        }
}

/* one iteration of karma3d.f90:160-295 (it = s->it + 1) */
static void karma_one(orc_karma* s)
{
    const int it = ++s->it;
    const double idx = 1.0 / s->dx;
    const double eps4 = s->eps4, lambda = s->lambda, dt = s->dt, Fnoise = s->Fnoise, k = s->k, D = s->D;
    double* phi = s->phi;
    double* U = s->U;
    double* dphi = s->dphi;
#define P(a, b, c) phi[at3(s, (a), (b), (c))]
#define UU(a, b, c) U[at3(s, (a), (b), (c))]
#define DP(a, b, c) dphi[at3(s, (a), (b), (c))]
    espelho(s, phi);
    espelho(s, U);

    /* phase equation, karma3d.f90:166-207 */
#pragma omp parallel for collapse(2) schedule(static)
    for (int kk = 1; kk <= s->nz; ++kk)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                const double pp = P(i, j, kk);
                const double q = 0.25 * idx;
                double Jxp = fluxn((P(i + 1, j, kk) - pp) * idx,
                                   q * (P(i, j + 1, kk) + P(i + 1, j + 1, kk) - P(i, j - 1, kk) - P(i + 1, j - 1, kk)),
                                   q * (P(i, j, kk + 1) + P(i + 1, j, kk + 1) - P(i, j, kk - 1) - P(i + 1, j, kk - 1)),
                                   eps4);
                double Jxm = fluxn((pp - P(i - 1, j, kk)) * idx,
                                   q * (P(i, j + 1, kk) + P(i - 1, j + 1, kk) - P(i, j - 1, kk) - P(i - 1, j - 1, kk)),
                                   q * (P(i, j, kk + 1) + P(i - 1, j, kk + 1) - P(i, j, kk - 1) - P(i - 1, j, kk - 1)),
                                   eps4);
                double Jyp = fluxn((P(i, j + 1, kk) - pp) * idx,
                                   q * (P(i + 1, j, kk) + P(i + 1, j + 1, kk) - P(i - 1, j, kk) - P(i - 1, j + 1, kk)),
                                   q * (P(i, j, kk + 1) + P(i, j + 1, kk + 1) - P(i, j, kk - 1) - P(i, j + 1, kk - 1)),
                                   eps4);
                double Jym = fluxn((pp - P(i, j - 1, kk)) * idx,
                                   q * (P(i + 1, j, kk) + P(i + 1, j - 1, kk) - P(i - 1, j, kk) - P(i - 1, j - 1, kk)),
                                   q * (P(i, j, kk + 1) + P(i, j - 1, kk + 1) - P(i, j, kk - 1) - P(i, j - 1, kk - 1)),
                                   eps4);
                double Jzp = fluxn((P(i, j, kk + 1) - pp) * idx,
                                   q * (P(i + 1, j, kk) + P(i + 1, j, kk + 1) - P(i - 1, j, kk) - P(i - 1, j, kk + 1)),
                                   q * (P(i, j + 1, kk) + P(i, j + 1, kk + 1) - P(i, j - 1, kk) - P(i, j - 1, kk + 1)),
                                   eps4);
                double Jzm = fluxn((pp - P(i, j, kk - 1)) * idx,
                                   q * (P(i + 1, j, kk) + P(i + 1, j, kk - 1) - P(i - 1, j, kk) - P(i - 1, j, kk - 1)),
                                   q * (P(i, j + 1, kk) + P(i, j + 1, kk - 1) - P(i, j - 1, kk) - P(i, j - 1, kk - 1)),
                                   eps4);
                const double divJ = (Jxp - Jxm + Jyp - Jym + Jzp - Jzm) * idx;
                const double h = 0.5 * idx;
                const double g1 = h * (P(i + 1, j, kk) - P(i - 1, j, kk));
                const double g2 = h * (P(i, j + 1, kk) - P(i, j - 1, kk));
                const double g3 = h * (P(i, j, kk + 1) - P(i, j, kk - 1));
                const double gm = g1 * g1 + g2 * g2 + g3 * g3;
                double as2;
                if (gm > 1.e-20) {
                    const double q1 = g1 * g1, q2 = g2 * g2, q3 = g3 * g3;
                    const double s4 = (q1 * q1 + q2 * q2 + q3 * q3) / (gm * gm);
                    const double t = 1.0 - 3.0 * eps4 + 4.0 * eps4 * s4;
                    as2 = t * t;
                } else {
                    const double t = 1.0 - 3.0 * eps4;
                    as2 = t * t;
                }
                const double om = 1.0 - pp * pp;
                const double d = (divJ + pp - (pp * pp) * pp - lambda * (om * om) * UU(i, j, kk)) / as2 +
                                 Fnoise * orc_karma_ruido(i, j, kk, it) * (1.0 - pp * pp) / sqrt(dt);
                DP(i, j, kk) = d;
                s->phin[at3(s, i, j, kk)] = pp + dt * d;
            }

    espelho(s, dphi);

    /* U equation with the anti-trapping current, karma3d.f90:212-276 */
#pragma omp parallel for collapse(2) schedule(static)
    for (int kk = 1; kk <= s->nz; ++kk)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                const double pp = P(i, j, kk);
                const double q = 0.25 * idx;
                const double uc = UU(i, j, kk), dc = DP(i, j, kk);
                double g1, g2, g3, gm, qf, cf;
                /* x+ */
                g1 = (P(i + 1, j, kk) - pp) * idx;
                g2 = q * (P(i, j + 1, kk) + P(i + 1, j + 1, kk) - P(i, j - 1, kk) - P(i + 1, j - 1, kk));
                g3 = q * (P(i, j, kk + 1) + P(i + 1, j, kk + 1) - P(i, j, kk - 1) - P(i + 1, j, kk - 1));
                gm = sqrt(g1 * g1 + g2 * g2 + g3 * g3);
                qf = 0.25 * (2.0 - pp - P(i + 1, j, kk));
                cf = 0.5 * ((1.0 + (1.0 - k) * uc) * dc + (1.0 + (1.0 - k) * UU(i + 1, j, kk)) * DP(i + 1, j, kk));
                double Fxp = D * qf * (UU(i + 1, j, kk) - uc) * idx;
                if (gm > 1.e-10) Fxp = Fxp + KAT * cf * g1 / gm;
                /* x- */
                g1 = (pp - P(i - 1, j, kk)) * idx;
                g2 = q * (P(i, j + 1, kk) + P(i - 1, j + 1, kk) - P(i, j - 1, kk) - P(i - 1, j - 1, kk));
                g3 = q * (P(i, j, kk + 1) + P(i - 1, j, kk + 1) - P(i, j, kk - 1) - P(i - 1, j, kk - 1));
                gm = sqrt(g1 * g1 + g2 * g2 + g3 * g3);
                qf = 0.25 * (2.0 - pp - P(i - 1, j, kk));
                cf = 0.5 * ((1.0 + (1.0 - k) * uc) * dc + (1.0 + (1.0 - k) * UU(i - 1, j, kk)) * DP(i - 1, j, kk));
                double Fxm = D * qf * (uc - UU(i - 1, j, kk)) * idx;
                if (gm > 1.e-10) Fxm = Fxm + KAT * cf * g1 / gm;
                /* y+ */
                g2 = (P(i, j + 1, kk) - pp) * idx;
                g1 = q * (P(i + 1, j, kk) + P(i + 1, j + 1, kk) - P(i - 1, j, kk) - P(i - 1, j + 1, kk));
                g3 = q * (P(i, j, kk + 1) + P(i, j + 1, kk + 1) - P(i, j, kk - 1) - P(i, j + 1, kk - 1));
                gm = sqrt(g1 * g1 + g2 * g2 + g3 * g3);
                qf = 0.25 * (2.0 - pp - P(i, j + 1, kk));
                cf = 0.5 * ((1.0 + (1.0 - k) * uc) * dc + (1.0 + (1.0 - k) * UU(i, j + 1, kk)) * DP(i, j + 1, kk));
                double Fyp = D * qf * (UU(i, j + 1, kk) - uc) * idx;
                if (gm > 1.e-10) Fyp = Fyp + KAT * cf * g2 / gm;
                /* y- */
                g2 = (pp - P(i, j - 1, kk)) * idx;
                g1 = q * (P(i + 1, j, kk) + P(i + 1, j - 1, kk) - P(i - 1, j, kk) - P(i - 1, j - 1, kk));
                g3 = q * (P(i, j, kk + 1) + P(i, j - 1, kk + 1) - P(i, j, kk - 1) - P(i, j - 1, kk - 1));
                gm = sqrt(g1 * g1 + g2 * g2 + g3 * g3);
                qf = 0.25 * (2.0 - pp - P(i, j - 1, kk));
                cf = 0.5 * ((1.0 + (1.0 - k) * uc) * dc + (1.0 + (1.0 - k) * UU(i, j - 1, kk)) * DP(i, j - 1, kk));
                double Fym = D * qf * (uc - UU(i, j - 1, kk)) * idx;
                if (gm > 1.e-10) Fym = Fym + KAT * cf * g2 / gm;
                /* z+ */
                g3 = (P(i, j, kk + 1) - pp) * idx;
                g1 = q * (P(i + 1, j, kk) + P(i + 1, j, kk + 1) - P(i - 1, j, kk) - P(i - 1, j, kk + 1));
                g2 = q * (P(i, j + 1, kk) + P(i, j + 1, kk + 1) - P(i, j - 1, kk) - P(i, j - 1, kk + 1));
                gm = sqrt(g1 * g1 + g2 * g2 + g3 * g3);
                qf = 0.25 * (2.0 - pp - P(i, j, kk + 1));
                cf = 0.5 * ((1.0 + (1.0 - k) * uc) * dc + (1.0 + (1.0 - k) * UU(i, j, kk + 1)) * DP(i, j, kk + 1));
                double Fzp = D * qf * (UU(i, j, kk + 1) - uc) * idx;
                if (gm > 1.e-10) Fzp = Fzp + KAT * cf * g3 / gm;
                /* z- */
                g3 = (pp - P(i, j, kk - 1)) * idx;
                g1 = q * (P(i + 1, j, kk) + P(i + 1, j, kk - 1) - P(i - 1, j, kk) - P(i - 1, j, kk - 1));
                g2 = q * (P(i, j + 1, kk) + P(i, j + 1, kk - 1) - P(i, j - 1, kk) - P(i, j - 1, kk - 1));
                gm = sqrt(g1 * g1 + g2 * g2 + g3 * g3);
                qf = 0.25 * (2.0 - pp - P(i, j, kk - 1));
                cf = 0.5 * ((1.0 + (1.0 - k) * uc) * dc + (1.0 + (1.0 - k) * UU(i, j, kk - 1)) * DP(i, j, kk - 1));
                double Fzm = D * qf * (uc - UU(i, j, kk - 1)) * idx;
                if (gm > 1.e-10) Fzm = Fzm + KAT * cf * g3 / gm;

                const double Au = 0.5 * (1.0 + k) - 0.5 * (1.0 - k) * pp;
                const double rhsU = (Fxp - Fxm + Fyp - Fym + Fzp - Fzm) * idx + 0.5 * (1.0 + (1.0 - k) * uc) * dc;
                s->Un[at3(s, i, j, kk)] = uc + dt * rhsU / Au;
            }

    /* advance, karma3d.f90:279-287 */
#pragma omp parallel for collapse(2) schedule(static)
    for (int kk = 1; kk <= s->nz; ++kk)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                const size_t a = at3(s, i, j, kk);
                phi[a] = fmax(-1.0, fmin(1.0, s->phin[a]));
                U[a] = s->Un[a];
            }
#undef P
#undef UU
#undef DP
}

void orc_karma_set_it(orc_karma* s, int it) { s->it = it; }

void orc_karma_step(orc_karma* s, int n)
{
    for (int q = 0; q < n; ++q) karma_one(s);
}

/* karma3d.f90:290-296: largest i with phi(i,1,1) > 0 and with phi(i,i,i) > 0 */
void orc_karma_tip(const orc_karma* s, int* tip_x, int* tip_d)
{
    int tx = 0, td = 0;
    int nd = s->nx < s->ny ? s->nx : s->ny;
    nd = nd < s->nz ? nd : s->nz;
    for (int i = 1; i <= s->nx; ++i)
        if (s->phi[at3(s, i, 1, 1)] > 0.0) tx = i;
    for (int i = 1; i <= nd; ++i)
        if (s->phi[at3(s, i, i, i)] > 0.0) td = i;
    *tip_x = tx;
    *tip_d = td;
}
