/*
 * pf_oracle.c -- CPU oracle for the coupled explicit time step of the 3-D
 * Al-Cu phase-field model of ileaof/phase-field-project-3D.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/, the smoke
 * check of __graft_entry__.py and the cpu_baseline / reference arm of
 * bench.py may load it.  The product (libpf3d) never links or calls it.
 *
 * It restates, in plain C with OpenMP, the reference's Fortran for the hot
 * path, statement by statement and in the same evaluation order:
 *   - pseudo_random / ruido_suave        source/variaveis.f90:73-111
 *   - W0_E0                              source/W0_E0.f90:10-31
 *   - auxiliar (M0)                      source/auxiliar.f90:12-42
 *   - dt and AAA scaling                 source/entrada.f90:159-185
 *   - temperatura + temp_body.inc        source/temperatura.f90:89-115, temp_body.inc:11-45
 *   - equacao_campo_fase + phase_body    source/equacao_campo_fase.f90:105-167, phase_body.inc:14-198
 *   - concentracao_soluto + conc_body    source/concentracao_soluto.f90:78-124, conc_body.inc:11-149
 *   - diagnosticos + diag_body.inc       source/diagnosticos.f90:242-287, diag_body.inc:8-22
 *   - the step order of the time loop    source/principal.f90:93-226
 * The whole-array copies and the boundary "decoration" plane copies are
 * executed literally (sequential plane copies in the reference's order), not
 * in closed form, so they check the kernels' closed-form mapping.
 *
 * Fortran evaluation rules reproduced (gfortran, strict IEEE, x86-64 SSE):
 * left-to-right association, x**2 = x*x, x**3 = (x*x)*x, x**4 = (x*x)*(x*x),
 * x**2.d0 = x*x, divisions kept as divisions, no FMA contraction (build with
 * -ffp-contract=off), REAL(4) variables (Ke, Sigma, Beta, ajuste, ran, time)
 * and REAL(4) literals (0.0000001, 0.01, 54.39180136) rounded to float.
 *
 * PARITY UNPINNED against a reference binary: no Fortran compiler exists in
 * this environment and the reference ships no tests, fixtures or golden
 * vectors, so this restatement is not compared with the reference's output
 * bit for bit.  It is cross-checked against an independent numpy restatement
 * (tests/golden/np_restatement.py) and its known-answer vectors are committed
 * under tests/golden/.  The reference's run log does record macroscopic
 * output of one of its runs (the tip heights of run6, registro_runs.md:
 * 138-140); the GPU form, held to this oracle within 1e-12 at small sizes,
 * reproduces them (tests/test_run6_record_gpu.py), but the oracle itself is
 * too slow to run those 52 500 steps on 81 M cells.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "pf_oracle.h"
#ifdef _OPENMP
#include <omp.h>
#endif

#define IDX(s, i, j, k) ((size_t)((i) - 1) + (size_t)(s)->nx * ((size_t)((j) - 1) + (size_t)(s)->ny * (size_t)((k) - 1)))

/* ---------------- noise: variaveis.f90:73-111 ---------------- */

double orc_pseudo_random(int i, int j, int k, int it, int salt)
{
    /* hval = int(i,8)*2654435761 + ... + 1 ; wrapping 64-bit arithmetic */
    uint64_t h = (uint64_t)(int64_t)i * 2654435761ull + (uint64_t)(int64_t)j * 2246822519ull +
                 (uint64_t)(int64_t)k * 3266489917ull + (uint64_t)(int64_t)it * 668265263ull +
                 (uint64_t)(int64_t)salt * 374761393ull + 1ull;
    h = h ^ (h >> 33);                 /* ieor(hval, ishft(hval,-33)): logical shift */
    h = h * 0xff51afd7ed558ccdull;
    h = h ^ (h >> 33);
    h = h * 0xc4ceb9fe1a85ec53ull;
    h = h ^ (h >> 33);
    /* real(iand(hval,MASK63),8) / real(MASK63,8); MASK63 rounds to 2^63 */
    int64_t m = (int64_t)(h & 0x7fffffffffffffffull);
    return (double)m / (double)INT64_MAX;
}

double orc_ruido_suave(int i, int j, int k, int it)
{
    const int LR = 6, TR = 20;         /* LR_RUIDO, TR_RUIDO (variaveis.f90:62) */
    int i0 = i / LR, j0 = j / LR, k0 = k / LR, tb = it / TR;
    double fx = (double)(i % LR) / (double)LR;
    double fy = (double)(j % LR) / (double)LR;
    double fz = (double)(k % LR) / (double)LR;
    double r =
        (1.0 - fz) * ((1.0 - fy) * ((1.0 - fx) * orc_pseudo_random(i0, j0, k0, tb, 3) +
                                    fx * orc_pseudo_random(i0 + 1, j0, k0, tb, 3)) +
                      fy * ((1.0 - fx) * orc_pseudo_random(i0, j0 + 1, k0, tb, 3) +
                            fx * orc_pseudo_random(i0 + 1, j0 + 1, k0, tb, 3))) +
        fz * ((1.0 - fy) * ((1.0 - fx) * orc_pseudo_random(i0, j0, k0 + 1, tb, 3) +
                            fx * orc_pseudo_random(i0 + 1, j0, k0 + 1, tb, 3)) +
              fy * ((1.0 - fx) * orc_pseudo_random(i0, j0 + 1, k0 + 1, tb, 3) +
                    fx * orc_pseudo_random(i0 + 1, j0 + 1, k0 + 1, tb, 3)));
    return r;
}

/* ---------------- scalar set-up ---------------- */

/* W0_E0.f90:10-31.  DO EPSLON_Try = 0, 1, 0.0000001: a REAL DO loop whose
 * step is the REAL(4) literal 1e-7 converted to double; the variable is
 * advanced by repeated addition.  Exits at the first |E0-eps| < 1e-5. */
void orc_w0_e0(double Lambda, float ajuste, float Sigma, double* W0, double* E0, long* iters)
{
    const double step = (double)0.0000001f;
    const double from = 0.0, to = 1.0;
    long count = (long)((to - from + step) / step);
    double eps = from, w0 = 0.0, e0 = 0.0;
    long n = 0;
    float as = ajuste * Sigma;         /* REAL(4) product */
    for (; n < count; ++n) {
        w0 = ((1.5556349186104 / Lambda) * eps) * ((1.5556349186104 / Lambda) * eps);
        e0 = (double)as * 4.24264068711929 / sqrt(w0);
        if (fabs(e0 - eps) < 1e-5) break;
        eps = eps + step;
    }
    *W0 = w0;
    *E0 = e0;
    if (iters) *iters = n + 1;
}

/* auxiliar.f90:12-42 */
double orc_auxiliar(const orc_params* p, double TP, double Cs_eq, double Cl_eq, double E0, double W0)
{
    double acc = 0.0;
    double phi = 0.11;
    for (;;) {
        double h = phi * phi * (3.0 - 2.0 * phi);
        double f1 = phi * (1.0 - phi);
        double num = h * (1.0 - h);
        double den = ((1.0 - h) * Cl_eq * (1.0 - Cl_eq) + h * Cs_eq * (1.0 - Cs_eq)) * f1;
        double fi = num / den;
        acc = acc + fi;
        phi = phi + 0.01;
        if (!(phi <= 0.8999)) break;
    }
    /* (0.01/2.d0)*( 54.39180136 + 2.d0*acc + 234.073053d0 ): the first two
       literals are REAL(4) */
    double integral = ((double)0.01f / 2.0) * ((double)54.39180136f + 2.0 * acc + 234.073053);
    double qsi = p->R * TP * (1.0 / p->Vm) * (Cl_eq - Cs_eq) * (Cl_eq - Cs_eq) * integral;
    float one_minus_ke = 1.0f - p->Ke;  /* (1-Ke) is REAL(4) */
    double inv_m0 = (E0 * E0 / (double)p->Sigma) *
                    (((double)p->Beta * p->R * TP * (double)one_minus_ke / (p->Vm * p->Me)) +
                     (E0 * qsi / (p->D_liq * sqrt(2.0 * W0))));
    return (double)p->ajuste * 1.0 / inv_m0;
}

/* ---------------- state ---------------- */

static size_t ncell(const orc_state* s) { return (size_t)s->nx * s->ny * s->nz; }

orc_state* orc_create(int nx, int ny, int nz, double dx, double dy, double dz, const orc_params* p)
{
    if (nx < 5 || ny < 5 || nz < 5) return NULL;
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    if (!s) return NULL;
    s->nx = nx; s->ny = ny; s->nz = nz;
    s->dx = dx; s->dy = dy; s->dz = dz;
    s->p = *p;
    size_t n = ncell(s);
    double** f[7] = {&s->phi_old, &s->phi_new, &s->c_old, &s->c_new, &s->T_old, &s->T_new, &s->dpp};
    for (int q = 0; q < 7; ++q) {
        *f[q] = (double*)calloc(n, sizeof(double));
        if (!*f[q]) { orc_destroy(s); return NULL; }
    }
    /* entrada.f90:159-185 */
    s->Lambda = p->Thin_Interface * dx;
    s->dt = (dx * dx) / (7.5 * p->D_liq);
    if (p->ruido_tipo == 0)
        s->AAA = p->AAA * (s->dt / ((dx * dx) / (5.0 * p->D_liq)));
    else
        s->AAA = p->AAA * sqrt(s->dt / ((dx * dx) / (5.0 * p->D_liq)));
    s->TP = p->TP;
    if (p->taxa_resfr > 0.0) s->TP = p->T0;  /* entrada.f90:81 */
    s->M0 = p->M0;
    orc_w0_e0(s->Lambda, p->ajuste, p->Sigma, &s->W0, &s->E0, &s->w0e0_iters);
    s->it = 0;
    s->time = 0.0f;
    return s;
}

void orc_destroy(orc_state* s)
{
    if (!s) return;
    free(s->phi_old); free(s->phi_new); free(s->c_old); free(s->c_new);
    free(s->T_old); free(s->T_new); free(s->dpp);
    free(s);
}

double* orc_field(orc_state* s, int field)
{
    switch (field) {
    case 0: return s->phi_old;
    case 1: return s->phi_new;
    case 2: return s->c_old;
    case 3: return s->c_new;
    case 4: return s->T_old;
    case 5: return s->T_new;
    case 6: return s->dpp;
    }
    return NULL;
}

void orc_set_field(orc_state* s, int field, const double* src) { memcpy(orc_field(s, field), src, ncell(s) * sizeof(double)); }
void orc_get_field(orc_state* s, int field, double* dst) { memcpy(dst, orc_field(s, field), ncell(s) * sizeof(double)); }

/* ---------------- temperatura.f90:89-115 + temp_body.inc ---------------- */

void orc_temperatura(orc_state* s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double dx = s->dx, dy = s->dy, dz = s->dz;
    const double TP = s->TP, dt = s->dt, D = s->p.D, delta_H = s->p.delta_H;
    const double cp = s->p.Cp_s;      /* temperatura.f90:9 */
    const int hq = s->p.h_quintico;
    memcpy(s->T_new, s->T_old, ncell(s) * sizeof(double));  /* TNEW = TOLD */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 2; k <= nz - 1; ++k)
        for (int j = 2; j <= ny - 1; ++j)
            for (int i = 2; i <= nx - 1; ++i) {
                double TE = s->T_old[IDX(s, i + 1, j, k)];
                double TW = s->T_old[IDX(s, i - 1, j, k)];
                double TN = s->T_old[IDX(s, i, j + 1, k)];
                double TS = s->T_old[IDX(s, i, j - 1, k)];
                double TT = s->T_old[IDX(s, i, j, k + 1)];
                double TB = s->T_old[IDX(s, i, j, k - 1)];
                double PP = s->phi_old[IDX(s, i, j, k)];
                double h_linha;
                if (hq == 1)
                    h_linha = 30.0 * PP * PP * (1.0 - PP) * (1.0 - PP);
                else
                    h_linha = 2.0 * PP * (3.0 - 2.0 * PP) - 2.0 * PP * PP;
                double FONTE = (delta_H / cp) * h_linha * s->dpp[IDX(s, i, j, k)];
                double TNEW1 = D * dt * (((TE - 2.0 * TP + TW) / (dx * dx)) + ((TN - 2.0 * TP + TS) / (dy * dy)) +
                                         ((TT - 2.0 * TP + TB) / (dz * dz))) +
                               FONTE + TP;
                s->T_new[IDX(s, i, j, k)] = TNEW1;
            }
}

/* ---------------- equacao_campo_fase.f90:105-167 + phase_body.inc ---------------- */

static inline double sq(double x) { return x * x; }
static inline double p4(double x) { double t = x * x; return t * t; }

void orc_equacao_campo_fase(orc_state* s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double dx = s->dx, dy = s->dy, dz = s->dz;
    const double E0 = s->E0, w0 = s->W0, DELTA_EPSLON = s->p.DELTA_EPSLON;
    const double DELTA_T = s->dt, M0 = s->M0, AAA = s->AAA, TP = s->TP;
    const double R = s->p.R, Vm = s->p.Vm, Tm = s->p.Tm, Me = s->p.Me;
    const float Ke = s->p.Ke;
    const int hq = s->p.h_quintico, rt = s->p.ruido_tipo, it = s->it;
    /* equacao_campo_fase.f90:21-22 */
    const double Cs_eq = ((Tm - TP) * (double)Ke) / Me;
    const double Cl_eq = (Tm - TP) / Me;
    s->Cs_eq = Cs_eq;
    s->Cl_eq = Cl_eq;
    const double* po = s->phi_old;
    double* pn = s->phi_new;

    memcpy(pn, po, ncell(s) * sizeof(double));  /* phase_field_new = phase_field_old */

#define PO(a, b, c) po[IDX(s, a, b, c)]
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 3; k <= nz - 2; ++k)
        for (int j = 3; j <= ny - 2; ++j)
            for (int i = 3; i <= nx - 2; ++i) {
                double PP = PO(i, j, k);
                double PN = PO(i, j + 1, k);
                double PS = PO(i, j - 1, k);
                double PE = PO(i + 1, j, k);
                double PW = PO(i - 1, j, k);
                double PT = PO(i, j, k + 1);
                double PB = PO(i, j, k - 1);
                double PNE = PO(i + 1, j + 1, k), PSE = PO(i + 1, j - 1, k);
                double PNW = PO(i - 1, j + 1, k), PSW = PO(i - 1, j - 1, k);
                double PNT = PO(i, j + 1, k + 1), PNB = PO(i, j + 1, k - 1);
                double PST = PO(i, j - 1, k + 1), PSB = PO(i, j - 1, k - 1);
                double PET = PO(i + 1, j, k + 1), PEB = PO(i + 1, j, k - 1);
                double PWT = PO(i - 1, j, k + 1), PWB = PO(i - 1, j, k - 1);
                const double small = 1e-23;
                double K_aniso = 16.0 * E0 * DELTA_EPSLON;

                /* PONTO E */
                double phix_E = (PO(i + 2, j, k) - PP) * 0.5 / dx;
                double phiy_E = (PO(i + 1, j + 1, k) - PO(i + 1, j - 1, k)) * 0.5 / dy;
                double phiz_E = (PO(i + 1, j, k + 1) - PO(i + 1, j, k - 1)) * 0.5 / dz;
                double Q_E = sq(phix_E) + sq(phiy_E) + sq(phiz_E) + small;
                double S4_E = p4(phix_E) + p4(phiy_E) + p4(phiz_E);
                double eps_E = E0 * (1.0 + DELTA_EPSLON * (4.0 * S4_E / sq(Q_E) - 3.0));
                double exy_E = K_aniso * eps_E * phix_E * phiy_E * (sq(phix_E) - sq(phiy_E)) / sq(Q_E);
                double ezx_E = K_aniso * eps_E * phiz_E * phix_E * (sq(phiz_E) - sq(phix_E)) / sq(Q_E);
                /* PONTO W */
                double phix_W = (PP - PO(i - 2, j, k)) * 0.5 / dx;
                double phiy_W = (PO(i - 1, j + 1, k) - PO(i - 1, j - 1, k)) * 0.5 / dy;
                double phiz_W = (PO(i - 1, j, k + 1) - PO(i - 1, j, k - 1)) * 0.5 / dz;
                double Q_W = sq(phix_W) + sq(phiy_W) + sq(phiz_W) + small;
                double S4_W = p4(phix_W) + p4(phiy_W) + p4(phiz_W);
                double eps_W = E0 * (1.0 + DELTA_EPSLON * (4.0 * S4_W / sq(Q_W) - 3.0));
                double exy_W = K_aniso * eps_W * phix_W * phiy_W * (sq(phix_W) - sq(phiy_W)) / sq(Q_W);
                double ezx_W = K_aniso * eps_W * phiz_W * phix_W * (sq(phiz_W) - sq(phix_W)) / sq(Q_W);
                /* PONTO N */
                double phix_N = (PO(i + 1, j + 1, k) - PO(i - 1, j + 1, k)) * 0.5 / dx;
                double phiy_N = (PO(i, j + 2, k) - PP) * 0.5 / dy;
                double phiz_N = (PO(i, j + 1, k + 1) - PO(i, j + 1, k - 1)) * 0.5 / dz;
                double Q_N = sq(phix_N) + sq(phiy_N) + sq(phiz_N) + small;
                double S4_N = p4(phix_N) + p4(phiy_N) + p4(phiz_N);
                double eps_N = E0 * (1.0 + DELTA_EPSLON * (4.0 * S4_N / sq(Q_N) - 3.0));
                double exy_N = K_aniso * eps_N * phix_N * phiy_N * (sq(phix_N) - sq(phiy_N)) / sq(Q_N);
                double eyz_N = K_aniso * eps_N * phiy_N * phiz_N * (sq(phiy_N) - sq(phiz_N)) / sq(Q_N);
                /* PONTO S */
                double phix_S = (PO(i + 1, j - 1, k) - PO(i - 1, j - 1, k)) * 0.5 / dx;
                double phiy_S = (PP - PO(i, j - 2, k)) * 0.5 / dy;
                double phiz_S = (PO(i, j - 1, k + 1) - PO(i, j - 1, k - 1)) * 0.5 / dz;
                double Q_S = sq(phix_S) + sq(phiy_S) + sq(phiz_S) + small;
                double S4_S = p4(phix_S) + p4(phiy_S) + p4(phiz_S);
                double eps_S = E0 * (1.0 + DELTA_EPSLON * (4.0 * S4_S / sq(Q_S) - 3.0));
                double exy_S = K_aniso * eps_S * phix_S * phiy_S * (sq(phix_S) - sq(phiy_S)) / sq(Q_S);
                double eyz_S = K_aniso * eps_S * phiy_S * phiz_S * (sq(phiy_S) - sq(phiz_S)) / sq(Q_S);
                /* PONTO T */
                double phix_T = (PO(i + 1, j, k + 1) - PO(i - 1, j, k + 1)) * 0.5 / dx;
                double phiy_T = (PO(i, j + 1, k + 1) - PO(i, j - 1, k + 1)) * 0.5 / dy;
                double phiz_T = (PO(i, j, k + 2) - PP) * 0.5 / dz;
                double Q_T = sq(phix_T) + sq(phiy_T) + sq(phiz_T) + small;
                double S4_T = p4(phix_T) + p4(phiy_T) + p4(phiz_T);
                double eps_T = E0 * (1.0 + DELTA_EPSLON * (4.0 * S4_T / sq(Q_T) - 3.0));
                double eyz_T = K_aniso * eps_T * phiy_T * phiz_T * (sq(phiy_T) - sq(phiz_T)) / sq(Q_T);
                double ezx_T = K_aniso * eps_T * phiz_T * phix_T * (sq(phiz_T) - sq(phix_T)) / sq(Q_T);
                /* PONTO B */
                double phix_B = (PO(i + 1, j, k - 1) - PO(i - 1, j, k - 1)) * 0.5 / dx;
                double phiy_B = (PO(i, j + 1, k - 1) - PO(i, j - 1, k - 1)) * 0.5 / dy;
                double phiz_B = (PP - PO(i, j, k - 2)) * 0.5 / dz;
                double Q_B = sq(phix_B) + sq(phiy_B) + sq(phiz_B) + small;
                double S4_B = p4(phix_B) + p4(phiy_B) + p4(phiz_B);
                double eps_B = E0 * (1.0 + DELTA_EPSLON * (4.0 * S4_B / sq(Q_B) - 3.0));
                double eyz_B = K_aniso * eps_B * phiy_B * phiz_B * (sq(phiy_B) - sq(phiz_B)) / sq(Q_B);
                double ezx_B = K_aniso * eps_B * phiz_B * phix_B * (sq(phiz_B) - sq(phix_B)) / sq(Q_B);

                double AA = (sq(eps_E) * (PE - PP) + sq(eps_W) * (PW - PP)) / sq(dx) +
                            (sq(eps_N) * (PN - PP) + sq(eps_S) * (PS - PP)) / sq(dy) +
                            (sq(eps_T) * (PT - PP) + sq(eps_B) * (PB - PP)) / sq(dz);

                double Cross_xy = (0.25 / (dx * dy)) * (PNE * (-exy_N - (-exy_E)) + PSE * (-exy_E - (-exy_S)) +
                                                        PNW * (-exy_W - (-exy_N)) + PSW * (-exy_S - (-exy_W))) +
                                  PN * (0.25 / (dx * dy)) * (-exy_W - (-exy_E)) + PS * (0.25 / (dx * dy)) * (-exy_E - (-exy_W)) +
                                  PE * (0.25 / (dx * dy)) * (-exy_N - (-exy_S)) + PW * (0.25 / (dx * dy)) * (-exy_S - (-exy_N));

                double Cross_yz = (0.25 / (dy * dz)) * (PNT * (-eyz_T - (-eyz_N)) + PNB * (-eyz_N - (-eyz_B)) +
                                                        PST * (-eyz_S - (-eyz_T)) + PSB * (-eyz_B - (-eyz_S))) +
                                  PT * (0.25 / (dy * dz)) * (-eyz_S - (-eyz_N)) + PB * (0.25 / (dy * dz)) * (-eyz_N - (-eyz_S)) +
                                  PN * (0.25 / (dy * dz)) * (-eyz_T - (-eyz_B)) + PS * (0.25 / (dy * dz)) * (-eyz_B - (-eyz_T));

                double Cross_zx = (0.25 / (dz * dx)) * (PET * (-ezx_E - (-ezx_T)) + PWT * (-ezx_T - (-ezx_W)) +
                                                        PEB * (-ezx_B - (-ezx_E)) + PWB * (-ezx_W - (-ezx_B))) +
                                  PE * (0.25 / (dz * dx)) * (-ezx_B - (-ezx_T)) + PW * (0.25 / (dz * dx)) * (-ezx_T - (-ezx_B)) +
                                  PT * (0.25 / (dz * dx)) * (-ezx_E - (-ezx_W)) + PB * (0.25 / (dz * dx)) * (-ezx_W - (-ezx_E));

                AA = AA + Cross_xy + Cross_yz + Cross_zx;

                double g_linha = 2.0 * PP * (1.0 - PP) * (1.0 - PP) - 2.0 * PP * PP * (1.0 - PP);
                double CPP = s->c_old[IDX(s, i, j, k)];
                double h_linha, h;
                if (hq == 1) {
                    h_linha = 30.0 * PP * PP * (1.0 - PP) * (1.0 - PP);
                    h = PP * PP * PP * (10.0 - 15.0 * PP + 6.0 * PP * PP);
                } else {
                    h_linha = 2.0 * PP * (3.0 - 2.0 * PP) - 2.0 * PP * PP;
                    h = PP * PP * (3.0 - 2.0 * PP);
                }
                double CLP = CPP / ((double)Ke * h + (1.0 - h));
                double CSP = (double)Ke * CPP / ((double)Ke * h + (1.0 - h));
                double GG = (-(w0 * g_linha)) +
                            (R * TP / Vm) * h_linha * log(fabs(((1.0 - Cs_eq) * (1.0 - CLP)) / ((1.0 - Cl_eq) * (1.0 - CSP))));

                float ran;
                if (rt == 2)
                    ran = (float)orc_ruido_suave(i, j, k, it);
                else
                    ran = (float)orc_pseudo_random(i, j, k, it, 1);
                double ruidos;
                if (rt == 0)
                    ruidos = (double)ran * AAA * 16.0 * sq(PP) * sq(1.0 - PP);
                else
                    ruidos = (2.0 * (double)ran - 1.0) * AAA * 16.0 * sq(PP) * sq(1.0 - PP);

                double PPNEW = PP + (M0 * DELTA_T) * (AA + GG) + ruidos;
                s->dpp[IDX(s, i, j, k)] = PPNEW - PO(i, j, k);
                double t = (PPNEW < 1.0) ? PPNEW : 1.0;   /* dmin1(1.d0, PPNEW) */
                pn[IDX(s, i, j, k)] = (t > 0.0) ? t : 0.0; /* dmax1(0.d0, .)     */
            }
#undef PO

    /* equacao_campo_fase.f90:151-167, literally, in order */
#define PNW_(a, b, c) pn[IDX(s, a, b, c)]
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) PNW_(i, 1, k) = PNW_(i, 2, k);
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) PNW_(i, 2, k) = PNW_(i, 3, k);
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) PNW_(i, ny, k) = PNW_(i, ny - 1, k);
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) PNW_(i, ny - 1, k) = PNW_(i, ny - 2, k);
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) PNW_(1, j, k) = PNW_(2, j, k);
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) PNW_(2, j, k) = PNW_(3, j, k);
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) PNW_(nx, j, k) = PNW_(nx - 1, j, k);
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) PNW_(nx - 1, j, k) = PNW_(nx - 2, j, k);
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) PNW_(i, j, 1) = PNW_(i, j, 2);
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) PNW_(i, j, 2) = PNW_(i, j, 3);
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) PNW_(i, j, nz) = PNW_(i, j, nz - 1);
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) PNW_(i, j, nz - 1) = PNW_(i, j, nz - 2);
#undef PNW_
}

/* principal.f90:140-148 */
void orc_copy_phase_new_to_old(orc_state* s) { memcpy(s->phi_old, s->phi_new, ncell(s) * sizeof(double)); }

/* ---------------- concentracao_soluto.f90:78-124 + conc_body.inc ---------------- */

void orc_concentracao_soluto(orc_state* s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double InvDX = 1.0 / (s->dx * s->dx);
    const double InvDY = 1.0 / (s->dy * s->dy);
    const double InvDZ = 1.0 / (s->dz * s->dz);
    const double DELTA_T = s->dt, D_liq = s->p.D_liq, D_sol = s->p.D_sol;
    const double Ke = (double)s->p.Ke;
    const int hq = s->p.h_quintico;
    const double* po = s->phi_old;
    const double* co = s->c_old;
    double* cn = s->c_new;

    memcpy(cn, co, ncell(s) * sizeof(double));  /* conc_soluto_new = conc_soluto_old */

#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 2; k <= nz - 1; ++k)
        for (int j = 2; j <= ny - 1; ++j)
            for (int i = 2; i <= nx - 1; ++i) {
                double PP = po[IDX(s, i, j, k)];
                double PN = po[IDX(s, i, j + 1, k)];
                double PS = po[IDX(s, i, j - 1, k)];
                double PW = po[IDX(s, i - 1, j, k)];
                double PE = po[IDX(s, i + 1, j, k)];
                double PT = po[IDX(s, i, j, k + 1)];
                double PB = po[IDX(s, i, j, k - 1)];
                double CPP = co[IDX(s, i, j, k)];
                double CPS = co[IDX(s, i, j - 1, k)];
                double CPN = co[IDX(s, i, j + 1, k)];
                double CPW = co[IDX(s, i - 1, j, k)];
                double CPE = co[IDX(s, i + 1, j, k)];
                double CPT = co[IDX(s, i, j, k + 1)];
                double CPB = co[IDX(s, i, j, k - 1)];
                double h, h_E, h_W, h_N, h_S, h_T, h_B;
                if (hq == 1) {
                    h = (PP * PP * PP) * (10.0 - (15.0 * PP) + (6.0 * (PP * PP)));
                    h_E = (PE * PE * PE) * (10.0 - (15.0 * PE) + (6.0 * (PE * PE)));
                    h_W = (PW * PW * PW) * (10.0 - (15.0 * PW) + (6.0 * (PW * PW)));
                    h_N = (PN * PN * PN) * (10.0 - (15.0 * PN) + (6.0 * (PN * PN)));
                    h_S = (PS * PS * PS) * (10.0 - (15.0 * PS) + (6.0 * (PS * PS)));
                    h_T = (PT * PT * PT) * (10.0 - (15.0 * PT) + (6.0 * (PT * PT)));
                    h_B = (PB * PB * PB) * (10.0 - (15.0 * PB) + (6.0 * (PB * PB)));
                } else {
                    h = PP * PP * (3.0 - 2.0 * PP);
                    h_E = PE * PE * (3.0 - 2.0 * PE);
                    h_W = PW * PW * (3.0 - 2.0 * PW);
                    h_N = PN * PN * (3.0 - 2.0 * PN);
                    h_S = PS * PS * (3.0 - 2.0 * PS);
                    h_T = PT * PT * (3.0 - 2.0 * PT);
                    h_B = PB * PB * (3.0 - 2.0 * PB);
                }
                double CSP = (Ke * CPP) / ((Ke * h) + (1.0 - h));
                double CSN = (Ke * CPN) / ((Ke * h_N) + (1.0 - h_N));
                double CSS = (Ke * CPS) / ((Ke * h_S) + (1.0 - h_S));
                double CSE = (Ke * CPE) / ((Ke * h_E) + (1.0 - h_E));
                double CSW = (Ke * CPW) / ((Ke * h_W) + (1.0 - h_W));
                double CST = (Ke * CPT) / ((Ke * h_T) + (1.0 - h_T));
                double CSB = (Ke * CPB) / ((Ke * h_B) + (1.0 - h_B));
                double CLP = CPP / (Ke * h + (1.0 - h));
                double CLN = CPN / (Ke * h_N + (1.0 - h_N));
                double CLS = CPS / (Ke * h_S + (1.0 - h_S));
                double CLE = CPE / (Ke * h_E + (1.0 - h_E));
                double CLW = CPW / (Ke * h_W + (1.0 - h_W));
                double CLT = CPT / (Ke * h_T + (1.0 - h_T));
                double CLB = CPB / (Ke * h_B + (1.0 - h_B));
                double D_soluto_C = (PP <= 0.95) ? D_liq : D_sol;
                double GAMA_P = D_soluto_C * ((1.0 - h) * CLP * (1.0 - CLP) + h * CSP * (1.0 - CSP));
                double GAMA_S = D_soluto_C * ((1.0 - h_S) * CLS * (1.0 - CLS) + h_S * CSS * (1.0 - CSS));
                double GAMA_N = D_soluto_C * ((1.0 - h_N) * CLN * (1.0 - CLN) + h_N * CSN * (1.0 - CSN));
                double GAMA_W = D_soluto_C * ((1.0 - h_W) * CLW * (1.0 - CLW) + h_W * CSW * (1.0 - CSW));
                double GAMA_E = D_soluto_C * ((1.0 - h_E) * CLE * (1.0 - CLE) + h_E * CSE * (1.0 - CSE));
                double GAMA_T = D_soluto_C * ((1.0 - h_T) * CLT * (1.0 - CLT) + h_T * CST * (1.0 - CST));
                double GAMA_B = D_soluto_C * ((1.0 - h_B) * CLB * (1.0 - CLB) + h_B * CSB * (1.0 - CSB));
                double GAMAs = 2.0 / ((1.0 / GAMA_P) + (1.0 / GAMA_S));
                double GAMAn = 2.0 / ((1.0 / GAMA_N) + (1.0 / GAMA_P));
                double GAMAw = 2.0 / ((1.0 / GAMA_P) + (1.0 / GAMA_W));
                double GAMAe = 2.0 / ((1.0 / GAMA_E) + (1.0 / GAMA_P));
                double GAMAt = 2.0 / ((1.0 / GAMA_T) + (1.0 / GAMA_P));
                double GAMAb = 2.0 / ((1.0 / GAMA_P) + (1.0 / GAMA_B));
                /* conc_body.inc:134-136: the solute noise is computed but unused */
                double c_new = (GAMAe * InvDX * (log(CLE / (1.0 - CLE)) - log(CLP / (1.0 - CLP))) -
                                GAMAw * InvDX * (log(CLP / (1.0 - CLP)) - log(CLW / (1.0 - CLW))) +
                                GAMAn * InvDY * (log(CLN / (1.0 - CLN)) - log(CLP / (1.0 - CLP))) -
                                GAMAs * InvDY * (log(CLP / (1.0 - CLP)) - log(CLS / (1.0 - CLS))) +
                                GAMAt * InvDZ * (log(CLT / (1.0 - CLT)) - log(CLP / (1.0 - CLP))) -
                                GAMAb * InvDZ * (log(CLP / (1.0 - CLP)) - log(CLB / (1.0 - CLB)))) *
                                   DELTA_T +
                               CPP;
                cn[IDX(s, i, j, k)] = c_new;
            }

    /* concentracao_soluto.f90:116-124, literally */
    memcpy(s->c_old, cn, ncell(s) * sizeof(double));  /* conc_soluto_old = conc_soluto_new */
    double* co2 = s->c_old;
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) cn[IDX(s, i, 1, k)] = co2[IDX(s, i, 2, k)];
    for (int k = 1; k <= nz; ++k) for (int i = 1; i <= nx; ++i) cn[IDX(s, i, ny, k)] = co2[IDX(s, i, ny - 1, k)];
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) cn[IDX(s, 1, j, k)] = co2[IDX(s, 2, j, k)];
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) cn[IDX(s, nx, j, k)] = co2[IDX(s, nx - 1, j, k)];
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) cn[IDX(s, i, j, 1)] = co2[IDX(s, i, j, 2)];
    for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) cn[IDX(s, i, j, nz)] = co2[IDX(s, i, j, nz - 1)];
}

/* ---------------- diagnosticos.f90 + diag_body.inc (serial order) ---------------- */

void orc_diagnosticos(const orc_state* s, double out[5])
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double dx = s->dx, dy = s->dy, dz = s->dz, E0 = s->E0, w0 = s->W0;
    const double* pn = s->phi_new;
    double L2 = 0.0, pmax = -1.7976931348623157e308, pmin = 1.7976931348623157e308, sol = 0.0, fe = 0.0;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double phi_p = pn[IDX(s, i, j, k)];
                L2 = L2 + phi_p * phi_p;
                if (phi_p > pmax) pmax = phi_p;
                if (phi_p < pmin) pmin = phi_p;
                sol = sol + s->c_new[IDX(s, i, j, k)];
                double w_term = w0 * phi_p * phi_p * (1.0 - phi_p) * (1.0 - phi_p);
                double grad2;
                if (i > 1 && i < nx && j > 1 && j < ny && k > 1 && k < nz)
                    grad2 = sq((pn[IDX(s, i + 1, j, k)] - pn[IDX(s, i - 1, j, k)]) * 0.5 / dx) +
                            sq((pn[IDX(s, i, j + 1, k)] - pn[IDX(s, i, j - 1, k)]) * 0.5 / dy) +
                            sq((pn[IDX(s, i, j, k + 1)] - pn[IDX(s, i, j, k - 1)]) * 0.5 / dz);
                else
                    grad2 = 0.0;
                fe = fe + (0.5 * E0 * E0 * grad2 + w_term) * dx * dy * dz;
            }
    out[0] = sqrt(L2);
    out[1] = pmax;
    out[2] = pmin;
    out[3] = sol;
    out[4] = fe;
}

/* principal.f90:213-225 */
void orc_swap(orc_state* s)
{
    size_t b = ncell(s) * sizeof(double);
    memcpy(s->phi_old, s->phi_new, b);
    memcpy(s->T_old, s->T_new, b);
    memcpy(s->c_old, s->c_new, b);
}

/* ---------------- time loop: principal.f90:93-226 ---------------- */

void orc_step(orc_state* s)
{
    int it = s->it + 1;
    s->it = it;
    s->time = (float)(s->dt + (double)s->time);                   /* :96  */
    orc_temperatura(s);                                           /* :98  */
    if (s->p.taxa_resfr > 0.0) s->TP = s->p.T0 - s->p.taxa_resfr * s->dt * it;  /* :104 */
    int nsw = s->p.n_varreduras < 1 ? 1 : s->p.n_varreduras;
    for (int n_sw = 1; n_sw <= nsw; ++n_sw) {                     /* :127-152 */
        if (n_sw > 1) orc_copy_phase_new_to_old(s);
        orc_equacao_campo_fase(s);
    }
    orc_concentracao_soluto(s);                                   /* :154 */
    s->M0 = orc_auxiliar(&s->p, s->TP, s->Cs_eq, s->Cl_eq, s->E0, s->W0);  /* :157 */
    orc_swap(s);                                                  /* :200-226 */
}

void orc_run(orc_state* s, int nsteps)
{
    for (int n = 0; n < nsteps; ++n) orc_step(s);
}

void orc_get_scalars(const orc_state* s, double out[10])
{
    out[0] = s->dt;
    out[1] = s->AAA;
    out[2] = s->Lambda;
    out[3] = s->W0;
    out[4] = s->E0;
    out[5] = s->TP;
    out[6] = s->M0;
    out[7] = (double)s->it;
    out[8] = (double)s->time;
    out[9] = (double)s->w0e0_iters;
}

void orc_set_scalars(orc_state* s, int it, double TP, double M0, float time)
{
    s->it = it;
    s->TP = TP;
    s->M0 = M0;
    s->time = time;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
