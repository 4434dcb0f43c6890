// pf3d_scalar.cpp -- host-side FP64 scalar set-up of the phase-field step:
// the W0/E0 fixed-point scan (W0_E0.f90), the per-step mobility M0
// (auxiliar.f90) and the dt / noise-amplitude rescale (entrada.f90:159-185).
// These run once per run or once per step on a handful of scalars, so they
// stay on the host in FP64 for every storage precision.  REAL(4) variables
// and literals of the reference are rounded to float where it rounds them.
// Built with -ffp-contract=off: no multiply-add contraction.
#include <cmath>
#include <cstring>
#include "../../include/pf3d.h"
#include "pf3d_scalar.h"

namespace pf3d {

void setup_derived(const pf_grid& g, const pf_params& p, pf_derived& out)
{
    std::memset(&out, 0, sizeof(out));
    const double dx = g.dx;
    out.Lambda = p.Thin_Interface * dx;             // entrada.f90:161
    out.DELTA_T = (dx * dx) / (7.5 * p.D_liq);      // entrada.f90:173
    const double ratio = out.DELTA_T / ((dx * dx) / (5.0 * p.D_liq));
    out.AAA = (p.ruido_tipo == 0) ? p.AAA * ratio : p.AAA * std::sqrt(ratio);  // :179-185
    pf_w0_e0(&g, &p, &out.W0, &out.E0, &out.w0e0_iterations);
}

double initial_tp(const pf_params& p)
{
    // TP line of the deck, replaced by T0 under continuous cooling (entrada.f90:81)
    return (p.taxa_resfr > 0.0) ? p.T0 : p.TP;
}

double step_tp(const pf_params& p, double dt, int it, double tp_prev)
{
    // principal.f90:104: TP = T0 - taxa_resfr*DELTA_T*IT
    if (p.taxa_resfr > 0.0) return p.T0 - p.taxa_resfr * dt * (double)it;
    return tp_prev;
}

void equilibrium(const pf_params& p, double TP, double* Cs_eq, double* Cl_eq)
{
    // equacao_campo_fase.f90:21-22
    *Cs_eq = ((p.Tm - TP) * (double)p.Ke) / p.Me;
    *Cl_eq = (p.Tm - TP) / p.Me;
}

}  // namespace pf3d

extern "C" int pf_w0_e0(const pf_grid* g, const pf_params* p, double* W0, double* E0, long* iterations)
{
    if (!g || !p || !W0 || !E0 || !(g->dx > 0.0) || !(p->Thin_Interface > 0.0)) return PF_E_ARG;
    // DO EPSLON_Try = 0, 1, 0.0000001 -- a REAL DO loop: trip count fixed up
    // front, variable advanced by adding the (REAL(4)) step each trip.
    const double lambda = p->Thin_Interface * g->dx;
    const double inc = (double)0.0000001f;
    const long trips = (long)((1.0 - 0.0 + inc) / inc);
    const float as = p->ajuste * p->Sigma;           // REAL(4) product
    const double k1 = 1.5556349186104 / lambda;
    double e = 0.0, w = 0.0, E = 0.0;
    long n = 0;
    while (n < trips) {
        const double t = k1 * e;
        w = t * t;
        E = (double)as * 4.24264068711929 / std::sqrt(w);
        ++n;
        if (std::fabs(E - e) < 1e-5) break;
        e = e + inc;
    }
    *W0 = w;
    *E0 = E;
    if (iterations) *iterations = n;
    return PF_OK;
}

extern "C" int pf_auxiliar_scalar(const pf_params* p, double E0, double W0, double TP, double Cs_eq, double Cl_eq,
                                  double* M0)
{
    if (!p || !M0) return PF_E_ARG;
    // repeated trapezoid over phi_i = 0.11, 0.12, ... <= 0.8999 (auxiliar.f90:15-29)
    double sum = 0.0;
    double ph = 0.11;
    do {
        const double hp = ph * ph * (3.0 - 2.0 * ph);
        const double f1 = ph * (1.0 - ph);
        const double numer = hp * (1.0 - hp);
        const double denom = ((1.0 - hp) * Cl_eq * (1.0 - Cl_eq) + hp * Cs_eq * (1.0 - Cs_eq)) * f1;
        sum = sum + numer / denom;
        ph = ph + 0.01;
    } while (ph <= 0.8999);
    // end points hard-coded; 0.01 and 54.39180136 are REAL(4) literals (:31)
    const double integral = ((double)0.01f / 2.0) * ((double)54.39180136f + 2.0 * sum + 234.073053);
    const double qsi = p->R * TP * (1.0 / p->Vm) * (Cl_eq - Cs_eq) * (Cl_eq - Cs_eq) * integral;
    const float omk = 1.0f - p->Ke;                  // (1-Ke) evaluated in REAL(4)
    const double kin = (double)p->Beta * p->R * TP * (double)omk / (p->Vm * p->Me);
    const double dif = E0 * qsi / (p->D_liq * std::sqrt(2.0 * W0));
    const double inv = (E0 * E0 / (double)p->Sigma) * (kin + dif);
    *M0 = (double)p->ajuste * 1.0 / inv;
    return PF_OK;
}
