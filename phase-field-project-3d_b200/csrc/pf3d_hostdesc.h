// pf3d_hostdesc.h -- host helpers shared by the context and batch code:
// validation, pitched layout, the device descriptor of a domain and the
// per-step scalars (all FP64, the reference's expressions).
#pragma once
#include <cmath>
#include <cstring>
#include <string>
#include "../../include/pf3d.h"
#include "pf3d_launch.h"
#include "pf3d_scalar.h"

namespace pf3d {

inline void fill_desc(const pf_grid& g, const pf_params& p, const pf_derived& dv, int px, DomainDesc& d)
{
    std::memset(&d, 0, sizeof(d));
    d.nx = g.nx; d.ny = g.ny; d.nz = g.nz;
    d.px = px;
    d.plane = (long long)px * g.ny;
    d.dx = g.dx; d.dy = g.dy; d.dz = g.dz;
    d.E0 = dv.E0; d.W0 = dv.W0; d.DE = p.DELTA_EPSLON;
    d.K_aniso = 16.0 * dv.E0 * p.DELTA_EPSLON;       // phase_body.inc:49
    d.AAA = dv.AAA;
    d.Ke = (double)p.Ke;
    d.D_liq = p.D_liq; d.D_sol = p.D_sol;
    d.dt = dv.DELTA_T;
    d.dH_cp = p.delta_H / p.Cp_s;                     // temp_body.inc:36, cp = cp_s
    d.Ddt = p.D * dv.DELTA_T;                         // temp_body.inc:41
    d.cxy = 0.25 / (g.dx * g.dy);
    d.cyz = 0.25 / (g.dy * g.dz);
    d.czx = 0.25 / (g.dz * g.dx);
    d.dx2 = g.dx * g.dx; d.dy2 = g.dy * g.dy; d.dz2 = g.dz * g.dz;
    d.InvDX = 1.0 / (g.dx * g.dx); d.InvDY = 1.0 / (g.dy * g.dy); d.InvDZ = 1.0 / (g.dz * g.dz);
    d.hx = 0.5 / g.dx; d.hy = 0.5 / g.dy; d.hz = 0.5 / g.dz;
    d.rdx2 = 1.0 / (g.dx * g.dx); d.rdy2 = 1.0 / (g.dy * g.dy); d.rdz2 = 1.0 / (g.dz * g.dz);
    d.AAA16 = dv.AAA * 16.0;
    d.omKe = 1.0 - (double)p.Ke;
    d.dtIX = dv.DELTA_T * d.InvDX; d.dtIY = dv.DELTA_T * d.InvDY; d.dtIZ = dv.DELTA_T * d.InvDZ;
    d.hq = p.h_quintico;
    d.rt = p.ruido_tipo;
    d.do_heat_lap = (p.D != 0.0) ? 1 : 0;
}

inline StepArgs make_step_args(const pf_params& p, const pf_derived& dv, int it, double TP_heat, double TP, double M0)
{
    StepArgs s;
    std::memset(&s, 0, sizeof(s));
    double Cs, Cl;
    equilibrium(p, TP, &Cs, &Cl);
    s.it = it;
    s.TP_heat = TP_heat;
    s.TP = TP;
    s.M0dt = M0 * dv.DELTA_T;
    s.RTV = p.R * TP / p.Vm;
    s.omCs = 1.0 - Cs;
    s.omCl = 1.0 - Cl;
    s.Lc = std::log(s.omCs / s.omCl);
    return s;
}

inline int validate(const pf_grid* g, const pf_params* p, int precision, std::string& why)
{
    if (!g || !p) { why = "null grid or params"; return PF_E_ARG; }
    if (g->nx < 5 || g->ny < 5 || g->nz < 5) { why = "every grid dimension must be >= 5"; return PF_E_ARG; }
    if (!(g->dx > 0) || !(g->dy > 0) || !(g->dz > 0)) { why = "grid spacings must be > 0"; return PF_E_ARG; }
    if (precision != PF_FP64 && precision != PF_FP32) { why = "precision must be 64 or 32"; return PF_E_ARG; }
    if (!(p->D_liq > 0) || !(p->Cp_s != 0) || !(p->Me != 0) || !(p->Vm != 0)) { why = "D_liq, Cp_s, Me, Vm must be nonzero"; return PF_E_ARG; }
    if (p->n_varreduras < 1) { why = "n_varreduras must be >= 1"; return PF_E_ARG; }
    if (p->h_quintico != 0 && p->h_quintico != 1) { why = "h_quintico must be 0 or 1"; return PF_E_ARG; }
    if (p->ruido_tipo < 0 || p->ruido_tipo > 2) { why = "ruido_tipo must be 0, 1 or 2"; return PF_E_ARG; }
    if (p->bc != PF_BC_REFERENCE) { why = "only the reference boundary treatment is available"; return PF_E_ARG; }
    return PF_OK;
}

inline size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
inline int pitch_of(int nx) { return (int)round_up((size_t)nx, 32); }


}  // namespace pf3d
