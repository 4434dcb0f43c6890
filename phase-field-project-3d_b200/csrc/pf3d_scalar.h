// pf3d_scalar.h -- host FP64 scalar helpers shared by the context and batch code.
#pragma once
#include "../../include/pf3d.h"

namespace pf3d {
void setup_derived(const pf_grid& g, const pf_params& p, pf_derived& out);
double initial_tp(const pf_params& p);
double step_tp(const pf_params& p, double dt, int it, double tp_prev);
void equilibrium(const pf_params& p, double TP, double* Cs_eq, double* Cl_eq);
}  // namespace pf3d
