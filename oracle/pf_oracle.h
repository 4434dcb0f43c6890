/*
 * pf_oracle.h -- CPU oracle (test infrastructure only) for the coupled explicit
 * time step of ileaof/phase-field-project-3D.  See pf_oracle.c.
 */
#ifndef PF_ORACLE_H
#define PF_ORACLE_H
#include "../include/pf3d.h"

#ifdef __cplusplus
extern "C" {
#endif

/* the deck parameters use the public pf_params layout */
typedef pf_params orc_params;

typedef struct orc_state {
    int nx, ny, nz;
    double dx, dy, dz;
    orc_params p;
    /* the seven resident fields, Fortran order */
    double *phi_old, *phi_new, *c_old, *c_new, *T_old, *T_new, *dpp;
    /* module scalars */
    double dt, AAA, Lambda, W0, E0, TP, M0, Cs_eq, Cl_eq;
    long w0e0_iters;
    int it;
    float time;
} orc_state;

double orc_pseudo_random(int i, int j, int k, int it, int salt);
double orc_ruido_suave(int i, int j, int k, int it);
void orc_w0_e0(double Lambda, float ajuste, float Sigma, double* W0, double* E0, long* iters);
double orc_auxiliar(const orc_params* p, double TP, double Cs_eq, double Cl_eq, double E0, double W0);

orc_state* orc_create(int nx, int ny, int nz, double dx, double dy, double dz, const orc_params* p);
void orc_destroy(orc_state* s);
double* orc_field(orc_state* s, int field);
void orc_set_field(orc_state* s, int field, const double* src);
void orc_get_field(orc_state* s, int field, double* dst);

void orc_temperatura(orc_state* s);
void orc_equacao_campo_fase(orc_state* s);
void orc_copy_phase_new_to_old(orc_state* s);
void orc_concentracao_soluto(orc_state* s);
void orc_diagnosticos(const orc_state* s, double out[5]);
void orc_swap(orc_state* s);
void orc_step(orc_state* s);
void orc_run(orc_state* s, int nsteps);
void orc_get_scalars(const orc_state* s, double out[10]);
void orc_set_scalars(orc_state* s, int it, double TP, double M0, float time);
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
