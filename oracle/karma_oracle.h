/*
 * karma_oracle.h -- CPU oracle (test infrastructure only) of the quantitative
 * Karma model of karma/karma3d.f90.  See karma_oracle.c.
 */
#ifndef KARMA_ORACLE_H
#define KARMA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_karma {
    int nx, ny, nz;
    double lambda, eps4, dx, dt, Fnoise, k, D;
    /* (nx+2)(ny+2)(nz+2) arrays with the ghost layer, i fastest */
    double *phi, *phin, *U, *Un, *dphi;
    int it;
} orc_karma;

double orc_karma_ruido(int i, int j, int k, int it);
orc_karma* orc_karma_create(int nx, int ny, int nz, double lambda, double eps4, double dx, double dt, double Fnoise,
                            double k);
void orc_karma_destroy(orc_karma* s);
void orc_karma_set(orc_karma* s, const double* phi, const double* U);
void orc_karma_get(const orc_karma* s, double* phi, double* U, double* dphi);
void orc_karma_step(orc_karma* s, int n);
void orc_karma_set_it(orc_karma* s, int it);   /* steps done (noise counter) */
void orc_karma_tip(const orc_karma* s, int* tip_x, int* tip_d);

#ifdef __cplusplus
}
#endif
#endif
