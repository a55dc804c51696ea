/* kem_oracle.h -- plain-C restatement of KEMField's electrostatic BEM hot path (test
 * infrastructure only; the product never links it). See kem_oracle.c for the reference
 * file:line each function follows. Element encoding as include/kemcu.h. */
#ifndef KEM_ORACLE_H
#define KEM_ORACLE_H

#include <stddef.h>

/* rule tables: node (s, t, w) triples of the six cubature rules and (x, w) pairs of the two
   Gauss-Legendre half rules, as the reference tabulates them (taken from the reference's
   own GaussPoints_* functions on canonical elements) */
void kemo_set_rules(const double* tri7, const double* tri12, const double* tri33, const double* rect7,
                    const double* rect12, const double* rect33, const double* gl4, const double* gl16);
void kemo_set_constants(double one_over_four_pi_eps0, double eps0);

/* normalised (sigma = 1) field and potential of one element at P: out[4] = Ex, Ey, Ez, phi
   (shapes 0-2 planar; 3 conic section, 4 ring: the analytic axisymmetric integrators) */
void kemo_element(int shape, const double* geom11, const double* P, double* out4);
/* Kahan-summed direct sum over n elements at m points (out: m x 4) */
void kemo_field(size_t n, const int* shape, const double* geom, const double* sigma, size_t m, const double* P,
                double* out);
/* boundary-integral matrix A (n x n, row-major) and right-hand side */
void kemo_matrix(size_t n, const int* shape, const int* boundary, const double* geom, const double* value,
                 double* A, double* b);
/* GMRES (MGS, Givens, back-substitution) on a dense matrix; returns iterations */
int kemo_gmres(size_t n, const double* A, const double* b, double tol, int max_iter, double* x, double* resid);
/* nsteps RK8 steps of one particle in the field of the elements; state[8] in/out */
void kemo_rk8(size_t n, const int* shape, const double* geom, const double* sigma, double* state, double dt,
              int nsteps, double charge, double mass, double* traj);

#endif
