/*
 * CPU oracle for the Wilson-clover hot path - TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C (C11 + OpenMP) restatement of the reference algorithm
 * (YellowBicycleee/Qcu_Cg_Inverter, directory cg_inverter/), used by tests/,
 * the smoke check and bench.py's CPU-baseline legs as the checker. The product
 * library never links or calls it.
 *
 * Parity pins: the oracle is checked against the reference library itself,
 * compiled unmodified into oracle/_ref/ and run on a GPU; the outputs of those
 * runs are committed as golden fixtures under tests/golden/ together with the
 * script that made them.
 *
 * Layouts are the reference's own AoS layouts (complex = two doubles):
 *   gauge       [dir 4][parity 2][t][z][y][x/2][3][3]            (include/qcu_point.cuh:65-67)
 *   half spinor [t][z][y][x/2][spin 4][colour 3]                  (include/qcu_point.cuh:70-72)
 *   full spinor [parity 2][half spinor]                           (src/qcu_clover_dslash.cu:1001-1004)
 *   clover      [parity 2][t][z][y][x/2][block 2][6][6]           (include/qcu_point.cuh:89-91)
 * Parity 0 holds the even sites, (x+y+z+t) even; the full x coordinate of a
 * checkerboard site is x = 2*(x/2) + ((y+z+t+parity) & 1).
 */
#ifndef QCU_ORACLE_H
#define QCU_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- seeded synthetic fields (counter-based; same values on any thread count) ---- */
void orc_gauge_random(double* gauge, const int L[4], uint64_t seed, double eps);
void orc_gauge_unit(double* gauge, const int L[4]);
void orc_gauge_pure(double* gauge, const int L[4], uint64_t seed);  /* U_mu(x) = g(x) g(x+mu)^dag */
void orc_gauge_transform(double* out, const double* gauge, const double* g, const int L[4]);
void orc_su3_random_field(double* g, const int L[4], uint64_t seed); /* one SU(3) matrix per site */
void orc_spinor_random(double* psi, size_t nsites, uint64_t seed);
void orc_spinor_transform(double* out, const double* psi, const double* g, const int L[4]); /* full spinor */

/* ---- reference operators (kappa = kappa*c_sw = 1, periodic) ---- */
/* out(parity) = D_{parity,1-parity} in, dagger flips the sign of gamma
 * (src/qcu_clover_dslash.cu:570-772). bc_t multiplies hops across the t boundary. */
void orc_dslash(double* out_half, const double* in_half, const double* gauge, const int L[4],
                int parity, int dagger, double bc_t);
/* A = 1 + csw*T per site for both parities (src/qcu_clover_dslash.cu:173-458, 509-544). */
void orc_clover_build(double* clover, const double* gauge, const int L[4], double csw);
/* block-wise 6x6 inverse of both blocks of each of nsites sites (src/qcu_clover_dslash.cu:42-100). */
int orc_clover_invert(double* inv, const double* clover, size_t nsites);
/* in place psi <- blockdiag(B0,B1) psi per site (src/qcu_clover_dslash.cu:461-506). */
void orc_clover_apply(double* psi, const double* mat, size_t nsites);

/* complex BLAS on n complex numbers (src/qcu_complex_computation.cu:10-133) */
void orc_cdot(const double* x, const double* y, size_t n, double out[2]); /* sum conj(x)*y */
void orc_caxpy(double* y, const double* x, const double a[2], size_t n);  /* y += a*x */
void orc_cscale(double* x, const double a[2], size_t n);                  /* x *= a */

/* reference compositions on full spinors */
void orc_full_dslash_ref(double* out, const double* in, const double* gauge, const double* clover,
                         const double* clover_inv, const int L[4], int dagger);
void orc_new_full_ref(double* out, const double* in, const double* gauge, const double* clover_inv,
                      const int L[4], int dagger);
void orc_mmv_ref(double* out, const double* in, const double* gauge, const double* clover_inv,
                 const int L[4]);
void orc_invert_clover_ref(double* out, const double* clover_inv, const int L[4]);
/* the reference CG flow (src/cg_inverter.cu:181-369). Returns iterations done;
 * *converged set to 1 when the reference's own test passed. maxiter <= 0 -> V. */
int orc_cg_inverter_ref(double* x, const double* b, const double* gauge, const int L[4],
                        int maxiter, int* converged);

/* ---- extended physics: M = A(kappa*csw) - kappa*D, antiperiodic t via bc_t ---- */
void orc_apply_full(double* out, const double* in, const double* gauge, const double* clover,
                    const int L[4], double kappa, double bc_t, int dagger);
/* Even-odd Schur CGNR on Mhat^dag Mhat, Mhat = 1 - kappa^2 A_ee^-1 D_eo A_oo^-1 D_oe,
 * odd sites reconstructed. Stops when the true full residual |b-Mx|/|b| < tol, checked
 * where the iterated residual predicts it (see orc_solve_schur_cl).
 * Returns iterations; *true_res receives the final true relative residual. */
int orc_solve_schur(double* x, const double* b, const double* gauge, const int L[4], double kappa,
                    double csw, double bc_t, double tol, int maxiter, double* true_res);
/* The same with a prebuilt clover A (clover) and its inverse (clover_inv), so
 * that the setup is timed apart from the solve; *checks (may be NULL) receives
 * the number of true-residual checks. */
int orc_solve_schur_cl(double* x, const double* b, const double* gauge, const double* clover,
                       const double* clover_inv, const int L[4], double kappa, double bc_t, double tol,
                       int maxiter, double* true_res, int* checks);
/* The Schur operator and its adjoint on even half spinors (for operator tests). */
void orc_schur_apply(double* out, const double* in, const double* gauge, const double* clover_inv,
                     const int L[4], double kappa, double bc_t, int dagger);

int orc_num_threads(void);
void orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
