/*
 * nufht_oracle.h -- CPU oracle for the batched nonuniform fast Hankel transform.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * library's algorithm (Ansal06/NUFHT: src/fast_hankel_nufht.c, src/expansions.c)
 * used as the parity checker for the CUDA product and as the timed CPU baseline.
 * Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline and
 * reference arms) may load it.  The product library never links or calls it.
 *
 * Third-party arithmetic the reference delegates to, and what stands in here:
 *   - GSL gsl_sf_bessel_Jn / gsl_sf_bessel_Jnu (version not pinned by the
 *     reference): integer orders use the C library's jn() (POSIX), half-integer
 *     orders a spherical-Bessel restatement; both are pinned against mpmath
 *     values committed under tests/golden/.
 *   - FINUFFT finufft1d3 / finufft1d3many (version not pinned): either an exact
 *     O(n m) evaluation of sum_j c_j exp(+i k r_j) (mode ORACLE_T3_EXACT, the
 *     parity mode) or a type-3 NUFFT with the exponential-of-semicircle kernel
 *     of Barnett, Magland & af Klinteberg (SIAM J. Sci. Comput. 2019) and a
 *     radix-2 FFT (mode ORACLE_T3_NUFFT, used for timing the CPU baseline).
 */
#ifndef NUFHT_ORACLE_H
#define NUFHT_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_T3_EXACT = 0, ORACLE_T3_NUFFT = 1 };

/* Table cache in the reference's binary format (src/fast_hankel_nufht.c:183-312). */
int oracle_load_tables(const char *path);

/* Plan parameters: restates fill_plan_parameters (src/fast_hankel_nufht.c:322-414).
 * Returns 0 or the reference's negative codes -1..-6. */
int oracle_plan_params(double nu, double tol, double z_opt, int K_asy_opt, int K_loc_opt,
                       double *z_split, int *K_asy, int *K_loc, double *asy_coef64);

/* Box partition: restates generate_boxes (src/fast_hankel_nufht.c:578-744).
 * Writes box counts to counts[3] = {loc, asy, dir}; boxes (4 ints each, loc then asy
 * then dir) to out if cap (in boxes) suffices.  Returns total box count. */
long oracle_generate_boxes(const double *rs, int m, const double *ws, int n,
                           double z_split, int max_levels, int min_dim_prod, int K_loc_threshold,
                           long *counts, int *out, long cap);

/* Restated evaluators (src/expansions.c).  Signatures follow the reference's. */
void oracle_add_dir(double *gs, double nu, const double *rs, const double *cs,
                    const double *ws, int m, int n);
void oracle_add_dir_batch(double *gs, double nu, const double *rs, const double *cs,
                          const double *ws, int m, int n, int batch, int ld_cs, int ld_gs);
void oracle_add_loc(double *gs, double nu, const double *rs, const double *cs,
                    const double *ws, int m, int n, int K,
                    double *cheb_buffer, double *bessel_buffer_1, double *bessel_buffer_2);
void oracle_add_loc_batch(double *gs, double nu, const double *rs, const double *cs,
                          const double *ws, int m, int n, int K, int batch, int ld_cs, int ld_gs,
                          double *cheb_buffer_batch, double *bessel_buffer_1,
                          double *bessel_buffer_2);
void oracle_add_asy(double *gs, double nu, const double *rs, const double *cs,
                    const double *ws, int m, int n, int K, double tol, const double *asy_coef,
                    double *real_buffer_1, double *real_buffer_2,
                    double *in_buffer, double *out_buffer);
void oracle_add_asy_batch(double *gs, double nu, const double *rs, const double *cs,
                          const double *ws, int m, int n, int K, double tol,
                          const double *asy_coef, int batch, int ld_cs, int ld_gs,
                          double *in_buffer, double *out_buffer);

/* Whole transform: restates nufht_batch (src/fast_hankel_nufht.c:989-1107) with the
 * plan built as nufht_plan_init (:759-786) builds it.
 * faithful != 0 keeps the reference's batch==1 double negation for odd nu < 0
 * (:916-920 then :1090-1095); faithful == 0 applies the sign once. */
int oracle_nufht_batch(double nu, const double *rs, int m, const double *ws, int n,
                       const double *cs, int ld_cs, double *gs, int ld_gs, int batch,
                       double tol, int max_levels, int min_dim_prod,
                       double z_opt, int K_asy_opt, int K_loc_opt, int faithful);

/* Independent FP64 ground truth g[i,t] = sum_j c[j,t] J_|nu|(k_i r_j) (sign of
 * J_{-n} = (-1)^n J_n for integer nu) at the listed target indices. */
void oracle_direct_sum(double nu, const double *rs, int m, const double *ws,
                       const double *cs, int ld_cs, int batch,
                       const long *idx, int nidx, double *out /* nidx x batch, col-major */);

void oracle_set_type3_mode(int mode);
int oracle_get_type3_mode(void);
/* Set the number of host threads the oracle may use (1 = faithful single thread). */
void oracle_set_threads(int nthreads);

/* Bessel functions used by the oracle (ORACLE ONLY). */
double oracle_besselj(double nu, double x);
void oracle_besselj_all(int nmax, double z, double *out);

/* Type-3 transform f_k = sum_j c_j exp(i s_k x_j) for ntr vectors (complex interleaved). */
int oracle_type3(int ntr, int nj, const double *xj, const double *cj, double eps,
                 int nk, const double *sk, double *fk);

#ifdef __cplusplus
}
#endif
#endif
