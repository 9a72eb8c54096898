/*
 * ref_glue.c -- TEST INFRASTRUCTURE ONLY.  Provides the evaluator symbols the reference's
 * own driver (src/fast_hankel_nufht.c, compiled unchanged from the reference tree into
 * oracle/_ref/) calls, so that the reference's planner and nufht_batch control flow run
 * here on top of the oracle's restated evaluators (GSL and FINUFFT are absent).
 */
#include "nufht_oracle.h"

void add_dir(double *gs, double nu, const double *rs, const double *cs, const double *ws,
             int m, int n)
{ oracle_add_dir(gs, nu, rs, cs, ws, m, n); }

void add_dir_batch(double *gs, double nu, const double *rs, const double *cs,
                   const double *ws, int m, int n, int batch, int ld_cs, int ld_gs)
{ oracle_add_dir_batch(gs, nu, rs, cs, ws, m, n, batch, ld_cs, ld_gs); }

void add_loc(double *gs, double nu, const double *rs, const double *cs, const double *ws,
             int m, int n, int K, double *b0, double *b1, double *b2)
{ oracle_add_loc(gs, nu, rs, cs, ws, m, n, K, b0, b1, b2); }

void add_loc_batch(double *gs, double nu, const double *rs, const double *cs,
                   const double *ws, int m, int n, int K, int batch, int ld_cs, int ld_gs,
                   double *b0, double *b1, double *b2)
{ oracle_add_loc_batch(gs, nu, rs, cs, ws, m, n, K, batch, ld_cs, ld_gs, b0, b1, b2); }

void add_asy(double *gs, double nu, const double *rs, const double *cs, const double *ws,
             int m, int n, int K, double tol, const double *coef, double *r1, double *r2,
             double *in, double *out)
{ oracle_add_asy(gs, nu, rs, cs, ws, m, n, K, tol, coef, r1, r2, in, out); }

void add_asy_batch(double *gs, double nu, const double *rs, const double *cs,
                   const double *ws, int m, int n, int K, double tol, const double *coef,
                   int batch, int ld_cs, int ld_gs, double *in, double *out)
{ oracle_add_asy_batch(gs, nu, rs, cs, ws, m, n, K, tol, coef, batch, ld_cs, ld_gs, NULL, NULL); }
