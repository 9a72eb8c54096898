// Internal declarations shared by the host planner, the tables and the CUDA executor.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "nufht_b200.h"

#define NUFHT_NU_ROWS 401
#define NUFHT_MAX_COEF 64
#define NUFHT_MAX_I 401
#define NUFHT_MAX_J 32
#define NUFHT_MAX_K 16

namespace hankel {

struct Tables {
  double coef[NUFHT_NU_ROWS][NUFHT_MAX_COEF];
  double z[NUFHT_MAX_I][NUFHT_MAX_J][NUFHT_MAX_K];
  int kw[NUFHT_MAX_I][NUFHT_MAX_J][NUFHT_MAX_K];
};

int tables_load(Tables* T, const char* path);
int tables_save(const Tables* T, const char* path);
const Tables* tables();
const Tables* tables_extended();
const char* tables_source();
void tables_regenerate_into(Tables* T);

struct PlanParams {
  double nu = 0, tol = 0, z_split = 0;
  int K_asy = 0, K_loc = -1;
  double asy_coef[64] = {0};
  // z_terms[K] (K <= K_asy, integer orders): the table's switch point for K + 1 term pairs at
  // this order and tolerance -- from there on K + 1 pairs of the Hankel expansion meet tol.
  // n_z_terms = 0 when unknown (half-integer orders, single boxes with a given K).
  double z_terms[16] = {0};
  int n_z_terms = 0;
};

// Order/tolerance validation and table lookup (fill_plan_parameters,
// src/fast_hankel_nufht.c:322-414).  Returns 0 or -1..-6.
int fill_params(double nu, const NufhtOptions& opt, bool extended, PlanParams* out);

struct HBox {
  int i0, i1, j0, j1;
};
struct HBoxes {
  std::vector<HBox> loc, asy, dir;
};

// generate_boxes (src/fast_hankel_nufht.c:578-744) with binary search on the sorted grids.
void make_boxes(const double* rs, int m, const double* ws, int n, double z, int max_levels,
                int min_dim_prod, int Kthr, HBoxes* out);
void split_box_bs(const double* rs, int m, const double* ws, const HBox& b, double z,
                  int* ispl, int* jspl);

// 0 when a[0..len) is finite, non-negative and non-decreasing.
int check_grid(const double* a, int len);
bool is_integer(double x);
bool is_odd_integer(double x);


}  // namespace hankel
