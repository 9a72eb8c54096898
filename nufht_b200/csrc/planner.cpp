// Host planner: order/tolerance parameters and the box partition of the (k, r) index
// rectangle.  Produces exactly the reference's boxes (src/fast_hankel_nufht.c:498-744);
// the reference scans the sorted grids linearly for the first element above a threshold
// (:454-466), which is std::upper_bound on a non-decreasing array.
#include <algorithm>
#include <cmath>

#include "nufht_internal.h"

namespace hankel {

bool is_integer(double x) { return std::fabs(x - std::nearbyint(x)) < 1e-12; }

bool is_odd_integer(double x) {
  if (!is_integer(x)) return false;
  return (std::llround(x) & 1LL) != 0;
}

int check_grid(const double* a, int len) {
  for (int i = 0; i < len; ++i) {
    if (!std::isfinite(a[i]) || a[i] < 0.0) return -1;
    if (i > 0 && a[i] < a[i - 1]) return -1;
  }
  return 0;
}

int fill_params(double nu, const NufhtOptions& opt, bool extended, PlanParams* P) {
  if (opt.tol < 1e-15) return -1;
  bool is2 = is_integer(2.0 * nu), isi = is_integer(nu);
  if (!is2 || (isi && std::fabs(nu) > 200.0) || (!isi && is2 && std::fabs(nu) > 19.0 / 2.0))
    return -2;
  const Tables* T = extended ? tables_extended() : tables();
  int i_idx = (int)std::llround(std::fabs(nu));
  if (i_idx < 0 || i_idx >= NUFHT_MAX_I) return -3;
  int row = (int)std::llround(2.0 * std::fabs(nu) + 1.0) - 1;
  if (row < 0 || row >= NUFHT_NU_ROWS) return -4;
  for (int k = 0; k < NUFHT_MAX_COEF; ++k) P->asy_coef[k] = T->coef[row][k];
  int j = (int)std::ceil(-std::log10(opt.tol) - 3.0);
  if (j < 1) j = 1;
  int j_idx = j - 1;
  if (j_idx >= NUFHT_MAX_J) return -5;
  P->nu = nu;
  P->tol = opt.tol;
  if (isi) {
    int kv;
    if (opt.K_asy <= 0) {
      int k0 = (int)std::floor(std::fabs(nu) / 5.0 + std::log10(1.0 / opt.tol) / 4.0 + 1.0);
      kv = k0 < 10 ? k0 : 10;
    } else {
      kv = opt.K_asy;
    }
    if (kv < 0 || kv >= NUFHT_MAX_K) return -6;
    P->K_asy = kv;
    P->z_split = std::isnan(opt.z_split) ? T->z[i_idx][j_idx][kv] : opt.z_split;
    // switch points of the smaller term counts (entries the tables leave empty are unusable)
    P->n_z_terms = 0;
    for (int K = 0; K <= kv && K < 16; ++K) {
      const double zk = T->z[i_idx][j_idx][K];
      P->z_terms[K] = zk > 0.0 ? zk : HUGE_VAL;
    }
    P->n_z_terms = kv + 1 <= 16 ? kv + 1 : 16;
    P->K_loc = opt.K_loc <= 0 ? T->kw[i_idx][j_idx][kv] : opt.K_loc;
  } else {
    P->K_asy = (int)std::llround(std::fabs(nu) - 0.5);
    P->z_split = NAN;
    P->K_loc = -1;
  }
  return 0;
}

namespace {

// Index of the first element > thr in a non-decreasing array, or -1.
inline int first_greater(const double* a, int len, double thr) {
  const double* p = std::upper_bound(a, a + len, thr);
  return p == a + len ? -1 : (int)(p - a);
}

}  // namespace

void split_box_bs(const double* rs, int m, const double* ws, const HBox& b, double z,
                  int* ispl, int* jspl) {
  int cand[10], nc = 0;
  if (b.i1 <= b.i0) {
    cand[nc++] = b.i0;
  } else {
    for (int k = 0; k < 10; ++k) {
      double t = (double)k / 9.0;
      int idx = (int)std::llround(b.i0 + t * (double)(b.i1 - b.i0));
      idx = std::min(std::max(idx, b.i0), b.i1);
      if (nc == 0 || idx != cand[nc - 1]) cand[nc++] = idx;
    }
  }
  long long best = -1;
  int bi = b.i0;
  for (int c = 0; c < nc; ++c) {
    int i = cand[c];
    int j = first_greater(rs, m, z / ws[i]);
    long long v = 0;
    if (j >= 0)
      v = (long long)(i - b.i0 + 1) * (long long)(j - b.j0 + 1) +
          (long long)(b.i1 - i + 1) * (long long)(b.j1 - j + 1);
    if (v > best) {
      best = v;
      bi = i;
    }
  }
  int j = first_greater(rs, m, z / ws[bi]);
  if (j < 0) j = b.j0;
  *ispl = bi;
  *jspl = j;
}

void make_boxes(const double* rs, int m, const double* ws, int n, double z, int max_levels,
                int min_dim_prod, int Kthr, HBoxes* out) {
  out->loc.clear();
  out->asy.clear();
  out->dir.clear();
  if (n <= 0 || m <= 0) return;
  if (max_levels <= 0) {
    int mn = std::min(n, m);
    double ratio = (double)mn * (double)mn / (double)min_dim_prod;
    max_levels = ratio < 1.0 ? 0 : (int)std::floor(std::log2(ratio));
    if (max_levels < 0) max_levels = 0;
  }
  int i0 = first_greater(ws, n, z / rs[m - 1]), i1, j0, j1;
  if (m == 1) {
    i1 = i0 == -1 ? -1 : i0 - 1;
  } else {
    int idx = first_greater(ws, n, z / rs[0]);
    i1 = idx == -1 ? n - 1 : idx - 1;
  }
  j0 = first_greater(rs, m, z / ws[n - 1]);
  if (n == 1) {
    j1 = j0 == -1 ? -1 : j0 - 1;
  } else {
    int idx = first_greater(rs, m, z / ws[0]);
    j1 = idx == -1 ? m - 1 : idx - 1;
  }
  if (i0 == -1) {
    out->loc.push_back({0, n - 1, 0, m - 1});
    return;
  }
  if (i1 < 0) {
    out->asy.push_back({0, n - 1, 0, m - 1});
    return;
  }
  std::vector<HBox> loc, asy, dir;
  if (i0 > 0) loc.push_back({0, i0 - 1, 0, m - 1});
  if (j0 > 0) loc.push_back({i0, n - 1, 0, j0 - 1});
  if (i1 < n - 1) asy.push_back({i1 + 1, n - 1, 0, m - 1});
  if (j1 < m - 1) asy.push_back({0, i1, j1 + 1, m - 1});
  if (m == 1 || n == 1) {
    out->loc = loc;
    out->asy = asy;
    return;
  }
  dir.push_back({i0, i1, j0, j1});
  for (int lev = 0; lev < max_levels; ++lev) {
    std::vector<HBox> nd;
    nd.reserve(dir.size() * 2);
    for (const HBox& b : dir) {
      long long d1 = b.i1 - b.i0 + 1, d2 = b.j1 - b.j0 + 1;
      if (d1 * d2 > 4LL * (long long)min_dim_prod) {
        int is, js;
        split_box_bs(rs, m, ws, b, z, &is, &js);
        if (is > b.i0) {
          loc.push_back({b.i0, is - 1, b.j0, js - 1});
          nd.push_back({b.i0, is - 1, js, b.j1});
        }
        asy.push_back({is, b.i1, js, b.j1});
        nd.push_back({is, b.i1, b.j0, js - 1});
      } else {
        nd.push_back(b);
      }
    }
    dir.swap(nd);
  }
  for (const HBox& b : loc) {
    int d1 = b.i1 - b.i0 + 1, d2 = b.j1 - b.j0 + 1;
    if (std::min(d1, d2) < Kthr) dir.push_back(b);
    else out->loc.push_back(b);
  }
  for (const HBox& b : asy) {
    long long area = (long long)(b.i1 - b.i0 + 1) * (long long)(b.j1 - b.j0 + 1);
    if (area < (long long)min_dim_prod) dir.push_back(b);
    else out->asy.push_back(b);
  }
  out->dir = dir;
}

}  // namespace hankel
