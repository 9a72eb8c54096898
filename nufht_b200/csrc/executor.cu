// GPU executor of the batched NUFHT on B200 (sm_100a).
//
// A device plan holds device copies of the sorted grids rs (sources) and ws (targets),
// the reference's box partition turned into flat work lists, plan-time tables and a
// device workspace.  One transform g = H c runs as a fixed sequence of kernels on one
// stream:
//
//   local boxes      k_loc_proj -> k_loc_reduce -> k_loc_eval        (kernels_loc.cuh)
//   asymptotic boxes k_asy_spread -> cuFFT (Z2Z, one batched call per FFT length)
//                    -> k_asy_interp                                  (kernels_asy.cuh)
//   direct boxes     k_dir                                            (kernels_dir.cuh)
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "executor.h"
#include "kernels_asy.cuh"
#include "kernels_dir.cuh"
#include "kernels_loc.cuh"
#include "kernels_loc_mma.cuh"

namespace hankel {

std::atomic<long long> g_launch_counter{0};

// Optional per-phase device timing: CUDA events recorded on the launching stream around
// each phase of run(); read (and released) by phase_times().
std::atomic<bool> g_phase_timing{false};

// Local boxes on the SIMT kernels instead of the tensor-core ones (NUFHT_B200_LOC_SIMT=1; the
// tests compare the two forms).
const bool g_loc_simt = [] {
  const char* e = std::getenv("NUFHT_B200_LOC_SIMT");
  return e && e[0] == '1';
}();

// Direct boxes on the tensor-core kernel (Bessel tiles in shared memory, DMMA products;
// NUFHT_B200_DIR_MMA=1) instead of the SIMT one (one thread or a few lanes per target, the
// multiply-adds on the FP64 pipe), which measured faster on B200 (direct phase 3.0 against 4.8
// ms per step at the 1e6-point workload).
const bool g_dir_simt = [] {
  const char* e = std::getenv("NUFHT_B200_DIR_MMA");
  return !(e && e[0] == '1');
}();

// Sources per direct work item (NUFHT_B200_DIR_SOURCES, 256..16384, default kDirSources):
// each item adds its targets' partial sums into g with FP64 atomics, so fewer, longer items
// mean less atomic traffic, more items a better balance.
int dir_sources_per_item() {
  static const int v = [] {
    const char* e = std::getenv("NUFHT_B200_DIR_SOURCES");
    const int q = e ? std::atoi(e) : kDirSources;
    return (q >= 256 && q <= 16384) ? q : kDirSources;
  }();
  return v;
}

// Direct boxes evaluate J_nu directly instead of through the plan-time table
// (NUFHT_B200_DIR_NO_TABLE=1).
const bool g_dir_no_table = [] {
  const char* e = std::getenv("NUFHT_B200_DIR_NO_TABLE");
  return e && e[0] == '1';
}();

namespace {

std::mutex g_phase_mu;
struct PhaseMark {
  int phase;
  cudaEvent_t a, b;
};
std::vector<PhaseMark> g_phase_marks;

}  // namespace

void phase_record(int phase, cudaEvent_t a, cudaEvent_t b) {
  std::lock_guard<std::mutex> lk(g_phase_mu);
  g_phase_marks.push_back({phase, a, b});
}

namespace {

template <typename T>
int upload(const std::vector<T>& h, T** d) {
  *d = nullptr;
  if (h.empty()) return 0;
  NUFHT_CUDA_TRY(cudaMalloc((void**)d, h.size() * sizeof(T)));
  NUFHT_CUDA_TRY(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

// Smallest 2^a 3^b 5^c >= n (lengths cuFFT handles with its fastest radices).
long long fft_len(long long n) {
  long long best = LLONG_MAX;
  for (long long p2 = 1; p2 < 2 * n + 2; p2 *= 2)
    for (long long p3 = p2; p3 < 2 * n + 2; p3 *= 3)
      for (long long p5 = p3; p5 < 2 * n + 2; p5 *= 5)
        if (p5 >= n && p5 < best) best = p5;
  return best;
}

void gauss_legendre(int n, double* x, double* w) {
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

double host_es(double u, int W, double beta) {
  double z = 2.0 * u / W;
  double s = 1.0 - z * z;
  return s > 0.0 ? std::exp(beta * (std::sqrt(s) - 1.0)) : 0.0;
}

int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

// Direct boxes with the same sources and adjacent targets (or the same targets and adjacent
// sources) merged into one: the sum over the union is the same, each source's coefficients
// are staged once instead of once per box, and each target's partial sums are added into g
// once.  Sibling boxes of the partition often qualify (at the 1e6-point workload 483 boxes
// become 260, with 17% fewer summed sources and targets).
void merge_direct_boxes(std::vector<HBox>* boxes) {
  std::vector<HBox>& bs = *boxes;
  for (bool changed = true; changed;) {
    changed = false;
    std::sort(bs.begin(), bs.end(), [](const HBox& a, const HBox& b) {
      return a.j0 != b.j0 ? a.j0 < b.j0 : (a.j1 != b.j1 ? a.j1 < b.j1 : a.i0 < b.i0);
    });
    std::vector<HBox> out;
    for (const HBox& b : bs) {
      if (!out.empty() && out.back().j0 == b.j0 && out.back().j1 == b.j1 && out.back().i1 + 1 == b.i0) {
        out.back().i1 = b.i1;
        changed = true;
      } else {
        out.push_back(b);
      }
    }
    std::sort(out.begin(), out.end(), [](const HBox& a, const HBox& b) {
      return a.i0 != b.i0 ? a.i0 < b.i0 : (a.i1 != b.i1 ? a.i1 < b.i1 : a.j0 < b.j0);
    });
    bs.clear();
    for (const HBox& b : out) {
      if (!bs.empty() && bs.back().i0 == b.i0 && bs.back().i1 == b.i1 && bs.back().j1 + 1 == b.j0) {
        bs.back().j1 = b.j1;
        changed = true;
      } else {
        bs.push_back(b);
      }
    }
  }
}

// Expansion-term classes per oversampling class: NLP = 2, 4, ..., 2 kNlpClasses.
constexpr int kNlpClasses = kMaxNLP / 2;

// Asymptotic boxes split by expansion terms (NUFHT_B200_TERM_SPLIT=0 turns it off: every box
// then takes the plan's 2 (K_asy + 1) terms, as the reference does).
const bool term_split = [] {
  const char* e = std::getenv("NUFHT_B200_TERM_SPLIT");
  return !(e && e[0] == '0');
}();

// Oversampling factors tried for each asymptotic box.  sigma = 2 keeps the kernel
// narrow (spreading-bound boxes with many points per cell); smaller sigma shrinks the
// grid and the FFT (memory-bound boxes with few points per cell).
const double kSigmas[3] = {2.0, 1.5, 1.25};

// psi-hat(0) / psi-hat(pi / sigma) for the three oversampling classes: the factor by which
// deconvolution amplifies rounding at the edge of the band.
const double kKappa[3] = {3.0, 26.0, 1100.0};

// Worst-case error of the asymptotic boxes in FP32 arithmetic, per unit ||c||_1 (all of c
// on one source), for deconvolution amplification kappa.  Every FP32 stage rounds relative
// to the magnitude of the expansion term it carries, and term lp of a box is at most
// |coef_lp| x^-(lp+1/2) per unit |c_j| with x = k r >= k_lo rref over the box, so
//   err = max over boxes of  kFp32Err kappa sum_lp sqrt(2/pi) |a_lp| x_min^-(lp+1/2),
// kFp32Err fitted to single-source columns on B200 (the measured error stayed below 0.9 of
// the model over orders 0 to 25, half-integer orders and tolerances 1e-6 to 1e-8).
double fp32_error_bound(const DevicePlan& D, double kappa) {
  constexpr double kFp32Err = 5e-7;
  const int NLP = 2 * (D.P.K_asy + 1);
  const double s2p = std::sqrt(2.0 / M_PI);
  const double* rs = D.h_rs.data();
  const double* ws = D.h_ws.data();
  double err = 0.0;
  for (size_t q = 0; q < D.asy_eval.size(); ++q) {
    const HBox& hb = D.asy_eval[q];
    const int nlp = q < D.asy_eval_nlp.size() ? D.asy_eval_nlp[q] : NLP;
    const double* p = std::upper_bound(rs + hb.j0, rs + hb.j1 + 1, 0.0);
    if (p > rs + hb.j1) continue;  // only sources at r = 0: nothing to evaluate
    const double x = ws[hb.i0] * *p;
    if (!(x > 0.0)) continue;
    double sum = 0.0;
    for (int lp = 0; lp < nlp && lp < 64; ++lp) sum += s2p * std::fabs(D.P.asy_coef[lp]) * std::pow(x, -(lp + 0.5));
    err = std::max(err, kFp32Err * kappa * sum);
  }
  return err;
}

// Wimp degree the local boxes need.  Term l of the expansion is b_l(z) C_l with
// |b_l(z)| <= |J_{l0+odd+l}(z)| <= (z/2)^n / n!  (n = l0+odd+l; |J_m| <= 1) and
// |C_l| <= 2 ||c||_1 (|T_l| <= 1, weight <= 2), so all terms from l = L+1 on add at most
//   2 ||c||_1 sum_{n >= n0} (z/2)^n / n!  <=  2 ||c||_1 (z/2)^n0 / n0! / (1 - z / (2 (n0+1))),
// n0 = l0+odd+L+1, at the largest z = k r_end / 2 of any local box.  The degree is the
// table's K_loc, lowered to the smallest L whose tail stays below 1e-3 tol ||c||_1 (large
// orders: K_loc = 551 at nu = 100, tol 1e-8, while z < 80 needs about 80 terms).
int wimp_degree_needed(const PlanParams& P, const std::vector<HBox>& boxes, const double* rs, const double* ws) {
  const int K = P.K_loc;
  if (K <= 0 || boxes.empty()) return std::max(K, 0);
  double zmax = 0.0;
  for (const HBox& hb : boxes) zmax = std::max(zmax, ws[hb.i1] * rs[hb.j1] / 2.0);
  if (!(zmax > 0.0)) return 0;
  const int nu_int = (int)std::llround(std::fabs(P.nu));
  const int base = nu_int / 2 + (nu_int & 1);  // l0 + odd
  const double lh = std::log(zmax / 2.0);
  const double target = std::log(1e-3 * P.tol / 2.0);
  for (int L = 0; L < K; ++L) {
    const int n0 = base + L + 1;
    const double q = zmax / (2.0 * (n0 + 1.0));
    if (q >= 1.0) continue;
    const double lt = n0 * lh - std::lgamma(n0 + 1.0) - std::log1p(-q);
    if (lt <= target) return L;
  }
  return K;
}

// Kernel shape for oversampling sigma and width W: beta = 2.30 W at sigma = 2 (the
// value of Barnett, Magland & af Klinteberg 2019), 0.97 pi (1 - 1/(2 sigma)) W otherwise.
double es_beta(double sigma, int W) {
  return sigma == 2.0 ? 2.30 * W : 0.97 * M_PI * (1.0 - 1.0 / (2.0 * sigma)) * W;
}

AsyConst make_asy_const(const PlanParams& P, int NLP, int W, double beta) {
  AsyConst A;
  std::memset(&A, 0, sizeof(A));
  A.NLP = NLP;
  A.beta = beta;
  double anu = std::fabs(P.nu);
  double ph = M_PI * (-anu / 2.0 - 0.25);
  A.cos_phi = std::cos(ph);
  A.sin_phi = std::sin(ph);
  double s2p = std::sqrt(2.0 / M_PI);
  for (int lp = 0; lp < NLP && lp < kMaxNLP; ++lp) {
    int l = lp / 2;
    A.coef[lp] = s2p * ((l & 1) ? -1.0 : 1.0) * P.asy_coef[lp];
  }
  A.nq = std::min(2 * W + 16, kMaxQuad);
  double gx[kMaxQuad], gw[kMaxQuad];
  gauss_legendre(A.nq, gx, gw);
  for (int q = 0; q < A.nq; ++q) {
    A.qx[q] = (gx[q] + 1.0) * 0.25 * W;
    A.qwpsi[q] = gw[q] * 0.25 * W * host_es(A.qx[q], W, beta);
  }
  return A;
}

// Expansion terms an asymptotic box needs: the smallest 2 (K + 1) whose table switch point
// z_terms[K] is at most the box's smallest argument x_min = k_lo r_ref, never more than the
// plan's 2 (K_asy + 1).
int terms_needed(const PlanParams& P, int NLP, double xmin) {
  for (int K = 0; K < P.n_z_terms && 2 * (K + 1) < NLP; ++K)
    if (xmin >= P.z_terms[K]) return 2 * (K + 1);
  return NLP;
}

// Split of the asymptotic boxes by expansion terms.  The reference evaluates every
// asymptotic box with the K_asy + 1 term pairs that its smallest arguments (k r near z_split)
// need; most of a large box lies at far larger k r, where fewer pairs meet the same
// tolerance (the table's switch points for smaller K).  A box is cut along r at
// r = z_terms[K] / k_lo or along k at k = z_terms[K] / r_ref when the modelled time of the two
// parts (each with its own term count) is below the whole box's; the parts are split again
// (greedily, a few levels).  Model per column, from B200 phase times at the 1e6-point
// workload: spreading 71 ps per source and term, interpolation 99 ps per target and term,
// FFT and grid traffic 288 ps per grid cell and term (sigma = 2).
struct TermBox {
  HBox b;
  int nlp;
};

// Cost model of an asymptotic box for the term split (seconds at 32 columns on B200): per
// source-term, target-term and cell-term, and per source and per target of the box
// independent of its terms (record copies and the walks' control).  NUFHT_B200_SPLIT_MODEL
// ("a,b,c,d,e" in picoseconds) replaces the fitted values (tuning).
const double* split_model() {
  static const std::vector<double> m = [] {
    std::vector<double> v = {71e-12, 99e-12, 288e-12, 0.0, 0.0};
    if (const char* e = std::getenv("NUFHT_B200_SPLIT_MODEL")) {
      double q[5];
      if (std::sscanf(e, "%lf,%lf,%lf,%lf,%lf", &q[0], &q[1], &q[2], &q[3], &q[4]) == 5)
        for (int i = 0; i < 5; ++i) v[i] = q[i] * 1e-12;
    }
    return v;
  }();
  return m.data();
}

void split_by_terms(const PlanParams& P, int NLP, int W, const double* rs, const double* ws, const HBox& hb,
                    int depth, std::vector<TermBox>* out) {
  auto rref_of = [&](int j0, int j1) {
    const double* p = std::upper_bound(rs + j0, rs + j1 + 1, 0.0);
    return p <= rs + j1 ? *p : 0.0;
  };
  auto model = [&](const HBox& b, int* nlp_out) {
    const double rref = rref_of(b.j0, b.j1);
    const int nlp = rref > 0.0 ? terms_needed(P, NLP, ws[b.i0] * rref) : NLP;
    if (nlp_out) *nlp_out = nlp;
    const double X = 0.5 * (rs[b.j1] - rs[b.j0]);
    const double S = std::max(0.5 * (ws[b.i1] - ws[b.i0]), 1e-12 * std::max(std::fabs(ws[b.i0]), 1.0));
    const double half = std::ceil(X / (M_PI / (2.0 * S)) + 0.5 * W);
    const double n2 = 2.0 * (2.0 * half + 1.0);
    const double nj = b.j1 - b.j0 + 1, ni = b.i1 - b.i0 + 1;
    const double* m = split_model();
    return nlp * (m[0] * nj + m[1] * ni + m[2] * n2) + m[3] * nj + m[4] * ni;
  };
  int nlp0 = NLP;
  const double c0 = model(hb, &nlp0);
  if (P.n_z_terms == 0 || depth >= 6 || nlp0 <= 2) {
    out->push_back({hb, nlp0});
    return;
  }
  double best = c0;
  HBox a{}, b{};
  bool found = false;
  const double rref = rref_of(hb.j0, hb.j1);
  for (int K = 0; K < P.n_z_terms && 2 * (K + 1) < nlp0; ++K) {
    const double zk = P.z_terms[K];
    if (!std::isfinite(zk)) continue;
    // along r: sources with r >= z_K / k_lo need at most K + 1 pairs
    const int js = (int)(std::lower_bound(rs + hb.j0, rs + hb.j1 + 1, zk / ws[hb.i0]) - rs);
    if (js > hb.j0 && js <= hb.j1) {
      const HBox l{hb.i0, hb.i1, hb.j0, js - 1}, r{hb.i0, hb.i1, js, hb.j1};
      const double c = model(l, nullptr) + model(r, nullptr);
      if (c < best) {
        best = c;
        a = l;
        b = r;
        found = true;
      }
    }
    // along k: targets with k >= z_K / r_ref
    if (rref > 0.0) {
      const int is = (int)(std::lower_bound(ws + hb.i0, ws + hb.i1 + 1, zk / rref) - ws);
      if (is > hb.i0 && is <= hb.i1) {
        const HBox l{hb.i0, is - 1, hb.j0, hb.j1}, r{is, hb.i1, hb.j0, hb.j1};
        const double c = model(l, nullptr) + model(r, nullptr);
        if (c < best) {
          best = c;
          a = l;
          b = r;
          found = true;
        }
      }
    }
  }
  if (!found) {
    out->push_back({hb, nlp0});
    return;
  }
  split_by_terms(P, NLP, W, rs, ws, a, depth + 1, out);
  split_by_terms(P, NLP, W, rs, ws, b, depth + 1, out);
}

}  // namespace

int phase_times(double* ms, int nphase) {
  for (int p = 0; p < nphase; ++p) ms[p] = 0.0;
  std::lock_guard<std::mutex> lk(g_phase_mu);
  int cnt = 0;
  for (PhaseMark& mk : g_phase_marks) {
    cudaEventSynchronize(mk.b);
    float t = 0.f;
    if (cudaEventElapsedTime(&t, mk.a, mk.b) == cudaSuccess && mk.phase < nphase) ms[mk.phase] += t;
    cudaEventDestroy(mk.a);
    cudaEventDestroy(mk.b);
    ++cnt;
  }
  g_phase_marks.clear();
  return cnt;
}

// Kernel width for tolerance tol at oversampling sigma: ceil(log10(1/tol)) + 1 at
// sigma = 2, ceil(ln(10/tol) / (pi sqrt(1 - 1/sigma))) otherwise (0 if above 16).
int spread_width(double tol, double sigma) {
  int w;
  if (sigma == 2.0) {
    w = (int)std::ceil(std::log10(1.0 / tol)) + 1;
  } else {
    w = (int)std::ceil(std::log(10.0 / tol) / (M_PI * std::sqrt(1.0 - 1.0 / sigma)));
    if (w > 16) return 0;
  }
  return std::min(std::max(w, 2), 16);
}

int spread_width_for_tol(double tol) { return spread_width(tol, 2.0); }

// ------------------------------------------------------------------------------------
// Work lists.
// ------------------------------------------------------------------------------------
void DevicePlan::build_lists() {
  const double* rs = h_rs.data();
  const double* ws = h_ws.data();
  // ---- local boxes
  locb.clear();
  proj.clear();
  eval.clear();
  K_eval = wimp_degree_needed(P, loc_boxes, rs, ws);
  KL1 = K_eval + 1;
  for (size_t b = 0; b < loc_boxes.size(); ++b) {
    const HBox& hb = loc_boxes[b];
    LocBoxD d;
    d.i0 = hb.i0;
    d.ni = hb.i1 - hb.i0 + 1;
    d.j0 = hb.j0;
    d.nj = hb.j1 - hb.j0 + 1;
    d.r_end = rs[hb.j1];
    d.item0 = (int)proj.size();
    for (int j = hb.j0; j <= hb.j1; j += kLocSources)
      proj.push_back({(int)b, j, std::min(kLocSources, hb.j1 - j + 1)});
    d.nitems = (int)proj.size() - d.item0;
    for (int i = hb.i0; i <= hb.i1; i += kLocTargets)
      eval.push_back({(int)b, i, std::min(kLocTargets, hb.i1 - i + 1)});
    locb.push_back(d);
  }
  // ---- direct boxes: one target per thread for tall boxes, several for thin ones.
  // Asymptotic boxes with at most kThinDirect sources or targets are summed directly too:
  // there the pairs are few (at most kThinDirect per point) while the NUFFT would still
  // interpolate (or spread) every point for all NLP x B vectors.
  dir.clear();
  asy_direct.clear();
  asy_eval.clear();
  asy_eval_nlp.clear();
  W = spread_width(P.tol, 2.0);
  NLP = 2 * (P.K_asy + 1);
  {
    std::vector<TermBox> parts;
    for (const HBox& hb : asy_boxes) {
      const int ni = hb.i1 - hb.i0 + 1, nj = hb.j1 - hb.j0 + 1;
      if (std::min(ni, nj) <= kThinDirect) {
        asy_direct.push_back(hb);
        continue;
      }
      parts.clear();
      if (term_split) split_by_terms(P, NLP, W, rs, ws, hb, 0, &parts);
      else parts.push_back({hb, NLP});
      for (const TermBox& tb : parts) {
        const int pi = tb.b.i1 - tb.b.i0 + 1, pj = tb.b.j1 - tb.b.j0 + 1;
        if (std::min(pi, pj) <= kThinDirect) {
          asy_direct.push_back(tb.b);
        } else {
          asy_eval.push_back(tb.b);
          asy_eval_nlp.push_back(tb.nlp);
        }
      }
    }
  }
  std::vector<HBox> all_dir = dir_boxes;
  all_dir.insert(all_dir.end(), asy_direct.begin(), asy_direct.end());
  merge_direct_boxes(&all_dir);
  dir_thin = 0;
  dir_simt = g_dir_simt;
  if (dir_simt) {
    for (const HBox& hb : all_dir) {
      int ni = hb.i1 - hb.i0 + 1;
      int lanes = ni >= kDirThreads ? 1 : std::min(32, kDirThreads / next_pow2(ni));
      int tpc = kDirThreads / lanes;  // targets per CTA
      // The same number of sources per item for every shape: thin boxes (few targets, many
      // sources) split into many CTAs instead of a few long-running ones.
      const int spi = dir_sources_per_item();
      for (int i = hb.i0; i <= hb.i1; i += tpc)
        for (int j = hb.j0; j <= hb.j1; j += spi)
          dir.push_back({i, std::min(tpc, hb.i1 - i + 1), j, std::min(spi, hb.j1 - j + 1), lanes});
    }
  } else {
    // Tensor-core items: blocks of up to 64 targets x kDirMmaSources sources; blocks of at most
    // 16 targets take the thin tile shape and come first in the list.
    std::vector<DirItem> wide;
    for (const HBox& hb : all_dir)
      for (int i = hb.i0; i <= hb.i1; i += 64) {
        const int nb = std::min(64, hb.i1 - i + 1);
        std::vector<DirItem>& to = nb <= 16 ? dir : wide;
        for (int j = hb.j0; j <= hb.j1; j += kDirMmaSources)
          to.push_back({i, nb, j, std::min(kDirMmaSources, hb.j1 - j + 1), 0});
      }
    dir_thin = (int)dir.size();
    dir.insert(dir.end(), wide.begin(), wide.end());
  }
  // ---- asymptotic boxes
  asyb.clear();
  spread.clear();
  interp.clear();
  groups.clear();
  classes.clear();
  int Wc[3];
  for (int c = 0; c < 3; ++c) Wc[c] = spread_width(P.tol, kSigmas[c]);
  // In FP32 the deconvolution by psi-hat amplifies rounding by psi-hat(0)/psi-hat(pi/sigma):
  // about 3 at sigma = 2, 26 at 1.5 and 1100 at 1.25, so mixed precision keeps sigma = 2
  // unless NUFHT_B200_MIXED_SIGMAS lists the classes to allow (tuning: "2,1.5").  It runs
  // only where the modelled worst case of FP32 rounding stays within a quarter of the
  // tolerance (other plans evaluate their asymptotic boxes in FP64), unless the caller
  // accepts rounding that averages out over many sources (mixed_averaged).
  {
    static const int allowed = [] {
      const char* e = std::getenv("NUFHT_B200_MIXED_SIGMAS");
      int mask = 1;
      if (e) {
        if (std::strstr(e, "1.5")) mask |= 2;
        if (std::strstr(e, "1.25")) mask |= 4;
      }
      return mask;
    }();
    const double kappa = (allowed & 4) ? kKappa[2] : (allowed & 2) ? kKappa[1] : kKappa[0];
    fp32_err = fp32_error_bound(*this, kappa);
    if (mixed_asy && !mixed_averaged && fp32_err > 0.25 * P.tol) mixed_asy = false;
    if (mixed_asy) {
      if (!(allowed & 2)) Wc[1] = 0;
      if (!(allowed & 4)) Wc[2] = 0;
    }
  }
  std::vector<AsyBoxD> tmp;
  for (size_t q = 0; q < asy_eval.size(); ++q) {
    const HBox& hb = asy_eval[q];
    AsyBoxD d;
    std::memset(&d, 0, sizeof(d));
    d.nlp = asy_eval_nlp[q];
    d.i0 = hb.i0;
    d.i1 = hb.i1;
    d.j0 = hb.j0;
    d.j1 = hb.j1;
    double rlo = rs[hb.j0], rhi = rs[hb.j1], klo = ws[hb.i0], khi = ws[hb.i1];
    d.C = 0.5 * (rlo + rhi);
    // smallest positive radius of the box (sources at r = 0 contribute nothing here:
    // J_nu(0) = 0 for every order that reaches an asymptotic box)
    {
      const double* p = std::upper_bound(rs + hb.j0, rs + hb.j1 + 1, 0.0);
      d.rref = p <= rs + hb.j1 ? *p : 1.0;
    }
    double X = 0.5 * (rhi - rlo);
    d.D = 0.5 * (klo + khi);
    double S = 0.5 * (khi - klo);
    double Smin = 1e-12 * std::max(std::fabs(d.D), 1.0);
    if (S < Smin) S = Smin;
    // Choose the oversampling with the smallest modelled time: FP64 multiply-adds of
    // spreading and interpolation (2 W per point and vector) at ~20 T/s against ~7 passes
    // of 16-byte grid traffic per FFT cell and vector at ~6 TB/s.
    const double pts = (double)(hb.i1 - hb.i0 + 1) + (double)(hb.j1 - hb.j0 + 1);
    int best = 0;
    double best_t = 1e300;
    for (int c = 0; c < 3; ++c) {
      if (Wc[c] == 0) continue;
      double h = M_PI / (kSigmas[c] * S);
      double half = std::ceil(X / h + 0.5 * Wc[c]);
      double n2 = kSigmas[c] * (2.0 * half + 1.0);
      double t = pts * 2.0 * Wc[c] / 20e12 + n2 * 16.0 * 7.0 / 6e12;
      if (t < best_t * 0.97) {  // prefer larger sigma unless clearly cheaper
        best_t = t;
        best = c;
      }
    }
    const int Wb = Wc[best];
    const double sigma = kSigmas[best];
    d.cls = best * kNlpClasses + std::min(d.nlp / 2 - 1, kNlpClasses - 1);  // class: (oversampling, terms)
    d.h = M_PI / (sigma * S);
    long long half = (long long)std::ceil(X / d.h + 0.5 * Wb);
    d.half = (int)half;
    d.n2 = (int)fft_len(std::max<long long>((long long)std::ceil(sigma * (2 * half + 1)), (long long)kMinFft));
    // Dense boxes (many sources per grid cell) are spread by source chunks.
    auto l0_of = [&](int j) { return (long long)std::ceil((rs[j] - d.C) / d.h - 0.5 * Wb); };
    auto first_ge = [&](long long lo) {
      int a = d.j0, c = d.j1 + 1;
      while (a < c) {
        int mid = a + (c - a) / 2;
        if (l0_of(mid) >= lo) c = mid;
        else a = mid + 1;
      }
      return a;
    };
    // A box is dense when one of its tiles (the layout of the work items below) would have
    // more than kTileMaxSources sources.
    const int TC = kSpreadTile;
    int worst = 0;
    for (long long l = 0; l <= half; l += TC)
      worst = std::max(worst, first_ge(l + std::min<long long>(TC, half - l + 1)) - first_ge(l - Wb + 1));
    for (long long l = -1; l >= -half; l -= TC) {
      const long long lo = std::max(l - TC + 1, -half);
      worst = std::max(worst, first_ge(l + 1) - first_ge(lo - Wb + 1));
    }
    d.mode = worst > kTileMaxSources ? 1 : 0;
    tmp.push_back(d);
  }
  // Layout: groups of consecutive boxes with equal (mode, n2, terms), mode-1 groups first so
  // that their cells form one range to zero before spreading.
  std::vector<int> order(tmp.size());
  for (size_t q = 0; q < order.size(); ++q) order[q] = (int)q;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    if (tmp[a].mode != tmp[b].mode) return tmp[a].mode > tmp[b].mode;
    if (tmp[a].cls != tmp[b].cls) return tmp[a].cls < tmp[b].cls;
    return tmp[a].n2 < tmp[b].n2;
  });
  long long row = 0, coff = 0, poff = 0;
  long long roff = 0, rwoff = 0, rpoff = 0, twoff = 0, tmoff = 0;
  chunk_cell_begin = chunk_cell_end = 0;
  for (size_t q = 0; q < order.size();) {
    size_t e = q;
    while (e < order.size() && tmp[order[e]].n2 == tmp[order[q]].n2 && tmp[order[e]].mode == tmp[order[q]].mode &&
           tmp[order[e]].cls == tmp[order[q]].cls)
      ++e;
    FftGroup gr;
    gr.n2 = tmp[order[q]].n2;
    gr.nbox = (int)(e - q);
    gr.mode = tmp[order[q]].mode;
    gr.nlp = tmp[order[q]].nlp;
    gr.cls = tmp[order[q]].cls;
    gr.slot = 0;
    gr.cell_off = row;
    gr.plan = 0;
    for (size_t z = q; z < e; ++z) {
      AsyBoxD d = tmp[order[z]];
      d.cell_off = row;
      d.corr_off = coff;
      d.post_off = poff;
      coff += 2LL * d.half + 1;
      const long long ni = d.i1 - d.i0 + 1;
      d.tw_off = twoff;
      d.tm_off = tmoff;
      poff += ni;
      twoff += ni * (mixed_asy ? interp_we<float>(Wc[d.cls / kNlpClasses]) : interp_we<double>(Wc[d.cls / kNlpClasses]));
      tmoff += ni * d.nlp;
      row += (long long)d.n2 * d.nlp;
      // source records: first cells, W weights and nlp factors per source (factor rows of a
      // box start on a multiple of 4 values, for vector loads)
      const long long nj = d.j1 - d.j0 + 1;
      d.rec_off = roff;
      d.recw_off = rwoff;
      d.recp_off = rpoff;
      roff += nj;
      rwoff += nj * Wc[d.cls / kNlpClasses];
      rpoff += (nj * d.nlp + 3) / 4 * 4;
      asyb.push_back(d);
    }
    if (gr.mode == 1) chunk_cell_end = row;
    groups.push_back(gr);
    q = e;
  }
  total_cells = row;
  total_corr = coff;
  total_post = poff;
  total_rec = roff;
  total_recw = rwoff;
  total_recp = rpoff;
  total_tw = twoff;
  total_tm = tmoff;
  // Work items, grouped by kernel class: windowed spreading items (mode 0 tiles and mode 2
  // zero padding), then atomic ones (mode 1 chunks of dense boxes).
  std::vector<SpreadItem> atomic_items;
  for (int c = 0; c < 3 * kNlpClasses; ++c) {
    AsyClass K;
    K.sigma = kSigmas[c / kNlpClasses];
    K.W = Wc[c / kNlpClasses];
    K.nlp = 2 * (c % kNlpClasses + 1);
    K.spread0 = (int)spread.size();
    K.interp0 = (int)interp.size();
    bool any = false;
    // Sources per dense-box chunk: at most kChunkSources, fewer when the class's dense boxes
    // would otherwise give less than about four CTAs per SM (a chunk is one CTA walking its
    // sources in order).
    int chunk_src = kChunkSources;
    {
      long long dense = 0;
      for (const AsyBoxD& d : asyb)
        if (d.cls == c && d.mode == 1) dense += d.j1 - d.j0 + 1;
      if (dense > 0) {
        static const long long per_sm = [] {  // NUFHT_B200_CHUNK_CTAS (1..32, tuning)
          const char* e = std::getenv("NUFHT_B200_CHUNK_CTAS");
          const int v = e ? std::atoi(e) : 4;
          return (long long)((v >= 1 && v <= 32) ? v : 4);
        }();
        const long long want = dense / (148LL * per_sm);
        chunk_src = (int)std::min<long long>(kChunkSources, std::max<long long>(256, (want + 63) / 64 * 64));
      }
    }
    for (size_t b = 0; b < asyb.size(); ++b) {
      const AsyBoxD& d = asyb[b];
      if (d.cls != c) continue;
      any = true;
      const int Wb = K.W;
      auto l0_of = [&](int j) { return (long long)std::ceil((rs[j] - d.C) / d.h - 0.5 * Wb); };
      auto first_ge = [&](long long lo) {
        int a = d.j0, cc = d.j1 + 1;
        while (a < cc) {
          int mid = a + (cc - a) / 2;
          if (l0_of(mid) >= lo) cc = mid;
          else a = mid + 1;
        }
        return a;
      };
      if (d.mode == 0) {
        auto add_tile = [&](int l_start, int ncell, int fft_start) {
          SpreadItem s;
          s.box = (int)b;
          s.mode = 0;
          s.l_start = l_start;
          s.ncell = ncell;
          s.fft_start = fft_start;
          // sources whose support [l0, l0 + W) meets the tile's cells
          s.js = first_ge((long long)l_start - Wb + 1);
          s.je = first_ge((long long)l_start + ncell);
          spread.push_back(s);
        };
        const int TC = kSpreadTile;
        for (int l = 0; l <= d.half; l += TC) add_tile(l, std::min(TC, d.half - l + 1), l);
        for (int l = -1; l >= -d.half; l -= TC) {
          int lo = std::max(l - TC + 1, -d.half);
          add_tile(lo, l - lo + 1, d.n2 + lo);
        }
        for (int f = d.half + 1; f <= d.n2 - d.half - 1; f += 4 * TC) {
          SpreadItem s;
          s.box = (int)b;
          s.mode = 2;
          s.l_start = 0;
          s.fft_start = f;
          s.ncell = std::min(4 * TC, d.n2 - d.half - f);
          s.js = s.je = 0;
          spread.push_back(s);
        }
      } else {
        // Dense box: chunks of chunk_src sources, added atomically to the grid.
        for (int js = d.j0; js <= d.j1; js += chunk_src) {
          SpreadItem s;
          s.box = (int)b;
          s.mode = 1;
          s.l_start = 0;
          s.ncell = 0;
          s.fft_start = 0;
          s.js = js;
          s.je = std::min(js + chunk_src, d.j1 + 1);
          atomic_items.push_back(s);
        }
      }
      for (int i = d.i0; i <= d.i1; i += kInterpTile)
        interp.push_back({(int)b, i, std::min(i + kInterpTile, d.i1 + 1)});
    }
    K.nspread = (int)spread.size() - K.spread0;
    K.spreadA0 = (int)spread.size();
    spread.insert(spread.end(), atomic_items.begin(), atomic_items.end());
    K.nspreadA = (int)atomic_items.size();
    atomic_items.clear();
    K.ninterp = (int)interp.size() - K.interp0;
    if (any) {
      K.ac = make_asy_const(P, K.nlp, K.W, es_beta(K.sigma, K.W));
    }
    else std::memset(&K.ac, 0, sizeof(K.ac));
    classes.push_back(K);
  }
  // Stream slots: the classes with boxes in turn; each FFT group takes its class's slot.
  int nslot = 0;
  for (AsyClass& K : classes) K.slot = (K.nspread + K.nspreadA + K.ninterp > 0) ? nslot++ % (kAuxStreams - 2) : -1;
  for (FftGroup& gr : groups) gr.slot = std::max(0, classes[gr.cls].slot);
}

int DevicePlan::upload_all() {
  NUFHT_CUDA_TRY(cudaSetDevice(device));
  if (!d_rs) {  // the device planner uploads the grids first
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_rs, sizeof(double) * (size_t)m));
    NUFHT_CUDA_TRY(cudaMemcpy(d_rs, h_rs.data(), sizeof(double) * m, cudaMemcpyHostToDevice));
  }
  if (!d_ws) {
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_ws, sizeof(double) * (size_t)n));
    NUFHT_CUDA_TRY(cudaMemcpy(d_ws, h_ws.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  }
  int rc;
  if ((rc = upload(locb, &d_locb)) || (rc = upload(proj, &d_proj)) || (rc = upload(eval, &d_eval)) ||
      (rc = upload(dir, &d_dir)) || (rc = upload(asyb, &d_asyb)) || (rc = upload(spread, &d_spread)) ||
      (rc = upload(interp, &d_interp)))
    return rc;
  // J_nu table for the direct boxes where J_nu costs a recurrence over the order (integer
  // orders from 2, half-integer orders from 3/2), for their arguments k r below the table's
  // reach (larger arguments are evaluated directly).  Orders 0, 1 and 1/2 evaluate directly:
  // there the table's 128 bytes per pair, a different line for each lane of a tall box,
  // measured slower on B200 than the Chebyshev and Hankel forms (direct phase 2.97 against
  // 3.22 ms per step at the 1e6-point workload).
  if (!dir.empty() && nu2 >= 3 && !g_dir_no_table) {
    double xmax = 0.0;
    for (const DirItem& it : dir) xmax = std::max(xmax, h_ws[it.i0 + it.ni - 1] * h_rs[it.j0 + it.nj - 1]);
    jtab_n = (int)std::min<double>(std::ceil(xmax) + 1.0, (double)kJTabMaxIntervals);
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_jtab, sizeof(double) * (size_t)jtab_n * kJTabCoefs));
    k_build_jtable<<<jtab_n, kJTabCoefs>>>(nu2, d_jtab, jtab_n);
    NUFHT_LAUNCH_CHECK();
    NUFHT_CUDA_TRY(cudaDeviceSynchronize());
  }
  if (!asyb.empty()) {
    if (NLP > kMaxNLP) return NUFHT_E_TOO_LARGE;
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_corr, sizeof(double) * (size_t)total_corr));
    // Tables per box with the constants of the box's kernel class.
    for (size_t b0 = 0; b0 < asyb.size();) {
      size_t b1 = b0;
      while (b1 < asyb.size() && asyb[b1].cls == asyb[b0].cls && b1 - b0 < 65535) ++b1;
      const AsyConst& A = classes[asyb[b0].cls].ac;
      unsigned cnt = (unsigned)(b1 - b0);
      k_asy_setup_cells<<<dim3(64, cnt), 256>>>(d_asyb + b0, A, d_corr);
      NUFHT_LAUNCH_CHECK();
      b0 = b1;
    }
    const int rc2 = mixed_asy ? asy_records_f32(*this) : asy_records_f64(*this);
    if (rc2) return rc2;
    NUFHT_CUDA_TRY(cudaDeviceSynchronize());
  }
  return 0;
}

void DevicePlan::release_fft() {
  for (auto& kv : fft_cache)
    for (cufftHandle h : kv.second) cufftDestroy(h);
  fft_cache.clear();
  for (FftGroup& g : groups) g.plan = 0;
  fft_B = 0;
}

void DevicePlan::drop_buffer(void* p) {
  if (!p) return;
  if (pins > 0) retired.push_back(p);
  else cudaFree(p);
}

void DevicePlan::pin() { ++pins; }

void DevicePlan::unpin() {
  if (pins > 0) --pins;
  if (pins > 0 || retired.empty()) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaDeviceSynchronize();  // a launch of a released graph may still read them
  for (void* p : retired) cudaFree(p);
  retired.clear();
  if (prev >= 0) cudaSetDevice(prev);
}

DevicePlan::~DevicePlan() {
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  release_fft();
  cudaFree(d_rs); cudaFree(d_ws); cudaFree(d_locb); cudaFree(d_proj); cudaFree(d_eval);
  cudaFree(d_dir); cudaFree(d_asyb); cudaFree(d_spread); cudaFree(d_interp);
  cudaFree(d_corr); cudaFree(d_jtab);
  cudaFree(d_rec_l0); cudaFree(d_rec_w); cudaFree(d_rec_p); cudaFree(d_ct);
  cudaFree(d_tq0); cudaFree(d_tw); cudaFree(d_tmu);
  cudaFree(d_grid); cudaFree(d_partial); cudaFree(d_cheb); cudaFree(d_fft_work);
  for (void* p : retired) cudaFree(p);
  cudaFree(d_stage_c); cudaFree(d_stage_g); cudaFree(d_stage_t);
  for (int q = 0; q < kAuxStreams; ++q) {
    if (aux[q]) cudaStreamDestroy(aux[q]);
    if (ev_join[q]) cudaEventDestroy(ev_join[q]);
  }
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (copy_in) cudaStreamDestroy(copy_in);
  if (copy_out) cudaStreamDestroy(copy_out);
  for (int q = 0; q < 4; ++q) {
    if (ev_in[q]) cudaEventDestroy(ev_in[q]);
    if (ev_done[q]) cudaEventDestroy(ev_done[q]);
  }
  if (prev >= 0) cudaSetDevice(prev);
}

// FFT plans for batch size B: group g transforms nbox * V contiguous vectors of length n2.
// Plans are made once per batch size and kept (a captured batch graph may refer to the plans
// of any size it used); the shared work area only grows.
int DevicePlan::ensure_fft(int B) {
  if (asyb.empty() || B == fft_B) return 0;
  auto it = fft_cache.find(B);
  if (it == fft_cache.end()) {
    size_t need = 0;
    std::vector<cufftHandle> hs;
    auto destroy = [&]() {
      for (cufftHandle h : hs) cufftDestroy(h);
    };
    for (FftGroup& gr : groups) {
      cufftHandle h;
      if (cufftCreate(&h) != CUFFT_SUCCESS) {
        destroy();
        return NUFHT_E_CUDA;
      }
      hs.push_back(h);
      cufftSetAutoAllocation(h, 0);
      int nn = gr.n2;
      long long batch = (long long)gr.nbox * gr.nlp * B;
      if (batch > INT_MAX) {
        destroy();
        return NUFHT_E_TOO_LARGE;
      }
      size_t wsz = 0;
      if (cufftMakePlanMany(h, 1, &nn, nullptr, 1, nn, nullptr, 1, nn, mixed_asy ? CUFFT_C2C : CUFFT_Z2Z,
                            (int)batch, &wsz) != CUFFT_SUCCESS) {
        destroy();
        std::fprintf(stderr, "nufht_b200: cufftMakePlanMany failed (n=%d batch=%lld)\n", nn, batch);
        return NUFHT_E_CUDA;
      }
      need = std::max(need, wsz);
    }
    // One slice of the work area per stream slot: groups of different classes run
    // concurrently on their classes' streams.
    need = (need + 255) / 256 * 256;
    auto slice = [&](const FftGroup& gr) -> void* {
      return d_fft_work ? static_cast<char*>(d_fft_work) + (size_t)gr.slot * fft_slot_bytes : nullptr;
    };
    if (need > fft_slot_bytes) {
      drop_buffer(d_fft_work);
      d_fft_work = nullptr;
      fft_work_bytes = fft_slot_bytes = 0;
      const size_t bytes = need * (size_t)(kAuxStreams - 2);
      if (cudaMalloc(&d_fft_work, bytes) != cudaSuccess) {
        destroy();
        std::fprintf(stderr, "nufht_b200: cudaMalloc of %zu bytes of FFT work area failed\n", bytes);
        return NUFHT_E_CUDA;
      }
      fft_work_bytes = bytes;
      fft_slot_bytes = need;
      for (auto& kv : fft_cache)
        for (size_t g = 0; g < kv.second.size(); ++g) cufftSetWorkArea(kv.second[g], slice(groups[g]));
    }
    for (size_t g = 0; g < hs.size(); ++g) cufftSetWorkArea(hs[g], slice(groups[g]));
    it = fft_cache.emplace(B, std::move(hs)).first;
  }
  for (size_t g = 0; g < groups.size(); ++g) groups[g].plan = it->second[g];
  fft_B = B;
  return 0;
}

int DevicePlan::ensure_aux() {
  if (ev_fork) return 0;
  for (int q = 0; q < kAuxStreams; ++q) {
    NUFHT_CUDA_TRY(cudaStreamCreateWithFlags(&aux[q], cudaStreamNonBlocking));
    NUFHT_CUDA_TRY(cudaEventCreateWithFlags(&ev_join[q], cudaEventDisableTiming));
  }
  NUFHT_CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
  return 0;
}

// Fork: streams s[0..n) wait for the work queued so far on st.  Join: st waits for all of
// them.  Both are ordinary event records and waits, so they are captured into CUDA graphs as
// dependencies.
int fork_streams(DevicePlan& D, cudaStream_t st, const int* which, int n) {
  if (D.serial) return 0;
  NUFHT_CUDA_TRY(cudaEventRecord(D.ev_fork, st));
  for (int q = 0; q < n; ++q) NUFHT_CUDA_TRY(cudaStreamWaitEvent(D.aux[which[q]], D.ev_fork, 0));
  return 0;
}
int join_streams(DevicePlan& D, cudaStream_t st, const int* which, int n) {
  if (D.serial) return 0;
  for (int q = 0; q < n; ++q) {
    NUFHT_CUDA_TRY(cudaEventRecord(D.ev_join[which[q]], D.aux[which[q]]));
    NUFHT_CUDA_TRY(cudaStreamWaitEvent(st, D.ev_join[which[q]], 0));
  }
  return 0;
}

int DevicePlan::ensure_workspace(int B) {
  if (B <= ws_B) return ensure_fft(B);
  drop_buffer(d_grid); drop_buffer(d_partial); drop_buffer(d_cheb); drop_buffer(d_ct);
  d_grid = nullptr; d_partial = nullptr; d_cheb = nullptr; d_ct = nullptr;
  ws_B = 0;
  size_t bytes = 0;
  if (!asyb.empty()) {
    size_t g = (size_t)total_cells * (size_t)B * (mixed_asy ? sizeof(float2) : sizeof(double2));
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_grid, g));
    bytes += g;
    ldct = packed_ld(B);
    const size_t c = (size_t)m * (size_t)ldct * (mixed_asy ? sizeof(float) : sizeof(double));
    NUFHT_CUDA_TRY(cudaMalloc(&d_ct, c));
    bytes += c;
  }
  if (!locb.empty()) {
    size_t p = (size_t)proj.size() * KL1 * B * sizeof(double);
    size_t c = (size_t)locb.size() * KL1 * B * sizeof(double);
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_partial, p));
    NUFHT_CUDA_TRY(cudaMalloc((void**)&d_cheb, c));
    bytes += p + c;
  }
  ws_B = B;
  int rc = ensure_fft(B);
  ws_bytes = bytes + fft_work_bytes;
  return rc;
}

namespace {

int run_asy(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
            double sgn) {
  return D.mixed_asy ? run_asy_f32(D, cs, ld_cs, gs, ld_gs, B, st, sgn)
                     : run_asy_f64(D, cs, ld_cs, gs, ld_gs, B, st, sgn);
}

template <int BT>
int launch_dir(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B,
               cudaStream_t st, double sgn) {
  dim3 g((unsigned)D.dir.size(), (unsigned)((B + BT - 1) / BT));
  k_dir<BT><<<g, kDirThreads, 0, st>>>(D.d_rs, D.d_ws, cs, ld_cs, gs, ld_gs, B, D.d_dir, D.nu2, sgn, D.d_jtab,
                                       D.jtab_n);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

template <int ROWS, int NTN>
int launch_dir_mma_items(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B,
                         cudaStream_t st, double sgn, int item0, int nitems) {
  if (nitems <= 0) return 0;
  const size_t sm = DirMmaSmem<ROWS>::bytes(8 * NTN);
  static bool attr_set = false;
  if (!attr_set) {
    NUFHT_CUDA_TRY(cudaFuncSetAttribute(k_dir_mma<ROWS, NTN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    attr_set = true;
  }
  dim3 g((unsigned)nitems, (unsigned)((B + 8 * NTN - 1) / (8 * NTN)));
  k_dir_mma<ROWS, NTN><<<g, 128, sm, st>>>(D.d_rs, D.d_ws, cs, ld_cs, gs, ld_gs, B, D.d_dir + item0, D.nu2, sgn,
                                            D.d_jtab, D.jtab_n);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

template <int NTN>
int launch_dir_mma(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
                   double sgn) {
  int rc = launch_dir_mma_items<16, NTN>(D, cs, ld_cs, gs, ld_gs, B, st, sgn, 0, D.dir_thin);
  if (rc) return rc;
  return launch_dir_mma_items<64, NTN>(D, cs, ld_cs, gs, ld_gs, B, st, sgn, D.dir_thin,
                                       (int)D.dir.size() - D.dir_thin);
}

// Shared-memory budget of the local-expansion kernels (doubles).
constexpr size_t kLocSmemDoubles = 200 * 1024 / 8;

template <int MAXO>
int launch_loc_eval_t(const double* ws, double* gs, int ld_gs, int B, const LocBoxD* d_box, const EvalItem* d_eval,
                      int neval, const double* d_cheb, int K, int nu_int, double sgn, cudaStream_t st) {
  const int KL1 = K + 1;
  const int BTC = (int)std::max<size_t>(1, std::min<size_t>((size_t)B, kLocSmemDoubles / (size_t)KL1));
  const size_t sm = sizeof(double) * ((size_t)KL1 * BTC + kLocEvalCols);  // rows + register-block padding
  if (sm > 48 * 1024) cudaFuncSetAttribute(k_loc_eval<MAXO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_loc_eval<MAXO><<<(unsigned)neval, kLocTargets, sm, st>>>(ws, gs, ld_gs, B, d_box, d_eval, d_cheb, K, nu_int,
                                                            sgn, BTC);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

// Projection on the FP64 tensor cores (k_loc_proj_mma): CTAs of (source chunk item, block
// of up to 128 orders, block of up to 64 columns), so that every table entry a CTA fills
// serves all its columns; staged sources per round chosen for the shared-memory budget.
// Returns 1 when the layout does not fit (SIMT path then).
int launch_loc_proj_mma(const double* rs, const double* cs, int ld_cs, int B, const LocBoxD* d_box,
                        const ProjItem* d_proj, int nproj, double* d_partial, int KL1, int odd, cudaStream_t st) {
  const int MB = std::min(128, round8(KL1));
  const int BT = std::min(64, round8(B));
  const int tiles = (MB / 8) * (BT / 8);
  if (tiles > kLocMmaWarps * 16) return 1;
  int chunk = 128;
  LocProjMma L = loc_proj_mma_layout(MB, BT, chunk);
  while (chunk > 4 && L.doubles() > (size_t)(100 * 1024 / 8)) {
    chunk -= 4;
    L = loc_proj_mma_layout(MB, BT, chunk);
  }
  if (L.doubles() > kLocSmemDoubles) return 1;
  const size_t sm = sizeof(double) * L.doubles();
  dim3 g((unsigned)nproj, (unsigned)((KL1 + MB - 1) / MB), (unsigned)((B + BT - 1) / BT));
  if (tiles <= kLocMmaWarps * 4) {
    if (sm > 48 * 1024) cudaFuncSetAttribute(k_loc_proj_mma<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_loc_proj_mma<4><<<g, kLocThreads, sm, st>>>(rs, cs, ld_cs, B, d_box, d_proj, KL1, odd, d_partial, L);
  } else {
    if (sm > 48 * 1024) cudaFuncSetAttribute(k_loc_proj_mma<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_loc_proj_mma<16><<<g, kLocThreads, sm, st>>>(rs, cs, ld_cs, B, d_box, d_proj, KL1, odd, d_partial, L);
  }
  NUFHT_LAUNCH_CHECK();
  return 0;
}

// Evaluation on the FP64 tensor cores (k_loc_eval_mma): the largest tile of targets (128,
// 32, 16 or 8) whose Bessel table fits in 100 KB of shared memory (two CTAs per SM), else
// the largest that fits at all.  Returns 1 when even 8 targets do not fit.
template <int TI>
int launch_loc_eval_mma_t(const double* ws, double* gs, int ld_gs, int B, const LocBoxD* d_box, const EvalItem* d_eval,
                          int neval, const double* d_cheb, int K, int nu_int, double sgn, const LocEvalMma& L,
                          cudaStream_t st) {
  const size_t sm = sizeof(double) * L.doubles();
  if (sm > 48 * 1024) cudaFuncSetAttribute(k_loc_eval_mma<TI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_loc_eval_mma<TI><<<(unsigned)neval, kLocThreads, sm, st>>>(ws, gs, ld_gs, B, d_box, d_eval, d_cheb, K, nu_int, sgn,
                                                               L);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

int launch_loc_eval_mma(const double* ws, double* gs, int ld_gs, int B, const LocBoxD* d_box, const EvalItem* d_eval,
                        int neval, const double* d_cheb, int K, int nu_int, double sgn, cudaStream_t st) {
  const int maxo = nu_int / 2 + K + (nu_int & 1);
  // The tile with the most targets resident per SM (shared memory decides how many CTAs
  // fit); at equal counts the one with more CTAs per SM, so that one CTA's Bessel recurrences
  // overlap another's products.
  const int tis[4] = {128, 32, 16, 8};
  int pick = -1, best = 0, best_ctas = 0;
  for (int q = 0; q < 4; ++q) {
    const size_t bytes = sizeof(double) * loc_eval_mma_layout(tis[q], maxo).doubles();
    if (bytes > sizeof(double) * kLocSmemDoubles) continue;
    const int ctas = (int)std::min<size_t>(8, (size_t)(224 * 1024) / (bytes + 1024));
    const int per_sm = tis[q] * ctas;
    if (per_sm > best || (per_sm == best && ctas > best_ctas)) {
      best = per_sm;
      best_ctas = ctas;
      pick = tis[q];
    }
  }
  if (pick < 0) return 1;
  const LocEvalMma L = loc_eval_mma_layout(pick, maxo);
  switch (pick) {
    case 128: return launch_loc_eval_mma_t<128>(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, L, st);
    case 32: return launch_loc_eval_mma_t<32>(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, L, st);
    case 16: return launch_loc_eval_mma_t<16>(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, L, st);
    default: return launch_loc_eval_mma_t<8>(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, L, st);
  }
}

// The local-expansion kernels over `nbox` boxes (g += their contribution): projection per
// source chunk, reduction of the partial projections per box, evaluation at the targets.
// Both contractions run on the FP64 tensor cores; the SIMT kernels remain for Wimp degrees
// beyond their tile limits.
int launch_loc(const double* rs, const double* ws, const double* cs, int ld_cs, double* gs, int ld_gs, int B,
               const LocBoxD* d_box, int nbox, const ProjItem* d_proj, int nproj, const EvalItem* d_eval, int neval,
               double* d_partial, double* d_cheb, int K, int nu_int, double sgn, cudaStream_t st) {
  const int KL1 = K + 1;
  const int maxo = nu_int / 2 + K + (nu_int & 1);
  if (KL1 > kLocThreads * kLocMaxNL || maxo > 2304) return NUFHT_E_TOO_LARGE;
  {
    PhaseScope ps(kPhaseLocProj, st);
    int rc = g_loc_simt ? 1 : launch_loc_proj_mma(rs, cs, ld_cs, B, d_box, d_proj, nproj, d_partial, KL1, nu_int & 1, st);
    if (rc < 0) return rc;
    if (rc == 1) {
      // columns per projection CTA: the widest power of two (<= 32, <= B) for which each
      // thread owns one order, or, for very large degrees, at most kLocMaxNL orders
      const int cap = KL1 <= kLocThreads ? kLocThreads : kLocThreads * kLocMaxNL;
      int BT = 32;
      while (BT > 1 && KL1 * BT > cap) BT >>= 1;
      BT = std::max(1, std::min(BT, B));
      const int LS = kLocThreads / BT;
      const int NL = (KL1 + LS - 1) / LS;
      if (NL > kLocMaxNL) return NUFHT_E_TOO_LARGE;
      // sources per staging round: even (the projection reads the table in 16-byte pairs)
      const int chunk = (int)std::min<size_t>(kLocChunk, kLocSmemDoubles / (size_t)(KL1 + BT)) & ~1;
      if (chunk < 2) return NUFHT_E_TOO_LARGE;
      const size_t sm = sizeof(double) * ((size_t)KL1 * chunk + (size_t)chunk * BT);
      dim3 g((unsigned)nproj, (unsigned)((B + BT - 1) / BT));
      if (NL == 1) {
        if (sm > 48 * 1024) cudaFuncSetAttribute(k_loc_proj<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_loc_proj<1><<<g, kLocThreads, sm, st>>>(rs, cs, ld_cs, B, d_box, d_proj, KL1, nu_int & 1, d_partial, BT,
                                                 chunk);
      } else {
        if (sm > 48 * 1024)
          cudaFuncSetAttribute(k_loc_proj<kLocMaxNL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_loc_proj<kLocMaxNL><<<g, kLocThreads, sm, st>>>(rs, cs, ld_cs, B, d_box, d_proj, KL1, nu_int & 1,
                                                          d_partial, BT, chunk);
      }
      NUFHT_LAUNCH_CHECK();
    }
    long long tot = (long long)nbox * KL1 * B;
    k_loc_reduce<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(d_box, nbox, KL1, B, d_partial, d_cheb);
    NUFHT_LAUNCH_CHECK();
  }
  PhaseScope ps(kPhaseLocEval, st);
  if (!g_loc_simt) {
    int rc = launch_loc_eval_mma(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, st);
    if (rc <= 0) return rc;
  }
  if (maxo <= 64) return launch_loc_eval_t<64>(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, st);
  if (maxo <= 160) return launch_loc_eval_t<160>(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, st);
  if (maxo <= 640) return launch_loc_eval_t<640>(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, st);
  if (maxo <= 1280)
    return launch_loc_eval_t<1280>(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, st);
  return launch_loc_eval_t<2304>(ws, gs, ld_gs, B, d_box, d_eval, neval, d_cheb, K, nu_int, sgn, st);
}

}  // namespace

int DevicePlan::run(const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
                    bool zero_output) {
  NUFHT_CUDA_TRY(cudaSetDevice(device));
  int rc = ensure_workspace(B);
  if (rc) return rc;
  if ((rc = ensure_aux())) return rc;
  // With per-phase timing on, everything runs in order on st (the phase times then add up to
  // the transform's time; concurrent phases would overlap in time and share the GPU).
  serial = g_phase_timing.load(std::memory_order_relaxed);
  if (zero_output) {
    PhaseScope ps(kPhaseZero, st);
    NUFHT_CUDA_TRY(cudaMemset2DAsync(gs, sizeof(double) * (size_t)ld_gs, 0, sizeof(double) * (size_t)n, B, st));
  }
  const double sgn = sign;
  // The three box families add into g with atomics and share no workspace, so the local and
  // direct boxes run on their own streams beside the asymptotic ones (the FP64 Bessel work of
  // the direct boxes overlaps the memory-bound FFT and grid passes).
  const int side[2] = {0, 1};
  if ((rc = fork_streams(*this, st, side, 2))) return rc;
  const cudaStream_t s_loc = serial ? st : aux[0], s_dir = serial ? st : aux[1];
  if (!locb.empty()) {
    rc = launch_loc(d_rs, d_ws, cs, ld_cs, gs, ld_gs, B, d_locb, (int)locb.size(), d_proj, (int)proj.size(), d_eval,
                    (int)eval.size(), d_partial, d_cheb, K_eval, nu2 / 2, sgn, s_loc);
    if (rc) return rc;
  }
  if (!dir.empty()) {
    PhaseScope ps(kPhaseDir, s_dir);
    if (!dir_simt) {
      if (B >= 25) rc = launch_dir_mma<4>(*this, cs, ld_cs, gs, ld_gs, B, s_dir, sgn);
      else if (B >= 17) rc = launch_dir_mma<3>(*this, cs, ld_cs, gs, ld_gs, B, s_dir, sgn);
      else if (B >= 9) rc = launch_dir_mma<2>(*this, cs, ld_cs, gs, ld_gs, B, s_dir, sgn);
      else rc = launch_dir_mma<1>(*this, cs, ld_cs, gs, ld_gs, B, s_dir, sgn);
    } else if (B >= 32) rc = launch_dir<32>(*this, cs, ld_cs, gs, ld_gs, B, s_dir, sgn);
    else if (B >= 16) rc = launch_dir<16>(*this, cs, ld_cs, gs, ld_gs, B, s_dir, sgn);
    else if (B >= 8) rc = launch_dir<8>(*this, cs, ld_cs, gs, ld_gs, B, s_dir, sgn);
    else if (B >= 4) rc = launch_dir<4>(*this, cs, ld_cs, gs, ld_gs, B, s_dir, sgn);
    else rc = launch_dir<1>(*this, cs, ld_cs, gs, ld_gs, B, s_dir, sgn);
    if (rc) return rc;
  }
  if (!asyb.empty()) {
    rc = run_asy(*this, cs, ld_cs, gs, ld_gs, B, st, sgn);
    if (rc) return rc;
  }
  return join_streams(*this, st, side, 2);
}

// The local-expansion kernels of one box on caller-provided device buffers (work lists,
// partial projections and coefficients), without any allocation; g += the box's
// contribution.  Used by the allocation-free entry point (noalloc.cu).
int run_loc_box(const double* rs, const double* ws, const double* cs, int ld_cs, double* gs, int ld_gs,
                int B, const LocBoxD* d_box, const ProjItem* d_proj, int nproj, const EvalItem* d_eval,
                int neval, double* d_partial, double* d_cheb, int K, int nu_int, double sgn, cudaStream_t st) {
  return launch_loc(rs, ws, cs, ld_cs, gs, ld_gs, B, d_box, 1, d_proj, nproj, d_eval, neval, d_partial, d_cheb, K,
                    nu_int, sgn, st);
}

int run_besselj(double nu, const double* x, double* out, long count, cudaStream_t st) {
  double anu = std::fabs(nu);
  int nu2 = (int)std::llround(2.0 * anu);
  if (std::fabs(2.0 * anu - nu2) > 1e-12) return -2;
  if ((nu2 & 1) == 0 && nu2 / 2 > 200) return -2;
  if ((nu2 & 1) && nu2 > 19) return -2;
  if (count <= 0) return 0;
  k_besselj<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(nu2, x, out, count);
  NUFHT_LAUNCH_CHECK();
  return 0;
}

}  // namespace hankel
