// Device plan and work-list types of the GPU executor.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <atomic>
#include <map>
#include <mutex>
#include <vector>

#include "nufht_internal.h"

namespace hankel {

constexpr int kMaxNLP = 32;    // 2 (K_asy + 1) expansion terms per box, at most
constexpr int kMaxQuad = 48;   // quadrature nodes for the kernel's Fourier transform

struct LocBoxD {
  int i0, ni, j0, nj;
  double r_end;
  int item0, nitems;  // projection work items of this box
};
struct ProjItem { int box, j0, nj; };
struct EvalItem { int box, i0, ni; };
struct DirItem { int i0, ni, j0, nj; };

// Geometry of one asymptotic box's type-3 transform: sources x = r - C, targets s = k - D,
// spreading grid spacing h (cells l in [-half, half]), FFT length n2, and the offset of its
// grid (in cells per vector) in the workspace.
struct AsyBoxD {
  int i0, i1, j0, j1;
  double C, D, h;
  int half, n2;
  long long cell_off;
};
struct SpreadItem {
  int box, l_start, fft_start, ncell, js, je, padding;
};
struct InterpItem { int box, ks, ke; };
struct FftGroup {
  int n2, box0, nbox;
  long long cell_off;
};

struct AsyConst {
  int NLP;      // 2 (K + 1)
  int nq;       // quadrature nodes
  double beta;  // kernel shape
  double cos_phi, sin_phi;  // exp(i pi (-nu/2 - 1/4))
  double coef[kMaxNLP];     // sqrt(2/pi) (-1)^l a_{2l+p}, index 2l+p
  double qx[kMaxQuad];      // nodes on [0, W/2]
  double qwpsi[kMaxQuad];   // weight * psi(node)
};

int spread_width_for_tol(double tol);

struct DevicePlan {
  int device = 0;
  int flags = 0;
  PlanParams P;
  int m = 0, n = 0;
  int path = 0;   // 0 boxes, 1 all-direct, 2 all-asymptotic
  int nu2 = 0;    // 2 |nu|
  double sign = 1.0;
  std::vector<double> h_rs, h_ws;
  std::vector<HBox> loc_boxes, asy_boxes, dir_boxes;  // boxes as evaluated
  std::vector<HBox> plan_loc, plan_asy, plan_dir;     // the planner's partition

  // work lists
  int KL1 = 0, W = 0;
  std::vector<LocBoxD> locb;
  std::vector<ProjItem> proj;
  std::vector<EvalItem> eval;
  std::vector<DirItem> dir;
  std::vector<AsyBoxD> asyb;
  std::vector<SpreadItem> spread;
  std::vector<InterpItem> interp;
  std::vector<FftGroup> groups;
  long long total_cells = 0;
  AsyConst ac{};

  // device copies
  double *d_rs = nullptr, *d_ws = nullptr;
  LocBoxD* d_locb = nullptr;
  ProjItem* d_proj = nullptr;
  EvalItem* d_eval = nullptr;
  DirItem* d_dir = nullptr;
  AsyBoxD* d_asyb = nullptr;
  SpreadItem* d_spread = nullptr;
  InterpItem* d_interp = nullptr;

  // workspace, sized for the largest batch executed so far
  int ws_B = 0;
  size_t ws_bytes = 0;
  double2* d_grid = nullptr;
  double* d_partial = nullptr;
  double* d_cheb = nullptr;
  void* d_fft_work = nullptr;
  std::map<int, cufftHandle> fft_plans;

  // staging for host-pointer calls through the reference-compatible entry points
  double* d_stage_c = nullptr;
  double* d_stage_g = nullptr;
  size_t stage_c_bytes = 0, stage_g_bytes = 0;

  std::mutex mu;

  ~DevicePlan();
  void build_lists();
  int upload_all();
  int ensure_workspace(int B);
  // g (+)= H c on stream st; cs / gs are device pointers.
  int run(const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
          bool zero_output);
};

extern std::atomic<long long> g_launch_counter;

int run_besselj(double nu, const double* x, double* out, long count, cudaStream_t st);

}  // namespace hankel
