// C ABI of libnufht_b200.so: the reference library's entry points (src/fast_hankel_nufht.h)
// backed by the GPU executor, and this library's device-plan extension.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "capi_internal.h"
#include "executor.h"
#include "nufht_internal.h"

using hankel::DevicePlan;
using hankel::HBox;
using hankel::HBoxes;
using hankel::PlanParams;

namespace {

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int has_device() {
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt <= 0) {
    cudaGetLastError();
    return 0;
  }
  return 1;
}

// Host copy of a grid that may live on the device.
int host_copy(const double* p, int len, std::vector<double>* out) {
  out->resize((size_t)len);
  if (is_device_ptr(p)) {
    if (cudaMemcpy(out->data(), p, sizeof(double) * (size_t)len, cudaMemcpyDeviceToHost) != cudaSuccess)
      return NUFHT_E_CUDA;
  } else {
    std::memcpy(out->data(), p, sizeof(double) * (size_t)len);
  }
  return 0;
}

// Host view of a grid for planning: the caller's array itself when it is host memory, a copy
// read back when it is device memory.
int host_view(const double* p, int len, DevicePlan::HostGrid* out) {
  if (!is_device_ptr(p)) {
    out->borrow(p);
    return 0;
  }
  int rc = host_copy(p, len, &out->own);
  out->p = out->own.data();
  return rc;
}

std::vector<HBox> to_hbox(const BoxVector& v) {
  std::vector<HBox> out;
  for (size_t q = 0; q < v.length; ++q) out.push_back({v.data[q].i0, v.data[q].i1, v.data[q].j0, v.data[q].j1});
  return out;
}

BoxVector to_boxvec(const std::vector<HBox>& v) {
  BoxVector b;
  b.length = v.size();
  b.capacity = v.size();
  b.data = v.empty() ? nullptr : (Box*)std::malloc(sizeof(Box) * v.size());
  for (size_t q = 0; q < v.size(); ++q) b.data[q] = {v[q].i0, v[q].i1, v[q].j0, v[q].j1};
  return b;
}

// Smallest argument x from which the terminating Hankel expansion of J_{n+1/2},
//   J_{n+1/2}(x) = sqrt(2/(pi x)) (cos chi sum_{k even} (-1)^{k/2} a_k x^-k
//                                  - sin chi sum_{k odd} (-1)^{(k-1)/2} a_k x^-k),
//   a_k = prod_{i=1..k} (4 nu^2 - (2i-1)^2) / (k! 8^k),  a_k = 0 for k > n,
// is evaluated without cancellation: there the terms sum to at most kHalfTermSum in
// magnitude, so the asymptotic boxes' per-term tolerance is amplified at most that much (the
// integer-order boxes of the planner work at similar term sums, about 10 at z_split).  0 for
// nu = 1/2, whose expansion is the single term sin(x).
constexpr double kHalfTermSum = 8.0;
double half_integer_split(double anu) {
  const int n = (int)std::llround(anu - 0.5);
  if (n <= 0) return 0.0;
  std::vector<double> a(n + 1);
  a[0] = 1.0;
  for (int k = 1; k <= n; ++k) a[k] = a[k - 1] * (4.0 * anu * anu - (2.0 * k - 1) * (2.0 * k - 1)) / (8.0 * k);
  auto sum = [&](double x) {
    double s = 0.0, p = 1.0;
    for (int k = 0; k <= n; ++k, p /= x) s += std::fabs(a[k]) * p;
    return s;
  };
  double lo = 1e-6, hi = 1e6;
  for (int it = 0; it < 200 && hi - lo > 1e-12 * hi; ++it) {
    double mid = std::sqrt(lo * hi);
    if (sum(mid) > kHalfTermSum) lo = mid;
    else hi = mid;
  }
  return hi;
}

// Decide which evaluation path nufht_batch takes (src/fast_hankel_nufht.c:1018-1080) and
// fill the boxes the executor evaluates.  Half-integer orders: the reference evaluates the
// whole rectangle with the terminating expansion (:1052-1078), which cancels
// catastrophically at small k r for nu >= 3/2; here pairs with k r below
// half_integer_split(nu) are summed directly (the planner's partition at that z, local
// boxes included) and only the rest is asymptotic.
void choose_path(DevicePlan* D, int min_dim_prod) {
  long long dp = (long long)D->m * (long long)D->n;
  D->loc_boxes.clear();
  D->asy_boxes.clear();
  D->dir_boxes.clear();
  HBox whole{0, D->n - 1, 0, D->m - 1};
  if (dp < (long long)min_dim_prod) {
    D->path = 1;
    D->dir_boxes.push_back(whole);
  } else if (!hankel::is_integer(D->P.nu)) {
    D->path = 2;
    const double zh = half_integer_split(std::fabs(D->P.nu));
    if (zh <= 0.0) {
      D->asy_boxes.push_back(whole);
    } else {
      hankel::HBoxes hb;
      hankel::make_boxes(D->h_rs.data(), D->m, D->h_ws.data(), D->n, zh, 0, min_dim_prod, INT_MAX, &hb);
      D->asy_boxes = hb.asy;
      D->dir_boxes = hb.dir;
      D->dir_boxes.insert(D->dir_boxes.end(), hb.loc.begin(), hb.loc.end());
    }
  } else {
    D->path = 0;
    if (D->P.K_loc >= 0) D->loc_boxes = D->plan_loc;
    D->asy_boxes = D->plan_asy;
    D->dir_boxes = D->plan_dir;
  }
}

double wall_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

int finish_device_plan(DevicePlan* D, int device) {
  D->device = device;
  D->nu2 = (int)std::llround(2.0 * std::fabs(D->P.nu));
  D->sign = (D->P.nu < 0.0 && hankel::is_odd_integer(D->P.nu)) ? -1.0 : 1.0;
  const double t0 = wall_ms();
  D->build_lists();
  const double t1 = wall_ms();
  const int rc = D->upload_all();
  D->plan_ms[1] = t1 - t0;
  D->plan_ms[2] = wall_ms() - t1;
  // the host views may borrow the caller's arrays, which need not outlive planning
  D->h_rs.release();
  D->h_ws.release();
  return rc;
}

// The partition runs on the device unless NUFHT_B200_HOST_PLANNER=1 (the host planner then
// gives the same boxes; the tests compare the two).
bool use_device_planner() {
  const char* e = std::getenv("NUFHT_B200_HOST_PLANNER");
  return !(e && e[0] == '1');
}

// Grids of a device plan: device copies (uploaded from host pointers or copied from device
// pointers), validated and partitioned on the device, plus the host copies the work lists
// are built from.  Fills D->h_rs, D->h_ws, D->d_rs, D->d_ws and hb.
int device_grids_and_boxes(DevicePlan* D, const double* rs, const double* ws, const NufhtOptions& opt,
                           HBoxes* hb) {
  const int m = D->m, n = D->n;
  const double t0 = wall_ms();
  static const bool report = [] {
    const char* e = std::getenv("NUFHT_B200_PLAN_TIMING");
    return e && e[0] == '1';
  }();
  int rc;
  if ((rc = host_view(rs, m, &D->h_rs)) || (rc = host_view(ws, n, &D->h_ws))) return rc;
  const double t_copy = wall_ms();
  const int Kthr = D->P.K_loc < 0 ? 0 : D->P.K_loc;
  if (!use_device_planner()) {
    if (hankel::check_grid(D->h_rs.data(), m)) return NUFHT_E_UNSORTED_RS;
    if (hankel::check_grid(D->h_ws.data(), n)) return NUFHT_E_UNSORTED_WS;
    hankel::make_boxes(D->h_rs.data(), m, D->h_ws.data(), n, D->P.z_split, opt.max_levels, opt.min_dim_prod,
                       Kthr, hb);
    D->plan_ms[0] = wall_ms() - t0;
    return 0;
  }
  if (cudaMalloc((void**)&D->d_rs, sizeof(double) * (size_t)m) != cudaSuccess ||
      cudaMalloc((void**)&D->d_ws, sizeof(double) * (size_t)n) != cudaSuccess)
    return NUFHT_E_CUDA;
  if (cudaMemcpy(D->d_rs, D->h_rs.data(), sizeof(double) * m, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(D->d_ws, D->h_ws.data(), sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    return NUFHT_E_CUDA;
  const double t_up = wall_ms();
  int bad = 0;
  if ((rc = hankel::device_make_boxes(D->d_rs, m, D->d_ws, n, D->P.z_split, opt.max_levels, opt.min_dim_prod,
                                      Kthr, hb, 0, &bad)))
    return rc;
  if (bad) return bad == 1 ? NUFHT_E_UNSORTED_RS : NUFHT_E_UNSORTED_WS;
  D->partition_on_device = 1;
  D->plan_ms[0] = wall_ms() - t0;
  if (report)
    std::fprintf(stderr, "nufht_b200 plan: host copies %.2f ms, upload %.2f ms, validation + partition %.2f ms\n",
                 t_copy - t0, t_up - t_copy, wall_ms() - t_up);
  return 0;
}

// ---- registry of device state for reference-style plans (NufhtPlan has no spare field)
struct Entry {
  const double* rs;
  const double* ws;
  int m, n, K_asy, K_loc;
  double nu, tol, z_split;
  const Box *dl, *da, *dd;
  size_t nl, na, nd;
  std::unique_ptr<DevicePlan> dp;
};
std::mutex g_reg_mu;
std::map<const NufhtPlan*, std::unique_ptr<Entry>> g_reg;

bool entry_matches(const Entry& e, const NufhtPlan* p) {
  return e.rs == p->rs && e.ws == p->ws && e.m == p->m && e.n == p->n && e.K_asy == p->K_asy &&
         e.K_loc == p->K_loc && e.nu == p->nu && e.tol == p->tol &&
         (e.z_split == p->z_split || (std::isnan(e.z_split) && std::isnan(p->z_split))) &&
         e.dl == p->boxes.loc.data && e.da == p->boxes.asy.data && e.dd == p->boxes.dir.data &&
         e.nl == p->boxes.loc.length && e.na == p->boxes.asy.length && e.nd == p->boxes.dir.length;
}

int device_state_for(const NufhtPlan* plan, DevicePlan** out) {
  std::lock_guard<std::mutex> lk(g_reg_mu);
  auto it = g_reg.find(plan);
  if (it != g_reg.end() && entry_matches(*it->second, plan)) {
    *out = it->second->dp.get();
    return 0;
  }
  if (!has_device()) return NUFHT_E_NO_DEVICE;
  std::unique_ptr<Entry> e(new Entry);
  e->rs = plan->rs; e->ws = plan->ws; e->m = plan->m; e->n = plan->n;
  e->K_asy = plan->K_asy; e->K_loc = plan->K_loc; e->nu = plan->nu; e->tol = plan->tol;
  e->z_split = plan->z_split;
  e->dl = plan->boxes.loc.data; e->da = plan->boxes.asy.data; e->dd = plan->boxes.dir.data;
  e->nl = plan->boxes.loc.length; e->na = plan->boxes.asy.length; e->nd = plan->boxes.dir.length;
  std::unique_ptr<DevicePlan> D(new DevicePlan);
  D->m = plan->m;
  D->n = plan->n;
  D->P.nu = plan->nu; D->P.tol = plan->tol; D->P.z_split = plan->z_split;
  D->P.K_asy = plan->K_asy; D->P.K_loc = plan->K_loc;
  std::memcpy(D->P.asy_coef, plan->asy_coef, sizeof(plan->asy_coef));
  {
    // the table's switch points for fewer expansion terms at this order and tolerance
    NufhtOptions o = nufht_default_options();
    o.tol = plan->tol;
    PlanParams Q;
    if (hankel::fill_params(plan->nu, o, false, &Q) == 0) {
      std::memcpy(D->P.z_terms, Q.z_terms, sizeof(Q.z_terms));
      D->P.n_z_terms = std::min(Q.n_z_terms, plan->K_asy + 1);
    }
  }
  int rc;
  if ((rc = host_view(plan->rs, plan->m, &D->h_rs)) || (rc = host_view(plan->ws, plan->n, &D->h_ws)))
    return rc;
  D->plan_loc = to_hbox(plan->boxes.loc);
  D->plan_asy = to_hbox(plan->boxes.asy);
  D->plan_dir = to_hbox(plan->boxes.dir);
  // The reference's entry points carry no precision argument; NUFHT_B200_PRECISION=mixed
  // or mixed-averaged selects the mixed-precision asymptotic path for them (the rules of
  // NUFHT_B200_MIXED and NUFHT_B200_MIXED_AVERAGED).
  if (const char* pr = std::getenv("NUFHT_B200_PRECISION")) {
    D->mixed_averaged = std::strcmp(pr, "mixed-averaged") == 0;
    D->mixed_asy = (std::strcmp(pr, "mixed") == 0 || D->mixed_averaged) && D->P.tol >= 1e-9;
  }
  choose_path(D.get(), plan->min_dim_prod);
  int dev = 0;
  cudaGetDevice(&dev);
  if ((rc = finish_device_plan(D.get(), dev))) return rc;
  e->dp = std::move(D);
  *out = e->dp.get();
  g_reg[plan] = std::move(e);
  return 0;
}

void drop_device_state(const NufhtPlan* plan) {
  std::lock_guard<std::mutex> lk(g_reg_mu);
  g_reg.erase(plan);
}

// Run D on cs/gs that may be host or device pointers (synchronous, legacy stream).
// Device buffer of at least `need` bytes (grown, never shrunk).
int stage_buffer(double** buf, size_t* have, size_t need) {
  if (need <= *have) return 0;
  cudaFree(*buf);
  *buf = nullptr;
  *have = 0;
  if (cudaMalloc((void**)buf, need) != cudaSuccess) return NUFHT_E_CUDA;
  *have = need;
  return 0;
}

// Column blocks of the pipelined host-buffer path: the transfers of one block overlap the
// transform of another, so large calls are cut into 2 to 4 equal blocks (equal, so that
// the FFT plans made for one width serve every block) of at least 16 columns (narrower
// blocks spread and interpolate less efficiently).
int pipeline_blocks(const DevicePlan* D, int B) {
  static const int forced = [] {  // NUFHT_B200_PIPELINE_BLOCKS=1 turns the pipeline off (tuning)
    const char* e = std::getenv("NUFHT_B200_PIPELINE_BLOCKS");
    return e ? std::atoi(e) : 0;
  }();
  if (forced > 0) return (B % forced == 0) ? forced : 1;
  const double bytes = 8.0 * ((double)D->m + (double)D->n) * (double)B;
  if (bytes < 64.0 * 1024 * 1024) return 1;
  for (int nb : {4, 3, 2})
    if (B % nb == 0 && B / nb >= 16) return nb;
  return 1;
}

int run_any(DevicePlan* D, const double* cs, int ld_cs, double* gs, int ld_gs, int B, bool zero) {
  std::lock_guard<std::mutex> lk(D->mu);
  if (cudaSetDevice(D->device) != cudaSuccess) return NUFHT_E_CUDA;
  cudaStream_t st = 0;
  const bool cdev = is_device_ptr(cs), gdev = is_device_ptr(gs);
  int rc;
  if (cdev && gdev) {
    rc = D->run(cs, ld_cs, gs, ld_gs, B, st, zero);
    if (rc) return rc;
    return cudaStreamSynchronize(st) == cudaSuccess ? 0 : NUFHT_E_CUDA;
  }
  if ((rc = stage_buffer(&D->d_stage_c, &D->stage_c_bytes, cdev ? 0 : sizeof(double) * (size_t)D->m * B)) ||
      (rc = stage_buffer(&D->d_stage_g, &D->stage_g_bytes, gdev ? 0 : sizeof(double) * (size_t)D->n * B)))
    return rc;
  const double* dc = cdev ? cs : D->d_stage_c;
  double* dg = gdev ? gs : D->d_stage_g;
  const int ldc = cdev ? ld_cs : D->m, ldg = gdev ? ld_gs : D->n;
  const int nb = zero ? pipeline_blocks(D, B) : 1;
  if (nb == 1) {
    if (!cdev && cudaMemcpy2DAsync(D->d_stage_c, sizeof(double) * D->m, cs, sizeof(double) * (size_t)ld_cs,
                                   sizeof(double) * D->m, B, cudaMemcpyHostToDevice, st) != cudaSuccess)
      return NUFHT_E_CUDA;
    if (!gdev && !zero &&
        cudaMemcpy2DAsync(dg, sizeof(double) * D->n, gs, sizeof(double) * (size_t)ld_gs, sizeof(double) * D->n, B,
                          cudaMemcpyHostToDevice, st) != cudaSuccess)
      return NUFHT_E_CUDA;
    if ((rc = D->run(dc, ldc, dg, ldg, B, st, zero))) return rc;
    if (!gdev && cudaMemcpy2DAsync(gs, sizeof(double) * (size_t)ld_gs, dg, sizeof(double) * D->n,
                                   sizeof(double) * D->n, B, cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return NUFHT_E_CUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? 0 : NUFHT_E_CUDA;
  }
  // Pipelined: block q's host-to-device copy (copy_in), transform (st) and device-to-host
  // copy (copy_out) overlap the neighbouring blocks' stages.
  if (!D->copy_in) {
    if (cudaStreamCreateWithFlags(&D->copy_in, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&D->copy_out, cudaStreamNonBlocking) != cudaSuccess)
      return NUFHT_E_CUDA;
    for (int q = 0; q < 4; ++q)
      if (cudaEventCreateWithFlags(&D->ev_in[q], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&D->ev_done[q], cudaEventDisableTiming) != cudaSuccess)
        return NUFHT_E_CUDA;
  }
  const int Bc = B / nb;
  // the copy streams start after all earlier work on st (e.g. a previous call's transform)
  if (cudaEventRecord(D->ev_done[0], st) != cudaSuccess || cudaStreamWaitEvent(D->copy_in, D->ev_done[0], 0) ||
      cudaStreamWaitEvent(D->copy_out, D->ev_done[0], 0))
    return NUFHT_E_CUDA;
  for (int q = 0; q < nb; ++q) {
    if (!cdev) {
      if (cudaMemcpy2DAsync(D->d_stage_c + (size_t)q * Bc * D->m, sizeof(double) * D->m,
                            cs + (size_t)q * Bc * ld_cs, sizeof(double) * (size_t)ld_cs, sizeof(double) * D->m, Bc,
                            cudaMemcpyHostToDevice, D->copy_in) != cudaSuccess)
        return NUFHT_E_CUDA;
    }
    if (cudaEventRecord(D->ev_in[q], D->copy_in) != cudaSuccess) return NUFHT_E_CUDA;
  }
  for (int q = 0; q < nb; ++q) {
    if (cudaStreamWaitEvent(st, D->ev_in[q], 0) != cudaSuccess) return NUFHT_E_CUDA;
    if ((rc = D->run(dc + (size_t)q * Bc * ldc, ldc, dg + (size_t)q * Bc * ldg, ldg, Bc, st, true))) return rc;
    if (cudaEventRecord(D->ev_done[q], st) != cudaSuccess) return NUFHT_E_CUDA;
    if (!gdev) {
      if (cudaStreamWaitEvent(D->copy_out, D->ev_done[q], 0) != cudaSuccess ||
          cudaMemcpy2DAsync(gs + (size_t)q * Bc * ld_gs, sizeof(double) * (size_t)ld_gs,
                            D->d_stage_g + (size_t)q * Bc * D->n, sizeof(double) * D->n, sizeof(double) * D->n, Bc,
                            cudaMemcpyDeviceToHost, D->copy_out) != cudaSuccess)
        return NUFHT_E_CUDA;
    }
  }
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaStreamSynchronize(D->copy_out) != cudaSuccess ||
      cudaStreamSynchronize(D->copy_in) != cudaSuccess)
    return NUFHT_E_CUDA;
  return 0;
}

// nufht_batch with either layout of cs and gs (column-major with leading dimension ld, or
// row-major with row pitch ld >= B), host or device pointers, synchronous.  Row-major
// batches are transposed on the GPU (one contiguous host copy each way, no host-side
// transposes); the transform itself runs on column-major device buffers in one block.
int run_layout(DevicePlan* D, const double* cs, bool crow, int ld_cs, double* gs, bool grow, int ld_gs, int B) {
  std::lock_guard<std::mutex> lk(D->mu);
  if (cudaSetDevice(D->device) != cudaSuccess) return NUFHT_E_CUDA;
  cudaStream_t st = 0;
  const bool cdev = is_device_ptr(cs), gdev = is_device_ptr(gs);
  const size_t m = (size_t)D->m, n = (size_t)D->n;
  int rc;
  const bool need_t = (crow && !cdev) || (grow && !gdev);
  if ((rc = stage_buffer(&D->d_stage_c, &D->stage_c_bytes, (cdev && !crow) ? 0 : sizeof(double) * m * B)) ||
      (rc = stage_buffer(&D->d_stage_g, &D->stage_g_bytes, (gdev && !grow) ? 0 : sizeof(double) * n * B)) ||
      (rc = stage_buffer(&D->d_stage_t, &D->stage_t_bytes, need_t ? sizeof(double) * std::max(m, n) * B : 0)))
    return rc;
  // c -> column-major device matrix dc (leading dimension ldc)
  const double* dc = cs;
  int ldc = ld_cs;
  if (crow) {
    const double* src = cs;
    int lds = ld_cs;
    if (!cdev) {
      if (cudaMemcpy2DAsync(D->d_stage_t, sizeof(double) * B, cs, sizeof(double) * (size_t)ld_cs, sizeof(double) * B,
                            m, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return NUFHT_E_CUDA;
      src = D->d_stage_t;
      lds = B;
    }
    if ((rc = hankel::transpose_f64(src, lds, D->d_stage_c, D->m, D->m, B, st))) return rc;
    dc = D->d_stage_c;
    ldc = D->m;
  } else if (!cdev) {
    if (cudaMemcpy2DAsync(D->d_stage_c, sizeof(double) * m, cs, sizeof(double) * (size_t)ld_cs, sizeof(double) * m,
                          B, cudaMemcpyHostToDevice, st) != cudaSuccess)
      return NUFHT_E_CUDA;
    dc = D->d_stage_c;
    ldc = D->m;
  }
  // transform into a column-major device matrix dg
  double* dg = (gdev && !grow) ? gs : D->d_stage_g;
  const int ldg = (gdev && !grow) ? ld_gs : D->n;
  if ((rc = D->run(dc, ldc, dg, ldg, B, st, true))) return rc;
  // dg -> gs
  if (grow) {
    double* dst = gdev ? gs : D->d_stage_t;
    const int ldd = gdev ? ld_gs : B;
    if ((rc = hankel::transpose_f64(dg, ldg, dst, ldd, B, D->n, st))) return rc;
    if (!gdev && cudaMemcpy2DAsync(gs, sizeof(double) * (size_t)ld_gs, D->d_stage_t, sizeof(double) * B,
                                   sizeof(double) * B, n, cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return NUFHT_E_CUDA;
  } else if (!gdev) {
    if (cudaMemcpy2DAsync(gs, sizeof(double) * (size_t)ld_gs, dg, sizeof(double) * n, sizeof(double) * n, B,
                          cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return NUFHT_E_CUDA;
  }
  return cudaStreamSynchronize(st) == cudaSuccess ? 0 : NUFHT_E_CUDA;
}

// One-box evaluator for the add_* entry points.
void run_single_box(int kind, double* gs, double nu, const double* rs, const double* cs,
                    const double* ws, int m, int n, int K, double tol, const double* asy_coef,
                    int batch, int ld_cs, int ld_gs, const char* who) {
  if (!gs || !rs || !cs || !ws || m <= 0 || n <= 0 || batch <= 0) return;
  if (!has_device()) {
    std::fprintf(stderr, "%s: no CUDA device\n", who);
    return;
  }
  std::unique_ptr<DevicePlan> D(new DevicePlan);
  D->m = m;
  D->n = n;
  D->P.nu = std::fabs(nu);
  D->P.tol = tol > 0 ? tol : 1e-8;
  if (kind == 1) D->P.K_loc = K;
  if (kind == 2) {
    D->P.K_asy = K;
    if (asy_coef) std::memcpy(D->P.asy_coef, asy_coef, sizeof(double) * 64);
  }
  if (host_view(rs, m, &D->h_rs) || host_view(ws, n, &D->h_ws)) {
    std::fprintf(stderr, "%s: cannot read grids\n", who);
    return;
  }
  HBox whole{0, n - 1, 0, m - 1};
  if (kind == 0) D->dir_boxes.push_back(whole);
  if (kind == 1) D->loc_boxes.push_back(whole);
  if (kind == 2) D->asy_boxes.push_back(whole);
  int dev = 0;
  cudaGetDevice(&dev);
  int rc = finish_device_plan(D.get(), dev);
  D->sign = 1.0;
  if (!rc) rc = run_any(D.get(), cs, ld_cs, gs, ld_gs, batch, false);
  if (rc) std::fprintf(stderr, "%s: %s\n", who, nufht_b200_strerror(rc));
}

}  // namespace

extern "C" {

NufhtOptions nufht_default_options(void) {
  NufhtOptions o;
  o.tol = 1e-8;
  o.max_levels = 0;
  o.min_dim_prod = 10000;
  o.z_split = NAN;
  o.K_asy = 0;
  o.K_loc = 0;
  return o;
}

void boxes_free(Boxes* b) {
  if (!b) return;
  std::free(b->loc.data);
  std::free(b->asy.data);
  std::free(b->dir.data);
  std::memset(b, 0, sizeof(*b));
}

Boxes generate_boxes(const double* rs, int m, const double* ws, int n, double z_split,
                     int max_levels, int min_dim_prod, int K_loc_threshold) {
  Boxes out;
  std::memset(&out, 0, sizeof(out));
  if (!rs || !ws || m <= 0 || n <= 0) return out;
  HBoxes hb;
  hankel::make_boxes(rs, m, ws, n, z_split, max_levels, min_dim_prod, K_loc_threshold, &hb);
  out.loc = to_boxvec(hb.loc);
  out.asy = to_boxvec(hb.asy);
  out.dir = to_boxvec(hb.dir);
  return out;
}

void split_box(const double* rs, int m, const double* ws, int n, const Box* box, double z,
               int* ispl_out, int* jspl_out) {
  (void)n;
  HBox b{box->i0, box->i1, box->j0, box->j1};
  hankel::split_box_bs(rs, m, ws, b, z, ispl_out, jspl_out);
}

int nufht_plan_init(NufhtPlan* plan, double nu, const double* rs, int m, const double* ws, int n,
                    const NufhtOptions* opt_in) {
  if (!plan || !rs || !ws || m <= 0 || n <= 0) return -200;
  NufhtOptions opt = opt_in ? *opt_in : nufht_default_options();
  drop_device_state(plan);
  std::memset(plan, 0, sizeof(*plan));
  plan->rs = rs;
  plan->ws = ws;
  plan->m = m;
  plan->n = n;
  plan->max_levels = opt.max_levels;
  plan->min_dim_prod = opt.min_dim_prod;
  PlanParams P;
  int rc = hankel::fill_params(nu, opt, false, &P);
  if (rc) return rc;
  plan->nu = P.nu;
  plan->tol = P.tol;
  plan->z_split = P.z_split;
  plan->K_asy = P.K_asy;
  plan->K_loc = P.K_loc;
  std::memcpy(plan->asy_coef, P.asy_coef, sizeof(plan->asy_coef));
  plan->tables_loaded = 1;
  std::vector<double> hr, hw;
  if ((rc = host_copy(rs, m, &hr)) || (rc = host_copy(ws, n, &hw))) return rc;
  if (hankel::check_grid(hr.data(), m)) return NUFHT_E_UNSORTED_RS;
  if (hankel::check_grid(hw.data(), n)) return NUFHT_E_UNSORTED_WS;
  plan->boxes = generate_boxes(hr.data(), m, hw.data(), n, P.z_split, opt.max_levels,
                               opt.min_dim_prod, P.K_loc < 0 ? 0 : P.K_loc);
  return 0;
}

void nufht_plan_free(NufhtPlan* plan) {
  if (!plan) return;
  drop_device_state(plan);
  boxes_free(&plan->boxes);
  std::memset(plan, 0, sizeof(*plan));
}

// Host buffers of the reference's sizes (src/fast_hankel_nufht.c:802-845).
int nufht_scratch_init(NufhtScratch* s, const NufhtPlan* plan) {
  if (!s || !plan) return -300;
  std::memset(s, 0, sizeof(*s));
  int m = plan->m, n = plan->n;
  int Kloc = plan->K_loc < 0 ? 0 : plan->K_loc;
  int extra = 0;
  if (plan->K_loc >= 0) {
    long ni = std::lround(plan->nu);
    extra = (int)(std::labs(ni) / 2) + ((ni & 1L) ? 1 : 0);
  }
  s->in_buffer = (double*)std::calloc((size_t)m * 2, sizeof(double));
  s->out_buffer = (double*)std::calloc((size_t)n * 2, sizeof(double));
  s->real_buffer_1 = (double*)std::calloc((size_t)n, sizeof(double));
  s->real_buffer_2 = (double*)std::calloc((size_t)n, sizeof(double));
  s->cheb_buffer = (double*)std::calloc((size_t)Kloc + 1, sizeof(double));
  s->bessel_buffer_1 = (double*)std::calloc((size_t)Kloc + 1, sizeof(double));
  s->bessel_buffer_2 = (double*)std::calloc((size_t)Kloc + 1 + (size_t)extra, sizeof(double));
  if (!s->in_buffer || !s->out_buffer || !s->real_buffer_1 || !s->real_buffer_2 ||
      !s->cheb_buffer || !s->bessel_buffer_1 || !s->bessel_buffer_2) {
    nufht_scratch_free(s);
    return -301;
  }
  s->m_alloc = m;
  s->n_alloc = n;
  s->Kloc_alloc = Kloc;
  s->extra_alloc = extra;
  return 0;
}

void nufht_scratch_free(NufhtScratch* s) {
  if (!s) return;
  std::free(s->in_buffer);
  std::free(s->out_buffer);
  std::free(s->real_buffer_1);
  std::free(s->real_buffer_2);
  std::free(s->cheb_buffer);
  std::free(s->bessel_buffer_1);
  std::free(s->bessel_buffer_2);
  std::memset(s, 0, sizeof(*s));
}

int nufht_batch(const NufhtPlan* plan, const double* cs, int ld_cs, double* gs, int ld_gs,
                int batch, NufhtScratch* scratch) {
  (void)scratch;
  if (!plan || !cs || !gs || batch <= 0) return -400;
  if (ld_cs < plan->m || ld_gs < plan->n) return -401;
  DevicePlan* D = nullptr;
  int rc = device_state_for(plan, &D);
  if (rc) {
    std::fprintf(stderr, "nufht_batch: %s\n", nufht_b200_strerror(rc));
    return rc;
  }
  rc = run_any(D, cs, ld_cs, gs, ld_gs, batch, true);
  if (rc) std::fprintf(stderr, "nufht_batch: %s\n", nufht_b200_strerror(rc));
  return rc;
}

extern "C" int nufht_b200_batch_layout(const NufhtPlan* plan, const double* cs, int c_rowmajor, int ld_cs,
                                       double* gs, int g_rowmajor, int ld_gs, int batch) {
  if (!plan || !cs || !gs || batch <= 0) return -400;
  if ((c_rowmajor != 0 && c_rowmajor != 1) || (g_rowmajor != 0 && g_rowmajor != 1)) return -400;
  if (ld_cs < (c_rowmajor ? batch : plan->m) || ld_gs < (g_rowmajor ? batch : plan->n)) return -401;
  DevicePlan* D = nullptr;
  int rc = device_state_for(plan, &D);
  if (!rc) {
    rc = (c_rowmajor || g_rowmajor) ? run_layout(D, cs, c_rowmajor != 0, ld_cs, gs, g_rowmajor != 0, ld_gs, batch)
                                    : run_any(D, cs, ld_cs, gs, ld_gs, batch, true);
  }
  if (rc) std::fprintf(stderr, "nufht_b200_batch_layout: %s\n", nufht_b200_strerror(rc));
  return rc;
}

void nufht_inplace(double* gs, double nu, const double* rs, int m, const double* cs,
                   const double* ws, int n, const NufhtOptions* opt) {
  if (!gs || !rs || !cs || !ws || m <= 0 || n <= 0) {
    std::fprintf(stderr, "nufht_inplace: invalid arguments\n");
    return;
  }
  NufhtPlan plan;
  std::memset(&plan, 0, sizeof(plan));
  if (nufht_plan_init(&plan, nu, rs, m, ws, n, opt) != 0) {
    std::fprintf(stderr, "nufht_inplace: plan init failed\n");
    nufht_plan_free(&plan);
    return;
  }
  if (nufht_batch(&plan, cs, m, gs, n, 1, nullptr) != 0)
    std::fprintf(stderr, "nufht_inplace: batch execution failed\n");
  nufht_plan_free(&plan);
}

double* nufht(double nu, const double* rs, int m, const double* cs, const double* ws, int n,
              const NufhtOptions* opt) {
  double* gs = (double*)std::calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  if (!gs) return nullptr;
  nufht_inplace(gs, nu, rs, m, cs, ws, n, opt);
  return gs;
}

void add_dir(double* gs, double nu, const double* rs, const double* cs, const double* ws, int m,
             int n) {
  run_single_box(0, gs, nu, rs, cs, ws, m, n, 0, 1e-8, nullptr, 1, m, n, "add_dir");
}

void add_dir_batch(double* gs, double nu, const double* rs, const double* cs, const double* ws,
                   int m, int n, int batch, int ld_cs, int ld_gs) {
  run_single_box(0, gs, nu, rs, cs, ws, m, n, 0, 1e-8, nullptr, batch, ld_cs, ld_gs, "add_dir_batch");
}

void add_loc(double* gs, double nu, const double* rs, const double* cs, const double* ws, int m,
             int n, int K, double*, double*, double*) {
  if (!hankel::is_integer(nu)) {
    std::fprintf(stderr, "add_loc: nu must be integer\n");
    return;
  }
  run_single_box(1, gs, nu, rs, cs, ws, m, n, K, 1e-8, nullptr, 1, m, n, "add_loc");
}

void add_loc_batch(double* gs, double nu, const double* rs, const double* cs, const double* ws,
                   int m, int n, int K, int batch, int ld_cs, int ld_gs, double*, double*, double*) {
  if (!hankel::is_integer(nu)) {
    std::fprintf(stderr, "add_loc_batch: nu must be integer\n");
    return;
  }
  run_single_box(1, gs, nu, rs, cs, ws, m, n, K, 1e-8, nullptr, batch, ld_cs, ld_gs, "add_loc_batch");
}

void add_asy(double* gs, double nu, const double* rs, const double* cs, const double* ws, int m,
             int n, int K, double tol, const double* asy_coef, double*, double*, double*, double*) {
  run_single_box(2, gs, nu, rs, cs, ws, m, n, K, tol, asy_coef, 1, m, n, "add_asy");
}

void add_asy_batch(double* gs, double nu, const double* rs, const double* cs, const double* ws,
                   int m, int n, int K, double tol, const double* asy_coef, int batch, int ld_cs,
                   int ld_gs, double*, double*) {
  run_single_box(2, gs, nu, rs, cs, ws, m, n, K, tol, asy_coef, batch, ld_cs, ld_gs, "add_asy_batch");
}

// ------------------------------- extension -------------------------------

int nufht_b200_plan_create(NufhtDevicePlan** out, double nu, const double* rs, int m,
                           const double* ws, int n, const NufhtOptions* opt_in, int flags,
                           int device) {
  if (!out) return -200;
  *out = nullptr;
  if (!rs || !ws || m <= 0 || n <= 0) return -200;
  if (flags & ~(NUFHT_B200_MIXED | NUFHT_B200_MIXED_AVERAGED | NUFHT_B200_EXTENDED_TABLES)) return NUFHT_E_BAD_FLAGS;
  NufhtOptions opt = opt_in ? *opt_in : nufht_default_options();
  std::unique_ptr<DevicePlan> D(new DevicePlan);
  int rc = hankel::fill_params(nu, opt, (flags & NUFHT_B200_EXTENDED_TABLES) != 0, &D->P);
  if (rc) return rc;
  if (!has_device()) return NUFHT_E_NO_DEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return NUFHT_E_CUDA;
  D->m = m;
  D->n = n;
  D->flags = flags;
  // Mixed precision requested: the asymptotic boxes (the bulk of the work) run in FP32 if
  // the planner finds the worst-case FP32 rounding within tol / 4 (NUFHT_B200_MIXED) or
  // regardless of it (NUFHT_B200_MIXED_AVERAGED), else in FP64; always FP64 below 1e-9.
  D->mixed_asy = (flags & (NUFHT_B200_MIXED | NUFHT_B200_MIXED_AVERAGED)) != 0 && D->P.tol >= 1e-9;
  D->mixed_averaged = (flags & NUFHT_B200_MIXED_AVERAGED) != 0;
  HBoxes hb;
  D->device = device;
  if ((rc = device_grids_and_boxes(D.get(), rs, ws, opt, &hb))) return rc;
  D->plan_loc = hb.loc;
  D->plan_asy = hb.asy;
  D->plan_dir = hb.dir;
  choose_path(D.get(), opt.min_dim_prod);
  if ((rc = finish_device_plan(D.get(), device))) return rc;
  NufhtDevicePlan* h = new NufhtDevicePlan;
  h->dp = std::move(D);
  *out = h;
  return 0;
}

int nufht_b200_generate_boxes_device(const double* rs, int m, const double* ws, int n, double z_split,
                                     int max_levels, int min_dim_prod, int K_loc_threshold, Boxes* out) {
  if (!out) return -200;
  std::memset(out, 0, sizeof(*out));
  if (!rs || !ws || m <= 0 || n <= 0) return -200;
  if (!has_device()) return NUFHT_E_NO_DEVICE;
  int rc;
  // device grids are used where they are; host grids are uploaded
  const double* dr = rs;
  const double* dw = ws;
  double *ur = nullptr, *uw = nullptr;
  auto release = [&]() {
    cudaFree(ur);
    cudaFree(uw);
  };
  if (!is_device_ptr(rs)) {
    if (cudaMalloc((void**)&ur, sizeof(double) * (size_t)m) != cudaSuccess ||
        cudaMemcpy(ur, rs, sizeof(double) * m, cudaMemcpyHostToDevice) != cudaSuccess) {
      release();
      return NUFHT_E_CUDA;
    }
    dr = ur;
  }
  if (!is_device_ptr(ws)) {
    if (cudaMalloc((void**)&uw, sizeof(double) * (size_t)n) != cudaSuccess ||
        cudaMemcpy(uw, ws, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
      release();
      return NUFHT_E_CUDA;
    }
    dw = uw;
  }
  HBoxes hb;
  int bad = 0;
  rc = hankel::device_make_boxes(dr, m, dw, n, z_split, max_levels, min_dim_prod, K_loc_threshold, &hb, 0, &bad);
  release();
  if (rc) return rc;
  if (bad) return bad == 1 ? NUFHT_E_UNSORTED_RS : NUFHT_E_UNSORTED_WS;
  out->loc = to_boxvec(hb.loc);
  out->asy = to_boxvec(hb.asy);
  out->dir = to_boxvec(hb.dir);
  return 0;
}

int nufht_b200_execute(NufhtDevicePlan* plan, const double* cs, int ld_cs, double* gs, int ld_gs,
                       int batch, void* stream) {
  if (!plan || !cs || !gs || batch <= 0) return -400;
  DevicePlan* D = plan->dp.get();
  if (ld_cs < D->m || ld_gs < D->n) return -401;
  std::lock_guard<std::mutex> lk(D->mu);
  return D->run(cs, ld_cs, gs, ld_gs, batch, (cudaStream_t)stream, true);
}

int nufht_b200_plan_info(const NufhtDevicePlan* plan, NufhtB200Info* info) {
  if (!plan || !info) return -400;
  const DevicePlan* D = plan->dp.get();
  std::memset(info, 0, sizeof(*info));
  info->nu = D->P.nu;
  info->tol = D->P.tol;
  info->z_split = D->P.z_split;
  info->K_asy = D->P.K_asy;
  info->K_loc = D->P.K_loc;
  info->n_loc = (long)D->loc_boxes.size();
  info->n_asy = (long)D->asy_boxes.size();
  info->n_dir = (long)D->dir_boxes.size();
  info->fft_points = D->NLP > 0 ? D->total_cells / D->NLP : D->total_cells;
  info->spread_width = D->W;
  info->path = D->path;
  info->workspace_bytes = D->ws_bytes;
  info->mixed = D->mixed_asy ? 1 : 0;
  return 0;
}

void nufht_b200_plan_destroy(NufhtDevicePlan* plan) { delete plan; }

long nufht_b200_plan_boxes(const NufhtDevicePlan* plan, int* out, long cap) {
  if (!plan) return -400;
  const DevicePlan* D = plan->dp.get();
  long tot = (long)(D->plan_loc.size() + D->plan_asy.size() + D->plan_dir.size());
  if (out && cap >= tot) {
    long p = 0;
    for (const auto* v : {&D->plan_loc, &D->plan_asy, &D->plan_dir})
      for (const HBox& b : *v) {
        out[4 * p] = b.i0; out[4 * p + 1] = b.i1; out[4 * p + 2] = b.j0; out[4 * p + 3] = b.j1;
        ++p;
      }
  }
  return tot;
}

const char* nufht_b200_strerror(int code) {
  switch (code) {
    case 0: return "success";
    case -1: return "tolerance below 1e-15";
    case -2: return "only integer |nu| <= 200 and half-integer |nu| <= 19/2 are implemented";
    case -3: case -4: case -5: case -6: return "table index out of range";
    case -100: return "NULL plan or options";
    case -200: return "NULL grid or non-positive size";
    case -300: return "NULL scratch or plan";
    case -301: return "scratch allocation failed";
    case -400: return "invalid argument";
    case -401: return "leading dimension smaller than the grid size";
    case -402: case -403: return "allocation failed";
    case NUFHT_E_UNSORTED_RS: return "rs must be finite, non-negative and non-decreasing";
    case NUFHT_E_UNSORTED_WS: return "ws must be finite, non-negative and non-decreasing";
    case NUFHT_E_CUDA: return "CUDA runtime or cuFFT error";
    case NUFHT_E_NO_DEVICE: return "no CUDA device";
    case NUFHT_E_TOO_LARGE: return "sizes exceed what this entry point accepts";
    case NUFHT_E_BAD_FLAGS: return "unknown flag bits";
    default: return "unknown error";
  }
}

long long nufht_b200_launch_count(void) { return hankel::g_launch_counter.load(); }

int nufht_b200_besselj(double nu, const double* x, double* out, long count, void* stream) {
  if (!x || !out || count < 0) return -400;
  return hankel::run_besselj(nu, x, out, count, (cudaStream_t)stream);
}

const char* nufht_b200_table_source(void) { return hankel::tables_source(); }

void nufht_b200_set_phase_timing(int on) { hankel::g_phase_timing.store(on != 0); }

int nufht_b200_phase_times(double* ms, int nphase) {
  if (!ms || nphase <= 0) return -400;
  return hankel::phase_times(ms, nphase);
}

}  // extern "C"

extern "C" int nufht_b200_plan_stats(const NufhtDevicePlan* plan, double* out, int n) {
  if (!plan || !out || n <= 0) return -400;
  hankel::plan_stats(*plan->dp, out, n);
  return 0;
}

extern "C" int nufht_b200_fp64_peak(double* tflops) {
  if (!tflops) return -400;
  return hankel::fp64_peak(tflops);
}

extern "C" int nufht_b200_fp32_peak(double* tflops) {
  if (!tflops) return -400;
  return hankel::fp32_peak(tflops);
}
