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
// Direct work item: targets [i0, i0+ni), sources [j0, j0+nj); `lanes` threads share one
// target (thin boxes) and split its sources.
struct DirItem { int i0, ni, j0, nj, lanes; };

// Geometry of one asymptotic box's type-3 transform: sources x = r - C, targets s = k - D,
// spreading grid spacing h (cells l in [-half, half]), FFT length n2, its rows in the
// per-cell deconvolution and per-target phase tables, and its place in the workspace:
// n2 * V contiguous complex values from cell_off * V, vector v at offset v * n2.
struct AsyBoxD {
  int i0, i1, j0, j1;
  double C, D, h;
  double rref;          // smallest source radius of the box: the source factors are
                        // (rref/r)^(lp+1/2) <= 1 and the target factors (k rref)^-(lp+1/2)
                        // <= z_split^-(lp+1/2), so both stay in single-precision range
  int half, n2;
  int mode;             // 0: CTAs own grid tiles; 1: CTAs own source chunks (dense boxes)
  int cls;              // kernel class (oversampling, kernel width, expansion terms)
  int nlp;              // expansion terms of this box: 2 (K + 1) with K <= K_asy
  long long cell_off;   // workspace offset in cells of one vector
  long long corr_off;   // first of 2 half + 1 entries in the cell table
  long long post_off;   // target records of the box (targets i0..i1): first cells from post_off,
  long long tw_off;     // interpolation weights (rows padded to 16 bytes) from tw_off,
  long long tm_off;     // nlp target factors each from tm_off
  long long rec_off;    // source records of the box (sources j0..j1): first cells from rec_off,
  long long recw_off;   // W weights each from recw_off,
  long long recp_off;   // nlp amplitude factors each from recp_off
};
// Spreading work item.  mode 0: cells [l_start, l_start+ncell) of the box, FFT index
// fft_start.., sources [js, je) whose support meets them; mode 1: all taps of sources
// [js, je) into a window of cells [l_start, l_start+ncell) added atomically; mode 2: FFT
// indices [fft_start, fft_start+ncell) of the zero padding.
struct SpreadItem {
  int box, mode, l_start, fft_start, ncell, js, je;
};
struct InterpItem { int box, ks, ke; };
struct FftGroup {
  int n2, nbox, mode, nlp;
  int cls;             // kernel class of the group's boxes
  int slot;            // stream slot of that class (and of its slice of the FFT work area)
  long long cell_off;  // the group's boxes are consecutive in the workspace
  cufftHandle plan;
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

// A kernel class: oversampling factor sigma of both type-3 stages, kernel width W and
// shape beta, expansion terms NLP (ac.NLP), and the contiguous ranges of its boxes'
// spreading / interpolation items.
struct AsyClass {
  double sigma;
  int W;
  int nlp;
  AsyConst ac;
  int spread0, nspread;    // windowed spreading items (modes 0 and 2)
  int spreadA0, nspreadA;  // atomic spreading items (mode 1)
  int interp0, ninterp;
  int slot;  // stream slot (0 .. kAuxStreams - 3) of the class's pipeline, -1 without boxes
};

int spread_width_for_tol(double tol);
int spread_width(double tol, double sigma);

struct DevicePlan {
  int device = 0;
  int flags = 0;
  PlanParams P;
  int m = 0, n = 0;
  int path = 0;   // 0 boxes, 1 all-direct, 2 all-asymptotic
  int nu2 = 0;    // 2 |nu|
  double sign = 1.0;
  // Host view of the grids, used while planning only: the caller's own array when the grid
  // is in host memory (no copy), else a copy read back from the device.
  struct HostGrid {
    std::vector<double> own;
    const double* p = nullptr;
    const double* data() const { return p; }
    double operator[](size_t i) const { return p[i]; }
    void borrow(const double* q) {
      own.clear();
      p = q;
    }
    void release() {
      std::vector<double>().swap(own);
      p = nullptr;
    }
  };
  HostGrid h_rs, h_ws;
  std::vector<HBox> loc_boxes, asy_boxes, dir_boxes;  // boxes as evaluated
  std::vector<HBox> plan_loc, plan_asy, plan_dir;     // the planner's partition
  std::vector<HBox> asy_eval, asy_direct;  // asymptotic boxes evaluated by NUFFT / summed directly
  std::vector<int> asy_eval_nlp;            // expansion terms of each asy_eval box

  // work lists
  int KL1 = 0, W = 0;
  int K_eval = 0;  // Wimp degree evaluated: K_loc, or fewer where the dropped terms are negligible
  std::vector<LocBoxD> locb;
  std::vector<ProjItem> proj;
  std::vector<EvalItem> eval;
  std::vector<DirItem> dir;       // direct items (tensor-core form: the dir_thin thin ones first)
  int dir_thin = 0;
  bool dir_simt = false;          // direct items of the SIMT kernel
  std::vector<AsyBoxD> asyb;
  std::vector<SpreadItem> spread;
  std::vector<InterpItem> interp;
  std::vector<FftGroup> groups;
  std::vector<AsyClass> classes;
  long long total_cells = 0;       // grid values per column: sum of n2 * NLP over asymptotic boxes
  long long chunk_cell_begin = 0;  // grid rows of the mode-1 boxes (zeroed before spreading)
  long long chunk_cell_end = 0;
  long long total_corr = 0, total_post = 0;
  long long total_rec = 0, total_recw = 0, total_recp = 0;  // source record counts
  long long total_tw = 0, total_tm = 0;                      // target record counts
  int NLP = 0;                     // 2 (K_asy + 1)

  // device copies
  double *d_rs = nullptr, *d_ws = nullptr;
  LocBoxD* d_locb = nullptr;
  ProjItem* d_proj = nullptr;
  EvalItem* d_eval = nullptr;
  DirItem* d_dir = nullptr;
  AsyBoxD* d_asyb = nullptr;
  SpreadItem* d_spread = nullptr;
  InterpItem* d_interp = nullptr;
  double* d_jtab = nullptr;   // J_nu table of the direct boxes (orders whose evaluation is costly)
  int jtab_n = 0;             // unit intervals of d_jtab: it covers [0, jtab_n)
  double* d_corr = nullptr;   // 1 / psi-hat of the second stage, per box cell
  // Source records of the asymptotic boxes (arithmetic type of the boxes): first cell of
  // each source's kernel support, its complex weights and its amplitude factors.
  int* d_rec_l0 = nullptr;
  void* d_rec_w = nullptr;
  void* d_rec_p = nullptr;
  // Target records: first cell of each target's stencil, its W kernel weights and its NLP
  // factors mu (expansion coefficient, target power, phase and deconvolution).
  int* d_tq0 = nullptr;
  void* d_tw = nullptr;
  void* d_tmu = nullptr;
  size_t rec_bytes = 0;

  // workspace, sized for the largest batch executed so far
  int ws_B = 0;
  int fft_B = 0;             // batch size of the FFT plans in groups[].plan
  std::map<int, std::vector<cufftHandle>> fft_cache;  // FFT plans per batch size, one per group
  size_t fft_work_bytes = 0;
  size_t fft_slot_bytes = 0;  // the work area holds one slice per stream slot
  // Batches (CUDA graphs) that recorded this plan's buffers and FFT plans: while pins > 0 a
  // buffer that must grow is replaced by a new allocation and the old one is kept in
  // `retired` (the graphs still use it) until the last batch lets go.
  int pins = 0;
  std::vector<void*> retired;
  size_t ws_bytes = 0;
  void* d_grid = nullptr;    // complex FP64 (double2) or, in mixed precision, FP32 (float2)
  void* d_ct = nullptr;      // coefficients source-major, in the asymptotic boxes' type
  int ldct = 0;              // row length of d_ct (columns, padded)
  bool mixed_asy = false;    // asymptotic boxes in FP32 (NUFHT_B200_MIXED, where FP32 meets tol)
  bool mixed_averaged = false;  // FP32 regardless of the worst-case bound (NUFHT_B200_MIXED_AVERAGED)
  double fp32_err = 0.0;     // modelled worst-case FP32 error of the asymptotic boxes per ||c||_1
  double* d_partial = nullptr;
  double* d_cheb = nullptr;
  void* d_fft_work = nullptr;

  // staging for host-pointer calls through the reference-compatible entry points
  double* d_stage_c = nullptr;
  double* d_stage_g = nullptr;
  double* d_stage_t = nullptr;  // row-major copies of cs / gs (nufht_b200_batch_layout)
  size_t stage_c_bytes = 0, stage_g_bytes = 0, stage_t_bytes = 0;
  // Streams on which run() executes independent phases and kernel classes concurrently
  // (forked from and joined back to the caller's stream with events; created on first use):
  // 0 local boxes, 1 direct boxes, 2.. asymptotic kernel classes.
  static constexpr int kAuxStreams = 8;
  cudaStream_t aux[kAuxStreams] = {};
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[kAuxStreams] = {};
  int ensure_aux();
  bool serial = false;  // this run() queues everything on the caller's stream
  // copy streams and events of the pipelined host-buffer path (created on first use)
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ev_in[4] = {}, ev_done[4] = {};

  // planning cost (host wall-clock ms): validation and box partition, work lists, device
  // tables and uploads; 1 when the partition ran on the device
  double plan_ms[3] = {0, 0, 0};
  int partition_on_device = 0;

  std::mutex mu;

  ~DevicePlan();
  void build_lists();
  int upload_all();
  int ensure_workspace(int B);
  int ensure_fft(int B);
  void release_fft();
  void drop_buffer(void* p);  // cudaFree, or keep in `retired` while pinned
  void pin();                 // called with mu held
  void unpin();               // called with mu held; frees retired buffers at zero pins
  // g (+)= H c on stream st; cs / gs are device pointers.
  int run(const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
          bool zero_output);
};

extern std::atomic<long long> g_launch_counter;
extern std::atomic<bool> g_phase_timing;

// Phases of run() reported by the optional device timers.
enum { kPhaseZero = 0, kPhaseLocProj, kPhaseLocEval, kPhaseSpread, kPhaseFft, kPhaseInterp, kPhaseDir,
       kNumPhases };
int phase_times(double* ms, int nphase);
void phase_record(int phase, cudaEvent_t a, cudaEvent_t b);

// Device events around one phase of run(), when phase timing is on.
struct PhaseScope {
  int phase = -1;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t st;
  PhaseScope(int ph, cudaStream_t s) : st(s) {
    if (!g_phase_timing.load(std::memory_order_relaxed)) return;
    phase = ph;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
  }
  ~PhaseScope() {
    if (phase < 0) return;
    cudaEventRecord(b, st);
    phase_record(phase, a, b);
  }
};

// The asymptotic boxes of one run() in single (mixed) or double precision.
int run_asy_f32(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
                double sgn);
int run_asy_f64(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
                double sgn);
// Source records of the asymptotic boxes (after the cell tables), in single or double precision.
int asy_records_f32(DevicePlan& D);
int asy_records_f64(DevicePlan& D);
// Row length of the packed coefficients for batch size B: whole column blocks of a spreading
// CTA (up to 32 columns) in 16-byte pieces.
inline int packed_ld(int B) { return B <= 32 ? (B + 3) / 4 * 4 : (B + 31) / 32 * 32; }

int run_besselj(double nu, const double* x, double* out, long count, cudaStream_t st);

// Fork streams D.aux[which[0..n)] from st (they wait for st's work so far) and join them back
// (st waits for their work), with events.
int fork_streams(DevicePlan& D, cudaStream_t st, const int* which, int n);
int join_streams(DevicePlan& D, cudaStream_t st, const int* which, int n);

// Device planner (planner_dev.cu): validation of a device-resident grid (0, or -1 when not
// finite, non-negative and non-decreasing) and the box partition from device-resident grids.
int device_check_grid(const double* d_a, int len, cudaStream_t st);
// bad_grid (optional): also validate both grids; set to 0, or 1 / 2 when rs / ws is not
// finite, non-negative and non-decreasing (the boxes are then not computed).
int device_make_boxes(const double* d_rs, int m, const double* d_ws, int n, double z, int max_levels,
                      int min_dim_prod, int Kthr, HBoxes* out, cudaStream_t st, int* bad_grid = nullptr);

// out[c * ldo + r] = in[r * ldi + c] for r < rows, c < cols (device pointers): a row-major
// batch to the executor's column-major one and back.
int transpose_f64(const double* in, int ldi, double* out, int ldo, int rows, int cols, cudaStream_t st);

}  // namespace hankel

namespace hankel {
// Algorithmic work of a plan per batch column, for roofline accounting (see stats order in
// nufht_b200_plan_stats).
void plan_stats(const DevicePlan& D, double* out, int n);
// Measured FP32 (packed f32x2) fused-multiply-add throughput of the current device in TFLOP/s.
int fp32_peak(double* tflops);
// Measured FP64 fused-multiply-add throughput of the current device in TFLOP/s.
int fp64_peak(double* tflops);
}  // namespace hankel

namespace hankel {
int run_loc_box(const double* rs, const double* ws, const double* cs, int ld_cs, double* gs, int ld_gs,
                int B, const LocBoxD* d_box, const ProjItem* d_proj, int nproj, const EvalItem* d_eval,
                int neval, double* d_partial, double* d_cheb, int K, int nu_int, double sgn, cudaStream_t st);
}  // namespace hankel
