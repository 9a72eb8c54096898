// Asymptotic boxes in double-precision arithmetic.
#include "asy_launch.cuh"

namespace hankel {

int run_asy_f64(DevicePlan& D, const double* cs, int ld_cs, double* gs, int ld_gs, int B, cudaStream_t st,
              double sgn) {
  return run_asy_t<double>(D, cs, ld_cs, gs, ld_gs, B, st, sgn);
}

int asy_records_f64(DevicePlan& D) { return build_records_t<double>(D); }

}  // namespace hankel
