// Device-resident AMG hierarchy (the object behind cfd_amg*).
#pragma once

#include <vector>

#include "amg_setup.h"
#include "internal.h"

namespace cfd {

template <typename XT>
struct LevelVecs {
  XT* b = nullptr;   // level right-hand side (restricted residual), l > 0
  XT* xa = nullptr;  // smoother iterate
  XT* xb = nullptr;  // smoother ping-pong partner
  XT* r = nullptr;   // level residual
  XT* e = nullptr;   // level output (coarse correction handed to the finer level)
};

// Pattern of R_l A_l on the device (the intermediate product of the Galerkin
// recompute), with a value buffer.
struct DevRA {
  int* rp = nullptr;
  int* ci = nullptr;
  double* v = nullptr;
  int64_t nrows = 0, nnz = 0;
};

struct DevLevel {
  DevMat A, P, R;
  DevRA ra;
  double* d64 = nullptr;  // diagonal of A (FP64)
  float* d32 = nullptr;
  LevelVecs<double> v64;
  LevelVecs<float> v32;
};

}  // namespace cfd

struct cfd_amg {
  cfd_context* ctx = nullptr;
  cfd_amg_config cfg{};
  std::vector<cfd::HostLevel> host;
  std::vector<cfd::DevLevel> dev;
  double* coarse_inv = nullptr;  // dense FP64 inverse of the coarsest operator (CFD_COARSE_DENSE)
  float* coarse_inv32 = nullptr;  // its FP32 rounding, applied by the FP32 (inner) V-cycle
  int64_t coarse_n = 0;
  bool have32 = false;
  bool host_values_stale = false;  // level A values re-formed on the device (cfd_amg_recompute)
  double setup_seconds = 0.0;
};

namespace cfd {
cfd_status amg_upload(cfd_amg* amg, bool want32);
cfd_status amg_ensure32(cfd_amg* amg);
void amg_free_device(cfd_amg* amg);
// Galerkin recompute on the device for the fine values of `a` (pattern fixed):
// A_{l+1} = (R_l A_l) P_l in the host spgemm's summation order, level
// diagonals, FP32 copies and the dense coarsest inverse (recompute.cu).
cfd_status amg_recompute_device(cfd_amg* amg, const cfd_csr* a);
// Brings the host copies of the level A values up to date after a device recompute.
cfd_status amg_sync_host_values(cfd_amg* amg);
void free_ra(DevRA& ra);
// Gauss-Jordan inverse (partial pivoting, the host dense_inverse's operations
// in its order) of an n x n device CSR operator into inv (n x n, row-major),
// for n <= kDenseInverseDeviceMaxRows (the staged pivot rows and row tables fit
// one CTA's shared memory).
constexpr int64_t kDenseInverseDeviceMaxRows = 8192;
cfd_status dense_inverse_device(cfd_context* ctx, int64_t n, const int* rp, const int* ci, const double* v,
                                double* inv);
}  // namespace cfd
