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

struct DevLevel {
  DevMat A, P, R;
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
  int64_t coarse_n = 0;
  bool have32 = false;
  double setup_seconds = 0.0;
};

namespace cfd {
cfd_status amg_upload(cfd_amg* amg, bool want32);
cfd_status amg_ensure32(cfd_amg* amg);
void amg_free_device(cfd_amg* amg);
}  // namespace cfd
