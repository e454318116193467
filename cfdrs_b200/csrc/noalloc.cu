// cfd_residual_norm_noalloc: r = b - A x and ||r||_2^2 for callers that cannot
// allocate device memory. See the declaration in include/cfdgpu.h.
//
// Some callers of this library cannot call cudaMalloc: a solver embedded in a
// host application whose memory manager has already reserved the device
// memory (a further cudaMalloc fails or breaks its accounting), and
// latency-critical outer loops (a pressure-correction convergence monitor
// checked every time step, many network solves issued from parallel design
// search workers) where cudaMalloc / cudaFree synchronize the device and
// serialize the threads. This entry point computes the same fused residual and
// squared norm as the library's outer-residual kernel, but keeps the scratch
// of its two-stage reduction (per-CTA partial sums and the last-CTA ticket) in
// a fixed device array compiled into the library instead of memory it
// allocates. The caller passes every input and output.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"
#include "kernels.cuh"

namespace cfd {
namespace {

constexpr int kNoAllocRowsPerCta = kThreads;                  // one thread per row
constexpr size_t kNoAllocScratchBytes = size_t(1) << 20;      // 1 MiB, held by every GPU that loads the library
constexpr size_t kNoAllocPartialOffset = 256;                 // ticket counter lives in the first 256 bytes
constexpr int64_t kNoAllocMaxCtas = (int64_t)((kNoAllocScratchBytes - kNoAllocPartialOffset) / sizeof(double));
constexpr int64_t kNoAllocMaxRows = kNoAllocMaxCtas * kNoAllocRowsPerCta;  // 33 546 240 rows

// The shared scratch: [0, 4) ticket counter, [256, 1 MiB) one partial per CTA.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
// Device address of g_noalloc_scratch, per device, looked up once and kept for
// the life of the process: stale after a cudaDeviceReset of that device, after
// which the entry point must not be used there (documented in cfdgpu.h).
unsigned char* g_scratch_addr[kMaxDevices] = {};

__global__ void __launch_bounds__(kThreads) k_residual_norm_noalloc(int nrows, const int* __restrict__ rp,
                                                                    const int* __restrict__ col,
                                                                    const double* __restrict__ val,
                                                                    const double* __restrict__ x,
                                                                    const double* __restrict__ b,
                                                                    double* __restrict__ r, double* out,
                                                                    unsigned char* scratch) {
  const int row = blockIdx.x * kNoAllocRowsPerCta + threadIdx.x;
  double acc[1] = {0.0};
  if (row < nrows) {
    double s = 0.0;
    for (int k = rp[row]; k < rp[row + 1]; ++k) s += val[k] * __ldg(x + col[k]);
    const double ri = b[row] - s;
    r[row] = ri;
    acc[0] = ri * ri;
  }
  Red red{reinterpret_cast<double*>(scratch + kNoAllocPartialOffset), reinterpret_cast<unsigned*>(scratch)};
  double tot[1];
  if (grid_reduce<1>(acc, red, tot) && threadIdx.x == 0) *out = tot[0];
}

}  // namespace
}  // namespace cfd

using namespace cfd;

extern "C" cfd_status cfd_residual_norm_noalloc(int64_t nrows, int64_t ncols, const int32_t* row_ptr,
                                                const int32_t* col, const double* val, const double* x,
                                                const double* b, double* r, double* norm2, void* cuda_stream) {
  if (nrows < 0 || ncols < 0) {
    set_error("cfd_residual_norm_noalloc: negative dimension");
    return CFD_ERR_DIM;
  }
  if (nrows > kNoAllocMaxRows || ncols >= INT32_MAX) {
    set_error("cfd_residual_norm_noalloc: %lld rows exceed the fixed scratch limit of %lld rows "
              "(1 MiB of reduction partials); use cfd_spmv on a cfd_csr handle instead",
              (long long)nrows, (long long)kNoAllocMaxRows);
    return CFD_ERR_DIM;
  }
  if (!norm2 || (nrows > 0 && (!row_ptr || !x || !b || !r || (!col && ncols > 0)))) {
    set_error("cfd_residual_norm_noalloc: null pointer argument");
    return CFD_ERR_STATE;
  }
  int dev = 0;
  CFD_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("cfd_residual_norm_noalloc: device ordinal %d out of range", dev);
    return CFD_ERR_CONFIG;
  }
  unsigned char* scratch = nullptr;
  {
    // Once per device, with that device current: the device address of the
    // scratch array (its host-side name is only a stand-in).
    std::lock_guard<std::mutex> g(g_setup_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) {
        set_error("cfd_residual_norm_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return CFD_ERR_CUDA;
      }
      g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  if (nrows == 0) {
    CFD_TRY_CUDA(cudaMemsetAsync(norm2, 0, sizeof(double), s));
    return CFD_OK;
  }
  // The array keeps the previous call's contents: the ticket must start at zero.
  CFD_TRY_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned), s));
  const int grid = (int)((nrows + kNoAllocRowsPerCta - 1) / kNoAllocRowsPerCta);
  k_residual_norm_noalloc<<<grid, kThreads, 0, s>>>((int)nrows, row_ptr, col, val, x, b, r, norm2, scratch);
  CFD_TRY_CUDA(cudaGetLastError());
  return CFD_OK;
}
