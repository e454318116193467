// Diagnostics of the failure path (no reference counterpart): every wait of
// the bulk-copy pipelines is an mbarrier parity wait bounded by a number of
// tries; when it runs out the kernel flags the context's error word and
// leaves, and the host call reports CFD_ERR_TIMEOUT. cfd_selftest_wait_timeout
// runs that wait on a barrier nothing completes, with a small bound, so the
// path can be checked on a GPU without a fault or a hang.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"
#include "kernels.cuh"

namespace cfd {
namespace {

__global__ void k_selftest_wait(unsigned tries, int* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // one arrival expected; none is made
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0u, tries)) atomicExch(err, 1);
}

}  // namespace
}  // namespace cfd

cfd_status cfd_selftest_wait_timeout(cfd_context* ctx, int32_t tries) {
  if (!ctx || tries < 1) {
    cfd::set_error("cfd_selftest_wait_timeout: null context or tries < 1");
    return CFD_ERR_CONFIG;
  }
  std::lock_guard<std::mutex> g(ctx->mu);
  CFD_TRY_CUDA(cudaSetDevice(ctx->device));
  cfd::k_selftest_wait<<<1, 32, 0, ctx->stream>>>((unsigned)tries, ctx->err);
  CFD_TRY_CUDA(cudaGetLastError());
  return cfd::check_device_flag(ctx);
}
