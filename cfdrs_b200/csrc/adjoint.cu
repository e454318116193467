// Adjoint building blocks: the sparsity-pattern outer product that turns an
// adjoint vector into dL/dA on A's pattern, and a device-side value update so
// a differentiable assembly on the device can feed the solver directly.
//
// For x = A^{-1} b and a loss L(x), with lambda = A^{-T} dL/dx:
//   dL/db = lambda,   dL/da_ij = -lambda_i x_j   for every stored (i, j).
// (No reference counterpart: CFDrs has no differentiable solve; its Python
// layer, crates/cfd-python/src/lib.rs:85-158, exposes physics solvers only.)
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "amg_device.h"
#include "internal.h"

namespace cfd {
namespace {

// g_e = -scale * lambda[row(e)] * x[col(e)], one thread per row.
__global__ void __launch_bounds__(kThreads) k_pattern_outer(int64_t nrows, const int* __restrict__ rp,
                                                            const int* __restrict__ col,
                                                            const double* __restrict__ lambda,
                                                            const double* __restrict__ x, double scale,
                                                            double* __restrict__ g) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += (int64_t)gridDim.x * blockDim.x) {
    const double li = -scale * lambda[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) g[k] = li * __ldg(x + col[k]);
  }
}

__global__ void k_cast64to32(int64_t n, const double* __restrict__ s, float* __restrict__ d) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (float)s[i];
}

}  // namespace
}  // namespace cfd

using namespace cfd;

extern "C" {

cfd_status cfd_pattern_outer(cfd_csr* a, const double* lambda, const double* x, double scale, double* g) {
  if (!a || !lambda || !x || !g) {
    set_error("cfd_pattern_outer: null argument");
    return CFD_ERR_STATE;
  }
  std::lock_guard<std::mutex> lk(a->ctx->mu);
  CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
  const int64_t n = a->dev.nrows;
  if (n == 0) return CFD_OK;
  const int grid = (int)std::min<int64_t>((n + kThreads - 1) / kThreads, (int64_t)a->ctx->num_sms * 8);
  k_pattern_outer<<<grid, kThreads, 0, a->ctx->stream>>>(n, a->dev.rp, a->dev.col, lambda, x, scale, g);
  CFD_TRY_CUDA(cudaGetLastError());
  return CFD_OK;
}

cfd_status cfd_csr_set_values_device(cfd_csr* a, const double* val_dev) {
  if (!a || !val_dev) {
    set_error("cfd_csr_set_values_device: null argument");
    return CFD_ERR_STATE;
  }
  std::lock_guard<std::mutex> lk(a->ctx->mu);
  CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
  cudaStream_t s = a->ctx->stream;
  const int64_t nnz = a->dev.nnz;
  CFD_TRY_CUDA(cudaMemcpyAsync(a->dev.v64, val_dev, nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (a->dev.v32 && nnz > 0) {
    const int grid = (int)std::min<int64_t>((nnz + 255) / 256, (int64_t)a->ctx->num_sms * 16);
    k_cast64to32<<<grid, 256, 0, s>>>(nnz, a->dev.v64, a->dev.v32);
    CFD_TRY_CUDA(cudaGetLastError());
  }
  a->dev.sl_stale = true;
  a->dev.dia_stale = true;
  // The host copy feeds AMG setup (the Galerkin recompute reads the device values).
  CFD_TRY_CUDA(cudaMemcpyAsync(a->host.v.data(), val_dev, nnz * sizeof(double), cudaMemcpyDeviceToHost, s));
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  a->simple_stale = a->simple_nv >= 0;
    a->cblock_stale = a->cblock_nv >= 0;
  if (a->diag64) {
    cudaFree(a->diag64);
    cudaFree(a->diag32);
    cudaFree(a->jinv64);
    cudaFree(a->jinv32);
    a->diag64 = nullptr;
    a->diag32 = nullptr;
    a->jinv64 = nullptr;
    a->jinv32 = nullptr;
    a->jacobi_status = -1;
  }
  return CFD_OK;
}

}  // extern "C"
