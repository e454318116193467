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

// 2-D Darcy system of an n x n cell grid, -div(k grad p) = 0 with k = exp(theta)
// per cell (row r = i + n j, theta[r]), harmonic-mean faces 2 k_a k_b / (k_a + k_b)
// (a the lower-numbered cell), Dirichlet p = 1 on the left and p = 0 on the
// right wall at half a cell (2 k on the diagonal, 2 k p in b), no flux on top
// and bottom. Row entries in column order: south, west, diagonal, east, north.
// The operations and their order are those of a plain elementwise assembly
// ((2a) b / (a + b), the diagonal -(((s + w) + e) + n) + wall), so the values
// equal such an assembly's bit for bit.
__device__ __forceinline__ double darcy_hmean(double a, double b) { return 2.0 * a * b / (a + b); }

__global__ void __launch_bounds__(kThreads) k_darcy2d_assemble(int n, const double* __restrict__ theta,
                                                               const int* __restrict__ rp, double* __restrict__ val,
                                                               double* __restrict__ b) {
  const int64_t cells = (int64_t)n * n;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < cells; r += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(r % n), j = (int)(r / n);
    const double kc = exp(theta[r]);
    const double south = j > 0 ? -darcy_hmean(exp(theta[r - n]), kc) : 0.0;
    const double west = i > 0 ? -darcy_hmean(exp(theta[r - 1]), kc) : 0.0;
    const double east = i < n - 1 ? -darcy_hmean(kc, exp(theta[r + 1])) : 0.0;
    const double north = j < n - 1 ? -darcy_hmean(kc, exp(theta[r + n])) : 0.0;
    const double wall = (0.0 + (i == 0 ? 2.0 * kc : 0.0)) + (i == n - 1 ? 2.0 * kc : 0.0);
    const double diag = -(((south + west) + east) + north) + wall;
    int k = rp[r];
    if (j > 0) val[k++] = south;
    if (i > 0) val[k++] = west;
    val[k++] = diag;
    if (i < n - 1) val[k++] = east;
    if (j < n - 1) val[k] = north;
    b[r] = i == 0 ? 2.0 * kc : 0.0;
  }
}

// dL/dtheta of the system above from x = A^-1 b and lambda = A^-T dL/dx
// (the face-coefficient chain rule; A symmetric). A face f between cells a and
// b adds k_f (e_a - e_b)(e_a - e_b)^T to A, so dL/dk_f = -(lambda_a - lambda_b)
// (x_a - x_b), and dk_f/dk_a = 2 k_b^2 / (k_a + k_b)^2. A left-wall cell has
// 2 k on the diagonal and 2 k in b: dL/dk += 2 lambda (1 - x); a right-wall
// cell 2 k on the diagonal: dL/dk -= 2 lambda x. Then dL/dtheta = k dL/dk.
__global__ void __launch_bounds__(kThreads) k_darcy2d_theta_grad(int n, const double* __restrict__ theta,
                                                                 const double* __restrict__ lam,
                                                                 const double* __restrict__ x,
                                                                 double* __restrict__ grad) {
  const int64_t cells = (int64_t)n * n;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < cells; r += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(r % n), j = (int)(r / n);
    const double kc = exp(theta[r]), lc = lam[r], xc = x[r];
    double g = 0.0;
    auto face = [&](int64_t q) {
      const double kq = exp(theta[q]);
      const double s = kc + kq;
      g += -(lc - lam[q]) * (xc - x[q]) * (2.0 * kq * kq / (s * s));
    };
    if (j > 0) face(r - n);
    if (i > 0) face(r - 1);
    if (i < n - 1) face(r + 1);
    if (j < n - 1) face(r + n);
    if (i == 0) g += 2.0 * lc * (1.0 - xc);
    if (i == n - 1) g -= 2.0 * lc * xc;
    grad[r] = g * kc;
  }
}

// The pattern of an n x n Darcy system as k_darcy2d_assemble writes it.
bool darcy2d_pattern_ok(const HostCsr& h, int64_t n) {
  if (n < 1 || h.nrows != n * n || h.ncols != n * n || h.nnz() != 5 * n * n - 4 * n) return false;
  for (int64_t r = 0; r < n * n; ++r) {
    const int64_t i = r % n, j = r / n;
    int64_t want[5], c = 0;
    if (j > 0) want[c++] = r - n;
    if (i > 0) want[c++] = r - 1;
    want[c++] = r;
    if (i < n - 1) want[c++] = r + 1;
    if (j < n - 1) want[c++] = r + n;
    if (h.rp[r + 1] - h.rp[r] != c) return false;
    for (int64_t q = 0; q < c; ++q)
      if (h.ci[h.rp[r] + q] != want[q]) return false;
  }
  return true;
}

cfd_status darcy2d_check(cfd_csr* a, int64_t n, const char* who) {
  if (a->darcy_n == n) return CFD_OK;
  if (n < 1 || n > 46340 || !darcy2d_pattern_ok(a->host, n)) {
    set_error("%s: the matrix is not the %lld x %lld cell Darcy pattern (rows i + n j; south, west, diagonal, "
              "east, north)", who, (long long)n, (long long)n);
    return CFD_ERR_DIM;
  }
  a->darcy_n = n;
  return CFD_OK;
}

__global__ void k_cast64to32(int64_t n, const double* __restrict__ s, float* __restrict__ d) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (float)s[i];
}

}  // namespace

cfd_status pattern_outer_launch(cfd_csr* a, const double* lambda, const double* x, double scale, double* g) {
  const int64_t n = a->dev.nrows;
  if (n == 0) return CFD_OK;
  const int grid = (int)std::min<int64_t>((n + kThreads - 1) / kThreads, (int64_t)a->ctx->num_sms * 8);
  k_pattern_outer<<<grid, kThreads, 0, a->ctx->stream>>>(n, a->dev.rp, a->dev.col, lambda, x, scale, g);
  a->ctx->stats.launches++;
  CFD_TRY_CUDA(cudaGetLastError());
  return CFD_OK;
}

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
  return pattern_outer_launch(a, lambda, x, scale, g);
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
  a->values_version++;
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

cfd_status cfd_darcy2d_assemble(cfd_csr* a, int64_t n, const double* theta, double* val, double* b) {
  return guarded("cfd_darcy2d_assemble", [&]() -> cfd_status {
    if (!a || !theta || !val || !b) {
      set_error("cfd_darcy2d_assemble: null argument");
      return CFD_ERR_STATE;
    }
    std::lock_guard<std::mutex> lk(a->ctx->mu);
    CFD_TRY(darcy2d_check(a, n, "cfd_darcy2d_assemble"));
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    const int grid = (int)std::min<int64_t>((n * n + kThreads - 1) / kThreads, (int64_t)a->ctx->num_sms * 8);
    k_darcy2d_assemble<<<grid, kThreads, 0, a->ctx->stream>>>((int)n, theta, a->dev.rp, val, b);
    a->ctx->stats.launches++;
    CFD_TRY_CUDA(cudaGetLastError());
    return CFD_OK;
  });
}

cfd_status cfd_darcy2d_theta_grad(cfd_csr* a, int64_t n, const double* theta, const double* lambda, const double* x,
                                  double* grad) {
  return guarded("cfd_darcy2d_theta_grad", [&]() -> cfd_status {
    if (!a || !theta || !lambda || !x || !grad) {
      set_error("cfd_darcy2d_theta_grad: null argument");
      return CFD_ERR_STATE;
    }
    std::lock_guard<std::mutex> lk(a->ctx->mu);
    CFD_TRY(darcy2d_check(a, n, "cfd_darcy2d_theta_grad"));
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    const int grid = (int)std::min<int64_t>((n * n + kThreads - 1) / kThreads, (int64_t)a->ctx->num_sms * 8);
    k_darcy2d_theta_grad<<<grid, kThreads, 0, a->ctx->stream>>>((int)n, theta, lambda, x, grad);
    a->ctx->stats.launches++;
    CFD_TRY_CUDA(cudaGetLastError());
    return CFD_OK;
  });
}

}  // extern "C"
