// ComponentBlockPreconditioner (crates/cfd-math/src/linear_solver/
// block_preconditioner.rs:609-976), the preconditioner of LinearSolverChain's
// GMRES + ComponentBlock tier (chain.rs:193-217), for 3-D saddle systems whose
// velocity block is component-major with three equal components and no
// coupling between them.
//
// Setup (host, from the matrix's values, new_with_symbols :707-826): each
// component block with cross-component entries above 1e-14 refused, its zero
// diagonals stabilized (stabilize_preconditioner_diagonal :71-107), then an
// exact inverse: the reference factors each block with its provider's sparse
// LU; here the block's dense inverse is formed on the device by the
// partial-pivoting Gauss-Jordan of the AMG coarsest level (an exact solve too;
// blocks of at most 8192 rows). The pressure Schur approximation
// C - D diag(A)^-1 G is assembled in the reference's entry order, stabilized,
// and lumped by signed row sums (lumped_pressure_preconditioner :112-137).
// Apply (the athena apply, :920-975), per component a dense product with the
// block inverse:
//   u* = A_c^-1 r_u;  p = (r_p - D u*) / lumped;  u = u* - A_c^-1 (G p).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "amg_device.h"
#include "internal.h"
#include "kernels.cuh"
#include "simple.h"

namespace cfd {

namespace {

constexpr double kCbEps = 1e-14;  // diagonal_epsilon (block_preconditioner.rs:40-42)

template <typename T>
cfd_status cb_put(T** d, const std::vector<T>& h, cudaStream_t s) {
  if (cudaMalloc((void**)d, std::max<size_t>(h.size(), 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *d = nullptr;
    set_error("cudaMalloc failed for a component-block array of %zu elements", h.size());
    return CFD_ERR_ALLOC;
  }
  if (!h.empty()) CFD_TRY_CUDA(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return CFD_OK;
}

std::vector<float> cb_narrow(const std::vector<double>& v) { return std::vector<float>(v.begin(), v.end()); }

// stabilize_preconditioner_diagonal over rows of (column -> value summed in
// entry order): a row whose diagonal is at most 1e-14 in magnitude gets
// max(row_scale * pivot_tolerance, 1e-14) added on the diagonal.
void cb_stabilize(std::vector<std::map<int64_t, double>>& rows, double pivot_tolerance) {
  for (int64_t r = 0; r < (int64_t)rows.size(); ++r) {
    double diag = 0.0, scale = 0.0;
    for (const auto& cv : rows[r]) {
      scale = std::max(scale, std::fabs(cv.second));
      if (cv.first == r) diag += cv.second;
    }
    if (std::fabs(diag) <= kCbEps) rows[r][r] += std::max(scale * pivot_tolerance, kCbEps);
  }
}

// y = inv x (sub = 0) or y -= inv x (sub = 1), inv an n x n FP64 row-major
// matrix; one warp per row, FP64 accumulation.
template <typename T>
__global__ void __launch_bounds__(256) k_cb_gemv(int n, const double* __restrict__ inv, const T* __restrict__ x,
                                                 T* __restrict__ y, int sub, const int* skip) {
  if (skip && *skip) return;
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (row >= n) return;
  const double* a = inv + (size_t)row * n;
  double s = 0.0;
  for (int k = lane; k < n; k += 32) s += a[k] * (double)x[k];
  s = warp_sum(s);
  if (lane == 0) y[row] = sub ? (T)((double)y[row] - s) : (T)s;
}

// z_p = (r_p - D z_u) / lumped, row by row in the reference's order.
template <typename T>
__global__ void k_cb_pressure(int64_t np, int64_t nv, const int* __restrict__ d_rp, const int* __restrict__ d_col,
                              const T* __restrict__ d_val, const T* __restrict__ pinv, const T* __restrict__ r,
                              T* __restrict__ z, const int* skip) {
  if (skip && *skip) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    T t = r[nv + i];
    for (int k = d_rp[i]; k < d_rp[i + 1]; ++k) t -= d_val[k] * z[d_col[k]];
    z[nv + i] = t * pinv[i];
  }
}

// gp_v = sum over the pressure columns of velocity row v (ascending) of G_vk p_k.
template <typename T>
__global__ void k_cb_grad(int64_t nv, const int* __restrict__ g_rp, const int* __restrict__ g_col,
                          const T* __restrict__ g_val, const T* __restrict__ z, T* __restrict__ gp, const int* skip) {
  if (skip && *skip) return;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    T t = T(0);
    for (int k = g_rp[v]; k < g_rp[v + 1]; ++k) t += g_val[k] * z[nv + g_col[k]];
    gp[v] = t;
  }
}

int cb_grid(const cfd_context* ctx, int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
}

}  // namespace

void component_free(ComponentDev* C) {
  if (!C) return;
  for (void* p : {(void*)C->inv[0], (void*)C->inv[1], (void*)C->inv[2], (void*)C->d_rp, (void*)C->d_col,
                  (void*)C->g_rp, (void*)C->g_col, (void*)C->d_val64, (void*)C->g_val64, (void*)C->pinv64,
                  (void*)C->d_val32, (void*)C->g_val32, (void*)C->pinv32, (void*)C->gp64, (void*)C->gp32})
    if (p) cudaFree(p);
  delete C;
}

// Builds the component blocks and the lumped pressure inverse from the host
// values. CFD_ERR_DIM for a split that is not three equal components,
// CFD_ERR_CONFIG for cross-component coupling, a block beyond the dense
// inverse limit or a singular block (the reference's constructor Errs).
cfd_status component_build(cfd_csr* a, int64_t nv, double pivot_tolerance, ComponentDev** out) {
  *out = nullptr;
  const HostCsr& h = a->host;
  const int64_t n = h.nrows;
  if (h.ncols != n || nv <= 0 || nv > n || nv % 3 != 0) {
    set_error("component-block preconditioner: velocity count %lld is not three equal components of a square "
              "system of %lld rows (block_preconditioner.rs:713-725)", (long long)nv, (long long)n);
    return CFD_ERR_DIM;
  }
  const int64_t cs = nv / 3;
  if (cs > kDenseInverseDeviceMaxRows) {
    set_error("component-block preconditioner: %lld rows per component exceed the dense inverse limit %lld",
              (long long)cs, (long long)kDenseInverseDeviceMaxRows);
    return CFD_ERR_CONFIG;
  }
  cudaStream_t s = a->ctx->stream;
  // freed on every early return and on unwinding; released to the caller at the end
  std::unique_ptr<ComponentDev, void (*)(ComponentDev*)> C(new ComponentDev, component_free);
  C->nv = nv;
  C->np = n - nv;
  C->cs = cs;
  for (int comp = 0; comp < 3; ++comp) {
    const int64_t off = comp * cs;
    std::vector<std::map<int64_t, double>> rows(cs);
    for (int64_t lr = 0; lr < cs; ++lr) {
      const int64_t g = off + lr;
      for (int64_t k = h.rp[g]; k < h.rp[g + 1]; ++k) {
        const int64_t col = h.ci[k];
        if (col >= nv) continue;
        if (col / cs != comp) {
          if (std::fabs(h.v[k]) > kCbEps) {
            set_error("velocity component coupling (%lld, %lld) is not supported by component-block "
                      "preconditioning (block_preconditioner.rs:736-742)", (long long)g, (long long)col);
            return CFD_ERR_CONFIG;
          }
          continue;
        }
        rows[lr][col - off] += h.v[k];
      }
    }
    cb_stabilize(rows, pivot_tolerance);
    std::vector<int> rp(cs + 1, 0), ci;
    std::vector<double> v;
    for (int64_t r = 0; r < cs; ++r) {
      for (const auto& cv : rows[r]) {
        ci.push_back((int)cv.first);
        v.push_back(cv.second);
      }
      rp[r + 1] = (int)ci.size();
    }
    int *drp = nullptr, *dci = nullptr;
    double* dv = nullptr;
    cfd_status st = cb_put(&drp, rp, s);
    if (st == CFD_OK) st = cb_put(&dci, ci, s);
    if (st == CFD_OK) st = cb_put(&dv, v, s);
    if (st == CFD_OK && cudaMalloc((void**)&C->inv[comp], (size_t)std::max<int64_t>(cs * cs, 1) * sizeof(double)) !=
                            cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc failed for a component-block inverse of %lld rows", (long long)cs);
      st = CFD_ERR_ALLOC;
    }
    if (st == CFD_OK) st = dense_inverse_device(a->ctx, cs, drp, dci, dv, C->inv[comp]);
    cudaStreamSynchronize(s);
    for (void* p : {(void*)drp, (void*)dci, (void*)dv})
      if (p) cudaFree(p);
    if (st != CFD_OK) {
      if (st == CFD_ERR_CONFIG)
        set_error("component-block preconditioner: velocity component %d block is singular", comp);
      return st;
    }
  }
  SimpleHost S;
  CFD_TRY(simple_build(h, nv, S));
  // pressure Schur approximation in the reference's entry order: the C block,
  // then per D entry (v, d) the G entries (v, pc, g) in ascending pc as -d dinv_v g
  std::vector<std::map<int64_t, double>> prow(C->np);
  for (int64_t i = 0; i < C->np; ++i) {
    auto& row = prow[i];
    for (int64_t k = h.rp[nv + i]; k < h.rp[nv + i + 1]; ++k)
      if (h.ci[k] >= nv && h.ci[k] < n) row[h.ci[k] - nv] += h.v[k];
    for (int32_t k = S.d_rp[i]; k < S.d_rp[i + 1]; ++k) {
      const int32_t vv = S.d_col[k];
      const double minv = S.dinv[vv];
      for (int32_t q = S.g_rp[vv]; q < S.g_rp[vv + 1]; ++q) row[S.g_col[q]] += -S.d_val[k] * minv * S.g_val[q];
    }
  }
  cb_stabilize(prow, pivot_tolerance);
  std::vector<double> pinv(C->np, 1.0);
  for (int64_t i = 0; i < C->np; ++i) {
    double sum = 0.0, diag = 0.0;
    for (const auto& cv : prow[i]) {
      sum += cv.second;
      if (cv.first == i) diag = cv.second;
    }
    const double scale = std::fabs(sum) > kCbEps ? sum : diag;
    pinv[i] = std::fabs(scale) > kCbEps ? 1.0 / scale : 1.0;
  }
  CFD_TRY(cb_put(&C->d_rp, S.d_rp, s));
  CFD_TRY(cb_put(&C->d_col, S.d_col, s));
  CFD_TRY(cb_put(&C->g_rp, S.g_rp, s));
  CFD_TRY(cb_put(&C->g_col, S.g_col, s));
  CFD_TRY(cb_put(&C->d_val64, S.d_val, s));
  CFD_TRY(cb_put(&C->g_val64, S.g_val, s));
  CFD_TRY(cb_put(&C->pinv64, pinv, s));
  CFD_TRY(cb_put(&C->d_val32, cb_narrow(S.d_val), s));
  CFD_TRY(cb_put(&C->g_val32, cb_narrow(S.g_val), s));
  CFD_TRY(cb_put(&C->pinv32, cb_narrow(pinv), s));
  CFD_TRY(cb_put(&C->gp64, std::vector<double>(nv, 0.0), s));
  CFD_TRY(cb_put(&C->gp32, std::vector<float>(nv, 0.0f), s));
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  *out = C.release();
  return CFD_OK;
}

cfd_status component_ensure(cfd_csr* a) {
  if (a->cblock_nv < 0) {
    set_error("component-block preconditioner requested but not set up on this matrix (cfd_component_block_setup)");
    return CFD_ERR_STATE;
  }
  if (a->cblock && !a->cblock_stale) return CFD_OK;
  ComponentDev* C = nullptr;
  CFD_TRY(component_build(a, a->cblock_nv, a->cblock_pivot_tolerance, &C));
  component_free(a->cblock);
  a->cblock = C;
  a->cblock_stale = false;
  return CFD_OK;
}

template <typename T>
cfd_status component_apply_device(cfd_csr* a, const T* r, T* z, const int* skip, cudaStream_t s) {
  const ComponentDev* C = a->cblock;
  const int cs = (int)C->cs;
  const int gg = (cs + 7) / 8;
  const T* dval;
  const T* gval;
  const T* pinv;
  T* gp;
  if constexpr (sizeof(T) == 8) {
    dval = C->d_val64;
    gval = C->g_val64;
    pinv = C->pinv64;
    gp = C->gp64;
  } else {
    dval = C->d_val32;
    gval = C->g_val32;
    pinv = C->pinv32;
    gp = C->gp32;
  }
  for (int comp = 0; comp < 3; ++comp)
    k_cb_gemv<T><<<gg, 256, 0, s>>>(cs, C->inv[comp], r + (int64_t)comp * cs, z + (int64_t)comp * cs, 0, skip);
  if (C->np > 0)
    k_cb_pressure<T><<<cb_grid(a->ctx, C->np), 256, 0, s>>>(C->np, C->nv, C->d_rp, C->d_col, dval, pinv, r, z,
                                                             skip);
  k_cb_grad<T><<<cb_grid(a->ctx, C->nv), 256, 0, s>>>(C->nv, C->g_rp, C->g_col, gval, z, gp, skip);
  for (int comp = 0; comp < 3; ++comp)
    k_cb_gemv<T><<<gg, 256, 0, s>>>(cs, C->inv[comp], gp + (int64_t)comp * cs, z + (int64_t)comp * cs, 1, skip);
  a->ctx->stats.launches += 7 + (C->np > 0);
  CFD_TRY_CUDA(cudaGetLastError());
  return CFD_OK;
}
template cfd_status component_apply_device<double>(cfd_csr*, const double*, double*, const int*, cudaStream_t);
template cfd_status component_apply_device<float>(cfd_csr*, const float*, float*, const int*, cudaStream_t);

}  // namespace cfd

using namespace cfd;

extern "C" {

cfd_status cfd_component_block_setup(cfd_csr* a, int64_t n_velocity, double pivot_tolerance) {
  return guarded("cfd_component_block_setup", [&]() -> cfd_status {
    if (!a) return CFD_ERR_STATE;
    if (!(pivot_tolerance >= 0.0) || !std::isfinite(pivot_tolerance)) {
      set_error("cfd_component_block_setup: pivot tolerance must be finite and >= 0");
      return CFD_ERR_CONFIG;
    }
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    ComponentDev* C = nullptr;
    CFD_TRY(component_build(a, n_velocity, pivot_tolerance, &C));
    component_free(a->cblock);
    a->cblock = C;
    a->cblock_nv = n_velocity;
    a->cblock_pivot_tolerance = pivot_tolerance;
    a->cblock_stale = false;
    return CFD_OK;
  });
}

cfd_status cfd_component_block_apply(cfd_csr* a, const double* r, double* z) {
  return guarded("cfd_component_block_apply", [&]() -> cfd_status {
    if (!a || !r || !z) return CFD_ERR_STATE;
    if (r == z) {
      set_error("cfd_component_block_apply: r and z must be different arrays");
      return CFD_ERR_STATE;
    }
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    CFD_TRY(component_ensure(a));
    CFD_TRY(component_apply_device<double>(a, r, z, nullptr, a->ctx->stream));
    CFD_TRY_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return CFD_OK;
  });
}

}  // extern "C"
