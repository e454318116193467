// Galerkin recompute of the AMG hierarchy on the device (AlgebraicMultigrid::
// recompute, amg.rs:179-214): with the transfer operators and every sparsity
// pattern fixed, new fine-level values flow down as A_{l+1} = (R_l A_l) P_l.
//
//  * k_spgemm_fixed forms the values of C = A B on C's known pattern: one warp
//    per row, one lane per entry, the entry summed over A's row in order with
//    separately rounded products, exactly as the host spgemm (stable order of
//    the terms per column) does, so device and host recomputes agree bit for
//    bit.
//  * The dense coarsest inverse is Gauss-Jordan with partial pivoting, the
//    host's dense_inverse step for step: per pivot one CTA finds the pivot
//    (first maximum), swaps, scales and saves the pivot column, then one grid
//    eliminates every other row.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "amg_device.h"
#include "amg_setup.h"
#include "internal.h"

namespace cfd {
namespace {

template <typename T>
cfd_status dalloc(T** p, int64_t n) {
  const cudaError_t e = cudaMalloc((void**)p, (size_t)std::max<int64_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) {
    set_error("cudaMalloc (%lld elements): %s", (long long)n, cudaGetErrorString(e));
    *p = nullptr;
    return CFD_ERR_ALLOC;
  }
  return CFD_OK;
}

// C = A B on C's pattern.
__global__ void __launch_bounds__(256) k_spgemm_fixed(int64_t nrows, const int* __restrict__ c_rp,
                                                      const int* __restrict__ c_ci, const int* __restrict__ a_rp,
                                                      const int* __restrict__ a_ci, const double* __restrict__ a_v,
                                                      const int* __restrict__ b_rp, const int* __restrict__ b_ci,
                                                      const double* __restrict__ b_v, double* __restrict__ c_v) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < nrows; row += warps) {
    const int a0 = a_rp[row], a1 = a_rp[row + 1];
    for (int e = c_rp[row] + lane; e < c_rp[row + 1]; e += 32) {
      const int j = c_ci[e];
      double s = 0.0;
      for (int ka = a0; ka < a1; ++ka) {
        const int k = a_ci[ka];
        int lo = b_rp[k], hi = b_rp[k + 1] - 1;
        while (lo <= hi) {
          const int mid = (lo + hi) >> 1;
          const int cm = b_ci[mid];
          if (cm == j) {
            s = __dadd_rn(s, __dmul_rn(a_v[ka], b_v[mid]));
            break;
          }
          if (cm < j)
            lo = mid + 1;
          else
            hi = mid - 1;
        }
      }
      c_v[e] = s;
    }
  }
}

__global__ void k_diag(int64_t n, const int* __restrict__ rp, const int* __restrict__ ci,
                       const double* __restrict__ v, double* __restrict__ d64, float* __restrict__ d32) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) d = v[k];
    d64[i] = d;
    if (d32) d32[i] = (float)d;
  }
}

__global__ void k_cast32(int64_t n, const double* __restrict__ s, float* __restrict__ d) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (float)s[i];
}

// m = A (dense, row-major), inv = I.
__global__ void k_dense_fill(int64_t n, const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ v, double* __restrict__ m, double* __restrict__ inv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    for (int k = rp[i]; k < rp[i + 1]; ++k) m[i * n + ci[k]] += v[k];
    inv[i * n + i] = 1.0;
  }
}

constexpr int kPivotThreads = 1024;

// Pivot c: first row of maximum |m[r][c]|, r >= c; swap it into row c (m from
// column c on, where the rows differ, inv whole); scale row c by 1/m[c][c];
// save the pivot column for the elimination. A zero pivot sets *err.
__global__ void __launch_bounds__(kPivotThreads) k_gj_pivot(int64_t n, int64_t c, double* m, double* inv,
                                                            double* fcol, int* err) {
  __shared__ double sv[kPivotThreads / 32];
  __shared__ int64_t sr[kPivotThreads / 32];
  __shared__ int64_t s_p;
  __shared__ double s_d;
  if (*err) return;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  double best = -1.0;
  int64_t br = n;
  for (int64_t r = c + tid; r < n; r += blockDim.x) {
    const double a = fabs(m[r * n + c]);
    if (a > best) {  // ascending r per thread: the first maximum
      best = a;
      br = r;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_down_sync(0xffffffffu, best, o);
    const int64_t orow = __shfl_down_sync(0xffffffffu, br, o);
    if (ob > best || (ob == best && orow < br)) {
      best = ob;
      br = orow;
    }
  }
  if (lane == 0) {
    sv[w] = best;
    sr[w] = br;
  }
  __syncthreads();
  if (tid == 0) {
    double b = sv[0];
    int64_t r = sr[0];
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q)
      if (sv[q] > b || (sv[q] == b && sr[q] < r)) {
        b = sv[q];
        r = sr[q];
      }
    s_p = r;
    if (!(b > 0.0)) *err = 1;
  }
  __syncthreads();
  if (*err) return;
  const int64_t p = s_p;
  if (p != c) {
    for (int64_t k = c + tid; k < n; k += blockDim.x) {
      const double t = m[c * n + k];
      m[c * n + k] = m[p * n + k];
      m[p * n + k] = t;
    }
    for (int64_t k = tid; k < n; k += blockDim.x) {
      const double t = inv[c * n + k];
      inv[c * n + k] = inv[p * n + k];
      inv[p * n + k] = t;
    }
  }
  __syncthreads();
  if (tid == 0) s_d = 1.0 / m[c * n + c];
  __syncthreads();
  const double d = s_d;
  __syncthreads();
  for (int64_t k = c + tid; k < n; k += blockDim.x) m[c * n + k] = __dmul_rn(m[c * n + k], d);
  for (int64_t k = tid; k < n; k += blockDim.x) inv[c * n + k] = __dmul_rn(inv[c * n + k], d);
  for (int64_t r = tid; r < n; r += blockDim.x) fcol[r] = r == c ? 0.0 : m[r * n + c];
}

// Rows r != c: row_r -= f_r row_c (m from column c on, inv whole); rows with
// f_r = 0 are left alone, as the host does.
__global__ void __launch_bounds__(256) k_gj_elim(int64_t n, int64_t c, double* m, double* inv,
                                                 const double* __restrict__ fcol, const int* err) {
  if (*err) return;
  const int64_t r = blockIdx.y;
  const double f = fcol[r];
  if (r == c || f == 0.0) return;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    if (k >= c) m[r * n + k] = __dsub_rn(m[r * n + k], __dmul_rn(f, m[c * n + k]));
    inv[r * n + k] = __dsub_rn(inv[r * n + k], __dmul_rn(f, inv[c * n + k]));
  }
}

cfd_status ensure_ra(cfd_amg* amg, cudaStream_t s) {
  for (size_t l = 0; l + 1 < amg->dev.size(); ++l) {
    DevRA& ra = amg->dev[l].ra;
    if (ra.rp) continue;
    const HostCsr RA = spgemm(amg->host[l].R, amg->host[l].A);  // pattern only (fixed)
    std::vector<int> rp(RA.nrows + 1);
    for (int64_t i = 0; i <= RA.nrows; ++i) rp[i] = (int)RA.rp[i];
    ra.nrows = RA.nrows;
    ra.nnz = RA.nnz();
    CFD_TRY(dalloc(&ra.rp, ra.nrows + 1));
    CFD_TRY(dalloc(&ra.ci, ra.nnz));
    CFD_TRY(dalloc(&ra.v, ra.nnz));
    CFD_TRY_CUDA(cudaMemcpyAsync(ra.rp, rp.data(), rp.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(ra.ci, RA.ci.data(), ra.nnz * sizeof(int), cudaMemcpyHostToDevice, s));
    CFD_TRY_CUDA(cudaStreamSynchronize(s));
  }
  return CFD_OK;
}

int grid_for(int64_t n, int per) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + per - 1) / per, 148 * 16)); }

}  // namespace

void free_ra(DevRA& ra) {
  if (ra.rp) cudaFree(ra.rp);
  if (ra.ci) cudaFree(ra.ci);
  if (ra.v) cudaFree(ra.v);
  ra = DevRA();
}

cfd_status amg_recompute_device(cfd_amg* amg, const cfd_csr* a) {
  cudaStream_t s = amg->ctx->stream;
  const size_t L = amg->dev.size();
  CFD_TRY(ensure_ra(amg, s));
  DevMat& A0 = amg->dev[0].A;
  CFD_TRY_CUDA(cudaMemcpyAsync(A0.v64, a->dev.v64, A0.nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
  for (size_t l = 0; l + 1 < L; ++l) {
    DevLevel& D = amg->dev[l];
    DevMat& Ac = amg->dev[l + 1].A;
    k_spgemm_fixed<<<grid_for(D.ra.nrows, 8), 256, 0, s>>>(D.ra.nrows, D.ra.rp, D.ra.ci, D.R.rp, D.R.col, D.R.v64,
                                                           D.A.rp, D.A.col, D.A.v64, D.ra.v);
    k_spgemm_fixed<<<grid_for(Ac.nrows, 8), 256, 0, s>>>(Ac.nrows, Ac.rp, Ac.col, D.ra.rp, D.ra.ci, D.ra.v, D.P.rp,
                                                         D.P.col, D.P.v64, Ac.v64);
    CFD_TRY_CUDA(cudaGetLastError());
  }
  for (size_t l = 0; l < L; ++l) {
    DevLevel& D = amg->dev[l];
    if (D.A.v32) k_cast32<<<grid_for(D.A.nnz, 256), 256, 0, s>>>(D.A.nnz, D.A.v64, D.A.v32);
    k_diag<<<grid_for(D.A.nrows, 256), 256, 0, s>>>(D.A.nrows, D.A.rp, D.A.col, D.A.v64, D.d64, D.d32);
    CFD_TRY_CUDA(cudaGetLastError());
  }
  if (amg->cfg.coarse_solve == CFD_COARSE_DENSE) {
    const DevMat& Ac = amg->dev[L - 1].A;
    const int64_t n = Ac.nrows;
    if (n > 65535) {  // one elimination row per grid row
      set_error("dense coarsest inverse: %lld rows exceed 65535", (long long)n);
      return CFD_ERR_CONFIG;
    }
    double *m = nullptr, *inv = nullptr, *fcol = nullptr;
    int* err = nullptr;
    cfd_status st = dalloc(&m, n * n);
    if (st == CFD_OK) st = dalloc(&inv, n * n);
    if (st == CFD_OK) st = dalloc(&fcol, n);
    if (st == CFD_OK) st = dalloc(&err, 1);
    int herr = 0;
    if (st == CFD_OK) {
      cudaMemsetAsync(m, 0, sizeof(double) * n * n, s);
      cudaMemsetAsync(inv, 0, sizeof(double) * n * n, s);
      cudaMemsetAsync(err, 0, sizeof(int), s);
      k_dense_fill<<<grid_for(n, 256), 256, 0, s>>>(n, Ac.rp, Ac.col, Ac.v64, m, inv);
      const dim3 eg((unsigned)std::min<int64_t>((n + 255) / 256, 64), (unsigned)n);
      for (int64_t c = 0; c < n; ++c) {
        k_gj_pivot<<<1, kPivotThreads, 0, s>>>(n, c, m, inv, fcol, err);
        k_gj_elim<<<eg, 256, 0, s>>>(n, c, m, inv, fcol, err);
      }
      cudaError_t e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) {
        set_error("coarsest inverse: %s", cudaGetErrorString(e));
        st = CFD_ERR_CUDA;
      } else if (herr) {
        set_error("AMG coarsest operator (%lld rows) is singular", (long long)n);
        st = CFD_ERR_CONFIG;
      }
    }
    if (st == CFD_OK) {
      if (amg->coarse_inv) cudaFree(amg->coarse_inv);
      amg->coarse_inv = inv;
      amg->coarse_n = n;
      inv = nullptr;
    }
    if (m) cudaFree(m);
    if (inv) cudaFree(inv);
    if (fcol) cudaFree(fcol);
    if (err) cudaFree(err);
    CFD_TRY(st);
  }
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  amg->host_values_stale = true;
  return CFD_OK;
}

cfd_status amg_sync_host_values(cfd_amg* amg) {
  if (!amg->host_values_stale) return CFD_OK;
  cudaStream_t s = amg->ctx->stream;
  for (size_t l = 0; l < amg->dev.size(); ++l)
    CFD_TRY_CUDA(cudaMemcpyAsync(amg->host[l].A.v.data(), amg->dev[l].A.v64, amg->dev[l].A.nnz * sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  amg->host_values_stale = false;
  return CFD_OK;
}

}  // namespace cfd
