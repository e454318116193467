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
//    host's dense_inverse operation for operation, in one cooperative launch
//    with one grid barrier per pivot (k_gj_coop, below).
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

// Blocks for n items at `per` items per block, capped at 16 blocks per SM.
int grid_for(const cfd_context* ctx, int64_t n, int per) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + per - 1) / per, (int64_t)ctx->num_sms * 16));
}

constexpr int kGjMaxRows = (int)kDenseInverseDeviceMaxRows;

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

// ---------------------------------------------------------------------------
// Dense coarsest inverse: Gauss-Jordan with partial pivoting in one
// cooperative launch, every element updated by the host's operations in the
// host's order (dense_inverse: pivot = first row of largest |m[r][c]|, r >= c;
// swap; scale the pivot row by d = 1/m[c][c]; row_r -= m[r][c] row_c for every
// r != c with m[r][c] != 0).
//
// Storage: row r of W (n + 1 entries) holds, at step c, the inverse columns
// already in use at 0..c-1 followed by m's live columns c..n-1 at c+1..n. An
// inverse column stays the unit vector of its row until that row becomes a
// pivot, so unit columns are not stored: the pivot of step c brings its
// column in at slot c, where m's column c-1 (dead from step c on) was. The
// final inverse is scattered by the pivots' original row numbers. Skipping
// the unit columns' zero updates changes at most the sign of a zero entry.
//
// Rows live in physical buffers reached through a per-CTA table; the swap is
// a table update and the new pivot row and the displaced row are written to
// two spare buffers, so no buffer read during a step is written in it and
// one grid barrier per step suffices. Per-CTA argmax partials of the next
// column (double-buffered by step parity) give every CTA the same pivot.

struct GjArgs {
  double* W;         // (n + 2) physical rows of ldw entries
  int ldw, n;
  double* part_v;    // 2 x grid: |value| of each CTA's candidate
  int* part_r;       // 2 x grid: its row (first of equal maxima)
  int* qcol;         // original row of the pivot of step j
  int* phys_out;     // final row table
  unsigned* bar;     // arrivals (monotone)
  int* err;          // 1: zero pivot, 2: barrier wait ran out
};

constexpr int kGjThreads = 512;
constexpr int kGjBatch = 16;
constexpr unsigned kGjSpinLimit = 1u << 21;  // each try is an L2 round trip: a second or two

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier (the launch is cooperative, so all CTAs are resident); the
// wait is bounded and gives up when another CTA has flagged an error.
__device__ bool gj_barrier(const GjArgs& g, unsigned target) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(g.bar, 1u);
    int ok = 1;
    unsigned i = 0;
    while (ld_acquire_u32(g.bar) < target) {
      if (++i > kGjSpinLimit) {
        atomicExch(g.err, 2);
        ok = 0;
        break;
      }
      if (*reinterpret_cast<volatile int*>(g.err)) {
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ void argmax_merge(double& bv, int& br, double v, int r) {
  if (v > bv || (v == bv && r < br)) {
    bv = v;
    br = r;
  }
}

// CTA-wide argmax of the per-warp candidates in lane 0 of each warp; thread 0 writes the partial.
__device__ void gj_cta_partial(const GjArgs& g, double bv, int br, int slot) {
  __shared__ double s_v[kGjThreads / 32];
  __shared__ int s_r[kGjThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s_v[warp] = bv;
    s_r[warp] = br;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = -1.0;
    int r = g.n;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) argmax_merge(v, r, s_v[w], s_r[w]);
    __stcg(g.part_v + (size_t)slot * gridDim.x + blockIdx.x, v);
    __stcg(g.part_r + (size_t)slot * gridDim.x + blockIdx.x, r);
  }
}

// W rows from the coarsest operator: slot 0 unused, m[r][k] at slot k + 1
// (duplicates summed in stored order, as the host fills its dense copy).
__global__ void k_gj_fill(int n, int ldw, const int* __restrict__ rp, const int* __restrict__ ci,
                          const double* __restrict__ v, double* __restrict__ W) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double* row = W + (size_t)i * ldw;
    for (int k = rp[i]; k < rp[i + 1]; ++k) row[ci[k] + 1] += v[k];
  }
}

__global__ void __launch_bounds__(kGjThreads, 1) k_gj_coop(GjArgs g) {
  extern __shared__ double gsm[];
  const int n = g.n, ldw = g.ldw;
  double* PW = gsm;        // scaled pivot row
  double* OC = gsm + ldw;  // old row c (moves to the pivot's position)
  int* phys = reinterpret_cast<int*>(gsm + 2 * ldw);
  int* orig = phys + n;
  __shared__ int s_spare[2];
  __shared__ int s_p;
  __shared__ double s_best;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nw = blockDim.x >> 5;
  const int gw = blockIdx.x * nw + warp, GW = gridDim.x * nw;
  for (int r = tid; r < n; r += blockDim.x) {
    phys[r] = r;
    orig[r] = r;
  }
  if (tid == 0) {
    s_spare[0] = n;
    s_spare[1] = n + 1;
  }
  {
    double bv = -1.0;
    int br = n;
    if (lane == 0)
      for (int r = gw; r < n; r += GW) argmax_merge(bv, br, fabs(__ldcg(g.W + (size_t)r * ldw + 1)), r);
    gj_cta_partial(g, bv, br, 0);
  }
  if (!gj_barrier(g, gridDim.x)) return;
  for (int c = 0; c < n; ++c) {
    // 1. pivot: every CTA reduces the same partials in the same order
    if (warp == 0) {
      double bv = -1.0;
      int br = n;
      for (int b = lane; b < (int)gridDim.x; b += 32)
        argmax_merge(bv, br, __ldcg(g.part_v + (size_t)(c & 1) * gridDim.x + b),
                     __ldcg(g.part_r + (size_t)(c & 1) * gridDim.x + b));
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, bv, o);
        const int orow = __shfl_down_sync(0xffffffffu, br, o);
        argmax_merge(bv, br, ov, orow);
      }
      if (lane == 0) {
        s_p = br;
        s_best = bv;
      }
    }
    __syncthreads();
    if (!(s_best > 0.0)) {  // zero pivot: the matrix is singular (every CTA sees it)
      if (tid == 0) atomicExch(g.err, 1);
      return;
    }
    const int p = s_p;
    const double* Wp = g.W + (size_t)phys[p] * ldw;
    const double* Wc = g.W + (size_t)phys[c] * ldw;
    const double d = 1.0 / __ldcg(Wp + c + 1);
    for (int j = tid; j <= n; j += blockDim.x) {
      PW[j] = j == c ? d : __dmul_rn(__ldcg(Wp + j), d);
      if (p != c) OC[j] = __ldcg(Wc + j);
    }
    __syncthreads();
    // 2. every row: r == c takes the pivot row, r == p the old row c; the rest in place
    double bv = -1.0;
    int br = n;
    const bool next = c + 1 < n;
    for (int r = gw; r < n; r += GW) {
      if (r == c) {
        double* dst = g.W + (size_t)s_spare[0] * ldw;
        for (int j = lane; j <= n; j += 32) __stcg(dst + j, PW[j]);
        continue;
      }
      const bool moved = (r == p);
      const double* src = moved ? OC : g.W + (size_t)phys[r] * ldw;
      double* dst = moved ? g.W + (size_t)s_spare[1] * ldw : g.W + (size_t)phys[r] * ldw;
      const double f = moved ? OC[c + 1] : __ldcg(src + c + 1);
      double nv = 0.0;
      if (f == 0.0) {
        if (moved) {
          for (int j = lane; j <= n; j += 32) __stcg(dst + j, j == c ? 0.0 : OC[j]);
        } else if (lane == 0) {
          __stcg(dst + c, 0.0);
        }
        if (next && lane == 0) nv = moved ? OC[c + 2] : __ldcg(src + c + 2);
      } else {
        // kGjBatch entries per lane are loaded before any is stored (dst may
        // be src, so the compiler would otherwise keep every load behind the
        // previous store)
        for (int base = 0; base <= n; base += 32 * kGjBatch) {
          double sv[kGjBatch];
#pragma unroll
          for (int u = 0; u < kGjBatch; ++u) {
            const int j = base + u * 32 + lane;
            sv[u] = (j <= n && j != c) ? (moved ? OC[j] : __ldcg(src + j)) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kGjBatch; ++u) {
            const int j = base + u * 32 + lane;
            if (j <= n) {
              const double v = __dsub_rn(sv[u], __dmul_rn(f, PW[j]));
              __stcg(dst + j, v);
              if (j == c + 2) nv = v;
            }
          }
        }
        if (next) nv = __shfl_sync(0xffffffffu, nv, (c + 2) & 31);
      }
      if (next && lane == 0 && r > c) argmax_merge(bv, br, fabs(nv), r);
    }
    __syncthreads();  // the row table is read above; update it
    if (tid == 0) {
      const int oc = phys[c], op = phys[p];
      phys[c] = s_spare[0];
      if (p != c) {
        phys[p] = s_spare[1];
        s_spare[1] = op;
        const int t = orig[c];
        orig[c] = orig[p];
        orig[p] = t;
      }
      s_spare[0] = oc;
      if (blockIdx.x == 0) g.qcol[c] = orig[c];
    }
    if (next) gj_cta_partial(g, bv, br, (c + 1) & 1);
    if (!gj_barrier(g, (unsigned)(c + 2) * gridDim.x)) return;
  }
  if (blockIdx.x == 0)
    for (int r = tid; r < n; r += blockDim.x) g.phys_out[r] = phys[r];
}

// inv[r][qcol[j]] = W[phys[r]][j].
__global__ void k_gj_scatter(int n, int ldw, const double* __restrict__ W, const int* __restrict__ phys,
                             const int* __restrict__ qcol, double* __restrict__ inv) {
  const int r = blockIdx.y;
  const double* row = W + (size_t)phys[r] * ldw;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    inv[(size_t)r * n + qcol[j]] = row[j];
}

}  // namespace

// Dense inverse of the n x n CSR operator (rp, ci, v on the device) into
// inv (n x n, row-major, device). Returns CFD_ERR_CONFIG for a singular operator.
cfd_status dense_inverse_device(cfd_context* ctx, int64_t n64, const int* rp, const int* ci, const double* v,
                                double* inv) {
  cudaStream_t s = ctx->stream;
  if (n64 > kGjMaxRows) {
    set_error("dense coarsest inverse: %lld rows exceed %d", (long long)n64, kGjMaxRows);
    return CFD_ERR_CONFIG;
  }
  const int n = (int)n64;
  if (n == 0) return CFD_OK;
  const int ldw = (n + 2) & ~1;
  const size_t smem = (size_t)2 * ldw * sizeof(double) + (size_t)2 * n * sizeof(int);
  CFD_TRY_CUDA(cudaFuncSetAttribute(k_gj_coop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  CFD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_gj_coop, kGjThreads, smem));
  if (occ < 1) {
    set_error("dense coarsest inverse: no resident CTA with %zu bytes of shared memory", smem);
    return CFD_ERR_CONFIG;
  }
  const int grid = ctx->num_sms;  // one CTA per SM keeps the grid barrier short
  GjArgs g{};
  g.ldw = ldw;
  g.n = n;
  double* W = nullptr;
  double* part_v = nullptr;
  int *part_r = nullptr, *qcol = nullptr, *phys = nullptr, *err = nullptr;
  unsigned* bar = nullptr;
  cfd_status st = dalloc(&W, (int64_t)(n + 2) * ldw);
  if (st == CFD_OK) st = dalloc(&part_v, 2 * grid);
  if (st == CFD_OK) st = dalloc(&part_r, 2 * grid);
  if (st == CFD_OK) st = dalloc(&qcol, n);
  if (st == CFD_OK) st = dalloc(&phys, n);
  if (st == CFD_OK) st = dalloc(&err, 1);
  if (st == CFD_OK) st = dalloc(&bar, 1);
  int herr = 0;
  if (st == CFD_OK) {
    cudaError_t e = cudaMemsetAsync(W, 0, sizeof(double) * (size_t)(n + 2) * ldw, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(bar, 0, sizeof(unsigned), s);
    if (e == cudaSuccess) {
      k_gj_fill<<<grid_for(ctx, n, 256), 256, 0, s>>>(n, ldw, rp, ci, v, W);
      e = cudaGetLastError();
    }
    g.W = W;
    g.part_v = part_v;
    g.part_r = part_r;
    g.qcol = qcol;
    g.phys_out = phys;
    g.bar = bar;
    g.err = err;
    if (e == cudaSuccess) {
      void* args[] = {&g};
      e = cudaLaunchCooperativeKernel((const void*)k_gj_coop, dim3(grid), dim3(kGjThreads), args, smem, s);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && herr == 0) {
      k_gj_scatter<<<dim3((unsigned)std::min((n + 255) / 256, 16), (unsigned)n), 256, 0, s>>>(n, ldw, W, phys,
                                                                                               qcol, inv);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e != cudaSuccess) {
      set_error("dense coarsest inverse: %s", cudaGetErrorString(e));
      st = CFD_ERR_CUDA;
    } else if (herr == 1) {
      set_error("AMG coarsest operator (%d rows) is singular", n);
      st = CFD_ERR_CONFIG;
    } else if (herr != 0) {
      set_error("dense coarsest inverse: a grid barrier wait ran out");
      st = CFD_ERR_CUDA;
    }
  }
  for (void* q : {(void*)W, (void*)part_v, (void*)part_r, (void*)qcol, (void*)phys, (void*)err, (void*)bar})
    if (q) cudaFree(q);
  return st;
}

namespace {

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
  const int64_t nc = amg->dev[L - 1].A.nrows;
  if (amg->cfg.coarse_solve == CFD_COARSE_DENSE && nc > kGjMaxRows) {
    set_error("dense coarsest inverse: %lld rows exceed %d", (long long)nc, kGjMaxRows);
    return CFD_ERR_CONFIG;
  }
  DevMat& A0 = amg->dev[0].A;
  amg->host_values_stale = true;  // from here on the device holds the newer values
  CFD_TRY_CUDA(cudaMemcpyAsync(A0.v64, a->dev.v64, A0.nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
  for (size_t l = 0; l + 1 < L; ++l) {
    DevLevel& D = amg->dev[l];
    DevMat& Ac = amg->dev[l + 1].A;
    k_spgemm_fixed<<<grid_for(amg->ctx, D.ra.nrows, 8), 256, 0, s>>>(
        D.ra.nrows, D.ra.rp, D.ra.ci, D.R.rp, D.R.col, D.R.v64, D.A.rp, D.A.col, D.A.v64, D.ra.v);
    k_spgemm_fixed<<<grid_for(amg->ctx, Ac.nrows, 8), 256, 0, s>>>(
        Ac.nrows, Ac.rp, Ac.col, D.ra.rp, D.ra.ci, D.ra.v, D.P.rp, D.P.col, D.P.v64, Ac.v64);
    CFD_TRY_CUDA(cudaGetLastError());
  }
  for (size_t l = 0; l < L; ++l) {
    DevLevel& D = amg->dev[l];
    if (D.A.v32) k_cast32<<<grid_for(amg->ctx, D.A.nnz, 256), 256, 0, s>>>(D.A.nnz, D.A.v64, D.A.v32);
    D.A.sl_stale = true;   // the sliced FP32 values are gathered again before their next use
    D.A.dia_stale = true;  // and the diagonal-major ones refilled
    k_diag<<<grid_for(amg->ctx, D.A.nrows, 256), 256, 0, s>>>(D.A.nrows, D.A.rp, D.A.col, D.A.v64, D.d64, D.d32);
    CFD_TRY_CUDA(cudaGetLastError());
  }
  if (amg->cfg.coarse_solve == CFD_COARSE_DENSE) {
    const DevMat& Ac = amg->dev[L - 1].A;
    double* inv = nullptr;
    CFD_TRY(dalloc(&inv, Ac.nrows * Ac.nrows));
    const cfd_status st = dense_inverse_device(amg->ctx, Ac.nrows, Ac.rp, Ac.col, Ac.v64, inv);
    if (st != CFD_OK) {
      cudaFree(inv);
      return st;
    }
    if (amg->coarse_inv) cudaFree(amg->coarse_inv);
    amg->coarse_inv = inv;
    amg->coarse_n = Ac.nrows;
    if (amg->coarse_inv32) {
      const int64_t nn = Ac.nrows * Ac.nrows;
      k_cast32<<<grid_for(amg->ctx, nn, 256), 256, 0, s>>>(nn, inv, amg->coarse_inv32);
      CFD_TRY_CUDA(cudaGetLastError());
    }
  }
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
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
