// Batched Jacobi-PCG for many small independent systems (Kirchhoff networks of
// the 1-D solver, one per design candidate) in one persistent launch per size
// bucket, replayed from a captured CUDA graph.
//
// Each CTA takes systems from a longest-first queue (atomic ticket) and keeps
// the whole system -- values, 16-bit local columns, row offsets and the PCG
// vectors -- resident in shared memory for the entire solve, so an iteration
// touches no global memory. Per bucket of system sizes the CTA width (one warp
// up to 512 threads) is chosen by timing the candidates on the batch itself
// (cfd_batch_autotune).
//
// Recurrence: the PCG of krylov::cg_preconditioned with the DiagJacobi
// preconditioner (crates/cfd-1d/src/solver/core/linear_system.rs:270-332). The
// convergence test is the row-equilibrated residual of the same solver,
// ||D (b - A x)|| <= tol * ||D b||, D = 1 / max_j |a_ij| (linear_system.rs:157-204).
// FP32_REFINE keeps the inner recurrence in FP32 shared memory and forms the
// outer residual b - A x and the solution update in FP64 from global memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <vector>

#include "batch_internal.h"
#include "internal.h"
#include "kernels.cuh"

namespace cfd {
namespace {

constexpr int kCandidates[] = {32, 64, 128, 256, 512};  // threads per system
constexpr int kGroupCandidates[] = {1, 2, 4};             // systems per CTA

struct BatchSys {
  const int* __restrict__ sys_row;   // first global row of each system (nsys + 1)
  const int* __restrict__ rp;        // global row offsets (total_rows + 1)
  const int* __restrict__ col;       // local column index within the system
  const double* __restrict__ v64;
  const float* __restrict__ v32;
};

struct BatchOut {
  double* __restrict__ x;  // solution / initial guess (FP64, global rows)
  const double* __restrict__ b;
  int* term;
  int* iters;
  double* resid;  // final equilibrated relative residual
};

// Shared-memory layout of a bucket, every region starting on a 16-byte
// boundary: values (T[zmax]), local columns (u16[zmax]), row offsets
// (int[nmax + 1]), then six T[nmax] vectors.
__host__ __device__ constexpr size_t round16(size_t b) { return (b + 15) / 16 * 16; }
template <typename T>
__host__ __device__ constexpr size_t batch_col_off(int zmax) {
  return round16((size_t)zmax * sizeof(T));
}
template <typename T>
__host__ __device__ constexpr size_t batch_rp_off(int zmax) {
  return batch_col_off<T>(zmax) + round16((size_t)zmax * 2);
}
template <typename T>
__host__ __device__ constexpr size_t batch_vec_off(int nmax, int zmax) {
  return batch_rp_off<T>(zmax) + round16((size_t)(nmax + 1) * 4);
}
template <typename T>
__host__ __device__ constexpr size_t batch_smem(int nmax, int zmax) {
  return batch_vec_off<T>(nmax, zmax) + 6 * round16((size_t)nmax * sizeof(T));
}

// A CTA runs G independent system groups of blockDim / G threads (G = 1, 2 or
// 4; a group is a whole number of warps). A group synchronises on its own
// named barrier (1 + group; the CTA-wide barrier 0 when G = 1; the warp
// barrier when the group is one warp), so groups that run systems of
// different lengths never wait for one another.
constexpr int kMaxGroups = 4;
struct Group {
  int g, gsz, t;  // group, threads per group, thread within the group
  __device__ Group(int groups) {
    gsz = (int)blockDim.x / groups;
    g = (int)threadIdx.x / gsz;
    t = (int)threadIdx.x - g * gsz;
  }
  __device__ __forceinline__ void sync(int groups) const {
    if (groups == 1)
      __syncthreads();
    else if (gsz == 32)
      __syncwarp();
    else
      asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(gsz) : "memory");
  }
};

// Sum over the group, result in every thread. `slot` alternates between calls
// so one barrier suffices between consecutive reductions.
__device__ __forceinline__ double group_sum(double v, double* buf, const Group& G, int groups) {
  const int lane = G.t & 31, w = G.t >> 5, nw = G.gsz >> 5;
  v = warp_sum(v);
  if (nw == 1) return __shfl_sync(0xffffffffu, v, 0);
  if (lane == 0) buf[w] = v;
  G.sync(groups);
  double t = lane < nw ? buf[lane] : 0.0;
  t = warp_sum(t);
  t = __shfl_sync(0xffffffffu, t, 0);
  return t;
}

template <typename T, bool REFINE>
__global__ void k_batch_pcg(BatchSys S, BatchOut O, const int* __restrict__ order, int count, unsigned* queue,
                            const BatchParams* __restrict__ prm, int nmax, int zmax, int groups) {
  extern __shared__ __align__(16) unsigned char smem_all[];
  const Group G(groups);
  unsigned char* sm = smem_all + (size_t)G.g * round16(batch_smem<T>(nmax, zmax));
  T* sv = reinterpret_cast<T*>(sm);
  unsigned short* sc = reinterpret_cast<unsigned short*>(sm + batch_col_off<T>(zmax));
  int* srp = reinterpret_cast<int*>(sm + batch_rp_off<T>(zmax));
  const size_t vstride = round16((size_t)nmax * sizeof(T));
  unsigned char* vbase = sm + batch_vec_off<T>(nmax, zmax);
  T* vx = reinterpret_cast<T*>(vbase);
  T* vr = reinterpret_cast<T*>(vbase + vstride);
  T* vp = reinterpret_cast<T*>(vbase + 2 * vstride);
  T* vq = reinterpret_cast<T*>(vbase + 3 * vstride);
  T* vj = reinterpret_cast<T*>(vbase + 4 * vstride);  // 1 / a_ii (identity where |a_ii| <= eps)
  T* vs = reinterpret_cast<T*>(vbase + 5 * vstride);  // equilibration scale 1 / max_j |a_ij|
  __shared__ double reds[kMaxGroups][2][32];
  __shared__ int s_ks[kMaxGroups];
  double(*red)[32] = reds[G.g];
  int& s_k = s_ks[G.g];
  const int tid = G.t, nt = G.gsz;
  const BatchParams P = *prm;
  auto gsync = [&]() { G.sync(groups); };

  for (;;) {
    if (tid == 0) s_k = (int)atomicAdd(queue, 1u);
    gsync();
    const int k = s_k;
    gsync();
    if (k >= count) break;
    const int sys = order[k];
    const int r0 = S.sys_row[sys], n = S.sys_row[sys + 1] - r0;
    const int k0 = S.rp[r0], nnz = S.rp[r0 + n] - k0;
    // ---- stage the system ----
    for (int i = tid; i <= n; i += nt) srp[i] = S.rp[r0 + i] - k0;
    for (int e = tid; e < nnz; e += nt) {
      sv[e] = REFINE ? (T)S.v32[k0 + e] : (T)S.v64[k0 + e];
      sc[e] = (unsigned short)S.col[k0 + e];
    }
    gsync();
    for (int i = tid; i < n; i += nt) {
      double d = 0.0, mx = 0.0;
      for (int e = srp[i]; e < srp[i + 1]; ++e) {
        const double a = REFINE ? (double)S.v64[k0 + e] : (double)sv[e];
        if (sc[e] == i) d = a;
        mx = fmax(mx, fabs(a));
      }
      vj[i] = (T)(fabs(d) <= DBL_EPSILON ? 1.0 : 1.0 / d);
      vs[i] = (T)((mx > DBL_EPSILON && isfinite(mx)) ? 1.0 / mx : 1.0);
    }
    gsync();
    int term = CFD_TERM_MAX_ITERATIONS, it_total = 0;
    double e_rel = 0.0;
    int slot = 0;
    auto sum = [&](double v) {
      const double t = group_sum(v, red[slot], G, groups);
      slot ^= 1;
      return t;
    };
    // Inner PCG on (A, rhs in vr) from x = vx; returns iterations; sets term.
    auto pcg = [&](double thr_rel, int max_it, double& e0_out, double& e_out, int& term_out, bool abs_thr,
                   double thr_abs) {
      double rho = 0.0, e2 = 0.0;
      for (int i = tid; i < n; i += nt) {
        const T ri = vr[i];
        const T zi = ri * vj[i];
        vp[i] = zi;
        rho += (double)ri * (double)zi;
        const double si = (double)vs[i] * (double)ri;
        e2 += si * si;
      }
      rho = sum(rho);
      e2 = sum(e2);
      const double e0 = sqrt(e2);
      e0_out = e0;
      e_out = e0;
      const double thr = abs_thr ? fmax(thr_abs, thr_rel * e0) : thr_rel * e0;
      if (!isfinite(e0)) {
        term_out = CFD_TERM_BREAKDOWN;
        return 0;
      }
      if (e0 <= thr) {
        term_out = CFD_TERM_INITIAL_RESIDUAL;
        return 0;
      }
      gsync();
      for (int it = 1; it <= max_it; ++it) {
        double pq = 0.0;
        for (int i = tid; i < n; i += nt) {
          T s = T(0);
          for (int e = srp[i]; e < srp[i + 1]; ++e) s += sv[e] * vp[sc[e]];
          vq[i] = s;
          pq += (double)vp[i] * (double)s;
        }
        pq = sum(pq);
        if (!(pq > 0.0)) {
          term_out = CFD_TERM_NON_POSITIVE_CURVATURE;
          return it - 1;
        }
        const T alpha = (T)(rho / pq);
        double rz = 0.0;
        e2 = 0.0;
        for (int i = tid; i < n; i += nt) {
          vx[i] = vx[i] + alpha * vp[i];
          const T ri = vr[i] - alpha * vq[i];
          vr[i] = ri;
          rz += (double)ri * (double)(ri * vj[i]);
          const double si = (double)vs[i] * (double)ri;
          e2 += si * si;
        }
        rz = sum(rz);
        e2 = sum(e2);
        const double e = sqrt(e2);
        e_out = e;
        if (!isfinite(e)) {
          term_out = CFD_TERM_BREAKDOWN;
          return it;
        }
        if (e <= thr) {
          term_out = CFD_TERM_CONVERGED;
          return it;
        }
        if (rz == 0.0 || !isfinite(rz)) {
          term_out = CFD_TERM_BREAKDOWN;
          return it;
        }
        const T beta = (T)(rz / rho);
        rho = rz;
        for (int i = tid; i < n; i += nt) vp[i] = vr[i] * vj[i] + beta * vp[i];
        gsync();
      }
      term_out = CFD_TERM_MAX_ITERATIONS;
      return max_it;
    };

    if (!REFINE) {
      // r = b - A x0 in shared memory.
      for (int i = tid; i < n; i += nt) vx[i] = (T)O.x[r0 + i];
      gsync();
      for (int i = tid; i < n; i += nt) {
        T s = T(0);
        for (int e = srp[i]; e < srp[i + 1]; ++e) s += sv[e] * vx[sc[e]];
        vr[i] = (T)O.b[r0 + i] - s;
      }
      gsync();
      double e0, e;
      it_total = pcg(P.tol_rel, P.max_iter, e0, e, term, true, P.tol_abs);
      e_rel = e0 > 0.0 ? e / e0 : 0.0;
      gsync();
      for (int i = tid; i < n; i += nt) O.x[r0 + i] = (double)vx[i];
    } else {
      // Outer FP64 residual and update from global memory, inner FP32 PCG.
      double e_first = -1.0, thr = 0.0;
      term = CFD_TERM_MAX_ITERATIONS;
      for (int outer = 0; outer <= P.max_outer; ++outer) {
        double r2 = 0.0, e2 = 0.0;
        for (int i = tid; i < n; i += nt) {
          double s = 0.0;
          for (int e = srp[i]; e < srp[i + 1]; ++e) s += S.v64[k0 + e] * O.x[r0 + sc[e]];
          const double ri = O.b[r0 + i] - s;
          r2 += ri * ri;
          const double si = (double)vs[i] * ri;
          e2 += si * si;
        }
        r2 = sum(r2);
        e2 = sum(e2);
        const double e = sqrt(e2), rn = sqrt(r2);
        if (e_first < 0.0) {
          e_first = e;
          thr = fmax(P.tol_abs, P.tol_rel * e);
        }
        e_rel = e_first > 0.0 ? e / e_first : 0.0;
        if (!isfinite(e)) {
          term = CFD_TERM_BREAKDOWN;
          break;
        }
        if (e <= thr) {
          term = (outer == 0) ? CFD_TERM_INITIAL_RESIDUAL : CFD_TERM_CONVERGED;
          break;
        }
        if (outer == P.max_outer || it_total >= P.max_iter) break;
        const double scale = 1.0 / rn;
        gsync();
        for (int i = tid; i < n; i += nt) {
          double s = 0.0;
          for (int e2i = srp[i]; e2i < srp[i + 1]; ++e2i) s += S.v64[k0 + e2i] * O.x[r0 + sc[e2i]];
          vr[i] = (T)((O.b[r0 + i] - s) * scale);
          vx[i] = T(0);
        }
        gsync();
        double ie0, ie;
        int iterm = CFD_TERM_MAX_ITERATIONS;
        const int its = pcg(P.inner_tol, P.max_iter - it_total, ie0, ie, iterm, false, 0.0);
        it_total += its;
        gsync();
        for (int i = tid; i < n; i += nt) O.x[r0 + i] += (double)vx[i] / scale;
        gsync();
        if (iterm == CFD_TERM_BREAKDOWN || iterm == CFD_TERM_NON_POSITIVE_CURVATURE) {
          term = iterm;
          break;
        }
      }
    }
    if (tid == 0) {
      O.term[sys] = term;
      O.iters[sys] = it_total;
      O.resid[sys] = e_rel;
    }
    gsync();
  }
}

}  // namespace
}  // namespace cfd

using namespace cfd;

namespace {

template <typename T>
cfd_status dalloc(T** p, int64_t n) {
  if (cudaMalloc((void**)p, (size_t)std::max<int64_t>(n + 16, 16) * sizeof(T)) != cudaSuccess) {
    set_error("cudaMalloc failed for a batch buffer of %lld elements", (long long)n);
    *p = nullptr;
    return CFD_ERR_ALLOC;
  }
  return CFD_OK;
}

// Shared-memory size, attribute and persistent grid of bucket k at `threads`.
// `threads` per system, `groups` systems per CTA.
template <bool REFINE>
cfd_status prepare_bucket(cfd_batch* bt, int bkt, int threads, int groups, int* grid, size_t* smem_out) {
  using T = typename std::conditional<REFINE, float, double>::type;
  const int count = bt->bucket_begin[bkt + 1] - bt->bucket_begin[bkt];
  *grid = 0;
  if (count == 0) return CFD_OK;
  const size_t smem = (size_t)groups * round16(batch_smem<T>(bt->bucket_nmax[bkt], bt->bucket_zmax[bkt]));
  threads *= groups;
  auto kern = k_batch_pcg<T, REFINE>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    set_error("batch bucket %d: %zu bytes of shared memory are not available", bkt, smem);
    return CFD_ERR_CONFIG;
  }
  int occ = 0;
  CFD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem));
  if (occ < 1) {
    set_error("batch bucket %d: %zu bytes of shared memory at %d threads do not fit", bkt, smem, threads);
    return CFD_ERR_CONFIG;
  }
  *grid = std::min((count + groups - 1) / groups, bt->ctx->num_sms * occ);
  *smem_out = smem;
  return CFD_OK;
}

template <bool REFINE>
cfd_status launch_bucket(cfd_batch* bt, int bkt, int threads, int groups, int grid, size_t smem, cudaStream_t s) {
  using T = typename std::conditional<REFINE, float, double>::type;
  const int count = bt->bucket_begin[bkt + 1] - bt->bucket_begin[bkt];
  if (count == 0 || grid == 0) return CFD_OK;
  BatchSys S{bt->sys_row, bt->rp, bt->col, bt->v64, bt->v32};
  BatchOut O{bt->x, bt->b, bt->term, bt->iters, bt->resid};
  k_batch_pcg<T, REFINE><<<grid, threads * groups, smem, s>>>(S, O, bt->order + bt->bucket_begin[bkt], count,
                                                               bt->queues + bkt, bt->params, bt->bucket_nmax[bkt],
                                                               bt->bucket_zmax[bkt], groups);
  CFD_TRY_CUDA(cudaGetLastError());
  return CFD_OK;
}

template <bool REFINE>
cfd_status run_bucket(cfd_batch* bt, int bkt, int threads, int groups, cudaStream_t s) {
  int grid = 0;
  size_t smem = 0;
  CFD_TRY(prepare_bucket<REFINE>(bt, bkt, threads, groups, &grid, &smem));
  return launch_bucket<REFINE>(bt, bkt, threads, groups, grid, smem, s);
}

// The device part of one batched solve: reset the queues, one persistent
// launch per bucket (largest systems first).
cfd_status enqueue_solve(cfd_batch* bt, int prec, const int* grid, const size_t* smem, cudaStream_t s) {
  CFD_TRY_CUDA(cudaMemsetAsync(bt->queues, 0, kBuckets * sizeof(unsigned), s));
  for (int k = kBuckets - 1; k >= 0; --k) {
    if (prec)
      CFD_TRY(launch_bucket<true>(bt, k, bt->threads[prec][k], bt->groups[prec][k], grid[k], smem[k], s));
    else
      CFD_TRY(launch_bucket<false>(bt, k, bt->threads[prec][k], bt->groups[prec][k], grid[k], smem[k], s));
  }
  return CFD_OK;
}

cfd_status capture_graph(cfd_batch* bt, int prec) {
  if (bt->graph[prec]) return CFD_OK;
  // Captured on the context's own stream, whatever stream the solve runs on:
  // CUDA does not capture the legacy default stream (torch's default stream
  // arrives as cudaStreamLegacy), and the graph launches into any stream.
  cudaStream_t s = bt->ctx->own;
  int grid[kBuckets];
  size_t smem[kBuckets] = {};
  for (int k = 0; k < kBuckets; ++k) {
    if (prec)
      CFD_TRY(prepare_bucket<true>(bt, k, bt->threads[prec][k], bt->groups[prec][k], &grid[k], &smem[k]));
    else
      CFD_TRY(prepare_bucket<false>(bt, k, bt->threads[prec][k], bt->groups[prec][k], &grid[k], &smem[k]));
  }
  // The buckets share one kernel per precision: its shared-memory limit must
  // cover the largest of them (with several systems per CTA a small-row
  // bucket can need more than a larger one).
  const size_t smem_max = *std::max_element(smem, smem + kBuckets);
  if (smem_max > 0) {
    const cudaError_t ea =
        prec ? cudaFuncSetAttribute(k_batch_pcg<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_max)
             : cudaFuncSetAttribute(k_batch_pcg<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_max);
    if (ea != cudaSuccess) {
      cudaGetLastError();
      set_error("batch: %zu bytes of shared memory are not available", smem_max);
      return CFD_ERR_CONFIG;
    }
  }
  cudaGraph_t g = nullptr;
  CFD_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cfd_status st = enqueue_solve(bt, prec, grid, smem, s);
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (st != CFD_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) {
    set_error("batch graph capture: %s", cudaGetErrorString(e));
    return CFD_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&bt->graph[prec], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    set_error("batch graph instantiate: %s", cudaGetErrorString(e));
    bt->graph[prec] = nullptr;
    return CFD_ERR_CUDA;
  }
  return CFD_OK;
}

void drop_graphs(cfd_batch* bt) {
  for (auto& g : bt->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

cfd_status set_params(cfd_batch* bt, const cfd_solver_config& cfg, const cfd_solve_options& opt) {
  bt->h_params->tol_abs = cfg.tolerance;
  bt->h_params->tol_rel = cfg.relative_tolerance;
  bt->h_params->inner_tol = opt.inner_tolerance > 0 ? opt.inner_tolerance : 1e-4;
  bt->h_params->max_iter = (int32_t)std::min<int64_t>(cfg.max_iterations, INT32_MAX);
  bt->h_params->max_outer = opt.max_outer > 0 ? opt.max_outer : 20;
  CFD_TRY_CUDA(cudaMemcpyAsync(bt->params, bt->h_params, sizeof(BatchParams), cudaMemcpyHostToDevice,
                               bt->ctx->stream));
  return CFD_OK;
}

}  // namespace

namespace cfd {

// The caller's layout, checked in an order that never indexes past what the
// earlier checks have bounded: the offsets (num_systems + 1 of them, from 0,
// non-decreasing, ending at the total row count), then per system its rows
// (row_ptr non-decreasing and within [0, nnz]) before its local columns.
// Touches no device state.
cfd_status batch_validate(int32_t num_systems, const int64_t* sys_row_offsets, const int64_t* row_ptr,
                          const int32_t* col, const double* val) {
  if (num_systems < 0 || !sys_row_offsets || !row_ptr) {
    set_error("cfd_batch_create: invalid arguments");
    return CFD_ERR_STATE;
  }
  const int64_t rows = sys_row_offsets[num_systems];
  if (sys_row_offsets[0] != 0 || rows < 0 || rows >= INT32_MAX) {
    set_error("cfd_batch_create: system offsets must start at 0 and end at a row count that fits int32");
    return CFD_ERR_DIM;
  }
  const int64_t nnz = row_ptr[rows];
  if (row_ptr[0] != 0 || nnz < 0 || nnz >= INT32_MAX) {
    set_error("cfd_batch_create: row_ptr must start at 0 and end at a nonzero count that fits int32");
    return CFD_ERR_DIM;
  }
  if (nnz > 0 && (!col || !val)) {
    set_error("cfd_batch_create: null column or value array");
    return CFD_ERR_DIM;
  }
  for (int s = 0; s < num_systems; ++s) {
    const int64_t r0 = sys_row_offsets[s], r1 = sys_row_offsets[s + 1];
    if (r1 < r0 || r1 > rows) {
      set_error("cfd_batch_create: system offsets decrease or pass the row count at system %d", s);
      return CFD_ERR_DIM;
    }
    for (int64_t i = r0; i < r1; ++i)
      if (row_ptr[i + 1] < row_ptr[i] || row_ptr[i + 1] > nnz) {
        set_error("cfd_batch_create: row_ptr decreases or passes nnz at row %lld", (long long)i);
        return CFD_ERR_DIM;
      }
    if (r1 - r0 > kBatchMaxRows || row_ptr[r1] - row_ptr[r0] > kBatchMaxNnz) {
      set_error("cfd_batch_create: system %d has %lld rows / %lld nonzeros; the batched solver holds at most "
                "%d rows and %d nonzeros per system (use cfd_solve for larger systems)",
                s, (long long)(r1 - r0), (long long)(row_ptr[r1] - row_ptr[r0]), kBatchMaxRows, kBatchMaxNnz);
      return CFD_ERR_DIM;
    }
    for (int64_t e = row_ptr[r0]; e < row_ptr[r1]; ++e)
      if (col[e] < 0 || col[e] >= r1 - r0) {
        set_error("cfd_batch_create: local column %d out of range in system %d", col[e], s);
        return CFD_ERR_DIM;
      }
  }
  return CFD_OK;
}

cfd_status batch_build(cfd_context* ctx, int32_t num_systems, const int64_t* sys_row_offsets,
                       const int64_t* row_ptr, const int32_t* col, const double* val, cfd_batch** out) {
  const int64_t rows = sys_row_offsets[num_systems];
  const int64_t nnz = row_ptr[rows];
  std::lock_guard<std::mutex> g(ctx->mu);
  CFD_TRY_CUDA(cudaSetDevice(ctx->device));
  cfd_batch* bt = new cfd_batch;
  OnUnwind release([&] { cfd_batch_destroy(bt); });
  bt->ctx = ctx;
  bt->nsys = num_systems;
  bt->rows = rows;
  bt->nnz = nnz;
  bt->h_sys_row.resize(num_systems + 1);
  for (int s = 0; s <= num_systems; ++s) bt->h_sys_row[s] = (int)sys_row_offsets[s];
  std::vector<int> rp32(rows + 1);
  for (int64_t i = 0; i <= rows; ++i) rp32[i] = (int)row_ptr[i];
  // Buckets by row count (bucket 0 also takes empty systems), largest system
  // first inside each bucket.
  std::vector<int> ord(num_systems);
  std::iota(ord.begin(), ord.end(), 0);
  auto nrows = [&](int s) { return bt->h_sys_row[s + 1] - bt->h_sys_row[s]; };
  auto bucket_of = [&](int s) {
    int k = 0;
    while (k + 1 < kBuckets && nrows(s) > kBucketRows[k]) ++k;
    return k;
  };
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
    const int ka = bucket_of(a), kb = bucket_of(b);
    return ka != kb ? ka < kb : nrows(a) > nrows(b);
  });
  std::vector<int> sorted = ord;
  bt->h_order = sorted;
  for (int k = 0; k <= kBuckets; ++k) bt->bucket_begin[k] = num_systems;
  for (int q = num_systems - 1; q >= 0; --q) bt->bucket_begin[bucket_of(sorted[q])] = q;
  for (int k = kBuckets - 1; k >= 0; --k)
    if (bt->bucket_begin[k] > bt->bucket_begin[k + 1]) bt->bucket_begin[k] = bt->bucket_begin[k + 1];
  for (int k = 0; k < kBuckets; ++k) {
    int nmax = 1, zmax = 1;
    for (int q = bt->bucket_begin[k]; q < bt->bucket_begin[k + 1]; ++q) {
      const int sy = sorted[q];
      nmax = std::max(nmax, nrows(sy));
      zmax = std::max(zmax, (int)(row_ptr[bt->h_sys_row[sy + 1]] - row_ptr[bt->h_sys_row[sy]]));
    }
    bt->bucket_nmax[k] = nmax;
    bt->bucket_zmax[k] = zmax;
  }
  cudaStream_t s = ctx->stream;
  cfd_status st = CFD_OK;
  auto fail = [&](cfd_status e) {
    cfd_batch_destroy(bt);
    return e;
  };
  if ((st = dalloc(&bt->sys_row, num_systems + 1)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->rp, rows + 1)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->col, nnz)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->v64, nnz)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->v32, nnz)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->x, rows)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->b, rows)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->term, num_systems)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->iters, num_systems)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->resid, num_systems)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->order, num_systems)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->queues, kBuckets)) != CFD_OK) return fail(st);
  if ((st = dalloc(&bt->params, 1)) != CFD_OK) return fail(st);
  if (cudaMallocHost((void**)&bt->h_params, sizeof(BatchParams)) != cudaSuccess) return fail(CFD_ERR_ALLOC);
  std::vector<float> v32(val, val + nnz);
  for (int64_t k = 0; k < nnz; ++k)
    if (std::isfinite(val[k]) && !std::isfinite(v32[k])) bt->f32_out_of_range = true;
  if (cudaMemcpyAsync(bt->sys_row, bt->h_sys_row.data(), (num_systems + 1) * sizeof(int), cudaMemcpyHostToDevice,
                      s) != cudaSuccess ||
      cudaMemcpyAsync(bt->rp, rp32.data(), (rows + 1) * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(bt->col, col, nnz * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(bt->v64, val, nnz * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(bt->v32, v32.data(), nnz * sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      (num_systems > 0 &&
       cudaMemcpyAsync(bt->order, sorted.data(), num_systems * sizeof(int), cudaMemcpyHostToDevice, s) !=
           cudaSuccess) ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    set_error("cfd_batch_create: upload failed");
    return fail(CFD_ERR_CUDA);
  }
  *out = bt;
  return CFD_OK;
}

}  // namespace cfd

extern "C" {

cfd_status cfd_batch_create(cfd_context* ctx, int32_t num_systems, const int64_t* sys_row_offsets,
                            const int64_t* row_ptr, const int32_t* col, const double* val, cfd_batch** out) {
  return guarded("cfd_batch_create", [&]() -> cfd_status {
    if (!out) {
      set_error("cfd_batch_create: null output handle");
      return CFD_ERR_STATE;
    }
    *out = nullptr;
    CFD_TRY(batch_validate(num_systems, sys_row_offsets, row_ptr, col, val));
    if (!ctx) {
      set_error("cfd_batch_create: null context");
      return CFD_ERR_STATE;
    }
    return batch_build(ctx, num_systems, sys_row_offsets, row_ptr, col, val, out);
  });
}

cfd_status cfd_batch_update_values(cfd_batch* bt, const double* val) {
  return guarded("cfd_batch_update_values", [&]() -> cfd_status {
    if (!bt || !val) return CFD_ERR_STATE;
    std::lock_guard<std::mutex> g(bt->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(bt->ctx->device));
    std::vector<float> v32(val, val + bt->nnz);
    bool out_of_range = false;
    for (int64_t k = 0; k < bt->nnz; ++k)
      if (std::isfinite(val[k]) && !std::isfinite(v32[k])) out_of_range = true;
    CFD_TRY_CUDA(cudaMemcpyAsync(bt->v64, val, bt->nnz * sizeof(double), cudaMemcpyHostToDevice, bt->ctx->stream));
    CFD_TRY_CUDA(
        cudaMemcpyAsync(bt->v32, v32.data(), bt->nnz * sizeof(float), cudaMemcpyHostToDevice, bt->ctx->stream));
    CFD_TRY_CUDA(cudaStreamSynchronize(bt->ctx->stream));
    bt->values_valid = true;
    bt->f32_out_of_range = out_of_range;
    return CFD_OK;
  });
}

cfd_status cfd_batch_solve(cfd_batch* bt, const cfd_solve_options* opt, const double* b, double* x,
                           const cfd_solver_config* cfg, int32_t* term_out, int32_t* iters_out,
                           double* resid_out, cfd_batch_report* rep) {
  return guarded("cfd_batch_solve", [&]() -> cfd_status {
    if (!bt || !opt || !x || !cfg || !rep) {
      set_error("null argument to cfd_batch_solve");
      return CFD_ERR_STATE;
    }
    if (!b && !bt->rhs_resident) {
      set_error("cfd_batch_solve: b is NULL but no assembled right-hand side is resident (cfd_batch_assemble)");
      return CFD_ERR_STATE;
    }
    if (!bt->values_valid) {
      set_error("cfd_batch_solve: the batch holds no valid matrix (assemble it, or update its values, first)");
      return CFD_ERR_STATE;
    }
    if (!(cfg->tolerance >= 0.0) || !(cfg->relative_tolerance >= 0.0) || cfg->max_iterations <= 0 ||
        opt->solver != CFD_SOLVER_CG || opt->precond != CFD_PRECOND_JACOBI || opt->precision < 0 ||
        opt->precision > 1) {
      set_error("cfd_batch_solve: needs CG with Jacobi, valid tolerances and a positive iteration budget");
      return CFD_ERR_CONFIG;
    }
    if (bt->f32_out_of_range && opt->precision == CFD_PRECISION_FP32_REFINE) {
      set_error("cfd_batch_solve: an entry of the batch exceeds the FP32 range; solve in FP64");
      return CFD_ERR_NONFINITE;
    }
    std::lock_guard<std::mutex> g(bt->ctx->mu);
    cfd_context* ctx = bt->ctx;
    CFD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const int prec = opt->precision;
    std::memset(rep, 0, sizeof(*rep));
    rep->num_systems = bt->nsys;
    if (bt->nsys == 0) return CFD_OK;
    const cudaMemcpyKind in = opt->memory == CFD_MEMORY_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind outk = opt->memory == CFD_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    CFD_TRY(capture_graph(bt, prec));
    CFD_TRY_CUDA(cudaEventRecord(ctx->ev0, s));
    CFD_TRY(set_params(bt, *cfg, *opt));
    if (b) {
      bt->rhs_resident = false;  // the caller's b replaces an assembled one
      CFD_TRY_CUDA(cudaMemcpyAsync(bt->b, b, bt->rows * sizeof(double), in, s));
    }
    CFD_TRY_CUDA(cudaMemcpyAsync(bt->x, x, bt->rows * sizeof(double), in, s));
    CFD_TRY_CUDA(cudaGraphLaunch(bt->graph[prec], s));
    CFD_TRY_CUDA(cudaMemcpyAsync(x, bt->x, bt->rows * sizeof(double), outk, s));
    CFD_TRY_CUDA(cudaEventRecord(ctx->ev1, s));
    std::vector<int> term(bt->nsys), iters(bt->nsys);
    std::vector<double> resid(bt->nsys);
    CFD_TRY_CUDA(cudaMemcpyAsync(term.data(), bt->term, bt->nsys * sizeof(int), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(iters.data(), bt->iters, bt->nsys * sizeof(int), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(resid.data(), bt->resid, bt->nsys * sizeof(double), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    CFD_TRY_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    for (int k = 0; k < bt->nsys; ++k) {
      if (term[k] == CFD_TERM_CONVERGED || term[k] == CFD_TERM_INITIAL_RESIDUAL) rep->converged_systems++;
      rep->total_iterations += iters[k];
      rep->max_iterations = std::max(rep->max_iterations, iters[k]);
      rep->max_rel_residual = std::max(rep->max_rel_residual, resid[k]);
    }
    rep->device_ms = ms;
    if (term_out) std::copy(term.begin(), term.end(), term_out);
    if (iters_out) std::copy(iters.begin(), iters.end(), iters_out);
    if (resid_out) std::copy(resid.begin(), resid.end(), resid_out);
    return CFD_OK;
  });
}

cfd_status cfd_batch_autotune(cfd_batch* bt, int32_t precision, int32_t sample_iterations) {
  return guarded("cfd_batch_autotune", [&]() -> cfd_status {
    if (!bt || precision < 0 || precision > 1 || sample_iterations <= 0) return CFD_ERR_CONFIG;
    if (!bt->values_valid) {
      set_error("cfd_batch_autotune: the batch holds no valid matrix (assemble it, or update its values, first)");
      return CFD_ERR_STATE;
    }
    std::lock_guard<std::mutex> g(bt->ctx->mu);
    cfd_context* ctx = bt->ctx;
    CFD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    // Representative inputs: x = 0, b = 1; a fixed iteration budget and a zero
    // tolerance make every candidate do the same work. b = 1 replaces an
    // assembled right-hand side.
    bt->rhs_resident = false;
    std::vector<double> ones(bt->rows, 1.0);
    CFD_TRY_CUDA(cudaMemcpyAsync(bt->b, ones.data(), bt->rows * sizeof(double), cudaMemcpyHostToDevice, s));
    cfd_solver_config cfg{0.0, 0.0, sample_iterations};
    cfd_solve_options opt;
    cfd_solve_options_default(&opt);
    opt.max_outer = 1;
    opt.inner_tolerance = 0.0;
    CFD_TRY(set_params(bt, cfg, opt));
    bt->h_params->inner_tol = 0.0;
    CFD_TRY_CUDA(cudaMemcpyAsync(bt->params, bt->h_params, sizeof(BatchParams), cudaMemcpyHostToDevice, s));
    for (int k = 0; k < kBuckets; ++k) {
      if (bt->bucket_begin[k + 1] == bt->bucket_begin[k]) continue;
      float best = 1e30f;
      int best_t = bt->threads[precision][k], best_g = bt->groups[precision][k];
      for (int t : kCandidates)
        for (int gr : kGroupCandidates) {
          if (t > 2 * std::max(32, bt->bucket_nmax[k]) || (gr > 1 && t * gr > 512)) continue;
          float ms_min = 1e30f;
          for (int rep = 0; rep < 2; ++rep) {
            CFD_TRY_CUDA(cudaMemsetAsync(bt->x, 0, bt->rows * sizeof(double), s));
            CFD_TRY_CUDA(cudaMemsetAsync(bt->queues + k, 0, sizeof(unsigned), s));
            CFD_TRY_CUDA(cudaEventRecord(ctx->ev0, s));
            cfd_status st = precision ? run_bucket<true>(bt, k, t, gr, s) : run_bucket<false>(bt, k, t, gr, s);
            if (st == CFD_ERR_CONFIG) break;  // does not fit at this width
            CFD_TRY(st);
            CFD_TRY_CUDA(cudaEventRecord(ctx->ev1, s));
            CFD_TRY_CUDA(cudaStreamSynchronize(s));
            float ms = 0.f;
            CFD_TRY_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
            ms_min = std::min(ms_min, ms);
          }
          if (ms_min < best) {
            best = ms_min;
            best_t = t;
            best_g = gr;
          }
        }
      bt->threads[precision][k] = best_t;
      bt->groups[precision][k] = best_g;
    }
    bt->tuned[precision] = true;
    drop_graphs(bt);
    return CFD_OK;
  });
}

cfd_status cfd_batch_config(const cfd_batch* bt, int32_t precision, int32_t* bucket_rows, int32_t* threads,
                            int32_t* systems) {
  if (!bt || precision < 0 || precision > 1) return CFD_ERR_STATE;
  for (int k = 0; k < kBuckets; ++k) {
    if (bucket_rows) bucket_rows[k] = kBucketRows[k];
    if (threads) threads[k] = bt->threads[precision][k];
    if (systems) systems[k] = bt->bucket_begin[k + 1] - bt->bucket_begin[k];
  }
  return CFD_OK;
}

cfd_status cfd_batch_set_config(cfd_batch* bt, int32_t precision, const int32_t* threads, const int32_t* groups) {
  return guarded("cfd_batch_set_config", [&]() -> cfd_status {
    if (!bt || precision < 0 || precision > 1 || !threads || !groups) return CFD_ERR_CONFIG;
    for (int k = 0; k < kBuckets; ++k) {
      const bool tok = std::find(std::begin(kCandidates), std::end(kCandidates), threads[k]) != std::end(kCandidates);
      const bool gok = std::find(std::begin(kGroupCandidates), std::end(kGroupCandidates), groups[k]) !=
                       std::end(kGroupCandidates);
      if (!tok || !gok || threads[k] * groups[k] > 1024) {
        set_error("cfd_batch_set_config: bucket %d: %d threads per system x %d systems per CTA is not a candidate",
                  k, threads[k], groups[k]);
        return CFD_ERR_CONFIG;
      }
    }
    std::lock_guard<std::mutex> g(bt->ctx->mu);
    for (int k = 0; k < kBuckets; ++k) {
      bt->threads[precision][k] = threads[k];
      bt->groups[precision][k] = groups[k];
    }
    drop_graphs(bt);
    return CFD_OK;
  });
}

cfd_status cfd_batch_groups(const cfd_batch* bt, int32_t precision, int32_t* groups) {
  if (!bt || precision < 0 || precision > 1 || !groups) return CFD_ERR_STATE;
  for (int k = 0; k < kBuckets; ++k) groups[k] = bt->groups[precision][k];
  return CFD_OK;
}

cfd_status cfd_batch_destroy(cfd_batch* bt) {
  if (!bt) return CFD_OK;
  cudaSetDevice(bt->ctx->device);
  cudaStreamSynchronize(bt->ctx->stream);
  drop_graphs(bt);
  for (void* p : {(void*)bt->sys_row, (void*)bt->rp, (void*)bt->col, (void*)bt->v64, (void*)bt->v32, (void*)bt->x,
                  (void*)bt->b, (void*)bt->term, (void*)bt->iters, (void*)bt->resid, (void*)bt->order,
                  (void*)bt->queues, (void*)bt->params, (void*)bt->ls_method, (void*)bt->ls_path,
                  (void*)bt->ls_list, (void*)bt->ls_params, (void*)bt->ls_queue, (void*)bt->ls_scratch,
                  (void*)bt->ls_pivot})
    if (p) cudaFree(p);
  if (bt->h_params) cudaFreeHost(bt->h_params);
  network_plan_free(bt->net);
  delete bt;
  return CFD_OK;
}

}  // extern "C"
