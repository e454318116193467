// Whole-solve PCG for small systems in one thread-block cluster: the plain CG
// and Jacobi-PCG of krylov::cg[_preconditioned] (krylov.rs:318-360, with
// DiagJacobi) in FP64, for systems whose rows fit the shared memory of a
// cluster of up to 16 CTAs (the 2-D 128^2 pressure Poisson system of 16 384
// unknowns among them).
//
// A multi-kernel PCG iteration on such a system is bound by launch and
// grid-reduction latency (about 19 us per iteration at 128^2: three to four
// kernels on data that sits in L2). Here one launch runs the whole solve:
// every CTA of the cluster keeps its block of rows (CSR values, columns as
// (owning CTA, local index), row offsets) and its slices of x, r, p, q and
// D^-1 in shared memory; the SpMV reads p of other rows from their owners'
// shared memory (distributed shared memory); a dot product is a per-CTA partial
// written to shared memory, one cluster barrier, and every CTA summing all
// partials in rank order, so every CTA holds the same value and takes the same
// branch. Three cluster barriers per iteration: before the SpMV (p complete),
// after the p.q partials, after the r.r and r.z partials. The barriers are the
// hardware cluster barrier; control flow is uniform across the cluster, so no
// CTA can wait for one that has left.
//
// Recurrence and termination are pcg_loop's: r0 = b - A x0, threshold
// max(tol, rtol ||r0||), InitialResidual / Breakdown on the initial residual;
// per iteration q = A p, NonPositiveCurvature when p.q <= 0, alpha = rho / p.q,
// x += alpha p, r -= alpha q, Breakdown / Converged / MaxIterations on ||r||,
// rho' = r.z (z = D^-1 r, or r), Breakdown when rho' is 0 or not finite,
// beta = rho' / rho, p = z + beta p. The row sums run in CSR order as the
// one-thread-per-row pipelines do; the dot products sum per-CTA partials in a
// different tree than the grid reductions, so iterates agree with the
// multi-kernel solve to rounding.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.h"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace cfd {
namespace {

constexpr int kClThreads = 512;
constexpr int kClMaxCtas = 16;

struct ClusterArgs {
  const int* __restrict__ rp;  // global CSR (int32)
  const int* __restrict__ col;
  const double* __restrict__ val;
  const double* __restrict__ jinv;  // nullptr: no preconditioner
  const double* __restrict__ b;
  double* __restrict__ x;
  DevState* st;
  int n, rpc, nnz_cap;  // rows, rows per CTA, nonzeros per CTA at most
};

struct ClusterLayout {
  size_t val, ent, rpl, vec, bytes;
};

__host__ __device__ inline size_t cl_round16(size_t b) { return (b + 15) / 16 * 16; }

__host__ __device__ inline ClusterLayout cluster_layout(int rpc, int nnz_cap) {
  ClusterLayout L;
  L.val = 0;
  L.ent = cl_round16((size_t)nnz_cap * 8);
  L.rpl = L.ent + cl_round16((size_t)nnz_cap * 4);
  L.vec = L.rpl + cl_round16((size_t)(rpc + 1) * 4);
  L.bytes = L.vec + 5 * cl_round16((size_t)rpc * 8);
  return L;
}

// Sums of a and b over the CTA, written by thread 0 to out[0..1].
__device__ __forceinline__ void cl_block_sum2(double a, double b, double (&buf)[2][32], double* out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  if (lane == 0) {
    buf[0][w] = a;
    buf[1][w] = b;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = (int)(blockDim.x >> 5);
    double ta = lane < nw ? buf[0][lane] : 0.0, tb = lane < nw ? buf[1][lane] : 0.0;
    ta = warp_sum(ta);
    tb = warp_sum(tb);
    if (lane == 0) {
      out[0] = ta;
      out[1] = tb;
    }
  }
}

__global__ void __launch_bounds__(kClThreads) k_cluster_pcg(ClusterArgs A) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int ncta = (int)cluster.num_blocks();
  extern __shared__ __align__(16) unsigned char sm[];
  const ClusterLayout L = cluster_layout(A.rpc, A.nnz_cap);
  double* sval = reinterpret_cast<double*>(sm + L.val);
  int* sent = reinterpret_cast<int*>(sm + L.ent);  // owner << 16 | local index
  int* srp = reinterpret_cast<int*>(sm + L.rpl);
  const size_t vs = cl_round16((size_t)A.rpc * 8);
  double* sx = reinterpret_cast<double*>(sm + L.vec);
  double* sr = reinterpret_cast<double*>(sm + L.vec + vs);
  double* sp = reinterpret_cast<double*>(sm + L.vec + 2 * vs);
  double* sq = reinterpret_cast<double*>(sm + L.vec + 3 * vs);
  double* sj = reinterpret_cast<double*>(sm + L.vec + 4 * vs);
  __shared__ double part[2][2];  // [slot][value]: this CTA's partial sums
  __shared__ double redbuf[2][32];
  __shared__ double tot[2];
  __shared__ double* px[kClMaxCtas];  // every CTA's x and p in the cluster's shared window
  __shared__ double* pp[kClMaxCtas];

  const int r0 = rank * A.rpc;
  const int nrow = max(0, min(A.rpc, A.n - r0));
  const int k0 = nrow > 0 ? A.rp[r0] : 0;
  const int nnz = nrow > 0 ? A.rp[r0 + nrow] - k0 : 0;
  for (int i = threadIdx.x; i <= nrow; i += blockDim.x) srp[i] = A.rp[r0 + i] - k0;
  for (int e = threadIdx.x; e < nnz; e += blockDim.x) {
    const int c = A.col[k0 + e];
    const int owner = c / A.rpc;
    sent[e] = (owner << 16) | (c - owner * A.rpc);
    sval[e] = A.val[k0 + e];
  }
  for (int i = threadIdx.x; i < nrow; i += blockDim.x) {
    sx[i] = A.x[r0 + i];
    sj[i] = A.jinv ? A.jinv[r0 + i] : 1.0;
  }
  if (threadIdx.x < ncta) {
    px[threadIdx.x] = cluster.map_shared_rank(sx, threadIdx.x);
    pp[threadIdx.x] = cluster.map_shared_rank(sp, threadIdx.x);
  }
  cluster.sync();  // every CTA's x staged

  auto row_sum = [&](int i, double* const* vec) {
    double s = 0.0;
    for (int k = srp[i]; k < srp[i + 1]; ++k) {
      const int e = sent[k];
      s += sval[k] * vec[e >> 16][e & 0xffff];
    }
    return s;
  };
  // CTA partials -> cluster totals: lane k of warp 0 fetches CTA k's partials
  // and the warp sums them by a fixed butterfly, so every CTA gets the same bits
  auto cluster_totals = [&](int slot, double a, double b2, double* ta, double* tb) {
    cl_block_sum2(a, b2, redbuf, &part[slot][0]);
    cluster.sync();
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      double ua = 0.0, ub = 0.0;
      if (lane < ncta) {
        const double* pk = cluster.map_shared_rank(&part[slot][0], lane);
        ua = pk[0];
        ub = pk[1];
      }
      ua = warp_sum(ua);
      ub = warp_sum(ub);
      if (lane == 0) {
        tot[0] = ua;
        tot[1] = ub;
      }
    }
    __syncthreads();
    *ta = tot[0];
    *tb = tot[1];
    __syncthreads();  // tot is rewritten by the next reduction
  };

  // r0 = b - A x0, z0 = D^-1 r0, p0 = z0, rho = r0.z0
  double arr = 0.0, arz = 0.0;
  for (int i = threadIdx.x; i < nrow; i += blockDim.x) {
    const double ri = A.b[r0 + i] - row_sum(i, px);
    sr[i] = ri;
    const double zi = ri * sj[i];
    sp[i] = zi;
    arr += ri * ri;
    arz += ri * zi;
  }
  double rr, rho;
  cluster_totals(0, arr, arz, &rr, &rho);
  const double rnorm0 = sqrt(rr);
  const double thr = fmax(A.st->tol_abs, A.st->tol_rel * rnorm0);
  const int max_iter = A.st->max_iter;
  int iter = 0, term = CFD_TERM_MAX_ITERATIONS;
  double rn = rnorm0;
  if (!isfinite(rnorm0)) {
    term = CFD_TERM_BREAKDOWN;
  } else if (rnorm0 <= thr) {
    term = CFD_TERM_INITIAL_RESIDUAL;
  } else {
    for (;;) {
      cluster.sync();  // p complete in every CTA
      double apq = 0.0;
      for (int i = threadIdx.x; i < nrow; i += blockDim.x) {
        const double qi = row_sum(i, pp);
        sq[i] = qi;
        apq += sp[i] * qi;
      }
      double pq, unused;
      cluster_totals(1, apq, 0.0, &pq, &unused);
      if (!(pq > 0.0)) {
        term = CFD_TERM_NON_POSITIVE_CURVATURE;
        break;
      }
      const double alpha = rho / pq;
      arr = 0.0;
      arz = 0.0;
      for (int i = threadIdx.x; i < nrow; i += blockDim.x) {
        sx[i] = sx[i] + alpha * sp[i];
        const double ri = sr[i] - alpha * sq[i];
        sr[i] = ri;
        arr += ri * ri;
        arz += ri * (ri * sj[i]);
      }
      double rz;
      cluster_totals(0, arr, arz, &rr, &rz);
      ++iter;
      rn = sqrt(rr);
      if (!isfinite(rn)) {
        term = CFD_TERM_BREAKDOWN;
        break;
      }
      if (rn <= thr) {
        term = CFD_TERM_CONVERGED;
        break;
      }
      if (iter >= max_iter) {
        term = CFD_TERM_MAX_ITERATIONS;
        break;
      }
      if (rz == 0.0 || !isfinite(rz)) {
        term = CFD_TERM_BREAKDOWN;
        break;
      }
      const double beta = rz / rho;
      rho = rz;
      for (int i = threadIdx.x; i < nrow; i += blockDim.x) sp[i] = sr[i] * sj[i] + beta * sp[i];
    }
  }
  for (int i = threadIdx.x; i < nrow; i += blockDim.x) A.x[r0 + i] = sx[i];
  if (rank == 0 && threadIdx.x == 0) {
    DevState* st = A.st;
    st->rnorm0 = rnorm0;
    st->threshold = thr;
    st->rnorm = rn;
    st->rr = rn * rn;
    st->iter = iter;
    st->term = term;
    st->done = 1;
  }
  cluster.sync();  // no CTA leaves while its shared memory may still be read
}

}  // namespace

// The cluster solve applies when the system's rows, split over at most 16
// CTAs, fit their shared memory; *ok = false otherwise (nothing launched).
cfd_status cluster_pcg_solve(cfd_context* ctx, const DevMat& m, const double* jinv, const double* b, double* x,
                             DevState* st, bool* ok) {
  *ok = false;
  const int64_t n = m.nrows;
  if (n <= 0 || n >= (int64_t)kClMaxCtas * 65536 || m.nrows != m.ncols) return CFD_OK;
  int max_smem = 0;
  CFD_TRY_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
  const size_t budget = (size_t)max_smem - 2048;  // static shared arrays
  // about 1024 rows per CTA (two per thread) where the cluster allows it,
  // more CTAs where a block does not fit the shared memory
  int first = 2;
  while (first < kClMaxCtas && (n + first - 1) / first > 2 * kClThreads) first *= 2;
  std::vector<int> rp32;
  for (int ncta = first; ncta <= kClMaxCtas; ncta *= 2) {
    const int rpc = (int)((n + ncta - 1) / ncta);
    if (rpc >= 65536) continue;
    if (rp32.empty()) {
      rp32.resize(n + 1);
      CFD_TRY_CUDA(cudaMemcpyAsync(rp32.data(), m.rp, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      CFD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    int nnz_cap = 0;
    for (int c = 0; c < ncta; ++c) {
      const int64_t a = std::min<int64_t>((int64_t)c * rpc, n), e = std::min<int64_t>((int64_t)(c + 1) * rpc, n);
      nnz_cap = std::max(nnz_cap, rp32[e] - rp32[a]);
    }
    const ClusterLayout L = cluster_layout(rpc, nnz_cap);
    if (L.bytes > budget) continue;
    CFD_TRY_CUDA(cudaFuncSetAttribute(k_cluster_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes));
    if (ncta > 8)
      CFD_TRY_CUDA(cudaFuncSetAttribute(k_cluster_pcg, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfgl = {};
    cfgl.gridDim = dim3(ncta);
    cfgl.blockDim = dim3(kClThreads);
    cfgl.dynamicSmemBytes = L.bytes;
    cfgl.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ncta;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfgl.attrs = attr;
    cfgl.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_cluster_pcg, &cfgl) != cudaSuccess || clusters < 1) {
      cudaGetLastError();
      continue;
    }
    ClusterArgs args{m.rp, m.col, m.v64, jinv, b, x, st, (int)n, rpc, nnz_cap};
    CFD_TRY_CUDA(cudaLaunchKernelEx(&cfgl, k_cluster_pcg, args));
    ctx->stats.launches++;
    *ok = true;
    return CFD_OK;
  }
  return CFD_OK;
}

}  // namespace cfd
