// The 1-D network solve of CFDrs, LinearSystemSolver::solve_with_initial_guess
// (crates/cfd-1d/src/solver/core/linear_system.rs:114-155), for every system
// of a batch (cfd_batch_linear_system_solve):
//
//   method   NetworkSolver::detect_solver_method (solver_detection.rs:36-64),
//            or the one the caller fixes (LinearSystemSolver::with_method);
//   scaling  rows equilibrated by 1 / max_j |a_ij| (:157-186);
//   n <= 256 dense LU of the equilibrated system, kept when its residual
//            target holds on the original system (:188-204), else dense LU of
//            the original system (:124-130);
//   n > 256  CG or BiCGSTAB on the equilibrated system with DiagJacobi of it
//            (:131-143), IterativeSolverConfig::new(tolerance): an absolute
//            threshold on the 2-norm of that system's residual; kept when it
//            converged and the residual target holds, else dense LU of the
//            original system (:144-155).
//
// Krylov: one CTA per system from a longest-first queue, the whole system in
// shared memory (k_ls_krylov), as the batched Jacobi-PCG of batch.cu.
// Dense LU: one CTA per system on an n x n FP64 slot in global memory, blocked
// right-looking with partial pivoting (k_ls_dense): 32-column panels factored
// in place, the trailing matrix updated by 64 x 64 tiles staged in shared
// memory. The systems whose Krylov solve is not kept are collected on the
// host after the Krylov launches and solved by a second dense launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "batch_internal.h"
#include "internal.h"
#include "kernels.cuh"

namespace cfd {
namespace {

constexpr int kLsThreads = 256;  // dense LU CTA
constexpr int kLuNb = 32;        // panel width
constexpr int kLuTile = 64;      // trailing-update tile edge

struct LsArgs {
  const int* __restrict__ sys_row;
  const int* __restrict__ rp;
  const int* __restrict__ col;
  const double* __restrict__ v64;
  const float* __restrict__ v32;
  const double* __restrict__ b;
  double* __restrict__ x;
  int* method;  // per system: CFD_LS_CG / CFD_LS_BICGSTAB
  int* path;    // per system: CFD_LS_PATH_*
  int* term;    // per system: Krylov termination, -1 when none ran
  int* iters;
  double* resid;  // ||D (A x - b)|| / ||D b|| of the returned x
};

struct LsParams {
  double tol, inner_tol;
  int32_t max_iter, max_outer, method;
};

__host__ __device__ constexpr size_t ls_round16(size_t b) { return (b + 15) / 16 * 16; }
template <typename T>
__host__ __device__ constexpr size_t ls_col_off(int zmax) {
  return ls_round16((size_t)zmax * sizeof(T));
}
template <typename T>
__host__ __device__ constexpr size_t ls_rp_off(int zmax) {
  return ls_col_off<T>(zmax) + ls_round16((size_t)zmax * 2);
}
template <typename T>
__host__ __device__ constexpr size_t ls_vec_off(int zmax, int nmax) {
  return ls_rp_off<T>(zmax) + ls_round16((size_t)(nmax + 1) * 4);
}
constexpr int kLsVectors = 8;  // x, r, r^, p, v, w (p^ / s^), t, D^-1
template <typename T>
__host__ __device__ constexpr size_t ls_smem(int nmax, int zmax) {
  return ls_vec_off<T>(zmax, nmax) + kLsVectors * ls_round16((size_t)nmax * sizeof(T));
}

// Sums of one or two values over the CTA, result in every thread; `slot`
// alternates so one barrier separates consecutive reductions.
__device__ __forceinline__ void ls_cta_sum2(double& a, double& b, double (*buf)[2][32], int& slot) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  if (nw > 1) {
    if (lane == 0) {
      buf[slot][0][w] = a;
      buf[slot][1][w] = b;
    }
    __syncthreads();
    a = warp_sum(lane < nw ? buf[slot][0][lane] : 0.0);
    b = warp_sum(lane < nw ? buf[slot][1][lane] : 0.0);
    slot ^= 1;
  }
  a = __shfl_sync(0xffffffffu, a, 0);
  b = __shfl_sync(0xffffffffu, b, 0);
}

// 1 / max_j |a_ij| of a row of the original values (identity where the
// maximum is not above f64::EPSILON or not finite).
__device__ __forceinline__ double ls_scale(const double* __restrict__ v, int k0, int k1) {
  double mx = 0.0;
  for (int k = k0; k < k1; ++k) mx = fmax(mx, fabs(v[k]));
  return (mx > DBL_EPSILON && isfinite(mx)) ? 1.0 / mx : 1.0;
}

// ||D (A x - b)|| / ||D b|| (or ||D (A x - b)|| when ||D b|| <= f64::EPSILON)
// of system rows [r0, r0 + n) for x in global memory (linear_system.rs:188-246).
__device__ double ls_target_ratio(const LsArgs& A, int r0, int n, double (*buf)[2][32], int& slot) {
  double r2 = 0.0, b2 = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int g = r0 + i, k0 = A.rp[g], k1 = A.rp[g + 1];
    double ax = 0.0;
    for (int k = k0; k < k1; ++k) ax += A.v64[k] * A.x[r0 + A.col[k]];
    const double s = ls_scale(A.v64, k0, k1);
    const double r = (ax - A.b[g]) * s, bb = A.b[g] * s;
    r2 += r * r;
    b2 += bb * bb;
  }
  ls_cta_sum2(r2, b2, buf, slot);
  const double rn = sqrt(r2), bn = sqrt(b2);
  if (!isfinite(rn)) return rn;
  return bn > DBL_EPSILON ? rn / bn : rn;
}

template <typename T, bool REFINE>
__global__ void __launch_bounds__(512) k_ls_krylov(LsArgs A, const int* __restrict__ order, int count,
                                                   unsigned* queue, const LsParams* __restrict__ prm, int nmax,
                                                   int zmax) {
  extern __shared__ __align__(16) unsigned char sm[];
  T* sv = reinterpret_cast<T*>(sm);
  unsigned short* sc = reinterpret_cast<unsigned short*>(sm + ls_col_off<T>(zmax));
  int* srp = reinterpret_cast<int*>(sm + ls_rp_off<T>(zmax));
  const size_t vs = ls_round16((size_t)nmax * sizeof(T));
  unsigned char* vb = sm + ls_vec_off<T>(zmax, nmax);
  T* vx = reinterpret_cast<T*>(vb);
  T* vr = reinterpret_cast<T*>(vb + vs);
  T* vrh = reinterpret_cast<T*>(vb + 2 * vs);
  T* vp = reinterpret_cast<T*>(vb + 3 * vs);
  T* vv = reinterpret_cast<T*>(vb + 4 * vs);
  T* vw = reinterpret_cast<T*>(vb + 5 * vs);
  T* vt = reinterpret_cast<T*>(vb + 6 * vs);
  T* vinv = reinterpret_cast<T*>(vb + 7 * vs);
  __shared__ double red[2][2][32];
  __shared__ int s_k;
  const int tid = threadIdx.x, nt = blockDim.x;
  const LsParams P = *prm;
  int slot = 0;
  auto sum1 = [&](double a) {
    double z = 0.0;
    ls_cta_sum2(a, z, red, slot);
    return a;
  };

  for (;;) {
    if (tid == 0) s_k = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int q = s_k;
    __syncthreads();
    if (q >= count) break;
    const int sys = order[q];
    const int r0 = A.sys_row[sys], n = A.sys_row[sys + 1] - r0;
    const int k0 = A.rp[r0], nnz = A.rp[r0 + n] - k0;
    for (int i = tid; i <= n; i += nt) srp[i] = A.rp[r0 + i] - k0;
    for (int e = tid; e < nnz; e += nt) sc[e] = (unsigned short)A.col[k0 + e];
    __syncthreads();
    // Equilibrated values, DiagJacobi of the equilibrated matrix and the
    // dominance test of detect_solver_method on the original values.
    bool not_spd = false, bad_diag = false;
    for (int i = tid; i < n; i += nt) {
      const int e0 = srp[i], e1 = srp[i + 1];
      const double s = ls_scale(A.v64, k0 + e0, k0 + e1);
      double diag = 0.0, sum_off = 0.0, dd = 0.0;
      bool row_bad = false;
      for (int e = e0; e < e1; ++e) {
        const double a = A.v64[k0 + e];
        const double as = a * s;
        sv[e] = (T)as;
        if (sc[e] == i) {
          diag = a;
          dd = as;
        } else if (a > 0.0) {
          row_bad = true;
        } else {
          sum_off += fabs(a);
        }
      }
      const bool identity = diag == 1.0 && sum_off == 0.0;
      if (row_bad || ((diag < sum_off || diag <= 0.0) && !identity)) not_spd = true;
      if (!isfinite(dd)) bad_diag = true;
      vinv[i] = (T)(fabs(dd) <= DBL_EPSILON ? 1.0 : 1.0 / dd);
      if (!REFINE) vt[i] = (T)s;  // the row scale, until the solve needs t
    }
    not_spd = __syncthreads_or(not_spd);
    bad_diag = __syncthreads_or(bad_diag);
    const int method = P.method == CFD_LS_DETECT ? (not_spd ? CFD_LS_BICGSTAB : CFD_LS_CG) : P.method;
    if (bad_diag) {
      if (tid == 0) {
        A.method[sys] = method;
        A.path[sys] = CFD_LS_PATH_ERROR;
        A.term[sys] = -1;
        A.iters[sys] = 0;
        A.resid[sys] = NAN;
      }
      __syncthreads();
      continue;
    }

    // y = (D A) u in shared memory for the rows of this thread.
    auto spmv_row = [&](int i, const T* u) {
      T s = T(0);
      for (int e = srp[i]; e < srp[i + 1]; ++e) s += sv[e] * u[sc[e]];
      return s;
    };

    // Krylov on (D A) x = rhs from x = vx, rhs - (D A) x in vr; threshold
    // max(thr_abs, thr_rel * ||r0||). Returns the iterations, sets term.
    auto krylov = [&](double thr_abs, double thr_rel, int max_it, int& term_out) -> int {
      double e2 = 0.0, rho = 0.0;
      for (int i = tid; i < n; i += nt) {
        const T ri = vr[i];
        e2 += (double)ri * (double)ri;
        if (method == CFD_LS_CG) {
          const T zi = ri * vinv[i];
          vp[i] = zi;
          rho += (double)ri * (double)zi;
        } else {
          vrh[i] = ri;
        }
      }
      ls_cta_sum2(e2, rho, red, slot);
      const double e0 = sqrt(e2);
      const double thr = fmax(thr_abs, thr_rel * e0);
      if (!isfinite(e0)) {
        term_out = CFD_TERM_BREAKDOWN;
        return 0;
      }
      if (e0 <= thr) {
        term_out = CFD_TERM_INITIAL_RESIDUAL;
        return 0;
      }
      __syncthreads();
      if (method == CFD_LS_CG) {
        for (int it = 1; it <= max_it; ++it) {
          double pq = 0.0;
          for (int i = tid; i < n; i += nt) {
            const T qi = spmv_row(i, vp);
            vv[i] = qi;
            pq += (double)vp[i] * (double)qi;
          }
          pq = sum1(pq);
          if (!(pq > 0.0)) {
            term_out = CFD_TERM_NON_POSITIVE_CURVATURE;
            return it - 1;
          }
          const T alpha = (T)(rho / pq);
          double ee = 0.0, rz = 0.0;
          for (int i = tid; i < n; i += nt) {
            vx[i] = vx[i] + alpha * vp[i];
            const T ri = vr[i] - alpha * vv[i];
            vr[i] = ri;
            ee += (double)ri * (double)ri;
            rz += (double)ri * (double)(ri * vinv[i]);
          }
          ls_cta_sum2(ee, rz, red, slot);
          const double e = sqrt(ee);
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
          for (int i = tid; i < n; i += nt) vp[i] = vr[i] * vinv[i] + beta * vp[i];
          __syncthreads();
        }
        term_out = CFD_TERM_MAX_ITERATIONS;
        return max_it;
      }
      // BiCGSTAB, right preconditioned (Saad 2003, Alg. 7.7), x updated by
      // alpha p^ and omega s^ in turn so that p^ and s^ share w.
      double rho_old = 1.0, alpha = 1.0, omega = 1.0;
      for (int it = 1; it <= max_it; ++it) {
        double rho_new = 0.0;
        for (int i = tid; i < n; i += nt) rho_new += (double)vrh[i] * (double)vr[i];
        rho_new = sum1(rho_new);
        if (rho_new == 0.0 || !isfinite(rho_new)) {
          term_out = CFD_TERM_BREAKDOWN;
          return it - 1;
        }
        const T beta = (T)((rho_new / rho_old) * (alpha / omega));
        for (int i = tid; i < n; i += nt) {
          const T pi = it == 1 ? vr[i] : vr[i] + beta * (vp[i] - (T)omega * vv[i]);
          vp[i] = pi;
          vw[i] = pi * vinv[i];
        }
        __syncthreads();
        double rv = 0.0;
        for (int i = tid; i < n; i += nt) {
          const T vi = spmv_row(i, vw);
          vv[i] = vi;
          rv += (double)vrh[i] * (double)vi;
        }
        rv = sum1(rv);
        if (rv == 0.0 || !isfinite(rv)) {
          term_out = CFD_TERM_BREAKDOWN;
          return it - 1;
        }
        alpha = rho_new / rv;
        const T a = (T)alpha;
        double sn = 0.0;
        for (int i = tid; i < n; i += nt) {
          const T si = vr[i] - a * vv[i];
          vr[i] = si;  // s
          vx[i] = vx[i] + a * vw[i];
          sn += (double)si * (double)si;
        }
        sn = sum1(sn);
        if (sqrt(sn) <= thr) {
          term_out = CFD_TERM_CONVERGED;
          return it;
        }
        for (int i = tid; i < n; i += nt) vw[i] = vr[i] * vinv[i];  // s^
        __syncthreads();
        double tt = 0.0, ts = 0.0;
        for (int i = tid; i < n; i += nt) {
          const T ti = spmv_row(i, vw);
          vt[i] = ti;
          tt += (double)ti * (double)ti;
          ts += (double)ti * (double)vr[i];
        }
        ls_cta_sum2(tt, ts, red, slot);
        if (tt == 0.0 || !isfinite(tt)) {
          term_out = CFD_TERM_BREAKDOWN;
          return it;
        }
        omega = ts / tt;
        const T w = (T)omega;
        double rn = 0.0;
        for (int i = tid; i < n; i += nt) {
          vx[i] = vx[i] + w * vw[i];
          const T ri = vr[i] - w * vt[i];
          vr[i] = ri;
          rn += (double)ri * (double)ri;
        }
        rn = sqrt(sum1(rn));
        if (!isfinite(rn)) {
          term_out = CFD_TERM_BREAKDOWN;
          return it;
        }
        if (rn <= thr) {
          term_out = CFD_TERM_CONVERGED;
          return it;
        }
        if (omega == 0.0) {
          term_out = CFD_TERM_BREAKDOWN;
          return it;
        }
        rho_old = rho_new;
      }
      term_out = CFD_TERM_MAX_ITERATIONS;
      return max_it;
    };

    int term = CFD_TERM_MAX_ITERATIONS, it_total = 0;
    if (!REFINE) {
      for (int i = tid; i < n; i += nt) vx[i] = (T)A.x[r0 + i];
      __syncthreads();
      for (int i = tid; i < n; i += nt) vr[i] = (T)(A.b[r0 + i] * (double)vt[i]) - spmv_row(i, vx);
      __syncthreads();
      it_total = krylov(P.tol, 0.0, P.max_iter, term);
      __syncthreads();
      for (int i = tid; i < n; i += nt) A.x[r0 + i] = (double)vx[i];
    } else {
      // Outer FP64 residual of the equilibrated system from global memory
      // (the products a_ij * s rounded as the equilibrated matrix holds
      // them), FP32 inner solves of the normalised residual.
      term = CFD_TERM_MAX_ITERATIONS;
      for (int outer = 0; outer <= P.max_outer; ++outer) {
        double e2 = 0.0, z = 0.0;
        for (int i = tid; i < n; i += nt) {
          const int g = r0 + i, e0 = A.rp[g], e1 = A.rp[g + 1];
          const double s = ls_scale(A.v64, e0, e1);
          double ax = 0.0;
          for (int e = e0; e < e1; ++e) ax += (A.v64[e] * s) * A.x[r0 + A.col[e]];
          const double ri = A.b[g] * s - ax;
          e2 += ri * ri;
        }
        ls_cta_sum2(e2, z, red, slot);
        const double e = sqrt(e2);
        if (!isfinite(e)) {
          term = CFD_TERM_BREAKDOWN;
          break;
        }
        if (e <= P.tol) {
          term = outer == 0 ? CFD_TERM_INITIAL_RESIDUAL : CFD_TERM_CONVERGED;
          break;
        }
        if (outer == P.max_outer || it_total >= P.max_iter) break;
        // the inner right-hand side: the same residual, normalised (FP32)
        const double sc_ = 1.0 / e;
        for (int i = tid; i < n; i += nt) {
          const int g = r0 + i, e0 = A.rp[g], e1 = A.rp[g + 1];
          const double s = ls_scale(A.v64, e0, e1);
          double ax = 0.0;
          for (int ee = e0; ee < e1; ++ee) ax += (A.v64[ee] * s) * A.x[r0 + A.col[ee]];
          vr[i] = (T)((A.b[g] * s - ax) * sc_);
          vx[i] = T(0);
        }
        __syncthreads();
        int iterm = CFD_TERM_MAX_ITERATIONS;
        it_total += krylov(0.0, P.inner_tol, P.max_iter - it_total, iterm);
        __syncthreads();
        for (int i = tid; i < n; i += nt) A.x[r0 + i] += (double)vx[i] * e;
        __syncthreads();
        if (iterm == CFD_TERM_BREAKDOWN || iterm == CFD_TERM_NON_POSITIVE_CURVATURE) {
          term = iterm;
          break;
        }
      }
    }
    __syncthreads();
    const bool converged = term == CFD_TERM_CONVERGED || term == CFD_TERM_INITIAL_RESIDUAL;
    double ratio = NAN;
    bool meets = false;
    if (converged) {
      ratio = ls_target_ratio(A, r0, n, red, slot);
      meets = ratio <= P.tol;
    }
    if (tid == 0) {
      A.method[sys] = method;
      A.path[sys] = meets ? CFD_LS_PATH_KRYLOV : CFD_LS_PATH_KRYLOV_FALLBACK;
      A.term[sys] = term;
      A.iters[sys] = it_total;
      A.resid[sys] = ratio;
    }
    __syncthreads();
  }
}

// In-place dense LU with partial pivoting of the n x n row-major matrix M
// (first largest |m_ik| at or below the diagonal), the swaps applied to b,
// then L y = P b and U x = y; the solution replaces b. Returns false on a
// zero or non-finite pivot (every thread gets the same answer).
__device__ bool lu_solve(double* __restrict__ M, double* __restrict__ b, int n, double* s_val, int* s_idx,
                         double (*Ls)[kLuNb + 1], double (*Us)[kLuTile + 1]) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  for (int k0 = 0; k0 < n; k0 += kLuNb) {
    const int kb = min(kLuNb, n - k0);
    // panel: columns [k0, k0 + kb), unblocked
    for (int k = k0; k < k0 + kb; ++k) {
      double best = -1.0;
      int bi = n;
      for (int i = k + tid; i < n; i += nt) {
        const double v = fabs(M[(size_t)i * n + k]);
        if (v > best || (v == best && i < bi) || v != v) {
          best = v != v ? INFINITY : v;  // a NaN pivot candidate fails the factorization below
          bi = i;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) {
          best = ov;
          bi = oi;
        }
      }
      if (lane == 0) {
        s_val[w] = best;
        s_idx[w] = bi;
      }
      __syncthreads();
      if (tid == 0) {
        double bv = s_val[0];
        int bj = s_idx[0];
        for (int q = 1; q < nw; ++q)
          if (s_val[q] > bv || (s_val[q] == bv && s_idx[q] < bj)) {
            bv = s_val[q];
            bj = s_idx[q];
          }
        s_val[32] = bv;
        s_idx[32] = bj;
      }
      __syncthreads();
      const double pv = s_val[32];
      const int p = s_idx[32];
      if (!(pv > 0.0) || !isfinite(pv) || p >= n) return false;
      if (p != k) {
        for (int j = tid; j < n; j += nt) {
          const double t = M[(size_t)k * n + j];
          M[(size_t)k * n + j] = M[(size_t)p * n + j];
          M[(size_t)p * n + j] = t;
        }
        if (tid == 0) {
          const double t = b[k];
          b[k] = b[p];
          b[p] = t;
        }
      }
      __syncthreads();
      const double piv = M[(size_t)k * n + k];
      for (int i = k + 1 + tid; i < n; i += nt) {
        double* row = M + (size_t)i * n;
        const double l = row[k] / piv;
        row[k] = l;
        for (int j = k + 1; j < k0 + kb; ++j) row[j] -= l * M[(size_t)k * n + j];
      }
      __syncthreads();
    }
    const int m0 = k0 + kb;
    if (m0 >= n) break;
    // U12 = L11^-1 A12, one column per thread
    for (int j = m0 + tid; j < n; j += nt)
      for (int k = k0; k < m0; ++k) {
        const double u = M[(size_t)k * n + j];
        for (int i = k + 1; i < m0; ++i) M[(size_t)i * n + j] -= M[(size_t)i * n + k] * u;
      }
    __syncthreads();
    // A22 -= L21 U12 by 64 x 64 tiles
    const int m = n - m0, tiles = (m + kLuTile - 1) / kLuTile;
    const int tx = tid & 15, ty = tid >> 4;  // 16 x 16 threads, 4 x 4 entries each
    for (int t = 0; t < tiles * tiles; ++t) {
      const int ti = t / tiles, tj = t % tiles;
      const int rb = m0 + ti * kLuTile, cb = m0 + tj * kLuTile;
      for (int q = tid; q < kLuTile * kLuNb; q += nt) {
        const int r = q / kLuNb, c = q % kLuNb;
        Ls[r][c] = (rb + r < n && c < kb) ? M[(size_t)(rb + r) * n + k0 + c] : 0.0;
      }
      for (int q = tid; q < kLuNb * kLuTile; q += nt) {
        const int r = q / kLuTile, c = q % kLuTile;
        Us[r][c] = (r < kb && cb + c < n) ? M[(size_t)(k0 + r) * n + cb + c] : 0.0;
      }
      __syncthreads();
      if (nt >= 256 && tid < 256) {
        double acc[4][4] = {};
        for (int c = 0; c < kb; ++c) {
          double lv[4], uv[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) lv[a] = Ls[ty + 16 * a][c];
#pragma unroll
          for (int q = 0; q < 4; ++q) uv[q] = Us[c][tx + 16 * q];
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][q] += lv[a] * uv[q];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const int r = rb + ty + 16 * a;
          if (r >= n) continue;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int c = cb + tx + 16 * q;
            if (c < n) M[(size_t)r * n + c] -= acc[a][q];
          }
        }
      }
      __syncthreads();
    }
  }
  // L y = P b (unit lower), column by column
  for (int k = 0; k < n - 1; ++k) {
    const double bk = b[k];
    for (int i = k + 1 + tid; i < n; i += nt) b[i] -= M[(size_t)i * n + k] * bk;
    __syncthreads();
  }
  // U x = y, column by column from the last
  for (int k = n - 1; k >= 0; --k) {
    const double xk = b[k] / M[(size_t)k * n + k];
    for (int i = tid; i < k; i += nt) b[i] -= M[(size_t)i * n + k] * xk;
    __syncthreads();
    if (tid == 0) b[k] = xk;
    __syncthreads();
  }
  return true;
}

// Dense solves of the listed systems: DIRECT mode (n <= 256) tries the
// equilibrated system first and keeps it when the residual target holds, else
// solves the original one; FALLBACK mode solves the original system. Each CTA
// owns one scratch slot of slot_elems doubles (matrix, then right-hand side).
__global__ void __launch_bounds__(kLsThreads) k_ls_dense(LsArgs A, const int* __restrict__ list, int count,
                                                        int direct, unsigned* queue, double* scratch,
                                                        size_t slot_elems, const LsParams* __restrict__ prm) {
  __shared__ double Ls[kLuTile][kLuNb + 1];
  __shared__ double Us[kLuNb][kLuTile + 1];
  __shared__ double s_val[33];
  __shared__ int s_idx[33];
  __shared__ double red[2][2][32];
  __shared__ int s_k;
  const int tid = threadIdx.x, nt = blockDim.x;
  double* M = scratch + (size_t)blockIdx.x * slot_elems;
  int slot = 0;
  const double tol = prm->tol;
  for (;;) {
    if (tid == 0) s_k = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int q = s_k;
    __syncthreads();
    if (q >= count) break;
    const int sys = list[q];
    const int r0 = A.sys_row[sys], n = A.sys_row[sys + 1] - r0;
    double* bv = M + (size_t)n * n;
    int path = direct ? CFD_LS_PATH_DIRECT : A.path[sys];
    double ratio = NAN;
    for (int attempt = direct ? 0 : 1; attempt < 2; ++attempt) {
      const bool scaled = attempt == 0;
      for (size_t e = tid; e < (size_t)n * n; e += nt) M[e] = 0.0;
      __syncthreads();
      for (int i = tid; i < n; i += nt) {
        const int g = r0 + i, e0 = A.rp[g], e1 = A.rp[g + 1];
        const double s = scaled ? ls_scale(A.v64, e0, e1) : 1.0;
        for (int e = e0; e < e1; ++e) M[(size_t)i * n + A.col[e]] += A.v64[e] * s;
        bv[i] = A.b[g] * s;
      }
      __syncthreads();
      const bool ok = lu_solve(M, bv, n, s_val, s_idx, Ls, Us);
      if (ok) {
        for (int i = tid; i < n; i += nt) A.x[r0 + i] = bv[i];
        __syncthreads();
        ratio = ls_target_ratio(A, r0, n, red, slot);
        if (!scaled || ratio <= tol) break;
        path = CFD_LS_PATH_DIRECT_UNSCALED;
      } else if (scaled) {
        path = CFD_LS_PATH_DIRECT_UNSCALED;
      } else {
        path = CFD_LS_PATH_FAILED;
        ratio = NAN;
      }
      __syncthreads();
    }
    if (tid == 0) {
      A.path[sys] = path;
      A.resid[sys] = ratio;
      if (direct) {
        A.term[sys] = -1;
        A.iters[sys] = 0;
      }
    }
    __syncthreads();
  }
}

// ---- dense LU, blocked, without row exchanges (the common case) --------------
// The same factorization as lu_solve for the systems on which partial
// pivoting keeps every diagonal pivot: by panels of kFb columns, the
// diagonal block is factored in shared memory, its triangular factors are
// inverted there, and L21 = A21 U11^-1, U12 = L11^-1 A12 and A22 -= L21 U12
// run as 64 x 64 shared-memory tile products (the right-hand side rides as
// column n, so forward elimination is part of the factorization). Back
// substitution runs panel by panel with the stored U11^-1. Partial pivoting
// would exchange rows only where some |l_ik| > 1; a multiplier above 1 by more
// than rounding (1e-8), or a zero or non-finite pivot, stops the fast path and
// marks the system for lu_solve (pivot[sys] = 1), which starts it over.
constexpr int kFb = 64;
constexpr int kFld = kFb + 1;
constexpr double kPivotSlack = 1e-8;
constexpr size_t kFastSmem = 5 * (size_t)kFb * kFld * sizeof(double);

__host__ __device__ constexpr size_t fast_slot_elems(int n) {
  return (size_t)n * (n + 1) + (size_t)((n + kFb - 1) / kFb) * kFb * kFb + 64;
}

// dst[r][c] = M[(r0 + r) ld + c0 + c] for r < rows, c < cols, else 0. The
// kernel runs kLsThreads threads (one CTA per SM): each issues all of its
// kFb^2 / kLsThreads loads before the stores, so they are in flight together.
constexpr int kFastPer = kFb * kFb / kLsThreads;
__device__ __forceinline__ void fast_load(double (*dst)[kFld], const double* __restrict__ M, size_t ld, int r0,
                                          int c0, int rows, int cols) {
  double v[kFastPer];
#pragma unroll
  for (int t = 0; t < kFastPer; ++t) {
    const int q = threadIdx.x + t * kLsThreads, r = q / kFb, c = q % kFb;
    v[t] = (r < rows && c < cols) ? M[(size_t)(r0 + r) * ld + c0 + c] : 0.0;
  }
#pragma unroll
  for (int t = 0; t < kFastPer; ++t) {
    const int q = threadIdx.x + t * kLsThreads;
    dst[q / kFb][q % kFb] = v[t];
  }
}

// acc[a][q] = sum_c A[ty + 16 a][c] B[c][tx + 16 q], c < kb.
__device__ __forceinline__ void fast_mm(const double (*A)[kFld], const double (*B)[kFld], int kb,
                                        double (&acc)[4][4]) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[a][q] = 0.0;
  for (int c = 0; c < kb; ++c) {
    double lv[4], uv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) lv[a] = A[ty + 16 * a][c];
#pragma unroll
    for (int q = 0; q < 4; ++q) uv[q] = B[c][tx + 16 * q];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[a][q] += lv[a] * uv[q];
  }
}

// Factor and solve the n x n system in M (row stride n + 1, right-hand side in
// column n); on success column n holds x. Returns false (uniformly) when the
// pivot guard stops the fast path.
__device__ bool lu_solve_fast(double* __restrict__ M, double* __restrict__ Uinv_store, int n, unsigned char* smem,
                              int* s_bad, double* s_tmp) {
  double(*Da)[kFld] = reinterpret_cast<double(*)[kFld]>(smem);
  double(*Li)[kFld] = Da + kFb;
  double(*Ui)[kFld] = Li + kFb;
  double(*At)[kFld] = Ui + kFb;
  double(*Bt)[kFld] = At + kFb;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int tx = tid & 15, ty = tid >> 4;
  const size_t ld = (size_t)n + 1;
  if (tid == 0) *s_bad = 0;
  __syncthreads();
  for (int k0 = 0, p = 0; k0 < n; k0 += kFb, ++p) {
    const int kb = min(kFb, n - k0), m0 = k0 + kb;
    fast_load(Da, M, ld, k0, k0, kb, kb);
    __syncthreads();
    for (int k = 0; k < kb; ++k) {
      const double piv = Da[k][k];
      if (tid == 0 && (!(fabs(piv) > 0.0) || !isfinite(piv))) *s_bad = 1;
      for (int i = k + 1 + tid; i < kb; i += nt) {
        const double v = Da[i][k];
        if (fabs(v) > fabs(piv) * (1.0 + kPivotSlack)) *s_bad = 1;
        Da[i][k] = v / piv;
      }
      __syncthreads();
      const int w = kb - k - 1;
      for (int q = tid; q < w * w; q += nt) {
        const int i = k + 1 + q / w, j = k + 1 + q % w;
        Da[i][j] -= Da[i][k] * Da[k][j];
      }
      __syncthreads();
    }
    if (*s_bad) return false;
    // U11^-1 (upper) and L11^-1 (unit lower), one column per thread; zero elsewhere
    for (int q = tid; q < kFb * kFb; q += nt) {
      Ui[q / kFb][q % kFb] = 0.0;
      Li[q / kFb][q % kFb] = 0.0;
    }
    __syncthreads();
    if (tid < kb) {
      const int j = tid;
      Ui[j][j] = 1.0 / Da[j][j];
      for (int i = j - 1; i >= 0; --i) {
        double t = 0.0;
        for (int k = i + 1; k <= j; ++k) t += Da[i][k] * Ui[k][j];
        Ui[i][j] = -t / Da[i][i];
      }
      Li[j][j] = 1.0;
      for (int i = j + 1; i < kb; ++i) {
        double t = 0.0;
        for (int k = j; k < i; ++k) t += Da[i][k] * Li[k][j];
        Li[i][j] = -t;
      }
    }
    __syncthreads();
    for (int q = tid; q < kFb * kFb; q += nt) Uinv_store[(size_t)p * kFb * kFb + q] = Ui[q / kFb][q % kFb];
    // L21 = A21 U11^-1
    for (int rt = m0; rt < n; rt += kFb) {
      const int rows = min(kFb, n - rt);
      fast_load(At, M, ld, rt, k0, rows, kb);
      __syncthreads();
      double acc[4][4];
      fast_mm(At, Ui, kb, acc);
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = ty + 16 * a, c = tx + 16 * q;
          if (r < rows && c < kb) {
            if (fabs(acc[a][q]) > 1.0 + kPivotSlack || !isfinite(acc[a][q])) *s_bad = 1;
            M[(size_t)(rt + r) * ld + k0 + c] = acc[a][q];
          }
        }
      __syncthreads();
    }
    if (*s_bad) return false;
    // U12 = L11^-1 A12, the right-hand side column included
    for (int ct = m0; ct <= n; ct += kFb) {
      const int cols = min(kFb, n + 1 - ct);
      fast_load(Bt, M, ld, k0, ct, kb, cols);
      __syncthreads();
      double acc[4][4];
      fast_mm(Li, Bt, kb, acc);
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = ty + 16 * a, c = tx + 16 * q;
          if (r < kb && c < cols) M[(size_t)(k0 + r) * ld + ct + c] = acc[a][q];
        }
      __syncthreads();
    }
    // A22 -= L21 U12 (columns through the right-hand side)
    for (int rt = m0; rt < n; rt += kFb) {
      const int rows = min(kFb, n - rt);
      fast_load(At, M, ld, rt, k0, rows, kb);
      for (int ct = m0; ct <= n; ct += kFb) {
        const int cols = min(kFb, n + 1 - ct);
        fast_load(Bt, M, ld, k0, ct, kb, cols);
        __syncthreads();
        // this thread's C entries are loaded before the product, so their
        // latency overlaps it
        double cv[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = ty + 16 * a, c = tx + 16 * q;
            cv[a][q] = (r < rows && c < cols) ? M[(size_t)(rt + r) * ld + ct + c] : 0.0;
          }
        double acc[4][4];
        fast_mm(At, Bt, kb, acc);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = ty + 16 * a, c = tx + 16 * q;
            if (r < rows && c < cols) M[(size_t)(rt + r) * ld + ct + c] = cv[a][q] - acc[a][q];
          }
        __syncthreads();
      }
    }
  }
  // back substitution by panels, from the last: x_p = U11^-1 (y_p - U12 x_rest)
  const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int np = (n + kFb - 1) / kFb;
  for (int p = np - 1; p >= 0; --p) {
    const int k0 = p * kFb, kb = min(kFb, n - k0), m0 = k0 + kb;
    for (int i = warp; i < kb; i += nw) {
      double t = 0.0;
      for (int j = m0 + lane; j < n; j += 32) t += M[(size_t)(k0 + i) * ld + j] * M[(size_t)j * ld + n];
      t = warp_sum(t);
      if (lane == 0) s_tmp[i] = M[(size_t)(k0 + i) * ld + n] - t;
    }
    __syncthreads();
    for (int i = tid; i < kb; i += nt) {
      double t = 0.0;
      for (int k = 0; k < kb; ++k) t += Uinv_store[(size_t)p * kFb * kFb + i * kFb + k] * s_tmp[k];
      M[(size_t)(k0 + i) * ld + n] = t;
    }
    __syncthreads();
  }
  return true;
}

// Dense solves of the listed systems on the fast path (modes as k_ls_dense);
// a system whose pivot guard fires gets pivot[sys] = 1 and is left to k_ls_dense.
__global__ void __launch_bounds__(kLsThreads) k_ls_dense_fast(LsArgs A, const int* __restrict__ list, int count,
                                                             int direct, unsigned* queue, double* scratch,
                                                             size_t slot_elems, const LsParams* __restrict__ prm,
                                                             int* pivot) {
  extern __shared__ __align__(16) unsigned char fsm[];
  __shared__ double red[2][2][32];
  __shared__ double s_tmp[kFb];
  __shared__ int s_k, s_bad;
  const int tid = threadIdx.x, nt = blockDim.x;
  double* slot = scratch + (size_t)blockIdx.x * slot_elems;
  int rslot = 0;
  const double tol = prm->tol;
  for (;;) {
    if (tid == 0) s_k = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int q = s_k;
    __syncthreads();
    if (q >= count) break;
    const int sys = list[q];
    const int r0 = A.sys_row[sys], n = A.sys_row[sys + 1] - r0;
    const size_t ld = (size_t)n + 1;
    double* M = slot;
    double* Uinv = slot + (size_t)n * ld;
    int path = direct ? CFD_LS_PATH_DIRECT : A.path[sys];
    double ratio = NAN;
    bool need_pivot = false;
    for (int attempt = direct ? 0 : 1; attempt < 2; ++attempt) {
      const bool scaled = attempt == 0;
      for (size_t e = tid; e < (size_t)n * ld; e += nt) M[e] = 0.0;
      __syncthreads();
      for (int i = tid; i < n; i += nt) {
        const int g = r0 + i, e0 = A.rp[g], e1 = A.rp[g + 1];
        const double s = scaled ? ls_scale(A.v64, e0, e1) : 1.0;
        for (int e = e0; e < e1; ++e) M[(size_t)i * ld + A.col[e]] += A.v64[e] * s;
        M[(size_t)i * ld + n] = A.b[g] * s;
      }
      __syncthreads();
      if (!lu_solve_fast(M, Uinv, n, fsm, &s_bad, s_tmp)) {
        need_pivot = true;
        break;
      }
      for (int i = tid; i < n; i += nt) A.x[r0 + i] = M[(size_t)i * ld + n];
      __syncthreads();
      ratio = ls_target_ratio(A, r0, n, red, rslot);
      if (!scaled || ratio <= tol) break;
      path = CFD_LS_PATH_DIRECT_UNSCALED;
      __syncthreads();
    }
    if (tid == 0) {
      pivot[sys] = need_pivot ? 1 : 0;
      if (!need_pivot) {
        A.path[sys] = path;
        A.resid[sys] = ratio;
        if (direct) {
          A.term[sys] = -1;
          A.iters[sys] = 0;
        }
      }
    }
    __syncthreads();
  }
}

// Detection alone for the direct systems (the method is reported for every system).
__global__ void k_ls_detect(LsArgs A, const int* __restrict__ list, int count, int fixed) {
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (q >= count) return;
  const int sys = list[q];
  const int r0 = A.sys_row[sys], n = A.sys_row[sys + 1] - r0;
  bool not_spd = false;
  for (int i = lane; i < n; i += 32) {
    const int g = r0 + i;
    double diag = 0.0, sum_off = 0.0;
    bool row_bad = false;
    for (int e = A.rp[g]; e < A.rp[g + 1]; ++e) {
      const double a = A.v64[e];
      if (A.col[e] == i)
        diag = a;
      else if (a > 0.0)
        row_bad = true;
      else
        sum_off += fabs(a);
    }
    const bool identity = diag == 1.0 && sum_off == 0.0;
    if (row_bad || ((diag < sum_off || diag <= 0.0) && !identity)) not_spd = true;
  }
  not_spd = __any_sync(0xffffffffu, not_spd);
  if (lane == 0) A.method[sys] = fixed >= 0 ? fixed : (not_spd ? CFD_LS_BICGSTAB : CFD_LS_CG);
}

template <typename T>
cfd_status ls_alloc(T** p, int64_t n) {
  if (cudaMalloc((void**)p, (size_t)std::max<int64_t>(n + 16, 16) * sizeof(T)) != cudaSuccess) {
    *p = nullptr;
    set_error("cudaMalloc failed for a batch buffer of %lld elements", (long long)n);
    return CFD_ERR_ALLOC;
  }
  return CFD_OK;
}

// Per-system result arrays, the device lists and the parameter block, made
// at the first cascade solve of a batch.
cfd_status ls_prepare(cfd_batch* bt) {
  if (bt->ls_path) return CFD_OK;
  CFD_TRY(ls_alloc(&bt->ls_method, bt->nsys));
  CFD_TRY(ls_alloc(&bt->ls_path, bt->nsys));
  CFD_TRY(ls_alloc(&bt->ls_list, bt->nsys));
  CFD_TRY(ls_alloc(&bt->ls_params, (int64_t)((sizeof(LsParams) + 7) / 8)));
  CFD_TRY(ls_alloc(&bt->ls_queue, 2));
  CFD_TRY(ls_alloc(&bt->ls_pivot, bt->nsys));
  return CFD_OK;
}

cfd_status ls_ensure_scratch(cfd_batch* bt, size_t slot_elems, int slots) {
  const size_t need = slot_elems * (size_t)slots;
  if (need <= bt->ls_scratch_elems) return CFD_OK;
  if (bt->ls_scratch) cudaFree(bt->ls_scratch);
  bt->ls_scratch = nullptr;
  bt->ls_scratch_elems = 0;
  if (cudaMalloc((void**)&bt->ls_scratch, need * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    set_error("cfd_batch_linear_system_solve: cudaMalloc of %zu bytes of dense-solve scratch failed",
              need * sizeof(double));
    return CFD_ERR_ALLOC;
  }
  bt->ls_scratch_elems = need;
  return CFD_OK;
}

// Dense solves of `list` (host, systems of at most nmax rows): the blocked
// fast path for all, then lu_solve for the systems whose pivot guard fired.
cfd_status ls_dense_launch(cfd_batch* bt, const LsArgs& A, const std::vector<int>& list, int nmax, bool direct,
                           cudaStream_t s) {
  if (list.empty()) return CFD_OK;
  const LsParams* prm = reinterpret_cast<const LsParams*>(bt->ls_params);
  if (cudaFuncSetAttribute(k_ls_dense_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFastSmem) !=
      cudaSuccess) {
    cudaGetLastError();
    set_error("cfd_batch_linear_system_solve: %zu bytes of shared memory for the dense solve are not available",
              kFastSmem);
    return CFD_ERR_CONFIG;
  }
  int occ = 0;
  CFD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ls_dense_fast, kLsThreads, kFastSmem));
  int grid = std::min<int>((int)list.size(), bt->ctx->num_sms * std::max(1, occ));
  const size_t slot = fast_slot_elems(nmax);
  CFD_TRY(ls_ensure_scratch(bt, slot, grid));
  CFD_TRY_CUDA(cudaMemcpyAsync(bt->ls_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  CFD_TRY_CUDA(cudaMemsetAsync(bt->ls_queue, 0, sizeof(unsigned), s));
  k_ls_dense_fast<<<grid, kLsThreads, kFastSmem, s>>>(A, bt->ls_list, (int)list.size(), direct ? 1 : 0,
                                                      bt->ls_queue, bt->ls_scratch, slot, prm, bt->ls_pivot);
  CFD_TRY_CUDA(cudaGetLastError());
  bt->ctx->stats.launches++;
  std::vector<int> piv(bt->nsys);
  CFD_TRY_CUDA(cudaMemcpyAsync(piv.data(), bt->ls_pivot, bt->nsys * sizeof(int), cudaMemcpyDeviceToHost, s));
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  std::vector<int> slow;
  int smax = 1;
  for (int sy : list)
    if (piv[sy]) {
      slow.push_back(sy);
      smax = std::max(smax, bt->h_sys_row[sy + 1] - bt->h_sys_row[sy]);
    }
  bt->ls_pivoted += (int64_t)slow.size();
  if (slow.empty()) return CFD_OK;
  CFD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ls_dense, kLsThreads, 0));
  grid = std::min<int>((int)slow.size(), bt->ctx->num_sms * std::max(1, occ));
  if (smax > 512) grid = std::min(grid, bt->ctx->num_sms);
  const size_t slot2 = (size_t)smax * smax + (size_t)smax + 16;
  CFD_TRY(ls_ensure_scratch(bt, slot2, grid));
  CFD_TRY_CUDA(cudaMemcpyAsync(bt->ls_list, slow.data(), slow.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  CFD_TRY_CUDA(cudaMemsetAsync(bt->ls_queue, 0, sizeof(unsigned), s));
  k_ls_dense<<<grid, kLsThreads, 0, s>>>(A, bt->ls_list, (int)slow.size(), direct ? 1 : 0, bt->ls_queue,
                                         bt->ls_scratch, slot2, prm);
  CFD_TRY_CUDA(cudaGetLastError());
  bt->ctx->stats.launches++;
  return CFD_OK;
}

template <bool REFINE>
cfd_status ls_krylov_bucket(cfd_batch* bt, const LsArgs& A, int bkt, cudaStream_t s) {
  using T = typename std::conditional<REFINE, float, double>::type;
  const int count = bt->bucket_begin[bkt + 1] - bt->bucket_begin[bkt];
  if (count == 0) return CFD_OK;
  const int nmax = bt->bucket_nmax[bkt], zmax = bt->bucket_zmax[bkt];
  const size_t smem = ls_smem<T>(nmax, zmax);
  auto kern = k_ls_krylov<T, REFINE>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    set_error("cfd_batch_linear_system_solve: bucket %d needs %zu bytes of shared memory", bkt, smem);
    return CFD_ERR_CONFIG;
  }
  int threads = std::min(512, std::max(32, bt->threads[REFINE ? 1 : 0][bkt]));
  int occ = 0;
  CFD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem));
  if (occ < 1) {
    set_error("cfd_batch_linear_system_solve: bucket %d: %zu bytes of shared memory at %d threads do not fit", bkt,
              smem, threads);
    return CFD_ERR_CONFIG;
  }
  const int grid = std::min(count, bt->ctx->num_sms * occ);
  CFD_TRY_CUDA(cudaMemsetAsync(bt->ls_queue + 1, 0, sizeof(unsigned), s));
  kern<<<grid, threads, smem, s>>>(A, bt->order + bt->bucket_begin[bkt], count, bt->ls_queue + 1,
                                   reinterpret_cast<const LsParams*>(bt->ls_params), nmax, zmax);
  CFD_TRY_CUDA(cudaGetLastError());
  bt->ctx->stats.launches++;
  return CFD_OK;
}

}  // namespace

size_t ls_krylov_smem_bytes(int precision, int nmax, int zmax) {
  return precision ? ls_smem<float>(nmax, zmax) : ls_smem<double>(nmax, zmax);
}

}  // namespace cfd

using namespace cfd;

extern "C" {

void cfd_ls_options_default(cfd_ls_options* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->tolerance = 1e-6;  // LinearSystemSolver::new (linear_system.rs:63-69)
  opt->max_iterations = 1000;
  opt->method = CFD_LS_DETECT;
  opt->precision = CFD_PRECISION_FP64;
  opt->memory = CFD_MEMORY_HOST;
  opt->inner_tolerance = 1e-4;
  opt->max_outer = 40;
}

cfd_status cfd_batch_linear_system_solve(cfd_batch* bt, const cfd_ls_options* opt, const double* b, double* x,
                                         cfd_ls_result* results, cfd_batch_report* rep) {
  return guarded("cfd_batch_linear_system_solve", [&]() -> cfd_status {
    if (!bt || !opt || !x || !rep) {
      set_error("cfd_batch_linear_system_solve: null argument");
      return CFD_ERR_STATE;
    }
    if (!b && !bt->rhs_resident) {
      set_error("cfd_batch_linear_system_solve: b is NULL but no assembled right-hand side is resident");
      return CFD_ERR_STATE;
    }
    if (!bt->values_valid) {
      set_error("cfd_batch_linear_system_solve: the batch holds no valid matrix (assemble it, or update its values, "
                "first)");
      return CFD_ERR_STATE;
    }
    if (!(opt->tolerance >= 0.0) || opt->max_iterations <= 0 || opt->method < CFD_LS_CG ||
        opt->method > CFD_LS_DETECT || opt->precision < 0 || opt->precision > 1 ||
        (opt->memory != CFD_MEMORY_HOST && opt->memory != CFD_MEMORY_DEVICE) ||
        (opt->precision == CFD_PRECISION_FP32_REFINE && !(opt->inner_tolerance > 0.0 && opt->inner_tolerance < 1.0))) {
      set_error("cfd_batch_linear_system_solve: needs a tolerance >= 0, a positive iteration budget, a method "
                "(CG, BiCGSTAB or detect), a precision and, for FP32_REFINE, an inner tolerance in (0, 1)");
      return CFD_ERR_CONFIG;
    }
    std::lock_guard<std::mutex> g(bt->ctx->mu);
    cfd_context* ctx = bt->ctx;
    CFD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    std::memset(rep, 0, sizeof(*rep));
    rep->num_systems = bt->nsys;
    if (bt->nsys == 0) return CFD_OK;
    CFD_TRY(ls_prepare(bt));
    if (bt->f32_out_of_range && opt->precision == CFD_PRECISION_FP32_REFINE) {
      set_error("cfd_batch_linear_system_solve: an assembled entry exceeds the FP32 range; solve in FP64");
      return CFD_ERR_NONFINITE;
    }
    LsParams hp{opt->tolerance, opt->inner_tolerance,
                (int32_t)std::min<int64_t>(opt->max_iterations, INT32_MAX), std::max(1, opt->max_outer),
                opt->method};
    const cudaMemcpyKind in = opt->memory == CFD_MEMORY_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind outk = opt->memory == CFD_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    CFD_TRY_CUDA(cudaEventRecord(ctx->ev0, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(bt->ls_params, &hp, sizeof(hp), cudaMemcpyHostToDevice, s));
    if (b) {
      bt->rhs_resident = false;
      CFD_TRY_CUDA(cudaMemcpyAsync(bt->b, b, bt->rows * sizeof(double), in, s));
    }
    CFD_TRY_CUDA(cudaMemcpyAsync(bt->x, x, bt->rows * sizeof(double), in, s));
    LsArgs A{bt->sys_row, bt->rp, bt->col, bt->v64, bt->v32, bt->b, bt->x,
             bt->ls_method, bt->ls_path, bt->term, bt->iters, bt->resid};
    // direct systems: rows <= 256, the buckets below kBucketRows[2]
    std::vector<int> direct;
    int dmax = 1;
    for (int q = bt->bucket_begin[0]; q < bt->bucket_begin[2]; ++q) {
      const int sy = bt->h_order[q];
      direct.push_back(sy);
      dmax = std::max(dmax, bt->h_sys_row[sy + 1] - bt->h_sys_row[sy]);
    }
    // Phase boundaries: start, after the direct solves, after the Krylov
    // launches, after the fallback (events released on every return).
    struct PhaseEvents {
      cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
      ~PhaseEvents() {
        for (cudaEvent_t& q : e)
          if (q) cudaEventDestroy(q);
      }
    } ph;
    for (cudaEvent_t& q : ph.e) CFD_TRY_CUDA(cudaEventCreate(&q));
    CFD_TRY_CUDA(cudaEventRecord(ph.e[0], s));
    if (!direct.empty()) {
      CFD_TRY_CUDA(cudaMemcpyAsync(bt->ls_list, direct.data(), direct.size() * sizeof(int), cudaMemcpyHostToDevice, s));
      const int fixed = opt->method == CFD_LS_DETECT ? -1 : opt->method;
      k_ls_detect<<<(int)((direct.size() + 7) / 8), 256, 0, s>>>(A, bt->ls_list, (int)direct.size(), fixed);
      CFD_TRY_CUDA(cudaGetLastError());
      ctx->stats.launches++;
      CFD_TRY(ls_dense_launch(bt, A, direct, dmax, true, s));
    }
    CFD_TRY_CUDA(cudaEventRecord(ph.e[1], s));
    for (int k = kBuckets - 1; k >= 2; --k) {
      if (opt->precision)
        CFD_TRY(ls_krylov_bucket<true>(bt, A, k, s));
      else
        CFD_TRY(ls_krylov_bucket<false>(bt, A, k, s));
    }
    CFD_TRY_CUDA(cudaEventRecord(ph.e[2], s));
    std::vector<int> path(bt->nsys), method(bt->nsys), term(bt->nsys), iters(bt->nsys);
    std::vector<double> resid(bt->nsys);
    CFD_TRY_CUDA(cudaMemcpyAsync(path.data(), bt->ls_path, bt->nsys * sizeof(int), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaStreamSynchronize(s));
    CFD_TRY(check_device_flag(ctx));
    // Krylov solves that were not kept: dense LU of the original system.
    std::vector<int> fallback;
    int fmax = 1;
    for (int q = bt->bucket_begin[2]; q < bt->nsys; ++q) {
      const int sy = bt->h_order[q];
      if (path[sy] == CFD_LS_PATH_KRYLOV_FALLBACK) {
        fallback.push_back(sy);
        fmax = std::max(fmax, bt->h_sys_row[sy + 1] - bt->h_sys_row[sy]);
      }
    }
    CFD_TRY(ls_dense_launch(bt, A, fallback, fmax, false, s));
    CFD_TRY_CUDA(cudaEventRecord(ph.e[3], s));
    CFD_TRY_CUDA(cudaMemcpyAsync(x, bt->x, bt->rows * sizeof(double), outk, s));
    CFD_TRY_CUDA(cudaEventRecord(ctx->ev1, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(path.data(), bt->ls_path, bt->nsys * sizeof(int), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(method.data(), bt->ls_method, bt->nsys * sizeof(int), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(term.data(), bt->term, bt->nsys * sizeof(int), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(iters.data(), bt->iters, bt->nsys * sizeof(int), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(resid.data(), bt->resid, bt->nsys * sizeof(double), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    CFD_TRY_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    rep->device_ms = ms;
    float pm[3] = {0.f, 0.f, 0.f};
    for (int q = 0; q < 3; ++q) CFD_TRY_CUDA(cudaEventElapsedTime(&pm[q], ph.e[q], ph.e[q + 1]));
    rep->direct_ms = pm[0];
    rep->krylov_ms = pm[1];
    rep->fallback_ms = pm[2];
    for (int k = 0; k < bt->nsys; ++k) {
      if (path[k] != CFD_LS_PATH_FAILED && path[k] != CFD_LS_PATH_ERROR) rep->converged_systems++;
      rep->total_iterations += iters[k];
      rep->max_iterations = std::max(rep->max_iterations, iters[k]);
      if (std::isfinite(resid[k])) rep->max_rel_residual = std::max(rep->max_rel_residual, resid[k]);
      if (results) results[k] = cfd_ls_result{method[k], path[k], term[k], iters[k], resid[k]};
    }
    return CFD_OK;
  });
}

}  // extern "C"
