// Device orchestration: SpMV launch helpers, the AMG V-cycle, preconditioned
// CG and BiCGSTAB, and FP32-inner / FP64-refinement solves.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <chrono>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "amg_device.h"
#include "internal.h"
#include "simple.h"
#include "kernels.cuh"

namespace cfd {

namespace {

constexpr int kPreNone = 0, kPreJacobi = 1, kPreAmg = 2, kPreSimple = 3, kPreBlockDiag = 4, kPreComponent = 5;

inline int vec_grid(int64_t n) {
  int64_t g = (n + kThreads - 1) / kThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, kVecGrid));
}

#define GRID_STRIDE(i, n) for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < (n); i += (int64_t)gridDim.x * kThreads)
// The same loop with four strided elements per pass: the elements are visited
// in the same order (so per-thread sums are unchanged), but the loads of four
// iterations are in flight together. One 4- or 8-byte element per thread at a
// time leaves too few bytes in flight per SM to reach the HBM bandwidth.
#define GRID_STRIDE_U4(i, n, ...)                                                       \
  {                                                                                    \
    const int64_t gs_t_ = (int64_t)gridDim.x * kThreads;                               \
    int64_t gs_i_ = (int64_t)blockIdx.x * kThreads + threadIdx.x;                      \
    for (; gs_i_ + 3 * gs_t_ < (n); gs_i_ += 4 * gs_t_) {                              \
      _Pragma("unroll") for (int gs_u_ = 0; gs_u_ < 4; ++gs_u_) {                      \
        const int64_t i = gs_i_ + gs_u_ * gs_t_;                                       \
        __VA_ARGS__                                                                    \
      }                                                                                \
    }                                                                                  \
    for (; gs_i_ < (n); gs_i_ += gs_t_) {                                              \
      const int64_t i = gs_i_;                                                         \
      __VA_ARGS__                                                                      \
    }                                                                                  \
  }

// ---------------------------------------------------------------------------
// Vector kernels.

// First damped-Jacobi sweep from a zero iterate: x = w (b / a_ii)
// (smooth0_value: the FP32 sweep divides with the fast division).
template <typename XT>
__global__ void __launch_bounds__(kThreads) k_smooth0(int64_t n, const XT* __restrict__ b, const XT* __restrict__ d,
                                                      XT omega, XT* __restrict__ x, const int* done) {
  pdl_enter();
  if (flag_set(done)) return;
  GRID_STRIDE_U4(i, n, {
    x[i] = smooth0_value<XT>(b[i], d[i], omega);
  })
}

template <typename XT>
__global__ void __launch_bounds__(kThreads) k_fill(int64_t n, XT* __restrict__ x, XT v, const int* done) {
  pdl_enter();
  if (flag_set(done)) return;
  GRID_STRIDE_U4(i, n, x[i] = v;)
}

template <typename XT>
__global__ void __launch_bounds__(kThreads) k_copy(int64_t n, const XT* __restrict__ s, XT* __restrict__ d, const int* done) {
  pdl_enter();
  if (flag_set(done)) return;
  GRID_STRIDE_U4(i, n, d[i] = s[i];)
}

// Dense coarsest-level solve x = A_c^{-1} b with the inverse (FP64, or its FP32
// rounding in the FP32 V-cycle), FP64 sums; one warp per row.
template <typename XT, typename IT>
__global__ void __launch_bounds__(kThreads) k_dense_gemv(int n, const IT* __restrict__ inv, const XT* __restrict__ b,
                                                         XT* __restrict__ x, const int* done) {
  pdl_enter();
  if (flag_set(done)) return;
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (row >= n) return;
  const IT* a = inv + (size_t)row * n;
  double s = 0.0;
  for (int k = lane; k < n; k += 32) s += (double)a[k] * (double)b[k];
  s = warp_sum(s);
  if (lane == 0) x[row] = (XT)s;
}

// PCG: x += alpha p; r -= alpha q; ||r||; with Jacobi also rho_new = r.(D^-1 r).
// The last CTA applies the termination tests (converged / non-finite / budget)
// and, for Jacobi or no preconditioner, beta = rho_new / rho.
// With AMG, x0 != NULL also writes the V-cycle's first pre-smoothing sweep on
// the new r (x0 = w r / a_ii, smooth0_value with the fine level's diagonal d0).
template <typename XT, int PRE>
__global__ void __launch_bounds__(kThreads) k_cg_update(int64_t n, XT* __restrict__ x, const XT* __restrict__ p,
                                                        XT* __restrict__ r, const XT* __restrict__ q,
                                                        const XT* __restrict__ jinv, DevState* st, Red red,
                                                        XT* __restrict__ x0, const XT* __restrict__ d0, XT omega) {
  pdl_enter();
  if (st->done) return;
  const XT a = (XT)st->alpha;
  double acc[2] = {0.0, 0.0};
  GRID_STRIDE_U4(i, n, {
    x[i] = x[i] + a * p[i];
    const XT ri = r[i] - a * q[i];
    r[i] = ri;
    acc[0] += (double)ri * (double)ri;
    if (PRE == kPreJacobi) acc[1] += (double)ri * (double)(ri * jinv[i]);
    if (PRE == kPreAmg && x0) x0[i] = smooth0_value<XT>(ri, d0[i], omega);
  })
  double tot[2];
  if (grid_reduce<2>(acc, red, tot) && threadIdx.x == 0) {
    const double rn = sqrt(tot[0]);
    st->rr = tot[0];
    st->rnorm = rn;
    st->iter += 1;
    if (!isfinite(rn)) {
      st->term = CFD_TERM_BREAKDOWN;
      st->done = 1;
    } else if (rn <= st->threshold) {
      st->term = CFD_TERM_CONVERGED;
      st->done = 1;
    } else if (st->iter >= st->max_iter) {
      st->term = CFD_TERM_MAX_ITERATIONS;
      st->done = 1;
    } else if (PRE == kPreJacobi) {
      pcg_rho_update(st, tot[1]);
    } else if (PRE == kPreNone) {
      pcg_rho_update(st, tot[0]);
    }
  }
}

// PCG start: p = M r and rho = r.p.
template <typename XT, int PRE>
__global__ void __launch_bounds__(kThreads) k_pcg_init(int64_t n, XT* __restrict__ p, const XT* __restrict__ r,
                                                       const XT* __restrict__ z, const XT* __restrict__ jinv,
                                                       DevState* st, Red red) {
  pdl_enter();
  if (st->done) return;
  double acc[1] = {0.0};
  GRID_STRIDE_U4(i, n, {
    const XT ri = r[i];
    const XT zi = PRE == kPreAmg ? z[i] : (PRE == kPreJacobi ? ri * jinv[i] : ri);
    p[i] = zi;
    acc[0] += (double)ri * (double)zi;
  })
  double tot[1];
  if (grid_reduce<1>(acc, red, tot) && threadIdx.x == 0) st->rho = tot[0];
}

// PCG direction: p = z + beta p (z = D^-1 r, r or the V-cycle output).
template <typename XT, int PRE>
__global__ void __launch_bounds__(kThreads) k_p_update(int64_t n, XT* __restrict__ p, const XT* __restrict__ r,
                                                       const XT* __restrict__ z, const XT* __restrict__ jinv,
                                                       const DevState* st) {
  pdl_enter();
  if (st->done) return;
  const XT beta = (XT)st->beta;
  GRID_STRIDE_U4(i, n, {
    const XT zi = PRE == kPreAmg ? z[i] : (PRE == kPreJacobi ? r[i] * jinv[i] : r[i]);
    p[i] = zi + beta * p[i];
  })
}

// rho_new = r.z after a preconditioner whose last kernel could not fuse it.
template <typename XT>
__global__ void __launch_bounds__(kThreads) k_rz(int64_t n, const XT* __restrict__ r, const XT* __restrict__ z,
                                                 DevState* st, int mode, Red red) {
  pdl_enter();
  if (st->done) return;
  double acc[1] = {0.0};
  GRID_STRIDE_U4(i, n, acc[0] += (double)r[i] * (double)z[i];)
  double tot[1];
  if (grid_reduce<1>(acc, red, tot) && threadIdx.x == 0) {
    if (mode == 1)
      st->rho = tot[0];
    else
      pcg_rho_update(st, tot[0]);
  }
}

// ---- BiCGSTAB (Saad 2003, Alg. 7.7, right preconditioning) --------------------
// rho_new = r_hat.r; beta = (rho_new / rho)(alpha / omega).
template <typename XT>
__global__ void __launch_bounds__(kThreads) k_bicg_rho(int64_t n, const XT* __restrict__ rhat, const XT* __restrict__ r,
                                                       DevState* st, Red red) {
  pdl_enter();
  if (st->done) return;
  double acc[1] = {0.0};
  GRID_STRIDE_U4(i, n, acc[0] += (double)rhat[i] * (double)r[i];)
  double tot[1];
  if (grid_reduce<1>(acc, red, tot) && threadIdx.x == 0) {
    const double rho_new = tot[0];
    if (rho_new == 0.0 || !isfinite(rho_new)) {
      st->term = CFD_TERM_BREAKDOWN;
      st->done = 1;
      return;
    }
    st->beta = (rho_new / st->rho) * (st->alpha / st->omega);
    st->rho = rho_new;
  }
}

// p = r + beta (p - omega v) (first: p = r); with Jacobi also p_hat = D^-1 p.
template <typename XT, int PRE>
__global__ void __launch_bounds__(kThreads) k_bicg_p(int64_t n, XT* __restrict__ p, XT* __restrict__ ph,
                                                     const XT* __restrict__ r, const XT* __restrict__ v,
                                                     const XT* __restrict__ jinv, const DevState* st, int first) {
  pdl_enter();
  if (st->done) return;
  const XT beta = (XT)st->beta, om = (XT)st->omega;
  GRID_STRIDE_U4(i, n, {
    const XT pi = first ? r[i] : r[i] + beta * (p[i] - om * v[i]);
    p[i] = pi;
    if (PRE == kPreJacobi) ph[i] = pi * jinv[i];
    if (PRE == kPreNone) ph[i] = pi;
  })
}

// s = r - alpha v; ||s|| (early exit: the host then adds alpha p_hat to x);
// with Jacobi also s_hat = D^-1 s.
template <typename XT, int PRE>
__global__ void __launch_bounds__(kThreads) k_bicg_s(int64_t n, XT* __restrict__ s, XT* __restrict__ sh,
                                                     const XT* __restrict__ r, const XT* __restrict__ v,
                                                     const XT* __restrict__ jinv, DevState* st, Red red) {
  pdl_enter();
  if (st->done) return;
  const XT a = (XT)st->alpha;
  double acc[1] = {0.0};
  GRID_STRIDE_U4(i, n, {
    const XT si = r[i] - a * v[i];
    s[i] = si;
    if (PRE == kPreJacobi) sh[i] = si * jinv[i];
    if (PRE == kPreNone) sh[i] = si;
    acc[0] += (double)si * (double)si;
  })
  double tot[1];
  if (grid_reduce<1>(acc, red, tot) && threadIdx.x == 0) {
    const double sn = sqrt(tot[0]);
    st->iter += 1;
    if (sn <= st->threshold) {
      st->rnorm = sn;
      st->term = CFD_TERM_CONVERGED;
      st->spare0 = 1.0;  // x still needs alpha p_hat
      st->done = 1;
    }
  }
}

// x += alpha p_hat + omega s_hat; r = s - omega t; ||r|| and termination tests.
template <typename XT>
__global__ void __launch_bounds__(kThreads) k_bicg_x(int64_t n, XT* __restrict__ x, XT* __restrict__ r,
                                                     const XT* __restrict__ ph, const XT* __restrict__ sh,
                                                     const XT* __restrict__ s, const XT* __restrict__ t,
                                                     DevState* st, Red red) {
  pdl_enter();
  if (st->done) return;
  const XT a = (XT)st->alpha, om = (XT)st->omega;
  double acc[1] = {0.0};
  GRID_STRIDE_U4(i, n, {
    x[i] = x[i] + (a * ph[i] + om * sh[i]);
    const XT ri = s[i] - om * t[i];
    r[i] = ri;
    acc[0] += (double)ri * (double)ri;
  })
  double tot[1];
  if (grid_reduce<1>(acc, red, tot) && threadIdx.x == 0) {
    const double rn = sqrt(tot[0]);
    st->rnorm = rn;
    if (!isfinite(rn)) {
      st->term = CFD_TERM_BREAKDOWN;
      st->done = 1;
    } else if (rn <= st->threshold) {
      st->term = CFD_TERM_CONVERGED;
      st->done = 1;
    } else if (st->omega == 0.0) {
      st->term = CFD_TERM_BREAKDOWN;
      st->done = 1;
    } else if (st->iter >= st->max_iter) {
      st->term = CFD_TERM_MAX_ITERATIONS;
      st->done = 1;
    }
  }
}

template <typename XT>
__global__ void __launch_bounds__(kThreads) k_axpy_state(int64_t n, XT* __restrict__ x, const XT* __restrict__ y,
                                                         const DevState* st) {
  pdl_enter();
  const XT a = (XT)st->alpha;
  GRID_STRIDE_U4(i, n, x[i] = x[i] + a * y[i];)
}

// ---- GMRES(m): restarted, right preconditioned (krylov.rs:150-221) -----------
// Arnoldi with classical Gram-Schmidt applied twice (CGS2): the j + 1
// projections of a step are dot products over the whole basis at once
// (k_mdot per-CTA partials, k_mdot_finish in fixed order), the subtraction one
// pass (k_gemv_sub); the Hessenberg column, the Givens rotations and the
// implicit residual live on the device (k_gmres_rot, one thread).
constexpr int kGmresGrid = 148 * 2;
constexpr int kDotTile = 8;

struct GmresDev {
  int m;            // restart width
  int* flags;       // [0] columns of the cycle, [1] cycle ended
  double* H;        // (m + 1) x m Hessenberg, column j at H + j (m + 1)
  double* cs;       // Givens cosines
  double* sn;       // Givens sines
  double* g;        // rotated right-hand side, m + 1
  double* y;        // least-squares solution, m
  double* h;        // second-pass projection coefficients, m + 1
  double* partials; // kGmresGrid x (m + 1)
};

// partials[cta (m+1) + k] = this CTA's share of V_k . w, k < nv.
template <typename XT>
__global__ void __launch_bounds__(kThreads) k_mdot(int64_t n, const XT* __restrict__ V, int64_t ldv, int nv,
                                                   const XT* __restrict__ w, int stride, double* partials,
                                                   const int* skip) {
  if (flag_set(skip)) return;
  for (int t0 = 0; t0 < nv; t0 += kDotTile) {
    double acc[kDotTile];
#pragma unroll
    for (int u = 0; u < kDotTile; ++u) acc[u] = 0.0;
    GRID_STRIDE(i, n) {
      const double wi = (double)w[i];
#pragma unroll
      for (int u = 0; u < kDotTile; ++u)
        if (t0 + u < nv) acc[u] += (double)V[(int64_t)(t0 + u) * ldv + i] * wi;
    }
#pragma unroll
    for (int u = 0; u < kDotTile; ++u) {
      const double b = block_sum(acc[u]);
      if (threadIdx.x == 0 && t0 + u < nv) partials[(size_t)blockIdx.x * stride + t0 + u] = b;
    }
  }
}

// out[k] = sum over CTAs of partials (one CTA per k, fixed order); mode 1: sqrt.
__global__ void __launch_bounds__(kThreads) k_mdot_finish(int grid, const double* __restrict__ partials, int stride,
                                                          double* out, int mode, const int* skip) {
  if (flag_set(skip)) return;
  const int k = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < grid; b += blockDim.x) s += partials[(size_t)b * stride + k];
  s = block_sum(s);
  if (threadIdx.x == 0) out[k] = mode == 1 ? sqrt(s) : s;
}

// w -= sum_k h_k V_k (k < nv), summed in k order in FP64.
template <typename XT>
__global__ void __launch_bounds__(kThreads) k_gemv_sub(int64_t n, const XT* __restrict__ V, int64_t ldv, int nv,
                                                       const double* __restrict__ h, XT* __restrict__ w,
                                                       const int* skip) {
  pdl_enter();
  if (flag_set(skip)) return;
  GRID_STRIDE(i, n) {
    double s = 0.0;
    for (int k = 0; k < nv; ++k) s += h[k] * (double)V[(int64_t)k * ldv + i];
    w[i] = (XT)((double)w[i] - s);
  }
}

// u = sum_k y_k V_k over the cycle's columns.
template <typename XT>
__global__ void __launch_bounds__(kThreads) k_gemv_cols(int64_t n, const XT* __restrict__ V, int64_t ldv,
                                                        const int* __restrict__ cols, const double* __restrict__ y,
                                                        XT* __restrict__ u, const int* skip) {
  pdl_enter();
  if (flag_set(skip)) return;
  const int nc = *cols;
  GRID_STRIDE(i, n) {
    double s = 0.0;
    for (int k = 0; k < nc; ++k) s += y[k] * (double)V[(int64_t)k * ldv + i];
    u[i] = (XT)s;
  }
}

// dst = src / *div (nothing when *div is 0: the Krylov space is exhausted).
template <typename XT>
__global__ void __launch_bounds__(kThreads) k_scale_div(int64_t n, const XT* src, XT* dst,
                                                        const double* __restrict__ div, const int* skip) {
  pdl_enter();
  if (flag_set(skip)) return;
  const double d = *div;
  if (d == 0.0) return;
  GRID_STRIDE(i, n) dst[i] = (XT)((double)src[i] / d);
}

template <typename XT>
__global__ void __launch_bounds__(kThreads) k_jacobi_apply(int64_t n, const XT* __restrict__ r,
                                                           const XT* __restrict__ jinv, XT* __restrict__ z,
                                                           const int* skip) {
  pdl_enter();
  if (flag_set(skip)) return;
  GRID_STRIDE_U4(i, n, z[i] = r[i] * jinv[i];)
}

template <typename XT>
__global__ void __launch_bounds__(kThreads) k_add(int64_t n, XT* __restrict__ x, const XT* __restrict__ z,
                                                  const int* skip) {
  pdl_enter();
  if (flag_set(skip)) return;
  GRID_STRIDE_U4(i, n, x[i] = x[i] + z[i];)
}

// Cycle start: no columns yet, the cycle open unless the solve is done;
// g = (beta, 0, ..., 0) once beta lands in g[0].
__global__ void k_gmres_begin(GmresDev G, const DevState* st) {
  G.flags[0] = 0;
  G.flags[1] = st->done ? 1 : 0;
  for (int k = 1; k <= G.m; ++k) G.g[k] = 0.0;
}

// Step j: second projection pass added to the column, earlier rotations
// applied, the new rotation formed, the implicit residual |g_{j+1}| tested.
__global__ void k_gmres_rot(GmresDev G, int j, DevState* st) {
  if (G.flags[1]) return;
  const int m = G.m;
  double* h = G.H + (size_t)j * (m + 1);
  for (int q = 0; q <= j; ++q) h[q] += G.h[q];
  const double hn = h[j + 1];
  for (int q = 0; q < j; ++q) {
    const double t = G.cs[q] * h[q] + G.sn[q] * h[q + 1];
    h[q + 1] = -G.sn[q] * h[q] + G.cs[q] * h[q + 1];
    h[q] = t;
  }
  const double d = hypot(h[j], h[j + 1]);
  G.cs[j] = d > 0.0 ? h[j] / d : 1.0;
  G.sn[j] = d > 0.0 ? h[j + 1] / d : 0.0;
  h[j] = d;
  h[j + 1] = 0.0;
  G.g[j + 1] = -G.sn[j] * G.g[j];
  G.g[j] = G.cs[j] * G.g[j];
  st->iter += 1;
  const double res = fabs(G.g[j + 1]);
  st->rnorm = res;
  G.flags[0] = j + 1;
  if (!isfinite(res)) {
    G.flags[1] = 1;
    st->term = CFD_TERM_BREAKDOWN;
    st->done = 1;
  } else if (res <= st->threshold || st->iter >= st->max_iter || hn == 0.0 || j + 1 == m) {
    G.flags[1] = 1;
  }
}

// y = R^-1 g on the cycle's columns (back substitution).
__global__ void k_gmres_lsq(GmresDev G, const int* skip) {
  if (flag_set(skip)) return;
  const int m = G.m, cols = G.flags[0];
  for (int q = cols - 1; q >= 0; --q) {
    double s = G.g[q];
    for (int l = q + 1; l < cols; ++l) s -= G.H[(size_t)l * (m + 1) + q] * G.y[l];
    const double dqq = G.H[(size_t)q * (m + 1) + q];
    G.y[q] = dqq != 0.0 ? s / dqq : 0.0;
  }
}

// After x += M^-1 V y and r = b - A x (rnorm = ||r||): the true residual decides.
__global__ void k_gmres_check(DevState* st) {
  if (st->done) return;
  const double rn = st->rnorm;
  if (!isfinite(rn)) {
    st->term = CFD_TERM_BREAKDOWN;
    st->done = 1;
  } else if (rn <= st->threshold) {
    st->term = CFD_TERM_CONVERGED;
    st->done = 1;
  } else if (st->iter >= st->max_iter) {
    st->term = CFD_TERM_MAX_ITERATIONS;
    st->done = 1;
  }
}

// ---- refinement ----------------------------------------------------------------
// Inner right-hand side r32 = r64 / ||r64||, inner iterate zeroed; sets up the
// inner state (threshold = inner_tol * ||r32||).
__global__ void __launch_bounds__(kThreads) k_refine_start(int64_t n, const double* __restrict__ r64,
                                                           float* __restrict__ r32, float* __restrict__ x32,
                                                           const DevState* outer, DevState* inner, Red red) {
  pdl_enter();
  const double sc = 1.0 / outer->rnorm;
  double acc[1] = {0.0};
  GRID_STRIDE_U4(i, n, {
    const float ri = (float)(r64[i] * sc);
    r32[i] = ri;
    x32[i] = 0.0f;
    acc[0] += (double)ri * (double)ri;
  })
  double tot[1];
  if (grid_reduce<1>(acc, red, tot) && threadIdx.x == 0) {
    const double rn = sqrt(tot[0]);
    inner->rnorm0 = rn;
    inner->rnorm = rn;
    inner->rr = tot[0];
    inner->threshold = fmax(inner->tol_abs, inner->tol_rel * rn);
    inner->iter = 0;
    inner->done = 0;
    inner->spare0 = 0.0;
    inner->term = CFD_TERM_MAX_ITERATIONS;
    inner->rho = inner->alpha = inner->omega = 1.0;
    inner->beta = 0.0;
    if (!(rn > inner->threshold)) {
      inner->term = CFD_TERM_INITIAL_RESIDUAL;
      inner->done = 1;
    }
  }
}

// x64 += ||r64|| * d32 (the FP64 solution accumulation).
__global__ void __launch_bounds__(kThreads) k_refine_accumulate(int64_t n, double* __restrict__ x64,
                                                                const float* __restrict__ d32, const DevState* outer) {
  pdl_enter();
  const double sc = outer->rnorm;
  GRID_STRIDE_U4(i, n, x64[i] += sc * (double)d32[i];)
}

}  // namespace

// ---------------------------------------------------------------------------
// Launch helpers.

struct Launcher {
  cfd_context* ctx;
  cudaStream_t s;
  Red red() const { return Red{ctx->partials, ctx->counter}; }
  // Every SpMV runs the persistent bulk-copy pipeline, one CTA per row block
  // up to num_sms * (resident CTAs per SM).
  template <typename VT, typename XT, bool OFF, class Epi, bool CODES>
  cfd_status spmv_launch(const DevMat& m, const XT* x, Epi epi) {
    auto kern = k_spmv_pipe<VT, XT, OFF, Epi, CODES>;
    constexpr int smem = PipeLayout<VT, CODES>::kSmemBytes;
    static int occ[kLaunchCacheDevices] = {};
    if (ctx->device >= kLaunchCacheDevices) {
      set_error("device ordinal %d beyond %d", ctx->device, kLaunchCacheDevices);
      return CFD_ERR_CUDA;
    }
    if (occ[ctx->device] <= 0) {
      CFD_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      int o = 0;
      CFD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, kPipeThreads, smem));
      occ[ctx->device] = std::max(1, o);
    }
    const int grid = std::min(m.nblk, ctx->num_sms * occ[ctx->device]);
    launch(kern, grid, kPipeThreads, smem, mat_view<VT>(m), m.nblk, x, epi, ctx->err);
    return CFD_OK;
  }
  // x-staged pipeline: one CTA per SM.
  template <typename VT, bool OFF, class Epi>
  cfd_status spmv_xs_launch(const DevMat& m, const VT* x, Epi epi) {
    auto kern = k_spmv_xs<VT, OFF, Epi>;
    constexpr int smem = XsLayout<VT>::kSmemBytes;
    static bool attr[kLaunchCacheDevices] = {};
    if (ctx->device >= kLaunchCacheDevices) {
      set_error("device ordinal %d beyond %d", ctx->device, kLaunchCacheDevices);
      return CFD_ERR_CUDA;
    }
    if (!attr[ctx->device]) {
      CFD_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      attr[ctx->device] = true;
    }
    const int grid = std::min(m.nblk, ctx->num_sms);
    const XsView xv{m.xdesc, m.xwin, m.rec, (int)m.ncols};
    launch(kern, grid, kXsThreads, smem, mat_view<VT>(m), xv, m.nblk, x, epi, ctx->err);
    ctx->stats.xs_launches++;
    return CFD_OK;
  }
  // Every SpMV runs a persistent bulk-copy pipeline: the split one (values,
  // columns or codes, row offsets and dictionary copied separately; any
  // matrix), the record one (values plus one block record; fully coded
  // matrices) or the x-staged one (x windows staged with the block). All three
  // sum each row in the same order (fused dot products add per-CTA partials
  // over each pipeline's own grid), so the choice changes speed, not the row
  // results
  // (spmv_path: by default FP32 takes the record pipeline, whose x gathers hit
  // L2, and FP64 the x-staged one for one-thread rows, whose x no longer fits
  // L2 at large sizes; CFD_PATH_TIMED times the eligible ones once).
  // Sliced pipeline (FP32 values only): one warp per 32-row slice. The
  // slot-major values are gathered from v32 first when v32 changed since.
  template <typename XT, bool OFF, class Epi>
  cfd_status sl_launch(const DevMat& m, const XT* x, Epi epi) {
    if (m.sl_stale) {
      const int g = (int)std::max<int64_t>(1, std::min<int64_t>((m.sl_slots + kThreads - 1) / kThreads,
                                                                (int64_t)ctx->num_sms * 8));
      k_sl_gather<<<g, kThreads, 0, s>>>(m.sl_slots, m.sl_src, m.v32, m.sl_v32);
      CFD_TRY(check());
      ctx->stats.launches++;
      m.sl_stale = false;
    }
    auto kern = k_spmv_sl<XT, OFF, Epi>;
    static int occ[kLaunchCacheDevices] = {};
    if (ctx->device >= kLaunchCacheDevices) {
      set_error("device ordinal %d beyond %d", ctx->device, kLaunchCacheDevices);
      return CFD_ERR_CUDA;
    }
    if (occ[ctx->device] <= 0) {
      int o = 0;
      CFD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, kThreads, 0));
      occ[ctx->device] = std::max(1, o);
    }
    const int64_t chunks = (m.sl_slices + kSlChunkSlices - 1) / kSlChunkSlices;
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>({chunks, (int64_t)ctx->num_sms * occ[ctx->device], (int64_t)ctx->partial_capacity}));
    const SlView sv{m.sl_off, m.sl_code, m.sl_dict, m.sl_doff, m.sl_v32, (unsigned long long)m.base_mult,
                    (int)m.sl_slices, (int)m.nrows};
    launch(kern, grid, kThreads, 0, sv, x, epi);
    return CFD_OK;
  }
  // Diagonal pipeline: refills the diagonal-major values first when the CSR
  // values changed since.
  template <typename VT>
  DiaView<VT> dia_view(const DevMat& m) const {
    DiaView<VT> D{};
    if constexpr (sizeof(VT) == 8)
      D.val = m.dia64;
    else
      D.val = m.dia32;
    D.ld = m.dia_ld;
    D.mask = m.dia_mask;
    D.nrows = (int)m.nrows;
    D.n = m.dia_n;
    D.main = m.dia_main;
    for (int d = 0; d < kDiaMax; ++d) D.off[d] = m.dia_off[d];
    return D;
  }
  cfd_status dia_refresh(const DevMat& m) {
    if (!m.dia_stale) return CFD_OK;
    const int g = (int)std::max<int64_t>(1, std::min<int64_t>((m.nrows + kThreads - 1) / kThreads,
                                                              (int64_t)ctx->num_sms * 8));
    if (m.dia64) {
      k_dia_fill<double><<<g, kThreads, 0, s>>>(dia_view<double>(m), m.rp, m.col, m.v64, m.dia64);
      ctx->stats.launches++;
    }
    if (m.dia32 && m.v32) {
      k_dia_fill<float><<<g, kThreads, 0, s>>>(dia_view<float>(m), m.rp, m.col, m.v32, m.dia32);
      ctx->stats.launches++;
    }
    CFD_TRY(check());
    m.dia_stale = false;
    return CFD_OK;
  }
  // Rows per thread of the streaming diagonal kernel: FP32 two (8-byte value
  // loads, half the scalar x loads of four rows per thread), FP64 two.
  template <typename VT>
  static constexpr int kDiaGenRows = 2;
  template <typename VT, bool OFF, class Epi>
  cfd_status dia_launch(const DevMat& m, const VT* x, Epi epi) {
    return dia_launch_xs<VT, OFF, Epi>(m, DiaXPlain<VT>{x}, ((uintptr_t)x & 15) == 0, epi);
  }
  // xvec: every array the x source reads (and stores) is 16-byte aligned.
  template <typename VT, bool OFF, class Epi, class XS>
  cfd_status dia_launch_xs(const DevMat& m, XS xs, bool xvec, Epi epi) {
    constexpr int V = DiaVec<VT>::V, VG = kDiaGenRows<VT>;
    if (m.tpr == 1 && m.dia_n == 7)
      return dia_launch_k<VT, Epi, V>(m, k_spmv_dia<VT, OFF, Epi, 7, XS>, xs, xvec, epi);
    if (m.tpr == 1 && m.dia_n == 5)
      return dia_launch_k<VT, Epi, V>(m, k_spmv_dia<VT, OFF, Epi, 5, XS>, xs, xvec, epi);
    if (m.tpr == 1) return dia_launch_k<VT, Epi, VG>(m, k_spmv_dia_gen<VT, OFF, Epi, 1, XS, VG>, xs, xvec, epi);
    return dia_launch_k<VT, Epi, VG>(m, k_spmv_dia_gen<VT, OFF, Epi, 2, XS, VG>, xs, xvec, epi);
  }
  // One launch of a diagonal kernel of V rows per thread and span (its
  // occupancy looked up once per device).
  template <typename VT, class Epi, int V, class XS>
  cfd_status dia_launch_k(const DevMat& m, void (*kern)(DiaView<VT>, XS, Epi), XS xs, bool xvec, Epi epi) {
    CFD_TRY(dia_refresh(m));
    static std::mutex occ_mu;
    static std::map<const void*, int> occ_by_kernel[kLaunchCacheDevices];
    if (ctx->device >= kLaunchCacheDevices) {
      set_error("device ordinal %d beyond %d", ctx->device, kLaunchCacheDevices);
      return CFD_ERR_CUDA;
    }
    int occ = 0;
    {
      std::lock_guard<std::mutex> g(occ_mu);
      int& o = occ_by_kernel[ctx->device][(const void*)kern];
      if (o <= 0) {
        CFD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, kThreads, 0));
        o = std::max(1, o);
      }
      occ = o;
    }
    const int64_t span = (int64_t)kThreads * V;
    const int64_t spans = (m.nrows + span - 1) / span;
    // at most one reduction slot per CTA (the context's partials)
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>({spans, (int64_t)ctx->num_sms * occ, (int64_t)ctx->partial_capacity}));
    DiaView<VT> D = dia_view<VT>(m);
    D.xvec = xvec ? 1 : 0;
    launch(kern, grid, kThreads, 0, D, xs, epi);
    return CFD_OK;
  }
  // The diagonal pipeline runs when the values of this precision are there
  // (the FP32 diagonal copy exists once the FP32 values do).
  template <typename VT>
  static bool dia_ready(const DevMat& m) {
    return m.dia && (sizeof(VT) == 8 ? m.dia64 != nullptr : (m.dia32 != nullptr && m.v32 != nullptr));
  }
  static constexpr int kPathTimed = -2, kPathSplit = 0, kPathRecord = 1, kPathXs = 2, kPathSliced = 3,
                       kPathDiag = 4;
  template <typename VT, typename XT, bool OFF, class Epi>
  cfd_status spmv(const DevMat& m, const XT* x, Epi epi) {
    if (m.nrows == 0) return CFD_OK;
    epi.red = red();
    const int p = sizeof(VT) == 4 ? 0 : 1;
    if (m.path[p] == kPathTimed) CFD_TRY(tune<VT>(m));
    int path = spmv_path(m, p);
    if (path == kPathXs && ((uintptr_t)x & 15) != 0) path = m.all_compressed ? kPathRecord : kPathSplit;
    if constexpr (std::is_same<VT, float>::value) {
      if (path == kPathSliced && m.v32) {
        CFD_TRY((sl_launch<XT, OFF, Epi>(m, x, epi)));
        return finish_spmv<VT, XT>(m);
      }
      if (path == kPathSliced) path = m.all_compressed ? kPathRecord : kPathSplit;
    }
    if constexpr (std::is_same<VT, XT>::value) {
      if (path == kPathDiag && dia_ready<VT>(m)) {
        CFD_TRY((dia_launch<VT, OFF, Epi>(m, x, epi)));
        return finish_spmv<VT, XT>(m);
      }
    }
    if (path == kPathDiag) path = m.all_compressed ? kPathRecord : kPathSplit;
    if constexpr (std::is_same<VT, XT>::value) {
      if (path == kPathXs) {
        CFD_TRY((spmv_xs_launch<VT, OFF, Epi>(m, x, epi)));
        return finish_spmv<VT, XT>(m);
      }
    }
    if (path == kPathRecord)
      CFD_TRY((spmv_launch<VT, XT, OFF, Epi, true>(m, x, epi)));
    else
      CFD_TRY((spmv_launch<VT, XT, OFF, Epi, false>(m, x, epi)));
    return finish_spmv<VT, XT>(m);
  }
  // Times y = A x on each eligible pipeline (two warm-up and five timed
  // launches on scratch vectors) and records the fastest in m.path.
  template <typename VT>
  cfd_status tune(const DevMat& m) {
    const int p = sizeof(VT) == 4 ? 0 : 1;
    if (!m.all_compressed && !dia_ready<VT>(m)) {
      m.path[p] = kPathSplit;
      return CFD_OK;
    }
    VT *xs = nullptr, *ys = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const KernelStats keep = ctx->stats;
    cfd_status st = CFD_OK;
    float best_ms = 0.0f;
    int best = kPathSplit;
    auto fail = [&](cudaError_t e) {
      set_error("SpMV pipeline timing: %s", cudaGetErrorString(e));
      st = CFD_ERR_CUDA;
    };
    cudaError_t e = cudaMalloc((void**)&xs, (size_t)(m.ncols + 16) * sizeof(VT));
    if (e == cudaSuccess) e = cudaMalloc((void**)&ys, (size_t)(m.nrows + 16) * sizeof(VT));
    if (e == cudaSuccess) e = cudaMemsetAsync(xs, 0, (size_t)m.ncols * sizeof(VT), s);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e != cudaSuccess) fail(e);
    const bool sl_ok = std::is_same<VT, float>::value && m.sl && m.v32;
    for (int path = kPathSplit; st == CFD_OK && path <= kPathDiag; ++path) {
      if ((path == kPathRecord && !m.all_compressed) || (path == kPathXs && !m.xs) || (path == kPathSliced && !sl_ok) ||
          (path == kPathDiag && !dia_ready<VT>(m)))
        continue;
      const EpiStore<VT> epi{ys, nullptr, red()};
      auto run = [&]() -> cfd_status {
        if (path == kPathDiag) return dia_launch<VT, false, EpiStore<VT>>(m, xs, epi);
        if constexpr (std::is_same<VT, float>::value) {
          if (path == kPathSliced) return sl_launch<VT, false, EpiStore<VT>>(m, xs, epi);
        }
        if (path == kPathXs) return spmv_xs_launch<VT, false, EpiStore<VT>>(m, xs, epi);
        if (path == kPathRecord) return spmv_launch<VT, VT, false, EpiStore<VT>, true>(m, xs, epi);
        return spmv_launch<VT, VT, false, EpiStore<VT>, false>(m, xs, epi);
      };
      for (int i = 0; i < 2 && st == CFD_OK; ++i) st = run();
      if (st == CFD_OK) st = check();
      if (st != CFD_OK) break;
      cudaEventRecord(e0, s);
      for (int i = 0; i < 5 && st == CFD_OK; ++i) st = run();
      cudaEventRecord(e1, s);
      if (st == CFD_OK) st = check();
      e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) {
        fail(e);
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (path == kPathSplit || ms < best_ms) {
        best_ms = ms;
        best = path;
      }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(xs);
    cudaFree(ys);
    ctx->stats = keep;
    if (st != CFD_OK) return st;
    m.path[p] = (int8_t)best;
    return check_device_flag(ctx);
  }
  template <typename VT, typename XT>
  cfd_status finish_spmv(const DevMat& m) {
    ctx->stats.launches++;
    ctx->stats.spmv_launches++;
    ctx->stats.spmv_bytes += (double)m.nnz * (sizeof(VT) + 4) + 4.0 * (m.nrows + 1) +
                             (double)sizeof(XT) * (m.nrows + m.ncols);
    return check();
  }
  cfd_status check() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error("kernel launch failed: %s", cudaGetErrorString(e));
      return CFD_ERR_CUDA;
    }
    return CFD_OK;
  }
  template <typename... KArgs, typename... Args>
  cfd_status vec(int64_t n, void (*kernel)(KArgs...), Args... args) {
    launch(kernel, vec_grid(n), kThreads, 0, n, args...);
    ctx->stats.launches++;
    return check();
  }
  // Launch with programmatic stream serialization (the kernel begins with
  // pdl_enter, which waits for the stream's preceding grid on the device).
  template <typename... KArgs, typename... Args>
  void launch(void (*kernel)(KArgs...), int grid, int block, size_t smem, Args... args) const {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
  }
};

// ---------------------------------------------------------------------------
// V-cycle, AlgebraicMultigrid::v_cycle (amg.rs:423-503) from a zero iterate
// (amg.rs:464-466, :553-554). `out` receives the level result; at level 0 with
// dot != 0 the last kernel also forms b.out (PCG rho).

template <typename XT>
LevelVecs<XT>& vecs(DevLevel& L);
template <>
LevelVecs<double>& vecs<double>(DevLevel& L) {
  return L.v64;
}
template <>
LevelVecs<float>& vecs<float>(DevLevel& L) {
  return L.v32;
}
template <typename XT>
const XT* diag_of(const DevLevel& L);
template <>
const double* diag_of<double>(const DevLevel& L) {
  return L.d64;
}
template <>
const float* diag_of<float>(const DevLevel& L) {
  return L.d32;
}

template <typename XT>
static cfd_status jacobi_sweep(Launcher& lc, const DevLevel& L, const XT* xo, XT* xn, const XT* b, XT omega,
                               int dot, DevState* st, const int* done) {
  if constexpr (std::is_same<XT, float>::value) {
    // FP32 (inner) sweeps: the residual form over the full row (EpiJacobiR)
    const float* d = diag_of<float>(L);
    if (dot == 1) return lc.spmv<float, float, false>(L.A, xo, EpiJacobiR<float, 1>{xn, xo, b, d, omega, st, done, {}});
    if (dot == 2) return lc.spmv<float, float, false>(L.A, xo, EpiJacobiR<float, 2>{xn, xo, b, d, omega, st, done, {}});
    return lc.spmv<float, float, false>(L.A, xo, EpiJacobiR<float, 0>{xn, xo, b, d, omega, st, done, {}});
  } else {
    const XT* d = diag_of<XT>(L);
    if (dot == 1) return lc.spmv<XT, XT, true>(L.A, xo, EpiJacobi<XT, 1>{xn, xo, b, d, omega, st, done, {}});
    if (dot == 2) return lc.spmv<XT, XT, true>(L.A, xo, EpiJacobi<XT, 2>{xn, xo, b, d, omega, st, done, {}});
    return lc.spmv<XT, XT, true>(L.A, xo, EpiJacobi<XT, 0>{xn, xo, b, d, omega, st, done, {}});
  }
}

// Whether level l's first pre-smoothing sweep can be written by the kernel
// that produces its right-hand side (into the level's vecs().xa).
template <typename XT>
static bool smooth0_fusable(const cfd_amg* amg, size_t l) {
  return l + 1 < amg->dev.size() && amg->cfg.pre_smooth >= 1;
}

// x0_ready: the producer of b already wrote the first pre-smoothing sweep
// (smooth0_value) into this level's vecs().xa.
template <typename XT>
static cfd_status vcycle(Launcher& lc, cfd_amg* amg, size_t l, const XT* b, XT* out, int dot, DevState* st,
                         const int* done, bool x0_ready = false) {
  DevLevel& L = amg->dev[l];
  LevelVecs<XT>& V = vecs<XT>(L);
  const int64_t n = L.A.nrows;
  const cfd_amg_config& c = amg->cfg;
  const XT omega = (XT)c.relaxation;
  const bool coarsest = (l + 1 == amg->dev.size());
  if (coarsest) {
    if (c.coarse_solve == CFD_COARSE_DENSE && amg->coarse_inv) {
      if (sizeof(XT) == 4 && amg->coarse_inv32)
        lc.launch(k_dense_gemv<XT, float>, (int)((n + 7) / 8), kThreads, 0, (int)n,
                  (const float*)amg->coarse_inv32, b, out, done);
      else
        lc.launch(k_dense_gemv<XT, double>, (int)((n + 7) / 8), kThreads, 0, (int)n,
                  (const double*)amg->coarse_inv, b, out, done);
      lc.ctx->stats.launches++;
      CFD_TRY(lc.check());
      if (dot) CFD_TRY(lc.vec(n, k_rz<XT>, b, (const XT*)out, st, dot, lc.red()));
      return CFD_OK;
    }
    const int sweeps = std::max(0, (int)c.coarse_sweeps);
    if (sweeps == 0) {
      CFD_TRY(lc.vec(n, k_fill<XT>, out, XT(0), done));
      if (dot) CFD_TRY(lc.vec(n, k_rz<XT>, b, (const XT*)out, st, dot, lc.red()));
      return CFD_OK;
    }
    XT* cur = V.xa;
    XT* nxt = V.xb;
    CFD_TRY(lc.vec(n, k_smooth0<XT>, b, diag_of<XT>(L), omega, sweeps == 1 ? out : cur, done));
    if (sweeps == 1) {
      if (dot) CFD_TRY(lc.vec(n, k_rz<XT>, b, (const XT*)out, st, dot, lc.red()));
      return CFD_OK;
    }
    for (int s = 1; s < sweeps; ++s) {
      XT* dst = (s == sweeps - 1) ? out : nxt;
      CFD_TRY(jacobi_sweep<XT>(lc, L, cur, dst, b, omega, s == sweeps - 1 ? dot : 0, st, done));
      std::swap(cur, nxt);
    }
    return CFD_OK;
  }
  // 1. pre-smoothing from x = 0
  XT* x = V.xa;
  XT* y = V.xb;
  if (c.pre_smooth >= 1) {
    if (!x0_ready) CFD_TRY(lc.vec(n, k_smooth0<XT>, b, diag_of<XT>(L), omega, x, done));
    for (int s = 1; s < c.pre_smooth; ++s) {
      CFD_TRY(jacobi_sweep<XT>(lc, L, x, y, b, omega, 0, st, done));
      std::swap(x, y);
    }
  } else {
    CFD_TRY(lc.vec(n, k_fill<XT>, x, XT(0), done));
  }
  // 2. residual r = b - A x
  CFD_TRY(lc.spmv<XT, XT, false>(L.A, x, EpiResidual<XT, 0>{V.r, b, nullptr, done, {}}));
  // 3. restriction to the next level's right-hand side
  DevLevel& Lc = amg->dev[l + 1];
  LevelVecs<XT>& Vc = vecs<XT>(Lc);
  const bool fuse = smooth0_fusable<XT>(amg, l + 1);
  if (fuse)
    CFD_TRY(lc.spmv<XT, XT, false>(L.R, V.r,
                                   EpiStoreSmooth<XT>{Vc.b, Vc.xa, diag_of<XT>(Lc), omega, done, {}}));
  else
    CFD_TRY(lc.spmv<XT, XT, false>(L.R, V.r, EpiStore<XT>{Vc.b, done, {}}));
  // 4. coarse solve from zero
  CFD_TRY(vcycle<XT>(lc, amg, l + 1, Vc.b, Vc.e, 0, st, done, fuse));
  // 5-6. x += P e_c
  CFD_TRY(lc.spmv<XT, XT, false>(L.P, Vc.e, EpiAddTo<XT>{x, x, done, {}}));
  // 7. post-smoothing
  if (c.post_smooth <= 0) {
    CFD_TRY(lc.vec(n, k_copy<XT>, (const XT*)x, out, done));
    if (dot) CFD_TRY(lc.vec(n, k_rz<XT>, b, (const XT*)out, st, dot, lc.red()));
    return CFD_OK;
  }
  for (int s = 0; s < c.post_smooth; ++s) {
    const bool last = (s == c.post_smooth - 1);
    XT* dst = last ? out : y;
    CFD_TRY(jacobi_sweep<XT>(lc, L, x, dst, b, omega, last ? dot : 0, st, done));
    if (!last) std::swap(x, y);
  }
  return CFD_OK;
}

// ---------------------------------------------------------------------------
// Krylov drivers. The recurrences run on device-resident scalars; the host
// only polls the state to stop launching, choosing how many iterations to
// enqueue from the observed convergence rate.

// Stream-ordered workspace (the default memory pool keeps freed blocks for reuse).
template <typename XT>
struct Alloc {
  cudaStream_t s;
  std::vector<void*> ptrs;
  XT* get(int64_t n) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, (size_t)std::max<int64_t>(n, 1) * sizeof(XT), s) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return (XT*)p;
  }
  ~Alloc() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
  }
};

struct Poller {
  cfd_context* ctx;
  DevState* dev;
  DevState* host;  // pinned slot
  int64_t last_iter = 0;
  double last_rn = 0.0;
  int chunk = 1;
  int fixed = 0;
  cfd_status poll() {
    CFD_TRY_CUDA(cudaMemcpyAsync(host, dev, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    CFD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFD_OK;
  }
  void next_chunk() {
    if (fixed > 0) {
      chunk = fixed;
      return;
    }
    const DevState& h = *host;
    int c = std::min(2 * chunk, 64);
    if (last_rn == 0.0 && h.iter >= 3 && h.rnorm0 > 0.0) {
      // first look after a predicted chunk: measure from the start
      last_iter = 0;
      last_rn = h.rnorm0;
    }
    if (h.iter > last_iter && last_rn > 0.0 && h.rnorm > 0.0 && h.rnorm < last_rn) {
      const double rate = std::pow(h.rnorm / last_rn, 1.0 / (double)(h.iter - last_iter));
      if (rate < 1.0 && rate > 0.0) {
        const double rem = std::log(h.threshold / h.rnorm) / std::log(rate);
        c = (int)std::ceil(std::max(1.0, std::min(64.0, rem)));
      }
    }
    last_iter = h.iter;
    last_rn = h.rnorm;
    chunk = std::max(1, c);
  }
};

template <typename XT>
struct KrylovBufs {
  XT *x, *b, *r, *p, *q, *z, *rh, *v, *s, *sh, *t;
};

template <typename XT>
static const XT* jinv_of(cfd_csr* a);
template <>
const double* jinv_of<double>(cfd_csr* a) {
  return a->jinv64;
}
template <>
const float* jinv_of<float>(cfd_csr* a) {
  return a->jinv32;
}

// Preconditioned CG. Expects the state's start (rnorm0, threshold, done, iter)
// already set and r holding the initial residual.
template <typename XT, int PRE>
static cfd_status pcg_loop(Launcher& lc, cfd_csr* a, cfd_amg* amg, KrylovBufs<XT>& B, DevState* st, Poller& pl) {
  const int64_t n = a->dev.nrows;
  const XT* jinv = jinv_of<XT>(a);
  const int* done = &st->done;
  if (PRE == kPreAmg) CFD_TRY(vcycle<XT>(lc, amg, 0, B.r, B.z, 0, st, done));
  CFD_TRY(lc.vec(n, k_pcg_init<XT, PRE>, B.p, (const XT*)B.r, (const XT*)B.z, jinv, st, lc.red()));
  const int64_t max_launch = std::max<int64_t>(1, st ? (int64_t)1 << 40 : 1);
  (void)max_launch;
  int64_t launched = 0;
  // the V-cycle's first sweep on the fine level comes from k_cg_update
  XT* x0 = nullptr;
  const XT* d0 = nullptr;
  XT omega = XT(0);
  if (PRE == kPreAmg && smooth0_fusable<XT>(amg, 0)) {
    x0 = vecs<XT>(amg->dev[0]).xa;
    d0 = diag_of<XT>(amg->dev[0]);
    omega = (XT)amg->cfg.relaxation;
  }
  for (;;) {
    for (int k = 0; k < pl.chunk; ++k) {
      CFD_TRY(lc.spmv<XT, XT, false>(a->dev, B.p, EpiCgDot<XT>{B.q, B.p, st, {}}));
      CFD_TRY(lc.vec(n, k_cg_update<XT, PRE>, B.x, (const XT*)B.p, B.r, (const XT*)B.q, jinv, st, lc.red(), x0,
                     d0, omega));
      if (PRE == kPreAmg) CFD_TRY(vcycle<XT>(lc, amg, 0, B.r, B.z, 2, st, done, x0 != nullptr));
      CFD_TRY(lc.vec(n, k_p_update<XT, PRE>, B.p, (const XT*)B.r, (const XT*)B.z, jinv, (const DevState*)st));
      ++launched;
    }
    CFD_TRY(pl.poll());
    if (pl.host->done) break;
    if (launched > pl.host->max_iter + 64) {
      set_error("PCG did not terminate within its iteration budget");
      return CFD_ERR_TIMEOUT;
    }
    pl.next_chunk();
  }
  return CFD_OK;
}

template <typename XT, int PRE>
static cfd_status bicgstab_loop(Launcher& lc, cfd_csr* a, cfd_amg* amg, KrylovBufs<XT>& B, DevState* st,
                                Poller& pl) {
  const int64_t n = a->dev.nrows;
  const XT* jinv = jinv_of<XT>(a);
  const int* done = &st->done;
  CFD_TRY(lc.vec(n, k_copy<XT>, (const XT*)B.r, B.rh, (const int*)nullptr));
  int64_t launched = 0;
  bool first = true;
  for (;;) {
    for (int k = 0; k < pl.chunk; ++k) {
      CFD_TRY(lc.vec(n, k_bicg_rho<XT>, (const XT*)B.rh, (const XT*)B.r, st, lc.red()));
      CFD_TRY(lc.vec(n, k_bicg_p<XT, PRE>, B.p, B.z, (const XT*)B.r, (const XT*)B.v, jinv, (const DevState*)st,
                     first ? 1 : 0));
      if (PRE == kPreAmg) CFD_TRY(vcycle<XT>(lc, amg, 0, B.p, B.z, 0, st, done));
      CFD_TRY(lc.spmv<XT, XT, false>(a->dev, B.z, EpiBicgV<XT>{B.v, B.rh, st, {}}));
      CFD_TRY(lc.vec(n, k_bicg_s<XT, PRE>, B.s, B.sh, (const XT*)B.r, (const XT*)B.v, jinv, st, lc.red()));
      if (PRE == kPreAmg) CFD_TRY(vcycle<XT>(lc, amg, 0, B.s, B.sh, 0, st, done));
      CFD_TRY(lc.spmv<XT, XT, false>(a->dev, B.sh, EpiBicgT<XT>{B.t, B.s, st, {}}));
      CFD_TRY(lc.vec(n, k_bicg_x<XT>, B.x, B.r, (const XT*)B.z, (const XT*)B.sh, (const XT*)B.s, (const XT*)B.t, st,
                     lc.red()));
      first = false;
      ++launched;
    }
    CFD_TRY(pl.poll());
    if (pl.host->done) break;
    if (launched > pl.host->max_iter + 64) {
      set_error("BiCGSTAB did not terminate within its iteration budget");
      return CFD_ERR_TIMEOUT;
    }
    pl.next_chunk();
  }
  if (pl.host->spare0 != 0.0) {
    // Converged on ||s||: x += alpha p_hat (the Krylov loop stopped before k_bicg_x).
    CFD_TRY(lc.vec(n, k_axpy_state<XT>, B.x, (const XT*)B.z, (const DevState*)st));
  }
  return CFD_OK;
}

// Restart width for a requested restart: RestartWidth::covering (krylov.rs:96-120).
int gmres_width(int64_t requested) {
  int w = 8;
  while (w < 256 && w < requested) w *= 2;
  return w;
}

// Restarted GMRES(m) with right preconditioning. Expects the state's start
// (rnorm0, threshold, done, iter) set, r = b - A x and b the right-hand side.
// One host poll per restart cycle; the steps of a cycle after it ended are
// launched but return at once.
template <typename XT, int PRE>
static cfd_status gmres_loop(Launcher& lc, cfd_csr* a, cfd_amg* amg, KrylovBufs<XT>& B, DevState* st, Poller& pl,
                             int64_t restart) {
  const int64_t n = a->dev.nrows;
  const int m = gmres_width(restart);
  const XT* jinv = jinv_of<XT>(a);
  Alloc<XT> ax{lc.s, {}};
  Alloc<double> ad{lc.s, {}};
  Alloc<int> ai{lc.s, {}};
  XT* V = ax.get((int64_t)(m + 1) * n);
  GmresDev G{m, ai.get(4), ad.get((int64_t)(m + 1) * m), ad.get(m), ad.get(m), ad.get(m + 1), ad.get(m),
             ad.get(m + 1), ad.get((int64_t)kGmresGrid * (m + 1))};
  if (!V || !G.flags || !G.H || !G.cs || !G.sn || !G.g || !G.y || !G.h || !G.partials) {
    set_error("GMRES workspace allocation failed (%lld unknowns, restart %d)", (long long)n, m);
    return CFD_ERR_ALLOC;
  }
  CFD_TRY_CUDA(cudaMemsetAsync(G.H, 0, sizeof(double) * (m + 1) * m, lc.s));
  const int stride = m + 1;
  const int* done = &st->done;
  const int* ended = G.flags + 1;
  auto dots = [&](const XT* Vb, int nv, const XT* w, double* out, int mode, const int* skip) -> cfd_status {
    k_mdot<XT><<<kGmresGrid, kThreads, 0, lc.s>>>(n, Vb, n, nv, w, stride, G.partials, skip);
    k_mdot_finish<<<nv, kThreads, 0, lc.s>>>(kGmresGrid, G.partials, stride, out, mode, skip);
    lc.ctx->stats.launches += 2;
    return lc.check();
  };
  auto precond = [&](const XT* v, XT* z, const int* skip) -> const XT* {
    if (PRE == kPreAmg) {
      if (vcycle<XT>(lc, amg, 0, v, z, 0, st, skip) != CFD_OK) return nullptr;
      return z;
    }
    if (PRE == kPreJacobi) {
      if (lc.vec(n, k_jacobi_apply<XT>, v, jinv, z, skip) != CFD_OK) return nullptr;
      return z;
    }
    if (PRE == kPreSimple) {
      if (simple_apply_device<XT>(a, v, z, skip, lc.s) != CFD_OK) return nullptr;
      return z;
    }
    if (PRE == kPreBlockDiag) {
      if (block_diagonal_apply_device<XT>(a, v, z, skip, lc.s) != CFD_OK) return nullptr;
      return z;
    }
    if (PRE == kPreComponent) {
      if (component_apply_device<XT>(a, v, z, skip, lc.s) != CFD_OK) return nullptr;
      return z;
    }
    return v;
  };
  int64_t cycles = 0;
  for (;;) {
    // cycle start: beta = ||r||, v_0 = r / beta
    k_gmres_begin<<<1, 1, 0, lc.s>>>(G, st);
    CFD_TRY(dots(B.r, 1, B.r, G.g, 1, done));
    CFD_TRY(lc.vec(n, k_scale_div<XT>, (const XT*)B.r, V, (const double*)G.g, done));
    for (int j = 0; j < m; ++j) {
      XT* vj = V + (int64_t)j * n;
      XT* w = V + (int64_t)(j + 1) * n;
      double* hc = G.H + (size_t)j * (m + 1);
      const XT* z = precond(vj, B.z, ended);
      if (!z) return CFD_ERR_CUDA;
      CFD_TRY(lc.spmv<XT, XT, false>(a->dev, z, EpiStore<XT>{w, ended, {}}));
      CFD_TRY(dots(V, j + 1, w, hc, 0, ended));
      CFD_TRY(lc.vec(n, k_gemv_sub<XT>, (const XT*)V, n, j + 1, (const double*)hc, w, ended));
      CFD_TRY(dots(V, j + 1, w, G.h, 0, ended));
      CFD_TRY(lc.vec(n, k_gemv_sub<XT>, (const XT*)V, n, j + 1, (const double*)G.h, w, ended));
      CFD_TRY(dots(w, 1, w, hc + j + 1, 1, ended));
      CFD_TRY(lc.vec(n, k_scale_div<XT>, (const XT*)w, w, (const double*)(hc + j + 1), ended));
      k_gmres_rot<<<1, 1, 0, lc.s>>>(G, j, st);
      CFD_TRY(lc.check());
    }
    // x += M^-1 (V y); r = b - A x; the true residual decides
    k_gmres_lsq<<<1, 1, 0, lc.s>>>(G, done);
    CFD_TRY(lc.vec(n, k_gemv_cols<XT>, (const XT*)V, n, (const int*)G.flags, (const double*)G.y, B.q, done));
    const XT* zc = precond(B.q, B.z, done);
    if (!zc) return CFD_ERR_CUDA;
    CFD_TRY(lc.vec(n, k_add<XT>, B.x, zc, done));
    CFD_TRY(lc.spmv<XT, XT, false>(a->dev, B.x, EpiResidual<XT, 2>{B.r, B.b, st, done, {}}));
    k_gmres_check<<<1, 1, 0, lc.s>>>(st);
    CFD_TRY(lc.check());
    CFD_TRY(pl.poll());
    if (pl.host->done) break;
    if (++cycles > pl.host->max_iter + 2) {
      set_error("GMRES did not terminate within its iteration budget");
      return CFD_ERR_TIMEOUT;
    }
  }
  return CFD_OK;
}

template <typename XT>
static cfd_status krylov_loop(Launcher& lc, int solver, int pre, cfd_csr* a, cfd_amg* amg, KrylovBufs<XT>& B,
                              DevState* st, Poller& pl, int64_t restart) {
  if (solver == CFD_SOLVER_GMRES) {
    if (pre == kPreJacobi) return gmres_loop<XT, kPreJacobi>(lc, a, amg, B, st, pl, restart);
    if (pre == kPreAmg) return gmres_loop<XT, kPreAmg>(lc, a, amg, B, st, pl, restart);
    if (pre == kPreSimple) return gmres_loop<XT, kPreSimple>(lc, a, amg, B, st, pl, restart);
    if (pre == kPreBlockDiag) return gmres_loop<XT, kPreBlockDiag>(lc, a, amg, B, st, pl, restart);
    if (pre == kPreComponent) return gmres_loop<XT, kPreComponent>(lc, a, amg, B, st, pl, restart);
    return gmres_loop<XT, kPreNone>(lc, a, amg, B, st, pl, restart);
  }
  if (pre == kPreSimple || pre == kPreBlockDiag || pre == kPreComponent) {
    set_error("the saddle-point preconditioners are applied with GMRES only");
    return CFD_ERR_CONFIG;
  }
  if (solver == CFD_SOLVER_BICGSTAB) {
    if (pre == kPreJacobi) return bicgstab_loop<XT, kPreJacobi>(lc, a, amg, B, st, pl);
    if (pre == kPreAmg) return bicgstab_loop<XT, kPreAmg>(lc, a, amg, B, st, pl);
    return bicgstab_loop<XT, kPreNone>(lc, a, amg, B, st, pl);
  }
  if (pre == kPreJacobi) return pcg_loop<XT, kPreJacobi>(lc, a, amg, B, st, pl);
  if (pre == kPreAmg) return pcg_loop<XT, kPreAmg>(lc, a, amg, B, st, pl);
  return pcg_loop<XT, kPreNone>(lc, a, amg, B, st, pl);
}

static void init_state(DevState& h, const cfd_solver_config& cfg) {
  std::memset(&h, 0, sizeof(h));
  h.tol_abs = cfg.tolerance;
  h.tol_rel = cfg.relative_tolerance;
  h.max_iter = (int32_t)std::min<int64_t>(cfg.max_iterations, INT32_MAX);
  h.rho = h.alpha = h.omega = 1.0;
  h.term = CFD_TERM_MAX_ITERATIONS;
}

cfd_status check_precond(cfd_csr* a, const cfd_solve_options& opt, cfd_amg* amg) {
  if (opt.precond == CFD_PRECOND_AMG) {
    if (!amg) {
      set_error("AMG preconditioner requested without an AMG handle");
      return CFD_ERR_CONFIG;
    }
    if (!amg->ctx) {
      set_error("AMG preconditioner: the hierarchy was built on the host only (cfd_amg_setup_host)");
      return CFD_ERR_STATE;
    }
    // The V-cycle runs on the matrix's context (its stream, its device, its
    // lock held): level buffers of another context may sit on another device.
    if (amg->ctx != a->ctx) {
      set_error("AMG preconditioner: the matrix and the hierarchy belong to different contexts");
      return CFD_ERR_STATE;
    }
    if (amg->dev.empty() || amg->dev[0].A.nrows != a->dev.nrows) {
      set_error("AMG hierarchy does not match the matrix (%lld rows)", (long long)a->dev.nrows);
      return CFD_ERR_DIM;
    }
  }
  if (opt.precond == CFD_PRECOND_SIMPLE || opt.precond == CFD_PRECOND_BLOCK_DIAGONAL) {
    // LinearSolverChain pairs both with GMRES (chain.rs:216-238, 265-285).
    if (opt.solver != CFD_SOLVER_GMRES) {
      set_error("the saddle-point preconditioners are applied with GMRES only (chain.rs:216-285)");
      return CFD_ERR_CONFIG;
    }
    CFD_TRY(simple_ensure(a));
  }
  if (opt.precond == CFD_PRECOND_COMPONENT_BLOCK) {
    // LinearSolverChain pairs it with GMRES (chain.rs:193-217).
    if (opt.solver != CFD_SOLVER_GMRES) {
      set_error("the component-block preconditioner is applied with GMRES only (chain.rs:193-217)");
      return CFD_ERR_CONFIG;
    }
    CFD_TRY(component_ensure(a));
  }
  if (opt.precond == CFD_PRECOND_JACOBI) {
    CFD_TRY(ensure_diagonals(a));
    if (a->jacobi_status != 0) {
      set_error("Jacobi preconditioner: non-finite diagonal entry");
      return CFD_ERR_NONFINITE;
    }
  }
  return CFD_OK;
}

// Plain FP64 solve.
cfd_status solve_fp64(cfd_csr* a, const cfd_solve_options& opt, cfd_amg* amg, const double* b, double* x,
                      const cfd_solver_config& cfg, cfd_solve_report& rep) {
  cfd_context* ctx = a->ctx;
  Launcher lc{ctx, ctx->stream};
  const int64_t n = a->dev.nrows;
  Alloc<double> al{ctx->stream, {}};
  KrylovBufs<double> B{};
  const bool host_mem = opt.memory == CFD_MEMORY_HOST;
  B.x = host_mem ? al.get(n) : x;
  B.b = host_mem ? al.get(n) : const_cast<double*>(b);
  B.r = al.get(n);
  B.p = al.get(n);
  B.q = al.get(n);
  B.z = al.get(n);
  if (opt.solver == CFD_SOLVER_BICGSTAB) {
    B.rh = al.get(n);
    B.v = al.get(n);
    B.s = al.get(n);
    B.sh = al.get(n);
    B.t = al.get(n);
  }
  if (!B.x || !B.b || !B.r || !B.p || !B.q || !B.z || (opt.solver == CFD_SOLVER_BICGSTAB && !B.t)) {
    set_error("device workspace allocation failed (%lld unknowns)", (long long)n);
    return CFD_ERR_ALLOC;
  }
  DevState* st = ctx->state;
  DevState* hs = ctx->h_state;
  init_state(*hs, cfg);
  CFD_TRY_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  if (host_mem) {
    CFD_TRY_CUDA(cudaMemcpyAsync(B.b, b, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CFD_TRY_CUDA(cudaMemcpyAsync(B.x, x, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  }
  CFD_TRY_CUDA(cudaMemcpyAsync(st, hs, sizeof(DevState), cudaMemcpyHostToDevice, ctx->stream));
  if (opt.solver == CFD_SOLVER_BICGSTAB) {
    CFD_TRY_CUDA(cudaMemsetAsync(B.v, 0, n * sizeof(double), ctx->stream));
    CFD_TRY_CUDA(cudaMemsetAsync(B.p, 0, n * sizeof(double), ctx->stream));
  }
  Poller pl{ctx, st, hs};
  pl.fixed = opt.check_every;
  bool whole = false;
  if (ctx->cluster_solve && opt.solver == CFD_SOLVER_CG &&
      (opt.precond == CFD_PRECOND_NONE || opt.precond == CFD_PRECOND_JACOBI))
    CFD_TRY(cluster_pcg_solve(ctx, a->dev, opt.precond == CFD_PRECOND_JACOBI ? a->jinv64 : nullptr, B.b, B.x, st,
                              &whole));
  if (!whole) {
    // r0 = b - A x0, ||r0||, threshold, InitialResidual test.
    CFD_TRY(lc.spmv<double, double, false>(a->dev, B.x, EpiResidual<double, 1>{B.r, B.b, st, nullptr, {}}));
    CFD_TRY(krylov_loop<double>(lc, opt.solver, opt.precond, a, amg, B, st, pl, opt.restart));
  }
  if (host_mem) CFD_TRY_CUDA(cudaMemcpyAsync(x, B.x, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CFD_TRY_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  CFD_TRY(pl.poll());
  float ms = 0.f;
  CFD_TRY_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  rep.termination = hs->term;
  rep.outer_iterations = 0;
  rep.iterations = hs->iter;
  rep.initial_residual = hs->rnorm0;
  rep.final_residual = hs->rnorm;
  rep.threshold = hs->threshold;
  rep.device_ms = ms;
  return CFD_OK;
}

// FP32 inner Krylov/AMG solves inside FP64 iterative refinement. FP64 is kept
// for the outer residual r = b - A x, the solution accumulation, the reduction
// accumulators and the coarsest-level solve.
cfd_status solve_refine(cfd_csr* a, const cfd_solve_options& opt, cfd_amg* amg, const double* b, double* x,
                        const cfd_solver_config& cfg, cfd_solve_report& rep) {
  cfd_context* ctx = a->ctx;
  Launcher lc{ctx, ctx->stream};
  const int64_t n = a->dev.nrows;
  CFD_TRY(devmat_ensure32(a->dev, ctx->stream));
  if (opt.precond == CFD_PRECOND_AMG) CFD_TRY(amg_ensure32(amg));
  Alloc<double> ad{ctx->stream, {}};
  Alloc<float> af{ctx->stream, {}};
  const bool host_mem = opt.memory == CFD_MEMORY_HOST;
  double* x64 = host_mem ? ad.get(n) : x;
  double* b64 = host_mem ? ad.get(n) : const_cast<double*>(b);
  double* r64 = ad.get(n);
  KrylovBufs<float> B{};
  B.x = af.get(n);
  if (opt.solver == CFD_SOLVER_GMRES) B.b = af.get(n);  // inner right-hand side for restarts
  B.r = af.get(n);
  B.p = af.get(n);
  B.q = af.get(n);
  B.z = af.get(n);
  if (opt.solver == CFD_SOLVER_BICGSTAB) {
    B.rh = af.get(n);
    B.v = af.get(n);
    B.s = af.get(n);
    B.sh = af.get(n);
    B.t = af.get(n);
  }
  if (!x64 || !b64 || !r64 || !B.x || !B.r || !B.p || !B.q || !B.z ||
      (opt.solver == CFD_SOLVER_BICGSTAB && !B.t) || (opt.solver == CFD_SOLVER_GMRES && !B.b)) {
    set_error("device workspace allocation failed (%lld unknowns)", (long long)n);
    return CFD_ERR_ALLOC;
  }
  DevState* outer = ctx->state;
  DevState* inner = ctx->state + 1;
  DevState* hs = ctx->h_state;
  init_state(hs[0], cfg);
  cfd_solver_config icfg = cfg;
  icfg.tolerance = 0.0;
  icfg.relative_tolerance = opt.inner_tolerance > 0 ? opt.inner_tolerance : 1e-4;
  init_state(hs[1], icfg);
  CFD_TRY_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  if (host_mem) {
    CFD_TRY_CUDA(cudaMemcpyAsync(b64, b, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CFD_TRY_CUDA(cudaMemcpyAsync(x64, x, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  }
  CFD_TRY_CUDA(cudaMemcpyAsync(ctx->state, hs, 2 * sizeof(DevState), cudaMemcpyHostToDevice, ctx->stream));
  CFD_TRY(lc.spmv<double, double, false>(a->dev, x64, EpiResidual<double, 1>{r64, b64, outer, nullptr, {}}));
  Poller pl_out{ctx, outer, hs};
  CFD_TRY(pl_out.poll());
  const double r0 = hs[0].rnorm0, thr = hs[0].threshold;
  int term = hs[0].term;
  double rn = hs[0].rnorm;
  int64_t inner_iters = 0;
  int outer_steps = 0;
  double inner_rate = 0.0;
  const int max_outer = opt.max_outer > 0 ? opt.max_outer : 20;
  while (!hs[0].done) {
    if (outer_steps >= max_outer || inner_iters >= cfg.max_iterations) {
      term = CFD_TERM_MAX_ITERATIONS;
      break;
    }
    // inner budget: what is left of the outer one
    hs[1].max_iter = (int32_t)std::min<int64_t>(cfg.max_iterations - inner_iters, INT32_MAX);
    CFD_TRY_CUDA(cudaMemcpyAsync(&inner->max_iter, &hs[1].max_iter, sizeof(int32_t), cudaMemcpyHostToDevice,
                                 ctx->stream));
    CFD_TRY(lc.vec(n, k_refine_start, (const double*)r64, B.r, B.x, (const DevState*)outer, inner, lc.red()));
    Poller pl{ctx, inner, hs + 1};
    pl.fixed = opt.check_every;
    // The previous inner solve's contraction rate predicts this one's length:
    // its first chunk stops one iteration short of the prediction, so the
    // host's first look at the state comes near the end instead of after one
    // iteration (no look at all before the first chunk).
    if (inner_rate > 0.0 && inner_rate < 1.0 && opt.solver == CFD_SOLVER_CG) {
      const double k = std::log(icfg.relative_tolerance) / std::log(inner_rate);
      pl.chunk = (int)std::max(1.0, std::min(64.0, std::floor(k) - 1.0));
    }
    if (opt.solver == CFD_SOLVER_GMRES) CFD_TRY(lc.vec(n, k_copy<float>, (const float*)B.r, B.b, (const int*)nullptr));
    CFD_TRY(krylov_loop<float>(lc, opt.solver, opt.precond, a, amg, B, inner, pl, opt.restart));
    inner_iters += hs[1].iter;
    ++outer_steps;
    if (hs[1].iter > 0 && hs[1].rnorm0 > 0.0 && hs[1].rnorm > 0.0)
      inner_rate = std::pow(hs[1].rnorm / hs[1].rnorm0, 1.0 / (double)hs[1].iter);
    const int iterm = hs[1].term;
    CFD_TRY(lc.vec(n, k_refine_accumulate, x64, (const float*)B.x, (const DevState*)outer));
    // outer FP64 residual and convergence test
    CFD_TRY(lc.spmv<double, double, false>(a->dev, x64, EpiResidual<double, 2>{r64, b64, outer, nullptr, {}}));
    CFD_TRY(pl_out.poll());
    rn = hs[0].rnorm;
    if (!std::isfinite(rn)) {
      term = CFD_TERM_BREAKDOWN;
      break;
    }
    if (rn <= thr) {
      term = CFD_TERM_CONVERGED;
      break;
    }
    if (iterm == CFD_TERM_BREAKDOWN || iterm == CFD_TERM_NON_POSITIVE_CURVATURE) {
      term = iterm;
      break;
    }
  }
  if (host_mem) CFD_TRY_CUDA(cudaMemcpyAsync(x, x64, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CFD_TRY_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  CFD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  CFD_TRY_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  rep.termination = term;
  rep.outer_iterations = outer_steps;
  rep.iterations = inner_iters;
  rep.initial_residual = r0;
  rep.final_residual = rn;
  rep.threshold = thr;
  rep.device_ms = ms;
  return CFD_OK;
}

// Standalone preconditioner application z = M^-1 r (FP64).
cfd_status amg_apply_fp64(cfd_amg* amg, const double* r, double* z) {
  cfd_context* ctx = amg->ctx;
  Launcher lc{ctx, ctx->stream};
  return vcycle<double>(lc, amg, 0, r, z, 0, nullptr, nullptr);
}

cfd_status spmv_fp64(cfd_csr* a, const double* x, double* y) {
  Launcher lc{a->ctx, a->ctx->stream};
  return lc.spmv<double, double, false>(a->dev, x, EpiStore<double>{y, nullptr, {}});
}

cfd_status spmv_fp32(cfd_csr* a, const float* x, float* y) {
  CFD_TRY(devmat_ensure32(a->dev, a->ctx->stream));
  Launcher lc{a->ctx, a->ctx->stream};
  return lc.spmv<float, float, false>(a->dev, x, EpiStore<float>{y, nullptr, {}});
}

}  // namespace cfd
