// Device kernels of the sparse solve path (sm_100a). All are HBM-bound.
//
//  * k_spmv_pipe: persistent, warp-specialized CSR SpMV. A producer warp walks
//    the CTA's row blocks (b = blockIdx.x + k * gridDim.x) and moves each
//    block's value, column and row-offset streams into a ring of shared-memory
//    stages with 1-D bulk copies (cp.async.bulk, the TMA engine); full/empty
//    mbarrier pairs hand stages between the producer and 8 consumer warps.
//    Consumers never touch global metadata: they read offsets and entries from
//    shared memory, gather x through the read-only path, and pass the row
//    result to a fused epilogue whose own operands were loaded before the
//    gathers. Row groups of 2^k threads serve operators with long rows.
//  * k_spmv_xs: the same pipeline for matrices whose blocks all have compact
//    column windows: x is staged in shared memory with the block, so no
//    gather leaves the SM.
//  * Epilogue functors (plain store, residual, damped Jacobi, PCG / BiCGSTAB
//    dots, prolongation-correction) consume the row result so no kernel
//    re-reads what another just wrote.
//  * Reductions are two-stage and deterministic: per-CTA partials in fixed
//    slots, and the last CTA to arrive (atomic ticket) sums them in a fixed
//    order and applies the Krylov scalar update on the device.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <type_traits>

#include "internal.h"

namespace cfd {

template <typename VT>
struct MatView {
  const int* __restrict__ rp;
  const int* __restrict__ col;
  const VT* __restrict__ val;
  const int* __restrict__ blk;
  const int4* __restrict__ desc;  // per row block {r0, r1, k0, k1}
  const uint8_t* __restrict__ code;    // dictionary codes (nullptr: no compressed block)
  const int* __restrict__ dict;        // concatenated offset dictionaries
  const int2* __restrict__ dict_desc;  // per block {first entry, entries}
  const uint8_t* __restrict__ rec;     // BlockRecords (fully coded matrices)
  const int* __restrict__ roff;        // per block record offset / 16
  unsigned long long base_mult;        // base(row) = (row * base_mult) >> 20
  int tpr_log2;  // log2 of the threads cooperating on one row
};

inline int ilog2(int v) {
  int l = 0;
  while ((1 << (l + 1)) <= v) ++l;
  return l;
}

template <typename VT>
inline MatView<VT> mat_view(const DevMat& m);
template <>
inline MatView<double> mat_view<double>(const DevMat& m) {
  return {m.rp,        m.col,   m.v64,  m.blk, m.desc, m.code, m.dict, m.dict_desc,
          m.rec,       m.roff,  (unsigned long long)m.base_mult,      ilog2(m.tpr)};
}
template <>
inline MatView<float> mat_view<float>(const DevMat& m) {
  return {m.rp,        m.col,   m.v32,  m.blk, m.desc, m.code, m.dict, m.dict_desc,
          m.rec,       m.roff,  (unsigned long long)m.base_mult,      ilog2(m.tpr)};
}

// Scratch of one two-stage reduction.
struct Red {
  double* partials;
  unsigned* counter;
};

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the CTA; the result is valid in thread 0.
template <typename T>
__device__ __forceinline__ T block_sum(T v) {
  __shared__ T sm[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sm[w] = v;
  __syncthreads();
  T t = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : T(0);
  if (w == 0) t = warp_sum(t);
  return t;
}

// Two-stage grid reduction of NV doubles. Every thread of every CTA must call
// it. Returns true in the last CTA, whose thread 0 then holds the totals.
template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], Red red, double (&tot)[NV]) {
  __shared__ bool s_last;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const double b = block_sum(v[q]);
    if (threadIdx.x == 0) red.partials[(size_t)blockIdx.x * NV + q] = b;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(red.counter, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += __ldcg(red.partials + (size_t)b * NV + q);
    tot[q] = block_sum(s);
  }
  if (threadIdx.x == 0) *red.counter = 0u;
  return true;
}

__device__ __forceinline__ bool flag_set(const int* done) { return done != nullptr && *done != 0; }

template <typename T>
__device__ __forceinline__ bool diag_ok(T d);
template <>
__device__ __forceinline__ bool diag_ok<double>(double d) {
  return fabs(d) > 1e-15;
}
template <>
__device__ __forceinline__ bool diag_ok<float>(float d) {
  return fabsf(d) > 1e-15f;
}

// Quotient of the damped-Jacobi sweeps: the FP32 (inner) sweeps divide with
// the fast single-precision division (within 2 ulp; the IEEE division's
// multi-instruction sequence made the sweep passes compute-bound), the FP64
// sweeps with the IEEE division.
template <typename XT>
__device__ __forceinline__ XT sweep_div(XT a, XT b) {
  return a / b;
}
template <>
__device__ __forceinline__ float sweep_div<float>(float a, float b) {
  return __fdividef(a, b);
}
// First damped-Jacobi sweep from a zero iterate, one entry: w b / a_ii, or 0
// where |a_ii| <= 1e-15 (the smoother's skip).
template <typename XT>
__device__ __forceinline__ XT smooth0_value(XT b, XT d, XT omega) {
  return diag_ok<XT>(d) ? omega * sweep_div<XT>(b, d) : XT(0);
}

// Programmatic dependent launch. The solve's kernels are launched with
// programmatic stream serialization, so the next kernel of the stream can be
// scheduled while this one drains. Every such kernel first waits for the
// stream's preceding grid to complete and its memory to be visible
// (griddepcontrol.wait; it returns at once for a launch without the
// attribute), then lets its own successor be scheduled.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Epilogues. load(i) fetches the row's own operands (issued before the x
// gathers so the latencies overlap); row(i, sum, diag, pre, acc) finishes it.

struct NoPre {};

// y = A x
template <typename XT>
struct EpiStore {
  static constexpr int NRED = 0;
  using Pre = NoPre;
  XT* __restrict__ y;
  const int* done;
  Red red;
  __device__ bool skip() const { return flag_set(done); }
  __device__ Pre load(int) const { return {}; }
  template <typename S>
  __device__ void row(int i, S s, S, const Pre&, double*) const {
    y[i] = (XT)s;
  }
  __device__ void finish(const double*) const {}
};

// y = A x, and x0 = the first damped-Jacobi sweep from zero on y (w y / a_ii,
// smooth0_value) for the level whose right-hand side y is: the restriction
// hands the coarse level its pre-smoothed start, so that level needs no
// separate pass over b. Bit for bit what the separate pass computes.
template <typename XT>
struct EpiStoreSmooth {
  static constexpr int NRED = 0;
  using Pre = XT;  // a_ii of the row of y
  XT* __restrict__ y;
  XT* __restrict__ x0;
  const XT* __restrict__ d;
  XT omega;
  const int* done;
  Red red;
  __device__ bool skip() const { return flag_set(done); }
  __device__ Pre load(int i) const { return d[i]; }
  template <typename S>
  __device__ void row(int i, S s, S, const Pre& di, double*) const {
    const XT yi = (XT)s;
    y[i] = yi;
    x0[i] = smooth0_value<XT>(yi, di, omega);
  }
  __device__ void finish(const double*) const {}
};

// y = base + A x (prolongation with correction, amg.rs:475-489; y may alias base)
template <typename XT>
struct EpiAddTo {
  static constexpr int NRED = 0;
  using Pre = XT;
  XT* y;
  const XT* base;
  const int* done;
  Red red;
  __device__ bool skip() const { return flag_set(done); }
  __device__ Pre load(int i) const { return base[i]; }
  template <typename S>
  __device__ void row(int i, S s, S, const Pre& bi, double*) const {
    y[i] = bi + (XT)s;
  }
  __device__ void finish(const double*) const {}
};

// r = b - A x. MODE 0: plain. MODE 1: Krylov start (||r0||, threshold, the
// InitialResidual test). MODE 2: refinement outer residual (||r|| into rnorm).
template <typename XT, int MODE>
struct EpiResidual {
  static constexpr int NRED = MODE ? 1 : 0;
  using Pre = XT;
  XT* __restrict__ r;
  const XT* __restrict__ b;
  DevState* st;
  const int* done;
  Red red;
  __device__ bool skip() const { return flag_set(done); }
  __device__ Pre load(int i) const { return b[i]; }
  template <typename S>
  __device__ void row(int i, S s, S, const Pre& bi, double* acc) const {
    const XT ri = bi - (XT)s;
    r[i] = ri;
    if (MODE) acc[0] += (double)ri * (double)ri;
  }
  __device__ void finish(const double* tot) const {
    const double rn = sqrt(tot[0]);
    st->rr = tot[0];
    st->rnorm = rn;
    if (MODE == 1) {
      st->rnorm0 = rn;
      st->threshold = fmax(st->tol_abs, st->tol_rel * rn);
      st->iter = 0;
      st->done = 0;
      st->term = CFD_TERM_MAX_ITERATIONS;
      if (!isfinite(rn)) {
        st->term = CFD_TERM_BREAKDOWN;
        st->done = 1;
      } else if (rn <= st->threshold) {
        st->term = CFD_TERM_INITIAL_RESIDUAL;
        st->done = 1;
      }
    }
  }
};

__device__ __forceinline__ void pcg_rho_update(DevState* st, double rho_new) {
  if (rho_new == 0.0 || !isfinite(rho_new)) {
    st->term = CFD_TERM_BREAKDOWN;
    st->done = 1;
    return;
  }
  st->beta = rho_new / st->rho;
  st->rho = rho_new;
}

// One damped-Jacobi sweep, JacobiSmoother::apply (smoothers.rs:160-194):
//   xn_i = xo_i + w ((b_i - sum_{j != i} a_ij xo_j) / a_ii - xo_i),  xn_i = xo_i if |a_ii| <= 1e-15.
// DOT 1: also accumulate b.xn and store it as rho (PCG start, z = M r).
// DOT 2: b.xn is rho_new of the PCG recurrence: breakdown test, beta, rho.
// a_ii comes from the level's diagonal array (the value of the row's diagonal
// entry), not from the SpMV's diagonal argument.
template <typename XT, int DOT>
struct EpiJacobi {
  static constexpr int NRED = DOT ? 1 : 0;
  struct Pre {
    XT xo, b, d;
  };
  XT* __restrict__ xn;
  const XT* __restrict__ xo;
  const XT* __restrict__ b;
  const XT* __restrict__ dg;
  XT omega;
  DevState* st;
  const int* done;
  Red red;
  __device__ bool skip() const { return flag_set(done); }
  __device__ Pre load(int i) const { return {xo[i], b[i], dg[i]}; }
  template <typename S>
  __device__ void row(int i, S s, S, const Pre& p, double* acc) const {
    XT out = p.xo;
    if (diag_ok<XT>(p.d)) {
      // FP32 (inner) sweeps: the fast single-precision division (within 2 ulp)
      const XT nv = sweep_div<XT>(p.b - (XT)s, p.d);
      out = p.xo + omega * (nv - p.xo);
    }
    xn[i] = out;
    if (DOT) acc[0] += (double)p.b * (double)out;
  }
  __device__ void finish(const double* tot) const {
    if (DOT == 1) st->rho = tot[0];
    if (DOT == 2) pcg_rho_update(st, tot[0]);
  }
};

// The same damped-Jacobi sweep for the FP32 (inner) V-cycle, in residual form
// over the full row sum s = sum_j a_ij xo_j (no per-entry diagonal test):
//   xn_i = xo_i + w (b_i - s) / a_ii,  xn_i = xo_i if |a_ii| <= 1e-15,
// a_ii from the level's diagonal array. Equal to the split form above in exact
// arithmetic; it rounds differently, and the inner solve only needs a fixed
// symmetric smoother (the FP64 sweeps keep the split form of
// smoothers.rs:177-186).
template <typename XT, int DOT>
struct EpiJacobiR {
  static constexpr int NRED = DOT ? 1 : 0;
  struct Pre {
    XT xo, b, d;
  };
  XT* __restrict__ xn;
  const XT* __restrict__ xo;
  const XT* __restrict__ b;
  const XT* __restrict__ diag;
  XT omega;
  DevState* st;
  const int* done;
  Red red;
  __device__ bool skip() const { return flag_set(done); }
  __device__ Pre load(int i) const { return {xo[i], b[i], diag[i]}; }
  template <typename S>
  __device__ void row(int i, S s, S, const Pre& p, double* acc) const {
    XT out = p.xo;
    if (diag_ok<XT>(p.d)) {
      const XT q = sweep_div<XT>(p.b - (XT)s, p.d);
      out = p.xo + omega * q;
    }
    xn[i] = out;
    if (DOT) acc[0] += (double)p.b * (double)out;
  }
  __device__ void finish(const double* tot) const {
    if (DOT == 1) st->rho = tot[0];
    if (DOT == 2) pcg_rho_update(st, tot[0]);
  }
};

// PCG q = A p with p.q: alpha = rho / p.q, or NonPositiveCurvature.
template <typename XT>
struct EpiCgDot {
  static constexpr int NRED = 1;
  using Pre = XT;
  XT* __restrict__ q;
  const XT* __restrict__ p;
  DevState* st;
  Red red;
  __device__ bool skip() const { return st->done != 0; }
  __device__ Pre load(int i) const { return p[i]; }
  template <typename S>
  __device__ void row(int i, S s, S, const Pre& pi, double* acc) const {
    const XT qi = (XT)s;
    q[i] = qi;
    acc[0] += (double)pi * (double)qi;
  }
  __device__ void finish(const double* tot) const {
    st->pq = tot[0];
    if (!(tot[0] > 0.0)) {
      st->term = CFD_TERM_NON_POSITIVE_CURVATURE;
      st->done = 1;
    } else {
      st->alpha = st->rho / tot[0];
    }
  }
};

// BiCGSTAB v = A p_hat with r_hat.v: alpha = rho / r_hat.v, or Breakdown.
template <typename XT>
struct EpiBicgV {
  static constexpr int NRED = 1;
  using Pre = XT;
  XT* __restrict__ v;
  const XT* __restrict__ rhat;
  DevState* st;
  Red red;
  __device__ bool skip() const { return st->done != 0; }
  __device__ Pre load(int i) const { return rhat[i]; }
  template <typename S>
  __device__ void row(int i, S s, S, const Pre& ri, double* acc) const {
    const XT vi = (XT)s;
    v[i] = vi;
    acc[0] += (double)ri * (double)vi;
  }
  __device__ void finish(const double* tot) const {
    if (tot[0] == 0.0 || !isfinite(tot[0])) {
      st->term = CFD_TERM_BREAKDOWN;
      st->done = 1;
    } else {
      st->alpha = st->rho / tot[0];
    }
  }
};

// BiCGSTAB t = A s_hat with (t.s, t.t): omega = t.s / t.t, or Breakdown.
template <typename XT>
struct EpiBicgT {
  static constexpr int NRED = 2;
  using Pre = XT;
  XT* __restrict__ t;
  const XT* __restrict__ s;
  DevState* st;
  Red red;
  __device__ bool skip() const { return st->done != 0; }
  __device__ Pre load(int i) const { return s[i]; }
  template <typename S>
  __device__ void row(int i, S sum, S, const Pre& si, double* acc) const {
    const XT ti = (XT)sum;
    t[i] = ti;
    acc[0] += (double)ti * (double)si;
    acc[1] += (double)ti * (double)ti;
  }
  __device__ void finish(const double* tot) const {
    if (tot[1] == 0.0 || !isfinite(tot[1])) {
      st->term = CFD_TERM_BREAKDOWN;
      st->done = 1;
    } else {
      st->omega = tot[0] / tot[1];
      st->ts = tot[0];
      st->tt = tot[1];
    }
  }
};

// ---------------------------------------------------------------------------
// Row-group dot products over staged entries. A group of 2^tl threads owns
// kRowsPerThread rows of the block (g and g + 256 >> tl, ...); the groups read
// strided shares of both rows in one interleaved loop so their x gathers are in
// flight together, then reduce with a butterfly. OFFDIAG=true forms
// sum_{j != i} a_ij x_j for the Jacobi smoother's split form
// (smoothers.rs:177-186), whose epilogue reads a_ii from the level's diagonal
// array. srp/sc/sv index rows and nonzeros directly.
// Column of staged entry k: int32 as stored, or base(row) + dict[code[k]]
// with base(row) = (row * mult) >> 20, mult = (ncols << 20) / nrows (row
// itself for square matrices), computed identically by the host encoder.
struct ColRaw {
  const int* sc;
  __device__ __forceinline__ int base(int) const { return 0; }
  __device__ __forceinline__ int at(int k, int) const { return sc[k]; }
};
struct ColDict {
  const uint8_t* scode;
  const int* sdict;
  unsigned long long mult;
  __device__ __forceinline__ int base(int row) const { return (int)(((unsigned long long)row * mult) >> 20); }
  __device__ __forceinline__ int at(int k, int rowbase) const { return rowbase + sdict[scode[k]]; }
};

// Row offsets as staged: int32 absolute, or the record's uint16 offsets from
// the block's first nonzero.
struct RpAbs {
  const int* p;
  __device__ __forceinline__ int operator()(int row) const { return p[row]; }
};
struct RpRec {
  const uint16_t* p;
  int r0, k0;
  __device__ __forceinline__ int operator()(int row) const { return (int)p[row - r0] + k0; }
};

template <typename VT, typename XT, bool OFFDIAG, class Epi, class Col, class Rp>
__device__ __forceinline__ void rows_from_stage(const Epi& epi, const Rp& srp, const Col& sc, const VT* sv, int r0,
                                                int r1, int tl, int tid, const XT* __restrict__ x, double* red) {
  const int lane = tid & ((1 << tl) - 1);
  const int step = 1 << tl;
  const int g = tid >> tl;
  const int ngroups = kThreads >> tl;
  int row[kRowsPerThread], ra[kRowsPerThread], re[kRowsPerThread], rb[kRowsPerThread];
  typename Epi::Pre pre[kRowsPerThread];
  VT sum[kRowsPerThread];
#pragma unroll
  for (int q = 0; q < kRowsPerThread; ++q) {
    row[q] = r0 + g + q * ngroups;
    const bool live = row[q] < r1;
    ra[q] = live ? srp(row[q]) + lane : 0;
    re[q] = live ? srp(row[q] + 1) : 0;
    rb[q] = live ? sc.base(row[q]) : 0;
    pre[q] = typename Epi::Pre{};
    if (live && lane == 0) pre[q] = epi.load(row[q]);
    sum[q] = VT(0);
  }
  int len = 0;
#pragma unroll
  for (int q = 0; q < kRowsPerThread; ++q) len = max(len, re[q] - ra[q]);
#pragma unroll 4
  for (int j = 0; j < len; j += step) {
#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q) {
      const int k = ra[q] + j;
      if (k < re[q]) {
        const int c = sc.at(k, rb[q]);
        const VT v = sv[k];
        // The gather is issued for the diagonal entry too (a valid, cached
        // address). With OFFDIAG the diagonal entry enters the row sum as
        // 0 * x_i: the sum starts at +0, so it is never -0, and adding the
        // product (+-0) leaves it unchanged for finite x_i, so the row sum
        // equals the off-diagonal sum bit for bit. a_ii itself is not kept
        // here: the sweep's epilogue reads it from the level's diagonal
        // array (keeping it in the loop made the FP64 sweeps take 1.8x their
        // residual's time).
        const VT xv = (VT)__ldg(x + c);
        if constexpr (OFFDIAG)
          sum[q] += (c == row[q] ? VT(0) : v) * xv;
        else
          sum[q] += v * xv;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kRowsPerThread; ++q) {
    for (int o = step >> 1; o > 0; o >>= 1) sum[q] += __shfl_xor_sync(0xffffffffu, sum[q], o);
    if (row[q] < r1 && lane == 0) epi.row(row[q], sum[q], VT(0), pre[q], red);
  }
}

// ---------------------------------------------------------------------------
// Persistent warp-specialized pipeline. Every wait is bounded: when one runs
// out the CTA records the failure in *err, drains the copies it issued (again
// bounded) and leaves without joining the reduction.
constexpr int kPipeThreads = kThreads + 32;  // 8 consumer warps + 1 producer warp
constexpr unsigned kWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned limit = kWaitLimit) {
  for (unsigned i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Stage layout. CODES: every staged block is dictionary-coded and arrives as
// values plus its BlockRecord (two bulk copies), so the column region holds
// the record; otherwise values, columns (int32 or codes), row offsets and
// dictionary arrive separately.
template <typename VT, bool CODES>
struct PipeLayout {
  // FP32 record stages are small enough for four CTAs per SM with two stages
  // each: 36 warps per SM hide the x-gather latency better than a deeper ring
  // (256^3 fine operator: 178 us at 2 stages x 4 CTAs, 215 us at 3 x 3).
  static constexpr int kStages = 2;
  static constexpr int kMinBlocks = (CODES && sizeof(VT) == 4) ? 4 : 2;
  static constexpr int kValSlack = 16 / (int)sizeof(VT);
  static constexpr int kValBytes = ((kNnzCap + 2 * kValSlack) * (int)sizeof(VT) + 127) / 128 * 128;
  static constexpr int kColBytes = CODES ? (kRecordCap + 127) / 128 * 128 : ((kNnzCap + 8) * 4 + 127) / 128 * 128;
  static constexpr int kRpBytes = CODES ? 0 : ((kRowsPerBlock + 1 + 8) * 4 + 127) / 128 * 128;
  static constexpr int kDictBytes = CODES ? 0 : ((256 + 8) * 4 + 127) / 128 * 128;
  static constexpr int kStageBytes = kValBytes + kColBytes + kRpBytes + kDictBytes;
  static constexpr int kSmemBytes = kStages * kStageBytes;
};

template <typename VT, typename XT, bool OFFDIAG, class Epi, bool CODES>
__global__ void __launch_bounds__(kPipeThreads, PipeLayout<VT, CODES>::kMinBlocks) k_spmv_pipe(MatView<VT> A, int nblk, const XT* __restrict__ x,
                                                                Epi epi, int* err) {
  pdl_enter();
  if (epi.skip()) return;
  using L = PipeLayout<VT, CODES>;
  constexpr int kStages = L::kStages;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ __align__(8) uint64_t empty[kStages];
  __shared__ int4 meta[kStages];  // r0, r1, k0, k1 of the staged block
  __shared__ int2 dmeta[kStages];  // dictionary {first entry, entries} of the staged block
  __shared__ VT s_psum[kStages][kThreads / 32], s_pdiag[kStages][kThreads / 32];  // long-row partials
  __shared__ int s_pcnt[kStages];
  __shared__ volatile int s_abort;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  constexpr int mv = L::kValSlack;
  auto stage_val = [&](int s) { return reinterpret_cast<VT*>(smem + s * L::kStageBytes); };
  auto stage_col = [&](int s) { return reinterpret_cast<int*>(smem + s * L::kStageBytes + L::kValBytes); };
  auto stage_rp = [&](int s) {
    return reinterpret_cast<int*>(smem + s * L::kStageBytes + L::kValBytes + L::kColBytes);
  };
  auto stage_dict = [&](int s) {
    return reinterpret_cast<int*>(smem + s * L::kStageBytes + L::kValBytes + L::kColBytes + L::kRpBytes);
  };

  if (tid == kThreads) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kThreads / 32);
      s_pcnt[s] = 0;
    }
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  double red[Epi::NRED > 0 ? Epi::NRED : 1];
#pragma unroll
  for (int q = 0; q < (Epi::NRED > 0 ? Epi::NRED : 1); ++q) red[q] = 0.0;

  if (warp == kThreads / 32) {
    // ---- producer warp: descriptors of 32 blocks are fetched at once (one per
    // lane); lane 0 waits for free stages and issues the copies.
    const int lane = tid & 31;
    int it = 0;
    bool stop = false;
    for (int base = blockIdx.x; base < nblk && !stop; base += 32 * gridDim.x) {
      const int bl = base + lane * gridDim.x;
      const int4 dl = bl < nblk ? A.desc[bl] : make_int4(0, 0, 0, 0);
      const int2 ddl = (bl < nblk && A.dict_desc) ? A.dict_desc[bl] : make_int2(0, 0);
      const int rol = (CODES && bl < nblk) ? A.roff[bl] : 0;
      for (int j = 0; j < 32; ++j, ++it) {
        const int b = base + j * gridDim.x;
        if (b >= nblk) {
          stop = true;
          break;
        }
        int4 m;
        m.x = __shfl_sync(0xffffffffu, dl.x, j);
        m.y = __shfl_sync(0xffffffffu, dl.y, j);
        m.z = __shfl_sync(0xffffffffu, dl.z, j);
        m.w = __shfl_sync(0xffffffffu, dl.w, j);
        int2 md;
        md.x = __shfl_sync(0xffffffffu, ddl.x, j);
        md.y = __shfl_sync(0xffffffffu, ddl.y, j);
        const int ro = __shfl_sync(0xffffffffu, rol, j);
        int ok = 1;
        if (lane == 0) {
          const int s = it % kStages;
          if (it >= kStages && !mbar_wait_bounded(&empty[s], (unsigned)((it / kStages) - 1) & 1u)) {
            s_abort = 1;
            atomicExch(err, 1);
          }
          if (s_abort) {
            ok = 0;
          } else {
            meta[s] = m;
            dmeta[s] = md;
            const int p0 = m.x & ~3, p1 = (m.y + 1 + 3) & ~3;
            const unsigned brp = (unsigned)(p1 - p0) * 4u;
            if constexpr (CODES) {
              if (m.w - m.z <= kNnzCap && m.y - m.x <= kRowsPerBlock) {
                // values and the block record
                const unsigned br = (unsigned)BlockRecord::of(m.y - m.x, m.w - m.z, md.y, false).bytes();
                const uint8_t* rec = A.rec + (size_t)ro * 16;
                if (m.w > m.z) {
                  const int v0 = m.z & ~(mv - 1), v1 = (m.w + mv - 1) & ~(mv - 1);
                  const unsigned bv = (unsigned)(v1 - v0) * sizeof(VT);
                  mbar_expect_tx(&full[s], bv + br);
                  bulk_g2s(stage_val(s), A.val + v0, bv, &full[s]);
                } else {
                  mbar_expect_tx(&full[s], br);
                }
                bulk_g2s(stage_col(s), rec, br, &full[s]);
              } else {
                // a block outside the codes-only invariant: complete the
                // phase without data and flag it
                atomicExch(err, 2);
                mbar_arrive(&full[s]);
              }
            } else if (m.w - m.z > kNnzCap || m.w == m.z) {
              mbar_expect_tx(&full[s], brp);
              bulk_g2s(stage_rp(s), A.rp + p0, brp, &full[s]);
            } else if (md.y > 0) {
              // dictionary-coded columns: values, one-byte codes, offsets, dictionary
              const int v0 = m.z & ~(mv - 1), v1 = (m.w + mv - 1) & ~(mv - 1);
              const int c0 = m.z & ~15, c1 = (m.w + 15) & ~15;
              const int d0 = md.x & ~3, d1 = (md.x + md.y + 3) & ~3;
              const unsigned bv = (unsigned)(v1 - v0) * sizeof(VT), bc = (unsigned)(c1 - c0);
              const unsigned bd = (unsigned)(d1 - d0) * 4u;
              mbar_expect_tx(&full[s], bv + bc + brp + bd);
              bulk_g2s(stage_val(s), A.val + v0, bv, &full[s]);
              bulk_g2s(stage_col(s), A.code + c0, bc, &full[s]);
              bulk_g2s(stage_rp(s), A.rp + p0, brp, &full[s]);
              bulk_g2s(stage_dict(s), A.dict + d0, bd, &full[s]);
            } else {
              const int v0 = m.z & ~(mv - 1), v1 = (m.w + mv - 1) & ~(mv - 1);
              const int c0 = m.z & ~3, c1 = (m.w + 3) & ~3;
              const unsigned bv = (unsigned)(v1 - v0) * sizeof(VT), bc = (unsigned)(c1 - c0) * 4u;
              mbar_expect_tx(&full[s], bv + bc + brp);
              bulk_g2s(stage_val(s), A.val + v0, bv, &full[s]);
              bulk_g2s(stage_col(s), A.col + c0, bc, &full[s]);
              bulk_g2s(stage_rp(s), A.rp + p0, brp, &full[s]);
            }
          }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) {
          stop = true;
          break;
        }
      }
    }
    if (lane == 0 && s_abort) {
      // Drain what was issued before leaving (bounded).
      for (int j = (it > kStages ? it - kStages : 0); j < it; ++j)
        mbar_wait_bounded(&full[j % kStages], (unsigned)(j / kStages) & 1u);
    }
  } else {
    // ---- consumers ----
    // Each warp takes the stages in order on its own (no CTA-wide barrier per
    // stage). A stage is refilled only after all consumer warps released it,
    // so a warp runs at most kStages blocks ahead of the slowest one and the
    // full-barrier phase it waits for is always the pending one.
    const int tl = A.tpr_log2;
    const int lane = tid & 31;
    const int G = (int)gridDim.x;
    int it = 0;
    for (int b = blockIdx.x; b < nblk; b += G, ++it) {
      const int s = it % kStages;
      const unsigned parity = (unsigned)(it / kStages) & 1u;
      int ok = 1;
      if (lane == 0) ok = (!s_abort && mbar_wait_bounded(&full[s], parity)) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) {
          s_abort = 1;
          atomicExch(err, 1);
        }
        break;
      }
      mbar_wait_bounded(&full[s], parity);  // completes at once; acquires the stage for this lane
      const int4 m = meta[s];
      const int2 md = dmeta[s];
      if constexpr (CODES) {
        if (m.w - m.z <= kNnzCap && m.y - m.x <= kRowsPerBlock) {
          // row offsets, codes and dictionary from the staged block record
          const BlockRecord R = BlockRecord::of(m.y - m.x, m.w - m.z, md.y, false);
          const uint8_t* rec = reinterpret_cast<const uint8_t*>(stage_col(s));
          const RpRec rp{reinterpret_cast<const uint16_t*>(rec), m.x, m.z};
          const ColDict cd{rec + R.rp_bytes - m.z, reinterpret_cast<const int*>(rec + R.rp_bytes + R.code_bytes),
                           A.base_mult};
          rows_from_stage<VT, XT, OFFDIAG>(epi, rp, cd, stage_val(s) - (m.z & ~(mv - 1)), m.x, m.y, tl, tid, x, red);
        }
        __syncwarp();
        if ((tid & 31) == 0) mbar_arrive(&empty[s]);
        continue;
      }
      const RpAbs srp{stage_rp(s) - (m.x & ~3)};
      if (m.w - m.z <= kNnzCap && (md.y > 0 || m.w == m.z)) {
        // codes index the block's own dictionary, staged from entry md.x & ~3
        // (a block of empty rows reads no entry and still runs its epilogue)
        const ColDict cd{reinterpret_cast<const uint8_t*>(stage_col(s)) - (m.z & ~15), stage_dict(s) + (md.x & 3),
                         A.base_mult};
        rows_from_stage<VT, XT, OFFDIAG>(epi, srp, cd, stage_val(s) - (m.z & ~(mv - 1)), m.x, m.y, tl, tid, x, red);
      } else if (m.w - m.z <= kNnzCap) {
        const ColRaw cr{stage_col(s) - (m.z & ~3)};
        rows_from_stage<VT, XT, OFFDIAG>(epi, srp, cr, stage_val(s) - (m.z & ~(mv - 1)), m.x, m.y, tl, tid, x, red);
      } else {
        // One row longer than kNnzCap, shared by all consumer warps: each warp
        // leaves its partial sums in shared memory and warp 0 adds them in a
        // fixed order after a bounded wait. No named barrier: a warp that
        // leaves the loop early cannot hold the others.
        const int row = m.x;
        typename Epi::Pre pre{};
        if (tid == 0) pre = epi.load(row);
        VT sum = VT(0), diag = VT(0);
        for (int k = m.z + tid; k < m.w; k += kThreads) {
          const int c = __ldcs(A.col + k);
          const VT v = __ldcs(A.val + k);
          if (OFFDIAG && c == row)
            diag += v;
          else
            sum += v * (VT)__ldg(x + c);
        }
        sum = warp_sum(sum);
        diag = warp_sum(diag);
        if (lane == 0) {
          s_psum[s][warp] = sum;
          s_pdiag[s][warp] = diag;
          __threadfence_block();
          atomicAdd(&s_pcnt[s], 1);
        }
        if (warp == 0) {
          int all = 1;
          if (lane == 0) {
            unsigned i = 0;
            while (*reinterpret_cast<volatile int*>(&s_pcnt[s]) < kThreads / 32 && ++i < kWaitLimit) {
            }
            all = i < kWaitLimit;
            __threadfence_block();
          }
          all = __shfl_sync(0xffffffffu, all, 0);
          __threadfence_block();
          if (all) {
            VT ts = lane < kThreads / 32 ? s_psum[s][lane] : VT(0);
            VT td = lane < kThreads / 32 ? s_pdiag[s][lane] : VT(0);
            ts = warp_sum(ts);
            td = warp_sum(td);
            if (lane == 0) {
              s_pcnt[s] = 0;  // the stage is refilled only after this warp releases it
              epi.row(row, ts, td, pre, red);
            }
          } else if (lane == 0) {
            s_abort = 1;
            atomicExch(err, 1);
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  if (s_abort) return;
  if constexpr (Epi::NRED > 0) {
    double tot[Epi::NRED];
    if (grid_reduce<Epi::NRED>(red, epi.red, tot) && tid == 0) epi.finish(tot);
  }
}

// ---------------------------------------------------------------------------
// Sliced pipeline (DevMat::sl, FP32 values): one warp per slice of 32 rows,
// one row per lane. Slot k of the slice holds the k-th entry of each of its
// 32 rows, so a warp's value load covers 128 contiguous bytes and its code
// load 32; the x gathers of neighbouring rows fall on neighbouring entries.
// No shared-memory staging and no producer: every warp keeps its own loads in
// flight, so occupancy, not copy issue, hides the latency. Padding slots
// (code kSlPadCode) are skipped; the row sum adds the entries in CSR order, as
// the other pipelines do, so y = A x is bit-identical to theirs.
struct SlView {
  const int* __restrict__ off;       // slice slot offsets
  const uint8_t* __restrict__ code;  // per slot dictionary code
  const int* __restrict__ dict;      // chunk dictionaries
  const int* __restrict__ doff;      // chunk dictionary offsets
  const float* __restrict__ val;     // slot-major FP32 values
  unsigned long long base_mult;
  int nslices, nrows;
};

// One CTA per chunk of kSlChunkSlices slices (grid-stride over chunks): the
// chunk's dictionary is staged in shared memory, each warp takes two slices,
// and a slice is read in batches of kSlBatch slots whose code and value loads
// are all issued before the x gathers they feed, which are again issued
// together, so a warp has 2 x kSlBatch loads in flight instead of a chain.
constexpr int kSlBatch = 8;

template <typename XT, bool OFFDIAG, class Epi>
__global__ void __launch_bounds__(kThreads) k_spmv_sl(SlView S, const XT* __restrict__ x, Epi epi) {
  pdl_enter();
  if (epi.skip()) return;
  __shared__ int sdict[256];
  double red[Epi::NRED > 0 ? Epi::NRED : 1];
#pragma unroll
  for (int q = 0; q < (Epi::NRED > 0 ? Epi::NRED : 1); ++q) red[q] = 0.0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nchunks = (S.nslices + kSlChunkSlices - 1) / kSlChunkSlices;
  for (int ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int d0 = S.doff[ch], nd = S.doff[ch + 1] - d0;
    for (int q = threadIdx.x; q < 256; q += kThreads) sdict[q] = q < nd ? S.dict[d0 + q] : 0;
    __syncthreads();
    for (int sl = ch * kSlChunkSlices + warp; sl < min(S.nslices, (ch + 1) * kSlChunkSlices); sl += kThreads / 32) {
      const int row = sl * kSlRows + lane;
      const bool live = row < S.nrows;
      typename Epi::Pre pre{};
      if (live) pre = epi.load(row);
      const int e0 = S.off[sl], w = (S.off[sl + 1] - e0) / kSlRows;
      const int base = (int)(((unsigned long long)row * S.base_mult) >> 20);
      float sum = 0.0f, diag = 0.0f;
      for (int k0 = 0; k0 < w; k0 += kSlBatch) {
        unsigned c[kSlBatch];
        float v[kSlBatch], xv[kSlBatch];
        int col[kSlBatch];
#pragma unroll
        for (int j = 0; j < kSlBatch; ++j) {
          const int q = e0 + (k0 + j) * kSlRows + lane;
          const bool ok = k0 + j < w;
          c[j] = ok ? (unsigned)S.code[q] : (unsigned)kSlPadCode;
          v[j] = ok ? S.val[q] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < kSlBatch; ++j) {
          col[j] = base + sdict[c[j]];
          xv[j] = c[j] != (unsigned)kSlPadCode ? (float)__ldg(x + col[j]) : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < kSlBatch; ++j) {
          if (c[j] != (unsigned)kSlPadCode) {
            if constexpr (OFFDIAG) {
              const bool isd = (col[j] == row);
              diag = isd ? v[j] : diag;
              sum = isd ? sum : sum + v[j] * xv[j];
            } else {
              sum += v[j] * xv[j];
            }
          }
        }
      }
      if (live) epi.row(row, sum, diag, pre, red);
    }
    __syncthreads();
  }
  if constexpr (Epi::NRED > 0) {
    double tot[Epi::NRED];
    if (grid_reduce<Epi::NRED>(red, epi.red, tot) && threadIdx.x == 0) epi.finish(tot);
  }
}

// Slot-major FP32 values of the sliced layout from the CSR-order ones.
static __global__ void __launch_bounds__(kThreads) k_sl_gather(int64_t slots, const int* __restrict__ src,
                                                        const float* __restrict__ v32, float* __restrict__ out) {
  for (int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x; q < slots; q += (int64_t)gridDim.x * kThreads) {
    const int k = src[q];
    out[q] = k >= 0 ? v32[k] : 0.0f;
  }
}

// ---------------------------------------------------------------------------
// Diagonal pipeline (DevMat::dia): values stored diagonal-major, no indices.
// Grid-stride over spans of kThreads * V rows, V = 16 / sizeof(VT) (4 FP32
// rows, 2 FP64 rows per thread). Each row adds its diagonals in ascending
// offset (= the CSR order) one product at a time with the same expression as
// rows_from_stage, so y = A x is bit-identical to the other pipelines for
// finite x (a slot without an entry holds 0 and adds +-0). Values are read
// with the streaming hint: they are used once, while x is re-read by the rows
// one grid line or plane away. Three paths per span:
//  - interior span (every row live, every x index of every diagonal inside
//    [0, nrows)) with 16-byte aligned x arrays: each thread owns V consecutive
//    rows; per diagonal one 16-byte value load; x for the offset 0 by one
//    16-byte load, for offsets that are multiples of V by one 16-byte load,
//    for offsets -1 and +1 from the offset-0 vectors of the neighbouring lanes
//    by shuffle (the warp's end lanes load their one missing entry), for any
//    other offset entry by entry. All loads of a span are issued before the
//    products.
//  - interior span, x not 16-byte aligned: V rows kThreads apart per thread,
//    loads at immediate offsets from one base pointer per diagonal.
//  - boundary span: the same mapping with every load predicated.
// k_spmv_dia takes the 5- and 7-point stencils (ND diagonals fixed at compile
// time, one thread per row in the other pipelines); k_spmv_dia_gen any count
// up to kDiaMax and row groups of TPR <= kDiaMaxTpr = 2 threads.
template <typename VT>
struct DiaView {
  const VT* __restrict__ val;      // n diagonals of ld entries
  const uint32_t* __restrict__ mask;  // TPR = 2: per-row lane bits of the diagonals
  int64_t ld;
  int nrows, n, main, xvec;  // xvec: x is 16-byte aligned
  int off[kDiaMax];
};
template <typename VT>
struct DiaVec;
template <>
struct DiaVec<float> {
  using type = float4;
  static constexpr int V = 4;
  __device__ static void unpack(const float4& a, float (&o)[4]) {
    o[0] = a.x;
    o[1] = a.y;
    o[2] = a.z;
    o[3] = a.w;
  }
};
template <>
struct DiaVec<double> {
  using type = double2;
  static constexpr int V = 2;
  __device__ static void unpack(const double2& a, double (&o)[2]) {
    o[0] = a.x;
    o[1] = a.y;
  }
};

// N consecutive entries by one vector load (N * sizeof(VT) = 8 or 16 bytes).
template <typename VT, int N>
struct DiaVecN;
template <>
struct DiaVecN<float, 4> : DiaVec<float> {};
template <>
struct DiaVecN<double, 2> : DiaVec<double> {};
template <typename VT>
struct DiaVecN<VT, 1> {
  using type = VT;
  static constexpr int V = 1;
  __device__ static void unpack(const VT& a, VT (&o)[1]) { o[0] = a; }
};
template <>
struct DiaVecN<float, 2> {
  using type = float2;
  static constexpr int V = 2;
  __device__ static void unpack(const float2& a, float (&o)[2]) {
    o[0] = a.x;
    o[1] = a.y;
  }
};

// x operand of the diagonal kernels (a stored vector; the kernels take it as
// a source object so a fused producer of x can take its place).
template <typename VT>
struct DiaXPlain {
  using Vec = DiaVec<VT>;
  static constexpr bool kStore = false;
  const VT* __restrict__ x;
  __device__ VT one(int j) const { return __ldg(x + j); }
  __device__ void vec(int j, VT (&o)[Vec::V]) const {
    Vec::unpack(__ldg(reinterpret_cast<const typename Vec::type*>(x + j)), o);
  }
  template <int N>
  __device__ void vecn(int j, VT (&o)[N]) const {
    using W = DiaVecN<VT, N>;
    W::unpack(__ldg(reinterpret_cast<const typename W::type*>(x + j)), o);
  }
  __device__ void store(int, const VT (&)[Vec::V]) const {}
  __device__ void store1(int, VT) const {}
};

template <typename VT, bool OFFDIAG, int NS>
__device__ __forceinline__ void dia_sum(const VT (&v)[NS], const VT (&xv)[NS], int nd, int main, VT& sum,
                                        VT& diag) {
#pragma unroll
  for (int d = 0; d < NS; ++d) {
    if (d < nd) {
      if (OFFDIAG && d == main) {
        diag = v[d];
      } else {
        sum = fma(v[d], xv[d], sum);
      }
    }
  }
}

template <typename VT, bool OFFDIAG, class Epi, int ND, class XS>
__global__ void __launch_bounds__(kThreads) k_spmv_dia(DiaView<VT> D, XS xs, Epi epi) {
  pdl_enter();
  static_assert(ND > 0 && ND <= 8, "k_spmv_dia holds every diagonal of a row in registers");
  if (epi.skip()) return;
  using Vec = DiaVec<VT>;
  constexpr int V = Vec::V;
  constexpr int NS = ND;  // slots per row in registers
  double red[Epi::NRED > 0 ? Epi::NRED : 1];
#pragma unroll
  for (int q = 0; q < (Epi::NRED > 0 ? Epi::NRED : 1); ++q) red[q] = 0.0;
  const int nd = ND > 0 ? ND : D.n;
  const int64_t span = (int64_t)kThreads * V;
  const int omin = D.off[0], omax = D.off[nd - 1];
  const int lane = threadIdx.x & 31;
  for (int64_t s0 = (int64_t)blockIdx.x * span; s0 < D.nrows; s0 += (int64_t)gridDim.x * span) {
    const bool interior = s0 + omin >= 0 && s0 + span + omax <= D.nrows && s0 + span <= D.nrows;
    typename Epi::Pre pre[V];
    VT v[V][NS], xv[V][NS];
    if (interior && D.xvec) {
      const int r0 = (int)s0 + threadIdx.x * V;  // V consecutive rows
#pragma unroll
      for (int q = 0; q < V; ++q) pre[q] = epi.load(r0 + q);
      VT x0[V];
      xs.vec(r0, x0);
      if constexpr (XS::kStore) xs.store(r0, x0);
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        VT vd[V], xd[V];
        if (ND > 0 || d < nd) {
          const int o = D.off[d];
          Vec::unpack(__ldcs(reinterpret_cast<const typename Vec::type*>(D.val + (int64_t)d * D.ld + r0)), vd);
          if (o == 0) {
#pragma unroll
            for (int q = 0; q < V; ++q) xd[q] = x0[q];
          } else if (o % V == 0) {
            xs.vec(r0 + o, xd);
          } else if (o == -1) {
            VT prev = __shfl_up_sync(0xffffffffu, x0[V - 1], 1);
            if (lane == 0) prev = xs.one(r0 - 1);
            xd[0] = prev;
#pragma unroll
            for (int q = 1; q < V; ++q) xd[q] = x0[q - 1];
          } else if (o == 1) {
            VT next = __shfl_down_sync(0xffffffffu, x0[0], 1);
            if (lane == 31) next = xs.one(r0 + V);
#pragma unroll
            for (int q = 0; q < V - 1; ++q) xd[q] = x0[q + 1];
            xd[V - 1] = next;
          } else {
#pragma unroll
            for (int q = 0; q < V; ++q) xd[q] = xs.one(r0 + q + o);
          }
        } else {
#pragma unroll
          for (int q = 0; q < V; ++q) vd[q] = xd[q] = VT(0);
        }
#pragma unroll
        for (int q = 0; q < V; ++q) {
          v[q][d] = vd[q];
          xv[q][d] = xd[q];
        }
      }
#pragma unroll
      for (int q = 0; q < V; ++q) {
        VT sum = VT(0), diag = VT(0);
        dia_sum<VT, OFFDIAG, NS>(v[q], xv[q], nd, D.main, sum, diag);
        epi.row(r0 + q, sum, diag, pre[q], red);
      }
    } else if (interior) {
      const int r0 = (int)s0 + threadIdx.x;  // V rows kThreads apart
#pragma unroll
      for (int q = 0; q < V; ++q) {
        pre[q] = epi.load(r0 + q * kThreads);
        if constexpr (XS::kStore) xs.store1(r0 + q * kThreads, xs.one(r0 + q * kThreads));
      }
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        if (ND > 0 || d < nd) {
          const VT* vp = D.val + (int64_t)d * D.ld + r0;
          const int xo = r0 + D.off[d];
#pragma unroll
          for (int q = 0; q < V; ++q) {
            v[q][d] = __ldcs(vp + q * kThreads);
            xv[q][d] = xs.one(xo + q * kThreads);
          }
        } else {
#pragma unroll
          for (int q = 0; q < V; ++q) v[q][d] = xv[q][d] = VT(0);
        }
      }
#pragma unroll
      for (int q = 0; q < V; ++q) {
        VT sum = VT(0), diag = VT(0);
        dia_sum<VT, OFFDIAG, NS>(v[q], xv[q], nd, D.main, sum, diag);
        epi.row(r0 + q * kThreads, sum, diag, pre[q], red);
      }
    } else {
      const int r0 = (int)s0 + threadIdx.x;
      bool live[V];
#pragma unroll
      for (int q = 0; q < V; ++q) {
        const int row = r0 + q * kThreads;
        live[q] = row < D.nrows;
        pre[q] = typename Epi::Pre{};
        if (live[q]) {
          pre[q] = epi.load(row);
          if constexpr (XS::kStore) xs.store1(row, xs.one(row));
        }
      }
#pragma unroll
      for (int d = 0; d < NS; ++d) {
        const bool act = d < nd;
        const VT* vd = D.val + (int64_t)d * D.ld;
        const int o = act ? D.off[d] : 0;
#pragma unroll
        for (int q = 0; q < V; ++q) {
          const int row = r0 + q * kThreads;
          const int j = row + o;
          const bool in = act && live[q];
          v[q][d] = in ? __ldcs(vd + row) : VT(0);
          xv[q][d] = (in && j >= 0 && j < D.nrows) ? xs.one(j) : VT(0);
        }
      }
#pragma unroll
      for (int q = 0; q < V; ++q) {
        VT sum = VT(0), diag = VT(0);
        dia_sum<VT, OFFDIAG, NS>(v[q], xv[q], nd, D.main, sum, diag);
        if (live[q]) epi.row(r0 + q * kThreads, sum, diag, pre[q], red);
      }
    }
  }
  if constexpr (Epi::NRED > 0) {
    double tot[Epi::NRED];
    if (grid_reduce<Epi::NRED>(red, epi.red, tot) && threadIdx.x == 0) epi.finish(tot);
  }
}

// Sum of a row group's partial sums in the order of its butterfly
// (rows_from_stage): steps TPR/2, ..., 1, lane 0 adding its partner's.
template <typename VT, int TPR>
__device__ __forceinline__ VT dia_butterfly(VT (&s)[TPR]) {
#pragma unroll
  for (int o = TPR / 2; o > 0; o >>= 1) {
#pragma unroll
    for (int l = 0; l < o; ++l) s[l] = s[l] + s[l + o];
  }
  return s[0];
}

// Adds one slot to the partial sums of its row. TPR = 1: every slot (an
// empty one holds 0 and adds +-0, which leaves a partial that started at +0
// unchanged for finite x). TPR = 2: bit d of the row's lane mask names the
// partial of the row group's thread that adds this entry in the CSR pipelines
// (its position among the row's stored entries, mod 2); an empty slot goes to
// partial 0 and adds +-0. Explicit fused multiply-adds: the CSR pipelines'
// sum += v * x contracts to one, and a product shared by the two predicated
// partials must not be split off.
template <typename VT, bool OFFDIAG, int TPR>
__device__ __forceinline__ void dia_add(VT v, VT xv, int d, int main, uint32_t lm, VT (&s)[TPR], VT& diag) {
  if (OFFDIAG && d == main) {
    diag = v;
  } else if (TPR == 1) {
    s[0] = fma(v, xv, s[0]);
  } else {
    if ((lm >> d) & 1u)
      s[TPR - 1] = fma(v, xv, s[TPR - 1]);
    else
      s[0] = fma(v, xv, s[0]);
  }
}

// Any number of diagonals up to kDiaMax: the diagonals are streamed in order,
// each adding into the rows' partial sums (unrolled by eight so the loads of
// several diagonals are in flight). Interior spans with aligned x: V
// consecutive rows per thread (V = 2: 32 registers, eight CTAs per SM), one
// V-entry vector load of values per diagonal, x by one vector load where the
// offset is a multiple of V and entry by entry otherwise (the entries of a
// warp's loads share their cache lines). Other spans: V rows kThreads apart,
// predicated loads.
template <typename VT, bool OFFDIAG, class Epi, int TPR, class XS, int V>
__global__ void __launch_bounds__(kThreads) k_spmv_dia_gen(DiaView<VT> D, XS xs, Epi epi) {
  pdl_enter();
  static_assert(TPR == 1 || TPR == 2, "row groups of one or two threads");
  if (epi.skip()) return;
  using Vec = DiaVecN<VT, V>;
  double red[Epi::NRED > 0 ? Epi::NRED : 1];
#pragma unroll
  for (int q = 0; q < (Epi::NRED > 0 ? Epi::NRED : 1); ++q) red[q] = 0.0;
  const int nd = D.n;
  const int64_t span = (int64_t)kThreads * V;
  const int omin = D.off[0], omax = D.off[nd - 1];
  for (int64_t s0 = (int64_t)blockIdx.x * span; s0 < D.nrows; s0 += (int64_t)gridDim.x * span) {
    const bool interior = s0 + omin >= 0 && s0 + span + omax <= D.nrows && s0 + span <= D.nrows;
    typename Epi::Pre pre[V];
    VT s[V][TPR], diag[V];
    uint32_t lm[V];
#pragma unroll
    for (int q = 0; q < V; ++q) {
      diag[q] = VT(0);
      lm[q] = 0u;
#pragma unroll
      for (int k = 0; k < TPR; ++k) s[q][k] = VT(0);
    }
    if (interior && D.xvec) {
      const int r0 = (int)s0 + threadIdx.x * V;  // V consecutive rows
#pragma unroll
      for (int q = 0; q < V; ++q) {
        pre[q] = epi.load(r0 + q);
        if (TPR > 1) lm[q] = D.mask[r0 + q];
      }
#pragma unroll 8
      for (int d = 0; d < nd; ++d) {
        const int o = D.off[d];
        VT vd[V], xd[V];
        Vec::unpack(__ldcs(reinterpret_cast<const typename Vec::type*>(D.val + (int64_t)d * D.ld + r0)), vd);
        if ((o & (V - 1)) == 0) {
          xs.template vecn<V>(r0 + o, xd);
        } else {
#pragma unroll
          for (int q = 0; q < V; ++q) xd[q] = xs.one(r0 + o + q);
        }
#pragma unroll
        for (int q = 0; q < V; ++q) dia_add<VT, OFFDIAG, TPR>(vd[q], xd[q], d, D.main, lm[q], s[q], diag[q]);
      }
#pragma unroll
      for (int q = 0; q < V; ++q) epi.row(r0 + q, dia_butterfly<VT, TPR>(s[q]), diag[q], pre[q], red);
    } else {
      const int r0 = (int)s0 + threadIdx.x;  // V rows kThreads apart
      bool live[V];
#pragma unroll
      for (int q = 0; q < V; ++q) {
        const int row = r0 + q * kThreads;
        live[q] = row < D.nrows;
        pre[q] = typename Epi::Pre{};
        if (live[q]) {
          pre[q] = epi.load(row);
          if (TPR > 1) lm[q] = D.mask[row];
        }
      }
#pragma unroll 4
      for (int d = 0; d < nd; ++d) {
        const int o = D.off[d];
        const VT* vd = D.val + (int64_t)d * D.ld;
#pragma unroll
        for (int q = 0; q < V; ++q) {
          const int row = r0 + q * kThreads;
          const int j = row + o;
          const VT v = live[q] ? __ldcs(vd + row) : VT(0);
          const VT xv = (live[q] && j >= 0 && j < D.nrows) ? xs.one(j) : VT(0);
          dia_add<VT, OFFDIAG, TPR>(v, xv, d, D.main, lm[q], s[q], diag[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < V; ++q)
        if (live[q]) epi.row(r0 + q * kThreads, dia_butterfly<VT, TPR>(s[q]), diag[q], pre[q], red);
    }
  }
  if constexpr (Epi::NRED > 0) {
    double tot[Epi::NRED];
    if (grid_reduce<Epi::NRED>(red, epi.red, tot) && threadIdx.x == 0) epi.finish(tot);
  }
}

// Diagonal-major values from the CSR ones, one thread per row (every slot of
// the row written: 0 where the row has no entry on that diagonal).
template <typename VT>
__global__ void __launch_bounds__(kThreads) k_dia_fill(DiaView<VT> D, const int* __restrict__ rp,
                                                       const int* __restrict__ col, const VT* __restrict__ v,
                                                       VT* __restrict__ out) {
  for (int r = blockIdx.x * kThreads + threadIdx.x; r < D.nrows; r += gridDim.x * kThreads) {
    VT slot[kDiaMax];
#pragma unroll
    for (int d = 0; d < kDiaMax; ++d) slot[d] = VT(0);
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
      const int o = col[k] - r;
#pragma unroll
      for (int d = 0; d < kDiaMax; ++d)
        if (d < D.n && D.off[d] == o) slot[d] = v[k];
    }
#pragma unroll
    for (int d = 0; d < kDiaMax; ++d)
      if (d < D.n) out[(int64_t)d * D.ld + r] = slot[d];
  }
}

// ---------------------------------------------------------------------------
// x-staged pipeline (DevMat::xs): each stage receives the block's values, its
// record (row offsets, codes, dictionary, displacement table) and its x
// windows by bulk copy, so the consumers read every operand from shared
// memory and no gather leaves the SM. One CTA per SM with 16 consumer warps (one row or row
// group per thread) on a ring sized to fill the SM's shared memory; the
// consumers take the stages in order, so a parity wait always names the phase
// it means. Copies address stages by 32-bit shared-window offsets. Summation order
// per row equals k_spmv_pipe's, so both paths give bit-identical results.
struct XsView {
  const int4* __restrict__ xdesc;    // per block {windows | tail << 16, zero code, record offset / 16, entries copied}
  const int4* __restrict__ xwin;     // per block 4 x int4 = 8 windows {src, len, src, len}
  const uint8_t* __restrict__ rec;   // BlockRecords, with displacement tables
  int ncols;
};

constexpr int kXsConsumers = 2 * kThreads;  // one thread per row of a full block
constexpr int kXsThreads = kXsConsumers + 32;

template <typename VT>
struct XsLayout {
  static constexpr int kValSlack = 16 / (int)sizeof(VT);
  static constexpr int kValBytes = ((kNnzCap + 2 * kValSlack) * (int)sizeof(VT) + 127) / 128 * 128;
  static constexpr int kRecBytes = (kRecordCap + 127) / 128 * 128;
  static constexpr int kXBytes = (kXsCap * (int)sizeof(VT) + 127) / 128 * 128;
  static constexpr int kStageBytes = kValBytes + kRecBytes + kXBytes;
  // 227 KB per CTA less 2 KB for the static barriers and reduction scratch
  static constexpr int kStages = (227 * 1024 - 2048) / kStageBytes;
  static constexpr int kSmemBytes = kStages * kStageBytes;
  static_assert(kStages >= 2, "x-staged ring needs two stages");
};

// Rows of one staged block (ctid in [0, kXsConsumers)): row group g of 2^tl
// threads owns row r0 + g; the strided loop and butterfly per row are those of
// rows_from_stage, so every row is summed in the same order. Entries are read
// eight at a time through plain shared-memory pointers, so the compiler can
// issue the code and value loads of a batch together before the dependent
// table and x loads (volatile asm loads would pin them in program order).
template <typename VT, bool OFFDIAG, class Epi>
__device__ __forceinline__ void rows_from_stage_xs(const Epi& epi, const uint16_t* srp, const uint8_t* scode,
                                                   const VT* sval, const int* se, const VT* sx, int zq, int r0,
                                                   int r1, unsigned long long mult, int tl, int ctid, double* red) {
  constexpr int kBatch = 8;
  const int lane = ctid & ((1 << tl) - 1);
  const int step = 1 << tl;
  const int i = ctid >> tl;
  const int row = r0 + i;
  const bool live = row < r1;
  int ka = 0, ke = 0;
  const VT* xr = sx;
  typename Epi::Pre pre{};
  if (live) {
    ka = srp[i] + lane;  // offsets from the block's first nonzero
    ke = srp[i + 1];
    const int b0 = (int)(((unsigned long long)r0 * mult) >> 20);
    xr += (int)(((unsigned long long)row * mult) >> 20) - b0;
    if (lane == 0) pre = epi.load(row);
  }
  VT sum = VT(0);
  for (int kb = ka; kb < ke; kb += kBatch * step) {
    unsigned c[kBatch];
    VT v[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int k = kb + u * step;
      c[u] = k < ke ? scode[k] : 0u;
      v[u] = k < ke ? sval[k] : VT(0);
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      if (kb + u * step < ke) {
        const VT xv = xr[se[c[u]]];
        if constexpr (OFFDIAG)
          sum += ((int)c[u] == zq ? VT(0) : v[u]) * xv;  // the diagonal as a zero product
        else
          sum += v[u] * xv;
      }
    }
  }
  for (int o = step >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if (live && lane == 0) epi.row(row, sum, VT(0), pre, red);
}

template <typename VT, bool OFFDIAG, class Epi>
__global__ void __launch_bounds__(kXsThreads, 1) k_spmv_xs(MatView<VT> A, XsView X, int nblk,
                                                            const VT* __restrict__ x, Epi epi, int* err) {
  pdl_enter();
  if (epi.skip()) return;
  using L = XsLayout<VT>;
  constexpr int kStages = L::kStages;
  constexpr int vs = (int)sizeof(VT);
  constexpr int mv = L::kValSlack;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ __align__(8) uint64_t empty[kStages];
  __shared__ int4 meta[kStages];   // r0, r1, k0, k1
  __shared__ int4 xmeta[kStages];  // dictionary entries, zero code, tail entries, entries copied
  __shared__ volatile int s_abort;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const uint32_t sbase = smem_u32(smem);
  auto a_val = [&](int s) { return sbase + (uint32_t)(s * L::kStageBytes); };
  auto a_rec = [&](int s) { return a_val(s) + (uint32_t)L::kValBytes; };
  auto a_x = [&](int s) { return a_rec(s) + (uint32_t)L::kRecBytes; };
  auto p_of = [&](uint32_t a) { return (void*)(smem + (a - sbase)); };

  if (tid == kXsConsumers) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kXsConsumers / 32);
    }
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  double red[Epi::NRED > 0 ? Epi::NRED : 1];
#pragma unroll
  for (int q = 0; q < (Epi::NRED > 0 ? Epi::NRED : 1); ++q) red[q] = 0.0;

  if (warp == kXsConsumers / 32) {
    // ---- producer warp: lane j holds the descriptors of the j-th of the next
    // 32 blocks and issues that block's copies itself.
    const int lane = tid & 31;
    int it = 0;
    bool stop = false;
    for (int base = blockIdx.x; base < nblk && !stop; base += 32 * gridDim.x) {
      const int bl = base + lane * gridDim.x;
      const bool have = bl < nblk;
      const int4 m = have ? A.desc[bl] : make_int4(0, 0, 0, 0);
      const int2 md = have ? A.dict_desc[bl] : make_int2(0, 0);
      const int4 xd = have ? X.xdesc[bl] : make_int4(0, -1, 0, 0);
      int4 w[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) w[i] = have ? X.xwin[(size_t)bl * 4 + i] : make_int4(0, 0, 0, 0);
      const int nj = min(32, (nblk - base + (int)gridDim.x - 1) / (int)gridDim.x);
      for (int j = 0; j < nj; ++j, ++it) {
        int ok = 1;
        if (lane == j) {
          const int s = it % kStages;
          if (it >= kStages && !mbar_wait_bounded(&empty[s], (unsigned)((it / kStages) - 1) & 1u)) {
            s_abort = 1;
            atomicExch(err, 1);
          }
          if (s_abort) {
            ok = 0;
          } else {
            meta[s] = m;
            const int nwin = xd.x & 0xffff;
            xmeta[s] = make_int4(md.y, xd.y, xd.x >> 16, xd.w);
            const BlockRecord R = BlockRecord::of(m.y - m.x, m.w - m.z, md.y, true);
            const uint8_t* rec = X.rec + (size_t)xd.z * 16;
            const int tail = xd.x >> 16;
            if (tail > 0 && m.w - m.z <= kNnzCap && m.y - m.x <= kRowsPerBlock) {
              // the 1-3 entries of x past its last 16-byte boundary, stored
              // after the copied windows; the arrive below publishes them
              asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
              VT* at = reinterpret_cast<VT*>(p_of(a_x(s))) + xd.w;
              for (int t = 0; t < tail; ++t) at[t] = x[(X.ncols & ~3) + t];
              asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            }
            if (m.w - m.z > kNnzCap || m.y - m.x > kRowsPerBlock) {
              // outside the x-staged invariant: complete the phase and flag it
              atomicExch(err, 2);
              mbar_arrive(&full[s]);
            } else if (m.w == m.z) {
              mbar_expect_tx(&full[s], (unsigned)R.bytes());
              bulk_g2s(p_of(a_rec(s)), rec, (unsigned)R.bytes(), &full[s]);
            } else {
              const int v0 = m.z & ~(mv - 1), v1 = (m.w + mv - 1) & ~(mv - 1);
              const unsigned bv = (unsigned)(v1 - v0) * vs, bx = (unsigned)xd.w * vs;
              mbar_expect_tx(&full[s], bv + (unsigned)R.bytes() + bx);
              bulk_g2s(p_of(a_val(s)), A.val + v0, bv, &full[s]);
              bulk_g2s(p_of(a_rec(s)), rec, (unsigned)R.bytes(), &full[s]);
              uint32_t soff = a_x(s);
#pragma unroll
              for (int i = 0; i < kXsMaxWin; ++i) {
                const int src = (i & 1) ? w[i >> 1].z : w[i >> 1].x;
                const int len = (i & 1) ? w[i >> 1].w : w[i >> 1].y;
                if (i < nwin && len > 0) {
                  bulk_g2s(p_of(soff), x + src, (unsigned)len * vs, &full[s]);
                  soff += (uint32_t)(len * vs);
                }
              }
            }
          }
        }
        ok = __shfl_sync(0xffffffffu, ok, j);
        if (!ok) {
          stop = true;
          break;
        }
      }
    }
    if (lane == 0 && s_abort) {
      // Drain what was issued before leaving (bounded).
      for (int j = (it > kStages ? it - kStages : 0); j < it; ++j)
        mbar_wait_bounded(&full[j % kStages], (unsigned)(j / kStages) & 1u);
    }
  } else {
    // ---- consumers: every block of this CTA in order. Each warp waits for
    // the stages itself; a stage is refilled only after all consumer warps
    // released it, so the phase a warp waits for is always the pending one.
    const int tl = A.tpr_log2;
    const int lane = tid & 31;
    int it = 0;
    for (int b = blockIdx.x; b < nblk; b += (int)gridDim.x, ++it) {
      const int s = it % kStages;
      const unsigned parity = (unsigned)(it / kStages) & 1u;
      int ok = 1;
      if (lane == 0) ok = (!s_abort && mbar_wait_bounded(&full[s], parity)) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) {
          s_abort = 1;
          atomicExch(err, 1);
        }
        break;
      }
      mbar_wait_bounded(&full[s], parity);  // completes at once; acquires the stage for this lane
      const int4 m = meta[s];
      const int4 xm = xmeta[s];
      if (m.w - m.z <= kNnzCap && m.y - m.x <= kRowsPerBlock) {
        const BlockRecord R = BlockRecord::of(m.y - m.x, m.w - m.z, xm.x, true);
        const unsigned char* rec = smem + (a_rec(s) - sbase);
        rows_from_stage_xs<VT, OFFDIAG>(
            epi, reinterpret_cast<const uint16_t*>(rec), rec + R.rp_bytes,
            reinterpret_cast<const VT*>(smem + (a_val(s) - sbase)) + (m.z & (mv - 1)),
            reinterpret_cast<const int*>(rec + R.rp_bytes + R.code_bytes + R.dict_bytes),
            reinterpret_cast<const VT*>(smem + (a_x(s) - sbase)), xm.y, m.x, m.y, A.base_mult, tl, tid, red);
      }
      __syncwarp();
      if ((tid & 31) == 0) mbar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  if (s_abort) return;
  if constexpr (Epi::NRED > 0) {
    double tot[Epi::NRED];
    if (grid_reduce<Epi::NRED>(red, epi.red, tot) && tid == 0) epi.finish(tot);
  }
}

}  // namespace cfd
