// The saddle-point preconditioners of LinearSolverChain over one
// velocity/pressure split: SimplePreconditioner
// (crates/cfd-math/src/linear_solver/block_preconditioner.rs:400-568, the
// GMRES + SIMPLE tier, chain.rs:216-238) and BlockDiagonalPreconditioner
// (:189-398, the GMRES + block-diagonal tier, chain.rs:265-285). The block
// diagonal is an inverse diagonal applied like Jacobi: the momentum diagonal
// (1 where |a_ii| <= 1e-14), and per pressure row the absolute row sum over
// the pressure block, or the mean |momentum diagonal| where that sum is <= 1e-14.
//
// SIMPLE:
// The first nv unknowns are velocities, the other np pressures. Setup (host,
// from the matrix's values): the momentum diagonal inverse dinv (1 where
// |a_ii| <= 1e-14, diagonal_epsilon :40-42), the divergence block D (pressure
// rows, velocity columns), the gradient block G (velocity rows, pressure
// columns), and sinv, the inverse of diag(C - D diag(A)^-1 G). Apply, in two
// row-parallel passes whose per-row operation order is the reference's:
//   pressure row i:  p_i = (g_i - sum_k D_ik (f_k dinv_k)) sinv_i
//   velocity row v:  u_v = f_v dinv_v, then u_v -= (dinv_v G_vi) p_i for the
//                    pressure columns i of row v in increasing order
// (the reference subtracts column by column over i, which for one v is the
// same sequence). Every product and difference is rounded on its own.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "cfdgpu.h"

namespace cfd {

struct HostCsr;

struct SimpleHost {
  int64_t nv = 0, np = 0;
  std::vector<int32_t> d_rp, d_col;  // D: np rows, velocity columns
  std::vector<double> d_val;
  std::vector<int32_t> g_rp, g_col;  // G: nv rows, pressure columns counted from 0
  std::vector<double> g_val;
  std::vector<double> dinv, sinv;
  std::vector<double> bdinv;  // BlockDiagonalPreconditioner's inverse diagonal, all n unknowns
};

// Arrays in one precision, the view both the host check and the kernels read.
template <typename T>
struct SimpleView {
  int64_t nv, np;
  const int32_t* d_rp;
  const int32_t* d_col;
  const T* d_val;
  const int32_t* g_rp;
  const int32_t* g_col;
  const T* g_val;
  const T* dinv;
  const T* sinv;
};

struct SimpleDev {
  int64_t nv = 0, np = 0;
  int32_t *d_rp = nullptr, *d_col = nullptr, *g_rp = nullptr, *g_col = nullptr;
  double *d_val64 = nullptr, *g_val64 = nullptr, *dinv64 = nullptr, *sinv64 = nullptr;
  float *d_val32 = nullptr, *g_val32 = nullptr, *dinv32 = nullptr, *sinv32 = nullptr;
  double* bdinv64 = nullptr;  // block-diagonal inverse, n entries
  float* bdinv32 = nullptr;
  template <typename T>
  SimpleView<T> view() const;
};

// Setup from a square CSR with sorted columns. CFD_ERR_DIM for n_velocity
// outside [0, n].
cfd_status simple_build(const HostCsr& a, int64_t n_velocity, SimpleHost& S);
cfd_status simple_upload(const SimpleHost& S, SimpleDev& D, cudaStream_t s);
void simple_free(SimpleDev* D);
// (Re)builds a matrix's device arrays when stale; CFD_ERR_STATE when SIMPLE
// was never set up on it. Caller holds the context lock, device selected.
cfd_status simple_ensure(cfd_csr* a);
// z = M^-1 r on stream s (r and z distinct); both passes return at once when
// skip is non-null and *skip is set.
template <typename T>
cfd_status simple_apply_device(cfd_csr* a, const T* r, T* z, const int* skip, cudaStream_t s);
// z = r * the block-diagonal inverse, same conventions.
template <typename T>
cfd_status block_diagonal_apply_device(cfd_csr* a, const T* r, T* z, const int* skip, cudaStream_t s);

// ComponentBlockPreconditioner (component.cu): three component-block dense
// inverses, D and G of the split, the lumped pressure inverse, scratch.
struct ComponentDev {
  int64_t nv = 0, np = 0, cs = 0;
  double* inv[3] = {nullptr, nullptr, nullptr};
  int32_t *d_rp = nullptr, *d_col = nullptr, *g_rp = nullptr, *g_col = nullptr;
  double *d_val64 = nullptr, *g_val64 = nullptr, *pinv64 = nullptr, *gp64 = nullptr;
  float *d_val32 = nullptr, *g_val32 = nullptr, *pinv32 = nullptr, *gp32 = nullptr;
};
void component_free(ComponentDev* C);
// (Re)builds the matrix's component-block arrays when stale; CFD_ERR_STATE
// when it was never set up. Caller holds the context lock, device selected.
cfd_status component_ensure(cfd_csr* a);
template <typename T>
cfd_status component_apply_device(cfd_csr* a, const T* r, T* z, const int* skip, cudaStream_t s);

template <typename T>
__host__ __device__ inline T sp_mul(T a, T b) {
#ifdef __CUDA_ARCH__
  if constexpr (sizeof(T) == 8)
    return __dmul_rn(a, b);
  else
    return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
template <typename T>
__host__ __device__ inline T sp_add(T a, T b) {
#ifdef __CUDA_ARCH__
  if constexpr (sizeof(T) == 8)
    return __dadd_rn(a, b);
  else
    return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
template <typename T>
__host__ __device__ inline T sp_sub(T a, T b) {
#ifdef __CUDA_ARCH__
  if constexpr (sizeof(T) == 8)
    return __dsub_rn(a, b);
  else
    return __fsub_rn(a, b);
#else
  return a - b;
#endif
}

// Pressure row i of z from r: (g_i - D_i u*) sinv_i, u* = f dinv.
template <typename T>
__host__ __device__ inline T simple_pressure_row(const SimpleView<T>& S, int64_t i, const T* r) {
  T bu = T(0);
  for (int32_t k = S.d_rp[i]; k < S.d_rp[i + 1]; ++k) {
    const int32_t v = S.d_col[k];
    bu = sp_add(bu, sp_mul(S.d_val[k], sp_mul(r[v], S.dinv[v])));
  }
  return sp_mul(sp_sub(r[S.nv + i], bu), S.sinv[i]);
}

// Velocity row v of z from r and the pressure part of z already formed.
template <typename T>
__host__ __device__ inline T simple_velocity_row(const SimpleView<T>& S, int64_t v, const T* r, const T* z) {
  const T dv = S.dinv[v];
  T u = sp_mul(r[v], dv);
  for (int32_t k = S.g_rp[v]; k < S.g_rp[v + 1]; ++k) u = sp_sub(u, sp_mul(sp_mul(dv, S.g_val[k]), z[S.nv + S.g_col[k]]));
  return u;
}

}  // namespace cfd
