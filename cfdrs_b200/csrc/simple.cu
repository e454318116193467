// SIMPLE saddle-point preconditioner: setup on the host from the matrix's
// values (SimplePreconditioner::new, block_preconditioner.rs:432-508), device
// arrays in FP64 and FP32, the apply as a standalone call (cfd_simple_apply)
// and as the host check of the same row code (cfd_simple_apply_host). The
// GMRES loop applies it through simple_apply_device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "internal.h"
#include "simple.h"

namespace cfd {

template <>
SimpleView<double> SimpleDev::view<double>() const {
  return {nv, np, d_rp, d_col, d_val64, g_rp, g_col, g_val64, dinv64, sinv64};
}
template <>
SimpleView<float> SimpleDev::view<float>() const {
  return {nv, np, d_rp, d_col, d_val32, g_rp, g_col, g_val32, dinv32, sinv32};
}

cfd_status simple_build(const HostCsr& a, int64_t n_velocity, SimpleHost& S) {
  const int64_t n = a.nrows;
  if (a.ncols != n) {
    set_error("SIMPLE needs a square matrix (%lld x %lld)", (long long)a.nrows, (long long)a.ncols);
    return CFD_ERR_DIM;
  }
  if (n_velocity < 0 || n_velocity > n) {
    set_error("SIMPLE: %lld velocity unknowns outside [0, %lld]", (long long)n_velocity, (long long)n);
    return CFD_ERR_DIM;
  }
  constexpr double eps = 1e-14;  // diagonal_epsilon (block_preconditioner.rs:40-42)
  S = SimpleHost();
  S.nv = n_velocity;
  S.np = n - n_velocity;
  auto diag = [&](int64_t r) {  // get_diagonal (:140-148): 0 when absent
    for (int64_t k = a.rp[r]; k < a.rp[r + 1]; ++k)
      if (a.ci[k] == r) return a.v[k];
    return 0.0;
  };
  S.dinv.resize(S.nv);
  for (int64_t i = 0; i < S.nv; ++i) {
    const double d = diag(i);
    S.dinv[i] = std::fabs(d) > eps ? 1.0 / d : 1.0;
  }
  S.d_rp.assign(1, 0);
  for (int64_t i = 0; i < S.np; ++i) {
    for (int64_t k = a.rp[S.nv + i]; k < a.rp[S.nv + i + 1]; ++k)
      if (a.ci[k] < S.nv) {
        S.d_col.push_back(a.ci[k]);
        S.d_val.push_back(a.v[k]);
      }
    S.d_rp.push_back((int32_t)S.d_col.size());
  }
  S.g_rp.assign(1, 0);
  for (int64_t v = 0; v < S.nv; ++v) {
    for (int64_t k = a.rp[v]; k < a.rp[v + 1]; ++k)
      if (a.ci[k] >= S.nv) {
        S.g_col.push_back((int32_t)(a.ci[k] - S.nv));
        S.g_val.push_back(a.v[k]);
      }
    S.g_rp.push_back((int32_t)S.g_col.size());
  }
  // diag(C - D diag(A)^-1 G): for each D entry (i, v) the G entry (v, i), found
  // in G's row v (columns sorted), in D's row order.
  S.sinv.resize(S.np);
  for (int64_t i = 0; i < S.np; ++i) {
    double s = diag(S.nv + i);
    for (int32_t k = S.d_rp[i]; k < S.d_rp[i + 1]; ++k) {
      const int32_t v = S.d_col[k];
      const auto b0 = S.g_col.begin() + S.g_rp[v], b1 = S.g_col.begin() + S.g_rp[v + 1];
      const auto it = std::lower_bound(b0, b1, (int32_t)i);
      if (it != b1 && *it == (int32_t)i) s -= S.d_val[k] * S.dinv[v] * S.g_val[it - S.g_col.begin()];
    }
    S.sinv[i] = std::fabs(s) > eps ? 1.0 / s : 1.0;
  }
  // BlockDiagonalPreconditioner::new (:258-366)
  S.bdinv.assign(n, 1.0);
  std::vector<double> md(S.nv);
  for (int64_t i = 0; i < S.nv; ++i) {
    const double d = diag(i);
    md[i] = std::fabs(d) > eps ? d : 1.0;
    S.bdinv[i] = std::fabs(md[i]) > eps ? 1.0 / md[i] : 1.0;
  }
  bool have_mean = false;
  double mean = 1.0;  // mean |momentum diagonal| over entries above eps; 1 without velocities
  for (int64_t i = 0; i < S.np; ++i) {
    double row_sum = 0.0;
    for (int64_t k = a.rp[S.nv + i]; k < a.rp[S.nv + i + 1]; ++k)
      if (a.ci[k] >= S.nv) row_sum += std::fabs(a.v[k]);
    double pd = row_sum;
    if (!(row_sum > eps)) {
      if (!have_mean) {
        double sum = 0.0;
        int64_t count = 0;
        for (int64_t v = 0; v < S.nv; ++v)
          if (std::fabs(md[v]) > eps) {
            sum += std::fabs(md[v]);
            ++count;
          }
        mean = count == 0 ? 1.0 : sum / (double)count;
        have_mean = true;
      }
      pd = mean;
    }
    S.bdinv[S.nv + i] = std::fabs(pd) > eps ? 1.0 / pd : 1.0;
  }
  return CFD_OK;
}

namespace {

template <typename T>
cfd_status put(T** d, const std::vector<T>& h, cudaStream_t s) {
  if (cudaMalloc((void**)d, std::max<size_t>(h.size(), 1) * sizeof(T)) != cudaSuccess) {
    *d = nullptr;
    set_error("cudaMalloc failed for a SIMPLE array of %zu elements", h.size());
    return CFD_ERR_ALLOC;
  }
  if (!h.empty()) CFD_TRY_CUDA(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return CFD_OK;
}

std::vector<float> narrow(const std::vector<double>& v) { return std::vector<float>(v.begin(), v.end()); }

template <typename T>
__global__ void k_simple_pressure(int64_t np, SimpleView<T> S, const T* __restrict__ r, T* __restrict__ z,
                                  const int* skip) {
  if (skip && *skip) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x)
    z[S.nv + i] = simple_pressure_row(S, i, r);
}

template <typename T>
__global__ void k_simple_velocity(int64_t nv, SimpleView<T> S, const T* __restrict__ r, T* __restrict__ z,
                                  const int* skip) {
  if (skip && *skip) return;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x)
    z[v] = simple_velocity_row(S, v, r, z);
}

int grid_of(const cfd_context* ctx, int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
}

}  // namespace

cfd_status simple_upload(const SimpleHost& S, SimpleDev& D, cudaStream_t s) {
  D.nv = S.nv;
  D.np = S.np;
  CFD_TRY(put(&D.d_rp, S.d_rp, s));
  CFD_TRY(put(&D.d_col, S.d_col, s));
  CFD_TRY(put(&D.g_rp, S.g_rp, s));
  CFD_TRY(put(&D.g_col, S.g_col, s));
  CFD_TRY(put(&D.d_val64, S.d_val, s));
  CFD_TRY(put(&D.g_val64, S.g_val, s));
  CFD_TRY(put(&D.dinv64, S.dinv, s));
  CFD_TRY(put(&D.sinv64, S.sinv, s));
  CFD_TRY(put(&D.d_val32, narrow(S.d_val), s));
  CFD_TRY(put(&D.g_val32, narrow(S.g_val), s));
  CFD_TRY(put(&D.dinv32, narrow(S.dinv), s));
  CFD_TRY(put(&D.sinv32, narrow(S.sinv), s));
  CFD_TRY(put(&D.bdinv64, S.bdinv, s));
  CFD_TRY(put(&D.bdinv32, narrow(S.bdinv), s));
  CFD_TRY_CUDA(cudaStreamSynchronize(s));  // the host vectors may go
  return CFD_OK;
}

void simple_free(SimpleDev* D) {
  if (!D) return;
  for (void* p : {(void*)D->d_rp, (void*)D->d_col, (void*)D->g_rp, (void*)D->g_col, (void*)D->d_val64,
                  (void*)D->g_val64, (void*)D->dinv64, (void*)D->sinv64, (void*)D->d_val32, (void*)D->g_val32,
                  (void*)D->dinv32, (void*)D->sinv32, (void*)D->bdinv64, (void*)D->bdinv32})
    if (p) cudaFree(p);
  delete D;
}

// (Re)builds the matrix's SIMPLE arrays when set up and stale. Caller holds
// the context lock with the device selected.
cfd_status simple_ensure(cfd_csr* a) {
  if (a->simple_nv < 0) {
    set_error("saddle-point preconditioner requested but no velocity/pressure split set on this matrix "
              "(cfd_saddle_setup)");
    return CFD_ERR_STATE;
  }
  if (a->simple && !a->simple_stale) return CFD_OK;
  SimpleHost S;
  CFD_TRY(simple_build(a->host, a->simple_nv, S));
  SimpleDev* D = new SimpleDev;
  OnUnwind release([&] { simple_free(D); });
  const cfd_status st = simple_upload(S, *D, a->ctx->stream);
  if (st != CFD_OK) {
    simple_free(D);
    return st;
  }
  simple_free(a->simple);
  a->simple = D;
  a->simple_stale = false;
  return CFD_OK;
}

// z = M^-1 r on stream s; the two passes return at once when *skip is set.
template <typename T>
cfd_status simple_apply_device(cfd_csr* a, const T* r, T* z, const int* skip, cudaStream_t s) {
  const SimpleView<T> S = a->simple->view<T>();
  if (S.np > 0) k_simple_pressure<T><<<grid_of(a->ctx, S.np), 256, 0, s>>>(S.np, S, r, z, skip);
  if (S.nv > 0) k_simple_velocity<T><<<grid_of(a->ctx, S.nv), 256, 0, s>>>(S.nv, S, r, z, skip);
  a->ctx->stats.launches += (S.np > 0) + (S.nv > 0);
  CFD_TRY_CUDA(cudaGetLastError());
  return CFD_OK;
}
template cfd_status simple_apply_device<double>(cfd_csr*, const double*, double*, const int*, cudaStream_t);
template cfd_status simple_apply_device<float>(cfd_csr*, const float*, float*, const int*, cudaStream_t);

namespace {
template <typename T>
__global__ void k_scale_by(int64_t n, const T* __restrict__ r, const T* __restrict__ inv, T* __restrict__ z,
                           const int* skip) {
  if (skip && *skip) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] = r[i] * inv[i];
}
}  // namespace

template <typename T>
cfd_status block_diagonal_apply_device(cfd_csr* a, const T* r, T* z, const int* skip, cudaStream_t s) {
  const int64_t n = a->simple->nv + a->simple->np;
  const T* inv;
  if constexpr (sizeof(T) == 8)
    inv = a->simple->bdinv64;
  else
    inv = a->simple->bdinv32;
  if (n > 0) {
    k_scale_by<T><<<grid_of(a->ctx, n), 256, 0, s>>>(n, r, inv, z, skip);
    a->ctx->stats.launches++;
  }
  CFD_TRY_CUDA(cudaGetLastError());
  return CFD_OK;
}
template cfd_status block_diagonal_apply_device<double>(cfd_csr*, const double*, double*, const int*, cudaStream_t);
template cfd_status block_diagonal_apply_device<float>(cfd_csr*, const float*, float*, const int*, cudaStream_t);

}  // namespace cfd

using namespace cfd;

extern "C" {

cfd_status cfd_saddle_setup(cfd_csr* a, int64_t n_velocity) {
  return guarded("cfd_saddle_setup", [&]() -> cfd_status {
    if (!a) return CFD_ERR_STATE;
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    SimpleHost S;
    CFD_TRY(simple_build(a->host, n_velocity, S));
    a->simple_nv = n_velocity;
    a->simple_stale = true;
    return simple_ensure(a);
  });
}

cfd_status cfd_simple_apply(cfd_csr* a, const double* r, double* z) {
  return guarded("cfd_simple_apply", [&]() -> cfd_status {
    if (!a || !r || !z) return CFD_ERR_STATE;
    if (r == z) {
      set_error("cfd_simple_apply: r and z must be different arrays");
      return CFD_ERR_STATE;
    }
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    CFD_TRY(simple_ensure(a));
    CFD_TRY(simple_apply_device<double>(a, r, z, nullptr, a->ctx->stream));
    CFD_TRY_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return CFD_OK;
  });
}

cfd_status cfd_block_diagonal_apply(cfd_csr* a, const double* r, double* z) {
  return guarded("cfd_block_diagonal_apply", [&]() -> cfd_status {
    if (!a || !r || !z) return CFD_ERR_STATE;
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    CFD_TRY(simple_ensure(a));
    CFD_TRY(block_diagonal_apply_device<double>(a, r, z, nullptr, a->ctx->stream));
    CFD_TRY_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return CFD_OK;
  });
}

cfd_status cfd_block_diagonal_host(int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val,
                                   int64_t n_velocity, double* inv_diag) {
  return guarded("cfd_block_diagonal_host", [&]() -> cfd_status {
    if (n < 0 || !row_ptr) {
      set_error("cfd_block_diagonal_host: invalid CSR arguments");
      return CFD_ERR_DIM;
    }
    const int64_t nnz = row_ptr[n];
    CFD_TRY(validate_csr(n, n, nnz, row_ptr, col, nullptr));
    if ((nnz > 0 && !val) || (n > 0 && !inv_diag)) {
      set_error("cfd_block_diagonal_host: null array");
      return CFD_ERR_DIM;
    }
    SimpleHost S;
    CFD_TRY(simple_build(host_from(n, n, nnz, row_ptr, col, nullptr, val), n_velocity, S));
    std::copy(S.bdinv.begin(), S.bdinv.end(), inv_diag);
    return CFD_OK;
  });
}

cfd_status cfd_simple_apply_host(int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val,
                                 int64_t n_velocity, const double* b, double* x) {
  return guarded("cfd_simple_apply_host", [&]() -> cfd_status {
    if (n < 0 || !row_ptr) {
      set_error("cfd_simple_apply_host: invalid CSR arguments");
      return CFD_ERR_DIM;
    }
    const int64_t nnz = row_ptr[n];
    CFD_TRY(validate_csr(n, n, nnz, row_ptr, col, nullptr));
    if ((nnz > 0 && !val) || (n > 0 && (!b || !x))) {
      set_error("cfd_simple_apply_host: null array");
      return CFD_ERR_DIM;
    }
    SimpleHost S;
    CFD_TRY(simple_build(host_from(n, n, nnz, row_ptr, col, nullptr, val), n_velocity, S));
    const SimpleView<double> V{S.nv, S.np, S.d_rp.data(), S.d_col.data(), S.d_val.data(),
                               S.g_rp.data(), S.g_col.data(), S.g_val.data(), S.dinv.data(), S.sinv.data()};
    for (int64_t i = 0; i < S.np; ++i) x[S.nv + i] = simple_pressure_row(V, i, b);
    for (int64_t v = 0; v < S.nv; ++v) x[v] = simple_velocity_row(V, v, b, x);
    return CFD_OK;
  });
}

}  // extern "C"
