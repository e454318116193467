// C ABI of libcfdgpu: handles, uploads and dispatch. See include/cfdgpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "amg_device.h"
#include "amg_setup.h"
#include "internal.h"
#include "simple.h"

namespace cfd {

cfd_status solve_fp64(cfd_csr* a, const cfd_solve_options& opt, cfd_amg* amg, const double* b, double* x,
                      const cfd_solver_config& cfg, cfd_solve_report& rep);
cfd_status solve_refine(cfd_csr* a, const cfd_solve_options& opt, cfd_amg* amg, const double* b, double* x,
                        const cfd_solver_config& cfg, cfd_solve_report& rep);
cfd_status check_precond(cfd_csr* a, const cfd_solve_options& opt, cfd_amg* amg);
cfd_status amg_apply_fp64(cfd_amg* amg, const double* r, double* z);
cfd_status spmv_fp64(cfd_csr* a, const double* x, double* y);
cfd_status spmv_fp32(cfd_csr* a, const float* x, float* y);

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

namespace {

__global__ void k_f64_to_f32(int64_t n, const double* __restrict__ s, float* __restrict__ d) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (float)s[i];
}

cfd_status cast_to_f32(const double* s, float* d, int64_t n, cudaStream_t st) {
  if (n == 0) return CFD_OK;
  int g = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_f64_to_f32<<<g, 256, 0, st>>>(n, s, d);
  CFD_TRY_CUDA(cudaGetLastError());
  return CFD_OK;
}

template <typename T>
cfd_status dmalloc(T** p, int64_t n) {
  // +16 elements of slack keeps vectorised loads of a row-block tail inside the allocation.
  cudaError_t e = cudaMalloc((void**)p, (size_t)(n + 16) * sizeof(T));
  if (e != cudaSuccess) {
    set_error("cudaMalloc(%lld bytes): %s", (long long)((n + 16) * sizeof(T)), cudaGetErrorString(e));
    *p = nullptr;
    return CFD_ERR_ALLOC;
  }
  return CFD_OK;
}

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace

// Threads per row: rows of ~6 or fewer nonzeros get a thread each; longer
// rows (Galerkin coarse operators) a power-of-two group of up to 32 threads.
int threads_per_row(int64_t nnz, int64_t nrows) {
  const double avg = nrows > 0 ? (double)nnz / (double)nrows : 0.0;
  int t = 1;
  while (t < 32 && 2.0 * t * 6.0 <= avg) t <<= 1;
  return t;
}

// Greedy row-block partition: up to kRowsPerBlock / tpr rows and kNnzCap
// nonzeros per block; a row with more nonzeros than the cap becomes a block
// of its own.
std::vector<int> row_partition(const int64_t* rp, int64_t nrows, int tpr) {
  const int64_t max_rows = kRowsPerBlock / tpr;
  std::vector<int> blk;
  blk.reserve(nrows / max_rows + 2);
  int64_t r = 0;
  blk.push_back(0);
  while (r < nrows) {
    int64_t start = r;
    int64_t nnz = rp[r + 1] - rp[r];
    ++r;
    if (nnz <= kNnzCap) {
      while (r < nrows && r - start < max_rows) {
        const int64_t rn = rp[r + 1] - rp[r];
        if (nnz + rn > kNnzCap) break;
        nnz += rn;
        ++r;
      }
    }
    blk.push_back((int)r);
  }
  return blk;
}

// Uploads the column dictionaries, the block records of fully coded matrices
// and, when every block qualifies, the x windows (encode_layout, layout.cpp).
static cfd_status upload_layout(DevMat& m, const HostCsr& h, const std::vector<int>& blk, cudaStream_t s) {
  HostLayout L;
  encode_layout(h, blk, L);
  m.base_mult = L.base_mult;
  m.compressed_nnz = L.compressed_nnz;
  m.all_compressed = L.all_compressed;
  if (L.compressed_nnz == 0) return CFD_OK;
  CFD_TRY(dmalloc(&m.code, h.nnz() + 16));
  CFD_TRY(dmalloc(&m.dict, (int64_t)L.dict.size() + 16));
  CFD_TRY(dmalloc(&m.dict_desc, (int64_t)L.dict_desc.size()));
  CFD_TRY_CUDA(cudaMemcpyAsync(m.code, L.code.data(), L.code.size(), cudaMemcpyHostToDevice, s));
  CFD_TRY_CUDA(cudaMemcpyAsync(m.dict, L.dict.data(), L.dict.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  CFD_TRY_CUDA(cudaMemcpyAsync(m.dict_desc, L.dict_desc.data(), L.dict_desc.size() * sizeof(int2),
                               cudaMemcpyHostToDevice, s));
  if (L.all_compressed) {
    CFD_TRY(dmalloc(&m.rec, (int64_t)L.rec.size()));
    CFD_TRY(dmalloc(&m.roff, (int64_t)L.roff.size()));
    CFD_TRY_CUDA(cudaMemcpyAsync(m.rec, L.rec.data(), L.rec.size(), cudaMemcpyHostToDevice, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(m.roff, L.roff.data(), L.roff.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  if (L.xs) {
    CFD_TRY(dmalloc(&m.xwin, (int64_t)L.xwin.size()));
    CFD_TRY(dmalloc(&m.xdesc, (int64_t)L.xdesc.size()));
    CFD_TRY_CUDA(cudaMemcpyAsync(m.xwin, L.xwin.data(), L.xwin.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    CFD_TRY_CUDA(cudaMemcpyAsync(m.xdesc, L.xdesc.data(), L.xdesc.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    m.xs = true;
  }
  CFD_TRY_CUDA(cudaStreamSynchronize(s));  // host staging buffers go out of scope
  return CFD_OK;
}

cfd_status devmat_upload(DevMat& m, const HostCsr& h, bool want32, cudaStream_t s) {
  devmat_free(m);
  m.nrows = h.nrows;
  m.ncols = h.ncols;
  m.nnz = h.nnz();
  if (m.nnz >= INT32_MAX || m.nrows >= INT32_MAX || m.ncols >= INT32_MAX) {
    set_error("matrix too large for int32 indices (nnz %lld)", (long long)m.nnz);
    return CFD_ERR_DIM;
  }
  std::vector<int> rp32(h.nrows + 1);
  for (int64_t i = 0; i <= h.nrows; ++i) rp32[i] = (int)h.rp[i];
  m.tpr = threads_per_row(m.nnz, m.nrows);
  std::vector<int> blk = row_partition(h.rp.data(), h.nrows, m.tpr);
  m.nblk = (int)blk.size() - 1;
  CFD_TRY(dmalloc(&m.rp, h.nrows + 1));
  CFD_TRY(dmalloc(&m.col, m.nnz));
  CFD_TRY(dmalloc(&m.v64, m.nnz));
  CFD_TRY(dmalloc(&m.blk, (int64_t)blk.size()));
  std::vector<int4> desc(m.nblk);
  for (int b = 0; b < m.nblk; ++b)
    desc[b] = make_int4(blk[b], blk[b + 1], (int)h.rp[blk[b]], (int)h.rp[blk[b + 1]]);
  CFD_TRY(dmalloc(&m.desc, (int64_t)m.nblk));
  CFD_TRY_CUDA(cudaMemcpyAsync(m.desc, desc.data(), desc.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
  CFD_TRY(upload_layout(m, h, blk, s));
  {
    HostSliced S;
    if (encode_sliced(h, m.tpr, m.base_mult, S)) {
      CFD_TRY(dmalloc(&m.sl_off, (int64_t)S.off.size()));
      CFD_TRY(dmalloc(&m.sl_code, (int64_t)S.code.size()));
      CFD_TRY(dmalloc(&m.sl_dict, (int64_t)S.dict.size()));
      CFD_TRY(dmalloc(&m.sl_doff, (int64_t)S.doff.size()));
      CFD_TRY(dmalloc(&m.sl_src, S.slots));
      CFD_TRY(dmalloc(&m.sl_v32, S.slots));
      CFD_TRY_CUDA(cudaMemcpyAsync(m.sl_off, S.off.data(), S.off.size() * sizeof(int), cudaMemcpyHostToDevice, s));
      CFD_TRY_CUDA(cudaMemcpyAsync(m.sl_code, S.code.data(), S.code.size(), cudaMemcpyHostToDevice, s));
      CFD_TRY_CUDA(cudaMemcpyAsync(m.sl_dict, S.dict.data(), S.dict.size() * sizeof(int), cudaMemcpyHostToDevice, s));
      CFD_TRY_CUDA(cudaMemcpyAsync(m.sl_doff, S.doff.data(), S.doff.size() * sizeof(int), cudaMemcpyHostToDevice, s));
      CFD_TRY_CUDA(cudaMemcpyAsync(m.sl_src, S.src.data(), S.src.size() * sizeof(int), cudaMemcpyHostToDevice, s));
      // the host vectors above are released when this block ends
      CFD_TRY_CUDA(cudaStreamSynchronize(s));
      m.sl = true;
      m.sl_slices = S.nslices;
      m.sl_slots = S.slots;
      m.sl_stale = true;
    }
  }
  {
    HostDiagonal D;
    if (encode_diagonal(h, m.tpr, D)) {
      CFD_TRY(dmalloc(&m.dia64, (int64_t)D.n * D.ld));
      CFD_TRY_CUDA(cudaMemsetAsync(m.dia64, 0, (size_t)D.n * D.ld * sizeof(double), s));
      m.dia = true;
      m.dia_n = D.n;
      m.dia_main = D.main;
      for (int d = 0; d < kDiaMax; ++d) m.dia_off[d] = D.off[d];
      m.dia_ld = D.ld;
      m.dia_stale = true;
      if (!D.mask.empty()) {
        CFD_TRY(dmalloc(&m.dia_mask, (int64_t)D.mask.size()));
        CFD_TRY_CUDA(cudaMemcpyAsync(m.dia_mask, D.mask.data(), D.mask.size() * sizeof(uint32_t),
                                     cudaMemcpyHostToDevice, s));
        CFD_TRY_CUDA(cudaStreamSynchronize(s));  // D.mask is released when this block ends
      }
    }
  }
  CFD_TRY_CUDA(cudaMemcpyAsync(m.rp, rp32.data(), rp32.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  CFD_TRY_CUDA(cudaMemcpyAsync(m.col, h.ci.data(), m.nnz * sizeof(int), cudaMemcpyHostToDevice, s));
  CFD_TRY_CUDA(cudaMemcpyAsync(m.v64, h.v.data(), m.nnz * sizeof(double), cudaMemcpyHostToDevice, s));
  CFD_TRY_CUDA(cudaMemcpyAsync(m.blk, blk.data(), blk.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  if (want32) CFD_TRY(devmat_ensure32(m, s));
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  return CFD_OK;
}

cfd_status devmat_ensure32(DevMat& m, cudaStream_t s) {
  if (m.v32 || m.nnz == 0) return CFD_OK;
  CFD_TRY(dmalloc(&m.v32, m.nnz));
  m.sl_stale = true;
  if (m.dia && !m.dia32) {
    CFD_TRY(dmalloc(&m.dia32, (int64_t)m.dia_n * m.dia_ld));
    CFD_TRY_CUDA(cudaMemsetAsync(m.dia32, 0, (size_t)m.dia_n * m.dia_ld * sizeof(float), s));
  }
  m.dia_stale = true;
  return cast_to_f32(m.v64, m.v32, m.nnz, s);
}

cfd_status devmat_update_values(DevMat& m, const double* v, int64_t nnz, bool want32, cudaStream_t s) {
  if (nnz != m.nnz) {
    set_error("value array length %lld does not match nnz %lld", (long long)nnz, (long long)m.nnz);
    return CFD_ERR_DIM;
  }
  CFD_TRY_CUDA(cudaMemcpyAsync(m.v64, v, nnz * sizeof(double), cudaMemcpyHostToDevice, s));
  if (m.v32 || want32) {
    if (!m.v32) CFD_TRY(devmat_ensure32(m, s));
    CFD_TRY(cast_to_f32(m.v64, m.v32, m.nnz, s));
  }
  m.sl_stale = true;
  m.dia_stale = true;
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  return CFD_OK;
}

void devmat_free(DevMat& m) {
  dfree(m.rp);
  dfree(m.col);
  dfree(m.v64);
  dfree(m.v32);
  dfree(m.blk);
  dfree(m.desc);
  dfree(m.code);
  dfree(m.dict);
  dfree(m.dict_desc);
  dfree(m.rec);
  dfree(m.roff);
  dfree(m.xwin);
  dfree(m.xdesc);
  dfree(m.sl_off);
  dfree(m.sl_code);
  dfree(m.sl_dict);
  dfree(m.sl_doff);
  dfree(m.sl_src);
  dfree(m.sl_v32);
  dfree(m.dia64);
  dfree(m.dia32);
  dfree(m.dia_mask);
  m.dia = false;
  m.dia_n = 0;
  m.dia_main = -1;
  m.dia_ld = 0;
  m.dia_stale = true;
  m.sl = false;
  m.sl_slices = m.sl_slots = 0;
  m.sl_stale = true;
  m.compressed_nnz = 0;
  m.all_compressed = false;
  m.xs = false;
  m.path[0] = m.path[1] = -1;
  m.nblk = 0;
}

cfd_status ensure_partials(cfd_context* ctx, int blocks) {
  if (blocks <= ctx->partial_capacity) return CFD_OK;
  dfree(ctx->partials);
  int cap = std::max(blocks, kVecGrid);
  CFD_TRY(dmalloc(&ctx->partials, (int64_t)cap * kMaxRed));
  ctx->partial_capacity = cap;
  return CFD_OK;
}

cfd_status check_device_flag(cfd_context* ctx) {
  CFD_TRY_CUDA(cudaMemcpyAsync(ctx->h_err, ctx->err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CFD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
  if (*ctx->h_err != 0) {
    const int code = *ctx->h_err;
    cudaMemsetAsync(ctx->err, 0, sizeof(int), ctx->stream);
    cudaMemsetAsync(ctx->counter, 0, sizeof(unsigned), ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    *ctx->h_err = 0;
    set_error(code == 2 ? "device-side layout check failed (int32 block in a codes-only SpMV); results are invalid"
                               : "a device-side bounded wait ran out (bulk-copy pipeline); results are invalid");
    return CFD_ERR_TIMEOUT;
  }
  return CFD_OK;
}

// Diagonal of A (FP64/FP32) and the DiagJacobi inverse: 1/a_ii, or 1 where
// |a_ii| <= f64::EPSILON (linear_system.rs:286-295); a non-finite diagonal
// entry makes the Jacobi preconditioner unavailable (linear_system.rs:281-285).
cfd_status ensure_diagonals(cfd_csr* a) {
  if (a->diag64) return CFD_OK;
  const HostCsr& h = a->host;
  const int64_t n = h.nrows;
  std::vector<double> d(n, 0.0), inv(n, 1.0);
  bool finite = true;
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t k = h.rp[i]; k < h.rp[i + 1]; ++k)
      if (h.ci[k] == i) d[i] = h.v[k];
    if (!std::isfinite(d[i])) finite = false;
    inv[i] = std::fabs(d[i]) <= DBL_EPSILON ? 1.0 : 1.0 / d[i];
  }
  a->jacobi_status = finite ? 0 : 1;
  cudaStream_t s = a->ctx->stream;
  CFD_TRY(dmalloc(&a->diag64, n));
  CFD_TRY(dmalloc(&a->diag32, n));
  CFD_TRY(dmalloc(&a->jinv64, n));
  CFD_TRY(dmalloc(&a->jinv32, n));
  CFD_TRY_CUDA(cudaMemcpyAsync(a->diag64, d.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
  CFD_TRY_CUDA(cudaMemcpyAsync(a->jinv64, inv.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
  CFD_TRY(cast_to_f32(a->diag64, a->diag32, n, s));
  CFD_TRY(cast_to_f32(a->jinv64, a->jinv32, n, s));
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  return CFD_OK;
}

// ---- AMG device hierarchy -------------------------------------------------------
template <typename XT>
static cfd_status alloc_level_vecs(LevelVecs<XT>& v, int64_t n) {
  CFD_TRY(dmalloc(&v.b, n));
  CFD_TRY(dmalloc(&v.xa, n));
  CFD_TRY(dmalloc(&v.xb, n));
  CFD_TRY(dmalloc(&v.r, n));
  CFD_TRY(dmalloc(&v.e, n));
  return CFD_OK;
}

template <typename XT>
static void free_level_vecs(LevelVecs<XT>& v) {
  dfree(v.b);
  dfree(v.xa);
  dfree(v.xb);
  dfree(v.r);
  dfree(v.e);
}

void amg_free_device(cfd_amg* amg) {
  for (DevLevel& L : amg->dev) {
    devmat_free(L.A);
    devmat_free(L.P);
    devmat_free(L.R);
    dfree(L.d64);
    dfree(L.d32);
    free_level_vecs(L.v64);
    free_level_vecs(L.v32);
    free_ra(L.ra);
  }
  amg->dev.clear();
  dfree(amg->coarse_inv);
  dfree(amg->coarse_inv32);
  amg->have32 = false;
}

cfd_status amg_upload(cfd_amg* amg, bool want32) {
  cudaStream_t s = amg->ctx->stream;
  amg_free_device(amg);
  amg->dev.resize(amg->host.size());
  int maxblk = 0;
  for (size_t l = 0; l < amg->host.size(); ++l) {
    const HostLevel& H = amg->host[l];
    DevLevel& D = amg->dev[l];
    CFD_TRY(devmat_upload(D.A, H.A, false, s));
    maxblk = std::max(maxblk, D.A.nblk);
    if (l + 1 < amg->host.size()) {
      CFD_TRY(devmat_upload(D.P, H.P, false, s));
      CFD_TRY(devmat_upload(D.R, H.R, false, s));
      maxblk = std::max({maxblk, D.P.nblk, D.R.nblk});
    }
    const int64_t n = H.A.nrows;
    std::vector<double> d(n, 0.0);
    for (int64_t i = 0; i < n; ++i)
      for (int64_t k = H.A.rp[i]; k < H.A.rp[i + 1]; ++k)
        if (H.A.ci[k] == i) d[i] = H.A.v[k];
    CFD_TRY(dmalloc(&D.d64, n));
    CFD_TRY(dmalloc(&D.d32, n));
    CFD_TRY_CUDA(cudaMemcpyAsync(D.d64, d.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    CFD_TRY(cast_to_f32(D.d64, D.d32, n, s));
    CFD_TRY(alloc_level_vecs(D.v64, n));
  }
  CFD_TRY(ensure_partials(amg->ctx, maxblk));
  if (amg->cfg.coarse_solve == CFD_COARSE_DENSE) {
    // The device Gauss-Jordan performs the host dense_inverse's operations in
    // its order (same inverse); the host one serves operators beyond its size.
    const DevMat& Ad = amg->dev.back().A;
    amg->coarse_n = Ad.nrows;
    CFD_TRY(dmalloc(&amg->coarse_inv, std::max<int64_t>(Ad.nrows * Ad.nrows, 1)));
    if (Ad.nrows <= kDenseInverseDeviceMaxRows) {
      CFD_TRY(dense_inverse_device(amg->ctx, Ad.nrows, Ad.rp, Ad.col, Ad.v64, amg->coarse_inv));
    } else {
      const HostCsr& Ac = amg->host.back().A;
      std::vector<double> inv;
      if (!dense_inverse(Ac, inv)) {
        set_error("AMG coarsest operator (%lld rows) is singular", (long long)Ac.nrows);
        return CFD_ERR_CONFIG;
      }
      CFD_TRY_CUDA(
          cudaMemcpyAsync(amg->coarse_inv, inv.data(), inv.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    }
  }
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  if (want32) CFD_TRY(amg_ensure32(amg));
  return CFD_OK;
}

cfd_status amg_ensure32(cfd_amg* amg) {
  if (amg->have32) return CFD_OK;
  cudaStream_t s = amg->ctx->stream;
  for (size_t l = 0; l < amg->dev.size(); ++l) {
    DevLevel& D = amg->dev[l];
    CFD_TRY(devmat_ensure32(D.A, s));
    if (l + 1 < amg->dev.size()) {
      CFD_TRY(devmat_ensure32(D.P, s));
      CFD_TRY(devmat_ensure32(D.R, s));
    }
    CFD_TRY(alloc_level_vecs(D.v32, D.A.nrows));
  }
  if (amg->coarse_inv) {
    const int64_t nn = std::max<int64_t>(amg->coarse_n * amg->coarse_n, 1);
    CFD_TRY(dmalloc(&amg->coarse_inv32, nn));
    CFD_TRY(cast_to_f32(amg->coarse_inv, amg->coarse_inv32, nn, s));
  }
  CFD_TRY_CUDA(cudaStreamSynchronize(s));
  amg->have32 = true;
  return CFD_OK;
}

HostCsr host_from(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* rp, const int32_t* c32,
                         const int64_t* c64, const double* v) {
  HostCsr h;
  h.nrows = nrows;
  h.ncols = ncols;
  h.rp.assign(rp, rp + nrows + 1);
  h.ci.resize(nnz);
  if (c32)
    std::memcpy(h.ci.data(), c32, nnz * sizeof(int32_t));
  else
    for (int64_t k = 0; k < nnz; ++k) h.ci[k] = (int32_t)c64[k];
  h.v.assign(v, v + nnz);
  return h;
}

cfd_status validate_csr(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* rp, const int32_t* c32,
                               const int64_t* c64) {
  if (nrows < 0 || ncols < 0 || nnz < 0 || !rp || (nnz > 0 && !c32 && !c64)) {
    set_error("invalid CSR arguments");
    return CFD_ERR_DIM;
  }
  if (nrows >= INT32_MAX || ncols >= INT32_MAX || nnz >= INT32_MAX) {
    set_error("matrix too large for int32 indices");
    return CFD_ERR_DIM;
  }
  if (rp[0] != 0 || rp[nrows] != nnz) {
    set_error("row_ptr must start at 0 and end at nnz (%lld != %lld)", (long long)rp[nrows], (long long)nnz);
    return CFD_ERR_DIM;
  }
  for (int64_t i = 0; i < nrows; ++i) {
    // rp[i + 1] <= nnz as well: the column scan below reads up to it before
    // the end of row_ptr has been compared with nnz.
    if (rp[i + 1] < rp[i] || rp[i + 1] > nnz) {
      set_error("row_ptr decreases or passes nnz at row %lld", (long long)i);
      return CFD_ERR_DIM;
    }
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      const int64_t c = c32 ? c32[k] : c64[k];
      if (c < 0 || c >= ncols) {
        set_error("column index %lld out of range in row %lld", (long long)c, (long long)i);
        return CFD_ERR_DIM;
      }
      if (k > rp[i]) {
        const int64_t cp = c32 ? c32[k - 1] : c64[k - 1];
        if (cp >= c) {
          set_error("column indices must be strictly increasing within row %lld", (long long)i);
          return CFD_ERR_DIM;
        }
      }
    }
  }
  return CFD_OK;
}

}  // namespace cfd

using namespace cfd;

extern "C" {

const char* cfd_last_error(void) { return g_err; }
const char* cfd_version(void) { return "cfdgpu 0.1.0 (sm_100a)"; }

cfd_status cfd_context_create(int device, cfd_context** out) {
  return guarded("cfd_context_create", [&]() -> cfd_status {
    if (!out) return CFD_ERR_CONFIG;
    *out = nullptr;
    int count = 0;
    CFD_TRY_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) {
      set_error("device %d not present (%d devices)", device, count);
      return CFD_ERR_CONFIG;
    }
    CFD_TRY_CUDA(cudaSetDevice(device));
    cfd_context* c = new cfd_context;
    c->device = device;
    // Any failure below releases what was made so far (destroy skips nulls).
    const cfd_status st = [&]() -> cfd_status {
      CFD_TRY_CUDA(cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking));
      c->stream = c->own;
      CFD_TRY(dmalloc(&c->counter, 1));
      CFD_TRY_CUDA(cudaMemset(c->counter, 0, sizeof(unsigned)));
      CFD_TRY(dmalloc(&c->state, 2));
      CFD_TRY_CUDA(cudaMallocHost((void**)&c->h_state, 2 * sizeof(DevState)));
      CFD_TRY_CUDA(cudaEventCreate(&c->ev0));
      CFD_TRY_CUDA(cudaEventCreate(&c->ev1));
      CFD_TRY_CUDA(cudaEventCreateWithFlags(&c->ev_switch, cudaEventDisableTiming));
      CFD_TRY(ensure_partials(c, kVecGrid));
      CFD_TRY(dmalloc(&c->err, 1));
      CFD_TRY_CUDA(cudaMemset(c->err, 0, sizeof(int)));
      CFD_TRY_CUDA(cudaMallocHost((void**)&c->h_err, sizeof(int)));
      *c->h_err = 0;
      CFD_TRY_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
      return CFD_OK;
    }();
    if (st != CFD_OK) {
      cfd_context_destroy(c);
      return st;
    }
    // Keep freed stream-ordered workspace in the pool for the next solve.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    *out = c;
    return CFD_OK;
  });
}

cfd_status cfd_context_set_stream(cfd_context* ctx, void* stream) {
  if (!ctx) return CFD_ERR_STATE;
  std::lock_guard<std::mutex> g(ctx->mu);
  const cudaStream_t next = stream ? (cudaStream_t)stream : ctx->own;
  if (next == ctx->stream) return CFD_OK;
  CFD_TRY_CUDA(cudaSetDevice(ctx->device));
  // What is queued on the old stream (an asynchronous SpMV, say) runs before
  // anything queued on the new one: an ordering on the device, the host does
  // not wait.
  CFD_TRY_CUDA(cudaEventRecord(ctx->ev_switch, ctx->stream));
  CFD_TRY_CUDA(cudaStreamWaitEvent(next, ctx->ev_switch, 0));
  ctx->stream = next;
  return CFD_OK;
}

cfd_status cfd_context_set_cluster_solve(cfd_context* ctx, int32_t enable) {
  if (!ctx) return CFD_ERR_STATE;
  std::lock_guard<std::mutex> g(ctx->mu);
  ctx->cluster_solve = enable != 0;
  return CFD_OK;
}

cfd_status cfd_context_synchronize(cfd_context* ctx) {
  if (!ctx) return CFD_ERR_STATE;
  std::lock_guard<std::mutex> g(ctx->mu);
  CFD_TRY_CUDA(cudaSetDevice(ctx->device));
  CFD_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
  return CFD_OK;
}

cfd_status cfd_context_destroy(cfd_context* ctx) {
  if (!ctx) return CFD_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  dfree(ctx->partials);
  dfree(ctx->counter);
  dfree(ctx->state);
  dfree(ctx->err);
  if (ctx->h_state) cudaFreeHost(ctx->h_state);
  if (ctx->h_err) cudaFreeHost(ctx->h_err);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->ev_switch) cudaEventDestroy(ctx->ev_switch);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
  return CFD_OK;
}

static cfd_status csr_create_common(cfd_context* ctx, int64_t nrows, int64_t ncols, int64_t nnz,
                                    const int64_t* rp, const int32_t* c32, const int64_t* c64, const double* val,
                                    cfd_csr** out) {
  return guarded("cfd_csr_create", [&]() -> cfd_status {
    if (!ctx || !out) {
      set_error("null context or output handle");
      return CFD_ERR_STATE;
    }
    *out = nullptr;
    CFD_TRY(validate_csr(nrows, ncols, nnz, rp, c32, c64));
    if (nnz > 0 && !val) {
      set_error("null value array");
      return CFD_ERR_DIM;
    }
    CFD_TRY_CUDA(cudaSetDevice(ctx->device));
    std::lock_guard<std::mutex> g(ctx->mu);
    cfd_csr* a = new cfd_csr;
    OnUnwind release([&] {
      devmat_free(a->dev);
      delete a;
    });
    a->ctx = ctx;
    a->host = host_from(nrows, ncols, nnz, rp, c32, c64, val);
    cfd_status s = devmat_upload(a->dev, a->host, false, ctx->stream);
    if (s == CFD_OK) s = ensure_partials(ctx, a->dev.nblk);
    if (s != CFD_OK) {
      devmat_free(a->dev);
      delete a;
      return s;
    }
    *out = a;
    return CFD_OK;
  });
}

cfd_status cfd_csr_create(cfd_context* ctx, int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* row_ptr,
                          const int64_t* col, const double* val, cfd_csr** out) {
  return csr_create_common(ctx, nrows, ncols, nnz, row_ptr, nullptr, col, val, out);
}

cfd_status cfd_csr_create_i32(cfd_context* ctx, int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* row_ptr,
                              const int32_t* col, const double* val, cfd_csr** out) {
  return csr_create_common(ctx, nrows, ncols, nnz, row_ptr, col, nullptr, val, out);
}

cfd_status cfd_csr_update_values(cfd_csr* a, const double* val) {
  return guarded("cfd_csr_update_values", [&]() -> cfd_status {
    if (!a || !val) return CFD_ERR_STATE;
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    // Device first: the host mirror (read by AMG setup) takes the new values
    // only once the device copy and the FP32 cast have succeeded.
    CFD_TRY(devmat_update_values(a->dev, val, a->host.nnz(), false, a->ctx->stream));
    std::copy(val, val + a->host.nnz(), a->host.v.begin());
    a->values_version++;
    a->simple_stale = a->simple_nv >= 0;
    a->cblock_stale = a->cblock_nv >= 0;
    dfree(a->diag64);
    dfree(a->diag32);
    dfree(a->jinv64);
    dfree(a->jinv32);
    a->jacobi_status = -1;
    return CFD_OK;
  });
}

cfd_status cfd_csr_info(const cfd_csr* a, int64_t* nrows, int64_t* ncols, int64_t* nnz) {
  if (!a) return CFD_ERR_STATE;
  if (nrows) *nrows = a->host.nrows;
  if (ncols) *ncols = a->host.ncols;
  if (nnz) *nnz = a->host.nnz();
  return CFD_OK;
}

cfd_status cfd_csr_layout(const cfd_csr* a, cfd_layout_info* out) {
  if (!a || !out) {
    set_error("cfd_csr_layout: null argument");
    return CFD_ERR_STATE;
  }
  const DevMat& m = a->dev;
  *out = cfd_layout_info{};
  out->blocks = m.nblk;
  out->compressed_nnz = m.compressed_nnz;
  out->all_compressed = m.all_compressed ? 1 : 0;
  out->x_staged = m.xs ? 1 : 0;
  out->threads_per_row = m.tpr;
  out->path_f32 = spmv_path(m, 0);
  out->path_f64 = spmv_path(m, 1);
  out->sliced = m.sl ? 1 : 0;
  out->sliced_slots = m.sl_slots;
  out->diagonals = m.dia ? m.dia_n : 0;
  return CFD_OK;
}

cfd_status cfd_csr_set_path(cfd_csr* a, int32_t fp32, int32_t path) {
  if (!a) {
    set_error("cfd_csr_set_path: null matrix");
    return CFD_ERR_STATE;
  }
  const DevMat& m = a->dev;
  const bool ok = path == CFD_PATH_AUTO || path == CFD_PATH_TIMED || path == CFD_PATH_SPLIT ||
                  (path == CFD_PATH_RECORD && m.all_compressed) || (path == CFD_PATH_X_STAGED && m.xs) ||
                  (path == CFD_PATH_SLICED && m.sl && fp32) || (path == CFD_PATH_DIAGONAL && m.dia);
  if (!ok) {
    set_error("SpMV pipeline %d not available for this matrix and precision (all blocks coded: %d, x staged: %d, "
              "sliced: %d, FP32 only; diagonals: %d)", path, (int)m.all_compressed, (int)m.xs, (int)m.sl,
              m.dia ? m.dia_n : 0);
    return CFD_ERR_CONFIG;
  }
  std::lock_guard<std::mutex> g(a->ctx->mu);
  m.path[fp32 ? 0 : 1] = (int8_t)path;
  return CFD_OK;
}

cfd_status cfd_layout_check(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* row_ptr, const int32_t* col,
                            const double* val, const double* x, double* y, cfd_layout_info* out) {
  return guarded("cfd_layout_check", [&]() -> cfd_status {
    CFD_TRY(validate_csr(nrows, ncols, nnz, row_ptr, col, nullptr));
    if ((nnz > 0 && !val) || (ncols > 0 && !x) || (nrows > 0 && !y)) {
      set_error("cfd_layout_check: null array");
      return CFD_ERR_DIM;
    }
    const HostCsr h = host_from(nrows, ncols, nnz, row_ptr, col, nullptr, val);
    const int tpr = threads_per_row(h.nnz(), h.nrows);
    const std::vector<int> blk = row_partition(h.rp.data(), h.nrows, tpr);
    HostLayout L;
    encode_layout(h, blk, L);
    std::string why;
    int64_t staged = 0;
    int maxw = 0;
    if (!check_layout(h, blk, L, x, y, &why, &staged, &maxw)) {
      set_error("layout check: %s", why.c_str());
      return CFD_ERR_STATE;
    }
    HostSliced S;
    const bool sliced = encode_sliced(h, tpr, L.base_mult, S);
    if (sliced && !check_sliced(h, L.base_mult, S, &why)) {
      set_error("sliced layout check: %s", why.c_str());
      return CFD_ERR_STATE;
    }
    HostDiagonal D;
    const bool diagonal = encode_diagonal(h, tpr, D);
    if (diagonal && !check_diagonal(h, D, x, &why)) {
      set_error("diagonal layout check: %s", why.c_str());
      return CFD_ERR_STATE;
    }
    if (out) {
      *out = cfd_layout_info{};
      out->blocks = (int64_t)blk.size() - 1;
      out->compressed_nnz = L.compressed_nnz;
      out->all_compressed = L.all_compressed ? 1 : 0;
      out->x_staged = L.xs ? 1 : 0;
      out->threads_per_row = tpr;
      out->max_windows = maxw;
      out->staged_x_entries = staged;
      out->sliced = sliced ? 1 : 0;
      out->sliced_slots = sliced ? S.slots : 0;
      out->diagonals = diagonal ? D.n : 0;
    }
    return CFD_OK;
  });
}

cfd_status cfd_csr_destroy(cfd_csr* a) {
  if (!a) return CFD_OK;
  cudaSetDevice(a->ctx->device);
  cudaStreamSynchronize(a->ctx->stream);
  devmat_free(a->dev);
  dfree(a->diag64);
  dfree(a->diag32);
  dfree(a->jinv64);
  dfree(a->jinv32);
  simple_free(a->simple);
  component_free(a->cblock);
  cfd_csr_destroy(a->tr);
  delete a;
  return CFD_OK;
}

cfd_status cfd_spmv(cfd_csr* a, const double* x, double* y) {
  return guarded("cfd_spmv", [&]() -> cfd_status {
    if (!a || !x || !y) return CFD_ERR_STATE;
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    CFD_TRY(spmv_fp64(a, x, y));
    return check_device_flag(a->ctx);
  });
}

cfd_status cfd_spmv_f32(cfd_csr* a, const float* x, float* y) {
  return guarded("cfd_spmv_f32", [&]() -> cfd_status {
    if (!a || !x || !y) return CFD_ERR_STATE;
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    CFD_TRY(spmv_fp32(a, x, y));
    return check_device_flag(a->ctx);
  });
}

void cfd_amg_config_default(cfd_amg_config* c) {
  // AMGConfig::default, multigrid/mod.rs:244-259 (smoother: damped Jacobi is the
  // device smoother; the reference default is Gauss-Seidel).
  c->max_levels = 10;
  c->coarsening = CFD_COARSEN_RUGE_STUEBEN;
  c->min_coarse_size = 50;
  c->interpolation = CFD_INTERP_CLASSICAL;
  c->smoother = CFD_SMOOTH_JACOBI;
  c->pre_smooth = 2;
  c->post_smooth = 2;
  c->relaxation = 1.0;
  c->strength_threshold = 0.25;
  c->coarse_solve = CFD_COARSE_SWEEPS;
  c->coarse_sweeps = 10;
  c->aggregate_size = 8;
  c->seed = 0;
  c->coarse_order = CFD_COARSE_ORDER_SELECTION;
  c->max_interp_points = 0;
}

static cfd_status check_amg_config(const cfd_amg_config* cfg) {
  if (cfg->max_levels < 1 || cfg->max_levels > 16 || cfg->smoother != CFD_SMOOTH_JACOBI ||
      cfg->pre_smooth < 0 || cfg->post_smooth < 0 || !(cfg->strength_threshold >= 0.0) ||
      !std::isfinite(cfg->relaxation) || cfg->coarsening < 0 || cfg->coarsening > 2 || cfg->interpolation < 0 ||
      cfg->interpolation > 2 || cfg->coarse_order < 0 || cfg->coarse_order > 1) {
    set_error("invalid AMG configuration");
    return CFD_ERR_CONFIG;
  }
  return CFD_OK;
}

// A hierarchy handle built by cfd_amg_setup_host has no context and no device data.
static cfd_status need_device_hierarchy(const cfd_amg* amg, const char* what) {
  if (!amg->ctx) {
    set_error("%s: the hierarchy was built on the host only (cfd_amg_setup_host)", what);
    return CFD_ERR_STATE;
  }
  return CFD_OK;
}

cfd_status cfd_amg_setup(cfd_csr* a, const cfd_amg_config* cfg, cfd_amg** out) {
  return guarded("cfd_amg_setup", [&]() -> cfd_status {
    if (!a || !cfg || !out) return CFD_ERR_STATE;
    *out = nullptr;
    CFD_TRY(check_amg_config(cfg));
    if (a->host.nrows != a->host.ncols) {
      set_error("AMG needs a square matrix");
      return CFD_ERR_DIM;
    }
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    auto t0 = std::chrono::steady_clock::now();
    cfd_amg* amg = new cfd_amg;
    OnUnwind release([&] {
      amg_free_device(amg);
      delete amg;
    });
    amg->ctx = a->ctx;
    amg->cfg = *cfg;
    amg->host = build_hierarchy(a->host, *cfg);
    cfd_status s = amg_upload(amg, false);
    if (s != CFD_OK) {
      amg_free_device(amg);
      delete amg;
      return s;
    }
    amg->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = amg;
    return CFD_OK;
  });
}

cfd_status cfd_amg_setup_host(int64_t n, const int64_t* row_ptr, const int64_t* col, const double* val,
                              const cfd_amg_config* cfg, cfd_amg** out) {
  return guarded("cfd_amg_setup_host", [&]() -> cfd_status {
    if (!cfg || !out) return CFD_ERR_STATE;
    *out = nullptr;
    CFD_TRY(check_amg_config(cfg));
    if (n < 0 || !row_ptr) {
      set_error("invalid CSR arguments");
      return CFD_ERR_DIM;
    }
    const int64_t nnz = row_ptr[n];
    CFD_TRY(validate_csr(n, n, nnz, row_ptr, nullptr, col));
    if (nnz > 0 && !val) {
      set_error("null value array");
      return CFD_ERR_DIM;
    }
    auto t0 = std::chrono::steady_clock::now();
    cfd_amg* amg = new cfd_amg;
    OnUnwind release([&] { delete amg; });
    amg->cfg = *cfg;
    amg->host = build_hierarchy(host_from(n, n, nnz, row_ptr, nullptr, col, val), *cfg);
    amg->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = amg;
    return CFD_OK;
  });
}

cfd_status cfd_amg_recompute(cfd_amg* amg, cfd_csr* a) {
  return guarded("cfd_amg_recompute", [&]() -> cfd_status {
    if (!amg || !a) return CFD_ERR_STATE;
    if (amg->host.empty()) return CFD_ERR_STATE;
    CFD_TRY(need_device_hierarchy(amg, "cfd_amg_recompute"));
    if (a->host.nrows != amg->host[0].A.nrows || a->host.nnz() != amg->host[0].A.nnz()) {
      set_error("recompute needs the hierarchy's sparsity pattern");
      return CFD_ERR_DIM;
    }
    if (a->ctx != amg->ctx) {
      set_error("recompute: the matrix and the hierarchy belong to different contexts");
      return CFD_ERR_STATE;
    }
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    return amg_recompute_device(amg, a);
  });
}

cfd_status cfd_amg_apply(cfd_amg* amg, const double* r, double* z) {
  return guarded("cfd_amg_apply", [&]() -> cfd_status {
    if (!amg || !r || !z) return CFD_ERR_STATE;
    CFD_TRY(need_device_hierarchy(amg, "cfd_amg_apply"));
    std::lock_guard<std::mutex> g(amg->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(amg->ctx->device));
    CFD_TRY(amg_apply_fp64(amg, r, z));
    return check_device_flag(amg->ctx);
  });
}

cfd_status cfd_amg_set_path(cfd_amg* amg, int32_t fp32, int32_t path) {
  if (!amg) {
    set_error("cfd_amg_set_path: null handle");
    return CFD_ERR_STATE;
  }
  if (path < CFD_PATH_TIMED || path > CFD_PATH_DIAGONAL) {
    set_error("cfd_amg_set_path: unknown pipeline %d", path);
    return CFD_ERR_CONFIG;
  }
  CFD_TRY(need_device_hierarchy(amg, "cfd_amg_set_path"));
  std::lock_guard<std::mutex> g(amg->ctx->mu);
  for (DevLevel& L : amg->dev)
    for (DevMat* m : {&L.A, &L.P, &L.R}) {
      int q = path;  // an ineligible request keeps the default rule for that operator
      if ((q == CFD_PATH_RECORD && !m->all_compressed) || (q == CFD_PATH_X_STAGED && !m->xs) ||
          (q == CFD_PATH_SLICED && !(m->sl && fp32)) || (q == CFD_PATH_DIAGONAL && !m->dia))
        q = CFD_PATH_AUTO;
      m->path[fp32 ? 0 : 1] = (int8_t)q;
    }
  return CFD_OK;
}

cfd_status cfd_amg_stats(const cfd_amg* amg, cfd_amg_stats_t* out) {
  if (!amg || !out) return CFD_ERR_STATE;
  std::memset(out, 0, sizeof(*out));
  out->num_levels = (int32_t)amg->host.size();
  double tot_nnz = 0, tot_rows = 0;
  for (size_t l = 0; l < amg->host.size(); ++l) {
    if (l < 16) {
      out->level_rows[l] = amg->host[l].A.nrows;
      out->level_nnz[l] = amg->host[l].A.nnz();
    }
    tot_nnz += (double)amg->host[l].A.nnz();
    tot_rows += (double)amg->host[l].A.nrows;
  }
  out->operator_complexity = tot_nnz / std::max<double>(1.0, (double)amg->host[0].A.nnz());
  out->grid_complexity = tot_rows / std::max<double>(1.0, (double)amg->host[0].A.nrows);
  out->setup_seconds = amg->setup_seconds;
  return CFD_OK;
}

cfd_status cfd_amg_level(const cfd_amg* amg, int level, int which, int64_t* nrows, int64_t* ncols, int64_t* nnz,
                         int64_t* row_ptr, int64_t* col, double* val) {
  return guarded("cfd_amg_level", [&]() -> cfd_status {
    if (!amg || level < 0 || level >= (int)amg->host.size() || which < 0 || which > 2) return CFD_ERR_DIM;
    if (which == 0 && val && amg->host_values_stale) {
      cfd_amg* mut = const_cast<cfd_amg*>(amg);  // the host mirror is a cache of the device values
      std::lock_guard<std::mutex> g(mut->ctx->mu);
      CFD_TRY_CUDA(cudaSetDevice(mut->ctx->device));
      CFD_TRY(amg_sync_host_values(mut));
    }
    const HostLevel& L = amg->host[level];
    if (which > 0 && level + 1 == (int)amg->host.size()) return CFD_ERR_DIM;
    const HostCsr& m = which == 0 ? L.A : (which == 1 ? L.P : L.R);
    if (nrows) *nrows = m.nrows;
    if (ncols) *ncols = m.ncols;
    if (nnz) *nnz = m.nnz();
    if (row_ptr) std::copy(m.rp.begin(), m.rp.end(), row_ptr);
    if (col)
      for (int64_t k = 0; k < m.nnz(); ++k) col[k] = m.ci[k];
    if (val) std::copy(m.v.begin(), m.v.end(), val);
    return CFD_OK;
  });
}

cfd_status cfd_amg_destroy(cfd_amg* amg) {
  if (!amg) return CFD_OK;
  if (amg->ctx) {
    cudaSetDevice(amg->ctx->device);
    cudaStreamSynchronize(amg->ctx->stream);
    amg_free_device(amg);
  }
  delete amg;
  return CFD_OK;
}

void cfd_solve_options_default(cfd_solve_options* o) {
  o->solver = CFD_SOLVER_CG;
  o->precond = CFD_PRECOND_JACOBI;
  o->precision = CFD_PRECISION_FP64;
  o->memory = CFD_MEMORY_HOST;
  o->inner_tolerance = 1e-4;
  o->max_outer = 20;
  o->check_every = 0;
  o->restart = 30;
}

// The solve arguments cfd_solve and cfd_adjoint share.
static cfd_status validate_solve(const cfd_csr* a, const cfd_solve_options* opt, const cfd_solver_config* cfg) {
  // convergence_policy (krylov.rs:123-139) rejects non-finite or negative
  // tolerances and a zero iteration budget at construction.
  if (!(cfg->tolerance >= 0.0) || !(cfg->relative_tolerance >= 0.0) || !std::isfinite(cfg->tolerance) ||
      !std::isfinite(cfg->relative_tolerance) || cfg->max_iterations <= 0) {
    set_error("invalid iterative solver configuration: tolerance %g, relative %g, max_iterations %lld",
              cfg->tolerance, cfg->relative_tolerance, (long long)cfg->max_iterations);
    return CFD_ERR_CONFIG;
  }
  if (opt->solver < 0 || opt->solver > 2 || opt->precond < 0 || opt->precond > 5 || opt->precision < 0 ||
      opt->precision > 1 || opt->memory < 0 || opt->memory > 1 || (opt->solver == CFD_SOLVER_GMRES && opt->restart < 1)) {
    set_error("invalid solve options");
    return CFD_ERR_CONFIG;
  }
  if (a->host.nrows != a->host.ncols) {
    set_error("Krylov solve needs a square matrix (%lld x %lld)", (long long)a->host.nrows,
              (long long)a->host.ncols);
    return CFD_ERR_DIM;
  }
  return CFD_OK;
}

// A's transpose as a matrix of its own context, formed on the host from A's
// current values (columns of each row ascending) and uploaded; its values are
// refreshed after A's change. Called with the context's lock held.
static cfd_status csr_transposed(cfd_csr* a, cfd_csr** out) {
  if (a->tr && a->tr_version == a->values_version) {
    *out = a->tr;
    return CFD_OK;
  }
  const HostCsr& h = a->host;
  HostCsr T;
  T.nrows = h.ncols;
  T.ncols = h.nrows;
  T.rp.assign(T.nrows + 1, 0);
  for (int64_t k = 0; k < h.nnz(); ++k) T.rp[h.ci[k] + 1]++;
  for (int64_t i = 0; i < T.nrows; ++i) T.rp[i + 1] += T.rp[i];
  T.ci.resize(h.nnz());
  T.v.resize(h.nnz());
  std::vector<int64_t> next(T.rp.begin(), T.rp.end() - 1);
  for (int64_t r = 0; r < h.nrows; ++r)
    for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) {
      const int64_t q = next[h.ci[k]]++;
      T.ci[q] = (int32_t)r;
      T.v[q] = h.v[k];
    }
  if (a->tr) {
    CFD_TRY(devmat_update_values(a->tr->dev, T.v.data(), T.nnz(), false, a->ctx->stream));
    a->tr->host.v = T.v;
    a->tr->values_version++;
    dfree(a->tr->diag64);
    dfree(a->tr->diag32);
    dfree(a->tr->jinv64);
    dfree(a->tr->jinv32);
    a->tr->jacobi_status = -1;
  } else {
    cfd_csr* t = new cfd_csr;
    t->ctx = a->ctx;
    t->host = std::move(T);
    cfd_status st = devmat_upload(t->dev, t->host, false, a->ctx->stream);
    if (st == CFD_OK) st = ensure_partials(a->ctx, t->dev.nblk);
    if (st != CFD_OK) {
      devmat_free(t->dev);
      delete t;
      return st;
    }
    a->tr = t;
  }
  a->tr_version = a->values_version;
  *out = a->tr;
  return CFD_OK;
}

cfd_status cfd_adjoint(cfd_csr* a, const cfd_solve_options* opt, cfd_amg* amg, const double* x, const double* g,
                       double* lambda, double* gvals, int32_t transpose, const cfd_solver_config* cfg,
                       cfd_solve_report* rep) {
  return guarded("cfd_adjoint", [&]() -> cfd_status {
    if (!a || !opt || !x || !g || !lambda || !cfg || !rep) {
      set_error("null argument to cfd_adjoint");
      return CFD_ERR_STATE;
    }
    CFD_TRY(validate_solve(a, opt, cfg));
    if (transpose && opt->precond != CFD_PRECOND_NONE && opt->precond != CFD_PRECOND_JACOBI) {
      set_error("cfd_adjoint: the transposed solve takes the Jacobi preconditioner or none (the AMG and "
                "saddle-point preconditioners were built for A)");
      return CFD_ERR_CONFIG;
    }
    cfd_solve_options o = *opt;
    o.memory = CFD_MEMORY_DEVICE;
    std::lock_guard<std::mutex> lk(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    cfd_csr* target = a;
    if (transpose) CFD_TRY(csr_transposed(a, &target));
    CFD_TRY(check_precond(target, o, amg));
    a->ctx->stats.reset();
    std::memset(rep, 0, sizeof(*rep));
    const int64_t n = a->host.nrows;
    if (n == 0) {
      rep->termination = CFD_TERM_INITIAL_RESIDUAL;
      return CFD_OK;
    }
    CFD_TRY_CUDA(cudaMemsetAsync(lambda, 0, n * sizeof(double), a->ctx->stream));
    if (o.precision == CFD_PRECISION_FP32_REFINE)
      CFD_TRY(solve_refine(target, o, amg, g, lambda, *cfg, *rep));
    else
      CFD_TRY(solve_fp64(target, o, amg, g, lambda, *cfg, *rep));
    if (gvals) CFD_TRY(pattern_outer_launch(a, lambda, x, 1.0, gvals));
    CFD_TRY_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return check_device_flag(a->ctx);
  });
}

cfd_status cfd_solve(cfd_csr* a, const cfd_solve_options* opt, cfd_amg* amg, const double* b, double* x,
                     const cfd_solver_config* cfg, cfd_solve_report* rep) {
  return guarded("cfd_solve", [&]() -> cfd_status {
    if (!a || !opt || !b || !x || !cfg || !rep) {
      set_error("null argument to cfd_solve");
      return CFD_ERR_STATE;
    }
    CFD_TRY(validate_solve(a, opt, cfg));
    std::lock_guard<std::mutex> g(a->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(a->ctx->device));
    CFD_TRY(check_precond(a, *opt, amg));
    a->ctx->stats.reset();
    std::memset(rep, 0, sizeof(*rep));
    if (a->host.nrows == 0) {
      rep->termination = CFD_TERM_INITIAL_RESIDUAL;
      return CFD_OK;
    }
    if (opt->precision == CFD_PRECISION_FP32_REFINE)
      CFD_TRY(solve_refine(a, *opt, amg, b, x, *cfg, *rep));
    else
      CFD_TRY(solve_fp64(a, *opt, amg, b, x, *cfg, *rep));
    return check_device_flag(a->ctx);
  });
}

cfd_status cfd_last_kernel_stats(cfd_context* ctx, cfd_kernel_stats* out) {
  if (!ctx || !out) return CFD_ERR_STATE;
  out->launches = ctx->stats.launches;
  out->spmv_launches = ctx->stats.spmv_launches;
  out->spmv_bytes = ctx->stats.spmv_bytes;
  return CFD_OK;
}

}  // extern "C"
