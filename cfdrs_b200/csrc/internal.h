// Internal declarations of libcfdgpu (host + device). Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "cfdgpu.h"

namespace cfd {

struct SimpleDev;     // simple.h
struct ComponentDev;  // simple.h

// Error message of the last failure on this thread (cfd_last_error()).
void set_error(const char* fmt, ...);

// Runs an entry point's body with C++ exceptions turned into status codes: a
// host allocation that fails (std::bad_alloc from a std::vector) must not
// unwind into a C, Rust or ctypes caller.
template <typename F>
cfd_status guarded(const char* what, F&& body) noexcept {
  try {
    return body();
  } catch (const std::bad_alloc&) {
    set_error("%s: host memory allocation failed", what);
    return CFD_ERR_ALLOC;
  } catch (const std::exception& e) {
    set_error("%s: %s", what, e.what());
    return CFD_ERR_STATE;
  } catch (...) {
    set_error("%s: unexpected exception", what);
    return CFD_ERR_STATE;
  }
}

// Runs `undo` when the scope is left by an exception, so that a half-built
// handle is released before guarded() turns the exception into a status.
// Returns by status code do not trigger it (those paths release for themselves).
template <typename F>
class OnUnwind {
 public:
  explicit OnUnwind(F f) : f_(f), depth_(std::uncaught_exceptions()) {}
  ~OnUnwind() {
    if (std::uncaught_exceptions() > depth_) f_();
  }
  OnUnwind(const OnUnwind&) = delete;
  OnUnwind& operator=(const OnUnwind&) = delete;

 private:
  F f_;
  int depth_;
};

#define CFD_TRY_CUDA(...)                                                                           \
  do {                                                                                              \
    cudaError_t e_ = (__VA_ARGS__);                                                                 \
    if (e_ != cudaSuccess) {                                                                        \
      ::cfd::set_error("%s: %s (%s:%d)", #__VA_ARGS__, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return CFD_ERR_CUDA;                                                                          \
    }                                                                                               \
  } while (0)

#define CFD_TRY(...)                  \
  do {                                \
    cfd_status s_ = (__VA_ARGS__);    \
    if (s_ != CFD_OK) return s_;      \
  } while (0)

// Row-blocked CSR SpMV geometry: 256 consumer threads per CTA, row blocks of
// at most kRowsPerBlock rows (two per consumer thread or row group) and
// kNnzCap nonzeros staged in shared memory; a row with more than kNnzCap
// nonzeros is a block of its own (block-stride reduction).
constexpr int kThreads = 256;
constexpr int kRowsPerThread = 2;
constexpr int kRowsPerBlock = kThreads * kRowsPerThread;
constexpr int kNnzCap = 4096;
// x staging: a dictionary-coded block whose columns fall in at most kXsMaxWin
// windows of kXsCap entries in total reads x from shared memory (the windows
// are bulk-copied with the block) instead of gathering it from global memory.
constexpr int kXsCap = 4096;
constexpr int kXsMaxWin = 8;
// Index record of a dictionary-coded block, moved by one bulk copy: row
// offsets relative to the block's first nonzero (uint16, rows + 1 of them),
// the one-byte codes, the offset dictionary (int32) and, for x-staged
// matrices, the code -> staged-x displacement table E (int32); each part is
// 16-byte aligned.
struct BlockRecord {
  int rp_bytes, code_bytes, dict_bytes, e_bytes;
  __host__ __device__ static BlockRecord of(int rows, int nnz, int nd, bool with_e) {
    const int d = (4 * nd + 15) & ~15;
    return {(2 * (rows + 1) + 15) & ~15, (nnz + 15) & ~15, d, with_e ? d : 0};
  }
  __host__ __device__ int bytes() const { return rp_bytes + code_bytes + dict_bytes + e_bytes; }
};
constexpr int kRecordCap = ((2 * (kRowsPerBlock + 1) + 15) & ~15) + kNnzCap + 2 * 4 * 256;
// Grid of the streaming vector kernels: 148 SMs x 8 resident CTAs.
constexpr int kVecGrid = 148 * 8;
// Device-side scratch for two-stage reductions (per-CTA partials, up to 4 values).
constexpr int kMaxRed = 4;
// Diagonals of the diagonal SpMV layout at most (DevMat::dia), and the
// largest threads-per-row whose summation order its kernels reproduce.
constexpr int kDiaMax = 32;
constexpr int kDiaMaxTpr = 2;
// Device ordinals covered by the per-device launch-attribute caches.
constexpr int kLaunchCacheDevices = 64;

// Host CSR (int64 offsets, int32 columns), the form AMG setup works on.
struct HostCsr {
  int64_t nrows = 0, ncols = 0;
  std::vector<int64_t> rp;
  std::vector<int32_t> ci;
  std::vector<double> v;
  int64_t nnz() const { return (int64_t)ci.size(); }
};

// A caller's CSR (int64 row offsets; int32 or int64 columns, one of c32/c64),
// checked without reading past a bound an earlier check established: sizes,
// row_ptr from 0 to nnz and non-decreasing, columns in range and strictly
// increasing within a row.
cfd_status validate_csr(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* rp, const int32_t* c32,
                        const int64_t* c64);
// Host copy of a CSR validate_csr accepted.
HostCsr host_from(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* rp, const int32_t* c32,
                  const int64_t* c64, const double* v);

// Device CSR. Indices are int32 (nnz < 2^31); values are kept in FP64 and,
// once asked for, an FP32 copy sharing the same index arrays.
struct DevMat {
  int64_t nrows = 0, ncols = 0, nnz = 0;
  int* rp = nullptr;
  int* col = nullptr;
  double* v64 = nullptr;
  float* v32 = nullptr;
  int* blk = nullptr;  // row-block partition, nblk + 1 entries
  int4* desc = nullptr;  // per row block {r0, r1, k0, k1}
  // Column compression: a block whose column offsets (col - base(row), base =
  // row * ncols / nrows) take at most 256 distinct values stores one byte per
  // nonzero indexing the block's offset dictionary; other blocks stay int32.
  uint8_t* code = nullptr;  // per-nonzero dictionary index (compressed blocks)
  int* dict = nullptr;      // concatenated per-block offset dictionaries
  int2* dict_desc = nullptr;  // per block {first entry, entries}; 0 entries = int32 columns
  int64_t compressed_nnz = 0;
  bool all_compressed = false;  // every staged block is dictionary-coded
  // base(row) = (row * base_mult) >> 20 with base_mult = (ncols << 20) / nrows:
  // the reference point of the column offsets (row itself for square matrices).
  uint64_t base_mult = 1u << 20;
  // Block records (all_compressed matrices): rec + 16 * roff[b] is block b's
  // BlockRecord, the staging unit of the codes-only and x-staged pipelines.
  uint8_t* rec = nullptr;
  int* roff = nullptr;
  // x staging (all blocks dictionary-coded and within kXsCap / kXsMaxWin).
  // Windows are 4-entry aligned column ranges [src, src + len) placed one after
  // another in shared memory; a window that would run past ncols copies up to
  // the last full 4-entry group and its `tail` (< 4) entries are read one by
  // one. The x entry of a nonzero with code q in row r sits at shared entry
  // base(r) - base(r0) + E[q], E being the table in the block's record.
  int4* xwin = nullptr;  // per block kXsMaxWin slots of {src, len}, two per int4
  // per block {windows | tail << 16, zero-offset code or -1, record offset / 16, entries copied}
  int4* xdesc = nullptr;
  bool xs = false;
  // SpMV pipeline per precision ([0] FP32, [1] FP64): a cfd_spmv_path value;
  // CFD_PATH_TIMED is replaced by the fastest after timing (Launcher::tune).
  mutable int8_t path[2] = {-1, -1};
  int nblk = 0;
  int tpr = 1;         // threads cooperating on one row (power of two, <= 32)
  // Sliced layout (FP32 SpMV only; HostSliced): slice offsets, codes,
  // dictionaries, the CSR entry of every slot and the slot-major FP32 values,
  // gathered from v32 before the first sliced SpMV after v32 changed.
  bool sl = false;
  int64_t sl_slices = 0, sl_slots = 0;
  int* sl_off = nullptr;
  uint8_t* sl_code = nullptr;
  int* sl_dict = nullptr;
  int* sl_doff = nullptr;
  int* sl_src = nullptr;
  float* sl_v32 = nullptr;
  mutable bool sl_stale = true;
  // Diagonal layout (HostDiagonal): values stored diagonal-major, ndia arrays
  // of dia_ld entries (0 where a row has no entry on that diagonal), refilled
  // from v64 / v32 before the first diagonal SpMV after the values changed;
  // for tpr = 2 the per-row lane bits of the diagonals (dia_mask).
  bool dia = false;
  int dia_n = 0, dia_main = -1;
  int dia_off[kDiaMax] = {};
  int64_t dia_ld = 0;
  double* dia64 = nullptr;
  float* dia32 = nullptr;
  uint32_t* dia_mask = nullptr;
  mutable bool dia_stale = true;
};

// Sliced layout (sliced.cpp, k_spmv_sl): rows in slices of kSlRows stored
// slot-major, one dictionary of column offsets per kSlChunkSlices slices.
constexpr int kSlRows = 32;
constexpr int kSlChunkSlices = 16;
constexpr int kSlMaxWidth = 32;
constexpr int kSlPadCode = 255;
constexpr double kSlMaxPadding = 1.15;
struct HostSliced {
  int64_t nslices = 0, slots = 0;
  std::vector<int> off;       // nslices + 1 slot offsets (multiples of kSlRows)
  std::vector<uint8_t> code;  // per slot, kSlPadCode for padding (slots + 16)
  std::vector<int> dict;      // concatenated chunk dictionaries
  std::vector<int> doff;      // chunk dictionary offsets
  std::vector<int> src;       // per slot: CSR entry, -1 for padding
};
bool encode_sliced(const HostCsr& h, int tpr, uint64_t base_mult, HostSliced& S);
bool check_sliced(const HostCsr& h, uint64_t base_mult, const HostSliced& S, std::string* why);

// Diagonal layout (diagonal.cpp, k_spmv_dia, k_spmv_dia_gen): a square matrix
// with at most kDiaMaxTpr threads per row whose entries lie on at most kDiaMax
// diagonals (column - row), stored as dense diagonals with at most
// kDiaMaxFill x nnz slots.
constexpr double kDiaMaxFill = 1.30;
struct HostDiagonal {
  int n = 0;          // diagonals, offsets ascending
  int main = -1;      // index of offset 0, -1 when the main diagonal is empty
  int off[kDiaMax] = {};
  int64_t ld = 0;     // entries per stored diagonal (rows rounded up to 32)
  int tpr = 1;
  // tpr = 2: bit d of row r set when (r, r + off[d]) is stored at an odd
  // position among the row's stored entries (the row group's second thread adds it)
  std::vector<uint32_t> mask;
};
bool encode_diagonal(const HostCsr& h, int tpr, HostDiagonal& D);
// Evaluates y = A x through the diagonal layout in the device kernel's order
// and compares it bit for bit with the CSR row sums in the order of the other
// pipelines for that threads-per-row (each thread of a row group sums every
// tpr-th stored entry with fused multiply-adds, then the butterfly).
bool check_diagonal(const HostCsr& h, const HostDiagonal& D, const double* x, std::string* why);

// SpMV pipeline that an SpMV of precision p ([0] FP32, [1] FP64) runs: the
// setting, with CFD_PATH_AUTO resolved to RECORD for FP32 and X_STAGED for
// FP64 one-thread rows (SPLIT for other FP64 matrices), as measured fastest on
// the 256^3 AMG hierarchy, and ineligible pipelines stepped down. CFD_PATH_TIMED
// is returned as is (the launcher times the pipelines first).
inline int spmv_path(const DevMat& m, int p) {
  int path = m.path[p];
  if (path == CFD_PATH_TIMED) return path;
  if (path == CFD_PATH_SLICED && (p != 0 || !m.sl)) path = p == 0 ? CFD_PATH_RECORD : CFD_PATH_AUTO;
  if (path == CFD_PATH_DIAGONAL && !m.dia) path = CFD_PATH_AUTO;
  if (path == CFD_PATH_AUTO && m.dia) path = CFD_PATH_DIAGONAL;
  if (path == CFD_PATH_AUTO) path = p == 0 ? CFD_PATH_RECORD : (m.xs && m.tpr == 1 ? CFD_PATH_X_STAGED : CFD_PATH_SPLIT);
  if (path == CFD_PATH_X_STAGED && !m.xs) path = CFD_PATH_RECORD;
  if (path == CFD_PATH_RECORD && !m.all_compressed) path = CFD_PATH_SPLIT;
  return path;
}

// Host image of DevMat's compression and x-staging arrays (layout.cpp).
struct HostLayout {
  uint64_t base_mult = 1u << 20;
  std::vector<uint8_t> code;  // nnz + 16
  std::vector<int> dict;
  std::vector<int2> dict_desc;
  int64_t compressed_nnz = 0;
  bool all_compressed = false;
  std::vector<uint8_t> rec;   // BlockRecords (all_compressed)
  std::vector<int> roff;      // per block record offset / 16
  std::vector<int> xe;        // code -> staged-x displacement (dictionary layout)
  std::vector<int4> xwin, xdesc;
  bool xs = false;
};
void encode_layout(const HostCsr& h, const std::vector<int>& blk, HostLayout& L);
bool check_layout(const HostCsr& h, const std::vector<int>& blk, const HostLayout& L, const double* x, double* y,
                  std::string* why, int64_t* staged_entries, int* max_windows);

cfd_status devmat_upload(DevMat& m, const HostCsr& h, bool want32, cudaStream_t s);
cfd_status devmat_update_values(DevMat& m, const double* v, int64_t nnz, bool want32, cudaStream_t s);
cfd_status devmat_ensure32(DevMat& m, cudaStream_t s);
void devmat_free(DevMat& m);
std::vector<int> row_partition(const int64_t* rp, int64_t nrows, int tpr);
int threads_per_row(int64_t nnz, int64_t nrows);

// Scalars of one Krylov recurrence, resident on the device so that the
// iteration runs without host round trips; the host polls `done`.
struct DevState {
  double rho, alpha, beta, omega;
  double pq, rr, rnorm, threshold;
  double rnorm0, rhat_v, ts, tt;
  double tol_abs, tol_rel, spare0, spare1;
  int32_t iter, max_iter, done, term;
};

struct KernelStats {
  int64_t launches = 0;
  int64_t spmv_launches = 0;
  int64_t xs_launches = 0;  // SpMV launches on the x-staged pipeline
  double spmv_bytes = 0.0;
  void reset() { *this = KernelStats(); }
};

}  // namespace cfd

struct cfd_context {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  double* partials = nullptr;      // kMaxRed * max grid
  unsigned* counter = nullptr;     // last-CTA ticket of the two-stage reduction
  int partial_capacity = 0;        // CTAs covered by `partials`
  cfd::DevState* state = nullptr;  // two states: [0] outer/FP64, [1] inner
  cfd::DevState* h_state = nullptr;  // pinned mirror
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_switch = nullptr;  // orders the old stream before the new one on a stream switch
  int* err = nullptr;    // set by a kernel whose bounded wait ran out
  int* h_err = nullptr;  // pinned mirror
  int num_sms = 148;
  // CG / Jacobi-PCG of small systems as one thread-block-cluster launch
  // (cluster_pcg.cu) where the system fits; cfd_context_set_cluster_solve
  bool cluster_solve = true;
  cfd::KernelStats stats;
  std::mutex mu;
};

struct cfd_csr {
  cfd_context* ctx = nullptr;
  cfd::HostCsr host;
  cfd::DevMat dev;
  double* diag64 = nullptr;
  float* diag32 = nullptr;
  double* jinv64 = nullptr;  // DiagJacobi inverse diagonal (identity for |d| <= eps)
  float* jinv32 = nullptr;
  int jacobi_status = -1;    // -1 unknown, 0 ok, 1 non-finite diagonal
  // Saddle-point split (cfd_saddle_setup): velocity count, or -1 when not
  // set up; the SIMPLE and block-diagonal arrays are rebuilt from the host
  // values after a value update.
  int64_t simple_nv = -1;
  cfd::SimpleDev* simple = nullptr;
  bool simple_stale = false;
  // Component-block split (cfd_component_block_setup): velocity count or -1,
  // the stabilization tolerance, and the arrays (rebuilt after a value update).
  int64_t cblock_nv = -1;
  double cblock_pivot_tolerance = 1e-12;
  cfd::ComponentDev* cblock = nullptr;
  bool cblock_stale = false;
  // Grid size n of the 2-D Darcy pattern the matrix was checked against
  // (cfd_darcy2d_*), -1 before the first check.
  int64_t darcy_n = -1;
  // Value updates so far, and the transpose (cfd_adjoint with transpose != 0),
  // formed from the values of update tr_version.
  uint64_t values_version = 0;
  cfd_csr* tr = nullptr;
  uint64_t tr_version = 0;
};

namespace cfd {
cfd_status ensure_partials(cfd_context* ctx, int blocks);
// Reads the device error flag; a set flag (a bounded wait ran out) is reported
// as CFD_ERR_TIMEOUT and the flag and reduction ticket are reset.
cfd_status check_device_flag(cfd_context* ctx);
cfd_status ensure_diagonals(cfd_csr* a);
// g_e = -scale * lambda[row(e)] * x[col(e)] over A's pattern, on the context stream.
cfd_status pattern_outer_launch(cfd_csr* a, const double* lambda, const double* x, double scale, double* g);
// Whole CG / Jacobi-PCG solve in one thread-block cluster (cluster_pcg.cu):
// *ok = false (nothing launched) when the system does not fit.
cfd_status cluster_pcg_solve(cfd_context* ctx, const DevMat& m, const double* jinv, const double* b, double* x,
                             DevState* st, bool* ok);
}  // namespace cfd
