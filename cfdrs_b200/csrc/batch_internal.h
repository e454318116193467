// Internal state of a batched small-system solve (cfd_batch), shared by the
// batched Jacobi-PCG (batch.cu) and the device network assembly (network.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "cfdgpu.h"

namespace cfd {

constexpr int kBatchMaxRows = 2048;  // rows per system held in shared memory
constexpr int kBatchMaxNnz = 8192;   // nonzeros per system held in shared memory
constexpr int kBuckets = 4;
constexpr int kBucketRows[kBuckets] = {64, 256, 1024, kBatchMaxRows};

struct BatchParams {
  double tol_abs, tol_rel, inner_tol;
  int32_t max_iter, max_outer;
};

struct NetworkPlanDev;  // network.cu

// Checks a batch layout (offsets, row_ptr, local columns) without touching
// any device state; see cfd_batch_create.
cfd_status batch_validate(int32_t num_systems, const int64_t* sys_row_offsets, const int64_t* row_ptr,
                          const int32_t* col, const double* val);
// Builds a batch from a layout batch_validate accepted.
cfd_status batch_build(cfd_context* ctx, int32_t num_systems, const int64_t* sys_row_offsets,
                       const int64_t* row_ptr, const int32_t* col, const double* val, cfd_batch** out);
// Releases the network part of a batch (network.cu).
void network_plan_free(NetworkPlanDev* p);

}  // namespace cfd

struct cfd_batch {
  cfd_context* ctx = nullptr;
  int nsys = 0;
  int64_t rows = 0, nnz = 0;
  std::vector<int> h_sys_row;
  int* sys_row = nullptr;
  int* rp = nullptr;
  int* col = nullptr;
  double* v64 = nullptr;
  float* v32 = nullptr;
  double* x = nullptr;
  double* b = nullptr;
  int* term = nullptr;
  int* iters = nullptr;
  double* resid = nullptr;
  int* order = nullptr;  // systems of each bucket, largest first, bucket after bucket
  int bucket_begin[cfd::kBuckets + 1] = {};
  int bucket_nmax[cfd::kBuckets] = {}, bucket_zmax[cfd::kBuckets] = {};
  int threads[2][cfd::kBuckets] = {{32, 64, 128, 256}, {32, 64, 128, 256}};  // [precision][bucket], per system
  int groups[2][cfd::kBuckets] = {{1, 1, 1, 1}, {1, 1, 1, 1}};  // systems per CTA of the Jacobi-PCG kernel
  bool tuned[2] = {false, false};
  unsigned* queues = nullptr;  // one ticket per bucket
  cfd::BatchParams* params = nullptr;
  cfd::BatchParams* h_params = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  // Right-hand side in `b` assembled on the device (cfd_batch_assemble) and
  // not yet replaced by a solve's own b: a solve may pass b = NULL.
  bool rhs_resident = false;
  // False for a network batch before its first assembly and after one that
  // failed: its values are not a matrix then.
  bool values_valid = true;
  cfd::NetworkPlanDev* net = nullptr;  // network batches only
  std::vector<int> h_order;            // `order` on the host
  // An entry that is finite in FP64 but not in FP32: FP32_REFINE solves refuse the batch.
  bool f32_out_of_range = false;
  // cfd_batch_linear_system_solve (batch_ls.cu): per-system method and path,
  // a device list of systems, its parameter block and queues, and the dense
  // LU scratch (one n x n slot per CTA, grown on demand).
  int* ls_method = nullptr;
  int* ls_path = nullptr;
  int* ls_list = nullptr;
  double* ls_params = nullptr;
  unsigned* ls_queue = nullptr;
  double* ls_scratch = nullptr;
  size_t ls_scratch_elems = 0;
  int* ls_pivot = nullptr;   // per system: the dense fast path's pivot guard fired
  int64_t ls_pivoted = 0;    // systems handed to the pivoting dense solve, all calls
};
