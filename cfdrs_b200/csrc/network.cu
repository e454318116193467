// Device assembly of a batch of Kirchhoff networks, so that a Picard loop
// (crates/cfd-1d/src/solver/core/network_solver.rs:289-340: assemble_into,
// then solve_with_initial_guess from the last iterate) re-assembles and
// re-solves from new conductances without the matrix crossing PCIe.
//
// The pattern step runs once on the host (build_network_plan); the value step
// is one kernel over the batch's edges (validity), CSR slots (values, FP64 and
// the FP32 copy the refined solve reads) and rows (right-hand side), each a
// gather in a fixed order: no atomics, so the result is the same every run and
// equals the host check (cfd_network_assemble_host) bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <mutex>
#include <vector>

#include "batch_internal.h"
#include "internal.h"
#include "network.h"

namespace cfd {

struct NetworkPlanDev {
  int64_t edges = 0;
  int32_t* slot_ptr = nullptr;
  int32_t* slot_src = nullptr;
  int32_t* rhs_ptr = nullptr;
  int32_t* rhs_edge = nullptr;
  int32_t* rhs_node = nullptr;
  int8_t* fixed = nullptr;
  double* fixed_value = nullptr;
  double* g = nullptr;  // staging for conductances given in host memory
  double* q = nullptr;  // staging for Neumann sources given in host memory
  int* bad = nullptr;    // [0] smallest rejected edge (>= edges when none); [1] non-finite flags
  int* h_bad = nullptr;  // pinned mirror of both

  NetworkView view() const { return {slot_ptr, slot_src, rhs_ptr, rhs_edge, rhs_node, fixed, fixed_value}; }
};

void network_plan_free(NetworkPlanDev* p) {
  if (!p) return;
  for (void* d : {(void*)p->slot_ptr, (void*)p->slot_src, (void*)p->rhs_ptr, (void*)p->rhs_edge,
                  (void*)p->rhs_node, (void*)p->fixed, (void*)p->fixed_value, (void*)p->g, (void*)p->q,
                  (void*)p->bad})
    if (d) cudaFree(d);
  if (p->h_bad) cudaFreeHost(p->h_bad);
  delete p;
}

namespace {

constexpr int kAsmThreads = 256;

// bad[0]: smallest edge with a rejected conductance; bad[1]: bit 0 a
// non-finite matrix entry, bit 1 a non-finite right-hand side, bit 2 a finite
// entry beyond the FP32 range (its FP32 copy is infinite: FP64 solves only).
__global__ void k_network_assemble(NetworkView V, int64_t edges, int64_t nnz, int64_t rows,
                                   const double* __restrict__ g, const double* __restrict__ q, double* v64,
                                   float* v32, double* b, int* bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t e = t0; e < edges; e += stride)
    if (!net_conductance_ok(g[e])) atomicMin(bad, (int)e);
  for (int64_t k = t0; k < nnz; k += stride) {
    const double v = net_slot_value(V, k, g);
    v64[k] = v;
    const float f = (float)v;
    v32[k] = f;
    if (!isfinite(v))
      atomicOr(bad + 1, 1);
    else if (!isfinite(f))
      atomicOr(bad + 1, 4);
  }
  for (int64_t r = t0; r < rows; r += stride) {
    const double br = net_rhs_value(V, r, g, q);
    b[r] = br;
    if (!isfinite(br)) atomicOr(bad + 1, 2);
  }
}

template <typename T>
cfd_status upload(T** d, const std::vector<T>& h, cudaStream_t s) {
  if (cudaMalloc((void**)d, std::max<size_t>(h.size(), 1) * sizeof(T)) != cudaSuccess) {
    *d = nullptr;
    set_error("cudaMalloc failed for a network plan array of %zu elements", h.size());
    return CFD_ERR_ALLOC;
  }
  if (!h.empty()) CFD_TRY_CUDA(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return CFD_OK;
}

cfd_status bad_conductance(const char* what, int64_t e, double g) {
  set_error("%s: %s conductance %g at edge %lld (matrix_assembly.rs:191-203)", what,
            std::isfinite(g) ? "non-positive" : "non-finite", g, (long long)e);
  return CFD_ERR_CONFIG;
}

// validate_linear_system (solver_detection.rs:66-93): the assembled matrix and
// right-hand side must be finite (a Neumann source or fixed pressure that is
// not, or a conductance sum that overflows).
cfd_status nonfinite_system(const char* what, int flags) {
  set_error("%s: %s", what, (flags & 1) ? "assembled matrix has a non-finite entry (solver_detection.rs:66-93)"
                                        : "RHS contains non-finite entries (solver_detection.rs:84-93)");
  return CFD_ERR_NONFINITE;
}

}  // namespace

cfd_status build_network_plan(int32_t nsys, const int64_t* node_off, const int64_t* edge_off, const int32_t* ei,
                              const int32_t* ej, const int8_t* fixed, const double* fixed_value, NetworkPlan& P) {
  if (nsys < 0 || !node_off || !edge_off) {
    set_error("network batch: invalid arguments");
    return CFD_ERR_STATE;
  }
  const int64_t rows = node_off[nsys], edges = edge_off[nsys];
  if (node_off[0] != 0 || edge_off[0] != 0 || rows < 0 || rows >= INT32_MAX || edges < 0 ||
      edges > kMaxNetworkEdges) {
    set_error("network batch: node and edge offsets must start at 0 and end at counts that fit (at most %lld edges)",
              (long long)kMaxNetworkEdges);
    return CFD_ERR_DIM;
  }
  if ((edges > 0 && (!ei || !ej)) || (rows > 0 && (!fixed || !fixed_value))) {
    set_error("network batch: null edge or node array");
    return CFD_ERR_DIM;
  }
  for (int32_t s = 0; s < nsys; ++s) {
    const int64_t r0 = node_off[s], r1 = node_off[s + 1], e0 = edge_off[s], e1 = edge_off[s + 1];
    if (r1 < r0 || r1 > rows || e1 < e0 || e1 > edges) {
      set_error("network batch: offsets decrease or pass their totals at network %d", s);
      return CFD_ERR_DIM;
    }
    if (r1 - r0 > kBatchMaxRows) {
      set_error("network batch: network %d has %lld nodes; the batched solver holds at most %d", s,
                (long long)(r1 - r0), kBatchMaxRows);
      return CFD_ERR_DIM;
    }
    for (int64_t e = e0; e < e1; ++e) {
      if (ei[e] < 0 || ei[e] >= r1 - r0 || ej[e] < 0 || ej[e] >= r1 - r0) {
        set_error("network batch: edge %lld of network %d joins nodes %d and %d outside its %lld nodes", (long long)e,
                  s, ei[e], ej[e], (long long)(r1 - r0));
        return CFD_ERR_DIM;
      }
      if (ei[e] == ej[e]) {
        set_error("network batch: self-loop edge %lld at node %d of network %d (matrix_assembly.rs:184-189)",
                  (long long)e, ei[e], s);
        return CFD_ERR_CONFIG;
      }
    }
  }
  P = NetworkPlan();
  P.nsys = nsys;
  P.rows = rows;
  P.edges = edges;
  P.sys_row.assign(node_off, node_off + nsys + 1);
  P.fixed.assign(fixed, fixed + rows);
  for (int8_t& f : P.fixed) f = f ? 1 : 0;
  P.fixed_value.assign(fixed_value, fixed_value + rows);
  P.row_ptr.assign(rows + 1, 0);
  P.slot_ptr.push_back(0);
  P.rhs_ptr.assign(rows + 1, 0);
  struct Push {
    int32_t r, c, code;
  };
  struct Elim {
    int32_t r, e, node;
  };
  std::vector<Push> coo;
  std::vector<Elim> elim;
  for (int32_t s = 0; s < nsys; ++s) {
    const int64_t r0 = node_off[s], n = node_off[s + 1] - r0;
    coo.clear();
    elim.clear();
    for (int64_t e = edge_off[s]; e < edge_off[s + 1]; ++e) {
      const int32_t i = ei[e], j = ej[e], code = (int32_t)(2 * e);
      const bool fi = P.fixed[r0 + i] != 0, fj = P.fixed[r0 + j] != 0;
      if (!fi && !fj) {
        coo.push_back({i, i, code});
        coo.push_back({j, j, code});
        coo.push_back({i, j, code + 1});
        coo.push_back({j, i, code + 1});
      } else if (fi && !fj) {
        coo.push_back({j, j, code});
        elim.push_back({j, (int32_t)e, (int32_t)(r0 + i)});
      } else if (!fi && fj) {
        coo.push_back({i, i, code});
        elim.push_back({i, (int32_t)e, (int32_t)(r0 + j)});
      }
    }
    for (int32_t k = 0; k < (int32_t)n; ++k)
      if (P.fixed[r0 + k]) coo.push_back({k, k, kUnitSlot});
    std::stable_sort(coo.begin(), coo.end(),
                     [](const Push& a, const Push& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
    std::stable_sort(elim.begin(), elim.end(), [](const Elim& a, const Elim& b) { return a.r < b.r; });
    for (size_t q = 0; q < coo.size();) {
      size_t t = q;
      while (t < coo.size() && coo[t].r == coo[q].r && coo[t].c == coo[q].c) P.slot_src.push_back(coo[t++].code);
      P.col.push_back(coo[q].c);
      P.slot_ptr.push_back((int32_t)P.slot_src.size());
      P.row_ptr[r0 + coo[q].r + 1]++;
      q = t;
    }
    for (const Elim& x : elim) {
      P.rhs_edge.push_back(x.e);
      P.rhs_node.push_back(x.node);
      P.rhs_ptr[r0 + x.r + 1]++;
    }
    if ((int64_t)P.slot_src.size() >= INT32_MAX || (int64_t)P.col.size() >= INT32_MAX) {
      set_error("network batch: more than %d matrix entries", INT32_MAX);
      return CFD_ERR_DIM;
    }
  }
  for (int64_t r = 0; r < rows; ++r) {
    P.row_ptr[r + 1] += P.row_ptr[r];
    P.rhs_ptr[r + 1] += P.rhs_ptr[r];
  }
  return CFD_OK;
}

}  // namespace cfd

using namespace cfd;

extern "C" {

cfd_status cfd_batch_create_networks(cfd_context* ctx, int32_t num_systems, const int64_t* node_offsets,
                                     const int64_t* edge_offsets, const int32_t* edge_i, const int32_t* edge_j,
                                     const int8_t* fixed, const double* fixed_value, cfd_batch** out) {
  return guarded("cfd_batch_create_networks", [&]() -> cfd_status {
    if (!out) {
      set_error("cfd_batch_create_networks: null output handle");
      return CFD_ERR_STATE;
    }
    *out = nullptr;
    NetworkPlan P;
    CFD_TRY(build_network_plan(num_systems, node_offsets, edge_offsets, edge_i, edge_j, fixed, fixed_value, P));
    const std::vector<double> zeros(P.col.size(), 0.0);  // values come with the first assembly
    CFD_TRY(batch_validate(num_systems, P.sys_row.data(), P.row_ptr.data(), P.col.data(), zeros.data()));
    if (!ctx) {
      set_error("cfd_batch_create_networks: null context");
      return CFD_ERR_STATE;
    }
    cfd_batch* bt = nullptr;
    CFD_TRY(batch_build(ctx, num_systems, P.sys_row.data(), P.row_ptr.data(), P.col.data(), zeros.data(), &bt));
    OnUnwind release([&] { cfd_batch_destroy(bt); });
    std::lock_guard<std::mutex> g(ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    NetworkPlanDev* d = new NetworkPlanDev;
    bt->net = d;
    bt->values_valid = false;
    d->edges = P.edges;
    cfd_status st = CFD_OK;
    if ((st = upload(&d->slot_ptr, P.slot_ptr, s)) != CFD_OK || (st = upload(&d->slot_src, P.slot_src, s)) != CFD_OK ||
        (st = upload(&d->rhs_ptr, P.rhs_ptr, s)) != CFD_OK || (st = upload(&d->rhs_edge, P.rhs_edge, s)) != CFD_OK ||
        (st = upload(&d->rhs_node, P.rhs_node, s)) != CFD_OK || (st = upload(&d->fixed, P.fixed, s)) != CFD_OK ||
        (st = upload(&d->fixed_value, P.fixed_value, s)) != CFD_OK ||
        (st = upload(&d->g, std::vector<double>(P.edges), s)) != CFD_OK ||
        (st = upload(&d->q, std::vector<double>(P.rows), s)) != CFD_OK ||
        (st = upload(&d->bad, std::vector<int>(2), s)) != CFD_OK) {
      cfd_batch_destroy(bt);
      return st;
    }
    if (cudaMallocHost((void**)&d->h_bad, 2 * sizeof(int)) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
      cfd_batch_destroy(bt);
      set_error("cfd_batch_create_networks: plan upload failed");
      return CFD_ERR_CUDA;
    }
    *out = bt;
    return CFD_OK;
  });
}

cfd_status cfd_batch_assemble(cfd_batch* bt, const double* conductance, const double* neumann, int32_t memory) {
  return guarded("cfd_batch_assemble", [&]() -> cfd_status {
    if (!bt || !conductance) {
      set_error("cfd_batch_assemble: null argument");
      return CFD_ERR_STATE;
    }
    if (!bt->net) {
      set_error("cfd_batch_assemble: not a network batch (cfd_batch_create_networks)");
      return CFD_ERR_STATE;
    }
    if (memory != CFD_MEMORY_HOST && memory != CFD_MEMORY_DEVICE) {
      set_error("cfd_batch_assemble: unknown memory kind %d", memory);
      return CFD_ERR_CONFIG;
    }
    cfd_context* ctx = bt->ctx;
    std::lock_guard<std::mutex> g(ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    NetworkPlanDev* d = bt->net;
    const double* gd = conductance;
    const double* qd = neumann;
    if (memory == CFD_MEMORY_HOST) {
      if (d->edges > 0)
        CFD_TRY_CUDA(cudaMemcpyAsync(d->g, conductance, d->edges * sizeof(double), cudaMemcpyHostToDevice, s));
      gd = d->g;
      if (neumann) {
        if (bt->rows > 0)
          CFD_TRY_CUDA(cudaMemcpyAsync(d->q, neumann, bt->rows * sizeof(double), cudaMemcpyHostToDevice, s));
        qd = d->q;
      }
    }
    // Every byte 0x7f: an int above any edge index (edges <= kMaxNetworkEdges).
    CFD_TRY_CUDA(cudaMemsetAsync(d->bad, 0x7f, sizeof(int), s));
    CFD_TRY_CUDA(cudaMemsetAsync(d->bad + 1, 0, sizeof(int), s));
    // From here until a successful end the batch holds no usable system.
    bt->values_valid = false;
    bt->rhs_resident = false;
    const int64_t work = std::max({d->edges, bt->nnz, bt->rows});
    if (work > 0) {
      const int grid = (int)std::max<int64_t>(
          1, std::min<int64_t>((work + kAsmThreads - 1) / kAsmThreads, (int64_t)ctx->num_sms * 8));
      k_network_assemble<<<grid, kAsmThreads, 0, s>>>(d->view(), d->edges, bt->nnz, bt->rows, gd, qd, bt->v64,
                                                       bt->v32, bt->b, d->bad);
      CFD_TRY_CUDA(cudaGetLastError());
      ctx->stats.launches++;
    }
    CFD_TRY_CUDA(cudaMemcpyAsync(d->h_bad, d->bad, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaStreamSynchronize(s));
    const int64_t e = *d->h_bad;
    if (e < d->edges) {
      double ge = 0.0;
      if (memory == CFD_MEMORY_HOST)
        ge = conductance[e];
      else
        CFD_TRY_CUDA(cudaMemcpy(&ge, conductance + e, sizeof(double), cudaMemcpyDeviceToHost));
      return bad_conductance("cfd_batch_assemble", e, ge);
    }
    if (d->h_bad[1] & 3) return nonfinite_system("cfd_batch_assemble", d->h_bad[1] & 3);
    // FP32 solves of this batch are refused while an entry exceeds the FP32 range
    bt->f32_out_of_range = (d->h_bad[1] & 4) != 0;
    bt->values_valid = true;
    bt->rhs_resident = true;
    return CFD_OK;
  });
}

cfd_status cfd_batch_values(cfd_batch* bt, double* val_host, double* rhs_host) {
  return guarded("cfd_batch_values", [&]() -> cfd_status {
    if (!bt) return CFD_ERR_STATE;
    std::lock_guard<std::mutex> g(bt->ctx->mu);
    CFD_TRY_CUDA(cudaSetDevice(bt->ctx->device));
    cudaStream_t s = bt->ctx->stream;
    if (val_host && bt->nnz > 0)
      CFD_TRY_CUDA(cudaMemcpyAsync(val_host, bt->v64, bt->nnz * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (rhs_host && bt->rows > 0)
      CFD_TRY_CUDA(cudaMemcpyAsync(rhs_host, bt->b, bt->rows * sizeof(double), cudaMemcpyDeviceToHost, s));
    CFD_TRY_CUDA(cudaStreamSynchronize(s));
    return CFD_OK;
  });
}

cfd_status cfd_network_assemble_host(int32_t num_systems, const int64_t* node_offsets, const int64_t* edge_offsets,
                                     const int32_t* edge_i, const int32_t* edge_j, const int8_t* fixed,
                                     const double* fixed_value, const double* conductance, const double* neumann,
                                     int64_t* nnz_out, int64_t* row_ptr, int32_t* col, double* val, double* rhs) {
  return guarded("cfd_network_assemble_host", [&]() -> cfd_status {
    if (!nnz_out) {
      set_error("cfd_network_assemble_host: null nnz_out");
      return CFD_ERR_STATE;
    }
    NetworkPlan P;
    CFD_TRY(build_network_plan(num_systems, node_offsets, edge_offsets, edge_i, edge_j, fixed, fixed_value, P));
    const int64_t nnz = (int64_t)P.col.size();
    *nnz_out = nnz;
    if (row_ptr) std::copy(P.row_ptr.begin(), P.row_ptr.end(), row_ptr);
    if (col) std::copy(P.col.begin(), P.col.end(), col);
    if (!val && !rhs) return CFD_OK;  // size or pattern query
    if (P.edges > 0 && !conductance) {
      set_error("cfd_network_assemble_host: null conductance array");
      return CFD_ERR_STATE;
    }
    for (int64_t e = 0; e < P.edges; ++e)
      if (!net_conductance_ok(conductance[e])) return bad_conductance("cfd_network_assemble_host", e, conductance[e]);
    const NetworkView V{P.slot_ptr.data(), P.slot_src.data(), P.rhs_ptr.data(), P.rhs_edge.data(),
                        P.rhs_node.data(), P.fixed.data(), P.fixed_value.data()};
    int flags = 0;
    if (val)
      for (int64_t k = 0; k < nnz; ++k) {
        val[k] = net_slot_value(V, k, conductance);
        if (!std::isfinite(val[k])) flags |= 1;
      }
    if (rhs)
      for (int64_t r = 0; r < P.rows; ++r) {
        rhs[r] = net_rhs_value(V, r, conductance, neumann);
        if (!std::isfinite(rhs[r])) flags |= 2;
      }
    return flags ? nonfinite_system("cfd_network_assemble_host", flags) : CFD_OK;
  });
}

}  // extern "C"
