// Kirchhoff network assembly as a gather plan: MatrixAssembler::assemble_into
// (crates/cfd-1d/src/solver/core/matrix_assembly.rs:163-250) for a whole batch
// of networks, split into a pattern step (once per network topology, on the
// host) and a value step (per set of conductances, on the device, or on the
// host for the check). The value step is written once, below, and compiled for
// both sides.
//
// assemble_into pushes COO entries edge by edge (free-free edge: +g at (i,i)
// and (j,j), -g at (i,j) and (j,i); an edge to a fixed node: +g on the free
// node's diagonal and g * p_fixed into its right-hand side; fixed-fixed:
// nothing), adds the Neumann sources, then gives every fixed node an identity
// row with right-hand side p. Converting the COO to CSR sums duplicate
// (row, column) entries; here they are summed in push order, as a stable sort
// by (row, column) does. So each CSR slot is a list of signed edge
// conductances in edge order, and each right-hand-side row a list of
// (edge, fixed neighbour) pairs in edge order.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <vector>

#include "cfdgpu.h"

namespace cfd {

// Contribution code of a CSR slot: 2 e for +g_e, 2 e + 1 for -g_e (e a global
// edge index), or kUnitSlot for the identity entry of a fixed node.
constexpr int32_t kUnitSlot = -1;
// Edge indices must leave room for the sign bit of the code.
constexpr int64_t kMaxNetworkEdges = (int64_t)(INT32_MAX / 2);

struct NetworkPlan {
  int32_t nsys = 0;
  int64_t rows = 0, edges = 0;
  std::vector<int64_t> sys_row;     // node offsets, nsys + 1
  std::vector<int64_t> row_ptr;     // global nonzero offsets, rows + 1
  std::vector<int32_t> col;         // column local to the row's network
  std::vector<int32_t> slot_ptr;    // nnz + 1
  std::vector<int32_t> slot_src;    // contribution codes
  std::vector<int32_t> rhs_ptr;     // rows + 1
  std::vector<int32_t> rhs_edge;    // an edge to a fixed neighbour ...
  std::vector<int32_t> rhs_node;    // ... and that neighbour (global node)
  std::vector<int8_t> fixed;        // per global node
  std::vector<double> fixed_value;  // per global node
};

// What the value step reads: host vectors for the check, device copies in
// the kernel.
struct NetworkView {
  const int32_t* slot_ptr;
  const int32_t* slot_src;
  const int32_t* rhs_ptr;
  const int32_t* rhs_edge;
  const int32_t* rhs_node;
  const int8_t* fixed;
  const double* fixed_value;
};

// The pattern step. Checks the description first (offsets, node ranges,
// self-loops, per-network size limits) and reads nothing it has not bounded.
cfd_status build_network_plan(int32_t nsys, const int64_t* node_off, const int64_t* edge_off, const int32_t* ei,
                              const int32_t* ej, const int8_t* fixed, const double* fixed_value, NetworkPlan& P);

// Each addition and product rounded on its own, on both sides (no fused
// multiply-add), so the device and the host check agree bit for bit.
__host__ __device__ inline double net_add(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
__host__ __device__ inline double net_mul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}

// The conductances assemble_into accepts (:191-203): finite and positive.
__host__ __device__ inline bool net_conductance_ok(double g) { return g > 0.0 && g <= DBL_MAX; }

__host__ __device__ inline double net_slot_value(const NetworkView& V, int64_t slot, const double* g) {
  double v = 0.0;
  for (int32_t k = V.slot_ptr[slot]; k < V.slot_ptr[slot + 1]; ++k) {
    const int32_t c = V.slot_src[k];
    if (c == kUnitSlot) {
      v = 1.0;
      continue;
    }
    const double ge = g[c >> 1];
    v = net_add(v, (c & 1) ? -ge : ge);
  }
  return v;
}

// neumann may be null. A fixed row's right-hand side is its pressure.
__host__ __device__ inline double net_rhs_value(const NetworkView& V, int64_t row, const double* g,
                                                const double* neumann) {
  if (V.fixed[row]) return V.fixed_value[row];
  double b = 0.0;
  for (int32_t k = V.rhs_ptr[row]; k < V.rhs_ptr[row + 1]; ++k)
    b = net_add(b, net_mul(g[V.rhs_edge[k]], V.fixed_value[V.rhs_node[k]]));
  if (neumann) b = net_add(b, neumann[row]);
  return b;
}

}  // namespace cfd
