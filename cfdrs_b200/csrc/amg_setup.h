// Host construction of the AMG hierarchy (coarsening, interpolation, Galerkin
// products). Runs once per pattern/value set; the V-cycle itself runs on the
// device (amg_device.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "internal.h"

namespace cfd {

HostCsr strength_matrix(const HostCsr& a, double theta);
HostCsr transpose(const HostCsr& a);
HostCsr spgemm(const HostCsr& a, const HostCsr& b);

struct Coarsening {
  std::vector<int32_t> coarse_points;  // selection order = coarse numbering
  std::vector<int32_t> f2c;            // fine -> coarse (-1: unassigned)
  HostCsr strength;
};

Coarsening ruge_stueben(const HostCsr& a, double theta);
Coarsening aggregation(const HostCsr& a, int64_t max_size);
Coarsening pmis(const HostCsr& a, double theta, uint64_t seed);

void renumber_ascending(Coarsening& c);
HostCsr classical_interpolation(const HostCsr& a, const Coarsening& c);
HostCsr modified_classical_interpolation(const HostCsr& a, const Coarsening& c);
HostCsr direct_interpolation(const Coarsening& c, int64_t n);

// Row-major inverse of a small dense SPD/nonsingular matrix (Gauss-Jordan
// with partial pivoting). Returns false when singular.
bool dense_inverse(const HostCsr& a, std::vector<double>& inv);

struct HostLevel {
  HostCsr A, P, R;
};

// AlgebraicMultigrid::setup / build_next_level.
std::vector<HostLevel> build_hierarchy(const HostCsr& a, const cfd_amg_config& cfg);

}  // namespace cfd
