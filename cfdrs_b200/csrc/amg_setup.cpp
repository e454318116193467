// Host AMG setup for the device V-cycle.
//
// Algorithms follow crates/cfd-math/src/linear_solver/preconditioners/multigrid/
// of CFDrs; the arithmetic order of every floating-point reduction is kept so
// the hierarchy is the same one the reference builds for the same matrix.
#include "amg_setup.h"

#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <numeric>

namespace cfd {

namespace {

inline double row_value(const HostCsr& a, int64_t row, int32_t col) {
  const int32_t* b = a.ci.data() + a.rp[row];
  const int32_t* e = a.ci.data() + a.rp[row + 1];
  const int32_t* it = std::lower_bound(b, e, col);
  return (it != e && *it == col) ? a.v[a.rp[row] + (it - b)] : 0.0;
}

// Prefix sum of per-row counts into row offsets.
void offsets_from_counts(std::vector<int64_t>& rp) {
  for (size_t i = 1; i < rp.size(); ++i) rp[i] += rp[i - 1];
}

}  // namespace

// compute_strength_matrix, coarsening/algorithms.rs:395-436: j != i is strong
// when |a_ij| >= theta * max_{k != i} |a_ik|; the value kept is |a_ij|.
HostCsr strength_matrix(const HostCsr& a, double theta) {
  HostCsr s;
  s.nrows = s.ncols = a.nrows;
  s.rp.assign(a.nrows + 1, 0);
  std::vector<double> thr(a.nrows);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < a.nrows; ++i) {
    double mx = 0.0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k)
      if (a.ci[k] != i) {
        double v = std::fabs(a.v[k]);
        mx = mx > v ? mx : v;
      }
    thr[i] = theta * mx;
    int64_t c = 0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k)
      if (a.ci[k] != i && std::fabs(a.v[k]) >= thr[i]) ++c;
    s.rp[i + 1] = c;
  }
  offsets_from_counts(s.rp);
  s.ci.resize(s.rp[a.nrows]);
  s.v.resize(s.rp[a.nrows]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < a.nrows; ++i) {
    int64_t o = s.rp[i];
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k)
      if (a.ci[k] != i && std::fabs(a.v[k]) >= thr[i]) {
        s.ci[o] = a.ci[k];
        s.v[o] = std::fabs(a.v[k]);
        ++o;
      }
  }
  return s;
}

HostCsr transpose(const HostCsr& a) {
  HostCsr t;
  t.nrows = a.ncols;
  t.ncols = a.nrows;
  t.rp.assign(t.nrows + 1, 0);
  for (int64_t k = 0; k < a.nnz(); ++k) t.rp[a.ci[k] + 1]++;
  offsets_from_counts(t.rp);
  t.ci.resize(a.nnz());
  t.v.resize(a.nnz());
  std::vector<int64_t> pos(t.rp.begin(), t.rp.end() - 1);
  for (int64_t i = 0; i < a.nrows; ++i)
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) {
      int64_t p = pos[a.ci[k]]++;
      t.ci[p] = (int32_t)i;
      t.v[p] = a.v[k];
    }
  return t;
}

// Row-wise product C = A B (Gustavson). Each output row accumulates its terms
// in a dense per-thread accumulator in the order A's row and then B's rows
// present them (first term assigned, the rest added), so every entry is the
// same left-to-right sum over A's row; the row's distinct columns are then
// sorted. The accumulator is stamped with the row index, so it is never reset.
HostCsr spgemm(const HostCsr& a, const HostCsr& b) {
  HostCsr c;
  c.nrows = a.nrows;
  c.ncols = b.ncols;
  c.rp.assign(a.nrows + 1, 0);
  // Pass 1: row lengths. Pass 2: values (the row is formed again).
#pragma omp parallel
  {
    std::vector<int32_t> stamp(b.ncols, -1);
#pragma omp for schedule(dynamic, 2048)
    for (int64_t i = 0; i < a.nrows; ++i) {
      int64_t u = 0;
      for (int64_t ka = a.rp[i]; ka < a.rp[i + 1]; ++ka) {
        const int64_t k = a.ci[ka];
        for (int64_t kb = b.rp[k]; kb < b.rp[k + 1]; ++kb) {
          const int32_t j = b.ci[kb];
          if (stamp[j] != (int32_t)i) {
            stamp[j] = (int32_t)i;
            ++u;
          }
        }
      }
      c.rp[i + 1] = u;
    }
  }
  offsets_from_counts(c.rp);
  c.ci.resize(c.rp[a.nrows]);
  c.v.resize(c.rp[a.nrows]);
#pragma omp parallel
  {
    std::vector<int32_t> stamp(b.ncols, -1);
    std::vector<double> acc(b.ncols);
    std::vector<int32_t> cols;
#pragma omp for schedule(dynamic, 2048)
    for (int64_t i = 0; i < a.nrows; ++i) {
      cols.clear();
      for (int64_t ka = a.rp[i]; ka < a.rp[i + 1]; ++ka) {
        const int64_t k = a.ci[ka];
        const double av = a.v[ka];
        for (int64_t kb = b.rp[k]; kb < b.rp[k + 1]; ++kb) {
          const int32_t j = b.ci[kb];
          const double t = av * b.v[kb];
          if (stamp[j] != (int32_t)i) {
            stamp[j] = (int32_t)i;
            acc[j] = t;
            cols.push_back(j);
          } else {
            acc[j] += t;
          }
        }
      }
      std::sort(cols.begin(), cols.end());
      int64_t o = c.rp[i];
      for (const int32_t j : cols) {
        c.ci[o] = j;
        c.v[o] = acc[j];
        ++o;
      }
    }
  }
  return c;
}

namespace {

// Leftmost-maximum tournament tree: the pick of "undecided point with the
// largest measure, lowest index first" in O(log n) per update.
class MaxTree {
 public:
  explicit MaxTree(const std::vector<int32_t>& key) {
    const int64_t n = (int64_t)key.size();
    while (size_ < n) size_ <<= 1;
    key_.assign(size_, -2);
    std::copy(key.begin(), key.end(), key_.begin());
    best_.resize(2 * size_);
    for (int64_t i = 0; i < size_; ++i) best_[size_ + i] = (int32_t)i;
    for (int64_t p = size_ - 1; p >= 1; --p) best_[p] = pick(best_[2 * p], best_[2 * p + 1]);
  }
  void set(int64_t i, int32_t k) {
    key_[i] = k;
    for (int64_t p = (i + size_) >> 1; p >= 1; p >>= 1) {
      const int32_t nb = pick(best_[2 * p], best_[2 * p + 1]);
      // Same winner here, and not the point whose key changed: every ancestor
      // compares the same keys as before, so the tree above is already right.
      if (nb == best_[p] && nb != (int32_t)i) break;
      best_[p] = nb;
    }
  }
  int32_t top() const { return best_[1]; }
  int32_t key(int64_t i) const { return key_[i]; }

 private:
  int32_t pick(int32_t l, int32_t r) const { return key_[r] > key_[l] ? r : l; }
  int64_t size_ = 1;
  std::vector<int32_t> key_, best_;
};

// assign_closest_coarse_points, coarsening/algorithms.rs:199-230.
void assign_closest(std::vector<int32_t>& f2c, const std::vector<int8_t>& status, const HostCsr& s) {
  for (int64_t i = 0; i < s.nrows; ++i) {
    if (f2c[i] >= 0) continue;
    double best = 0.0;
    int32_t best_idx = -1;
    bool have = false;
    for (int64_t k = s.rp[i]; k < s.rp[i + 1]; ++k) {
      const int32_t j = s.ci[k];
      if (status[j] == 1 && (!have || s.v[k] > best)) {
        best = s.v[k];
        best_idx = f2c[j];
        have = true;
      }
    }
    if (best_idx >= 0) f2c[i] = best_idx;
  }
}

}  // namespace

// ruge_stueben_coarsening, coarsening/algorithms.rs:34-126. The reference scans
// all points for the maximum measure on every pick (O(n^2)); the tournament
// tree returns the same point (largest lambda, lowest index) in O(log n).
Coarsening ruge_stueben(const HostCsr& a, double theta) {
  const int64_t n = a.nrows;
  Coarsening c;
  c.strength = strength_matrix(a, theta);
  const HostCsr& s = c.strength;
  const HostCsr st = transpose(s);
  std::vector<int32_t> lambda(n);
  for (int64_t i = 0; i < n; ++i) lambda[i] = (int32_t)(st.rp[i + 1] - st.rp[i]);
  std::vector<int8_t> status(n, 0);  // 0 undecided, 1 C, 2 F
  c.f2c.assign(n, -1);
  MaxTree tree(lambda);
  int64_t undecided = n;
  while (undecided > 0) {
    const int32_t i = tree.top();
    if (i >= n || tree.key(i) < 0) break;
    if (lambda[i] <= 0) break;
    status[i] = 1;
    tree.set(i, -1);
    --undecided;
    c.f2c[i] = (int32_t)c.coarse_points.size();
    c.coarse_points.push_back(i);
    for (int64_t k = st.rp[i]; k < st.rp[i + 1]; ++k) {
      const int32_t j = st.ci[k];
      if (status[j] != 0) continue;
      status[j] = 2;
      tree.set(j, -1);
      --undecided;
      for (int64_t m = s.rp[j]; m < s.rp[j + 1]; ++m) {
        const int32_t kk = s.ci[m];
        if (status[kk] == 0) tree.set(kk, ++lambda[kk]);
      }
    }
  }
  for (int64_t i = 0; i < n; ++i)
    if (status[i] == 0) {
      status[i] = 1;
      c.f2c[i] = (int32_t)c.coarse_points.size();
      c.coarse_points.push_back((int32_t)i);
    }
  assign_closest(c.f2c, status, s);
  return c;
}

// aggregation_coarsening, coarsening/algorithms.rs:129-172 (strength 0.5).
Coarsening aggregation(const HostCsr& a, int64_t max_size) {
  const int64_t n = a.nrows;
  Coarsening c;
  c.strength = strength_matrix(a, 0.5);
  const HostCsr& s = c.strength;
  std::vector<int8_t> agg(n, 0);
  c.f2c.assign(n, -1);
  std::vector<int32_t> members;
  int32_t id = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i]) continue;
    members.assign(1, (int32_t)i);
    agg[i] = 1;
    for (int64_t k = s.rp[i]; k < s.rp[i + 1]; ++k) {
      const int32_t j = s.ci[k];
      if (!agg[j] && (int64_t)members.size() < max_size) {
        members.push_back(j);
        agg[j] = 1;
      }
    }
    c.coarse_points.push_back(members[0]);
    for (int32_t p : members) c.f2c[p] = id;
    ++id;
  }
  return c;
}

// pmis_coarsening, coarsening/algorithms.rs:310-354, with SplitMix64-seeded
// priorities in place of the reference's unseeded thread_rng (:324).
Coarsening pmis(const HostCsr& a, double theta, uint64_t seed) {
  const int64_t n = a.nrows;
  Coarsening c;
  c.strength = strength_matrix(a, theta);
  const HostCsr& s = c.strength;
  std::vector<double> prio(n);
  uint64_t state = seed;
  for (int64_t i = 0; i < n; ++i) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    prio[i] = (double)(z >> 11) * 0x1.0p-53;
  }
  std::vector<int32_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return prio[x] > prio[y]; });
  std::vector<int8_t> status(n, 0);
  c.f2c.assign(n, -1);
  for (int32_t i : order) {
    if (status[i] != 0) continue;
    status[i] = 1;
    c.f2c[i] = (int32_t)c.coarse_points.size();
    c.coarse_points.push_back(i);
    for (int64_t k = s.rp[i]; k < s.rp[i + 1]; ++k)
      if (status[s.ci[k]] == 0) status[s.ci[k]] = 2;
  }
  assign_closest(c.f2c, status, s);
  return c;
}

// create_classical_interpolation, interpolation.rs:38-188. For an F-point i
// with strong C-neighbours C_i and strong F-neighbours F_i:
//   w_ij = (a_ij + sum_{k in F_i, |d_k| > eps} a_ik a_kj / d_k) * (1 / -(a_ii + sum_weak a_in)),
//   d_k  = sum_{m in C_i} a_km,
// C-points inject; rows without strong C-neighbours (or a vanishing lumped
// diagonal) stay empty.
HostCsr classical_interpolation(const HostCsr& a, const Coarsening& c) {
  const int64_t n = a.nrows;
  const int64_t nc = (int64_t)c.coarse_points.size();
  const HostCsr& s = c.strength;
  std::vector<int32_t> cmap(n, -1);
  for (int64_t l = 0; l < nc; ++l) cmap[c.coarse_points[l]] = (int32_t)l;
  std::vector<std::vector<std::pair<int32_t, double>>> rows(n);
#pragma omp parallel
  {
    std::vector<int32_t> ci, fi;
    std::vector<double> den;
#pragma omp for schedule(dynamic, 4096)
    for (int64_t i = 0; i < n; ++i) {
      auto& out = rows[i];
      if (cmap[i] >= 0) {
        out.emplace_back(cmap[i], 1.0);
        continue;
      }
      const int32_t* sc = s.ci.data() + s.rp[i];
      const int64_t ns = s.rp[i + 1] - s.rp[i];
      ci.clear();
      fi.clear();
      for (int64_t q = 0; q < ns; ++q) {
        if (cmap[sc[q]] >= 0)
          ci.push_back(sc[q]);
        else if (sc[q] != i)
          fi.push_back(sc[q]);
      }
      if (ci.empty()) continue;
      double a_ii = 0.0, weak = 0.0;
      for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) {
        const int32_t j = a.ci[k];
        if (j == i)
          a_ii = a.v[k];
        else if (!std::binary_search(sc, sc + ns, j))
          weak += a.v[k];
      }
      const double diagonal = a_ii + weak;
      if (!(std::fabs(diagonal) > DBL_EPSILON)) continue;
      den.resize(fi.size());
      for (size_t q = 0; q < fi.size(); ++q) {
        double d = 0.0;
        for (int32_t m : ci) d += row_value(a, fi[q], m);
        den[q] = d;
      }
      const double neg_inv = 1.0 / -diagonal;
      for (int32_t j : ci) {
        const double a_ij = row_value(a, i, j);
        double ind = 0.0;
        for (size_t q = 0; q < fi.size(); ++q)
          if (std::fabs(den[q]) > DBL_EPSILON) ind += row_value(a, i, fi[q]) * row_value(a, fi[q], j) / den[q];
        out.emplace_back(cmap[j], (a_ij + ind) * neg_inv);
      }
      std::stable_sort(out.begin(), out.end(),
                       [](const std::pair<int32_t, double>& x, const std::pair<int32_t, double>& y) {
                         return x.first < y.first;
                       });
    }
  }
  HostCsr p;
  p.nrows = n;
  p.ncols = nc;
  p.rp.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) p.rp[i + 1] = (int64_t)rows[i].size();
  offsets_from_counts(p.rp);
  p.ci.resize(p.rp[n]);
  p.v.resize(p.rp[n]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    for (size_t q = 0; q < rows[i].size(); ++q) {
      p.ci[p.rp[i] + q] = rows[i][q].first;
      p.v[p.rp[i] + q] = rows[i][q].second;
    }
  return p;
}

// Modified classical interpolation (Stueben 2001, App. A.7.2; the sign-
// restricted form of hypre BoomerAMG's classical-modified interpolation). The
// sets C_i / F_i and the weak-connection lumping are those of the reference
// formula above; what changes: for a strong F-neighbour k only entries a_km of
// sign opposite to a_kk are distributed (so the denominator cannot cancel on
// Galerkin levels whose off-diagonals turn positive), and a k with no such
// entry to C_i is lumped into the diagonal instead of dropped (so row sums are
// kept). The reference's form (interpolation.rs:116-158) loses convergence from
// the fourth level down on 3-D Poisson; the reference itself only builds
// hierarchies below 10 000 unknowns (crates/cfd-2d/src/pressure_velocity/correction.rs:40).
HostCsr modified_classical_interpolation(const HostCsr& a, const Coarsening& c) {
  const int64_t n = a.nrows;
  const int64_t nc = (int64_t)c.coarse_points.size();
  const HostCsr& s = c.strength;
  std::vector<int32_t> cmap(n, -1);
  for (int64_t l = 0; l < nc; ++l) cmap[c.coarse_points[l]] = (int32_t)l;
  std::vector<std::vector<std::pair<int32_t, double>>> rows(n);
#pragma omp parallel
  {
    std::vector<int32_t> ci, fi;
    std::vector<double> num;
#pragma omp for schedule(dynamic, 4096)
    for (int64_t i = 0; i < n; ++i) {
      auto& out = rows[i];
      if (cmap[i] >= 0) {
        out.emplace_back(cmap[i], 1.0);
        continue;
      }
      const int32_t* sc = s.ci.data() + s.rp[i];
      const int64_t ns = s.rp[i + 1] - s.rp[i];
      ci.clear();
      fi.clear();
      for (int64_t q = 0; q < ns; ++q) {
        if (cmap[sc[q]] >= 0)
          ci.push_back(sc[q]);
        else if (sc[q] != i)
          fi.push_back(sc[q]);
      }
      if (ci.empty()) continue;
      double diagonal = 0.0;
      for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) {
        const int32_t j = a.ci[k];
        if (j == i || !std::binary_search(sc, sc + ns, j)) diagonal += a.v[k];
      }
      num.assign(ci.size(), 0.0);
      for (size_t q = 0; q < ci.size(); ++q) num[q] = row_value(a, i, ci[q]);
      for (int32_t k : fi) {
        const double a_ik = row_value(a, i, k);
        const double a_kk = row_value(a, k, k);
        double den = 0.0;
        for (int32_t m : ci) {
          const double v = row_value(a, k, m);
          if (v * a_kk < 0.0) den += v;
        }
        if (den == 0.0) {
          diagonal += a_ik;
          continue;
        }
        for (size_t q = 0; q < ci.size(); ++q) {
          const double v = row_value(a, k, ci[q]);
          if (v * a_kk < 0.0) num[q] += a_ik * v / den;
        }
      }
      if (!(std::fabs(diagonal) > DBL_EPSILON)) continue;
      const double neg_inv = 1.0 / -diagonal;
      for (size_t q = 0; q < ci.size(); ++q) out.emplace_back(cmap[ci[q]], num[q] * neg_inv);
      std::stable_sort(out.begin(), out.end(),
                       [](const std::pair<int32_t, double>& x, const std::pair<int32_t, double>& y) {
                         return x.first < y.first;
                       });
    }
  }
  HostCsr p;
  p.nrows = n;
  p.ncols = nc;
  p.rp.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) p.rp[i + 1] = (int64_t)rows[i].size();
  offsets_from_counts(p.rp);
  p.ci.resize(p.rp[n]);
  p.v.resize(p.rp[n]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    for (size_t q = 0; q < rows[i].size(); ++q) {
      p.ci[p.rp[i] + q] = rows[i][q].first;
      p.v[p.rp[i] + q] = rows[i][q].second;
    }
  return p;
}

// create_direct_interpolation, interpolation.rs:191-217 (piecewise constant).
HostCsr direct_interpolation(const Coarsening& c, int64_t n) {
  HostCsr p;
  p.nrows = n;
  p.ncols = (int64_t)c.coarse_points.size();
  p.rp.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) {
    if (c.f2c[i] >= 0) {
      p.ci.push_back(c.f2c[i]);
      p.v.push_back(1.0);
    }
    p.rp[i + 1] = (int64_t)p.ci.size();
  }
  return p;
}

bool dense_inverse(const HostCsr& a, std::vector<double>& inv) {
  const int64_t n = a.nrows;
  std::vector<double> m((size_t)n * n, 0.0);
  inv.assign((size_t)n * n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    inv[(size_t)i * n + i] = 1.0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) m[(size_t)i * n + a.ci[k]] += a.v[k];
  }
  for (int64_t c = 0; c < n; ++c) {
    int64_t p = c;
    for (int64_t r = c + 1; r < n; ++r)
      if (std::fabs(m[(size_t)r * n + c]) > std::fabs(m[(size_t)p * n + c])) p = r;
    if (m[(size_t)p * n + c] == 0.0) return false;
    if (p != c)
      for (int64_t k = 0; k < n; ++k) {
        std::swap(m[(size_t)c * n + k], m[(size_t)p * n + k]);
        std::swap(inv[(size_t)c * n + k], inv[(size_t)p * n + k]);
      }
    const double d = 1.0 / m[(size_t)c * n + c];
    for (int64_t k = 0; k < n; ++k) {
      m[(size_t)c * n + k] *= d;
      inv[(size_t)c * n + k] *= d;
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = m[(size_t)r * n + c];
      if (f == 0.0) continue;
      for (int64_t k = 0; k < n; ++k) {
        m[(size_t)r * n + k] -= f * m[(size_t)c * n + k];
        inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
      }
    }
  }
  return true;
}

// Interpolation truncation (cfd_amg_config::max_interp_points): in every row
// of P with more than k weights keep the k of largest magnitude (ties: the
// smaller column) and scale them by (sum of all weights) / (sum of the kept
// ones), both sums taken in ascending column order, so the row sum is kept.
HostCsr truncate_interpolation(const HostCsr& p, int k) {
  if (k <= 0) return p;
  HostCsr t;
  t.nrows = p.nrows;
  t.ncols = p.ncols;
  t.rp.assign(p.nrows + 1, 0);
  std::vector<std::vector<std::pair<int32_t, double>>> rows(p.nrows);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t i = 0; i < p.nrows; ++i) {
    const int64_t a = p.rp[i], b = p.rp[i + 1];
    auto& out = rows[i];
    if (b - a <= k) {
      for (int64_t e = a; e < b; ++e) out.emplace_back(p.ci[e], p.v[e]);
      continue;
    }
    std::vector<int64_t> order;
    for (int64_t e = a; e < b; ++e) order.push_back(e);
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
      const double ax = std::fabs(p.v[x]), ay = std::fabs(p.v[y]);
      return ax != ay ? ax > ay : p.ci[x] < p.ci[y];
    });
    order.resize(k);
    std::sort(order.begin(), order.end());
    double all = 0.0, kept = 0.0;
    for (int64_t e = a; e < b; ++e) all += p.v[e];
    for (int64_t e : order) kept += p.v[e];
    const double scale = kept != 0.0 ? all / kept : 1.0;
    for (int64_t e : order) out.emplace_back(p.ci[e], p.v[e] * scale);
  }
  for (int64_t i = 0; i < p.nrows; ++i) t.rp[i + 1] = t.rp[i] + (int64_t)rows[i].size();
  t.ci.resize(t.rp[p.nrows]);
  t.v.resize(t.rp[p.nrows]);
  for (int64_t i = 0; i < p.nrows; ++i)
    for (size_t q = 0; q < rows[i].size(); ++q) {
      t.ci[t.rp[i] + q] = rows[i][q].first;
      t.v[t.rp[i] + q] = rows[i][q].second;
    }
  return t;
}

// Renumber the coarse points by ascending fine index (f2c follows).
void renumber_ascending(Coarsening& c) {
  std::vector<int32_t> sorted(c.coarse_points);
  std::sort(sorted.begin(), sorted.end());
  std::vector<int32_t> newid(c.f2c.size(), -1);
  for (size_t q = 0; q < sorted.size(); ++q) newid[sorted[q]] = (int32_t)q;
  for (size_t i = 0; i < c.f2c.size(); ++i)
    if (c.f2c[i] >= 0) c.f2c[i] = newid[c.coarse_points[c.f2c[i]]];
  c.coarse_points.swap(sorted);
}

// AlgebraicMultigrid::setup (amg.rs:217-288) and build_next_level (:290-380):
// coarsen while levels < max_levels and n > min_coarse_size; R = P^T; the
// Galerkin operator is (R A) P.
std::vector<HostLevel> build_hierarchy(const HostCsr& a, const cfd_amg_config& cfg) {
  std::vector<HostLevel> levels(1);
  levels[0].A = a;
  while ((int)levels.size() < cfg.max_levels && levels.back().A.nrows > cfg.min_coarse_size) {
    const HostCsr& cur = levels.back().A;
    Coarsening c;
    if (cfg.coarsening == CFD_COARSEN_AGGREGATION)
      c = aggregation(cur, cfg.aggregate_size);
    else if (cfg.coarsening == CFD_COARSEN_PMIS)
      c = pmis(cur, cfg.strength_threshold, cfg.seed);
    else
      c = ruge_stueben(cur, cfg.strength_threshold);
    const int64_t nc = (int64_t)c.coarse_points.size();
    if (cfg.coarse_order == CFD_COARSE_ORDER_ASCENDING) renumber_ascending(c);
    HostCsr p = cfg.interpolation == CFD_INTERP_DIRECT               ? direct_interpolation(c, cur.nrows)
                : cfg.interpolation == CFD_INTERP_MODIFIED_CLASSICAL ? modified_classical_interpolation(cur, c)
                                                                     : classical_interpolation(cur, c);
    if (cfg.max_interp_points > 0) p = truncate_interpolation(p, cfg.max_interp_points);
    HostCsr r = transpose(p);
    HostCsr ac = spgemm(spgemm(r, cur), p);
    levels.back().P = std::move(p);
    levels.back().R = std::move(r);
    const int64_t n_cur = cur.nrows;  // `cur` refers into `levels`, which the push_back may move
    HostLevel next;
    next.A = std::move(ac);
    levels.push_back(std::move(next));
    if (nc == 0 || nc >= n_cur) break;
  }
  return levels;
}

}  // namespace cfd
