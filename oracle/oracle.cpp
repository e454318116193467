// CPU oracle: plain restatement of the CFDrs FP64 sparse-solve path.
// Test infrastructure only -- see oracle.h for scope and the reference map.
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <map>
#include <vector>

struct or_csr {
  int64_t nrows = 0, ncols = 0;
  std::vector<int64_t> rp, ci;
  std::vector<double> v;
  int64_t nnz() const { return (int64_t)ci.size(); }
};

// SimplePreconditioner (crates/cfd-math/src/linear_solver/block_preconditioner.rs:411-424).
struct or_component_block {
  int64_t nv = 0, np = 0, cs = 0;
  std::vector<double> lu[3];      // per component: dense LU with partial pivoting
  std::vector<int64_t> piv[3];
  std::vector<double> pinv;       // lumped pressure inverse
  std::vector<std::vector<std::pair<int64_t, double>>> div_rows;  // D, per pressure row
  std::vector<std::vector<std::pair<int64_t, double>>> grad_rows; // G, per velocity row (pressure index, value)
};

struct or_simple {
  int64_t nv = 0, np = 0;
  std::vector<double> dinv, sinv;                                 // diag(A)^-1, diag(S)^-1
  std::vector<std::vector<std::pair<int64_t, double>>> div_rows;  // D, per pressure row
  std::vector<std::vector<std::pair<int64_t, double>>> grad_cols; // G, per pressure column
  std::vector<double> bdinv;  // BlockDiagonalPreconditioner's inverse diagonal (all n unknowns)
};

namespace {

// diagonal_epsilon() in multigrid/amg.rs:58-61 and smoothers.rs (|diag| > 1e-15).
constexpr double kDiagEps = 1e-15;

double dot(int64_t n, const double* a, const double* b) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

void spmv_raw(const or_csr& a, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < a.nrows; ++i) {
    double s = 0.0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) s += a.v[k] * x[a.ci[k]];
    y[i] = s;
  }
}

// csr_value (multigrid/mod.rs:205-215): binary search of column col in row.
double csr_value(const or_csr& a, int64_t row, int64_t col) {
  const int64_t* b = a.ci.data() + a.rp[row];
  const int64_t* e = a.ci.data() + a.rp[row + 1];
  const int64_t* it = std::lower_bound(b, e, col);
  if (it != e && *it == col) return a.v[a.rp[row] + (it - b)];
  return 0.0;
}

[[maybe_unused]] bool row_has(const or_csr& a, int64_t row, int64_t col) {
  const int64_t* b = a.ci.data() + a.rp[row];
  const int64_t* e = a.ci.data() + a.rp[row + 1];
  return std::binary_search(b, e, col);
}

or_csr transpose(const or_csr& a) {
  or_csr t;
  t.nrows = a.ncols;
  t.ncols = a.nrows;
  t.rp.assign(t.nrows + 1, 0);
  for (int64_t k = 0; k < a.nnz(); ++k) t.rp[a.ci[k] + 1]++;
  for (int64_t i = 0; i < t.nrows; ++i) t.rp[i + 1] += t.rp[i];
  t.ci.resize(a.nnz());
  t.v.resize(a.nnz());
  std::vector<int64_t> pos(t.rp.begin(), t.rp.end() - 1);
  for (int64_t i = 0; i < a.nrows; ++i)
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) {
      int64_t p = pos[a.ci[k]]++;
      t.ci[p] = i;
      t.v[p] = a.v[k];
    }
  return t;
}

// Gustavson row-by-row product; columns of each output row sorted, structural
// zeros kept (the product pattern is the symbolic pattern).
or_csr spgemm(const or_csr& a, const or_csr& b) {
  or_csr c;
  c.nrows = a.nrows;
  c.ncols = b.ncols;
  c.rp.assign(a.nrows + 1, 0);
  int nt = omp_get_max_threads();
  std::vector<std::vector<int64_t>> rows_ci(a.nrows);
  std::vector<std::vector<double>> rows_v(a.nrows);
#pragma omp parallel num_threads(nt)
  {
    std::vector<int64_t> marker(b.ncols, -1);
    std::vector<double> acc(b.ncols, 0.0);
    std::vector<int64_t> cols;
#pragma omp for schedule(dynamic, 1024)
    for (int64_t i = 0; i < a.nrows; ++i) {
      cols.clear();
      for (int64_t ka = a.rp[i]; ka < a.rp[i + 1]; ++ka) {
        int64_t k = a.ci[ka];
        double av = a.v[ka];
        for (int64_t kb = b.rp[k]; kb < b.rp[k + 1]; ++kb) {
          int64_t j = b.ci[kb];
          if (marker[j] != i) {
            marker[j] = i;
            acc[j] = av * b.v[kb];
            cols.push_back(j);
          } else {
            acc[j] += av * b.v[kb];
          }
        }
      }
      std::sort(cols.begin(), cols.end());
      rows_ci[i] = cols;
      rows_v[i].resize(cols.size());
      for (size_t q = 0; q < cols.size(); ++q) rows_v[i][q] = acc[cols[q]];
    }
  }
  for (int64_t i = 0; i < a.nrows; ++i) c.rp[i + 1] = c.rp[i] + (int64_t)rows_ci[i].size();
  c.ci.resize(c.rp[a.nrows]);
  c.v.resize(c.rp[a.nrows]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < a.nrows; ++i) {
    std::copy(rows_ci[i].begin(), rows_ci[i].end(), c.ci.begin() + c.rp[i]);
    std::copy(rows_v[i].begin(), rows_v[i].end(), c.v.begin() + c.rp[i]);
  }
  return c;
}

// compute_strength_matrix, coarsening/algorithms.rs:395-436.
or_csr strength(const or_csr& a, double theta) {
  or_csr s;
  s.nrows = a.nrows;
  s.ncols = a.nrows;
  s.rp.assign(a.nrows + 1, 0);
  for (int64_t i = 0; i < a.nrows; ++i) {
    double mx = 0.0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k)
      if (a.ci[k] != i) {
        double val = std::fabs(a.v[k]);
        mx = mx > val ? mx : val;
      }
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k)
      if (a.ci[k] != i) {
        double st = std::fabs(a.v[k]);
        if (st >= theta * mx) {
          s.ci.push_back(a.ci[k]);
          s.v.push_back(st);
        }
      }
    s.rp[i + 1] = (int64_t)s.ci.size();
  }
  return s;
}

// assign_closest_coarse_points, coarsening/algorithms.rs:199-230.
void assign_closest(std::vector<int64_t>& f2c, const std::vector<int>& status, const or_csr& s) {
  for (int64_t i = 0; i < s.nrows; ++i) {
    if (f2c[i] >= 0) continue;
    double best = 0.0;
    int64_t best_idx = -1;
    bool have = false;
    for (int64_t k = s.rp[i]; k < s.rp[i + 1]; ++k) {
      int64_t j = s.ci[k];
      if (status[j] == 1) {
        double st = s.v[k];
        if (!have || st > best) {
          best = st;
          best_idx = f2c[j];
          have = true;
        }
      }
    }
    if (best_idx >= 0) f2c[i] = best_idx;
  }
}

// Leftmost-maximum tournament tree over lambda (undecided points only);
// reproduces the reference's first-index-of-maximum linear scan exactly.
struct MaxTree {
  int64_t size = 1;
  std::vector<int64_t> key;   // per leaf, -1 when decided
  std::vector<int64_t> best;  // per node, leaf index of its leftmost maximum
  explicit MaxTree(const std::vector<int64_t>& k) {
    int64_t n = (int64_t)k.size();
    while (size < n) size <<= 1;
    key.assign(size, -2);
    for (int64_t i = 0; i < n; ++i) key[i] = k[i];
    best.assign(2 * size, 0);
    for (int64_t i = 0; i < size; ++i) best[size + i] = i;
    for (int64_t p = size - 1; p >= 1; --p) best[p] = pick(best[2 * p], best[2 * p + 1]);
  }
  int64_t pick(int64_t l, int64_t r) const { return key[r] > key[l] ? r : l; }
  void set(int64_t i, int64_t k) {
    key[i] = k;
    for (int64_t p = (i + size) >> 1; p >= 1; p >>= 1) {
      const int64_t nb = pick(best[2 * p], best[2 * p + 1]);
      if (nb == best[p] && nb != i) break;  // same winner, unchanged key: ancestors stand
      best[p] = nb;
    }
  }
  int64_t top() const { return best[1]; }
};

// ruge_stueben_coarsening, coarsening/algorithms.rs:34-126.
int64_t ruge_stueben(const or_csr& a, double theta, bool literal, std::vector<int64_t>& cpts,
                     std::vector<int64_t>& f2c, or_csr* s_out) {
  const int64_t n = a.nrows;
  or_csr s = strength(a, theta);
  or_csr st = transpose(s);
  std::vector<int64_t> lambda(n);
  for (int64_t i = 0; i < n; ++i) lambda[i] = st.rp[i + 1] - st.rp[i];
  std::vector<int> status(n, 0);
  f2c.assign(n, -1);
  cpts.clear();
  int64_t undecided = n;
  MaxTree* tree = literal ? nullptr : new MaxTree(lambda);
  auto decide = [&](int64_t j) {
    if (tree) tree->set(j, -1);
  };
  while (undecided > 0) {
    int64_t i_opt = -1;
    int64_t max_lambda = -1;
    if (literal) {
      for (int64_t k = 0; k < n; ++k)
        if (status[k] == 0 && lambda[k] > max_lambda) {
          max_lambda = lambda[k];
          i_opt = k;
        }
    } else {
      int64_t t = tree->top();
      if (t < n && tree->key[t] >= 0) {
        i_opt = t;
        max_lambda = lambda[t];
      }
    }
    if (i_opt < 0) break;
    if (max_lambda <= 0) break;
    int64_t i = i_opt;
    status[i] = 1;
    decide(i);
    undecided--;
    cpts.push_back(i);
    f2c[i] = (int64_t)cpts.size() - 1;
    for (int64_t k = st.rp[i]; k < st.rp[i + 1]; ++k) {
      int64_t j = st.ci[k];
      if (status[j] == 0) {
        status[j] = 2;
        decide(j);
        undecided--;
        for (int64_t m = s.rp[j]; m < s.rp[j + 1]; ++m) {
          int64_t kk = s.ci[m];
          if (status[kk] == 0) {
            lambda[kk] += 1;
            if (tree) tree->set(kk, lambda[kk]);
          }
        }
      }
    }
  }
  delete tree;
  for (int64_t i = 0; i < n; ++i)
    if (status[i] == 0) {
      status[i] = 1;
      cpts.push_back(i);
      f2c[i] = (int64_t)cpts.size() - 1;
    }
  assign_closest(f2c, status, s);
  if (s_out) *s_out = std::move(s);
  return (int64_t)cpts.size();
}

// aggregation_coarsening, coarsening/algorithms.rs:129-172 (strength theta fixed at 0.5).
int64_t aggregation(const or_csr& a, int64_t max_size, std::vector<int64_t>& cpts,
                    std::vector<int64_t>& f2c, or_csr* s_out) {
  const int64_t n = a.nrows;
  or_csr s = strength(a, 0.5);
  std::vector<char> agg(n, 0);
  f2c.assign(n, -1);
  cpts.clear();
  int64_t id = 0;
  std::vector<int64_t> members;
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i]) continue;
    members.assign(1, i);
    agg[i] = 1;
    for (int64_t k = s.rp[i]; k < s.rp[i + 1]; ++k) {
      int64_t j = s.ci[k];
      if (!agg[j] && (int64_t)members.size() < max_size) {
        members.push_back(j);
        agg[j] = 1;
      }
    }
    cpts.push_back(members[0]);
    for (int64_t p : members) f2c[p] = id;
    id++;
  }
  if (s_out) *s_out = std::move(s);
  return (int64_t)cpts.size();
}

uint64_t splitmix64(uint64_t& state) {
  uint64_t z = (state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// pmis_coarsening, coarsening/algorithms.rs:310-354; the reference draws the
// priorities from an unseeded thread_rng (:324) -- here a seeded SplitMix64.
int64_t pmis(const or_csr& a, double theta, uint64_t seed, std::vector<int64_t>& cpts,
             std::vector<int64_t>& f2c, or_csr* s_out) {
  const int64_t n = a.nrows;
  or_csr s = strength(a, theta);
  std::vector<double> prio(n);
  uint64_t state = seed;
  for (int64_t i = 0; i < n; ++i) prio[i] = (double)(splitmix64(state) >> 11) * 0x1.0p-53;
  std::vector<int64_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int64_t x, int64_t y) { return prio[x] > prio[y]; });
  std::vector<int> status(n, 0);
  f2c.assign(n, -1);
  cpts.clear();
  for (int64_t i : order) {
    if (status[i] != 0) continue;
    status[i] = 1;
    cpts.push_back(i);
    f2c[i] = (int64_t)cpts.size() - 1;
    for (int64_t k = s.rp[i]; k < s.rp[i + 1]; ++k)
      if (status[s.ci[k]] == 0) status[s.ci[k]] = 2;
  }
  assign_closest(f2c, status, s);
  if (s_out) *s_out = std::move(s);
  return (int64_t)cpts.size();
}

// create_classical_interpolation, interpolation.rs:38-188.
or_csr classical_interp(const or_csr& a, const std::vector<int64_t>& cpts, const or_csr& s) {
  const int64_t n = a.nrows;
  const int64_t nc = (int64_t)cpts.size();
  std::vector<int64_t> cmap(n, -1);
  for (int64_t l = 0; l < nc; ++l)
    if (cpts[l] < n) cmap[cpts[l]] = l;
  std::vector<std::vector<std::pair<int64_t, double>>> rows(n);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t i = 0; i < n; ++i) {
    auto& out = rows[i];
    if (cmap[i] >= 0) {
      out.emplace_back(cmap[i], 1.0);
      continue;
    }
    const int64_t* scols = s.ci.data() + s.rp[i];
    const int64_t ns = s.rp[i + 1] - s.rp[i];
    std::vector<int64_t> c_i, f_i;
    for (int64_t q = 0; q < ns; ++q) {
      int64_t nb = scols[q];
      if (cmap[nb] >= 0)
        c_i.push_back(nb);
      else if (nb != i)
        f_i.push_back(nb);
    }
    if (c_i.empty()) continue;
    double a_ii = 0.0, sum_weak = 0.0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) {
      int64_t nb = a.ci[k];
      if (nb == i)
        a_ii = a.v[k];
      else if (!std::binary_search(scols, scols + ns, nb))
        sum_weak += a.v[k];
    }
    double diagonal = a_ii + sum_weak;
    if (!(std::fabs(diagonal) > DBL_EPSILON)) continue;
    std::vector<double> denoms(f_i.size());
    for (size_t q = 0; q < f_i.size(); ++q) {
      double d = 0.0;
      for (int64_t m : c_i) d += csr_value(a, f_i[q], m);
      denoms[q] = d;
    }
    double neg_diag_inv = 1.0 / -diagonal;
    for (int64_t j : c_i) {
      double a_ij = csr_value(a, i, j);
      double indirect = 0.0;
      for (size_t q = 0; q < f_i.size(); ++q) {
        double den = denoms[q];
        if (std::fabs(den) > DBL_EPSILON) {
          double a_ik = csr_value(a, i, f_i[q]);
          double a_kj = csr_value(a, f_i[q], j);
          indirect += a_ik * a_kj / den;
        }
      }
      out.emplace_back(cmap[j], (a_ij + indirect) * neg_diag_inv);
    }
    std::stable_sort(out.begin(), out.end(),
                     [](const std::pair<int64_t, double>& x, const std::pair<int64_t, double>& y) {
                       return x.first < y.first;
                     });
  }
  or_csr p;
  p.nrows = n;
  p.ncols = nc;
  p.rp.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) p.rp[i + 1] = p.rp[i] + (int64_t)rows[i].size();
  p.ci.resize(p.rp[n]);
  p.v.resize(p.rp[n]);
  for (int64_t i = 0; i < n; ++i)
    for (size_t q = 0; q < rows[i].size(); ++q) {
      p.ci[p.rp[i] + q] = rows[i][q].first;
      p.v[p.rp[i] + q] = rows[i][q].second;
    }
  return p;
}

// Modified classical interpolation (Stueben 2001, "Algebraic multigrid (AMG):
// an introduction with applications", App. A.7.2; the sign-restricted form used by
// hypre BoomerAMG's classical-modified interpolation). Same sets C_i / F_i as
// classical_interp above, but for each strong F-neighbour k only the entries
// a_km whose sign is opposite to a_kk take part in the distribution, and an F
// neighbour with no such entry to C_i is lumped into the diagonal instead of
// being dropped, so row sums are preserved and no denominator can cancel.
or_csr modified_classical_interp(const or_csr& a, const std::vector<int64_t>& cpts, const or_csr& s) {
  const int64_t n = a.nrows;
  const int64_t nc = (int64_t)cpts.size();
  std::vector<int64_t> cmap(n, -1);
  for (int64_t l = 0; l < nc; ++l)
    if (cpts[l] < n) cmap[cpts[l]] = l;
  std::vector<std::vector<std::pair<int64_t, double>>> rows(n);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t i = 0; i < n; ++i) {
    auto& out = rows[i];
    if (cmap[i] >= 0) {
      out.emplace_back(cmap[i], 1.0);
      continue;
    }
    const int64_t* scols = s.ci.data() + s.rp[i];
    const int64_t ns = s.rp[i + 1] - s.rp[i];
    std::vector<int64_t> c_i, f_i;
    for (int64_t q = 0; q < ns; ++q) {
      int64_t nb = scols[q];
      if (cmap[nb] >= 0)
        c_i.push_back(nb);
      else if (nb != i)
        f_i.push_back(nb);
    }
    if (c_i.empty()) continue;
    double diagonal = 0.0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) {
      int64_t nb = a.ci[k];
      if (nb == i || !std::binary_search(scols, scols + ns, nb)) diagonal += a.v[k];
    }
    std::vector<double> num(c_i.size(), 0.0);
    for (size_t q = 0; q < c_i.size(); ++q) num[q] = csr_value(a, i, c_i[q]);
    for (int64_t k : f_i) {
      const double a_ik = csr_value(a, i, k);
      const double a_kk = csr_value(a, k, k);
      double den = 0.0;
      for (int64_t m : c_i) {
        const double v = csr_value(a, k, m);
        if (v * a_kk < 0.0) den += v;
      }
      if (den == 0.0) {
        diagonal += a_ik;
        continue;
      }
      for (size_t q = 0; q < c_i.size(); ++q) {
        const double v = csr_value(a, k, c_i[q]);
        if (v * a_kk < 0.0) num[q] += a_ik * v / den;
      }
    }
    if (!(std::fabs(diagonal) > DBL_EPSILON)) continue;
    const double neg_diag_inv = 1.0 / -diagonal;
    for (size_t q = 0; q < c_i.size(); ++q) out.emplace_back(cmap[c_i[q]], num[q] * neg_diag_inv);
    std::stable_sort(out.begin(), out.end(),
                     [](const std::pair<int64_t, double>& x, const std::pair<int64_t, double>& y) {
                       return x.first < y.first;
                     });
  }
  or_csr p;
  p.nrows = n;
  p.ncols = nc;
  p.rp.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) p.rp[i + 1] = p.rp[i] + (int64_t)rows[i].size();
  p.ci.resize(p.rp[n]);
  p.v.resize(p.rp[n]);
  for (int64_t i = 0; i < n; ++i)
    for (size_t q = 0; q < rows[i].size(); ++q) {
      p.ci[p.rp[i] + q] = rows[i][q].first;
      p.v[p.rp[i] + q] = rows[i][q].second;
    }
  return p;
}

// Truncation of the interpolation rows (the max_interpolation_points argument
// of interpolation.rs:42, unused by the reference): rows with more than k
// weights keep the k of largest magnitude (ties: the smaller column), scaled by
// (sum of all) / (sum of kept), both summed in ascending column order.
or_csr truncate_interp(const or_csr& p, int k) {
  if (k <= 0) return p;
  or_csr t;
  t.nrows = p.nrows;
  t.ncols = p.ncols;
  t.rp.assign(p.nrows + 1, 0);
  for (int64_t i = 0; i < p.nrows; ++i) {
    const int64_t a = p.rp[i], b = p.rp[i + 1];
    if (b - a <= k) {
      for (int64_t e = a; e < b; ++e) {
        t.ci.push_back(p.ci[e]);
        t.v.push_back(p.v[e]);
      }
    } else {
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
      for (int64_t e : order) {
        t.ci.push_back(p.ci[e]);
        t.v.push_back(p.v[e] * scale);
      }
    }
    t.rp[i + 1] = (int64_t)t.ci.size();
  }
  return t;
}

// create_direct_interpolation, interpolation.rs:191-217.
or_csr direct_interp(const std::vector<int64_t>& f2c, int64_t n, int64_t nc) {
  or_csr p;
  p.nrows = n;
  p.ncols = nc;
  p.rp.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) {
    if (f2c[i] >= 0) {
      p.ci.push_back(f2c[i]);
      p.v.push_back(1.0);
    }
    p.rp[i + 1] = (int64_t)p.ci.size();
  }
  return p;
}

// JacobiSmoother::apply, smoothers.rs:160-194.
void jacobi_sweeps(const or_csr& a, double* x, const double* b, double omega, int iters) {
  std::vector<double> xo(a.nrows);
  for (int it = 0; it < iters; ++it) {
    std::copy(x, x + a.nrows, xo.begin());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < a.nrows; ++i) {
      double sum = 0.0, diag = 0.0;
      for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) {
        if (a.ci[k] == i)
          diag = a.v[k];
        else
          sum += a.v[k] * xo[a.ci[k]];
      }
      if (std::fabs(diag) > kDiagEps) {
        double nv = (b[i] - sum) / diag;
        x[i] = xo[i] + omega * (nv - xo[i]);
      }
    }
  }
}

// GaussSeidelSmoother::apply, smoothers.rs:45-82 (forward) and the backward
// half of SymmetricGaussSeidelSmoother, smoothers.rs:84-138.
void gs_sweep(const or_csr& a, double* x, const double* b, double omega, bool backward) {
  for (int64_t q = 0; q < a.nrows; ++q) {
    int64_t i = backward ? a.nrows - 1 - q : q;
    double sum = 0.0, diag = 0.0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) {
      if (a.ci[k] == i)
        diag = a.v[k];
      else
        sum += a.v[k] * x[a.ci[k]];
    }
    if (std::fabs(diag) > kDiagEps) {
      double nv = (b[i] - sum) / diag;
      x[i] = x[i] + omega * (nv - x[i]);
    }
  }
}

void smooth(const or_csr& a, double* x, const double* b, int kind, double omega, int iters) {
  if (kind == OR_SMOOTH_JACOBI) {
    jacobi_sweeps(a, x, b, omega, iters);
  } else if (kind == OR_SMOOTH_GS) {
    for (int it = 0; it < iters; ++it) gs_sweep(a, x, b, omega, false);
  } else {
    for (int it = 0; it < iters; ++it) gs_sweep(a, x, b, omega, false);
    for (int it = 0; it < iters; ++it) gs_sweep(a, x, b, omega, true);
  }
}

// Dense LU with partial pivoting (coarsest-level direct solve).
int dense_solve(const or_csr& a, const double* b, double* x) {
  const int64_t n = a.nrows;
  std::vector<double> m((size_t)n * n, 0.0);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) m[(size_t)i * n + a.ci[k]] += a.v[k];
  std::vector<double> rhs(b, b + n);
  for (int64_t c = 0; c < n; ++c) {
    int64_t piv = c;
    for (int64_t r = c + 1; r < n; ++r)
      if (std::fabs(m[(size_t)r * n + c]) > std::fabs(m[(size_t)piv * n + c])) piv = r;
    if (m[(size_t)piv * n + c] == 0.0) return -1;
    if (piv != c) {
      for (int64_t k = 0; k < n; ++k) std::swap(m[(size_t)c * n + k], m[(size_t)piv * n + k]);
      std::swap(rhs[c], rhs[piv]);
    }
    double d = m[(size_t)c * n + c];
#pragma omp parallel for schedule(static) if (n > 512)
    for (int64_t r = c + 1; r < n; ++r) {
      double f = m[(size_t)r * n + c] / d;
      if (f == 0.0) continue;
      for (int64_t k = c; k < n; ++k) m[(size_t)r * n + k] -= f * m[(size_t)c * n + k];
      rhs[r] -= f * rhs[c];
    }
  }
  for (int64_t r = n - 1; r >= 0; --r) {
    double s = rhs[r];
    for (int64_t k = r + 1; k < n; ++k) s -= m[(size_t)r * n + k] * x[k];
    x[r] = s / m[(size_t)r * n + r];
  }
  return 0;
}

}  // namespace

struct or_amg {
  or_amg_config cfg;
  std::vector<or_csr> A, P, R;
  // Dense LU factor of the coarsest level (row-major, with pivots), when used.
  std::vector<double> lu;
  std::vector<int64_t> piv;
  mutable std::vector<std::vector<double>> ws_r, ws_rc, ws_xc, ws_e, ws_ax;
};

namespace {

void lu_factor(const or_csr& a, std::vector<double>& m, std::vector<int64_t>& piv) {
  const int64_t n = a.nrows;
  m.assign((size_t)n * n, 0.0);
  piv.resize(n);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) m[(size_t)i * n + a.ci[k]] += a.v[k];
  for (int64_t c = 0; c < n; ++c) {
    int64_t p = c;
    for (int64_t r = c + 1; r < n; ++r)
      if (std::fabs(m[(size_t)r * n + c]) > std::fabs(m[(size_t)p * n + c])) p = r;
    piv[c] = p;
    if (p != c)
      for (int64_t k = 0; k < n; ++k) std::swap(m[(size_t)c * n + k], m[(size_t)p * n + k]);
    double d = m[(size_t)c * n + c];
    if (d == 0.0) continue;
#pragma omp parallel for schedule(static) if (n > 256)
    for (int64_t r = c + 1; r < n; ++r) {
      double f = m[(size_t)r * n + c] / d;
      m[(size_t)r * n + c] = f;
      if (f == 0.0) continue;
      for (int64_t k = c + 1; k < n; ++k) m[(size_t)r * n + k] -= f * m[(size_t)c * n + k];
    }
  }
}

// Solve with the factors of lu_factor: P b first (every exchange, in order),
// then L y = P b and U x = y. (The stored multipliers of L are those of the
// rows' final positions, so the exchanges cannot be interleaved with the
// forward substitution.)
void lu_solve(const std::vector<double>& m, const std::vector<int64_t>& piv, int64_t n,
              const double* b, double* x) {
  std::vector<double> y(b, b + n);
  for (int64_t c = 0; c < n; ++c)
    if (piv[c] != c) std::swap(y[c], y[piv[c]]);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t r = c + 1; r < n; ++r) y[r] -= m[(size_t)r * n + c] * y[c];
  for (int64_t r = n - 1; r >= 0; --r) {
    double s = y[r];
    for (int64_t k = r + 1; k < n; ++k) s -= m[(size_t)r * n + k] * x[k];
    x[r] = s / m[(size_t)r * n + r];
  }
}

// AlgebraicMultigrid::v_cycle, amg.rs:423-503.
void v_cycle(const or_amg& h, size_t l, const double* b, double* x) {
  const or_csr& a = h.A[l];
  const int64_t n = a.nrows;
  const or_amg_config& c = h.cfg;
  if (l + 1 < h.A.size()) {
    smooth(a, x, b, c.smoother, c.relaxation, c.pre_smooth);
    std::vector<double>& ax = h.ws_ax[l];
    std::vector<double>& r = h.ws_r[l];
    spmv_raw(a, x, ax.data());
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
    std::vector<double>& rc = h.ws_rc[l];
    spmv_raw(h.R[l], r.data(), rc.data());
    std::vector<double>& xc = h.ws_xc[l];
    std::fill(xc.begin(), xc.end(), 0.0);
    v_cycle(h, l + 1, rc.data(), xc.data());
    std::vector<double>& e = h.ws_e[l];
    spmv_raw(h.P[l], xc.data(), e.data());
    for (int64_t i = 0; i < n; ++i) x[i] += e[i];
    smooth(a, x, b, c.smoother, c.relaxation, c.post_smooth);
  } else if (c.coarse_solve == OR_COARSE_DENSE) {
    lu_solve(h.lu, h.piv, n, b, x);
  } else {
    smooth(a, x, b, c.smoother, c.relaxation, c.coarse_sweeps);
  }
}

// DiagJacobi::new, cfd-1d/src/solver/core/linear_system.rs:270-299.
int jacobi_inverse(const or_csr& a, std::vector<double>& inv) {
  inv.assign(a.nrows, 1.0);
  for (int64_t i = 0; i < a.nrows; ++i) {
    double d = csr_value(a, i, i);
    if (!std::isfinite(d)) return -1;
    inv[i] = std::fabs(d) <= DBL_EPSILON ? 1.0 : 1.0 / d;
  }
  return 0;
}

struct Precond {
  int kind;
  const or_amg* amg;
  std::vector<double> inv;
  const or_simple* simple = nullptr;
  const or_component_block* cblock = nullptr;
  void apply(const double* r, double* z, int64_t n) const {
    if (kind == OR_PRE_JACOBI) {
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i) z[i] = r[i] * inv[i];
    } else if (kind == OR_PRE_AMG) {
      or_amg_apply(amg, r, z);
    } else if (kind == OR_PRE_SIMPLE) {
      or_simple_apply(simple, r, z);
    } else if (kind == OR_PRE_BLOCK_DIAGONAL) {
      for (int64_t i = 0; i < n; ++i) z[i] = r[i] * simple->bdinv[i];
    } else if (kind == OR_PRE_COMPONENT_BLOCK) {
      or_component_block_apply(cblock, r, z);
    } else {
      std::copy(r, r + n, z);
    }
  }
};

}  // namespace

extern "C" {

or_csr* or_csr_new(int64_t nrows, int64_t ncols, int64_t nnz, const int64_t* row_ptr,
                   const int64_t* col, const double* val) {
  or_csr* a = new or_csr;
  a->nrows = nrows;
  a->ncols = ncols;
  a->rp.assign(row_ptr, row_ptr + nrows + 1);
  a->ci.assign(col, col + nnz);
  a->v.assign(val, val + nnz);
  return a;
}

void or_csr_info(const or_csr* a, int64_t* nrows, int64_t* ncols, int64_t* nnz) {
  *nrows = a->nrows;
  *ncols = a->ncols;
  *nnz = a->nnz();
}

void or_csr_export(const or_csr* a, int64_t* row_ptr, int64_t* col, double* val) {
  std::copy(a->rp.begin(), a->rp.end(), row_ptr);
  std::copy(a->ci.begin(), a->ci.end(), col);
  std::copy(a->v.begin(), a->v.end(), val);
}

void or_csr_free(or_csr* a) { delete a; }

void or_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}
int or_get_threads(void) { return omp_get_max_threads(); }

void or_spmv(const or_csr* a, const double* x, double* y) { spmv_raw(*a, x, y); }
or_csr* or_strength(const or_csr* a, double theta) { return new or_csr(strength(*a, theta)); }
or_csr* or_transpose(const or_csr* a) { return new or_csr(transpose(*a)); }
or_csr* or_spgemm(const or_csr* a, const or_csr* b) { return new or_csr(spgemm(*a, *b)); }

int64_t or_coarsen(const or_csr* a, int kind, double theta, int64_t param, uint64_t seed,
                   int literal_scan, int64_t* coarse_points, int64_t* f2c) {
  std::vector<int64_t> cp, map;
  int64_t nc;
  if (kind == OR_RUGE_STUEBEN)
    nc = ruge_stueben(*a, theta, literal_scan != 0, cp, map, nullptr);
  else if (kind == OR_AGGREGATION)
    nc = aggregation(*a, param, cp, map, nullptr);
  else
    nc = pmis(*a, theta, seed, cp, map, nullptr);
  std::copy(cp.begin(), cp.end(), coarse_points);
  std::copy(map.begin(), map.end(), f2c);
  return nc;
}

or_csr* or_classical_interp(const or_csr* a, const int64_t* coarse_points, int64_t nc,
                            const or_csr* s) {
  std::vector<int64_t> cp(coarse_points, coarse_points + nc);
  return new or_csr(classical_interp(*a, cp, *s));
}

or_csr* or_direct_interp(const int64_t* f2c, int64_t n, int64_t nc) {
  std::vector<int64_t> m(f2c, f2c + n);
  return new or_csr(direct_interp(m, n, nc));
}

void or_smooth(const or_csr* a, double* x, const double* b, int kind, double omega, int iters) {
  smooth(*a, x, b, kind, omega, iters);
}

int or_dense_solve(const or_csr* a, const double* b, double* x) { return dense_solve(*a, b, x); }

// AlgebraicMultigrid::setup / build_next_level, amg.rs:217-380.
or_amg* or_amg_setup(const or_csr* a, const or_amg_config* cfg) {
  or_amg* h = new or_amg;
  h->cfg = *cfg;
  h->A.push_back(*a);
  while ((int)h->A.size() < cfg->max_levels && h->A.back().nrows > cfg->min_coarse_size) {
    const or_csr& cur = h->A.back();
    std::vector<int64_t> cp, map;
    or_csr s;
    int64_t nc;
    if (cfg->coarsening == OR_RUGE_STUEBEN)
      nc = ruge_stueben(cur, cfg->strength_threshold, false, cp, map, &s);
    else if (cfg->coarsening == OR_AGGREGATION)
      nc = aggregation(cur, cfg->aggregate_size, cp, map, &s);
    else
      nc = pmis(cur, cfg->strength_threshold, cfg->seed, cp, map, &s);
    if (cfg->coarse_order == 1) {
      // Number coarse points in ascending fine index instead of selection order.
      std::vector<int64_t> sorted(cp);
      std::sort(sorted.begin(), sorted.end());
      std::vector<int64_t> newid(cur.nrows, -1);
      for (size_t q = 0; q < sorted.size(); ++q) newid[sorted[q]] = (int64_t)q;
      for (int64_t i = 0; i < cur.nrows; ++i)
        if (map[i] >= 0) map[i] = newid[cp[map[i]]];
      cp.swap(sorted);
    }
    or_csr p = cfg->interpolation == 0   ? classical_interp(cur, cp, s)
               : cfg->interpolation == 2 ? modified_classical_interp(cur, cp, s)
                                         : direct_interp(map, cur.nrows, nc);
    if (cfg->max_interp_points > 0) p = truncate_interp(p, cfg->max_interp_points);
    or_csr r = transpose(p);
    or_csr ra = spgemm(r, cur);
    or_csr ac = spgemm(ra, p);
    const int64_t n_cur = cur.nrows;  // `cur` refers into h->A, which the push_back may move
    h->P.push_back(std::move(p));
    h->R.push_back(std::move(r));
    h->A.push_back(std::move(ac));
    if (nc == 0 || nc >= n_cur) break;  // no progress: stop coarsening
  }
  if (cfg->coarse_solve == OR_COARSE_DENSE) lu_factor(h->A.back(), h->lu, h->piv);
  size_t L = h->A.size();
  h->ws_r.resize(L);
  h->ws_rc.resize(L);
  h->ws_xc.resize(L);
  h->ws_e.resize(L);
  h->ws_ax.resize(L);
  for (size_t l = 0; l + 1 < L; ++l) {
    h->ws_r[l].assign(h->A[l].nrows, 0.0);
    h->ws_ax[l].assign(h->A[l].nrows, 0.0);
    h->ws_e[l].assign(h->A[l].nrows, 0.0);
    h->ws_rc[l].assign(h->A[l + 1].nrows, 0.0);
    h->ws_xc[l].assign(h->A[l + 1].nrows, 0.0);
  }
  return h;
}

// A hierarchy given level by level (e.g. exported from another setup), for
// timing the solve phase on an identical hierarchy.
or_amg* or_amg_from_levels(int nlev, const or_csr* const* a, const or_csr* const* p, const or_csr* const* r,
                           const or_amg_config* cfg) {
  or_amg* h = new or_amg;
  h->cfg = *cfg;
  for (int l = 0; l < nlev; ++l) {
    h->A.push_back(*a[l]);
    if (l + 1 < nlev) {
      h->P.push_back(*p[l]);
      h->R.push_back(*r[l]);
    }
  }
  if (cfg->coarse_solve == OR_COARSE_DENSE) lu_factor(h->A.back(), h->lu, h->piv);
  size_t L = h->A.size();
  h->ws_r.resize(L);
  h->ws_rc.resize(L);
  h->ws_xc.resize(L);
  h->ws_e.resize(L);
  h->ws_ax.resize(L);
  for (size_t l = 0; l + 1 < L; ++l) {
    h->ws_r[l].assign(h->A[l].nrows, 0.0);
    h->ws_ax[l].assign(h->A[l].nrows, 0.0);
    h->ws_e[l].assign(h->A[l].nrows, 0.0);
    h->ws_rc[l].assign(h->A[l + 1].nrows, 0.0);
    h->ws_xc[l].assign(h->A[l + 1].nrows, 0.0);
  }
  return h;
}

int or_amg_num_levels(const or_amg* h) { return (int)h->A.size(); }

const or_csr* or_amg_level(const or_amg* h, int level, int which) {
  if (level < 0 || level >= (int)h->A.size()) return nullptr;
  if (which == 0) return &h->A[level];
  if (level >= (int)h->P.size()) return nullptr;
  return which == 1 ? &h->P[level] : &h->R[level];
}

// Preconditioner::apply_to, amg.rs:507-557: z = 0, then one V-cycle.
void or_amg_apply(const or_amg* h, const double* r, double* z) {
  std::fill(z, z + h->A[0].nrows, 0.0);
  v_cycle(*h, 0, r, z);
}

void or_amg_free(or_amg* h) { delete h; }

// Preconditioned CG (Saad 2003, Alg. 9.1) with the termination mapping of
// krylov.rs:375-401. threshold = max(tolerance, relative_tolerance * ||r0||)
// (the absolute-or-relative test of cfd-core compute/solver/convergence.rs:26-30).
int or_pcg(const or_csr* a, int precond, const or_amg* amg, const double* b, double* x,
           const or_solver_config* cfg, or_report* rep, double* history) {
  const int64_t n = a->nrows;
  if (a->ncols != n) return -1;
  Precond M{precond, amg, {}};
  if (precond == OR_PRE_JACOBI && jacobi_inverse(*a, M.inv) != 0) return -2;
  std::vector<double> r(n), z(n), p(n), q(n);
  spmv_raw(*a, x, q.data());
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
  double rn = std::sqrt(dot(n, r.data(), r.data()));
  rep->initial_residual = rn;
  rep->threshold = std::max(cfg->tolerance, cfg->relative_tolerance * rn);
  rep->final_residual = rn;
  rep->iterations = 0;
  if (history) history[0] = rn;
  if (rn <= rep->threshold) {
    rep->termination = OR_TERM_INITIAL_RESIDUAL;
    return 0;
  }
  M.apply(r.data(), z.data(), n);
  double rho = dot(n, r.data(), z.data());
  std::copy(z.begin(), z.end(), p.begin());
  for (int64_t it = 1; it <= cfg->max_iterations; ++it) {
    spmv_raw(*a, p.data(), q.data());
    double pq = dot(n, p.data(), q.data());
    if (!(pq > 0.0)) {
      rep->termination = OR_TERM_NON_POSITIVE_CURVATURE;
      return 0;
    }
    double alpha = rho / pq;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    rn = std::sqrt(dot(n, r.data(), r.data()));
    rep->iterations = it;
    rep->final_residual = rn;
    if (history) history[it] = rn;
    if (!std::isfinite(rn)) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    if (rn <= rep->threshold) {
      rep->termination = OR_TERM_CONVERGED;
      return 0;
    }
    M.apply(r.data(), z.data(), n);
    double rho_new = dot(n, r.data(), z.data());
    if (rho_new == 0.0 || !std::isfinite(rho_new)) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    double beta = rho_new / rho;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rho = rho_new;
  }
  rep->termination = OR_TERM_MAX_ITERATIONS;
  return 0;
}

// Jacobi-PCG with the convergence test of the 1-D network solver: the
// row-equilibrated residual ||D (b - A x)||_2 with D = 1 / max_j |a_ij|
// (identity where the row maximum is not above f64::EPSILON or not finite),
// crates/cfd-1d/src/solver/core/linear_system.rs:157-204; threshold
// max(tolerance, relative_tolerance * ||D r0||).
int or_pcg_equilibrated(const or_csr* a, const double* b, double* x, const or_solver_config* cfg, or_report* rep) {
  const int64_t n = a->nrows;
  if (a->ncols != n) return -1;
  Precond M{OR_PRE_JACOBI, nullptr, {}};
  if (jacobi_inverse(*a, M.inv) != 0) return -2;
  std::vector<double> s(n, 1.0);
  for (int64_t i = 0; i < n; ++i) {
    double mx = 0.0;
    for (int64_t k = a->rp[i]; k < a->rp[i + 1]; ++k) mx = std::max(mx, std::fabs(a->v[k]));
    if (mx > DBL_EPSILON && std::isfinite(mx)) s[i] = 1.0 / mx;
  }
  auto enorm = [&](const std::vector<double>& r) {
    double t = 0.0;
    for (int64_t i = 0; i < n; ++i) t += (s[i] * r[i]) * (s[i] * r[i]);
    return std::sqrt(t);
  };
  std::vector<double> r(n), z(n), p(n), q(n);
  spmv_raw(*a, x, q.data());
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
  double e = enorm(r);
  rep->initial_residual = e;
  rep->threshold = std::max(cfg->tolerance, cfg->relative_tolerance * e);
  rep->final_residual = e;
  rep->iterations = 0;
  if (!std::isfinite(e)) {
    rep->termination = OR_TERM_BREAKDOWN;
    return 0;
  }
  if (e <= rep->threshold) {
    rep->termination = OR_TERM_INITIAL_RESIDUAL;
    return 0;
  }
  M.apply(r.data(), z.data(), n);
  double rho = 0.0;
  for (int64_t i = 0; i < n; ++i) rho += r[i] * z[i];
  p = z;
  for (int64_t it = 1; it <= cfg->max_iterations; ++it) {
    spmv_raw(*a, p.data(), q.data());
    double pq = 0.0;
    for (int64_t i = 0; i < n; ++i) pq += p[i] * q[i];
    if (!(pq > 0.0)) {
      rep->termination = OR_TERM_NON_POSITIVE_CURVATURE;
      return 0;
    }
    const double alpha = rho / pq;
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    e = enorm(r);
    rep->iterations = it;
    rep->final_residual = e;
    if (!std::isfinite(e)) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    if (e <= rep->threshold) {
      rep->termination = OR_TERM_CONVERGED;
      return 0;
    }
    M.apply(r.data(), z.data(), n);
    double rn = 0.0;
    for (int64_t i = 0; i < n; ++i) rn += r[i] * z[i];
    if (rn == 0.0 || !std::isfinite(rn)) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    const double beta = rn / rho;
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rho = rn;
  }
  rep->termination = OR_TERM_MAX_ITERATIONS;
  return 0;
}

// Right-preconditioned BiCGSTAB (Saad 2003, Alg. 7.7 with M^-1 applied to p and s).
// GMRES restart ladder, RestartWidth::covering (krylov.rs:96-120): the
// smallest of 8, 16, 32, 64, 128, 256 at least as large as the request,
// saturating at 256.
int or_gmres_width(int64_t requested) {
  int w = 8;
  while (w < 256 && w < requested) w *= 2;
  return w;
}

// Restarted GMRES(m) with right preconditioning, the solver behind
// krylov::gmres_preconditioned (krylov.rs:150-221; the recurrence lives in
// athena-core, not vendored, so it is restated from Saad 2003, Alg. 9.5):
//   cycle: beta = ||r||, v0 = r / beta; for j < m: w = A M^-1 v_j, classical
//   Gram-Schmidt against v_0..v_j applied twice (CGS2), h_{j+1,j} = ||w||,
//   Givens rotations on the Hessenberg column, implicit residual |g_{j+1}|;
//   the cycle ends at the threshold, at the budget or when h_{j+1,j} = 0;
//   then x += M^-1 (V y) with H y = g, and the true residual b - A x decides:
//   converged, budget spent, or restart.
// iterations counts Arnoldi steps over all cycles; history[k] is the implicit
// residual after step k (history[0] = ||r0||).
static int gmres_impl(const or_csr* a, const Precond& M, int64_t restart, const double* b, double* x,
                      const or_solver_config* cfg, or_report* rep, double* history) {
  const int64_t n = a->nrows;
  const int m = or_gmres_width(restart);
  std::vector<double> V((size_t)(m + 1) * n), w(n), z(n), r(n), t(n);
  std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1), y(m), h1(m + 1), h2(m + 1);
  auto vec = [&](int k) { return V.data() + (size_t)k * n; };
  auto residual = [&]() {
    spmv_raw(*a, x, t.data());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - t[i];
    return std::sqrt(dot(n, r.data(), r.data()));
  };
  // h = V[0..k)^T w (one dot per basis vector)
  auto project = [&](int k, std::vector<double>& h) {
    for (int q = 0; q < k; ++q) h[q] = dot(n, vec(q), w.data());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      double s = 0.0;
      for (int q = 0; q < k; ++q) s += h[q] * vec(q)[i];
      w[i] -= s;
    }
  };
  double rn = residual();
  rep->initial_residual = rn;
  rep->threshold = std::max(cfg->tolerance, cfg->relative_tolerance * rn);
  rep->final_residual = rn;
  rep->iterations = 0;
  if (history) history[0] = rn;
  if (rn <= rep->threshold) {
    rep->termination = OR_TERM_INITIAL_RESIDUAL;
    return 0;
  }
  int64_t it = 0;
  for (;;) {
    const double beta = rn;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) vec(0)[i] = r[i] / beta;
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int cols = 0;
    for (int j = 0; j < m; ++j) {
      M.apply(vec(j), z.data(), n);
      spmv_raw(*a, z.data(), w.data());
      project(j + 1, h1);
      project(j + 1, h2);
      double* h = H.data() + (size_t)j * (m + 1);
      for (int q = 0; q <= j; ++q) h[q] = h1[q] + h2[q];
      const double hn = std::sqrt(dot(n, w.data(), w.data()));
      h[j + 1] = hn;
      if (hn > 0.0) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) vec(j + 1)[i] = w[i] / hn;
      }
      for (int q = 0; q < j; ++q) {
        const double tq = cs[q] * h[q] + sn[q] * h[q + 1];
        h[q + 1] = -sn[q] * h[q] + cs[q] * h[q + 1];
        h[q] = tq;
      }
      const double d = std::hypot(h[j], h[j + 1]);
      cs[j] = d > 0.0 ? h[j] / d : 1.0;
      sn[j] = d > 0.0 ? h[j + 1] / d : 0.0;
      h[j] = d;
      h[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      ++it;
      cols = j + 1;
      const double res = std::fabs(g[j + 1]);
      rep->iterations = it;
      if (history) history[it] = res;
      if (!std::isfinite(res)) {
        rep->termination = OR_TERM_BREAKDOWN;
        return 0;
      }
      if (res <= rep->threshold || it >= cfg->max_iterations || hn == 0.0) break;
    }
    // y = H^-1 g (upper triangular), x += M^-1 (V y)
    for (int q = cols - 1; q >= 0; --q) {
      double s = g[q];
      for (int l = q + 1; l < cols; ++l) s -= H[(size_t)l * (m + 1) + q] * y[l];
      y[q] = H[(size_t)q * (m + 1) + q] != 0.0 ? s / H[(size_t)q * (m + 1) + q] : 0.0;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      double s = 0.0;
      for (int q = 0; q < cols; ++q) s += y[q] * vec(q)[i];
      w[i] = s;
    }
    M.apply(w.data(), z.data(), n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) x[i] += z[i];
    rn = residual();
    rep->final_residual = rn;
    if (!std::isfinite(rn)) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    if (rn <= rep->threshold) {
      rep->termination = OR_TERM_CONVERGED;
      return 0;
    }
    if (it >= cfg->max_iterations) {
      rep->termination = OR_TERM_MAX_ITERATIONS;
      return 0;
    }
  }
}

int or_gmres(const or_csr* a, int precond, const or_amg* amg, int64_t restart, const double* b, double* x,
             const or_solver_config* cfg, or_report* rep, double* history) {
  if (a->ncols != a->nrows) return -1;
  Precond M{precond, amg, {}};
  if (precond == OR_PRE_JACOBI && jacobi_inverse(*a, M.inv) != 0) return -2;
  return gmres_impl(a, M, restart, b, x, cfg, rep, history);
}

int or_gmres_saddle(const or_csr* a, const or_simple* simple, int precond, int64_t restart, const double* b,
                    double* x, const or_solver_config* cfg, or_report* rep, double* history) {
  if (a->ncols != a->nrows || !simple || simple->nv + simple->np != a->nrows) return -1;
  if (precond != OR_PRE_SIMPLE && precond != OR_PRE_BLOCK_DIAGONAL) return -1;
  Precond M{precond, nullptr, {}, simple};
  return gmres_impl(a, M, restart, b, x, cfg, rep, history);
}

// SimplePreconditioner::new (block_preconditioner.rs:432-508): the momentum
// diagonal inverse (1 where |a_ii| <= 1e-14, diagonal_epsilon :40-42), the
// divergence rows D (pressure rows, velocity columns) and gradient columns G
// (velocity rows' pressure columns, gathered per pressure column in velocity
// order), and the inverse of diag(C - D diag(A)^-1 G) over the entries of D
// whose transposed position holds a G entry.
or_simple* or_simple_new(const or_csr* a, int64_t n_velocity) {
  const int64_t n = a->nrows;
  if (a->ncols != n || n_velocity < 0 || n_velocity > n) return nullptr;
  constexpr double eps = 1e-14;
  or_simple* S = new or_simple;
  S->nv = n_velocity;
  S->np = n - n_velocity;
  auto diag = [&](int64_t r) {
    for (int64_t k = a->rp[r]; k < a->rp[r + 1]; ++k)
      if (a->ci[k] == r) return a->v[k];
    return 0.0;
  };
  S->dinv.resize(S->nv);
  for (int64_t i = 0; i < S->nv; ++i) {
    const double d = diag(i);
    S->dinv[i] = std::fabs(d) > eps ? 1.0 / d : 1.0;
  }
  S->div_rows.resize(S->np);
  for (int64_t i = 0; i < S->np; ++i)
    for (int64_t k = a->rp[S->nv + i]; k < a->rp[S->nv + i + 1]; ++k)
      if (a->ci[k] < S->nv) S->div_rows[i].push_back({a->ci[k], a->v[k]});
  S->grad_cols.resize(S->np);
  for (int64_t v = 0; v < S->nv; ++v)
    for (int64_t k = a->rp[v]; k < a->rp[v + 1]; ++k)
      if (a->ci[k] >= S->nv && a->ci[k] < n) S->grad_cols[a->ci[k] - S->nv].push_back({v, a->v[k]});
  S->sinv.resize(S->np);
  for (int64_t i = 0; i < S->np; ++i) {
    double s = diag(S->nv + i);
    for (const auto& dv : S->div_rows[i])
      for (const auto& gv : S->grad_cols[i])
        if (gv.first == dv.first) {
          s -= dv.second * S->dinv[dv.first] * gv.second;
          break;
        }
    S->sinv[i] = std::fabs(s) > eps ? 1.0 / s : 1.0;
  }
  // BlockDiagonalPreconditioner::new (:258-366): the momentum diagonal (1 where
  // |a_ii| <= eps) inverted; per pressure row the absolute row sum over the
  // pressure block, or, where that is <= eps, the mean |momentum diagonal|
  // over the entries above eps (1 without velocities), inverted.
  S->bdinv.assign(n, 1.0);
  std::vector<double> md(S->nv);
  for (int64_t i = 0; i < S->nv; ++i) {
    const double d = diag(i);
    md[i] = std::fabs(d) > eps ? d : 1.0;
    S->bdinv[i] = std::fabs(md[i]) > eps ? 1.0 / md[i] : 1.0;
  }
  for (int64_t i = 0; i < S->np; ++i) {
    double row_sum = 0.0;
    for (int64_t k = a->rp[S->nv + i]; k < a->rp[S->nv + i + 1]; ++k)
      if (a->ci[k] >= S->nv) row_sum += std::fabs(a->v[k]);
    double pd = row_sum;
    if (!(row_sum > eps)) {
      double sum = 0.0;
      int64_t count = 0;
      for (int64_t v = 0; v < S->nv; ++v)
        if (std::fabs(md[v]) > eps) {
          sum += std::fabs(md[v]);
          ++count;
        }
      pd = count == 0 ? 1.0 : sum / (double)count;
    }
    S->bdinv[S->nv + i] = std::fabs(pd) > eps ? 1.0 / pd : 1.0;
  }
  return S;
}

void or_block_diagonal_apply(const or_simple* S, const double* b, double* x) {
  for (int64_t i = 0; i < S->nv + S->np; ++i) x[i] = b[i] * S->bdinv[i];
}

// SimplePreconditioner::apply (block_preconditioner.rs:521-568):
// u* = diag(A)^-1 f; p = S^-1 (g - D u*); u = u* - diag(A)^-1 G p, the last
// step pressure column by pressure column.
void or_simple_apply(const or_simple* S, const double* b, double* x) {
  std::vector<double> us(S->nv), p(S->np);
  for (int64_t v = 0; v < S->nv; ++v) us[v] = b[v] * S->dinv[v];
  for (int64_t i = 0; i < S->np; ++i) {
    double bu = 0.0;
    for (const auto& dv : S->div_rows[i]) bu += dv.second * us[dv.first];
    p[i] = (b[S->nv + i] - bu) * S->sinv[i];
  }
  for (int64_t v = 0; v < S->nv; ++v) x[v] = us[v];
  for (int64_t i = 0; i < S->np; ++i)
    for (const auto& gv : S->grad_cols[i]) x[gv.first] -= S->dinv[gv.first] * gv.second * p[i];
  for (int64_t i = 0; i < S->np; ++i) x[S->nv + i] = p[i];
}

void or_simple_free(or_simple* S) { delete S; }

// ComponentBlockPreconditioner::new_with_symbols (block_preconditioner.rs:707-826).
or_component_block* or_component_block_new(const or_csr* a, int64_t nv, double pivot_tolerance, int* error) {
  constexpr double eps = 1e-14;  // diagonal_epsilon (:40-42)
  const int64_t n = a->nrows;
  *error = 0;
  if (a->ncols != n || nv <= 0 || nv > n || nv % 3 != 0) {
    *error = 1;  // size mismatch or velocity count not divisible by 3
    return nullptr;
  }
  // stabilize_preconditioner_diagonal (:71-107) of one block given as rows of
  // (column, value) in build order, summed per column: a row whose diagonal is
  // at most eps in magnitude gets max(row_scale * pivot_tolerance, eps) added.
  auto stabilize = [&](std::vector<std::map<int64_t, double>>& rows) {
    for (int64_t r = 0; r < (int64_t)rows.size(); ++r) {
      double diag = 0.0, scale = 0.0;
      for (const auto& cv : rows[r]) {
        scale = std::max(scale, std::fabs(cv.second));
        if (cv.first == r) diag += cv.second;
      }
      if (std::fabs(diag) <= eps) rows[r][r] += std::max(scale * pivot_tolerance, eps);
    }
  };
  auto* C = new or_component_block;
  C->nv = nv;
  C->np = n - nv;
  C->cs = nv / 3;
  const int64_t cs = C->cs;
  for (int comp = 0; comp < 3; ++comp) {
    const int64_t off = comp * cs;
    std::vector<std::map<int64_t, double>> rows(cs);
    for (int64_t lr = 0; lr < cs; ++lr) {
      const int64_t g = off + lr;
      for (int64_t k = a->rp[g]; k < a->rp[g + 1]; ++k) {
        const int64_t col = a->ci[k];
        if (col >= nv) continue;
        if (col / cs != comp) {
          if (std::fabs(a->v[k]) > eps) {
            *error = 2;  // velocity component coupling
            delete C;
            return nullptr;
          }
          continue;
        }
        rows[lr][col - off] += a->v[k];
      }
    }
    stabilize(rows);
    or_csr blk;
    blk.nrows = blk.ncols = cs;
    blk.rp.assign(cs + 1, 0);
    for (int64_t r = 0; r < cs; ++r) {
      for (const auto& cv : rows[r]) {
        blk.ci.push_back(cv.first);
        blk.v.push_back(cv.second);
      }
      blk.rp[r + 1] = (int64_t)blk.ci.size();
    }
    lu_factor(blk, C->lu[comp], C->piv[comp]);
    for (int64_t i = 0; i < cs; ++i)
      if (C->lu[comp][(size_t)i * cs + i] == 0.0) {
        *error = 3;  // singular component block
        delete C;
        return nullptr;
      }
  }
  // SIMPLE's parts (:432-508): diag(A)^-1, D rows, G per pressure column
  or_simple* S = or_simple_new(a, nv);
  C->div_rows = S->div_rows;
  C->grad_rows.assign(nv, {});
  for (int64_t pc = 0; pc < C->np; ++pc)
    for (const auto& gv : S->grad_cols[pc]) C->grad_rows[gv.first].push_back({pc, gv.second});
  for (auto& row : C->grad_rows) std::sort(row.begin(), row.end());
  // pressure Schur approximation in build order: C entries, then per D entry
  // (v, d) and pressure column pc in order every G entry (v, pc, g) as -d dinv_v g
  std::vector<std::map<int64_t, double>> prow(C->np);
  for (int64_t i = 0; i < C->np; ++i) {
    auto& row = prow[i];
    for (int64_t k = a->rp[nv + i]; k < a->rp[nv + i + 1]; ++k)
      if (a->ci[k] >= nv && a->ci[k] < n) row[a->ci[k] - nv] += a->v[k];
    for (const auto& dv : S->div_rows[i]) {
      const double minv = S->dinv[dv.first];
      for (const auto& gv : C->grad_rows[dv.first]) row[gv.first] += -dv.second * minv * gv.second;
    }
  }
  or_simple_free(S);
  stabilize(prow);
  // lumped_pressure_preconditioner (:112-137): signed row sum, else the diagonal
  C->pinv.assign(C->np, 1.0);
  for (int64_t i = 0; i < C->np; ++i) {
    double sum = 0.0, diag = 0.0;
    for (const auto& cv : prow[i]) {
      sum += cv.second;
      if (cv.first == i) diag = cv.second;
    }
    const double scale = std::fabs(sum) > eps ? sum : diag;
    C->pinv[i] = std::fabs(scale) > eps ? 1.0 / scale : 1.0;
  }
  return C;
}

// The athena apply of ComponentBlockPreconditioner (block_preconditioner.rs:920-975).
void or_component_block_apply(const or_component_block* C, const double* r, double* z) {
  const int64_t cs = C->cs, nv = C->nv, np = C->np;
  for (int comp = 0; comp < 3; ++comp) lu_solve(C->lu[comp], C->piv[comp], cs, r + comp * cs, z + comp * cs);
  for (int64_t i = 0; i < np; ++i) {
    double t = r[nv + i];
    for (const auto& dv : C->div_rows[i]) t -= dv.second * z[dv.first];
    z[nv + i] = t * C->pinv[i];
  }
  std::vector<double> rhs(cs), sol(cs);
  for (int comp = 0; comp < 3; ++comp) {
    const int64_t off = comp * cs;
    std::fill(rhs.begin(), rhs.end(), 0.0);
    // each velocity's gradient entries in ascending pressure column (the
    // reference loops over pressure columns, then their velocities)
    for (int64_t v = off; v < off + cs; ++v)
      for (const auto& gv : C->grad_rows[v]) rhs[v - off] += gv.second * z[nv + gv.first];
    lu_solve(C->lu[comp], C->piv[comp], cs, rhs.data(), sol.data());
    for (int64_t k = 0; k < cs; ++k) z[off + k] -= sol[k];
  }
}

void or_component_block_free(or_component_block* C) { delete C; }

int or_gmres_component_block(const or_csr* a, const or_component_block* c, int64_t restart, const double* b,
                             double* x, const or_solver_config* cfg, or_report* rep, double* history) {
  if (a->ncols != a->nrows || !c || c->nv + c->np != a->nrows) return -1;
  Precond M{OR_PRE_COMPONENT_BLOCK, nullptr, {}};
  M.cblock = c;
  return gmres_impl(a, M, restart, b, x, cfg, rep, history);
}

int or_bicgstab(const or_csr* a, int precond, const or_amg* amg, const double* b, double* x,
                const or_solver_config* cfg, or_report* rep, double* history) {
  const int64_t n = a->nrows;
  if (a->ncols != n) return -1;
  Precond M{precond, amg, {}};
  if (precond == OR_PRE_JACOBI && jacobi_inverse(*a, M.inv) != 0) return -2;
  std::vector<double> r(n), rh(n), p(n, 0.0), v(n, 0.0), ph(n), s(n), sh(n), t(n);
  spmv_raw(*a, x, t.data());
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - t[i];
  std::copy(r.begin(), r.end(), rh.begin());
  double rn = std::sqrt(dot(n, r.data(), r.data()));
  rep->initial_residual = rn;
  rep->threshold = std::max(cfg->tolerance, cfg->relative_tolerance * rn);
  rep->final_residual = rn;
  rep->iterations = 0;
  if (history) history[0] = rn;
  if (rn <= rep->threshold) {
    rep->termination = OR_TERM_INITIAL_RESIDUAL;
    return 0;
  }
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  for (int64_t it = 1; it <= cfg->max_iterations; ++it) {
    double rho_new = dot(n, rh.data(), r.data());
    if (rho_new == 0.0 || !std::isfinite(rho_new)) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    if (it == 1) {
      std::copy(r.begin(), r.end(), p.begin());
    } else {
      double beta = (rho_new / rho) * (alpha / omega);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    }
    M.apply(p.data(), ph.data(), n);
    spmv_raw(*a, ph.data(), v.data());
    double rv = dot(n, rh.data(), v.data());
    if (rv == 0.0 || !std::isfinite(rv)) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    alpha = rho_new / rv;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
    double sn = std::sqrt(dot(n, s.data(), s.data()));
    rep->iterations = it;
    if (sn <= rep->threshold) {
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i) x[i] += alpha * ph[i];
      rep->final_residual = sn;
      if (history) history[it] = sn;
      rep->termination = OR_TERM_CONVERGED;
      return 0;
    }
    M.apply(s.data(), sh.data(), n);
    spmv_raw(*a, sh.data(), t.data());
    double tt = dot(n, t.data(), t.data());
    if (tt == 0.0 || !std::isfinite(tt)) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    omega = dot(n, t.data(), s.data()) / tt;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * ph[i] + omega * sh[i];
      r[i] = s[i] - omega * t[i];
    }
    rn = std::sqrt(dot(n, r.data(), r.data()));
    rep->final_residual = rn;
    if (history) history[it] = rn;
    if (!std::isfinite(rn)) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    if (rn <= rep->threshold) {
      rep->termination = OR_TERM_CONVERGED;
      return 0;
    }
    if (omega == 0.0) {
      rep->termination = OR_TERM_BREAKDOWN;
      return 0;
    }
    rho = rho_new;
  }
  rep->termination = OR_TERM_MAX_ITERATIONS;
  return 0;
}

// MatrixAssembler::assemble_into (crates/cfd-1d/src/solver/core/matrix_assembly.rs:163-250):
// per edge in order, the self-loop and conductance checks (:184-203), then the
// COO pushes and RHS eliminations of the four cases (:208-231); Neumann
// sources added (:234-238); identity rows and RHS = p for fixed nodes
// (:240-246). The COO becomes CSR by a stable sort on (row, column) with
// duplicates summed in push order.
int or_network_assemble(int64_t n, int64_t m, const int64_t* ei, const int64_t* ej, const double* g,
                        const int8_t* fixed, const double* fixed_value, const double* neumann, or_csr** out,
                        double* rhs, int64_t* bad_edge) {
  struct Entry {
    int64_t r, c;
    double v;
  };
  *out = nullptr;
  *bad_edge = -1;
  std::vector<Entry> coo;
  std::fill(rhs, rhs + n, 0.0);
  for (int64_t e = 0; e < m; ++e) {
    const int64_t i = ei[e], j = ej[e];
    const double c = g[e];
    if (i == j || !std::isfinite(c) || c <= 0.0) {
      *bad_edge = e;
      return i == j ? 1 : (!std::isfinite(c) ? 2 : 3);
    }
    const bool fi = fixed[i] != 0, fj = fixed[j] != 0;
    if (!fi && !fj) {
      coo.push_back({i, i, c});
      coo.push_back({j, j, c});
      coo.push_back({i, j, -c});
      coo.push_back({j, i, -c});
    } else if (fi && !fj) {
      coo.push_back({j, j, c});
      rhs[j] += c * fixed_value[i];
    } else if (!fi && fj) {
      coo.push_back({i, i, c});
      rhs[i] += c * fixed_value[j];
    }
  }
  if (neumann)
    for (int64_t k = 0; k < n; ++k) rhs[k] += neumann[k];
  for (int64_t k = 0; k < n; ++k)
    if (fixed[k]) {
      coo.push_back({k, k, 1.0});
      rhs[k] = fixed_value[k];
    }
  std::stable_sort(coo.begin(), coo.end(),
                   [](const Entry& a, const Entry& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
  or_csr* a = new or_csr;
  a->nrows = a->ncols = n;
  a->rp.assign(n + 1, 0);
  for (size_t q = 0; q < coo.size();) {
    size_t t = q + 1;
    double v = coo[q].v;
    while (t < coo.size() && coo[t].r == coo[q].r && coo[t].c == coo[q].c) v += coo[t++].v;
    a->ci.push_back(coo[q].c);
    a->v.push_back(v);
    a->rp[coo[q].r + 1]++;
    q = t;
  }
  for (int64_t r = 0; r < n; ++r) a->rp[r + 1] += a->rp[r];
  *out = a;
  return 0;
}

// ---- the 1-D network solve (LinearSystemSolver, crates/cfd-1d/src/solver/core/linear_system.rs) ----

// NetworkSolver::detect_solver_method (solver_detection.rs:36-64): CG when
// every off-diagonal is <= 0 and every row has diag >= sum |off| and diag > 0
// (identity Dirichlet rows exempt), the sum taken in column order; else
// BiCGSTAB.
int or_detect_solver_method(const or_csr* a) {
  for (int64_t i = 0; i < a->nrows; ++i) {
    double diag = 0.0, sum_off = 0.0;
    for (int64_t k = a->rp[i]; k < a->rp[i + 1]; ++k) {
      const double v = a->v[k];
      if (a->ci[k] == i) {
        diag = v;
      } else if (v > 0.0) {
        return OR_LS_BICGSTAB;
      } else {
        sum_off += std::fabs(v);
      }
    }
    const bool identity_dirichlet = diag == 1.0 && sum_off == 0.0;
    if ((diag < sum_off || diag <= 0.0) && !identity_dirichlet) return OR_LS_BICGSTAB;
  }
  return OR_LS_CG;
}

// Dense LU with partial pivoting (right-looking Doolittle; the pivot is the
// first row of largest |a_ik| at or below the diagonal), forward elimination
// carried on b, then back substitution; the restated lu_decompose + solve of
// linear_system.rs:248-256 (leto_ops, not vendored).
int or_dense_lu_solve(int64_t n, double* m, double* b) {
  for (int64_t k = 0; k < n; ++k) {
    int64_t p = k;
    double best = std::fabs(m[k * n + k]);
    for (int64_t i = k + 1; i < n; ++i) {
      const double v = std::fabs(m[i * n + k]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (!(best > 0.0) || !std::isfinite(best)) return -1;
    if (p != k) {
      for (int64_t j = 0; j < n; ++j) std::swap(m[k * n + j], m[p * n + j]);
      std::swap(b[k], b[p]);
    }
    const double piv = m[k * n + k];
    for (int64_t i = k + 1; i < n; ++i) {
      const double l = m[i * n + k] / piv;
      m[i * n + k] = l;
      if (l == 0.0) continue;
      for (int64_t j = k + 1; j < n; ++j) m[i * n + j] -= l * m[k * n + j];
      b[i] -= l * b[k];
    }
  }
  for (int64_t i = n - 1; i >= 0; --i) {
    double t = b[i];
    for (int64_t j = i + 1; j < n; ++j) t -= m[i * n + j] * b[j];
    b[i] = t / m[i * n + i];
  }
  return 0;
}

namespace {

// 1 / max_j |a_ij| of row i, 1 where the maximum is not above f64::EPSILON or
// not finite (row_equilibrated_system, linear_system.rs:157-186).
double ls_row_scale(const or_csr& a, int64_t i) {
  double mx = 0.0;
  for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) mx = std::max(mx, std::fabs(a.v[k]));
  return (mx > DBL_EPSILON && std::isfinite(mx)) ? 1.0 / mx : 1.0;
}

// ||D (A x - b)|| / ||D b|| (or ||D (A x - b)|| when ||D b|| <= f64::EPSILON):
// compute_equilibrated_residual_norm / _rhs_norm (linear_system.rs:206-246).
double ls_target_ratio(const or_csr& a, const double* x, const double* b, bool* meets, double tol) {
  double r2 = 0.0, b2 = 0.0;
  for (int64_t i = 0; i < a.nrows; ++i) {
    double ax = 0.0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) ax += a.v[k] * x[a.ci[k]];
    const double s = ls_row_scale(a, i);
    const double r = (ax - b[i]) * s;
    r2 += r * r;
    const double bb = b[i] * s;
    b2 += bb * bb;
  }
  const double rn = std::sqrt(r2), bn = std::sqrt(b2);
  if (!std::isfinite(rn)) {
    *meets = false;
    return rn;
  }
  const double ratio = bn > DBL_EPSILON ? rn / bn : rn;
  *meets = ratio <= tol;
  return ratio;
}

int ls_dense(const or_csr& a, const double* b, double* x) {
  const int64_t n = a.nrows;
  std::vector<double> m((size_t)(n * n), 0.0), rhs(b, b + n);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) m[i * n + a.ci[k]] += a.v[k];
  if (or_dense_lu_solve(n, m.data(), rhs.data()) != 0) return -1;
  std::copy(rhs.begin(), rhs.end(), x);
  return 0;
}

double ls_dot(int64_t n, const double* u, const double* v) {
  double t = 0.0;
  for (int64_t i = 0; i < n; ++i) t += u[i] * v[i];
  return t;
}

void ls_spmv(const or_csr& a, const double* x, double* y) {
  for (int64_t i = 0; i < a.nrows; ++i) {
    double t = 0.0;
    for (int64_t k = a.rp[i]; k < a.rp[i + 1]; ++k) t += a.v[k] * x[a.ci[k]];
    y[i] = t;
  }
}

// Jacobi-PCG, the recurrence of or_pcg (serial: one network per thread, as
// the caller's parallel candidate loop runs them).
int ls_pcg(const or_csr& a, const std::vector<double>& inv, const double* b, double* x, double tol, int64_t max_it,
           int64_t* iters) {
  const int64_t n = a.nrows;
  std::vector<double> r(n), z(n), p(n), q(n);
  ls_spmv(a, x, q.data());
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
  double rn = std::sqrt(ls_dot(n, r.data(), r.data()));
  *iters = 0;
  if (rn <= tol) return OR_TERM_INITIAL_RESIDUAL;
  for (int64_t i = 0; i < n; ++i) z[i] = r[i] * inv[i];
  double rho = ls_dot(n, r.data(), z.data());
  p = z;
  for (int64_t it = 1; it <= max_it; ++it) {
    ls_spmv(a, p.data(), q.data());
    const double pq = ls_dot(n, p.data(), q.data());
    if (!(pq > 0.0)) return OR_TERM_NON_POSITIVE_CURVATURE;
    const double alpha = rho / pq;
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    *iters = it;
    rn = std::sqrt(ls_dot(n, r.data(), r.data()));
    if (!std::isfinite(rn)) return OR_TERM_BREAKDOWN;
    if (rn <= tol) return OR_TERM_CONVERGED;
    for (int64_t i = 0; i < n; ++i) z[i] = r[i] * inv[i];
    const double rz = ls_dot(n, r.data(), z.data());
    if (rz == 0.0 || !std::isfinite(rz)) return OR_TERM_BREAKDOWN;
    const double beta = rz / rho;
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rho = rz;
  }
  return OR_TERM_MAX_ITERATIONS;
}

// Jacobi-preconditioned BiCGSTAB, the recurrence of or_bicgstab (serial).
int ls_bicgstab(const or_csr& a, const std::vector<double>& inv, const double* b, double* x, double tol,
                int64_t max_it, int64_t* iters) {
  const int64_t n = a.nrows;
  std::vector<double> r(n), rh(n), p(n, 0.0), v(n, 0.0), ph(n), s(n), sh(n), t(n);
  ls_spmv(a, x, t.data());
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - t[i];
  rh = r;
  double rn = std::sqrt(ls_dot(n, r.data(), r.data()));
  *iters = 0;
  if (rn <= tol) return OR_TERM_INITIAL_RESIDUAL;
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  for (int64_t it = 1; it <= max_it; ++it) {
    const double rho_new = ls_dot(n, rh.data(), r.data());
    if (rho_new == 0.0 || !std::isfinite(rho_new)) return OR_TERM_BREAKDOWN;
    if (it == 1) {
      p = r;
    } else {
      const double beta = (rho_new / rho) * (alpha / omega);
      for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    }
    for (int64_t i = 0; i < n; ++i) ph[i] = p[i] * inv[i];
    ls_spmv(a, ph.data(), v.data());
    const double rv = ls_dot(n, rh.data(), v.data());
    if (rv == 0.0 || !std::isfinite(rv)) return OR_TERM_BREAKDOWN;
    alpha = rho_new / rv;
    // x takes alpha * p^ at once (the half step), then omega * s^ below: the
    // two updates of Saad's x += alpha p^ + omega s^ applied one after the
    // other, so that p^ and s^ can share storage on the device.
    for (int64_t i = 0; i < n; ++i) {
      s[i] = r[i] - alpha * v[i];
      x[i] += alpha * ph[i];
    }
    const double sn = std::sqrt(ls_dot(n, s.data(), s.data()));
    *iters = it;
    if (sn <= tol) return OR_TERM_CONVERGED;
    for (int64_t i = 0; i < n; ++i) sh[i] = s[i] * inv[i];
    ls_spmv(a, sh.data(), t.data());
    const double tt = ls_dot(n, t.data(), t.data());
    if (tt == 0.0 || !std::isfinite(tt)) return OR_TERM_BREAKDOWN;
    omega = ls_dot(n, t.data(), s.data()) / tt;
    for (int64_t i = 0; i < n; ++i) {
      x[i] += omega * sh[i];
      r[i] = s[i] - omega * t[i];
    }
    rn = std::sqrt(ls_dot(n, r.data(), r.data()));
    if (!std::isfinite(rn)) return OR_TERM_BREAKDOWN;
    if (rn <= tol) return OR_TERM_CONVERGED;
    if (omega == 0.0) return OR_TERM_BREAKDOWN;
    rho = rho_new;
  }
  return OR_TERM_MAX_ITERATIONS;
}

}  // namespace

int or_linear_system_solve(const or_csr* a, const double* b, double* x, int method, double tolerance,
                           int64_t max_iterations, or_ls_report* rep) {
  const int64_t n = a->nrows;
  if (a->ncols != n) return -1;
  *rep = or_ls_report{};
  rep->method = method == OR_LS_DETECT ? or_detect_solver_method(a) : method;
  rep->termination = -1;
  // Row-equilibrated copy (D A, D b).
  or_csr sa = *a;
  std::vector<double> sb(n);
  for (int64_t i = 0; i < n; ++i) {
    const double s = ls_row_scale(*a, i);
    for (int64_t k = sa.rp[i]; k < sa.rp[i + 1]; ++k) sa.v[k] *= s;
    sb[i] = b[i] * s;
  }
  bool meets = false;
  if (n <= 256) {
    std::vector<double> xd(n);
    if (ls_dense(sa, sb.data(), xd.data()) == 0) {
      rep->residual = ls_target_ratio(*a, xd.data(), b, &meets, tolerance);
      if (meets) {
        std::copy(xd.begin(), xd.end(), x);
        rep->path = OR_LS_PATH_DIRECT;
        return 0;
      }
    }
    rep->path = OR_LS_PATH_DIRECT_UNSCALED;
  } else {
    std::vector<double> inv(n, 1.0);
    for (int64_t i = 0; i < n; ++i) {
      const double d = csr_value(sa, i, i);
      if (!std::isfinite(d)) {
        rep->path = OR_LS_PATH_ERROR;
        return 0;
      }
      inv[i] = std::fabs(d) <= DBL_EPSILON ? 1.0 : 1.0 / d;
    }
    int64_t it = 0;
    rep->termination = rep->method == OR_LS_CG ? ls_pcg(sa, inv, sb.data(), x, tolerance, max_iterations, &it)
                                               : ls_bicgstab(sa, inv, sb.data(), x, tolerance, max_iterations, &it);
    rep->iterations = it;
    const bool converged = rep->termination == OR_TERM_CONVERGED || rep->termination == OR_TERM_INITIAL_RESIDUAL;
    if (converged) {
      rep->residual = ls_target_ratio(*a, x, b, &meets, tolerance);
      if (meets) {
        rep->path = OR_LS_PATH_KRYLOV;
        return 0;
      }
    }
    rep->path = OR_LS_PATH_KRYLOV_FALLBACK;
  }
  std::vector<double> xd(n);
  if (ls_dense(*a, b, xd.data()) != 0) {
    rep->path = OR_LS_PATH_FAILED;
    return 0;
  }
  std::copy(xd.begin(), xd.end(), x);
  rep->residual = ls_target_ratio(*a, x, b, &meets, tolerance);
  return 0;
}

}  // extern "C"
