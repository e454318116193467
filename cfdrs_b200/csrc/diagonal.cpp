// Diagonal SpMV layout (DevMat::dia, k_spmv_dia, k_spmv_dia_gen): eligibility
// and the host evaluation that mirrors the kernels.
//
// Stencil operators put every entry on a handful of diagonals column - row:
// 7 for the 3-D finite-volume operator, 5 in 2-D, and 23 for the Galerkin
// operator of the first coarse level of a Ruge-Stueben hierarchy on such a grid
// (its coarse points form a regular sub-lattice in ascending numbering). Stored
// diagonal-major, their values stream with coalesced loads and no index array:
// 4 (FP32) or 8 (FP64) bytes per slot instead of value + one-byte code + row
// record, and the x entries of a warp's rows are consecutive for every
// diagonal. Slots without an entry hold 0.
//
// Summation order. Every pipeline sums a row in the order of its row group of
// tpr threads: thread l adds the stored entries at positions l, l + tpr, ...
// (in column order) one product at a time, then the group combines its partial
// sums by a butterfly. The diagonal kernels keep tpr partial sums per row
// (tpr <= 2) and add each slot to the partial a per-row lane mask names (the
// parity of the stored entry's position), so their row sums are those of the
// other pipelines bit for bit: an empty slot holds 0 and adds 0 * x = +-0,
// which leaves a partial sum that started at +0 unchanged for finite x.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace cfd {

namespace {

// Small open-addressing set of diagonal offsets (at most kDiaMax members).
struct OffsetSet {
  static constexpr int kSlots = 128;
  int64_t key[kSlots];
  bool used[kSlots] = {};
  int count = 0;
  // false when a new offset would exceed kDiaMax
  bool insert(int64_t o) {
    uint64_t h = (uint64_t)o * 0x9E3779B97F4A7C15ull;
    int i = (int)(h >> 57);
    while (used[i]) {
      if (key[i] == o) return true;
      i = (i + 1) & (kSlots - 1);
    }
    if (count == kDiaMax) return false;
    used[i] = true;
    key[i] = o;
    ++count;
    return true;
  }
};

// The butterfly of a row group: partial l after the steps tpr/2, ..., 1 is
// s_l + s_{l^o} at each step; lane 0's value is returned.
double butterfly(std::vector<double> s) {
  for (int o = (int)s.size() / 2; o > 0; o >>= 1)
    for (int l = 0; l < o; ++l) s[l] = s[l] + s[l + o];
  return s[0];
}

}  // namespace

bool encode_diagonal(const HostCsr& h, int tpr, HostDiagonal& D) {
  D = HostDiagonal{};
  const int64_t n = h.nrows;
  if (n <= 0 || h.ncols != n || tpr < 1 || tpr > kDiaMaxTpr || n >= INT32_MAX || h.nnz() == 0) return false;
  OffsetSet set;
  for (int64_t r = 0; r < n; ++r)
    for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k)
      if (!set.insert((int64_t)h.ci[k] - r)) return false;
  const int cnt = set.count;
  if ((double)cnt * (double)n > kDiaMaxFill * (double)h.nnz()) return false;
  int64_t off[kDiaMax];
  int c = 0;
  for (int i = 0; i < OffsetSet::kSlots; ++i)
    if (set.used[i]) off[c++] = set.key[i];
  std::sort(off, off + cnt);
  D.n = cnt;
  for (int q = 0; q < cnt; ++q) {
    D.off[q] = (int)off[q];
    if (off[q] == 0) D.main = q;
  }
  D.ld = (n + 31) / 32 * 32;
  D.tpr = tpr;
  if (tpr == 2) {
    D.mask.assign((size_t)D.ld, 0u);
    for (int64_t r = 0; r < n; ++r) {
      int q = 0;
      for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) {
        const int64_t o = (int64_t)h.ci[k] - r;
        while (D.off[q] != o) ++q;  // columns ascend, so do the offsets
        if ((k - h.rp[r]) & 1) D.mask[r] |= 1u << q;
      }
    }
  }
  return true;
}

bool check_diagonal(const HostCsr& h, const HostDiagonal& D, const double* x, std::string* why) {
  const int64_t n = h.nrows;
  const int t = D.tpr;
  std::vector<double> val((size_t)D.n * D.ld, 0.0);
  for (int q = 1; q < D.n; ++q)
    if (D.off[q] <= D.off[q - 1]) {
      if (why) *why = "diagonal offsets not ascending";
      return false;
    }
  for (int64_t r = 0; r < n; ++r) {
    for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) {
      const int64_t o = (int64_t)h.ci[k] - r;
      int q = 0;
      while (q < D.n && D.off[q] != o) ++q;
      if (q == D.n) {
        if (why) *why = "entry (" + std::to_string(r) + ", " + std::to_string(h.ci[k]) + ") on no stored diagonal";
        return false;
      }
      val[(size_t)q * D.ld + r] = h.v[k];
    }
  }
  for (int64_t r = 0; r < n; ++r) {
    // the CSR pipelines: thread l of the row group adds positions l, l + t, ...
    std::vector<double> sc(t, 0.0), sd(t, 0.0);
    for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) {
      const int l = (int)((k - h.rp[r]) % t);
      sc[l] = std::fma(h.v[k], x[h.ci[k]], sc[l]);
    }
    // the diagonal kernels: every slot in diagonal order, to the partial its
    // lane bit names (empty slots hold 0 and go to partial 0)
    for (int q = 0; q < D.n; ++q) {
      const int64_t j = r + D.off[q];
      const double xv = (j >= 0 && j < n) ? x[j] : 0.0;
      const int l = t == 2 ? (int)((D.mask[r] >> q) & 1u) : 0;
      sd[l] = std::fma(val[(size_t)q * D.ld + r], xv, sd[l]);
    }
    const double ycsr = butterfly(sc), ydia = butterfly(sd);
    if (std::memcmp(&ycsr, &ydia, sizeof(double)) != 0) {
      if (why) *why = "row " + std::to_string(r) + " differs from the CSR row sum";
      return false;
    }
  }
  return true;
}

}  // namespace cfd
