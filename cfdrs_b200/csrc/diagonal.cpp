// Diagonal SpMV layout (DevMat::dia, k_spmv_dia): eligibility and the host
// evaluation that mirrors the kernel.
//
// Stencil operators (the 7-point finite-volume operator of a structured grid,
// the 5-point operator in 2-D) put every entry on a handful of diagonals
// column - row. Stored diagonal-major, their values stream with coalesced
// loads and no index array at all: 4 (FP32) or 8 (FP64) bytes per slot instead
// of value + one-byte code + row record, and the x entries of a warp's rows
// are consecutive for every diagonal. Slots without an entry hold 0.
//
// Summation order: each row adds its diagonals in ascending offset, which is
// ascending column and so the stored CSR order, one product at a time as the
// one-thread-per-row CSR pipelines do. A slot without an entry adds 0 * x = +-0,
// which leaves a finite partial sum unchanged (a sum that starts at +0 never
// becomes -0 by adding +-0 products), so y = A x is bit-identical to the other
// pipelines for finite x.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace cfd {

bool encode_diagonal(const HostCsr& h, int tpr, HostDiagonal& D) {
  D = HostDiagonal{};
  const int64_t n = h.nrows;
  if (n <= 0 || h.ncols != n || tpr != 1 || n >= INT32_MAX || h.nnz() == 0) return false;
  int cnt = 0;
  int64_t off[kDiaMax];
  for (int64_t r = 0; r < n; ++r) {
    for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) {
      const int64_t o = (int64_t)h.ci[k] - r;
      int q = 0;
      while (q < cnt && off[q] != o) ++q;
      if (q == cnt) {
        if (cnt == kDiaMax) return false;
        off[cnt++] = o;
      }
    }
  }
  if ((double)cnt * (double)n > kDiaMaxFill * (double)h.nnz()) return false;
  std::sort(off, off + cnt);
  D.n = cnt;
  for (int q = 0; q < cnt; ++q) {
    D.off[q] = (int)off[q];
    if (off[q] == 0) D.main = q;
  }
  D.ld = (n + 31) / 32 * 32;
  return true;
}

bool check_diagonal(const HostCsr& h, const HostDiagonal& D, const double* x, std::string* why) {
  const int64_t n = h.nrows;
  std::vector<double> val((size_t)D.n * D.ld, 0.0);
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
  for (int q = 1; q < D.n; ++q)
    if (D.off[q] <= D.off[q - 1]) {
      if (why) *why = "diagonal offsets not ascending";
      return false;
    }
  for (int64_t r = 0; r < n; ++r) {
    double ycsr = 0.0, ydia = 0.0;
    for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) ycsr = std::fma(h.v[k], x[h.ci[k]], ycsr);
    for (int q = 0; q < D.n; ++q) {
      const int64_t j = r + D.off[q];
      const double xv = (j >= 0 && j < n) ? x[j] : 0.0;
      ydia = std::fma(val[(size_t)q * D.ld + r], xv, ydia);
    }
    if (std::memcmp(&ycsr, &ydia, sizeof(double)) != 0) {
      if (why) *why = "row " + std::to_string(r) + " differs from the CSR row sum";
      return false;
    }
  }
  return true;
}

}  // namespace cfd
