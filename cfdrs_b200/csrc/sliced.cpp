// Host side of the sliced SpMV layout (DevMat::sl): rows in slices of 32, each
// slice stored slot-major (slot k of the slice's 32 rows is 32 consecutive
// entries) so that a warp reading one slot per row moves 128 contiguous bytes
// of FP32 values and 32 of codes. A slice is as wide as its longest row; the
// shorter rows are padded with code kSlPadCode and value 0. Columns are
// dictionary codes: col = base(row) + dict[chunk][code], one dictionary of at
// most 255 column offsets per chunk of kSlChunkSlices slices. The layout is
// built only when it pays: one thread per row, rows of at most kSlMaxWidth
// entries, at most kSlMaxPadding slots per stored nonzero.
#include <algorithm>
#include <vector>

#include "internal.h"

namespace cfd {

bool encode_sliced(const HostCsr& h, int tpr, uint64_t base_mult, HostSliced& S) {
  S = HostSliced();
  if (tpr != 1 || h.nrows == 0 || h.nnz() == 0) return false;
  const int64_t n = h.nrows;
  const int64_t ns = (n + kSlRows - 1) / kSlRows;
  const int64_t nch = (ns + kSlChunkSlices - 1) / kSlChunkSlices;
  auto row_base = [base_mult](int64_t r) { return (int64_t)(((uint64_t)r * base_mult) >> 20); };
  S.off.assign(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t w = 0;
    for (int64_t r = s * kSlRows; r < std::min(n, (s + 1) * kSlRows); ++r) w = std::max(w, h.rp[r + 1] - h.rp[r]);
    if (w > kSlMaxWidth) return false;
    S.off[s + 1] = S.off[s] + w * kSlRows;
  }
  const int64_t slots = S.off[ns];
  if ((double)slots > kSlMaxPadding * (double)h.nnz() || slots >= INT32_MAX) return false;
  std::vector<std::vector<int>> dicts(nch);
  bool ok = true;
#pragma omp parallel for schedule(dynamic, 16) reduction(&& : ok)
  for (int64_t c = 0; c < nch; ++c) {
    std::vector<int>& d = dicts[c];
    const int64_t r0 = c * kSlChunkSlices * kSlRows, r1 = std::min(n, (c + 1) * kSlChunkSlices * kSlRows);
    for (int64_t r = r0; r < r1; ++r)
      for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) d.push_back((int)(h.ci[k] - row_base(r)));
    std::sort(d.begin(), d.end());
    d.erase(std::unique(d.begin(), d.end()), d.end());
    if ((int)d.size() > kSlPadCode) ok = false;
  }
  if (!ok) {
    S = HostSliced();
    return false;
  }
  S.doff.assign(nch + 1, 0);
  for (int64_t c = 0; c < nch; ++c) S.doff[c + 1] = S.doff[c] + (int)dicts[c].size();
  S.dict.resize(S.doff[nch] + 16, 0);
  for (int64_t c = 0; c < nch; ++c) std::copy(dicts[c].begin(), dicts[c].end(), S.dict.begin() + S.doff[c]);
  S.code.assign(slots + 16, (uint8_t)kSlPadCode);
  S.src.assign(slots, -1);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t s = 0; s < ns; ++s) {
    const std::vector<int>& d = dicts[s / kSlChunkSlices];
    for (int lane = 0; lane < kSlRows; ++lane) {
      const int64_t r = s * kSlRows + lane;
      if (r >= n) break;
      const int64_t base = row_base(r);
      for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) {
        const int64_t q = S.off[s] + (k - h.rp[r]) * kSlRows + lane;
        const int off = (int)(h.ci[k] - base);
        S.code[q] = (uint8_t)(std::lower_bound(d.begin(), d.end(), off) - d.begin());
        S.src[q] = (int)k;
      }
    }
  }
  S.nslices = ns;
  S.slots = slots;
  return true;
}

// Walks the sliced layout as the kernel does: every real slot's column must
// equal the CSR column of its source entry and lie inside [0, ncols), every
// row's entries must appear once in order, padding must have no source.
bool check_sliced(const HostCsr& h, uint64_t base_mult, const HostSliced& S, std::string* why) {
  const int64_t n = h.nrows;
  auto fail = [&](const char* what, int64_t q) {
    if (why) *why = std::string(what) + " at slot " + std::to_string(q);
    return false;
  };
  if (S.nslices != (n + kSlRows - 1) / kSlRows || (int64_t)S.off.size() != S.nslices + 1) return fail("slice count", 0);
  for (int64_t s = 0; s < S.nslices; ++s) {
    const int64_t e0 = S.off[s], e1 = S.off[s + 1];
    if (e1 < e0 || (e1 - e0) % kSlRows != 0 || (e1 - e0) / kSlRows > kSlMaxWidth || e1 > S.slots)
      return fail("slice extent", e0);
    const int64_t c = s / kSlChunkSlices;
    if (c + 1 >= (int64_t)S.doff.size()) return fail("chunk index", e0);
    const int nd = S.doff[c + 1] - S.doff[c];
    for (int lane = 0; lane < kSlRows; ++lane) {
      const int64_t r = s * kSlRows + lane;
      int64_t next = r < n ? h.rp[r] : 0;
      const int64_t base = (int64_t)(((uint64_t)(r < n ? r : 0) * base_mult) >> 20);
      for (int64_t q = e0 + lane; q < e1; q += kSlRows) {
        const int code = S.code[q];
        if (code == kSlPadCode) {
          if (S.src[q] != -1) return fail("padding with a source", q);
          continue;
        }
        if (r >= n) return fail("entry past the last row", q);
        if (code >= nd) return fail("code outside its dictionary", q);
        const int64_t col = base + S.dict[S.doff[c] + code];
        if (col < 0 || col >= h.ncols) return fail("column out of range", q);
        if (S.src[q] != next || next >= h.rp[r + 1]) return fail("entry out of order", q);
        if (col != h.ci[next]) return fail("column differs from CSR", q);
        ++next;
      }
      if (r < n && next != h.rp[r + 1]) return fail("row entries missing", e0 + lane);
    }
  }
  return true;
}

}  // namespace cfd
