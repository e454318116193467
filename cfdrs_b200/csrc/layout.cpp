// Host side of the SpMV device layout: per-block column dictionaries, x
// windows and index records (see DevMat), and a host walk of the x-staged
// kernel's index arithmetic that checks every staged index and evaluates
// y = A x with it.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <vector>

#include "internal.h"

namespace cfd {

namespace {

// Windows of one dictionary-coded block. The columns of code q form the range
// [lo_q, hi_q]; each range widened to 4-entry boundaries is a window, and
// windows that overlap or lie within kWinGap entries of each other merge.
// Returns false when the block exceeds kXsCap entries or kXsMaxWin windows.
constexpr int64_t kWinGap = 16;

bool block_windows(const HostCsr& h, int r0, int r1, const std::vector<int>& d, const uint8_t* code,
                   uint64_t mult, int* slot, int4& xd, int* e) {
  const int nd = (int)d.size();
  const int64_t ncols = h.ncols, ncols4 = ncols & ~int64_t(3);
  std::vector<int64_t> lo(nd, INT64_MAX), hi(nd, -1);
  for (int64_t k = h.rp[r0]; k < h.rp[r1]; ++k) {
    const int q = code[k];
    lo[q] = std::min<int64_t>(lo[q], h.ci[k]);
    hi[q] = std::max<int64_t>(hi[q], h.ci[k]);
  }
  std::vector<int> order(nd);
  for (int q = 0; q < nd; ++q) order[q] = q;
  std::sort(order.begin(), order.end(), [&](int a, int c) { return lo[a] < lo[c]; });
  std::vector<int64_t> ws, we;
  std::vector<int> wof(nd);
  for (int q : order) {
    const int64_t a = lo[q] & ~int64_t(3), en = (hi[q] + 4) & ~int64_t(3);
    if (!ws.empty() && a <= we.back() + kWinGap) {
      we.back() = std::max(we.back(), en);
    } else {
      ws.push_back(a);
      we.push_back(en);
    }
    wof[q] = (int)ws.size() - 1;
  }
  int64_t total = 0;
  for (size_t w = 0; w < ws.size(); ++w) total += we[w] - ws[w];
  if (total > kXsCap || (int)ws.size() > kXsMaxWin) return false;
  // Windows sit back to back in shared memory; only the last one can reach
  // past the end of x, and it copies up to the last full 4-entry group.
  std::vector<int64_t> soff(ws.size());
  int64_t off = 0, copied = 0;
  int tail = 0;
  for (size_t w = 0; w < ws.size(); ++w) {
    soff[w] = off;
    int64_t len = we[w] - ws[w];
    if (we[w] > ncols) {
      len = ncols4 - ws[w];
      tail = (int)(ncols - ncols4);
    }
    slot[2 * w] = (int)ws[w];
    slot[2 * w + 1] = (int)len;
    copied += len;
    off += we[w] - ws[w];
  }
  const int64_t b0 = (int64_t)(((uint64_t)r0 * mult) >> 20);
  int zq = -1;
  for (int q = 0; q < nd; ++q) {
    e[q] = (int)(b0 + d[q] - ws[wof[q]] + soff[wof[q]]);
    if (h.nrows == h.ncols && d[q] == 0) zq = q;
  }
  xd = make_int4((int)ws.size() | (tail << 16), zq, 0, (int)copied);
  return true;
}

void drop_xs(HostLayout& L) {
  L.xs = false;
  L.xwin.clear();
  L.xdesc.clear();
  L.xe.clear();
}

}  // namespace

// Per-block offset dictionaries: a block whose offsets col - base(row) take at
// most 256 distinct values gets one-byte codes; blocks with more, and the
// single-row blocks beyond the staging capacity, keep int32 columns. When
// every non-empty block is coded, the x windows and index records are built
// as well (x staging), unless a block's windows exceed the staging limits.
void encode_layout(const HostCsr& h, const std::vector<int>& blk, HostLayout& L) {
  const int nb = (int)blk.size() - 1;
  const uint64_t mult = h.nrows ? (((uint64_t)h.ncols << 20) / (uint64_t)h.nrows) : (1u << 20);
  L = HostLayout();
  L.base_mult = mult;
  auto row_base = [mult](int r) { return (int)(((uint64_t)r * mult) >> 20); };
  int raw_blocks = 0;
  std::vector<std::vector<int>> dicts(nb);
  L.dict_desc.assign(nb, make_int2(0, 0));
  L.code.assign(h.nnz() + 16, 0);
  int64_t comp = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : comp, raw_blocks)
  for (int b = 0; b < nb; ++b) {
    const int r0 = blk[b], r1 = blk[b + 1];
    const int64_t k0 = h.rp[r0], k1 = h.rp[r1];
    if (k1 - k0 > kNnzCap || k1 == k0) continue;
    std::vector<int>& d = dicts[b];
    d.reserve(64);
    for (int r = r0; r < r1; ++r) {
      const int base = row_base(r);
      for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) d.push_back(h.ci[k] - base);
    }
    std::sort(d.begin(), d.end());
    d.erase(std::unique(d.begin(), d.end()), d.end());
    if (d.size() > 256) {
      d.clear();
      ++raw_blocks;
      continue;
    }
    for (int r = r0; r < r1; ++r) {
      const int base = row_base(r);
      for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k)
        L.code[k] = (uint8_t)(std::lower_bound(d.begin(), d.end(), h.ci[k] - base) - d.begin());
    }
    comp += k1 - k0;
  }
  for (int b = 0; b < nb; ++b) {
    L.dict_desc[b] = make_int2((int)L.dict.size(), (int)dicts[b].size());
    L.dict.insert(L.dict.end(), dicts[b].begin(), dicts[b].end());
  }
  L.compressed_nnz = comp;
  L.all_compressed = comp > 0 && raw_blocks == 0;
  if (!L.all_compressed) return;

  // x windows: every non-empty block must fit the staging limits
  L.xwin.assign((size_t)nb * (kXsMaxWin / 2), make_int4(0, 0, 0, 0));
  L.xdesc.assign(nb, make_int4(0, -1, 0, 0));
  L.xe.assign(L.dict.size(), 0);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : bad)
  for (int b = 0; b < nb; ++b) {
    if (dicts[b].empty()) continue;  // empty block: no columns, nothing staged
    int* slot = reinterpret_cast<int*>(&L.xwin[(size_t)b * (kXsMaxWin / 2)]);
    if (!block_windows(h, blk[b], blk[b + 1], dicts[b], L.code.data(), mult, slot, L.xdesc[b],
                       L.xe.data() + L.dict_desc[b].x))
      ++bad;
  }
  bool xs = bad == 0;
  if (!xs) drop_xs(L);
  // block records, back to back
  std::vector<int64_t> off(nb + 1, 0);
  for (int b = 0; b < nb; ++b) {
    const int rows = blk[b + 1] - blk[b];
    const int nnz = (int)(h.rp[blk[b + 1]] - h.rp[blk[b]]);
    if (rows > kRowsPerBlock) {  // partitions never make such blocks; stay on the int32 path
      drop_xs(L);
      L.all_compressed = false;
      return;
    }
    off[b + 1] = off[b] + BlockRecord::of(rows, nnz, L.dict_desc[b].y, xs).bytes();
  }
  if (off[nb] / 16 >= INT32_MAX) {
    drop_xs(L);
    L.all_compressed = false;
    return;
  }
  L.roff.resize(nb);
  for (int b = 0; b < nb; ++b) {
    L.roff[b] = (int)(off[b] / 16);
    if (xs) L.xdesc[b].z = L.roff[b];
  }
  L.rec.assign(off[nb] + 16, 0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int b = 0; b < nb; ++b) {
    const int r0 = blk[b], r1 = blk[b + 1];
    const int64_t k0 = h.rp[r0], k1 = h.rp[r1];
    const int2 dd = L.dict_desc[b];
    const BlockRecord R = BlockRecord::of(r1 - r0, (int)(k1 - k0), dd.y, xs);
    uint8_t* rec = L.rec.data() + off[b];
    uint16_t* rp16 = reinterpret_cast<uint16_t*>(rec);
    for (int r = r0; r <= r1; ++r) rp16[r - r0] = (uint16_t)(h.rp[r] - k0);
    std::copy(L.code.begin() + k0, L.code.begin() + k1, rec + R.rp_bytes);
    std::copy(L.dict.begin() + dd.x, L.dict.begin() + dd.x + dd.y,
              reinterpret_cast<int*>(rec + R.rp_bytes + R.code_bytes));
    if (xs)
      std::copy(L.xe.begin() + dd.x, L.xe.begin() + dd.x + dd.y,
                reinterpret_cast<int*>(rec + R.rp_bytes + R.code_bytes + R.dict_bytes));
  }
  L.xs = xs;
}

// Host walk of one SpMV through the device layout. Codes-only layouts are read
// from the block records as k_spmv_pipe reads them. For x-staged layouts it
// rebuilds each block's shared-memory x image from the windows and the tail
// exactly as k_spmv_xs does, reads row offsets, codes and the displacement
// table from the block's record, checks that every one of them lies inside its
// region and that the staged entry is x[col], and sums rows in the kernel's
// order for one thread per row. Returns false with a message on the
// first violation.
bool check_layout(const HostCsr& h, const std::vector<int>& blk, const HostLayout& L, const double* x, double* y,
                  std::string* why, int64_t* staged_entries, int* max_windows) {
  const int nb = (int)blk.size() - 1;
  const uint64_t mult = L.base_mult;
  auto row_base = [mult](int64_t r) { return (int64_t)(((uint64_t)r * mult) >> 20); };
  auto fail = [&](const char* fmt, int b, int64_t a, int64_t c) {
    char buf[256];
    snprintf(buf, sizeof(buf), fmt, b, (long long)a, (long long)c);
    if (why) *why = buf;
    return false;
  };
  int64_t staged = 0;
  int maxw = 0;
  std::vector<double> sx(kXsCap);
  std::vector<int64_t> src(kXsCap);
  for (int b = 0; b < nb; ++b) {
    const int r0 = blk[b], r1 = blk[b + 1];
    const int64_t k0 = h.rp[r0], k1 = h.rp[r1];
    const int2 dd = L.dict_desc.empty() ? make_int2(0, 0) : L.dict_desc[b];
    const bool coded = dd.y > 0;
    if (L.all_compressed && k1 > k0 && !coded)
      return fail("block %d: all_compressed but nonzeros %lld..%lld uncoded", b, k0, k1);
    if (!L.xs) {
      // codes-only pipeline: row offsets, codes and dictionary from the record
      const uint16_t* rp16 = nullptr;
      const uint8_t* rcode = nullptr;
      const int* rdict = nullptr;
      if (L.all_compressed) {
        const BlockRecord R = BlockRecord::of(r1 - r0, (int)(k1 - k0), dd.y, false);
        if (r1 - r0 > kRowsPerBlock || R.bytes() > kRecordCap)
          return fail("block %d: %lld rows, record of %lld bytes", b, r1 - r0, R.bytes());
        const int64_t ro = (int64_t)L.roff[b] * 16;
        if (ro + R.bytes() > (int64_t)L.rec.size())
          return fail("block %d: record end %lld > %lld", b, ro + R.bytes(), (int64_t)L.rec.size());
        rp16 = reinterpret_cast<const uint16_t*>(L.rec.data() + ro);
        rcode = L.rec.data() + ro + R.rp_bytes;
        rdict = reinterpret_cast<const int*>(L.rec.data() + ro + R.rp_bytes + R.code_bytes);
      }
      for (int r = r0; r < r1; ++r) {
        if (rp16 && (rp16[r - r0] != h.rp[r] - k0 || rp16[r - r0 + 1] != h.rp[r + 1] - k0))
          return fail("block %d: record row offsets %lld..%lld", b, rp16[r - r0], rp16[r - r0 + 1]);
        double s = 0.0;
        for (int64_t k = h.rp[r]; k < h.rp[r + 1]; ++k) {
          int64_t c = h.ci[k];
          if (coded) {
            const int q = rcode ? rcode[k - k0] : L.code[k];
            if (q >= dd.y) return fail("block %d: code %lld >= %lld entries", b, q, dd.y);
            c = row_base(r) + (rdict ? rdict[q] : L.dict[dd.x + q]);
            if (c != h.ci[k]) return fail("block %d: decoded column %lld != %lld", b, c, h.ci[k]);
          }
          s += h.v[k] * x[c];
        }
        y[r] = s;
      }
      continue;
    }
    // x-staged block: producer copy sizes and regions
    const int4 xd = L.xdesc[b];
    const int nwin = xd.x & 0xffff, tail = xd.x >> 16, copied = xd.w;
    if (k1 - k0 > kNnzCap) return fail("block %d: %lld nonzeros > cap %lld", b, k1 - k0, kNnzCap);
    if (nwin > kXsMaxWin) return fail("block %d: %lld windows > %lld", b, nwin, kXsMaxWin);
    if (tail < 0 || tail > 3 || copied + tail > kXsCap) return fail("block %d: tail %lld copied %lld", b, tail, copied);
    if ((k1 == k0) != (dd.y == 0)) return fail("block %d: dictionary size %lld for %lld nonzeros", b, dd.y, k1 - k0);
    const BlockRecord R = BlockRecord::of(r1 - r0, (int)(k1 - k0), dd.y, true);
    if (r1 - r0 > kRowsPerBlock || R.bytes() > kRecordCap)
      return fail("block %d: %lld rows, record of %lld bytes", b, r1 - r0, R.bytes());
    if (xd.z != L.roff[b]) return fail("block %d: record offset %lld != %lld", b, xd.z, L.roff[b]);
    const int64_t ro = (int64_t)xd.z * 16;
    if (ro + R.bytes() > (int64_t)L.rec.size())
      return fail("block %d: record end %lld > %lld", b, ro + R.bytes(), (int64_t)L.rec.size());
    const uint8_t* rec = L.rec.data() + ro;
    const uint16_t* rp16 = reinterpret_cast<const uint16_t*>(rec);
    const uint8_t* rcode = rec + R.rp_bytes;
    const int* rE = reinterpret_cast<const int*>(rec + R.rp_bytes + R.code_bytes + R.dict_bytes);
    std::fill(src.begin(), src.end(), -1);
    const int* slot = reinterpret_cast<const int*>(&L.xwin[(size_t)b * (kXsMaxWin / 2)]);
    int64_t soff = 0;
    for (int w = 0; w < nwin; ++w) {
      const int64_t s0 = slot[2 * w], len = slot[2 * w + 1];
      if (s0 % 4 || len % 4 || len < 0)
        return fail("block %d: window start %lld length %lld not 16-byte aligned", b, s0, len);
      if (s0 + len > h.ncols) return fail("block %d: window end %lld > ncols %lld", b, s0 + len, h.ncols);
      if (soff + len > kXsCap) return fail("block %d: staged end %lld > cap %lld", b, soff + len, kXsCap);
      for (int64_t t = 0; t < len; ++t) {
        sx[soff + t] = x[s0 + t];
        src[soff + t] = s0 + t;
      }
      soff += len;
    }
    if (soff != copied) return fail("block %d: windows copy %lld entries, descriptor %lld", b, soff, copied);
    const int64_t ncols4 = h.ncols & ~int64_t(3);
    for (int t = 0; t < tail; ++t) {
      if (ncols4 + t >= h.ncols) return fail("block %d: tail entry %lld beyond ncols %lld", b, ncols4 + t, h.ncols);
      sx[copied + t] = x[ncols4 + t];
      src[copied + t] = ncols4 + t;
    }
    staged += copied + tail;
    maxw = std::max(maxw, nwin);
    const int64_t b0 = row_base(r0);
    for (int r = r0; r < r1; ++r) {
      const int64_t lb = row_base(r) - b0;
      const int ka = rp16[r - r0], ke = rp16[r - r0 + 1];
      if (ka != h.rp[r] - k0 || ke != h.rp[r + 1] - k0) return fail("block %d: record row offsets %lld..%lld", b, ka, ke);
      double s = 0.0;
      for (int kl = ka; kl < ke; ++kl) {
        const int64_t k = k0 + kl;
        const int q = rcode[kl];
        if (q >= dd.y) return fail("block %d: code %lld >= %lld entries", b, q, dd.y);
        const int64_t idx = lb + rE[q];
        if (idx < 0 || idx >= copied + tail)
          return fail("block %d: staged index %lld outside [0, %lld)", b, idx, copied + tail);
        if (src[idx] != h.ci[k])
          return fail("block %d: staged entry holds column %lld, needs %lld", b, src[idx], h.ci[k]);
        const bool is_diag = q == xd.y;
        if (h.nrows == h.ncols && is_diag != (h.ci[k] == r))
          return fail("block %d: zero-offset code %lld disagrees with column %lld", b, xd.y, h.ci[k]);
        s += h.v[k] * sx[idx];
      }
      y[r] = s;
    }
  }
  if (staged_entries) *staged_entries = staged;
  if (max_windows) *max_windows = maxw;
  return true;
}

}  // namespace cfd
