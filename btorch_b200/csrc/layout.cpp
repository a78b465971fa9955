// Host-side static layout builder and error plumbing for the C ABI.
//
// Replaces the reference's per-source Python loop that builds its task layout
// (btorch/models/_sparse_preprocess.py:28-122): one counting-sort pass builds
// both the post-major (CSC) view used by the ordered gather and the pre-major
// (CSR) view used by the scatter, from the canonical (post, src) COO order the
// module stores (btorch/models/linear.py:278-292).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <vector>

#include "../../include/btorch_b200.h"

namespace {
thread_local char g_error[512] = {0};
}

extern "C" int bt_set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
  return status;
}

extern "C" const char* bt_last_error(void) { return g_error; }

extern "C" int bt_abi_version(void) { return BT_ABI_VERSION; }

extern "C" int bt_layout_build(int64_t nnz, const int64_t* post, const int64_t* src, int64_t n_post,
                               int64_t n_pre, int32_t n_bins, int32_t* csc_ptr, uint32_t* csc_src,
                               int32_t* csr_ptr, uint32_t* csr_dst, int32_t* csr_perm) {
  g_error[0] = 0;
  if (nnz < 0 || nnz >= (int64_t(1) << 31))
    return bt_set_error(BT_ERR_INVALID, "nnz=%lld outside [0, 2^31)", (long long)nnz);
  if (n_post < 0 || n_post >= BT_MAX_NEURONS || n_pre < 0 || n_pre >= BT_MAX_NEURONS)
    return bt_set_error(BT_ERR_INVALID, "n_post=%lld / n_pre=%lld must be below 2^25", (long long)n_post,
                        (long long)n_pre);
  if (n_bins < 1 || n_bins > BT_MAX_BINS)
    return bt_set_error(BT_ERR_INVALID, "n_bins=%d outside [1, %d]", n_bins, BT_MAX_BINS);
  if (nnz > 0 && (!post || !src || !csc_src || !csr_dst || !csr_perm))
    return bt_set_error(BT_ERR_INVALID, "null array");
  if (!csc_ptr || !csr_ptr) return bt_set_error(BT_ERR_INVALID, "null pointer array");

  const int64_t n_src = n_pre * n_bins;
  std::vector<int32_t> pre_count(size_t(n_pre) + 1, 0);
  std::memset(csc_ptr, 0, sizeof(int32_t) * size_t(n_post + 1));
  int64_t prev_post = -1, prev_src = -1;
  for (int64_t e = 0; e < nnz; ++e) {
    const int64_t p = post[e], s = src[e];
    if (p < 0 || p >= n_post || s < 0 || s >= n_src)
      return bt_set_error(BT_ERR_LAYOUT, "edge %lld: (post=%lld, src=%lld) outside (%lld, %lld)", (long long)e,
                          (long long)p, (long long)s, (long long)n_post, (long long)n_src);
    if (p < prev_post || (p == prev_post && s <= prev_src))
      return bt_set_error(BT_ERR_LAYOUT, "edge %lld breaks canonical (post, src) order or repeats an edge",
                          (long long)e);
    prev_post = p;
    prev_src = s;
    csc_ptr[p + 1]++;
    pre_count[size_t(s / n_bins) + 1]++;
    csc_src[e] = uint32_t(s / n_bins) | (uint32_t(s % n_bins) << BT_BIN_SHIFT);
  }
  for (int64_t i = 0; i < n_post; ++i) csc_ptr[i + 1] += csc_ptr[i];
  csr_ptr[0] = 0;
  for (int64_t j = 0; j < n_pre; ++j) csr_ptr[j + 1] = csr_ptr[j] + pre_count[size_t(j) + 1];
  // Stable placement: within one presynaptic neuron the edges keep canonical
  // order, i.e. ascending post then ascending delay bin.
  std::vector<int32_t> cursor(csr_ptr, csr_ptr + n_pre);
  for (int64_t e = 0; e < nnz; ++e) {
    const int64_t s = src[e];
    const int64_t j = s / n_bins;
    const int32_t pos = cursor[size_t(j)]++;
    csr_dst[pos] = uint32_t(post[e]) | (uint32_t(s % n_bins) << BT_BIN_SHIFT);
    csr_perm[pos] = int32_t(e);
  }
  return BT_OK;
}

// Sliced post-major view (SELL-32): posts are grouped in slices of 32; slice s
// holds rows [sl_ptr[s], sl_ptr[s+1]), row r storing entry k of each of its 32
// posts at [32 r + lane] -- so a warp with lane = post reads one row with one
// coalesced 128-byte load, and walks each post's in-edges in canonical order.
// Short posts are padded with `sentinel` (a presynaptic id that never spikes)
// and perm -1 (weight 0).
extern "C" int bt_layout_slices(int64_t n_post, const int32_t* csc_ptr, const uint32_t* csc_src, uint32_t sentinel,
                                int64_t* sl_ptr, uint32_t* sl_src, int32_t* sl_perm, int64_t capacity_rows,
                                int64_t* rows_out) {
  g_error[0] = 0;
  if (n_post < 0 || !csc_ptr || !sl_ptr || !rows_out) return bt_set_error(BT_ERR_INVALID, "null argument");
  const int64_t n_slices = (n_post + 31) / 32;
  int64_t rows = 0;
  sl_ptr[0] = 0;
  for (int64_t s = 0; s < n_slices; ++s) {
    int32_t len = 0;
    for (int64_t p = s * 32; p < std::min<int64_t>(n_post, s * 32 + 32); ++p)
      len = std::max(len, csc_ptr[p + 1] - csc_ptr[p]);
    rows += len;
    sl_ptr[s + 1] = rows;
  }
  *rows_out = rows;
  if (!sl_src || !sl_perm) return BT_OK;  // size query
  if (capacity_rows < rows) return bt_set_error(BT_ERR_INVALID, "slice capacity %lld < %lld rows",
                                                (long long)capacity_rows, (long long)rows);
  for (int64_t s = 0; s < n_slices; ++s) {
    for (int64_t r = sl_ptr[s]; r < sl_ptr[s + 1]; ++r) {
      const int64_t k = r - sl_ptr[s];
      for (int lane = 0; lane < 32; ++lane) {
        const int64_t p = s * 32 + lane;
        const int64_t at = r * 32 + lane;
        if (p < n_post && csc_ptr[p] + k < csc_ptr[p + 1]) {
          sl_src[at] = csc_src[csc_ptr[p] + k];
          sl_perm[at] = csc_ptr[p] + int32_t(k);
        } else {
          sl_src[at] = sentinel;
          sl_perm[at] = -1;
        }
      }
    }
  }
  return BT_OK;
}
