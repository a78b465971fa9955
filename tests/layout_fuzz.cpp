// Randomised check of the host layout builders (bt_layout_build, bt_layout_slices),
// compiled with AddressSanitizer and UndefinedBehaviorSanitizer by
// tests/test_layout_fuzz_cpu.py: every valid canonical COO must give the CSC,
// CSR and sliced views built directly here, every out-of-range or
// out-of-order one must be refused with BT_ERR_LAYOUT, and no access may
// leave its array.
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <random>
#include <vector>
#include <algorithm>
#include <tuple>
#include "btorch_b200.h"
extern "C" int bt_layout_build(int64_t, const int64_t*, const int64_t*, int64_t, int64_t, int32_t, int32_t*, uint32_t*, int32_t*, uint32_t*, int32_t*);
extern "C" int bt_layout_slices(int64_t, const int32_t*, const uint32_t*, uint32_t, int64_t*, uint32_t*, int32_t*, int64_t, int64_t*);
int main() {
  std::mt19937_64 rng(1234);
  int bad = 0, rejected = 0, accepted = 0;
  for (int it = 0; it < 20000; ++it) {
    int64_t n_post = rng() % 70, n_pre = rng() % 70; int32_t nb = 1 + rng() % 5;
    int64_t nsrc = n_pre * nb;
    std::vector<std::pair<int64_t,int64_t>> e;
    int64_t m = (n_post && nsrc) ? rng() % (1 + std::min<int64_t>(400, n_post * nsrc)) : 0;
    for (int64_t k = 0; k < m; ++k) e.push_back({int64_t(rng() % n_post), int64_t(rng() % nsrc)});
    std::sort(e.begin(), e.end()); e.erase(std::unique(e.begin(), e.end()), e.end());
    int mode = rng() % 6;  // 0-3 valid; 4 out of range; 5 order broken
    if (mode == 4 && !e.empty()) { auto& x = e[rng() % e.size()]; if (rng() & 1) x.first = n_post + int64_t(rng() % 3); else x.second = -1 - int64_t(rng() % 3); }
    if (mode == 5 && e.size() > 1) { std::swap(e[0], e[e.size() - 1]); }
    int64_t nnz = e.size();
    std::vector<int64_t> post(nnz), src(nnz);
    for (int64_t k = 0; k < nnz; ++k) { post[k] = e[k].first; src[k] = e[k].second; }
    std::vector<int32_t> csc_ptr(n_post + 1), csr_ptr(n_pre + 1), perm(std::max<int64_t>(nnz, 1));
    std::vector<uint32_t> csc_src(std::max<int64_t>(nnz, 1)), csr_dst(std::max<int64_t>(nnz, 1));
    int st = bt_layout_build(nnz, post.data(), src.data(), n_post, n_pre, nb, csc_ptr.data(), csc_src.data(), csr_ptr.data(), csr_dst.data(), perm.data());
    bool valid = true;
    for (int64_t k = 0; k < nnz; ++k) {
      if (post[k] < 0 || post[k] >= n_post || src[k] < 0 || src[k] >= nsrc) valid = false;
      if (k && std::make_pair(post[k], src[k]) <= std::make_pair(post[k-1], src[k-1])) valid = false;
    }
    if (!valid) { if (st != BT_ERR_LAYOUT) { printf("it %d: invalid input accepted (st %d)\n", it, st); ++bad; } else ++rejected; continue; }
    if (st != BT_OK) { printf("it %d: valid input rejected (st %d)\n", it, st); ++bad; continue; }
    ++accepted;
    // CSC check
    for (int64_t p = 0, k = 0; p < n_post; ++p) {
      if (csc_ptr[p] != k) { ++bad; printf("csc_ptr\n"); break; }
      while (k < nnz && post[k] == p) { uint32_t want = uint32_t(src[k] / nb) | (uint32_t(src[k] % nb) << 25); if (csc_src[k] != want) { ++bad; printf("csc_src\n"); } ++k; }
    }
    // CSR check: rows by pre, canonical order within, perm maps back
    std::vector<int64_t> seen;
    for (int64_t j = 0; j < n_pre; ++j) {
      int64_t last = -1;
      for (int32_t q = csr_ptr[j]; q < csr_ptr[j + 1]; ++q) {
        int64_t c = perm[q];
        if (c <= last || src[c] / nb != j) { ++bad; printf("csr order\n"); }
        last = c; seen.push_back(c);
        if (csr_dst[q] != (uint32_t(post[c]) | (uint32_t(src[c] % nb) << 25))) { ++bad; printf("csr_dst\n"); }
      }
    }
    if ((int64_t)seen.size() != nnz) { ++bad; printf("csr count\n"); }
    // slices
    int64_t rows = 0;
    std::vector<int64_t> sl_ptr((n_post + 31) / 32 + 1);
    if (bt_layout_slices(n_post, csc_ptr.data(), csc_src.data(), 999999u, sl_ptr.data(), nullptr, nullptr, 0, &rows) != BT_OK) { ++bad; printf("slice query\n"); continue; }
    std::vector<uint32_t> sl_src(std::max<int64_t>(rows * 32, 1)); std::vector<int32_t> sl_perm(std::max<int64_t>(rows * 32, 1));
    if (bt_layout_slices(n_post, csc_ptr.data(), csc_src.data(), 999999u, sl_ptr.data(), sl_src.data(), sl_perm.data(), rows, &rows) != BT_OK) { ++bad; printf("slices\n"); continue; }
    if (rows > 0 && bt_layout_slices(n_post, csc_ptr.data(), csc_src.data(), 999999u, sl_ptr.data(), sl_src.data(), sl_perm.data(), rows - 1, &rows) != BT_ERR_INVALID) { ++bad; printf("capacity\n"); }
    for (int64_t s = 0; s * 32 < n_post; ++s)
      for (int lane = 0; lane < 32; ++lane) {
        int64_t p = s * 32 + lane; if (p >= n_post) continue;
        for (int64_t r = sl_ptr[s]; r < sl_ptr[s + 1]; ++r) {
          int64_t k = r - sl_ptr[s]; int32_t pr = sl_perm[r * 32 + lane];
          if (csc_ptr[p] + k < csc_ptr[p + 1]) { if (pr != csc_ptr[p] + k || sl_src[r * 32 + lane] != csc_src[pr]) { ++bad; printf("slice entry\n"); } }
          else if (pr != -1 || sl_src[r * 32 + lane] != 999999u) { ++bad; printf("slice pad\n"); }
        }
      }
  }
  // argument checks
  int32_t cp[2]; uint32_t cs[1]; int32_t rp[2]; uint32_t rd[1]; int32_t pm[1]; int64_t pp[1] = {0}, ss[1] = {0};
  if (bt_layout_build(-1, pp, ss, 1, 1, 1, cp, cs, rp, rd, pm) != BT_ERR_INVALID) ++bad;
  if (bt_layout_build(1, pp, ss, 1, 1, 0, cp, cs, rp, rd, pm) != BT_ERR_INVALID) ++bad;
  if (bt_layout_build(1, pp, ss, 1, 1, 129, cp, cs, rp, rd, pm) != BT_ERR_INVALID) ++bad;
  if (bt_layout_build(1, pp, ss, int64_t(1) << 25, 1, 1, cp, cs, rp, rd, pm) != BT_ERR_INVALID) ++bad;
  if (bt_layout_build(1, nullptr, ss, 1, 1, 1, cp, cs, rp, rd, pm) != BT_ERR_INVALID) ++bad;
  printf("accepted %d rejected %d bad %d\n", accepted, rejected, bad);
  return bad != 0;
}
