// Event-driven sparse products for SparseConn (forward and backward).
//
// Replaces the reference's three Triton kernels (pack / direct / hash,
// btorch/models/_sparse_triton.py:20-200) and its torch index-op backward
// (_sparse_triton.py:389-415).  Two forward directions are provided:
//   * gather  -- pull over the post-major (CSC) view, ordered fmaf chain per
//                output, bit-identical to the reference's CPU product;
//   * scatter -- push over the pre-major (CSR) view: compacted nonzero inputs,
//                128-bit edge loads, fp32 reductions into L2-resident outputs.
#include "common.cuh"

namespace bt {

// bits[b][w] bit l  <=>  x[b][32 w + l] != 0.   One warp per 32-column word.
__global__ void k_nonzero_bits(int64_t rows, int64_t cols, int64_t words, const float* __restrict__ x,
                               uint32_t* __restrict__ bits) {
  const int64_t gw = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (gw >= rows * words) return;
  const int64_t r = gw / words, w = gw % words;
  const int64_t c = w * 32 + lane_id();
  const bool nz = c < cols && x[r * cols + c] != 0.0f;
  const uint32_t m = __ballot_sync(0xffffffffu, nz);
  if (lane_id() == 0) bits[gw] = m;
}

// One warp per output neuron i; for every sample the warp walks i's in-edges
// (ascending source) 32 at a time, ballots the ones whose input is nonzero and
// folds them in order with fmaf:  acc = fma(w, x, acc).  Zero inputs are
// skipped, which does not change the value: acc is never -0 (it starts at +0
// and an exact cancellation rounds to +0), so acc + (w * 0) == acc.
__global__ void k_spmv_gather(int64_t batch, int64_t n_in, int64_t n_out, int64_t words,
                              const int32_t* __restrict__ csc_ptr, const uint32_t* __restrict__ csc_src,
                              const float* __restrict__ csc_w, const float* __restrict__ x,
                              const uint32_t* __restrict__ bits, float* __restrict__ out) {
  const int64_t i = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (i >= n_out) return;
  const unsigned lane = lane_id();
  const int32_t beg = csc_ptr[i], end = csc_ptr[i + 1];
  for (int64_t b = 0; b < batch; ++b) {
    const uint32_t* brow = bits + b * words;
    const float* xrow = x + b * n_in;
    float acc = 0.0f;
    for (int32_t base = beg; base < end; base += 32) {
      const int32_t e = base + int32_t(lane);
      uint32_t j = 0;
      float w = 0.0f, xv = 0.0f;
      bool act = false;
      if (e < end) {
        j = __ldg(csc_src + e) & kIdMask;
        act = (__ldg(brow + (j >> 5)) >> (j & 31)) & 1u;
        if (act) {
          w = __ldg(csc_w + e);
          xv = __ldg(xrow + j);
        }
      }
      uint32_t m = __ballot_sync(0xffffffffu, act);
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1;
        acc = fmaf(__shfl_sync(0xffffffffu, w, k), __shfl_sync(0xffffffffu, xv, k), acc);
      }
    }
    if (lane == 0) out[b * n_out + i] = acc;
  }
}

// Compact the nonzero entries of x into work[2 + k] = b * n_in + j (order of
// arrival; the scatter's result does not depend on it beyond fp32 rounding).
// work[0] holds the count.  Warp ballot + one atomic per warp.
__global__ void k_compact_nonzero(int64_t total, const float* __restrict__ x, int32_t* __restrict__ work) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool nz = idx < total && x[idx] != 0.0f;
  const uint32_t m = __ballot_sync(0xffffffffu, nz);
  if (m == 0) return;
  const unsigned lane = lane_id();
  int32_t base = 0;
  if (lane == 0) base = atomicAdd(work, __popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (nz) work[2 + base + __popc(m & ((1u << lane) - 1u))] = int32_t(idx);
}

// Stream the out-edges [beg, end) of one source with 128-bit loads (4 edges
// per lane, 512 B per warp instruction on each array) and add val * w into
// out_row[post].  Edge arrays are padded to a multiple of 4 so the aligned
// vector window never leaves the allocation.
__device__ __forceinline__ void scatter_edges(int32_t beg, int32_t end, const uint32_t* __restrict__ dst,
                                              const float* __restrict__ wts, float val, float* out_row) {
  const unsigned lane = lane_id();
  for (int32_t g = (beg & ~3) + int32_t(lane) * 4; g < end; g += 128) {
    const uint4 d4 = __ldg(reinterpret_cast<const uint4*>(dst + g));
    const float4 w4 = __ldg(reinterpret_cast<const float4*>(wts + g));
    const uint32_t dd[4] = {d4.x, d4.y, d4.z, d4.w};
    const float ww[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int32_t e = g + q;
      if (e >= beg && e < end) atomicAdd(out_row + (dd[q] & kIdMask), ww[q] * val);
    }
  }
}

__global__ void k_spmv_scatter(int64_t n_in, int64_t n_out, const int32_t* __restrict__ csr_ptr,
                               const uint32_t* __restrict__ csr_dst, const float* __restrict__ csr_w,
                               const float* __restrict__ x, const int32_t* __restrict__ work,
                               float* __restrict__ out) {
  const int32_t count = *reinterpret_cast<const volatile int32_t*>(work);
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t it = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; it < count; it += warps) {
    const int32_t flat = work[2 + it];
    const int64_t b = flat / n_in, j = flat % n_in;
    scatter_edges(csr_ptr[j], csr_ptr[j + 1], csr_dst, csr_w, x[flat], out + b * n_out);
  }
}

// grad_x[b][j] = sum over out-edges of w * g[b][post]; one warp per source,
// lanes over edges, fixed-shape butterfly reduction (deterministic).
__global__ void k_spmv_grad_input(int64_t batch, int64_t n_in, int64_t n_out,
                                  const int32_t* __restrict__ csr_ptr, const uint32_t* __restrict__ csr_dst,
                                  const float* __restrict__ csr_w, const float* __restrict__ g,
                                  float* __restrict__ gx) {
  const int64_t j = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (j >= n_in) return;
  const unsigned lane = lane_id();
  const int32_t beg = csr_ptr[j], end = csr_ptr[j + 1];
  for (int64_t b = 0; b < batch; ++b) {
    const float* grow = g + b * n_out;
    float acc = 0.0f;
    for (int32_t e = beg + int32_t(lane); e < end; e += 32)
      acc = fmaf(__ldg(csr_w + e), __ldg(grow + (__ldg(csr_dst + e) & kIdMask)), acc);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) gx[b * n_in + j] = acc;
  }
}

// out[c][r] = in[r][c] for an rows x cols fp32 matrix, through 32 x 32
// shared-memory tiles (block 32 x 8: coalesced reads and writes).
__global__ void k_transpose(int64_t rows, int64_t cols, const float* __restrict__ in, float* __restrict__ out) {
  __shared__ float tile[32][33];
  const int64_t c0 = int64_t(blockIdx.x) * 32, r0 = int64_t(blockIdx.y) * 32;
#pragma unroll
  for (int k = 0; k < 32; k += 8) {
    const int64_t r = r0 + threadIdx.y + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[threadIdx.y + k][threadIdx.x] = in[r * cols + c];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 32; k += 8) {
    const int64_t c = c0 + threadIdx.y + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][threadIdx.y + k];
  }
}

// grad_x[b][j] = sum over j's out-edges e in CSR order of w_e * g[b][dst_e],
// read from gT = g transposed ([n_out][batch]): one warp per source j, lane =
// V consecutive samples, so every edge reads one contiguous run of gT (a
// 512-byte row for 128 samples) instead of one scattered word per sample.
// The warp loads 32 edges at a time and broadcasts them in order; each
// (b, j) is an fmaf chain in ascending edge order (deterministic).
template <int V>
__global__ void k_spmv_grad_input_t(int64_t batch, int64_t n_in, const int32_t* __restrict__ csr_ptr,
                                    const uint32_t* __restrict__ csr_dst, const float* __restrict__ csr_w,
                                    const float* __restrict__ gT, float* __restrict__ gx) {
  const int64_t j = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (j >= n_in) return;
  const unsigned lane = lane_id();
  const int32_t beg = csr_ptr[j], end = csr_ptr[j + 1];
  for (int64_t b0 = 0; b0 < batch; b0 += 32 * V) {
    const int64_t bl = b0 + int64_t(lane) * V;  // this lane's first sample
    float acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = 0.0f;
    for (int32_t base = beg; base < end; base += 32) {
      const int32_t e = base + int32_t(lane);
      const uint32_t dst = e < end ? (__ldg(csr_dst + e) & kIdMask) : 0u;
      const float w = e < end ? __ldg(csr_w + e) : 0.0f;
      const int cnt = end - base < 32 ? end - base : 32;
#pragma unroll 4
      for (int q = 0; q < cnt; ++q) {
        const uint32_t dq = __shfl_sync(0xffffffffu, dst, q);
        const float wq = __shfl_sync(0xffffffffu, w, q);
        const float* row = gT + int64_t(dq) * batch + bl;
        if constexpr (V == 4) {
          if (bl < batch) {
            const float4 g4 = __ldg(reinterpret_cast<const float4*>(row));
            acc[0] = fmaf(wq, g4.x, acc[0]);
            acc[1] = fmaf(wq, g4.y, acc[1]);
            acc[2] = fmaf(wq, g4.z, acc[2]);
            acc[3] = fmaf(wq, g4.w, acc[3]);
          }
        } else {
#pragma unroll
          for (int v = 0; v < V; ++v)
            if (bl + v < batch) acc[v] = fmaf(wq, __ldg(row + v), acc[v]);
        }
      }
    }
#pragma unroll
    for (int v = 0; v < V; ++v)
      if (bl + v < batch) gx[(bl + v) * n_in + j] = acc[v];
  }
}

// masks[j][q] bit l <=> x[32 q + l][j] != 0.  One thread per source; the 32
// samples of a word are loaded before any is tested.
__global__ void k_source_masks(int64_t batch, int64_t n_in, int64_t mwords, const float* __restrict__ x,
                               uint32_t* __restrict__ masks) {
  const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= n_in) return;
  for (int64_t q = 0; q < mwords; ++q) {
    float xv[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) xv[l] = q * 32 + l < batch ? x[(q * 32 + l) * n_in + j] : 0.0f;
    uint32_t m = 0;
#pragma unroll
    for (int l = 0; l < 32; ++l) m |= (xv[l] != 0.0f ? 1u : 0u) << l;
    masks[j * mwords + q] = m;
  }
}

// grad_w in canonical order: one warp per post neuron i, lanes over i's
// in-edges; each edge folds x[b][j] * g[b][i] over its source's active samples.
__global__ void k_spmv_grad_weight(int64_t batch, int64_t n_in, int64_t n_out, int64_t mwords,
                                   const int32_t* __restrict__ csc_ptr, const uint32_t* __restrict__ csc_src,
                                   const float* __restrict__ x, const float* __restrict__ g,
                                   const uint32_t* __restrict__ masks, float* __restrict__ gw) {
  const int64_t i = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (i >= n_out) return;
  const int32_t beg = csc_ptr[i], end = csc_ptr[i + 1];
  for (int32_t e = beg + int32_t(lane_id()); e < end; e += 32) {
    const uint32_t j = __ldg(csc_src + e) & kIdMask;
    float acc = 0.0f;
    for (int64_t q = 0; q < mwords; ++q) {
      uint32_t m = __ldg(masks + j * mwords + q);
      while (m) {
        const int l = __ffs(m) - 1;
        m &= m - 1;
        const int64_t b = q * 32 + l;
        acc = fmaf(__ldg(x + b * n_in + j), __ldg(g + b * n_out + i), acc);
      }
    }
    gw[e] = acc;
  }
}

}  // namespace bt

using namespace bt;

static inline int grid_for_warps(int64_t warps, int threads = 256) {
  return int(ceil_div(warps * 32, threads));
}

extern "C" int bt_spmv_gather(int64_t batch, int64_t n_in, int64_t n_out, const int32_t* csc_ptr,
                              const uint32_t* csc_src, const float* csc_w, const float* x, float* out,
                              uint32_t* bits, void* stream) {
  BT_CHECK_ARG(batch >= 0 && n_in >= 0 && n_out >= 0, "negative size");
  BT_CHECK_ARG(n_in < BT_MAX_NEURONS && n_out < BT_MAX_NEURONS, "sizes must be below 2^25");
  if (batch == 0 || n_out == 0) return BT_OK;
  BT_CHECK_ARG(csc_ptr && x && out && bits, "null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t words = ceil_div(n_in, 32);
  if (words > 0) {
    k_nonzero_bits<<<grid_for_warps(batch * words), 256, 0, s>>>(batch, n_in, words, x, bits);
    BT_CHECK_LAUNCH("k_nonzero_bits");
  }
  k_spmv_gather<<<grid_for_warps(n_out), 256, 0, s>>>(batch, n_in, n_out, words, csc_ptr, csc_src, csc_w, x,
                                                       bits, out);
  BT_CHECK_LAUNCH("k_spmv_gather");
  return BT_OK;
}

extern "C" int bt_spmv_scatter(int64_t batch, int64_t n_in, int64_t n_out, const int32_t* csr_ptr,
                               const uint32_t* csr_dst, const float* csr_w, const float* x, float* out,
                               int32_t* work, void* stream) {
  BT_CHECK_ARG(batch >= 0 && n_in >= 0 && n_out >= 0, "negative size");
  BT_CHECK_ARG(batch * n_in < (int64_t(1) << 31), "batch * n_in must be below 2^31");
  if (batch == 0 || n_out == 0) return BT_OK;
  BT_CHECK_ARG(csr_ptr && x && out && work, "null pointer");
  BT_CHECK_ARG((reinterpret_cast<uintptr_t>(csr_dst) & 15) == 0 && (reinterpret_cast<uintptr_t>(csr_w) & 15) == 0,
               "edge arrays must be 16-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(out, 0, sizeof(float) * size_t(batch * n_out), s) != cudaSuccess ||
      cudaMemsetAsync(work, 0, sizeof(int32_t) * 2, s) != cudaSuccess)
    return bt_set_error(BT_ERR_CUDA, "memset failed");
  const int64_t total = batch * n_in;
  if (total == 0) return BT_OK;
  k_compact_nonzero<<<int(ceil_div(total, 256)), 256, 0, s>>>(total, x, work);
  BT_CHECK_LAUNCH("k_compact_nonzero");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_spmv_scatter<<<sms * 8, 256, 0, s>>>(n_in, n_out, csr_ptr, csr_dst, csr_w, x, work, out);
  BT_CHECK_LAUNCH("k_spmv_scatter");
  return BT_OK;
}

extern "C" int bt_spmv_grad_input(int64_t batch, int64_t n_in, int64_t n_out, const int32_t* csr_ptr,
                                  const uint32_t* csr_dst, const float* csr_w, const float* grad_out,
                                  float* grad_x, void* stream) {
  BT_CHECK_ARG(batch >= 0 && n_in >= 0 && n_out >= 0, "negative size");
  if (batch == 0 || n_in == 0) return BT_OK;
  BT_CHECK_ARG(csr_ptr && grad_out && grad_x, "null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_spmv_grad_input<<<grid_for_warps(n_in), 256, 0, s>>>(batch, n_in, n_out, csr_ptr, csr_dst, csr_w, grad_out,
                                                          grad_x);
  BT_CHECK_LAUNCH("k_spmv_grad_input");
  return BT_OK;
}

extern "C" int bt_spmv_grad_input_t(int64_t batch, int64_t n_in, int64_t n_out, const int32_t* csr_ptr,
                                    const uint32_t* csr_dst, const float* csr_w, const float* grad_out,
                                    float* grad_x, float* work, void* stream) {
  BT_CHECK_ARG(batch >= 0 && n_in >= 0 && n_out >= 0, "negative size");
  if (batch == 0 || n_in == 0) return BT_OK;
  BT_CHECK_ARG(csr_ptr && grad_out && grad_x && work, "null pointer");
  BT_CHECK_ARG(batch * n_out < (int64_t(1) << 40), "too large");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n_out > 0) {
    const dim3 tgrid(unsigned(ceil_div(n_out, 32)), unsigned(ceil_div(batch, 32)));
    BT_CHECK_ARG(tgrid.y < 65536, "batch too large for the transpose grid");
    k_transpose<<<tgrid, dim3(32, 8), 0, s>>>(batch, n_out, grad_out, work);
    BT_CHECK_LAUNCH("k_transpose");
  }
  // 16-byte sample runs need batch % 4 == 0 and an aligned transpose buffer
  if (batch % 4 == 0 && (reinterpret_cast<uintptr_t>(work) & 15) == 0)
    k_spmv_grad_input_t<4><<<grid_for_warps(n_in), 256, 0, s>>>(batch, n_in, csr_ptr, csr_dst, csr_w, work, grad_x);
  else
    k_spmv_grad_input_t<1><<<grid_for_warps(n_in), 256, 0, s>>>(batch, n_in, csr_ptr, csr_dst, csr_w, work, grad_x);
  BT_CHECK_LAUNCH("k_spmv_grad_input_t");
  return BT_OK;
}

extern "C" int bt_spmv_grad_weight(int64_t batch, int64_t n_in, int64_t n_out, const int32_t* csc_ptr,
                                   const uint32_t* csc_src, const float* x, const float* grad_out, float* grad_w,
                                   uint32_t* masks, void* stream) {
  BT_CHECK_ARG(batch >= 0 && n_in >= 0 && n_out >= 0, "negative size");
  if (n_out == 0) return BT_OK;
  BT_CHECK_ARG(csc_ptr && grad_w && masks, "null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t mwords = ceil_div(batch, 32);
  if (n_in > 0 && mwords > 0) {
    k_source_masks<<<int(ceil_div(n_in, 256)), 256, 0, s>>>(batch, n_in, mwords, x, masks);
    BT_CHECK_LAUNCH("k_source_masks");
  }
  k_spmv_grad_weight<<<grid_for_warps(n_out), 256, 0, s>>>(batch, n_in, n_out, mwords, csc_ptr, csc_src, x,
                                                            grad_out, masks, grad_w);
  BT_CHECK_LAUNCH("k_spmv_grad_weight");
  return BT_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of bt_spmv_gather.
//
// Some callers cannot allocate device memory at the point where they need the
// product: code running on a stream that is being captured into a CUDA graph
// under a fixed memory plan, real-time loops that must never hit the implicit
// device synchronisation of cudaMalloc/cudaFree, and foreign-language hosts
// (JNI, cgo, plain C) that bind this library without any device allocator.
// This entry point needs no caller scratch: its bitmap lives in a file-scope
// device array that every GPU loading the library holds until process exit.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr int kNoAllocMaxDevices = 64;
__device__ __align__(256) uint32_t g_noalloc_gather_bits[BT_NOALLOC_GATHER_MAX_WORDS];

std::mutex g_noalloc_mu;
uint32_t* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_gather_bits on the current device.  The array's
// name in host code is only a host-side stand-in, so the address must come
// from cudaGetSymbolAddress, looked up once per device with that device current.
// The address is cached for the life of the process: it is not looked up
// again after cudaDeviceReset or after the primary context is destroyed and
// recreated, so the library must not be used across such a reset.
int noalloc_scratch(uint32_t** out) {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return bt_set_error(BT_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(err));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return bt_set_error(BT_ERR_UNSUPPORTED, "device %d", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    err = cudaGetSymbolAddress(&p, g_noalloc_gather_bits);
    if (err != cudaSuccess || !p)
      return bt_set_error(BT_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(err));
    g_noalloc_addr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_noalloc_addr[dev];
  return BT_OK;
}

}  // namespace

extern "C" int bt_spmv_gather_noalloc(int64_t batch, int64_t n_in, int64_t n_out, const int32_t* csc_ptr,
                                      const uint32_t* csc_src, const float* csc_w, const float* x, float* out,
                                      void* stream) {
  BT_CHECK_ARG(batch >= 0 && n_in >= 0 && n_out >= 0, "negative size");
  BT_CHECK_ARG(n_in < BT_MAX_NEURONS && n_out < BT_MAX_NEURONS, "sizes must be below 2^25");
  const int64_t words = ceil_div(n_in, 32);
  // compare without forming batch * words first: a huge batch must not wrap
  // the product back under the limit
  BT_CHECK_ARG(words == 0 || batch <= BT_NOALLOC_GATHER_MAX_WORDS / words,
               "batch %lld x ceil(n_in / 32) = %lld words exceeds the built-in scratch of %d words; use "
               "bt_spmv_gather", (long long)batch, (long long)words, BT_NOALLOC_GATHER_MAX_WORDS);
  if (batch == 0 || n_out == 0) return BT_OK;
  BT_CHECK_ARG(csc_ptr && out && (n_in == 0 || x), "null pointer");
  uint32_t* bits = nullptr;
  if (int st = noalloc_scratch(&bits)) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // k_nonzero_bits rewrites every word the gather reads, so the contents left
  // by an earlier call never leak into this one.
  if (words > 0) {
    k_nonzero_bits<<<grid_for_warps(batch * words), 256, 0, s>>>(batch, n_in, words, x, bits);
    BT_CHECK_LAUNCH("k_nonzero_bits");
  }
  k_spmv_gather<<<grid_for_warps(n_out), 256, 0, s>>>(batch, n_in, n_out, words, csc_ptr, csc_src, csc_w, x, bits,
                                                       out);
  BT_CHECK_LAUNCH("k_spmv_gather");
  return BT_OK;
}
