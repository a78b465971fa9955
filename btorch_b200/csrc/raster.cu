// Spike rasters as sparse coordinates (the output side of the step).
//
// The reference serialises recorded spikes by converting the dense fp32
// (T, B, N) stack to COO index arrays, row-major (np.nonzero), one int32 index
// array per dimension (btorch/io/serialization.py:80-141).  Here the engine's
// bitmask raster ([rows = T * B][ceil(N/32)] words) is compacted on the device:
// one pass counts the spikes per row, the caller scans the counts, a second
// pass writes the coordinates of every set bit in the same row-major order.
#include "common.cuh"

namespace {

using bt::ceil_div;
using bt::lane_id;

// Warp per row: number of set bits among the row's first n bits.
__global__ void k_raster_count(int64_t rows, int64_t n, const uint32_t* __restrict__ bits, int64_t* __restrict__ counts) {
  const int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (r >= rows) return;  // whole warps
  const int64_t words = (n + 31) >> 5;
  const uint32_t tail = (n & 31) ? (1u << (n & 31)) - 1u : 0xffffffffu;
  int64_t c = 0;
  for (int64_t w = lane_id(); w < words; w += 32) {
    uint32_t m = bits[r * words + w];
    if (w == words - 1) m &= tail;
    c += __popc(m);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane_id() == 0) counts[r] = c;
}

// Warp per row: coordinates of the row's set bits in ascending neuron order,
// starting at offsets[r] (exclusive scan of the counts).
__global__ void k_raster_coords(int64_t rows, int64_t batch, int64_t n, const uint32_t* __restrict__ bits,
                                const int64_t* __restrict__ offsets, int32_t* __restrict__ idx_time,
                                int32_t* __restrict__ idx_batch, int32_t* __restrict__ idx_neuron) {
  const int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (r >= rows) return;
  const unsigned lane = lane_id();
  const int64_t words = (n + 31) >> 5;
  const uint32_t tail = (n & 31) ? (1u << (n & 31)) - 1u : 0xffffffffu;
  const int32_t t = int32_t(r / batch), b = int32_t(r % batch);
  int64_t base = offsets[r];
  for (int64_t w0 = 0; w0 < words; w0 += 32) {
    const int64_t w = w0 + lane;
    uint32_t m = w < words ? bits[r * words + w] : 0u;
    if (w == words - 1) m &= tail;
    // exclusive prefix of the lanes' bit counts
    const int c = __popc(m);
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (int(lane) >= o) incl += y;
    }
    int64_t pos = base + incl - c;
    while (m) {
      const int l = __ffs(m) - 1;
      m &= m - 1;
      idx_time[pos] = t;
      idx_batch[pos] = b;
      idx_neuron[pos] = int32_t(w * 32 + l);
      ++pos;
    }
    base += __shfl_sync(0xffffffffu, incl, 31);
  }
}

}  // namespace

extern "C" int bt_raster_count(int64_t rows, int64_t n, const uint32_t* bits, int64_t* counts, void* stream) {
  BT_CHECK_ARG(rows >= 0 && n >= 0, "negative size");
  if (rows == 0) return BT_OK;
  BT_CHECK_ARG(bits && counts, "null pointer");
  k_raster_count<<<int(ceil_div(rows * 32, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(rows, n, bits, counts);
  BT_CHECK_LAUNCH("k_raster_count");
  return BT_OK;
}

extern "C" int bt_raster_coords(int64_t rows, int64_t batch, int64_t n, const uint32_t* bits, const int64_t* offsets,
                                int32_t* idx_time, int32_t* idx_batch, int32_t* idx_neuron, void* stream) {
  BT_CHECK_ARG(rows >= 0 && n >= 0, "negative size");
  if (rows == 0) return BT_OK;  // an empty raster (T = 0 or batch = 0) has no coordinates
  BT_CHECK_ARG(batch > 0 && rows % batch == 0, "rows must be a multiple of batch");
  BT_CHECK_ARG(n < (int64_t(1) << 31) && rows / batch < (int64_t(1) << 31), "coordinates exceed int32");
  BT_CHECK_ARG(bits && offsets && idx_time && idx_batch && idx_neuron, "null pointer");
  k_raster_coords<<<int(ceil_div(rows * 32, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, batch, n, bits, offsets, idx_time, idx_batch, idx_neuron);
  BT_CHECK_LAUNCH("k_raster_coords");
  return BT_OK;
}
