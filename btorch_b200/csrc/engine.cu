// Fused multi-step recurrent engine: RecurrentNN(neuron, synapse, inp) for
// LIF/ALIF neurons with exponential (optionally delayed) synapses on a sparse
// connectivity, btorch/models/rnn.py:517-528 repeated over time
// (rnn.py:200-332).
//
// Reference step t (per sample b, neuron i):
//   I     = psc_{t-1} + x_t                     (rnn.py:524)
//   z_t   = neuron(I)                           (base.py:1108-1116)
//   psc_t = decay(psc_{t-1}) + sum_d W_d z_{t-d} (synapse.py:99-103, delay bins
//                                                 via history.py:299-345 and
//                                                 connection.py:973-1027)
//
// SCATTER mode, two launches per step:
//   k_eng_neuron  (step t): P = stored + ring[(t-1) mod R]; zero that slot;
//                 neuron update with I = P + x_t; stored = decay(P); spike
//                 bitmaps; union of active presynaptic neurons compacted
//                 (warp ballot + block prefix + one atomic per block).
//   k_eng_scatter (step t): for each active neuron j (any sample), stream its
//                 out-edges once with 128-bit loads and add w into
//                 ring[(t + bin) mod R][b][post] for every sample b that
//                 spiked (fp32 reductions, resolved in L2).
//   "stored" holds decay(psc_{t-1}) during a run; the ring holds the pending
//   sums of W z for every arrival step, so the reference's rounding of
//   psc = decay(psc) + Wz is kept (exact sums when weights are dyadic).
//
// GATHER mode, one launch per step (k_eng_gather): each warp owns a neuron,
//   computes P_{t-1} = decay(P_{t-2}) + sum over its in-edges (pre, bin) in
//   ascending canonical order of w * z_{t-1-bin}[pre] (fmaf chain, exactly the
//   reference's CPU rounding), then runs the neuron update of step t.  The
//   last synapse update of a run is k_eng_gather_final.
#include "neuron.cuh"

namespace bt {

constexpr int kEngThreads = 256;

struct EngCounters {
  int32_t list_count[2];  // active-list length, double buffered by step parity
  int32_t pad[2];
};

__host__ __device__ __forceinline__ int mask_words(int64_t batch) { return int((batch + 31) >> 5); }

// ---------------------------------------------------------------- scatter --

template <int KIND, bool HARD, bool USE_REF>
__global__ void __launch_bounds__(kEngThreads) k_eng_neuron(bt_engine_desc d, int64_t k, int sg) {
  extern __shared__ uint32_t sh[];
  const int nt = kEngThreads / sg;
  const int tid = threadIdx.x;
  const int tn = tid % nt, g = tid / nt;
  const int64_t n = d.n, B = d.batch;
  const int64_t i0 = int64_t(blockIdx.x) * nt;
  const int64_t i = i0 + tn;
  const bool valid = i < n;
  const int mw = mask_words(B);
  const int64_t words = (n + 31) >> 5;
  const int64_t t = d.t0 + k;
  const int R = d.n_bins;
  const int64_t slot_in = ((t - 1) % R + R) % R;
  uint32_t* smask = sh;  // [nt][mw]
  for (int q = tid; q < nt * mw; q += kEngThreads) smask[q] = 0;
  __syncthreads();

  for (int64_t b = g; b < B; b += sg) {
    float s = 0.0f;
    if (valid) {
      const int64_t idx = b * n + i;
      float* ring_in = d.ring + (slot_in * B) * n;
      const float pending = ring_in[idx];
      ring_in[idx] = 0.0f;
      const int64_t len = d.sample_len ? d.sample_len[b] : INT64_MAX;
      if (k < len) {
        const float P = add(d.psc[idx], pending);
        const float I = d.x ? add(P, d.x[(k * B) * n + idx]) : P;
        float v = d.v[idx];
        float ref = USE_REF ? d.refractory[idx] : 0.0f;
        float gk = KIND == BT_NEURON_ALIF ? d.g_k[idx] : 0.0f;
        const NeuronOut o = neuron_update<KIND, HARD, USE_REF>(d.neuron, i, I, v, ref, gk);
        s = o.spike;
        d.v[idx] = v;
        if (USE_REF) d.refractory[idx] = ref;
        if (KIND == BT_NEURON_ALIF) d.g_k[idx] = gk;
        d.psc[idx] = psc_decay(d.psc_coef, d.psc_tau, i, P);
        if (d.v_trace) d.v_trace[(k * B) * n + idx] = v;
        if (USE_REF && d.ref_trace) d.ref_trace[(k * B) * n + idx] = ref;
        if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[(k * B) * n + idx] = gk;
        if (d.psc_trace && k > 0) d.psc_trace[((k - 1) * B) * n + idx] = P;
      } else {
        // Finished sample: its state freezes at its last step.  On the first
        // step past the end the pending sum completes psc of that last step;
        // later arrivals are dropped.
        if (k == len) d.psc[idx] = add(d.psc[idx], pending);
        if (d.v_trace) d.v_trace[(k * B) * n + idx] = d.v[idx];
        if (USE_REF && d.ref_trace) d.ref_trace[(k * B) * n + idx] = d.refractory[idx];
        if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[(k * B) * n + idx] = d.g_k[idx];
        if (d.psc_trace && k > 0) d.psc_trace[((k - 1) * B) * n + idx] = d.psc[idx];
      }
      if (d.spikes) d.spikes[(k * B) * n + idx] = s;
    }
    const uint32_t word = __ballot_sync(0xffffffffu, s != 0.0f);
    if ((tid & 31) == 0 && i < n) {
      const int64_t w = i >> 5;
      d.hist[((t % d.hist_len) * B + b) * words + w] = word;
      if (d.raster) d.raster[(k * B + b) * words + w] = word;
    }
    if (s != 0.0f) atomicOr(&smask[tn * mw + (b >> 5)], 1u << (b & 31));
  }
  __syncthreads();

  // Compact the neurons of this tile that spiked in any sample.
  EngCounters* cnt = reinterpret_cast<EngCounters*>(d.work);
  int32_t* list_j = d.work + 4;
  uint32_t* list_m = reinterpret_cast<uint32_t*>(d.work + 4 + 2 * n);  // [2][n][mw]
  const int par = int(t & 1);
  __shared__ int32_t warp_tot[kEngThreads / 32];
  __shared__ int32_t block_base;
  bool act = false;
  if (tid < nt) {
    for (int q = 0; q < mw; ++q) act |= smask[tid * mw + q] != 0;
  }
  const uint32_t bal = __ballot_sync(0xffffffffu, act);
  const int wid = tid >> 5;
  if ((tid & 31) == 0) warp_tot[wid] = __popc(bal);
  __syncthreads();
  if (tid == 0) {
    int32_t tot = 0;
    for (int q = 0; q < kEngThreads / 32; ++q) {
      const int32_t c = warp_tot[q];
      warp_tot[q] = tot;
      tot += c;
    }
    block_base = tot ? atomicAdd(&cnt->list_count[par], tot) : 0;
  }
  __syncthreads();
  if (act) {
    const int32_t pos = block_base + warp_tot[wid] + __popc(bal & ((1u << (tid & 31)) - 1u));
    list_j[par * n + pos] = int32_t(i);
    for (int q = 0; q < mw; ++q) list_m[(int64_t(par) * n + pos) * mw + q] = smask[tid * mw + q];
  }
}

__global__ void __launch_bounds__(kEngThreads) k_eng_scatter(bt_engine_desc d, int64_t k) {
  const int64_t n = d.n, B = d.batch;
  const int64_t t = d.t0 + k;
  const int R = d.n_bins;
  const int mw = mask_words(B);
  EngCounters* cnt = reinterpret_cast<EngCounters*>(d.work);
  const int par = int(t & 1);
  const int32_t count = cnt->list_count[par];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    cnt->list_count[par ^ 1] = 0;  // consumed by the next step's neuron kernel
    if (d.stats) d.stats[k * 4 + 0] = count;
  }
  const int32_t* list_j = d.work + 4 + par * n;
  const uint32_t* list_m = reinterpret_cast<const uint32_t*>(d.work + 4 + 2 * n) + int64_t(par) * n * mw;
  const unsigned lane = lane_id();
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  long long ev = 0, ed = 0;
  for (int64_t it = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; it < count; it += warps) {
    const int32_t j = list_j[it];
    const int32_t beg = d.csr_ptr[j], end = d.csr_ptr[j + 1];
    int nsamp = 0;
    for (int q = 0; q < mw; ++q) nsamp += __popc(list_m[it * mw + q]);
    ev += (long long)nsamp * (end - beg);
    ed += end - beg;
    for (int32_t gidx = (beg & ~3) + int32_t(lane) * 4; gidx < end; gidx += 128) {
      const uint4 d4 = __ldg(reinterpret_cast<const uint4*>(d.csr_dst + gidx));
      const float4 w4 = __ldg(reinterpret_cast<const float4*>(d.csr_w + gidx));
      const uint32_t dd[4] = {d4.x, d4.y, d4.z, d4.w};
      const float ww[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        const int32_t e = gidx + qq;
        if (e < beg || e >= end) continue;
        const uint32_t post = dd[qq] & kIdMask;
        const int64_t slot = (t + (dd[qq] >> BT_BIN_SHIFT)) % R;
        float* base = d.ring + (slot * B) * n + post;
        for (int q = 0; q < mw; ++q) {
          uint32_t m = list_m[it * mw + q];
          while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            atomicAdd(base + (int64_t(q) * 32 + l) * n, ww[qq]);
          }
        }
      }
    }
  }
  if (d.stats && lane == 0 && ed) {
    atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 1), (unsigned long long)ev);
    atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 2), (unsigned long long)ed);
  }
}

// psc_{t_end-1} = stored + pending(t_end - 1); clears that slot.
__global__ void k_eng_scatter_final(bt_engine_desc d) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t n = d.n, B = d.batch;
  if (idx >= B * n) return;
  const int64_t t_last = d.t0 + d.n_steps - 1;
  const int R = d.n_bins;
  float* ring = d.ring + (((t_last % R + R) % R) * B) * n;
  const float pending = ring[idx];
  ring[idx] = 0.0f;
  const int64_t b = idx / n;
  const int64_t len = d.sample_len ? d.sample_len[b] : INT64_MAX;
  if (d.n_steps - 1 < len) {
    const float P = add(d.psc[idx], pending);
    d.psc[idx] = P;
    if (d.psc_trace) d.psc_trace[((d.n_steps - 1) * B) * n + idx] = P;
  } else if (d.psc_trace) {
    d.psc_trace[((d.n_steps - 1) * B) * n + idx] = d.psc[idx];
  }
}

// ----------------------------------------------------------------- gather --

// Ordered in-edge gather of W z for (b, i) at arrival step `ta`:
// sum over in-edges (pre, bin) ascending of w * z_{ta - bin}[pre].
__device__ __forceinline__ float gather_in(const bt_engine_desc& d, int64_t i, int64_t b, int64_t ta, int64_t words) {
  const unsigned lane = lane_id();
  const int32_t beg = __ldg(d.csc_ptr + i), end = __ldg(d.csc_ptr + i + 1);
  const int64_t H = d.hist_len;
  float acc = 0.0f;
  for (int32_t base = beg; base < end; base += 32) {
    const int32_t e = base + int32_t(lane);
    float w = 0.0f;
    bool act = false;
    if (e < end) {
      const uint32_t src = __ldg(d.csc_src + e);
      const uint32_t pre = src & kIdMask;
      const int64_t s = ta - int64_t(src >> BT_BIN_SHIFT);
      const uint32_t word = d.hist[(((s % H) + H) % H * d.batch + b) * words + (pre >> 5)];
      act = (word >> (pre & 31)) & 1u;
      if (act) w = __ldg(d.csc_w + e);
    }
    uint32_t m = __ballot_sync(0xffffffffu, act);
    while (m) {
      const int q = __ffs(m) - 1;
      m &= m - 1;
      acc = fmaf(__shfl_sync(0xffffffffu, w, q), 1.0f, acc);
    }
  }
  return acc;
}

// One launch per step.  Block = 32 warps = 32 consecutive neurons, so each
// (sample, 32-neuron word) of the spike bitmap is written by one thread.
template <int KIND, bool HARD, bool USE_REF>
__global__ void __launch_bounds__(1024) k_eng_gather(bt_engine_desc d, int64_t k) {
  extern __shared__ uint32_t sbits[];  // [batch]
  const int64_t n = d.n, B = d.batch;
  const int64_t words = (n + 31) >> 5;
  const int64_t t = d.t0 + k;
  const int wid = threadIdx.x >> 5;
  const unsigned lane = lane_id();
  const int64_t i = int64_t(blockIdx.x) * 32 + wid;
  for (int64_t b = threadIdx.x; b < B; b += blockDim.x) sbits[b] = 0;
  __syncthreads();
  if (i < n) {
    for (int64_t b = 0; b < B; ++b) {
      const int64_t idx = b * n + i;
      const int64_t len = d.sample_len ? d.sample_len[b] : INT64_MAX;
      // synapse update of step t-1 (skipped on the first step of a call: the
      // stored psc already is psc_{t0-1}; skipped after a sample's last step)
      float P = d.psc[idx];
      if (k > 0 && k - 1 < len) {
        const float wz = gather_in(d, i, b, t - 1, words);
        P = add(psc_decay(d.psc_coef, d.psc_tau, i, P), wz);
      }
      float s = 0.0f;
      if (lane == 0) {
        if (k < len) {
          const float I = d.x ? add(P, d.x[(k * B) * n + idx]) : P;
          float v = d.v[idx];
          float ref = USE_REF ? d.refractory[idx] : 0.0f;
          float gk = KIND == BT_NEURON_ALIF ? d.g_k[idx] : 0.0f;
          const NeuronOut o = neuron_update<KIND, HARD, USE_REF>(d.neuron, i, I, v, ref, gk);
          s = o.spike;
          d.v[idx] = v;
          if (USE_REF) d.refractory[idx] = ref;
          if (KIND == BT_NEURON_ALIF) d.g_k[idx] = gk;
        }
        d.psc[idx] = P;
        if (d.v_trace) d.v_trace[(k * B) * n + idx] = d.v[idx];
        if (USE_REF && d.ref_trace) d.ref_trace[(k * B) * n + idx] = d.refractory[idx];
        if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[(k * B) * n + idx] = d.g_k[idx];
        if (d.psc_trace && k > 0) d.psc_trace[((k - 1) * B) * n + idx] = P;
        if (d.spikes) d.spikes[(k * B) * n + idx] = s;
        if (s != 0.0f) atomicOr(&sbits[b], 1u << (i & 31));
      }
    }
  }
  __syncthreads();
  const int64_t w = int64_t(blockIdx.x);
  for (int64_t b = threadIdx.x; b < B; b += blockDim.x) {
    d.hist[((t % d.hist_len) * B + b) * words + w] = sbits[b];
    if (d.raster) d.raster[(k * B + b) * words + w] = sbits[b];
  }
}

// Synapse update of the last step of a call: psc_{t_end-1}.
__global__ void __launch_bounds__(1024) k_eng_gather_final(bt_engine_desc d) {
  const int64_t n = d.n, B = d.batch;
  const int64_t words = (n + 31) >> 5;
  const int64_t k = d.n_steps - 1;
  const int64_t t = d.t0 + k;
  const int64_t i = int64_t(blockIdx.x) * 32 + (threadIdx.x >> 5);
  if (i >= n) return;
  for (int64_t b = 0; b < B; ++b) {
    const int64_t idx = b * n + i;
    const int64_t len = d.sample_len ? d.sample_len[b] : INT64_MAX;
    if (k >= len) {
      if (lane_id() == 0 && d.psc_trace) d.psc_trace[(k * B) * n + idx] = d.psc[idx];
      continue;
    }
    const float wz = gather_in(d, i, b, t, words);
    if (lane_id() == 0) {
      const float P = add(psc_decay(d.psc_coef, d.psc_tau, i, d.psc[idx]), wz);
      d.psc[idx] = P;
      if (d.psc_trace) d.psc_trace[(k * B) * n + idx] = P;
    }
  }
}

// ------------------------------------------------------------ ring rebuild --

// One warp per (past step s, presynaptic neuron j): re-add the still-pending
// contributions of z_s (arrivals >= t0) into the ring.
__global__ void k_ring_from_history(bt_engine_desc d) {
  const int64_t gw = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t n = d.n, B = d.batch;
  const int R = d.n_bins;
  const int64_t back = R - 1;  // steps t0-1 .. t0-back can still have pending arrivals
  if (gw >= back * n) return;
  const int64_t s = d.t0 - 1 - gw / n;
  const int64_t j = gw % n;
  const int64_t words = (n + 31) >> 5;
  const int64_t H = d.hist_len;
  const unsigned lane = lane_id();
  const int32_t beg = d.csr_ptr[j], end = d.csr_ptr[j + 1];
  for (int64_t b = 0; b < B; ++b) {
    const uint32_t word = d.hist[((((s % H) + H) % H) * B + b) * words + (j >> 5)];
    if (!((word >> (j & 31)) & 1u)) continue;
    for (int32_t e = beg + int32_t(lane); e < end; e += 32) {
      const uint32_t dd = d.csr_dst[e];
      const int64_t arrival = s + (dd >> BT_BIN_SHIFT);
      if (arrival < d.t0) continue;
      atomicAdd(d.ring + ((arrival % R) * B + b) * n + (dd & kIdMask), d.csr_w[e]);
    }
  }
}

// ------------------------------------------------------- input projection --

// Per row r: ascending list of nonzero input channels (warp ballot + prefix).
__global__ void k_row_nonzeros(int64_t rows, int64_t c_in, const float* __restrict__ xin, int32_t* __restrict__ cnt,
                               int32_t* __restrict__ idx) {
  const int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (r >= rows) return;
  const unsigned lane = lane_id();
  int32_t total = 0;
  for (int64_t c0 = 0; c0 < c_in; c0 += 32) {
    const int64_t c = c0 + lane;
    const bool nz = c < c_in && xin[r * c_in + c] != 0.0f;
    const uint32_t m = __ballot_sync(0xffffffffu, nz);
    if (nz) idx[r * c_in + total + __popc(m & ((1u << lane) - 1u))] = int32_t(c);
    total += __popc(m);
  }
  if (lane == 0) cnt[r] = total;
}

// out[r][i] = sum over nonzero xin[r][c] (ascending c) of xin * w_t[c][i] (+ bias).
// grid.x walks row blocks fastest so that concurrently resident blocks share a
// narrow slice of w_t in L2.
constexpr int kProjRows = 8;
__global__ void __launch_bounds__(256) k_input_project(int64_t rows, int64_t c_in, int64_t n,
                                                       const float* __restrict__ xin,
                                                       const float* __restrict__ w_t,
                                                       const float* __restrict__ bias,
                                                       const int32_t* __restrict__ cnt,
                                                       const int32_t* __restrict__ idx, float* __restrict__ out) {
  const int64_t i = int64_t(blockIdx.y) * 256 + threadIdx.x;
  const int64_t r0 = int64_t(blockIdx.x) * kProjRows;
  if (i >= n) return;
  const float bi = bias ? bias[i] : 0.0f;
  for (int64_t r = r0; r < r0 + kProjRows && r < rows; ++r) {
    const int32_t c_n = cnt[r];
    const int32_t* ri = idx + r * c_in;
    const float* xr = xin + r * c_in;
    float acc = 0.0f;
    for (int32_t q = 0; q < c_n; ++q) {
      const int32_t c = ri[q];
      acc = fmaf(xr[c], __ldg(w_t + int64_t(c) * n + i), acc);
    }
    out[r * n + i] = bias ? add(acc, bi) : acc;
  }
}

// --------------------------------------------------------------- bitmaps --

__global__ void k_bits_to_float(int64_t rows, int64_t n, const uint32_t* __restrict__ bits, float* __restrict__ out) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= rows * n) return;
  const int64_t r = idx / n, i = idx % n;
  const int64_t words = (n + 31) >> 5;
  out[idx] = float((bits[r * words + (i >> 5)] >> (i & 31)) & 1u);
}

__global__ void k_float_to_bits(int64_t rows, int64_t n, const float* __restrict__ in, uint32_t* __restrict__ bits) {
  const int64_t words = (n + 31) >> 5;
  const int64_t gw = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (gw >= rows * words) return;
  const int64_t r = gw / words, w = gw % words;
  const int64_t i = w * 32 + lane_id();
  const bool nz = i < n && in[r * n + i] != 0.0f;
  const uint32_t m = __ballot_sync(0xffffffffu, nz);
  if (lane_id() == 0) bits[gw] = m;
}

}  // namespace bt

using namespace bt;

namespace {

int engine_check(const bt_engine_desc* d) {
  if (!d) return bt_set_error(BT_ERR_INVALID, "null engine descriptor");
  if (int st = bt_check_neuron_desc(&d->neuron)) return st;
  BT_CHECK_ARG(d->n > 0 && d->n < BT_MAX_NEURONS, "n=%lld outside (0, 2^25)", (long long)d->n);
  BT_CHECK_ARG(d->batch > 0 && d->batch * d->n < (int64_t(1) << 40), "bad batch");
  BT_CHECK_ARG(d->n_bins >= 1 && d->n_bins <= BT_MAX_BINS, "n_bins=%d outside [1, 128]", d->n_bins);
  BT_CHECK_ARG(d->hist_len >= d->n_bins + 2, "hist_len=%d must be >= n_bins + 2", d->hist_len);
  BT_CHECK_ARG(d->n_steps >= 0 && d->t0 >= 0, "negative step index");
  BT_CHECK_ARG(d->mode == BT_MODE_SCATTER || d->mode == BT_MODE_GATHER, "mode=%d", d->mode);
  BT_CHECK_ARG(d->v && d->psc && d->hist, "state pointer missing (v / psc / hist)");
  BT_CHECK_ARG(!d->neuron.use_refractory || d->refractory, "refractory state missing");
  BT_CHECK_ARG(d->neuron.kind != BT_NEURON_ALIF || d->g_k, "g_k state missing");
  BT_CHECK_ARG(d->psc_coef.ptr && d->psc_tau.ptr, "PSC coefficients missing");
  BT_CHECK_ARG(d->neuron.spiking, "the fused engine needs a spiking (Heaviside) forward");
  if (d->mode == BT_MODE_SCATTER) {
    BT_CHECK_ARG(d->csr_ptr && d->csr_dst && d->csr_w && d->ring && d->work, "scatter needs CSR, ring and work");
    BT_CHECK_ARG((reinterpret_cast<uintptr_t>(d->csr_dst) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(d->csr_w) & 15) == 0,
                 "CSR edge arrays must be 16-byte aligned and padded to a multiple of 4");
  } else {
    BT_CHECK_ARG(d->csc_ptr && d->csc_src && d->csc_w, "gather needs CSC");
  }
  return BT_OK;
}

int sample_groups(int64_t batch) {
  int sg = 1;
  while (sg * 2 <= 8 && sg * 2 <= batch) sg *= 2;
  return sg;
}

template <int KIND, bool HARD, bool USE_REF>
int run_typed(const bt_engine_desc& d, cudaStream_t s) {
  const int64_t n = d.n;
  if (d.mode == BT_MODE_SCATTER) {
    const int sg = sample_groups(d.batch);
    const int nt = kEngThreads / sg;
    const int grid = int(ceil_div(n, nt));
    const size_t smem = sizeof(uint32_t) * size_t(nt) * size_t(mask_words(d.batch));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (smem > 48 * 1024) {
      if (cudaFuncSetAttribute(k_eng_neuron<KIND, HARD, USE_REF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(smem)) != cudaSuccess)
        return bt_set_error(BT_ERR_CUDA, "shared memory request of %zu bytes refused", smem);
    }
    if (cudaMemsetAsync(d.work, 0, sizeof(EngCounters), s) != cudaSuccess)
      return bt_set_error(BT_ERR_CUDA, "memset failed");
    for (int64_t k = 0; k < d.n_steps; ++k) {
      k_eng_neuron<KIND, HARD, USE_REF><<<grid, kEngThreads, smem, s>>>(d, k, sg);
      k_eng_scatter<<<sms * 8, kEngThreads, 0, s>>>(d, k);
    }
    BT_CHECK_LAUNCH("k_eng_neuron/k_eng_scatter");
    if (d.n_steps > 0) {
      k_eng_scatter_final<<<int(ceil_div(d.batch * n, 256)), 256, 0, s>>>(d);
      BT_CHECK_LAUNCH("k_eng_scatter_final");
    }
  } else {
    const int grid = int(ceil_div(n, 32));
    const size_t smem = sizeof(uint32_t) * size_t(d.batch);
    BT_CHECK_ARG(smem <= 48 * 1024, "batch too large for the gather engine");
    for (int64_t k = 0; k < d.n_steps; ++k)
      k_eng_gather<KIND, HARD, USE_REF><<<grid, 1024, smem, s>>>(d, k);
    BT_CHECK_LAUNCH("k_eng_gather");
    if (d.n_steps > 0) {
      k_eng_gather_final<<<grid, 1024, 0, s>>>(d);
      BT_CHECK_LAUNCH("k_eng_gather_final");
    }
  }
  return BT_OK;
}

}  // namespace

extern "C" int bt_engine_run(const bt_engine_desc* d, void* stream) {
  if (int st = engine_check(d)) return st;
  if (d->n_steps == 0) return BT_OK;
  if (d->stats && cudaMemsetAsync(d->stats, 0, sizeof(int64_t) * 4 * size_t(d->n_steps),
                                  static_cast<cudaStream_t>(stream)) != cudaSuccess)
    return bt_set_error(BT_ERR_CUDA, "memset failed");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool h = d->neuron.hard_reset != 0, r = d->neuron.use_refractory != 0;
  if (d->neuron.kind == BT_NEURON_LIF) {
    if (h && r) return run_typed<BT_NEURON_LIF, true, true>(*d, s);
    if (h) return run_typed<BT_NEURON_LIF, true, false>(*d, s);
    if (r) return run_typed<BT_NEURON_LIF, false, true>(*d, s);
    return run_typed<BT_NEURON_LIF, false, false>(*d, s);
  }
  if (h && r) return run_typed<BT_NEURON_ALIF, true, true>(*d, s);
  if (h) return run_typed<BT_NEURON_ALIF, true, false>(*d, s);
  if (r) return run_typed<BT_NEURON_ALIF, false, true>(*d, s);
  return run_typed<BT_NEURON_ALIF, false, false>(*d, s);
}

extern "C" int bt_engine_ring_from_history(const bt_engine_desc* d, void* stream) {
  if (int st = engine_check(d)) return st;
  BT_CHECK_ARG(d->mode == BT_MODE_SCATTER, "the ring exists in scatter mode only");
  const int64_t back = d->n_bins - 1;
  if (back == 0) return BT_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_ring_from_history<<<int(ceil_div(back * d->n * 32, 256)), 256, 0, s>>>(*d);
  BT_CHECK_LAUNCH("k_ring_from_history");
  return BT_OK;
}

extern "C" int bt_input_project(int64_t rows, int64_t c_in, int64_t n, const float* xin, const float* w_t,
                                const float* bias, float* out, int32_t* work, void* stream) {
  BT_CHECK_ARG(rows >= 0 && c_in >= 0 && n >= 0, "negative size");
  if (rows == 0 || n == 0) return BT_OK;
  BT_CHECK_ARG(xin && w_t && out && work, "null pointer");
  BT_CHECK_ARG(rows * c_in < (int64_t(1) << 40), "too large");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int32_t* cnt = work;
  int32_t* idx = work + rows;
  k_row_nonzeros<<<int(ceil_div(rows * 32, 256)), 256, 0, s>>>(rows, c_in, xin, cnt, idx);
  BT_CHECK_LAUNCH("k_row_nonzeros");
  dim3 grid(unsigned(ceil_div(rows, kProjRows)), unsigned(ceil_div(n, 256)));
  BT_CHECK_ARG(grid.y < 65536, "n too large for the projection grid");
  k_input_project<<<grid, 256, 0, s>>>(rows, c_in, n, xin, w_t, bias, cnt, idx, out);
  BT_CHECK_LAUNCH("k_input_project");
  return BT_OK;
}

extern "C" int bt_bits_to_float(int64_t rows, int64_t n, const uint32_t* bits, float* out, void* stream) {
  BT_CHECK_ARG(rows >= 0 && n >= 0, "negative size");
  if (rows * n == 0) return BT_OK;
  BT_CHECK_ARG(bits && out, "null pointer");
  k_bits_to_float<<<int(ceil_div(rows * n, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(rows, n, bits, out);
  BT_CHECK_LAUNCH("k_bits_to_float");
  return BT_OK;
}

extern "C" int bt_float_to_bits(int64_t rows, int64_t n, const float* in, uint32_t* bits, void* stream) {
  BT_CHECK_ARG(rows >= 0 && n >= 0, "negative size");
  if (rows * n == 0) return BT_OK;
  BT_CHECK_ARG(bits && in, "null pointer");
  const int64_t words = (n + 31) >> 5;
  k_float_to_bits<<<int(ceil_div(rows * words * 32, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(rows, n, in,
                                                                                                         bits);
  BT_CHECK_LAUNCH("k_float_to_bits");
  return BT_OK;
}
