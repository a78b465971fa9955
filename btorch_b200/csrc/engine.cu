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
//   k_eng_neuron  (step t): P = stored + acc; zero acc; neuron update with
//                 I = P + x_t; stored = decay(P); spike bitmaps; the step's
//                 spike set: a mask of spiking samples per neuron and the
//                 compacted list of neurons that spiked in any sample (warp
//                 ballot + one warp-aggregated atomic on one of 64 counters).
//   k_eng_scatter (step t): for every delay bin d and every neuron j in the
//                 spike set of step t - d, stream the out-edges of row
//                 j * R + d of the delay-expanded matrix with 128-bit loads
//                 and add w into acc[b][post] for every sample b in j's mask
//                 (fp32 reductions, resolved in L2: acc is [B][n], the size
//                 of one state variable, whatever the delay range).
//   The spike sets of the last R steps live in a ring of R + 1 slots (slot =
//   step mod (R + 1)) in the scratch; the last reader of a set clears it.
//   "stored" holds decay(psc_{t-1}) during a run and acc the sum W z of the
//   step, so the reference's rounding of psc = decay(psc) + Wz is kept
//   (exact sums when weights are dyadic).
//
// GATHER mode, one launch per step (k_eng_gather): each warp owns a neuron,
//   computes P_{t-1} = decay(P_{t-2}) + sum over its in-edges (pre, bin) in
//   ascending canonical order of w * z_{t-1-bin}[pre] (fmaf chain, exactly the
//   reference's CPU rounding), then runs the neuron update of step t.  The
//   last synapse update of a run is k_eng_gather_final.
//
// RECEPTOR CHANNELS (HeterSynapsePSC with n_receptor = C > 1,
// synapse.py:626-847): the matrix has C columns per neuron (post * C + r, the
// layout make_hetersynapse_conn builds, connection.py:218-587); PSC state,
// acc and the PSC coefficients are [batch][n * C], and the neuron's input is
// the receptor sum of its C channels (receptor_sum, the reference's
// psc.reshape(..., n, C).sum(-1) rounding).  Scatter and gather modes.
#include <algorithm>
#include <climits>
#include <cstring>
#include <type_traits>

#include "neuron.cuh"

namespace bt {

constexpr int kEngThreads = 256;
constexpr int kMaxRec = 16;  // receptor channels per neuron

// Receptor columns per neuron (0 in the descriptor means 1).
__host__ __device__ __forceinline__ int n_rec(const bt_engine_desc& d) { return d.n_rec > 1 ? d.n_rec : 1; }

// Sum of one neuron's C receptor PSCs p[0..C) in the order torch's CPU sum
// reduces a contiguous row of C floats, which the reference runs as
// psc.reshape(..., n, C).sum(-1) (synapse.py:744-747):
//   C < 4       left to right;
//   4 <= C < 8  a_j = p_j (j < 4), p_4 .. p_{C-1} added to a_0 in turn, then
//               ((a_0 + a_1) + a_2) + a_3;
//   C >= 8      a_j = p_j + p_{8+j} + ... over the whole groups of 8, the
//               left-to-right sum of the remaining tail added to a_0, then
//               a_0 + a_1 + ... + a_7 left to right.
// (Established against torch.sum for every C up to 39; the host mirror in
// btorch_b200/models/synapse.py is checked against torch.sum in the CPU
// tests.)  p holds M >= C values; indices are compile-time after unrolling.
template <int M>
__device__ __forceinline__ float receptor_sum(const float (&p)[M], int C) {
  if (C < 4 || M < 4) {
    float s = p[0];
#pragma unroll
    for (int r = 1; r < 4 && r < M; ++r)
      if (r < C) s = add(s, p[r]);
    return s;
  }
  if constexpr (M >= 4) {
    if (C < 8 || M < 8) {
      float a0 = p[0];
#pragma unroll
      for (int r = 4; r < 8 && r < M; ++r)
        if (r < C) a0 = add(a0, p[r]);
      return add(add(add(a0, p[1]), p[2]), p[3]);
    }
  }
  if constexpr (M >= 8) {
    const int full = C & ~7;
    float a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = p[j];
#pragma unroll
    for (int r = 8; r < M; ++r)
      if (r < full) a[r & 7] = add(a[r & 7], p[r]);
    if (full < C) {
      float t = 0.0f;
      bool first = true;
#pragma unroll
      for (int r = 8; r < M; ++r)
        if (r >= full && r < C) {
          t = first ? p[r] : add(t, p[r]);
          first = false;
        }
      a[0] = add(a[0], t);
    }
    float s = a[0];
#pragma unroll
    for (int j = 1; j < 8; ++j) s = add(s, a[j]);
    return s;
  }
  return p[0];  // not reached: C <= M
}

__host__ __device__ __forceinline__ int mask_words(int64_t batch) { return int((batch + 31) >> 5); }

// Words per neuron in the pull engine's sample masks: the word count rounded up
// to the vector width the kernel loads with (1, 2 or 4 words), unchanged above 4.
__host__ __device__ __forceinline__ int mask_stride(int64_t batch) {
  const int mw = mask_words(batch);
  return mw <= 1 ? 1 : mw <= 2 ? 2 : mw <= 4 ? 4 : mw;
}

// Slot indices of one step, computed on the host per launch so that no kernel
// evaluates a 64-bit modulo per element.
struct StepIdx {
  int q_t;     // t mod (R + 1): spike-set slot of step t (scatter)
  int h_t;     // t mod H:       history slot written at step t
  int h_prev;  // (t - 1) mod H: history slot of step t - 1
};

inline StepIdx step_idx(int64_t t, int R, int H) {
  StepIdx s;
  s.q_t = int(t % (R + 1));
  s.h_t = int(t % H);
  s.h_prev = int((t - 1) % H);
  return s;
}

// ---------------------------------------------------------------- scatter --

// Scatter-mode scratch (d.work, int32 words), Q = R + 1 spike-set slots:
//   [0, 2*Q*kSub)                  active-list counts and spike totals,
//                                  [slot][count | spikes][sub-list]
//   next Q*n                       "listed" flags, [slot][neuron]
//   next Q*kSub*cap                list entries, [slot][sub-list][cap]
//   next Q n S                     sample masks, [slot][neuron][S words], S = mask_stride(batch)
//   next kSub                      control words (ctrl[0]: blocks done with a dense step)
// Sub-list s only lists neurons [s*cap, (s+1)*cap) and each neuron is listed at
// most once per step (its flag), so a sub-list never holds more than cap
// entries.  cap is a multiple of 32, so the 32 neurons of a warp share one
// sub-list.
constexpr int kSub = 64;
// Dense delivery needs at least this many spiking samples per listed neuron on
// average: below it the per-event reductions of the list path are cheaper
// than the dense pull's random mask reads (measured crossover about 2.5).
constexpr int kDenseSpikesPerRow = 3;

// A power of two (>= 32), so the sub-list of neuron i is i >> log2(cap).
__host__ __device__ __forceinline__ int64_t sub_cap(int64_t n) {
  const int64_t c = (n + kSub - 1) / kSub;
  int64_t p = 32;
  while (p < c) p <<= 1;
  return p;
}

__host__ __device__ __forceinline__ int64_t scatter_work_words(int64_t n, int64_t batch, int n_bins) {
  const int64_t Q = int64_t(n_bins) + 1;
  return Q * (2 * kSub + n + kSub * sub_cap(n) + n * mask_stride(batch)) + kSub;
}

struct ScatterScratch {
  int32_t* count;
  int32_t* spk;   // spikes (sample-neuron pairs) listed per sub-list
  int32_t* flag;
  int32_t* list;
  uint32_t* mask;
  int32_t* ctrl;
  int64_t cap;
  int cap_shift;  // log2(cap)
  int ms;
};

__host__ __device__ __forceinline__ int log2_pow2(int64_t c) {
  int s = 0;
  while ((int64_t(1) << s) < c) ++s;
  return s;
}

__host__ __device__ __forceinline__ ScatterScratch scatter_scratch(const bt_engine_desc& d, int q) {
  ScatterScratch w;
  const int64_t n = d.n;
  const int64_t Q = int64_t(d.n_bins) + 1;
  w.ms = mask_stride(d.batch);
  w.cap = sub_cap(n);
  w.cap_shift = log2_pow2(w.cap);
  w.count = d.work + q * 2 * kSub;
  w.spk = w.count + kSub;
  w.flag = d.work + Q * 2 * kSub + q * n;
  w.list = d.work + Q * 2 * kSub + Q * n + q * kSub * w.cap;
  w.mask = reinterpret_cast<uint32_t*>(d.work + Q * 2 * kSub + Q * n + Q * kSub * w.cap) + int64_t(q) * n * w.ms;
  w.ctrl = d.work + Q * (2 * kSub + n + kSub * w.cap + n * w.ms);
  return w;
}

// Publish neuron i's spikes of step t in the step's spike set `ws` (bit u of
// `spiked`: sample b0 + u): the samples' bits in the neuron's mask -- one
// atomic, the S samples lie in one 32-sample word (b0 % S == 0, S | 32) --
// and the neuron in the compacted list if this warp's samples are the first
// to spike (one warp-aggregated atomic on one of kSub counters).  Called by
// every lane of the warp.
__device__ __forceinline__ void publish_spikes_ws(const ScatterScratch& ws, int i, int b0, uint32_t spiked) {
  if (__ballot_sync(0xffffffffu, spiked != 0) == 0) return;  // warp-uniform
  const unsigned lane = lane_id();
  bool first = false;
  if (spiked) {
    atomicOr(ws.mask + int64_t(i) * ws.ms + (b0 >> 5), spiked << (b0 & 31));
    first = atomicOr(ws.flag + i, 1) == 0;
  }
  const uint32_t fb = __ballot_sync(0xffffffffu, first);
  const int sub = (i - int(lane)) >> ws.cap_shift;  // same for the whole warp (cap % 32 == 0)
  const int nspk = __reduce_add_sync(0xffffffffu, unsigned(__popc(spiked)));
  if (lane == 0 && nspk) atomicAdd(ws.spk + sub, nspk);
  if (fb == 0) return;
  int32_t base = 0;
  if (lane == 0) base = atomicAdd(ws.count + sub, __popc(fb));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (first) ws.list[int64_t(sub) * ws.cap + base + __popc(fb & ((1u << lane) - 1u))] = i;
}

// The same for a kernel that derives the spike set from the descriptor.
template <int S>
__device__ __forceinline__ void publish_spikes(const bt_engine_desc& d, const StepIdx& si, int64_t i, int64_t b0,
                                               uint32_t spiked) {
  if (__ballot_sync(0xffffffffu, spiked != 0) == 0) return;  // warp-uniform
  const unsigned lane = lane_id();
  const ScatterScratch ws = scatter_scratch(d, si.q_t);
  bool first = false;
  if (spiked) {
    uint32_t* mrow = ws.mask + i * ws.ms;
#pragma unroll
    for (int u = 0; u < S; ++u)
      if (spiked & (1u << u)) atomicOr(mrow + ((b0 + u) >> 5), 1u << ((b0 + u) & 31));
    first = atomicOr(ws.flag + i, 1) == 0;
  }
  const uint32_t fb = __ballot_sync(0xffffffffu, first);
  const int sub = int((i - lane) >> ws.cap_shift);  // same for the whole warp (cap % 32 == 0)
  const int nspk = __reduce_add_sync(0xffffffffu, unsigned(__popc(spiked)));
  if (lane == 0 && nspk) atomicAdd(ws.spk + sub, nspk);
  if (fb == 0) return;
  int32_t base = 0;
  if (lane == 0) base = atomicAdd(ws.count + sub, __popc(fb));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (first) ws.list[sub * ws.cap + base + __popc(fb & ((1u << lane) - 1u))] = int32_t(i);
}

// Grid (ceil(n / 256), ceil(batch / S)): a thread owns neuron i for S
// consecutive samples; a warp covers one 32-neuron bitmap word of each of
// them.  All S samples' state is loaded before any is updated (memory-level
// parallelism), and the neuron's parameters are read once for the S samples.
// `ws` is the step's spike set, its pointers computed on the host; indices
// are 32-bit (batch * n < 2^31 in scatter mode, checked on the host) except
// into the per-step input and trace arrays.
template <int KIND, bool HARD, bool USE_REF, int S, bool FAST>
__global__ void __launch_bounds__(kEngThreads) k_eng_neuron(bt_engine_desc d, int k, StepIdx si, ScatterScratch ws) {
  const int n = int(d.n), B = int(d.batch);
  const int words = (n + 31) >> 5;
  const int i = int(blockIdx.x) * kEngThreads + int(threadIdx.x);
  const int b0 = int(blockIdx.y) * S;
  if ((i & ~31) >= n) return;  // whole warps past the last word
  const bool valid = i < n;
  const int nb = B - b0 < S ? B - b0 : S;  // samples of this block (uniform)
  const int off0 = b0 * n + (valid ? i : 0);
  float* __restrict__ ring_p = d.ring + off0;  // acc: W z of the previous step
  float* __restrict__ psc_p = d.psc + off0;
  float* __restrict__ v_p = d.v + off0;
  float* __restrict__ ref_p = USE_REF ? d.refractory + off0 : nullptr;
  float* __restrict__ gk_p = KIND == BT_NEURON_ALIF ? d.g_k + off0 : nullptr;
  const float* __restrict__ x_p = d.x ? d.x + int64_t(k) * B * n + off0 : nullptr;
  const uint64_t pol_stream = l2_evict_first(), pol_keep = l2_evict_last();
  // Every load before the first store: a load behind a store through a
  // pointer that may alias it waits for the store.  A sample past its length
  // (k > len) reads and writes no state unless state traces are requested:
  // its state is frozen and its accumulator is not read again in this call.
  const bool traces = d.v_trace || d.psc_trace || d.ref_trace || d.gk_trace || d.spikes;
  const bool st_traces = d.v_trace || d.psc_trace || d.ref_trace || d.gk_trace;
  float pend[S], pv[S], xv[S], vv[S], rv[S], gv[S];
  int lenv[S];
#pragma unroll
  for (int u = 0; u < S; ++u) lenv[u] = (valid && u < nb && d.sample_len) ? d.sample_len[b0 + u] : INT_MAX;
#pragma unroll
  for (int u = 0; u < S; ++u) {
    const bool in = valid && u < nb;
    const bool live = in && k < lenv[u], edge = in && k <= lenv[u], frozen = in && st_traces;
    const int o = u * n;
    pend[u] = edge ? ld_f32(ring_p + o, pol_keep) : 0.0f;
    pv[u] = (edge || frozen) ? psc_p[o] : 0.0f;
    xv[u] = (live && x_p) ? ld_nc_f32(x_p + o, pol_stream) : 0.0f;
    vv[u] = (live || frozen) ? v_p[o] : 0.0f;
    rv[u] = ((live || frozen) && USE_REF) ? ref_p[o] : 0.0f;
    gv[u] = ((live || frozen) && KIND == BT_NEURON_ALIF) ? gk_p[o] : 0.0f;
  }
  const int ip = valid ? i : 0;
  const NeuronParams prm = load_params<KIND, USE_REF>(d.neuron, ip);
  const float pc = d.psc_uniform ? d.psc_coef_s : ld(d.psc_coef, ip);
  const float pt = d.psc_uniform ? d.psc_tau_s : ld(d.psc_tau, ip);
  const Div dpt = make_div(pt, d.psc_uniform && d.psc_fast_div, d.psc_rcp);
  const unsigned lane = lane_id();
  uint32_t* hist_p = d.hist + (int64_t(si.h_t) * B + b0) * words + (i >> 5);
  uint32_t* raster_p = d.raster ? d.raster + (int64_t(k) * B + b0) * words + (i >> 5) : nullptr;
  uint32_t spiked = 0;  // bit u: spiked in sample b0 + u
#pragma unroll
  for (int u = 0; u < S; ++u) {
    if (u >= nb) break;  // uniform across the block
    const int o = u * n;
    float s = 0.0f;
    if (valid) {
      const int len = lenv[u];
      if (k <= len) st_f32(ring_p + o, 0.0f, pol_keep);
      float v = vv[u], ref = rv[u], gk = gv[u];
      float P;
      if (k < len) {
        P = add(pv[u], pend[u]);
        const float I = x_p ? add(P, xv[u]) : P;
        const NeuronOut out = neuron_update<KIND, HARD, USE_REF, true, FAST>(prm, I, v, ref, gk);
        s = out.spike;
        v_p[o] = v;
        if (USE_REF) ref_p[o] = ref;
        if (KIND == BT_NEURON_ALIF) gk_p[o] = gk;
        psc_p[o] = psc_decay_k<FAST>(pc, dpt, P);
      } else {
        // Finished sample: its state freezes at its last step.  On the first
        // step past the end the pending sum completes psc of that last step;
        // later arrivals are dropped.
        P = pv[u];
        if (k == len) {
          P = add(P, pend[u]);
          psc_p[o] = P;
        }
      }
      if (traces) {
        const int64_t tix = (int64_t(k) * B + b0 + u) * n + i;
        if (d.psc_trace && k > 0) d.psc_trace[tix - int64_t(B) * n] = P;
        if (d.v_trace) d.v_trace[tix] = v;
        if (USE_REF && d.ref_trace) d.ref_trace[tix] = ref;
        if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[tix] = gk;
        if (d.spikes) d.spikes[tix] = s;
      }
    }
    const uint32_t word = __ballot_sync(0xffffffffu, s != 0.0f);
    if (lane == 0) {
      hist_p[u * words] = word;
      if (raster_p) raster_p[u * words] = word;
    }
    if (s != 0.0f) spiked |= 1u << u;
  }
  publish_spikes_ws(ws, i, b0, spiked);
}

// SCATTER neuron step with receptor channels (n_rec = C > 1): for each
// channel column c = i * C + r, P_r = stored + acc (acc zeroed); the neuron's
// input is receptor_sum(P) (+ x); stored = decay_r(P_r).  Grid
// (ceil(n / 256), batch): a thread owns (neuron i, sample b).  CT = C known
// at compile time (2 or 4: the channels of (b, i) are one 8- or 16-byte
// vector) or 0 (any C up to kMaxRec).  Every load of the thread is issued
// before its first store: a load behind a store through a pointer that may
// alias it waits for the store, which made this step latency bound.
template <int KIND, bool HARD, bool USE_REF, int CT>
__global__ void __launch_bounds__(kEngThreads) k_eng_neuron_rec(bt_engine_desc d, int64_t k, StepIdx si) {
  constexpr int M = CT > 0 ? CT : kMaxRec;
  const int64_t n = d.n, B = d.batch;
  const int C = CT > 0 ? CT : n_rec(d);
  const int64_t nc = n * C;
  const int64_t words = (n + 31) >> 5;
  const int64_t i = int64_t(blockIdx.x) * kEngThreads + threadIdx.x;
  const int64_t b = blockIdx.y;
  if ((i & ~int64_t(31)) >= n) return;  // whole warps past the last word
  float s = 0.0f;
  const int64_t len = (i < n && d.sample_len) ? d.sample_len[b] : INT64_MAX;
  const bool st_traces = d.v_trace || d.psc_trace || d.ref_trace || d.gk_trace;
  if (i < n && (k <= len || st_traces)) {  // else: past its length, nothing to read or write
    const int64_t idx = b * n + i, c0 = b * nc + i * C;
    float* __restrict__ ring = d.ring + c0;
    float* __restrict__ psc = d.psc + c0;
    // loads
    float pend[M], stv[M], pc[M], pt[M];
    if constexpr (CT == 4) {
      const float4 a = *reinterpret_cast<const float4*>(ring), q = *reinterpret_cast<const float4*>(psc);
      pend[0] = a.x, pend[1] = a.y, pend[2] = a.z, pend[3] = a.w;
      stv[0] = q.x, stv[1] = q.y, stv[2] = q.z, stv[3] = q.w;
    } else if constexpr (CT == 2) {
      const float2 a = *reinterpret_cast<const float2*>(ring), q = *reinterpret_cast<const float2*>(psc);
      pend[0] = a.x, pend[1] = a.y;
      stv[0] = q.x, stv[1] = q.y;
    } else {
      for (int r = 0; r < C; ++r) {
        pend[r] = ring[r];
        stv[r] = psc[r];
      }
    }
#pragma unroll
    for (int r = 0; r < M; ++r) {
      if (r >= C) break;
      pc[r] = d.psc_uniform ? d.psc_coef_s : ld(d.psc_coef, i * C + r);
      pt[r] = d.psc_uniform ? d.psc_tau_s : ld(d.psc_tau, i * C + r);
    }
    float v = d.v[idx];
    float ref = USE_REF ? d.refractory[idx] : 0.0f;
    float gk = KIND == BT_NEURON_ALIF ? d.g_k[idx] : 0.0f;
    const float xv = d.x ? d.x[(k * B) * n + idx] : 0.0f;
    const NeuronParams prm = load_params<KIND, USE_REF>(d.neuron, i);
    // past a sample's end: the first step completes psc of its last step,
    // later arrivals are dropped (as k_eng_neuron)
    float P[M];
#pragma unroll
    for (int r = 0; r < M; ++r) {
      if (r >= C) break;
      P[r] = k <= len ? add(stv[r], pend[r]) : stv[r];
    }
    // stores
    if constexpr (CT == 4) {
      *reinterpret_cast<float4*>(ring) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else if constexpr (CT == 2) {
      *reinterpret_cast<float2*>(ring) = make_float2(0.0f, 0.0f);
    } else {
      for (int r = 0; r < C; ++r) ring[r] = 0.0f;
    }
    float out[M];
    bool write = k <= len;
    if (k < len) {
      const float I0 = receptor_sum(P, C);
      const float I = d.x ? add(I0, xv) : I0;
      const NeuronOut o = neuron_update<KIND, HARD, USE_REF, true>(prm, I, v, ref, gk);
      s = o.spike;
      d.v[idx] = v;
      if (USE_REF) d.refractory[idx] = ref;
      if (KIND == BT_NEURON_ALIF) d.g_k[idx] = gk;
#pragma unroll
      for (int r = 0; r < M; ++r) {
        if (r >= C) break;
        out[r] = psc_decay(pc[r], make_div(pt[r], d.psc_uniform && d.psc_fast_div, d.psc_rcp), P[r]);
      }
    } else {
#pragma unroll
      for (int r = 0; r < M; ++r) {
        if (r >= C) break;
        out[r] = P[r];
      }
    }
    if (write) {
      if constexpr (CT == 4) {
        *reinterpret_cast<float4*>(psc) = make_float4(out[0], out[1], out[2], out[3]);
      } else if constexpr (CT == 2) {
        *reinterpret_cast<float2*>(psc) = make_float2(out[0], out[1]);
      } else {
        for (int r = 0; r < C; ++r) psc[r] = out[r];
      }
    }
    if (d.psc_trace && k > 0) {
      float* tr = d.psc_trace + ((k - 1) * B) * nc + c0;
#pragma unroll
      for (int r = 0; r < M; ++r) {
        if (r >= C) break;
        tr[r] = P[r];
      }
    }
    const int64_t tix = (k * B) * n + idx;
    if (d.v_trace) d.v_trace[tix] = v;
    if (USE_REF && d.ref_trace) d.ref_trace[tix] = ref;
    if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[tix] = gk;
  }
  if (i < n && d.spikes) d.spikes[(k * B + b) * n + i] = s;
  const uint32_t word = __ballot_sync(0xffffffffu, s != 0.0f);
  if (lane_id() == 0) {
    d.hist[(int64_t(si.h_t) * B + b) * words + (i >> 5)] = word;
    if (d.raster) d.raster[(k * B + b) * words + (i >> 5)] = word;
  }
  publish_spikes<1>(d, si, i, b, s != 0.0f ? 1u : 0u);
}

// Offsets of the kSub sub-lists of one spike set in shared memory (warp 0
// scans the counts; two per lane).
__device__ __forceinline__ void sub_offsets(const ScatterScratch& ws, int32_t* s_off, int32_t* s_spk) {
  if (threadIdx.x < 32) {
    const int l = threadIdx.x;
    const int32_t c0 = ws.count[2 * l], c1 = ws.count[2 * l + 1];
    int32_t v = c0 + c1;
    int32_t sp = ws.spk[2 * l] + ws.spk[2 * l + 1];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, v, o);
      if (l >= o) v += y;
      sp += __shfl_xor_sync(0xffffffffu, sp, o);
    }
    s_off[2 * l] = v - c0 - c1;
    s_off[2 * l + 1] = v - c1;
    if (l == 31) s_off[kSub] = v;
    if (l == 0) *s_spk = sp;
  }
  __syncthreads();
}

// Sub-list holding item `it`: the last s with s_off[s] <= it (s_off[kSub] > it).
__device__ __forceinline__ int find_sub(const int32_t* s_off, int64_t it) {
  int lo = 0, hi = kSub - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (s_off[mid] <= it) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Block-level sum of per-thread event / edge counts, one pair of atomics per
// block (same-address atomics serialise in L2).  Every thread of the block
// must call it.
__device__ __forceinline__ void block_stats(const bt_engine_desc& d, int64_t k, long long ev, long long ed) {
  __shared__ long long s_ev[kEngThreads / 32], s_ed[kEngThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ev += __shfl_xor_sync(0xffffffffu, ev, o);
    ed += __shfl_xor_sync(0xffffffffu, ed, o);
  }
  if (lane_id() == 0) {
    s_ev[threadIdx.x >> 5] = ev;
    s_ed[threadIdx.x >> 5] = ed;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long tev = 0, ted = 0;
    for (int w = 0; w < kEngThreads / 32; ++w) {
      tev += s_ev[w];
      ted += s_ed[w];
    }
    if (ted) {
      atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 1), (unsigned long long)tev);
      atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 2), (unsigned long long)ted);
    }
  }
}

// Dense delivery of one spike set (single delay bin): a block owns a slice of
// 32 posts (lane = post); its 8 warps split the slice's rows of the sliced
// in-edge view and accumulate, one 32-sample mask word per pass, into
// per-warp shared-memory columns (no conflicts, no atomics); the block then
// sums the 8 partial columns and stores the totals into acc with plain
// stores (acc is zero on entry, each (sample, post) has one writer).  Used
// for steps where most neurons spike in some sample, where per-event
// reductions would cost more than reading every in-edge once.  The spike
// set's masks and flags are then cleared by the last block to finish
// (block-completion counter in ctrl[0]; no block waits for another).
template <int MS>
__device__ void scatter_dense(const bt_engine_desc& d, int64_t k, const ScatterScratch& ws, long long& ev,
                              long long& ed) {
  constexpr int W = kEngThreads / 32;
  __shared__ float s_acc[W][32][32];
  const int lane = int(lane_id()), wid = int(threadIdx.x >> 5);
  const int64_t n = d.n, B = d.batch;
  const int64_t nc = n * n_rec(d);  // acc columns (post * C + r)
  const int n32 = int(nc);
  const int64_t n_slices = (nc + 31) >> 5;
  const int64_t nblocks = int64_t(gridDim.x) * gridDim.y;
  const int64_t bid = int64_t(blockIdx.y) * gridDim.x + blockIdx.x;
  float(*acc)[32] = s_acc[wid];
  const uint64_t pol_stream = l2_evict_first();
  const uint32_t sentinel = uint32_t(n);
  for (int64_t sl = bid; sl < n_slices; sl += nblocks) {  // uniform per block
    const int64_t r0 = d.sl_ptr[sl], r1 = d.sl_ptr[sl + 1];
    const int64_t per = (r1 - r0 + W - 1) / W;
    const int64_t ra = r0 + wid * per, rb = ra + per < r1 ? ra + per : r1;
    for (int w = 0; w < ws.ms; ++w) {
#pragma unroll 8
      for (int l = 0; l < 32; ++l) acc[l][lane] = 0.0f;
      __syncwarp();
      constexpr int U = 8;
      for (int64_t r = ra; r < rb; r += U) {
        uint32_t src[U];
        float wg[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const bool in = r + u < rb;
          src[u] = in ? ld_nc_u32(d.sl_src + (r + u) * 32 + lane, pol_stream) & kIdMask : sentinel;
          wg[u] = in ? ld_nc_f32(d.sl_w + (r + u) * 32 + lane, pol_stream) : 0.0f;
        }
        uint32_t m[U];
#pragma unroll
        for (int u = 0; u < U; ++u) m[u] = src[u] < sentinel ? ws.mask[int64_t(src[u]) * ws.ms + w] : 0u;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (w == 0 && src[u] < sentinel) {
            bool any = m[u] != 0;
            for (int x = 1; x < ws.ms && !any; ++x) any = ws.mask[int64_t(src[u]) * ws.ms + x] != 0;
            ed += any ? 1 : 0;
          }
          ev += __popc(m[u]);
          uint32_t mm = m[u];
          while (mm) {
            const int l = __ffs(mm) - 1;
            mm &= mm - 1;
            acc[l][lane] = add(acc[l][lane], wg[u]);
          }
        }
      }
      __syncthreads();
      for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
        const int l = idx >> 5, ln = idx & 31;
        float sum = 0.0f;
#pragma unroll
        for (int v = 0; v < W; ++v) sum = add(sum, s_acc[v][l][ln]);
        const int64_t b = int64_t(w) * 32 + l, p = sl * 32 + ln;
        if (b < B && p < nc && sum != 0.0f) d.ring[b * n32 + p] = sum;
      }
      __syncthreads();
    }
  }
  // the last block to finish clears the spike set (no other block reads it)
  __shared__ int s_last;
  if (threadIdx.x == 0) {
    __threadfence();
    const int done = atomicAdd(ws.ctrl, 1);
    s_last = done == int(nblocks) - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    for (int64_t i = threadIdx.x; i < n * ws.ms; i += blockDim.x) ws.mask[i] = 0u;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) ws.flag[i] = 0;
    if (threadIdx.x == 0) ws.ctrl[0] = 0;
  }
}

// Grid (x, bin_hi - bin_lo + 1): plane y delivers delay bin d = bin_lo + y,
// i.e. the spike set of step t - d through rows j * R + d.  G lanes share one
// row (G = 32 for long rows, 8 for the short rows of a wide delay range), each
// lane loading 4 edges with one 128-bit load of posts and one of weights, then
// adding them for every sample in the row's mask (MS words; the sample loop is
// outside the edge loop, so a lane issues 4 reductions per mask bit).
// Launch bounds: at least 4 (MS <= 4) or 3 resident blocks per SM, which
// leaves ptxas 64 / 85 registers -- without a bound its occupancy heuristic
// has settled on 48 registers and spilled the reduction loop.
template <int G, int MS>
__global__ void __launch_bounds__(kEngThreads, MS <= 4 ? 4 : 3) k_eng_scatter(bt_engine_desc d, int64_t k, StepIdx si) {
  const int64_t n = d.n;
  const int R = d.n_bins, Q = R + 1;
  const int bin = d.bin_lo + int(blockIdx.y);
  int q = si.q_t - bin;
  if (q < 0) q += Q;
  const ScatterScratch ws = scatter_scratch(d, q);
  __shared__ int32_t s_off[kSub + 1];
  __shared__ int32_t s_spk;
  sub_offsets(ws, s_off, &s_spk);
  const int32_t count = s_off[kSub];
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x < kSub) {
    // the counts of slot (t + 1) mod Q, i.e. of step t - R, were last read by
    // the previous step's scatter: clear them for the next neuron launch
    const int qc = si.q_t + 1 == Q ? 0 : si.q_t + 1;
    d.work[qc * 2 * kSub + threadIdx.x] = 0;
    d.work[qc * 2 * kSub + kSub + threadIdx.x] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && d.stats)
    atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 0), (unsigned long long)count);
  // dense when most neurons spike and they do so in several samples each
  if (d.dense_rows > 0 && count >= d.dense_rows && s_spk >= kDenseSpikesPerRow * count) {  // grid-uniform
    long long ev = 0, ed = 0;
    scatter_dense<MS>(d, k, ws, ev, ed);
    if (d.stats) block_stats(d, k, ev, ed);
    return;
  }
  const bool last_use = bin == d.bin_hi;  // this set is not read again: clear it
  const unsigned lane = lane_id();
  const int grp = int(lane) / G, lig = int(lane) % G;
  constexpr int kPerWarp = 32 / G;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int n32 = int(n * n_rec(d));  // acc row stride; batch * n * C < 2^31 (checked on the host)
  const uint64_t pol_stream = l2_evict_first(), pol_keep = l2_evict_last();
  long long ev = 0, ed = 0;
  for (int64_t base = ((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * kPerWarp; base < count;
       base += warps * kPerWarp) {
    const int64_t it = base + grp;
    uint32_t mw_local[MS];
    int32_t beg = 0, end = 0;
    uint32_t* mrow = nullptr;
    int32_t j = -1;
    if (it < count) {
      const int sub = find_sub(s_off, it);
      j = ws.list[sub * ws.cap + (it - s_off[sub])];
      mrow = ws.mask + int64_t(j) * ws.ms;
      const int64_t row = int64_t(j) * R + bin;
      beg = d.csr_ptr[row];
      end = d.csr_ptr[row + 1];
    }
    // MS is the compile-time bound (1, 2, 4 or 8); the row holds ws.ms words
    // (5..8 samples words above 128 samples run with MS = 8)
    int nsamp = 0;
#pragma unroll
    for (int w = 0; w < MS; ++w) {
      mw_local[w] = (mrow && w < ws.ms) ? mrow[w] : 0u;
      nsamp += __popc(mw_local[w]);
    }
    __syncwarp();
    if (last_use && lig == 0 && j >= 0) {
#pragma unroll
      for (int w = 0; w < MS; ++w)
        if (w < ws.ms) mrow[w] = 0;
      ws.flag[j] = 0;
    }
    if (lig == 0) {
      ev += (long long)nsamp * (end - beg);
      ed += end - beg;
    }
    // U quads per lane in flight: all loads of an iteration are issued before
    // its reductions
    constexpr int U = 2;
    for (int32_t g0 = (beg & ~3) + lig * 4; g0 < end; g0 += G * 4 * U) {
      uint4 dq[U], wq[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int32_t gi = g0 + u * G * 4;
        if (gi < end) {
          // edges gi .. gi+3 as (post, weight) records: two 128-bit loads
          const uint4 a = ld_nc_u4(d.csr_edges + 2 * int64_t(gi), pol_stream);
          const uint4 b = ld_nc_u4(d.csr_edges + 2 * int64_t(gi) + 4, pol_stream);
          dq[u] = make_uint4(a.x, a.z, b.x, b.z);
          wq[u] = make_uint4(a.y, a.w, b.y, b.w);
        } else {
          dq[u] = make_uint4(0u, 0u, 0u, 0u);
          wq[u] = dq[u];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int32_t gidx = g0 + u * G * 4;
        // edges outside [beg, end) of the first and last quad add nothing
        const bool v0 = gidx >= beg && gidx < end, v1 = gidx + 1 >= beg && gidx + 1 < end,
                   v2 = gidx + 2 >= beg && gidx + 2 < end, v3 = gidx + 3 >= beg && gidx + 3 < end;
        const int p0 = int(dq[u].x & kIdMask), p1 = int(dq[u].y & kIdMask), p2 = int(dq[u].z & kIdMask),
                  p3 = int(dq[u].w & kIdMask);
#pragma unroll
        for (int w = 0; w < MS; ++w) {
          uint32_t m = mw_local[w];
          while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            float* row = d.ring + (w * 32 + l) * n32;
            if (v0) red_add_f32(row + p0, __uint_as_float(wq[u].x), pol_keep);
            if (v1) red_add_f32(row + p1, __uint_as_float(wq[u].y), pol_keep);
            if (v2) red_add_f32(row + p2, __uint_as_float(wq[u].z), pol_keep);
            if (v3) red_add_f32(row + p3, __uint_as_float(wq[u].w), pol_keep);
          }
        }
      }
    }
  }
  if (d.stats) block_stats(d, k, ev, ed);
}

// Scatter for short rows (a wide delay range splits each neuron's out-edges
// into n_bins rows): a warp takes 32 rows, one per lane, scans their lengths
// and walks their edges as one flattened range, 32 consecutive edges per
// iteration -- each lane finds its row by a 5-step binary search over the
// lanes' exclusive offsets (shuffles), so no lane idles on a short row and
// consecutive lanes load consecutive edges.  Grid as k_eng_scatter.
template <int MS>
__global__ void __launch_bounds__(kEngThreads, MS <= 4 ? 4 : 3) k_eng_scatter_flat(bt_engine_desc d, int64_t k,
                                                                              StepIdx si) {
  const int R = d.n_bins, Q = R + 1;
  const int bin = d.bin_lo + int(blockIdx.y);
  int q = si.q_t - bin;
  if (q < 0) q += Q;
  const ScatterScratch ws = scatter_scratch(d, q);
  __shared__ int32_t s_off[kSub + 1];
  __shared__ int32_t s_spk;
  sub_offsets(ws, s_off, &s_spk);
  const int32_t count = s_off[kSub];
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x < kSub) {
    const int qc = si.q_t + 1 == Q ? 0 : si.q_t + 1;  // step t - R: last read by the previous step
    d.work[qc * 2 * kSub + threadIdx.x] = 0;
    d.work[qc * 2 * kSub + kSub + threadIdx.x] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && d.stats)
    atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 0), (unsigned long long)count);
  // dense when most neurons spike and they do so in several samples each
  if (d.dense_rows > 0 && count >= d.dense_rows && s_spk >= kDenseSpikesPerRow * count) {  // grid-uniform
    long long ev = 0, ed = 0;
    scatter_dense<MS>(d, k, ws, ev, ed);
    if (d.stats) block_stats(d, k, ev, ed);
    return;
  }
  const bool last_use = bin == d.bin_hi;
  const int lane = int(lane_id());
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int n32 = int(d.n * n_rec(d));  // acc row stride; batch * n * C < 2^31 (checked on the host)
  const uint64_t pol_stream = l2_evict_first(), pol_keep = l2_evict_last();
  long long ev = 0, ed = 0;
  for (int64_t base = ((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * 32; base < count;
       base += warps * 32) {
    const int64_t it = base + lane;
    uint32_t mw[MS];
    int32_t beg = 0, len = 0;
    if (it < count) {
      const int sub = find_sub(s_off, it);
      const int32_t j = ws.list[sub * ws.cap + (it - s_off[sub])];
      uint32_t* mrow = ws.mask + int64_t(j) * ws.ms;
      const int64_t row = int64_t(j) * R + bin;
      beg = d.csr_ptr[row];
      len = d.csr_ptr[row + 1] - beg;
      int nsamp = 0;
#pragma unroll
      for (int w = 0; w < MS; ++w) {
        mw[w] = w < ws.ms ? mrow[w] : 0u;
        nsamp += __popc(mw[w]);
      }
      if (last_use) {
#pragma unroll
        for (int w = 0; w < MS; ++w)
          if (w < ws.ms) mrow[w] = 0;
        ws.flag[j] = 0;
      }
      ev += (long long)nsamp * len;
      ed += len;
    } else {
#pragma unroll
      for (int w = 0; w < MS; ++w) mw[w] = 0u;
    }
    // exclusive offsets of the 32 rows in the flattened edge range
    int32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int32_t excl = incl - len;
    const int32_t total = __shfl_sync(0xffffffffu, incl, 31);
    // U edges per lane in flight: the row searches and loads of an iteration
    // come before its reductions
    constexpr int U = 4;
    for (int32_t e0 = 0; e0 < total; e0 += 32 * U) {
      int pp[U];
      float wv[U];
      uint32_t mm[U][MS];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int32_t e = e0 + u * 32 + lane;
        // r = the last lane whose excl <= e (rows of length 0 are skipped over)
        int r = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int32_t x = __shfl_sync(0xffffffffu, excl, r + step);
          if (x <= e) r += step;
        }
        const int32_t rbeg = __shfl_sync(0xffffffffu, beg, r);
        const int32_t rexcl = __shfl_sync(0xffffffffu, excl, r);
#pragma unroll
        for (int w = 0; w < MS; ++w) mm[u][w] = __shfl_sync(0xffffffffu, mw[w], r);
        pp[u] = 0;
        wv[u] = 0.0f;
        if (e < total) {
          const int32_t g = rbeg + (e - rexcl);
          const uint2 e = ld_nc_u2(d.csr_edges + 2 * int64_t(g), pol_stream);
          pp[u] = int(e.x & kIdMask);
          wv[u] = __uint_as_float(e.y);
        } else {
#pragma unroll
          for (int w = 0; w < MS; ++w) mm[u][w] = 0u;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int w = 0; w < MS; ++w) {
          uint32_t m = mm[u][w];
          while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            red_add_f32(d.ring + (w * 32 + l) * n32 + pp[u], wv[u], pol_keep);
          }
        }
      }
    }
  }
  if (d.stats) block_stats(d, k, ev, ed);
}

// psc_{t_end-1} = stored + acc; clears acc.
__global__ void k_eng_scatter_final(bt_engine_desc d) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nc = d.n * n_rec(d), B = d.batch;  // one thread per PSC column
  if (idx >= B * nc) return;
  // all loads before the first store (see k_eng_neuron_rec)
  float* __restrict__ ring = d.ring;
  float* __restrict__ psc = d.psc;
  const float pending = ring[idx];
  const float stored = psc[idx];
  const int64_t b = idx / nc;
  const int64_t len = d.sample_len ? d.sample_len[b] : INT64_MAX;
  ring[idx] = 0.0f;
  const float P = d.n_steps - 1 < len ? add(stored, pending) : stored;
  if (d.n_steps - 1 < len) psc[idx] = P;
  if (d.psc_trace) d.psc_trace[((d.n_steps - 1) * B) * nc + idx] = P;
}

// ----------------------------------------------------------------- gather --

// Ordered in-edge gather of W z for (b, i) at arrival step `ta`:
// sum over in-edges (pre, bin) ascending of w * z_{ta - bin}[pre].
__device__ __forceinline__ float gather_in(const bt_engine_desc& d, int64_t i, int64_t b, int ta_mod_h, int64_t words) {
  const unsigned lane = lane_id();
  const int32_t beg = __ldg(d.csc_ptr + i), end = __ldg(d.csc_ptr + i + 1);
  const int H = d.hist_len;  // slot of bin b is ta_mod_h - b (mod H), b < H
  float acc = 0.0f;
  for (int32_t base = beg; base < end; base += 32) {
    const int32_t e = base + int32_t(lane);
    float w = 0.0f;
    bool act = false;
    if (e < end) {
      const uint32_t src = __ldg(d.csc_src + e);
      const uint32_t pre = src & kIdMask;
      int slot = ta_mod_h - int(src >> BT_BIN_SHIFT);
      if (slot < 0) slot += H;
      const uint32_t word = d.hist[(int64_t(slot) * d.batch + b) * words + (pre >> 5)];
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
// REC: receptor channels, the warp gathers the C columns i * C + r in turn.
template <int KIND, bool HARD, bool USE_REF, bool REC>
__global__ void __launch_bounds__(1024) k_eng_gather(bt_engine_desc d, int64_t k, StepIdx si) {
  extern __shared__ uint32_t sbits[];  // [batch]
  const int64_t n = d.n, B = d.batch;
  const int64_t words = (n + 31) >> 5;
  const int wid = threadIdx.x >> 5;
  const unsigned lane = lane_id();
  const int64_t i = int64_t(blockIdx.x) * 32 + wid;
  for (int64_t b = threadIdx.x; b < B; b += blockDim.x) sbits[b] = 0;
  __syncthreads();
  int nspk = 0;
  if (i < n) {
    for (int64_t b = 0; b < B; ++b) {
      const int64_t idx = b * n + i;
      const int64_t len = d.sample_len ? d.sample_len[b] : INT64_MAX;
      // synapse update of step t-1 (skipped on the first step of a call: the
      // stored psc already is psc_{t0-1}; skipped after a sample's last step)
      const bool syn = k > 0 && k - 1 < len;
      float P;
      float Pr[REC ? kMaxRec : 1];
      const int C = REC ? d.n_rec : 1;
      const int64_t c0 = (b * n + i) * C;  // first PSC column of (b, i)
      if constexpr (!REC) {
        P = d.psc[idx];
        if (syn) P = add(psc_decay(d.psc_coef, d.psc_tau, i, P), gather_in(d, i, b, si.h_prev, words));
      } else {
        for (int r = 0; r < C; ++r) {
          float q = d.psc[c0 + r];
          if (syn) q = add(psc_decay(d.psc_coef, d.psc_tau, i * C + r, q), gather_in(d, i * C + r, b, si.h_prev, words));
          Pr[r] = q;
        }
        P = receptor_sum(Pr, C);
      }
      float s = 0.0f;
      if (lane == 0) {
        if (k < len) {
          const float I = d.x ? add(P, d.x[(k * B) * n + idx]) : P;
          float v = d.v[idx];
          float ref = USE_REF ? d.refractory[idx] : 0.0f;
          float gk = KIND == BT_NEURON_ALIF ? d.g_k[idx] : 0.0f;
          const NeuronParams prm = load_params<KIND, USE_REF>(d.neuron, i);
          const NeuronOut o = neuron_update<KIND, HARD, USE_REF, true>(prm, I, v, ref, gk);
          s = o.spike;
          d.v[idx] = v;
          if (USE_REF) d.refractory[idx] = ref;
          if (KIND == BT_NEURON_ALIF) d.g_k[idx] = gk;
        }
        if constexpr (!REC) {
          d.psc[idx] = P;
          if (d.psc_trace && k > 0) d.psc_trace[((k - 1) * B) * n + idx] = P;
        } else {
          for (int r = 0; r < C; ++r) {
            d.psc[c0 + r] = Pr[r];
            if (d.psc_trace && k > 0) d.psc_trace[((k - 1) * B) * n * C + c0 + r] = Pr[r];
          }
        }
        if (d.v_trace) d.v_trace[(k * B) * n + idx] = d.v[idx];
        if (USE_REF && d.ref_trace) d.ref_trace[(k * B) * n + idx] = d.refractory[idx];
        if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[(k * B) * n + idx] = d.g_k[idx];
        if (d.spikes) d.spikes[(k * B) * n + idx] = s;
        if (s != 0.0f) {
          atomicOr(&sbits[b], 1u << (i & 31));
          ++nspk;
        }
      }
    }
  }
  __shared__ long long s_stat[32][3];  // per warp: union, events, edges
  if (d.stats && lane == 0) {
    const long long deg = (i < n && nspk && d.outdeg) ? d.outdeg[i] : 0;
    s_stat[wid][0] = nspk ? 1 : 0;
    s_stat[wid][1] = nspk * deg;
    s_stat[wid][2] = nspk ? deg : 0;
  }
  __syncthreads();
  if (d.stats && threadIdx.x < 3) {
    // one atomic per block and counter (same-address atomics serialise in L2)
    long long tot = 0;
    for (int q = 0; q < 32; ++q) tot += s_stat[q][threadIdx.x];
    if (tot) atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + threadIdx.x), (unsigned long long)tot);
  }
  const int64_t w = int64_t(blockIdx.x);
  for (int64_t b = threadIdx.x; b < B; b += blockDim.x) {
    d.hist[(int64_t(si.h_t) * B + b) * words + w] = sbits[b];
    if (d.raster) d.raster[(k * B + b) * words + w] = sbits[b];
  }
}

// Synapse update of the last step of a call: psc_{t_end-1}.
__global__ void __launch_bounds__(1024) k_eng_gather_final(bt_engine_desc d, StepIdx si) {
  const int64_t n = d.n, B = d.batch;
  const int64_t words = (n + 31) >> 5;
  const int64_t k = d.n_steps - 1;
  const int64_t i = int64_t(blockIdx.x) * 32 + (threadIdx.x >> 5);
  if (i >= n) return;
  const int C = n_rec(d);
  const int64_t nc = n * C;
  for (int64_t b = 0; b < B; ++b) {
    const int64_t len = d.sample_len ? d.sample_len[b] : INT64_MAX;
    for (int r = 0; r < C; ++r) {
      const int64_t col = i * C + r, idx = b * nc + col;  // PSC column
      if (k >= len) {
        if (lane_id() == 0 && d.psc_trace) d.psc_trace[(k * B) * nc + idx] = d.psc[idx];
        continue;
      }
      const float wz = gather_in(d, col, b, si.h_t, words);
      if (lane_id() == 0) {
        const float P = add(psc_decay(d.psc_coef, d.psc_tau, col, d.psc[idx]), wz);
        d.psc[idx] = P;
        if (d.psc_trace) d.psc_trace[(k * B) * nc + idx] = P;
      }
    }
  }
}

// ------------------------------------------------------------ sliced pull --
//
// PULL mode, one launch per step for batched runs.  Warp = (slice of 32 posts,
// 32-sample word q); lane = post.  The warp walks the slice's SELL-32 rows
// (each post's in-edges in canonical order down its lane), looks up the
// presynaptic neuron's sample mask for the step the edge's delay bin points
// at, and adds w into acc[sample][lane] in shared memory -- conflict-free and
// in ascending in-edge order for every (sample, post), i.e. the reference's
// fma chain (acc + w == fma(w, 1, acc)).  Then each lane runs the neuron
// update of its post for the warp's 32 samples and publishes its new mask.
constexpr int kPullWarps = 8;
constexpr int kPullUnroll = 8;

template <int MW>
struct MaskVec;
template <>
struct MaskVec<1> {
  using T = uint32_t;
  __device__ static void split(T v, uint32_t* m) { m[0] = v; }
};
template <>
struct MaskVec<2> {
  using T = uint2;
  __device__ static void split(T v, uint32_t* m) { m[0] = v.x; m[1] = v.y; }
};
template <>
struct MaskVec<4> {
  using T = uint4;
  __device__ static void split(T v, uint32_t* m) { m[0] = v.x; m[1] = v.y; m[2] = v.z; m[3] = v.w; }
};

// MW: sample words a warp covers (1, 2 or 4 -> batch up to 32, 64, 128).  For
// larger batches MW = 1 and the grid has one warp per (slice, word): `split`.
template <int KIND, bool HARD, bool USE_REF, bool FINAL, int MW>
__global__ void __launch_bounds__(kPullWarps * 32, 3) k_eng_pull(bt_engine_desc d, int64_t k, int split, StepIdx si) {
  extern __shared__ float acc_dyn[];  // [kPullWarps][MW * 32][32]
  const int wid = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t n = d.n, B = d.batch;
  const int mw_all = mask_stride(B);
  const int64_t n_slices = (n + 31) >> 5;
  const int64_t gw = int64_t(blockIdx.x) * kPullWarps + wid;
  const int64_t sl = split ? gw / mw_all : gw;
  const int q0 = split ? int(gw % mw_all) : 0;  // first sample word of this warp
  if (sl >= n_slices) return;  // warp-uniform; the kernel has no block barrier
  const int64_t p = sl * 32 + lane;
  const bool valid = p < n;
  const int H = d.hist_len;
  // history slot of the arrival step whose PSC this launch completes
  const int ta_mod_h = FINAL ? si.h_t : si.h_prev;
  const bool gather = FINAL || k > 0;
  float(*acc)[32] = reinterpret_cast<float(*)[32]>(acc_dyn + wid * (MW * 32 * 32));
  using V = typename MaskVec<MW>::T;
  const int64_t row_stride = int64_t(n + 1) * mw_all;  // words per history slot
  if (gather) {
#pragma unroll 8
    for (int l = 0; l < MW * 32; ++l) acc[l][lane] = 0.0f;
    __syncwarp();
    const int64_t r0 = d.sl_ptr[sl], r1 = d.sl_ptr[sl + 1];
    const uint32_t sentinel = uint32_t(n);
    for (int64_t r = r0; r < r1; r += kPullUnroll) {
      uint32_t src[kPullUnroll];
      float w[kPullUnroll];
      V mv[kPullUnroll];
#pragma unroll
      for (int u = 0; u < kPullUnroll; ++u) {
        const bool in = r + u < r1;
        src[u] = in ? __ldg(d.sl_src + (r + u) * 32 + lane) : sentinel;
        w[u] = in ? __ldg(d.sl_w + (r + u) * 32 + lane) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kPullUnroll; ++u) {
        int slot = ta_mod_h - int(src[u] >> BT_BIN_SHIFT);
        if (slot < 0) slot += H;
        const uint32_t* mrow = d.masks + slot * row_stride + int64_t(src[u] & kIdMask) * mw_all + q0;
        mv[u] = __ldg(reinterpret_cast<const V*>(mrow));
      }
#pragma unroll
      for (int u = 0; u < kPullUnroll; ++u) {
        uint32_t m[MW];
        MaskVec<MW>::split(mv[u], m);
#pragma unroll
        for (int q = 0; q < MW; ++q) {
          uint32_t mm = m[q];
          while (mm) {
            const int l = __ffs(mm) - 1;
            mm &= mm - 1;
            acc[q * 32 + l][lane] = add(acc[q * 32 + l][lane], w[u]);
          }
        }
      }
    }
    __syncwarp();
  }
  const int64_t words = n_slices;
  uint32_t my_mask[MW];
#pragma unroll
  for (int q = 0; q < MW; ++q) my_mask[q] = 0;
  constexpr int U = 4;
  const float* __restrict__ xk = d.x ? d.x + (k * B) * n : nullptr;
  const NeuronParams prm = load_params<KIND, USE_REF>(d.neuron, valid ? p : 0);
  const float pc = ld(d.psc_coef, valid ? p : 0), pt = ld(d.psc_tau, valid ? p : 0), rpt = pow2_recip(pt);
#pragma unroll
  for (int q = 0; q < MW; ++q) {
    for (int l0 = 0; l0 < 32; l0 += U) {
      const int64_t b0 = int64_t(q0 + q) * 32 + l0;
      if (b0 >= B) break;  // warp-uniform
      // load phase: U samples' state at once (independent loads in flight)
      float pv[U], xv[U], vv[U], rv[U], gv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t b = b0 + u;
        const bool in = valid && b < B;
        const int64_t idx = b * n + p;
        pv[u] = in ? d.psc[idx] : 0.0f;
        xv[u] = (in && xk && !FINAL) ? xk[idx] : 0.0f;
        vv[u] = (in && !FINAL) ? d.v[idx] : 0.0f;
        rv[u] = (in && USE_REF && !FINAL) ? d.refractory[idx] : 0.0f;
        gv[u] = (in && KIND == BT_NEURON_ALIF && !FINAL) ? d.g_k[idx] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t b = b0 + u;
        if (b >= B) break;  // warp-uniform
        const int l = l0 + u;
        float spk = 0.0f;
        if (valid) {
          const int64_t idx = b * n + p;
          const int64_t len = d.sample_len ? d.sample_len[b] : INT64_MAX;
          float P = pv[u];
          const bool syn_live = FINAL ? (k < len) : (k - 1 < len);
          if (gather && syn_live) P = add(psc_decay(pc, pt, rpt, P), acc[q * 32 + l][lane]);
          if (FINAL) {
            d.psc[idx] = P;
            if (d.psc_trace) d.psc_trace[(k * B) * n + idx] = P;
            continue;
          }
          float v = vv[u], ref = rv[u], gk = gv[u];
          if (k < len) {
            const float I = xk ? add(P, xv[u]) : P;
            const NeuronOut o = neuron_update<KIND, HARD, USE_REF, true>(prm, I, v, ref, gk);
            spk = o.spike;
            d.v[idx] = v;
            if (USE_REF) d.refractory[idx] = ref;
            if (KIND == BT_NEURON_ALIF) d.g_k[idx] = gk;
          }
          d.psc[idx] = P;
          if (d.v_trace) d.v_trace[(k * B) * n + idx] = v;
          if (USE_REF && d.ref_trace) d.ref_trace[(k * B) * n + idx] = ref;
          if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[(k * B) * n + idx] = gk;
          if (d.psc_trace && k > 0) d.psc_trace[((k - 1) * B) * n + idx] = P;
          if (d.spikes) d.spikes[(k * B) * n + idx] = spk;
        }
        if (!FINAL) {
          const uint32_t word = __ballot_sync(0xffffffffu, spk != 0.0f);
          if (lane == 0 && d.raster) d.raster[(k * B + b) * words + sl] = word;
          if (spk != 0.0f) my_mask[q] |= 1u << l;
        }
      }
    }
  }
  if (FINAL) return;
  if (valid) {
    uint32_t* mrow = d.masks + int64_t(si.h_t) * row_stride + p * mw_all + q0;
#pragma unroll
    for (int q = 0; q < MW; ++q) mrow[q] = my_mask[q];
  }
  if (d.stats) {
    // events = spikes x out-degree; union counted by the warp that owns word 0
    int nspk = 0;
#pragma unroll
    for (int q = 0; q < MW; ++q) nspk += __popc(my_mask[q]);
    const int deg = (valid && d.outdeg) ? d.outdeg[p] : 0;
    long long ev = (long long)nspk * deg;
    long long ed = (!split && nspk) ? deg : 0;
    long long un = (!split && nspk) ? 1 : 0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      ev += __shfl_xor_sync(0xffffffffu, ev, off);
      ed += __shfl_xor_sync(0xffffffffu, ed, off);
      un += __shfl_xor_sync(0xffffffffu, un, off);
    }
    if (lane == 0) {
      if (ev) atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 1), (unsigned long long)ev);
      if (ed) atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 2), (unsigned long long)ed);
      if (un) atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 0), (unsigned long long)un);
    }
  }
}

// masks[i][q] bit l  <=>  in[(32 q + l) * n + i] != 0   (sample-minor from [B][n]).
__global__ void k_float_to_masks(int64_t batch, int64_t n, const float* __restrict__ in, uint32_t* __restrict__ masks) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int mw = mask_stride(batch);
  if (idx >= n * mw) return;
  const int64_t i = idx / mw;
  const int q = int(idx % mw);
  uint32_t m = 0;
  for (int l = 0; l < 32 && int64_t(q) * 32 + l < batch; ++l)
    if (in[(int64_t(q) * 32 + l) * n + i] != 0.0f) m |= 1u << l;
  masks[idx] = m;
}

__global__ void k_masks_to_float(int64_t batch, int64_t n, const uint32_t* __restrict__ masks, float* __restrict__ out) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= batch * n) return;
  const int64_t b = idx / n, i = idx % n;
  const int mw = mask_stride(batch);
  out[idx] = float((masks[i * mw + (b >> 5)] >> (b & 31)) & 1u);
}

// ---------------------------------------------------------- run priming --

// One thread per (steps ago a in 1..bin_hi, neuron i): the spike set of step
// t0 - a rebuilt from the history bitmaps -- the mask of samples in which i
// spiked, and i listed once if any did (warp-aggregated atomic).  Rows are
// padded to whole 32-neuron words, so every warp has a single a.
__global__ void k_prime_history(bt_engine_desc d) {
  const int64_t n = d.n, B = d.batch;
  const int64_t words = (n + 31) >> 5;
  const int64_t npad = words * 32;
  const int64_t gid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t a = 1 + gid / npad;
  const int64_t i = gid - (a - 1) * npad;
  if (a > d.bin_hi) return;  // whole warps
  const int64_t s = d.t0 - a;  // >= 0: t0 >= hist_len > n_bins > bin_hi
  const int64_t hs = s % d.hist_len;
  const int q = int(s % (d.n_bins + 1));
  const ScatterScratch ws = scatter_scratch(d, q);
  uint32_t mw[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  bool any = false;
  if (i < n) {
    const uint32_t* h = d.hist + hs * B * words + (i >> 5);
    for (int64_t b = 0; b < B; ++b) {
      if ((h[b * words] >> (i & 31)) & 1u) {
        mw[b >> 5] |= 1u << (b & 31);
        any = true;
      }
    }
    if (any) {
#pragma unroll
      for (int w = 0; w < 8; ++w)
        if (w < ws.ms) ws.mask[i * ws.ms + w] = mw[w];
      ws.flag[i] = 1;
    }
  }
  const unsigned lane = lane_id();
  const uint32_t fb = __ballot_sync(0xffffffffu, any);
  if (fb == 0) return;
  const int sub = int((i - lane) >> ws.cap_shift);
  int32_t base = 0;
  if (lane == 0) base = atomicAdd(ws.count + sub, __popc(fb));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (any) ws.list[sub * ws.cap + base + __popc(fb & ((1u << lane) - 1u))] = int32_t(i);
}

// ------------------------------------------------------- input projection --

// Per row r: its nonzero inputs as (channel, value) pairs in ascending channel
// order (warp ballot + prefix), and their count.  With live_len, row
// r = t * batch + b of a sample past its length (t >= live_len[b]) gets
// count -1 and no pairs: nothing reads its projection.
__global__ void k_row_pairs(int64_t rows, int64_t c_in, const float* __restrict__ xin, int32_t* __restrict__ cnt,
                            int2* __restrict__ pairs, const int32_t* __restrict__ live_len, int64_t batch) {
  const int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (r >= rows) return;
  const unsigned lane = lane_id();
  if (live_len && r / batch >= __ldg(live_len + r % batch)) {  // warp-uniform
    if (lane == 0) cnt[r] = -1;
    return;
  }
  int32_t total = 0;
  for (int64_t c0 = 0; c0 < c_in; c0 += 32) {
    const int64_t c = c0 + lane;
    const float v = c < c_in ? xin[r * c_in + c] : 0.0f;
    const bool nz = v != 0.0f;
    const uint32_t m = __ballot_sync(0xffffffffu, nz);
    if (nz) pairs[r * c_in + total + __popc(m & ((1u << lane) - 1u))] = make_int2(int(c), __float_as_int(v));
    total += __popc(m);
  }
  if (lane == 0) cnt[r] = total;
}

// out[r][i] = sum over the row's pairs (ascending channel) of v * w_t[c][i],
// as an fmaf chain (+ bias).  Each thread owns kProjNPT neurons spaced by the
// block size, so one broadcast pair load feeds kProjNPT coalesced weight loads
// and fmas.  grid.x walks row blocks fastest: the resident blocks then share a
// narrow column slice of w_t, which stays in L2.
constexpr int kProjRows = 8;
constexpr int kProjNPT = 4;
__global__ void __launch_bounds__(256) k_input_project(int64_t rows, int64_t c_in, int64_t n,
                                                       const float* __restrict__ w_t,
                                                       const float* __restrict__ bias,
                                                       const int32_t* __restrict__ cnt,
                                                       const int2* __restrict__ pairs, float* __restrict__ out) {
  const int64_t tile = int64_t(blockIdx.y) * (256 * kProjNPT);
  const int64_t r0 = int64_t(blockIdx.x) * kProjRows;
  int64_t ii[kProjNPT];
  bool ok[kProjNPT];
#pragma unroll
  for (int j = 0; j < kProjNPT; ++j) {
    ii[j] = tile + threadIdx.x + j * 256;
    ok[j] = ii[j] < n;
  }
  for (int64_t r = r0; r < r0 + kProjRows && r < rows; ++r) {
    const int32_t c_n = cnt[r];
    if (c_n < 0) continue;  // a finished sample's step: left unwritten
    const int2* rp = pairs + r * c_in;
    float acc[kProjNPT];
#pragma unroll
    for (int j = 0; j < kProjNPT; ++j) acc[j] = 0.0f;
    for (int32_t q = 0; q < c_n; ++q) {
      const int2 pr = __ldg(rp + q);
      const float v = __int_as_float(pr.y);
      const float* wr = w_t + int64_t(pr.x) * n;
#pragma unroll
      for (int j = 0; j < kProjNPT; ++j)
        if (ok[j]) acc[j] = fmaf(v, __ldg(wr + ii[j]), acc[j]);
    }
#pragma unroll
    for (int j = 0; j < kProjNPT; ++j)
      if (ok[j]) out[r * n + ii[j]] = bias ? add(acc[j], bias[ii[j]]) : acc[j];
  }
}

// Per channel c, the rows r (ascending) whose input x[r][c] is nonzero, and
// their count: one warp per channel (ballot + prefix keeps the order).
__global__ void k_channel_rows(int64_t rows, int64_t c_in, const float* __restrict__ x, int32_t* __restrict__ lists,
                               int32_t* __restrict__ counts) {
  const int64_t c = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (c >= c_in) return;
  const unsigned lane = lane_id();
  int32_t total = 0;
  for (int64_t r0 = 0; r0 < rows; r0 += 32) {
    const int64_t r = r0 + lane;
    const bool nz = r < rows && x[r * c_in + c] != 0.0f;
    const uint32_t m = __ballot_sync(0xffffffffu, nz);
    if (nz) lists[c * rows + total + __popc(m & ((1u << lane) - 1u))] = int32_t(r);
    total += __popc(m);
  }
  if (lane == 0) counts[c] = total;
}

// Gradient of the input layer's weight (w_t [c_in][n]) from the gradient of
// its projection g [rows][n]: out[c][i] = sum over the rows r of channel c
// (ascending) of x[r][c] * g[r][i] -- an fmaf chain over the nonzero inputs
// only; accumulate adds it to out.  Block = (channel, 1024 columns), each
// thread kProjNPT columns spaced by the block size (coalesced rows of g).
__global__ void __launch_bounds__(256) k_input_grad_weight(int64_t rows, int64_t c_in, int64_t n,
                                                           const float* __restrict__ x, const float* __restrict__ g,
                                                           const int32_t* __restrict__ lists,
                                                           const int32_t* __restrict__ counts,
                                                           float* __restrict__ out, int accumulate) {
  const int64_t c = blockIdx.x;
  const int64_t tile = int64_t(blockIdx.y) * (256 * kProjNPT);
  const int32_t cnt = counts[c];
  const int32_t* rl = lists + c * rows;
  float acc[kProjNPT];
#pragma unroll
  for (int j = 0; j < kProjNPT; ++j) acc[j] = 0.0f;
  for (int32_t q = 0; q < cnt; ++q) {
    const int64_t r = __ldg(rl + q);
    const float xv = __ldg(x + r * c_in + c);
    const float* gr = g + r * n;
#pragma unroll
    for (int j = 0; j < kProjNPT; ++j) {
      const int64_t i = tile + threadIdx.x + j * 256;
      if (i < n) acc[j] = fmaf(xv, __ldg(gr + i), acc[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < kProjNPT; ++j) {
    const int64_t i = tile + threadIdx.x + j * 256;
    if (i < n) out[c * n + i] = accumulate ? add(out[c * n + i], acc[j]) : acc[j];
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

namespace bt {
int run_tile(const bt_engine_desc& d, bool fast, cudaStream_t s);     // tile.cu
int run_cluster(const bt_engine_desc& d, bool fast, cudaStream_t s);  // cluster.cu
}

namespace {

int engine_check(const bt_engine_desc* d) {
  if (!d) return bt_set_error(BT_ERR_INVALID, "null engine descriptor");
  if (int st = bt_check_neuron_desc(&d->neuron)) return st;
  BT_CHECK_ARG(d->n > 0 && d->n < BT_MAX_NEURONS, "n=%lld outside (0, 2^25)", (long long)d->n);
  BT_CHECK_ARG(d->batch > 0 && d->batch * d->n < (int64_t(1) << 40), "bad batch");
  BT_CHECK_ARG(d->n_bins >= 1 && d->n_bins <= BT_MAX_BINS, "n_bins=%d outside [1, 128]", d->n_bins);
  BT_CHECK_ARG(d->hist_len >= d->n_bins + 2, "hist_len=%d must be >= n_bins + 2", d->hist_len);
  BT_CHECK_ARG(d->n_steps >= 0 && d->t0 >= 0, "negative step index");
  BT_CHECK_ARG(d->n_steps < (int64_t(1) << 31), "n_steps must be below 2^31");
  BT_CHECK_ARG(d->mode == BT_MODE_SCATTER || d->mode == BT_MODE_GATHER || d->mode == BT_MODE_PULL ||
                   d->mode == BT_MODE_TILE || d->mode == BT_MODE_CLUSTER,
               "mode=%d", d->mode);
  BT_CHECK_ARG(d->v && d->psc && d->hist, "state pointer missing (v / psc / hist)");
  BT_CHECK_ARG(!d->neuron.use_refractory || d->refractory, "refractory state missing");
  BT_CHECK_ARG(d->neuron.kind != BT_NEURON_ALIF || d->g_k, "g_k state missing");
  BT_CHECK_ARG(d->psc_coef.ptr && d->psc_tau.ptr, "PSC coefficients missing");
  BT_CHECK_ARG(d->neuron.spiking, "the fused engine needs a spiking (Heaviside) forward");
  BT_CHECK_ARG(d->n_rec >= 0 && d->n_rec <= kMaxRec, "n_rec=%d outside [0, %d]", d->n_rec, kMaxRec);
  BT_CHECK_ARG(d->n * n_rec(*d) < BT_MAX_NEURONS, "n * n_rec must be < 2^25");
  BT_CHECK_ARG(n_rec(*d) == 1 || d->mode != BT_MODE_PULL, "pull mode has no receptor channels");
  if (d->mode == BT_MODE_SCATTER) {
    BT_CHECK_ARG(d->csr_ptr && d->csr_edges && d->ring && d->work, "scatter needs CSR, ring and work");
    BT_CHECK_ARG((reinterpret_cast<uintptr_t>(d->csr_edges) & 15) == 0, "csr_edges must be 16-byte aligned");
    BT_CHECK_ARG(d->bin_lo >= 0 && d->bin_lo <= d->bin_hi && d->bin_hi < d->n_bins, "bins [%d, %d] outside [0, %d)",
                 d->bin_lo, d->bin_hi, d->n_bins);
    BT_CHECK_ARG(d->scatter_lanes == 0 || d->scatter_lanes == 1 || d->scatter_lanes == 8 || d->scatter_lanes == 32,
                 "scatter_lanes=%d (0, 1, 8 or 32)", d->scatter_lanes);
    BT_CHECK_ARG(mask_stride(d->batch) <= 8, "scatter mode supports up to 256 samples");
    BT_CHECK_ARG(d->batch * d->n * n_rec(*d) < (int64_t(1) << 31), "scatter mode needs batch * n * n_rec < 2^31");
    BT_CHECK_ARG(d->dense_rows == 0 || (d->bin_lo == d->bin_hi && d->sl_ptr && d->sl_src && d->sl_w),
                 "dense delivery needs a single delay bin and the sliced in-edge view");
    BT_CHECK_ARG(d->neuron_spt == 0 || d->neuron_spt == 1 || d->neuron_spt == 2 || d->neuron_spt == 4,
                 "neuron_spt=%d (0, 1, 2 or 4)", d->neuron_spt);
  } else if (d->mode == BT_MODE_TILE) {
    BT_CHECK_ARG(d->csr_ptr && d->csr_edges && d->ring && d->tile_off && d->tile_work,
                 "tile mode needs CSR, ring, tile offsets and tile work");
    BT_CHECK_ARG((reinterpret_cast<uintptr_t>(d->tile_work) & 63) == 0, "tile_work must be 64-byte aligned");
    BT_CHECK_ARG((reinterpret_cast<uintptr_t>(d->csr_edges) & 15) == 0, "csr_edges must be 16-byte aligned");
    BT_CHECK_ARG(d->n_bins == 1 && d->bin_lo == 0 && d->bin_hi == 0, "tile mode has no synaptic delays");
    BT_CHECK_ARG(n_rec(*d) == 1, "tile mode has no receptor channels");
    BT_CHECK_ARG(d->tile_posts > 0 && (d->tile_posts & 31) == 0, "tile_posts=%d must be a positive multiple of 32",
                 d->tile_posts);
    BT_CHECK_ARG(d->n_tiles > 0 && int64_t(d->n_tiles) * d->tile_posts >= d->n &&
                     int64_t(d->n_tiles - 1) * d->tile_posts < d->n,
                 "n_tiles=%d x tile_posts=%d does not tile n=%lld", d->n_tiles, d->tile_posts, (long long)d->n);
    BT_CHECK_ARG(d->batch <= 256 && d->batch * d->n < (int64_t(1) << 31), "tile mode: batch <= 256, batch * n < 2^31");
  } else if (d->mode == BT_MODE_CLUSTER) {
    BT_CHECK_ARG(d->cl_w && d->cl_src && d->cl_gptr, "cluster mode needs the packed in-edges cl_w / cl_src / cl_gptr");
    BT_CHECK_ARG(((reinterpret_cast<uintptr_t>(d->cl_w) | reinterpret_cast<uintptr_t>(d->cl_src)) & 15) == 0,
                 "cl_w and cl_src must be 16-byte aligned (bulk copies)");
    BT_CHECK_ARG(d->n_bins >= 1 && d->n_bins <= 32 && (d->n_bins == 1 || d->n + 32 <= (int64_t(1) << 20)),
                 "cluster mode: n_bins=%d (1..32; with delays n + 32 <= 2^20)", d->n_bins);
    BT_CHECK_ARG(d->tile_rows >= 0 && d->tile_rows % 16 == 0 && d->tile_rows < (int64_t(1) << 24),
                 "tile_rows=%lld must be a multiple of 16", (long long)d->tile_rows);
    BT_CHECK_ARG(n_rec(*d) == 1, "cluster mode has no receptor channels");
    BT_CHECK_ARG(d->tile_posts > 0 && (d->tile_posts & 31) == 0, "tile_posts=%d must be a positive multiple of 32",
                 d->tile_posts);
    BT_CHECK_ARG(d->n_tiles >= 1 && d->n_tiles <= 16 && int64_t(d->n_tiles) * d->tile_posts >= d->n &&
                     int64_t(d->n_tiles - 1) * d->tile_posts < d->n,
                 "n_tiles=%d (1..16) x tile_posts=%d does not tile n=%lld", d->n_tiles, d->tile_posts,
                 (long long)d->n);
    BT_CHECK_ARG(d->batch <= 256 && d->batch * d->n < (int64_t(1) << 31), "cluster mode: batch <= 256");
  } else if (d->mode == BT_MODE_GATHER) {
    BT_CHECK_ARG(d->csc_ptr && d->csc_src && d->csc_w, "gather needs CSC");
  } else {
    BT_CHECK_ARG(d->sl_ptr && d->sl_src && d->sl_w && d->masks, "pull needs the sliced layout and masks");
  }
  return BT_OK;
}

// The device's Div kind of divisor c (neuron.cuh make_div) is 1 or 2.
bool fast_divisor(float c, bool verified) {
  uint32_t u;
  std::memcpy(&u, &c, sizeof(u));
  const uint32_t e = u >> 23;
  return ((u & 0x7fffffu) == 0u && e >= 1u && e <= 253u) || verified;
}

// Uniform scalar parameters whose divisions all avoid the IEEE path.
bool fast_divisors(const bt_engine_desc& d, int kind) {
  const bt_neuron_desc& nd = d.neuron;
  if (!nd.uniform || !d.psc_uniform) return false;
  const float den = nd.sv[0] - nd.sv[1];  // v_threshold - v_reset, as the device computes it
  bool ok = fast_divisor(nd.sv[2], nd.fast_div & 1) && fast_divisor(den, nd.fast_div & 2) &&
            fast_divisor(d.psc_tau_s, d.psc_fast_div != 0);
  ok = ok && (kind == BT_NEURON_LIF ? fast_divisor(nd.sv[3], nd.fast_div & 4) : fast_divisor(nd.sv[9], nd.fast_div & 8));
  return ok;
}

template <int KIND, bool HARD, bool USE_REF>
int run_typed(const bt_engine_desc& d, cudaStream_t s) {
  const int64_t n = d.n;
  if (d.mode == BT_MODE_CLUSTER) return run_cluster(d, fast_divisors(d, KIND), s);  // no final launch
  if (d.mode == BT_MODE_TILE) {
    if (int st = run_tile(d, fast_divisors(d, KIND), s)) return st;
    k_eng_scatter_final<<<int(ceil_div(d.batch * n, 256)), 256, 0, s>>>(d);
    BT_CHECK_LAUNCH("k_eng_scatter_final");
    return BT_OK;
  }
  if (d.mode == BT_MODE_SCATTER) {
    const int S = d.neuron_spt > 0 ? d.neuron_spt : 4;
    const dim3 grid(unsigned(ceil_div(n, kEngThreads)), unsigned(ceil_div(d.batch, S)));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned planes = unsigned(d.bin_hi - d.bin_lo + 1);
    // a plane lists at most n rows: no more blocks than n rows need (small
    // networks would otherwise launch mostly idle blocks every step)
    const int64_t rows_per_block = d.scatter_lanes == 1 ? kEngThreads : d.scatter_lanes == 8 ? kEngThreads / 8
                                                                                            : kEngThreads / 32;
    const int64_t xblocks = std::min(ceil_div(int64_t(sms) * 8, planes), ceil_div(n, rows_per_block));
    const dim3 sgrid(unsigned(std::max<int64_t>(xblocks, 1)), planes);
    const int ms = mask_stride(d.batch);
    // every divisor a power of two or a verified reciprocal: no IEEE division compiled in
    const bool fast = fast_divisors(d, KIND);
    auto neuron = fast ? (S == 1 ? k_eng_neuron<KIND, HARD, USE_REF, 1, true>
                          : S == 2 ? k_eng_neuron<KIND, HARD, USE_REF, 2, true> : k_eng_neuron<KIND, HARD, USE_REF, 4, true>)
                       : (S == 1 ? k_eng_neuron<KIND, HARD, USE_REF, 1, false>
                          : S == 2 ? k_eng_neuron<KIND, HARD, USE_REF, 2, false> : k_eng_neuron<KIND, HARD, USE_REF, 4, false>);
    auto pick = [&](auto g) {
      constexpr int G = decltype(g)::value;
      // MS >= ms: mask_stride gives 1, 2, 4, or 5..8 words (MS = 8)
    return ms == 1 ? k_eng_scatter<G, 1> : ms == 2 ? k_eng_scatter<G, 2> : ms <= 4 ? k_eng_scatter<G, 4>
                                                                                      : k_eng_scatter<G, 8>;
    };
    auto scatter = d.scatter_lanes == 1   ? (ms == 1 ? k_eng_scatter_flat<1> : ms == 2 ? k_eng_scatter_flat<2>
                                             : ms <= 4 ? k_eng_scatter_flat<4> : k_eng_scatter_flat<8>)
                   : d.scatter_lanes == 8 ? pick(std::integral_constant<int, 8>())
                                          : pick(std::integral_constant<int, 32>());
    const int C = n_rec(d);
    const dim3 rgrid(unsigned(ceil_div(n, kEngThreads)), unsigned(d.batch));
    // vector access to the C channels of (b, i) needs 8 / 16-byte aligned state and acc
    const bool aligned = ((reinterpret_cast<uintptr_t>(d.psc) | reinterpret_cast<uintptr_t>(d.ring)) & 15) == 0;
    auto rec = C == 4 && aligned ? k_eng_neuron_rec<KIND, HARD, USE_REF, 4>
             : C == 2 && aligned ? k_eng_neuron_rec<KIND, HARD, USE_REF, 2> : k_eng_neuron_rec<KIND, HARD, USE_REF, 0>;
    for (int64_t k = 0; k < d.n_steps; ++k) {
      const StepIdx si = step_idx(d.t0 + k, d.n_bins, d.hist_len);
      if (C > 1) rec<<<rgrid, kEngThreads, 0, s>>>(d, k, si);
      else neuron<<<grid, kEngThreads, 0, s>>>(d, int(k), si, scatter_scratch(d, si.q_t));
      scatter<<<sgrid, kEngThreads, 0, s>>>(d, k, si);
    }
    BT_CHECK_LAUNCH("k_eng_neuron/k_eng_scatter");
    if (d.n_steps > 0) {
      k_eng_scatter_final<<<int(ceil_div(d.batch * n * C, 256)), 256, 0, s>>>(d);
      BT_CHECK_LAUNCH("k_eng_scatter_final");
    }
  } else if (d.mode == BT_MODE_PULL) {
    // Words of the sample mask per warp: the descriptor may ask for 2 or 4
    // (fewer warps, one vector mask load per edge); by default every warp
    // takes one 32-sample word, which gives the most warps in flight.
    const int mw = mask_stride(d.batch);
    int MWT = d.pull_words_per_warp > 0 ? d.pull_words_per_warp : 1;
    if (MWT != 1 && MWT != mw) MWT = 1;
    const int split = MWT < mw ? 1 : 0;
    const int64_t warps = ceil_div(n, 32) * (split ? mw : 1);
    const int grid = int(ceil_div(warps, kPullWarps));
    const size_t smem = sizeof(float) * kPullWarps * MWT * 32 * 32;
#define BT_PULL_LAUNCH(M)                                                                                        \
  do {                                                                                                           \
    auto kern = k_eng_pull<KIND, HARD, USE_REF, false, M>;                                                      \
    auto kfin = k_eng_pull<KIND, HARD, USE_REF, true, M>;                                                       \
    if (smem > 48 * 1024 &&                                                                                      \
        (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess ||    \
         cudaFuncSetAttribute(kfin, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess))     \
      return bt_set_error(BT_ERR_CUDA, "shared memory request of %zu bytes refused", smem);                     \
    for (int64_t k = 0; k < d.n_steps; ++k)                                                                     \
      kern<<<grid, kPullWarps * 32, smem, s>>>(d, k, split, step_idx(d.t0 + k, d.n_bins, d.hist_len));          \
    BT_CHECK_LAUNCH("k_eng_pull");                                                                               \
    kfin<<<grid, kPullWarps * 32, smem, s>>>(d, d.n_steps - 1, split,                                           \
                                             step_idx(d.t0 + d.n_steps - 1, d.n_bins, d.hist_len));              \
    BT_CHECK_LAUNCH("k_eng_pull final");                                                                         \
  } while (0)
    if (d.n_steps > 0) {
      if (MWT == 1) BT_PULL_LAUNCH(1);
      else if (MWT == 2) BT_PULL_LAUNCH(2);
      else BT_PULL_LAUNCH(4);
    }
#undef BT_PULL_LAUNCH
  } else {
    const int grid = int(ceil_div(n, 32));
    const size_t smem = sizeof(uint32_t) * size_t(d.batch);
    BT_CHECK_ARG(smem <= 48 * 1024, "batch too large for the gather engine");
    auto gather = n_rec(d) > 1 ? k_eng_gather<KIND, HARD, USE_REF, true> : k_eng_gather<KIND, HARD, USE_REF, false>;
    for (int64_t k = 0; k < d.n_steps; ++k)
      gather<<<grid, 1024, smem, s>>>(d, k, step_idx(d.t0 + k, d.n_bins, d.hist_len));
    BT_CHECK_LAUNCH("k_eng_gather");
    if (d.n_steps > 0) {
      k_eng_gather_final<<<grid, 1024, 0, s>>>(d, step_idx(d.t0 + d.n_steps - 1, d.n_bins, d.hist_len));
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

extern "C" int bt_engine_prime(const bt_engine_desc* d, void* stream) {
  if (int st = engine_check(d)) return st;
  if (d->mode != BT_MODE_SCATTER) return BT_OK;
  BT_CHECK_ARG(d->t0 >= d->hist_len, "t0=%lld must be >= hist_len", (long long)d->t0);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t words = size_t(scatter_work_words(d->n, d->batch, d->n_bins));
  if (cudaMemsetAsync(d->work, 0, sizeof(int32_t) * words, s) != cudaSuccess ||
      cudaMemsetAsync(d->ring, 0, sizeof(float) * size_t(d->batch * d->n * n_rec(*d)), s) != cudaSuccess)
    return bt_set_error(BT_ERR_CUDA, "memset failed");
  if (d->bin_hi > 0) {
    const int64_t npad = ((d->n + 31) >> 5) * 32;
    k_prime_history<<<int(ceil_div(int64_t(d->bin_hi) * npad, 256)), 256, 0, s>>>(*d);
    BT_CHECK_LAUNCH("k_prime_history");
  }
  return BT_OK;
}

namespace {
int input_project(int64_t rows, int64_t c_in, int64_t n, const float* xin, const float* w_t, const float* bias,
                  float* out, int32_t* work, const int32_t* live_len, int64_t batch, void* stream) {
  BT_CHECK_ARG(rows >= 0 && c_in >= 0 && n >= 0, "negative size");
  if (rows == 0 || n == 0) return BT_OK;
  BT_CHECK_ARG(xin && w_t && out && work, "null pointer");
  BT_CHECK_ARG(rows * c_in < (int64_t(1) << 40), "too large");
  BT_CHECK_ARG((reinterpret_cast<uintptr_t>(work) & 7) == 0, "work must be 8-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int2* pairs = reinterpret_cast<int2*>(work);
  int32_t* cnt = work + 2 * rows * c_in;
  k_row_pairs<<<int(ceil_div(rows * 32, 256)), 256, 0, s>>>(rows, c_in, xin, cnt, pairs, live_len, batch);
  BT_CHECK_LAUNCH("k_row_pairs");
  dim3 grid(unsigned(ceil_div(rows, kProjRows)), unsigned(ceil_div(n, 256 * kProjNPT)));
  BT_CHECK_ARG(grid.y < 65536 && grid.x < (1u << 31), "projection grid too large");
  k_input_project<<<grid, 256, 0, s>>>(rows, c_in, n, w_t, bias, cnt, pairs, out);
  BT_CHECK_LAUNCH("k_input_project");
  return BT_OK;
}
}  // namespace

extern "C" int bt_input_project(int64_t rows, int64_t c_in, int64_t n, const float* xin, const float* w_t,
                                const float* bias, float* out, int32_t* work, void* stream) {
  return input_project(rows, c_in, n, xin, w_t, bias, out, work, nullptr, 1, stream);
}

extern "C" int bt_input_project_live(int64_t steps, int64_t batch, int64_t c_in, int64_t n, const float* xin,
                                     const float* w_t, const float* bias, const int32_t* sample_len, float* out,
                                     int32_t* work, void* stream) {
  BT_CHECK_ARG(steps >= 0 && batch > 0, "bad steps / batch");
  return input_project(steps * batch, c_in, n, xin, w_t, bias, out, work, sample_len, batch, stream);
}

extern "C" int bt_input_grad_weight(int64_t rows, int64_t c_in, int64_t n, const float* x, const float* g,
                                    float* out, int32_t accumulate, int32_t* work, void* stream) {
  BT_CHECK_ARG(rows >= 0 && c_in >= 0 && n >= 0, "negative size");
  if (c_in == 0 || n == 0) return BT_OK;
  BT_CHECK_ARG(x && g && out && work, "null pointer");
  BT_CHECK_ARG(c_in * (rows + 1) < (int64_t(1) << 31), "c_in * rows too large");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int32_t* lists = work;
  int32_t* counts = work + c_in * rows;
  k_channel_rows<<<int(ceil_div(c_in * 32, 256)), 256, 0, s>>>(rows, c_in, x, lists, counts);
  BT_CHECK_LAUNCH("k_channel_rows");
  const dim3 grid(unsigned(c_in), unsigned(ceil_div(n, 256 * kProjNPT)));
  BT_CHECK_ARG(grid.y < 65536, "n too large");
  k_input_grad_weight<<<grid, 256, 0, s>>>(rows, c_in, n, x, g, lists, counts, out, accumulate);
  BT_CHECK_LAUNCH("k_input_grad_weight");
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

extern "C" int bt_mask_stride(int64_t batch) { return batch > 0 ? mask_stride(batch) : 0; }

extern "C" int64_t bt_engine_work_words(int64_t n, int64_t batch, int32_t n_bins) {
  return (n > 0 && batch > 0 && n_bins >= 1 && n_bins <= BT_MAX_BINS) ? scatter_work_words(n, batch, n_bins) : 0;
}

extern "C" int bt_float_to_masks(int64_t batch, int64_t n, const float* in, uint32_t* masks, void* stream) {
  BT_CHECK_ARG(batch >= 0 && n >= 0, "negative size");
  if (batch * n == 0) return BT_OK;
  BT_CHECK_ARG(in && masks, "null pointer");
  const int64_t total = n * mask_stride(batch);
  k_float_to_masks<<<int(ceil_div(total, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(batch, n, in, masks);
  BT_CHECK_LAUNCH("k_float_to_masks");
  return BT_OK;
}

extern "C" int bt_masks_to_float(int64_t batch, int64_t n, const uint32_t* masks, float* out, void* stream) {
  BT_CHECK_ARG(batch >= 0 && n >= 0, "negative size");
  if (batch * n == 0) return BT_OK;
  BT_CHECK_ARG(out && masks, "null pointer");
  k_masks_to_float<<<int(ceil_div(batch * n, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(batch, n, masks, out);
  BT_CHECK_LAUNCH("k_masks_to_float");
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
