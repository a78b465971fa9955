// Persistent tile engine (BT_MODE_TILE): many recurrent steps in one launch
// for networks without synaptic delays (a single delay bin 0), the
// counterpart of RecurrentNN's time loop (btorch/models/rnn.py:200-332)
// with the step of rnn.py:517-528.
//
// The posts are cut into n_tiles tiles of tile_posts neurons.  One CTA owns
// a tile for every sample of the batch and keeps the tile's synaptic input
// (the accumulator W z of the next step, [batch][tile_posts] fp32) in shared
// memory for the whole launch.  Per step:
//
//   neuron phase   every (sample, neuron) of the tile: P = stored + acc,
//                  acc = 0, I = P + x, LIF/ALIF update, stored = decay(P),
//                  spike bitmaps (warp ballot); the tile's spiking neurons
//                  are compacted into the tile's spike list, one record per
//                  neuron: its id and the mask of samples in which it spiked.
//   grid barrier   (bounded wait, see below)
//   delivery       every CTA walks the spike lists of all tiles and, for
//                  each listed neuron j, the run of j's out-edges that lands
//                  in its own tile (tile_off: the CSR row of j split at the
//                  tile boundaries; rows are sorted by post), adding w into
//                  the shared accumulator of every sample in j's mask
//                  (shared-memory fp32 atomics).
//
// So the synaptic input of a step never leaves the SM: no accumulator
// traffic to L2/HBM and no per-event L2 reduction, which is what bounds the
// two-launch scatter step.  The spike lists are double-buffered by step
// parity: the neuron phase of step k + 1 may overwrite nothing that the
// delivery of step k still reads, and the barrier after the neuron phase of
// step k + 1 waits for every CTA's delivery of step k, so one barrier per
// step suffices.  The order of the additions into one accumulator is not
// fixed (as in the scatter step): exact whenever the partial sums are
// (dyadic weights).
//
// Grid barrier: every CTA must be resident (cooperative launch, grid <= the
// co-resident limit checked on the host).  A CTA's thread 0 arrives on a
// counter and waits for the generation word to move on, at most
// spin_limit polls; a wait that gives up sets the status word, and every CTA
// leaves the launch at its next barrier once the status word is set, so the
// kernel always ends.  The host reads the status word after the call
// (BT_ERR_TIMEOUT).
//
// At the end of the launch the shared accumulators are written to d.ring,
// which the call's final launch (k_eng_scatter_final) adds into psc -- the
// hand-over the two-launch scatter step uses, so calls of either mode
// interleave freely.
#include "neuron.cuh"

namespace bt {

constexpr int kTileThreads = 512;
constexpr int kTileWarps = kTileThreads / 32;
constexpr unsigned kDefaultSpinLimit = 4u << 20;  // polls with a 256 ns back-off: about a second

__host__ __device__ __forceinline__ int tile_mask_words(int64_t batch) { return int((batch + 31) >> 5); }

// Mask words a record is laid out for: the kernel's compile-time bucket
// MS >= the batch's mask words (1, 2, 4 or 8).
__host__ __device__ __forceinline__ int tile_mask_bucket(int64_t batch) {
  const int ms = tile_mask_words(batch);
  return ms <= 1 ? 1 : ms <= 2 ? 2 : ms <= 4 ? 4 : 8;
}

// Words of one spike-list record: the neuron id and MS mask words, padded to
// 2, 4, 8 or 16 words (MS = 1, 2, 4, 8) -- exactly what load_record<MS>
// reads with 8- or 16-byte vector loads.
__host__ __device__ __forceinline__ int tile_rec_words(int64_t batch) { return 2 * tile_mask_bucket(batch); }

// Work layout (int32 words): [0, 32) control (0: barrier arrivals,
// 1: barrier generation, 2: status), then counts [2][n_tiles], then, from
// the next multiple of 16 words (64 bytes: every record 16-byte aligned),
// records [2][n_tiles][tile_posts][rec_words].
constexpr int kTileCtrl = 32;
__host__ __device__ __forceinline__ int64_t tile_rec_offset(int n_tiles) {
  return (kTileCtrl + 2 * int64_t(n_tiles) + 15) & ~int64_t(15);
}
__host__ __device__ __forceinline__ int64_t tile_work_words(int64_t batch, int tile_posts, int n_tiles) {
  return tile_rec_offset(n_tiles) + 2 * int64_t(n_tiles) * tile_posts * tile_rec_words(batch);
}

// Dynamic shared memory: accumulators [batch][tile_posts], sample masks
// [tile_posts][mask words], list offsets [n_tiles + 1] (+ scan scratch).
__host__ __device__ __forceinline__ size_t tile_smem_bytes(int64_t batch, int tile_posts, int n_tiles) {
  return sizeof(float) * size_t(batch) * tile_posts + sizeof(uint32_t) * size_t(tile_posts) * tile_mask_words(batch) +
         sizeof(int32_t) * (size_t(n_tiles) + 1 + kTileWarps + 2 + size_t(batch));
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier with a bounded wait.  Returns false (every thread) if the
// status word is set, by this wait or another CTA's.
__device__ bool tile_barrier(unsigned* ctrl, unsigned nblocks, unsigned& gen, unsigned spin_limit, int* s_flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned* count = ctrl;
    unsigned* genw = ctrl + 1;
    int* status = reinterpret_cast<int*>(ctrl + 2);
    __threadfence();  // this CTA's spike list and counts before the arrival
    const unsigned arrived = atomicAdd(count, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(count, 0u);  // reset before the generation moves: no CTA arrives again before that
      __threadfence();
      atomicAdd(genw, 1u);
    } else {
      unsigned polls = 0;
      while (ld_acquire_u32(genw) == gen) {
        if (++polls > spin_limit || *reinterpret_cast<volatile int*>(status) != 0) {
          atomicCAS(status, 0, BT_ERR_TIMEOUT);
          break;
        }
        __nanosleep(256);
      }
    }
    __threadfence();
    ++gen;
    *s_flag = *reinterpret_cast<volatile int*>(status);
  }
  __syncthreads();
  return *s_flag == 0;
}

constexpr int kTileU = 4;     // samples per warp item of the neuron phase (loads in flight)
constexpr int kTileGroups = 4;  // groups of 32 spike records a warp prefetches in the delivery

// One item of the neuron phase: a 32-neuron word of the tile (lane = neuron)
// for kTileU consecutive samples b0 .. b0+kTileU-1.  All the samples' loads
// are issued before the first update (memory-level parallelism for a phase
// that streams the state once); per sample the update is the reference's
// (see k_eng_neuron), the spike bitmaps go out by warp ballot and the
// neuron's sample bits of this word are or-ed into the tile's mask with one
// shared atomic.
template <int KIND, bool HARD, bool USE_REF, bool FAST>
__device__ __forceinline__ void tile_neuron_item(const bt_engine_desc& d, const NeuronParams& prm_u, int64_t k,
                                                 int b0, int64_t i, bool valid, int l, int Tp, float* s_acc,
                                                 const int* s_len, uint32_t* s_mask, int ms, float pc_u,
                                                 const Div& dpt_u, int h_t, int64_t words, int64_t wg,
                                                 bool traces) {
  const int B = int(d.batch), n32 = int(d.n);
  const unsigned lane = lane_id();
  float pend[kTileU], pv[kTileU], xv[kTileU], vv[kTileU], rv[kTileU], gv[kTileU];
  bool live[kTileU], edge[kTileU];
  const int off0 = b0 * n32 + int(valid ? i : 0);
  const float* xk = d.x ? d.x + k * int64_t(n32) * B : nullptr;
#pragma unroll
  for (int u = 0; u < kTileU; ++u) {
    const int b = b0 + u;
    const bool in = valid && b < B;
    const int len = in ? s_len[b] : 0;
    live[u] = in && k < len;
    edge[u] = in && k <= len;
    const bool rd = live[u] || (in && traces);
    const int off = off0 + u * n32;
    pend[u] = edge[u] ? s_acc[b * Tp + l] : 0.0f;
    pv[u] = (edge[u] || (in && traces)) ? d.psc[off] : 0.0f;
    xv[u] = (live[u] && xk) ? __ldcs(xk + off) : 0.0f;
    vv[u] = rd ? d.v[off] : 0.0f;
    rv[u] = (rd && USE_REF) ? d.refractory[off] : 0.0f;
    gv[u] = (rd && KIND == BT_NEURON_ALIF) ? d.g_k[off] : 0.0f;
  }
  NeuronParams prm = prm_u;
  float pc = pc_u;
  Div dpt = dpt_u;
  if (!d.neuron.uniform) prm = load_params<KIND, USE_REF>(d.neuron, valid ? i : 0);
  if (!d.psc_uniform) {
    const int64_t ip = valid ? i : 0;
    pc = ld(d.psc_coef, ip);
    dpt = make_div(ld(d.psc_tau, ip), false, 0.0f);
  }
  uint32_t bits = 0;
#pragma unroll
  for (int u = 0; u < kTileU; ++u) {
    const int b = b0 + u;
    if (b >= B) break;  // warp-uniform
    const int off = off0 + u * n32;
    float s = 0.0f;
    float v = vv[u], ref = rv[u], gk = gv[u];
    float P = pv[u];
    if (edge[u]) s_acc[b * Tp + l] = 0.0f;
    if (live[u]) {
      P = add(pv[u], pend[u]);
      const float I = xk ? add(P, xv[u]) : P;
      s = neuron_update<KIND, HARD, USE_REF, true, FAST>(prm, I, v, ref, gk).spike;
      d.v[off] = v;
      if (USE_REF) d.refractory[off] = ref;
      if (KIND == BT_NEURON_ALIF) d.g_k[off] = gk;
      d.psc[off] = psc_decay_k<FAST>(pc, dpt, P);
    } else if (edge[u]) {
      // the first step past the sample's end completes psc of its last step
      P = add(P, pend[u]);
      d.psc[off] = P;
    }
    if (traces && valid) {
      const int64_t tix = (k * B + b) * d.n + i;
      if (d.psc_trace && k > 0) d.psc_trace[tix - int64_t(B) * d.n] = P;
      if (d.v_trace) d.v_trace[tix] = v;
      if (USE_REF && d.ref_trace) d.ref_trace[tix] = ref;
      if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[tix] = gk;
      if (d.spikes) d.spikes[tix] = s;
    }
    const uint32_t word = __ballot_sync(0xffffffffu, s != 0.0f);
    if (lane == 0 && wg < words) {
      d.hist[(int64_t(h_t) * B + b) * words + wg] = word;
      if (d.raster) d.raster[(k * B + b) * words + wg] = word;
    }
    if (s != 0.0f) bits |= 1u << (b & 31);
  }
  if (bits) atomicOr(s_mask + l * ms + (b0 >> 5), bits);
}

// Record loads of the delivery: the neuron id and MS mask words (records of
// tile_rec_words(batch) words, 16-byte aligned for MS >= 2).
template <int MS>
__device__ __forceinline__ uint32_t load_record(const uint32_t* r, uint32_t (&m)[MS]) {
  if constexpr (MS == 1) {
    const uint2 a = __ldcg(reinterpret_cast<const uint2*>(r));
    m[0] = a.y;
    return a.x;
  } else if constexpr (MS == 2) {
    const uint4 a = __ldcg(reinterpret_cast<const uint4*>(r));
    m[0] = a.y;
    m[1] = a.z;
    return a.x;
  } else {
    // MS = 4: records of 8 words, two 16-byte loads; MS = 8: records of 16
    // words, the first 12 read (the id and 8 mask words)
    uint32_t w[MS + 4];
#pragma unroll
    for (int q = 0; q < (MS + 4) / 4; ++q) {
      const uint4 a = __ldcg(reinterpret_cast<const uint4*>(r) + q);
      w[4 * q] = a.x;
      w[4 * q + 1] = a.y;
      w[4 * q + 2] = a.z;
      w[4 * q + 3] = a.w;
    }
#pragma unroll
    for (int q = 0; q < MS; ++q) m[q] = w[1 + q];
    return w[0];
  }
}

template <int KIND, bool HARD, bool USE_REF, bool FAST, int MS>
__global__ void __launch_bounds__(kTileThreads, 1) k_tile_engine(bt_engine_desc d) {
  extern __shared__ float tile_smem[];
  const int Tp = d.tile_posts, P = d.n_tiles;
  const int64_t n = d.n, B = d.batch;
  const int ms = tile_mask_words(B), RW = tile_rec_words(B);
  const int64_t words = (n + 31) >> 5;
  const int tile = blockIdx.x;
  const int64_t p0 = int64_t(tile) * Tp;
  const int NW = Tp >> 5;  // 32-neuron words of the tile
  const int NG = int((B + kTileU - 1) / kTileU);
  float* s_acc = tile_smem;                                            // [B][Tp]
  uint32_t* s_mask = reinterpret_cast<uint32_t*>(s_acc + B * Tp);     // [Tp][ms]
  int32_t* s_pre = reinterpret_cast<int32_t*>(s_mask + Tp * ms);      // [P + 1] list offsets
  int32_t* s_scan = s_pre + P + 1;                                    // [kTileWarps] + flag + total
  int* s_flag = s_scan + kTileWarps;
  int* s_len = s_flag + 2;                                            // [B] sample lengths
  unsigned* ctrl = reinterpret_cast<unsigned*>(d.tile_work);
  int32_t* counts = d.tile_work + kTileCtrl;                            // [2][P]
  uint32_t* recs = reinterpret_cast<uint32_t*>(d.tile_work + tile_rec_offset(P));  // [2][P][Tp][RW]
  const unsigned spin = d.spin_limit > 0 ? unsigned(d.spin_limit) : kDefaultSpinLimit;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int H = d.hist_len;
  const bool traces = d.v_trace || d.psc_trace || d.ref_trace || d.gk_trace || d.spikes;

  for (int64_t q = threadIdx.x; q < B * Tp; q += kTileThreads) s_acc[q] = 0.0f;
  for (int q = threadIdx.x; q < int(B); q += kTileThreads)
    s_len[q] = d.sample_len ? int(min(int64_t(d.sample_len[q]), int64_t(INT32_MAX))) : INT32_MAX;
  unsigned gen = 0;
  if (threadIdx.x == 0) gen = ld_acquire_u32(ctrl + 1);

  const NeuronParams prm_u = load_params<KIND, USE_REF>(d.neuron, 0);
  const float pc_u = d.psc_uniform ? d.psc_coef_s : 0.0f;
  const Div dpt_u = make_div(d.psc_uniform ? d.psc_tau_s : 1.0f, d.psc_uniform && d.psc_fast_div, d.psc_rcp);

  for (int64_t k = 0; k < d.n_steps; ++k) {
    const int buf = int(k & 1);
    const int h_t = int((d.t0 + k) % H);
    for (int q = threadIdx.x; q < Tp * ms; q += kTileThreads) s_mask[q] = 0u;
    __syncthreads();
    // ---- neuron phase: items (word w, group of kTileU samples), groups fastest
    for (int it = warp; it < NW * NG; it += kTileWarps) {
      const int w = it / NG;
      const int b0 = (it - w * NG) * kTileU;
      const int l = w * 32 + lane;
      const int64_t i = p0 + l;
      tile_neuron_item<KIND, HARD, USE_REF, FAST>(d, prm_u, k, b0, i, i < n, l, Tp, s_acc, s_len, s_mask, ms, pc_u,
                                                  dpt_u, h_t, words, (p0 >> 5) + w, traces);
    }
    __syncthreads();
    // ---- compaction: the tile's spiking neurons, in ascending id order
    int32_t* cnt = counts + buf * P;
    uint32_t* rec = recs + (int64_t(buf) * P + tile) * Tp * RW;
    long long ev = 0, ed = 0;
    int base = 0;
    for (int l0 = 0; l0 < Tp; l0 += kTileThreads) {
      const int l = l0 + threadIdx.x;
      bool any = false;
      if (l < Tp)
        for (int m = 0; m < ms; ++m) any |= s_mask[l * ms + m] != 0u;
      const uint32_t bal = __ballot_sync(0xffffffffu, any);
      if (lane == 0) s_scan[warp] = __popc(bal);
      __syncthreads();
      if (warp == 0) {
        const int c = lane < kTileWarps ? s_scan[lane] : 0;
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        if (lane < kTileWarps) s_scan[lane] = incl - c;
        if (lane == 31) s_flag[1] = incl;
      }
      __syncthreads();
      if (any) {
        const int slot = base + s_scan[warp] + __popc(bal & ((1u << lane) - 1u));
        uint32_t* r = rec + int64_t(slot) * RW;
        r[0] = uint32_t(p0 + l);
        int pop = 0;
        for (int m = 0; m < ms; ++m) {
          const uint32_t mv = s_mask[l * ms + m];
          r[1 + m] = mv;
          pop += __popc(mv);
        }
        if (d.stats) {
          const long long deg = d.outdeg ? d.outdeg[p0 + l] : 0;
          ev += pop * deg;
          ed += deg;
        }
      }
      base += s_flag[1];
      __syncthreads();
    }
    if (threadIdx.x == 0) cnt[tile] = base;
    if (d.stats) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ev += __shfl_xor_sync(0xffffffffu, ev, o);
        ed += __shfl_xor_sync(0xffffffffu, ed, o);
      }
      __shared__ long long s_ev[kTileWarps], s_ed[kTileWarps];
      if (lane == 0) {
        s_ev[warp] = ev;
        s_ed[warp] = ed;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        long long tev = 0, ted = 0;
        for (int q = 0; q < kTileWarps; ++q) {
          tev += s_ev[q];
          ted += s_ed[q];
        }
        if (base) atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 0), (unsigned long long)base);
        if (tev) atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 1), (unsigned long long)tev);
        if (ted) atomicAdd(reinterpret_cast<unsigned long long*>(d.stats + k * 4 + 2), (unsigned long long)ted);
      }
    }
    if (!tile_barrier(ctrl, unsigned(P), gen, spin, s_flag)) return;
    // ---- delivery: every listed neuron's out-edges into this tile
    if (warp == 0) {
      // offsets of the P lists (one pass of 32-wide scans)
      int carry = 0;
      for (int q0 = 0; q0 < P; q0 += 32) {
        const int q = q0 + lane;
        const int c = q < P ? int(ld_acquire_u32(reinterpret_cast<const unsigned*>(cnt + q))) : 0;
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        if (q < P) s_pre[q] = carry + incl - c;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) s_pre[P] = carry;
    }
    __syncthreads();
    const int total = s_pre[P];
    const uint32_t* recb = recs + int64_t(buf) * P * Tp * RW;
    const int32_t* toff = d.tile_off;
    const uint64_t pol_stream = l2_evict_first();
    constexpr int G = kTileGroups;
    for (int base0 = warp * 32 * G; base0 < total; base0 += kTileWarps * 32 * G) {
      // kTileGroups records per lane: their ids, masks and tile segments,
      // every load issued before any is used
      int32_t e0[G], cntg[G];
      uint32_t mk[G][MS];
      uint32_t jj[G];
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int idx = base0 + g * 32 + lane;
        jj[g] = 0xffffffffu;
#pragma unroll
        for (int q = 0; q < MS; ++q) mk[g][q] = 0u;
        if (idx < total) {
          int lo = 0, hi = P - 1;  // the list holding entry idx: the last q with s_pre[q] <= idx
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_pre[mid] <= idx) lo = mid;
            else hi = mid - 1;
          }
          jj[g] = load_record<MS>(recb + (int64_t(lo) * Tp + (idx - s_pre[lo])) * RW, mk[g]);
        }
      }
#pragma unroll
      for (int g = 0; g < G; ++g) {
        e0[g] = 0;
        cntg[g] = 0;
        if (jj[g] != 0xffffffffu) {
          const int32_t* tj = toff + int64_t(jj[g]) * (P + 1) + tile;
          e0[g] = __ldg(tj);
          cntg[g] = __ldg(tj + 1) - e0[g];
        }
      }
#pragma unroll
      for (int g = 0; g < G; ++g) {
        // the 32 records' segments walked as one flattened edge range, a lane per edge
        int incl = cntg[g];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        const int excl = incl - cntg[g];
        const int tot = __shfl_sync(0xffffffffu, incl, 31);
        // EU passes of 32 edges per iteration: every edge load of the
        // iteration is issued before its additions (memory-level parallelism)
        constexpr int EU = 4;
        for (int f0 = 0; f0 < tot; f0 += 32 * EU) {
          uint2 rec2[EU];
          uint32_t mm[EU][MS];
#pragma unroll
          for (int uu = 0; uu < EU; ++uu) {
            const int f = f0 + uu * 32 + lane;
            int r = 0;  // the last lane whose excl <= f
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
              const int x = __shfl_sync(0xffffffffu, excl, r + step);
              if (x <= f) r += step;
            }
            const int eb = __shfl_sync(0xffffffffu, e0[g], r) + (f - __shfl_sync(0xffffffffu, excl, r));
#pragma unroll
            for (int q = 0; q < MS; ++q) mm[uu][q] = __shfl_sync(0xffffffffu, mk[g][q], r);
            if (f < tot) {
              rec2[uu] = ld_nc_u2(d.csr_edges + 2 * int64_t(eb), pol_stream);
            } else {
              rec2[uu] = make_uint2(0u, 0u);
#pragma unroll
              for (int q = 0; q < MS; ++q) mm[uu][q] = 0u;
            }
          }
#pragma unroll
          for (int uu = 0; uu < EU; ++uu) {
            const int lp = int((rec2[uu].x & kIdMask) - uint32_t(p0));
            const float wv = __uint_as_float(rec2[uu].y);
#pragma unroll
            for (int q = 0; q < MS; ++q) {
              uint32_t bits = q < ms ? mm[uu][q] : 0u;
              while (bits) {
                const int bit = __ffs(bits) - 1;
                bits &= bits - 1;
                atomicAdd(s_acc + (q * 32 + bit) * Tp + lp, wv);
              }
            }
          }
        }
      }
    }
    __syncthreads();
  }
  // hand the pending synaptic input over to the call's final launch
  for (int64_t q = threadIdx.x; q < B * Tp; q += kTileThreads) {
    const int64_t b = q / Tp, l = q - b * Tp;
    if (p0 + l < n) d.ring[b * n + p0 + l] = s_acc[q];
  }
}

// Tile boundaries of every CSR row: off[r][t] = the first edge of row r whose
// post is >= t * tile_posts (rows sorted by post), t = 0 .. n_tiles.
__global__ void k_tile_offsets(int64_t rows, const int32_t* __restrict__ csr_ptr,
                               const uint32_t* __restrict__ edges, int tile_posts, int n_tiles,
                               int32_t* __restrict__ off) {
  const int64_t gid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t r = gid / (n_tiles + 1);
  const int t = int(gid - r * (n_tiles + 1));
  if (r >= rows) return;
  int32_t lo = csr_ptr[r], hi = csr_ptr[r + 1];
  const uint32_t key = uint32_t(int64_t(t) * tile_posts);
  while (lo < hi) {  // first edge with post >= key
    const int32_t mid = lo + ((hi - lo) >> 1);
    if ((edges[2 * int64_t(mid)] & kIdMask) < key) lo = mid + 1;
    else hi = mid;
  }
  off[gid] = lo;
}

template <int KIND, bool HARD, bool USE_REF, bool FAST>
auto tile_kernel(int ms) {
  // the record layout's bucket (tile_mask_bucket): 1, 2, 4 (3..4 words) or 8 (5..8)
  return ms == 1 ? k_tile_engine<KIND, HARD, USE_REF, FAST, 1>
         : ms == 2 ? k_tile_engine<KIND, HARD, USE_REF, FAST, 2>
         : ms == 4 ? k_tile_engine<KIND, HARD, USE_REF, FAST, 4> : k_tile_engine<KIND, HARD, USE_REF, FAST, 8>;
}

template <int KIND, bool HARD, bool USE_REF>
int tile_launch(const bt_engine_desc& d, bool fast, cudaStream_t s) {
  const int ms = tile_mask_bucket(d.batch);
  void (*kern)(bt_engine_desc) = fast ? tile_kernel<KIND, HARD, USE_REF, true>(ms)
                                      : tile_kernel<KIND, HARD, USE_REF, false>(ms);
  const size_t smem = tile_smem_bytes(d.batch, d.tile_posts, d.n_tiles);
  int dev = 0;
  cudaGetDevice(&dev);
  if (!launch_setup_known(reinterpret_cast<const void*>(kern), dev, smem, d.n_tiles)) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(launch_smem_allow(reinterpret_cast<const void*>(kern), dev, smem))) != cudaSuccess)
      return bt_set_error(BT_ERR_UNSUPPORTED, "tile engine: %zu bytes of shared memory refused", smem);
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTileThreads, smem) != cudaSuccess)
      return bt_set_error(BT_ERR_CUDA, "tile engine: occupancy query failed");
    if (int64_t(per_sm) * sms < d.n_tiles)
      return bt_set_error(BT_ERR_UNSUPPORTED, "tile engine: %d tiles but only %d co-resident blocks", d.n_tiles,
                          per_sm * sms);
    launch_setup_add(reinterpret_cast<const void*>(kern), dev, smem, d.n_tiles);
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(d.n_tiles));
  cfg.blockDim = dim3(kTileThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t err = cudaLaunchKernelEx(&cfg, kern, d);
  if (err != cudaSuccess) return bt_set_error(BT_ERR_CUDA, "tile engine launch: %s", cudaGetErrorString(err));
  return BT_OK;
}

int run_tile(const bt_engine_desc& d, bool fast, cudaStream_t s) {
  const bool h = d.neuron.hard_reset != 0, r = d.neuron.use_refractory != 0;
  if (d.neuron.kind == BT_NEURON_LIF) {
    if (h && r) return tile_launch<BT_NEURON_LIF, true, true>(d, fast, s);
    if (h) return tile_launch<BT_NEURON_LIF, true, false>(d, fast, s);
    if (r) return tile_launch<BT_NEURON_LIF, false, true>(d, fast, s);
    return tile_launch<BT_NEURON_LIF, false, false>(d, fast, s);
  }
  if (h && r) return tile_launch<BT_NEURON_ALIF, true, true>(d, fast, s);
  if (h) return tile_launch<BT_NEURON_ALIF, true, false>(d, fast, s);
  if (r) return tile_launch<BT_NEURON_ALIF, false, true>(d, fast, s);
  return tile_launch<BT_NEURON_ALIF, false, false>(d, fast, s);
}

}  // namespace bt

extern "C" int64_t bt_tile_work_words(int64_t batch, int32_t tile_posts, int32_t n_tiles) {
  return (batch > 0 && tile_posts > 0 && n_tiles > 0) ? bt::tile_work_words(batch, tile_posts, n_tiles) : 0;
}

extern "C" int64_t bt_tile_smem_bytes(int64_t batch, int32_t tile_posts, int32_t n_tiles) {
  return (batch > 0 && tile_posts > 0 && n_tiles > 0) ? int64_t(bt::tile_smem_bytes(batch, tile_posts, n_tiles)) : 0;
}

extern "C" int bt_tile_offsets(int64_t rows, const int32_t* csr_ptr, const uint32_t* csr_edges, int32_t tile_posts,
                               int32_t n_tiles, int32_t* off, void* stream) {
  BT_CHECK_ARG(rows >= 0 && tile_posts > 0 && (tile_posts & 31) == 0 && n_tiles > 0, "bad tile shape");
  if (rows == 0) return BT_OK;
  BT_CHECK_ARG(csr_ptr && csr_edges && off, "null pointer");
  const int64_t total = rows * (int64_t(n_tiles) + 1);
  bt::k_tile_offsets<<<int(bt::ceil_div(total, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, csr_ptr, csr_edges, tile_posts, n_tiles, off);
  BT_CHECK_LAUNCH("k_tile_offsets");
  return BT_OK;
}
