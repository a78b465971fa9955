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

constexpr int kTileThreads = 1024;
constexpr int kTileWarps = kTileThreads / 32;
constexpr unsigned kDefaultSpinLimit = 4u << 20;  // polls with a 256 ns back-off: about a second

__host__ __device__ __forceinline__ int tile_mask_words(int64_t batch) { return int((batch + 31) >> 5); }

// Words of one spike-list record: the neuron id and its sample mask words,
// rounded up to a power of two (2, 4, 8 or 16) for vector loads.
__host__ __device__ __forceinline__ int tile_rec_words(int64_t batch) {
  const int need = 1 + tile_mask_words(batch);
  return need <= 2 ? 2 : need <= 4 ? 4 : need <= 8 ? 8 : 16;
}

// Work layout (int32 words): [0, 32) control (0: barrier arrivals,
// 1: barrier generation, 2: status), then counts [2][n_tiles], then records
// [2][n_tiles][tile_posts][rec_words].
constexpr int kTileCtrl = 32;
__host__ __device__ __forceinline__ int64_t tile_work_words(int64_t batch, int tile_posts, int n_tiles) {
  return kTileCtrl + 2 * int64_t(n_tiles) + 2 * int64_t(n_tiles) * tile_posts * tile_rec_words(batch);
}

// Dynamic shared memory: accumulators [batch][tile_posts], sample masks
// [tile_posts][mask words], list offsets [n_tiles + 1] (+ scan scratch).
__host__ __device__ __forceinline__ size_t tile_smem_bytes(int64_t batch, int tile_posts, int n_tiles) {
  return sizeof(float) * size_t(batch) * tile_posts + sizeof(uint32_t) * size_t(tile_posts) * tile_mask_words(batch) +
         sizeof(int32_t) * (size_t(n_tiles) + 1 + kTileWarps + 2);
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

// One (sample b, 32-neuron word) item of the neuron phase: the lanes are the
// word's neurons.  Returns the spike (0 or 1) of this lane's neuron.
template <int KIND, bool HARD, bool USE_REF, bool FAST, bool TRACES>
__device__ __forceinline__ float tile_neuron_item(const bt_engine_desc& d, const NeuronParams& prm_u, int64_t k,
                                                  int64_t b, int64_t i, bool valid, float* acc, float pc,
                                                  const Div& dpt, int n32) {
  const int64_t len = d.sample_len ? d.sample_len[b] : INT64_MAX;
  const bool live = valid && k < len, edge = valid && k <= len;
  const int off = int(b) * n32 + int(valid ? i : 0);
  const bool frozen = valid && TRACES;
  float* __restrict__ psc_p = d.psc + off;
  float* __restrict__ v_p = d.v + off;
  float* __restrict__ ref_p = USE_REF ? d.refractory + off : nullptr;
  float* __restrict__ gk_p = KIND == BT_NEURON_ALIF ? d.g_k + off : nullptr;
  // loads before stores (a load behind a store to a maybe-aliasing pointer waits)
  const float pend = edge ? *acc : 0.0f;
  const float pv = (edge || frozen) ? *psc_p : 0.0f;
  const float xv = (live && d.x) ? __ldcs(d.x + k * int64_t(n32) * d.batch + off) : 0.0f;
  float v = (live || frozen) ? *v_p : 0.0f;
  float ref = ((live || frozen) && USE_REF) ? *ref_p : 0.0f;
  float gk = ((live || frozen) && KIND == BT_NEURON_ALIF) ? *gk_p : 0.0f;
  NeuronParams prm = prm_u;
  if (!d.neuron.uniform) prm = load_params<KIND, USE_REF>(d.neuron, valid ? i : 0);
  float s = 0.0f;
  if (valid) {
    float P = pv;
    if (edge) *acc = 0.0f;
    if (live) {
      P = add(pv, pend);
      const float I = d.x ? add(P, xv) : P;
      s = neuron_update<KIND, HARD, USE_REF, true, FAST>(prm, I, v, ref, gk).spike;
      *v_p = v;
      if (USE_REF) *ref_p = ref;
      if (KIND == BT_NEURON_ALIF) *gk_p = gk;
      *psc_p = psc_decay_k<FAST>(pc, dpt, P);
    } else if (edge) {
      // the first step past the sample's end completes psc of its last step
      P = add(P, pend);
      *psc_p = P;
    }
    if (TRACES) {
      const int64_t tix = (k * d.batch + b) * d.n + i;
      if (d.psc_trace && k > 0) d.psc_trace[tix - d.batch * d.n] = P;
      if (d.v_trace) d.v_trace[tix] = v;
      if (USE_REF && d.ref_trace) d.ref_trace[tix] = ref;
      if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[tix] = gk;
      if (d.spikes) d.spikes[tix] = s;
    }
  }
  return s;
}

template <int KIND, bool HARD, bool USE_REF, bool FAST, bool TRACES>
__global__ void __launch_bounds__(kTileThreads, 1) k_tile_engine(bt_engine_desc d) {
  extern __shared__ float tile_smem[];
  const int Tp = d.tile_posts, P = d.n_tiles;
  const int64_t n = d.n, B = d.batch;
  const int ms = tile_mask_words(B), RW = tile_rec_words(B);
  const int64_t words = (n + 31) >> 5;
  const int tile = blockIdx.x;
  const int64_t p0 = int64_t(tile) * Tp;
  const int NW = Tp >> 5;  // 32-neuron words of the tile
  float* s_acc = tile_smem;                                            // [B][Tp]
  uint32_t* s_mask = reinterpret_cast<uint32_t*>(s_acc + B * Tp);     // [Tp][ms]
  int32_t* s_pre = reinterpret_cast<int32_t*>(s_mask + Tp * ms);      // [P + 1] list offsets
  int32_t* s_scan = s_pre + P + 1;                                    // [kTileWarps] + flag + total
  int* s_flag = s_scan + kTileWarps;
  unsigned* ctrl = reinterpret_cast<unsigned*>(d.tile_work);
  int32_t* counts = d.tile_work + kTileCtrl;                            // [2][P]
  uint32_t* recs = reinterpret_cast<uint32_t*>(counts + 2 * P);        // [2][P][Tp][RW]
  const unsigned spin = d.spin_limit > 0 ? unsigned(d.spin_limit) : kDefaultSpinLimit;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n32 = int(n);
  const int H = d.hist_len;

  for (int64_t q = threadIdx.x; q < B * Tp; q += kTileThreads) s_acc[q] = 0.0f;
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
    // ---- neuron phase: items (word w, sample b), b fastest
    for (int64_t it = warp; it < int64_t(NW) * B; it += kTileWarps) {
      const int w = int(it / B);
      const int64_t b = it - int64_t(w) * B;
      const int l = w * 32 + lane;
      const int64_t i = p0 + l;
      const bool valid = i < n;
      float pc = pc_u;
      Div dpt = dpt_u;
      if (!d.psc_uniform) {
        const int64_t ip = valid ? i : 0;
        pc = ld(d.psc_coef, ip);
        dpt = make_div(ld(d.psc_tau, ip), false, 0.0f);
      }
      const float s = tile_neuron_item<KIND, HARD, USE_REF, FAST, TRACES>(d, prm_u, k, b, i, valid,
                                                                          s_acc + b * Tp + l, pc, dpt, n32);
      const uint32_t word = __ballot_sync(0xffffffffu, s != 0.0f);
      if (lane == 0 && (p0 >> 5) + w < words) {
        d.hist[(int64_t(h_t) * B + b) * words + (p0 >> 5) + w] = word;
        if (d.raster) d.raster[(k * B + b) * words + (p0 >> 5) + w] = word;
      }
      if (s != 0.0f) atomicOr(s_mask + l * ms + int(b >> 5), 1u << (b & 31));
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
        const int c = s_scan[lane];
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        s_scan[lane] = incl - c;
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
        const int c = q < P ? ld_acquire_u32(reinterpret_cast<const unsigned*>(cnt + q)) : 0;
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
    for (int idx = threadIdx.x; idx < total; idx += kTileThreads) {
      // list holding entry idx: the last q with s_pre[q] <= idx
      int lo = 0, hi = P - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_pre[mid] <= idx) lo = mid;
        else hi = mid - 1;
      }
      const uint32_t* r = recb + (int64_t(lo) * Tp + (idx - s_pre[lo])) * RW;
      const uint32_t j = __ldcg(r);
      const int32_t* tj = toff + int64_t(j) * (P + 1) + tile;
      const int32_t e0 = __ldg(tj), e1 = __ldg(tj + 1);
      if (e0 == e1) continue;
      uint32_t m[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) m[q] = q < ms ? __ldcg(r + 1 + q) : 0u;
      for (int32_t e = e0; e < e1; ++e) {
        const uint2 rec2 = ld_nc_u2(d.csr_edges + 2 * int64_t(e), pol_stream);
        const int lp = int((rec2.x & kIdMask) - uint32_t(p0));
        const float wv = __uint_as_float(rec2.y);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          if (q >= ms) break;
          uint32_t mm = m[q];
          while (mm) {
            const int bit = __ffs(mm) - 1;
            mm &= mm - 1;
            atomicAdd(s_acc + (q * 32 + bit) * Tp + lp, wv);
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

template <int KIND, bool HARD, bool USE_REF>
int tile_launch(const bt_engine_desc& d, bool fast, bool traces, cudaStream_t s) {
  void (*kern)(bt_engine_desc) =
      fast ? (traces ? k_tile_engine<KIND, HARD, USE_REF, true, true> : k_tile_engine<KIND, HARD, USE_REF, true, false>)
           : (traces ? k_tile_engine<KIND, HARD, USE_REF, false, true>
                     : k_tile_engine<KIND, HARD, USE_REF, false, false>);
  const size_t smem = tile_smem_bytes(d.batch, d.tile_posts, d.n_tiles);
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return bt_set_error(BT_ERR_UNSUPPORTED, "tile engine: %zu bytes of shared memory refused", smem);
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTileThreads, smem) != cudaSuccess)
    return bt_set_error(BT_ERR_CUDA, "tile engine: occupancy query failed");
  if (int64_t(per_sm) * sms < d.n_tiles)
    return bt_set_error(BT_ERR_UNSUPPORTED, "tile engine: %d tiles but only %d co-resident blocks", d.n_tiles,
                        per_sm * sms);
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
  const bool traces = d.v_trace || d.psc_trace || d.ref_trace || d.gk_trace || d.spikes;
  const bool h = d.neuron.hard_reset != 0, r = d.neuron.use_refractory != 0;
  if (d.neuron.kind == BT_NEURON_LIF) {
    if (h && r) return tile_launch<BT_NEURON_LIF, true, true>(d, fast, traces, s);
    if (h) return tile_launch<BT_NEURON_LIF, true, false>(d, fast, traces, s);
    if (r) return tile_launch<BT_NEURON_LIF, false, true>(d, fast, traces, s);
    return tile_launch<BT_NEURON_LIF, false, false>(d, fast, traces, s);
  }
  if (h && r) return tile_launch<BT_NEURON_ALIF, true, true>(d, fast, traces, s);
  if (h) return tile_launch<BT_NEURON_ALIF, true, false>(d, fast, traces, s);
  if (r) return tile_launch<BT_NEURON_ALIF, false, true>(d, fast, traces, s);
  return tile_launch<BT_NEURON_ALIF, false, false>(d, fast, traces, s);
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
