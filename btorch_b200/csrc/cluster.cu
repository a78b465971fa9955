// Single-cluster persistent engine (BT_MODE_CLUSTER) for small networks,
// with or without synaptic delay bins: every step of a call in ONE launch of one
// thread-block cluster of up to 16 CTAs, the step of btorch/models/rnn.py:
// 517-528 repeated over time (rnn.py:200-332).
//
// The cluster's CTAs split the posts into tiles of tile_posts (a multiple of
// 32).  A CTA keeps in shared memory, for the whole launch:
//   - its tile's state (v, psc, refractory, g_k) for every sample;
//   - its tile's in-edges, the SELL-32 slices of the CSC (lane = post, the
//     k-th in-edge of each post in row k, ascending canonical order), the
//     presynaptic id stored as id ^ 31 (16 bits when n + 32 <= 2^16);
//   - copies of the whole network's spike bitmap ([copies][batch][words + 1],
//     the last word of each sample zero: the slices' padding points there),
//     step k in copy k mod copies: 2 copies, or R + 1 with R delay bins
//     (bin b of step k reads the spikes of step k - 1 - b).
// Per step k, each warp takes (32-post word of the tile, sample):
//   synapse   P = decay(P) + sum over the post's in-edges (pre, bin) in
//             ascending order of w * z_{k-1-bin}[pre] (local bitmaps), the
//             fp32 chain of the gather engine: the reference's rounding for
//             ANY weights, not only dyadic ones;
//   neuron    I = P + x, LIF/ALIF update, the spike word by ballot;
//   publish   the word into bitmap copy k mod copies of every other CTA of the
//             cluster (st.async, one lane per CTA, its bytes counted on the
//             receiver's mbarrier for that copy) and of its own (plain store).
// Then thread 0 waits (bounded) for the barrier phase of the step (two
// mbarriers, by step parity) and the CTA synchronises: every word of step k
// is in this CTA's copy.  No cluster-wide barrier: a CTA arms a barrier for
// step s + 1 right after its wait for step s - 1 and before it publishes step
// s, which every sender of step s + 1 has to have received first; and a copy
// is overwritten (step k into the copy of step k - copies) only by a sender
// that has received every CTA's step k - 1, published after that CTA's last
// read of the copy (its step k - 1 reads steps k - 2 .. k - 1 - R).  With
// delay bins the copies of the call's first steps' history come from the
// history ring (d.hist) at the start.
// After the last step the launch applies the synapse update of that step
// (the gather engine's final launch) and writes the state back: one launch
// per call, nothing per step in global memory but the input read and the
// spike bitmaps written.
#include <cooperative_groups.h>

#include <type_traits>

#include "neuron.cuh"

namespace cg = cooperative_groups;

namespace bt {

constexpr int kClThreads = 256;
// in-edge rows of a slice are padded to a multiple of kClRows; the sum walks
// them kClRows at a time with every load of the block issued first
constexpr int kClRows = 16;
constexpr int kClMaxCtas = 16;

// Shared-memory carve-up of one CTA (bytes, every part 16-byte aligned):
// state [4][B][Tp] f32 | edge weights [rows][32] f32 | presynaptic ids
// [rows][32] (u16 when src16, else u32) | bitmaps [copies][B][Wd] u32 | slice
// group offsets [NW + 1] i32 | sample lengths [B] i32 | out-degrees [Tp] i32.
// rows: the tile's slice rows, each slice rounded up to a multiple of kClRows
// and stored as groups of 4 rows per lane ([group][lane][4]), so that one
// 8- or 16-byte load brings 4 in-edges of a post.
struct ClusterSmem {
  size_t state, w, src, bits, gptr, len, deg, total;
};

__host__ __device__ __forceinline__ size_t cl_align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ __forceinline__ bool cluster_src16(int64_t n) { return n + 32 <= 65536; }

// Presynaptic id encodings (template IDS): 0 = pre ^ 31 in 16 bits (no
// delay bins, n + 32 <= 2^16), 1 = the same in 32 bits, 2 = (pre ^ 31) in
// bits 0..19 and the delay bin in bits 20..24 (n + 32 <= 2^20, R <= 32).
constexpr int kClBinShift = 20;
__host__ __device__ __forceinline__ int cluster_ids(int64_t n, int n_bins) {
  return n_bins > 1 ? 2 : cluster_src16(n) ? 0 : 1;
}
__host__ __device__ __forceinline__ int cluster_copies(int n_bins) { return n_bins > 1 ? n_bins + 1 : 2; }

__host__ __device__ __forceinline__ ClusterSmem cluster_smem(int64_t n, int64_t batch, int tp, int64_t rows,
                                                            bool src16, int copies) {
  ClusterSmem s;
  const int64_t wd = ((n + 31) >> 5) + 1;
  s.state = 0;
  s.w = cl_align16(sizeof(float) * 4 * size_t(batch) * tp);
  s.src = s.w + cl_align16(sizeof(float) * size_t(rows) * 32);
  s.bits = s.src + cl_align16((src16 ? 2 : 4) * size_t(rows) * 32);
  s.gptr = s.bits + cl_align16(sizeof(uint32_t) * size_t(copies) * size_t(batch) * size_t(wd));
  s.len = s.gptr + cl_align16(sizeof(int32_t) * size_t(tp / 32 + 1));
  s.deg = s.len + cl_align16(sizeof(int32_t) * size_t(batch));
  s.total = s.deg + cl_align16(sizeof(int32_t) * size_t(tp));
  return s;
}

// Word exchange: a CTA's spike words go to the other CTAs of the cluster as
// asynchronous remote shared-memory stores (st.async) that each count their
// bytes on the receiving CTA's mbarrier for that bitmap copy; the receiver
// arms the barrier with the bytes it expects and waits for the phase (one
// thread, bounded polls).  No cluster-wide barrier and no release fence per
// step.
constexpr unsigned kClDefaultSpinLimit = 1u << 24;  // polls without back-off: about a second

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// one arrival that also expects `bytes` more transaction bytes in this phase
__device__ __forceinline__ void mbar_arm(uint64_t* bar, uint32_t bytes) {
  uint64_t state;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
               : "=l"(state)
               : "r"(smem_addr(bar)), "r"(bytes)
               : "memory");
  (void)state;
}
// phase with this parity complete? (acquire at cluster scope: the remote
// stores it counted are visible)
__device__ __forceinline__ bool mbar_done(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// the shared::cluster address of `local` in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* local, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_addr(local)), "r"(rank));
  return r;
}
// bulk copy (no multicast) of `bytes` (a multiple of 16, both addresses
// 16-byte aligned) from global into this CTA's shared memory, completing on
// the CTA's mbarrier `bar`
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(smem_dst)),
               "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void st_async_word(uint32_t raddr, uint32_t v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.u32 [%0], %1, [%2];" ::"r"(raddr), "r"(v),
               "r"(rbar)
               : "memory");
}

// 4 presynaptic ids of one lane's group (stored as pre ^ 31: the word index
// pre >> 5 is unchanged and the low 5 bits are 31 - (pre & 31), the left
// rotation that brings the neuron's bit to bit 31).
template <bool SRC16>
struct SrcGroup;
template <>
struct SrcGroup<true> {
  using T = uint2;
  __device__ static void split(T v, uint32_t* s) {
    s[0] = v.x & 0xffffu;
    s[1] = v.x >> 16;
    s[2] = v.y & 0xffffu;
    s[3] = v.y >> 16;
  }
};
template <>
struct SrcGroup<false> {
  using T = uint4;
  __device__ static void split(T v, uint32_t* s) {
    s[0] = v.x;
    s[1] = v.y;
    s[2] = v.z;
    s[3] = v.w;
  }
};

template <int KIND, bool HARD, bool USE_REF, bool FAST, int IDS>
__global__ void __launch_bounds__(kClThreads, 1) k_cluster_engine(bt_engine_desc d) {
  constexpr bool SRC16 = IDS == 0, DELAY = IDS == 2;
  extern __shared__ __align__(16) unsigned char cl_smem[];
  using Src = typename std::conditional<SRC16, uint16_t, uint32_t>::type;
  using G4 = typename SrcGroup<SRC16>::T;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = int(cluster.block_rank());
  const int CL = int(cluster.num_blocks());
  const int Tp = d.tile_posts;
  const int64_t n = d.n;
  const int B = int(d.batch);
  const int words = int((n + 31) >> 5);
  const int Wd = words + 1;
  const int64_t p0 = int64_t(rank) * Tp;
  const int tile_n = int(p0 + Tp <= n ? Tp : (p0 < n ? n - p0 : 0));  // posts of this tile
  const int NWv = (tile_n + 31) >> 5;                                  // its words
  const int w0 = int(p0 >> 5);                                         // its first word
  const int R = DELAY ? d.n_bins : 1;
  const int Hc = DELAY ? R + 1 : 2;  // bitmap copies
  const ClusterSmem L = cluster_smem(n, B, Tp, d.tile_rows, SRC16, Hc);
  const int g_max = int(d.tile_rows >> 2);  // groups of 4 rows the shared memory holds
  float* s_v = reinterpret_cast<float*>(cl_smem + L.state);
  float* s_psc = s_v + B * Tp;
  float* s_ref = s_psc + B * Tp;
  float* s_gk = s_ref + B * Tp;
  float* s_w = reinterpret_cast<float*>(cl_smem + L.w);
  Src* s_src = reinterpret_cast<Src*>(cl_smem + L.src);
  uint32_t* s_bits = reinterpret_cast<uint32_t*>(cl_smem + L.bits);
  int* s_gptr = reinterpret_cast<int*>(cl_smem + L.gptr);
  int* s_len = reinterpret_cast<int*>(cl_smem + L.len);
  int* s_deg = reinterpret_cast<int*>(cl_smem + L.deg);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int W = kClThreads / 32;
  const int H = d.hist_len;
  const bool traces = d.v_trace || d.psc_trace || d.ref_trace || d.gk_trace || d.spikes;

  // ---- load the tile: state, lengths, out-degrees; zero the bitmaps
  for (int q = threadIdx.x; q < B * Tp; q += kClThreads) {
    const int b = q / Tp, l = q - b * Tp;
    const bool in = l < tile_n;
    const int64_t g = int64_t(b) * n + p0 + l;
    s_v[q] = in ? d.v[g] : 0.0f;
    s_psc[q] = in ? d.psc[g] : 0.0f;
    s_ref[q] = (in && USE_REF) ? d.refractory[g] : 0.0f;
    s_gk[q] = (in && KIND == BT_NEURON_ALIF) ? d.g_k[g] : 0.0f;
  }
  // bitmaps: zero, but for the copies of the steps before the call that
  // delay bins read (steps -1 .. -(R - 1) in copies Hc - 1 .. Hc - R + 1),
  // which come from the history ring
  for (int q = threadIdx.x; q < Hc * B * Wd; q += kClThreads) {
    const int c = q / (B * Wd), rem = q - c * (B * Wd);
    const int b = rem / Wd, wi = rem - b * Wd;
    const int j = Hc - c;  // the copy of step -j
    uint32_t word = 0u;
    if (DELAY && j >= 1 && j <= R - 1 && wi < words)
      word = uint32_t(d.hist[(((d.t0 - j) % H) * B + b) * words + wi]);
    s_bits[q] = word;
  }
  for (int q = threadIdx.x; q < B; q += kClThreads)
    s_len[q] = d.sample_len ? int(min(int64_t(d.sample_len[q]), int64_t(INT32_MAX))) : INT32_MAX;
  for (int l = threadIdx.x; l < Tp; l += kClThreads) s_deg[l] = (d.outdeg && l < tile_n) ? d.outdeg[p0 + l] : 0;
  // the tile's in-edges: its packed block of each array, one bulk copy each,
  // completing on s_mbar[2]; its slice group offsets (clamped to the groups
  // the shared memory holds: the accesses stay in bounds whatever is passed)
  const int gstride = Tp / 32 + 1;
  for (int q = threadIdx.x; q <= NWv; q += kClThreads) s_gptr[q] = min(d.cl_gptr[rank * gstride + q], g_max);
  __shared__ __align__(8) uint64_t s_mbar[3];  // [0], [1]: the bitmap copies; [2]: the in-edge copies
  if (threadIdx.x == 0) {
    mbar_init(&s_mbar[2], 1);
    mbar_init_fence();
    const int ng = NWv ? min(d.cl_gptr[rank * gstride + NWv], g_max) : 0;
    const uint32_t bw = uint32_t(ng) * 128u * 4u, bs = uint32_t(ng) * 128u * uint32_t(sizeof(Src));
    mbar_arm(&s_mbar[2], bw + bs);
    if (ng) {
      const int64_t blk = int64_t(rank) * g_max * 128;  // the tile's first element
      bulk_load(s_w, d.cl_w + blk, bw, &s_mbar[2]);
      bulk_load(s_src, static_cast<const Src*>(d.cl_src) + blk, bs, &s_mbar[2]);
    }
  }
  const NeuronParams prm_u = load_params<KIND, USE_REF>(d.neuron, 0);
  const float pc_u = d.psc_uniform ? d.psc_coef_s : 0.0f;
  const Div dpt_u = make_div(d.psc_uniform ? d.psc_tau_s : 1.0f, d.psc_uniform && d.psc_fast_div, d.psc_rcp);
  // bitmap copy c's barrier counts the other CTAs' words of the steps k = c mod 2:
  // (words - NWv) words per sample.  Armed for steps 0 and 1 here; after the
  // wait for step s - 1, for step s + 1 -- before this CTA publishes step s,
  // which every sender of step s + 1 has to have received first.
  // a wait gave up somewhere in the cluster: every CTA stops waiting and
  // publishing, runs out its loop and meets the others at the final barrier
  __shared__ int s_dead;
  volatile int* dead = &s_dead;
  const uint32_t expect = uint32_t(4 * B * (words - NWv));
  if (threadIdx.x == 0) {
    mbar_init(&s_mbar[0], 1);
    mbar_init(&s_mbar[1], 1);
    mbar_init_fence();
    s_dead = 0;
    mbar_arm(&s_mbar[0], expect);
    if (d.n_steps > 1) mbar_arm(&s_mbar[1], expect);
  }
  const unsigned spin = d.spin_limit > 0 ? unsigned(d.spin_limit) : kClDefaultSpinLimit;
  cluster.sync();  // every CTA resident, its bitmaps zeroed and barriers armed before the first remote store
  // the in-edges have landed (bounded wait by one thread; then every thread's
  // own acquire of the completed phase)
  if (threadIdx.x == 0) {
    unsigned polls = 0;
    while (!mbar_done(&s_mbar[2], 0)) {
      if (++polls > spin) {
        if (d.tile_work) atomicCAS(d.tile_work + 2, 0, BT_ERR_TIMEOUT);
        for (int r = 0; r < CL; ++r) *reinterpret_cast<volatile int*>(cluster.map_shared_rank(&s_dead, r)) = 1;
        break;
      }
    }
  }
  __syncthreads();
  if (!*dead) (void)mbar_done(&s_mbar[2], 0);

  const int items = NWv * B;  // (word, sample) pairs of this tile; item it = (b, w) = divmod(it, NWv)
  int h_t = int(d.t0 % H);
  // the drive of the warp's first item, loaded one step ahead (behind the barrier)
  float x_ahead = 0.0f;
  auto drive = [&](int64_t kk, int it) -> float {
    const int b = it / NWv, l = (it - b * NWv) * 32 + lane;
    return (d.x && kk < d.n_steps && l < tile_n && kk < s_len[b]) ? __ldcs(d.x + (kk * B + b) * n + p0 + l) : 0.0f;
  };
  if (warp < items) x_ahead = drive(0, warp);
  int kc = 0, kp = Hc - 1;  // the copies of steps k and k - 1
  for (int64_t k = 0; k <= d.n_steps; ++k) {
    const bool last = k == d.n_steps;  // only the synapse update of step n_steps - 1
    const int cur = int(k & 1), prv = cur ^ 1;  // mbarriers by step parity
    if (k > 0) {
      // z_{k-1}: every CTA's words of step k - 1 in copy prv
      if (threadIdx.x == 0 && !*dead) {
        unsigned polls = 0;
        while (!mbar_done(&s_mbar[prv], uint32_t(((k - 1) >> 1) & 1))) {
          if (*dead) break;  // another CTA gave up
          if (++polls > spin) {
            if (d.tile_work) atomicCAS(d.tile_work + 2, 0, BT_ERR_TIMEOUT);
            for (int r = 0; r < CL; ++r) *reinterpret_cast<volatile int*>(cluster.map_shared_rank(&s_dead, r)) = 1;
            break;
          }
        }
        if (!*dead && k + 1 < d.n_steps) mbar_arm(&s_mbar[prv], expect);  // for step k + 1
      }
      __syncthreads();  // also orders this CTA's own words (plain stores) before they are read
    }
    long long st_un = 0, st_ev = 0;  // this lane's statistics of the step
    for (int it = warp; it < items; it += W) {
      const int b = it / NWv, w = it - b * NWv;
      const int l = w * 32 + lane;
      const bool valid = l < tile_n;
      const int64_t i = p0 + l;
      const int q = b * Tp + l;
      const int len = s_len[b];
      // the drive's load is issued first: its latency overlaps the in-edge sum
      const float xv = it == warp ? x_ahead : drive(k, it);
      float P = s_psc[q];
      if (k > 0 && k - 1 < len) {
        // ordered in-edge sum over z_{k-1-bin} (zero terms skipped: exact)
        const uint32_t* bits = s_bits + (kp * B + b) * Wd;
        const G4* srcg = reinterpret_cast<const G4*>(s_src);
        const float4* wg = reinterpret_cast<const float4*>(s_w);
        float g = 0.0f;
        const int ge = s_gptr[w + 1];
        // blocks of kClRows rows (kClRows / 4 groups): the ids, the bitmap
        // words and the weights of a block are loaded before its additions
        constexpr int NG = kClRows / 4;
        for (int gc = s_gptr[w]; gc < ge; gc += NG) {
          uint32_t sr[kClRows], rot[kClRows];
          float wv[kClRows];
#pragma unroll
          for (int j = 0; j < NG; ++j) {
            SrcGroup<SRC16>::split(srcg[(gc + j) * 32 + lane], sr + 4 * j);
            const float4 w4 = wg[(gc + j) * 32 + lane];
            wv[4 * j] = w4.x;
            wv[4 * j + 1] = w4.y;
            wv[4 * j + 2] = w4.z;
            wv[4 * j + 3] = w4.w;
          }
#pragma unroll
          for (int u = 0; u < kClRows; ++u) {
            uint32_t bw;
            if constexpr (DELAY) {
              int c = kp - int(sr[u] >> kClBinShift);  // the copy of step k - 1 - bin
              c += c < 0 ? Hc : 0;
              bw = s_bits[(c * B + b) * Wd + ((sr[u] & ((1u << kClBinShift) - 1u)) >> 5)];
            } else {
              bw = bits[sr[u] >> 5];
            }
            rot[u] = __funnelshift_l(bw, bw, sr[u]);
          }
#pragma unroll
          for (int u = 0; u < kClRows; ++u)
            if (int(rot[u]) < 0) g = add(g, wv[u]);
        }
        float pc = pc_u;
        Div dpt = dpt_u;
        if (valid && !d.psc_uniform) {
          pc = ld(d.psc_coef, i);
          dpt = make_div(ld(d.psc_tau, i), false, 0.0f);
        }
        P = add(psc_decay_k<FAST>(pc, dpt, P), g);
      }
      if (valid) {
        s_psc[q] = P;
        if (d.psc_trace && k > 0) d.psc_trace[((k - 1) * B + b) * n + i] = P;
      }
      if (last) continue;
      float s = 0.0f;
      if (valid) {
        float v = s_v[q], ref = s_ref[q], gk = s_gk[q];
        if (k < len) {
          NeuronParams prm = prm_u;
          if (!d.neuron.uniform) prm = load_params<KIND, USE_REF>(d.neuron, i);
          const float I = d.x ? add(P, xv) : P;
          s = neuron_update<KIND, HARD, USE_REF, true, FAST>(prm, I, v, ref, gk).spike;
          s_v[q] = v;
          if (USE_REF) s_ref[q] = ref;
          if (KIND == BT_NEURON_ALIF) s_gk[q] = gk;
        }
        if (traces) {
          const int64_t tix = (k * B + b) * n + i;
          if (d.v_trace) d.v_trace[tix] = v;
          if (USE_REF && d.ref_trace) d.ref_trace[tix] = ref;
          if (KIND == BT_NEURON_ALIF && d.gk_trace) d.gk_trace[tix] = gk;
          if (d.spikes) d.spikes[tix] = s;
        }
      }
      const uint32_t word = __ballot_sync(0xffffffffu, s != 0.0f);
      // publish: lane c stores the word into CTA c's copy (c = rank: its own)
      const int off = (kc * B + b) * Wd + w0 + w;
      if (lane == rank) s_bits[off] = word;
      else if (lane < CL && !*dead) st_async_word(cluster_addr(s_bits + off, lane), word, cluster_addr(&s_mbar[cur], lane));
      if (s != 0.0f) {
        st_ev += s_deg[l];
        st_un += 1;
      }
    }
    if (last) break;
    long long st_ed = st_ev;
    if (d.stats && B > 1) {
      // union and edges over samples from this tile's own words (events, the
      // per-sample sum, were counted above)
      __syncthreads();
      st_un = st_ed = 0;
      for (int l = threadIdx.x; l < tile_n; l += kClThreads) {
        uint32_t any = 0u;
        for (int b = 0; b < B; ++b) any |= s_bits[(kc * B + b) * Wd + w0 + (l >> 5)];
        if ((any >> (l & 31)) & 1u) {
          st_un += 1;
          st_ed += s_deg[l];
        }
      }
    }
    __syncwarp();
    // the history ring holds the last H steps: only those are written
    const bool hist = k + H >= d.n_steps;
    for (int it = warp; it < items; it += W) {
      const int b = it / NWv, w = it - b * NWv;
      if (lane == 0) {
        const uint32_t word = s_bits[(kc * B + b) * Wd + w0 + w];  // this warp's own store
        if (hist) d.hist[(int64_t(h_t) * B + b) * words + w0 + w] = word;
        if (d.raster) d.raster[(k * B + b) * words + w0 + w] = word;
      }
    }
    if (d.stats && (warp < items || B > 1)) {
      // warp sums in 32 bits: a step's counts are at most batch x synapses,
      // which a network that fits one cluster keeps below 2^32
      const unsigned un = __reduce_add_sync(0xffffffffu, unsigned(st_un));
      const unsigned ev = __reduce_add_sync(0xffffffffu, unsigned(st_ev));
      const unsigned ed = __reduce_add_sync(0xffffffffu, unsigned(st_ed));
      if (lane == 0) {
        unsigned long long* st = reinterpret_cast<unsigned long long*>(d.stats + k * 4);
        if (un) atomicAdd(st + 0, (unsigned long long)un);
        if (ev) atomicAdd(st + 1, (unsigned long long)ev);
        if (ed) atomicAdd(st + 2, (unsigned long long)ed);
      }
    }
    if (warp < items) x_ahead = drive(k + 1, warp);
    h_t = h_t + 1 == H ? 0 : h_t + 1;
    kp = kc;
    kc = kc + 1 == Hc ? 0 : kc + 1;
  }
  // every remote store into this CTA was waited for (the last iteration's
  // wait covers the last step); the barrier keeps every CTA resident until
  // all have left the loop, also when a wait gave up
  cluster.sync();
  for (int q = threadIdx.x; q < B * Tp; q += kClThreads) {
    const int b = q / Tp, l = q - b * Tp;
    if (l >= tile_n) continue;
    const int64_t g = int64_t(b) * n + p0 + l;
    d.v[g] = s_v[q];
    d.psc[g] = s_psc[q];
    if (USE_REF) d.refractory[g] = s_ref[q];
    if (KIND == BT_NEURON_ALIF) d.g_k[g] = s_gk[q];
  }
}

template <int KIND, bool HARD, bool USE_REF, bool FAST, int IDS>
int cluster_launch(const bt_engine_desc& d, cudaStream_t s) {
  void (*kern)(bt_engine_desc) = k_cluster_engine<KIND, HARD, USE_REF, FAST, IDS>;
  const int CL = d.n_tiles;
  const size_t smem = cluster_smem(d.n, d.batch, d.tile_posts, d.tile_rows, IDS == 0, cluster_copies(d.n_bins)).total;
  int dev = 0;
  cudaGetDevice(&dev);
  const bool known = launch_setup_known(reinterpret_cast<const void*>(kern), dev, smem, CL);
  if (!known && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(launch_smem_allow(reinterpret_cast<const void*>(kern), dev, smem))) !=
                    cudaSuccess)
    return bt_set_error(BT_ERR_UNSUPPORTED, "cluster engine: %zu bytes of shared memory refused", smem);
  if (!known && CL > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    return bt_set_error(BT_ERR_UNSUPPORTED, "cluster engine: clusters of %d CTAs refused", CL);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(CL));
  cfg.blockDim = dim3(kClThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = unsigned(CL);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (!known) {
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1)
      return bt_set_error(BT_ERR_UNSUPPORTED, "cluster engine: a cluster of %d CTAs with %zu bytes each does not fit",
                          CL, smem);
    launch_setup_add(reinterpret_cast<const void*>(kern), dev, smem, CL);
  }
  const cudaError_t err = cudaLaunchKernelEx(&cfg, kern, d);
  if (err != cudaSuccess) return bt_set_error(BT_ERR_CUDA, "cluster engine launch: %s", cudaGetErrorString(err));
  return BT_OK;
}

template <int KIND, bool HARD, bool USE_REF>
int cluster_pick(const bt_engine_desc& d, bool fast, cudaStream_t s) {
  switch (cluster_ids(d.n, d.n_bins)) {  // the encoding the packed ids were written in
    case 0:
      return fast ? cluster_launch<KIND, HARD, USE_REF, true, 0>(d, s) : cluster_launch<KIND, HARD, USE_REF, false, 0>(d, s);
    case 1:
      return fast ? cluster_launch<KIND, HARD, USE_REF, true, 1>(d, s) : cluster_launch<KIND, HARD, USE_REF, false, 1>(d, s);
    default:
      return fast ? cluster_launch<KIND, HARD, USE_REF, true, 2>(d, s) : cluster_launch<KIND, HARD, USE_REF, false, 2>(d, s);
  }
}

int run_cluster(const bt_engine_desc& d, bool fast, cudaStream_t s) {
  const bool h = d.neuron.hard_reset != 0, r = d.neuron.use_refractory != 0;
  if (d.neuron.kind == BT_NEURON_LIF) {
    if (h && r) return cluster_pick<BT_NEURON_LIF, true, true>(d, fast, s);
    if (h) return cluster_pick<BT_NEURON_LIF, true, false>(d, fast, s);
    if (r) return cluster_pick<BT_NEURON_LIF, false, true>(d, fast, s);
    return cluster_pick<BT_NEURON_LIF, false, false>(d, fast, s);
  }
  if (h && r) return cluster_pick<BT_NEURON_ALIF, true, true>(d, fast, s);
  if (h) return cluster_pick<BT_NEURON_ALIF, true, false>(d, fast, s);
  if (r) return cluster_pick<BT_NEURON_ALIF, false, true>(d, fast, s);
  return cluster_pick<BT_NEURON_ALIF, false, false>(d, fast, s);
}

}  // namespace bt

extern "C" int64_t bt_cluster_smem_bytes(int64_t n, int64_t batch, int32_t tile_posts, int64_t tile_rows,
                                         int32_t n_bins) {
  if (n <= 0 || batch <= 0 || tile_posts <= 0 || (tile_posts & 31) || tile_rows < 0 || (tile_rows & 3) ||
      n_bins < 1 || n_bins > 32 || (n_bins > 1 && n + 32 > (int64_t(1) << bt::kClBinShift)))
    return 0;
  return int64_t(bt::cluster_smem(n, batch, tile_posts, tile_rows, bt::cluster_ids(n, n_bins) == 0,
                                  bt::cluster_copies(n_bins))
                     .total);
}
