/*
 * btorch_b200.h -- C ABI of the B200-native recurrent spiking step.
 *
 * This is the drop-in boundary underneath the btorch module API
 * (SparseConn, LIF, ALIF, ExponentialPSC, DelayedPSC, HeterSynapsePSC,
 * RecurrentNN).  Every entry point takes plain pointers and sizes, never a
 * framework type.  Device pointers are raw CUDA global-memory addresses,
 * host pointers are ordinary process memory, and `stream` is a cudaStream_t
 * passed as void*.  No entry point allocates device memory or synchronises
 * the stream (except bt_layout_build, which is host-only), so every device
 * entry point can be captured in a CUDA graph.  Each returns a bt_status.
 *
 * Sparse layout conventions (shared by all entry points):
 *   canonical order  -- the reference's COO order: edges sorted by
 *                       (post, src) where src is the (possibly
 *                       delay-expanded) presynaptic row  pre*n_bins + bin
 *                       (btorch/models/linear.py:278-292,
 *                        btorch/connectome/connection.py:1021-1027).
 *                       `magnitude` is stored in this order.
 *   CSC (by post)    -- csc_ptr[n_post+1], csc_src[nnz] = packed
 *                       (pre | bin << BT_BIN_SHIFT), weights = magnitude.
 *   CSR (by pre)     -- csr_ptr[n_pre+1], csr_dst[nnz] = packed
 *                       (post | bin << BT_BIN_SHIFT), csr_perm[nnz] maps a
 *                       CSR position to its canonical index.
 *
 * Trust boundary: the device entry points check sizes, null pointers and
 * alignment, but read the contents of the layout arrays (row pointers,
 * packed ids) as indices without checking them on the device.  Pass arrays
 * made by bt_layout_build / bt_layout_slices, which reject COO indices that
 * are out of range or not canonical (BT_ERR_LAYOUT), with the sizes they were
 * built for, and weight arrays with one value per stored nonzero.
 *
 * Numerics: every elementwise update is evaluated op by op with IEEE
 * round-to-nearest single precision in the reference's operator order (no
 * contraction to FMA); the ordered gather accumulates each output in
 * ascending source order with fused multiply-add, which is how the
 * reference's CPU sparse product (torch.sparse.mm) rounds.
 */
#ifndef BTORCH_B200_H
#define BTORCH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BT_API __attribute__((visibility("default")))
#else
#define BT_API
#endif

#define BT_ABI_VERSION 11
#define BT_BIN_SHIFT 25              /* low 25 bits: neuron id, high 7: delay bin */
#define BT_MAX_NEURONS (1 << 25)
#define BT_MAX_BINS 128

typedef enum bt_status {
  BT_OK = 0,
  BT_ERR_INVALID = 1,      /* bad argument: the message names it */
  BT_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  BT_ERR_TIMEOUT = 3,      /* a bounded device-side wait gave up */
  BT_ERR_UNSUPPORTED = 4,  /* configuration the kernels do not implement */
  BT_ERR_LAYOUT = 5        /* COO indices out of range or not canonical */
} bt_status;

/* Text of the most recent error on the calling thread ("" if none). */
BT_API const char* bt_last_error(void);
BT_API int bt_abi_version(void);

/* ------------------------------------------------------------------ */
/* Static layout (host only).                                          */
/* Replaces preprocess_sparse  btorch/models/_sparse_preprocess.py:28-122 */
/* and BaseSparseConn._rebuild_triton_layout  linear.py:329-349.        */
/* ------------------------------------------------------------------ */

/* SELL-32 view of the CSC for BT_MODE_PULL: slice s = posts [32 s, 32 s + 32)
 * holds rows [sl_ptr[s], sl_ptr[s + 1]); row r stores the k-th in-edge of each
 * of its posts at [32 r + lane] (k = r - sl_ptr[s]); shorter posts are padded
 * with src = sentinel (a neuron id that never spikes) and perm = -1.
 * sl_src / sl_perm NULL: only fill sl_ptr and *rows_out (size query). */
BT_API int bt_layout_slices(int64_t n_post, const int32_t* csc_ptr,
                            const uint32_t* csc_src, uint32_t sentinel,
                            int64_t* sl_ptr, uint32_t* sl_src, int32_t* sl_perm,
                            int64_t capacity_rows, int64_t* rows_out);

/* Build CSC and CSR views of a canonical COO matrix in one O(nnz) pass.
 * post[e], src[e]: canonical COO (sorted by (post, src)); src is the
 * delay-expanded row index pre*n_bins + bin (n_bins = 1 for a plain
 * matrix).  Outputs are caller-allocated host arrays of the stated sizes.
 * Fails with BT_ERR_LAYOUT if an index is out of range or the order is not
 * canonical, BT_ERR_INVALID if nnz >= 2^31 or sizes exceed the packing. */
BT_API int bt_layout_build(int64_t nnz, const int64_t* post, const int64_t* src,
                    int64_t n_post, int64_t n_pre, int32_t n_bins,
                    int32_t* csc_ptr,   /* [n_post + 1] */
                    uint32_t* csc_src,  /* [nnz] pre | bin << 25 */
                    int32_t* csr_ptr,   /* [n_pre + 1] */
                    uint32_t* csr_dst,  /* [nnz] post | bin << 25 */
                    int32_t* csr_perm); /* [nnz] CSR position -> canonical */

/* ------------------------------------------------------------------ */
/* Event-driven sparse product  out = x @ W  for SparseConn.forward.   */
/* Replaces triton_sparse_mm / _launch_sparse_mm                        */
/* btorch/models/_sparse_triton.py:272-355,418-444.                     */
/* x: [batch, n_in] dense (graded values allowed), out: [batch, n_out]. */
/* ------------------------------------------------------------------ */

/* Pull: each output walks its in-edges in ascending source order and
 * accumulates x[b, src] * w with fmaf, skipping zero inputs.  Deterministic
 * and bit-identical to the reference's CPU product.  `bits` is scratch of
 * batch * ceil(n_in / 32) uint32 words. */
BT_API int bt_spmv_gather(int64_t batch, int64_t n_in, int64_t n_out,
                   const int32_t* csc_ptr, const uint32_t* csc_src,
                   const float* csc_w, const float* x, float* out,
                   uint32_t* bits, void* stream);

/* Push: nonzero inputs are compacted (warp ballot + prefix sum), then one
 * warp per active (sample, source) streams that source's out-edges with
 * 128-bit loads and adds into `out` with fp32 reductions in L2.  Order of
 * the additions is not fixed; exact whenever the partial sums are (dyadic
 * weights).  `work` is scratch of batch * n_in + 2 int32 words. */
BT_API int bt_spmv_scatter(int64_t batch, int64_t n_in, int64_t n_out,
                    const int32_t* csr_ptr, const uint32_t* csr_dst,
                    const float* csr_w, const float* x, float* out,
                    int32_t* work, void* stream);

/* Allocation-free bt_spmv_gather.  No counterpart in the reference: it exists
 * for callers that cannot allocate device memory when they need the product
 * (stream capture under a fixed memory plan, loops that must not take the
 * device-wide synchronisation of cudaMalloc/cudaFree, foreign-language hosts
 * with no device allocator).  Same arguments and result as bt_spmv_gather
 * without `bits`: the scratch is a file-scope device array of
 * BT_NOALLOC_GATHER_MAX_WORDS uint32 words (1 MiB) that every GPU loading the
 * library holds until exit.  batch * ceil(n_in / 32) above that limit is
 * rejected with BT_ERR_INVALID.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress with that device current);
 * make that first call before any stream capture.  The address is cached
 * per device for the life of the process and is not refreshed after
 * cudaDeviceReset or a re-created primary context: do not call this entry
 * point across such a reset.  Every call shares the one array: calls that
 * overlap on the GPU (other streams, other threads) race and must be
 * serialised by the caller.  x may be NULL when n_in == 0.  Nothing is
 * allocated or freed. */
#define BT_NOALLOC_GATHER_MAX_WORDS (1 << 18)
BT_API int bt_spmv_gather_noalloc(int64_t batch, int64_t n_in, int64_t n_out,
                                  const int32_t* csc_ptr, const uint32_t* csc_src,
                                  const float* csc_w, const float* x, float* out,
                                  void* stream);

/* Backward of the product (replaces _TritonSparseMM.backward
 * btorch/models/_sparse_triton.py:389-415).
 * grad_x[b, j] = sum over out-edges (j -> i) of w * grad_out[b, i]:
 * a transpose gather in ascending post order, deterministic. */
BT_API int bt_spmv_grad_input(int64_t batch, int64_t n_in, int64_t n_out,
                       const int32_t* csr_ptr, const uint32_t* csr_dst,
                       const float* csr_w, const float* grad_out,
                       float* grad_x, void* stream);

/* The same product through grad_out transposed into `work` (batch * n_out
 * floats, caller scratch): every edge then reads one contiguous run of
 * samples instead of one scattered word per sample.  Each grad_x[b, j] is
 * an fmaf chain over j's out-edges in CSR order (deterministic; rounding
 * differs from bt_spmv_grad_input's lane-split sum). */
BT_API int bt_spmv_grad_input_t(int64_t batch, int64_t n_in, int64_t n_out,
                       const int32_t* csr_ptr, const uint32_t* csr_dst,
                       const float* csr_w, const float* grad_out,
                       float* grad_x, float* work, void* stream);

/* grad_w[canonical e = (j -> i)] = sum_b x[b, j] * grad_out[b, i], over
 * stored nonzeros only and only over samples whose input x[b, j] is nonzero
 * (ascending b, fmaf); entries whose source is silent in every sample are
 * written as 0.  Written in canonical order (coalesced), deterministic.
 * `masks` is scratch of n_in * ceil(batch / 32) uint32 words. */
BT_API int bt_spmv_grad_weight(int64_t batch, int64_t n_in, int64_t n_out,
                        const int32_t* csc_ptr, const uint32_t* csc_src,
                        const float* x, const float* grad_out, float* grad_w,
                        uint32_t* masks, void* stream);

/* ------------------------------------------------------------------ */
/* Neuron and synapse parameter descriptors.                           */
/* ------------------------------------------------------------------ */

/* A per-neuron parameter: value(i) = ptr[i * stride]; stride 0 = scalar. */
typedef struct bt_param {
  const float* ptr;
  int64_t stride;
} bt_param;

#define BT_NEURON_LIF 0
#define BT_NEURON_ALIF 1

/* LIF (btorch/models/neurons/lif.py:29-200) and ALIF
 * (btorch/models/neurons/alif.py:30-268) through
 * BaseNode.single_step_forward (btorch/models/base.py:1108-1116). */
typedef struct bt_neuron_desc {
  int32_t kind;            /* BT_NEURON_LIF / BT_NEURON_ALIF */
  int32_t hard_reset;      /* 1: v -= (v - v_reset) * s; 0: v -= (v_th - v_reset) * s */
  int32_t use_refractory;  /* tau_ref given */
  int32_t spiking;         /* 1: Heaviside forward; 0: sigmoid(k*alpha*u) (smooth) */
  float dt;                /* environ dt, as fp32 */
  float sg_alpha;          /* surrogate alpha * 2 ln(1 + sqrt 2), as fp32 */
  float sg_damping;        /* surrogate damping factor */
  float pad_;
  bt_param v_threshold, v_reset, c_m;
  bt_param tau;            /* LIF membrane time constant */
  bt_param tau_ref;
  bt_param g_leak, E_leak, E_k, dg_k, tau_adapt; /* ALIF */
  bt_param coef_gk;        /* ALIF: expm1(dt * (-1/tau_adapt)) / (-1/tau_adapt), host-rounded */
  /* When every parameter above is a scalar (stride 0) the caller may set
     uniform = 1 and copy the values into sv[] = {v_threshold, v_reset, c_m,
     tau, tau_ref, g_leak, E_leak, E_k, dg_k, tau_adapt, coef_gk} (unused
     entries 0): the kernels then read no parameter memory.  The copies must
     equal the pointed-to values. */
  int32_t uniform;
  float sv[11];
  /* With uniform = 1: bit k of fast_div says that x / divisor_k equals
     fma(fma(-q, c, x), rcp[k], q) with q = x * rcp[k] for every fp32 x that
     gives 2^-100 <= |q| <= 2^100 (IEEE division otherwise), as verified for
     that divisor by bt_fast_div_check; divisors {c_m, v_threshold - v_reset,
     tau, tau_adapt}, rcp = the correctly rounded reciprocal. */
  int32_t fast_div;
  float rcp[4];
} bt_neuron_desc;

/* One BaseNode.single_step_forward (charge -> adaptation -> fire -> reset),
 * one launch.  x: input current [batch, n].  State inputs v_in, ref_in
 * (NULL unless use_refractory), gk_in (ALIF only) and the matching outputs
 * are [batch, n]; an output may alias its input (in-place update).
 * spike: [batch, n] output.  Saved for the surrogate backward (each may be
 * NULL): u_save = (v_charged - v_th) / (v_th - v_reset), mask_save = 1 where
 * the neuron was not refractory, vch_save = v after charge. */
BT_API int bt_neuron_step(const bt_neuron_desc* d, int64_t batch, int64_t n,
                   const float* x, const float* v_in, const float* ref_in,
                   const float* gk_in, float* v_out, float* ref_out,
                   float* gk_out, float* spike, float* u_save,
                   float* mask_save, float* vch_save, void* stream);

/* Surrogate-gradient backward of one neuron step (sigmoid surrogate
 * btorch/models/surrogate/sigmoid.py:23-29; reset as in
 * btorch/models/neurons/lif.py:170-187, alif.py:230-249).  Inputs: the
 * step's input current x, grads of
 * the step outputs g_spike, g_v_new, g_gk_new (each may be NULL = 0) and the
 * forward's saved u, spike, mask, v_charged plus v_prev / gk_prev.  Outputs:
 * g_x (input current), g_v_prev, g_gk_prev (ALIF; may be NULL).  The
 * refractory counter only feeds a detached comparison, so it carries no
 * gradient into the spike path. */
BT_API int bt_neuron_step_backward(const bt_neuron_desc* d, int64_t batch, int64_t n,
                            const float* x, const float* g_spike, const float* g_v_new,
                            const float* g_gk_new, const float* u_save,
                            const float* spike, const float* mask_save,
                            const float* v_charged, const float* v_prev,
                            const float* gk_prev, float* g_x,
                            float* g_v_prev, float* g_gk_prev,
                            int32_t detach_reset, void* stream);

/* Validate a neuron descriptor without launching anything. */
BT_API int bt_check_neuron_desc(const bt_neuron_desc* d);

/* Exhaustive check of the reciprocal division for one divisor c (finite,
 * nonzero) with rcp = the correctly rounded 1/c: over all 2^32 fp32 bit
 * patterns x, sets *mismatches (device int32, zeroed by the caller) to 1 if
 * the fast quotient of any x (as in bt_neuron_desc.fast_div) differs from the
 * IEEE quotient x / c (NaN results compare equal).  0 makes the fast path
 * bit-identical to division for that divisor.  About 2 ms on one B200;
 * asynchronous on `stream`. */
BT_API int bt_fast_div_check(float c, float rcp, int32_t* mismatches, void* stream);

/* Exponential PSC step (btorch/models/synapse.py:99-103,171-178):
 * out = psc + coef * ((-psc) / tau_syn), then out = out + wz (wz may be
 * NULL).  out may alias psc.  Because the decay is linear, the same call
 * with wz = NULL applied to a gradient is the decay's backward. */
BT_API int bt_psc_step(int64_t batch, int64_t n, bt_param coef, bt_param tau_syn,
                const float* psc, const float* wz, float* out, void* stream);

/* ------------------------------------------------------------------ */
/* Fused multi-step engine for RecurrentNN                             */
/* (btorch/models/rnn.py:517-528 driven by rnn.py:200-332).            */
/* ------------------------------------------------------------------ */

#define BT_MODE_SCATTER 0  /* push: 2 launches per step, L2 fp32 reductions */
#define BT_MODE_GATHER 1   /* pull, warp per post: 1 launch per step, ordered, bit-exact */
#define BT_MODE_PULL 2     /* pull over SELL-32 slices, lane per post, sample masks:
                              1 launch per step, ordered, bit-exact, for batches */
#define BT_MODE_TILE 3     /* persistent: one launch for all n_steps, one CTA per tile
                              of posts with its synaptic input in shared memory, a
                              bounded grid barrier per step; single delay bin 0 */
#define BT_MODE_CLUSTER 4  /* persistent, small networks: one launch for all n_steps,
                              one thread-block cluster of n_tiles <= 16 CTAs holds
                              state and in-edges in shared memory, ordered in-edge
                              sums (bit-exact), spike words exchanged through
                              distributed shared memory (asynchronous stores counted
                              on mbarriers, bounded waits); delay bins up to 32, no
                              receptor channels */

typedef struct bt_engine_desc {
  /* sizes */
  int64_t n;              /* neurons */
  int64_t batch;          /* samples */
  int32_t n_bins;         /* delay bins R: a spike at step s through an edge
                             with bin d reaches the PSC of step s + d */
  int32_t mode;           /* BT_MODE_SCATTER / BT_MODE_GATHER */
  int64_t t0;             /* absolute index of the first step of this call */
  int64_t n_steps;        /* steps in this call */
  int32_t bin_lo;         /* scatter: lowest and highest delay bin that holds */
  int32_t bin_hi;         /*   edges (0 <= bin_lo <= bin_hi < n_bins)        */
  int32_t hist_len;       /* H: slots of the spike-history bitmap ring (>= n_bins + 2) */
  int32_t scatter_lanes;  /* scatter: lanes per active row, 8 or 32, or 1 = the 32
                             rows of a warp walked as one flattened edge range
                             (short rows); 0 = 32 */

  bt_neuron_desc neuron;
  bt_param psc_coef, psc_tau;  /* ExponentialPSC decay, per PSC column (n * n_rec) */

  /* connectivity (n_pre == n).  Scatter: CSR over the rows pre * n_bins + bin
     of the delay-expanded matrix, csr_dst = post, both edge arrays 16-byte
     aligned and padded to a multiple of 4.  Gather: CSC by post with
     csc_src = pre | bin << BT_BIN_SHIFT. */
  const int32_t* csr_ptr; const uint32_t* csr_dst; const float* csr_w;
  const int32_t* csc_ptr; const uint32_t* csc_src; const float* csc_w;

  /* state [batch, n], updated in place; psc is [batch, n * n_rec] (column
     post * n_rec + r: the base PSC of HeterSynapsePSC) */
  float* v; float* refractory; float* g_k; float* psc;
  float* ring;            /* [batch][n * n_rec] scatter: synaptic input W z accumulated
                             for the next neuron step (zero between runs) */
  uint32_t* hist;         /* [hist_len][batch][words] spike bitmaps, slot = step mod H */

  /* inputs */
  const float* x;         /* [n_steps][batch][n] input current (already projected) */
  const int32_t* sample_len; /* [batch] steps each sample runs (absolute, from step 0); NULL = all */

  /* outputs (any may be NULL) */
  uint32_t* raster;       /* [n_steps][batch][words] spike bitmaps */
  float* spikes;          /* [n_steps][batch][n] spikes as fp32 (reference output layout) */
  float* v_trace;         /* [n_steps][batch][n] v after each step */
  float* psc_trace;       /* [n_steps][batch][n * n_rec] psc after each step */
  float* ref_trace;       /* [n_steps][batch][n] refractory after each step */
  float* gk_trace;        /* [n_steps][batch][n] g_k after each step (ALIF) */

  /* sliced post-major view and sample masks (pull mode) */
  const int64_t* sl_ptr;  /* [ceil(n/32) + 1] first row of each 32-post slice */
  const uint32_t* sl_src; /* [rows * 32] pre | bin << 25, pre = n on padding */
  const float* sl_w;      /* [rows * 32] weights, 0 on padding */
  uint32_t* masks;        /* [hist_len][n + 1][S] spikes of each neuron by sample (bit l
                             of word q = sample 32 q + l), slot = step mod hist_len,
                             row n stays 0; S = bt_mask_stride(batch) */
  const int32_t* outdeg;  /* [n] out-degrees, for the stats of pull mode (may be NULL) */
  int32_t pull_words_per_warp; /* pull mode: 32-sample mask words one warp covers:
                                  0 or 1 = one word per warp (default), or the whole
                                  bt_mask_stride(batch) when that is 2 or 4 */
  int32_t neuron_spt;     /* scatter: samples per thread of the neuron launch, 1, 2 or 4
                             (0 = 4) */

  /* scratch (scatter mode) */
  int32_t* work;          /* bt_engine_work_words(n, batch, n_bins) int32: the spike
                             sets (active lists and sample masks) of the last
                             n_bins steps; bt_engine_prime initialises it */
  int64_t* stats;         /* [n_steps][4]: active union, events, edges, 0; may be NULL */

  /* scatter with a single delay bin (bin_lo == bin_hi): a step whose spike
     set lists at least dense_rows neurons is delivered by a dense pull over
     the sliced in-edge view sl_ptr / sl_src / sl_w instead (lane per post,
     ascending in-edge order, plain stores), 0 = never */
  int64_t dense_rows;
  /* scalar PSC coefficients (psc_coef, psc_tau of stride 0): psc_uniform = 1
     and their values, which must equal the pointed-to ones */
  int32_t psc_uniform;
  float psc_coef_s, psc_tau_s;
  int32_t psc_fast_div;   /* 1: psc_tau verified as above, reciprocal psc_rcp */
  float psc_rcp;
  int32_t n_rec;          /* receptor channels per neuron, C (0 or 1: none; at most 16;
                             scatter and gather modes): the matrix has n * C columns,
                             post * C + r, and the neuron's input is the sum of its C
                             PSCs in torch's CPU row-sum order (HeterSynapsePSC with
                             n_receptor = C, btorch/models/synapse.py:626-847) */
  /* scatter: the expanded CSR's edges interleaved, [2 * len(csr_dst)] words:
     post, weight bits, post, weight bits, ... (one 8-byte record per edge, so
     a short row occupies the fewest memory sectors); 16-byte aligned */
  const uint32_t* csr_edges;

  /* tile mode (BT_MODE_TILE, no counterpart in the reference: its time loop
     launches per step).  Tile t owns posts [t * tile_posts, (t + 1) *
     tile_posts); tile_posts is a multiple of 32 and n_tiles the number of
     tiles covering n, all co-resident (at most one per SM for large tiles).
     tile_off: [n][n_tiles + 1] from bt_tile_offsets (the CSR row of each
     source split at the tile boundaries).  tile_work:
     bt_tile_work_words(batch, tile_posts, n_tiles) int32 words, 64-byte
     aligned, whose first 32 are zero before the first call; word 2 is the status word, nonzero
     (BT_ERR_TIMEOUT) after a grid barrier wait gave up -- the caller reads
     it after the call and clears the first 32 words before reusing them.
     spin_limit: polls of one barrier wait before it gives up (0 = about a
     second). */
  int32_t tile_posts;
  int32_t n_tiles;
  const int32_t* tile_off;
  int32_t* tile_work;
  int32_t spin_limit;
  /* cluster mode (BT_MODE_CLUSTER, no counterpart in the reference): rank t
     of the cluster owns posts [t * tile_posts, (t + 1) * tile_posts), n_tiles
     <= 16 CTAs cover n (one launch per call, no final launch, no ring).  The
     tiles' in-edges are packed as the kernel keeps them in shared memory and
     copied there with one bulk copy per array:
       tile_rows  rows per tile (the SELL-32 rows of its slices, each slice
                  rounded up to a multiple of 16), a multiple of 16;
       cl_w       [n_tiles][tile_rows / 4][32][4] fp32: group g, lane l, u =
                  the weight of row 4 g + u of lane l's post, 0 on padding;
       cl_src     the same shape, the presynaptic id XOR 31 (padding: n XOR
                  31), uint16 when n + 32 <= 65536, else uint32; with
                  delay bins (n_bins > 1, n + 32 <= 2^20) uint32, the id
                  XOR 31 in bits 0..19 and the edge's bin in bits 20..24;
       cl_gptr    [n_tiles][tile_posts / 32 + 1] int32: the first group of each
                  of the tile's 32-post slices, then the tile's group count;
     all three 16-byte aligned.  tile_work: 32 int32 words, word 2 the status
     (nonzero after a wait gave up), zero before the call. */
  int64_t tile_rows;
  const float* cl_w;
  const void* cl_src;
  const int32_t* cl_gptr;
} bt_engine_desc;

/* Cluster mode shared memory per CTA (0 for a bad shape): n neurons, a
   tile of tile_posts posts (a multiple of 32) holding tile_rows slice rows
   (a multiple of 16), n_bins delay bins (1..32). */
BT_API int64_t bt_cluster_smem_bytes(int64_t n, int64_t batch, int32_t tile_posts, int64_t tile_rows,
                                     int32_t n_bins);

/* Tile mode scratch words and shared memory bytes per CTA for a shape
   (0 for a bad shape). */
BT_API int64_t bt_tile_work_words(int64_t batch, int32_t tile_posts, int32_t n_tiles);
BT_API int64_t bt_tile_smem_bytes(int64_t batch, int32_t tile_posts, int32_t n_tiles);

/* off[r][t] (r < rows, t <= n_tiles) = the first edge of CSR row r whose post
   is >= t * tile_posts; rows must be sorted by post (bt_layout_build's CSR
   is).  csr_edges: the interleaved (post, weight) records of
   bt_engine_desc.csr_edges. */
BT_API int bt_tile_offsets(int64_t rows, const int32_t* csr_ptr, const uint32_t* csr_edges,
                           int32_t tile_posts, int32_t n_tiles, int32_t* off, void* stream);

/* Weight gradient of the input layer (replaces the autograd of the
 * reference's DenseConn / nn.Linear, btorch/models/linear.py:163-228):
 * out[c][i] (+)= sum over rows r with x[r][c] != 0, ascending, of
 * x[r][c] * g[r][i] (fmaf chain), for x [rows][c_in] and the projection's
 * gradient g [rows][n]; out is the gradient of the transposed weight
 * [c_in][n]; accumulate != 0 adds to it.  `work`: c_in * (rows + 1) int32. */
BT_API int bt_input_grad_weight(int64_t rows, int64_t c_in, int64_t n, const float* x, const float* g,
                                float* out, int32_t accumulate, int32_t* work, void* stream);

/* Scratch words (int32) the scatter mode needs in bt_engine_desc.work. */
BT_API int64_t bt_engine_work_words(int64_t n, int64_t batch, int32_t n_bins);

/* Run n_steps recurrent steps.  Per step: I = psc + x; neuron update;
 * psc = psc + coef*((-psc)/tau) + sum over delay bins d of W_d z_{t-d}.
 * Scatter mode needs bt_engine_prime once per run. */
BT_API int bt_engine_run(const bt_engine_desc* d, void* stream);

/* Start a run in scatter mode (no-op in the other modes): clear work and
 * ring, and list the spikes of steps t0 - bin_hi .. t0 - 1 (read from the
 * hist bitmaps, slot = step mod hist_len) in their spike sets, so that their
 * arrivals at steps >= t0 are delivered.  Call once before the first
 * bt_engine_run of a run; later calls that continue the run (t0 advanced by
 * the previous n_steps) must not prime again.  Replaces the reference's
 * rebuild of the flattened delay history (btorch/models/history.py:299-345)
 * at the start of a multi-step call. */
BT_API int bt_engine_prime(const bt_engine_desc* d, void* stream);

/* Input projection for DenseConn as neuron_inp_module (nn.Linear,
 * btorch/models/linear.py:163-228): out[r, i] = bias[i] + sum over nonzero
 * xin[r, c] (ascending c) of xin[r, c] * w_t[c, i].  rows = steps*batch;
 * w_t: [c_in, n] (transpose of the module weight); bias may be NULL.
 * work: scratch of rows * (2 * c_in + 1) int32, 8-byte aligned. */
BT_API int bt_input_project(int64_t rows, int64_t c_in, int64_t n,
                     const float* xin, const float* w_t, const float* bias,
                     float* out, int32_t* work, void* stream);

/* bt_input_project over steps * batch rows (row t * batch + b) that skips the
 * steps of finished samples: rows with t >= sample_len[b] (this call's steps,
 * as bt_engine_desc.sample_len) are neither scanned nor written -- the engine
 * does not read them.  Same work scratch. */
BT_API int bt_input_project_live(int64_t steps, int64_t batch, int64_t c_in, int64_t n,
                     const float* xin, const float* w_t, const float* bias,
                     const int32_t* sample_len, float* out, int32_t* work, void* stream);

/* Expand spike bitmaps [rows][words] to fp32 [rows][n] (words = ceil(n/32),
 * bit i%32 of word i/32 is neuron i). */
BT_API int bt_bits_to_float(int64_t rows, int64_t n, const uint32_t* bits,
                     float* out, void* stream);

/* Words per neuron of the pull engine's sample masks: ceil(batch/32) rounded
 * up to 1, 2 or 4 (the kernel's vector load width), unchanged above 4. */
BT_API int bt_mask_stride(int64_t batch);

/* [batch][n] fp32 <-> sample masks [n][bt_mask_stride(batch)] (bit l of word q
 * set where sample 32 q + l is nonzero) -- the pull engine's history layout. */
BT_API int bt_float_to_masks(int64_t batch, int64_t n, const float* in,
                             uint32_t* masks, void* stream);
BT_API int bt_masks_to_float(int64_t batch, int64_t n, const uint32_t* masks,
                             float* out, void* stream);

/* Pack fp32 rows [rows][n] into bitmaps (bit set where the value != 0). */
/* Spike rasters as sparse coordinates (replaces the dense np.nonzero of the
 * reference's to_sparse_repr, btorch/io/serialization.py:80-141, for spike
 * stacks).  bits: [rows = T * batch][ceil(n/32)] bitmask raster.
 * bt_raster_count: counts[r] = spikes in row r.  bt_raster_coords: with
 * offsets = exclusive scan of counts, writes the (time, batch, neuron)
 * coordinates of every spike, row-major (time, then batch, then ascending
 * neuron), as int32. */
BT_API int bt_raster_count(int64_t rows, int64_t n, const uint32_t* bits, int64_t* counts, void* stream);
BT_API int bt_raster_coords(int64_t rows, int64_t batch, int64_t n, const uint32_t* bits,
                            const int64_t* offsets, int32_t* idx_time, int32_t* idx_batch,
                            int32_t* idx_neuron, void* stream);

BT_API int bt_float_to_bits(int64_t rows, int64_t n, const float* in,
                     uint32_t* bits, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BTORCH_B200_H */
