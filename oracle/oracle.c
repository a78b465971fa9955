/*
 * oracle.c -- CPU restatement of btorch's recurrent spiking step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product
 * is compared against (tests/, __graft_entry__.smoke, bench.py's CPU
 * baseline and --impl reference arm).  Nothing in btorch_b200/ links or
 * calls it.
 *
 * It restates, in the reference's operator order and rounding:
 *   - the native sparse product  (btorch/models/linear.py:474-483:
 *     torch.sparse.mm over canonical (post, src) COO; each output is a
 *     fused-multiply-add chain over its in-edges in ascending source order,
 *     zero inputs included -- verified against the reference in this repo's
 *     golden fixtures);
 *   - LIF   (btorch/models/neurons/lif.py:144-187) via euler_step
 *     (btorch/models/ode.py:53-55);
 *   - ALIF  (btorch/models/neurons/alif.py:193-249) via exp_euler_step
 *     (btorch/models/ode.py:20-50);
 *   - BaseNode.single_step_forward (btorch/models/base.py:1108-1116);
 *   - ExponentialPSC (btorch/models/synapse.py:99-103,171-178);
 *   - delays: DelayedPSC (synapse.py:537-623, uniform delay through
 *     SpikeHistory.get_delay, history.py:252-281) and HeterSynapsePSC
 *     (synapse.py:626-761 with expand_conn_for_delays rows pre*D + d,
 *     connection.py:973-1027, and SpikeHistory.get_flattened,
 *     history.py:299-345);
 *   - RecurrentNN.single_step_forward (btorch/models/rnn.py:517-528):
 *     I = psc + x; z = neuron(I); psc = decay(psc) + W z_delayed;
 *   - receptor channels of HeterSynapsePSC (synapse.py:626-847): C PSC
 *     columns per neuron (post * C + r, each with its own coefficients), the
 *     neuron's input the sum of its C columns in the order torch's CPU sum
 *     reduces a contiguous row (synapse.py:744-747).
 * Every torch op is one correctly rounded fp32 op here; the file must be
 * compiled with -ffp-contract=off so that no multiply-add is fused.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Hot loops are compiled twice, with and without the FMA instruction set,
 * and the loader picks the variant the host supports.  fmaf is correctly
 * rounded either way; only its speed differs (a libm call per element
 * without FMA).  Contraction stays off, so no other multiply-add fuses. */
#if defined(__x86_64__) && defined(__GNUC__) && !defined(__clang__) && !defined(__SANITIZE_ADDRESS__)
#define ORC_HOT __attribute__((target_clones("fma", "default")))
#else
#define ORC_HOT
#endif

typedef struct orc_net {
  int64_t n, batch, steps;
  int32_t kind;        /* 0 LIF, 1 ALIF */
  int32_t hard_reset;
  int32_t use_ref;
  int32_t max_delay;   /* largest edge delay in steps (0 = none) */
  float dt;
  /* per-neuron parameters, each an array of n floats */
  const float *vth, *vr, *cm, *tau, *tau_ref;
  const float *g_leak, *E_leak, *E_k, *dg_k, *tau_adapt, *coef_gk;
  const float *psc_coef, *psc_tau;
  /* connectivity, canonical CSC by post: in-edges of i are
   * [ptr[i], ptr[i+1]) in ascending (pre, delay) order */
  const int64_t* ptr;
  const int32_t* pre;
  const int32_t* delay;
  const float* w;
  /* input current [steps][batch][n]; may be NULL (zero input) */
  const float* x;
  const int32_t* sample_len; /* [batch] or NULL */
  /* state [batch][n], updated in place */
  float *v, *ref, *gk, *psc;
  /* spike history [max_delay + 1][batch][n]: slot (t mod H) = z_t */
  float* hist;
  int64_t t0;          /* absolute index of the first step (history slots) */
  /* outputs (any may be NULL) */
  uint8_t* spikes;     /* [steps][batch][n] */
  float* v_trace;      /* [steps][batch][n] */
  float* psc_trace;    /* [steps][batch][n * n_rec] */
  int32_t threads;
  int32_t n_rec;       /* receptor columns per neuron (0 or 1: none); psc, psc_coef,
                          psc_tau and the columns of ptr are then n * n_rec wide */
  /* Event-driven synapse phase (orc_run_events): the same edges by source
   * row r = pre * (max_delay + 1) + delay, rows ascending, each row's edges
   * [row_ptr[r], row_ptr[r+1]) as (PSC column, weight). */
  const int64_t* row_ptr;
  const int32_t* row_col;
  const float* row_w;
  float* acc;          /* [batch][n * n_rec] scratch */
  uint64_t* zmask;     /* [max_delay + 1][n][ceil(batch / 64)]: hist as sample bit masks */
} orc_net;

static inline float relu_keep_nan(float x) { return (x != x) ? x : (x > 0.0f ? x : 0.0f); }

/* Sum of C floats in torch's CPU order for a contiguous row (C < 4: left to
 * right; 4 <= C < 8: four accumulators, the rest folded into the first in
 * turn; C >= 8: eight accumulators over whole groups of 8, the tail's sum
 * added to the first), as the reference's .sum(-1) over receptors rounds. */
static float receptor_sum(const float* p, int C) {
  if (C < 4) {
    float s = p[0];
    for (int r = 1; r < C; ++r) s = s + p[r];
    return s;
  }
  if (C < 8) {
    float a0 = p[0];
    for (int r = 4; r < C; ++r) a0 = a0 + p[r];
    return ((a0 + p[1]) + p[2]) + p[3];
  }
  const int full = C & ~7;
  float a[8];
  for (int j = 0; j < 8; ++j) a[j] = p[j];
  for (int r = 8; r < full; ++r) a[r & 7] = a[r & 7] + p[r];
  if (full < C) {
    float t = p[full];
    for (int r = full + 1; r < C; ++r) t = t + p[r];
    a[0] = a[0] + t;
  }
  float s = a[0];
  for (int j = 1; j < 8; ++j) s = s + a[j];
  return s;
}

ORC_HOT static void neuron_phase(const orc_net* d, int64_t k, int64_t lo, int64_t hi) {
  const int64_t n = d->n, B = d->batch, H = d->max_delay + 1;
  const int64_t t = d->t0 + k;
  const float dt = d->dt;
  const int64_t W64 = (B + 63) >> 6;
  uint64_t* zm = d->zmask ? d->zmask + (t % H) * n * W64 : NULL;
  if (zm) memset(zm + lo * W64, 0, sizeof(uint64_t) * (size_t)((hi - lo) * W64));
  for (int64_t b = 0; b < B; ++b) {
    const int live = !d->sample_len || k < d->sample_len[b];
    float* hrow = d->hist + ((t % H) * B + b) * n;
    for (int64_t i = lo; i < hi; ++i) {
      const int64_t idx = b * n + i;
      float s = 0.0f;
      if (live) {
        const int C = d->n_rec > 1 ? d->n_rec : 1;
        const float P = C > 1 ? receptor_sum(d->psc + idx * C, C) : d->psc[idx];
        const float I = d->x ? P + d->x[(k * B) * n + idx] : P;
        float v = d->v[idx];
        const float vth = d->vth[i], vr = d->vr[i], cm = d->cm[i];
        float v1;
        float gk = 0.0f;
        if (d->kind == 0) {
          /* v + dt * ((-(v - v_reset)) / tau + x / c_m) */
          const float a = (-(v - vr)) / d->tau[i];
          const float c = I / cm;
          const float der = a + c;
          const float step = dt * der;
          v1 = v + step;
        } else {
          gk = d->gk[idx];
          const float ngl = -d->g_leak[i];
          const float leak = ngl * (v - d->E_leak[i]);
          const float adapt = (-gk) * (v - d->E_k[i]);
          const float s1 = leak + adapt;
          const float s2 = s1 + I;
          const float der = s2 / cm;
          const float lin = (ngl - gk) / cm;
          const float e = expm1f(dt * lin);
          const float coef = e / lin;
          const float step = coef * der;
          v1 = v + step;
          /* neuronal_adaptation: g_k + coef_gk * ((-g_k) / tau_adapt) */
          const float dg = (-gk) / d->tau_adapt[i];
          gk = gk + d->coef_gk[i] * dg;
        }
        /* fire: Heaviside((v - v_th) / (v_th - v_reset)) * (refractory == 0) */
        const float den = vth - vr;
        const float u = (v1 - vth) / den;
        s = (u >= 0.0f) ? 1.0f : 0.0f;
        float r = 0.0f;
        if (d->use_ref) {
          r = d->ref[idx];
          s = s * ((r == 0.0f) ? 1.0f : 0.0f);
        }
        /* reset */
        if (d->hard_reset) {
          const float dv = (v1 - vr) * s;
          v = v1 - dv;
        } else {
          const float dv = den * s;
          v = v1 - dv;
        }
        if (d->kind == 1) {
          const float inc = d->dg_k[i] * s;
          gk = gk + inc;
          d->gk[idx] = gk;
        }
        if (d->use_ref) {
          const float add = s * d->tau_ref[i];
          const float r1 = r + add;
          d->ref[idx] = relu_keep_nan(r1 - dt);
        }
        d->v[idx] = v;
      }
      hrow[i] = s;
      if (zm && s != 0.0f) zm[i * W64 + (b >> 6)] |= (uint64_t)1 << (b & 63);
      if (d->spikes) d->spikes[(k * B) * n + idx] = (uint8_t)(s != 0.0f);
      if (d->v_trace) d->v_trace[(k * B) * n + idx] = d->v[idx];
    }
  }
}

ORC_HOT static void synapse_phase(const orc_net* d, int64_t k, int64_t lo, int64_t hi) {
  const int64_t n = d->n, B = d->batch, H = d->max_delay + 1;
  const int64_t t = d->t0 + k;
  const int64_t C = d->n_rec > 1 ? d->n_rec : 1, nc = n * C;
  for (int64_t b = 0; b < B; ++b) {
    const int live = !d->sample_len || k < d->sample_len[b];
    for (int64_t col = lo * C; col < hi * C; ++col) {  /* the PSC columns of neurons [lo, hi) */
      const int64_t idx = b * nc + col;
      if (live) {
        /* W z: fmaf chain over in-edges in canonical order */
        float acc = 0.0f;
        for (int64_t e = d->ptr[col]; e < d->ptr[col + 1]; ++e) {
          const int64_t s = t - d->delay[e];
          const float z = s >= 0 ? d->hist[((s % H) * B + b) * n + d->pre[e]] : 0.0f;
          acc = fmaf(d->w[e], z, acc);
        }
        const float p = d->psc[idx];
        const float dec = d->psc_coef[col] * ((-p) / d->psc_tau[col]);
        const float q = p + dec;
        d->psc[idx] = q + acc;
      }
      if (d->psc_trace) d->psc_trace[(k * B) * nc + idx] = d->psc[idx];
    }
  }
}

/* The synapse phase of samples [slo, shi), event-driven: W z is formed by
 * pushing the edges of every source row whose presynaptic neuron spiked
 * `delay` steps ago, rows in ascending (pre, delay) order.  Each PSC column
 * then receives its terms in ascending canonical source order -- the order
 * of synapse_phase's chain -- and the terms it skips are exact zeros
 * (fmaf(w, 0, acc) == acc: acc starts at +0 and a sum of nonzero terms
 * never rounds to -0), so the result is bit-identical to synapse_phase's,
 * at a cost proportional to the spikes instead of the synapses.  A row's
 * edges are read once for all the samples of the range in which it spiked
 * (up to 64 at a time). */
ORC_HOT static void synapse_phase_events(const orc_net* d, int64_t k, int64_t slo, int64_t shi) {
  const int64_t n = d->n, B = d->batch, H = d->max_delay + 1;
  const int64_t t = d->t0 + k;
  const int64_t C = d->n_rec > 1 ? d->n_rec : 1, nc = n * C;
  const int64_t R = d->max_delay + 1;  /* source rows per presynaptic neuron */
  const int64_t W64 = (B + 63) >> 6;
  for (int64_t g0 = slo; g0 < shi; g0 += 64) {
    const int64_t g1 = g0 + 64 < shi ? g0 + 64 : shi;
    uint64_t live = 0;
    for (int64_t b = g0; b < g1; ++b)
      if (!d->sample_len || k < d->sample_len[b]) {
        live |= (uint64_t)1 << (b - g0);
        memset(d->acc + b * nc, 0, sizeof(float) * (size_t)nc);
      }
    for (int64_t pre = 0; pre < n && live; ++pre) {
      for (int64_t dl = 0; dl < R; ++dl) {
        const int64_t r = pre * R + dl;
        const int64_t e0 = d->row_ptr[r], e1 = d->row_ptr[r + 1];
        const int64_t s = t - dl;
        if (e0 == e1 || s < 0) continue;
        /* bits g0 .. g1-1 of the step's sample mask of `pre` */
        const uint64_t* zw = d->zmask + ((s % H) * n + pre) * W64 + (g0 >> 6);
        const int sh = (int)(g0 & 63);
        uint64_t m = zw[0] >> sh;
        if (sh && (g0 >> 6) + 1 < W64) m |= zw[1] << (64 - sh);
        m &= live;
        if (!m) continue;
        for (int64_t e = e0; e < e1; ++e) {
          const int64_t col = d->row_col[e];
          const float w = d->row_w[e];
          for (uint64_t mm = m; mm; mm &= mm - 1) {
            float* a = d->acc + (g0 + __builtin_ctzll(mm)) * nc + col;
            *a = *a + w;  /* fmaf(w, 1, a): one rounding of a + w */
          }
        }
      }
    }
    for (int64_t b = g0; b < g1; ++b) {
      if ((live >> (b - g0)) & 1) {
        const float* acc = d->acc + b * nc;
        for (int64_t col = 0; col < nc; ++col) {
          const int64_t idx = b * nc + col;
          const float p = d->psc[idx];
          const float dec = d->psc_coef[col] * ((-p) / d->psc_tau[col]);
          const float q = p + dec;
          d->psc[idx] = q + acc[col];
        }
      }
      if (d->psc_trace)
        memcpy(d->psc_trace + (k * B) * nc + b * nc, d->psc + b * nc, sizeof(float) * (size_t)nc);
    }
  }
}

typedef struct {
  const orc_net* net;
  int64_t lo, hi;   /* neuron range */
  int64_t slo, shi; /* sample range (event-driven synapse phase) */
  int events;
  pthread_barrier_t* bar;
} run_arg;

static void* worker(void* p) {
  run_arg* a = (run_arg*)p;
  const orc_net* d = a->net;
  for (int64_t k = 0; k < d->steps; ++k) {
    neuron_phase(d, k, a->lo, a->hi);
    pthread_barrier_wait(a->bar);
    if (a->events) synapse_phase_events(d, k, a->slo, a->shi);
    else synapse_phase(d, k, a->lo, a->hi);
    pthread_barrier_wait(a->bar);
  }
  return NULL;
}

static int run_threads(const orc_net* d, int events) {
  int T = d->threads > 0 ? d->threads : 1;
  if (T > d->n) T = (int)d->n;
  if (T < 1) T = 1;
  pthread_barrier_t bar;
  pthread_barrier_init(&bar, NULL, (unsigned)T);
  pthread_t* th = (pthread_t*)calloc((size_t)T, sizeof(pthread_t));
  run_arg* args = (run_arg*)calloc((size_t)T, sizeof(run_arg));
  if (!th || !args) return 1;
  for (int q = 0; q < T; ++q) {
    args[q].net = d;
    args[q].lo = d->n * q / T;
    args[q].hi = d->n * (q + 1) / T;
    args[q].slo = d->batch * q / T;
    args[q].shi = d->batch * (q + 1) / T;
    args[q].events = events;
    args[q].bar = &bar;
    if (q > 0) pthread_create(&th[q], NULL, worker, &args[q]);
  }
  worker(&args[0]);
  for (int q = 1; q < T; ++q) pthread_join(th[q], NULL);
  pthread_barrier_destroy(&bar);
  free(th);
  free(args);
  return 0;
}

/* Run `steps` recurrent steps (the reference's algorithm: every synapse of
 * every step, as torch.sparse.mm computes it).  Returns 0 on success. */
int orc_run(const orc_net* d) { return run_threads(d, 0); }

/* The same steps with the event-driven synapse phase (bit-identical results;
 * needs row_ptr, row_col, row_w and acc).  Returns 0 on success. */
int orc_run_events(const orc_net* d) {
  if (!d->row_ptr || !d->row_col || !d->row_w || !d->acc || !d->zmask) return 2;
  return run_threads(d, 1);
}

/* out[b][i] = fmaf chain over in-edges of i (ascending canonical order) of
 * w * x[b][src], zero inputs included (the reference's torch.sparse.mm). */
typedef struct {
  int64_t n_out, batch, n_in, lo, hi;
  const int64_t* ptr;
  const int64_t* src;
  const float *w, *x;
  float* out;
} spmm_arg;

ORC_HOT static void* spmm_worker(void* p) {
  spmm_arg* a = (spmm_arg*)p;
  for (int64_t b = 0; b < a->batch; ++b)
    for (int64_t i = a->lo; i < a->hi; ++i) {
      float acc = 0.0f;
      for (int64_t e = a->ptr[i]; e < a->ptr[i + 1]; ++e) acc = fmaf(a->w[e], a->x[b * a->n_in + a->src[e]], acc);
      a->out[b * a->n_out + i] = acc;
    }
  return NULL;
}

int orc_spmm(int64_t n_out, int64_t batch, int64_t n_in, const int64_t* ptr, const int64_t* src, const float* w,
             const float* x, float* out, int32_t threads) {
  int T = threads > 0 ? threads : 1;
  if (T > n_out) T = n_out > 0 ? (int)n_out : 1;
  pthread_t* th = (pthread_t*)calloc((size_t)T, sizeof(pthread_t));
  spmm_arg* args = (spmm_arg*)calloc((size_t)T, sizeof(spmm_arg));
  if (!th || !args) return 1;
  for (int q = 0; q < T; ++q) {
    spmm_arg a = {n_out, batch, n_in, n_out * q / T, n_out * (q + 1) / T, ptr, src, w, x, out};
    args[q] = a;
    if (q > 0) pthread_create(&th[q], NULL, spmm_worker, &args[q]);
  }
  spmm_worker(&args[0]);
  for (int q = 1; q < T; ++q) pthread_join(th[q], NULL);
  free(th);
  free(args);
  return 0;
}

/* Input projection restated as an ascending-channel fmaf chain over the
 * nonzero inputs (nn.Linear in the reference runs through MKL, whose
 * summation order is not reproducible; this order is the one the CUDA
 * projection uses).  out[r][i] = sum_c x[r][c] * W[i][c] (+ bias[i]). */
typedef struct {
  int64_t r0, r1, c_in, n;
  const float *x, *W, *bias;
  float* out;
  int status;
} linear_arg;

ORC_HOT static void* linear_worker(void* p) {
  linear_arg* a = (linear_arg*)p;
  const int64_t c_in = a->c_in, n = a->n;
  int64_t* nz = (int64_t*)malloc(sizeof(int64_t) * (size_t)(c_in > 0 ? c_in : 1));
  if (!nz) {
    a->status = 1;
    return NULL;
  }
  for (int64_t r = a->r0; r < a->r1; ++r) {
    const float* xr = a->x + r * c_in;
    int64_t cnt = 0;
    for (int64_t c = 0; c < c_in; ++c)
      if (xr[c] != 0.0f) nz[cnt++] = c;
    for (int64_t i = 0; i < n; ++i) {
      const float* wi = a->W + i * c_in;
      float acc = 0.0f;
      for (int64_t q = 0; q < cnt; ++q) acc = fmaf(xr[nz[q]], wi[nz[q]], acc);
      a->out[r * n + i] = a->bias ? acc + a->bias[i] : acc;
    }
  }
  free(nz);
  return NULL;
}

int orc_linear_mt(int64_t rows, int64_t c_in, int64_t n, const float* x, const float* W, const float* bias,
                  float* out, int32_t threads) {
  int T = threads > 0 ? threads : 1;
  if (T > rows) T = rows > 0 ? (int)rows : 1;
  pthread_t* th = (pthread_t*)calloc((size_t)T, sizeof(pthread_t));
  linear_arg* args = (linear_arg*)calloc((size_t)T, sizeof(linear_arg));
  if (!th || !args) return 1;
  for (int q = 0; q < T; ++q) {
    linear_arg a = {rows * q / T, rows * (q + 1) / T, c_in, n, x, W, bias, out, 0};
    args[q] = a;
    if (q > 0) pthread_create(&th[q], NULL, linear_worker, &args[q]);
  }
  linear_worker(&args[0]);
  int st = 0;
  for (int q = 0; q < T; ++q) {
    if (q > 0) pthread_join(th[q], NULL);
    st |= args[q].status;
  }
  free(th);
  free(args);
  return st;
}

/* The same projection from W_t [c_in][n] (the layout DenseConn's weight
 * has transposed): each nonzero channel's weight row is added into the
 * output row in ascending channel order, so every out[r][i] is the same fmaf
 * chain as orc_linear's; rows split over threads. */
typedef struct {
  int64_t r0, r1, c_in, n;
  const float *x, *Wt, *bias;
  float* out;
} linear_t_arg;

ORC_HOT static void* linear_t_worker(void* p) {
  linear_t_arg* a = (linear_t_arg*)p;
  const int64_t c_in = a->c_in, n = a->n;
  for (int64_t r = a->r0; r < a->r1; ++r) {
    const float* xr = a->x + r * c_in;
    float* o = a->out + r * n;
    for (int64_t i = 0; i < n; ++i) o[i] = 0.0f;
    for (int64_t c = 0; c < c_in; ++c) {
      const float xv = xr[c];
      if (xv == 0.0f) continue;
      const float* w = a->Wt + c * n;
      for (int64_t i = 0; i < n; ++i) o[i] = fmaf(xv, w[i], o[i]);
    }
    if (a->bias)
      for (int64_t i = 0; i < n; ++i) o[i] = o[i] + a->bias[i];
  }
  return NULL;
}

int orc_linear_t(int64_t rows, int64_t c_in, int64_t n, const float* x, const float* Wt, const float* bias,
                 float* out, int32_t threads) {
  int T = threads > 0 ? threads : 1;
  if (T > rows) T = rows > 0 ? (int)rows : 1;
  pthread_t* th = (pthread_t*)calloc((size_t)T, sizeof(pthread_t));
  linear_t_arg* args = (linear_t_arg*)calloc((size_t)T, sizeof(linear_t_arg));
  if (!th || !args) return 1;
  for (int q = 0; q < T; ++q) {
    linear_t_arg a = {rows * q / T, rows * (q + 1) / T, c_in, n, x, Wt, bias, out};
    args[q] = a;
    if (q > 0) pthread_create(&th[q], NULL, linear_t_worker, &args[q]);
  }
  linear_t_worker(&args[0]);
  for (int q = 1; q < T; ++q) pthread_join(th[q], NULL);
  free(th);
  free(args);
  return 0;
}

int orc_linear(int64_t rows, int64_t c_in, int64_t n, const float* x, const float* W, const float* bias, float* out) {
  return orc_linear_mt(rows, c_in, n, x, W, bias, out, 1);
}
