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

typedef struct {
  const orc_net* net;
  int64_t lo, hi; /* neuron range */
  pthread_barrier_t* bar;
} worker_arg;

static void neuron_phase(const orc_net* d, int64_t k, int64_t lo, int64_t hi) {
  const int64_t n = d->n, B = d->batch, H = d->max_delay + 1;
  const int64_t t = d->t0 + k;
  const float dt = d->dt;
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
      if (d->spikes) d->spikes[(k * B) * n + idx] = (uint8_t)(s != 0.0f);
      if (d->v_trace) d->v_trace[(k * B) * n + idx] = d->v[idx];
    }
  }
}

static void synapse_phase(const orc_net* d, int64_t k, int64_t lo, int64_t hi) {
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

static void* worker(void* p) {
  worker_arg* a = (worker_arg*)p;
  const orc_net* d = a->net;
  for (int64_t k = 0; k < d->steps; ++k) {
    neuron_phase(d, k, a->lo, a->hi);
    pthread_barrier_wait(a->bar);
    synapse_phase(d, k, a->lo, a->hi);
    pthread_barrier_wait(a->bar);
  }
  return NULL;
}

/* Run `steps` recurrent steps.  Returns 0 on success. */
int orc_run(const orc_net* d) {
  int T = d->threads > 0 ? d->threads : 1;
  if (T > d->n) T = (int)d->n;
  if (T < 1) T = 1;
  pthread_barrier_t bar;
  pthread_barrier_init(&bar, NULL, (unsigned)T);
  pthread_t* th = (pthread_t*)calloc((size_t)T, sizeof(pthread_t));
  worker_arg* args = (worker_arg*)calloc((size_t)T, sizeof(worker_arg));
  if (!th || !args) return 1;
  for (int q = 0; q < T; ++q) {
    args[q].net = d;
    args[q].lo = d->n * q / T;
    args[q].hi = d->n * (q + 1) / T;
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

/* out[b][i] = fmaf chain over in-edges of i (ascending canonical order) of
 * w * x[b][src], zero inputs included (the reference's torch.sparse.mm). */
typedef struct {
  int64_t n_out, batch, n_in, lo, hi;
  const int64_t* ptr;
  const int64_t* src;
  const float *w, *x;
  float* out;
} spmm_arg;

static void* spmm_worker(void* p) {
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
int orc_linear(int64_t rows, int64_t c_in, int64_t n, const float* x, const float* W, const float* bias, float* out) {
  int64_t* nz = (int64_t*)malloc(sizeof(int64_t) * (size_t)(c_in > 0 ? c_in : 1));
  if (!nz) return 1;
  for (int64_t r = 0; r < rows; ++r) {
    int64_t cnt = 0;
    for (int64_t c = 0; c < c_in; ++c)
      if (x[r * c_in + c] != 0.0f) nz[cnt++] = c;
    for (int64_t i = 0; i < n; ++i) {
      float acc = 0.0f;
      for (int64_t q = 0; q < cnt; ++q) acc = fmaf(x[r * c_in + nz[q]], W[i * c_in + nz[q]], acc);
      out[r * n + i] = bias ? acc + bias[i] : acc;
    }
  }
  free(nz);
  return 0;
}
