// Single-step neuron and synapse kernels (the per-module path used when a
// model is stepped module by module, and for autograd).
#include "neuron.cuh"

namespace bt {

template <int KIND, bool HARD, bool USE_REF>
__global__ void k_neuron_step(bt_neuron_desc d, int64_t batch, int64_t n, const float* __restrict__ x,
                              const float* v_in, const float* ref_in, const float* gk_in, float* v_out,
                              float* ref_out, float* gk_out, float* __restrict__ spike, float* __restrict__ u_save,
                              float* __restrict__ mask_save, float* __restrict__ vch_save) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= batch * n) return;
  const int64_t i = idx % n;
  float v = v_in[idx];
  float ref = USE_REF ? ref_in[idx] : 0.0f;
  float gk = KIND == BT_NEURON_ALIF ? gk_in[idx] : 0.0f;
  const NeuronOut o = neuron_update<KIND, HARD, USE_REF>(d, i, x[idx], v, ref, gk);
  v_out[idx] = v;
  if (USE_REF) ref_out[idx] = ref;
  if (KIND == BT_NEURON_ALIF) gk_out[idx] = gk;
  spike[idx] = o.spike;
  if (u_save) u_save[idx] = o.u;
  if (mask_save) mask_save[idx] = o.mask;
  if (vch_save) vch_save[idx] = o.v_charged;
}

// Reverse-mode derivative of one neuron step, following the autograd graph
// the reference builds from its eager ops.  The fire step's surrogate is the
// sigmoid one: damping * 4 * s(k a u) * (1 - s(k a u)).
__global__ void k_neuron_step_backward(bt_neuron_desc d, int64_t batch, int64_t n, const float* x,
                                       const float* g_spike, const float* g_v_new, const float* g_gk_new,
                                       const float* u_save, const float* spike, const float* mask_save,
                                       const float* v_charged, const float* v_prev, const float* gk_prev, float* g_x,
                                       float* g_v_prev, float* g_gk_prev, int detach_reset) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= batch * n) return;
  const int64_t i = idx % n;
  const float vth = ld(d.v_threshold, i), vr = ld(d.v_reset, i), cm = ld(d.c_m, i);
  const float dt = d.dt;
  const float s = spike[idx], u = u_save[idx], mask = mask_save[idx], v1 = v_charged[idx];
  const float gv2 = g_v_new ? g_v_new[idx] : 0.0f;
  const bool alif = d.kind == BT_NEURON_ALIF;
  const float ggk2 = (alif && g_gk_new) ? g_gk_new[idx] : 0.0f;
  float gs = g_spike ? g_spike[idx] : 0.0f;
  const float den = vth - vr;
  // reset:  hard v2 = v1 - (v1 - vr) * s ;  soft v2 = v1 - (vth - vr) * s
  float gv1, gs_reset;
  if (d.hard_reset) {
    gv1 = gv2 - gv2 * s;
    gs_reset = -gv2 * (v1 - vr);
  } else {
    gv1 = gv2;
    gs_reset = -gv2 * den;
  }
  if (alif) gs_reset += ggk2 * ld(d.dg_k, i);  // gk2 = gk1 + dg_k * s
  if (!detach_reset) gs += gs_reset;
  // fire:  s = H(u) * mask with the surrogate derivative at u;  u = (v1 - vth) / den
  const float sig = sigmoidf_dev(d.sg_alpha * u);
  const float gu = (gs * mask) * (d.sg_damping * 4.0f * sig * (1.0f - sig));
  gv1 += gu / den;
  const float v = v_prev[idx];
  if (!alif) {
    // charge: v1 = v + dt * ((-(v - vr)) / tau + I / cm)
    const float gD = dt * gv1;
    g_x[idx] = gD / cm;
    if (g_v_prev) g_v_prev[idx] = gv1 - gD / ld(d.tau, i);
    return;
  }
  // charge: v1 = v + C(lin) * D,  D = (ngl (v - El) + (-gk)(v - Ek) + I) / cm,  lin = (ngl - gk) / cm
  const float gk = gk_prev[idx];
  const float ngl = -ld(d.g_leak, i);
  const float Ek = ld(d.E_k, i);
  const float lin = (ngl - gk) / cm;
  const float em1 = expm1f(dt * lin);
  const float C = em1 / lin;
  const float D = (ngl * (v - ld(d.E_leak, i)) + (-gk) * (v - Ek) + x[idx]) / cm;
  const float gC = gv1 * D, gD = gv1 * C;
  g_x[idx] = gD / cm;
  if (g_v_prev) g_v_prev[idx] = gv1 + gD * lin;
  // dC/dlin = (dt e^{dt lin} lin - expm1(dt lin)) / lin^2 ; dlin/dgk = -1/cm ; dD/dgk = -(v - Ek)/cm
  const float dCdl = (dt * (em1 + 1.0f) * lin - em1) / (lin * lin);
  const float g_gk_charge = -(gC * dCdl) / cm - gD * (v - Ek) / cm;
  // adaptation: gk1 = gk + coef_gk * ((-gk) / tau_adapt)
  const float dgk1 = 1.0f - ld(d.coef_gk, i) / ld(d.tau_adapt, i);
  if (g_gk_prev) g_gk_prev[idx] = ggk2 * dgk1 + g_gk_charge;
}

__global__ void k_psc_step(int64_t batch, int64_t n, bt_param coef, bt_param tau, const float* psc,
                           const float* wz, float* out) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= batch * n) return;
  float p = psc_decay(coef, tau, idx % n, psc[idx]);
  if (wz) p = add(p, wz[idx]);
  out[idx] = p;
}

}  // namespace bt

using namespace bt;

namespace {

template <int KIND, bool HARD, bool USE_REF>
void launch_neuron_step(const bt_neuron_desc& d, int64_t batch, int64_t n, const float* x, const float* v_in,
                        const float* ref_in, const float* gk_in, float* v_out, float* ref_out, float* gk_out,
                        float* spike, float* u_save, float* mask_save, float* vch_save, cudaStream_t s) {
  const int64_t total = batch * n;
  k_neuron_step<KIND, HARD, USE_REF><<<int(ceil_div(total, 256)), 256, 0, s>>>(
      d, batch, n, x, v_in, ref_in, gk_in, v_out, ref_out, gk_out, spike, u_save, mask_save, vch_save);
}

int check_neuron_desc(const bt_neuron_desc* d) {
  if (!d) return bt_set_error(BT_ERR_INVALID, "null neuron descriptor");
  if (d->kind != BT_NEURON_LIF && d->kind != BT_NEURON_ALIF)
    return bt_set_error(BT_ERR_UNSUPPORTED, "neuron kind %d", d->kind);
  if (!d->v_threshold.ptr || !d->v_reset.ptr || !d->c_m.ptr)
    return bt_set_error(BT_ERR_INVALID, "missing v_threshold / v_reset / c_m");
  if (d->kind == BT_NEURON_LIF && !d->tau.ptr) return bt_set_error(BT_ERR_INVALID, "LIF needs tau");
  if (d->kind == BT_NEURON_ALIF && (!d->g_leak.ptr || !d->E_leak.ptr || !d->E_k.ptr || !d->dg_k.ptr ||
                                    !d->tau_adapt.ptr || !d->coef_gk.ptr))
    return bt_set_error(BT_ERR_INVALID, "ALIF parameter missing");
  if (d->use_refractory && !d->tau_ref.ptr) return bt_set_error(BT_ERR_INVALID, "refractory needs tau_ref");
  return BT_OK;
}

}  // namespace

extern "C" int bt_check_neuron_desc(const bt_neuron_desc* d) { return check_neuron_desc(d); }

namespace {

// Every fp32 bit pattern x once: fast quotient vs IEEE quotient.
__global__ void k_fast_div_check(float c, float r, int32_t* mismatches) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  int bad = 0;
  for (uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < (uint64_t(1) << 32); u += stride) {
    const float x = __uint_as_float(uint32_t(u));
    const float f = bt::div_recip(x, c, r), g = bt::div(x, c);
    bad += (__float_as_uint(f) == __float_as_uint(g) || (f != f && g != g)) ? 0 : 1;
  }
  // a flag, not a count: up to 2^32 mismatches would overflow an int32 sum
  if (__any_sync(0xffffffffu, bad != 0) && (threadIdx.x & 31) == 0) atomicOr(mismatches, 1);
}

}  // namespace

extern "C" int bt_fast_div_check(float c, float rcp, int32_t* mismatches, void* stream) {
  BT_CHECK_ARG(mismatches, "null mismatches");
  BT_CHECK_ARG(c == c && c != 0.0f && c - c == 0.0f, "divisor must be finite and nonzero");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_fast_div_check<<<sms * 16, 256, 0, static_cast<cudaStream_t>(stream)>>>(c, rcp, mismatches);
  BT_CHECK_LAUNCH("k_fast_div_check");
  return BT_OK;
}

extern "C" int bt_neuron_step(const bt_neuron_desc* d, int64_t batch, int64_t n, const float* x, const float* v_in,
                              const float* ref_in, const float* gk_in, float* v_out, float* ref_out, float* gk_out,
                              float* spike, float* u_save, float* mask_save, float* vch_save, void* stream) {
  if (int st = check_neuron_desc(d)) return st;
  BT_CHECK_ARG(batch >= 0 && n >= 0, "negative size");
  if (batch * n == 0) return BT_OK;
  BT_CHECK_ARG(x && v_in && v_out && spike, "null x / v / spike");
  BT_CHECK_ARG(!d->use_refractory || (ref_in && ref_out), "refractory state missing");
  BT_CHECK_ARG(d->kind != BT_NEURON_ALIF || (gk_in && gk_out), "g_k state missing");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
#define BT_NS(K, H, R)                                                                                        \
  launch_neuron_step<K, H, R>(*d, batch, n, x, v_in, ref_in, gk_in, v_out, ref_out, gk_out, spike, u_save, \
                              mask_save, vch_save, s)
  const bool h = d->hard_reset != 0, r = d->use_refractory != 0;
  if (d->kind == BT_NEURON_LIF) {
    if (h && r) BT_NS(BT_NEURON_LIF, true, true);
    else if (h) BT_NS(BT_NEURON_LIF, true, false);
    else if (r) BT_NS(BT_NEURON_LIF, false, true);
    else BT_NS(BT_NEURON_LIF, false, false);
  } else {
    if (h && r) BT_NS(BT_NEURON_ALIF, true, true);
    else if (h) BT_NS(BT_NEURON_ALIF, true, false);
    else if (r) BT_NS(BT_NEURON_ALIF, false, true);
    else BT_NS(BT_NEURON_ALIF, false, false);
  }
#undef BT_NS
  BT_CHECK_LAUNCH("k_neuron_step");
  return BT_OK;
}

extern "C" int bt_neuron_step_backward(const bt_neuron_desc* d, int64_t batch, int64_t n, const float* x,
                                       const float* g_spike, const float* g_v_new, const float* g_gk_new,
                                       const float* u_save, const float* spike, const float* mask_save,
                                       const float* v_charged, const float* v_prev, const float* gk_prev,
                                       float* g_x, float* g_v_prev, float* g_gk_prev, int32_t detach_reset,
                                       void* stream) {
  if (int st = check_neuron_desc(d)) return st;
  BT_CHECK_ARG(batch >= 0 && n >= 0, "negative size");
  if (batch * n == 0) return BT_OK;
  BT_CHECK_ARG(x && u_save && spike && mask_save && v_charged && v_prev && g_x, "null saved tensor");
  BT_CHECK_ARG(d->kind != BT_NEURON_ALIF || gk_prev, "ALIF backward needs gk_prev");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_neuron_step_backward<<<int(ceil_div(batch * n, 256)), 256, 0, s>>>(
      *d, batch, n, x, g_spike, g_v_new, g_gk_new, u_save, spike, mask_save, v_charged, v_prev, gk_prev, g_x,
      g_v_prev, g_gk_prev, detach_reset);
  BT_CHECK_LAUNCH("k_neuron_step_backward");
  return BT_OK;
}

extern "C" int bt_psc_step(int64_t batch, int64_t n, bt_param coef, bt_param tau_syn, const float* psc,
                           const float* wz, float* out, void* stream) {
  BT_CHECK_ARG(batch >= 0 && n >= 0, "negative size");
  if (batch * n == 0) return BT_OK;
  BT_CHECK_ARG(psc && out && coef.ptr && tau_syn.ptr, "null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_psc_step<<<int(ceil_div(batch * n, 256)), 256, 0, s>>>(batch, n, coef, tau_syn, psc, wz, out);
  BT_CHECK_LAUNCH("k_psc_step");
  return BT_OK;
}
