// Device-side neuron and synapse updates, op by op in the reference's order.
//
// LIF   btorch/models/neurons/lif.py:144-187   (dV, charge, fire, reset)
// ALIF  btorch/models/neurons/alif.py:193-249  (dV, dgk, charge, adaptation, fire, reset)
// step  btorch/models/base.py:1108-1116         (charge -> adaptation -> fire -> reset)
// ODE   btorch/models/ode.py:20-55              (euler: x + dt*f ; exp-euler: x + expm1(dt*A)/A*f)
// PSC   btorch/models/synapse.py:171-178,79-103 (psc + coef*((-psc)/tau), then psc + W z)
//
// Every arithmetic torch op of the reference becomes one correctly rounded
// fp32 op here (bt::add/sub/mul/div), so the LIF and PSC updates reproduce the
// reference's CPU results bit for bit.  The only transcendental evaluated per
// element on the device is ALIF's expm1 of the state-dependent linear term
// (CUDA's expm1f; it differs from the CPU's in the last ulp at most).
#pragma once

#include "common.cuh"

namespace bt {

struct NeuronOut {
  float spike;      // emitted spike (after the refractory mask)
  float u;          // (v_charged - v_th) / (v_th - v_reset)
  float mask;       // 1 if not refractory before this step (else 0)
  float v_charged;  // v after charge, before reset
};

__device__ __forceinline__ float relu_keep_nan(float x) { return (x != x) ? x : fmaxf(x, 0.0f); }

__device__ __forceinline__ float sigmoidf_dev(float x) { return 1.0f / (1.0f + expf(-x)); }

// One BaseNode.single_step_forward for neuron i with input current I.
// v, ref, gk are updated in place.  KIND/HARD/USE_REF may be template
// constants (engine) or runtime values (single-step kernel).
template <int KIND, bool HARD, bool USE_REF>
__device__ __forceinline__ NeuronOut neuron_update(const bt_neuron_desc& d, int64_t i, float I, float& v, float& ref,
                                                   float& gk) {
  const float vth = ld(d.v_threshold, i);
  const float vr = ld(d.v_reset, i);
  const float cm = ld(d.c_m, i);
  const float dt = d.dt;
  float v1;
  if (KIND == BT_NEURON_LIF) {
    // euler_step(dV): v + dt * ((-(v - v_reset)) / tau + x / c_m)
    const float tau = ld(d.tau, i);
    v1 = add(v, mul(dt, add(div(-sub(v, vr), tau), div(I, cm))));
  } else {
    // exp_euler_step(dV): derivative = ((-g_leak)(v - E_leak) + (-g_k)(v - E_k) + x) / c_m
    //                     linear     = ((-g_leak) - g_k) / c_m
    const float ngl = -ld(d.g_leak, i);
    const float leak = mul(ngl, sub(v, ld(d.E_leak, i)));
    const float adapt = mul(-gk, sub(v, ld(d.E_k, i)));
    const float deriv = div(add(add(leak, adapt), I), cm);
    const float lin = div(sub(ngl, gk), cm);
    const float coef = div(expm1f(mul(dt, lin)), lin);
    v1 = add(v, mul(coef, deriv));
    // neuronal_adaptation: g_k + coef_gk * ((-g_k) / tau_adapt)
    gk = add(gk, mul(ld(d.coef_gk, i), div(-gk, ld(d.tau_adapt, i))));
  }
  NeuronOut o;
  o.v_charged = v1;
  // neuronal_fire: surrogate((v - v_th) / (v_th - v_reset)) * (refractory == 0)
  const float den = sub(vth, vr);
  o.u = div(sub(v1, vth), den);
  float s = d.spiking ? (o.u >= 0.0f ? 1.0f : 0.0f) : sigmoidf_dev(mul(d.sg_alpha, o.u));
  o.mask = 1.0f;
  if (USE_REF) {
    o.mask = (ref == 0.0f) ? 1.0f : 0.0f;
    s = mul(s, o.mask);
  }
  o.spike = s;
  // neuronal_reset
  if (HARD)
    v = sub(v1, mul(sub(v1, vr), s));
  else
    v = sub(v1, mul(den, s));
  if (KIND == BT_NEURON_ALIF) gk = add(gk, mul(ld(d.dg_k, i), s));
  if (USE_REF) ref = relu_keep_nan(sub(add(ref, mul(s, ld(d.tau_ref, i))), dt));
  return o;
}

// ExponentialPSC.conductance_charge: psc + coef * ((-psc) / tau_syn)
__device__ __forceinline__ float psc_decay(const bt_param& coef, const bt_param& tau, int64_t i, float p) {
  return add(p, mul(ld(coef, i), div(-p, ld(tau, i))));
}

}  // namespace bt
