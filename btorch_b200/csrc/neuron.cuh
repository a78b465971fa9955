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

// Exact reciprocal of c if c is a power of two (then x / c == x * (1/c) for
// every x: both are the correctly rounded value of the same real number), 0
// otherwise.  Lets the kernels replace IEEE division by a multiply whenever a
// divisor such as c_m = 1 or (v_threshold - v_reset) = 1 allows it.
__device__ __forceinline__ float pow2_recip(float c) {
  // positive normal power of two: zero mantissa, biased exponent e in [1, 253]
  // so that 1/c = 2^(127 - (e - 127)) has biased exponent 254 - e in [1, 253]
  const uint32_t u = __float_as_uint(c);
  const uint32_t e = u >> 23;  // sign bit included: negative c gives e > 255
  return ((u & 0x7fffffu) == 0u && e >= 1u && e <= 253u) ? __uint_as_float((254u - e) << 23) : 0.0f;
}

// x / c with the reference's rounding; rc = pow2_recip(c).
__device__ __forceinline__ float divc(float x, float c, float rc) { return rc != 0.0f ? mul(x, rc) : div(x, c); }

// x / c from the correctly rounded reciprocal r of c: q = x r, then one FMA
// correction with the exact remainder x - q c (Markstein's division step,
// IBM J. Res. Dev. 34(1), 1990).  A zero x gives q = x r, which is already
// the IEEE quotient (a zero whose sign is sign(x) xor sign(c)).  A tiny
// quotient, 2^-124 <= |q| < 2^-100, is computed for x 2^64 and scaled back by
// 2^-64 (both scalings exact: the result stays normal).  These cases are
// common -- a silent synapse, a neuron at rest, a decaying trace long after
// its last input -- and must not take the slow path.  Otherwise, outside
// 2^-100 <= |q| <= 2^100 (subnormal or huge quotients, inf, nan), it divides.
// Whether this equals the IEEE quotient for every x depends on c; the host
// enables it only for divisors checked against __fdiv_rn for every fp32 bit
// pattern of x (bt_fast_div_check).
static __device__ __noinline__ float div_recip_rare(float x, float c, float r) {
  const float q = mul(x, r);
  if (x == 0.0f) return q;
  const float aq = fabsf(q);
  if (aq < 0x1p-100f && aq >= 0x1p-124f) {
    const float xs = mul(x, 0x1p64f);
    const float qs = mul(xs, r);
    const float e = __fmaf_rn(-qs, c, xs);
    return mul(__fmaf_rn(e, r, qs), 0x1p-64f);
  }
  return div(x, c);
}

__device__ __forceinline__ float div_recip(float x, float c, float r) {
  const float q = mul(x, r);
  const float aq = fabsf(q);
  if (aq >= 0x1p-100f && aq <= 0x1p100f) {  // the common case: six instructions
    const float e = __fmaf_rn(-q, c, x);
    return __fmaf_rn(e, r, q);
  }
  return div_recip_rare(x, c, r);
}

// A divisor with its exact evaluation: kind 1 = power of two (multiply by the
// exact reciprocal), 2 = verified reciprocal (div_recip), 0 = IEEE division.
struct Div {
  float c, r;
  int kind;
};

__device__ __forceinline__ Div make_div(float c, bool verified, float rcp) {
  Div d;
  d.c = c;
  d.r = pow2_recip(c);
  d.kind = d.r != 0.0f ? 1 : 0;
  if (d.kind == 0 && verified) {
    d.r = rcp;
    d.kind = 2;
  }
  return d;
}

__device__ __forceinline__ float divc(float x, const Div& d) {
  return d.kind == 1 ? mul(x, d.r) : d.kind == 2 ? div_recip(x, d.c, d.r) : div(x, d.c);
}

// divc for a launch whose divisors are all of kind 1 or 2 (FAST, decided on
// the host from the parameter values): the IEEE-division branch is compiled
// out, which shortens the per-sample update of the issue-bound neuron steps.
template <bool FAST>
__device__ __forceinline__ float divk(float x, const Div& d) {
  if constexpr (FAST)
    return d.kind == 1 ? mul(x, d.r) : div_recip(x, d.c, d.r);
  else
    return divc(x, d);
}

// The parameters of one neuron, read once into registers (the kernels update
// many samples of the same neuron with them).
struct NeuronParams {
  float vth, vr, cm, den, dt;
  float tau;                           // LIF
  float tau_ref;
  float ngl, El, Ek, dgk, tau_a, cgk;  // ALIF: -g_leak, E_leak, E_k, dg_k, tau_adapt, coef_gk
  float sg_alpha;
  Div d_cm, d_den, d_tau, d_tau_a;     // the divisors with their evaluation
  int spiking;
};

template <int KIND, bool USE_REF>
__device__ __forceinline__ NeuronParams load_params(const bt_neuron_desc& d, int64_t i) {
  NeuronParams p;
  if (d.uniform) {  // scalar parameters passed by value: no parameter loads
    p.vth = d.sv[0];
    p.vr = d.sv[1];
    p.cm = d.sv[2];
    p.den = sub(p.vth, p.vr);
    p.dt = d.dt;
    p.sg_alpha = d.sg_alpha;
    p.spiking = d.spiking;
    p.tau = KIND == BT_NEURON_LIF ? d.sv[3] : 0.0f;
    p.tau_ref = USE_REF ? d.sv[4] : 0.0f;
    if (KIND == BT_NEURON_ALIF) {
      p.ngl = -d.sv[5];
      p.El = d.sv[6];
      p.Ek = d.sv[7];
      p.dgk = d.sv[8];
      p.tau_a = d.sv[9];
      p.cgk = d.sv[10];
    } else {
      p.ngl = p.El = p.Ek = p.dgk = p.tau_a = p.cgk = 0.0f;
    }
    p.d_cm = make_div(p.cm, d.fast_div & 1, d.rcp[0]);
    p.d_den = make_div(p.den, d.fast_div & 2, d.rcp[1]);
    p.d_tau = make_div(p.tau, d.fast_div & 4, d.rcp[2]);
    p.d_tau_a = make_div(p.tau_a, d.fast_div & 8, d.rcp[3]);
    return p;
  }
  p.vth = ld(d.v_threshold, i);
  p.vr = ld(d.v_reset, i);
  p.cm = ld(d.c_m, i);
  p.den = sub(p.vth, p.vr);  // (v_threshold - v_reset), one torch op in the reference
  p.dt = d.dt;
  p.sg_alpha = d.sg_alpha;
  p.spiking = d.spiking;
  p.tau = KIND == BT_NEURON_LIF ? ld(d.tau, i) : 0.0f;
  p.tau_ref = USE_REF ? ld(d.tau_ref, i) : 0.0f;
  if (KIND == BT_NEURON_ALIF) {
    p.ngl = -ld(d.g_leak, i);
    p.El = ld(d.E_leak, i);
    p.Ek = ld(d.E_k, i);
    p.dgk = ld(d.dg_k, i);
    p.tau_a = ld(d.tau_adapt, i);
    p.cgk = ld(d.coef_gk, i);
  } else {
    p.ngl = p.El = p.Ek = p.dgk = p.tau_a = p.cgk = 0.0f;
  }
  p.d_cm = make_div(p.cm, false, 0.0f);
  p.d_den = make_div(p.den, false, 0.0f);
  p.d_tau = make_div(p.tau, false, 0.0f);
  p.d_tau_a = make_div(p.tau_a, false, 0.0f);
  return p;
}

// One BaseNode.single_step_forward with input current I.  v, ref, gk are
// updated in place.  SPIKING selects the Heaviside forward at compile time
// (the fused engine); otherwise pr.spiking decides at run time.
template <int KIND, bool HARD, bool USE_REF, bool SPIKING = false, bool FAST = false>
__device__ __forceinline__ NeuronOut neuron_update(const NeuronParams& pr, float I, float& v, float& ref, float& gk) {
  const float dt = pr.dt;
  float v1;
  if (KIND == BT_NEURON_LIF) {
    // euler_step(dV): v + dt * ((-(v - v_reset)) / tau + x / c_m)
    v1 = add(v, mul(dt, add(divk<FAST>(-sub(v, pr.vr), pr.d_tau), divk<FAST>(I, pr.d_cm))));
  } else {
    // exp_euler_step(dV): derivative = ((-g_leak)(v - E_leak) + (-g_k)(v - E_k) + x) / c_m
    //                     linear     = ((-g_leak) - g_k) / c_m
    const float leak = mul(pr.ngl, sub(v, pr.El));
    const float adapt = mul(-gk, sub(v, pr.Ek));
    const float deriv = divk<FAST>(add(add(leak, adapt), I), pr.d_cm);
    const float lin = divk<FAST>(sub(pr.ngl, gk), pr.d_cm);
    const float coef = div(expm1f(mul(dt, lin)), lin);
    v1 = add(v, mul(coef, deriv));
    // neuronal_adaptation: g_k + coef_gk * ((-g_k) / tau_adapt)
    gk = add(gk, mul(pr.cgk, divk<FAST>(-gk, pr.d_tau_a)));
  }
  NeuronOut o;
  o.v_charged = v1;
  // neuronal_fire: surrogate((v - v_th) / (v_th - v_reset)) * (refractory == 0)
  o.u = divk<FAST>(sub(v1, pr.vth), pr.d_den);
  float s;
  if (SPIKING || pr.spiking)
    s = o.u >= 0.0f ? 1.0f : 0.0f;
  else
    s = sigmoidf_dev(mul(pr.sg_alpha, o.u));
  o.mask = 1.0f;
  if (USE_REF) {
    o.mask = (ref == 0.0f) ? 1.0f : 0.0f;
    s = mul(s, o.mask);
  }
  o.spike = s;
  // neuronal_reset
  if (HARD)
    v = sub(v1, mul(sub(v1, pr.vr), s));
  else
    v = sub(v1, mul(pr.den, s));
  if (KIND == BT_NEURON_ALIF) gk = add(gk, mul(pr.dgk, s));
  if (USE_REF) ref = relu_keep_nan(sub(add(ref, mul(s, pr.tau_ref)), dt));
  return o;
}

// Convenience overload: parameters read for neuron i.
template <int KIND, bool HARD, bool USE_REF>
__device__ __forceinline__ NeuronOut neuron_update(const bt_neuron_desc& d, int64_t i, float I, float& v, float& ref,
                                                   float& gk) {
  const NeuronParams pr = load_params<KIND, USE_REF>(d, i);
  return neuron_update<KIND, HARD, USE_REF>(pr, I, v, ref, gk);
}

// ExponentialPSC.conductance_charge: psc + coef * ((-psc) / tau_syn)
__device__ __forceinline__ float psc_decay(float coef, float tau, float rtau, float p) {
  return add(p, mul(coef, divc(-p, tau, rtau)));
}
__device__ __forceinline__ float psc_decay(float coef, const Div& tau, float p) {
  return add(p, mul(coef, divc(-p, tau)));
}
template <bool FAST>
__device__ __forceinline__ float psc_decay_k(float coef, const Div& tau, float p) {
  return add(p, mul(coef, divk<FAST>(-p, tau)));
}
__device__ __forceinline__ float psc_decay(float coef, float tau, float p) {
  return psc_decay(coef, tau, pow2_recip(tau), p);
}
__device__ __forceinline__ float psc_decay(const bt_param& coef, const bt_param& tau, int64_t i, float p) {
  return psc_decay(ld(coef, i), ld(tau, i), p);
}

}  // namespace bt
