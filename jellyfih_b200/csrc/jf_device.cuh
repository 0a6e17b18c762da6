// Device math of the 2-D MLS-MPM substep, shared by the plain and batched
// paths.  Each function follows the reference engine mpm_sim.py (line numbers
// cited per function) in its operation order, FP32 throughout.
//
// Rounding: the chain F update -> SVD -> plasticity -> stress -> APIC affine
// ends in the cancellation F - R, so every operation there is rounded on its
// own (the _rn intrinsics below), as the reference's FP32 arithmetic rounds
// it; letting the compiler fuse multiply-adds in that chain moves a
// substep's fields by ~1e-5.  The G2P gather, the node contributions and the
// stencil weights are insensitive (~2e-7) and are left to FMA contraction.
// The waveform phase and the position update are also rounded step by step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Static per-instance description, built on the host.  FP32 constants are the
// reference's Python-double expressions rounded once (mpm_sim.py:18-58).
struct JfInst {
  int32_t nx, ny;       // grid nodes along x and y (n_grid, n_grid_y)
  int32_t dcx, dcy;     // damping band widths n_grid // 20, n_grid_y // 20 (:283-284)
  int32_t band_h;       // nominal grid rows per CTA band (batched path): ceil(ny / CTAs)
  int32_t band_cap;     // most rows a band may take when the sort balances bands (batched)
  int32_t n_slots;      // particle slots of this instance
  int64_t p_off;        // first particle slot in the engine arrays
  int64_t g_off;        // first grid node in the engine grid array
  float inv_dx, dx, dt, p_mass;
  float stress_scale;   // -dt * p_vol * 4 * inv_dx^2 (:250)
  float c4;             // 4 * inv_dx (:326)
  float dtg;            // dt * gravity (:329)
  float y_hi;           // domain_height - 0.001 (:333)
  float rref_lo;        // axisymmetric: dx * 0.1, floor of the load radius (:246)
  float r_lo;           // axisymmetric: dx * 0.05, floor of the radius (:247)
  int32_t axisym;       // JELLY_AXISYM (:17): r-weighted P2G, hoop correction, axis condition
  double domain_h;      // domain_height as the caller gave it (fitness ceiling, evolve.py:101)
};

// Mutable per-instance waveform / material parameters (mpm_sim.py:116-149).
struct JfParams {
  float actuation;        // instance_actuation
  float contraction;      // instance_act_contraction
  float freq;             // instance_freq
  float payload_density;  // instance_payload_density
};

// Lame parameters by material id: 0 water, 1 jelly, 2 payload, 3 muscle,
// anything else the E_base / nu_base default (mpm_sim.py:192-203).
struct JfMaterials {
  float mu[5];
  float la[5];
};

__device__ __forceinline__ int jf_mat_slot(int mt) { return (mt >= 0 && mt <= 3) ? mt : 4; }

// separately rounded FP32 operations (never fused)
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
// a*b + c*d with each product and the sum rounded on its own
__device__ __forceinline__ float rdot2(float a, float b, float c, float d) {
  return __fadd_rn(__fmul_rn(a, b), __fmul_rn(c, d));
}

// Activation of the 2-phase waveform (mpm_sim.py:173-180): Python float
// modulo as a - b*floor(a/b), half-cosine arch while phase < contraction.
// cos is taken in double and rounded once.
__host__ __device__ inline float jf_activation(float freq, float contraction, float t) {
#ifdef __CUDA_ARCH__
  float period = __fdiv_rn(1.0f, __fmul_rn(1.0f, freq));
  float q = floorf(__fdiv_rn(t, period));
  float r = __fsub_rn(t, __fmul_rn(period, q));
  float phase = __fdiv_rn(r, period);
  float a = 0.0f;
  if (phase < contraction) {
    float arg = __fmul_rn(__fdiv_rn(phase, contraction), 3.14159265f);
    a = __fmul_rn(0.5f, __fsub_rn(1.0f, (float)cos((double)arg)));
  }
  return a;
#else
  // host: volatile stores keep every operation rounded on its own, as the
  // device's __f*_rn do (no contraction into fused multiply-adds)
  volatile float period = 1.0f / (1.0f * freq);
  volatile float q = floorf(t / period);
  volatile float pq = period * q;
  volatile float r = t - pq;
  volatile float phase = r / period;
  float a = 0.0f;
  if (phase < contraction) {
    volatile float ratio = phase / contraction;
    volatile float arg = ratio * 3.14159265f;
    volatile float cs = (float)cos((double)arg);
    volatile float om = 1.0f - cs;
    a = 0.5f * om;
  }
  return a;
#endif
}

// 2x2 SVD as taichi 1.7.4 ti.svd computes it (_svd2d): polar decomposition
// A = R S with R = [[c,-s],[s,c]] from (A00 + A11, A10 - A01), one Jacobi
// rotation (cc, ss) of S unless |S01| < 1e-5, singular values ordered
// s1 >= s2 with the matching V, U = R V.  Matrices row-major in float4
// (00, 01, 10, 11).  jf_svd2_values stops before the ordering: it returns the
// rotations and the two singular values in Jacobi order.
struct JfSvdRot {
  float c, s, cc, ss, s1, s2;
};

__device__ __forceinline__ JfSvdRot jf_svd2_values(float4 A) {
  JfSvdRot o;
  const float x = radd(A.x, A.w);
  const float y = rsub(A.z, A.y);
  const float scale = 1.0f / sqrtf(radd(rmul(x, x), rmul(y, y)));
  o.c = rmul(x, scale);
  o.s = rmul(y, scale);
  const float ms = -o.s;
  const float S00 = rdot2(o.c, A.x, o.s, A.z);
  const float S01 = rdot2(o.c, A.y, o.s, A.w);
  const float S11 = rdot2(ms, A.y, o.c, A.w);
  // Both branches of the reference's |S01| < 1e-5 test are evaluated and the
  // result selected, so lanes of a warp do not diverge; the selected values
  // are those of the taken branch (the other one may be NaN and is dropped).
  const float tao = rmul(0.5f, rsub(S00, S11));
  const float w = sqrtf(radd(rmul(tao, tao), rmul(S01, S01)));
  const float t = S01 / (tao > 0.0f ? radd(tao, w) : rsub(tao, w));
  const float jc = 1.0f / sqrtf(radd(rmul(t, t), 1.0f));
  const float js = rmul(-t, jc);
  const float cc2 = rmul(jc, jc), ss2 = rmul(js, js);
  const float cs2 = rmul(rmul(2.0f, jc), js);
  const float j1 = radd(rsub(rmul(cc2, S00), rmul(cs2, S01)), rmul(ss2, S11));
  const float j2 = radd(radd(rmul(ss2, S00), rmul(cs2, S01)), rmul(cc2, S11));
  const bool diagonal = fabsf(S01) < 1e-5f;
  o.cc = diagonal ? 1.0f : jc;
  o.ss = diagonal ? 0.0f : js;
  o.s1 = diagonal ? S00 : j1;
  o.s2 = diagonal ? S11 : j2;
  return o;
}

__device__ __forceinline__ void jf_svd2_vectors(const JfSvdRot& r, float4& U, float2& sig, float4& V) {
  float s1 = r.s1, s2 = r.s2;
  const float cc = r.cc, ss = r.ss, c = r.c, s = r.s, ms = -r.s;
  float V00, V01, V10, V11;
  if (s1 < s2) {
    const float tmp = s1; s1 = s2; s2 = tmp;
    V00 = -ss; V01 = cc; V10 = -cc; V11 = -ss;
  } else {
    V00 = cc; V01 = ss; V10 = -ss; V11 = cc;
  }
  U = make_float4(rdot2(c, V00, ms, V10), rdot2(c, V01, ms, V11), rdot2(s, V00, c, V10),
                  rdot2(s, V01, c, V11));
  V = make_float4(V00, V01, V10, V11);
  sig = make_float2(s1, s2);
}

// Quadratic B-spline stencil of one particle (mpm_sim.py:183-187).  Returns
// false when the particle lies outside [0, n-2) in either axis; the cast
// truncates toward zero, as Taichi's .cast(int) does.
struct JfStencil {
  int bx, by;
  float fx0, fx1;
  float wx0, wx1, wx2, wy0, wy1, wy2;
};

__device__ __forceinline__ bool jf_stencil(const JfInst& I, float2 x, JfStencil& st) {
  st.bx = (int)(x.x * I.inv_dx - 0.5f);
  st.by = (int)(x.y * I.inv_dx - 0.5f);
  if (st.bx < 0 || st.by < 0 || st.bx >= I.nx - 2 || st.by >= I.ny - 2) return false;
  st.fx0 = x.x * I.inv_dx - (float)st.bx;
  st.fx1 = x.y * I.inv_dx - (float)st.by;
  float a0 = 1.5f - st.fx0, a1 = 1.5f - st.fx1;
  float b0 = st.fx0 - 1.0f, b1 = st.fx1 - 1.0f;
  float e0 = st.fx0 - 0.5f, e1 = st.fx1 - 0.5f;
  st.wx0 = 0.5f * (a0 * a0); st.wx1 = 0.75f - b0 * b0; st.wx2 = 0.5f * (e0 * e0);
  st.wy0 = 0.5f * (a1 * a1); st.wy1 = 0.75f - b1 * b1; st.wy2 = 0.5f * (e1 * e1);
  return true;
}

// jf_stencil with every operation rounded on its own, as the reference's FP32
// arithmetic rounds it (the base cast, fx and the weights; no fused
// multiply-adds).  The differentiable rollout's deterministic forward and its
// adjoints use it, so that their stencils match the oracle's bit for bit.
__device__ __forceinline__ bool jf_stencil_strict(const JfInst& I, float2 x, JfStencil& st) {
  const float X = __fmul_rn(x.x, I.inv_dx), Y = __fmul_rn(x.y, I.inv_dx);
  st.bx = (int)__fsub_rn(X, 0.5f);
  st.by = (int)__fsub_rn(Y, 0.5f);
  if (st.bx < 0 || st.by < 0 || st.bx >= I.nx - 2 || st.by >= I.ny - 2) return false;
  st.fx0 = __fsub_rn(X, (float)st.bx);
  st.fx1 = __fsub_rn(Y, (float)st.by);
  const float a0 = __fsub_rn(1.5f, st.fx0), a1 = __fsub_rn(1.5f, st.fx1);
  const float b0 = __fsub_rn(st.fx0, 1.0f), b1 = __fsub_rn(st.fx1, 1.0f);
  const float e0 = __fsub_rn(st.fx0, 0.5f), e1 = __fsub_rn(st.fx1, 0.5f);
  st.wx0 = __fmul_rn(0.5f, __fmul_rn(a0, a0));
  st.wx1 = __fsub_rn(0.75f, __fmul_rn(b0, b0));
  st.wx2 = __fmul_rn(0.5f, __fmul_rn(e0, e0));
  st.wy0 = __fmul_rn(0.5f, __fmul_rn(a1, a1));
  st.wy1 = __fsub_rn(0.75f, __fmul_rn(b1, b1));
  st.wy2 = __fmul_rn(0.5f, __fmul_rn(e1, e1));
  return true;
}

__device__ __forceinline__ float jf_w(const JfStencil& s, int axis, int k) {
  if (axis == 0) return k == 0 ? s.wx0 : (k == 1 ? s.wx1 : s.wx2);
  return k == 0 ? s.wy0 : (k == 1 ? s.wy1 : s.wy2);
}

// Per-particle scatter terms of P2G: the mass channel (mass, times the radius
// r_p in the axisymmetric variant), APIC affine matrix, momentum (mass r_p v
// there) and, axisymmetric only, mass * (sigma_rr - sigma_thetatheta).
struct JfScatter {
  float mass;
  float af00, af01, af10, af11;
  float mv0, mv1;
  float hoop;
};

// P2G for one particle (mpm_sim.py:189-254): F <- (I + dt C) F, SVD,
// plasticity (payload clamps sigma to [1-5e-3, 1+5e-3]; water resets
// F = sqrt(J) I), fixed-corotated Kirchhoff stress plus the muscle's active
// fibre stress, scaled, plus the APIC term.  Jp is updated only when the
// material is payload (for every other material the ratio is exactly 1).
// Axisymmetric variant (:235-268): xr = the particle's radius x[0], rref its
// load radius; the hoop stress uses the stretch max(xr, dx/20) / max(rref, dx/10).
__device__ __forceinline__ void jf_p2g_particle(const JfInst& I, const JfMaterials& mats, int mt,
                                                float2 v, float4 C, float4& F, float& Jp,
                                                float2 fiber, float pressure, float pdens,
                                                JfScatter& o, float xr = 0.0f, float rref = 1.0f) {
  const float dt = I.dt;
  {
    const float A00 = radd(1.0f, rmul(dt, C.x)), A01 = rmul(dt, C.y);
    const float A10 = rmul(dt, C.z), A11 = radd(1.0f, rmul(dt, C.w));
    F = make_float4(rdot2(A00, F.x, A01, F.z), rdot2(A00, F.y, A01, F.w), rdot2(A10, F.x, A11, F.z),
                    rdot2(A10, F.y, A11, F.w));
  }
  // constant-index selects keep the table in registers (no local-memory copy)
  const int ms = jf_mat_slot(mt);
  const float mu = ms == 0 ? mats.mu[0] : ms == 1 ? mats.mu[1] : ms == 2 ? mats.mu[2]
                 : ms == 3 ? mats.mu[3] : mats.mu[4];
  const float la = ms == 0 ? mats.la[0] : ms == 1 ? mats.la[1] : ms == 2 ? mats.la[2]
                 : ms == 3 ? mats.la[3] : mats.la[4];
  float mass = I.p_mass;
  if (mt == 2) mass = rmul(mass, pdens);

  const JfSvdRot rot = jf_svd2_values(F);
  float s00, s01, s10, s11, J;
  if (mt == 0) {
    // water: mu = 0, so the corotated term 2 mu (F - R) F^T of the stress is
    // exactly zero for finite F and only J = s1 s2 is needed (the product
    // does not depend on the singular values' order); F = sqrt(J) I
    J = rmul(fmaxf(rot.s1, 1e-6f), fmaxf(rot.s2, 1e-6f));
    const float sj = sqrtf(J);
    F = make_float4(sj, 0.0f, 0.0f, sj);
    const float diag = rmul(rmul(la, J), rsub(J, 1.0f));
    s00 = diag;
    s01 = 0.0f;
    s10 = 0.0f;
    s11 = diag;
  } else {
    float4 U, V;
    float2 sig;
    jf_svd2_vectors(rot, U, sig, V);
    sig.x = fmaxf(sig.x, 1e-6f);
    sig.y = fmaxf(sig.y, 1e-6f);
    if (mt == 2) {
      const float n0 = fminf(fmaxf(sig.x, 0.995f), 1.005f);
      const float n1 = fminf(fmaxf(sig.y, 0.995f), 1.005f);
      Jp = rmul(Jp, sig.x / n0);
      Jp = rmul(Jp, sig.y / n1);
      sig = make_float2(n0, n1);
    }
    J = rmul(sig.x, sig.y);
    if (mt == 2) {
      const float US00 = rmul(U.x, sig.x), US01 = rmul(U.y, sig.y);
      const float US10 = rmul(U.z, sig.x), US11 = rmul(U.w, sig.y);
      F = make_float4(rdot2(US00, V.x, US01, V.y), rdot2(US00, V.z, US01, V.w),
                      rdot2(US10, V.x, US11, V.y), rdot2(US10, V.z, US11, V.w));
    }
    const float R00 = rdot2(U.x, V.x, U.y, V.y);
    const float R01 = rdot2(U.x, V.z, U.y, V.w);
    const float R10 = rdot2(U.z, V.x, U.w, V.y);
    const float R11 = rdot2(U.z, V.z, U.w, V.w);
    const float twomu = rmul(2.0f, mu);
    const float E00 = rmul(twomu, rsub(F.x, R00)), E01 = rmul(twomu, rsub(F.y, R01));
    const float E10 = rmul(twomu, rsub(F.z, R10)), E11 = rmul(twomu, rsub(F.w, R11));
    const float diag = rmul(rmul(la, J), rsub(J, 1.0f));
    s00 = radd(rdot2(E00, F.x, E01, F.y), diag);
    s01 = rdot2(E00, F.z, E01, F.w);
    s10 = rdot2(E10, F.x, E11, F.y);
    s11 = radd(rdot2(E10, F.z, E11, F.w), diag);
    if (mt == 3) {
      s00 = radd(s00, rmul(rmul(rmul(fiber.x, fiber.x), pressure), J));
      s01 = radd(s01, rmul(rmul(rmul(fiber.x, fiber.y), pressure), J));
      s10 = radd(s10, rmul(rmul(rmul(fiber.y, fiber.x), pressure), J));
      s11 = radd(s11, rmul(rmul(rmul(fiber.y, fiber.y), pressure), J));
    }
  }
  const float k = I.stress_scale;
  float mch = mass;
  o.hoop = 0.0f;
  if (I.axisym) {
    // sigma_rr is the unscaled stress s00; for water (mu = 0) sigma_thetatheta
    // equals it exactly, so its hoop term is zero
    if (mt != 0) {
      const float lam = __fdiv_rn(fmaxf(xr, I.r_lo), fmaxf(rref, I.rref_lo));
      const float khoop = radd(rmul(rmul(2.0f, mu), rsub(lam, 1.0f)), rmul(rmul(la, J), rsub(J, 1.0f)));
      o.hoop = rmul(mass, rsub(s00, khoop));
    }
    mch = rmul(mass, xr);
  }
  o.mass = mch;
  o.af00 = rdot2(k, s00, mass, C.x);
  o.af01 = rdot2(k, s01, mass, C.y);
  o.af10 = rdot2(k, s10, mass, C.z);
  o.af11 = rdot2(k, s11, mass, C.w);
  o.mv0 = rmul(mch, v.x);
  o.mv1 = rmul(mch, v.y);
}

// Contribution of a particle to stencil node (i, j), i, j in 0..2
// (mpm_sim.py:256-271): (weight * momentum_x, weight * momentum_y, weight * mass).
__device__ __forceinline__ float3 jf_node_contrib(const JfInst& I, const JfStencil& st,
                                                  const JfScatter& sc, int i, int j) {
  float d0 = ((float)i - st.fx0) * I.dx;
  float d1 = ((float)j - st.fx1) * I.dx;
  float weight = jf_w(st, 0, i) * jf_w(st, 1, j);
  float c0 = weight * (sc.mv0 + (sc.af00 * d0 + sc.af01 * d1));
  float c1 = weight * (sc.mv1 + (sc.af10 * d0 + sc.af11 * d1));
  return make_float3(c0, c1, weight * sc.mass);
}

// jf_node_contrib with every operation rounded on its own (mpm_sim.py:256-271
// evaluated as the reference's FP32 code evaluates it).
__device__ __forceinline__ float3 jf_node_contrib_strict(const JfInst& I, const JfStencil& st,
                                                         const JfScatter& sc, int i, int j) {
  const float d0 = __fmul_rn(__fsub_rn((float)i, st.fx0), I.dx);
  const float d1 = __fmul_rn(__fsub_rn((float)j, st.fx1), I.dx);
  const float weight = __fmul_rn(jf_w(st, 0, i), jf_w(st, 1, j));
  const float c0 = __fmul_rn(weight, __fadd_rn(sc.mv0, rdot2(sc.af00, d0, sc.af01, d1)));
  const float c1 = __fmul_rn(weight, __fadd_rn(sc.mv1, rdot2(sc.af10, d0, sc.af11, d1)));
  return make_float3(c0, c1, __fmul_rn(weight, sc.mass));
}

// Grid node update (mpm_sim.py:274-309): normalise by mass, damp in a band of
// n//20 nodes on all four sides, zero the velocity component pointing into a
// wall within 3 nodes.  Nodes without mass keep their (zero) momentum.
// Axisymmetric variant (:292-303): h = sum of mass * (sigma_rr - sigma_tt);
// v_r += dt (h / m) / r_node off the axis cell, v_r = 0 on the axis (i = 0)
// instead of the i < 3 wall.
__device__ __forceinline__ float2 jf_grid_node(const JfInst& I, int i, int j, float gx, float gy,
                                               float m, float h = 0.0f) {
  if (!(m > 0.0f)) return make_float2(gx, gy);
  float g0 = gx / m, g1 = gy / m;
  float damp = 1.0f;
  if (i < I.dcx) damp = damp * (0.95f + 0.05f * (float)i / (float)I.dcx);
  if (i > I.nx - I.dcx) damp = damp * (0.95f + 0.05f * (float)(I.nx - i) / (float)I.dcx);
  if (j < I.dcy) damp = damp * (0.95f + 0.05f * (float)j / (float)I.dcy);
  if (j > I.ny - I.dcy) damp = damp * (0.95f + 0.05f * (float)(I.ny - j) / (float)I.dcy);
  g0 = g0 * damp;
  g1 = g1 * damp;
  if (I.axisym) {
    const float r_node = ((float)i + 0.5f) * I.dx;
    if (r_node > I.dx) g0 = g0 + (I.dt * (h / m)) / r_node;
    if (i == 0) g0 = 0.0f;
  } else if (i < 3 && g0 < 0.0f) {
    g0 = 0.0f;
  }
  if (i > I.nx - 3 && g0 > 0.0f) g0 = 0.0f;
  if (j < 3 && g1 < 0.0f) g1 = 0.0f;
  if (j > I.ny - 3 && g1 > 0.0f) g1 = 0.0f;
  return make_float2(g0, g1);
}

// APIC gather of G2P (mpm_sim.py:317-327) for a particle whose stencil is in
// range: new v and C from the updated grid.  `gather(i, j)` returns the
// updated velocity of stencil node (bx + i, by + j), i, j in 0..2.  The sums
// are formed row by row (sum over i, then weighted by the y weight), a
// re-association of the reference's node-by-node sum that moves results by
// rounding only.
template <class Gather>
__device__ __forceinline__ void jf_g2p_apic(const JfInst& I, const JfStencil& st, float2& v, float4& C,
                                            Gather gather) {
  const float wx[3] = {st.wx0, st.wx1, st.wx2};
  const float wy[3] = {st.wy0, st.wy1, st.wy2};
  float wxd[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) wxd[i] = wx[i] * ((float)i - st.fx0);
  float nv0 = 0.f, nv1 = 0.f, c00 = 0.f, c01 = 0.f, c10 = 0.f, c11 = 0.f;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    float sx = 0.f, sy = 0.f, tx = 0.f, ty = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float2 g = gather(i, j);
      sx += wx[i] * g.x;
      sy += wx[i] * g.y;
      tx += wxd[i] * g.x;
      ty += wxd[i] * g.y;
    }
    const float wyd = wy[j] * ((float)j - st.fx1);
    nv0 += wy[j] * sx;
    nv1 += wy[j] * sy;
    c00 += wy[j] * tx;
    c01 += wyd * sx;
    c10 += wy[j] * ty;
    c11 += wyd * sy;
  }
  v = make_float2(nv0, nv1);
  C = make_float4(I.c4 * c00, I.c4 * c01, I.c4 * c10, I.c4 * c11);
}

// The APIC gather of G2P in the reference's own operation order
// (mpm_sim.py:317-327): nodes i outer, j inner, weight = w_i w_j,
// new_v += weight g_v and new_C += (4 inv_dx weight) (g_v outer dpos), every
// operation rounded on its own.  The deterministic forward of the
// differentiable rollout uses it, so that the rollout reproduces the oracle's
// arithmetic exactly apart from the order of the P2G sums.
template <class Gather>
__device__ __forceinline__ void jf_g2p_apic_nodes(const JfInst& I, const JfStencil& st, float2& v, float4& C,
                                                  Gather gather) {
  const float wx[3] = {st.wx0, st.wx1, st.wx2};
  const float wy[3] = {st.wy0, st.wy1, st.wy2};
  float nv0 = 0.f, nv1 = 0.f, c00 = 0.f, c01 = 0.f, c10 = 0.f, c11 = 0.f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float d0 = __fsub_rn((float)i, st.fx0), d1 = __fsub_rn((float)j, st.fx1);
      const float2 g = gather(i, j);
      const float w = __fmul_rn(wx[i], wy[j]);
      nv0 = __fadd_rn(nv0, __fmul_rn(w, g.x));
      nv1 = __fadd_rn(nv1, __fmul_rn(w, g.y));
      const float k = __fmul_rn(I.c4, w);
      c00 = __fadd_rn(c00, __fmul_rn(k, __fmul_rn(g.x, d0)));
      c01 = __fadd_rn(c01, __fmul_rn(k, __fmul_rn(g.x, d1)));
      c10 = __fadd_rn(c10, __fmul_rn(k, __fmul_rn(g.y, d0)));
      c11 = __fadd_rn(c11, __fmul_rn(k, __fmul_rn(g.y, d1)));
    }
  }
  v = make_float2(nv0, nv1);
  C = make_float4(c00, c01, c10, c11);
}

// Gravity, advection and the wall clamp of every live particle
// (mpm_sim.py:329-333).
__device__ __forceinline__ void jf_g2p_advect(const JfInst& I, float2& x, float2& v) {
  v.y = v.y - I.dtg;
  // rounded as the reference rounds it (product, then sum): a fused
  // multiply-add here shifts 1,000-step payload displacement by ~0.2%
  x.x = __fadd_rn(x.x, __fmul_rn(I.dt, v.x));
  x.y = __fadd_rn(x.y, __fmul_rn(I.dt, v.y));
  x.x = fmaxf(fminf(x.x, 0.999f), 0.001f);
  x.y = fmaxf(fminf(x.y, I.y_hi), 0.001f);
}

// G2P for one particle (mpm_sim.py:315-333).  `gather(i_node, j_node)`
// returns the updated grid velocity of an absolute node.
template <class Gather>
__device__ __forceinline__ void jf_g2p_particle(const JfInst& I, float2& x, float2& v, float4& C,
                                                Gather gather) {
  JfStencil st;
  if (jf_stencil(I, x, st)) {
    jf_g2p_apic(I, st, v, C, [&](int i, int j) { return gather(st.bx + i, st.by + j); });
  }
  jf_g2p_advect(I, x, v);
}

// visual_glow decay (mpm_sim.py:336-338), render-only.
__device__ __forceinline__ float jf_glow(float glow, float Jp) {
  return fmaxf(glow * 0.9f, fabsf(1.0f - Jp));
}
