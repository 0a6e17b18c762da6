// FP64 versions of the device math the differentiable rollout uses, for its
// FP64 build (JF_FLAG_GRAD_FP64).  Each function has the name and the
// operation order of its FP32 counterpart in jf_device.cuh, which follows the
// reference engine mpm_sim.py; here every constant is the reference's Python
// double expression itself (not rounded to FP32) and every operation is a
// separately rounded double operation, as the oracle's REAL=double build
// evaluates it.  The axisymmetric variant has no FP64 build (the
// differentiable rollout rejects it).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "jf_device.cuh"

// separately rounded FP64 operations (never fused)
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rdot2(double a, double b, double c, double d) {
  return __dadd_rn(__dmul_rn(a, b), __dmul_rn(c, d));
}

// Per-instance description in FP64 (the JfInst of the FP32 path with its
// constants as doubles, mpm_sim.py:18-58).
struct JfInst64 {
  int32_t nx, ny, dcx, dcy;
  int32_t n_slots;
  int64_t p_off, g_off;
  double inv_dx, dx, dt, p_mass;
  double stress_scale;  // -dt * p_vol * 4 * inv_dx^2
  double c4;            // 4 * inv_dx
  double dtg;           // dt * gravity
  double y_hi;          // domain_height - 0.001
};

struct JfMaterials64 {
  double mu[5];
  double la[5];
};

struct JfStencil64 {
  int bx, by;
  double fx0, fx1;
  double wx0, wx1, wx2, wy0, wy1, wy2;
};

struct JfScatter64 {
  double mass;
  double af00, af01, af10, af11;
  double mv0, mv1;
  double hoop;  // unused (no axisymmetric FP64 build); kept for the shared kernel code
};

struct JfSvdRot64 {
  double c, s, cc, ss, s1, s2;
};

// activation of the waveform (mpm_sim.py:173-180) in FP64
__device__ __forceinline__ double jf_activation64(double freq, double contraction, double t) {
  const double period = 1.0 / rmul(1.0, freq);
  const double q = floor(t / period);
  const double r = rsub(t, rmul(period, q));
  const double phase = r / period;
  double a = 0.0;
  if (phase < contraction) {
    const double arg = rmul(phase / contraction, 3.14159265);
    a = rmul(0.5, rsub(1.0, cos(arg)));
  }
  return a;
}

__device__ __forceinline__ bool jf_stencil_strict(const JfInst64& I, double2 x, JfStencil64& st) {
  const double X = rmul(x.x, I.inv_dx), Y = rmul(x.y, I.inv_dx);
  st.bx = (int)rsub(X, 0.5);
  st.by = (int)rsub(Y, 0.5);
  if (st.bx < 0 || st.by < 0 || st.bx >= I.nx - 2 || st.by >= I.ny - 2) return false;
  st.fx0 = rsub(X, (double)st.bx);
  st.fx1 = rsub(Y, (double)st.by);
  const double a0 = rsub(1.5, st.fx0), a1 = rsub(1.5, st.fx1);
  const double b0 = rsub(st.fx0, 1.0), b1 = rsub(st.fx1, 1.0);
  const double e0 = rsub(st.fx0, 0.5), e1 = rsub(st.fx1, 0.5);
  st.wx0 = rmul(0.5, rmul(a0, a0));
  st.wx1 = rsub(0.75, rmul(b0, b0));
  st.wx2 = rmul(0.5, rmul(e0, e0));
  st.wy0 = rmul(0.5, rmul(a1, a1));
  st.wy1 = rsub(0.75, rmul(b1, b1));
  st.wy2 = rmul(0.5, rmul(e1, e1));
  return true;
}

__device__ __forceinline__ double jf_w(const JfStencil64& s, int axis, int k) {
  if (axis == 0) return k == 0 ? s.wx0 : (k == 1 ? s.wx1 : s.wx2);
  return k == 0 ? s.wy0 : (k == 1 ? s.wy1 : s.wy2);
}

__device__ __forceinline__ double3 jf_node_contrib_strict(const JfInst64& I, const JfStencil64& st,
                                                          const JfScatter64& sc, int i, int j) {
  const double d0 = rmul(rsub((double)i, st.fx0), I.dx);
  const double d1 = rmul(rsub((double)j, st.fx1), I.dx);
  const double weight = rmul(jf_w(st, 0, i), jf_w(st, 1, j));
  const double c0 = rmul(weight, radd(sc.mv0, rdot2(sc.af00, d0, sc.af01, d1)));
  const double c1 = rmul(weight, radd(sc.mv1, rdot2(sc.af10, d0, sc.af11, d1)));
  return make_double3(c0, c1, rmul(weight, sc.mass));
}

__device__ __forceinline__ JfSvdRot64 jf_svd2_values(double4 A) {
  JfSvdRot64 o;
  const double x = radd(A.x, A.w);
  const double y = rsub(A.z, A.y);
  const double scale = 1.0 / sqrt(radd(rmul(x, x), rmul(y, y)));
  o.c = rmul(x, scale);
  o.s = rmul(y, scale);
  const double ms = -o.s;
  const double S00 = rdot2(o.c, A.x, o.s, A.z);
  const double S01 = rdot2(o.c, A.y, o.s, A.w);
  const double S11 = rdot2(ms, A.y, o.c, A.w);
  const double tao = rmul(0.5, rsub(S00, S11));
  const double w = sqrt(radd(rmul(tao, tao), rmul(S01, S01)));
  const double t = S01 / (tao > 0.0 ? radd(tao, w) : rsub(tao, w));
  const double jc = 1.0 / sqrt(radd(rmul(t, t), 1.0));
  const double js = rmul(-t, jc);
  const double cc2 = rmul(jc, jc), ss2 = rmul(js, js);
  const double cs2 = rmul(rmul(2.0, jc), js);
  const double j1 = radd(rsub(rmul(cc2, S00), rmul(cs2, S01)), rmul(ss2, S11));
  const double j2 = radd(radd(rmul(ss2, S00), rmul(cs2, S01)), rmul(cc2, S11));
  const bool diagonal = fabs(S01) < 1e-5;
  o.cc = diagonal ? 1.0 : jc;
  o.ss = diagonal ? 0.0 : js;
  o.s1 = diagonal ? S00 : j1;
  o.s2 = diagonal ? S11 : j2;
  return o;
}

__device__ __forceinline__ void jf_svd2_vectors(const JfSvdRot64& r, double4& U, double2& sig, double4& V) {
  double s1 = r.s1, s2 = r.s2;
  const double cc = r.cc, ss = r.ss, c = r.c, s = r.s, ms = -r.s;
  double V00, V01, V10, V11;
  if (s1 < s2) {
    const double tmp = s1; s1 = s2; s2 = tmp;
    V00 = -ss; V01 = cc; V10 = -cc; V11 = -ss;
  } else {
    V00 = cc; V01 = ss; V10 = -ss; V11 = cc;
  }
  U = make_double4(rdot2(c, V00, ms, V10), rdot2(c, V01, ms, V11), rdot2(s, V00, c, V10),
                   rdot2(s, V01, c, V11));
  V = make_double4(V00, V01, V10, V11);
  sig = make_double2(s1, s2);
}

// P2G material update and scatter terms of one particle (mpm_sim.py:189-254).
__device__ __forceinline__ void jf_p2g_particle(const JfInst64& I, const JfMaterials64& mats, int mt, double2 v,
                                                double4 C, double4& F, double& Jp, float2 fiber,
                                                double pressure, double pdens, JfScatter64& o) {
  const double dt = I.dt;
  {
    const double A00 = radd(1.0, rmul(dt, C.x)), A01 = rmul(dt, C.y);
    const double A10 = rmul(dt, C.z), A11 = radd(1.0, rmul(dt, C.w));
    F = make_double4(rdot2(A00, F.x, A01, F.z), rdot2(A00, F.y, A01, F.w), rdot2(A10, F.x, A11, F.z),
                     rdot2(A10, F.y, A11, F.w));
  }
  const int ms = jf_mat_slot(mt);
  const double mu = ms == 0 ? mats.mu[0] : ms == 1 ? mats.mu[1] : ms == 2 ? mats.mu[2]
                  : ms == 3 ? mats.mu[3] : mats.mu[4];
  const double la = ms == 0 ? mats.la[0] : ms == 1 ? mats.la[1] : ms == 2 ? mats.la[2]
                  : ms == 3 ? mats.la[3] : mats.la[4];
  double mass = I.p_mass;
  if (mt == 2) mass = rmul(mass, pdens);
  const JfSvdRot64 rot = jf_svd2_values(F);
  double s00, s01, s10, s11, J;
  if (mt == 0) {
    J = rmul(fmax(rot.s1, 1e-6), fmax(rot.s2, 1e-6));
    const double sj = sqrt(J);
    F = make_double4(sj, 0.0, 0.0, sj);
    const double diag = rmul(rmul(la, J), rsub(J, 1.0));
    s00 = diag; s01 = 0.0; s10 = 0.0; s11 = diag;
  } else {
    double4 U, V;
    double2 sig;
    jf_svd2_vectors(rot, U, sig, V);
    sig.x = fmax(sig.x, 1e-6);
    sig.y = fmax(sig.y, 1e-6);
    if (mt == 2) {
      const double n0 = fmin(fmax(sig.x, 1 - 5e-3), 1 + 5e-3);
      const double n1 = fmin(fmax(sig.y, 1 - 5e-3), 1 + 5e-3);
      Jp = rmul(Jp, sig.x / n0);
      Jp = rmul(Jp, sig.y / n1);
      sig = make_double2(n0, n1);
    }
    J = rmul(sig.x, sig.y);
    if (mt == 2) {
      const double US00 = rmul(U.x, sig.x), US01 = rmul(U.y, sig.y);
      const double US10 = rmul(U.z, sig.x), US11 = rmul(U.w, sig.y);
      F = make_double4(rdot2(US00, V.x, US01, V.y), rdot2(US00, V.z, US01, V.w), rdot2(US10, V.x, US11, V.y),
                       rdot2(US10, V.z, US11, V.w));
    }
    const double R00 = rdot2(U.x, V.x, U.y, V.y);
    const double R01 = rdot2(U.x, V.z, U.y, V.w);
    const double R10 = rdot2(U.z, V.x, U.w, V.y);
    const double R11 = rdot2(U.z, V.z, U.w, V.w);
    const double twomu = rmul(2.0, mu);
    const double E00 = rmul(twomu, rsub(F.x, R00)), E01 = rmul(twomu, rsub(F.y, R01));
    const double E10 = rmul(twomu, rsub(F.z, R10)), E11 = rmul(twomu, rsub(F.w, R11));
    const double diag = rmul(rmul(la, J), rsub(J, 1.0));
    s00 = radd(rdot2(E00, F.x, E01, F.y), diag);
    s01 = rdot2(E00, F.z, E01, F.w);
    s10 = rdot2(E10, F.x, E11, F.y);
    s11 = radd(rdot2(E10, F.z, E11, F.w), diag);
    if (mt == 3) {
      const double fx = fiber.x, fy = fiber.y;
      s00 = radd(s00, rmul(rmul(rmul(fx, fx), pressure), J));
      s01 = radd(s01, rmul(rmul(rmul(fx, fy), pressure), J));
      s10 = radd(s10, rmul(rmul(rmul(fy, fx), pressure), J));
      s11 = radd(s11, rmul(rmul(rmul(fy, fy), pressure), J));
    }
  }
  const double k = I.stress_scale;
  o.hoop = 0.0;
  o.mass = mass;
  o.af00 = rdot2(k, s00, mass, C.x);
  o.af01 = rdot2(k, s01, mass, C.y);
  o.af10 = rdot2(k, s10, mass, C.z);
  o.af11 = rdot2(k, s11, mass, C.w);
  o.mv0 = rmul(mass, v.x);
  o.mv1 = rmul(mass, v.y);
}

// grid node update (mpm_sim.py:274-309), Cartesian
__device__ __forceinline__ double2 jf_grid_node(const JfInst64& I, int i, int j, double gx, double gy, double m) {
  if (!(m > 0.0)) return make_double2(gx, gy);
  double g0 = gx / m, g1 = gy / m;
  double damp = 1.0;
  if (i < I.dcx) damp = rmul(damp, radd(0.95, (rmul(0.05, (double)i)) / (double)I.dcx));
  if (i > I.nx - I.dcx) damp = rmul(damp, radd(0.95, (rmul(0.05, (double)(I.nx - i))) / (double)I.dcx));
  if (j < I.dcy) damp = rmul(damp, radd(0.95, (rmul(0.05, (double)j)) / (double)I.dcy));
  if (j > I.ny - I.dcy) damp = rmul(damp, radd(0.95, (rmul(0.05, (double)(I.ny - j))) / (double)I.dcy));
  g0 = rmul(g0, damp);
  g1 = rmul(g1, damp);
  if (i < 3 && g0 < 0.0) g0 = 0.0;
  if (i > I.nx - 3 && g0 > 0.0) g0 = 0.0;
  if (j < 3 && g1 < 0.0) g1 = 0.0;
  if (j > I.ny - 3 && g1 > 0.0) g1 = 0.0;
  return make_double2(g0, g1);
}

template <class Gather>
__device__ __forceinline__ void jf_g2p_apic_nodes(const JfInst64& I, const JfStencil64& st, double2& v, double4& C,
                                                  Gather gather) {
  const double wx[3] = {st.wx0, st.wx1, st.wx2};
  const double wy[3] = {st.wy0, st.wy1, st.wy2};
  double nv0 = 0.0, nv1 = 0.0, c00 = 0.0, c01 = 0.0, c10 = 0.0, c11 = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double d0 = rsub((double)i, st.fx0), d1 = rsub((double)j, st.fx1);
      const double2 g = gather(i, j);
      const double w = rmul(wx[i], wy[j]);
      nv0 = radd(nv0, rmul(w, g.x));
      nv1 = radd(nv1, rmul(w, g.y));
      const double k = rmul(I.c4, w);
      c00 = radd(c00, rmul(k, rmul(g.x, d0)));
      c01 = radd(c01, rmul(k, rmul(g.x, d1)));
      c10 = radd(c10, rmul(k, rmul(g.y, d0)));
      c11 = radd(c11, rmul(k, rmul(g.y, d1)));
    }
  }
  v = make_double2(nv0, nv1);
  C = make_double4(c00, c01, c10, c11);
}

__device__ __forceinline__ void jf_g2p_advect(const JfInst64& I, double2& x, double2& v) {
  v.y = rsub(v.y, I.dtg);
  x.x = radd(x.x, rmul(I.dt, v.x));
  x.y = radd(x.y, rmul(I.dt, v.y));
  x.x = fmax(fmin(x.x, 0.999), 0.001);
  x.y = fmax(fmin(x.y, I.y_hi), 0.001);
}
