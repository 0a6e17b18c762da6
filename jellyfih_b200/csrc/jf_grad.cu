// Differentiable rollout: d(payload displacement) / d(actuation amplitude,
// contraction fraction, frequency multiplier, initial positions).
//
// Forward: the substep of the plain path with one change, a deterministic
// P2G (momentum and mass accumulated in 2^-44 fixed point with 64-bit integer
// atomics, whose sums do not depend on the order of the atomics), so that a
// segment recomputed from its checkpoint reproduces the forward bit for bit.
// The state (x, v, C, F) is checkpointed every K substeps.
//
// Backward, per segment in reverse: restore the checkpoint, recompute the
// segment's K pre-step states and keep each substep's grid (updated
// velocity, momentum and mass per node), then for each substep in reverse run the
// hand-written adjoints of G2P (mpm_sim.py:312-333), of the grid update
// (:274-309) and of P2G (:168-271).  The material map F* -> (F_out, tau)
// (SVD, plasticity, stress) is differentiated with four-tangent dual numbers
// (jf_dual.cuh); everything else is written out by hand.  Integer cell bases,
// clamps at their bounds and boundary-zeroed grid components carry no
// gradient, as in an autodiff of the same code.
//
// The waveform drops from 1 to 0 when the phase reaches the contraction
// fraction (mpm_sim.py:176-180).  A discrete adjoint does not see that jump
// (nor would Taichi's autodiff), but moving the contraction fraction or the
// frequency moves the instant of the drop, and the loss moves with it.  The
// backward therefore records dL/dpressure of every substep and adds, for every
// drop inside the rollout, the boundary term of the time integral:
// dL/dc += A g* / (f dt) and dL/df -= A g* t* / (f dt) (t* the instant of
// the drop, g* dL/dpressure there, interpolated between the substeps around
// it; a(c-) = 1).
//
// Non-finite states: G2P flags an instance whose position or velocity is NaN
// or Inf, and P2G flags a contribution too large for the fixed-point sums
// (|value| >= 64, far beyond any physical momentum or mass of a particle), and
// adds zero for it; the adjoint flags non-finite adjoint states.  The flags
// are the engine's non-finite flags (jf_error_flags).

// Every operation of the deterministic forward is rounded on its own (the
// stencil, the node contributions and the G2P gather in the reference's node
// order), so that, apart from the order-free fixed-point P2G sums, it performs
// the reference's FP32 arithmetic exactly.
//
// Everything here is written once for a real type R and built twice: R =
// float (the default) and R = double (JF_FLAG_GRAD_FP64), the FP64 build of
// the same kernels, whose math (jf_device64.cuh) follows the oracle's FP64
// build.  In FP64 the P2G sums are plain double atomics (their order moves
// results by ~1e-16), the working state is a double copy of the engine's
// particles, and the final state is written back to them rounded to FP32.
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "jf_device64.cuh"
#include "jf_dual.cuh"
#include "jf_engine.h"

namespace {

constexpr int kT = 256;
constexpr float kFix = 17592186044416.0f;        // 2^44
constexpr double kFixInv = 1.0 / 17592186044416.0;

// The types of each precision: the instance description, materials,
// stencil and scatter terms of jf_device.cuh (FP32) or jf_device64.cuh
// (FP64), vector types, and the P2G accumulator (2^-44 fixed point in FP32,
// double in FP64).
template <class R> struct GT;
template <> struct GT<float> {
  using Inst = JfInst;
  using Mats = JfMaterials;
  using Stencil = JfStencil;
  using Scatter = JfScatter;
  using Rot = JfSvdRot;
  using V2 = float2;
  using V4 = float4;
  using Acc = unsigned long long;
};
template <> struct GT<double> {
  using Inst = JfInst64;
  using Mats = JfMaterials64;
  using Stencil = JfStencil64;
  using Scatter = JfScatter64;
  using Rot = JfSvdRot64;
  using V2 = double2;
  using V4 = double4;
  using Acc = double;
};
template <class R> using V2 = typename GT<R>::V2;
template <class R> using V4 = typename GT<R>::V4;

__host__ __device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ float4 mk4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
__host__ __device__ __forceinline__ double4 mk4(double a, double b, double c, double d) {
  return make_double4(a, b, c, d);
}

template <class R>
struct GradState {
  V4<R>* xv;
  V4<R>* C;
  V4<R>* F;
};

template <class R>
struct GradArgs {
  const typename GT<R>::Inst* inst;
  const JfParams* params;
  typename GT<R>::Mats mats;
  GradState<R> s;              // the state the kernel reads (pre-step)
  GradState<R> o;              // where it writes the post-step state (s itself in the forward)
  const int32_t* mat;
  R* Jp;
  const float2* fiber;
  typename GT<R>::Acc* fix;    // 3 per node: momentum x, momentum y, mass
  V2<R>* u;                    // updated grid velocity
  V4<R>* pmv;                  // if set: (momentum x, momentum y, mass) per node, kept for the adjoint
  int32_t* err;                // per-instance non-finite flags
  R t;
};

// Largest contribution the P2G sums take: |v| < 64 keeps v * 2^44 below
// 2^50, so 8,192 contributions to one node cannot overflow 2^63 (the FP64
// build keeps the same bound).
constexpr float kFixMax = 64.0f;

// v in 2^-44 fixed point; a non-finite or out-of-range v sets the instance's
// flag (bit 2) and contributes zero.
__device__ __forceinline__ unsigned long long to_fixed(float v, int32_t* flag) {
  if (!(fabsf(v) < kFixMax)) {
    atomicOr(flag, 2);
    return 0ull;
  }
  return (unsigned long long)__float2ll_rn(v * kFix);
}
// the same bound in FP64, where the contribution is added as it is
__device__ __forceinline__ double to_fixed(double v, int32_t* flag) {
  if (!(fabs(v) < (double)kFixMax)) {
    atomicOr(flag, 2);
    return 0.0;
  }
  return v;
}

template <class Acc, class R>
__device__ __forceinline__ void add_fixed(Acc* p, R v, int32_t* flag) {
  const Acc q = to_fixed(v, flag);
  if (q != Acc(0)) atomicAdd(p, q);
}
__device__ __forceinline__ float from_fixed(unsigned long long v) {
  return (float)((double)(long long)v * kFixInv);
}
__device__ __forceinline__ double from_fixed(double v) { return v; }

// the waveform's activation in each precision
__device__ __forceinline__ float activation(float freq, float contraction, float t) {
  return jf_activation(freq, contraction, t);
}
__device__ __forceinline__ double activation(double freq, double contraction, double t) {
  return jf_activation64(freq, contraction, t);
}

// per-block activation pressure of instance blockIdx.y at time a.t
template <class R>
__device__ __forceinline__ R block_pressure(const GradArgs<R>& a, int m) {
  __shared__ R s_p;
  if (threadIdx.x == 0) {
    const JfParams P = a.params[m];
    s_p = (R)P.actuation * activation((R)P.freq, (R)P.contraction, a.t);
  }
  __syncthreads();
  return s_p;
}

// Deterministic P2G.  A block's particles (consecutive slots of one
// instance) first add their contributions into a shared-memory tile covering
// the block's stencil bounding box, when that box has at most kTileNodes
// nodes, and the tile then goes to the grid with one atomic per touched node
// and component; otherwise each contribution goes to the grid directly.  In
// FP32 the contributions are integers, so every grouping gives the same sums
// bit for bit.
constexpr int kTileNodes = 1024;

template <class R>
__global__ void __launch_bounds__(kT) gf_p2g(GradArgs<R> a) {
  using Acc = typename GT<R>::Acc;
  __shared__ Acc s_acc[3 * kTileNodes];
  __shared__ int s_box[4];  // stencil bases: min x, min y, max x, max y
  const int m = blockIdx.y;
  const R pressure = block_pressure(a, m);
  const auto I = a.inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t g = I.p_off + k;
  const bool copy = a.o.F != a.s.F;
  bool valid = false;
  typename GT<R>::Stencil st;
  typename GT<R>::Scatter sc;
  if (k < I.n_slots) {
    const int mt = a.mat[g];
    const V4<R> xv = mt >= 0 ? a.s.xv[g] : mk4(R(0), R(0), R(0), R(0));
    if (mt >= 0 && jf_stencil_strict(I, mk2(xv.x, xv.y), st)) {
      V4<R> F = a.s.F[g];
      R jp = (mt == 2) ? a.Jp[g] : R(1);
      const float2 fb = (mt == 3) ? a.fiber[g] : make_float2(0.0f, 1.0f);
      jf_p2g_particle(I, a.mats, mt, mk2(xv.z, xv.w), a.s.C[g], F, jp, fb, pressure,
                      (R)a.params[m].payload_density, sc);
      a.o.F[g] = F;
      if (mt == 2) a.Jp[g] = jp;
      valid = true;
    } else if (copy) {
      a.o.F[g] = a.s.F[g];
    }
  }
  if (threadIdx.x == 0) {
    s_box[0] = s_box[1] = 0x7fffffff;
    s_box[2] = s_box[3] = -1;
  }
  __syncthreads();
  if (valid) {
    atomicMin(&s_box[0], st.bx);
    atomicMin(&s_box[1], st.by);
    atomicMax(&s_box[2], st.bx);
    atomicMax(&s_box[3], st.by);
  }
  __syncthreads();
  const int x0 = s_box[0], y0 = s_box[1];
  const int W = s_box[2] - x0 + 3, H = s_box[3] - y0 + 3;
  if (s_box[2] < 0) return;  // no particle of the block scatters (uniform)
  Acc* fix = a.fix + 3 * I.g_off;
  if (W * H > kTileNodes) {  // uniform: the direct path
    if (!valid) return;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const auto c = jf_node_contrib_strict(I, st, sc, i, j);
        const int64_t n = 3 * ((int64_t)(st.by + j) * I.nx + st.bx + i);
        add_fixed(fix + n + 0, c.x, a.err + m);
        add_fixed(fix + n + 1, c.y, a.err + m);
        add_fixed(fix + n + 2, c.z, a.err + m);
      }
    }
    return;
  }
  const int entries = 3 * W * H;
  for (int e = threadIdx.x; e < entries; e += blockDim.x) s_acc[e] = Acc(0);
  __syncthreads();
  if (valid) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const auto c = jf_node_contrib_strict(I, st, sc, i, j);
        Acc* t = s_acc + 3 * ((st.by + j - y0) * W + (st.bx + i - x0));
        atomicAdd(t + 0, to_fixed(c.x, a.err + m));
        atomicAdd(t + 1, to_fixed(c.y, a.err + m));
        atomicAdd(t + 2, to_fixed(c.z, a.err + m));
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < entries; e += blockDim.x) {
    const Acc v = s_acc[e];
    if (v == Acc(0)) continue;
    const int node = e / 3, comp = e - 3 * node;
    const int ty = node / W, tx = node - ty * W;
    atomicAdd(fix + 3 * ((int64_t)(y0 + ty) * I.nx + x0 + tx) + comp, v);
  }
}

template <class R>
__global__ void gf_grid(GradArgs<R> a) {
  const int m = blockIdx.y;
  const auto I = a.inst[m];
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= I.nx * I.ny) return;
  const typename GT<R>::Acc* q = a.fix + 3 * (I.g_off + n);
  const R px = from_fixed(q[0]), py = from_fixed(q[1]), pm = from_fixed(q[2]);
  a.u[I.g_off + n] = jf_grid_node(I, n % I.nx, n / I.nx, px, py, pm);
  if (a.pmv) a.pmv[I.g_off + n] = mk4(px, py, pm, R(0));
}

template <class R>
__global__ void gf_g2p(GradArgs<R> a) {
  const int m = blockIdx.y;
  const auto I = a.inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  if (a.mat[g] < 0) {
    if (a.o.xv != a.s.xv) {
      a.o.xv[g] = a.s.xv[g];
      a.o.C[g] = a.s.C[g];
    }
    return;
  }
  const V4<R> xv = a.s.xv[g];
  V2<R> x = mk2(xv.x, xv.y), v = mk2(xv.z, xv.w);
  V4<R> C = a.s.C[g];
  const V2<R>* u = a.u + I.g_off;
  const int nx = I.nx;
  typename GT<R>::Stencil st;
  if (jf_stencil_strict(I, x, st)) {
    jf_g2p_apic_nodes(I, st, v, C, [&](int i, int j) { return u[(st.by + j) * nx + st.bx + i]; });
  }
  jf_g2p_advect(I, x, v);
  if (!(isfinite(x.x) && isfinite(x.y) && isfinite(v.x) && isfinite(v.y))) atomicOr(a.err + m, 1);
  a.o.xv[g] = mk4(x.x, x.y, v.x, v.y);
  a.o.C[g] = C;
}

template <class R>
struct AdjArgs {
  GradArgs<R> f;       // pre-step state of this substep (segment buffer) and its kept grid (u, pmv)
  V4<R>* lxv;          // adjoint (x, v): in = post-step, out = pre-step
  V4<R>* lC;
  V4<R>* lF;
  V2<R>* ubar;         // adjoint of the updated grid velocity
  V4<R>* pmbar;        // adjoint of the accumulated momentum (x, y) and mass (z)
  V2<R>* xtmp;         // G2P part of the position adjoint
  V2<R>* vtmp;         // velocity adjoint of particles outside the stencil range
  double* gparam;      // M x 3: d/d actuation, d/d contraction, d/d freq
  double* dLdp;        // M: d L / d pressure of this substep, per instance
  double* fac;         // M x 3: d pressure / d (actuation, contraction, freq) of this substep
};

template <class R>
__device__ __forceinline__ R wd(int k, R f) {  // d W_k / d f
  return k == 0 ? -(R(1.5) - f) : (k == 1 ? R(-2) * (f - R(1)) : (f - R(0.5)));
}

template <class R>
__device__ __forceinline__ R clamp_pass(R xpp, R lo, R hi) {
  return (xpp > lo && xpp < hi) ? R(1) : R(0);
}

__device__ __forceinline__ void atomic_add2(float2* p, float a, float b) { atomicAdd(p, make_float2(a, b)); }
__device__ __forceinline__ void atomic_add2(double2* p, double a, double b) {
  atomicAdd(&p->x, a);
  atomicAdd(&p->y, b);
}

template <class R>
__global__ void ad_g2p(AdjArgs<R> A) {
  const GradArgs<R>& a = A.f;
  const int m = blockIdx.y;
  const auto I = a.inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  if (a.mat[g] < 0) return;
  const V4<R> xv = a.s.xv[g];
  V2<R> x = mk2(xv.x, xv.y), v = mk2(xv.z, xv.w);
  const V4<R> lxv = A.lxv[g];
  const V4<R> Cb = A.lC[g];
  typename GT<R>::Stencil st;
  const bool inr = jf_stencil_strict(I, x, st);
  const V2<R>* u = a.u + I.g_off;
  const int nx = I.nx;
  V2<R> vn = v;
  if (inr) {
    V4<R> Cn;
    jf_g2p_apic_nodes(I, st, vn, Cn, [&](int i, int j) { return u[(st.by + j) * nx + st.bx + i]; });
  }
  vn.y = vn.y - I.dtg;
  const R xpp0 = radd(x.x, rmul(I.dt, vn.x));
  const R xpp1 = radd(x.y, rmul(I.dt, vn.y));
  const R xd0 = lxv.x * clamp_pass(xpp0, R(0.001), R(0.999));
  const R xd1 = lxv.y * clamp_pass(xpp1, R(0.001), I.y_hi);
  const R vt0 = lxv.z + I.dt * xd0;
  const R vt1 = lxv.w + I.dt * xd1;
  if (!inr) {
    A.xtmp[g] = mk2(xd0, xd1);
    A.vtmp[g] = mk2(vt0, vt1);
    return;
  }
  const R wx[3] = {st.wx0, st.wx1, st.wx2};
  const R wy[3] = {st.wy0, st.wy1, st.wy2};
  R xb0 = R(0), xb1 = R(0), xe0 = R(0), xe1 = R(0);
  V2<R>* ub = A.ubar + I.g_off;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int n = (st.by + j) * nx + st.bx + i;
      const V2<R> uu = u[n];
      const R w = wx[i] * wy[j];
      const R e0 = (R)i - st.fx0, e1 = (R)j - st.fx1;
      const R ce0 = Cb.x * e0 + Cb.y * e1;  // (C_bar e)_0
      const R ce1 = Cb.z * e0 + Cb.w * e1;  // (C_bar e)_1
      atomic_add2(ub + n, w * vt0 + I.c4 * w * ce0, w * vt1 + I.c4 * w * ce1);
      const R sgl = uu.x * vt0 + uu.y * vt1 + I.c4 * (uu.x * ce0 + uu.y * ce1);
      xb0 += wd(i, st.fx0) * wy[j] * sgl;
      xb1 += wx[i] * wd(j, st.fx1) * sgl;
      xe0 += w * (Cb.x * uu.x + Cb.z * uu.y);
      xe1 += w * (Cb.y * uu.x + Cb.w * uu.y);
    }
  }
  const R cf = I.c4 * I.inv_dx;
  A.xtmp[g] = mk2(xd0 + I.inv_dx * xb0 - cf * xe0, xd1 + I.inv_dx * xb1 - cf * xe1);
  A.vtmp[g] = mk2(R(0), R(0));
}

// d pressure / d (actuation, contraction, freq) of instance m at time t: the
// activation a, A da/dc and A da/df (mpm_sim.py:173-180; the drop at
// phase == c is added on the host, see add_waveform_drop_terms).
template <class R>
__device__ __forceinline__ void pressure_factors(const JfParams& P, R tf, double* fac) {
  const double f = P.freq, c = P.contraction, t = tf;
  const R act = activation((R)P.freq, (R)P.contraction, tf);
  const double period = 1.0 / f;
  const double phase = (t - period * floor(t / period)) / period;
  double da_dc = 0.0, da_df = 0.0;
  if (act != R(0) && phase < c) {
    const double sn = 0.5 * sin(3.14159265 * phase / c);
    da_dc = sn * 3.14159265 * (-phase / (c * c));
    da_df = sn * (3.14159265 / c) * t;
  }
  fac[0] = act;
  fac[1] = P.actuation * da_dc;
  fac[2] = P.actuation * da_df;
}

template <class R>
__global__ void ad_grid(AdjArgs<R> A) {
  const GradArgs<R>& a = A.f;
  const int m = blockIdx.y;
  if (blockIdx.x == 0 && threadIdx.x == 0) pressure_factors(a.params[m], a.t, A.fac + 3 * m);
  const auto I = a.inst[m];
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= I.nx * I.ny) return;
  const int64_t node = I.g_off + n;
  const V4<R> q = a.pmv[node];
  const R px = q.x, py = q.y, pm = q.z;
  const V2<R> ub = A.ubar[node];
  if (!(pm > R(0))) {
    A.pmbar[node] = mk4(ub.x, ub.y, R(0), R(0));
    return;
  }
  const int i = n % I.nx, j = n / I.nx;
  R damp = R(1);
  if (i < I.dcx) damp = damp * (R(0.95) + R(0.05) * (R)i / (R)I.dcx);
  if (i > I.nx - I.dcx) damp = damp * (R(0.95) + R(0.05) * (R)(I.nx - i) / (R)I.dcx);
  if (j < I.dcy) damp = damp * (R(0.95) + R(0.05) * (R)j / (R)I.dcy);
  if (j > I.ny - I.dcy) damp = damp * (R(0.95) + R(0.05) * (R)(I.ny - j) / (R)I.dcy);
  const R g0 = (px / pm) * damp, g1 = (py / pm) * damp;
  const bool z0 = (i < 3 && g0 < R(0)) || (i > I.nx - 3 && g0 > R(0));
  const bool z1 = (j < 3 && g1 < R(0)) || (j > I.ny - 3 && g1 > R(0));
  const R a0 = z0 ? R(0) : damp * ub.x / pm;
  const R a1 = z1 ? R(0) : damp * ub.y / pm;
  A.pmbar[node] = mk4(a0, a1, -(a0 * px + a1 * py) / pm, R(0));
}

// The P2G adjoint of one live particle g of instance m.  kWater: only water
// particles whose singular values are both above the 1e-6 floor are done here
// (closed-form Jacobian: J = det F*, dJ = cof F*, F_out = sqrt(J) I,
// tau = lambda J (J - 1) I; mpm_sim.py:219-227 with mu = 0), and false is
// returned for every other particle in range (it goes to the second kernel);
// otherwise the material map is differentiated with dual numbers.  Returns
// true when the particle is done; *pbar = d L / d pressure of the particle.
template <class R, bool kWater>
__device__ __forceinline__ bool ad_p2g_particle(const AdjArgs<R>& A, const typename GT<R>::Inst& I, int m,
                                                int64_t g, int mt, R pressure, R* pbar) {
  const GradArgs<R>& a = A.f;
  *pbar = R(0);
  const V4<R> xv = a.s.xv[g];
  const V2<R> x = mk2(xv.x, xv.y), v = mk2(xv.z, xv.w);
  typename GT<R>::Stencil st;
  const V2<R> xt = A.xtmp[g];
  if (!jf_stencil_strict(I, x, st)) {
    A.lxv[g] = mk4(xt.x, xt.y, A.vtmp[g].x, A.vtmp[g].y);
    return true;  // C and F pass through unchanged outside the stencil range
  }
  if (kWater && mt != 0) return false;
  const V4<R> C = a.s.C[g], F = a.s.F[g];
  const R dt = I.dt;
  const R M00 = radd(R(1), rmul(dt, C.x)), M01 = rmul(dt, C.y);
  const R M10 = rmul(dt, C.z), M11 = radd(R(1), rmul(dt, C.w));
  const R fsv[4] = {rdot2(M00, F.x, M01, F.z), rdot2(M00, F.y, M01, F.w),
                    rdot2(M10, F.x, M11, F.z), rdot2(M10, F.y, M11, F.w)};
  const int ms = jf_mat_slot(mt);
  const auto& mats = a.mats;
  const R la = ms == 0 ? mats.la[0] : ms == 1 ? mats.la[1] : ms == 2 ? mats.la[2]
             : ms == 3 ? mats.la[3] : mats.la[4];
  const float2 fb = (mt == 3) ? a.fiber[g] : make_float2(0.0f, 1.0f);
  // the material map F* -> (F_out, tau): values and Jacobians d./dF*[e]
  R tv[4];                    // tau values
  D4T<R> Fo[4], tau[4], J;    // full path: values and Jacobians
  R dJ[4], kf = R(0), kt = R(0);  // water path: J = det F*, dJ = cof F*
  if constexpr (kWater) {
    // water, no singular value at the 1e-6 floor: J = s1 s2 = det F*, so
    // dJ = cof F*, dF_out = dJ / (2 sqrt J) I, dtau = lambda (2 J - 1) dJ I;
    // values as the forward rounds them
    const auto rot = jf_svd2_values(mk4(fsv[0], fsv[1], fsv[2], fsv[3]));
    if (!(rot.s1 > R(1e-6) && rot.s2 > R(1e-6))) return false;
    const R Jw = rmul(rot.s1, rot.s2);
    dJ[0] = fsv[3]; dJ[1] = -fsv[2]; dJ[2] = -fsv[1]; dJ[3] = fsv[0];
    kf = R(0.5) / sqrt(Jw);
    kt = la * (R(2) * Jw - R(1));
    const R diag = rmul(rmul(la, Jw), rsub(Jw, R(1)));
    tv[0] = diag; tv[1] = R(0); tv[2] = R(0); tv[3] = diag;
  } else {
    const R mu = ms == 0 ? mats.mu[0] : ms == 1 ? mats.mu[1] : ms == 2 ? mats.mu[2]
               : ms == 3 ? mats.mu[3] : mats.mu[4];
    D4T<R> Fs[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      Fs[q] = d4c(fsv[q]);
      Fs[q].d[q] = R(1);
    }
    jf_phi<D4T<R>>(Fs, mt, mu, la, pressure, fb, Fo, tau, J);
#pragma unroll
    for (int q = 0; q < 4; ++q) tv[q] = tau[q].v;
  }
  R mass = I.p_mass;
  if (mt == 2) mass = mass * (R)a.params[m].payload_density;
  const R ks = I.stress_scale;
  const R Af00 = ks * tv[0] + mass * C.x, Af01 = ks * tv[1] + mass * C.y;
  const R Af10 = ks * tv[2] + mass * C.z, Af11 = ks * tv[3] + mass * C.w;
  const R wx[3] = {st.wx0, st.wx1, st.wx2};
  const R wy[3] = {st.wy0, st.wy1, st.wy2};
  const V4<R>* pmb = A.pmbar + I.g_off;
  R vb0 = R(0), vb1 = R(0), Ab00 = R(0), Ab01 = R(0), Ab10 = R(0), Ab11 = R(0);
  R xb0 = R(0), xb1 = R(0), xa0 = R(0), xa1 = R(0);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const V4<R> pb = pmb[(st.by + j) * I.nx + st.bx + i];
      const R w = wx[i] * wy[j];
      const R d0 = ((R)i - st.fx0) * I.dx, d1 = ((R)j - st.fx1) * I.dx;
      vb0 += w * pb.x;
      vb1 += w * pb.y;
      Ab00 += w * pb.x * d0; Ab01 += w * pb.x * d1;
      Ab10 += w * pb.y * d0; Ab11 += w * pb.y * d1;
      const R mom0 = mass * v.x + (Af00 * d0 + Af01 * d1);
      const R mom1 = mass * v.y + (Af10 * d0 + Af11 * d1);
      const R qv = pb.x * mom0 + pb.y * mom1 + pb.z * mass;
      xb0 += wd(i, st.fx0) * wy[j] * qv;
      xb1 += wx[i] * wd(j, st.fx1) * qv;
      xa0 += w * (Af00 * pb.x + Af10 * pb.y);
      xa1 += w * (Af01 * pb.x + Af11 * pb.y);
    }
  }
  const R tb[4] = {ks * Ab00, ks * Ab01, ks * Ab10, ks * Ab11};
  const V4<R> Fob = A.lF[g];
  const R fob[4] = {Fob.x, Fob.y, Fob.z, Fob.w};
  R Fsb[4];
  if constexpr (kWater) {
    const R cw = (fob[0] + fob[3]) * kf + (tb[0] + tb[3]) * kt;
#pragma unroll
    for (int e = 0; e < 4; ++e) Fsb[e] = cw * dJ[e];
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      R acc = R(0);
#pragma unroll
      for (int q = 0; q < 4; ++q) acc += fob[q] * Fo[q].d[e] + tb[q] * tau[q].d[e];
      Fsb[e] = acc;
    }
    if (mt == 3) {
      const R fx = fb.x, fy = fb.y;
      *pbar = (tb[0] * fx * fx + tb[1] * fx * fy + tb[2] * fy * fx + tb[3] * fy * fy) * J.v;
    }
  }
  // F* = M F: F_bar = M^T F*_bar, C_bar += dt F*_bar F^T
  const R Fb00 = M00 * Fsb[0] + M10 * Fsb[2], Fb01 = M00 * Fsb[1] + M10 * Fsb[3];
  const R Fb10 = M01 * Fsb[0] + M11 * Fsb[2], Fb11 = M01 * Fsb[1] + M11 * Fsb[3];
  const R Cb00 = mass * Ab00 + dt * (Fsb[0] * F.x + Fsb[1] * F.y);
  const R Cb01 = mass * Ab01 + dt * (Fsb[0] * F.z + Fsb[1] * F.w);
  const R Cb10 = mass * Ab10 + dt * (Fsb[2] * F.x + Fsb[3] * F.y);
  const R Cb11 = mass * Ab11 + dt * (Fsb[2] * F.z + Fsb[3] * F.w);
  const V4<R> lx = mk4(xt.x + I.inv_dx * xb0 - xa0, xt.y + I.inv_dx * xb1 - xa1, mass * vb0, mass * vb1);
  A.lxv[g] = lx;
  A.lC[g] = mk4(Cb00, Cb01, Cb10, Cb11);
  A.lF[g] = mk4(Fb00, Fb01, Fb10, Fb11);
  const R chk = ((lx.x + lx.y) + (lx.z + lx.w)) + ((Cb00 + Cb01) + (Cb10 + Cb11)) +
                ((Fb00 + Fb01) + (Fb10 + Fb11));
  if (!isfinite(chk)) atomicOr(a.err + m, 4);
  return true;
}

// P2G adjoint of the water particles (most of the tank): the closed-form
// Jacobian at the register budget of that path; water at the singular-value
// floor is listed for ad_p2g_list (the full path), and every other material is
// done by ad_p2g_list over the rollout's list of non-water particles, which
// runs beside this kernel on a second stream.
template <class R>
__global__ void __launch_bounds__(kT, sizeof(R) == 4 ? 4 : 1) ad_p2g_water(AdjArgs<R> A, int32_t* floor_list, int32_t* n_floor) {
  const GradArgs<R>& a = A.f;
  const int m = blockIdx.y;
  const auto I = a.inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  if (a.mat[g] != 0) return;
  R pbar;
  if (!ad_p2g_particle<R, true>(A, I, m, g, 0, R(0), &pbar)) floor_list[atomicAdd(n_floor, 1)] = (int32_t)g;
}

// P2G adjoint with the full material map (dual-number SVD) over a list of
// particles; the muscle's d L / d pressure goes into the parameter gradients
// of its instance.
template <class R>
__global__ void __launch_bounds__(kT) ad_p2g_list(AdjArgs<R> A, const int32_t* list, const int32_t* n_list,
                                                  const int32_t* inst_of) {
  const GradArgs<R>& a = A.f;
  const int n = *n_list;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int64_t g = list[r];
    const int m = inst_of[g];
    const auto I = a.inst[m];
    const double* fm = A.fac + 3 * m;
    const R pressure = (R)a.params[m].actuation * (R)fm[0];
    R pbar = R(0);
    ad_p2g_particle<R, false>(A, I, m, g, a.mat[g], pressure, &pbar);
    if (pbar != R(0)) {
      atomicAdd(A.gparam + 3 * m + 0, (double)pbar * fm[0]);
      atomicAdd(A.gparam + 3 * m + 1, (double)pbar * fm[1]);
      atomicAdd(A.gparam + 3 * m + 2, (double)pbar * fm[2]);
      atomicAdd(A.dLdp + m, (double)pbar);
    }
  }
}

// the live particles that are not water (the list ad_p2g_list takes beside
// the water kernel)
__global__ void nonwater_list_kernel(const JfInst* __restrict__ inst, const int32_t* __restrict__ mat,
                                     int32_t* __restrict__ list, int32_t* __restrict__ n) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  if (mat[g] > 0) list[atomicAdd(n, 1)] = (int32_t)g;
}

// d L / d x at the final state: +1/n on the y of the selected particles
// (payload, or jelly + muscle without payload); sign = -1 subtracts the
// initial-CoM term at the end of the backward pass.
template <class R>
__global__ void seed_kernel(const JfInst* __restrict__ inst, const int32_t* __restrict__ mat,
                            const int32_t* __restrict__ body_mode, const double* __restrict__ inv_n,
                            V4<R>* lxv, V4<R>* lC, V4<R>* lF, int init, R sign) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const int mt = mat[g];
  const bool sel = body_mode[m] ? (mt == 1 || mt == 3) : (mt == 2);
  const R s = sel ? sign * (R)inv_n[m] : R(0);
  if (init) {
    lxv[g] = mk4(R(0), s, R(0), R(0));
    lC[g] = mk4(R(0), R(0), R(0), R(0));
    lF[g] = mk4(R(0), R(0), R(0), R(0));
  } else if (sel) {
    lxv[g].y += s;
  }
}

// instance index of every particle slot
__global__ void inst_of_kernel(const JfInst* __restrict__ inst, int32_t* __restrict__ out) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < I.n_slots) out[I.p_off + k] = m;
}

// FP64 build: the engine's FP32 state (x, v, C, F, Jp) into the double
// working state and back (rounded to FP32)
__global__ void widen_kernel(const JfInst* __restrict__ inst, JfParticles p, double4* xv, double4* C, double4* F,
                             double* Jp) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const float4 a = p.xv[g], b = p.C[g], c = p.F[g];
  xv[g] = make_double4(a.x, a.y, a.z, a.w);
  C[g] = make_double4(b.x, b.y, b.z, b.w);
  F[g] = make_double4(c.x, c.y, c.z, c.w);
  Jp[g] = p.Jp[g];
}
__global__ void narrow_kernel(const JfInst* __restrict__ inst, JfParticles p, const double4* xv, const double4* C,
                              const double4* F, const double* Jp) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const double4 a = xv[g], b = C[g], c = F[g];
  p.xv[g] = make_float4((float)a.x, (float)a.y, (float)a.z, (float)a.w);
  p.C[g] = make_float4((float)b.x, (float)b.y, (float)b.z, (float)b.w);
  p.F[g] = make_float4((float)c.x, (float)c.y, (float)c.z, (float)c.w);
  p.Jp[g] = (float)Jp[g];
}

// The loss sums of the FP64 build from its own final state (the FP32 slots
// hold it rounded): per instance payload [sum_y, count, sum_x] and body
// (jelly + muscle) [sum_y, count, sum_x], as stats_kernel sums the FP32 slots.
__global__ void stats64_kernel(const JfInst* __restrict__ inst, const double4* __restrict__ xv,
                               const int32_t* __restrict__ mat, double* __restrict__ out) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  double py = 0, pc = 0, px = 0, by = 0, bc = 0, bx = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < I.n_slots; k += gridDim.x * blockDim.x) {
    const int64_t g = I.p_off + k;
    const int mt = mat[g];
    if (mt == 2) {
      const double4 a = xv[g];
      py += a.y; pc += 1.0; px += a.x;
    } else if (mt == 1 || mt == 3) {
      const double4 a = xv[g];
      by += a.y; bc += 1.0; bx += a.x;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    py += __shfl_down_sync(0xffffffffu, py, off);
    pc += __shfl_down_sync(0xffffffffu, pc, off);
    px += __shfl_down_sync(0xffffffffu, px, off);
    by += __shfl_down_sync(0xffffffffu, by, off);
    bc += __shfl_down_sync(0xffffffffu, bc, off);
    bx += __shfl_down_sync(0xffffffffu, bx, off);
  }
  if ((threadIdx.x & 31) == 0 && (pc > 0 || bc > 0)) {
    double* o = out + 6 * m;
    atomicAdd(o + 0, py); atomicAdd(o + 1, pc); atomicAdd(o + 2, px);
    atomicAdd(o + 3, by); atomicAdd(o + 4, bc); atomicAdd(o + 5, bx);
  }
}

template <class T>
cudaError_t alloc_n(T** p, size_t n) {
  return cudaMalloc((void**)p, sizeof(T) * (n > 0 ? n : 1));
}

// A CUDA graph of a rollout's device work, replayed while its key (sizes,
// start time, buffer addresses) is unchanged.
struct GradGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> key;
  int64_t launches = 0;  // kernels one replay launches
};

// Device buffers of the differentiable rollout in one precision.
template <class R>
struct GradBuffers {
  int64_t steps = 0;
  int32_t K = 0;
  R t0 = R(0);
  size_t n_ck = 0, seg_cap = 0;
  typename GT<R>::Inst* inst = nullptr;  // the instances' constants in this precision
  typename GT<R>::Acc* fix = nullptr;
  V2<R>* u = nullptr;
  V2<R>* ubar = nullptr;
  V4<R>* pmbar = nullptr;
  V4<R> *lxv = nullptr, *lC = nullptr, *lF = nullptr;
  V2<R> *xtmp = nullptr, *vtmp = nullptr;
  V4<R>* ck = nullptr;     // n_ck checkpoints x 3 arrays x total slots
  // FP64: the working state (x, v, C, F) and Jp; FP32 works on the engine's
  V4<R>* work = nullptr;   // 3 arrays x total slots
  R* wJp = nullptr;
  // two sets of segment buffers: the backward recomputes segment k - 1 into
  // one while the adjoint of segment k reads the other
  V4<R>* seg[2] = {nullptr, nullptr};    // K states x 3 arrays x total slots
  V2<R>* useg[2] = {nullptr, nullptr};   // K grids: updated velocity per node
  V4<R>* pmseg[2] = {nullptr, nullptr};  // K grids: (momentum x, momentum y, mass) per node
  cudaStream_t rstream = nullptr;        // the recompute's stream
  cudaEvent_t ready[2] = {nullptr, nullptr}, released[2] = {nullptr, nullptr};
  V4<R>* fin = nullptr;    // final state (3 arrays)
  R* fin_Jp = nullptr;     // final Jp (the backward's recompute updates Jp in place)
  double* gparam = nullptr;
  double* dLdp = nullptr;  // steps x M: d L / d pressure per substep and instance
  size_t dLdp_cap = 0;
  double* fac = nullptr;       // M x 3 pressure factors of the current substep
  int32_t* solid = nullptr;    // the rollout's non-water live particles
  int32_t* floor_list = nullptr;  // water at the singular-value floor, per substep
  int32_t* counts = nullptr;   // [non-water, floor]
  int32_t* inst_of = nullptr;  // instance of every particle slot
  cudaStream_t side = nullptr; // second stream of the backward (the non-water P2G adjoint)
  cudaEvent_t fork = nullptr, join = nullptr;
  int32_t* body_mode = nullptr;
  double* inv_n = nullptr;
  bool have_forward = false;   // the latest rollout's forward completed
  bool have_backward = false;  // and its backward (the adjoint in lxv, lC, lF)
  int n_sm = 148;
  GradGraph fwd_graph, bwd_graph, step_graph;  // forward, backward, forward + backward

  void release() {
    cudaFree(fix); cudaFree(u); cudaFree(ubar); cudaFree(pmbar); cudaFree(inst);
    cudaFree(lxv); cudaFree(lC); cudaFree(lF); cudaFree(xtmp); cudaFree(vtmp);
    cudaFree(ck); cudaFree(work); cudaFree(wJp); cudaFree(fin); cudaFree(fin_Jp); cudaFree(gparam);
    for (int b = 0; b < 2; ++b) {
      cudaFree(seg[b]); cudaFree(useg[b]); cudaFree(pmseg[b]);
      if (ready[b]) cudaEventDestroy(ready[b]);
      if (released[b]) cudaEventDestroy(released[b]);
    }
    if (rstream) cudaStreamDestroy(rstream);
    for (GradGraph* gg : {&fwd_graph, &bwd_graph, &step_graph})
      if (gg->exec) cudaGraphExecDestroy(gg->exec);
    cudaFree(dLdp); cudaFree(fac); cudaFree(solid); cudaFree(floor_list); cudaFree(counts);
    cudaFree(inst_of);
    if (side) cudaStreamDestroy(side);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    cudaFree(body_mode); cudaFree(inv_n);
  }
};

}  // namespace

// The differentiable rollout's buffers of both precisions (an engine uses
// the one its JF_FLAG_GRAD_FP64 flag selects).
struct JfGrad {
  GradBuffers<float> f32;
  GradBuffers<double> f64;
};

void jf_grad_free(jf_engine* e) {
  JfGrad* G = e->grad;
  if (!G) return;
  G->f32.release();
  G->f64.release();
  delete G;
  e->grad = nullptr;
}

namespace {

template <class R> GradBuffers<R>& bufs(jf_engine* e);
template <> GradBuffers<float>& bufs<float>(jf_engine* e) { return e->grad->f32; }
template <> GradBuffers<double>& bufs<double>(jf_engine* e) { return e->grad->f64; }

// the instances' constants in this precision: the engine's table in FP32,
// the FP64 copy in FP64
template <class R> const typename GT<R>::Inst* inst_table(jf_engine* e);
template <> const JfInst* inst_table<float>(jf_engine* e) { return e->d_inst; }
template <> const JfInst64* inst_table<double>(jf_engine* e) { return bufs<double>(e).inst; }

// the FP64 materials (mpm_sim.py:25-48, the Python doubles themselves)
JfMaterials64 materials64() {
  const double E_base = 0.1e4, nu_base = 0.2, E_jelly = 0.7e3, nu_jelly = 0.3;
  const double E_pay = 2.0e5, nu_pay = 0.2, water_lambda = 100000.0;
  JfMaterials64 m;
  m.mu[0] = 0.0; m.la[0] = water_lambda;
  m.mu[1] = E_jelly / (2 * (1 + nu_jelly)); m.la[1] = E_jelly * nu_jelly / ((1 + nu_jelly) * (1 - 2 * nu_jelly));
  m.mu[2] = E_pay / (2 * (1 + nu_pay)); m.la[2] = E_pay * nu_pay / ((1 + nu_pay) * (1 - 2 * nu_pay));
  m.mu[3] = m.mu[1]; m.la[3] = m.la[1];
  m.mu[4] = E_base / (2 * (1 + nu_base)); m.la[4] = E_base * nu_base / ((1 + nu_base) * (1 - 2 * nu_base));
  return m;
}

// the instances' constants in FP64 (mpm_sim.py:18-58, as the oracle's FP64
// build folds them)
std::vector<JfInst64> insts64(const jf_engine* e) {
  std::vector<JfInst64> out;
  for (const JfInst& I : e->inst) {
    JfInst64 d = {};
    d.nx = I.nx; d.ny = I.ny; d.dcx = I.dcx; d.dcy = I.dcy;
    d.n_slots = I.n_slots; d.p_off = I.p_off; d.g_off = I.g_off;
    const double nx = I.nx, dx = 1.0 / nx, p_vol = (dx * 0.5) * (dx * 0.5);
    d.inv_dx = nx;
    d.dx = dx;
    d.dt = e->dt;
    d.p_mass = p_vol * 1;
    d.stress_scale = -e->dt * p_vol * 4 * nx * nx;
    d.c4 = 4 * nx;
    d.dtg = e->dt * 10.0;
    d.y_hi = I.domain_h - 0.001;
    out.push_back(d);
  }
  return out;
}

template <class R> typename GT<R>::Mats mats_of();
template <> JfMaterials mats_of<float>() { return jf_materials(); }
template <> JfMaterials64 mats_of<double>() { return materials64(); }

// the working state: the engine's particles in FP32, the double copy in FP64
template <class R> GradState<R> work_state(jf_engine* e);
template <> GradState<float> work_state<float>(jf_engine* e) { return GradState<float>{e->p.xv, e->p.C, e->p.F}; }
template <> GradState<double> work_state<double>(jf_engine* e) {
  GradBuffers<double>& G = bufs<double>(e);
  const size_t slots = (size_t)e->total_slots;
  return GradState<double>{G.work, G.work + slots, G.work + 2 * slots};
}
template <class R> R* work_Jp(jf_engine* e);
template <> float* work_Jp<float>(jf_engine* e) { return e->p.Jp; }
template <> double* work_Jp<double>(jf_engine* e) { return bufs<double>(e).wJp; }

template <class R>
GradArgs<R> grad_args(jf_engine* e, GradState<R> s, R t) {
  GradBuffers<R>& G = bufs<R>(e);
  GradArgs<R> a;
  a.inst = inst_table<R>(e);
  a.params = e->d_params;
  a.mats = mats_of<R>();
  a.s = s;
  a.o = s;
  a.mat = e->p.mat;
  a.Jp = work_Jp<R>(e);
  a.fiber = e->p.fiber;
  a.fix = G.fix;
  a.u = G.u;
  a.pmv = nullptr;
  a.err = e->d_err;
  a.t = t;
  return a;
}

template <class R>
GradState<R> state_at(V4<R>* base, size_t slots, size_t idx) {
  V4<R>* b = base + 3 * slots * idx;
  return GradState<R>{b, b + slots, b + 2 * slots};
}

template <class R>
cudaError_t copy_state(jf_engine* e, GradState<R> dst, GradState<R> src, cudaStream_t st = nullptr) {
  const size_t bytes = sizeof(V4<R>) * (size_t)e->total_slots;
  if (!st) st = e->stream;
  cudaError_t err;
  if ((err = cudaMemcpyAsync(dst.xv, src.xv, bytes, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return err;
  if ((err = cudaMemcpyAsync(dst.C, src.C, bytes, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return err;
  return cudaMemcpyAsync(dst.F, src.F, bytes, cudaMemcpyDeviceToDevice, st);
}

// one deterministic substep of every instance from state s at time t into
// state o (s itself when o is not given); with u_keep / pmv_keep set, its grid
// is written there for the adjoint
template <class R>
cudaError_t det_substep(jf_engine* e, GradState<R> s, R t, V2<R>* u_keep = nullptr, V4<R>* pmv_keep = nullptr,
                        const GradState<R>* o = nullptr, cudaStream_t st = nullptr) {
  if (!st) st = e->stream;
  GradBuffers<R>& G = bufs<R>(e);
  GradArgs<R> a = grad_args<R>(e, s, t);
  if (o) a.o = *o;
  if (u_keep) {
    a.u = u_keep;
    a.pmv = pmv_keep;
  }
  cudaError_t err = cudaMemsetAsync(G.fix, 0, sizeof(typename GT<R>::Acc) * 3 * (size_t)e->total_nodes, st);
  if (err != cudaSuccess) return err;
  const dim3 gp((e->max_slots + kT - 1) / kT, e->M), gn((e->max_cells + kT - 1) / kT, e->M);
  gf_p2g<R><<<gp, kT, 0, st>>>(a);
  gf_grid<R><<<gn, kT, 0, st>>>(a);
  gf_g2p<R><<<gp, kT, 0, st>>>(a);
  e->launches += 3;
  return cudaGetLastError();
}


// Every buffer of a rollout of `steps` substeps with a checkpoint every K
// (allocated before any graph capture: capture allows no allocation).
template <class R>
cudaError_t grad_alloc(jf_engine* e, int64_t steps, int32_t K) {
  if (!e->grad) e->grad = new JfGrad();
  GradBuffers<R>& G = bufs<R>(e);
  const size_t slots = (size_t)e->total_slots;
  const size_t n_ck = (size_t)((steps + K - 1) / K);
  cudaError_t err = cudaSuccess;
  if (!G.fix) {
    if ((err = alloc_n(&G.fix, 3 * (size_t)e->total_nodes)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.u, e->total_nodes)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.ubar, e->total_nodes)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.pmbar, e->total_nodes)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.lxv, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.lC, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.lF, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.xtmp, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.vtmp, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.fin, 3 * slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.fin_Jp, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.gparam, 3 * (size_t)e->M)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.body_mode, e->M)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.inv_n, e->M)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.fac, 3 * (size_t)e->M)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.solid, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.floor_list, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.counts, 2)) != cudaSuccess) return err;
    if ((err = alloc_n(&G.inst_of, slots)) != cudaSuccess) return err;
    if constexpr (std::is_same<R, double>::value) {
      if ((err = alloc_n(&G.work, 3 * slots)) != cudaSuccess) return err;
      if ((err = alloc_n(&G.wJp, slots)) != cudaSuccess) return err;
      if ((err = alloc_n(&G.inst, (size_t)e->M)) != cudaSuccess) return err;
      const std::vector<JfInst64> h = insts64(e);
      if ((err = cudaMemcpy(G.inst, h.data(), sizeof(JfInst64) * h.size(), cudaMemcpyHostToDevice))) return err;
    }
    if ((err = cudaStreamCreateWithFlags(&G.side, cudaStreamNonBlocking)) != cudaSuccess) return err;
    if ((err = cudaEventCreateWithFlags(&G.fork, cudaEventDisableTiming)) != cudaSuccess) return err;
    if ((err = cudaEventCreateWithFlags(&G.join, cudaEventDisableTiming)) != cudaSuccess) return err;
    if ((err = cudaStreamCreateWithFlags(&G.rstream, cudaStreamNonBlocking)) != cudaSuccess) return err;
    for (int b = 0; b < 2; ++b) {
      if ((err = cudaEventCreateWithFlags(&G.ready[b], cudaEventDisableTiming)) != cudaSuccess) return err;
      if ((err = cudaEventCreateWithFlags(&G.released[b], cudaEventDisableTiming)) != cudaSuccess) return err;
    }
    const dim3 gp((e->max_slots + kT - 1) / kT, e->M);
    inst_of_kernel<<<gp, kT, 0, e->stream>>>(e->d_inst, G.inst_of);
    e->launches += 1;
    cudaDeviceGetAttribute(&G.n_sm, cudaDevAttrMultiProcessorCount, e->device);
  }
  if (G.n_ck < n_ck) {
    cudaFree(G.ck);
    G.ck = nullptr;
    if ((err = alloc_n(&G.ck, 3 * slots * n_ck)) != cudaSuccess) return err;
    G.n_ck = n_ck;
  }
  if (G.dLdp_cap < (size_t)steps * e->M) {
    cudaFree(G.dLdp);
    G.dLdp = nullptr;
    G.dLdp_cap = 0;
    if ((err = alloc_n(&G.dLdp, (size_t)steps * e->M)) != cudaSuccess) return err;
    G.dLdp_cap = (size_t)steps * e->M;
  }
  return cudaSuccess;
}

// The backward's segment buffers (K pre-step states and grids, two sets),
// allocated only when a backward runs, so that a forward-only rollout with a
// long checkpoint interval does not hold them.
template <class R>
cudaError_t seg_alloc(jf_engine* e, int32_t K) {
  GradBuffers<R>& G = bufs<R>(e);
  const size_t slots = (size_t)e->total_slots;
  cudaError_t err = cudaSuccess;
  if (G.seg_cap < (size_t)K) {
    G.seg_cap = 0;
    for (int b = 0; b < 2; ++b) {
      cudaFree(G.seg[b]);
      cudaFree(G.useg[b]);
      cudaFree(G.pmseg[b]);
      G.seg[b] = nullptr;
      G.useg[b] = nullptr;
      G.pmseg[b] = nullptr;
      if ((err = alloc_n(&G.seg[b], 3 * slots * (size_t)K)) != cudaSuccess) return err;
      if ((err = alloc_n(&G.useg[b], (size_t)e->total_nodes * K)) != cudaSuccess) return err;
      if ((err = alloc_n(&G.pmseg[b], (size_t)e->total_nodes * K)) != cudaSuccess) return err;
    }
    G.seg_cap = (size_t)K;
  }
  return cudaSuccess;
}

// FP64: the engine's FP32 state into the working state, and back
template <class R>
cudaError_t widen(jf_engine* e) {
  if constexpr (std::is_same<R, double>::value) {
    GradBuffers<double>& G = bufs<double>(e);
    const GradState<double> w = work_state<double>(e);
    const dim3 gp((e->max_slots + kT - 1) / kT, e->M);
    widen_kernel<<<gp, kT, 0, e->stream>>>(e->d_inst, e->p, w.xv, w.C, w.F, G.wJp);
    e->launches += 1;
  }
  return cudaGetLastError();
}
template <class R>
cudaError_t narrow(jf_engine* e) {
  if constexpr (std::is_same<R, double>::value) {
    GradBuffers<double>& G = bufs<double>(e);
    const GradState<double> w = work_state<double>(e);
    const dim3 gp((e->max_slots + kT - 1) / kT, e->M);
    narrow_kernel<<<gp, kT, 0, e->stream>>>(e->d_inst, e->p, w.xv, w.C, w.F, G.wJp);
    e->launches += 1;
  }
  return cudaGetLastError();
}

// the times of the rollout's substeps: a running sum in the rollout's precision
// (mpm_sim.py:340; the oracle's FP64 build sums in double)
template <class R>
std::vector<R> substep_times(const jf_engine* e, R t0, int64_t steps) {
  const R dt = (R)e->dt;
  std::vector<R> ts((size_t)steps + 1);
  ts[0] = t0;
  for (int64_t s = 0; s < steps; ++s) ts[s + 1] = ts[s] + dt;
  return ts;
}

// The forward's device work: the non-water list, the substeps from G.t0 with
// their checkpoints, and copies of the final state (in FP64 also written back
// to the engine's particles).
template <class R>
cudaError_t fwd_record(jf_engine* e) {
  GradBuffers<R>& G = bufs<R>(e);
  const size_t slots = (size_t)e->total_slots;
  const int64_t steps = G.steps;
  const int32_t K = G.K;
  cudaError_t err;
  // the rollout's non-water particles, for the backward's second stream
  if ((err = cudaMemsetAsync(G.counts, 0, sizeof(int32_t), e->stream))) return err;
  {
    const dim3 gp((e->max_slots + kT - 1) / kT, e->M);
    nonwater_list_kernel<<<gp, kT, 0, e->stream>>>(e->d_inst, e->p.mat, G.solid, G.counts);
    e->launches += 1;
  }
  if ((err = widen<R>(e))) return err;
  const GradState<R> work = work_state<R>(e);
  const std::vector<R> ts = substep_times<R>(e, G.t0, steps);
  for (int64_t s = 0; s < steps; ++s) {
    if (s % K == 0) {
      if ((err = copy_state<R>(e, state_at<R>(G.ck, slots, s / K), work)) != cudaSuccess) return err;
    }
    {
      JfTimed timed(e, false);
      if ((err = det_substep<R>(e, work, ts[(size_t)s])) != cudaSuccess) return err;
    }
  }
  if ((err = copy_state<R>(e, state_at<R>(G.fin, slots, 0), work)) != cudaSuccess) return err;
  if ((err = cudaMemcpyAsync(G.fin_Jp, work_Jp<R>(e), sizeof(R) * slots, cudaMemcpyDeviceToDevice, e->stream)))
    return err;
  return narrow<R>(e);
}

// Phase of the waveform at time t as the rollout's precision computes it
// (mpm_sim.py:173-174); the volatile stores keep every operation rounded on
// its own, as the device code does.
float waveform_phase(float freq, float t) {
  volatile float period = 1.0f / (1.0f * freq);
  volatile float q = floorf(t / period);
  volatile float pq = period * q;
  volatile float r = t - pq;
  volatile float phase = r / period;
  return phase;
}
double waveform_phase(double freq, double t) {
  volatile double period = 1.0 / (1.0 * freq);
  volatile double q = floor(t / period);
  volatile double pq = period * q;
  volatile double r = t - pq;
  volatile double phase = r / period;
  return phase;
}

// Boundary terms of the waveform's drop from 1 to 0 at phase == contraction
// (mpm_sim.py:176-180): for every drop between substeps n - 1 and n of the
// rollout, at the instant t* where the phase, advancing by f per unit time,
// reaches c, d L / d c += A g* / (f dt) and d L / d f -= A g* t* / (f dt), with
// g* = d L / d pressure interpolated between the two substeps (the rollout's
// pressure at substep n is A a(phase(t_n)), and a(c-) = 1).
template <class R>
void add_waveform_drop_terms(const jf_engine* e, const std::vector<R>& ts, const std::vector<double>& dLdp,
                             double* gparam) {
  const int64_t steps = (int64_t)ts.size() - 1;
  for (int m = 0; m < e->M; ++m) {
    const JfParams& P = e->params[m];
    const double A = P.actuation, c = P.contraction, f = P.freq;
    const R cr = (R)P.contraction;
    if (!(f > 0.0) || !(c > 0.0) || A == 0.0) continue;
    R prev = waveform_phase((R)P.freq, ts[0]);
    for (int64_t n = 1; n < steps; ++n) {
      const R ph = waveform_phase((R)P.freq, ts[(size_t)n]);
      if (prev < cr && !(ph < cr) && ph >= prev) {
        const double theta = (c - (double)prev) / ((double)ph - (double)prev);
        const double tstar = (double)ts[(size_t)n - 1] + theta * ((double)ts[(size_t)n] - (double)ts[(size_t)n - 1]);
        const double g = (1.0 - theta) * dLdp[(size_t)(n - 1) * e->M + m] + theta * dLdp[(size_t)n * e->M + m];
        gparam[3 * m + 1] += A * g / (f * e->dt);
        gparam[3 * m + 2] -= A * g * tstar / (f * e->dt);
      }
      prev = ph;
    }
  }
}

// The backward's device work: seeds, the recompute of every segment (on its
// own stream, overlapped with the adjoint of the segment after it), the
// adjoint substeps in reverse, and the engine's state restored to the
// forward's final state.
template <class R>
cudaError_t bwd_record(jf_engine* e) {
  GradBuffers<R>& G = bufs<R>(e);
  const size_t slots = (size_t)e->total_slots;
  const int64_t steps = G.steps;
  const int32_t K = G.K;
  const std::vector<R> ts = substep_times<R>(e, G.t0, steps);
  const dim3 gp((e->max_slots + kT - 1) / kT, e->M), gn((e->max_cells + kT - 1) / kT, e->M);
  cudaError_t err = cudaMemsetAsync(G.gparam, 0, sizeof(double) * 3 * e->M, e->stream);
  if (err != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(G.dLdp, 0, sizeof(double) * (size_t)steps * e->M, e->stream))) return err;
  seed_kernel<R><<<gp, kT, 0, e->stream>>>(e->d_inst, e->p.mat, G.body_mode, G.inv_n, G.lxv, G.lC, G.lF, 1, R(1));
  e->launches += 1;
  const GradState<R> work = work_state<R>(e);
  const int64_t n_seg = (steps + K - 1) / K;
  const size_t nodes = (size_t)e->total_nodes;
  const int list_blocks = 2 * G.n_sm;  // grid-stride over the listed particles
  const int floor_blocks = 16;         // water at the singular-value floor: rare
  auto seg_len = [&](int64_t seg) { return (int)((steps - seg * K) < K ? (steps - seg * K) : K); };
  // Recompute of segment `seg` into buffer set b on the recompute stream: its
  // pre-step states (substep j reads state j and writes state j + 1; the last
  // writes the working state, which nothing reads) and every substep's grid.
  // It waits until the adjoint that last read buffer set b is done.  The
  // recompute needs only its checkpoint, so it runs while the main stream
  // runs the adjoint of the segment after it.
  auto recompute = [&](int64_t seg, int b) -> cudaError_t {
    cudaError_t r;
    if ((r = cudaStreamWaitEvent(G.rstream, G.released[b], 0))) return r;
    if ((r = copy_state<R>(e, state_at<R>(G.seg[b], slots, 0), state_at<R>(G.ck, slots, (size_t)seg),
                           G.rstream)))
      return r;
    const int n = seg_len(seg);
    for (int j = 0; j < n; ++j) {
      const GradState<R> next = (j + 1 < n) ? state_at<R>(G.seg[b], slots, (size_t)j + 1) : work;
      if ((r = det_substep<R>(e, state_at<R>(G.seg[b], slots, (size_t)j), ts[seg * K + j], G.useg[b] + nodes * j,
                              G.pmseg[b] + nodes * j, &next, G.rstream)))
        return r;
    }
    return cudaEventRecord(G.ready[b], G.rstream);
  };
  // the recompute stream starts after everything queued on the main stream
  // (the forward's state and the seeds above)
  if ((err = cudaEventRecord(G.released[0], e->stream))) return err;
  if ((err = cudaEventRecord(G.released[1], e->stream))) return err;
  if ((err = recompute(n_seg - 1, 0))) return err;
  for (int64_t seg = n_seg - 1; seg >= 0; --seg) {
    const int b = (int)((n_seg - 1 - seg) & 1);
    if (seg > 0 && (err = recompute(seg - 1, b ^ 1))) return err;
    if ((err = cudaStreamWaitEvent(e->stream, G.ready[b], 0))) return err;
    const int64_t s0 = seg * K;
    const int n = seg_len(seg);
    for (int j = n - 1; j >= 0; --j) {
      JfTimed timed(e, false);
      AdjArgs<R> A;
      A.f = grad_args<R>(e, state_at<R>(G.seg[b], slots, (size_t)j), ts[s0 + j]);
      A.lxv = G.lxv;
      A.lC = G.lC;
      A.lF = G.lF;
      A.ubar = G.ubar;
      A.pmbar = G.pmbar;
      A.xtmp = G.xtmp;
      A.vtmp = G.vtmp;
      A.gparam = G.gparam;
      A.dLdp = G.dLdp + (size_t)(s0 + j) * e->M;
      A.fac = G.fac;
      // the substep's grid as the recompute left it
      A.f.u = G.useg[b] + nodes * j;
      A.f.pmv = G.pmseg[b] + nodes * j;
      if ((err = cudaMemsetAsync(G.ubar, 0, sizeof(V2<R>) * nodes, e->stream))) return err;
      if ((err = cudaMemsetAsync(G.counts + 1, 0, sizeof(int32_t), e->stream))) return err;
      ad_g2p<R><<<gp, kT, 0, e->stream>>>(A);
      ad_grid<R><<<gn, kT, 0, e->stream>>>(A);
      // P2G adjoint: the non-water particles on the second stream, beside the water
      if ((err = cudaEventRecord(G.fork, e->stream))) return err;
      if ((err = cudaStreamWaitEvent(G.side, G.fork, 0))) return err;
      ad_p2g_list<R><<<list_blocks, kT, 0, G.side>>>(A, G.solid, G.counts, G.inst_of);
      if ((err = cudaEventRecord(G.join, G.side))) return err;
      ad_p2g_water<R><<<gp, kT, 0, e->stream>>>(A, G.floor_list, G.counts + 1);
      ad_p2g_list<R><<<floor_blocks, kT, 0, e->stream>>>(A, G.floor_list, G.counts + 1, G.inst_of);
      if ((err = cudaStreamWaitEvent(e->stream, G.join, 0))) return err;
      e->launches += 5;
      if ((err = cudaGetLastError()) != cudaSuccess) return err;
    }
    if ((err = cudaEventRecord(G.released[b], e->stream))) return err;
  }
  // the initial CoM term of the displacement
  seed_kernel<R><<<gp, kT, 0, e->stream>>>(e->d_inst, e->p.mat, G.body_mode, G.inv_n, G.lxv, G.lC, G.lF, 0, R(-1));
  e->launches += 1;
  // leave the engine at the forward's final state
  if ((err = copy_state<R>(e, work, state_at<R>(G.fin, slots, 0))) != cudaSuccess) return err;
  if ((err = cudaMemcpyAsync(work_Jp<R>(e), G.fin_Jp, sizeof(R) * slots, cudaMemcpyDeviceToDevice, e->stream)))
    return err;
  return narrow<R>(e);
}

// After the backward's device work: the parameter gradients and the
// per-substep d L / d pressure to the host, then the waveform-drop terms.
template <class R>
cudaError_t bwd_finish(jf_engine* e, double* gparam_host) {
  GradBuffers<R>& G = bufs<R>(e);
  const int64_t steps = G.steps;
  const std::vector<R> ts = substep_times<R>(e, G.t0, steps);
  cudaError_t err;
  if ((err = cudaMemcpyAsync(gparam_host, G.gparam, sizeof(double) * 3 * e->M, cudaMemcpyDeviceToHost, e->stream)))
    return err;
  std::vector<double> dLdp((size_t)steps * e->M);
  if ((err = cudaMemcpyAsync(dLdp.data(), G.dLdp, sizeof(double) * dLdp.size(), cudaMemcpyDeviceToHost,
                             e->stream)))
    return err;
  if ((err = cudaStreamSynchronize(e->stream))) return err;
  add_waveform_drop_terms<R>(e, ts, dLdp, gparam_host);
  return cudaSuccess;
}

// Runs `record` (device work on the engine's stream) directly, or, with
// graphs on and per-kernel timing off, from a CUDA graph captured on first
// use and replayed while `key` is unchanged.
template <class Record>
cudaError_t run_graph(jf_engine* e, GradGraph& gg, const std::vector<uint64_t>& key, Record record) {
  if (!e->use_graphs || e->timing) return record();
  if (!gg.exec || gg.key != key) {
    if (gg.exec) {
      cudaGraphExecDestroy(gg.exec);
      gg.exec = nullptr;
    }
    const int64_t launches = e->launches;
    cudaGraph_t graph = nullptr;
    cudaError_t err = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) return err;
    e->capturing = true;
    const cudaError_t rec = record();
    e->capturing = false;
    err = cudaStreamEndCapture(e->stream, &graph);
    gg.launches = e->launches - launches;
    e->launches = launches;  // nothing ran yet
    if (rec != cudaSuccess || err != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return rec != cudaSuccess ? rec : err;
    }
    err = cudaGraphInstantiate(&gg.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) return err;
    gg.key = key;
  }
  e->launches += gg.launches;
  return cudaGraphLaunch(gg.exec, e->stream);
}

// What a captured graph depends on.  The forward (tag 1) does not touch the
// segment buffers, which the first backward allocates: they stay out of its
// key, so that a forward captured before any backward is still replayed.
template <class R>
std::vector<uint64_t> graph_key(jf_engine* e, int tag) {
  const GradBuffers<R>& G = bufs<R>(e);
  uint64_t tbits = 0;
  memcpy(&tbits, &G.t0, sizeof(R));
  const bool segs = tag != 1;
  return {(uint64_t)tag, (uint64_t)sizeof(R), (uint64_t)G.steps, (uint64_t)G.K, tbits,
          (uint64_t)(uintptr_t)e->p.xv, (uint64_t)(uintptr_t)e->p.C, (uint64_t)(uintptr_t)e->p.F,
          (uint64_t)(uintptr_t)e->p.Jp, (uint64_t)(uintptr_t)e->p.mat, (uint64_t)(uintptr_t)G.ck,
          segs ? (uint64_t)(uintptr_t)G.seg[0] : 0, segs ? (uint64_t)(uintptr_t)G.seg[1] : 0,
          segs ? (uint64_t)(uintptr_t)G.useg[0] : 0, segs ? (uint64_t)(uintptr_t)G.useg[1] : 0,
          segs ? (uint64_t)(uintptr_t)G.pmseg[0] : 0, segs ? (uint64_t)(uintptr_t)G.pmseg[1] : 0,
          (uint64_t)(uintptr_t)G.dLdp, (uint64_t)(uintptr_t)e->d_stats};
}

template <class R>
cudaError_t grad_begin(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode, const double* inv_n) {
  if (e->grad) bufs<R>(e).have_forward = bufs<R>(e).have_backward = false;  // a new rollout
  cudaError_t err = grad_alloc<R>(e, steps, K);
  if (err != cudaSuccess) return err;
  GradBuffers<R>& G = bufs<R>(e);
  if ((err = cudaMemcpyAsync(G.body_mode, body_mode, sizeof(int32_t) * e->M, cudaMemcpyHostToDevice, e->stream)))
    return err;
  if ((err = cudaMemcpyAsync(G.inv_n, inv_n, sizeof(double) * e->M, cudaMemcpyHostToDevice, e->stream)))
    return err;
  G.steps = steps;
  G.K = K;
  G.t0 = (R)e->t;
  return cudaSuccess;
}

// the engine's FP32 time after the rollout (its own running sum)
void grad_advance_time(jf_engine* e, int64_t steps) {
  const float dtf = (float)e->dt;
  float t = e->t;
  for (int64_t s = 0; s < steps; ++s) t = t + dtf;
  e->t = t;
}

template <class R>
cudaError_t forward_impl(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode, const double* inv_n) {
  cudaError_t err = grad_begin<R>(e, steps, K, body_mode, inv_n);
  if (err != cudaSuccess) return err;
  if ((err = run_graph(e, bufs<R>(e).fwd_graph, graph_key<R>(e, 1), [&] { return fwd_record<R>(e); }))) return err;
  grad_advance_time(e, steps);
  bufs<R>(e).have_forward = true;
  return cudaSuccess;
}

template <class R>
cudaError_t backward_impl(jf_engine* e, double* gparam_host) {
  cudaError_t err = seg_alloc<R>(e, bufs<R>(e).K);
  if (err != cudaSuccess) return err;
  err = run_graph(e, bufs<R>(e).bwd_graph, graph_key<R>(e, 2), [&] { return bwd_record<R>(e); });
  if (err != cudaSuccess) return err;
  if ((err = bwd_finish<R>(e, gparam_host)) == cudaSuccess) bufs<R>(e).have_backward = true;
  return err;
}

// The loss sums into e->d_stats after a rollout: the engine's stats over its
// FP32 slots, or, in the FP64 build, over the FP64 final state.
template <class R>
cudaError_t loss_stats(jf_engine* e) {
  if constexpr (std::is_same<R, double>::value) {
    GradBuffers<double>& G = bufs<double>(e);
    cudaError_t err = cudaMemsetAsync(e->d_stats, 0, sizeof(double) * 6 * e->M, e->stream);
    if (err != cudaSuccess) return err;
    const int blocks = std::max(1, std::min(64, (int)((e->max_slots + kT - 1) / kT)));
    stats64_kernel<<<dim3(blocks, e->M), kT, 0, e->stream>>>(e->d_inst, state_at<double>(G.fin, e->total_slots, 0).xv,
                                                             e->p.mat, e->d_stats);
    e->launches += 1;
    return cudaGetLastError();
  } else {
    return jf_stats_launch(e);
  }
}

template <class R>
cudaError_t step_impl(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode, const double* inv_n,
                      double* gparam_host) {
  cudaError_t err = grad_begin<R>(e, steps, K, body_mode, inv_n);
  if (err != cudaSuccess) return err;
  if ((err = seg_alloc<R>(e, K)) != cudaSuccess) return err;
  err = run_graph(e, bufs<R>(e).step_graph, graph_key<R>(e, 3), [&] {
    cudaError_t r = fwd_record<R>(e);
    if (r == cudaSuccess) r = loss_stats<R>(e);
    if (r == cudaSuccess) r = bwd_record<R>(e);
    return r;
  });
  if (err != cudaSuccess) return err;
  grad_advance_time(e, steps);
  bufs<R>(e).have_forward = true;
  if ((err = bwd_finish<R>(e, gparam_host)) == cudaSuccess) bufs<R>(e).have_backward = true;
  return err;
}

template <class R>
cudaError_t x0_impl(jf_engine* e, int m, std::vector<float4>& out) {
  const JfInst& I = e->inst[m];
  out.resize((size_t)I.n_slots);
  if (I.n_slots == 0) return cudaSuccess;
  std::vector<V4<R>> tmp((size_t)I.n_slots);
  cudaError_t err = cudaMemcpyAsync(tmp.data(), bufs<R>(e).lxv + I.p_off, sizeof(V4<R>) * I.n_slots,
                                    cudaMemcpyDeviceToHost, e->stream);
  if (err != cudaSuccess) return err;
  if ((err = cudaStreamSynchronize(e->stream))) return err;
  for (size_t k = 0; k < tmp.size(); ++k)
    out[k] = make_float4((float)tmp[k].x, (float)tmp[k].y, (float)tmp[k].z, (float)tmp[k].w);
  return cudaSuccess;
}

bool fp64(const jf_engine* e) { return (e->flags & JF_FLAG_GRAD_FP64) != 0; }

}  // namespace

cudaError_t jf_grad_forward_impl(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode,
                                 const double* inv_n) {
  return fp64(e) ? forward_impl<double>(e, steps, K, body_mode, inv_n)
                 : forward_impl<float>(e, steps, K, body_mode, inv_n);
}

cudaError_t jf_grad_loss_stats(jf_engine* e) {
  return fp64(e) ? loss_stats<double>(e) : loss_stats<float>(e);
}

cudaError_t jf_grad_backward_impl(jf_engine* e, double* gparam_host) {
  return fp64(e) ? backward_impl<double>(e, gparam_host) : backward_impl<float>(e, gparam_host);
}

// Forward and backward of one rollout as one graph; the final state's CoM
// sums are left in e->d_stats for the loss.
cudaError_t jf_grad_step_impl(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode,
                              const double* inv_n, double* gparam_host) {
  return fp64(e) ? step_impl<double>(e, steps, K, body_mode, inv_n, gparam_host)
                 : step_impl<float>(e, steps, K, body_mode, inv_n, gparam_host);
}

// Position adjoint of the initial state for one instance, in engine order.
cudaError_t jf_grad_x0_impl(jf_engine* e, int m, std::vector<float4>& out) {
  return fp64(e) ? x0_impl<double>(e, m, out) : x0_impl<float>(e, m, out);
}

// Whether the engine's latest rollout completed its forward (stage 1) or its
// backward too (stage 2), in the engine's gradient precision.
bool jf_grad_done(const jf_engine* e, int stage) {
  if (!e->grad) return false;
  const bool f = fp64(e) ? e->grad->f64.have_forward : e->grad->f32.have_forward;
  const bool b = fp64(e) ? e->grad->f64.have_backward : e->grad->f32.have_backward;
  return stage >= 2 ? (f && b) : f;
}
