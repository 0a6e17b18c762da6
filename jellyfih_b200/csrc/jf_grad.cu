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
// dL/dc += A g* / (f dt) and dL/df -= A g* t* / (f^2 dt) (t* the instant of
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
#include <cstring>
#include <vector>

#include "jf_dual.cuh"
#include "jf_engine.h"

namespace {

constexpr int kT = 256;
constexpr float kFix = 17592186044416.0f;        // 2^44
constexpr double kFixInv = 1.0 / 17592186044416.0;

struct GradState {
  float4* xv;
  float4* C;
  float4* F;
};

struct GradArgs {
  const JfInst* inst;
  const JfParams* params;
  JfMaterials mats;
  GradState s;                 // the state the kernel reads (pre-step)
  GradState o;                 // where it writes the post-step state (s itself in the forward)
  const int32_t* mat;
  float* Jp;
  const float2* fiber;
  unsigned long long* fix;     // 3 per node: momentum x, momentum y, mass (fixed point)
  float2* u;                   // updated grid velocity
  float4* pmv;                 // if set: (momentum x, momentum y, mass) per node, kept for the adjoint
  int32_t* err;                // per-instance non-finite flags
  float t;
};

// Largest contribution the fixed-point sums take: |v| < 64 keeps v * 2^44
// below 2^50, so 8,192 contributions to one node cannot overflow 2^63.
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

__device__ __forceinline__ void add_fixed(unsigned long long* p, float v, int32_t* flag) {
  const unsigned long long q = to_fixed(v, flag);
  if (q) atomicAdd(p, q);
}
__device__ __forceinline__ float from_fixed(unsigned long long v) {
  return (float)((double)(long long)v * kFixInv);
}

// per-block activation pressure of instance blockIdx.y at time a.t
__device__ __forceinline__ float block_pressure(const GradArgs& a, int m) {
  __shared__ float s_p;
  if (threadIdx.x == 0) {
    const JfParams P = a.params[m];
    s_p = P.actuation * jf_activation(P.freq, P.contraction, a.t);
  }
  __syncthreads();
  return s_p;
}

// Deterministic P2G.  A block's particles (consecutive slots of one
// instance) first add their fixed-point contributions into a shared-memory
// tile covering the block's stencil bounding box, when that box has at most
// kTileNodes nodes, and the tile then goes to the grid with one atomic per
// touched node and component; otherwise each contribution goes to the grid
// directly.  The contributions are integers, so every grouping gives the same
// sums bit for bit.
constexpr int kTileNodes = 1024;

__global__ void __launch_bounds__(kT) gf_p2g(GradArgs a) {
  __shared__ unsigned long long s_acc[3 * kTileNodes];
  __shared__ int s_box[4];  // stencil bases: min x, min y, max x, max y
  const int m = blockIdx.y;
  const float pressure = block_pressure(a, m);
  const JfInst I = a.inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t g = I.p_off + k;
  const bool copy = a.o.F != a.s.F;
  bool valid = false;
  JfStencil st;
  JfScatter sc;
  if (k < I.n_slots) {
    const int mt = a.mat[g];
    const float4 xv = mt >= 0 ? a.s.xv[g] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (mt >= 0 && jf_stencil_strict(I, make_float2(xv.x, xv.y), st)) {
      float4 F = a.s.F[g];
      float jp = (mt == 2) ? a.Jp[g] : 1.0f;
      const float2 fb = (mt == 3) ? a.fiber[g] : make_float2(0.0f, 1.0f);
      jf_p2g_particle(I, a.mats, mt, make_float2(xv.z, xv.w), a.s.C[g], F, jp, fb, pressure,
                      a.params[m].payload_density, sc);
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
  unsigned long long* fix = a.fix + 3 * I.g_off;
  if (W * H > kTileNodes) {  // uniform: the direct path
    if (!valid) return;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float3 c = jf_node_contrib_strict(I, st, sc, i, j);
        const int64_t n = 3 * ((int64_t)(st.by + j) * I.nx + st.bx + i);
        add_fixed(fix + n + 0, c.x, a.err + m);
        add_fixed(fix + n + 1, c.y, a.err + m);
        add_fixed(fix + n + 2, c.z, a.err + m);
      }
    }
    return;
  }
  const int entries = 3 * W * H;
  for (int e = threadIdx.x; e < entries; e += blockDim.x) s_acc[e] = 0ull;
  __syncthreads();
  if (valid) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float3 c = jf_node_contrib_strict(I, st, sc, i, j);
        unsigned long long* t = s_acc + 3 * ((st.by + j - y0) * W + (st.bx + i - x0));
        atomicAdd(t + 0, to_fixed(c.x, a.err + m));
        atomicAdd(t + 1, to_fixed(c.y, a.err + m));
        atomicAdd(t + 2, to_fixed(c.z, a.err + m));
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < entries; e += blockDim.x) {
    const unsigned long long v = s_acc[e];
    if (v == 0ull) continue;
    const int node = e / 3, comp = e - 3 * node;
    const int ty = node / W, tx = node - ty * W;
    atomicAdd(fix + 3 * ((int64_t)(y0 + ty) * I.nx + x0 + tx) + comp, v);
  }
}

__global__ void gf_grid(GradArgs a) {
  const int m = blockIdx.y;
  const JfInst I = a.inst[m];
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= I.nx * I.ny) return;
  const unsigned long long* q = a.fix + 3 * (I.g_off + n);
  const float px = from_fixed(q[0]), py = from_fixed(q[1]), pm = from_fixed(q[2]);
  a.u[I.g_off + n] = jf_grid_node(I, n % I.nx, n / I.nx, px, py, pm);
  if (a.pmv) a.pmv[I.g_off + n] = make_float4(px, py, pm, 0.0f);
}

__global__ void gf_g2p(GradArgs a) {
  const int m = blockIdx.y;
  const JfInst I = a.inst[m];
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
  const float4 xv = a.s.xv[g];
  float2 x = make_float2(xv.x, xv.y), v = make_float2(xv.z, xv.w);
  float4 C = a.s.C[g];
  const float2* u = a.u + I.g_off;
  const int nx = I.nx;
  JfStencil st;
  if (jf_stencil_strict(I, x, st)) {
    jf_g2p_apic_nodes(I, st, v, C, [&](int i, int j) { return u[(st.by + j) * nx + st.bx + i]; });
  }
  jf_g2p_advect(I, x, v);
  if (!(isfinite(x.x) && isfinite(x.y) && isfinite(v.x) && isfinite(v.y))) atomicOr(a.err + m, 1);
  a.o.xv[g] = make_float4(x.x, x.y, v.x, v.y);
  a.o.C[g] = C;
}

struct AdjArgs {
  GradArgs f;          // pre-step state of this substep (segment buffer) and its kept grid (u, pmv)
  float4* lxv;         // adjoint (x, v): in = post-step, out = pre-step
  float4* lC;
  float4* lF;
  float2* ubar;        // adjoint of the updated grid velocity
  float4* pmbar;       // adjoint of the accumulated momentum (x, y) and mass (z)
  float2* xtmp;        // G2P part of the position adjoint
  float2* vtmp;        // velocity adjoint of particles outside the stencil range
  double* gparam;      // M x 3: d/d actuation, d/d contraction, d/d freq
  double* dLdp;        // M: d L / d pressure of this substep, per instance
  double* fac;         // M x 3: d pressure / d (actuation, contraction, freq) of this substep
};

__device__ __forceinline__ float wd(int k, float f) {  // d W_k / d f
  return k == 0 ? -(1.5f - f) : (k == 1 ? -2.0f * (f - 1.0f) : (f - 0.5f));
}

__device__ __forceinline__ float clamp_pass(float xpp, float lo, float hi) {
  return (xpp > lo && xpp < hi) ? 1.0f : 0.0f;
}

__global__ void ad_g2p(AdjArgs A) {
  const GradArgs& a = A.f;
  const int m = blockIdx.y;
  const JfInst I = a.inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  if (a.mat[g] < 0) return;
  const float4 xv = a.s.xv[g];
  float2 x = make_float2(xv.x, xv.y), v = make_float2(xv.z, xv.w);
  const float4 lxv = A.lxv[g];
  const float4 Cb = A.lC[g];
  JfStencil st;
  const bool inr = jf_stencil_strict(I, x, st);
  const float2* u = a.u + I.g_off;
  const int nx = I.nx;
  float2 vn = v;
  if (inr) {
    float4 Cn;
    jf_g2p_apic_nodes(I, st, vn, Cn, [&](int i, int j) { return u[(st.by + j) * nx + st.bx + i]; });
  }
  vn.y = vn.y - I.dtg;
  const float xpp0 = __fadd_rn(x.x, __fmul_rn(I.dt, vn.x));
  const float xpp1 = __fadd_rn(x.y, __fmul_rn(I.dt, vn.y));
  const float xd0 = lxv.x * clamp_pass(xpp0, 0.001f, 0.999f);
  const float xd1 = lxv.y * clamp_pass(xpp1, 0.001f, I.y_hi);
  const float vt0 = lxv.z + I.dt * xd0;
  const float vt1 = lxv.w + I.dt * xd1;
  if (!inr) {
    A.xtmp[g] = make_float2(xd0, xd1);
    A.vtmp[g] = make_float2(vt0, vt1);
    return;
  }
  const float wx[3] = {st.wx0, st.wx1, st.wx2};
  const float wy[3] = {st.wy0, st.wy1, st.wy2};
  float xb0 = 0.0f, xb1 = 0.0f, xe0 = 0.0f, xe1 = 0.0f;
  float2* ub = A.ubar + I.g_off;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int n = (st.by + j) * nx + st.bx + i;
      const float2 uu = u[n];
      const float w = wx[i] * wy[j];
      const float e0 = (float)i - st.fx0, e1 = (float)j - st.fx1;
      const float ce0 = Cb.x * e0 + Cb.y * e1;  // (C_bar e)_0
      const float ce1 = Cb.z * e0 + Cb.w * e1;  // (C_bar e)_1
      atomicAdd(ub + n, make_float2(w * vt0 + I.c4 * w * ce0, w * vt1 + I.c4 * w * ce1));
      const float sgl = uu.x * vt0 + uu.y * vt1 + I.c4 * (uu.x * ce0 + uu.y * ce1);
      xb0 += wd(i, st.fx0) * wy[j] * sgl;
      xb1 += wx[i] * wd(j, st.fx1) * sgl;
      xe0 += w * (Cb.x * uu.x + Cb.z * uu.y);
      xe1 += w * (Cb.y * uu.x + Cb.w * uu.y);
    }
  }
  const float cf = I.c4 * I.inv_dx;
  A.xtmp[g] = make_float2(xd0 + I.inv_dx * xb0 - cf * xe0, xd1 + I.inv_dx * xb1 - cf * xe1);
  A.vtmp[g] = make_float2(0.0f, 0.0f);
}

// d pressure / d (actuation, contraction, freq) of instance m at time t: the
// activation a, A da/dc and A da/df (mpm_sim.py:173-180; the drop at
// phase == c is added on the host, see add_waveform_drop_terms).
__device__ __forceinline__ void pressure_factors(const JfParams& P, float tf, double* fac) {
  const double f = P.freq, c = P.contraction, t = tf;
  const float act = jf_activation(P.freq, P.contraction, tf);
  const double period = 1.0 / f;
  const double phase = (t - period * floor(t / period)) / period;
  double da_dc = 0.0, da_df = 0.0;
  if (act != 0.0f && phase < c) {
    const double sn = 0.5 * sin(3.14159265 * phase / c);
    da_dc = sn * 3.14159265 * (-phase / (c * c));
    da_df = sn * (3.14159265 / c) * t;
  }
  fac[0] = act;
  fac[1] = P.actuation * da_dc;
  fac[2] = P.actuation * da_df;
}

__global__ void ad_grid(AdjArgs A) {
  const GradArgs& a = A.f;
  const int m = blockIdx.y;
  if (blockIdx.x == 0 && threadIdx.x == 0) pressure_factors(a.params[m], a.t, A.fac + 3 * m);
  const JfInst I = a.inst[m];
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= I.nx * I.ny) return;
  const int64_t node = I.g_off + n;
  const float4 q = a.pmv[node];
  const float px = q.x, py = q.y, pm = q.z;
  const float2 ub = A.ubar[node];
  if (!(pm > 0.0f)) {
    A.pmbar[node] = make_float4(ub.x, ub.y, 0.0f, 0.0f);
    return;
  }
  const int i = n % I.nx, j = n / I.nx;
  float damp = 1.0f;
  if (i < I.dcx) damp = damp * (0.95f + 0.05f * (float)i / (float)I.dcx);
  if (i > I.nx - I.dcx) damp = damp * (0.95f + 0.05f * (float)(I.nx - i) / (float)I.dcx);
  if (j < I.dcy) damp = damp * (0.95f + 0.05f * (float)j / (float)I.dcy);
  if (j > I.ny - I.dcy) damp = damp * (0.95f + 0.05f * (float)(I.ny - j) / (float)I.dcy);
  const float g0 = (px / pm) * damp, g1 = (py / pm) * damp;
  const bool z0 = (i < 3 && g0 < 0.0f) || (i > I.nx - 3 && g0 > 0.0f);
  const bool z1 = (j < 3 && g1 < 0.0f) || (j > I.ny - 3 && g1 > 0.0f);
  const float a0 = z0 ? 0.0f : damp * ub.x / pm;
  const float a1 = z1 ? 0.0f : damp * ub.y / pm;
  A.pmbar[node] = make_float4(a0, a1, -(a0 * px + a1 * py) / pm, 0.0f);
}

// The P2G adjoint of one live particle g of instance m.  kWater: only water
// particles whose singular values are both above the 1e-6 floor are done here
// (closed-form Jacobian: J = det F*, dJ = cof F*, F_out = sqrt(J) I,
// tau = lambda J (J - 1) I; mpm_sim.py:219-227 with mu = 0), and false is
// returned for every other particle in range (it goes to the second kernel);
// otherwise the material map is differentiated with dual numbers.  Returns
// true when the particle is done; *pbar = d L / d pressure of the particle.
template <bool kWater>
__device__ __forceinline__ bool ad_p2g_particle(const AdjArgs& A, const JfInst& I, int m, int64_t g, int mt,
                                                float pressure, float* pbar) {
  const GradArgs& a = A.f;
  *pbar = 0.0f;
  const float4 xv = a.s.xv[g];
  const float2 x = make_float2(xv.x, xv.y), v = make_float2(xv.z, xv.w);
  JfStencil st;
  const float2 xt = A.xtmp[g];
  if (!jf_stencil_strict(I, x, st)) {
    A.lxv[g] = make_float4(xt.x, xt.y, A.vtmp[g].x, A.vtmp[g].y);
    return true;  // C and F pass through unchanged outside the stencil range
  }
  if (kWater && mt != 0) return false;
  const float4 C = a.s.C[g], F = a.s.F[g];
  const float dt = I.dt;
  const float M00 = radd(1.0f, rmul(dt, C.x)), M01 = rmul(dt, C.y);
  const float M10 = rmul(dt, C.z), M11 = radd(1.0f, rmul(dt, C.w));
  const float fsv[4] = {rdot2(M00, F.x, M01, F.z), rdot2(M00, F.y, M01, F.w),
                        rdot2(M10, F.x, M11, F.z), rdot2(M10, F.y, M11, F.w)};
  const int ms = jf_mat_slot(mt);
  const JfMaterials& mats = a.mats;
  const float la = ms == 0 ? mats.la[0] : ms == 1 ? mats.la[1] : ms == 2 ? mats.la[2]
                 : ms == 3 ? mats.la[3] : mats.la[4];
  const float2 fb = (mt == 3) ? a.fiber[g] : make_float2(0.0f, 1.0f);
  // the material map F* -> (F_out, tau): values and Jacobians d./dF*[e]
  float tv[4];        // tau values
  D4 Fo[4], tau[4], J;  // full path: values and Jacobians
  float dJ[4], kf = 0.0f, kt = 0.0f;  // water path: J = det F*, dJ = cof F*
  if constexpr (kWater) {
    // water, no singular value at the 1e-6 floor: J = s1 s2 = det F*, so
    // dJ = cof F*, dF_out = dJ / (2 sqrt J) I, dtau = lambda (2 J - 1) dJ I;
    // values as the forward rounds them
    const JfSvdRot rot = jf_svd2_values(make_float4(fsv[0], fsv[1], fsv[2], fsv[3]));
    if (!(rot.s1 > 1e-6f && rot.s2 > 1e-6f)) return false;
    const float Jw = rmul(rot.s1, rot.s2);
    dJ[0] = fsv[3]; dJ[1] = -fsv[2]; dJ[2] = -fsv[1]; dJ[3] = fsv[0];
    kf = 0.5f / sqrtf(Jw);
    kt = la * (2.0f * Jw - 1.0f);
    const float diag = rmul(rmul(la, Jw), rsub(Jw, 1.0f));
    tv[0] = diag; tv[1] = 0.0f; tv[2] = 0.0f; tv[3] = diag;
  } else {
    const float mu = ms == 0 ? mats.mu[0] : ms == 1 ? mats.mu[1] : ms == 2 ? mats.mu[2]
                   : ms == 3 ? mats.mu[3] : mats.mu[4];
    D4 Fs[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      Fs[q] = d4c(fsv[q]);
      Fs[q].d[q] = 1.0f;
    }
    jf_phi<D4>(Fs, mt, mu, la, pressure, fb, Fo, tau, J);
#pragma unroll
    for (int q = 0; q < 4; ++q) tv[q] = tau[q].v;
  }
  float mass = I.p_mass;
  if (mt == 2) mass = mass * a.params[m].payload_density;
  const float ks = I.stress_scale;
  const float Af00 = ks * tv[0] + mass * C.x, Af01 = ks * tv[1] + mass * C.y;
  const float Af10 = ks * tv[2] + mass * C.z, Af11 = ks * tv[3] + mass * C.w;
  const float wx[3] = {st.wx0, st.wx1, st.wx2};
  const float wy[3] = {st.wy0, st.wy1, st.wy2};
  const float4* pmb = A.pmbar + I.g_off;
  float vb0 = 0.f, vb1 = 0.f, Ab00 = 0.f, Ab01 = 0.f, Ab10 = 0.f, Ab11 = 0.f;
  float xb0 = 0.f, xb1 = 0.f, xa0 = 0.f, xa1 = 0.f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float4 pb = pmb[(st.by + j) * I.nx + st.bx + i];
      const float w = wx[i] * wy[j];
      const float d0 = ((float)i - st.fx0) * I.dx, d1 = ((float)j - st.fx1) * I.dx;
      vb0 += w * pb.x;
      vb1 += w * pb.y;
      Ab00 += w * pb.x * d0; Ab01 += w * pb.x * d1;
      Ab10 += w * pb.y * d0; Ab11 += w * pb.y * d1;
      const float mom0 = mass * v.x + (Af00 * d0 + Af01 * d1);
      const float mom1 = mass * v.y + (Af10 * d0 + Af11 * d1);
      const float qv = pb.x * mom0 + pb.y * mom1 + pb.z * mass;
      xb0 += wd(i, st.fx0) * wy[j] * qv;
      xb1 += wx[i] * wd(j, st.fx1) * qv;
      xa0 += w * (Af00 * pb.x + Af10 * pb.y);
      xa1 += w * (Af01 * pb.x + Af11 * pb.y);
    }
  }
  const float tb[4] = {ks * Ab00, ks * Ab01, ks * Ab10, ks * Ab11};
  const float4 Fob = A.lF[g];
  const float fob[4] = {Fob.x, Fob.y, Fob.z, Fob.w};
  float Fsb[4];
  if constexpr (kWater) {
    const float cw = (fob[0] + fob[3]) * kf + (tb[0] + tb[3]) * kt;
#pragma unroll
    for (int e = 0; e < 4; ++e) Fsb[e] = cw * dJ[e];
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float acc = 0.0f;
#pragma unroll
      for (int q = 0; q < 4; ++q) acc += fob[q] * Fo[q].d[e] + tb[q] * tau[q].d[e];
      Fsb[e] = acc;
    }
    if (mt == 3) {
      *pbar = (tb[0] * fb.x * fb.x + tb[1] * fb.x * fb.y + tb[2] * fb.y * fb.x + tb[3] * fb.y * fb.y) * J.v;
    }
  }
  // F* = M F: F_bar = M^T F*_bar, C_bar += dt F*_bar F^T
  const float Fb00 = M00 * Fsb[0] + M10 * Fsb[2], Fb01 = M00 * Fsb[1] + M10 * Fsb[3];
  const float Fb10 = M01 * Fsb[0] + M11 * Fsb[2], Fb11 = M01 * Fsb[1] + M11 * Fsb[3];
  const float Cb00 = mass * Ab00 + dt * (Fsb[0] * F.x + Fsb[1] * F.y);
  const float Cb01 = mass * Ab01 + dt * (Fsb[0] * F.z + Fsb[1] * F.w);
  const float Cb10 = mass * Ab10 + dt * (Fsb[2] * F.x + Fsb[3] * F.y);
  const float Cb11 = mass * Ab11 + dt * (Fsb[2] * F.z + Fsb[3] * F.w);
  const float4 lx = make_float4(xt.x + I.inv_dx * xb0 - xa0, xt.y + I.inv_dx * xb1 - xa1, mass * vb0,
                                mass * vb1);
  A.lxv[g] = lx;
  A.lC[g] = make_float4(Cb00, Cb01, Cb10, Cb11);
  A.lF[g] = make_float4(Fb00, Fb01, Fb10, Fb11);
  const float chk = ((lx.x + lx.y) + (lx.z + lx.w)) + ((Cb00 + Cb01) + (Cb10 + Cb11)) +
                    ((Fb00 + Fb01) + (Fb10 + Fb11));
  if (!isfinite(chk)) atomicOr(a.err + m, 4);
  return true;
}

// P2G adjoint of the water particles (most of the tank): the closed-form
// Jacobian at the register budget of that path; water at the singular-value
// floor is listed for ad_p2g_list (the full path), and every other material is
// done by ad_p2g_list over the rollout's list of non-water particles, which
// runs beside this kernel on a second stream.
__global__ void __launch_bounds__(kT, 4) ad_p2g_water(AdjArgs A, int32_t* floor_list, int32_t* n_floor) {
  const GradArgs& a = A.f;
  const int m = blockIdx.y;
  const JfInst I = a.inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  if (a.mat[g] != 0) return;
  float pbar;
  if (!ad_p2g_particle<true>(A, I, m, g, 0, 0.0f, &pbar)) floor_list[atomicAdd(n_floor, 1)] = (int32_t)g;
}

// P2G adjoint with the full material map (dual-number SVD) over a list of
// particles; the muscle's d L / d pressure goes into the parameter gradients
// of its instance.
__global__ void __launch_bounds__(kT) ad_p2g_list(AdjArgs A, const int32_t* list, const int32_t* n_list,
                                                  const int32_t* inst_of) {
  const GradArgs& a = A.f;
  const int n = *n_list;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int64_t g = list[r];
    const int m = inst_of[g];
    const JfInst I = a.inst[m];
    const double* fm = A.fac + 3 * m;
    const float pressure = a.params[m].actuation * (float)fm[0];
    float pbar = 0.0f;
    ad_p2g_particle<false>(A, I, m, g, a.mat[g], pressure, &pbar);
    if (pbar != 0.0f) {
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
__global__ void seed_kernel(const JfInst* __restrict__ inst, const int32_t* __restrict__ mat,
                            const int32_t* __restrict__ body_mode, const double* __restrict__ inv_n,
                            float4* lxv, float4* lC, float4* lF, int init, float sign) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const int mt = mat[g];
  const bool sel = body_mode[m] ? (mt == 1 || mt == 3) : (mt == 2);
  const float s = sel ? sign * (float)inv_n[m] : 0.0f;
  if (init) {
    lxv[g] = make_float4(0.0f, s, 0.0f, 0.0f);
    lC[g] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    lF[g] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
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

template <class T>
cudaError_t alloc_n(T** p, size_t n) {
  return cudaMalloc((void**)p, sizeof(T) * (n > 0 ? n : 1));
}

}  // namespace

// A CUDA graph of a rollout's device work, replayed while its key (sizes,
// start time, buffer addresses) is unchanged.
struct GradGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> key;
  int64_t launches = 0;  // kernels one replay launches
};

// Device buffers of the differentiable rollout, owned by the engine.
struct JfGrad {
  int64_t steps = 0;
  int32_t K = 0;
  float t0 = 0.0f;
  size_t n_ck = 0, seg_cap = 0;
  unsigned long long* fix = nullptr;
  float2* u = nullptr;
  float2* ubar = nullptr;
  float4* pmbar = nullptr;
  float4 *lxv = nullptr, *lC = nullptr, *lF = nullptr;
  float2 *xtmp = nullptr, *vtmp = nullptr;
  float4* ck = nullptr;     // n_ck checkpoints x 3 arrays x total slots
  // two sets of segment buffers: the backward recomputes segment k - 1 into
  // one while the adjoint of segment k reads the other
  float4* seg[2] = {nullptr, nullptr};    // K states x 3 arrays x total slots
  float2* useg[2] = {nullptr, nullptr};   // K grids: updated velocity per node
  float4* pmseg[2] = {nullptr, nullptr};  // K grids: (momentum x, momentum y, mass) per node
  cudaStream_t rstream = nullptr;         // the recompute's stream
  cudaEvent_t ready[2] = {nullptr, nullptr}, released[2] = {nullptr, nullptr};
  float4* fin = nullptr;    // final state (3 arrays)
  float* fin_Jp = nullptr;  // final Jp (the backward's recompute updates Jp in place)
  double* gparam = nullptr;
  double* dLdp = nullptr;   // steps x M: d L / d pressure per substep and instance
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
  std::vector<double> loss;
  bool have_forward = false;
  int n_sm = 148;
  GradGraph fwd_graph, bwd_graph, step_graph;  // forward, backward, forward + backward
};

void jf_grad_free(jf_engine* e) {
  JfGrad* G = e->grad;
  if (!G) return;
  cudaFree(G->fix); cudaFree(G->u); cudaFree(G->ubar); cudaFree(G->pmbar);
  cudaFree(G->lxv); cudaFree(G->lC); cudaFree(G->lF); cudaFree(G->xtmp); cudaFree(G->vtmp);
  cudaFree(G->ck); cudaFree(G->fin); cudaFree(G->fin_Jp); cudaFree(G->gparam);
  for (int b = 0; b < 2; ++b) {
    cudaFree(G->seg[b]); cudaFree(G->useg[b]); cudaFree(G->pmseg[b]);
    if (G->ready[b]) cudaEventDestroy(G->ready[b]);
    if (G->released[b]) cudaEventDestroy(G->released[b]);
  }
  if (G->rstream) cudaStreamDestroy(G->rstream);
  for (GradGraph* gg : {&G->fwd_graph, &G->bwd_graph, &G->step_graph})
    if (gg->exec) cudaGraphExecDestroy(gg->exec);
  cudaFree(G->dLdp); cudaFree(G->fac); cudaFree(G->solid); cudaFree(G->floor_list); cudaFree(G->counts);
  cudaFree(G->inst_of);
  if (G->side) cudaStreamDestroy(G->side);
  if (G->fork) cudaEventDestroy(G->fork);
  if (G->join) cudaEventDestroy(G->join);
  cudaFree(G->body_mode); cudaFree(G->inv_n);
  delete G;
  e->grad = nullptr;
}

static GradArgs grad_args(jf_engine* e, GradState s, float t) {
  JfGrad* G = e->grad;
  GradArgs a;
  a.inst = e->d_inst;
  a.params = e->d_params;
  a.mats = jf_materials();
  a.s = s;
  a.o = s;
  a.mat = e->p.mat;
  a.Jp = e->p.Jp;
  a.fiber = e->p.fiber;
  a.fix = G->fix;
  a.u = G->u;
  a.pmv = nullptr;
  a.err = e->d_err;
  a.t = t;
  return a;
}

static GradState state_at(float4* base, size_t slots, size_t idx) {
  float4* b = base + 3 * slots * idx;
  return GradState{b, b + slots, b + 2 * slots};
}

static cudaError_t copy_state(jf_engine* e, GradState dst, GradState src, cudaStream_t st = nullptr) {
  const size_t bytes = sizeof(float4) * (size_t)e->total_slots;
  if (!st) st = e->stream;
  cudaError_t err;
  if ((err = cudaMemcpyAsync(dst.xv, src.xv, bytes, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return err;
  if ((err = cudaMemcpyAsync(dst.C, src.C, bytes, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return err;
  return cudaMemcpyAsync(dst.F, src.F, bytes, cudaMemcpyDeviceToDevice, st);
}

// one deterministic substep of every instance from state s at time t into
// state o (s itself when o is not given); with u_keep / pmv_keep set, its grid
// is written there for the adjoint
static cudaError_t det_substep(jf_engine* e, GradState s, float t, float2* u_keep = nullptr,
                               float4* pmv_keep = nullptr, const GradState* o = nullptr,
                               cudaStream_t st = nullptr) {
  if (!st) st = e->stream;
  JfGrad* G = e->grad;
  GradArgs a = grad_args(e, s, t);
  if (o) a.o = *o;
  if (u_keep) {
    a.u = u_keep;
    a.pmv = pmv_keep;
  }
  cudaError_t err = cudaMemsetAsync(G->fix, 0, sizeof(unsigned long long) * 3 * (size_t)e->total_nodes, st);
  if (err != cudaSuccess) return err;
  const dim3 gp((e->max_slots + kT - 1) / kT, e->M), gn((e->max_cells + kT - 1) / kT, e->M);
  gf_p2g<<<gp, kT, 0, st>>>(a);
  gf_grid<<<gn, kT, 0, st>>>(a);
  gf_g2p<<<gp, kT, 0, st>>>(a);
  e->launches += 3;
  return cudaGetLastError();
}

// Every buffer of a rollout of `steps` substeps with a checkpoint every K
// (allocated before any graph capture: capture allows no allocation).
static cudaError_t grad_alloc(jf_engine* e, int64_t steps, int32_t K) {
  if (!e->grad) e->grad = new JfGrad();
  JfGrad* G = e->grad;
  const size_t slots = (size_t)e->total_slots;
  const size_t n_ck = (size_t)((steps + K - 1) / K);
  cudaError_t err = cudaSuccess;
  if (!G->fix) {
    if ((err = alloc_n(&G->fix, 3 * (size_t)e->total_nodes)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->u, e->total_nodes)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->ubar, e->total_nodes)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->pmbar, e->total_nodes)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->lxv, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->lC, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->lF, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->xtmp, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->vtmp, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->fin, 3 * slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->fin_Jp, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->gparam, 3 * (size_t)e->M)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->body_mode, e->M)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->inv_n, e->M)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->fac, 3 * (size_t)e->M)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->solid, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->floor_list, slots)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->counts, 2)) != cudaSuccess) return err;
    if ((err = alloc_n(&G->inst_of, slots)) != cudaSuccess) return err;
    if ((err = cudaStreamCreateWithFlags(&G->side, cudaStreamNonBlocking)) != cudaSuccess) return err;
    if ((err = cudaEventCreateWithFlags(&G->fork, cudaEventDisableTiming)) != cudaSuccess) return err;
    if ((err = cudaEventCreateWithFlags(&G->join, cudaEventDisableTiming)) != cudaSuccess) return err;
    if ((err = cudaStreamCreateWithFlags(&G->rstream, cudaStreamNonBlocking)) != cudaSuccess) return err;
    for (int b = 0; b < 2; ++b) {
      if ((err = cudaEventCreateWithFlags(&G->ready[b], cudaEventDisableTiming)) != cudaSuccess) return err;
      if ((err = cudaEventCreateWithFlags(&G->released[b], cudaEventDisableTiming)) != cudaSuccess) return err;
    }
    const dim3 gp((e->max_slots + kT - 1) / kT, e->M);
    inst_of_kernel<<<gp, kT, 0, e->stream>>>(e->d_inst, G->inst_of);
    e->launches += 1;
    cudaDeviceGetAttribute(&G->n_sm, cudaDevAttrMultiProcessorCount, e->device);
  }
  if (G->n_ck < n_ck) {
    cudaFree(G->ck);
    G->ck = nullptr;
    if ((err = alloc_n(&G->ck, 3 * slots * n_ck)) != cudaSuccess) return err;
    G->n_ck = n_ck;
  }
  if (G->dLdp_cap < (size_t)steps * e->M) {
    cudaFree(G->dLdp);
    G->dLdp = nullptr;
    G->dLdp_cap = 0;
    if ((err = alloc_n(&G->dLdp, (size_t)steps * e->M)) != cudaSuccess) return err;
    G->dLdp_cap = (size_t)steps * e->M;
  }
  return cudaSuccess;
}

// The backward's segment buffers (K pre-step states and grids, two sets),
// allocated only when a backward runs, so that a forward-only rollout with a
// long checkpoint interval does not hold them.
static cudaError_t seg_alloc(jf_engine* e, int32_t K) {
  JfGrad* G = e->grad;
  const size_t slots = (size_t)e->total_slots;
  cudaError_t err = cudaSuccess;
  if (G->seg_cap < (size_t)K) {
    G->seg_cap = 0;
    for (int b = 0; b < 2; ++b) {
      cudaFree(G->seg[b]);
      cudaFree(G->useg[b]);
      cudaFree(G->pmseg[b]);
      G->seg[b] = nullptr;
      G->useg[b] = nullptr;
      G->pmseg[b] = nullptr;
      if ((err = alloc_n(&G->seg[b], 3 * slots * (size_t)K)) != cudaSuccess) return err;
      if ((err = alloc_n(&G->useg[b], (size_t)e->total_nodes * K)) != cudaSuccess) return err;
      if ((err = alloc_n(&G->pmseg[b], (size_t)e->total_nodes * K)) != cudaSuccess) return err;
    }
    G->seg_cap = (size_t)K;
  }
  return cudaSuccess;
}

// The forward's device work: the non-water list, the substeps from G->t0
// with their checkpoints, and copies of the final state.
static cudaError_t fwd_record(jf_engine* e) {
  JfGrad* G = e->grad;
  const size_t slots = (size_t)e->total_slots;
  const int64_t steps = G->steps;
  const int32_t K = G->K;
  cudaError_t err;
  // the rollout's non-water particles, for the backward's second stream
  if ((err = cudaMemsetAsync(G->counts, 0, sizeof(int32_t), e->stream))) return err;
  {
    const dim3 gp((e->max_slots + kT - 1) / kT, e->M);
    nonwater_list_kernel<<<gp, kT, 0, e->stream>>>(e->d_inst, e->p.mat, G->solid, G->counts);
    e->launches += 1;
  }
  const GradState work{e->p.xv, e->p.C, e->p.F};
  const float dtf = (float)e->dt;
  float t = G->t0;
  for (int64_t s = 0; s < steps; ++s) {
    if (s % K == 0) {
      if ((err = copy_state(e, state_at(G->ck, slots, s / K), work)) != cudaSuccess) return err;
    }
    {
      JfTimed timed(e, false);
      if ((err = det_substep(e, work, t)) != cudaSuccess) return err;
    }
    t = t + dtf;
  }
  if ((err = copy_state(e, state_at(G->fin, slots, 0), work)) != cudaSuccess) return err;
  return cudaMemcpyAsync(G->fin_Jp, e->p.Jp, sizeof(float) * slots, cudaMemcpyDeviceToDevice, e->stream);
}

// Phase of the waveform at time t in FP32, as jf_activation computes it
// (mpm_sim.py:173-174).
static float waveform_phase(float freq, float t) {
  volatile float period = 1.0f / (1.0f * freq);
  volatile float q = floorf(t / period);
  volatile float pq = period * q;
  volatile float r = t - pq;
  volatile float phase = r / period;
  return phase;
}

// Boundary terms of the waveform's drop from 1 to 0 at phase == contraction
// (mpm_sim.py:176-180): for every drop between substeps n - 1 and n of the
// rollout, at the instant t* where the phase, advancing by f per unit time,
// reaches c, d L / d c += A g* / (f dt) and d L / d f -= A g* t* / (f dt), with
// g* = d L / d pressure interpolated between the two substeps (the rollout's
// pressure at substep n is A a(phase(t_n)), and a(c-) = 1).
static void add_waveform_drop_terms(const jf_engine* e, const std::vector<float>& ts,
                                    const std::vector<double>& dLdp, double* gparam) {
  const int64_t steps = (int64_t)ts.size() - 1;
  for (int m = 0; m < e->M; ++m) {
    const JfParams& P = e->params[m];
    const double A = P.actuation, c = P.contraction, f = P.freq;
    if (!(f > 0.0) || !(c > 0.0) || A == 0.0) continue;
    float prev = waveform_phase(P.freq, ts[0]);
    for (int64_t n = 1; n < steps; ++n) {
      const float ph = waveform_phase(P.freq, ts[(size_t)n]);
      if (prev < P.contraction && !(ph < P.contraction) && ph >= prev) {
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
static cudaError_t bwd_record(jf_engine* e) {
  JfGrad* G = e->grad;
  const size_t slots = (size_t)e->total_slots;
  const int64_t steps = G->steps;
  const int32_t K = G->K;
  const float dtf = (float)e->dt;
  std::vector<float> ts((size_t)steps + 1);
  ts[0] = G->t0;
  for (int64_t s = 0; s < steps; ++s) ts[s + 1] = ts[s] + dtf;
  const dim3 gp((e->max_slots + kT - 1) / kT, e->M), gn((e->max_cells + kT - 1) / kT, e->M);
  cudaError_t err = cudaMemsetAsync(G->gparam, 0, sizeof(double) * 3 * e->M, e->stream);
  if (err != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(G->dLdp, 0, sizeof(double) * (size_t)steps * e->M, e->stream))) return err;
  seed_kernel<<<gp, kT, 0, e->stream>>>(e->d_inst, e->p.mat, G->body_mode, G->inv_n, G->lxv, G->lC, G->lF, 1, 1.0f);
  e->launches += 1;
  const GradState work{e->p.xv, e->p.C, e->p.F};
  const int64_t n_seg = (steps + K - 1) / K;
  const size_t nodes = (size_t)e->total_nodes;
  const int list_blocks = 2 * G->n_sm;  // grid-stride over the listed particles
  const int floor_blocks = 16;       // water at the singular-value floor: rare
  auto seg_len = [&](int64_t seg) { return (int)((steps - seg * K) < K ? (steps - seg * K) : K); };
  // Recompute of segment `seg` into buffer set b on the recompute stream: its
  // pre-step states (substep j reads state j and writes state j + 1; the last
  // writes the engine's work arrays, which nothing reads) and every substep's
  // grid.  It waits until the adjoint that last read buffer set b is done.
  // The recompute needs only its checkpoint, so it runs while the main stream
  // runs the adjoint of the segment after it.
  auto recompute = [&](int64_t seg, int b) -> cudaError_t {
    cudaError_t r;
    if ((r = cudaStreamWaitEvent(G->rstream, G->released[b], 0))) return r;
    if ((r = copy_state(e, state_at(G->seg[b], slots, 0), state_at(G->ck, slots, (size_t)seg), G->rstream)))
      return r;
    const int n = seg_len(seg);
    for (int j = 0; j < n; ++j) {
      const GradState next = (j + 1 < n) ? state_at(G->seg[b], slots, (size_t)j + 1) : work;
      if ((r = det_substep(e, state_at(G->seg[b], slots, (size_t)j), ts[seg * K + j], G->useg[b] + nodes * j,
                           G->pmseg[b] + nodes * j, &next, G->rstream)))
        return r;
    }
    return cudaEventRecord(G->ready[b], G->rstream);
  };
  // the recompute stream starts after everything queued on the main stream
  // (the forward's state and the seeds above)
  if ((err = cudaEventRecord(G->released[0], e->stream))) return err;
  if ((err = cudaEventRecord(G->released[1], e->stream))) return err;
  if ((err = recompute(n_seg - 1, 0))) return err;
  for (int64_t seg = n_seg - 1; seg >= 0; --seg) {
    const int b = (int)((n_seg - 1 - seg) & 1);
    if (seg > 0 && (err = recompute(seg - 1, b ^ 1))) return err;
    if ((err = cudaStreamWaitEvent(e->stream, G->ready[b], 0))) return err;
    const int64_t s0 = seg * K;
    const int n = seg_len(seg);
    for (int j = n - 1; j >= 0; --j) {
      JfTimed timed(e, false);
      AdjArgs A;
      A.f = grad_args(e, state_at(G->seg[b], slots, (size_t)j), ts[s0 + j]);
      A.lxv = G->lxv;
      A.lC = G->lC;
      A.lF = G->lF;
      A.ubar = G->ubar;
      A.pmbar = G->pmbar;
      A.xtmp = G->xtmp;
      A.vtmp = G->vtmp;
      A.gparam = G->gparam;
      A.dLdp = G->dLdp + (size_t)(s0 + j) * e->M;
      A.fac = G->fac;
      // the substep's grid as the recompute left it
      A.f.u = G->useg[b] + nodes * j;
      A.f.pmv = G->pmseg[b] + nodes * j;
      if ((err = cudaMemsetAsync(G->ubar, 0, sizeof(float2) * nodes, e->stream))) return err;
      if ((err = cudaMemsetAsync(G->counts + 1, 0, sizeof(int32_t), e->stream))) return err;
      ad_g2p<<<gp, kT, 0, e->stream>>>(A);
      ad_grid<<<gn, kT, 0, e->stream>>>(A);
      // P2G adjoint: the non-water particles on the second stream, beside the water
      if ((err = cudaEventRecord(G->fork, e->stream))) return err;
      if ((err = cudaStreamWaitEvent(G->side, G->fork, 0))) return err;
      ad_p2g_list<<<list_blocks, kT, 0, G->side>>>(A, G->solid, G->counts, G->inst_of);
      if ((err = cudaEventRecord(G->join, G->side))) return err;
      ad_p2g_water<<<gp, kT, 0, e->stream>>>(A, G->floor_list, G->counts + 1);
      ad_p2g_list<<<floor_blocks, kT, 0, e->stream>>>(A, G->floor_list, G->counts + 1, G->inst_of);
      if ((err = cudaStreamWaitEvent(e->stream, G->join, 0))) return err;
      e->launches += 5;
      if ((err = cudaGetLastError()) != cudaSuccess) return err;
    }
    if ((err = cudaEventRecord(G->released[b], e->stream))) return err;
  }
  // the initial CoM term of the displacement
  seed_kernel<<<gp, kT, 0, e->stream>>>(e->d_inst, e->p.mat, G->body_mode, G->inv_n, G->lxv, G->lC, G->lF, 0, -1.0f);
  e->launches += 1;
  // leave the engine at the forward's final state
  if ((err = copy_state(e, work, state_at(G->fin, slots, 0))) != cudaSuccess) return err;
  if ((err = cudaMemcpyAsync(e->p.Jp, G->fin_Jp, sizeof(float) * slots, cudaMemcpyDeviceToDevice, e->stream)))
    return err;
  return cudaSuccess;
}

// After the backward's device work: the parameter gradients and the
// per-substep d L / d pressure to the host, then the waveform-drop terms.
static cudaError_t bwd_finish(jf_engine* e, double* gparam_host) {
  JfGrad* G = e->grad;
  const int64_t steps = G->steps;
  const float dtf = (float)e->dt;
  std::vector<float> ts((size_t)steps + 1);
  ts[0] = G->t0;
  for (int64_t s = 0; s < steps; ++s) ts[s + 1] = ts[s] + dtf;
  cudaError_t err;
  if ((err = cudaMemcpyAsync(gparam_host, G->gparam, sizeof(double) * 3 * e->M, cudaMemcpyDeviceToHost, e->stream)))
    return err;
  std::vector<double> dLdp((size_t)steps * e->M);
  if ((err = cudaMemcpyAsync(dLdp.data(), G->dLdp, sizeof(double) * dLdp.size(), cudaMemcpyDeviceToHost,
                             e->stream)))
    return err;
  if ((err = cudaStreamSynchronize(e->stream))) return err;
  add_waveform_drop_terms(e, ts, dLdp, gparam_host);
  return cudaSuccess;
}

// Runs `record` (device work on the engine's stream) directly, or, with
// graphs on and per-kernel timing off, from a CUDA graph captured on first
// use and replayed while `key` is unchanged.
template <class Record>
static cudaError_t run_graph(jf_engine* e, GradGraph& gg, const std::vector<uint64_t>& key, Record record) {
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

static std::vector<uint64_t> graph_key(const jf_engine* e, int tag) {
  const JfGrad* G = e->grad;
  uint32_t tbits;
  memcpy(&tbits, &G->t0, sizeof(tbits));
  return {(uint64_t)tag, (uint64_t)G->steps, (uint64_t)G->K, tbits, (uint64_t)(uintptr_t)e->p.xv,
          (uint64_t)(uintptr_t)e->p.C, (uint64_t)(uintptr_t)e->p.F, (uint64_t)(uintptr_t)e->p.Jp,
          (uint64_t)(uintptr_t)e->p.mat, (uint64_t)(uintptr_t)G->ck, (uint64_t)(uintptr_t)G->seg[0],
          (uint64_t)(uintptr_t)G->seg[1], (uint64_t)(uintptr_t)G->dLdp, (uint64_t)(uintptr_t)e->d_stats};
}

static cudaError_t grad_begin(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode,
                              const double* inv_n) {
  cudaError_t err = grad_alloc(e, steps, K);
  if (err != cudaSuccess) return err;
  JfGrad* G = e->grad;
  if ((err = cudaMemcpyAsync(G->body_mode, body_mode, sizeof(int32_t) * e->M, cudaMemcpyHostToDevice, e->stream)))
    return err;
  if ((err = cudaMemcpyAsync(G->inv_n, inv_n, sizeof(double) * e->M, cudaMemcpyHostToDevice, e->stream)))
    return err;
  G->steps = steps;
  G->K = K;
  G->t0 = e->t;
  return cudaSuccess;
}

static void grad_advance_time(jf_engine* e) {
  const float dtf = (float)e->dt;
  float t = e->grad->t0;
  for (int64_t s = 0; s < e->grad->steps; ++s) t = t + dtf;
  e->t = t;
}

cudaError_t jf_grad_forward_impl(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode,
                                 const double* inv_n) {
  cudaError_t err = grad_begin(e, steps, K, body_mode, inv_n);
  if (err != cudaSuccess) return err;
  if ((err = run_graph(e, e->grad->fwd_graph, graph_key(e, 1), [&] { return fwd_record(e); }))) return err;
  grad_advance_time(e);
  e->grad->have_forward = true;
  return cudaSuccess;
}

cudaError_t jf_grad_backward_impl(jf_engine* e, double* gparam_host) {
  cudaError_t err = seg_alloc(e, e->grad->K);
  if (err != cudaSuccess) return err;
  err = run_graph(e, e->grad->bwd_graph, graph_key(e, 2), [&] { return bwd_record(e); });
  if (err != cudaSuccess) return err;
  return bwd_finish(e, gparam_host);
}

// Forward and backward of one rollout as one graph; the final state's CoM
// sums are left in e->d_stats for the loss.
cudaError_t jf_grad_step_impl(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode,
                              const double* inv_n, double* gparam_host) {
  cudaError_t err = grad_begin(e, steps, K, body_mode, inv_n);
  if (err != cudaSuccess) return err;
  if ((err = seg_alloc(e, K)) != cudaSuccess) return err;
  err = run_graph(e, e->grad->step_graph, graph_key(e, 3), [&] {
    cudaError_t r = fwd_record(e);
    if (r == cudaSuccess) r = jf_stats_launch(e);
    if (r == cudaSuccess) r = bwd_record(e);
    return r;
  });
  if (err != cudaSuccess) return err;
  grad_advance_time(e);
  e->grad->have_forward = true;
  return bwd_finish(e, gparam_host);
}

// Position adjoint of the initial state for one instance, in engine order.
cudaError_t jf_grad_x0_impl(jf_engine* e, int m, std::vector<float4>& out) {
  const JfInst& I = e->inst[m];
  out.resize((size_t)I.n_slots);
  if (I.n_slots == 0) return cudaSuccess;
  cudaError_t err = cudaMemcpyAsync(out.data(), e->grad->lxv + I.p_off, sizeof(float4) * I.n_slots,
                                    cudaMemcpyDeviceToHost, e->stream);
  if (err != cudaSuccess) return err;
  return cudaStreamSynchronize(e->stream);
}
