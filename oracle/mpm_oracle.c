/*
 * mpm_oracle.c -- CPU restatement of jellyfih's 2-D MLS-MPM substep.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only
 * as the checker or the timed CPU baseline.  The product path never calls it.
 *
 * It restates, operation by operation and in the same evaluation order, the
 * reference engine in mpm_sim.py:
 *   - constants                 mpm_sim.py:18-58
 *   - substep()                 mpm_sim.py:153-340
 *       grid clear              mpm_sim.py:160-165
 *       P2G                     mpm_sim.py:168-271
 *       grid update             mpm_sim.py:274-309
 *       G2P                     mpm_sim.py:312-333
 *       glow                    mpm_sim.py:336-338
 *       axisymmetric variant    mpm_sim.py:17,163-165,235-268,292-303
 *                               (JELLY_AXISYM=1; r_ref set at load, :727)
 *   - payload / body CoM sums   mpm_sim.py:746-762
 * and the third-party 2x2 SVD the reference calls (ti.svd, mpm_sim.py:206):
 * taichi==1.7.4 (uv.lock:1591-1592), python/taichi/_funcs.py _polar_decompose2d
 * and _svd2d -- a polar decomposition A = R S followed by one symmetric Jacobi
 * rotation of S, restated from that published algorithm in svd2() below.
 *
 * Parity pin: tests/golden holds fixtures produced by executing the reference's
 * own mpm_sim.py source under a numpy stand-in for the Taichi runtime (strict
 * FP32, sequential struct-for order); tests/test_oracle_golden.py checks this
 * file against them.
 *
 * The file is compiled twice (see oracle/Makefile): REAL=float gives the FP32
 * oracle whose rounding follows the reference (Taichi default_fp=f32, Python
 * scalar constants folded in double and rounded to f32 at use), REAL=double
 * gives the FP64 build of the same algorithm used to state FP32 error.
 * Build with -ffp-contract=off: every operation is rounded on its own.
 *
 * Layouts follow the reference fields (row-major 2x2 matrices):
 *   x, v, fiber: [n][2]   C, F: [n][4] = (00, 01, 10, 11)   material: int32[n]
 *   r_ref: [n] (load radius, read only in the axisymmetric variant)
 *   grid_v: [nx][ny][2]   grid_m: [nx][ny]      (mpm_sim.py:92-93)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL float
#define SFX f32
#endif

#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

/* One instance's static description.  dt is the reference's Python double
 * (mpm_sim.py:19); constants derived from it are folded in double, as the
 * reference's Python-level arithmetic does, and rounded to REAL at use. */
typedef struct {
  int32_t nx;          /* n_grid (x nodes)        mpm_sim.py:14 */
  int32_t ny;          /* n_grid_y (y nodes)      mpm_sim.py:15 */
  double domain_h;     /* domain_height           mpm_sim.py:16 */
  double dt;           /* dt                      mpm_sim.py:19 */
  double actuation;    /* instance_actuation[m]      mpm_sim.py:116,146 */
  double contraction;  /* instance_act_contraction[m] mpm_sim.py:121,148 */
  double freq;         /* instance_freq[m]           mpm_sim.py:125,149 */
  double payload_density; /* instance_payload_density[m] mpm_sim.py:142,147 */
  int32_t axisym;      /* JELLY_AXISYM            mpm_sim.py:17 */
  int32_t fixed_p2g;   /* not in the reference: sum P2G in 2^-44 fixed point (below) */
} oracle_inst;

/* Order-free P2G sums (fixed_p2g != 0).  Each momentum / mass contribution is
 * rounded to the nearest multiple of 2^-44 (an int64; contributions of
 * magnitude >= 64 count as zero), the node sums are integer sums, whose value
 * does not depend on the order of the additions, and each sum is converted
 * back as (REAL)((double)sum * 2^-44) before the grid update.  This is the
 * accumulation the GPU engine's deterministic forward (the differentiable
 * rollout) uses; with it the oracle and that forward can be compared over
 * long rollouts without the summation-order noise of floating-point sums.
 * The reference itself sums in FP32 (mpm_sim.py:269-270). */
static const double kFixScale = 17592186044416.0; /* 2^44 */

static uint64_t FN(to_fixed)(REAL v) {
  if (!(fabs((double)v) < 64.0)) return 0;
  return (uint64_t)llrint((double)v * kFixScale);
}

static REAL FN(from_fixed)(uint64_t v) { return (REAL)((double)(int64_t)v * (1.0 / kFixScale)); }

/* Material constants, Python doubles (mpm_sim.py:25-48). */
static const double E_base = 0.1e4, nu_base = 0.2;
static const double E_jelly = 0.7e3, nu_jelly = 0.3;
static const double E_payload = 2.0e5, nu_payload = 0.2;
static const double water_lambda = 100000.0;
static const double gravity = 10.0;

/* Taichi 1.7.4 _svd2d (polar decomposition + one Jacobi rotation).
 * Returns U (row-major), sig (s1 >= s2 after the swap rule), V (row-major). */
static void FN(svd2)(const REAL A[4], REAL U[4], REAL sig[2], REAL V[4]) {
  /* _polar_decompose2d: x = A00 + A11, y = A10 - A01, R = [[c,-s],[s,c]] */
  REAL x = A[0] + A[3];
  REAL y = A[2] - A[1];
  REAL scale = (REAL)1.0 / (REAL)sqrt(x * x + y * y);
  REAL c = x * scale;
  REAL s = y * scale;
  REAL ms = -s;
  /* S = R^T @ A, R^T = [[c, s], [-s, c]] */
  REAL S00 = c * A[0] + s * A[2];
  REAL S01 = c * A[1] + s * A[3];
  REAL S11 = ms * A[1] + c * A[3];
  REAL cc, ss, s1, s2;
  if ((REAL)fabs(S01) < (REAL)1e-5) {
    cc = (REAL)1; ss = (REAL)0;
    s1 = S00; s2 = S11;
  } else {
    REAL tao = (REAL)0.5 * (S00 - S11);
    REAL w = (REAL)sqrt(tao * tao + S01 * S01);
    REAL t;
    if (tao > (REAL)0) t = S01 / (tao + w);
    else t = S01 / (tao - w);
    cc = (REAL)1 / (REAL)sqrt(t * t + (REAL)1);
    ss = (-t) * cc;
    s1 = (cc * cc * S00 - (REAL)2 * cc * ss * S01) + ss * ss * S11;
    s2 = (ss * ss * S00 + (REAL)2 * cc * ss * S01) + cc * cc * S11;
  }
  REAL V00, V01, V10, V11;
  if (s1 < s2) {
    REAL tmp = s1; s1 = s2; s2 = tmp;
    V00 = -ss; V01 = cc; V10 = -cc; V11 = -ss;
  } else {
    V00 = cc; V01 = ss; V10 = -ss; V11 = cc;
  }
  /* U = R @ V */
  U[0] = c * V00 + ms * V10;
  U[1] = c * V01 + ms * V11;
  U[2] = s * V00 + c * V10;
  U[3] = s * V01 + c * V11;
  V[0] = V00; V[1] = V01; V[2] = V10; V[3] = V11;
  sig[0] = s1; sig[1] = s2;
}

void FN(oracle_svd2)(const REAL* A, REAL* U, REAL* sig, REAL* V) { FN(svd2)(A, U, sig, V); }

/* Per-instance activation of the 2-phase waveform, mpm_sim.py:173-180.
 * Python-semantics float modulo as Taichi lowers it: a - b * floor(a / b).
 * cos is evaluated in double and rounded once. */
REAL FN(oracle_activation)(const oracle_inst* I, REAL t) {
  REAL freq = (REAL)I->freq;
  REAL period = (REAL)1.0 / ((REAL)1 * freq);
  REAL q = (REAL)floor((double)(t / period));
  REAL r = t - period * q;
  REAL phase = r / period;
  REAL c_end = (REAL)I->contraction;
  REAL a = (REAL)0;
  if (phase < c_end) {
    REAL arg = phase / c_end * (REAL)3.14159265;
    a = (REAL)0.5 * ((REAL)1.0 - (REAL)cos((double)arg));
  }
  return a;
}

/* One substep of one instance (mpm_sim.py:153-340). t is sim_time[None]
 * before the step; the caller advances it by (REAL)dt afterwards (:340). */
void FN(oracle_substep)(const oracle_inst* I, int64_t n, REAL* x, REAL* v, REAL* C,
                        REAL* F, const int32_t* mat, REAL* Jp, REAL* glow,
                        const REAL* fiber, const REAL* r_ref, REAL* gv, REAL* gm, REAL t) {
  const int nx = I->nx, ny = I->ny;
  const double dx_d = 1.0 / nx;
  const double inv_dx_d = (double)nx;
  const double dt_d = I->dt;
  const double p_vol_d = (dx_d * 0.5) * (dx_d * 0.5);
  const double p_mass_d = p_vol_d * 1;

  const REAL dx = (REAL)dx_d, inv_dx = (REAL)inv_dx_d, dt = (REAL)dt_d;
  const REAL mu_0 = (REAL)(E_base / (2 * (1 + nu_base)));
  const REAL la_0 = (REAL)(E_base * nu_base / ((1 + nu_base) * (1 - 2 * nu_base)));
  const REAL mu_j = (REAL)(E_jelly / (2 * (1 + nu_jelly)));
  const REAL la_j = (REAL)(E_jelly * nu_jelly / ((1 + nu_jelly) * (1 - 2 * nu_jelly)));
  const REAL mu_p = (REAL)(E_payload / (2 * (1 + nu_payload)));
  const REAL la_p = (REAL)(E_payload * nu_payload / ((1 + nu_payload) * (1 - 2 * nu_payload)));
  const REAL la_w = (REAL)water_lambda;
  const REAL stress_scale = (REAL)(-dt_d * p_vol_d * 4 * inv_dx_d * inv_dx_d);
  const REAL c4 = (REAL)(4 * inv_dx_d);
  const REAL dtg = (REAL)(dt_d * gravity);
  const REAL x_lo = (REAL)0.001, x_hi = (REAL)0.999;
  const REAL y_hi = (REAL)(I->domain_h - 0.001);
  const REAL sig_lo = (REAL)(1 - 5e-3), sig_hi = (REAL)(1 + 5e-3);
  const REAL act = (REAL)I->actuation;
  const REAL pdens = (REAL)I->payload_density;

  const int axisym = I->axisym != 0;
  const REAL rref_lo = (REAL)(dx_d * 0.1), r_lo = (REAL)(dx_d * 0.05);

  /* 1. grid clear (:160-165); the axisymmetric stress sums are scratch here */
  memset(gv, 0, sizeof(REAL) * 2 * (size_t)nx * ny);
  memset(gm, 0, sizeof(REAL) * (size_t)nx * ny);
  uint64_t* gfix = NULL; /* fixed_p2g: momentum x, momentum y, mass per node */
  if (I->fixed_p2g && !axisym) gfix = (uint64_t*)calloc((size_t)3 * nx * ny, sizeof(uint64_t));
  REAL* gsr = NULL;
  REAL* gsh = NULL;
  if (axisym) {
    gsr = (REAL*)calloc((size_t)nx * ny, sizeof(REAL));
    gsh = (REAL*)calloc((size_t)nx * ny, sizeof(REAL));
  }

  const REAL activation = FN(oracle_activation)(I, t);

  /* 2. P2G (:168-271) */
  for (int64_t p = 0; p < n; ++p) {
    const int32_t mt = mat[p];
    if (mt < 0) continue;
    REAL* xp = x + 2 * p;
    REAL* vp = v + 2 * p;
    REAL* Cp = C + 4 * p;
    REAL* Fp = F + 4 * p;
    int bx = (int)(xp[0] * inv_dx - (REAL)0.5);
    int by = (int)(xp[1] * inv_dx - (REAL)0.5);
    if (bx < 0 || by < 0 || bx >= nx - 2 || by >= ny - 2) continue;
    REAL fx0 = xp[0] * inv_dx - (REAL)bx;
    REAL fx1 = xp[1] * inv_dx - (REAL)by;
    REAL a0 = (REAL)1.5 - fx0, a1 = (REAL)1.5 - fx1;
    REAL b0 = fx0 - (REAL)1, b1 = fx1 - (REAL)1;
    REAL e0 = fx0 - (REAL)0.5, e1 = fx1 - (REAL)0.5;
    REAL wx[3] = {(REAL)0.5 * (a0 * a0), (REAL)0.75 - b0 * b0, (REAL)0.5 * (e0 * e0)};
    REAL wy[3] = {(REAL)0.5 * (a1 * a1), (REAL)0.75 - b1 * b1, (REAL)0.5 * (e1 * e1)};

    /* F <- (I + dt C) F (:189) */
    {
      REAL A00 = (REAL)1 + dt * Cp[0], A01 = (REAL)0 + dt * Cp[1];
      REAL A10 = (REAL)0 + dt * Cp[2], A11 = (REAL)1 + dt * Cp[3];
      REAL F00 = A00 * Fp[0] + A01 * Fp[2];
      REAL F01 = A00 * Fp[1] + A01 * Fp[3];
      REAL F10 = A10 * Fp[0] + A11 * Fp[2];
      REAL F11 = A10 * Fp[1] + A11 * Fp[3];
      Fp[0] = F00; Fp[1] = F01; Fp[2] = F10; Fp[3] = F11;
    }

    /* material (:192-203) */
    REAL mu = mu_0, la = la_0;
    REAL mass = (REAL)p_mass_d;
    if (mt == 1 || mt == 3) { mu = mu_j; la = la_j; }
    else if (mt == 2) { mu = mu_p; la = la_p; mass = mass * pdens; }
    else if (mt == 0) { mu = (REAL)0.0; la = la_w; }

    /* SVD and plasticity (:206-223) */
    REAL U[4], sig[2], V[4];
    FN(svd2)(Fp, U, sig, V);
    for (int d = 0; d < 2; ++d) sig[d] = sig[d] > (REAL)1e-6 ? sig[d] : (REAL)1e-6;
    REAL J = (REAL)1.0;
    for (int d = 0; d < 2; ++d) {
      REAL ns = sig[d];
      if (mt == 2) {
        ns = sig[d] > sig_lo ? sig[d] : sig_lo;
        ns = ns < sig_hi ? ns : sig_hi;
      }
      Jp[p] = Jp[p] * (sig[d] / ns);
      sig[d] = ns;
      J = J * ns;
    }
    if (mt == 0) {
      REAL sj = (REAL)sqrt(J);
      Fp[0] = sj; Fp[1] = (REAL)0; Fp[2] = (REAL)0; Fp[3] = sj;
    } else if (mt == 2) {
      REAL US00 = U[0] * sig[0], US01 = U[1] * sig[1];
      REAL US10 = U[2] * sig[0], US11 = U[3] * sig[1];
      Fp[0] = US00 * V[0] + US01 * V[1];
      Fp[1] = US00 * V[2] + US01 * V[3];
      Fp[2] = US10 * V[0] + US11 * V[1];
      Fp[3] = US10 * V[2] + US11 * V[3];
    }

    /* stress (:226-233) */
    REAL R00 = U[0] * V[0] + U[1] * V[1];
    REAL R01 = U[0] * V[2] + U[1] * V[3];
    REAL R10 = U[2] * V[0] + U[3] * V[1];
    REAL R11 = U[2] * V[2] + U[3] * V[3];
    REAL twomu = (REAL)2 * mu;
    REAL E00 = twomu * (Fp[0] - R00), E01 = twomu * (Fp[1] - R01);
    REAL E10 = twomu * (Fp[2] - R10), E11 = twomu * (Fp[3] - R11);
    REAL diag = la * J * (J - (REAL)1);
    REAL s00 = (E00 * Fp[0] + E01 * Fp[1]) + diag;
    REAL s01 = (E00 * Fp[2] + E01 * Fp[3]);
    REAL s10 = (E10 * Fp[0] + E11 * Fp[1]);
    REAL s11 = (E10 * Fp[2] + E11 * Fp[3]) + diag;
    if (mt == 3) {
      REAL cp = act * activation;
      REAL f0 = fiber[2 * p], f1 = fiber[2 * p + 1];
      s00 = s00 + f0 * f0 * cp * J;
      s01 = s01 + f0 * f1 * cp * J;
      s10 = s10 + f1 * f0 * cp * J;
      s11 = s11 + f1 * f1 * cp * J;
    }
    /* axisymmetric hoop terms, before the scaling (:235-248) */
    REAL kirch_rr = (REAL)0, kirch_hoop = (REAL)0, r_p = (REAL)0;
    if (axisym) {
      kirch_rr = s00;
      r_p = xp[0];
      REAL r_ref_p = r_ref[p] > rref_lo ? r_ref[p] : rref_lo;
      REAL lam = (r_p > r_lo ? r_p : r_lo) / r_ref_p;
      kirch_hoop = (REAL)2.0 * mu * (lam - (REAL)1.0) + la * J * (J - (REAL)1.0);
    }
    s00 = stress_scale * s00; s01 = stress_scale * s01;
    s10 = stress_scale * s10; s11 = stress_scale * s11;
    /* APIC affine (:254) */
    REAL af00 = s00 + mass * Cp[0], af01 = s01 + mass * Cp[1];
    REAL af10 = s10 + mass * Cp[2], af11 = s11 + mass * Cp[3];
    REAL mv0 = mass * vp[0], mv1 = mass * vp[1];
    if (axisym) {  /* ring momentum (mass r_p) v (:264) */
      REAL mr = mass * r_p;
      mv0 = mr * vp[0];
      mv1 = mr * vp[1];
    }

    /* scatter (:256-271) */
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) {
        REAL d0 = ((REAL)i - fx0) * dx;
        REAL d1 = ((REAL)j - fx1) * dx;
        REAL weight = wx[i] * wy[j];
        REAL c0 = weight * (mv0 + (af00 * d0 + af01 * d1));
        REAL c1 = weight * (mv1 + (af10 * d0 + af11 * d1));
        size_t node = (size_t)(bx + i) * ny + (size_t)(by + j);
        if (gfix) {
          gfix[3 * node] += FN(to_fixed)(c0);
          gfix[3 * node + 1] += FN(to_fixed)(c1);
          gfix[3 * node + 2] += FN(to_fixed)(weight * mass);
          continue;
        }
        gv[2 * node] = gv[2 * node] + c0;
        gv[2 * node + 1] = gv[2 * node + 1] + c1;
        if (axisym) {  /* :264-268 */
          REAL wm = weight * mass;
          gm[node] = gm[node] + wm * r_p;
          gsr[node] = gsr[node] + wm * kirch_rr;
          gsh[node] = gsh[node] + wm * kirch_hoop;
        } else {
          gm[node] = gm[node] + weight * mass;
        }
      }
    }
  }

  if (gfix) {
    for (size_t node = 0; node < (size_t)nx * ny; ++node) {
      gv[2 * node] = FN(from_fixed)(gfix[3 * node]);
      gv[2 * node + 1] = FN(from_fixed)(gfix[3 * node + 1]);
      gm[node] = FN(from_fixed)(gfix[3 * node + 2]);
    }
    free(gfix);
  }

  /* 3. grid update (:274-309) */
  const int dcx = nx / 20, dcy = ny / 20;
  for (int i = 0; i < nx; ++i) {
    for (int j = 0; j < ny; ++j) {
      size_t node = (size_t)i * ny + j;
      REAL m = gm[node];
      if (!(m > (REAL)0)) continue;
      REAL g0 = gv[2 * node] / m, g1 = gv[2 * node + 1] / m;
      REAL damp = (REAL)1.0;
      if (i < dcx) damp = damp * ((REAL)0.95 + (REAL)0.05 * (REAL)i / (REAL)dcx);
      if (i > nx - dcx) damp = damp * ((REAL)0.95 + (REAL)0.05 * (REAL)(nx - i) / (REAL)dcx);
      if (j < dcy) damp = damp * ((REAL)0.95 + (REAL)0.05 * (REAL)j / (REAL)dcy);
      if (j > ny - dcy) damp = damp * ((REAL)0.95 + (REAL)0.05 * (REAL)(ny - j) / (REAL)dcy);
      g0 = g0 * damp; g1 = g1 * damp;
      if (axisym) {
        /* hoop correction (:295-299), then the axis condition (:302-304) */
        REAL r_node = ((REAL)i + (REAL)0.5) * dx;
        if (r_node > dx) {
          REAL hoop_diff = (gsr[node] - gsh[node]) / m;
          g0 = g0 + dt * hoop_diff / r_node;
        }
        if (i == 0) g0 = (REAL)0;
      } else if (i < 3 && g0 < (REAL)0) {
        g0 = (REAL)0;
      }
      if (i > nx - 3 && g0 > (REAL)0) g0 = (REAL)0;
      if (j < 3 && g1 < (REAL)0) g1 = (REAL)0;
      if (j > ny - 3 && g1 > (REAL)0) g1 = (REAL)0;
      gv[2 * node] = g0; gv[2 * node + 1] = g1;
    }
  }

  /* 4. G2P (:312-333) */
  for (int64_t p = 0; p < n; ++p) {
    if (mat[p] < 0) continue;
    REAL* xp = x + 2 * p;
    REAL* vp = v + 2 * p;
    REAL* Cp = C + 4 * p;
    int bx = (int)(xp[0] * inv_dx - (REAL)0.5);
    int by = (int)(xp[1] * inv_dx - (REAL)0.5);
    if (bx >= 0 && by >= 0 && bx < nx - 2 && by < ny - 2) {
      REAL fx0 = xp[0] * inv_dx - (REAL)bx;
      REAL fx1 = xp[1] * inv_dx - (REAL)by;
      REAL a0 = (REAL)1.5 - fx0, a1 = (REAL)1.5 - fx1;
      REAL b0 = fx0 - (REAL)1.0, b1 = fx1 - (REAL)1.0;
      REAL e0 = fx0 - (REAL)0.5, e1 = fx1 - (REAL)0.5;
      REAL wx[3] = {(REAL)0.5 * (a0 * a0), (REAL)0.75 - b0 * b0, (REAL)0.5 * (e0 * e0)};
      REAL wy[3] = {(REAL)0.5 * (a1 * a1), (REAL)0.75 - b1 * b1, (REAL)0.5 * (e1 * e1)};
      REAL nv0 = 0, nv1 = 0, nC00 = 0, nC01 = 0, nC10 = 0, nC11 = 0;
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
          REAL d0 = (REAL)i - fx0, d1 = (REAL)j - fx1;
          size_t node = (size_t)(bx + i) * ny + (size_t)(by + j);
          REAL g0 = gv[2 * node], g1 = gv[2 * node + 1];
          REAL weight = wx[i] * wy[j];
          nv0 = nv0 + weight * g0;
          nv1 = nv1 + weight * g1;
          REAL k = c4 * weight;
          nC00 = nC00 + k * (g0 * d0);
          nC01 = nC01 + k * (g0 * d1);
          nC10 = nC10 + k * (g1 * d0);
          nC11 = nC11 + k * (g1 * d1);
        }
      }
      vp[0] = nv0; vp[1] = nv1;
      Cp[0] = nC00; Cp[1] = nC01; Cp[2] = nC10; Cp[3] = nC11;
    }
    vp[1] = vp[1] - dtg;
    xp[0] = xp[0] + dt * vp[0];
    xp[1] = xp[1] + dt * vp[1];
    REAL q0 = xp[0] < x_hi ? xp[0] : x_hi;
    xp[0] = q0 > x_lo ? q0 : x_lo;
    REAL q1 = xp[1] < y_hi ? xp[1] : y_hi;
    xp[1] = q1 > x_lo ? q1 : x_lo;
  }

  free(gsr);
  free(gsh);

  /* 5. glow (:336-338), every slot */
  for (int64_t p = 0; p < n; ++p) {
    REAL g = glow[p] * (REAL)0.9;
    REAL d = (REAL)fabs((REAL)1.0 - Jp[p]);
    glow[p] = g > d ? g : d;
  }
}

/* Run `steps` substeps of one instance starting at time *t (advanced in REAL
 * like sim_time[None] += dt, mpm_sim.py:340). */
void FN(oracle_run)(const oracle_inst* I, int64_t n, REAL* x, REAL* v, REAL* C, REAL* F,
                    const int32_t* mat, REAL* Jp, REAL* glow, const REAL* fiber,
                    const REAL* r_ref, REAL* gv, REAL* gm, REAL* t, int64_t steps) {
  const REAL dt = (REAL)I->dt;
  for (int64_t s = 0; s < steps; ++s) {
    FN(oracle_substep)(I, n, x, v, C, F, mat, Jp, glow, fiber, r_ref, gv, gm, *t);
    *t = *t + dt;
  }
}

/* Many independent instances advanced together, parallel over instances with
 * OpenMP (the CPU baseline's batched form).  Instance m's particles start at
 * offsets[m] (in particles), its grid at goffsets[m] (in nodes). Every instance
 * sees the same time sequence. */
void FN(oracle_run_batch)(int32_t M, const oracle_inst* insts, const int64_t* counts,
                          const int64_t* offsets, const int64_t* goffsets, REAL* x, REAL* v,
                          REAL* C, REAL* F, const int32_t* mat, REAL* Jp, REAL* glow,
                          const REAL* fiber, const REAL* r_ref, REAL* gv, REAL* gm, REAL* t,
                          int64_t steps) {
  const REAL t0 = *t;
#pragma omp parallel for schedule(dynamic, 1)
  for (int32_t m = 0; m < M; ++m) {
    REAL tm = t0;
    const int64_t o = offsets[m], g = goffsets[m];
    FN(oracle_run)(&insts[m], counts[m], x + 2 * o, v + 2 * o, C + 4 * o, F + 4 * o, mat + o,
                   Jp + o, glow + o, fiber + 2 * o, r_ref + o, gv + 2 * g, gm + g, &tm, steps);
  }
  REAL tt = t0;
  const REAL dt = M > 0 ? (REAL)insts[0].dt : (REAL)0;
  for (int64_t s = 0; s < steps; ++s) tt = tt + dt;
  *t = tt;
}

/* CoM sums (mpm_sim.py:746-762): mode 0 = payload (material 2), mode 1 =
 * body (materials 1 and 3).  out = [sum_y, count, sum_x], accumulated in
 * double (the GPU engine also accumulates these in FP64). */
void FN(oracle_stats)(int64_t n, const REAL* x, const int32_t* mat, int32_t mode, double* out) {
  double sy = 0, cnt = 0, sx = 0;
  for (int64_t p = 0; p < n; ++p) {
    int32_t mt = mat[p];
    int hit = mode == 0 ? (mt == 2) : (mt == 1 || mt == 3);
    if (hit) { sy += (double)x[2 * p + 1]; cnt += 1.0; sx += (double)x[2 * p]; }
  }
  out[0] = sy; out[1] = cnt; out[2] = sx;
}
