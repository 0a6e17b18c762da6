// Plain path: one instance per launch sequence, structured like the
// reference's substep() offloads (mpm_sim.py:160-340): grid clear, P2G with
// global atomics, grid update, G2P.  Also the CoM reduction and the
// load / glow-reorder kernels shared with the batched path.
#include "jf_engine.h"

namespace {

constexpr int kThreads = 256;

JfMaterials host_materials() {
  // mpm_sim.py:25-48, Python doubles rounded once.
  const double E_base = 0.1e4, nu_base = 0.2, E_jelly = 0.7e3, nu_jelly = 0.3;
  const double E_pay = 2.0e5, nu_pay = 0.2, water_lambda = 100000.0;
  const float mu0 = (float)(E_base / (2 * (1 + nu_base)));
  const float la0 = (float)(E_base * nu_base / ((1 + nu_base) * (1 - 2 * nu_base)));
  const float muj = (float)(E_jelly / (2 * (1 + nu_jelly)));
  const float laj = (float)(E_jelly * nu_jelly / ((1 + nu_jelly) * (1 - 2 * nu_jelly)));
  const float mup = (float)(E_pay / (2 * (1 + nu_pay)));
  const float lap = (float)(E_pay * nu_pay / ((1 + nu_pay) * (1 - 2 * nu_pay)));
  JfMaterials m;
  m.mu[0] = 0.0f; m.la[0] = (float)water_lambda;  // water
  m.mu[1] = muj;  m.la[1] = laj;                  // jelly
  m.mu[2] = mup;  m.la[2] = lap;                  // payload
  m.mu[3] = muj;  m.la[3] = laj;                  // muscle
  m.mu[4] = mu0;  m.la[4] = la0;                  // any other id
  return m;
}

__global__ void plain_p2g(JfInst I, JfMaterials mats, JfParams P, float pressure,
                          const float4* __restrict__ xv, const float4* __restrict__ Cm,
                          float4* __restrict__ Fm, const int32_t* __restrict__ mat,
                          float* __restrict__ Jp, const float2* __restrict__ fiber,
                          const float* __restrict__ rref, float4* __restrict__ grid) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const int mt = mat[g];
  if (mt < 0) return;
  const float4 a = xv[g];
  const float2 x = make_float2(a.x, a.y), v = make_float2(a.z, a.w);
  JfStencil st;
  if (!jf_stencil(I, x, st)) return;
  float4 F = Fm[g];
  const float4 C = Cm[g];
  float jp = (mt == 2) ? Jp[g] : 1.0f;
  const float2 fb = (mt == 3) ? fiber[g] : make_float2(0.0f, 1.0f);
  JfScatter sc;
  jf_p2g_particle(I, mats, mt, v, C, F, jp, fb, pressure, P.payload_density, sc, x.x,
                  I.axisym ? rref[g] : 1.0f);
  Fm[g] = F;
  if (mt == 2) Jp[g] = jp;
  float4* gi = grid + I.g_off;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float3 c = jf_node_contrib(I, st, sc, i, j);
      const float hw = jf_w(st, 0, i) * jf_w(st, 1, j) * sc.hoop;  // axisymmetric hoop channel
      atomicAdd(gi + (int64_t)(st.by + j) * I.nx + (st.bx + i), make_float4(c.x, c.y, c.z, hw));
    }
  }
}

__global__ void plain_grid(JfInst I, float4* __restrict__ grid) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= I.nx * I.ny) return;
  const int i = n % I.nx, j = n / I.nx;
  const float4 g = grid[I.g_off + n];
  const float2 u = jf_grid_node(I, i, j, g.x, g.y, g.z, g.w);
  grid[I.g_off + n] = make_float4(u.x, u.y, g.z, 0.0f);
}

__global__ void plain_g2p(JfInst I, int m, float4* __restrict__ xv, float4* __restrict__ Cm,
                          const int32_t* __restrict__ mat, const float* __restrict__ Jp,
                          float* __restrict__ glow, const float4* __restrict__ grid,
                          int32_t* __restrict__ err, int do_glow) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  if (do_glow) glow[g] = jf_glow(glow[g], Jp[g]);
  if (mat[g] < 0) return;
  const float4 a = xv[g];
  float2 x = make_float2(a.x, a.y), v = make_float2(a.z, a.w);
  float4 C = Cm[g];
  const float4* gi = grid + I.g_off;
  const int nx = I.nx;
  jf_g2p_particle(I, x, v, C, [&](int ni, int nj) {
    const float4 q = gi[(int64_t)nj * nx + ni];
    return make_float2(q.x, q.y);
  });
  if (!(isfinite(x.x) && isfinite(x.y) && isfinite(v.x) && isfinite(v.y))) atomicOr(err + m, 1);
  xv[g] = make_float4(x.x, x.y, v.x, v.y);
  Cm[g] = C;
}

__global__ void stats_kernel(const JfInst* __restrict__ inst, const float4* __restrict__ xv,
                             const int32_t* __restrict__ mat, double* __restrict__ out) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  double py = 0, pc = 0, px = 0, by = 0, bc = 0, bx = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < I.n_slots; k += gridDim.x * blockDim.x) {
    const int64_t g = I.p_off + k;
    const int mt = mat[g];
    if (mt == 2) {
      const float4 a = xv[g];
      py += (double)a.y; pc += 1.0; px += (double)a.x;
    } else if (mt == 1 || mt == 3) {
      const float4 a = xv[g];
      by += (double)a.y; bc += 1.0; bx += (double)a.x;
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

// Reset one instance from staged host arrays (mpm_sim.py:715-727).
__global__ void load_kernel(JfInst I, int32_t n, const float* __restrict__ pos,
                            const int32_t* __restrict__ mt_in, const float* __restrict__ fib,
                            int has_fiber, JfParticles p, const float* __restrict__ glow_slot) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  float2 x = make_float2(-1.0f, -1.0f);
  int mt = -1;
  float2 fb = make_float2(0.0f, 1.0f);
  if (k < n) {
    x = make_float2(pos[2 * k], pos[2 * k + 1]);
    mt = mt_in[k];
    if (has_fiber) fb = make_float2(fib[2 * k], fib[2 * k + 1]);
  }
  p.xv[g] = make_float4(x.x, x.y, 0.0f, 0.0f);
  p.C[g] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  p.F[g] = make_float4(1.0f, 0.0f, 0.0f, 1.0f);
  p.mat[g] = mt;
  p.fiber[g] = fb;
  p.Jp[g] = 1.0f;
  p.glow[g] = glow_slot[k];
  p.slot[g] = k;
  p.rref[g] = x.x;  // mpm_sim.py:727
}

// Every instance at once (blockIdx.y = instance) from slot-ordered staging
// laid out as the engine's slots: the same reset as load_kernel.
__global__ void load_all_kernel(const JfInst* __restrict__ inst, const float* __restrict__ pos,
                                const int32_t* __restrict__ mt_in, const float* __restrict__ fib,
                                int has_fiber, JfParticles p, const float* __restrict__ glow_slot) {
  const JfInst I = inst[blockIdx.y];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const int mt = mt_in[g];
  const float2 x = make_float2(pos[2 * g], pos[2 * g + 1]);
  p.xv[g] = make_float4(x.x, x.y, 0.0f, 0.0f);
  p.C[g] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  p.F[g] = make_float4(1.0f, 0.0f, 0.0f, 1.0f);
  p.mat[g] = mt;
  p.fiber[g] = has_fiber ? make_float2(fib[2 * g], fib[2 * g + 1]) : make_float2(0.0f, 1.0f);
  p.Jp[g] = 1.0f;
  p.glow[g] = glow_slot[g];
  p.slot[g] = k;
  p.rref[g] = x.x;  // mpm_sim.py:727
}

// glow of every instance into slot order (blockIdx.y = instance)
__global__ void glow_all_to_slot_kernel(const JfInst* __restrict__ inst, const float* __restrict__ glow,
                                        const int32_t* __restrict__ slot, float* __restrict__ out) {
  const JfInst I = inst[blockIdx.y];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  out[I.p_off + slot[g]] = glow[g];
}

// run_batch_headless rows (mpm_sim.py:776-834) from the CoM sums before and
// after: the payload CoM, or the jelly + muscle CoM without payload;
// [init_y, init_x, final_y, final_x, final_y >= 0.01], zeros without either.
__global__ void rows_kernel(int M, const double* __restrict__ before, const double* __restrict__ after,
                            double* __restrict__ rows) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  const double* a = before + 6 * (size_t)m;
  const double* b = after + 6 * (size_t)m;
  if (a[1] == 0) a += 3;
  if (b[1] == 0) b += 3;
  double* o = rows + 5 * (size_t)m;
  o[0] = o[1] = o[2] = o[3] = o[4] = 0.0;
  if (a[1] > 0 && b[1] > 0) {
    o[0] = a[0] / a[1];
    o[1] = a[2] / a[1];
    o[2] = b[0] / b[1];
    o[3] = b[2] / b[1];
    o[4] = (o[2] < 0.01) ? 0.0 : 1.0;
  }
}

__global__ void glow_to_slot_kernel(JfInst I, const float* __restrict__ glow,
                                    const int32_t* __restrict__ slot, float* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  out[slot[g]] = glow[g];
}

// Fitness of every instance (evolve.py:90-124) in FP64: one block, the
// penalty for invalid instances is the block maximum of the valid scores + 1.
__global__ void fitness_kernel(const JfInst* __restrict__ inst, int M, const double* __restrict__ rows,
                               const int32_t* __restrict__ muscle, const double* __restrict__ contraction,
                               int has_contraction, int mode, double* __restrict__ out) {
  __shared__ double s_max[32];
  __shared__ int s_any[32];
  double best = -INFINITY;
  int any = 0;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    const double* r = rows + 5 * (size_t)m;
    const double valid = r[4];
    double score = NAN;
    if (!(valid == 0.0 || muscle[m] < 200)) {
      const double cap = inst[m].domain_h - 0.07;
      const double disp = (r[2] < cap ? r[2] : cap) - r[0];
      if (mode == 1) {
        score = -disp;
      } else {
        double frac = has_contraction ? contraction[m] : 0.20;
        frac = frac < 0.05 ? 0.05 : (frac > 0.60 ? 0.60 : frac);
        const double cost = sqrt((double)muscle[m] * frac / 500.0);
        score = -disp / cost;
      }
      best = score > best ? score : best;
      any = 1;
    }
    out[m] = score;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    best = fmax(best, __shfl_down_sync(0xffffffffu, best, off));
    any |= __shfl_down_sync(0xffffffffu, any, off);
  }
  if ((threadIdx.x & 31) == 0) {
    s_max[threadIdx.x >> 5] = best;
    s_any[threadIdx.x >> 5] = any;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = -INFINITY;
    int a = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      b = s_max[w] > b ? s_max[w] : b;
      a |= s_any[w];
    }
    s_max[0] = a ? b + 1.0 : 100.0;
  }
  __syncthreads();
  const double penalty = s_max[0];
  for (int m = threadIdx.x; m < M; m += blockDim.x)
    if (isnan(out[m])) out[m] = penalty;
}

inline int blocks_for(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

}  // namespace

JfMaterials jf_materials() { return host_materials(); }

cudaError_t jf_plain_step(jf_engine* e, int64_t n_steps) {
  const JfMaterials mats = host_materials();
  const float dtf = (float)e->dt;
  const int do_glow = (e->flags & JF_FLAG_GLOW) ? 1 : 0;
  float t_end = e->t;
  for (int m = 0; m < e->M; ++m) {
    const JfInst& I = e->inst[m];
    const JfParams P = e->params[m];
    const int nodes = I.nx * I.ny;
    float t = e->t;
    for (int64_t s = 0; s < n_steps; ++s) {
      const float pressure = P.actuation * jf_activation(P.freq, P.contraction, t);
      JfTimed timed(e, false);
      cudaError_t err = cudaMemsetAsync(e->d_grid + I.g_off, 0, sizeof(float4) * nodes, e->stream);
      if (err != cudaSuccess) return err;
      if (I.n_slots > 0) {
        plain_p2g<<<blocks_for(I.n_slots), kThreads, 0, e->stream>>>(
            I, mats, P, pressure, e->p.xv, e->p.C, e->p.F, e->p.mat, e->p.Jp, e->p.fiber, e->p.rref,
            e->d_grid);
      }
      plain_grid<<<blocks_for(nodes), kThreads, 0, e->stream>>>(I, e->d_grid);
      if (I.n_slots > 0) {
        plain_g2p<<<blocks_for(I.n_slots), kThreads, 0, e->stream>>>(
            I, m, e->p.xv, e->p.C, e->p.mat, e->p.Jp, e->p.glow, e->d_grid, e->d_err, do_glow);
      }
      e->launches += (I.n_slots > 0) ? 3 : 1;
      t = t + dtf;
    }
    t_end = t;
  }
  e->t = t_end;
  return cudaGetLastError();
}

cudaError_t jf_stats_launch(jf_engine* e) {
  cudaError_t err = cudaMemsetAsync(e->d_stats, 0, sizeof(double) * 6 * e->M, e->stream);
  if (err != cudaSuccess) return err;
  int blocks = blocks_for(e->max_slots);
  if (blocks > 64) blocks = 64;
  if (blocks < 1) blocks = 1;
  stats_kernel<<<dim3(blocks, e->M), kThreads, 0, e->stream>>>(e->d_inst, e->p.xv, e->p.mat,
                                                                 e->d_stats);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_fitness_launch(jf_engine* e, const double* d_rows, const int32_t* d_muscle,
                              const double* d_contraction, int mode, double* d_out) {
  fitness_kernel<<<1, 1024, 0, e->stream>>>(e->d_inst, e->M, d_rows, d_muscle, d_contraction,
                                            d_contraction != nullptr, mode, d_out);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_load_all_launch(jf_engine* e, const float* d_pos, const int32_t* d_mat, const float* d_fib,
                               float* d_glow_slot) {
  if (e->max_slots == 0) return cudaSuccess;
  const dim3 grid(blocks_for(e->max_slots), e->M);
  glow_all_to_slot_kernel<<<grid, kThreads, 0, e->stream>>>(e->d_inst, e->p.glow, e->p.slot, d_glow_slot);
  load_all_kernel<<<grid, kThreads, 0, e->stream>>>(e->d_inst, d_pos, d_mat, d_fib, d_fib != nullptr, e->p,
                                                    d_glow_slot);
  e->launches += 2;
  return cudaGetLastError();
}

cudaError_t jf_rows_launch(jf_engine* e, const double* d_before, const double* d_after, double* d_rows) {
  rows_kernel<<<(e->M + 127) / 128, 128, 0, e->stream>>>(e->M, d_before, d_after, d_rows);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_glow_to_slot_order(jf_engine* e, int m) {
  const JfInst& I = e->inst[m];
  if (I.n_slots == 0) return cudaSuccess;
  glow_to_slot_kernel<<<blocks_for(I.n_slots), kThreads, 0, e->stream>>>(
      I, e->p.glow, e->p.slot, e->d_stage + 4 * (int64_t)e->max_slots);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_load_launch(jf_engine* e, int m, int32_t n) {
  // staging layout: d_stage[0 .. 2S) pos, [2S .. 4S) fibre, [4S .. 5S) glow in slot
  // order; d_stage_i[0 .. S) material.
  const JfInst& I = e->inst[m];
  if (I.n_slots == 0) return cudaSuccess;
  const int64_t S = e->max_slots;
  load_kernel<<<blocks_for(I.n_slots), kThreads, 0, e->stream>>>(
      I, n, e->d_stage, e->d_stage_i, e->d_stage + 2 * S, 1, e->p, e->d_stage + 4 * S);
  e->launches += 1;
  return cudaGetLastError();
}
