// Batched path: every instance advances in one persistent launch per chunk
// of substeps.  Instance m is owned by one thread-block cluster of CS CTAs;
// CTA r of the cluster owns grid rows [r*H, r*H + H) of that instance and
// keeps them, plus a halo, in shared memory for the whole chunk, so the grid
// never touches HBM.  Particles are counting-sorted by cell between chunks so
// that each CTA streams exactly the particles whose stencils fall in its band.
//
// One pass over a CTA's particles fuses G2P of substep s-1 with P2G of
// substep s (mpm_sim.py:312-333 then :168-271), so each substep reads and
// writes the particle state (x, v, C, F) once.  Between passes the cluster
// exchanges halo rows through distributed shared memory and applies the grid
// update (:274-309) to its owned rows.  Particles that drifted beyond the
// halo since the last sort reach their rows' owners through DSMEM, so the
// result does not depend on the re-sort interval.
#include <cooperative_groups.h>

#include <utility>

#include "jf_engine.h"

namespace cg = cooperative_groups;

namespace {

constexpr int kHaloLo = 1;  // window rows below the band (drift of one row)
constexpr int kHaloHi = 3;  // rows above: the stencil's +2 plus one row of drift
constexpr int kHalo = kHaloLo + kHaloHi;
constexpr int kSortThreads = 256;
constexpr int kScanThreads = 1024;

struct ChunkArgs {
  const JfInst* inst;
  const JfParams* params;
  JfMaterials mats;
  float4* xv;
  float4* C;
  float4* F;
  const int32_t* mat;
  float* Jp;
  const float2* fiber;
  float* glow;
  const int32_t* band;   // M x (CS + 1) engine positions
  float4* grid;          // grid of the chunk's last substep, node = g_off + j * nx + i
  int32_t* err;
  int32_t M;
  int32_t CS;
  int32_t K;             // substeps in this chunk
  float t0;
  float dt;
  int32_t do_glow;
};

__global__ void __launch_bounds__(512, 1) chunk_kernel(ChunkArgs a) {
  extern __shared__ float4 smem4[];
  float* sm = reinterpret_cast<float*>(smem4);
  __shared__ float s_pressure;

  cg::cluster_group cluster = cg::this_cluster();
  const int CS = a.CS;
  const int r = (int)cluster.block_rank();
  const int m = blockIdx.x / CS;
  if (m >= a.M) return;  // a padding cluster leaves as a whole

  const JfInst I = a.inst[m];
  const JfParams P = a.params[m];
  const JfMaterials mats = a.mats;  // a register copy: no address taken in parameter space
  const int nx = I.nx, ny = I.ny, H = I.band_h;
  const int row0 = r * H;
  const int own_hi = min(row0 + H, ny);
  const int win0 = row0 - kHaloLo;
  const int WR = H + kHalo;
  const int WN = WR * nx;
  float* Gx = sm;
  float* Gy = Gx + WN;
  float* Ax = Gy + WN;
  float* Ay = Ax + WN;
  float* Am = Ay + WN;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int lo = a.band[m * (CS + 1) + r];
  const int hi = a.band[m * (CS + 1) + r + 1];

  for (int n = tid; n < 5 * WN; n += nth) sm[n] = 0.0f;
  cluster.sync();

  // window position of grid row j in the CTA that owns it
  auto owner_of = [&](int j) { return j / H; };
  auto owner_row = [&](int j, int o) { return j - (o * H - kHaloLo); };

  auto gather = [&](int ni, int nj) -> float2 {
    const int wr = nj - win0;
    if (wr >= 0 && wr < WR) {
      const int n = wr * nx + ni;
      return make_float2(Gx[n], Gy[n]);
    }
    const int o = owner_of(nj);
    const int n = owner_row(nj, o) * nx + ni;
    const float* rx = cluster.map_shared_rank(Gx, o);
    const float* ry = cluster.map_shared_rank(Gy, o);
    return make_float2(rx[n], ry[n]);
  };

  float t = a.t0;
  for (int s = 0; s <= a.K; ++s) {
    const bool do_g2p = s > 0;
    const bool do_p2g = s < a.K;
    if (tid == 0) s_pressure = P.actuation * jf_activation(P.freq, P.contraction, t);
    __syncthreads();
    const float pressure = s_pressure;

    for (int k = lo + tid; k < hi; k += nth) {
      const float4 xv = a.xv[k];
      float4 C = a.C[k];
      const int mt = a.mat[k];
      float2 x = make_float2(xv.x, xv.y), v = make_float2(xv.z, xv.w);
      float jp = 1.0f;
      if (mt == 2 || a.do_glow) jp = a.Jp[k];
      if (do_g2p) {
        jf_g2p_particle(I, x, v, C, gather);
        if (a.do_glow) a.glow[k] = jf_glow(a.glow[k], jp);
        if (!(isfinite(x.x) && isfinite(x.y) && isfinite(v.x) && isfinite(v.y))) atomicOr(a.err + m, 1);
      }
      if (do_p2g) {
        JfStencil st;
        if (jf_stencil(I, x, st)) {
          float4 F = a.F[k];
          const float2 fb = (mt == 3) ? a.fiber[k] : make_float2(0.0f, 1.0f);
          JfScatter sc;
          jf_p2g_particle(I, mats, mt, v, C, F, jp, fb, pressure, P.payload_density, sc);
          a.F[k] = F;
          if (mt == 2) a.Jp[k] = jp;
          const int wr0 = st.by - win0;
          if (wr0 >= 0 && wr0 + 2 < WR) {
            const int base = wr0 * nx + st.bx;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
#pragma unroll
              for (int i = 0; i < 3; ++i) {
                const float3 c = jf_node_contrib(I, st, sc, i, j);
                const int n = base + j * nx + i;
                atomicAdd(Ax + n, c.x);
                atomicAdd(Ay + n, c.y);
                atomicAdd(Am + n, c.z);
              }
            }
          } else {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              const int row = st.by + j;
              const int wr = row - win0;
              float *px, *py, *pm;
              int rn;
              if (wr >= 0 && wr < WR) {
                px = Ax; py = Ay; pm = Am;
                rn = wr * nx;
              } else {
                const int o = owner_of(row);
                px = cluster.map_shared_rank(Ax, o);
                py = cluster.map_shared_rank(Ay, o);
                pm = cluster.map_shared_rank(Am, o);
                rn = owner_row(row, o) * nx;
              }
#pragma unroll
              for (int i = 0; i < 3; ++i) {
                const float3 c = jf_node_contrib(I, st, sc, i, j);
                atomicAdd(px + rn + st.bx + i, c.x);
                atomicAdd(py + rn + st.bx + i, c.y);
                atomicAdd(pm + rn + st.bx + i, c.z);
              }
            }
          }
        }
      }
      if (do_g2p) {
        a.xv[k] = make_float4(x.x, x.y, v.x, v.y);
        a.C[k] = C;
      }
    }
    __syncthreads();

    if (do_p2g) {
      // halo rows of the accumulator go to the rows' owners
      for (int n = tid; n < WN; n += nth) {
        const int wr = n / nx;
        const int j = win0 + wr;
        if ((j >= row0 && j < own_hi) || j < 0 || j >= ny) continue;
        const float vx = Ax[n], vy = Ay[n], vm = Am[n];
        if (vx != 0.0f || vy != 0.0f || vm != 0.0f) {
          const int o = owner_of(j);
          const int rn = owner_row(j, o) * nx + (n - wr * nx);
          atomicAdd(cluster.map_shared_rank(Ax, o) + rn, vx);
          atomicAdd(cluster.map_shared_rank(Ay, o) + rn, vy);
          atomicAdd(cluster.map_shared_rank(Am, o) + rn, vm);
          Ax[n] = 0.0f;
          Ay[n] = 0.0f;
          Am[n] = 0.0f;
        }
      }
      cluster.sync();

      // grid update of the owned rows; the accumulator is cleared for the next pass
      const bool last = (s == a.K - 1);
      const int n_end = (kHaloLo + own_hi - row0) * nx;
      for (int n = kHaloLo * nx + tid; n < n_end; n += nth) {
        const int wr = n / nx;
        const int i = n - wr * nx;
        const int j = win0 + wr;
        const float mm = Am[n];
        const float2 u = jf_grid_node(I, i, j, Ax[n], Ay[n], mm);
        Gx[n] = u.x;
        Gy[n] = u.y;
        if (last) a.grid[I.g_off + (int64_t)j * nx + i] = make_float4(u.x, u.y, mm, 0.0f);
        Ax[n] = 0.0f;
        Ay[n] = 0.0f;
        Am[n] = 0.0f;
      }
      cluster.sync();

      // halo rows of the updated grid come from their owners
      for (int n = tid; n < WN; n += nth) {
        const int wr = n / nx;
        const int j = win0 + wr;
        if ((j >= row0 && j < own_hi) || j < 0 || j >= ny) continue;
        const int o = owner_of(j);
        const int rn = owner_row(j, o) * nx + (n - wr * nx);
        Gx[n] = cluster.map_shared_rank(Gx, o)[rn];
        Gy[n] = cluster.map_shared_rank(Gy, o)[rn];
      }
      __syncthreads();
      t = t + a.dt;
    }
  }
  // peers may still read this CTA's grid rows in their last G2P pass
  cluster.sync();
}

// Cell key of every particle: row-major cell index, then one bin for live
// particles outside the stencil range and one for dead slots.
__global__ void sort_keys_kernel(const JfInst* __restrict__ inst, const float4* __restrict__ xv,
                                 const int32_t* __restrict__ mat, int32_t* __restrict__ keys,
                                 int32_t* __restrict__ counts, int stride) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const int cells = I.nx * I.ny;
  int key;
  if (mat[g] < 0) {
    key = cells + 1;
  } else {
    const float4 a = xv[g];
    JfStencil st;
    key = jf_stencil(I, make_float2(a.x, a.y), st) ? st.by * I.nx + st.bx : cells;
  }
  keys[g] = key;
  atomicAdd(counts + (int64_t)m * stride + key, 1);
}

// Exclusive scan of one instance's bins (counts become start cursors) and the
// CTA band table: CTA r streams [band[r], band[r+1]); the last CTA also takes
// the out-of-range bin.
__global__ void __launch_bounds__(kScanThreads) sort_scan_kernel(const JfInst* __restrict__ inst,
                                                                int32_t* __restrict__ counts,
                                                                int stride, int32_t* __restrict__ band,
                                                                int CS) {
  __shared__ int warp_sums[kScanThreads / 32];
  const int m = blockIdx.x;
  const JfInst I = inst[m];
  const int cells = I.nx * I.ny;
  const int nbins = cells + 2;
  int32_t* c = counts + (int64_t)m * stride;
  const int per = (nbins + kScanThreads - 1) / kScanThreads;
  const int b0 = threadIdx.x * per;
  const int b1 = min(b0 + per, nbins);
  int local = 0;
  for (int b = b0; b < b1; ++b) local += c[b];
  // block exclusive scan of `local`
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = local;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += y;
  }
  if (lane == 31) warp_sums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int w = (lane < kScanThreads / 32) ? warp_sums[lane] : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += y;
    }
    if (lane < kScanThreads / 32) warp_sums[lane] = w;
  }
  __syncthreads();
  int run = (incl - local) + (wid > 0 ? warp_sums[wid - 1] : 0);
  for (int b = b0; b < b1; ++b) {
    const int cnt = c[b];
    c[b] = run;
    run += cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int H = I.band_h;
    for (int r = 0; r < CS; ++r) {
      const int row = min(r * H, I.ny);
      band[m * (CS + 1) + r] = (int32_t)I.p_off + c[row * I.nx];
    }
    band[m * (CS + 1) + CS] = (int32_t)I.p_off + c[cells + 1];
  }
}

__global__ void sort_scatter_kernel(const JfInst* __restrict__ inst, const int32_t* __restrict__ keys,
                                    int32_t* __restrict__ counts, int stride, JfParticles src,
                                    JfParticles dst) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const int key = keys[g];
  const int64_t d = I.p_off + atomicAdd(counts + (int64_t)m * stride + key, 1);
  dst.xv[d] = src.xv[g];
  dst.C[d] = src.C[g];
  dst.F[d] = src.F[g];
  dst.mat[d] = src.mat[g];
  dst.fiber[d] = src.fiber[g];
  dst.Jp[d] = src.Jp[g];
  dst.glow[d] = src.glow[g];
  dst.slot[d] = src.slot[g];
}

// Dead slots are not streamed by the chunk kernel; their render-only glow
// still decays once per substep (mpm_sim.py:336-338).
__global__ void dead_glow_kernel(const JfInst* __restrict__ inst, const int32_t* __restrict__ band,
                                 int CS, const int32_t* __restrict__ mat, const float* __restrict__ Jp,
                                 float* __restrict__ glow, int K) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int64_t end = I.p_off + I.n_slots;
  for (int64_t g = band[m * (CS + 1) + CS] + blockIdx.x * blockDim.x + threadIdx.x; g < end;
       g += (int64_t)gridDim.x * blockDim.x) {
    float gl = glow[g];
    const float jp = Jp[g];
    for (int s = 0; s < K; ++s) gl = jf_glow(gl, jp);
    glow[g] = gl;
  }
}

}  // namespace

size_t jf_batched_smem_bytes(const jf_engine* e) {
  return sizeof(float) * 5 * (size_t)e->win_nodes;
}

cudaError_t jf_batched_sort(jf_engine* e) {
  JfTimed timed(e, true);
  const int stride = e->max_cells + 2;
  cudaError_t err = cudaMemsetAsync(e->d_counts, 0, sizeof(int32_t) * (size_t)stride * e->M, e->stream);
  if (err != cudaSuccess) return err;
  const dim3 grid((e->max_slots + kSortThreads - 1) / kSortThreads, e->M);
  if (e->max_slots > 0) {
    sort_keys_kernel<<<grid, kSortThreads, 0, e->stream>>>(e->d_inst, e->p.xv, e->p.mat, e->d_keys,
                                                          e->d_counts, stride);
  }
  sort_scan_kernel<<<e->M, kScanThreads, 0, e->stream>>>(e->d_inst, e->d_counts, stride, e->d_band,
                                                         e->cluster);
  if (e->max_slots > 0) {
    sort_scatter_kernel<<<grid, kSortThreads, 0, e->stream>>>(e->d_inst, e->d_keys, e->d_counts, stride,
                                                             e->p, e->q);
  }
  e->launches += (e->max_slots > 0) ? 3 : 1;
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  std::swap(e->p, e->q);
  e->sorted = true;
  return cudaSuccess;
}

static cudaError_t launch_chunk(jf_engine* e, int K) {
  ChunkArgs a;
  a.inst = e->d_inst;
  a.params = e->d_params;
  a.mats = jf_materials();
  a.xv = e->p.xv;
  a.C = e->p.C;
  a.F = e->p.F;
  a.mat = e->p.mat;
  a.Jp = e->p.Jp;
  a.fiber = e->p.fiber;
  a.glow = e->p.glow;
  a.band = e->d_band;
  a.grid = e->d_grid;
  a.err = e->d_err;
  a.M = e->M;
  a.CS = e->cluster;
  a.K = K;
  a.t0 = e->t;
  a.dt = (float)e->dt;
  a.do_glow = (e->flags & JF_FLAG_GLOW) ? 1 : 0;

  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(e->M * e->cluster, 1, 1);
  cfg.blockDim = dim3(e->block_threads, 1, 1);
  cfg.dynamicSmemBytes = jf_batched_smem_bytes(e);
  cfg.stream = e->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = e->cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t err;
  {
    JfTimed timed(e, false);
    err = cudaLaunchKernelEx(&cfg, chunk_kernel, a);
  }
  e->launches += 1;
  if (err != cudaSuccess) return err;
  if (a.do_glow) {
    dead_glow_kernel<<<dim3(16, e->M), 256, 0, e->stream>>>(e->d_inst, e->d_band, e->cluster, e->p.mat,
                                                           e->p.Jp, e->p.glow, K);
    e->launches += 1;
  }
  return cudaGetLastError();
}

cudaError_t jf_batched_prepare(jf_engine* e) {
  const size_t smem = jf_batched_smem_bytes(e);
  cudaError_t err = cudaFuncSetAttribute(chunk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
  if (err != cudaSuccess) return err;
  if (e->cluster > 8) {
    err = cudaFuncSetAttribute(chunk_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

int jf_batched_max_active_clusters(jf_engine* e, int cluster, int* out) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster * 8, 1, 1);
  cfg.blockDim = dim3(e->block_threads, 1, 1);
  cfg.dynamicSmemBytes = jf_batched_smem_bytes(e);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return (int)cudaOccupancyMaxActiveClusters(out, chunk_kernel, &cfg);
}

cudaError_t jf_batched_step(jf_engine* e, int64_t n_steps) {
  const float dtf = (float)e->dt;
  while (n_steps > 0) {
    if (!e->sorted) {
      cudaError_t err = jf_batched_sort(e);
      if (err != cudaSuccess) return err;
    }
    const int K = (int)(n_steps < e->resort_interval ? n_steps : e->resort_interval);
    cudaError_t err = launch_chunk(e, K);
    if (err != cudaSuccess) return err;
    for (int s = 0; s < K; ++s) e->t = e->t + dtf;
    n_steps -= K;
    e->sorted = false;  // particles moved: re-sort before the next chunk
  }
  return cudaSuccess;
}
