// Batched path: every instance advances in one persistent launch per chunk
// of substeps.  Instance m is owned by one thread-block cluster of CS CTAs
// (clusters take instances in descending live count); CTA r of the cluster
// owns a band of grid rows of that instance — the bands are cut at each
// re-sort so that the CTAs carry equal work — and keeps them, plus a halo, in
// shared memory for the whole chunk, so the grid never touches HBM.
// Particles are counting-sorted by cell between chunks so that each CTA
// streams exactly the particles whose stencils fall in its band; a cell keeps
// at most a per-instance cap of particles for its lane, the rest go to the
// band's overflow list.
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
// Per-lane cap of a cell's particles: a warp's cell loop runs as many
// iterations as its fullest cell, so the particles a cell holds beyond the
// cap are listed per band at the re-sort and handled 32 at a time, one per
// lane with per-particle atomics, as extra tasks of the band's task queue.
// The cap is chosen per instance at each re-sort by the cost model
// 32 * sum_warps min(max count, cap) + 1.5 * overflow (lane-iterations), over
// caps 1 .. kCapCandidates - 1 and "no cap".
constexpr int kCapCandidates = 16;
constexpr int kMaxCluster = 16;
// Band boundaries follow the particles: at each re-sort the rows are split
// into CS bands of about equal cost (cell-loop iterations at the chosen cap,
// overflow, grid update), each at most band_cap rows (the shared-memory
// window's capacity).  Grids taller than kMaxBandRows keep equal-height bands.
constexpr int kMaxBandRows = kJfMaxBandRows;
constexpr int kRowCost = 40;  // grid update of one row, in the cost model's units
// A non-water particle takes the full SVD and stress path, which the whole
// warp of its cell segment then executes; robot cells are mostly full of
// such particles, so the extra cost spread over them is small: 1.5 units per
// particle (in half units here; measured best among 1 / 1.5 / 2 / 3 / 4 / 8,
// 2.3 % on the 32-instance batch against no weight).
constexpr int kSolidCostHalves = 3;
constexpr int kNoCap = 1 << 30;
// CTA size of the TMEM variant of the chunk kernel (24 warps per SM)
constexpr int kTmemThreads = 768;

// Sort cell of a particle: (floor(X - 1/4), floor(Y - 1/4)) in grid units,
// clamped at 0.  The stencil base trunc(X - 1/2) of a particle in sort cell k
// is k - 1 or k, so a lane that owns cell k accumulates a 4x4 node block.
// The reference's water lattice (spacing dx/2) puts half its lines exactly on
// X - 1/2 in Z, where the base flips with any motion; the quarter shift keeps
// every lattice point a quarter cell away from a sort-cell edge.
__device__ __forceinline__ int2 sort_cell(const JfInst& I, float2 x) {
  const int kx = max((int)floorf(x.x * I.inv_dx - 0.25f), 0);
  const int ky = max((int)floorf(x.y * I.inv_dx - 0.25f), 0);
  return make_int2(kx, ky);
}

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
  const float* rref;          // load radius (axisymmetric variant)
  const int32_t* cell_start;  // M x stride: start of each bin's run (relative to p_off)
  const int32_t* cap;         // M: particles a cell lane takes; the rest are overflow
  const int32_t* ovlist;      // overflow positions (relative to p_off), grouped by band
  const int32_t* ovband;      // M x (CS + 1): band starts in ovlist
  const int32_t* order;       // cluster -> instance
  const int32_t* brow;        // M x (CS + 1): band row starts
  int32_t stride;
  float4* grid;             // grid of the chunk's last substep, node = g_off + j * nx + i
  int32_t* err;
  int32_t M;
  int32_t CS;
  int32_t K;                // substeps in this chunk
  const float* t_dev;       // sim_time at the chunk's start (device scalar)
  float dt;
  int32_t do_glow;
  unsigned long long* path;  // [register scatters, generic scatters, generic gathers, overflow]
};

// Shared-memory window of one CTA: grid rows [win0, win0 + WR) of its
// instance: the updated velocity G as float2 pairs (one 64-bit load per node
// in G2P), then planar accumulators (momentum Ax, Ay,
// mass Am and, axisymmetric only, the hoop sum Ah).  Rows outside the window
// are reached in the owner CTA's window.
struct Window {
  float2* G;
  float *Ax, *Ay, *Am, *Ah;
  int nx, win0;
  int WR;  // rows of a plane (the largest band the sort may cut, plus the halo)
  int VR;  // rows in use: this band's rows plus the halo; rows VR .. WR - 1 stay idle
  int CS;
  const int* brow;  // shared copy of the instance's band row starts (CS + 1)
};

// Distributed shared memory in explicit shared::cluster form: the address of
// a local shared location in CTA `rank` of the cluster (mapa), and 32-bit
// loads / reductions there, so that no generic pointer into another CTA's
// window reaches the code that works on this CTA's window.
__device__ __forceinline__ uint32_t dsmem_addr(const void* local, int rank) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(local);
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void dsmem_add(uint32_t a, float v) {
  asm volatile("red.shared::cluster.add.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ float2 dsmem_ld2(uint32_t a) {
  float2 v;
  asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a) : "memory");
  return v;
}

// Tensor memory (TMEM) variant of the cell lanes' node block.  With more than
// 16 warps per SM the 48-float block no longer fits in registers beside one
// particle's state, so between the particles of its cell a lane keeps the
// block in TMEM: warp w of the CTA uses TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31
// (its threads' own lanes, the quadrant a warp may access) and the 48 columns
// starting at 48 (w / 4) of the CTA's allocation.  Each access starts at a
// multiple of its width in columns.  A load first waits for the thread's
// earlier stores (tcgen05.wait::st; the second half needs none of its own,
// see the cell loop) and waits for its data inside the same asm statement, so
// its outputs cannot be read before they arrive.
#define JF_TM_OUT16(b)                                                                                   \
  "=r"(r[b + 0]), "=r"(r[b + 1]), "=r"(r[b + 2]), "=r"(r[b + 3]), "=r"(r[b + 4]), "=r"(r[b + 5]),        \
      "=r"(r[b + 6]), "=r"(r[b + 7]), "=r"(r[b + 8]), "=r"(r[b + 9]), "=r"(r[b + 10]), "=r"(r[b + 11]), \
      "=r"(r[b + 12]), "=r"(r[b + 13]), "=r"(r[b + 14]), "=r"(r[b + 15])
#define JF_TM_IN16(b)                                                                                             \
  "r"(r[b + 0]), "r"(r[b + 1]), "r"(r[b + 2]), "r"(r[b + 3]), "r"(r[b + 4]), "r"(r[b + 5]), "r"(r[b + 6]),      \
      "r"(r[b + 7]), "r"(r[b + 8]), "r"(r[b + 9]), "r"(r[b + 10]), "r"(r[b + 11]), "r"(r[b + 12]), "r"(r[b + 13]), \
      "r"(r[b + 14]), "r"(r[b + 15])
#define JF_TM_OUT8(b) \
  "=r"(r[b + 0]), "=r"(r[b + 1]), "=r"(r[b + 2]), "=r"(r[b + 3]), "=r"(r[b + 4]), "=r"(r[b + 5]), "=r"(r[b + 6]), "=r"(r[b + 7])
#define JF_TM_IN8(b) \
  "r"(r[b + 0]), "r"(r[b + 1]), "r"(r[b + 2]), "r"(r[b + 3]), "r"(r[b + 4]), "r"(r[b + 5]), "r"(r[b + 6]), "r"(r[b + 7])

// columns 0 .. 47 of the warp's block set to zero (a task's start)
__device__ __forceinline__ void tm_zero48(uint32_t ta) {
  const uint32_t z = 0u;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3};\n\t"
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%1], {%3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3};\n\t"
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%2], {%3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3, %3};"
      :
      : "r"(ta), "r"(ta + 16u), "r"(ta + 32u), "r"(z)
      : "memory");
}
// columns 0 .. 23 (block rows 0 and 1): 16 at 0, 8 at 16
__device__ __forceinline__ void tm_load_rows01(uint32_t ta, float* acc) {
  uint32_t r[24];
  asm volatile(
      "tcgen05.wait::st.sync.aligned;\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%24];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16, %17, %18, %19, %20, %21, %22, %23}, [%25];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : JF_TM_OUT16(0), JF_TM_OUT8(16)
      : "r"(ta), "r"(ta + 16u)
      : "memory");
#pragma unroll
  for (int q = 0; q < 24; ++q) acc[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tm_store_rows01(uint32_t ta, const float* acc) {
  uint32_t r[24];
#pragma unroll
  for (int q = 0; q < 24; ++q) r[q] = __float_as_uint(acc[q]);
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17};\n\t"
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%1], {%18, %19, %20, %21, %22, %23, %24, %25};"
      :
      : "r"(ta), "r"(ta + 16u), JF_TM_IN16(0), JF_TM_IN8(16)
      : "memory");
}
// columns 24 .. 47 (block rows 2 and 3): 8 at 24, 16 at 32.  No wait for
// earlier stores: the last store to these columns came before the wait of the
// rows-0/1 load that precedes every use.
__device__ __forceinline__ void tm_load_rows23(uint32_t ta, float* acc) {
  uint32_t r[24];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%24];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23}, [%25];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : JF_TM_OUT8(0), JF_TM_OUT16(8)
      : "r"(ta + 24u), "r"(ta + 32u)
      : "memory");
#pragma unroll
  for (int q = 0; q < 24; ++q) acc[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tm_store_rows23(uint32_t ta, const float* acc) {
  uint32_t r[24];
#pragma unroll
  for (int q = 0; q < 24; ++q) r[q] = __float_as_uint(acc[q]);
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%2, %3, %4, %5, %6, %7, %8, %9};\n\t"
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%1], {%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25};"
      :
      : "r"(ta + 24u), "r"(ta + 32u), JF_TM_IN8(0), JF_TM_IN16(8)
      : "memory");
}
#undef JF_TM_OUT16
#undef JF_TM_IN16
#undef JF_TM_OUT8
#undef JF_TM_IN8

// the band (CTA of the cluster) that owns grid row j, and j's row in its window
__device__ __forceinline__ int owner_of(const Window& w, int j) {
  int o = 0;
  while (o + 1 < w.CS && w.brow[o + 1] <= j) ++o;
  return o;
}
__device__ __forceinline__ int owner_row(const Window& w, int j, int o) { return j - (w.brow[o] - kHaloLo); }

__device__ __forceinline__ float2 gather_node(const Window& w, cg::cluster_group& cl, int i, int j) {
  const int wr = j - w.win0;
  if (wr >= 0 && wr < w.VR) {
    const int n = wr * w.nx + i;
    return w.G[n];
  }
  const int o = owner_of(w, j);
  const int n = owner_row(w, j, o) * w.nx + i;
  return dsmem_ld2(dsmem_addr(w.G + n, o));
}

// Scatter of one particle's 9 stencil contributions with atomics, local when
// the rows are in this CTA's window, else into the owner CTA's window.
__device__ __forceinline__ void scatter_particle(const Window& w, cg::cluster_group& cl, const JfInst& I,
                                                 const JfStencil& st, const JfScatter& sc) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int row = st.by + j;
    const int wr = row - w.win0;
    if (wr >= 0 && wr < w.VR) {
      const int rn = wr * w.nx + st.bx;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const float3 c = jf_node_contrib(I, st, sc, i, j);
        atomicAdd(w.Ax + rn + i, c.x);
        atomicAdd(w.Ay + rn + i, c.y);
        atomicAdd(w.Am + rn + i, c.z);
        if (I.axisym) atomicAdd(w.Ah + rn + i, jf_w(st, 0, i) * jf_w(st, 1, j) * sc.hoop);
      }
    } else {
      const int o = owner_of(w, row);
      const int rn = owner_row(w, row, o) * w.nx + st.bx;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const float3 c = jf_node_contrib(I, st, sc, i, j);
        dsmem_add(dsmem_addr(w.Ax + rn + i, o), c.x);
        dsmem_add(dsmem_addr(w.Ay + rn + i, o), c.y);
        dsmem_add(dsmem_addr(w.Am + rn + i, o), c.z);
        if (I.axisym) dsmem_add(dsmem_addr(w.Ah + rn + i, o), jf_w(st, 0, i) * jf_w(st, 1, j) * sc.hoop);
      }
    }
  }
}

// Adds a particle's 3x3 stencil into the lane's 4x4 node block, shifted by
// (di, dj) = stencil base - (cell - 1), both 0 or 1.  Branch-free: the
// weights are shifted into 4-wide vectors with zeros outside the stencil, so
// lanes with different shifts run the same instructions.  Contributions are
// formed separably, weight_x * (m v + A (x_i - x_p)) per column and then
// weight_y per row, a re-association of mpm_sim.py:256-271 that moves results
// by rounding only.
__device__ __forceinline__ void accumulate_block(float* acc, const JfInst& I, const JfStencil& st,
                                                 const JfScatter& sc, int di, int dj) {
  const bool sx = di != 0, sy = dj != 0;
  const float wx4[4] = {sx ? 0.0f : st.wx0, sx ? st.wx0 : st.wx1, sx ? st.wx1 : st.wx2, sx ? st.wx2 : 0.0f};
  const float wy4[4] = {sy ? 0.0f : st.wy0, sy ? st.wy0 : st.wy1, sy ? st.wy1 : st.wy2, sy ? st.wy2 : 0.0f};
  // node offsets from the particle: (I - di - fx0) dx; di + fx0 is exact
  const float ex = (float)di + st.fx0, ey = (float)dj + st.fx1;
  float P[4], Q0[4], Q1[4], Pm[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float d0 = ((float)i - ex) * I.dx;
    P[i] = wx4[i];
    Q0[i] = wx4[i] * (sc.mv0 + sc.af00 * d0);
    Q1[i] = wx4[i] * (sc.mv1 + sc.af10 * d0);
    Pm[i] = wx4[i] * sc.mass;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float d1 = ((float)j - ey) * I.dx;
    const float r0 = sc.af01 * d1, r1 = sc.af11 * d1;
    const float wj = wy4[j];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int q = (j * 4 + i) * 3;
      acc[q + 0] += wj * (Q0[i] + P[i] * r0);
      acc[q + 1] += wj * (Q1[i] + P[i] * r1);
      acc[q + 2] += wj * Pm[i];
    }
  }
}

// accumulate_block restricted to block rows J0 and J0 + 1, whose 24 floats
// `acc` holds (the TMEM variant adds a particle half a block at a time).
template <int J0>
__device__ __forceinline__ void accumulate_rows(float* acc, const JfInst& I, const JfStencil& st,
                                                const JfScatter& sc, int di, int dj) {
  const bool sx = di != 0, sy = dj != 0;
  const float wx4[4] = {sx ? 0.0f : st.wx0, sx ? st.wx0 : st.wx1, sx ? st.wx1 : st.wx2, sx ? st.wx2 : 0.0f};
  const float wy4[4] = {sy ? 0.0f : st.wy0, sy ? st.wy0 : st.wy1, sy ? st.wy1 : st.wy2, sy ? st.wy2 : 0.0f};
  const float ex = (float)di + st.fx0, ey = (float)dj + st.fx1;
  float P[4], Q0[4], Q1[4], Pm[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float d0 = ((float)i - ex) * I.dx;
    P[i] = wx4[i];
    Q0[i] = wx4[i] * (sc.mv0 + sc.af00 * d0);
    Q1[i] = wx4[i] * (sc.mv1 + sc.af10 * d0);
    Pm[i] = wx4[i] * sc.mass;
  }
#pragma unroll
  for (int jj = 0; jj < 2; ++jj) {
    const int j = J0 + jj;
    const float d1 = ((float)j - ey) * I.dx;
    const float r0 = sc.af01 * d1, r1 = sc.af11 * d1;
    const float wj = wy4[j];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int q = (jj * 4 + i) * 3;
      acc[q + 0] += wj * (Q0[i] + P[i] * r0);
      acc[q + 1] += wj * (Q1[i] + P[i] * r1);
      acc[q + 2] += wj * Pm[i];
    }
  }
}

// Writes a warp's 4x4 node blocks into the window.  Lane l owns cell column
// cx = seg0 + l and covers node columns cx-1 .. cx+2; node column cx collects
// block column 1 of lane l, 0 of lane l+1, 2 of lane l-1 and 3 of lane l-2,
// so each lane issues one atomic per (row, component).  Lane 0 also writes
// column seg0-1, lane 31 columns seg0+32 and seg0+33.
// `acc` holds block rows J0 .. J0 + NJ - 1 (the TMEM variant flushes two rows
// at a time).
template <int J0 = 0, int NJ = 4>
__device__ __forceinline__ void flush_block(const float* acc, const Window& w, int lane, int cx, int cy,
                                            int seg0, int nx) {
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int J = J0; J < J0 + NJ; ++J) {
    const int rowo = (cy - 1 + J - w.win0) * nx;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float* A = q == 0 ? w.Ax : (q == 1 ? w.Ay : w.Am);
      const float a0 = acc[((J - J0) * 4 + 0) * 3 + q];
      const float a1 = acc[((J - J0) * 4 + 1) * 3 + q];
      const float a2 = acc[((J - J0) * 4 + 2) * 3 + q];
      const float a3 = acc[((J - J0) * 4 + 3) * 3 + q];
      const float from_right = __shfl_down_sync(full, a0, 1);
      const float from_left = __shfl_up_sync(full, a2, 1);
      const float from_left2 = __shfl_up_sync(full, a3, 2);
      const float a3_l30 = __shfl_sync(full, a3, 30);
      float col = a1;
      if (lane <= 30) col += from_right;
      if (lane >= 1) col += from_left;
      if (lane >= 2) col += from_left2;
      if (cx < nx && col != 0.0f) atomicAdd(A + rowo + cx, col);
      if (lane == 0 && seg0 >= 1 && a0 != 0.0f) atomicAdd(A + rowo + seg0 - 1, a0);
      if (lane == 31) {
        const float e32 = a2 + a3_l30;
        if (seg0 + 32 < nx && e32 != 0.0f) atomicAdd(A + rowo + seg0 + 32, e32);
        if (seg0 + 33 < nx && a3 != 0.0f) atomicAdd(A + rowo + seg0 + 33, a3);
      }
    }
  }
}

// kTmem: the node blocks live in TMEM (launched with 544 .. 768 threads, 80
// registers at 768); otherwise in registers (up to 512 threads, 128 registers).
template <bool kTmem>
__global__ void __launch_bounds__(kTmem ? kTmemThreads : 512, 1) chunk_kernel(ChunkArgs a) {
  extern __shared__ float4 smem4[];
  float* sm = reinterpret_cast<float*>(smem4);
  // per-substep values, double-buffered so that substep s + 1's are set
  // before the barrier that ends substep s
  __shared__ float s_pressure[2];
  __shared__ int s_next_task[2];

  cg::cluster_group cluster = cg::this_cluster();
  const int CS = a.CS;
  const int r = (int)cluster.block_rank();
  const int ci = blockIdx.x / CS;
  if (ci >= a.M) return;  // a padding cluster leaves as a whole
  const int m = a.order[ci];

  const JfInst I = a.inst[m];
  const JfParams P = a.params[m];
  const JfMaterials mats = a.mats;
  const int nx = I.nx, ny = I.ny;
  __shared__ int s_brow[kMaxCluster + 1];
  if (threadIdx.x <= CS) s_brow[threadIdx.x] = a.brow[m * (CS + 1) + threadIdx.x];
  __syncthreads();
  const int row0 = s_brow[r];
  const int own_hi = s_brow[r + 1];
  Window w;
  w.nx = nx;
  w.CS = CS;
  w.brow = s_brow;
  w.win0 = row0 - kHaloLo;
  w.WR = I.band_cap + kHalo;  // the window holds the largest band the sort may cut
  w.VR = max(own_hi - row0, 0) + kHalo;
  const int WN = w.WR * nx;
  w.G = reinterpret_cast<float2*>(sm);  // 2 * WN floats
  w.Ax = sm + 2 * WN;
  w.Ay = w.Ax + WN;
  w.Am = w.Ay + WN;
  w.Ah = w.Am + WN;  // a sixth plane exists only in the axisymmetric variant
  const int n_planes = I.axisym ? 6 : 5;
  const int cap = a.cap[m];
  const int tid = threadIdx.x, nth = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, n_warps = nth >> 5;
  const int cells = nx * ny;
  const int32_t* cstart = a.cell_start + (int64_t)m * a.stride;
  const int64_t p0 = I.p_off;
  // this instance's particle arrays, indexed by position within the instance
  float4* __restrict__ xv_m = a.xv + p0;
  float4* __restrict__ C_m = a.C + p0;
  float4* __restrict__ F_m = a.F + p0;
  const int32_t* __restrict__ mat_m = a.mat + p0;

  for (int n = tid; n < n_planes * WN; n += nth) sm[n] = 0.0f;
  // path counters of the CTA: register-block scatters, per-particle (generic)
  // scatters, generic gathers, overflow particles
  __shared__ unsigned s_path[4];
  if (tid < 4) s_path[tid] = 0u;
  bool nonfinite = false;  // a G2P result of this thread's particles was NaN/Inf
  // TMEM: 48 columns per warp of a lane quadrant, rounded up to a power of two
  // (256 for up to 16 + 4 warps, 512 for 24); one CTA per SM, so the
  // allocation never waits for another CTA's
  __shared__ uint32_t s_tmem;
  uint32_t tm_cols = 32, tm_base = 0, ta = 0;
  if constexpr (kTmem) {
    const int per_quad = (n_warps + 3) >> 2;
    while (tm_cols < (uint32_t)(48 * per_quad)) tm_cols <<= 1;
    __syncwarp();
    if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       (uint32_t)__cvta_generic_to_shared(&s_tmem)),
                   "r"(tm_cols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  cluster.sync();
  if constexpr (kTmem) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    tm_base = s_tmem;
    ta = tm_base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(48 * (warp >> 2));
  }

  // G2P of the previous substep, then P2G of this one, for a particle that
  // is not handled by a cell lane (generic gathers and scatters).
  auto particle_generic = [&](int64_t g, bool do_g2p, bool do_p2g, float pressure) {
    const float4 xv = a.xv[g];
    float4 C = a.C[g];
    const int mt = a.mat[g];
    float2 x = make_float2(xv.x, xv.y), v = make_float2(xv.z, xv.w);
    float jp = 1.0f;
    if (mt == 2 || a.do_glow) jp = a.Jp[g];
    if (do_g2p) {
      jf_g2p_particle(I, x, v, C, [&](int ni, int nj) { return gather_node(w, cluster, ni, nj); });
      if (a.do_glow) a.glow[g] = jf_glow(a.glow[g], jp);
      nonfinite |= !(isfinite(x.x) && isfinite(x.y) && isfinite(v.x) && isfinite(v.y));
      a.xv[g] = make_float4(x.x, x.y, v.x, v.y);
      if (!do_p2g) a.C[g] = C;  // stored when no later pass of the chunk recomputes it (see the cell loop)
    }
    if (do_p2g) {
      JfStencil st;
      if (jf_stencil(I, x, st)) {
        float4 F = a.F[g];
        const float2 fb = (mt == 3) ? a.fiber[g] : make_float2(0.0f, 1.0f);
        JfScatter sc;
        jf_p2g_particle(I, mats, mt, v, C, F, jp, fb, pressure, P.payload_density, sc, x.x,
                        I.axisym ? a.rref[g] : 1.0f);
        a.F[g] = F;
        if (mt == 2) a.Jp[g] = jp;
        scatter_particle(w, cluster, I, st, sc);
      } else if (do_g2p) {
        a.C[g] = C;  // out of range: the next G2P keeps this C
      }
    }
  };

  // tasks: groups of 32 generic particles (this band's overflow list, then,
  // in the last band, live particles outside every stencil range), then the
  // 32-cell row segments of the band.  The slower generic groups go first so
  // that the segments even out the end of the pass; a group's lanes take
  // entries n_gen_tasks apart, far apart in the list, so that their atomics
  // rarely meet on one node.
  const int segs = (nx + 31) >> 5;
  const int n_cell_tasks = max(own_hi - row0, 0) * segs;
  const int32_t* ov = a.ovlist + p0 + a.ovband[m * (CS + 1) + r];
  const int n_ov = a.ovband[m * (CS + 1) + r + 1] - a.ovband[m * (CS + 1) + r];
  int oor_beg = 0, n_oor = 0;
  if (r == CS - 1) {
    oor_beg = cstart[cells];
    n_oor = cstart[cells + 1] - oor_beg;
  }
  const int n_generic_all = n_ov + n_oor;
  const int n_gen_tasks = (n_generic_all + 31) >> 5;
  const int n_tasks = n_cell_tasks + n_gen_tasks;

  // window rows outside the band (pushed to / pulled from their owners):
  // row 0 and rows n_own + 1 .. VR - 1
  const int n_own = max(own_hi - row0, 0);
  const int n_halo_rows = w.VR - n_own;  // row 0 and rows n_own + 1 .. n_own + 3
  const bool rows_by_thread = (nth % nx) == 0;  // the grid update can step whole rows

  float t = *a.t_dev;
  if (tid == 0) {
    s_pressure[0] = P.actuation * jf_activation(P.freq, P.contraction, t);
    s_next_task[0] = n_warps;
  }
  __syncthreads();
  for (int s = 0; s <= a.K; ++s) {
    const bool do_g2p = s > 0;
    const bool do_p2g = s < a.K;
    const float pressure = s_pressure[s & 1];
    int* next_task = &s_next_task[s & 1];

    // cells of the band: a warp takes 32 consecutive cells of one row; warps
    // claim row segments from a shared counter so that they finish together
    for (int task_id = warp; task_id < n_tasks;) {
      if (task_id < n_gen_tasks) {
        const int e = task_id + lane * n_gen_tasks;
        if (e < n_generic_all) {
          const bool over = e < n_ov;
          particle_generic(p0 + (over ? ov[e] : oor_beg + e - n_ov), do_g2p, do_p2g, pressure);
          atomicAdd(&s_path[over ? 3 : 1], 1u);
        }
        int nt = 0;
        if (lane == 0) nt = atomicAdd(next_task, 1);
        task_id = __shfl_sync(0xffffffffu, nt, 0);
        continue;
      }
      const int task = task_id - n_gen_tasks;
      const int cy = row0 + task / segs;
      const int seg0 = (task % segs) << 5;
      const int cx = seg0 + lane;
      int beg = 0, end = 0;
      if (cx < nx) {
        const int c = cy * nx + cx;
        beg = cstart[c];
        end = min(cstart[c + 1], beg + cap);  // the rest of the cell is overflow
      }
      // G2P then P2G of particle k of this lane's cell (nxv / nmt: its
      // prefetched position-velocity and material, replaced by particle
      // k + 1's); returns true when its stencil lies in the lane's 4x4 node
      // block (columns cx-1 .. cx+2, rows cy-1 .. cy+2), with the stencil,
      // the scatter terms and the block offset for the caller to add
      auto cell_particle = [&](int k, float4& nxv, int& nmt, JfStencil& st, JfScatter& sc, int& di,
                               int& dj) -> bool {
        const float4 xv = nxv;
        const int mt = nmt;
        float4 F = F_m[k];  // first used by P2G, after the gather
        if (k + 1 < end) {  // next particle of this cell, loaded while this one computes
          nxv = xv_m[k + 1];
          nmt = mat_m[k + 1];
        }
        float2 x = make_float2(xv.x, xv.y), v = make_float2(xv.z, xv.w);
        float jp = 1.0f;
        if (mt == 2 || a.do_glow) jp = a.Jp[p0 + k];
        // G2P replaces v and C from the grid (mpm_sim.py:315-327); the stored
        // C is read only where G2P does not run
        float4 C;
        if (do_g2p) {
          JfStencil gs;
          if (!jf_stencil(I, x, gs)) {
            C = C_m[k];
          } else {
            const int wr0 = gs.by - w.win0;
            if (wr0 >= 0 && wr0 + 2 < w.VR) {
              const int wb = wr0 * nx + gs.bx;
              jf_g2p_apic(I, gs, v, C, [&](int i, int j) {
                const int n = wb + j * nx + i;
                return w.G[n];
              });
            } else {
              atomicAdd(&s_path[2], 1u);
              jf_g2p_apic(I, gs, v, C,
                          [&](int i, int j) { return gather_node(w, cluster, gs.bx + i, gs.by + j); });
            }
          }
          jf_g2p_advect(I, x, v);
          if (a.do_glow) a.glow[p0 + k] = jf_glow(a.glow[p0 + k], jp);
          nonfinite |= !(isfinite(x.x) && isfinite(x.y) && isfinite(v.x) && isfinite(v.y));
          xv_m[k] = make_float4(x.x, x.y, v.x, v.y);
          // this pass's P2G takes C from registers and the next pass's G2P
          // recomputes it, so C is stored only by the chunk's last pass and
          // where the particle leaves the stencil range (P2G below)
          if (!do_p2g) C_m[k] = C;
        } else {
          C = C_m[k];
        }
        if (!do_p2g) return false;
        if (!jf_stencil(I, x, st)) {
          if (do_g2p) C_m[k] = C;  // out of range: the next G2P keeps this C
          return false;
        }
        const float2 fb = (mt == 3) ? a.fiber[p0 + k] : make_float2(0.0f, 1.0f);
        jf_p2g_particle(I, mats, mt, v, C, F, jp, fb, pressure, P.payload_density, sc, x.x,
                        I.axisym ? a.rref[p0 + k] : 1.0f);
        F_m[k] = F;
        if (mt == 2) a.Jp[p0 + k] = jp;
        di = st.bx - (cx - 1);
        dj = st.by - (cy - 1);
        if ((unsigned)di < 2u && (unsigned)dj < 2u) {
          if (I.axisym) {  // the hoop sum goes straight to the window (rows in it)
            const int hb = (st.by - w.win0) * nx + st.bx;
#pragma unroll
            for (int jj = 0; jj < 3; ++jj)
#pragma unroll
              for (int ii = 0; ii < 3; ++ii)
                atomicAdd(w.Ah + hb + jj * nx + ii, jf_w(st, 0, ii) * jf_w(st, 1, jj) * sc.hoop);
          }
          return true;
        }
        atomicAdd(&s_path[1], 1u);
        scatter_particle(w, cluster, I, st, sc);
        return false;
      };
      float4 nxv;
      int nmt = -1;
      if (beg < end) {
        nxv = xv_m[beg];
        nmt = mat_m[beg];
      }
      if constexpr (!kTmem) {
        // the lane's cell runs as a loop of its own length; the block stays in registers
        unsigned n_block = 0;
        float acc[48];
#pragma unroll
        for (int q = 0; q < 48; ++q) acc[q] = 0.0f;
        for (int k = beg; k < end; ++k) {
          JfStencil st;
          JfScatter sc;
          int di, dj;
          if (cell_particle(k, nxv, nmt, st, sc, di, dj)) {
            accumulate_block(acc, I, st, sc, di, dj);
            ++n_block;
          }
        }
        __syncwarp();
        if (do_p2g) {
          flush_block(acc, w, lane, cx, cy, seg0, nx);
          const unsigned nb = __reduce_add_sync(0xffffffffu, n_block);
          if (lane == 0 && nb) atomicAdd(&s_path[0], nb);
        }
      } else {
        // the warp steps its cells' particles together (the TMEM accesses are
        // warp-wide) for as many iterations as its fullest cell; the block of
        // each lane is loaded from TMEM, added to and stored back, two rows at
        // a time, once per iteration in which some lane's particle adds to it
        const int iters = (int)__reduce_max_sync(0xffffffffu, (unsigned)(end - beg));
        unsigned n_block = 0;  // the same in every lane of the warp
        __syncwarp();
        if (do_p2g) tm_zero48(ta);
        for (int it = 0; it < iters; ++it) {
          const int k = beg + it;
          JfStencil st;
          JfScatter sc;
          int di = 0, dj = 0;
          const bool blk = k < end && cell_particle(k, nxv, nmt, st, sc, di, dj);
          if (do_p2g) {
            const unsigned bm = __ballot_sync(0xffffffffu, blk);
            if (bm) {
              n_block += (unsigned)__popc(bm);
              float half[24];
              tm_load_rows01(ta, half);
              if (blk) accumulate_rows<0>(half, I, st, sc, di, dj);
              __syncwarp();
              tm_store_rows01(ta, half);
              tm_load_rows23(ta, half);
              if (blk) accumulate_rows<2>(half, I, st, sc, di, dj);
              __syncwarp();
              tm_store_rows23(ta, half);
            }
          }
        }
        __syncwarp();
        if (do_p2g) {
          // the last store to columns 24 .. 47 precedes the wait of the first load
          float half[24];
          tm_load_rows01(ta, half);
          flush_block<0, 2>(half, w, lane, cx, cy, seg0, nx);
          tm_load_rows23(ta, half);
          flush_block<2, 2>(half, w, lane, cx, cy, seg0, nx);
          if (lane == 0 && n_block) atomicAdd(&s_path[0], n_block);
        }
      }
      int nt = 0;
      if (lane == 0) nt = atomicAdd(next_task, 1);
      task_id = __shfl_sync(0xffffffffu, nt, 0);
    }
    __syncthreads();

    if (do_p2g) {
      // halo rows of the accumulator go to the rows' owners
      for (int q = tid; q < n_halo_rows * nx; q += nth) {
        const int h = q / nx;
        const int wr = h == 0 ? 0 : n_own + h;
        const int j = w.win0 + wr;
        if (j < 0 || j >= ny) continue;
        const int n = wr * nx + (q - h * nx);
        const float vx = w.Ax[n], vy = w.Ay[n], vm = w.Am[n];
        const float vh = I.axisym ? w.Ah[n] : 0.0f;
        if (vx != 0.0f || vy != 0.0f || vm != 0.0f || vh != 0.0f) {
          const int o = owner_of(w, j);
          const int rn = owner_row(w, j, o) * nx + (n - wr * nx);
          dsmem_add(dsmem_addr(w.Ax + rn, o), vx);
          dsmem_add(dsmem_addr(w.Ay + rn, o), vy);
          dsmem_add(dsmem_addr(w.Am + rn, o), vm);
          w.Ax[n] = 0.0f;
          w.Ay[n] = 0.0f;
          w.Am[n] = 0.0f;
          if (I.axisym) {
            dsmem_add(dsmem_addr(w.Ah + rn, o), vh);
            w.Ah[n] = 0.0f;
          }
        }
      }
      cluster.sync();

      // grid update of the owned rows (window rows 1 .. n_own); the
      // accumulator is cleared for the next pass
      const bool last = (s == a.K - 1);
      auto update_node = [&](int n, int wr, int i) {
        const int j = w.win0 + wr;
        const float mm = w.Am[n];
        const float2 u = jf_grid_node(I, i, j, w.Ax[n], w.Ay[n], mm, I.axisym ? w.Ah[n] : 0.0f);
        w.G[n] = u;
        if (last) a.grid[I.g_off + (int64_t)j * nx + i] = make_float4(u.x, u.y, mm, 0.0f);
        w.Ax[n] = 0.0f;
        w.Ay[n] = 0.0f;
        w.Am[n] = 0.0f;
        if (I.axisym) w.Ah[n] = 0.0f;
      };
      if (rows_by_thread) {
        // a thread keeps one column and steps nth / nx rows at a time
        const int i = tid % nx, row_step = nth / nx;
        for (int wr = kHaloLo + tid / nx; wr < kHaloLo + n_own; wr += row_step) update_node(wr * nx + i, wr, i);
      } else {
        for (int n = kHaloLo * nx + tid; n < (kHaloLo + n_own) * nx; n += nth) {
          const int wr = n / nx;
          update_node(n, wr, n - wr * nx);
        }
      }
      cluster.sync();

      // halo rows of the updated grid come from their owners
      for (int q = tid; q < n_halo_rows * nx; q += nth) {
        const int h = q / nx;
        const int wr = h == 0 ? 0 : n_own + h;
        const int j = w.win0 + wr;
        if (j < 0 || j >= ny) continue;
        const int n = wr * nx + (q - h * nx);
        const int o = owner_of(w, j);
        const int rn = owner_row(w, j, o) * nx + (n - wr * nx);
        w.G[n] = dsmem_ld2(dsmem_addr(w.G + rn, o));
      }
      t = t + a.dt;
      if (tid == 0) {
        s_pressure[(s + 1) & 1] = P.actuation * jf_activation(P.freq, P.contraction, t);
        s_next_task[(s + 1) & 1] = n_warps;
      }
      __syncthreads();
    }
  }
  if (__any_sync(0xffffffffu, nonfinite) && lane == 0) atomicOr(a.err + m, 1);
  // the CTA's path counters, and the TMEM allocation freed once every warp
  // is past its last access
  if constexpr (kTmem) asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if constexpr (kTmem) {
    if (warp == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm_base), "r"(tm_cols)
                   : "memory");
    }
  }
  if (a.path && tid < 4 && s_path[tid]) atomicAdd(a.path + tid, (unsigned long long)s_path[tid]);
  // peers may still read this CTA's grid rows in their last G2P pass
  cluster.sync();
}

// Cell key of every particle: row-major cell index, then one bin for live
// particles outside the stencil range and one for dead slots.
__global__ void sort_keys_kernel(const JfInst* __restrict__ inst, const float4* __restrict__ xv,
                                 const int32_t* __restrict__ mat, int32_t* __restrict__ keys,
                                 int32_t* __restrict__ rank, int32_t* __restrict__ counts, int stride,
                                 int32_t* __restrict__ solid) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const int cells = I.nx * I.ny;
  int key;
  const int mt = mat[g];
  if (mt < 0) {
    key = cells + 1;
  } else {
    const float4 a = xv[g];
    JfStencil st;
    if (jf_stencil(I, make_float2(a.x, a.y), st)) {
      const int2 c = sort_cell(I, make_float2(a.x, a.y));
      key = c.y * I.nx + c.x;
    } else {
      key = cells;
    }
  }
  keys[g] = key;
  // lanes of the warp with the same cell take one atomic between them (lattice
  // neighbours share cells); each gets its rank from the group's base
  const unsigned group = __match_any_sync(__activemask(), key);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(group) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counts + (int64_t)m * stride + key, __popc(group));
  base = __shfl_sync(group, base, leader);
  rank[g] = base + __popc(group & ((1u << lane) - 1u));
  if (mt > 0 && key < cells && I.ny <= kMaxBandRows) atomicAdd(solid + m * kMaxBandRows + key / I.nx, 1);
}

// Per instance: the cell cap, the exclusive scan of the bins (counts become
// bin starts), the CTA band table (CTA r owns positions [band[r], band[r+1]);
// the last CTA also takes the out-of-range bin) and the band starts and
// cursors of the overflow list.
__global__ void __launch_bounds__(kScanThreads) sort_scan_kernel(const JfInst* __restrict__ inst,
                                                                int32_t* __restrict__ counts,
                                                                int stride, int32_t* __restrict__ band,
                                                                int32_t* __restrict__ brow,
                                                                int32_t* __restrict__ cap_out,
                                                                int32_t* __restrict__ ovband,
                                                                int32_t* __restrict__ ovcur, int CS,
                                                                int fixed_cap, const int32_t* __restrict__ solid) {
  __shared__ int warp_sums[kScanThreads / 32];
  __shared__ int s_cost[kCapCandidates];
  __shared__ int s_row_cost[kMaxBandRows];
  __shared__ int s_row_over[kMaxBandRows];
  __shared__ int s_brow[kMaxCluster + 1];
  __shared__ int s_cap;
  const int m = blockIdx.x;
  const JfInst I = inst[m];
  const int cells = I.nx * I.ny;
  const int nbins = cells + 2;
  int32_t* c = counts + (int64_t)m * stride;
  const int segs = (I.nx + 31) >> 5;
  const bool dynamic = I.ny <= kMaxBandRows;

  // per-lane cap from the cell counts (candidate 0 = no cap); costs in
  // quarter lane-iterations: 128 per warp iteration, 6 per overflow particle
  if (threadIdx.x < kCapCandidates) s_cost[threadIdx.x] = 0;
  for (int y = threadIdx.x; y < min(I.ny, kMaxBandRows); y += kScanThreads) {
    s_row_cost[y] = kRowCost + (kSolidCostHalves * solid[m * kMaxBandRows + y]) / 2;
    s_row_over[y] = 0;
  }
  __syncthreads();
  for (int sg = threadIdx.x; sg < I.ny * segs; sg += kScanThreads) {
    const int row = sg / segs;
    const int x0 = (sg - row * segs) << 5;
    const int xn = min(32, I.nx - x0);
    const int32_t* cr = c + row * I.nx + x0;
    int mx = 0;
    for (int i = 0; i < xn; ++i) mx = max(mx, cr[i]);
    if (mx == 0) continue;
    atomicAdd(&s_cost[0], 128 * mx);
    for (int k = 1; k < kCapCandidates; ++k) {
      int ov = 0;
      if (k < mx)
        for (int i = 0; i < xn; ++i) ov += max(0, cr[i] - k);
      atomicAdd(&s_cost[k], 128 * min(mx, k) + 6 * ov);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int best = 0;
    for (int k = 1; k < kCapCandidates; ++k)
      if (s_cost[k] < s_cost[best]) best = k;
    if (fixed_cap > 0) best = fixed_cap < kCapCandidates ? fixed_cap : 0;
    cap_out[m] = best == 0 ? kNoCap : best;
    s_cap = best == 0 ? kNoCap : best;
  }
  __syncthreads();
  // cost and overflow of every row at the chosen cap
  const int cap = s_cap;
  for (int sg = threadIdx.x; sg < I.ny * segs; sg += kScanThreads) {
    const int row = sg / segs;
    const int x0 = (sg - row * segs) << 5;
    const int xn = min(32, I.nx - x0);
    const int32_t* cr = c + row * I.nx + x0;
    int mx = 0, ov = 0;
    for (int i = 0; i < xn; ++i) {
      mx = max(mx, cr[i]);
      ov += max(0, cr[i] - cap);
    }
    if (dynamic) {
      atomicAdd(&s_row_cost[row], 128 * min(mx, cap) + 6 * ov);
      if (ov) atomicAdd(&s_row_over[row], ov);
    } else if (ov) {
      atomicAdd(&s_row_over[min(row / I.band_h, CS - 1)], ov);  // per band
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (dynamic) {
      // band r starts where the prefix cost reaches r / CS of the total,
      // clamped so that no band exceeds band_cap rows and the bands after it
      // can still cover the rows that are left
      long long total = 0;
      for (int y = 0; y < I.ny; ++y) total += s_row_cost[y];
      s_brow[0] = 0;
      long long pre = 0;
      int y = 0;
      for (int r = 1; r < CS; ++r) {
        const long long target = total * r / CS;
        while (y < I.ny && pre + s_row_cost[y] / 2 < target) pre += s_row_cost[y++];
        int b = y;
        b = min(b, s_brow[r - 1] + I.band_cap);
        b = max(b, I.ny - (CS - r) * I.band_cap);
        b = max(b, s_brow[r - 1]);
        b = min(b, I.ny);
        while (y > b) pre -= s_row_cost[--y];
        while (y < b) pre += s_row_cost[y++];
        s_brow[r] = b;
      }
      s_brow[CS] = I.ny;
    } else {
      for (int r = 0; r < CS; ++r) s_brow[r] = min(r * I.band_h, I.ny);
      s_brow[CS] = I.ny;
    }
    // overflow bins of the bands (in the position list order)
    int run = 0;
    for (int r = 0; r < CS; ++r) {
      ovband[m * (CS + 1) + r] = run;
      ovcur[m * CS + r] = run;
      if (cap != kNoCap) {
        if (dynamic)
          for (int yy = s_brow[r]; yy < s_brow[r + 1]; ++yy) run += s_row_over[yy];
        else
          run += s_row_over[r];
      }
    }
    ovband[m * (CS + 1) + CS] = run;
    for (int r = 0; r <= CS; ++r) brow[m * (CS + 1) + r] = s_brow[r];
  }
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
    for (int r = 0; r < CS; ++r) band[m * (CS + 1) + r] = (int32_t)I.p_off + c[s_brow[r] * I.nx];
    band[m * (CS + 1) + CS] = (int32_t)I.p_off + c[cells + 1];
  }
}

// Moves every particle to bin start + rank; particles of a cell beyond the
// cap are also listed in their band's part of the overflow list.
__global__ void sort_scatter_kernel(const JfInst* __restrict__ inst, const int32_t* __restrict__ keys,
                                    const int32_t* __restrict__ rank, const int32_t* __restrict__ starts,
                                    int stride, const int32_t* __restrict__ cap, int CS,
                                    const int32_t* __restrict__ brow, int32_t* __restrict__ ovcur,
                                    int32_t* __restrict__ ovlist, JfParticles src, JfParticles dst) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const int key = keys[g];
  const int rk = rank[g];
  const int32_t rel = starts[(int64_t)m * stride + key] + rk;
  const int64_t d = I.p_off + rel;
  if (key < I.nx * I.ny && rk >= cap[m]) {
    const int row = key / I.nx;
    const int32_t* br = brow + m * (CS + 1);
    int band = 0;
    while (band + 1 < CS && br[band + 1] <= row) ++band;
    ovlist[I.p_off + atomicAdd(ovcur + m * CS + band, 1)] = rel;
  }
  dst.xv[d] = src.xv[g];
  dst.C[d] = src.C[g];
  dst.F[d] = src.F[g];
  dst.mat[d] = src.mat[g];
  dst.fiber[d] = src.fiber[g];
  dst.Jp[d] = src.Jp[g];
  dst.glow[d] = src.glow[g];
  dst.slot[d] = src.slot[g];
  dst.rref[d] = src.rref[g];
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

// sim_time += dt, K times, as the FP32 running sum of mpm_sim.py:340
__global__ void advance_time_kernel(float* t, int K, float dt) {
  float v = *t;
  for (int s = 0; s < K; ++s) v = v + dt;
  *t = v;
}

}  // namespace

size_t jf_batched_smem_bytes(const jf_engine* e) {
  const size_t planes = (e->flags & JF_FLAG_AXISYM) ? 6 : 5;
  return sizeof(float) * planes * (size_t)e->win_nodes;
}

cudaError_t jf_batched_sort(jf_engine* e) {
  JfTimed timed(e, true, e->capturing);
  const int stride = e->max_cells + 2;
  cudaError_t err = cudaMemsetAsync(e->d_counts, 0, sizeof(int32_t) * (size_t)stride * e->M, e->stream);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(e->d_solid, 0, sizeof(int32_t) * (size_t)kMaxBandRows * e->M, e->stream);
  if (err != cudaSuccess) return err;
  const dim3 grid((e->max_slots + kSortThreads - 1) / kSortThreads, e->M);
  if (e->max_slots > 0) {
    sort_keys_kernel<<<grid, kSortThreads, 0, e->stream>>>(e->d_inst, e->p.xv, e->p.mat, e->d_keys,
                                                          e->d_rank, e->d_counts, stride, e->d_solid);
  }
  sort_scan_kernel<<<e->M, kScanThreads, 0, e->stream>>>(e->d_inst, e->d_counts, stride, e->d_band,
                                                         e->d_brow, e->d_cap, e->d_ovband, e->d_ovcur,
                                                         e->cluster, e->cell_cap, e->d_solid);
  if (e->max_slots > 0) {
    sort_scatter_kernel<<<grid, kSortThreads, 0, e->stream>>>(e->d_inst, e->d_keys, e->d_rank, e->d_counts,
                                                             stride, e->d_cap, e->cluster, e->d_brow,
                                                             e->d_ovcur, e->d_ovlist, e->p, e->q);
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
  a.rref = e->p.rref;
  a.cell_start = e->d_counts;
  a.cap = e->d_cap;
  a.ovlist = e->d_ovlist;
  a.ovband = e->d_ovband;
  a.order = e->d_order;
  a.brow = e->d_brow;
  a.stride = e->max_cells + 2;
  a.grid = e->d_grid;
  a.err = e->d_err;
  a.M = e->M;
  a.CS = e->cluster;
  a.K = K;
  a.t_dev = e->d_time;
  a.dt = (float)e->dt;
  a.do_glow = (e->flags & JF_FLAG_GLOW) ? 1 : 0;
  a.path = e->d_path;

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
    JfTimed timed(e, false, e->capturing);
    err = e->block_threads > 512 ? cudaLaunchKernelEx(&cfg, chunk_kernel<true>, a)
                                 : cudaLaunchKernelEx(&cfg, chunk_kernel<false>, a);
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

// the chunk kernel instantiation the engine's CTA size selects
static const void* chunk_kernel_for(const jf_engine* e) {
  return e->block_threads > 512 ? (const void*)chunk_kernel<true> : (const void*)chunk_kernel<false>;
}

cudaError_t jf_batched_prepare(jf_engine* e) {
  const size_t smem = jf_batched_smem_bytes(e);
  const void* k = chunk_kernel_for(e);
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  if (e->cluster > 8) {
    err = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
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
  return (int)cudaOccupancyMaxActiveClusters(out, chunk_kernel_for(e), &cfg);
}

static cudaError_t chunk_with_sort(jf_engine* e, int K) {
  cudaError_t err = jf_batched_sort(e);
  if (err != cudaSuccess) return err;
  if ((err = launch_chunk(e, K)) != cudaSuccess) return err;
  advance_time_kernel<<<1, 1, 0, e->stream>>>(e->d_time, K, (float)e->dt);
  e->launches += 1;
  e->sorted = false;  // particles moved: re-sort before the next chunk
  return cudaGetLastError();
}

// A graph of two (sort, chunk) pairs: two re-sorts swap the ping-pong particle
// buffers twice, so the graph leaves them as it found them and can be replayed.
static cudaError_t capture_pair(jf_engine* e, int K) {
  if (e->graph_exec) {
    cudaGraphExecDestroy(e->graph_exec);
    e->graph_exec = nullptr;
  }
  cudaGraph_t graph = nullptr;
  const int64_t launches = e->launches;
  cudaError_t err = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) return err;
  e->capturing = true;
  cudaError_t e1 = chunk_with_sort(e, K);
  cudaError_t e2 = (e1 == cudaSuccess) ? chunk_with_sort(e, K) : e1;
  e->capturing = false;
  err = cudaStreamEndCapture(e->stream, &graph);
  e->launches = launches;  // nothing ran yet
  if (e2 != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return e2;
  }
  if (err != cudaSuccess) return err;
  err = cudaGraphInstantiate(&e->graph_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (err != cudaSuccess) return err;
  e->graph_K = K;
  e->graph_p = e->p.xv;
  e->graph_launches = 2 * (e->max_slots > 0 ? 5 : 3) + ((e->flags & JF_FLAG_GLOW) ? 2 : 0);
  return cudaSuccess;
}

cudaError_t jf_batched_step(jf_engine* e, int64_t n_steps) {
  const float dtf = (float)e->dt;
  cudaError_t err = cudaMemcpyAsync(e->d_time, &e->t, sizeof(float), cudaMemcpyHostToDevice, e->stream);
  if (err != cudaSuccess) return err;
  const int R = e->resort_interval;
  while (n_steps > 0) {
    // graphs are replayed only when per-kernel timing is off (events cannot
    // attribute time inside a replayed graph)
    if (e->use_graphs && !e->timing && n_steps >= 2 * R) {
      if (!e->graph_exec || e->graph_K != R || e->graph_p != e->p.xv) {
        if ((err = capture_pair(e, R)) != cudaSuccess) return err;
      }
      {
        JfTimed timed(e, false);
        if ((err = cudaGraphLaunch(e->graph_exec, e->stream)) != cudaSuccess) return err;
      }
      e->launches += e->graph_launches;
      for (int s = 0; s < 2 * R; ++s) e->t = e->t + dtf;
      n_steps -= 2 * R;
      continue;
    }
    const int K = (int)(n_steps < R ? n_steps : R);
    if ((err = chunk_with_sort(e, K)) != cudaSuccess) return err;
    for (int s = 0; s < K; ++s) e->t = e->t + dtf;
    n_steps -= K;
  }
  // the host's copy is the authoritative time; the device copy keeps up with it
  return cudaSuccess;
}
