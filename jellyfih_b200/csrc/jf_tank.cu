// Tank fill on the GPU (make_jelly.py:336-402): the water lattice of one
// instance, minus the lattice points within the water margin of a robot
// particle, placed after the robot in slot order, written into the load
// staging of the engine.
//
// The lattice is numpy's np.arange(margin, stop, spacing) in x and y
// (element i = start + i * ((start + spacing) - start), length
// ceil((stop - start) / spacing)), the candidates in meshgrid-ravel order
// (y outer, x inner).  A candidate is dropped when its distance to the
// nearest robot particle, sqrt((x - rx)^2 + (y - ry)^2) in double with each
// operation rounded on its own, is <= the margin — the test the reference's
// KD-tree query makes.  Kept candidates keep their lattice order (a scan of
// keep flags), and water that does not fit in the instance's slots is cut.
#include "jf_engine.h"

namespace {

constexpr int kThreads = 256;
constexpr int kRobotTile = 1024;  // robot positions per shared-memory tile (16 KB)

struct Lattice {
  double x0, dx;  // x_i = x0 + i * dx
  double y0, dy;
  int nx, ny;     // candidates per row, rows
};

__device__ __forceinline__ double2 candidate(const Lattice& L, int64_t c) {
  const int j = (int)(c / L.nx), i = (int)(c - (int64_t)j * L.nx);
  return make_double2(__dadd_rn(L.x0, __dmul_rn((double)i, L.dx)), __dadd_rn(L.y0, __dmul_rn((double)j, L.dy)));
}

// keep[c] = 1 when candidate c is farther than `margin` from every robot
// particle; per-block keep counts into block_count.
__global__ void __launch_bounds__(kThreads) water_keep_kernel(Lattice L, const double2* __restrict__ robot,
                                                             int n_robot, double4 bbox, double margin,
                                                             int32_t* __restrict__ keep,
                                                             int32_t* __restrict__ block_count) {
  __shared__ double2 s_r[kRobotTile];
  __shared__ int s_count[kThreads / 32];
  const int64_t n = (int64_t)L.nx * L.ny;
  const int64_t c = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  const bool valid = c < n;
  const double2 p = valid ? candidate(L, c) : make_double2(0.0, 0.0);
  // the robot's bounding box grown by the margin: candidates outside it keep
  bool near = valid && p.x >= bbox.x && p.x <= bbox.z && p.y >= bbox.y && p.y <= bbox.w;
  bool drop = false;
  // the block scans the robot in tiles while any of its candidates needs it
  if (__syncthreads_or(near)) {
    for (int t0 = 0; t0 < n_robot; t0 += kRobotTile) {
      const int tn = min(kRobotTile, n_robot - t0);
      __syncthreads();
      for (int k = threadIdx.x; k < tn; k += kThreads) s_r[k] = robot[t0 + k];
      __syncthreads();
      if (near && !drop) {
        for (int k = 0; k < tn; ++k) {
          const double ex = __dsub_rn(p.x, s_r[k].x), ey = __dsub_rn(p.y, s_r[k].y);
          const double d2 = __dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey));
          if (sqrt(d2) <= margin) {
            drop = true;
            break;
          }
        }
      }
    }
  }
  const int kf = (valid && !drop) ? 1 : 0;
  if (valid) keep[c] = kf;
  const int wsum = __reduce_add_sync(0xffffffffu, kf);
  if ((threadIdx.x & 31) == 0) s_count[threadIdx.x >> 5] = wsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < kThreads / 32; ++w) s += s_count[w];
    block_count[blockIdx.x] = s;
  }
}

// Exclusive scan of the per-block counts (one block; blocks <= a few
// thousand), total into *total.
__global__ void __launch_bounds__(1024) block_scan_kernel(int32_t* __restrict__ block_count, int n_blocks,
                                                         int32_t* __restrict__ total) {
  __shared__ int s_carry;
  __shared__ int s_warp[32];
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < n_blocks; b0 += blockDim.x) {
    const int b = b0 + threadIdx.x;
    const int v = b < n_blocks ? block_count[b] : 0;
    // inclusive warp scan, then across warps
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if ((threadIdx.x & 31) >= o) x += y;
    }
    if ((threadIdx.x & 31) == 31) s_warp[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
      int w = (int)threadIdx.x < (int)(blockDim.x >> 5) ? s_warp[threadIdx.x] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if ((int)threadIdx.x >= o) w += y;
      }
      s_warp[threadIdx.x] = w;
    }
    __syncthreads();
    const int warp_base = (threadIdx.x >> 5) > 0 ? s_warp[(threadIdx.x >> 5) - 1] : 0;
    const int carry = s_carry;
    if (b < n_blocks) block_count[b] = carry + warp_base + x - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = carry + warp_base + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = s_carry;
}

// Kept candidate c goes to slot n_robot + (its rank among kept candidates),
// if that is below n_slots: staging position (f32), material 0, fibre (0, 1).
__global__ void __launch_bounds__(kThreads) water_place_kernel(Lattice L, const int32_t* __restrict__ keep,
                                                              const int32_t* __restrict__ block_base,
                                                              int n_robot, int n_slots, float* __restrict__ pos,
                                                              float* __restrict__ fib, int32_t* __restrict__ mat) {
  __shared__ int s_warp[kThreads / 32];
  const int64_t n = (int64_t)L.nx * L.ny;
  const int64_t c = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  const int kf = c < n ? keep[c] : 0;
  const unsigned ballot = __ballot_sync(0xffffffffu, kf);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_warp[warp] = __popc(ballot);
  __syncthreads();
  int base = block_base[blockIdx.x];
  for (int w = 0; w < warp; ++w) base += s_warp[w];
  if (!kf) return;
  const int rank = base + __popc(ballot & ((1u << lane) - 1u));
  const int64_t slot = (int64_t)n_robot + rank;
  if (slot >= n_slots) return;
  const double2 p = candidate(L, c);
  pos[2 * slot] = __double2float_rn(p.x);
  pos[2 * slot + 1] = __double2float_rn(p.y);
  fib[2 * slot] = 0.0f;
  fib[2 * slot + 1] = 1.0f;
  mat[slot] = 0;
}

}  // namespace

// numpy.arange(start, stop, step): length and element spacing as numpy forms them.
static void np_arange(double start, double stop, double step, double& x0, double& dx, int& n) {
  x0 = start;
  dx = (start + step) - start;
  const double len = ceil((stop - start) / step);
  n = len > 0 ? (int)len : 0;
}

cudaError_t jf_tank_water_launch(jf_engine* e, int m, const double* d_robot, int n_robot, const double* bbox,
                                 double water_margin, double spacing_div, int32_t* d_scratch,
                                 int64_t scratch_ints, int32_t* h_total) {
  const JfInst& I = e->inst[m];
  const int grid_res = I.nx;
  const double spacing = 1.0 / (grid_res * spacing_div);
  const double margin = (1.0 / (grid_res * 2.0)) * 3;
  Lattice L;
  np_arange(margin, 1.0 - margin, spacing, L.x0, L.dx, L.nx);
  np_arange(margin, I.domain_h - margin, spacing, L.y0, L.dy, L.ny);
  const int64_t n = (int64_t)L.nx * L.ny;
  const int n_blocks = (int)((n + kThreads - 1) / kThreads);
  // scratch: keep flags [n], block counts [n_blocks], total [1]
  if (n + n_blocks + 1 > scratch_ints) return cudaErrorInvalidValue;
  int32_t* keep = d_scratch;
  int32_t* counts = d_scratch + n;
  int32_t* total = counts + n_blocks;
  const double4 box = make_double4(bbox[0] - water_margin, bbox[1] - water_margin, bbox[2] + water_margin,
                                   bbox[3] + water_margin);
  if (n_blocks > 0) {
    water_keep_kernel<<<n_blocks, kThreads, 0, e->stream>>>(L, reinterpret_cast<const double2*>(d_robot), n_robot,
                                                            box, water_margin, keep, counts);
    block_scan_kernel<<<1, 1024, 0, e->stream>>>(counts, n_blocks, total);
    const int64_t S = e->max_slots;
    water_place_kernel<<<n_blocks, kThreads, 0, e->stream>>>(L, keep, counts, n_robot, I.n_slots, e->d_stage,
                                                             e->d_stage + 2 * S, e->d_stage_i);
    e->launches += 3;
    cudaError_t err = cudaMemcpyAsync(h_total, total, sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream);
    if (err != cudaSuccess) return err;
  } else {
    *h_total = 0;
  }
  return cudaGetLastError();
}

int64_t jf_tank_scratch_ints(const jf_engine* e, int m, double spacing_div) {
  const JfInst& I = e->inst[m];
  const double spacing = 1.0 / (I.nx * spacing_div);
  const double margin = (1.0 / (I.nx * 2.0)) * 3;
  double x0, dx;
  int nx, ny;
  np_arange(margin, 1.0 - margin, spacing, x0, dx, nx);
  np_arange(margin, I.domain_h - margin, spacing, x0, dx, ny);
  const int64_t n = (int64_t)nx * ny;
  return n + (n + kThreads - 1) / kThreads + 1;
}
