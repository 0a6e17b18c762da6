// Allocation-free substep of one instance (jf_substep_noalloc in
// include/jellyfih.h).
//
// Some callers cannot allocate device memory at the point where they step a
// simulation: code running inside a host callback or a memory pool that must
// not grow, embedders that forbid cudaMalloc after start-up, or programs that
// own all device memory through their own allocator.  This entry point needs
// no allocation: the caller passes the particle arrays (device pointers, the
// reference's layouts) and the grid scratch lives in the file-scope array
// below, which every GPU that loads the library holds until the process exits.
//
// The array holds at most kMaxNodes grid nodes; larger grids are rejected.
// All calls share it and it keeps the last call's contents, so each call
// clears the nodes it uses first, and calls whose work overlaps on the GPU
// (different streams, or different host threads on one device) race on it.
#include <string>

#include "jf_engine.h"

namespace {

constexpr int kMaxNodes = JF_NOALLOC_MAX_NODES;
constexpr int kThreads = 256;

static __device__ __align__(256) float4 g_noalloc_grid[kMaxNodes];

int fail(int code, const std::string& msg) {
  jf_set_global_error(msg);
  return code;
}

__global__ void noalloc_clear(float4* __restrict__ grid, int nodes) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < nodes) grid[n] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__global__ void noalloc_p2g(JfInst I, JfMaterials mats, JfParams P, float pressure, int n,
                            const float2* __restrict__ x, const float2* __restrict__ v,
                            const float4* __restrict__ C, float4* __restrict__ F,
                            const int32_t* __restrict__ mat, float* __restrict__ Jp,
                            const float2* __restrict__ fiber, float4* __restrict__ grid) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int mt = mat[k];
  if (mt < 0) return;
  JfStencil st;
  if (!jf_stencil(I, x[k], st)) return;
  float4 Fk = F[k];
  float jp = Jp[k];
  const float2 fb = (mt == 3 && fiber) ? fiber[k] : make_float2(0.0f, 1.0f);
  JfScatter sc;
  jf_p2g_particle(I, mats, mt, v[k], C[k], Fk, jp, fb, pressure, P.payload_density, sc);
  F[k] = Fk;
  if (mt == 2) Jp[k] = jp;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float3 c = jf_node_contrib(I, st, sc, i, j);
      atomicAdd(grid + (st.by + j) * I.nx + (st.bx + i), make_float4(c.x, c.y, c.z, 0.0f));
    }
  }
}

__global__ void noalloc_grid_update(JfInst I, float4* __restrict__ grid) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= I.nx * I.ny) return;
  const float4 g = grid[n];
  const float2 u = jf_grid_node(I, n % I.nx, n / I.nx, g.x, g.y, g.z);
  grid[n] = make_float4(u.x, u.y, g.z, 0.0f);
}

__global__ void noalloc_g2p(JfInst I, int n, float2* __restrict__ x, float2* __restrict__ v,
                            float4* __restrict__ C, const int32_t* __restrict__ mat,
                            const float* __restrict__ Jp, float* __restrict__ glow,
                            const float4* __restrict__ grid) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (glow) glow[k] = jf_glow(glow[k], Jp[k]);
  if (mat[k] < 0) return;
  float2 xk = x[k], vk = v[k];
  float4 Ck = C[k];
  const int nx = I.nx;
  jf_g2p_particle(I, xk, vk, Ck, [&](int ni, int nj) {
    const float4 q = grid[nj * nx + ni];
    return make_float2(q.x, q.y);
  });
  x[k] = xk;
  v[k] = vk;
  C[k] = Ck;
}

// Device address of the scratch array in the context current on this thread
// (cudaGetSymbolAddress; nullptr on failure).  It is looked up on every call,
// not cached: an address belongs to the context it was taken in, and after a
// cudaDeviceReset, or with another context made current on the same device,
// a cached address would point at memory that is no longer the array.
float4* scratch_in_current_context() {
  float4* ptr = nullptr;
  if (cudaGetSymbolAddress((void**)&ptr, g_noalloc_grid) != cudaSuccess) return nullptr;
  return ptr;
}

bool aligned(const void* p, size_t a) { return ((uintptr_t)p % a) == 0; }

}  // namespace

extern "C" int jf_substep_noalloc(int32_t n, int32_t n_grid, int32_t n_grid_y, float domain_height,
                                  double dt, float sim_time, float actuation, float contraction,
                                  float freq, float payload_density, float* x, float* v, float* C,
                                  float* F, const int32_t* material, float* Jp, float* glow,
                                  const float* fiber, void* stream) {
  if (n < 0) return fail(JF_ERR_INVALID, "jf_substep_noalloc: n must be >= 0");
  if (n_grid < 8 || n_grid_y < 8 || !(domain_height > 0) || !(dt > 0))
    return fail(JF_ERR_INVALID, "jf_substep_noalloc: bad grid size, domain height or dt");
  if ((int64_t)n_grid * n_grid_y > kMaxNodes)
    return fail(JF_ERR_UNSUPPORTED, "jf_substep_noalloc: grid of " + std::to_string(n_grid) + " x " +
                                        std::to_string(n_grid_y) + " nodes exceeds the " +
                                        std::to_string(kMaxNodes) + "-node scratch array");
  if (n > 0 && (!x || !v || !C || !F || !material || !Jp))
    return fail(JF_ERR_INVALID, "jf_substep_noalloc: x, v, C, F, material and Jp are required");
  if (!aligned(x, 8) || !aligned(v, 8) || !aligned(C, 16) || !aligned(F, 16) || !aligned(fiber, 8))
    return fail(JF_ERR_INVALID, "jf_substep_noalloc: x, v, fiber need 8-byte and C, F 16-byte alignment");
  float4* grid = scratch_in_current_context();
  if (!grid) return fail(JF_ERR_CUDA, "jf_substep_noalloc: scratch array unavailable on this device");

  const double dx_d = 1.0 / n_grid;
  const double p_vol = (dx_d * 0.5) * (dx_d * 0.5);
  JfInst I = {};
  I.nx = n_grid;
  I.ny = n_grid_y;
  I.dcx = n_grid / 20;
  I.dcy = n_grid_y / 20;
  I.band_h = n_grid_y;
  I.n_slots = n;
  I.inv_dx = (float)n_grid;
  I.dx = (float)dx_d;
  I.dt = (float)dt;
  I.p_mass = (float)(p_vol * 1);
  I.stress_scale = (float)(-dt * p_vol * 4 * (double)n_grid * n_grid);
  I.c4 = (float)(4.0 * n_grid);
  I.dtg = (float)(dt * 10.0);
  I.y_hi = (float)((double)domain_height - 0.001);
  I.domain_h = (double)domain_height;
  const JfParams P = {actuation, contraction, freq, payload_density};
  const float pressure = actuation * jf_activation(freq, contraction, sim_time);
  cudaStream_t s = (cudaStream_t)stream;
  const int nodes = n_grid * n_grid_y;

  noalloc_clear<<<(nodes + kThreads - 1) / kThreads, kThreads, 0, s>>>(grid, nodes);
  if (n > 0) {
    noalloc_p2g<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
        I, jf_materials(), P, pressure, n, (const float2*)x, (const float2*)v, (const float4*)C,
        (float4*)F, material, Jp, (const float2*)fiber, grid);
  }
  noalloc_grid_update<<<(nodes + kThreads - 1) / kThreads, kThreads, 0, s>>>(I, grid);
  if (n > 0) {
    noalloc_g2p<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(I, n, (float2*)x, (float2*)v,
                                                                   (float4*)C, material, Jp, glow, grid);
  }
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess)
    return fail(JF_ERR_CUDA, std::string("jf_substep_noalloc: launch failed: ") + cudaGetErrorString(err));
  return JF_OK;
}
