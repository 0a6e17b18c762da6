// Headless renderer: the reference's Taichi render kernels (mpm_sim.py:343-712)
// as CUDA kernels writing a device frame buffer (no graphics API).
//
// The frame is video_res x video_res pixels of float4 (r, g, b, unused), so
// that an additive splat is one 16-byte vector atomic per pixel instead of
// three scalar ones; jf_read_frame packs it to the reference's
// frame_buffer[py, px, c] layout.  Every kernel follows its reference kernel
// in FP32 with each operation rounded on its own (the _rn intrinsics keep the
// compiler from contracting a*b+c), so that which pixels a particle or grid
// cell touches is decided bit for bit as in the reference; cos, atan2, tanh and
// pow are evaluated in double and rounded once.  Additive splats land in
// arbitrary order (float atomics), so HDR sums agree with a serial renderer to
// rounding.
#include "jf_engine.h"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// mpm_sim.py:345-358
__device__ float3 hsv2rgb(float h, float s, float v) {
  const float h6 = fmul(h, 6.0f);
  const int i = (int)h6;
  const float f = fsub(h6, (float)i);
  const float p = fmul(v, fsub(1.0f, s));
  const float q = fmul(v, fsub(1.0f, fmul(f, s)));
  const float t = fmul(v, fsub(1.0f, fmul(fsub(1.0f, f), s)));
  switch (((i % 6) + 6) % 6) {  // Taichi's integer % is Python's (floor) modulo
    case 0: return make_float3(v, t, p);
    case 1: return make_float3(q, v, p);
    case 2: return make_float3(p, v, t);
    case 3: return make_float3(p, q, v);
    case 4: return make_float3(t, p, v);
    default: return make_float3(v, p, q);
  }
}

// Screen position of a particle of the instance in tile (row, col):
// mpm_sim.py:462-463 (abyss) and 503-504 (flat pass).
__device__ __forceinline__ float2 splat_centre(float2 x, float dh, int row, int col, int res_sub) {
  const float cx = fmul(fadd(fdiv(x.x, dh), (float)col), (float)res_sub);
  const float cy = fmul(fadd(fdiv(fsub(dh, x.y), dh), (float)row), (float)res_sub);
  return make_float2(cx, cy);
}

__global__ void clear_kernel(float4* __restrict__ fb, int64_t n, float value) {
  const float4 c = make_float4(value, value, value, 0.0f);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    fb[k] = c;
}

// render_frame_abyss, mpm_sim.py:385-481: one thread per particle slot.
__global__ void __launch_bounds__(kThreads) abyss_kernel(const JfInst* __restrict__ inst,
                                                        const JfParams* __restrict__ params,
                                                        const float4* __restrict__ xv,
                                                        const int32_t* __restrict__ mat,
                                                        const float* __restrict__ Jp,
                                                        const float2* __restrict__ hues, float t, int res_sub,
                                                        int grid_side, float radius, int water_mode, int res,
                                                        float4* __restrict__ fb) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t g = I.p_off + k;
  const int mt = mat[g];
  if (mt < 0) return;  // dead slots skip the position load
  const float4 a = xv[g];
  if (a.x < 0.0f) return;
  const float dh = (float)I.domain_h;
  const int row = m / grid_side, col = m % grid_side;
  const float vel = sqrtf(fadd(fmul(a.z, a.z), fmul(a.w, a.w)));
  float3 color = make_float3(0.0f, 0.0f, 0.0f);
  float intensity = 0.0f;
  if (mt == 0) {  // water
    if (vel > 0.02f) {
      if (water_mode == 0) {
        color = make_float3(0.15f, 0.15f, 0.18f);
        intensity = 0.008f;
      } else {
        const float br = fminf(fdiv(vel, 2.0f), 1.0f);
        if (water_mode == 1) {
          color = hsv2rgb(0.60f, 0.55f, br);
        } else {
          const float ang = (float)atan2((double)a.w, (double)a.z);
          const float h = fadd(fdiv(ang, (float)(2.0 * 3.14159265)), 0.5f);
          const float hue = fsub(h, fmul(1.0f, floorf(fdiv(h, 1.0f))));  // Taichi's float %
          color = hsv2rgb(hue, 0.8f, br);
        }
        intensity = fadd(0.025f, fmul(0.075f, br));
      }
    }
  } else if (mt == 1) {  // jelly
    const float gnf = grid_side > 1 ? (float)(grid_side - 1) : 1.0f;
    const float sat = fadd(0.4f, fmul(fdiv((float)row, gnf), 0.4f));
    const float3 base = hsv2rgb(hues[m].x, sat, 0.9f);
    const float glow = fadd(fmul(fabsf(fsub(1.0f, Jp[g])), 2.0f), 0.1f);
    color = make_float3(fadd(base.x, glow), fadd(base.y, glow), fadd(base.z, glow));
    intensity = fadd(0.05f, fmul(glow, 0.2f));
  } else if (mt == 3) {  // muscle: brightens with the instance's activation
    const JfParams P = params[m];
    const float act = jf_activation(P.freq, P.contraction, t);
    const float3 base = hsv2rgb(hues[m].y, 0.2f, 1.0f);
    color = make_float3(fadd(base.x, act), fadd(base.y, act), fadd(base.z, act));
    intensity = fadd(0.4f, fmul(act, 0.4f));
  } else if (mt == 2) {  // payload
    color = make_float3(1.0f, 0.2f, 0.0f);
    intensity = 0.8f;
  }
  if (!(intensity > 0.001f)) return;
  const float2 c = splat_centre(make_float2(a.x, a.y), dh, row, col, res_sub);
  const float dr = fmul(radius, 1.5f);
  const float dr2 = fmul(dr, dr);
  const int lx = (int)fsub(c.x, dr), hx = (int)fadd(c.x, dr);
  const int ly = (int)fsub(c.y, dr), hy = (int)fadd(c.y, dr);
  const float cr = fmul(color.x, intensity), cg = fmul(color.y, intensity), cb = fmul(color.z, intensity);
  for (int px = max(lx, 0); px <= min(hx, res - 1); ++px) {
    const float ddx = fsub((float)px, c.x);
    const float ddx2 = fmul(ddx, ddx);
    for (int py = max(ly, 0); py <= min(hy, res - 1); ++py) {
      const float ddy = fsub((float)py, c.y);
      const float dn = fdiv(fadd(ddx2, fmul(ddy, ddy)), dr2);
      if (dn < 1.0f) {
        // (1 - dn)^4: the double product is exact to 96 bits before the rounding
        const double u = (double)fsub(1.0f, dn);
        const double u2 = u * u;
        const float fo = (float)(u2 * u2);
        atomicAdd(fb + (int64_t)py * res + px, make_float4(fmul(cr, fo), fmul(cg, fo), fmul(cb, fo), 0.0f));
      }
    }
  }
}

// render_flat_pass, mpm_sim.py:489-517: one material in one colour.  Every
// covering write stores the same value, so the order of writes is immaterial.
__global__ void __launch_bounds__(kThreads) flat_kernel(const JfInst* __restrict__ inst,
                                                       const float4* __restrict__ xv,
                                                       const int32_t* __restrict__ mat, int res_sub, int grid_side,
                                                       float radius, int target, float r, float g, float b, int res,
                                                       float4* __restrict__ fb) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n_slots) return;
  const int64_t q = I.p_off + k;
  const float4 a = xv[q];
  if (mat[q] != target || a.x < 0.0f) return;
  const int row = m / grid_side, col = m % grid_side;
  const float2 c = splat_centre(make_float2(a.x, a.y), (float)I.domain_h, row, col, res_sub);
  const float dr = radius, dr2 = fmul(radius, radius);
  const int lx = (int)fsub(c.x, dr), hx = (int)fadd(c.x, dr);
  const int ly = (int)fsub(c.y, dr), hy = (int)fadd(c.y, dr);
  const float4 v = make_float4(r, g, b, 0.0f);
  for (int px = max(lx, 0); px <= min(hx, res - 1); ++px) {
    const float ddx = fsub((float)px, c.x);
    const float ddx2 = fmul(ddx, ddx);
    for (int py = max(ly, 0); py <= min(hy, res - 1); ++py) {
      const float ddy = fsub((float)py, c.y);
      if (fadd(ddx2, fmul(ddy, ddy)) <= dr2) fb[(int64_t)py * res + px] = v;
    }
  }
}

// curl of node (i, j) of instance I, mpm_sim.py:536-539 (grid node layout
// g_off + j * nx + i); false on the border and at nodes without mass.
__device__ __forceinline__ bool node_curl(const JfInst& I, const float4* __restrict__ grid, int i, int j,
                                          float& curl) {
  if (i < 1 || i >= I.nx - 1 || j < 1 || j >= I.ny - 1) return false;
  const float4* G = grid + I.g_off;
  if (!(G[(int64_t)j * I.nx + i].z > 0.0f)) return false;
  const float two_dx = (float)(2.0 * (1.0 / I.nx));
  const float dvx_dy = fdiv(fsub(G[(int64_t)(j + 1) * I.nx + i].x, G[(int64_t)(j - 1) * I.nx + i].x), two_dx);
  const float dvy_dx = fdiv(fsub(G[(int64_t)j * I.nx + i + 1].y, G[(int64_t)j * I.nx + i - 1].y), two_dx);
  curl = fsub(dvx_dy, dvy_dx);
  return true;
}

// render_vorticity_overlay, mpm_sim.py:520-558: one thread per grid node.
__global__ void __launch_bounds__(kThreads) overlay_kernel(const JfInst* __restrict__ inst,
                                                          const float4* __restrict__ grid, int res_sub,
                                                          int grid_side, float scale, int res,
                                                          float4* __restrict__ fb) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= I.nx * I.ny) return;
  const int j = n / I.nx, i = n - j * I.nx;
  float curl;
  if (!node_curl(I, grid, i, j, curl)) return;
  const float vi = fminf(fmul(fabsf(curl), scale), 1.0f);
  if (vi < 0.01f) return;
  const float4 col = curl > 0.0f ? make_float4(fmul(fmul(1.0f, vi), 0.5f), fmul(fmul(0.4f, vi), 0.5f), 0.0f, 0.0f)
                                 : make_float4(0.0f, fmul(fmul(0.4f, vi), 0.5f), fmul(fmul(1.0f, vi), 0.5f), 0.0f);
  const int row = m / grid_side, c = m % grid_side;
  const float dh = (float)I.domain_h, fnx = (float)I.nx;
  const int cell_x = (int)fmul(fadd(fdiv(fdiv((float)i, fnx), dh), (float)c), (float)res_sub);
  const int cell_y = (int)fmul(fadd(fdiv(fsub(dh, fdiv((float)j, fnx)), dh), (float)row), (float)res_sub);
  const int cell_px = max(1, res_sub / I.nx);
  for (int px = max(cell_x - cell_px / 2, 0); px <= min(cell_x + cell_px / 2, res - 1); ++px)
    for (int py = max(cell_y - cell_px / 2, 0); py <= min(cell_y + cell_px / 2, res - 1); ++py)
      atomicAdd(fb + (int64_t)py * res + px, col);
}

// compute_vorticity_grid, mpm_sim.py:561-579 (vort in grid node layout).
__global__ void __launch_bounds__(kThreads) vorticity_kernel(const JfInst* __restrict__ inst,
                                                            const float4* __restrict__ grid, float scale,
                                                            float* __restrict__ vort) {
  const int m = blockIdx.y;
  const JfInst I = inst[m];
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= I.nx * I.ny) return;
  const int j = n / I.nx, i = n - j * I.nx;
  float curl, out = 0.0f;
  if (node_curl(I, grid, i, j, curl)) out = (float)tanh((double)fmul(curl, scale));
  vort[I.g_off + n] = out;
}

// render_vorticity_rdbu / _hueshift / _white, mpm_sim.py:582-711: one thread
// per pixel.  style 2 writes every pixel (the white clear, then the blend).
__global__ void __launch_bounds__(kThreads) vort_blend_kernel(const JfInst* __restrict__ inst, int M,
                                                             const float* __restrict__ vort, int res_sub,
                                                             int grid_side, float alpha_max, int style, int res,
                                                             float4* __restrict__ fb) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= (int64_t)res * res) return;
  const int py = (int)(n / res), px = (int)(n - (int64_t)py * res);
  float4 o = style == 2 ? make_float4(1.0f, 1.0f, 1.0f, 0.0f) : fb[n];
  const int col = (int)((int64_t)px * grid_side / res);
  const int row = (int)((int64_t)py * grid_side / res);
  const int m = row * grid_side + col;
  if (m < M) {
    const JfInst I = inst[m];
    const float sub_x = fdiv((float)(px - col * res_sub), (float)res_sub);
    const float sub_y = fsub(1.0f, fdiv((float)(py - row * res_sub), (float)res_sub));
    const int gi = (int)fmul(fmul(sub_x, (float)I.nx), (float)I.domain_h);
    const int gj = (int)fmul(sub_y, (float)I.ny);
    if (gi >= 0 && gi < I.nx && gj >= 0 && gj < I.ny) {
      const float vv = vort[I.g_off + (int64_t)gj * I.nx + gi];
      const float mag = fabsf(vv);
      if (!(mag < 0.02f)) {
        const float alpha = fmul(alpha_max, mag);
        const float t = fadd(0.5f, fmul(0.5f, vv > 0.0f ? 1.0f : (vv < 0.0f ? -1.0f : 0.0f)));
        const bool warm = style == 1;
        const float pr = warm ? 0.90f : 0.84f, pg = warm ? 0.18f : 0.10f, pb = warm ? 0.15f : 0.11f;
        const float nr = warm ? 0.15f : 0.13f, ng = warm ? 0.35f : 0.31f, nb = warm ? 0.90f : 0.80f;
        const float u = fsub(1.0f, t);
        const float cr = fadd(fmul(t, pr), fmul(u, nr));
        const float cg = fadd(fmul(t, pg), fmul(u, ng));
        const float cb = fadd(fmul(t, pb), fmul(u, nb));
        const float keep = fsub(1.0f, alpha);
        if (style == 2) {
          o = make_float4(fadd(keep, fmul(alpha, cr)), fadd(keep, fmul(alpha, cg)), fadd(keep, fmul(alpha, cb)), 0.0f);
        } else {
          o = make_float4(fadd(fmul(keep, o.x), fmul(alpha, cr)), fadd(fmul(keep, o.y), fmul(alpha, cg)),
                          fadd(fmul(keep, o.z), fmul(alpha, cb)), 0.0f);
        }
      }
    }
  }
  if (style == 2 || m < M) fb[n] = o;
}

// tone_map_and_encode, mpm_sim.py:366-383.
__device__ __forceinline__ float tone(float hdr) {
  const float e = fmul(hdr, 2.5f);
  float mapped = fdiv(e, fadd(e, 1.0f));
  mapped = fdiv(mapped, fadd(mapped, 0.15f));
  return (float)pow((double)mapped, (double)(float)(1.0 / 2.2));
}

__global__ void tone_map_kernel(float4* __restrict__ fb, int64_t n) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const float4 h = fb[k];
    fb[k] = make_float4(tone(h.x), tone(h.y), tone(h.z), 0.0f);
  }
}

int pixel_blocks(const jf_engine* e) {
  const int64_t n = (int64_t)e->frame_res * e->frame_res;
  return (int)std::min<int64_t>((n + kThreads - 1) / kThreads, 148 * 16);
}

}  // namespace

cudaError_t jf_frame_clear_launch(jf_engine* e, float value) {
  clear_kernel<<<pixel_blocks(e), kThreads, 0, e->stream>>>(e->d_frame, (int64_t)e->frame_res * e->frame_res, value);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_render_abyss_launch(jf_engine* e, int res_sub, int grid_side, float radius, int water_mode) {
  if (e->max_slots == 0) return cudaSuccess;
  const dim3 grid((e->max_slots + kThreads - 1) / kThreads, e->M);
  abyss_kernel<<<grid, kThreads, 0, e->stream>>>(e->d_inst, e->d_params, e->p.xv, e->p.mat, e->p.Jp, e->d_hue, e->t,
                                                 res_sub, grid_side, radius, water_mode, e->frame_res, e->d_frame);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_render_flat_launch(jf_engine* e, int res_sub, int grid_side, float radius, int material, float r,
                                  float g, float b) {
  if (e->max_slots == 0) return cudaSuccess;
  const dim3 grid((e->max_slots + kThreads - 1) / kThreads, e->M);
  flat_kernel<<<grid, kThreads, 0, e->stream>>>(e->d_inst, e->p.xv, e->p.mat, res_sub, grid_side, radius, material, r,
                                                g, b, e->frame_res, e->d_frame);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_render_overlay_launch(jf_engine* e, int res_sub, int grid_side, float scale) {
  const dim3 grid((e->max_cells + kThreads - 1) / kThreads, e->M);
  overlay_kernel<<<grid, kThreads, 0, e->stream>>>(e->d_inst, e->d_grid, res_sub, grid_side, scale, e->frame_res,
                                                   e->d_frame);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_vorticity_launch(jf_engine* e, float scale) {
  const dim3 grid((e->max_cells + kThreads - 1) / kThreads, e->M);
  vorticity_kernel<<<grid, kThreads, 0, e->stream>>>(e->d_inst, e->d_grid, scale, e->d_vort);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_render_vort_launch(jf_engine* e, int res_sub, int grid_side, float alpha, int style) {
  const int64_t n = (int64_t)e->frame_res * e->frame_res;
  vort_blend_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, e->stream>>>(
      e->d_inst, e->M, e->d_vort, res_sub, grid_side, alpha, style, e->frame_res, e->d_frame);
  e->launches += 1;
  return cudaGetLastError();
}

cudaError_t jf_tone_map_launch(jf_engine* e) {
  tone_map_kernel<<<pixel_blocks(e), kThreads, 0, e->stream>>>(e->d_frame, (int64_t)e->frame_res * e->frame_res);
  e->launches += 1;
  return cudaGetLastError();
}
