/* CPU oracle of the reference's headless renderer (test infrastructure: only
 * tests/, the smoke check and the bench's CPU legs call it; the product path
 * is jellyfih_b200/csrc/jf_render.cu).
 *
 * Restates mpm_sim.py:343-712 of the reference in FP32 (Taichi default_fp),
 * serially in the reference's struct-for order (instance, particle, then
 * pixel columns outer and rows inner), so that additive splats accumulate in
 * the reference's order:
 *   hsv2rgb                    mpm_sim.py:345-358
 *   clear_frame_buffer(_white) mpm_sim.py:361-364, 483-486
 *   tone_map_and_encode        mpm_sim.py:366-383
 *   render_frame_abyss         mpm_sim.py:385-481
 *   render_flat_pass           mpm_sim.py:489-517
 *   render_vorticity_overlay   mpm_sim.py:520-558
 *   compute_vorticity_grid     mpm_sim.py:561-579
 *   render_vorticity_rdbu / _hueshift / _white
 *                              mpm_sim.py:582-711
 * Pinned: tests/golden/make_render_golden.py records the reference's own
 * kernels run under the numpy stand-in of Taichi, and
 * tests/test_oracle_render.py checks this file against those frames.
 * Transcendentals (cos, atan2, tanh) are evaluated in double and rounded once,
 * as the stand-in does; pow is powf.  Frames are HWC float arrays
 * (res x res x 3, frame_buffer[py, px, c]); grids are [nx][ny] per instance.
 * Compiled with -ffp-contract=off: every operation rounds on its own. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct {
  int32_t n_slots, nx, ny;
  float domain_h;
  float freq, contraction, hue, muscle_hue;
} RoInst;

static void hsv2rgb(float h, float s, float v, float* rgb) {
  const float h6 = h * 6.0f;
  const int i = (int)h6;
  const float f = h6 - (float)i;
  const float p = v * (1.0f - s);
  const float q = v * (1.0f - f * s);
  const float t = v * (1.0f - (1.0f - f) * s);
  float r = 0.0f, g = 0.0f, b = 0.0f;
  switch (((i % 6) + 6) % 6) { /* Taichi's integer % follows Python (floor) */
    case 0: r = v; g = t; b = p; break;
    case 1: r = q; g = v; b = p; break;
    case 2: r = p; g = v; b = t; break;
    case 3: r = p; g = q; b = v; break;
    case 4: r = t; g = p; b = v; break;
    default: r = v; g = p; b = q; break;
  }
  rgb[0] = r; rgb[1] = g; rgb[2] = b;
}

/* The per-instance waveform of mpm_sim.py:393-399 (the substep's, 172-180). */
static float activation(float freq, float contraction, float t) {
  const float period = 1.0f / (1.0f * freq);
  const float q = floorf(t / period);
  const float r = t - period * q;
  const float phase = r / period;
  float a = 0.0f;
  if (phase < contraction) {
    const float arg = (phase / contraction) * 3.14159265f;
    a = 0.5f * (1.0f - (float)cos((double)arg));
  }
  return a;
}

void ro_clear(float* fb, int res, float value) {
  for (long k = 0; k < (long)res * res * 3; ++k) fb[k] = value;
}

void ro_tone_map(float* fb, int res) {
  const float exposure = 2.5f;
  const float inv_gamma = (float)(1.0 / 2.2);
  for (long k = 0; k < (long)res * res; ++k) {
    for (int c = 0; c < 3; ++c) {
      const float hdr = fb[3 * k + c];
      float mapped = (hdr * exposure) / (hdr * exposure + 1.0f);
      mapped = mapped / (mapped + 0.15f);
      fb[3 * k + c] = powf(mapped, inv_gamma);
    }
  }
}

void ro_abyss(float* fb, int res, int M, const RoInst* inst, const float* x, const float* v,
              const int32_t* mat, const float* Jp, float t, int res_sub, int grid_side, float radius,
              int water_mode) {
  const float gnf = grid_side > 1 ? (float)(grid_side - 1) : 1.0f;
  const float two_pi = (float)(2.0 * 3.14159265);
  long off = 0;
  for (int m = 0; m < M; ++m) {
    const RoInst I = inst[m];
    const float act = activation(I.freq, I.contraction, t);
    const int row = m / grid_side, col = m % grid_side;
    const float norm_y = (float)row / gnf;
    for (int p = 0; p < I.n_slots; ++p) {
      const long g = off + p;
      const float px0 = x[2 * g], py0 = x[2 * g + 1];
      const int mt = mat[g];
      if (mt < 0 || px0 < 0.0f) continue;
      const float vx = v[2 * g], vy = v[2 * g + 1];
      const float vel = sqrtf(vx * vx + vy * vy);
      const float stress = 1.0f - Jp[g];
      float color[3] = {0.0f, 0.0f, 0.0f};
      float intensity = 0.0f;
      if (mt == 0) {
        if (water_mode == 0) {
          if (vel > 0.02f) {
            color[0] = 0.15f; color[1] = 0.15f; color[2] = 0.18f;
            intensity = 0.008f;
          }
        } else if (water_mode == 1) {
          if (vel > 0.02f) {
            const float br = fminf(vel / 2.0f, 1.0f);
            hsv2rgb(0.60f, 0.55f, br, color);
            intensity = 0.025f + 0.075f * br;
          }
        } else {
          if (vel > 0.02f) {
            const float br = fminf(vel / 2.0f, 1.0f);
            const float ang = (float)atan2((double)vy, (double)vx);
            const float h = ang / two_pi + 0.5f;
            const float hue = h - 1.0f * floorf(h / 1.0f);
            hsv2rgb(hue, 0.8f, br, color);
            intensity = 0.025f + 0.075f * br;
          }
        }
      } else if (mt == 1) {
        const float sat = 0.4f + norm_y * 0.4f;
        float base[3];
        hsv2rgb(I.hue, sat, 0.9f, base);
        const float glow = fabsf(stress) * 2.0f + 0.1f;
        for (int c = 0; c < 3; ++c) color[c] = base[c] + glow;
        intensity = 0.05f + glow * 0.2f;
      } else if (mt == 3) {
        float base[3];
        hsv2rgb(I.muscle_hue, 0.2f, 1.0f, base);
        for (int c = 0; c < 3; ++c) color[c] = base[c] + act;
        intensity = 0.4f + act * 0.4f;
      } else if (mt == 2) {
        color[0] = 1.0f; color[1] = 0.2f; color[2] = 0.0f;
        intensity = 0.8f;
      }
      if (!(intensity > 0.001f)) continue;
      const float cx = (px0 / I.domain_h + (float)col) * (float)res_sub;
      const float cy = ((I.domain_h - py0) / I.domain_h + (float)row) * (float)res_sub;
      const float dr = radius * 1.5f;
      const float dr2 = dr * dr;
      const int lx = (int)(cx - dr), hx = (int)(cx + dr);
      const int ly = (int)(cy - dr), hy = (int)(cy + dr);
      float ci[3];
      for (int c = 0; c < 3; ++c) ci[c] = color[c] * intensity;
      for (int px = lx; px <= hx; ++px) {
        for (int py = ly; py <= hy; ++py) {
          if (px < 0 || px >= res || py < 0 || py >= res) continue;
          const float ddx = (float)px - cx, ddy = (float)py - cy;
          const float dist_sq = ddx * ddx + ddy * ddy;
          const float dn = dist_sq / dr2;
          if (dn < 1.0f) {
            const float falloff = powf(1.0f - dn, 4.0f);
            float* o = fb + 3 * ((long)py * res + px);
            for (int c = 0; c < 3; ++c) o[c] = o[c] + ci[c] * falloff;
          }
        }
      }
    }
    off += I.n_slots;
  }
}

void ro_flat(float* fb, int res, int M, const RoInst* inst, const float* x, const int32_t* mat,
             int res_sub, int grid_side, float radius, int target, float r, float g, float b) {
  long off = 0;
  for (int m = 0; m < M; ++m) {
    const RoInst I = inst[m];
    const int row = m / grid_side, col = m % grid_side;
    for (int p = 0; p < I.n_slots; ++p) {
      const long k = off + p;
      const float px0 = x[2 * k], py0 = x[2 * k + 1];
      if (mat[k] != target || px0 < 0.0f) continue;
      const float cx = (px0 / I.domain_h + (float)col) * (float)res_sub;
      const float cy = ((I.domain_h - py0) / I.domain_h + (float)row) * (float)res_sub;
      const float dr = radius;
      const int lx = (int)(cx - dr), hx = (int)(cx + dr);
      const int ly = (int)(cy - dr), hy = (int)(cy + dr);
      for (int px = lx; px <= hx; ++px) {
        for (int py = ly; py <= hy; ++py) {
          if (px < 0 || px >= res || py < 0 || py >= res) continue;
          const float ddx = (float)px - cx, ddy = (float)py - cy;
          if (ddx * ddx + ddy * ddy <= dr * dr) {
            float* o = fb + 3 * ((long)py * res + px);
            o[0] = r; o[1] = g; o[2] = b;
          }
        }
      }
    }
    off += I.n_slots;
  }
}

/* curl of node (i, j) (mpm_sim.py:536-539); returns 0 when the node is on the
 * border or has no mass (the caller skips it). */
static int curl_at(const RoInst* I, const float* gv, const float* gm, int i, int j, float* curl) {
  if (i < 1 || i >= I->nx - 1 || j < 1 || j >= I->ny - 1) return 0;
  if (!(gm[(long)i * I->ny + j] > 0.0f)) return 0;
  const float two_dx = (float)(2.0 * (1.0 / I->nx));
  const float dvx_dy = (gv[2 * ((long)i * I->ny + j + 1)] - gv[2 * ((long)i * I->ny + j - 1)]) / two_dx;
  const float dvy_dx = (gv[2 * ((long)(i + 1) * I->ny + j) + 1] - gv[2 * ((long)(i - 1) * I->ny + j) + 1]) / two_dx;
  *curl = dvx_dy - dvy_dx;
  return 1;
}

void ro_vort_overlay(float* fb, int res, int M, const RoInst* inst, const float* gv, const float* gm,
                     int res_sub, int grid_side, float scale) {
  long goff = 0;
  for (int m = 0; m < M; ++m) {
    const RoInst* I = &inst[m];
    const float* v = gv + 2 * goff;
    const float* mm = gm + goff;
    const int row = m / grid_side, cc = m % grid_side;
    for (int i = 0; i < I->nx; ++i) {
      for (int j = 0; j < I->ny; ++j) {
        float curl;
        if (!curl_at(I, v, mm, i, j, &curl)) continue;
        const float vi = fminf(fabsf(curl) * scale, 1.0f);
        if (vi < 0.01f) continue;
        float col[3];
        if (curl > 0.0f) {
          col[0] = 1.0f * vi; col[1] = 0.4f * vi; col[2] = 0.0f * vi;
        } else {
          col[0] = 0.0f * vi; col[1] = 0.4f * vi; col[2] = 1.0f * vi;
        }
        const float fnx = (float)I->nx;
        const int cell_x = (int)(((float)i / fnx / I->domain_h + (float)cc) * (float)res_sub);
        const int cell_y = (int)(((I->domain_h - (float)j / fnx) / I->domain_h + (float)row) * (float)res_sub);
        int cell_px = res_sub / I->nx;
        if (cell_px < 1) cell_px = 1;
        for (int px = cell_x - cell_px / 2; px <= cell_x + cell_px / 2; ++px) {
          for (int py = cell_y - cell_px / 2; py <= cell_y + cell_px / 2; ++py) {
            if (px < 0 || px >= res || py < 0 || py >= res) continue;
            float* o = fb + 3 * ((long)py * res + px);
            for (int c = 0; c < 3; ++c) o[c] = o[c] + col[c] * 0.5f;
          }
        }
      }
    }
    goff += (long)I->nx * I->ny;
  }
}

void ro_vort_grid(float* vort, int M, const RoInst* inst, const float* gv, const float* gm, float scale) {
  long goff = 0;
  for (int m = 0; m < M; ++m) {
    const RoInst* I = &inst[m];
    for (int i = 0; i < I->nx; ++i) {
      for (int j = 0; j < I->ny; ++j) {
        float curl;
        float out = 0.0f;
        if (curl_at(I, gv + 2 * goff, gm + goff, i, j, &curl)) out = (float)tanh((double)(curl * scale));
        vort[goff + (long)i * I->ny + j] = out;
      }
    }
    goff += (long)I->nx * I->ny;
  }
}

/* style 0: rdbu (mpm_sim.py:582-625), 1: hueshift (628-670), 2: white (673-711) */
void ro_vort_blend(float* fb, int res, int M, const RoInst* inst, const float* vort, int res_sub,
                   int grid_side, float alpha_max, int style) {
  static const float kCol[3][2][3] = {
      {{0.84f, 0.10f, 0.11f}, {0.13f, 0.31f, 0.80f}},
      {{0.90f, 0.18f, 0.15f}, {0.15f, 0.35f, 0.90f}},
      {{0.84f, 0.10f, 0.11f}, {0.13f, 0.31f, 0.80f}},
  };
  if (style == 2) ro_clear(fb, res, 1.0f);
  long* goff = (long*)malloc(sizeof(long) * (size_t)(M > 0 ? M : 1));
  if (!goff) return;
  long acc = 0;
  for (int m = 0; m < M; ++m) {
    goff[m] = acc;
    acc += (long)inst[m].nx * inst[m].ny;
  }
  for (int px = 0; px < res; ++px) {
    for (int py = 0; py < res; ++py) {
      const int col = px * grid_side / res;
      const int row = py * grid_side / res;
      const int m = row * grid_side + col;
      if (m >= M) continue;
      const RoInst* I = &inst[m];
      const float sub_x = (float)(px - col * res_sub) / (float)res_sub;
      const float sub_y = 1.0f - (float)(py - row * res_sub) / (float)res_sub;
      const int gi = (int)(sub_x * (float)I->nx * I->domain_h);
      const int gj = (int)(sub_y * (float)I->ny);
      if (gi < 0 || gi >= I->nx || gj < 0 || gj >= I->ny) continue;
      const float vv = vort[goff[m] + (long)gi * I->ny + gj];
      const float mag = fabsf(vv);
      if (mag < 0.02f) continue;
      const float alpha = alpha_max * mag;
      const float t = 0.5f + 0.5f * (vv > 0.0f ? 1.0f : (vv < 0.0f ? -1.0f : 0.0f));
      const float* cp = kCol[style][0];
      const float* cn = kCol[style][1];
      float* o = fb + 3 * ((long)py * res + px);
      for (int c = 0; c < 3; ++c) {
        const float colc = t * cp[c] + (1.0f - t) * cn[c];
        if (style == 2)
          o[c] = (1.0f - alpha) + alpha * colc;
        else
          o[c] = (1.0f - alpha) * o[c] + alpha * colc;
      }
    }
  }
  free(goff);
}
