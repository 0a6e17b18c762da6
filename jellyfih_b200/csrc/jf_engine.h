// Internal engine state shared by the C-ABI entry points and the two step
// paths (plain per-instance launches, batched persistent cluster launch).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/jellyfih.h"
#include "jf_device.cuh"

// Particle arrays in engine order.  The plain path keeps slot order; the
// batched path keeps every instance's live particles sorted by grid cell, and
// slot[k] maps engine position k back to the caller's slot index.
struct JfParticles {
  float4* xv = nullptr;     // (x0, x1, v0, v1)
  float4* C = nullptr;      // APIC affine velocity, row-major
  float4* F = nullptr;      // deformation gradient, row-major
  int32_t* mat = nullptr;   // material id, -1 = dead slot
  float2* fiber = nullptr;  // muscle fibre direction
  float* Jp = nullptr;      // plastic volume ratio
  float* glow = nullptr;    // render-only glow
  int32_t* slot = nullptr;  // engine position -> slot index
  float* rref = nullptr;    // load radius x[0] (axisymmetric hoop stretch)
};

struct JfGrad;
// Grids up to this many rows get bands balanced by per-row cost at each
// re-sort (taller grids keep equal bands).
constexpr int kJfMaxBandRows = 1024;

struct jf_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int32_t M = 0;
  double dt = 2e-5;
  int32_t path = JF_PATH_PLAIN;
  uint32_t flags = 0;
  int32_t resort_interval = 16;
  int32_t block_threads = 768;
  int32_t cluster = 4;

  std::vector<JfInst> inst;        // host copy
  std::vector<JfParams> params;    // host mirror (authoritative)
  bool params_dirty = true;
  int64_t total_slots = 0;
  int64_t total_nodes = 0;
  int32_t max_slots = 0;
  int32_t max_cells = 0;           // max nx * ny
  int32_t win_nodes = 0;           // max (band_h + halo rows) * nx, batched smem window

  JfInst* d_inst = nullptr;
  JfParams* d_params = nullptr;
  JfParticles p;                   // live buffers
  JfParticles q;                   // batched path: sort destination
  int32_t* d_keys = nullptr;       // batched path: cell key per engine position
  int32_t* d_rank = nullptr;       // batched path: rank of the particle within its cell
  int32_t* d_counts = nullptr;     // batched path: M x (max_cells + 2) histogram, then bin starts
  int32_t* d_ovlist = nullptr;     // batched path: per band, sorted positions beyond the cell cap
  int32_t* d_ovband = nullptr;     // batched path: M x (cluster + 1) overflow list band starts
  int32_t* d_ovcur = nullptr;      // batched path: M x cluster overflow list cursors
  int32_t* d_band = nullptr;       // batched path: M x (cluster + 1) particle ranges
  int32_t* d_cap = nullptr;        // batched path: per-instance particles per cell lane
  int32_t* d_order = nullptr;      // batched path: cluster -> instance, most live particles first
  int32_t* d_brow = nullptr;       // batched path: M x (cluster + 1) band row starts
  float* d_ep = nullptr;           // episode staging: pos (2), fiber (2), glow (1) floats per slot
  int32_t* d_ep_mat = nullptr;     // episode staging: material per slot
  double* d_ep_stats = nullptr;    // episode: CoM sums before the run (6 per instance)
  std::vector<int32_t> n_live;     // live particles per instance at its last load
  std::vector<int32_t> h_order;    // host copy of d_order
  int32_t cell_cap = 0;            // batched path: fixed cell cap, 0 = cost model per re-sort
  int32_t* d_solid = nullptr;      // batched path: M x kJfMaxBandRows non-water particles per grid row
  float4* d_grid = nullptr;        // grid nodes (node = g_off + j * nx + i): (v0, v1, m, 0)
  double* d_stats = nullptr;       // M x 6 CoM sums (payload y, count, x; body y, count, x)
  int32_t* d_err = nullptr;        // per-instance non-finite flags
  float* d_stage = nullptr;        // host <-> device staging (max_slots * 8 floats)
  int32_t* d_stage_i = nullptr;    // staging for ints (max_slots * 2)
  unsigned long long* d_path = nullptr;  // batched path counters (see jf_path_counts)
  double* d_fit = nullptr;         // fitness staging: M x 5 rows + M scores
  double* d_fit_f = nullptr;       // fitness staging: M contraction genes
  int32_t* d_fit_i = nullptr;      // fitness staging: M muscle counts

  bool sorted = false;             // batched path: particle order valid for the current state
  float* d_time = nullptr;         // batched path: sim_time on the device (chunk start)
  bool use_graphs = true;          // batched path: replay (sort, chunk) pairs as a CUDA graph
  bool capturing = false;
  cudaGraphExec_t graph_exec = nullptr;
  int32_t graph_K = 0;
  float4* graph_p = nullptr;       // particle buffer the graph was captured with
  int64_t graph_launches = 0;
  float t = 0.0f;                  // sim_time (FP32 running sum, mpm_sim.py:340)
  int64_t launches = 0;            // kernels launched by this engine
  std::string err;

  JfGrad* grad = nullptr;          // differentiable rollout buffers (jf_grad.cu)
  // headless renderer (jf_render.cu)
  float4* d_frame = nullptr;       // frame_res^2 pixels (r, g, b, unused), row py = frame row
  int32_t frame_res = 0;
  float* d_vort = nullptr;         // tanh-mapped curl per grid node (node layout of d_grid)
  float2* d_hue = nullptr;         // per instance (jelly hue, muscle hue) of the last abyss pass

  // optional device timing of step and sort kernels
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> step_events, sort_events;
  std::vector<cudaEvent_t> event_pool;
  double step_ms = 0.0, sort_ms = 0.0;
  int64_t step_launches = 0, sort_launches = 0;
};

// Event pair bracketing one timed region (no-op when timing is off or when
// the work is being captured into a graph).
struct JfTimed {
  jf_engine* e;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>>* list;
  cudaEvent_t a = nullptr, b = nullptr;
  bool off = false;
  JfTimed(jf_engine* eng, bool sort, bool skip = false);
  ~JfTimed();
};

// Message of the last failed call made without an engine handle
// (jf_create, jf_substep_noalloc); returned by jf_last_error(NULL).
void jf_set_global_error(const std::string& msg);

// Lame parameters by material id (mpm_sim.py:25-48), passed to kernels by value.
JfMaterials jf_materials();

// Plain path: instance-by-instance launches of clear / P2G / grid update / G2P.
cudaError_t jf_plain_step(jf_engine* e, int64_t n_steps);

// Batched path: re-sort plus one persistent cluster launch per chunk.
cudaError_t jf_batched_step(jf_engine* e, int64_t n_steps);
cudaError_t jf_batched_sort(jf_engine* e);
size_t jf_batched_smem_bytes(const jf_engine* e);

// Episode helpers (jf_run_episode): load every instance from slot-ordered
// staging, and the (M, 5) rows from before / after CoM sums, on the device.
cudaError_t jf_load_all_launch(jf_engine* e, const float* d_pos, const int32_t* d_mat, const float* d_fib,
                               float* d_glow_slot);
cudaError_t jf_rows_launch(jf_engine* e, const double* d_before, const double* d_after, double* d_rows);

// Fitness of every instance from (M, 5) rows on the device (FP64).
cudaError_t jf_fitness_launch(jf_engine* e, const double* d_rows, const int32_t* d_muscle,
                              const double* d_contraction, int mode, double* d_out);

// Differentiable rollout (jf_grad.cu).
cudaError_t jf_grad_forward_impl(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode,
                                 const double* inv_n);
cudaError_t jf_grad_backward_impl(jf_engine* e, double* gparam_host);
cudaError_t jf_grad_step_impl(jf_engine* e, int64_t steps, int32_t K, const int32_t* body_mode,
                              const double* inv_n, double* gparam_host);
cudaError_t jf_grad_x0_impl(jf_engine* e, int m, std::vector<float4>& out);
bool jf_grad_done(const jf_engine* e, int stage);
void jf_grad_free(jf_engine* e);
// The rollout's loss sums into e->d_stats (from the FP64 final state in the FP64 build).
cudaError_t jf_grad_loss_stats(jf_engine* e);

// CoM sums of every instance into e->d_stats (M x 6 doubles).
cudaError_t jf_stats_launch(jf_engine* e);

// Kernels used by the C-ABI for loading, reading and writing particles.
cudaError_t jf_load_launch(jf_engine* e, int m, int32_t n);
// Copies instance m's glow into slot order at d_stage + 4 * max_slots.
cudaError_t jf_glow_to_slot_order(jf_engine* e, int m);
// Headless renderer (jf_render.cu): the reference's render kernels on e->d_frame.
cudaError_t jf_frame_clear_launch(jf_engine* e, float value);
cudaError_t jf_render_abyss_launch(jf_engine* e, int res_sub, int grid_side, float radius, int water_mode);
cudaError_t jf_render_flat_launch(jf_engine* e, int res_sub, int grid_side, float radius, int material, float r,
                                  float g, float b);
cudaError_t jf_render_overlay_launch(jf_engine* e, int res_sub, int grid_side, float scale);
cudaError_t jf_vorticity_launch(jf_engine* e, float scale);
cudaError_t jf_render_vort_launch(jf_engine* e, int res_sub, int grid_side, float alpha, int style);
cudaError_t jf_tone_map_launch(jf_engine* e);
// Tank fill (jf_tank.cu): water lattice of instance m minus the robot's
// margin, placed after the robot in the load staging; *h_total = kept
// candidates (read back on the engine's stream; valid after a sync).
cudaError_t jf_tank_water_launch(jf_engine* e, int m, const double* d_robot, int n_robot, const double* bbox,
                                 double water_margin, double spacing_div, int32_t* d_scratch,
                                 int64_t scratch_ints, int32_t* h_total);
int64_t jf_tank_scratch_ints(const jf_engine* e, int m, double spacing_div);
