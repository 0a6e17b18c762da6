/*
 * jellyfih.h -- C ABI of the B200 MLS-MPM engine (libjellyfih.so).
 *
 * The engine replaces the Taichi-backed module mpm_sim.py of jellyfih: one
 * handle owns every device buffer for its lifetime, as mpm_sim.py owns its
 * global fields from import (mpm_sim.py:86-142).  Plain pointers and sizes
 * only; host arrays use the reference's field layouts:
 *   positions, velocities, fibres  float[n][2]      (x, v, fiber_dir)
 *   C, F                           float[n][2][2]   row-major
 *   material                       int32[n]         -1 = dead slot
 *   grid_v                         float[nx][ny][2] grid_m float[nx][ny]
 *
 * Every call returns JF_OK (0) or an error code; jf_last_error() gives the
 * message.  A handle is not thread-safe.  Work is queued on the engine's CUDA
 * stream; calls that return host data synchronise that stream.
 */
#ifndef JELLYFIH_H
#define JELLYFIH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JF_OK 0
#define JF_ERR_INVALID 1      /* bad argument, shape or state */
#define JF_ERR_CUDA 2         /* a CUDA call failed */
#define JF_ERR_NONFINITE 3    /* a particle state became NaN/Inf: returned, after their outputs
                                 are written, by jf_sync, jf_run_headless, jf_run_episode,
                                 jf_grad_forward and jf_grad_backward while an instance's flag is
                                 set (jf_error_flags / jf_clear_error_flags); the gradient path
                                 also flags P2G contributions too large for its fixed-point sums
                                 and non-finite adjoint states */
#define JF_ERR_UNSUPPORTED 4  /* configuration outside what the chosen path supports */
#define JF_ERR_TIMEOUT 5      /* jf_sync_timeout: the engine's queued work had not finished
                                 within the limit; it keeps running, the engine stays usable */

#define JF_PATH_PLAIN 0       /* one instance per launch sequence (reference structure) */
#define JF_PATH_BATCHED 1     /* all instances in one persistent cluster launch per chunk */

#define JF_FLAG_GLOW 1u       /* keep the render-only visual_glow field up to date */
#define JF_FLAG_NO_GRAPHS 2u  /* batched: launch every chunk directly instead of replaying a CUDA graph */
#define JF_FLAG_AXISYM 4u     /* axisymmetric (r, z) substep, JELLY_AXISYM=1 (mpm_sim.py:17,163-165,
                                 235-268,292-303): r-weighted P2G, hoop-stress correction, v_r = 0
                                 on the axis; the differentiable rollout does not support it */
#define JF_FLAG_GRAD_FP64 8u  /* the differentiable rollout (jf_grad_*) in FP64: the same kernels
                                 built for double, every constant the reference's Python double,
                                 P2G summed with double atomics; the state is widened from the
                                 engine's FP32 particles and the final state written back rounded
                                 to FP32.  Stepping (jf_step etc.) stays FP32 */

typedef struct jf_engine jf_engine;

/* One simulation instance: slot capacity and grid (mpm_sim.py:11-19). */
typedef struct {
  int32_t n_slots;        /* particle slots (n_particles) */
  int32_t n_grid;         /* grid nodes along x (n_grid; dx = 1 / n_grid) */
  int32_t n_grid_y;       /* grid nodes along y (n_grid_y) */
  float domain_height;    /* physical height of the tank (domain_height) */
} jf_instance_desc;

typedef struct {
  int32_t n_instances;                  /* n_instances */
  const jf_instance_desc* instances;    /* n_instances entries */
  double dt;                            /* substep (mpm_sim.py:19), 0 = 2e-5 */
  int32_t path;                         /* JF_PATH_* */
  uint32_t flags;                       /* JF_FLAG_* */
  int32_t device;                       /* CUDA device ordinal */
  int32_t resort_interval;              /* batched: substeps between re-sorts, 0 = 64 */
  int32_t block_threads;                /* batched: threads per CTA (multiple of 32, <= 768); above
                                           512 the cell lanes keep their node blocks in tensor
                                           memory (TMEM), up to 512 in registers.  0 = 768 when the
                                           tallest instance's bands hold >= 32 rows
                                           (ceil(n_grid_y / cluster size)), else 512 */
  int32_t cluster_size;                 /* batched: CTAs per instance (1..16), 0 = automatic */
  int32_t cell_cap;                     /* batched: particles a cell lane accumulates per substep;
                                           the rest of the cell goes through per-particle atomics.
                                           0 = chosen per instance at every re-sort, >= 16 = no cap */
} jf_config;

/* Engine life cycle.  Replaces the import-time allocation of mpm_sim.py:86-149;
 * per-instance parameters start at the reference defaults (actuation 500,
 * contraction 0.2, frequency multiplier 1.0, payload density 2.5). */
int jf_create(const jf_config* cfg, jf_engine** out);
int jf_destroy(jf_engine* e);
/* Message of the engine's last failure; with e == NULL, of the calling
 * thread's last failed call made without a handle (jf_create,
 * jf_substep_noalloc, or any call given a NULL handle).  The pointer stays valid until that engine's, or that
 * thread's, next failure. */
const char* jf_last_error(const jf_engine* e);
const char* jf_version(void);

/* Stream the engine queues work on (a cudaStream_t); NULL restores the
 * engine's own stream. */
int jf_set_stream(jf_engine* e, void* stream);

/* Reset instance `m` from host arrays of n <= n_slots particles
 * (load_particles / _load_particles_kernel, mpm_sim.py:715-736): x, material
 * and fibre from the arrays (fiber == NULL gives (0, 1)), v = 0, F = I, C = 0,
 * Jp = 1; slots n..n_slots-1 become dead. */
int jf_load_instance(jf_engine* e, int32_t m, const float* pos, const int32_t* material,
                     const float* fiber, int32_t n);

/* Per-instance parameters, host arrays of n_instances floats; NULL leaves a
 * parameter unchanged (instance_actuation, instance_act_contraction,
 * instance_freq, instance_payload_density; mpm_sim.py:116-149). */
int jf_set_params(jf_engine* e, const float* actuation, const float* contraction,
                  const float* freq, const float* payload_density);
int jf_get_params(const jf_engine* e, float* actuation, float* contraction, float* freq,
                  float* payload_density);

/* sim_time[None] (mpm_sim.py:95), an FP32 running sum advanced by dt per substep. */
int jf_set_time(jf_engine* e, float t);
int jf_get_time(const jf_engine* e, float* t);

/* n substeps of every instance (n calls of substep(), mpm_sim.py:153-340). */
int jf_step(jf_engine* e, int64_t n_steps);
int jf_sync(jf_engine* e);

/* jf_sync with a watchdog limit: waits at most timeout_ms milliseconds for
 * the work queued on the engine's stream (jf_step returns once its launches
 * are queued; ti.sync(), run_population.py:37,47,73, is the reference's
 * unbounded wait).  JF_ERR_TIMEOUT if it has not finished by then: nothing is
 * cancelled, the work runs on, and a later jf_sync or jf_sync_timeout waits
 * for it.  Otherwise the same as jf_sync. */
int jf_sync_timeout(jf_engine* e, int64_t timeout_ms);

/* get_payload_stats (mpm_sim.py:764-777): out[n_instances][3] =
 * [com_y, com_x, count] of the payload (material 2), zeros without payload.
 * Sums are accumulated on the GPU in FP64. */
int jf_payload_stats(jf_engine* e, double* out);

/* _get_stats_any (mpm_sim.py:779-800): payload CoM where present, else the
 * CoM of jelly + muscle (materials 1 and 3). */
int jf_stats_any(jf_engine* e, double* out);

/* The FP64 sums behind the CoM (clear_fitness_buffer + compute_payload_stats
 * / compute_body_stats, mpm_sim.py:740-762): out[n_instances][6] =
 * [payload sum_y, payload count, payload sum_x, body sum_y, body count,
 * body sum_x], body = materials 1 and 3. */
int jf_stats_raw(jf_engine* e, double* out);

/* run_batch_headless (mpm_sim.py:802-834): time reset to 0, CoM before,
 * `steps` substeps, CoM after; out[n_instances][5] = [init_y, init_x,
 * final_y, final_x, valid] with valid = final_y >= 0.01. */
int jf_run_headless(jf_engine* e, int64_t steps, double* out);

/* Fitness of every instance from run_headless rows, computed on the GPU in
 * FP64 (evolve.py:90-124 compute_fitness): invalid when valid == 0 or
 * muscle_counts[m] < 200; displacement = min(final_y, domain_height - 0.07)
 * - init_y; mode 0 (efficiency) scores -displacement / sqrt(muscle_counts[m]
 * * clip(contraction[m], 0.05, 0.60) / 500) (contraction NULL: 0.20), mode 1
 * (displacement) scores -displacement; invalid instances get the worst valid
 * score + 1, or 100 when none is valid.  results: host [n_instances][5],
 * muscle_counts, contraction (gene 9, unclipped): host [n_instances], out:
 * host [n_instances]. */
int jf_fitness(jf_engine* e, const double* results, const int32_t* muscle_counts,
               const double* contraction, int32_t mode, double* out);

/* One evaluation episode of every instance with a single host round trip,
 * the loop body of evolve.py:127-155 and 90-124: load_particles for every
 * instance (mpm_sim.py:715-736), instance_act_contraction / instance_freq
 * set, run_batch_headless(steps) (:802-834), then compute_fitness on the GPU.
 * pos [total slots][2], material [total slots], fiber [total slots][2] (NULL:
 * (0, 1)) hold the instances' slot arrays back to back (instance m's
 * n_slots entries after those of instances 0 .. m-1; material -1 = empty
 * slot).  contraction, freq: [n_instances] (freq NULL keeps the current
 * values).  rows: [n_instances][5] as jf_run_headless.  muscle_counts NULL
 * skips the fitness; else fitness [n_instances] as jf_fitness in `mode`
 * with contraction as the gene.  One synchronisation at the end. */
int jf_run_episode(jf_engine* e, const float* pos, const int32_t* material, const float* fiber,
                   const float* contraction, const float* freq, int64_t steps,
                   const int32_t* muscle_counts, int32_t mode, double* rows, double* fitness);

/* Differentiable rollout.  jf_grad_forward runs `steps` substeps from the
 * current state with a deterministic P2G, checkpointing (x, v, C, F) every
 * `checkpoint_every` substeps, and returns loss[m] = the displacement of the
 * payload CoM height (jelly + muscle without payload) over the rollout, the
 * quantity evolve.py's fitness is built from (evolve.py:101).  jf_grad_backward
 * then returns d loss / d instance_actuation, instance_act_contraction and
 * instance_freq (host arrays, NULL to skip; the refractory fraction is
 * 1 - contraction, so its gradient is minus the contraction's), and
 * jf_grad_positions the gradient w.r.t. instance m's initial positions in slot
 * order ([n_slots][2]).  The waveform's drop from 1 to 0 when the phase
 * reaches the contraction fraction (mpm_sim.py:176-180) is differentiated as
 * the boundary term of the time integral: each drop inside the rollout adds
 * actuation * g / (freq * dt) to d/d contraction and minus that times the
 * drop's time to d/d freq, g being d loss / d pressure at the drop.  The
 * reference engine has no gradients; this replaces nothing in it.  The engine
 * is left at the rollout's final state, and so is it after jf_grad_backward,
 * which recomputes the rollout from its checkpoints and puts that final
 * particle state back (a state loaded or stepped in between is replaced; the
 * time is not changed).  jf_grad_backward needs a completed forward, and
 * jf_grad_positions the backward of the latest rollout (a new
 * jf_grad_forward discards the previous rollout's adjoint); otherwise they
 * return JF_ERR_INVALID. */
int jf_grad_forward(jf_engine* e, int64_t steps, int32_t checkpoint_every, double* loss);
int jf_grad_backward(jf_engine* e, double* d_actuation, double* d_contraction, double* d_freq);
int jf_grad_positions(jf_engine* e, int32_t m, float* dx0);
/* jf_grad_forward followed by jf_grad_backward with one host round trip
 * between none of their device work: both run as one CUDA graph, captured on
 * the first call and replayed while the sizes, start time and buffers are
 * unchanged (the gradient-refinement loop: every step restarts from time 0).
 * jf_grad_forward / jf_grad_backward each replay a graph of their own the
 * same way.  With JF_FLAG_NO_GRAPHS, or while kernel timing is on, the work
 * is launched directly.  Outputs as the two calls'; jf_grad_positions works
 * after it. */
int jf_grad_step(jf_engine* e, int64_t steps, int32_t checkpoint_every, double* loss, double* d_actuation,
                 double* d_contraction, double* d_freq);

/* Particle fields of instance m in slot order (field.to_numpy()); any
 * pointer may be NULL.  x, v, fiber: [n_slots][2]; C, F: [n_slots][4]. */
int jf_read_particles(jf_engine* e, int32_t m, float* x, float* v, float* C, float* F,
                      int32_t* material, float* Jp, float* glow, float* fiber);

/* Overwrite particle fields of instance m from slot-order host arrays
 * (field.from_numpy()); NULL leaves a field unchanged. */
int jf_write_particles(jf_engine* e, int32_t m, const float* x, const float* v, const float* C,
                       const float* F, const float* Jp, const float* glow);

/* grid_v / grid_m of instance m after the last substep (mpm_sim.py:92-93):
 * grid_v[nx][ny][2], grid_m[nx][ny]; either may be NULL. */
int jf_read_grid(jf_engine* e, int32_t m, float* grid_v, float* grid_m);

/* Load instance m from its robot alone, with the water filled on the GPU
 * (make_jelly.py:336-402, fill_tank with no jitter): slots hold the robot
 * particles (positions rounded to float), then the water lattice of spacing
 * 1 / (n_grid * spacing_div) between 3/(2 n_grid) of the walls, without every
 * lattice point within water_margin of a robot particle, in lattice order
 * (y outer, x inner); water beyond the slots is cut (the robot first, as the
 * reference truncates), the rest dead.  Then the load reset of
 * jf_load_instance.  robot_pos [n_robot][2] doubles; robot_fiber may be NULL
 * (0, 1); out_counts (may be NULL) = {robot particles kept, water particles}. */
int jf_load_robot(jf_engine* e, int32_t m, const double* robot_pos, const int32_t* robot_mat,
                  const float* robot_fiber, int32_t n_robot, double water_margin, double spacing_div,
                  int32_t* out_counts);

/* Overwrite grid_v / grid_m of instance m (grid_v.from_numpy, grid_m.from_numpy;
 * layouts as jf_read_grid).  The next substep recomputes the grid from the
 * particles, so this feeds the renderer and vorticity calls below. */
int jf_write_grid(jf_engine* e, int32_t m, const float* grid_v, const float* grid_m);

/* ---- Headless renderer (mpm_sim.py:343-712) --------------------------------
 * The reference's render kernels into a device frame buffer owned by the
 * engine (frame_buffer, mpm_sim.py:96); no graphics API is involved.  The
 * frame holds video_res x video_res RGB floats; instance m draws into tile
 * (m / grid_side, m % grid_side) of res_sub pixels.  Launches are queued on
 * the engine's stream; jf_read_frame / jf_read_vorticity synchronise. */
#define JF_VORT_RDBU 0      /* render_vorticity_rdbu (mpm_sim.py:582-625) */
#define JF_VORT_HUESHIFT 1  /* render_vorticity_hueshift (mpm_sim.py:628-670) */
#define JF_VORT_WHITE 2     /* render_vorticity_white (mpm_sim.py:673-711) */

/* (Re)allocate the frame (video_res x video_res) and clear it to 0. */
int jf_frame_create(jf_engine* e, int32_t video_res);
/* clear_frame_buffer (value 0, mpm_sim.py:361-364) / clear_frame_buffer_white
 * (0.98, mpm_sim.py:483-486). */
int jf_frame_clear(jf_engine* e, float value);
/* render_frame_abyss (mpm_sim.py:385-481): additive splats of radius
 * 1.5 * radius, coloured by material; hue / muscle_hue are the per-instance
 * instance_hue / instance_muscle_hue [n_instances]; water_mode is
 * water_angle_color (0 ghost, 1 plain, else rainbow).  Uses sim_time and the
 * per-instance waveform parameters for the muscle colour. */
int jf_render_abyss(jf_engine* e, int32_t res_sub, int32_t grid_side, float radius, const float* hue,
                    const float* muscle_hue, int32_t water_mode);
/* render_flat_pass (mpm_sim.py:489-517): discs of one material in one colour. */
int jf_render_flat(jf_engine* e, int32_t res_sub, int32_t grid_side, float radius, int32_t material, float r,
                   float g, float b);
/* render_vorticity_overlay (mpm_sim.py:520-558): additive curl squares from
 * the last substep's grid. */
int jf_render_vorticity_overlay(jf_engine* e, int32_t res_sub, int32_t grid_side, float vort_scale);
/* compute_vorticity_grid (mpm_sim.py:561-579): tanh(curl * vort_scale) per node. */
int jf_compute_vorticity(jf_engine* e, float vort_scale);
/* render_vorticity_rdbu / _hueshift / _white (style JF_VORT_*): blends the
 * vorticity grid over the frame (white: over a white clear). */
int jf_render_vorticity(jf_engine* e, int32_t res_sub, int32_t grid_side, float alpha, int32_t style);
/* tone_map_and_encode (mpm_sim.py:366-383). */
int jf_tone_map(jf_engine* e);
/* frame_buffer.to_numpy(): rgb[video_res][video_res][3], row = frame row py. */
int jf_read_frame(jf_engine* e, float* rgb);
/* vort_grid of instance m (mpm_sim.py:106): vort[nx][ny]. */
int jf_read_vorticity(jf_engine* e, int32_t m, float* vort);

/* Per-instance non-finite flags raised by the G2P update since the last
 * clear (out[n_instances]). */
int jf_error_flags(jf_engine* e, int32_t* out);
int jf_clear_error_flags(jf_engine* e);

/* Batched path counters since the last reset (out has 4 entries): out[0]
 * particle scatters accumulated in a lane's register block, out[1] scatters
 * through per-particle atomics (drifted or out-of-range particles), out[2] G2P
 * gathers outside the CTA's shared-memory window, out[3] particles beyond
 * their cell's per-lane cap, handed to the CTA's balanced overflow pass
 * (per-particle atomics).  All zero on the plain path. */
int jf_path_counts(jf_engine* e, int64_t* out, int32_t reset);

/* The batched launch layout the engine chose: CTAs per instance (cluster
 * size) and threads per CTA.  Either pointer may be NULL.  No counterpart in
 * the reference (its launch layout is Taichi's). */
int jf_get_layout(const jf_engine* e, int32_t* cluster_size, int32_t* block_threads);

/* Largest grid, in nodes (n_grid * n_grid_y), jf_substep_noalloc accepts. */
#define JF_NOALLOC_MAX_NODES 32768

/* One substep of one instance that allocates no device memory.
 *
 * No counterpart in the reference: it serves callers that cannot call
 * cudaMalloc when they step (allocators or memory pools that must not grow,
 * host callbacks, embedders that own all device memory).  The caller passes
 * device pointers in the reference's layouts -- x, v, fiber [n][2]; C, F
 * [n][2][2] row-major; material, Jp, glow [n] -- and advances sim_time by dt
 * itself; fiber NULL means (0, 1), glow NULL skips the render-only glow.
 * x, v, fiber must be 8-byte and C, F 16-byte aligned.  The grid scratch is a
 * file-scope device array of JF_NOALLOC_MAX_NODES float4 nodes (512 KiB) that
 * every GPU loading the library holds until exit; larger grids are rejected
 * with JF_ERR_UNSUPPORTED.  Every call looks the array's address up
 * (cudaGetSymbolAddress, which allocates nothing) in the CUDA context current
 * on the calling thread, so a device reset or another context on the same
 * device is followed; the first call on a device may load the library's device
 * code, so make that first call before any stream capture.  All calls share
 * the array and each call clears the nodes it uses; calls that overlap on the
 * GPU race.  A state that turns NaN or Inf is not reported by this entry point
 * (the engine's jf_error_flags do not see it): check the outputs where that
 * matters.  Work is queued on `stream` (a cudaStream_t, NULL = legacy default
 * stream). */
int jf_substep_noalloc(int32_t n, int32_t n_grid, int32_t n_grid_y, float domain_height, double dt,
                       float sim_time, float actuation, float contraction, float freq,
                       float payload_density, float* x, float* v, float* C, float* F,
                       const int32_t* material, float* Jp, float* glow, const float* fiber,
                       void* stream);

/* Number of kernels this engine has launched. */
int64_t jf_kernel_launches(const jf_engine* e);

/* Kernel timing with CUDA events on the engine's stream.  While enabled, every
 * step-kernel launch is bracketed by events; jf_kernel_timing synchronises and
 * returns the summed device time (ms) and launch counts of the step kernels
 * (batched chunk kernel, or the plain P2G / grid / G2P kernels) and of the
 * batched re-sort kernels, accumulated since timing was enabled. */
int jf_set_kernel_timing(jf_engine* e, int32_t enable);
int jf_kernel_timing(jf_engine* e, double* step_ms, int64_t* step_launches, double* sort_ms,
                     int64_t* sort_launches);

#ifdef __cplusplus
}
#endif

#endif /* JELLYFIH_H */
