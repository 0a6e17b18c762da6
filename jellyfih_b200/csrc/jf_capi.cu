// C-ABI entry points of libjellyfih.so (declared in include/jellyfih.h).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "jf_engine.h"

cudaError_t jf_batched_prepare(jf_engine* e);
int jf_batched_max_active_clusters(jf_engine* e, int cluster, int* out);

namespace {

// message of the last failed call without a handle, per host thread, so that
// the pointer jf_last_error(NULL) returns stays valid while other threads fail
thread_local std::string g_create_err;

constexpr int kHaloRows = 4;  // batched window rows beyond the band (1 below, 3 above)
constexpr size_t kMaxSmem = 227 * 1024;
constexpr size_t kStaticSmem = 1024;  // the chunk kernel's static shared variables, rounded up
constexpr size_t kBandSlackSmem = 128 * 1024;  // window size up to which bands get spare rows

int fail(jf_engine* e, int code, const std::string& msg) {
  if (e) e->err = msg;
  return code;
}

int cuda_fail(jf_engine* e, cudaError_t err, const char* what) {
  std::string msg = std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")";
  return fail(e, JF_ERR_CUDA, msg);
}

#define JF_CK(call, what)                                   \
  do {                                                      \
    cudaError_t _err = (call);                              \
    if (_err != cudaSuccess) return cuda_fail(e, _err, what); \
  } while (0)

template <class T>
cudaError_t alloc(T** p, size_t n) {
  return cudaMalloc((void**)p, sizeof(T) * (n > 0 ? n : 1));
}

cudaError_t alloc_particles(JfParticles& p, size_t n) {
  cudaError_t err;
  if ((err = alloc(&p.xv, n)) != cudaSuccess) return err;
  if ((err = alloc(&p.C, n)) != cudaSuccess) return err;
  if ((err = alloc(&p.F, n)) != cudaSuccess) return err;
  if ((err = alloc(&p.mat, n)) != cudaSuccess) return err;
  if ((err = alloc(&p.fiber, n)) != cudaSuccess) return err;
  if ((err = alloc(&p.Jp, n)) != cudaSuccess) return err;
  if ((err = alloc(&p.glow, n)) != cudaSuccess) return err;
  if ((err = alloc(&p.slot, n)) != cudaSuccess) return err;
  if ((err = alloc(&p.rref, n)) != cudaSuccess) return err;
  return cudaSuccess;
}

void free_particles(JfParticles& p) {
  cudaFree(p.xv); cudaFree(p.C); cudaFree(p.F); cudaFree(p.mat);
  cudaFree(p.fiber); cudaFree(p.Jp); cudaFree(p.glow); cudaFree(p.slot); cudaFree(p.rref);
  p = JfParticles();
}

// A call on a NULL handle fails with the thread's handle-less message set.
int check_engine(const jf_engine* e) {
  if (e) return JF_OK;
  jf_set_global_error("NULL engine handle");
  return JF_ERR_INVALID;
}

// JF_ERR_INVALID, with a message naming them, when required pointers are NULL.
int need_args(jf_engine* e, bool present, const char* what) {
  return present ? JF_OK : fail(e, JF_ERR_INVALID, std::string(what) + " must not be NULL");
}

int set_device(jf_engine* e) {
  JF_CK(cudaSetDevice(e->device), "cudaSetDevice");
  return JF_OK;
}

int upload_params(jf_engine* e) {
  if (!e->params_dirty) return JF_OK;
  JF_CK(cudaMemcpyAsync(e->d_params, e->params.data(), sizeof(JfParams) * e->M,
                        cudaMemcpyHostToDevice, e->stream),
        "upload params");
  JF_CK(cudaStreamSynchronize(e->stream), "upload params sync");
  e->params_dirty = false;
  return JF_OK;
}

// The batched path's clusters take instances in descending live count
// (e->n_live), so that the longest run first when the clusters do not all
// fit at once: re-sorts the order and queues its upload.
int upload_order(jf_engine* e) {
  if (!e->d_order) return JF_OK;
  for (int q = 0; q < e->M; ++q) e->h_order[q] = q;
  std::stable_sort(e->h_order.begin(), e->h_order.end(),
                   [&](int32_t a, int32_t b) { return e->n_live[a] > e->n_live[b]; });
  JF_CK(cudaMemcpyAsync(e->d_order, e->h_order.data(), sizeof(int32_t) * e->M, cudaMemcpyHostToDevice, e->stream),
        "cluster order");
  return JF_OK;
}

// Live count of instance m after a load, and the cluster order with it.
int set_live_count(jf_engine* e, int m, int32_t live) {
  if (!e->d_order) return JF_OK;
  e->n_live[m] = live;
  return upload_order(e);
}

// Instance m's particle arrays in engine order, copied to the host.
struct HostInstance {
  std::vector<float4> xv, C, F;
  std::vector<int32_t> mat, slot;
  std::vector<float2> fiber;
  std::vector<float> Jp, glow;
};

int download_instance(jf_engine* e, int m, HostInstance& h) {
  const JfInst& I = e->inst[m];
  const size_t n = (size_t)I.n_slots;
  h.xv.resize(n); h.C.resize(n); h.F.resize(n); h.mat.resize(n); h.slot.resize(n);
  h.fiber.resize(n); h.Jp.resize(n); h.glow.resize(n);
  if (n == 0) return JF_OK;
  const int64_t o = I.p_off;
  JF_CK(cudaMemcpyAsync(h.xv.data(), e->p.xv + o, n * sizeof(float4), cudaMemcpyDeviceToHost, e->stream), "read xv");
  JF_CK(cudaMemcpyAsync(h.C.data(), e->p.C + o, n * sizeof(float4), cudaMemcpyDeviceToHost, e->stream), "read C");
  JF_CK(cudaMemcpyAsync(h.F.data(), e->p.F + o, n * sizeof(float4), cudaMemcpyDeviceToHost, e->stream), "read F");
  JF_CK(cudaMemcpyAsync(h.mat.data(), e->p.mat + o, n * sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream), "read mat");
  JF_CK(cudaMemcpyAsync(h.slot.data(), e->p.slot + o, n * sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream), "read slot");
  JF_CK(cudaMemcpyAsync(h.fiber.data(), e->p.fiber + o, n * sizeof(float2), cudaMemcpyDeviceToHost, e->stream), "read fiber");
  JF_CK(cudaMemcpyAsync(h.Jp.data(), e->p.Jp + o, n * sizeof(float), cudaMemcpyDeviceToHost, e->stream), "read Jp");
  JF_CK(cudaMemcpyAsync(h.glow.data(), e->p.glow + o, n * sizeof(float), cudaMemcpyDeviceToHost, e->stream), "read glow");
  JF_CK(cudaStreamSynchronize(e->stream), "read particles sync");
  for (size_t k = 0; k < n; ++k) {
    if (h.slot[k] < 0 || (size_t)h.slot[k] >= n) return fail(e, JF_ERR_CUDA, "corrupt slot permutation");
  }
  return JF_OK;
}

int upload_instance(jf_engine* e, int m, const HostInstance& h) {
  const JfInst& I = e->inst[m];
  const size_t n = (size_t)I.n_slots;
  if (n == 0) return JF_OK;
  const int64_t o = I.p_off;
  JF_CK(cudaMemcpyAsync(e->p.xv + o, h.xv.data(), n * sizeof(float4), cudaMemcpyHostToDevice, e->stream), "write xv");
  JF_CK(cudaMemcpyAsync(e->p.C + o, h.C.data(), n * sizeof(float4), cudaMemcpyHostToDevice, e->stream), "write C");
  JF_CK(cudaMemcpyAsync(e->p.F + o, h.F.data(), n * sizeof(float4), cudaMemcpyHostToDevice, e->stream), "write F");
  JF_CK(cudaMemcpyAsync(e->p.Jp + o, h.Jp.data(), n * sizeof(float), cudaMemcpyHostToDevice, e->stream), "write Jp");
  JF_CK(cudaMemcpyAsync(e->p.glow + o, h.glow.data(), n * sizeof(float), cudaMemcpyHostToDevice, e->stream), "write glow");
  JF_CK(cudaStreamSynchronize(e->stream), "write particles sync");
  return JF_OK;
}

int stats_rows(jf_engine* e, double* out, bool any) {
  JF_CK(jf_stats_launch(e), "stats kernel");
  std::vector<double> raw(6 * (size_t)e->M);
  JF_CK(cudaMemcpyAsync(raw.data(), e->d_stats, sizeof(double) * raw.size(), cudaMemcpyDeviceToHost,
                        e->stream),
        "read stats");
  JF_CK(cudaStreamSynchronize(e->stream), "stats sync");
  for (int m = 0; m < e->M; ++m) {
    const double* r = &raw[6 * (size_t)m];
    if (any && r[1] == 0) r = r + 3;  // body CoM fallback (mpm_sim.py:786-792)
    double* o = out + 3 * (size_t)m;
    if (r[1] > 0) {
      o[0] = r[0] / r[1];
      o[1] = r[2] / r[1];
      o[2] = r[1];
    } else {
      o[0] = o[1] = o[2] = 0.0;
    }
  }
  return JF_OK;
}

int step_impl(jf_engine* e, int64_t n) {
  if (n < 0) return fail(e, JF_ERR_INVALID, "n_steps must be >= 0");
  if (n == 0) return JF_OK;
  int rc = set_device(e);
  if (rc) return rc;
  rc = upload_params(e);
  if (rc) return rc;
  cudaError_t err = (e->path == JF_PATH_BATCHED) ? jf_batched_step(e, n) : jf_plain_step(e, n);
  if (err != cudaSuccess) return cuda_fail(e, err, "step");
  return JF_OK;
}

// Folds recorded event pairs into the totals and returns the events to the pool.
cudaError_t collect_timing(jf_engine* e) {
  cudaError_t first = cudaSuccess;
  for (int which = 0; which < 2; ++which) {
    auto& list = which ? e->sort_events : e->step_events;
    for (auto& pr : list) {
      float ms = 0.0f;
      cudaError_t err = cudaEventElapsedTime(&ms, pr.first, pr.second);
      if (err != cudaSuccess && first == cudaSuccess) first = err;
      (which ? e->sort_ms : e->step_ms) += ms;
      (which ? e->sort_launches : e->step_launches) += 1;
      e->event_pool.push_back(pr.first);
      e->event_pool.push_back(pr.second);
    }
    list.clear();
  }
  return first;
}

}  // namespace

void jf_set_global_error(const std::string& msg) { g_create_err = msg; }

static cudaEvent_t pool_event(jf_engine* e) {
  if (!e->event_pool.empty()) {
    cudaEvent_t ev = e->event_pool.back();
    e->event_pool.pop_back();
    return ev;
  }
  cudaEvent_t ev = nullptr;
  cudaEventCreate(&ev);
  return ev;
}

JfTimed::JfTimed(jf_engine* eng, bool sort, bool skip)
    : e(eng), list(sort ? &eng->sort_events : &eng->step_events), off(skip) {
  if (!e->timing || off) return;
  a = pool_event(e);
  b = pool_event(e);
  cudaEventRecord(a, e->stream);
}

JfTimed::~JfTimed() {
  if (!e->timing || off || !a) return;
  cudaEventRecord(b, e->stream);
  list->push_back({a, b});
}

extern "C" {

const char* jf_version(void) { return "jellyfih-b200 0.1"; }

const char* jf_last_error(const jf_engine* e) {
  if (e) return e->err.c_str();
  return g_create_err.c_str();
}

int jf_create(const jf_config* cfg, jf_engine** out) {
  if (!out) return JF_ERR_INVALID;
  *out = nullptr;
  if (!cfg || cfg->n_instances <= 0 || !cfg->instances) {
    jf_set_global_error("config needs n_instances > 0 and an instance table");
    return JF_ERR_INVALID;
  }
  if (cfg->path != JF_PATH_PLAIN && cfg->path != JF_PATH_BATCHED) {
    jf_set_global_error("unknown path");
    return JF_ERR_INVALID;
  }
  jf_engine* e = new jf_engine();
  e->device = cfg->device;
  e->M = cfg->n_instances;
  e->dt = cfg->dt > 0 ? cfg->dt : 2e-5;
  e->path = cfg->path;
  e->flags = cfg->flags;
  e->resort_interval = cfg->resort_interval > 0 ? cfg->resort_interval : 64;
  e->block_threads = cfg->block_threads;  // 0: chosen below, once the cluster size is known
  e->cell_cap = cfg->cell_cap;
  e->use_graphs = (cfg->flags & JF_FLAG_NO_GRAPHS) == 0;
  auto bail = [&](int code, const std::string& msg) {
    jf_set_global_error(msg);
    jf_destroy(e);
    return code;
  };
  if (cfg->cell_cap < 0) return bail(JF_ERR_INVALID, "cell_cap must be >= 0");
  if (e->block_threads < 0 || e->block_threads > 768 || e->block_threads % 32)
    return bail(JF_ERR_INVALID, "block_threads must be 0 or a multiple of 32, <= 768");

  int ny_max = 0;
  for (int m = 0; m < e->M; ++m) {
    const jf_instance_desc& d = cfg->instances[m];
    if (d.n_slots < 0 || d.n_grid < 8 || d.n_grid_y < 8 || !(d.domain_height > 0))
      return bail(JF_ERR_INVALID, "instance " + std::to_string(m) + ": bad n_slots / n_grid / domain_height");
    ny_max = std::max(ny_max, (int)d.n_grid_y);
  }

  int rc = set_device(e);
  if (rc) return bail(rc, e->err);
  int n_sm = 148;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, e->device);

  // cluster size: grow while the launch still fits the SMs and bands keep >= 8 rows
  e->cluster = 4;
  if (cfg->cluster_size > 0) {
    if (cfg->cluster_size > 16) return bail(JF_ERR_INVALID, "cluster_size must be <= 16");
    e->cluster = cfg->cluster_size;
  } else if (e->path == JF_PATH_BATCHED) {
    while (e->cluster < 16 && (int64_t)e->M * e->cluster * 2 <= n_sm &&
           (ny_max + e->cluster * 2 - 1) / (e->cluster * 2) >= 8)
      e->cluster *= 2;
  }
  // CTA size: 24 warps (node blocks in TMEM) when a band has rows enough to
  // keep them busy to the end of a pass (32 rows = 128 cell tasks of 32 cells
  // on 128^2), else 16 warps (node blocks in registers): measured, 32-row
  // bands run 4 % faster at 768 threads, 16-row bands 16 % slower
  if (e->block_threads == 0) e->block_threads = (ny_max + e->cluster - 1) / e->cluster >= 32 ? 768 : 512;

  int64_t p_off = 0, g_off = 0;
  for (int m = 0; m < e->M; ++m) {
    const jf_instance_desc& d = cfg->instances[m];
    JfInst I = {};
    const double nx = d.n_grid;
    const double dx_d = 1.0 / nx;
    const double p_vol = (dx_d * 0.5) * (dx_d * 0.5);
    I.nx = d.n_grid;
    I.ny = d.n_grid_y;
    I.dcx = d.n_grid / 20;
    I.dcy = d.n_grid_y / 20;
    I.band_h = (d.n_grid_y + e->cluster - 1) / e->cluster;
    I.n_slots = d.n_slots;
    I.p_off = p_off;
    I.g_off = g_off;
    I.inv_dx = (float)nx;
    I.dx = (float)dx_d;
    I.dt = (float)e->dt;
    I.p_mass = (float)(p_vol * 1);
    I.stress_scale = (float)(-e->dt * p_vol * 4 * nx * nx);
    I.c4 = (float)(4 * nx);
    I.dtg = (float)(e->dt * 10.0);
    I.y_hi = (float)((double)d.domain_height - 0.001);
    I.rref_lo = (float)(dx_d * 0.1);
    I.r_lo = (float)(dx_d * 0.05);
    I.axisym = (cfg->flags & JF_FLAG_AXISYM) ? 1 : 0;
    I.domain_h = (double)d.domain_height;
    e->inst.push_back(I);
    JfParams P = {500.0f, 0.20f, 1.0f, 2.5f};  // mpm_sim.py:143-149
    e->params.push_back(P);
    p_off += d.n_slots;
    g_off += (int64_t)d.n_grid * d.n_grid_y;
    e->max_slots = std::max(e->max_slots, d.n_slots);
    e->max_cells = std::max(e->max_cells, d.n_grid * d.n_grid_y);
    {
      // the sort may give a band up to 25 % more rows than ceil(ny / CTAs)
      // when that balances the CTAs' work, as long as the window stays within
      // kBandSlackSmem: shared memory and L1 share an SM's 256 KB, and
      // particle loads slow down when the window takes most of it
      const int planes = (cfg->flags & JF_FLAG_AXISYM) ? 6 : 5;
      const long long fit = (long long)kBandSlackSmem / (4LL * planes * d.n_grid) - kHaloRows;
      long long bc = I.band_h + I.band_h / 4;
      bc = std::min(bc, fit);
      bc = std::max<long long>(bc, I.band_h);
      bc = std::min<long long>(bc, d.n_grid_y);
      e->inst.back().band_cap = (int32_t)bc;
    }
    e->win_nodes = std::max(e->win_nodes, (e->inst.back().band_cap + kHaloRows) * d.n_grid);
  }
  e->total_slots = p_off;
  e->total_nodes = g_off;
  if (p_off >= (int64_t)1 << 31) return bail(JF_ERR_UNSUPPORTED, "more than 2^31 particle slots");
  if (e->path == JF_PATH_BATCHED && jf_batched_smem_bytes(e) > kMaxSmem - kStaticSmem)
    return bail(JF_ERR_UNSUPPORTED, "grid band does not fit in shared memory (n_grid * rows too large)");

  if (!e->stream) {
    cudaError_t err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) return bail(JF_ERR_CUDA, "cudaStreamCreate failed");
    e->own_stream = true;
  }
  cudaError_t err = cudaSuccess;
  if ((err = alloc_particles(e->p, p_off)) != cudaSuccess ||
      (err = alloc(&e->d_inst, e->M)) != cudaSuccess ||
      (err = alloc(&e->d_params, e->M)) != cudaSuccess ||
      (err = alloc(&e->d_grid, g_off)) != cudaSuccess ||
      (err = alloc(&e->d_stats, 6 * (size_t)e->M)) != cudaSuccess ||
      (err = alloc(&e->d_err, e->M)) != cudaSuccess ||
      (err = alloc(&e->d_stage, 8 * (size_t)e->max_slots)) != cudaSuccess ||
      (err = alloc(&e->d_stage_i, 2 * (size_t)e->max_slots)) != cudaSuccess ||
      (err = alloc(&e->d_fit, 6 * (size_t)e->M)) != cudaSuccess ||
      (err = alloc(&e->d_fit_f, e->M)) != cudaSuccess ||
      (err = alloc(&e->d_fit_i, e->M)) != cudaSuccess)
    return bail(JF_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(err));
  if (e->path == JF_PATH_BATCHED) {
    if ((err = alloc_particles(e->q, p_off)) != cudaSuccess ||
        (err = alloc(&e->d_keys, p_off)) != cudaSuccess ||
        (err = alloc(&e->d_rank, p_off)) != cudaSuccess ||
        (err = alloc(&e->d_ovlist, p_off)) != cudaSuccess ||
        (err = alloc(&e->d_ovband, (size_t)(e->cluster + 1) * e->M)) != cudaSuccess ||
        (err = alloc(&e->d_ovcur, (size_t)e->cluster * e->M)) != cudaSuccess ||
        (err = alloc(&e->d_counts, (size_t)(e->max_cells + 2) * e->M)) != cudaSuccess ||
        (err = alloc(&e->d_band, (size_t)(e->cluster + 1) * e->M)) != cudaSuccess ||
        (err = alloc(&e->d_cap, e->M)) != cudaSuccess ||
        (err = alloc(&e->d_order, e->M)) != cudaSuccess ||
        (err = alloc(&e->d_brow, (size_t)(e->cluster + 1) * e->M)) != cudaSuccess ||
        (err = alloc(&e->d_solid, (size_t)kJfMaxBandRows * e->M)) != cudaSuccess ||
        (err = alloc(&e->d_path, 4)) != cudaSuccess ||
        (err = alloc(&e->d_time, 1)) != cudaSuccess ||
        (err = cudaMemset(e->d_path, 0, 4 * sizeof(unsigned long long))) != cudaSuccess)
      return bail(JF_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(err));
    e->n_live.assign(e->M, 0);
    e->h_order.resize(e->M);
    for (int m = 0; m < e->M; ++m) e->h_order[m] = m;
    if ((err = cudaMemcpy(e->d_order, e->h_order.data(), sizeof(int32_t) * e->M, cudaMemcpyHostToDevice)) !=
        cudaSuccess)
      return bail(JF_ERR_CUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(err));
    if ((err = jf_batched_prepare(e)) != cudaSuccess)
      return bail(JF_ERR_CUDA, std::string("kernel attributes: ") + cudaGetErrorString(err));
    int active = 0;
    jf_batched_max_active_clusters(e, e->cluster, &active);
    if (active == 0)
      return bail(JF_ERR_UNSUPPORTED, "clusters of " + std::to_string(e->cluster) + " CTAs cannot be scheduled");
  }
  if (cudaMemcpy(e->d_inst, e->inst.data(), sizeof(JfInst) * e->M, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(e->d_grid, 0, sizeof(float4) * std::max<int64_t>(g_off, 1)) != cudaSuccess ||
      cudaMemset(e->d_err, 0, sizeof(int32_t) * e->M) != cudaSuccess ||
      cudaMemset(e->p.glow, 0, sizeof(float) * std::max<int64_t>(p_off, 1)) != cudaSuccess)
    return bail(JF_ERR_CUDA, "initial upload failed");
  // every slot starts dead: position -1, material -1, F = I, Jp = 1
  {
    std::vector<float> zeros(5 * (size_t)std::max(e->max_slots, 1), 0.0f);
    cudaMemcpy(e->d_stage + 4 * (size_t)e->max_slots, zeros.data(), sizeof(float) * e->max_slots,
               cudaMemcpyHostToDevice);
    for (int m = 0; m < e->M; ++m) {
      if (jf_load_launch(e, m, 0) != cudaSuccess) return bail(JF_ERR_CUDA, "initial reset failed");
    }
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) return bail(JF_ERR_CUDA, "initial reset sync failed");
  }
  e->params_dirty = true;
  *out = e;
  return JF_OK;
}

int jf_destroy(jf_engine* e) {
  if (!e) return JF_ERR_INVALID;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  jf_grad_free(e);
  free_particles(e->p);
  free_particles(e->q);
  cudaFree(e->d_inst); cudaFree(e->d_params); cudaFree(e->d_keys); cudaFree(e->d_counts);
  cudaFree(e->d_rank); cudaFree(e->d_ovlist); cudaFree(e->d_ovband); cudaFree(e->d_ovcur);
  cudaFree(e->d_band); cudaFree(e->d_cap); cudaFree(e->d_order); cudaFree(e->d_brow); cudaFree(e->d_solid); cudaFree(e->d_ep); cudaFree(e->d_ep_mat);
  cudaFree(e->d_ep_stats); cudaFree(e->d_grid); cudaFree(e->d_stats); cudaFree(e->d_err);
  cudaFree(e->d_stage); cudaFree(e->d_stage_i); cudaFree(e->d_path);
  cudaFree(e->d_fit); cudaFree(e->d_fit_f); cudaFree(e->d_fit_i); cudaFree(e->d_time);
  cudaFree(e->d_frame); cudaFree(e->d_vort); cudaFree(e->d_hue);
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  for (auto& pr : e->step_events) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
  for (auto& pr : e->sort_events) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
  for (auto ev : e->event_pool) cudaEventDestroy(ev);
  if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return JF_OK;
}

int jf_set_stream(jf_engine* e, void* stream) {
  if (check_engine(e)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(cudaStreamSynchronize(e->stream), "sync old stream");
  if (stream) {
    if (e->own_stream) cudaStreamDestroy(e->stream);
    e->own_stream = false;
    e->stream = (cudaStream_t)stream;
  } else if (!e->own_stream) {
    JF_CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    e->own_stream = true;
  }
  return JF_OK;
}

int jf_load_instance(jf_engine* e, int32_t m, const float* pos, const int32_t* material,
                     const float* fiber, int32_t n) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (m < 0 || m >= e->M) return fail(e, JF_ERR_INVALID, "instance index out of range");
  const JfInst& I = e->inst[m];
  if (n < 0 || n > I.n_slots) return fail(e, JF_ERR_INVALID, "particle count exceeds the instance's slots");
  if (n > 0 && (!pos || !material)) return fail(e, JF_ERR_INVALID, "positions and materials are required");
  int rc = set_device(e);
  if (rc) return rc;
  const size_t S = (size_t)e->max_slots;
  // glow is not reset by a load (mpm_sim.py:715-727): keep it, in slot order
  JF_CK(jf_glow_to_slot_order(e, m), "glow reorder");
  std::vector<float> fib;
  if (!fiber && n > 0) {
    fib.assign(2 * (size_t)n, 0.0f);
    for (int k = 0; k < n; ++k) fib[2 * k + 1] = 1.0f;
    fiber = fib.data();
  }
  if (n > 0) {
    JF_CK(cudaMemcpyAsync(e->d_stage, pos, sizeof(float) * 2 * n, cudaMemcpyHostToDevice, e->stream), "stage pos");
    JF_CK(cudaMemcpyAsync(e->d_stage + 2 * S, fiber, sizeof(float) * 2 * n, cudaMemcpyHostToDevice, e->stream),
          "stage fiber");
    JF_CK(cudaMemcpyAsync(e->d_stage_i, material, sizeof(int32_t) * n, cudaMemcpyHostToDevice, e->stream),
          "stage material");
  }
  JF_CK(jf_load_launch(e, m, n), "load kernel");
  int32_t live = 0;
  for (int k = 0; k < n; ++k) live += material[k] >= 0 ? 1 : 0;
  if ((rc = set_live_count(e, m, live))) return rc;
  JF_CK(cudaStreamSynchronize(e->stream), "load sync");
  e->sorted = false;
  return JF_OK;
}

int jf_load_robot(jf_engine* e, int32_t m, const double* robot_pos, const int32_t* robot_mat,
                  const float* robot_fiber, int32_t n_robot, double water_margin, double spacing_div,
                  int32_t* out_counts) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (m < 0 || m >= e->M) return fail(e, JF_ERR_INVALID, "instance index out of range");
  if (n_robot < 0 || (n_robot > 0 && (!robot_pos || !robot_mat)))
    return fail(e, JF_ERR_INVALID, "robot positions and materials are required");
  if (!(spacing_div > 0.0) || !(water_margin >= 0.0))
    return fail(e, JF_ERR_INVALID, "spacing_div must be > 0 and water_margin >= 0");
  int rc = set_device(e);
  if (rc) return rc;
  const JfInst& I = e->inst[m];
  const size_t S = (size_t)e->max_slots;
  const int32_t nr = std::min(n_robot, I.n_slots);  // make_jelly.py:371-374: the robot keeps its slots
  JF_CK(jf_glow_to_slot_order(e, m), "glow reorder");
  double bbox[4] = {0.0, 0.0, -1.0, -1.0};
  if (nr > 0) {
    std::vector<float> pos(2 * (size_t)nr), fib(2 * (size_t)nr);
    for (int k = 0; k < nr; ++k) {
      pos[2 * k] = (float)robot_pos[2 * k];
      pos[2 * k + 1] = (float)robot_pos[2 * k + 1];
      fib[2 * k] = robot_fiber ? robot_fiber[2 * k] : 0.0f;
      fib[2 * k + 1] = robot_fiber ? robot_fiber[2 * k + 1] : 1.0f;
    }
    JF_CK(cudaMemcpyAsync(e->d_stage, pos.data(), sizeof(float) * pos.size(), cudaMemcpyHostToDevice, e->stream),
          "stage robot");
    JF_CK(cudaMemcpyAsync(e->d_stage + 2 * S, fib.data(), sizeof(float) * fib.size(), cudaMemcpyHostToDevice,
                          e->stream), "stage robot fibre");
    JF_CK(cudaMemcpyAsync(e->d_stage_i, robot_mat, sizeof(int32_t) * nr, cudaMemcpyHostToDevice, e->stream),
          "stage robot material");
  }
  if (n_robot > 0) {
    bbox[0] = bbox[2] = robot_pos[0];
    bbox[1] = bbox[3] = robot_pos[1];
    for (int k = 1; k < n_robot; ++k) {
      bbox[0] = std::min(bbox[0], robot_pos[2 * k]);
      bbox[2] = std::max(bbox[2], robot_pos[2 * k]);
      bbox[1] = std::min(bbox[1], robot_pos[2 * k + 1]);
      bbox[3] = std::max(bbox[3], robot_pos[2 * k + 1]);
    }
  }
  // every robot particle excludes water, also those cut from the slots
  double* d_robot = nullptr;
  int32_t* d_scratch = nullptr;
  const int64_t scratch = jf_tank_scratch_ints(e, m, spacing_div);
  int32_t total = 0;
  cudaError_t err = alloc(&d_robot, 2 * (size_t)std::max(n_robot, 1));
  if (err == cudaSuccess) err = alloc(&d_scratch, (size_t)scratch);
  if (err == cudaSuccess && n_robot > 0)
    err = cudaMemcpyAsync(d_robot, robot_pos, sizeof(double) * 2 * n_robot, cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess)
    err = jf_tank_water_launch(e, m, d_robot, n_robot, bbox, water_margin, spacing_div, d_scratch, scratch, &total);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
  cudaFree(d_robot);
  cudaFree(d_scratch);
  if (err != cudaSuccess) return cuda_fail(e, err, "tank water fill");
  const int32_t n_water = std::max(0, std::min(total, I.n_slots - n_robot));
  JF_CK(jf_load_launch(e, m, nr + n_water), "load kernel");
  if ((rc = set_live_count(e, m, nr + n_water))) return rc;
  JF_CK(cudaStreamSynchronize(e->stream), "load sync");
  e->sorted = false;
  if (out_counts) {
    out_counts[0] = nr;
    out_counts[1] = n_water;
  }
  return JF_OK;
}

int jf_set_params(jf_engine* e, const float* actuation, const float* contraction, const float* freq,
                  const float* payload_density) {
  if (check_engine(e)) return JF_ERR_INVALID;
  for (int m = 0; m < e->M; ++m) {
    if (actuation) e->params[m].actuation = actuation[m];
    if (contraction) e->params[m].contraction = contraction[m];
    if (freq) e->params[m].freq = freq[m];
    if (payload_density) e->params[m].payload_density = payload_density[m];
  }
  e->params_dirty = true;
  return JF_OK;
}

int jf_get_params(const jf_engine* e, float* actuation, float* contraction, float* freq,
                  float* payload_density) {
  if (check_engine(e)) return JF_ERR_INVALID;
  for (int m = 0; m < e->M; ++m) {
    if (actuation) actuation[m] = e->params[m].actuation;
    if (contraction) contraction[m] = e->params[m].contraction;
    if (freq) freq[m] = e->params[m].freq;
    if (payload_density) payload_density[m] = e->params[m].payload_density;
  }
  return JF_OK;
}

int jf_set_time(jf_engine* e, float t) {
  if (check_engine(e)) return JF_ERR_INVALID;
  e->t = t;
  return JF_OK;
}

int jf_get_time(const jf_engine* e, float* t) {
  if (check_engine(e) || !t) return JF_ERR_INVALID;
  *t = e->t;
  return JF_OK;
}

int jf_step(jf_engine* e, int64_t n_steps) {
  if (check_engine(e)) return JF_ERR_INVALID;
  return step_impl(e, n_steps);
}

// JF_ERR_NONFINITE when any instance's non-finite flag is set (the caller
// has synchronised the stream); the message names the instances.
static int nonfinite_status(jf_engine* e, const std::vector<int32_t>& flags) {
  std::string which;
  int n = 0;
  for (int m = 0; m < e->M; ++m) {
    if (!flags[m]) continue;
    if (n < 8) which += (n ? ", " : "") + std::to_string(m);
    ++n;
  }
  if (n == 0) return JF_OK;
  if (n > 8) which += ", ...";
  return fail(e, JF_ERR_NONFINITE, std::to_string(n) + " instance(s) with a non-finite particle state: " + which);
}

static int read_flags_and_sync(jf_engine* e, std::vector<int32_t>& flags) {
  flags.assign(e->M, 0);
  JF_CK(cudaMemcpyAsync(flags.data(), e->d_err, sizeof(int32_t) * e->M, cudaMemcpyDeviceToHost, e->stream),
        "read flags");
  JF_CK(cudaStreamSynchronize(e->stream), "sync");
  return JF_OK;
}

int jf_sync(jf_engine* e) {
  if (check_engine(e)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  std::vector<int32_t> flags;
  if ((rc = read_flags_and_sync(e, flags))) return rc;
  return nonfinite_status(e, flags);
}

int jf_sync_timeout(jf_engine* e, int64_t timeout_ms) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (timeout_ms < 0) return fail(e, JF_ERR_INVALID, "jf_sync_timeout: negative limit");
  int rc = set_device(e);
  if (rc) return rc;
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t q = cudaStreamQuery(e->stream);
    if (q == cudaSuccess) break;
    if (q != cudaErrorNotReady) return cuda_fail(e, q, "stream query");
    const auto waited = std::chrono::duration_cast<std::chrono::milliseconds>(
        std::chrono::steady_clock::now() - t0).count();
    if (waited >= timeout_ms)
      return fail(e, JF_ERR_TIMEOUT, "queued work not finished after " + std::to_string(waited) + " ms");
    std::this_thread::sleep_for(std::chrono::microseconds(100));
  }
  return jf_sync(e);
}

int jf_payload_stats(jf_engine* e, double* out) {
  if (check_engine(e) || need_args(e, out, "jf_payload_stats: out")) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  return stats_rows(e, out, false);
}

int jf_stats_any(jf_engine* e, double* out) {
  if (check_engine(e) || need_args(e, out, "jf_stats_any: out")) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  return stats_rows(e, out, true);
}

int jf_stats_raw(jf_engine* e, double* out) {
  if (check_engine(e) || need_args(e, out, "jf_stats_raw: out")) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(jf_stats_launch(e), "stats kernel");
  JF_CK(cudaMemcpyAsync(out, e->d_stats, sizeof(double) * 6 * e->M, cudaMemcpyDeviceToHost, e->stream),
        "read stats");
  JF_CK(cudaStreamSynchronize(e->stream), "stats sync");
  return JF_OK;
}

int jf_run_headless(jf_engine* e, int64_t steps, double* out) {
  if (check_engine(e) || need_args(e, out, "jf_run_headless: out")) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  e->t = 0.0f;
  std::vector<double> initial(3 * (size_t)e->M), final_(3 * (size_t)e->M);
  if ((rc = stats_rows(e, initial.data(), true))) return rc;
  if ((rc = step_impl(e, steps))) return rc;
  if ((rc = stats_rows(e, final_.data(), true))) return rc;
  for (int m = 0; m < e->M; ++m) {
    const double* a = &initial[3 * (size_t)m];
    const double* b = &final_[3 * (size_t)m];
    double* o = out + 5 * (size_t)m;
    o[0] = o[1] = o[2] = o[3] = o[4] = 0.0;
    if (a[2] > 0 && b[2] > 0) {
      o[0] = a[0]; o[1] = a[1]; o[2] = b[0]; o[3] = b[1];
      o[4] = (b[0] < 0.01) ? 0.0 : 1.0;
    }
  }
  std::vector<int32_t> flags;
  if ((rc = read_flags_and_sync(e, flags))) return rc;
  return nonfinite_status(e, flags);
}

int jf_fitness(jf_engine* e, const double* results, const int32_t* muscle_counts, const double* contraction,
               int32_t mode, double* out) {
  if (check_engine(e) || need_args(e, results && muscle_counts && out, "jf_fitness: results, muscle_counts and out"))
    return JF_ERR_INVALID;
  if (mode != 0 && mode != 1) return fail(e, JF_ERR_INVALID, "fitness mode must be 0 or 1");
  int rc = set_device(e);
  if (rc) return rc;
  const size_t M = (size_t)e->M;
  double* d_rows = e->d_fit;       // 5M doubles
  double* d_out = e->d_fit + 5 * M;  // M doubles
  double* d_con = e->d_fit_f;      // M doubles
  int32_t* d_mus = e->d_fit_i;     // M ints
  JF_CK(cudaMemcpyAsync(d_rows, results, sizeof(double) * 5 * M, cudaMemcpyHostToDevice, e->stream), "fitness rows");
  JF_CK(cudaMemcpyAsync(d_mus, muscle_counts, sizeof(int32_t) * M, cudaMemcpyHostToDevice, e->stream), "fitness counts");
  if (contraction)
    JF_CK(cudaMemcpyAsync(d_con, contraction, sizeof(double) * M, cudaMemcpyHostToDevice, e->stream), "fitness genes");
  JF_CK(jf_fitness_launch(e, d_rows, d_mus, contraction ? d_con : nullptr, mode, d_out), "fitness kernel");
  JF_CK(cudaMemcpyAsync(out, d_out, sizeof(double) * M, cudaMemcpyDeviceToHost, e->stream), "fitness read");
  JF_CK(cudaStreamSynchronize(e->stream), "fitness sync");
  return JF_OK;
}

int jf_run_episode(jf_engine* e, const float* pos, const int32_t* material, const float* fiber,
                   const float* contraction, const float* freq, int64_t steps,
                   const int32_t* muscle_counts, int32_t mode, double* rows, double* fitness) {
  if (check_engine(e) ||
      need_args(e, pos && material && contraction && rows, "jf_run_episode: pos, material, contraction and rows"))
    return JF_ERR_INVALID;
  if (steps < 0) return fail(e, JF_ERR_INVALID, "steps must be >= 0");
  if (muscle_counts && !fitness) return fail(e, JF_ERR_INVALID, "fitness output required with muscle_counts");
  if (mode != 0 && mode != 1) return fail(e, JF_ERR_INVALID, "fitness mode must be 0 or 1");
  int rc = set_device(e);
  if (rc) return rc;
  const size_t S = (size_t)e->total_slots, M = (size_t)e->M;
  if (!e->d_ep) {
    cudaError_t err;
    if ((err = cudaMalloc((void**)&e->d_ep, sizeof(float) * 5 * (S > 0 ? S : 1))) != cudaSuccess ||
        (err = cudaMalloc((void**)&e->d_ep_mat, sizeof(int32_t) * (S > 0 ? S : 1))) != cudaSuccess ||
        (err = cudaMalloc((void**)&e->d_ep_stats, sizeof(double) * 6 * M)) != cudaSuccess)
      return cuda_fail(e, err, "episode staging");
  }
  float* d_pos = e->d_ep;
  float* d_fib = e->d_ep + 2 * S;
  float* d_glow = e->d_ep + 4 * S;
  // loads of every instance (mpm_sim.py:715-727), one copy per array
  if (S > 0) {
    JF_CK(cudaMemcpyAsync(d_pos, pos, sizeof(float) * 2 * S, cudaMemcpyHostToDevice, e->stream), "episode pos");
    JF_CK(cudaMemcpyAsync(e->d_ep_mat, material, sizeof(int32_t) * S, cudaMemcpyHostToDevice, e->stream),
          "episode material");
    if (fiber)
      JF_CK(cudaMemcpyAsync(d_fib, fiber, sizeof(float) * 2 * S, cudaMemcpyHostToDevice, e->stream), "episode fiber");
  }
  JF_CK(jf_load_all_launch(e, d_pos, e->d_ep_mat, fiber ? d_fib : nullptr, d_glow), "episode load");
  e->sorted = false;
  if (e->d_order) {
    for (size_t m = 0; m < M; ++m) {
      const JfInst& I = e->inst[m];
      int32_t live = 0;
      for (int32_t k = 0; k < I.n_slots; ++k) live += material[I.p_off + k] >= 0 ? 1 : 0;
      e->n_live[m] = live;
    }
    int rc = upload_order(e);
    if (rc) return rc;
  }
  // timing genes (evolve.py:150-152)
  for (size_t m = 0; m < M; ++m) {
    e->params[m].contraction = contraction[m];
    if (freq) e->params[m].freq = freq[m];
  }
  e->params_dirty = true;
  // run_batch_headless (mpm_sim.py:802-834) with the rows formed on the device
  e->t = 0.0f;
  JF_CK(jf_stats_launch(e), "stats kernel");
  JF_CK(cudaMemcpyAsync(e->d_ep_stats, e->d_stats, sizeof(double) * 6 * M, cudaMemcpyDeviceToDevice, e->stream),
        "stats before");
  if ((rc = step_impl(e, steps))) return rc;
  JF_CK(jf_stats_launch(e), "stats kernel");
  double* d_rows = e->d_fit;          // 5M doubles
  double* d_out = e->d_fit + 5 * M;   // M doubles
  JF_CK(jf_rows_launch(e, e->d_ep_stats, e->d_stats, d_rows), "rows kernel");
  if (muscle_counts) {
    std::vector<double> con(M);
    for (size_t m = 0; m < M; ++m) con[m] = (double)contraction[m];
    JF_CK(cudaMemcpyAsync(e->d_fit_i, muscle_counts, sizeof(int32_t) * M, cudaMemcpyHostToDevice, e->stream),
          "fitness counts");
    JF_CK(cudaMemcpyAsync(e->d_fit_f, con.data(), sizeof(double) * M, cudaMemcpyHostToDevice, e->stream),
          "fitness genes");
    JF_CK(jf_fitness_launch(e, d_rows, e->d_fit_i, e->d_fit_f, mode, d_out), "fitness kernel");
    JF_CK(cudaMemcpyAsync(fitness, d_out, sizeof(double) * M, cudaMemcpyDeviceToHost, e->stream), "fitness read");
  }
  JF_CK(cudaMemcpyAsync(rows, d_rows, sizeof(double) * 5 * M, cudaMemcpyDeviceToHost, e->stream), "rows read");
  std::vector<int32_t> flags;
  if ((rc = read_flags_and_sync(e, flags))) return rc;
  return nonfinite_status(e, flags);
}

// The CoM each instance's loss follows (payload; jelly + muscle without
// payload, mpm_sim.py:786-792) from the current state: selection, 1 / count
// and the initial height.
static int grad_prologue(jf_engine* e, std::vector<int32_t>& body, std::vector<double>& inv_n,
                         std::vector<double>& init) {
  int rc = upload_params(e);
  if (rc) return rc;
  std::vector<double> raw(6 * (size_t)e->M);
  JF_CK(jf_stats_launch(e), "stats kernel");
  JF_CK(cudaMemcpyAsync(raw.data(), e->d_stats, sizeof(double) * raw.size(), cudaMemcpyDeviceToHost, e->stream),
        "read stats");
  JF_CK(cudaStreamSynchronize(e->stream), "stats sync");
  body.assign(e->M, 0);
  inv_n.assign(e->M, 0.0);
  init.assign(e->M, 0.0);
  for (int m = 0; m < e->M; ++m) {
    const double* r = &raw[6 * (size_t)m];
    body[m] = r[1] == 0 ? 1 : 0;
    const double cnt = body[m] ? r[4] : r[1];
    const double sy = body[m] ? r[3] : r[0];
    inv_n[m] = cnt > 0 ? 1.0 / cnt : 0.0;
    init[m] = cnt > 0 ? sy / cnt : 0.0;
  }
  return JF_OK;
}

// loss[m] = final CoM height - initial, from the sums in e->d_stats
static int grad_loss(jf_engine* e, const std::vector<int32_t>& body, const std::vector<double>& init,
                     double* loss) {
  std::vector<double> raw(6 * (size_t)e->M);
  JF_CK(cudaMemcpyAsync(raw.data(), e->d_stats, sizeof(double) * raw.size(), cudaMemcpyDeviceToHost, e->stream),
        "read stats");
  JF_CK(cudaStreamSynchronize(e->stream), "stats sync");
  for (int m = 0; m < e->M; ++m) {
    const double* r = &raw[6 * (size_t)m];
    const double cnt = body[m] ? r[4] : r[1];
    const double sy = body[m] ? r[3] : r[0];
    const double fin = cnt > 0 ? sy / cnt : 0.0;
    if (loss) loss[m] = fin - init[m];
  }
  return JF_OK;
}

static int grad_check_args(jf_engine* e, int64_t steps, int32_t checkpoint_every) {
  if (steps <= 0 || checkpoint_every <= 0) return fail(e, JF_ERR_INVALID, "steps and checkpoint_every must be > 0");
  if (e->flags & JF_FLAG_AXISYM)
    return fail(e, JF_ERR_UNSUPPORTED, "the differentiable rollout has no axisymmetric variant");
  return JF_OK;
}

int jf_grad_forward(jf_engine* e, int64_t steps, int32_t checkpoint_every, double* loss) {
  if (check_engine(e)) return JF_ERR_INVALID;
  int rc = grad_check_args(e, steps, checkpoint_every);
  if (rc) return rc;
  if ((rc = set_device(e))) return rc;
  std::vector<int32_t> body;
  std::vector<double> inv_n, init;
  if ((rc = grad_prologue(e, body, inv_n, init))) return rc;
  JF_CK(jf_grad_forward_impl(e, steps, checkpoint_every, body.data(), inv_n.data()), "gradient forward");
  JF_CK(jf_grad_loss_stats(e), "loss sums");
  if ((rc = grad_loss(e, body, init, loss))) return rc;
  e->sorted = false;
  std::vector<int32_t> flags;
  if ((rc = read_flags_and_sync(e, flags))) return rc;
  return nonfinite_status(e, flags);
}

int jf_grad_step(jf_engine* e, int64_t steps, int32_t checkpoint_every, double* loss, double* d_actuation,
                 double* d_contraction, double* d_freq) {
  if (check_engine(e)) return JF_ERR_INVALID;
  int rc = grad_check_args(e, steps, checkpoint_every);
  if (rc) return rc;
  if ((rc = set_device(e))) return rc;
  std::vector<int32_t> body;
  std::vector<double> inv_n, init;
  if ((rc = grad_prologue(e, body, inv_n, init))) return rc;
  std::vector<double> g(3 * (size_t)e->M);
  JF_CK(jf_grad_step_impl(e, steps, checkpoint_every, body.data(), inv_n.data(), g.data()), "gradient step");
  if ((rc = grad_loss(e, body, init, loss))) return rc;
  for (int m = 0; m < e->M; ++m) {
    if (d_actuation) d_actuation[m] = g[3 * (size_t)m + 0];
    if (d_contraction) d_contraction[m] = g[3 * (size_t)m + 1];
    if (d_freq) d_freq[m] = g[3 * (size_t)m + 2];
  }
  e->sorted = false;
  std::vector<int32_t> flags;
  if ((rc = read_flags_and_sync(e, flags))) return rc;
  return nonfinite_status(e, flags);
}

int jf_grad_backward(jf_engine* e, double* d_actuation, double* d_contraction, double* d_freq) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (!jf_grad_done(e, 1))
    return fail(e, JF_ERR_INVALID, "jf_grad_backward needs a completed jf_grad_forward first");
  int rc = set_device(e);
  if (rc) return rc;
  std::vector<double> g(3 * (size_t)e->M);
  JF_CK(jf_grad_backward_impl(e, g.data()), "gradient backward");
  for (int m = 0; m < e->M; ++m) {
    if (d_actuation) d_actuation[m] = g[3 * (size_t)m + 0];
    if (d_contraction) d_contraction[m] = g[3 * (size_t)m + 1];
    if (d_freq) d_freq[m] = g[3 * (size_t)m + 2];
  }
  std::vector<int32_t> flags;
  if ((rc = read_flags_and_sync(e, flags))) return rc;
  return nonfinite_status(e, flags);
}

int jf_grad_positions(jf_engine* e, int32_t m, float* dx0) {
  if (check_engine(e) || need_args(e, dx0, "jf_grad_positions: dx0")) return JF_ERR_INVALID;
  if (m < 0 || m >= e->M) return fail(e, JF_ERR_INVALID, "instance index out of range");
  if (!jf_grad_done(e, 2))
    return fail(e, JF_ERR_INVALID,
                "jf_grad_positions needs the backward of the latest rollout (jf_grad_backward or jf_grad_step)");
  int rc = set_device(e);
  if (rc) return rc;
  std::vector<float4> lx;
  JF_CK(jf_grad_x0_impl(e, m, lx), "read position adjoint");
  HostInstance h;
  if ((rc = download_instance(e, m, h))) return rc;
  for (size_t k = 0; k < lx.size(); ++k) {
    const size_t s = (size_t)h.slot[k];
    dx0[2 * s] = lx[k].x;
    dx0[2 * s + 1] = lx[k].y;
  }
  return JF_OK;
}

int jf_read_particles(jf_engine* e, int32_t m, float* x, float* v, float* C, float* F, int32_t* material,
                      float* Jp, float* glow, float* fiber) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (m < 0 || m >= e->M) return fail(e, JF_ERR_INVALID, "instance index out of range");
  int rc = set_device(e);
  if (rc) return rc;
  HostInstance h;
  if ((rc = download_instance(e, m, h))) return rc;
  const size_t n = h.slot.size();
  for (size_t k = 0; k < n; ++k) {
    const size_t s = (size_t)h.slot[k];
    if (x) { x[2 * s] = h.xv[k].x; x[2 * s + 1] = h.xv[k].y; }
    if (v) { v[2 * s] = h.xv[k].z; v[2 * s + 1] = h.xv[k].w; }
    if (C) { C[4 * s] = h.C[k].x; C[4 * s + 1] = h.C[k].y; C[4 * s + 2] = h.C[k].z; C[4 * s + 3] = h.C[k].w; }
    if (F) { F[4 * s] = h.F[k].x; F[4 * s + 1] = h.F[k].y; F[4 * s + 2] = h.F[k].z; F[4 * s + 3] = h.F[k].w; }
    if (material) material[s] = h.mat[k];
    if (Jp) Jp[s] = h.Jp[k];
    if (glow) glow[s] = h.glow[k];
    if (fiber) { fiber[2 * s] = h.fiber[k].x; fiber[2 * s + 1] = h.fiber[k].y; }
  }
  return JF_OK;
}

int jf_write_particles(jf_engine* e, int32_t m, const float* x, const float* v, const float* C, const float* F,
                       const float* Jp, const float* glow) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (m < 0 || m >= e->M) return fail(e, JF_ERR_INVALID, "instance index out of range");
  int rc = set_device(e);
  if (rc) return rc;
  HostInstance h;
  if ((rc = download_instance(e, m, h))) return rc;
  const size_t n = h.slot.size();
  for (size_t k = 0; k < n; ++k) {
    const size_t s = (size_t)h.slot[k];
    if (x) { h.xv[k].x = x[2 * s]; h.xv[k].y = x[2 * s + 1]; }
    if (v) { h.xv[k].z = v[2 * s]; h.xv[k].w = v[2 * s + 1]; }
    if (C) h.C[k] = make_float4(C[4 * s], C[4 * s + 1], C[4 * s + 2], C[4 * s + 3]);
    if (F) h.F[k] = make_float4(F[4 * s], F[4 * s + 1], F[4 * s + 2], F[4 * s + 3]);
    if (Jp) h.Jp[k] = Jp[s];
    if (glow) h.glow[k] = glow[s];
  }
  if ((rc = upload_instance(e, m, h))) return rc;
  if (x) e->sorted = false;
  return JF_OK;
}

int jf_read_grid(jf_engine* e, int32_t m, float* grid_v, float* grid_m) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (m < 0 || m >= e->M) return fail(e, JF_ERR_INVALID, "instance index out of range");
  int rc = set_device(e);
  if (rc) return rc;
  const JfInst& I = e->inst[m];
  std::vector<float4> g((size_t)I.nx * I.ny);
  JF_CK(cudaMemcpyAsync(g.data(), e->d_grid + I.g_off, sizeof(float4) * g.size(), cudaMemcpyDeviceToHost,
                        e->stream),
        "read grid");
  JF_CK(cudaStreamSynchronize(e->stream), "read grid sync");
  for (int j = 0; j < I.ny; ++j) {
    for (int i = 0; i < I.nx; ++i) {
      const float4 q = g[(size_t)j * I.nx + i];
      const size_t r = (size_t)i * I.ny + j;  // reference layout [nx][ny]
      if (grid_v) { grid_v[2 * r] = q.x; grid_v[2 * r + 1] = q.y; }
      if (grid_m) grid_m[r] = q.z;
    }
  }
  return JF_OK;
}

int jf_error_flags(jf_engine* e, int32_t* out) {
  if (check_engine(e) || need_args(e, out, "jf_error_flags: out")) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(cudaMemcpyAsync(out, e->d_err, sizeof(int32_t) * e->M, cudaMemcpyDeviceToHost, e->stream), "read flags");
  JF_CK(cudaStreamSynchronize(e->stream), "flags sync");
  return JF_OK;
}

int jf_clear_error_flags(jf_engine* e) {
  if (check_engine(e)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(cudaMemsetAsync(e->d_err, 0, sizeof(int32_t) * e->M, e->stream), "clear flags");
  return JF_OK;
}

int64_t jf_kernel_launches(const jf_engine* e) { return e ? e->launches : -1; }

int jf_path_counts(jf_engine* e, int64_t* out, int32_t reset) {
  if (check_engine(e) || need_args(e, out, "jf_path_counts: out")) return JF_ERR_INVALID;
  out[0] = out[1] = out[2] = out[3] = 0;
  if (!e->d_path) return JF_OK;
  int rc = set_device(e);
  if (rc) return rc;
  unsigned long long h[4] = {0, 0, 0, 0};
  JF_CK(cudaMemcpyAsync(h, e->d_path, sizeof(h), cudaMemcpyDeviceToHost, e->stream), "read path counters");
  JF_CK(cudaStreamSynchronize(e->stream), "path counters sync");
  for (int i = 0; i < 4; ++i) out[i] = (int64_t)h[i];
  if (reset) JF_CK(cudaMemsetAsync(e->d_path, 0, sizeof(h), e->stream), "reset path counters");
  return JF_OK;
}

int jf_get_layout(const jf_engine* e, int32_t* cluster_size, int32_t* block_threads) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (cluster_size) *cluster_size = e->cluster;
  if (block_threads) *block_threads = e->block_threads;
  return JF_OK;
}

int jf_set_kernel_timing(jf_engine* e, int32_t enable) {
  if (check_engine(e)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(cudaStreamSynchronize(e->stream), "timing sync");
  collect_timing(e);
  e->step_ms = e->sort_ms = 0.0;
  e->step_launches = e->sort_launches = 0;
  e->timing = enable != 0;
  return JF_OK;
}

int jf_kernel_timing(jf_engine* e, double* step_ms, int64_t* step_launches, double* sort_ms,
                     int64_t* sort_launches) {
  if (check_engine(e)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(cudaStreamSynchronize(e->stream), "timing sync");
  JF_CK(collect_timing(e), "event elapsed time");
  if (step_ms) *step_ms = e->step_ms;
  if (step_launches) *step_launches = e->step_launches;
  if (sort_ms) *sort_ms = e->sort_ms;
  if (sort_launches) *sort_launches = e->sort_launches;
  return JF_OK;
}

// --- headless renderer (mpm_sim.py:343-712) -----------------------------------

static int need_frame(jf_engine* e) {
  if (!e->d_frame) return fail(e, JF_ERR_INVALID, "no frame buffer: call jf_frame_create first");
  return JF_OK;
}

static int check_tiles(jf_engine* e, int32_t res_sub, int32_t grid_side) {
  if (res_sub <= 0 || grid_side <= 0) return fail(e, JF_ERR_INVALID, "res_sub and grid_side must be > 0");
  return JF_OK;
}

static int need_vort(jf_engine* e) {
  if (e->d_vort) return JF_OK;
  JF_CK(alloc(&e->d_vort, (size_t)e->total_nodes), "cudaMalloc vorticity");
  JF_CK(cudaMemsetAsync(e->d_vort, 0, sizeof(float) * std::max<int64_t>(e->total_nodes, 1), e->stream),
        "clear vorticity");
  return JF_OK;
}

int jf_frame_create(jf_engine* e, int32_t video_res) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (video_res <= 0 || video_res > 16384) return fail(e, JF_ERR_INVALID, "video_res must be in 1 .. 16384");
  int rc = set_device(e);
  if (rc) return rc;
  if (e->frame_res != video_res) {
    JF_CK(cudaStreamSynchronize(e->stream), "frame sync");
    cudaFree(e->d_frame);
    e->d_frame = nullptr;
    e->frame_res = 0;
    JF_CK(alloc(&e->d_frame, (size_t)video_res * video_res), "cudaMalloc frame");
    e->frame_res = video_res;
  }
  JF_CK(cudaMemsetAsync(e->d_frame, 0, sizeof(float4) * (size_t)video_res * video_res, e->stream), "clear frame");
  return JF_OK;
}

int jf_frame_clear(jf_engine* e, float value) {
  if (check_engine(e) || need_frame(e)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(jf_frame_clear_launch(e, value), "clear frame");
  return JF_OK;
}

int jf_render_abyss(jf_engine* e, int32_t res_sub, int32_t grid_side, float radius, const float* hue,
                    const float* muscle_hue, int32_t water_mode) {
  if (check_engine(e) || need_frame(e) || check_tiles(e, res_sub, grid_side)) return JF_ERR_INVALID;
  if (!hue || !muscle_hue) return fail(e, JF_ERR_INVALID, "hue and muscle_hue are required");
  int rc = set_device(e);
  if (rc) return rc;
  if ((rc = upload_params(e))) return rc;
  if (!e->d_hue) JF_CK(alloc(&e->d_hue, (size_t)e->M), "cudaMalloc hues");
  std::vector<float2> h(e->M);
  for (int m = 0; m < e->M; ++m) h[m] = make_float2(hue[m], muscle_hue[m]);
  // a copy from pageable memory has staged the source when it returns
  JF_CK(cudaMemcpyAsync(e->d_hue, h.data(), sizeof(float2) * e->M, cudaMemcpyHostToDevice, e->stream), "upload hues");
  JF_CK(jf_render_abyss_launch(e, res_sub, grid_side, radius, water_mode), "render abyss");
  return JF_OK;
}

int jf_render_flat(jf_engine* e, int32_t res_sub, int32_t grid_side, float radius, int32_t material, float r,
                   float g, float b) {
  if (check_engine(e) || need_frame(e) || check_tiles(e, res_sub, grid_side)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(jf_render_flat_launch(e, res_sub, grid_side, radius, material, r, g, b), "render flat pass");
  return JF_OK;
}

int jf_render_vorticity_overlay(jf_engine* e, int32_t res_sub, int32_t grid_side, float vort_scale) {
  if (check_engine(e) || need_frame(e) || check_tiles(e, res_sub, grid_side)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(jf_render_overlay_launch(e, res_sub, grid_side, vort_scale), "render vorticity overlay");
  return JF_OK;
}

int jf_compute_vorticity(jf_engine* e, float vort_scale) {
  if (check_engine(e)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc || (rc = need_vort(e))) return rc;
  JF_CK(jf_vorticity_launch(e, vort_scale), "compute vorticity");
  return JF_OK;
}

int jf_render_vorticity(jf_engine* e, int32_t res_sub, int32_t grid_side, float alpha, int32_t style) {
  if (check_engine(e) || need_frame(e) || check_tiles(e, res_sub, grid_side)) return JF_ERR_INVALID;
  if (style < JF_VORT_RDBU || style > JF_VORT_WHITE) return fail(e, JF_ERR_INVALID, "unknown vorticity style");
  int rc = set_device(e);
  if (rc || (rc = need_vort(e))) return rc;
  JF_CK(jf_render_vort_launch(e, res_sub, grid_side, alpha, style), "render vorticity");
  return JF_OK;
}

int jf_tone_map(jf_engine* e) {
  if (check_engine(e) || need_frame(e)) return JF_ERR_INVALID;
  int rc = set_device(e);
  if (rc) return rc;
  JF_CK(jf_tone_map_launch(e), "tone map");
  return JF_OK;
}

int jf_read_frame(jf_engine* e, float* rgb) {
  if (check_engine(e) || need_frame(e)) return JF_ERR_INVALID;
  if (!rgb) return fail(e, JF_ERR_INVALID, "rgb is NULL");
  int rc = set_device(e);
  if (rc) return rc;
  const size_t n = (size_t)e->frame_res * e->frame_res;
  std::vector<float4> f(n);
  JF_CK(cudaMemcpyAsync(f.data(), e->d_frame, sizeof(float4) * n, cudaMemcpyDeviceToHost, e->stream), "read frame");
  JF_CK(cudaStreamSynchronize(e->stream), "read frame sync");
  for (size_t k = 0; k < n; ++k) {
    rgb[3 * k] = f[k].x;
    rgb[3 * k + 1] = f[k].y;
    rgb[3 * k + 2] = f[k].z;
  }
  return JF_OK;
}

int jf_read_vorticity(jf_engine* e, int32_t m, float* vort) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (m < 0 || m >= e->M) return fail(e, JF_ERR_INVALID, "instance index out of range");
  if (!vort) return fail(e, JF_ERR_INVALID, "vort is NULL");
  int rc = set_device(e);
  if (rc || (rc = need_vort(e))) return rc;
  const JfInst& I = e->inst[m];
  std::vector<float> g((size_t)I.nx * I.ny);
  JF_CK(cudaMemcpyAsync(g.data(), e->d_vort + I.g_off, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, e->stream),
        "read vorticity");
  JF_CK(cudaStreamSynchronize(e->stream), "read vorticity sync");
  for (int j = 0; j < I.ny; ++j)
    for (int i = 0; i < I.nx; ++i) vort[(size_t)i * I.ny + j] = g[(size_t)j * I.nx + i];
  return JF_OK;
}

int jf_write_grid(jf_engine* e, int32_t m, const float* grid_v, const float* grid_m) {
  if (check_engine(e)) return JF_ERR_INVALID;
  if (m < 0 || m >= e->M) return fail(e, JF_ERR_INVALID, "instance index out of range");
  if (!grid_v || !grid_m) return fail(e, JF_ERR_INVALID, "grid_v and grid_m are required");
  int rc = set_device(e);
  if (rc) return rc;
  const JfInst& I = e->inst[m];
  std::vector<float4> g((size_t)I.nx * I.ny);
  for (int j = 0; j < I.ny; ++j) {
    for (int i = 0; i < I.nx; ++i) {
      const size_t r = (size_t)i * I.ny + j;  // reference layout [nx][ny]
      g[(size_t)j * I.nx + i] = make_float4(grid_v[2 * r], grid_v[2 * r + 1], grid_m[r], 0.0f);
    }
  }
  JF_CK(cudaMemcpyAsync(e->d_grid + I.g_off, g.data(), sizeof(float4) * g.size(), cudaMemcpyHostToDevice, e->stream),
        "write grid");
  JF_CK(cudaStreamSynchronize(e->stream), "write grid sync");
  return JF_OK;
}

}  // extern "C"
