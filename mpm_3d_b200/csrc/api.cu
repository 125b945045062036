// Host side of the C ABI declared in include/mpm_b200.h: the single-job
// handle (mpmgpu_*) and the batch (mpmgpu_batch_*), both on the step engine
// of engine.cuh. A handle is a batch of one job that starts at its first
// step.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "engine.cuh"
#include "points_file.h"
#include "server.cuh"

using namespace mpmb200;

struct mpmgpu_handle {
  mpmgpu_config cfg{};
  std::unique_ptr<BatchBase> b;
  int job = 0;
  bool started = false;
  int64_t extra_launches = 0;  // map exports (outside the engine)
  std::string last_error;
};

struct mpmgpu_batch {
  mpmgpu_batch_config cfg{};
  std::unique_ptr<BatchBase> b;
  std::string last_error;
};

struct mpmgpu_server {
  std::unique_ptr<Server> s;
};

namespace {

mpmgpu_status hfail(mpmgpu_handle* h, mpmgpu_status s, const std::string& msg) {
  if (h) {
    h->last_error = msg;
    if (h->b) h->b->last_error = msg;
  }
  return s;
}

#define CUDA_TRY(h, expr)                                                                                      \
  do {                                                                                                         \
    cudaError_t e_ = (expr);                                                                                   \
    if (e_ != cudaSuccess) return hfail((h), MPMGPU_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define TRY(expr)                   \
  do {                              \
    mpmgpu_status s_ = (expr);      \
    if (s_ != MPMGPU_OK) return s_; \
  } while (0)

int grid_blocks(int64_t work, int threads) {
  int64_t b = (work + threads - 1) / threads;
  const int64_t cap = 148 * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

mpmgpu_status check_launch(mpmgpu_handle* h, const char* what) {
  h->extra_launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return hfail(h, MPMGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return MPMGPU_OK;
}

std::unique_ptr<BatchBase> make_batch(int dim, int mode, int device, int sort_interval, int cap, int use_graph,
                                      int keep_debug, mpmgpu_status* st, std::string* msg) {
  std::unique_ptr<BatchBase> b;
  if (mode == MPMGPU_MODE_FP64 || mode == MPMGPU_MODE_FP64_DETERMINISTIC) {
    auto p = std::make_unique<Batch<double>>(dim, device, sort_interval, cap, use_graph, keep_debug,
                                             mode == MPMGPU_MODE_FP64_DETERMINISTIC);
    *st = p->init();
    *msg = p->last_error;
    b = std::move(p);
  } else {
    auto p = std::make_unique<Batch<float>>(dim, device, sort_interval, cap, use_graph, keep_debug);
    *st = p->init();
    *msg = p->last_error;
    b = std::move(p);
  }
  return b;
}

mpmgpu_status start(mpmgpu_handle* h) {
  if (h->started) return MPMGPU_OK;
  TRY(h->b->admit(h->job));
  h->started = true;
  return MPMGPU_OK;
}

}  // namespace

extern "C" {

const char* mpmgpu_status_string(mpmgpu_status s) {
  switch (s) {
    case MPMGPU_OK: return "ok";
    case MPMGPU_ERR_ARG: return "invalid argument";
    case MPMGPU_ERR_CUDA: return "CUDA error";
    case MPMGPU_ERR_NOMEM: return "out of memory";
    case MPMGPU_ERR_UNSUPPORTED: return "unsupported";
    case MPMGPU_ERR_STATE: return "invalid state";
    case MPMGPU_ERR_DEVICE: return "device error flag";
  }
  return "unknown";
}

const char* mpmgpu_last_error(const mpmgpu_handle* h) {
  if (!h) return "";
  return h->b ? h->b->last_error.c_str() : h->last_error.c_str();
}

mpmgpu_status mpmgpu_create(const mpmgpu_config* cfg, mpmgpu_handle** out) {
  if (!cfg || !out) return MPMGPU_ERR_ARG;
  *out = nullptr;
  if (cfg->dim != 2 && cfg->dim != 3) return MPMGPU_ERR_UNSUPPORTED;
  if (!(cfg->dt > 0)) return MPMGPU_ERR_ARG;
  if (cfg->cpdi_spec != 0 && cfg->cpdi_spec != 1) return MPMGPU_ERR_ARG;
  if (cfg->contact_spec != 0 && cfg->contact_spec != 1) return MPMGPU_ERR_ARG;
  if (cfg->mode != MPMGPU_MODE_FP64 && cfg->mode != MPMGPU_MODE_MIXED && cfg->mode != MPMGPU_MODE_FP64_DETERMINISTIC)
    return MPMGPU_ERR_UNSUPPORTED;
  if (cfg->sort_interval < 0) return MPMGPU_ERR_ARG;
  for (int d = 0; d < cfg->dim; d++)
    if (cfg->N[d] < 1 || !(cfg->L[d] > 0)) return MPMGPU_ERR_ARG;
  auto h = std::make_unique<mpmgpu_handle>();
  h->cfg = *cfg;
  mpmgpu_status st = MPMGPU_OK;
  std::string msg;
  h->b = make_batch(cfg->dim, cfg->mode, cfg->device, cfg->sort_interval, 0, 1, cfg->keep_debug, &st, &msg);
  if (st != MPMGPU_OK) return st;
  // one job that runs until the handle is destroyed
  TRY(h->b->new_job(*cfg, INT64_MAX, &h->job));
  *out = h.release();
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_add_body(mpmgpu_handle* h, const mpmgpu_body_desc* desc, int* body_id) {
  if (!h || !desc) return MPMGPU_ERR_ARG;
  if (h->started) return hfail(h, MPMGPU_ERR_STATE, "bodies must be added before the first step");
  return h->b->add_body(h->job, *desc, body_id);
}

mpmgpu_status mpmgpu_add_contact(mpmgpu_handle* h, int body1, int body2, double mu_f, int* contact_id) {
  if (!h) return MPMGPU_ERR_ARG;
  if (h->started) return hfail(h, MPMGPU_ERR_STATE, "contacts must be added before the first step");
  return h->b->add_contact(h->job, body1, body2, mu_f, contact_id);
}

mpmgpu_status mpmgpu_add_contact_reflected(mpmgpu_handle* h, int body1, int body2, double mu_f, int* contact_id) {
  if (!h) return MPMGPU_ERR_ARG;
  if (h->started) return hfail(h, MPMGPU_ERR_STATE, "contacts must be added before the first step");
  return h->b->add_contact(h->job, body1, body2, mu_f, contact_id, 1);
}

mpmgpu_status mpmgpu_set_gravity(mpmgpu_handle* h, int use_vector, const double g[3]) {
  if (!h) return MPMGPU_ERR_ARG;
  return h->b->set_gravity(h->job, use_vector, g);
}

mpmgpu_status mpmgpu_step(mpmgpu_handle* h, int nsteps) {
  if (!h || nsteps < 0) return MPMGPU_ERR_ARG;
  int64_t n = 0;
  TRY(h->b->sizes(h->job, 0, &n, nullptr) == MPMGPU_OK ? MPMGPU_OK : hfail(h, MPMGPU_ERR_STATE, "no bodies"));
  TRY(start(h));
  return h->b->step(nsteps);
}

mpmgpu_status mpmgpu_synchronize(mpmgpu_handle* h) {
  if (!h) return MPMGPU_ERR_ARG;
  return h->b->synchronize();
}

mpmgpu_status mpmgpu_sizes(const mpmgpu_handle* h, int body, int64_t* n_points, int64_t* n_nodes) {
  if (!h) return MPMGPU_ERR_ARG;
  return h->b->sizes(h->job, body, n_points, n_nodes);
}

int64_t mpmgpu_launch_count(const mpmgpu_handle* h) { return h ? h->b->launches() + h->extra_launches : 0; }

void* mpmgpu_stream(const mpmgpu_handle* h) { return h ? (void*)h->b->stream() : nullptr; }

mpmgpu_status mpmgpu_active_nodes(mpmgpu_handle* h, int64_t* nodes, int64_t* drifted) {
  if (!h) return MPMGPU_ERR_ARG;
  return h->b->active_nodes(nodes, drifted);
}

mpmgpu_status mpmgpu_set_kernel(mpmgpu_handle* h, int form, int points_per_item) {
  if (!h) return MPMGPU_ERR_ARG;
  return h->b->set_kernel(form, points_per_item);
}

mpmgpu_status mpmgpu_kernel(const mpmgpu_handle* h, int* form, int* points_per_item) {
  if (!h) return MPMGPU_ERR_ARG;
  if (form) *form = h->b->kernel_form();
  if (points_per_item) *points_per_item = h->b->points_per_item();
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_autotune(mpmgpu_handle* h, int steps, int* form, int* points_per_item) {
  if (!h || steps < 1) return MPMGPU_ERR_ARG;
  int64_t n = 0;
  TRY(h->b->sizes(h->job, 0, &n, nullptr) == MPMGPU_OK ? MPMGPU_OK : hfail(h, MPMGPU_ERR_STATE, "no bodies"));
  TRY(start(h));
  int cap = 0;
  TRY(h->b->autotune(steps, &cap));
  if (form) *form = h->b->kernel_form();
  if (points_per_item) *points_per_item = cap;
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_set_wait_limit(mpmgpu_handle* h, uint32_t polls) {
  if (!h) return MPMGPU_ERR_ARG;
  h->b->set_wait_limit(polls);
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_profile(mpmgpu_handle* h, int enable) {
  if (!h) return MPMGPU_ERR_ARG;
  return h->b->profile(enable);
}

mpmgpu_status mpmgpu_profile_read(mpmgpu_handle* h, int stage, int64_t* launches, double* total_ms) {
  if (!h) return MPMGPU_ERR_ARG;
  return h->b->profile_read(stage, launches, total_ms);
}

mpmgpu_status mpmgpu_download_points(mpmgpu_handle* h, int body, int field, double* out) {
  if (!h || !out) return MPMGPU_ERR_ARG;
  return h->b->download_points(h->job, body, field, out);
}

mpmgpu_status mpmgpu_download_nodes(mpmgpu_handle* h, int body, int field, double* out) {
  if (!h || !out) return MPMGPU_ERR_ARG;
  return h->b->download_nodes(h->job, body, field, out);
}

mpmgpu_status mpmgpu_download_contact(mpmgpu_handle* h, int contact, int field, double* out) {
  if (!h || !out) return MPMGPU_ERR_ARG;
  return h->b->download_contact(h->job, contact, field, out);
}

mpmgpu_status mpmgpu_frame_begin(mpmgpu_handle* h) {
  if (!h) return MPMGPU_ERR_ARG;
  return h->b->frame_begin(h->job);
}

mpmgpu_status mpmgpu_frame_points(mpmgpu_handle* h, int body, int field, double* out) {
  if (!h || !out) return MPMGPU_ERR_ARG;
  return h->b->frame_points(h->job, body, field, out);
}

mpmgpu_status mpmgpu_frame_nodes(mpmgpu_handle* h, int body, int field, double* out) {
  if (!h || !out) return MPMGPU_ERR_ARG;
  return h->b->frame_nodes(h->job, body, field, out);
}

mpmgpu_status mpmgpu_frame_contact(mpmgpu_handle* h, int contact, int field, double* out) {
  if (!h || !out) return MPMGPU_ERR_ARG;
  return h->b->frame_contact(h->job, contact, field, out);
}

mpmgpu_status mpmgpu_dump_map(mpmgpu_handle* h, int body, int32_t* node, int32_t* point, double* s_val, double* grad,
                              int64_t* count) {
  if (!h || !count) return MPMGPU_ERR_ARG;
  PointsDev P{};
  Geom g{};
  int cpdi = 1;
  TRY(h->b->body_points_fp64(h->job, body, &P, &g, &cpdi));
  cudaStream_t st = h->b->stream();
  const int cp = g.cp;
  const size_t slots = (size_t)P.n * cp * cp;
  int32_t* dnode = nullptr;
  double *ds = nullptr, *dg = nullptr;
  CUDA_TRY(h, cudaMalloc(&dnode, std::max<size_t>(slots, 1) * sizeof(int32_t)));
  CUDA_TRY(h, cudaMalloc(&ds, std::max<size_t>(slots, 1) * sizeof(double)));
  CUDA_TRY(h, cudaMalloc(&dg, std::max<size_t>(slots, 1) * 3 * sizeof(double)));
  if (P.n > 0) {
    if (g.dim == 3)
      k_export_map<3><<<grid_blocks(P.n, 128), 128, 0, st>>>(g, cpdi, P, dnode, ds, dg);
    else
      k_export_map<2><<<grid_blocks(P.n, 128), 128, 0, st>>>(g, cpdi, P, dnode, ds, dg);
  }
  mpmgpu_status r = check_launch(h, "k_export_map");
  std::vector<int32_t> hn(slots);
  std::vector<double> hs(slots), hg(3 * slots);
  if (r == MPMGPU_OK && slots > 0) {
    cudaError_t e = cudaMemcpyAsync(hn.data(), dnode, slots * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hs.data(), ds, slots * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hg.data(), dg, 3 * slots * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = hfail(h, MPMGPU_ERR_CUDA, std::string("dump_map copy: ") + cudaGetErrorString(e));
  }
  cudaFree(dnode);
  cudaFree(ds);
  cudaFree(dg);
  if (r != MPMGPU_OK) return r;
  int64_t k = 0;
  const size_t per = (size_t)cp * cp;
  for (size_t i = 0; i < slots; i++) {
    if (hn[i] < 0) continue;
    if (node) {
      node[k] = hn[i];
      if (point) point[k] = (int32_t)(i / per);
      if (s_val) s_val[k] = hs[i];
      if (grad)
        for (int d = 0; d < 3; d++) grad[3 * k + d] = hg[3 * i + d];
    }
    k++;
  }
  *count = k;
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_destroy(mpmgpu_handle* h) {
  delete h;
  return MPMGPU_OK;
}

// ---------------------------------------------------------------------------
// Batch
// ---------------------------------------------------------------------------

const char* mpmgpu_batch_last_error(const mpmgpu_batch* b) {
  if (!b) return "";
  return b->b ? b->b->last_error.c_str() : b->last_error.c_str();
}

mpmgpu_status mpmgpu_batch_create(const mpmgpu_batch_config* cfg, mpmgpu_batch** out) {
  if (!cfg || !out) return MPMGPU_ERR_ARG;
  *out = nullptr;
  if (cfg->dim != 2 && cfg->dim != 3) return MPMGPU_ERR_UNSUPPORTED;
  if (cfg->mode != MPMGPU_MODE_FP64 && cfg->mode != MPMGPU_MODE_MIXED && cfg->mode != MPMGPU_MODE_FP64_DETERMINISTIC)
    return MPMGPU_ERR_UNSUPPORTED;
  if (cfg->sort_interval < 0 || cfg->points_per_item < 0) return MPMGPU_ERR_ARG;
  if (cfg->points_per_item != 0 &&
      !form_available(cfg->dim, cfg->mode == MPMGPU_MODE_MIXED, cfg->mode == MPMGPU_MODE_FP64_DETERMINISTIC,
                      kFormLean, cfg->points_per_item) &&
      !cap_available(cfg->dim, cfg->mode == MPMGPU_MODE_MIXED, cfg->points_per_item))
    return MPMGPU_ERR_UNSUPPORTED;
  auto b = std::make_unique<mpmgpu_batch>();
  b->cfg = *cfg;
  mpmgpu_status st = MPMGPU_OK;
  std::string msg;
  b->b = make_batch(cfg->dim, cfg->mode, cfg->device, cfg->sort_interval, cfg->points_per_item, !cfg->no_graph,
                    cfg->keep_debug, &st, &msg);
  if (st != MPMGPU_OK) return st;
  *out = b.release();
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_batch_footprint(const mpmgpu_batch* b, const mpmgpu_job_desc* job, int64_t* bytes) {
  if (!b || !job || !job->grid || !bytes || job->nbodies < 0 || job->nbodies > kMaxBodies) return MPMGPU_ERR_ARG;
  if (job->nbodies > 0 && !job->bodies) return MPMGPU_ERR_ARG;
  *bytes = job_footprint(*job->grid, b->cfg.mode, b->cfg.keep_debug != 0, job->bodies, job->nbodies, job->ncontacts);
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_batch_add_job(mpmgpu_batch* b, const mpmgpu_job_desc* job, int* job_id) {
  if (!b || !job || !job->grid || job->nbodies < 1 || !job->bodies || job->ncontacts < 0 ||
      (job->ncontacts > 0 && !job->contacts))
    return MPMGPU_ERR_ARG;
  mpmgpu_config cfg = *job->grid;
  cfg.dim = b->cfg.dim;
  int id = -1;
  TRY(b->b->new_job(cfg, job->steps, &id));
  mpmgpu_status st = MPMGPU_OK;
  for (int i = 0; i < job->nbodies && st == MPMGPU_OK; i++) st = b->b->add_body(id, job->bodies[i], nullptr);
  for (int c = 0; c < job->ncontacts && st == MPMGPU_OK; c++)
    st = b->b->add_contact(id, job->contacts[c].body1, job->contacts[c].body2, job->contacts[c].mu, nullptr,
                           job->contacts[c].reflected);
  if (st == MPMGPU_OK) st = b->b->set_gravity(id, job->gravity_vector, job->gravity);
  if (st == MPMGPU_OK) st = b->b->admit(id);
  if (st != MPMGPU_OK) {
    const std::string msg = b->b->last_error;
    b->b->remove_job(id);
    b->b->last_error = msg;
    return st;
  }
  if (job_id) *job_id = id;
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_batch_step(mpmgpu_batch* b, int nsteps) {
  if (!b || nsteps < 0) return MPMGPU_ERR_ARG;
  return b->b->step(nsteps);
}

mpmgpu_status mpmgpu_batch_synchronize(mpmgpu_batch* b) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->synchronize();
}

mpmgpu_status mpmgpu_batch_job_state(const mpmgpu_batch* b, int job, int64_t* steps_done, int64_t* steps_left) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->job_state(job, steps_done, steps_left);
}

mpmgpu_status mpmgpu_batch_sizes(const mpmgpu_batch* b, int job, int body, int64_t* n_points, int64_t* n_nodes) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->sizes(job, body, n_points, n_nodes);
}

mpmgpu_status mpmgpu_batch_download_points(mpmgpu_batch* b, int job, int body, int field, double* out) {
  if (!b || !out) return MPMGPU_ERR_ARG;
  return b->b->download_points(job, body, field, out);
}

mpmgpu_status mpmgpu_batch_download_points_many(mpmgpu_batch* b, int count, const int* jobs, int body, int field,
                                                double* const* outs, int threads) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->download_points_many(count, jobs, body, field, outs, threads);
}

mpmgpu_status mpmgpu_batch_remove_job(mpmgpu_batch* b, int job) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->remove_job(job);
}

mpmgpu_status mpmgpu_batch_counts(const mpmgpu_batch* b, int* live_jobs, int64_t* live_points, int64_t* bytes_in_use) {
  if (!b) return MPMGPU_ERR_ARG;
  b->b->counts(live_jobs, live_points);
  if (bytes_in_use) *bytes_in_use = b->b->memory_in_use();
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_batch_autotune(mpmgpu_batch* b, int steps, int* points_per_item) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->autotune(steps, points_per_item);
}

mpmgpu_status mpmgpu_batch_profile(mpmgpu_batch* b, int enable) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->profile(enable);
}

mpmgpu_status mpmgpu_batch_profile_read(mpmgpu_batch* b, int stage, int64_t* launches, double* total_ms) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->profile_read(stage, launches, total_ms);
}

int mpmgpu_batch_points_per_item(const mpmgpu_batch* b) { return b ? b->b->points_per_item() : 0; }
int mpmgpu_batch_kernel_form(const mpmgpu_batch* b) { return b ? b->b->kernel_form() : -1; }

mpmgpu_status mpmgpu_batch_set_kernel(mpmgpu_batch* b, int form, int points_per_item) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->set_kernel(form, points_per_item);
}

int mpmgpu_batch_sort_interval(const mpmgpu_batch* b) { return b ? b->b->sort_interval() : 0; }

mpmgpu_status mpmgpu_batch_active_nodes(mpmgpu_batch* b, int64_t* nodes, int64_t* drifted) {
  if (!b) return MPMGPU_ERR_ARG;
  return b->b->active_nodes(nodes, drifted);
}

void* mpmgpu_batch_stream(const mpmgpu_batch* b) { return b ? (void*)b->b->stream() : nullptr; }

int64_t mpmgpu_batch_launch_count(const mpmgpu_batch* b) { return b ? b->b->launches() : 0; }

mpmgpu_status mpmgpu_batch_destroy(mpmgpu_batch* b) {
  delete b;
  return MPMGPU_OK;
}

// ---------------------------------------------------------------------------
// Server
// ---------------------------------------------------------------------------

mpmgpu_status mpmgpu_server_create(const mpmgpu_batch_config* cfg, int64_t budget_bytes, mpmgpu_server** out) {
  if (!cfg || !out || budget_bytes <= 0) return MPMGPU_ERR_ARG;
  *out = nullptr;
  if (cfg->dim != 2 && cfg->dim != 3) return MPMGPU_ERR_UNSUPPORTED;
  if (cfg->mode != MPMGPU_MODE_FP64 && cfg->mode != MPMGPU_MODE_MIXED && cfg->mode != MPMGPU_MODE_FP64_DETERMINISTIC)
    return MPMGPU_ERR_UNSUPPORTED;
  if (cfg->points_per_item != 0 &&
      !form_available(cfg->dim, cfg->mode == MPMGPU_MODE_MIXED, cfg->mode == MPMGPU_MODE_FP64_DETERMINISTIC,
                      kFormLean, cfg->points_per_item) &&
      !cap_available(cfg->dim, cfg->mode == MPMGPU_MODE_MIXED, cfg->points_per_item))
    return MPMGPU_ERR_UNSUPPORTED;
  mpmgpu_status st = MPMGPU_OK;
  std::string msg;
  // the batch's default kernel (in 3D point per thread, 512 points per
  // work item), unless the caller picks the size
  const int cap = cfg->points_per_item;
  auto b = make_batch(cfg->dim, cfg->mode, cfg->device, cfg->sort_interval, cap, !cfg->no_graph, cfg->keep_debug, &st,
                      &msg);
  if (st != MPMGPU_OK) return st;
  auto srv = std::make_unique<mpmgpu_server>();
  srv->s = std::make_unique<Server>(std::move(b), cfg->mode, cfg->keep_debug != 0, budget_bytes);
  *out = srv.release();
  return MPMGPU_OK;
}

const char* mpmgpu_server_last_error(const mpmgpu_server* s) { return s ? s->s->last_error.c_str() : ""; }

mpmgpu_status mpmgpu_server_footprint(const mpmgpu_server* s, const mpmgpu_job_desc* job, int64_t* bytes) {
  if (!s || !job || !bytes) return MPMGPU_ERR_ARG;
  return s->s->footprint(*job, bytes);
}

mpmgpu_status mpmgpu_server_submit(mpmgpu_server* s, const mpmgpu_job_desc* job, int* request_id) {
  if (!s || !job || !request_id) return MPMGPU_ERR_ARG;
  return s->s->submit(*job, request_id);
}

mpmgpu_status mpmgpu_server_advance(mpmgpu_server* s, int steps) {
  if (!s) return MPMGPU_ERR_ARG;
  return s->s->advance(steps);
}

int mpmgpu_server_poll(mpmgpu_server* s, int* ids, int max_ids) {
  if (!s || !ids || max_ids <= 0) return 0;
  return s->s->poll(ids, max_ids);
}

mpmgpu_status mpmgpu_server_request(const mpmgpu_server* s, int id, int* state, double* t_admit, double* t_done,
                                    int64_t* points, int64_t* steps) {
  if (!s) return MPMGPU_ERR_ARG;
  return s->s->request(id, state, t_admit, t_done, points, steps);
}

mpmgpu_status mpmgpu_server_result(mpmgpu_server* s, int id, int body, int field, double* out) {
  if (!s) return MPMGPU_ERR_ARG;
  return s->s->result(id, body, field, out);
}

mpmgpu_status mpmgpu_server_cancel(mpmgpu_server* s, int id) {
  if (!s) return MPMGPU_ERR_ARG;
  return s->s->cancel(id);
}

mpmgpu_status mpmgpu_server_release(mpmgpu_server* s, int id) {
  if (!s) return MPMGPU_ERR_ARG;
  return s->s->release(id);
}

mpmgpu_status mpmgpu_server_stats(const mpmgpu_server* s, int* running, int64_t* reserved_bytes, int64_t* live_points,
                                  int64_t* particle_steps_done) {
  if (!s) return MPMGPU_ERR_ARG;
  s->s->stats(running, reserved_bytes, live_points, particle_steps_done);
  return MPMGPU_OK;
}

double mpmgpu_server_clock(const mpmgpu_server* s) { return s ? s->s->clock() : 0.0; }

mpmgpu_status mpmgpu_server_destroy(mpmgpu_server* s) {
  delete s;
  return MPMGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free map export (mpmgpu_dump_map_noalloc).
//
// For callers that must not allocate device memory when they read the map
// (caller-owned memory pools, real-time loops): the slot buffers that
// mpmgpu_dump_map takes from cudaMalloc live here in one static device
// array, and the compaction to the reference's triplet order runs on the
// device into the caller's arrays. Nothing is allocated on the host or the
// device by the call. The call waits for its result (a stream
// synchronisation), so it refuses to run on a stream under capture.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {

// Slots served per call: points x 4^dim triplets of k_export_map.
constexpr int64_t kNoAllocSlots = (int64_t)1 << 19;
constexpr int64_t kNoAllocBlocks = kNoAllocSlots / 1024;
// Carved into: node ids (int32), slot positions (int32), block offsets
// (int32, +1 total), S values (double), gradients (3 doubles).
constexpr size_t kNoAllocOffNode = 0;
constexpr size_t kNoAllocOffPos = kNoAllocOffNode + 4 * kNoAllocSlots;
constexpr size_t kNoAllocOffBlk = kNoAllocOffPos + 4 * kNoAllocSlots;
constexpr size_t kNoAllocOffS = kNoAllocOffBlk + 256 * ((4 * (kNoAllocBlocks + 1) + 255) / 256);
constexpr size_t kNoAllocOffGrad = kNoAllocOffS + 8 * kNoAllocSlots;
constexpr size_t kNoAllocBytes = kNoAllocOffGrad + 24 * kNoAllocSlots;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_base[kNoAllocMaxDevices] = {};
void* g_noalloc_ctx[kNoAllocMaxDevices] = {};   // context the address belongs to

// The current driver context of the calling thread (cuCtxGetCurrent, taken
// through the runtime's driver entry point: the library does not link the
// driver library itself). Null if it cannot be queried.
void* current_context() {
  using CtxGet = int (*)(void**);
  static CtxGet fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGet>(f);
  }();
  void* ctx = nullptr;
  if (fn == nullptr || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of the scratch array on `device`, looked up with that
// device current (in host code the symbol is only a stand-in) the first time
// and again whenever the device's context has changed since (after a device
// reset the module is loaded anew and the array may move).
mpmgpu_status noalloc_scratch(mpmgpu_handle* h, int device, unsigned char** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return hfail(h, MPMGPU_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  int current = 0;
  CUDA_TRY(h, cudaGetDevice(&current));
  if (current != device) CUDA_TRY(h, cudaSetDevice(device));
  void* ctx = current_context();
  cudaError_t e = cudaSuccess;
  if (g_noalloc_base[device] == nullptr || ctx != g_noalloc_ctx[device]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e == cudaSuccess) {
      g_noalloc_base[device] = static_cast<unsigned char*>(p);
      g_noalloc_ctx[device] = ctx;
    }
  }
  if (current != device) CUDA_TRY(h, cudaSetDevice(current));
  if (e != cudaSuccess)
    return hfail(h, MPMGPU_ERR_CUDA, std::string("cudaGetSymbolAddress(map scratch): ") + cudaGetErrorString(e));
  *out = g_noalloc_base[device];
  return MPMGPU_OK;
}

// Exclusive scan, per 1024-slot block, of the "slot holds a triplet" flags;
// block totals go to blk[blockIdx.x].
__global__ void k_noalloc_slot_scan(const int32_t* node, int64_t nslots, int32_t* pos, int32_t* blk) {
  __shared__ int32_t warp_sums[32];
  const int64_t i = blockIdx.x * 1024LL + threadIdx.x;
  const int flag = (i < nslots && node[i] >= 0) ? 1 : 0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = flag;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int ws = warp_sums[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += y;
    }
    warp_sums[lane] = ws;
  }
  __syncthreads();
  const int before = wid > 0 ? warp_sums[wid - 1] : 0;
  if (i < nslots) pos[i] = before + incl - flag;
  if (threadIdx.x == 1023) blk[blockIdx.x] = before + incl;
}

// Writes the occupied slots, in slot order, to the caller's device arrays.
__global__ void k_noalloc_compact(const int32_t* node, const double* s, const double* grad, const int32_t* pos,
                                  const int32_t* blk, int64_t nslots, int per_point, int32_t* d_node, int32_t* d_point,
                                  double* d_s, double* d_grad, int64_t capacity) {
  const int64_t i = blockIdx.x * 1024LL + threadIdx.x;
  if (i >= nslots || node[i] < 0) return;
  const int64_t k = (int64_t)blk[blockIdx.x] + pos[i];
  if (k >= capacity) return;
  d_node[k] = node[i];
  d_point[k] = (int32_t)(i / per_point);
  d_s[k] = s[i];
  for (int c = 0; c < 3; c++) d_grad[3 * k + c] = grad[3 * i + c];
}

}  // namespace

extern "C" mpmgpu_status mpmgpu_dump_map_noalloc(mpmgpu_handle* h, int body, int32_t* d_node, int32_t* d_point,
                                                  double* d_s, double* d_grad, int64_t capacity, int64_t* count) {
  if (!h || !count) return MPMGPU_ERR_ARG;
  if (capacity < 0 || (capacity > 0 && (!d_node || !d_point || !d_s || !d_grad)))
    return hfail(h, MPMGPU_ERR_ARG, "output arrays missing");
  PointsDev P{};
  Geom g{};
  int cpdi = 1;
  TRY(h->b->body_points_fp64(h->job, body, &P, &g, &cpdi));
  const int per_point = g.cp * g.cp;
  const int64_t nslots = P.n * per_point;
  if (nslots > kNoAllocSlots)
    return hfail(h, MPMGPU_ERR_ARG,
                 "mpmgpu_dump_map_noalloc: body has " + std::to_string(P.n) + " points x " + std::to_string(per_point) +
                     " triplet slots = " + std::to_string(nslots) + " slots, above the static scratch limit of " +
                     std::to_string(kNoAllocSlots));
  cudaStream_t st = h->b->stream();
  {
    // the call ends with a wait for its result, which a stream under capture
    // cannot do; refuse before queuing anything, so the caller's capture
    // stays valid
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CUDA_TRY(h, cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone)
      return hfail(h, MPMGPU_ERR_UNSUPPORTED,
                   "mpmgpu_dump_map_noalloc waits for its result and cannot run while the handle's stream is captured");
  }
  unsigned char* base = nullptr;
  TRY(noalloc_scratch(h, h->cfg.device, &base));
  int32_t* node = reinterpret_cast<int32_t*>(base + kNoAllocOffNode);
  int32_t* pos = reinterpret_cast<int32_t*>(base + kNoAllocOffPos);
  int32_t* blk = reinterpret_cast<int32_t*>(base + kNoAllocOffBlk);
  double* s = reinterpret_cast<double*>(base + kNoAllocOffS);
  double* grad = reinterpret_cast<double*>(base + kNoAllocOffGrad);
  // every slot read below is written first by this call: nothing carries over
  if (P.n > 0) {
    if (g.dim == 3)
      k_export_map<3><<<grid_blocks(P.n, 128), 128, 0, st>>>(g, cpdi, P, node, s, grad);
    else
      k_export_map<2><<<grid_blocks(P.n, 128), 128, 0, st>>>(g, cpdi, P, node, s, grad);
    TRY(check_launch(h, "k_export_map"));
  }
  const int nblk = (int)((nslots + 1023) / 1024);
  if (nblk > 0) {
    k_noalloc_slot_scan<<<nblk, 1024, 0, st>>>(node, nslots, pos, blk);
    TRY(check_launch(h, "k_noalloc_slot_scan"));
  }
  k_scan_small<<<1, 1024, 0, st>>>(blk, nblk, blk + nblk);
  TRY(check_launch(h, "k_scan_small"));
  if (nblk > 0 && capacity > 0) {
    k_noalloc_compact<<<nblk, 1024, 0, st>>>(node, s, grad, pos, blk, nslots, per_point, d_node, d_point, d_s, d_grad,
                                             capacity);
    TRY(check_launch(h, "k_noalloc_compact"));
  }
  int32_t total = 0;
  CUDA_TRY(h, cudaMemcpyAsync(&total, blk + nblk, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  *count = total;
  if (total > capacity) return hfail(h, MPMGPU_ERR_ARG, "capacity below the triplet count");
  return MPMGPU_OK;
}

// ---- .points files (host only) ----

mpmgpu_status mpmgpu_points_file_count(const char* path, int64_t* n) {
  if (!path || !n) return MPMGPU_ERR_ARG;
  return mpmb200::points_file_count(path, n).ok ? MPMGPU_OK : MPMGPU_ERR_ARG;
}

mpmgpu_status mpmgpu_points_file_read(const char* path, int dim, int64_t n, double* m, double* v, double* x,
                                      double* x_t, int32_t* active, int threads, int64_t* bad_line) {
  if (bad_line) *bad_line = 0;
  if (!path || (dim != 2 && dim != 3) || n < 0 || (n > 0 && (!m || !v || !x || !x_t || !active)))
    return MPMGPU_ERR_ARG;
  const mpmb200::PointsFileResult r = mpmb200::points_file_read(path, dim, n, m, v, x, x_t, active, threads);
  if (bad_line) *bad_line = r.bad_line;
  return r.ok ? MPMGPU_OK : MPMGPU_ERR_ARG;
}
