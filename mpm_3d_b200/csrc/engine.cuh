// Host side of the step engine: a batch of independent jobs (each one the
// reference's Job: a CartesianLinear grid, its DefaultBodies and
// ContactHuang pairs) advanced together, one launch per stage for the whole
// batch:
//
//   compact   active node blocks flagged by the last scatter -> work list
//   grid      body force, contact, boundary, moveGrid on the active blocks
//   g2p2g     per bin of points: gather + point update (this step), map
//             build + scatter at the new positions (next step)
//
// plus, every sort_interval steps and whenever jobs join or leave, a
// re-binning of every body's points. A job that joins is binned and primed
// (a scatter-only pass of its bodies builds its first nodal sums) at the
// next step boundary while the others keep their state; a job that has run
// its steps stops advancing and keeps its state readable until removed.
//
// Kernels read sizes and per-job / per-body parameters from device tables,
// so the step and the re-binning are captured once in CUDA graphs and stay
// valid while jobs come and go (they are re-captured only when a capacity
// grows). The single-job C ABI (mpmgpu_handle) is a batch of one job.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <set>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "fused.cuh"
#include "frame.cuh"
#include "fused_lean.cuh"
#include "kernels_fp64.cuh"
#include "sort.cuh"

namespace mpmb200 {

#define MPM_CUDA_TRY(expr)                                                                            \
  do {                                                                                                \
    cudaError_t e_ = (expr);                                                                          \
    if (e_ != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define MPM_TRY(expr)               \
  do {                              \
    mpmgpu_status s_ = (expr);      \
    if (s_ != MPMGPU_OK) return s_; \
  } while (0)

// Stages of the per-stage event profile.
enum { kStageFused = 0, kStageGrid = 1, kStageCompact = 2, kStageRebin = 3, kStages = 4 };

// Grid geometry of a job from its config (CartesianLinear::init,
// cartesian.cpp:24-67) and the node-block / bin layouts.
inline void make_geometry(const mpmgpu_config& cfg, Geom& g, MapConst& mc, BinGeom& bg) {
  g = Geom{};
  mc = MapConst{};
  bg = BinGeom{};
  g.dim = cfg.dim;
  g.cp = 1 << cfg.dim;
  g.nnodes = 1;
  for (int d = 0; d < 3; d++) {
    if (d < cfg.dim) {
      g.L[d] = cfg.L[d];
      g.N[d] = cfg.N[d];
      g.h[d] = cfg.L[d] / cfg.N[d];  // cartesian.cpp:40
      g.nn[d] = cfg.N[d] + 1;
      g.nnodes *= g.nn[d];
      mc.NL[d] = (double)cfg.N[d] / cfg.L[d];
      mc.invh[d] = 1.0 / g.h[d];
    } else {
      g.nn[d] = 1;
    }
    mc.invhf[d] = (float)mc.invh[d];
  }
  if (cfg.dim == 3) {
    g.bsh[0] = g.bsh[1] = g.bsh[2] = 2;
  } else {
    g.bsh[0] = g.bsh[1] = 3;
    g.bsh[2] = 0;
  }
  g.nblocks = 1;
  for (int d = 0; d < 3; d++) {
    const int ext = 1 << g.bsh[d];
    g.nb[d] = (g.nn[d] + ext - 1) / ext;
    g.nblocks *= g.nb[d];
  }
  g.nslots = g.nblocks * 64;
  bg.B = cfg.dim == 3 ? 4 : 8;
  bg.cells_per_bin = 64;
  bg.nbx = (g.N[0] + bg.B - 1) / bg.B;
  bg.nby = (g.N[1] + bg.B - 1) / bg.B;
  bg.nbz = cfg.dim == 3 ? (g.N[2] + bg.B - 1) / bg.B : 1;
  bg.nbins = bg.nbx * bg.nby * bg.nbz;
  bg.T = bg.B + 3;
  bg.tile_nodes = cfg.dim == 3 ? bg.T * bg.T * bg.T : bg.T * bg.T;
}

// IsotropicLinearElasticity constants, isolin.cpp:34-38.
// props: a Sand_SachithLocal body's grain diameter, mu_s, grains_rho,
// rho_critical, mu_2 and I_0 (kind 2 only); flags bit 0:
// USE_DENSITY_FOR_PRESSURE.
inline MaterialParams make_material(int has_material, double E, double nu, int kind = 0,
                                    const double* props = nullptr, int flags = 0) {
  MaterialParams m{};
  m.has_material = has_material;
  m.kind = has_material ? kind : 0;
  if (has_material) {
    const double G = E / (2.0 * (1.0 + nu));
    const double K = E / (3.0 * (1.0 - 2 * nu));
    m.G = G;
    m.K = K;
    m.lambda = K - 2.0 * G / 3.0;
  }
  if (m.kind == 2 && props) {
    m.grains_d = props[0];
    m.mu_s = props[1];
    m.grains_rho = props[2];
    m.rho_critical = props[3];
    m.mu_2 = props[4];
    m.i_0 = props[5];
    m.use_density = flags & 1;
  }
  return m;
}

// Extent of a point, default_points.cpp:49-57 (computed once, never updated).
inline double point_extent(int dim, double vol) { return dim == 2 ? 0.5 * std::sqrt(vol) : 0.5 * std::cbrt(vol); }

// Particles per work item (CTA) of the staged kernel available for each
// dimension and precision.
inline bool cap_available(int dim, bool mixed, int cap) {
  if (dim == 3) return mixed ? (cap == 256 || cap == 512 || cap == 1024) : (cap == 256 || cap == 512);
  return cap == 512;
}

// Forms of the fused kernel (mpmgpu_set_kernel): the staged kernel
// (fused.cuh: point arrays staged in shared memory, gather and scatter
// phases apart, up to 1024 points per CTA) and the point-per-thread kernel
// (fused_lean.cuh, 3D, not the deterministic form).
enum { kFormStaged = 0, kFormLean = 1 };

inline bool form_available(int dim, bool mixed, bool det, int form, int cap) {
  if (form == kFormStaged) return cap_available(dim, mixed, cap);
  if (form == kFormLean) return dim == 3 && !det && lean_size_ok(cap);
  return false;
}

// Device bytes a job will hold: points (two buffers, with the material's
// per-point state), nodal arrays (with the deterministic form's second
// level), binning and its share of the batch's scratch.
inline int64_t job_footprint(const mpmgpu_config& cfg, int mode, bool keep_debug, const mpmgpu_body_desc* bodies,
                             int nbodies, int ncontacts) {
  Geom g;
  MapConst mc;
  BinGeom bg;
  make_geometry(cfg, g, mc, bg);
  const bool mixed = mode == MPMGPU_MODE_MIXED;
  const int64_t ps = mixed ? 4 : 8;
  int64_t bytes = 0;
  for (int b = 0; b < nbodies; b++) {
    const int64_t n = bodies[b].n + 8;
    const int nstate = material_state_arrays(bodies[b].has_material, bodies[b].material_kind);
    // two point buffers (+ the 256-byte alignment of every array); the
    // mixed form adds the low words of x, x_t and m
    const int nlow = mixed ? 7 : 0;
    bytes += 2 * n * ((18 + nstate + nlow) * ps + 8) + (96 + 2 * nlow) * 256;
    if (keep_debug && !mixed) bytes += 2 * n * 72;
    bytes += g.nslots * 8 * (7 + 6);            // accumulators + velocities
    if (mode == MPMGPU_MODE_FP64_DETERMINISTIC) bytes += g.nslots * 8 * 7;
    bytes += n * 10;                             // sort key, rank, class rank
    bytes += ((int64_t)bg.nbins * bg.cells_per_bin + 1) * 12 + ((int64_t)bg.nbins + 2) * 4;
    bytes += ((int64_t)bg.nbins + n / 256 + 1) * 16;
    if (keep_debug) bytes += g.nslots * 8 * 7;
  }
  bytes += (int64_t)ncontacts * g.nslots * 8 * (3 + (keep_debug ? 6 : 0));
  bytes += g.nblocks * (4 + 8 + 1 + 4);
  return bytes;
}

// Process-wide device memory pools, one per device: batches allocate their
// jobs' arrays from it in stream order, and a closed batch's memory stays
// reserved for the next batch (mapping and unmapping device pages is what
// makes a batch slow to create and to close). A closing batch trims the
// pool to kPoolKeepBytes.
constexpr size_t kPoolKeepBytes = (size_t)48 << 30;

inline cudaError_t shared_pool(int device, cudaMemPool_t* out) {
  static std::mutex m;
  static cudaMemPool_t pools[64] = {};
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(m);
  if (!pools[device]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    pools[device] = pool;
  }
  *out = pools[device];
  return cudaSuccess;
}

// Process-wide cache of pinned host buffers (staging of uploads, downloads
// and frames): pinning and unpinning pages costs about as much as the copy
// itself, so a closed batch's buffers serve the next one. At most
// kPinnedKeepBytes stay cached.
constexpr size_t kPinnedKeepBytes = (size_t)4 << 30;

struct PinnedCache {
  std::mutex m;
  std::vector<std::pair<void*, size_t>> free;
  size_t held = 0;
};
inline PinnedCache& pinned_cache() {
  static PinnedCache c;
  return c;
}
// A pinned buffer of at least `bytes` (its size in *cap).
inline cudaError_t pinned_take(size_t bytes, void** out, size_t* cap) {
  PinnedCache& c = pinned_cache();
  {
    std::lock_guard<std::mutex> lock(c.m);
    size_t best = c.free.size();
    for (size_t i = 0; i < c.free.size(); i++)
      if (c.free[i].second >= bytes && (best == c.free.size() || c.free[i].second < c.free[best].second)) best = i;
    if (best < c.free.size()) {
      *out = c.free[best].first;
      *cap = c.free[best].second;
      c.held -= c.free[best].second;
      c.free.erase(c.free.begin() + (std::ptrdiff_t)best);
      return cudaSuccess;
    }
  }
  *cap = bytes;
  return cudaHostAlloc(out, bytes, cudaHostAllocDefault);
}
inline void pinned_give(void* p, size_t cap) {
  if (!p) return;
  PinnedCache& c = pinned_cache();
  std::lock_guard<std::mutex> lock(c.m);
  c.free.emplace_back(p, cap);
  c.held += cap;
  while (c.held > kPinnedKeepBytes && !c.free.empty()) {
    // drop the smallest first: large buffers are the expensive ones to pin
    size_t small = 0;
    for (size_t i = 1; i < c.free.size(); i++)
      if (c.free[i].second < c.free[small].second) small = i;
    cudaFreeHost(c.free[small].first);
    c.held -= c.free[small].second;
    c.free.erase(c.free.begin() + (std::ptrdiff_t)small);
  }
}

// Type-independent interface of a batch (the C ABI holds this).
class BatchBase {
 public:
  virtual ~BatchBase() = default;
  std::string last_error;
  mpmgpu_status fail(mpmgpu_status s, const std::string& msg) {
    last_error = msg;
    return s;
  }
  virtual int dim() const = 0;
  virtual bool mixed() const = 0;
  virtual cudaStream_t stream() const = 0;
  virtual int64_t launches() const = 0;
  virtual mpmgpu_status new_job(const mpmgpu_config& cfg, int64_t steps, int* job) = 0;
  virtual mpmgpu_status add_body(int job, const mpmgpu_body_desc& desc, int* body) = 0;
  virtual mpmgpu_status add_contact(int job, int b1, int b2, double mu, int* contact, int reflected = 0) = 0;
  virtual mpmgpu_status set_gravity(int job, int use_vector, const double* g) = 0;
  virtual mpmgpu_status admit(int job) = 0;
  virtual mpmgpu_status step(int nsteps) = 0;
  virtual mpmgpu_status synchronize() = 0;
  virtual mpmgpu_status remove_job(int job) = 0;
  virtual mpmgpu_status job_state(int job, int64_t* done, int64_t* left) const = 0;
  virtual mpmgpu_status download_points(int job, int body, int field, double* out) = 0;
  // One point field of one body of each of `count` jobs, copied with one
  // wait and converted on up to `threads` host threads.
  virtual mpmgpu_status download_points_many(int count, const int* jobs, int body, int field, double* const* outs,
                                             int threads) = 0;
  // Raw point state of a body copied to host memory in stream order, i.e.
  // as it stands after the work queued so far (without waiting): x, u, x_t
  // (3 arrays each), stress (6) and V in the point precision (and the mixed
  // form's low words of x and x_t), then active and pid (int32). `host` is
  // pinned and holds snapshot_bytes(n).
  virtual size_t snapshot_bytes(int64_t n) const = 0;
  virtual mpmgpu_status snapshot_body(int job, int body, void* host) = 0;
  // The fields of a completed snapshot in reference point order, as
  // download_points gives them (x, u, x_t: 3 per point; T: 9; V; active).
  virtual void snapshot_fields(const void* host, int64_t n, double* x, double* u, double* x_t, double* T, double* v,
                               double* active) const = 0;
  virtual mpmgpu_status download_nodes(int job, int body, int field, double* out) = 0;
  virtual mpmgpu_status download_contact(int job, int contact, int field, double* out) = 0;
  // Frames: every body's point, node and contact fields of a job copied to
  // pinned host memory behind the work queued so far, without waiting
  // (frame_begin); frame_points / _nodes / _contact wait for those copies
  // (once) and convert one field to the reference layout, while later work
  // queued on the stream runs. A frame stays readable until the next
  // frame_begin.
  virtual mpmgpu_status frame_begin(int job) = 0;
  virtual mpmgpu_status frame_points(int job, int body, int field, double* out) = 0;
  virtual mpmgpu_status frame_nodes(int job, int body, int field, double* out) = 0;
  virtual mpmgpu_status frame_contact(int job, int contact, int field, double* out) = 0;
  virtual mpmgpu_status sizes(int job, int body, int64_t* n_points, int64_t* n_nodes) const = 0;
  virtual mpmgpu_status profile(int enable) = 0;
  virtual mpmgpu_status profile_read(int stage, int64_t* launches, double* ms) = 0;
  virtual mpmgpu_status autotune(int steps, int* best_cap) = 0;
  // Poll limit of the fused kernels' waits for bulk copies (kWaitPolls by
  // default); a wait that runs out makes the step report MPMGPU_ERR_DEVICE.
  virtual void set_wait_limit(uint32_t polls) = 0;
  virtual int64_t memory_in_use() const = 0;
  virtual void counts(int* live_jobs, int64_t* live_points) const = 0;
  virtual int points_per_item() const = 0;
  virtual int sort_interval() const = 0;
  // Form of the fused kernel (kFormStaged, kFormLean) and
  // its points per work item; chosen at creation (the point-per-thread
  // kernel with 512 points in 3D, the staged kernel otherwise), by the
  // autotuner, or by set_kernel.
  virtual int kernel_form() const = 0;
  virtual mpmgpu_status set_kernel(int form, int cap) = 0;
  virtual mpmgpu_status active_nodes(int64_t* nodes, int64_t* drifted) = 0;
  // FP64 map export support (single-job handle)
  virtual mpmgpu_status body_points_fp64(int job, int body, PointsDev* P, Geom* g, int* cpdi) = 0;
  virtual int device() const = 0;
};

template <typename PT>
class Batch : public BatchBase {
 public:
  struct HBody {
    int64_t n = 0;
    PointsT<PT> P{}, Palt{};
    NodesAcc A{}, snap{};
    NodesAcc Ar{};   // deterministic form: level-1 sums
    NodesVel V{};
    MaterialParams mat{};
    int has_boundary = 0;   // boundary kind (mpmgpu_body_desc.has_boundary)
    double mu_f = 0.0;
    int needs_normal = 0;
    int prime = 1;
    std::vector<void*> allocs;
  };
  struct HJob {
    mpmgpu_config cfg{};
    Geom g{};
    MapConst mc{};
    BinGeom bg{};
    StepParams sp{};
    std::vector<HBody> bodies;
    int nc = 0;
    int cb1[kMaxContacts] = {}, cb2[kMaxContacts] = {};
    double mu[kMaxContacts] = {};
    int reflected[kMaxContacts] = {};
    double* normal_out[kMaxContacts] = {};
    double* force_out[kMaxContacts] = {};
    std::vector<void*> allocs;
    int64_t block_off = -1;
    int slot = -1;           // stable index in the job table while stepped
    bool fill_pending = false;  // its block range still maps to another slot
    int64_t steps_done = 0, steps_left = 0;
    bool admitted = false;   // asked to join
    bool in_tables = false;  // part of the stepped set
    bool finished = false;
    bool removed = false;
    bool primed = false;     // has had its first scatter
    int64_t bytes = 0;
  };

  Batch(int dim, int device, int sort_interval, int cap, int use_graph, int keep_debug, bool det = false)
      : dim_(dim), device_(device), keep_debug_(keep_debug != 0), use_graph_(use_graph != 0), det_(det) {
    sort_interval_ = sort_interval > 0 ? sort_interval : 32;
    cap_ = cap;
  }

  mpmgpu_status init() {
    MPM_CUDA_TRY(cudaSetDevice(device_));
    MPM_CUDA_TRY(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device_));
    MPM_CUDA_TRY(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    MPM_CUDA_TRY(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
    MPM_CUDA_TRY(cudaEventCreateWithFlags(&upload_ev_, cudaEventDisableTiming));
    MPM_CUDA_TRY(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
    for (int i = 0; i < kSideStreams; i++) {
      MPM_CUDA_TRY(cudaStreamCreateWithFlags(&side_[i], cudaStreamNonBlocking));
      MPM_CUDA_TRY(cudaEventCreateWithFlags(&join_ev_[i], cudaEventDisableTiming));
    }
    // jobs' arrays come from the device's stream-ordered pool, which keeps
    // freed memory for the next job and the next batch (no device-wide
    // synchronisation per job)
    MPM_CUDA_TRY(shared_pool(device_, &pool_));
    // a requested item size is served by the point-per-thread kernel
    // where it has that size, else by the staged kernel
    if (cap_ == 0) cap_ = (dim_ == 3 && !det_) ? kDefaultLeanCap : default_cap();
    form_ = form_available(dim_, mixed(), det_, kFormLean, cap_) ? kFormLean : kFormStaged;
    if (!form_available(dim_, mixed(), det_, form_, cap_) || (det_ && cap_ != default_cap()))
      return fail(MPMGPU_ERR_ARG, "points_per_item " + std::to_string(cap_) + " not available for this form");
    if (det_ && mixed()) return fail(MPMGPU_ERR_UNSUPPORTED, "the deterministic form is FP64");
    MPM_TRY(alloc_raw(&hdr_, 1, scratch_allocs_));
    MPM_TRY(alloc_raw(&count_, 1, scratch_allocs_));
    MPM_TRY(alloc_raw(&err_, 1, scratch_allocs_));
    MPM_TRY(alloc_raw(&drift_, 1, scratch_allocs_));
    MPM_TRY(alloc_raw(&queue_, 2, scratch_allocs_));
    MPM_TRY(alloc_raw(&nwork_, 1, scratch_allocs_));
    MPM_TRY(alloc_raw(&active_nodes_, 1, scratch_allocs_));
    return MPMGPU_OK;
  }

  ~Batch() override {
    if (stream_) cudaStreamSynchronize(stream_);
    if (copy_stream_) cudaStreamSynchronize(copy_stream_);
    drop_graphs();
    for (int s = 0; s < kStages; s++)
      for (auto& pr : pending_[s]) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
      }
    for (cudaEvent_t e : event_pool_) cudaEventDestroy(e);
    for (auto& j : jobs_) free_job(j);
    if (stream_) cudaStreamSynchronize(stream_);
    for (void* p : scratch_allocs_) cudaFree(p);
    for (void* p : cap_allocs_) cudaFree(p);
    if (pool_) cudaMemPoolTrimTo(pool_, kPoolKeepBytes);
    pinned_give(stage_, stage_cap_);
    pinned_give(dl_stage_, dl_cap_);
    pinned_give(frame_stage_, frame_cap_);
    if (frame_dev_) cudaFree(frame_dev_);
    if (frame_ev_) cudaEventDestroy(frame_ev_);
    if (upload_ev_) cudaEventDestroy(upload_ev_);
    if (fork_ev_) cudaEventDestroy(fork_ev_);
    for (int i = 0; i < kSideStreams; i++) {
      if (side_[i]) cudaStreamSynchronize(side_[i]);
      if (side_[i]) cudaStreamDestroy(side_[i]);
      if (join_ev_[i]) cudaEventDestroy(join_ev_[i]);
    }
    if (copy_stream_) cudaStreamDestroy(copy_stream_);
    if (stream_) cudaStreamDestroy(stream_);
  }

  int dim() const override { return dim_; }
  bool mixed() const override { return sizeof(PT) == 4; }
  cudaStream_t stream() const override { return stream_; }
  int64_t launches() const override { return launches_; }
  int points_per_item() const override { return cap_; }

  // Nodes with mass (per body) in the last step's grid update, and points
  // found outside their bin's tile since the batch was created.
  mpmgpu_status active_nodes(int64_t* nodes, int64_t* drifted) override {
    MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
    unsigned long long a = 0, d = 0;
    MPM_CUDA_TRY(cudaMemcpy(&a, active_nodes_, sizeof(a), cudaMemcpyDeviceToHost));
    MPM_CUDA_TRY(cudaMemcpy(&d, drift_, sizeof(d), cudaMemcpyDeviceToHost));
    if (nodes) *nodes = (int64_t)a;
    if (drifted) *drifted = (int64_t)d;
    return MPMGPU_OK;
  }
  int device() const override { return device_; }

  mpmgpu_status new_job(const mpmgpu_config& cfg, int64_t steps, int* job) override {
    if (cfg.dim != dim_) return fail(MPMGPU_ERR_ARG, "job dimension differs from the batch's");
    if (!(cfg.dt > 0)) return fail(MPMGPU_ERR_ARG, "dt must be positive");
    if (cfg.cpdi_spec != 0 && cfg.cpdi_spec != 1) return fail(MPMGPU_ERR_ARG, "cpdi_spec must be 0 or 1");
    if (cfg.contact_spec != 0 && cfg.contact_spec != 1) return fail(MPMGPU_ERR_ARG, "contact_spec must be 0 or 1");
    for (int d = 0; d < cfg.dim; d++)
      if (cfg.N[d] < 1 || !(cfg.L[d] > 0)) return fail(MPMGPU_ERR_ARG, "grid sizes must be positive");
    if (steps < 0) return fail(MPMGPU_ERR_ARG, "negative step count");
    HJob j;
    j.cfg = cfg;
    make_geometry(cfg, j.g, j.mc, j.bg);
    j.sp.dt = cfg.dt;
    j.sp.cpdi = cfg.cpdi_spec;
    j.sp.contact_spec = cfg.contact_spec;
    j.sp.keep_debug = keep_debug_ ? 1 : 0;
    // DefaultDriver gravity until set otherwise (default_driver.cpp:90-105)
    j.sp.grav[cfg.dim == 2 ? 1 : 2] = -9.81;
    j.steps_left = steps;
    jobs_.push_back(std::move(j));
    *job = (int)jobs_.size() - 1;
    return MPMGPU_OK;
  }

  mpmgpu_status add_body(int job, const mpmgpu_body_desc& desc, int* body) override {
    HJob* j;
    MPM_TRY(editable_job(job, &j));
    if ((int)j->bodies.size() >= kMaxBodies) return fail(MPMGPU_ERR_UNSUPPORTED, "too many bodies in a job");
    if (desc.n < 0 || desc.n > (int64_t)INT32_MAX / 2 || (desc.n > 0 && (!desc.m || !desc.v || !desc.x || !desc.x_t)))
      return fail(MPMGPU_ERR_ARG, "body arrays missing or too many points");
    if (desc.has_boundary < 0 || desc.has_boundary > 3) return fail(MPMGPU_ERR_ARG, "unknown boundary kind");
    const int D = dim_;
    const int64_t n = desc.n;
    HBody B;
    B.n = n;
    MPM_TRY(stage_reserve((size_t)n * (28 * sizeof(PT) + 8) + 64 * 256));
    const size_t ns = (size_t)j->g.nslots;
    if (desc.has_material && (desc.material_kind < 0 || desc.material_kind > 2))
      return fail(MPMGPU_ERR_ARG, "unknown material kind");
    const int nstate = material_state_arrays(desc.has_material, desc.material_kind);
    // both point buffers and the nodal arrays of the body
    MPM_TRY(alloc_arena(
        [&](Arena& a) {
          layout_points(a, B.P, n, nstate);
          layout_points(a, B.Palt, n, nstate);
          if (det_) {
            carve(a, &B.Ar.m, ns);
            for (int d = 0; d < 3; d++) {
              carve(a, &B.Ar.mx[d], ns);
              carve(a, &B.Ar.f[d], ns);
            }
          }
          carve(a, &B.A.m, ns);
          for (int d = 0; d < 3; d++) {
            carve(a, &B.A.mx[d], ns);
            carve(a, &B.A.f[d], ns);
            carve(a, &B.V.vt[d], ns);
            carve(a, &B.V.dv[d], ns);
          }
          if (keep_debug_) {
            carve(a, &B.snap.m, ns);
            for (int d = 0; d < 3; d++) {
              carve(a, &B.snap.mx[d], ns);
              carve(a, &B.snap.f[d], ns);
            }
          }
        },
        B.allocs, j->bytes));
    if (n > 0) {
      // each array is written straight into the pinned staging buffer (on
      // several host threads for large bodies) and copied on the copy stream
      auto col = [&](PT* dst, const double* aos, int w, int d) {
        return upload_fill(dst, n, [=](PT* h, int64_t a, int64_t b) {
          for (int64_t i = a; i < b; i++) h[i] = (PT)aos[i * w + d];
        });
      };
      // the mixed form's low words of x, x_t and m (hi + lo = the value)
      auto col_lo = [&](PT* dst, const double* aos, int w, int d) {
        return upload_fill(dst, n, [=](PT* h, int64_t a, int64_t b) {
          for (int64_t i = a; i < b; i++) {
            float hi, lo;
            split_two_word(aos[i * w + d], hi, lo);
            h[i] = (PT)lo;
          }
        });
      };
      for (int d = 0; d < D; d++) {
        MPM_TRY(col(B.P.x[d], desc.x, 3, d));
        MPM_TRY(col(B.P.v[d], desc.x_t, 3, d));
        if constexpr (sizeof(PT) == 4) {
          MPM_TRY(col_lo(B.P.xl[d], desc.x, 3, d));
          MPM_TRY(col_lo(B.P.vl[d], desc.x_t, 3, d));
        }
      }
      MPM_TRY(col(B.P.m, desc.m, 1, 0));
      if constexpr (sizeof(PT) == 4) MPM_TRY(col_lo(B.P.ml, desc.m, 1, 0));
      MPM_TRY(col(B.P.vol, desc.v, 1, 0));
      const double* vol0 = desc.v;
      MPM_TRY(upload_fill(B.P.ext, n, [=](PT* h, int64_t a, int64_t b) {
        for (int64_t i = a; i < b; i++) h[i] = (PT)point_extent(D, vol0[i]);
      }));
      if (desc.u)
        for (int d = 0; d < D; d++) MPM_TRY(col(B.P.u[d], desc.u, 3, d));
      if (desc.T) {
        // stored as xx yy zz xy yz xz (row-major 9 -> symmetric 6)
        static const int idx[6] = {0, 4, 8, 1, 5, 2};
        for (int c = 0; c < 6; c++) MPM_TRY(col(B.P.s[c], desc.T, 9, idx[c]));
      }
      const int32_t* act0 = desc.active;
      MPM_TRY(upload_fill(B.P.active, n, [=](int32_t* h, int64_t a, int64_t b) {
        for (int64_t i = a; i < b; i++) h[i] = act0 ? (act0[i] != 0 ? 1 : 0) : 1;
      }));
      MPM_TRY(upload_fill(B.P.pid, n, [](int32_t* h, int64_t a, int64_t b) {
        for (int64_t i = a; i < b; i++) h[i] = (int32_t)i;
      }));
    }
    B.mat = make_material(desc.has_material, desc.E, desc.nu, desc.material_kind, desc.material_props,
                          desc.material_flags);
    B.has_boundary = desc.has_boundary;
    B.mu_f = desc.boundary_mu;
    MPM_TRY(finish_uploads());
    j->bodies.push_back(std::move(B));
    if (body) *body = (int)j->bodies.size() - 1;
    return MPMGPU_OK;
  }

  mpmgpu_status add_contact(int job, int b1, int b2, double mu, int* contact, int reflected = 0) override {
    HJob* j;
    MPM_TRY(editable_job(job, &j));
    const int nb = (int)j->bodies.size();
    if (b1 < 0 || b2 < 0 || b1 >= nb || b2 >= nb || b1 == b2) return fail(MPMGPU_ERR_ARG, "contact bodies out of range");
    if (j->nc >= kMaxContacts) return fail(MPMGPU_ERR_UNSUPPORTED, "too many contacts");
    HBody& B1 = j->bodies[(size_t)b1];
    const size_t ns = (size_t)j->g.nslots;
    if (!B1.needs_normal) {
      for (int d = 0; d < 3; d++) MPM_TRY(alloc_dev(&B1.A.nrm[d], ns, B1.allocs, j->bytes));
      if (det_)
        for (int d = 0; d < 3; d++) MPM_TRY(alloc_dev(&B1.Ar.nrm[d], ns, B1.allocs, j->bytes));
      B1.needs_normal = 1;
    }
    const int c = j->nc;
    j->cb1[c] = b1;
    j->cb2[c] = b2;
    j->mu[c] = mu;
    j->reflected[c] = reflected != 0 ? 1 : 0;
    if (keep_debug_) {
      MPM_TRY(alloc_dev(&j->normal_out[c], 3 * ns, j->allocs, j->bytes));
      MPM_TRY(alloc_dev(&j->force_out[c], 3 * ns, j->allocs, j->bytes));
    }
    j->nc++;
    MPM_TRY(finish_uploads());
    if (contact) *contact = c;
    return MPMGPU_OK;
  }

  mpmgpu_status set_gravity(int job, int use_vector, const double* gv) override {
    HJob* j;
    MPM_TRY(live_job(job, &j));
    double g3[3] = {0.0, 0.0, 0.0};
    if (use_vector) {
      if (!gv) return fail(MPMGPU_ERR_ARG, "gravity vector missing");
      for (int d = 0; d < dim_; d++) g3[d] = gv[d];
    } else {
      g3[dim_ == 2 ? 1 : 2] = -9.81;
    }
    for (int d = 0; d < 3; d++) j->sp.grav[d] = g3[d];
    tables_dirty_ = true;
    return MPMGPU_OK;
  }

  mpmgpu_status admit(int job) override {
    HJob* j;
    MPM_TRY(editable_job(job, &j));
    if (j->bodies.empty()) return fail(MPMGPU_ERR_STATE, "job has no bodies");
    j->admitted = true;
    membership_dirty_ = true;
    return MPMGPU_OK;
  }

  mpmgpu_status step(int nsteps) override {
    if (nsteps < 0) return fail(MPMGPU_ERR_ARG, "negative step count");
    for (int s = 0; s < nsteps; s++) {
      MPM_TRY(commit());
      if (live_jobs_ == 0) break;
      MPM_TRY(launch_step());
      steps_since_sort_++;
      bool finished_any = false;
      for (auto& j : jobs_) {
        if (!j.in_tables) continue;
        j.steps_done++;
        if (--j.steps_left <= 0) {
          j.finished = true;
          finished_any = true;
        }
      }
      if (finished_any) membership_dirty_ = true;
      if (steps_since_sort_ >= sort_interval_ && !membership_dirty_) MPM_TRY(launch_sort());
    }
    return MPMGPU_OK;
  }

  mpmgpu_status synchronize() override {
    MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
    int flag = 0;
    MPM_CUDA_TRY(cudaMemcpy(&flag, err_, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag & kErrWideSpan) return fail(MPMGPU_ERR_DEVICE, "point corners span more than two cells (extent > cell size)");
    if (flag & kErrElemAlias) return fail(MPMGPU_ERR_DEVICE, "point within rounding of the upper domain face");
    if (flag & kErrWaitTimeout) return fail(MPMGPU_ERR_DEVICE, "a bulk copy did not complete within the wait limit");
    if (flag & kErrItemCap) return fail(MPMGPU_ERR_DEVICE, "a work item holds more points than the kernel takes");
    return MPMGPU_OK;
  }

  mpmgpu_status remove_job(int job) override {
    if (job < 0 || job >= (int)jobs_.size() || jobs_[(size_t)job].removed) return fail(MPMGPU_ERR_ARG, "no such job");
    HJob& j = jobs_[(size_t)job];
    if (j.in_tables) membership_dirty_ = true;
    j.finished = true;
    j.admitted = false;
    if (j.block_off >= 0 && j.in_tables) {
      // the next compaction must not see its blocks
      MPM_CUDA_TRY(cudaMemsetAsync(flags_ + j.block_off, 0, sizeof(uint32_t) * j.g.nblocks, stream_));
    }
    // stream-ordered: the arrays return to the pool after the queued work;
    // the job leaves the device tables at the next step boundary, before
    // any later launch
    free_job(j);
    j.removed = true;
    return MPMGPU_OK;
  }

  mpmgpu_status job_state(int job, int64_t* done, int64_t* left) const override {
    if (job < 0 || job >= (int)jobs_.size()) return MPMGPU_ERR_ARG;
    const HJob& j = jobs_[(size_t)job];
    if (done) *done = j.steps_done;
    if (left) *left = j.finished ? 0 : j.steps_left;
    return MPMGPU_OK;
  }

  mpmgpu_status sizes(int job, int body, int64_t* n_points, int64_t* n_nodes) const override {
    if (job < 0 || job >= (int)jobs_.size()) return MPMGPU_ERR_ARG;
    const HJob& j = jobs_[(size_t)job];
    if (body < 0 || body >= (int)j.bodies.size()) return MPMGPU_ERR_ARG;
    if (n_points) *n_points = j.bodies[(size_t)body].n;
    if (n_nodes) *n_nodes = j.g.nnodes;
    return MPMGPU_OK;
  }

  mpmgpu_status body_points_fp64(int job, int body, PointsDev* P, Geom* g, int* cpdi) override {
    if (mixed()) return fail(MPMGPU_ERR_UNSUPPORTED, "map export needs the FP64 form");
    if (job < 0 || job >= (int)jobs_.size()) return fail(MPMGPU_ERR_ARG, "no such job");
    HJob& j = jobs_[(size_t)job];
    if (body < 0 || body >= (int)j.bodies.size()) return fail(MPMGPU_ERR_ARG, "no such body");
    std::memcpy(P, &j.bodies[(size_t)body].P, sizeof(PointsDev));
    *g = j.g;
    *cpdi = j.sp.cpdi;
    return MPMGPU_OK;
  }

  int64_t memory_in_use() const override {
    int64_t b = scratch_bytes_;
    for (const auto& j : jobs_)
      if (!j.removed) b += j.bytes;
    return b;
  }

  void counts(int* live_jobs, int64_t* live_points) const override {
    int lj = 0;
    int64_t lp = 0;
    for (const auto& j : jobs_)
      if (j.admitted && !j.finished && !j.removed) {
        lj++;
        for (const auto& b : j.bodies) lp += b.n;
      }
    if (live_jobs) *live_jobs = lj;
    if (live_points) *live_points = lp;
  }

  // ---- downloads (reference layout, original point order) ----

  // Host views of one body's point arrays (copies in pinned memory), from
  // which fields are converted to the reference's layout and point order.
  struct PointView {
    int64_t n = 0;
    const int32_t* pid = nullptr;
    const int32_t* active = nullptr;
    const PT* x[3] = {};
    const PT* u[3] = {};
    const PT* v[3] = {};
    const PT* s[6] = {};
    const PT* vol = nullptr;
    const PT* m = nullptr;
    const PT* ext = nullptr;
    const PT* ms[2] = {};
    const double* L = nullptr;
    // low words of the mixed form (null in the FP64 form)
    const PT* xl[3] = {};
    const PT* vl[3] = {};
    const PT* ml = nullptr;
  };

  static bool point_field_known(int field) {
    switch (field) {
      case MPMGPU_P_X: case MPMGPU_P_U: case MPMGPU_P_X_T: case MPMGPU_P_MX_T: case MPMGPU_P_L: case MPMGPU_P_T:
      case MPMGPU_P_M: case MPMGPU_P_V: case MPMGPU_P_EXTENT: case MPMGPU_P_ACTIVE: case MPMGPU_P_GAMMAP:
      case MPMGPU_P_GAMMAP_DOT:
        return true;
    }
    return false;
  }

  // The device arrays a point field is converted from (the point ids
  // first): add(source, bytes, slot of the view that receives its copy).
  template <typename F>
  void point_field_arrays(const HBody& B, int field, PointView& v, F&& add) const {
    const size_t nz = (size_t)B.n, np = nz * sizeof(PT);
    const int D = dim_;
    auto slot = [](auto& p) { return reinterpret_cast<const void**>(&p); };
    add(B.P.pid, nz * sizeof(int32_t), slot(v.pid));
    const bool two = B.P.ml != nullptr;   // the mixed form's low words
    switch (field) {
      case MPMGPU_P_X:
        for (int d = 0; d < D; d++) add(B.P.x[d], np, slot(v.x[d]));
        if (two)
          for (int d = 0; d < D; d++) add(B.P.xl[d], np, slot(v.xl[d]));
        break;
      case MPMGPU_P_U:
        for (int d = 0; d < D; d++) add(B.P.u[d], np, slot(v.u[d]));
        break;
      case MPMGPU_P_X_T:
        for (int d = 0; d < D; d++) add(B.P.v[d], np, slot(v.v[d]));
        if (two)
          for (int d = 0; d < D; d++) add(B.P.vl[d], np, slot(v.vl[d]));
        break;
      case MPMGPU_P_MX_T:
        for (int d = 0; d < D; d++) add(B.P.v[d], np, slot(v.v[d]));
        add(B.P.m, np, slot(v.m));
        if (two) {
          for (int d = 0; d < D; d++) add(B.P.vl[d], np, slot(v.vl[d]));
          add(B.P.ml, np, slot(v.ml));
        }
        break;
      case MPMGPU_P_L: add(B.P.L, nz * 9 * sizeof(double), slot(v.L)); break;
      case MPMGPU_P_T:
        for (int c = 0; c < 6; c++) add(B.P.s[c], np, slot(v.s[c]));
        break;
      case MPMGPU_P_M:
        add(B.P.m, np, slot(v.m));
        if (two) add(B.P.ml, np, slot(v.ml));
        break;
      case MPMGPU_P_V: add(B.P.vol, np, slot(v.vol)); break;
      case MPMGPU_P_EXTENT: add(B.P.ext, np, slot(v.ext)); break;
      case MPMGPU_P_ACTIVE: add(B.P.active, nz * sizeof(int32_t), slot(v.active)); break;
      case MPMGPU_P_GAMMAP: add(B.P.ms[0], np, slot(v.ms[0])); break;
      case MPMGPU_P_GAMMAP_DOT: add(B.P.ms[1], np, slot(v.ms[1])); break;
    }
  }

  // One point field from host views, in the layout of mpmgpu_download_points
  // and the reference's point order (pid).
  void points_to_ref(const PointView& v, int field, double* out) const {
    const int64_t n = v.n;
    const size_t nz = (size_t)n;
    const int D = dim_;
    const int32_t* pid = v.pid;
    // lo: the mixed form's low words (hi + lo), else null
    auto vec3 = [&](const PT* const* a, const PT* const* lo = nullptr) {
      for (int64_t i = 0; i < 3 * n; i++) out[i] = 0.0;
      for (int d = 0; d < D; d++)
        for (size_t i = 0; i < nz; i++)
          out[3 * (int64_t)pid[i] + d] = two_word(a[d], lo ? lo[d] : nullptr, (int64_t)i);
    };
    auto scalar = [&](const PT* a, const PT* lo = nullptr) {
      for (size_t i = 0; i < nz; i++) out[pid[i]] = two_word(a, lo, (int64_t)i);
    };
    switch (field) {
      case MPMGPU_P_X: vec3(v.x, v.xl[0] ? v.xl : nullptr); return;
      case MPMGPU_P_U: vec3(v.u); return;
      case MPMGPU_P_X_T: vec3(v.v, v.vl[0] ? v.vl : nullptr); return;
      case MPMGPU_P_MX_T:
        vec3(v.v, v.vl[0] ? v.vl : nullptr);
        // movePoints: mx_t = m * x_t (explicit_usl.cpp:295-297)
        for (size_t i = 0; i < nz; i++) {
          const int64_t q = pid[i];
          const double m = two_word(v.m, v.ml, (int64_t)i);
          for (int d = 0; d < D; d++) out[3 * q + d] = m * out[3 * q + d];
        }
        return;
      case MPMGPU_P_L:
        for (size_t i = 0; i < nz; i++)
          for (int k = 0; k < 9; k++) out[9 * (int64_t)pid[i] + k] = v.L[9 * i + (size_t)k];
        return;
      case MPMGPU_P_T: {
        static const int idx[9] = {0, 3, 5, 3, 1, 4, 5, 4, 2};
        for (size_t i = 0; i < nz; i++)
          for (int k = 0; k < 9; k++) out[9 * (int64_t)pid[i] + k] = (double)v.s[idx[k]][i];
        return;
      }
      case MPMGPU_P_M: scalar(v.m, v.ml); return;
      case MPMGPU_P_V: scalar(v.vol); return;
      case MPMGPU_P_EXTENT: scalar(v.ext); return;
      case MPMGPU_P_GAMMAP: scalar(v.ms[0]); return;
      case MPMGPU_P_GAMMAP_DOT: scalar(v.ms[1]); return;
      case MPMGPU_P_ACTIVE:
        // 2 = left the domain at the last move: still active until the next
        // map build deactivates it, as in the reference
        for (size_t i = 0; i < nz; i++) out[pid[i]] = v.active[i] != 0 ? 1.0 : 0.0;
        return;
    }
  }

  mpmgpu_status point_field_check(const HBody& B, int field) {
    if (!point_field_known(field)) return fail(MPMGPU_ERR_ARG, "unknown point field");
    if (field == MPMGPU_P_L && !B.P.L) return fail(MPMGPU_ERR_STATE, "L is kept only with keep_debug in the FP64 form");
    if ((field == MPMGPU_P_GAMMAP || field == MPMGPU_P_GAMMAP_DOT) && B.mat.kind != 2)
      return fail(MPMGPU_ERR_STATE, "gammap and gammap_dot belong to Sand_SachithLocal bodies");
    return MPMGPU_OK;
  }

  mpmgpu_status download_points(int job, int body, int field, double* out) override {
    HJob* j;
    HBody* B;
    MPM_TRY(readable_body(job, body, &j, &B));
    const int64_t n = B->n;
    if (field == MPMGPU_P_B) {
      MPM_TRY(synchronize());
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) out[3 * i + d] = j->sp.grav[d];
      return MPMGPU_OK;
    }
    MPM_TRY(point_field_check(*B, field));
    // the point ids and the arrays of the field, copied with one wait
    PointView pv;
    pv.n = n;
    std::vector<std::pair<const void*, size_t>> items;
    std::vector<const void**> slots;
    point_field_arrays(*B, field, pv, [&](const void* src, size_t bytes, const void** slot) {
      items.emplace_back(src, bytes);
      slots.push_back(slot);
    });
    std::vector<const unsigned char*> h;
    MPM_TRY(fetch(items, h));
    for (size_t k = 0; k < slots.size(); k++) *slots[k] = h[k];
    points_to_ref(pv, field, out);
    return MPMGPU_OK;
  }

  mpmgpu_status download_points_many(int count, const int* jobs, int body, int field, double* const* outs,
                                     int threads) override {
    if (count < 0 || (count > 0 && (!jobs || !outs))) return fail(MPMGPU_ERR_ARG, "job list missing");
    if (field == MPMGPU_P_B) {
      for (int k = 0; k < count; k++) MPM_TRY(download_points(jobs[k], body, field, outs[k]));
      return MPMGPU_OK;
    }
    std::vector<PointView> views((size_t)count);
    std::vector<std::pair<const void*, size_t>> items;
    std::vector<std::pair<size_t, const void**>> slots;   // (view, slot)
    std::vector<size_t> first_item((size_t)count + 1, 0);
    for (int k = 0; k < count; k++) {
      HJob* j;
      HBody* B;
      MPM_TRY(readable_body(jobs[k], body, &j, &B));
      MPM_TRY(point_field_check(*B, field));
      views[(size_t)k].n = B->n;
      first_item[(size_t)k] = items.size();
      point_field_arrays(*B, field, views[(size_t)k], [&](const void* src, size_t bytes, const void** slot) {
        items.emplace_back(src, bytes);
        slots.emplace_back((size_t)k, slot);
      });
    }
    first_item[(size_t)count] = items.size();
    // jobs in groups of at most kFetchGroupBytes staged bytes: one copy and
    // wait per group, then the group's conversion on host threads (a bounded
    // pinned buffer instead of one the size of the whole field)
    int k0 = 0;
    while (k0 < count) {
      int k1 = k0;
      size_t bytes = 0;
      while (k1 < count) {
        size_t b = 0;
        for (size_t i = first_item[(size_t)k1]; i < first_item[(size_t)k1 + 1]; i++) b += (items[i].second + 255) / 256 * 256;
        if (k1 > k0 && bytes + b > kFetchGroupBytes) break;
        bytes += b;
        k1++;
      }
      const size_t i0 = first_item[(size_t)k0], i1 = first_item[(size_t)k1];
      std::vector<std::pair<const void*, size_t>> group(items.begin() + (std::ptrdiff_t)i0,
                                                        items.begin() + (std::ptrdiff_t)i1);
      std::vector<const unsigned char*> h;
      MPM_TRY(fetch(group, h));
      for (size_t i = i0; i < i1; i++) *slots[i].second = h[i - i0];
      const int ng = k1 - k0;
      const int nt = std::max(1, std::min(threads, ng));
      std::vector<std::thread> pool;
      for (int t = 0; t < nt; t++)
        pool.emplace_back([&, t]() {
          for (int k = k0 + t; k < k1; k += nt) points_to_ref(views[(size_t)k], field, outs[k]);
        });
      for (auto& th : pool) th.join();
      k0 = k1;
    }
    return MPMGPU_OK;
  }
  static constexpr size_t kFetchGroupBytes = (size_t)192 << 20;

  // ---- frames ----

  mpmgpu_status frame_begin(int job) override {
    HJob* j;
    MPM_TRY(live_job(job, &j));
    MPM_TRY(frame_wait());   // the previous frame's buffers are reused
    Frame f;
    f.job = job;
    f.primed = j->primed && j->block_off >= 0;
    f.nnodes = j->g.nnodes;
    for (int d = 0; d < 3; d++) f.grav[d] = j->sp.grav[d];
    // layout of the frame: per body its point fields, then its node fields;
    // then the contacts
    int64_t off = 0;
    auto take = [&](int64_t n) {
      const int64_t o = off;
      off += (n + 31) / 32 * 32;   // 256-byte aligned fields
      return o;
    };
    const int64_t nn = j->g.nnodes;
    for (const HBody& B : j->bodies) {
      FramePointLayout pl;
      const int64_t n = B.n;
      pl.x = take(3 * n);
      pl.u = take(3 * n);
      pl.xt = take(3 * n);
      pl.mxt = take(3 * n);
      pl.T = take(9 * n);
      pl.v = take(n);
      pl.m = take(n);
      pl.ext = take(n);
      pl.active = take(n);
      pl.L = B.P.L ? take(9 * n) : -1;
      const bool sand = B.mat.has_material && B.mat.kind == 2 && B.P.ms[0] != nullptr;
      pl.gammap = sand ? take(n) : -1;
      pl.gammap_dot = sand ? take(n) : -1;
      f.pts.push_back(pl);
      f.npts.push_back(n);
      FrameNodeLayout nl;
      const bool dbg = B.snap.m != nullptr;
      nl.m = dbg ? take(nn) : -1;
      nl.mxt = dbg ? take(3 * nn) : -1;
      nl.f = dbg ? take(3 * nn) : -1;
      nl.xt = take(3 * nn);
      nl.u = take(3 * nn);
      nl.dxt = take(3 * nn);
      f.nodes.push_back(nl);
    }
    for (int c = 0; c < j->nc; c++) {
      const bool kept = j->normal_out[c] != nullptr && j->force_out[c] != nullptr;
      f.contact.push_back({kept ? take(3 * nn) : -1, kept ? take(3 * nn) : -1});
    }
    const size_t bytes = (size_t)off * sizeof(double) + 256;   // + the error flag
    if (bytes > frame_dev_cap_ || bytes > frame_cap_) {
      MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
      if (bytes > frame_dev_cap_) {
        if (frame_dev_) cudaFree(frame_dev_);
        frame_dev_ = nullptr;
        frame_dev_cap_ = 0;
        const cudaError_t e = cudaMalloc(&frame_dev_, bytes);
        if (e != cudaSuccess) return fail(MPMGPU_ERR_NOMEM, std::string("frame staging: ") + cudaGetErrorString(e));
        frame_dev_cap_ = bytes;
      }
      if (bytes > frame_cap_) {
        pinned_give(frame_stage_, frame_cap_);
        frame_stage_ = nullptr;
        frame_cap_ = 0;
        size_t cap = 0;
        MPM_CUDA_TRY(pinned_take(bytes, &frame_stage_, &cap));
        frame_cap_ = cap;
      }
    }
    double* out = reinterpret_cast<double*>(frame_dev_);
    const uint8_t* act = j->block_off >= 0 ? was_active_ + j->block_off : nullptr;
    const int blocks = sm_count_ * 8;
    for (size_t b = 0; b < j->bodies.size(); b++) {
      const HBody& B = j->bodies[b];
      if (B.n > 0) {
        k_frame_points<PT><<<blocks, 256, 0, stream_>>>(B.P, dim_, f.pts[b], out);
        MPM_TRY(check_launch("k_frame_points"));
      }
      if (f.primed) {
        k_frame_nodes<<<blocks, 256, 0, stream_>>>(j->g, j->sp.dt, act, B.snap, B.V, f.nodes[b], out);
        MPM_TRY(check_launch("k_frame_nodes"));
      } else {
        const FrameNodeLayout& nl = f.nodes[b];
        const int64_t first = nl.m >= 0 ? nl.m : nl.xt;
        const int64_t last = nl.dxt + 3 * nn;
        MPM_CUDA_TRY(cudaMemsetAsync(out + first, 0, (size_t)(last - first) * sizeof(double), stream_));
      }
    }
    for (int c = 0; c < j->nc; c++) {
      if (f.contact[(size_t)c].first < 0) continue;
      k_frame_contact<<<blocks, 256, 0, stream_>>>(j->g, f.primed ? 1 : 0, act, j->normal_out[c], 1,
                                                   out + f.contact[(size_t)c].first);
      k_frame_contact<<<blocks, 256, 0, stream_>>>(j->g, f.primed ? 1 : 0, act, j->force_out[c], 0,
                                                   out + f.contact[(size_t)c].second);
      MPM_TRY(check_launch("k_frame_contact"));
    }
    unsigned char* host = static_cast<unsigned char*>(frame_stage_);
    MPM_CUDA_TRY(cudaMemcpyAsync(host + (size_t)off * sizeof(double), err_, sizeof(int), cudaMemcpyDeviceToHost,
                                 stream_));
    if (off > 0)
      MPM_CUDA_TRY(
          cudaMemcpyAsync(host, frame_dev_, (size_t)off * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    if (!frame_ev_) MPM_CUDA_TRY(cudaEventCreateWithFlags(&frame_ev_, cudaEventDisableTiming));
    MPM_CUDA_TRY(cudaEventRecord(frame_ev_, stream_));
    f.data = reinterpret_cast<const double*>(host);
    f.err = reinterpret_cast<const int*>(host + (size_t)off * sizeof(double));
    f.pending = true;
    frame_ = std::move(f);
    return MPMGPU_OK;
  }

  mpmgpu_status frame_points(int job, int body, int field, double* out) override {
    HBody* B;
    MPM_TRY(frame_body(job, body, &B));
    const int64_t n = frame_.npts[(size_t)body];
    if (field == MPMGPU_P_B) {
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) out[3 * i + d] = frame_.grav[d];
      return MPMGPU_OK;
    }
    MPM_TRY(point_field_check(*B, field));
    const FramePointLayout& pl = frame_.pts[(size_t)body];
    int64_t o = -1, w = 1;
    switch (field) {
      case MPMGPU_P_X: o = pl.x; w = 3; break;
      case MPMGPU_P_U: o = pl.u; w = 3; break;
      case MPMGPU_P_X_T: o = pl.xt; w = 3; break;
      case MPMGPU_P_MX_T: o = pl.mxt; w = 3; break;
      case MPMGPU_P_T: o = pl.T; w = 9; break;
      case MPMGPU_P_L: o = pl.L; w = 9; break;
      case MPMGPU_P_V: o = pl.v; break;
      case MPMGPU_P_M: o = pl.m; break;
      case MPMGPU_P_EXTENT: o = pl.ext; break;
      case MPMGPU_P_ACTIVE: o = pl.active; break;
      case MPMGPU_P_GAMMAP: o = pl.gammap; break;
      case MPMGPU_P_GAMMAP_DOT: o = pl.gammap_dot; break;
    }
    if (o < 0) return fail(MPMGPU_ERR_STATE, "field not in the frame");
    MPM_TRY(frame_wait());
    std::memcpy(out, frame_.data + o, (size_t)(n * w) * sizeof(double));
    return MPMGPU_OK;
  }

  mpmgpu_status frame_nodes(int job, int body, int field, double* out) override {
    HBody* B;
    MPM_TRY(frame_body(job, body, &B));
    const FrameNodeLayout& nl = frame_.nodes[(size_t)body];
    int64_t o = -1, w = 3;
    switch (field) {
      case MPMGPU_N_M: o = nl.m; w = 1; break;
      case MPMGPU_N_MX_T: o = nl.mxt; break;
      case MPMGPU_N_F: o = nl.f; break;
      case MPMGPU_N_X_T: o = nl.xt; break;
      case MPMGPU_N_U: o = nl.u; break;
      case MPMGPU_N_DIFF_X_T: o = nl.dxt; break;
      default: return fail(MPMGPU_ERR_ARG, "unknown node field");
    }
    if (o < 0) return fail(MPMGPU_ERR_STATE, "nodal m, mx_t and f are kept only with keep_debug");
    MPM_TRY(frame_wait());
    std::memcpy(out, frame_.data + o, (size_t)(frame_.nnodes * w) * sizeof(double));
    return MPMGPU_OK;
  }

  mpmgpu_status frame_contact(int job, int contact, int field, double* out) override {
    if (job != frame_.job) return fail(MPMGPU_ERR_STATE, "no frame of this job was begun");
    if (contact < 0 || contact >= (int)frame_.contact.size()) return fail(MPMGPU_ERR_ARG, "no such contact");
    if (field != MPMGPU_C_NORMAL && field != MPMGPU_C_FORCE) return fail(MPMGPU_ERR_ARG, "unknown contact field");
    const auto& cl = frame_.contact[(size_t)contact];
    const int64_t o = field == MPMGPU_C_NORMAL ? cl.first : cl.second;
    if (o < 0) return fail(MPMGPU_ERR_STATE, "contact fields are kept only with keep_debug");
    MPM_TRY(frame_wait());
    std::memcpy(out, frame_.data + o, (size_t)(3 * frame_.nnodes) * sizeof(double));
    return MPMGPU_OK;
  }

  // Point arrays of a snapshot: x, u, x_t (3 each), the stress (6), V, and
  // in the mixed form the low words of x and x_t (3 each); then active and
  // the point ids.
  int snapshot_arrays() const { return mixed() ? 22 : 16; }

  size_t snapshot_bytes(int64_t n) const override {
    return (size_t)n * ((size_t)snapshot_arrays() * sizeof(PT) + 2 * sizeof(int32_t));
  }

  mpmgpu_status snapshot_body(int job, int body, void* host) override {
    HJob* j;
    HBody* B;
    MPM_TRY(readable_body(job, body, &j, &B));
    const size_t n = (size_t)B->n;
    if (n == 0) return MPMGPU_OK;
    PT* h = static_cast<PT*>(host);
    const PT* src[22] = {B->P.x[0],  B->P.x[1],  B->P.x[2],  B->P.u[0],  B->P.u[1],  B->P.u[2],  B->P.v[0],  B->P.v[1],
                         B->P.v[2],  B->P.s[0],  B->P.s[1],  B->P.s[2],  B->P.s[3],  B->P.s[4],  B->P.s[5],  B->P.vol,
                         B->P.xl[0], B->P.xl[1], B->P.xl[2], B->P.vl[0], B->P.vl[1], B->P.vl[2]};
    const int na = snapshot_arrays();
    for (int a = 0; a < na; a++) {
      // x, u, x_t and the low words exist for the grid's axes only
      if ((a < 9 || a >= 16) && (a < 16 ? a % 3 : (a - 16) % 3) >= dim_) continue;
      MPM_CUDA_TRY(cudaMemcpyAsync(h + a * n, src[a], n * sizeof(PT), cudaMemcpyDeviceToHost, stream_));
    }
    int32_t* hi = reinterpret_cast<int32_t*>(h + (size_t)na * n);
    MPM_CUDA_TRY(cudaMemcpyAsync(hi, B->P.active, n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
    MPM_CUDA_TRY(cudaMemcpyAsync(hi + n, B->P.pid, n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
    return MPMGPU_OK;
  }

  void snapshot_fields(const void* host, int64_t n64, double* x, double* u, double* x_t, double* T, double* v,
                       double* active) const override {
    const size_t n = (size_t)n64;
    const PT* h = static_cast<const PT*>(host);
    const int na = snapshot_arrays();
    const int32_t* act = reinterpret_cast<const int32_t*>(h + (size_t)na * n);
    const int32_t* pid = act + n;
    static const int idx[9] = {0, 3, 5, 3, 1, 4, 5, 4, 2};
    for (size_t i = 0; i < n; i++) {
      const size_t q = (size_t)pid[i];
      for (int d = 0; d < 3; d++) {
        const bool on = d < dim_;
        x[3 * q + d] = on ? two_word(h + d * n, mixed() ? h + (16 + d) * n : nullptr, (int64_t)i) : 0.0;
        u[3 * q + d] = on ? (double)h[(3 + d) * n + i] : 0.0;
        x_t[3 * q + d] = on ? two_word(h + (6 + d) * n, mixed() ? h + (19 + d) * n : nullptr, (int64_t)i) : 0.0;
      }
      for (int k = 0; k < 9; k++) T[9 * q + k] = (double)h[(9 + idx[k]) * n + i];
      v[q] = (double)h[15 * n + i];
      // 2 = left the domain at the last move: still active, as download_points
      active[q] = act[i] != 0 ? 1.0 : 0.0;
    }
  }

  mpmgpu_status download_nodes(int job, int body, int field, double* out) override {
    HJob* j;
    HBody* B;
    MPM_TRY(readable_body(job, body, &j, &B));
    MPM_TRY(synchronize());
    const int D = dim_;
    const bool dbg = B->snap.m != nullptr;
    if (!j->primed || j->block_off < 0) {
      for (int64_t i = 0; i < j->g.nnodes * (field == MPMGPU_N_M ? 1 : 3); i++) out[i] = 0.0;
      return MPMGPU_OK;
    }
    switch (field) {
      case MPMGPU_N_M:
        if (!dbg) return fail(MPMGPU_ERR_STATE, "nodal m is kept only with keep_debug");
        return nodes_to_ref(*j, &B->snap.m, 1, 1, out);
      case MPMGPU_N_MX_T:
        if (!dbg) return fail(MPMGPU_ERR_STATE, "nodal mx_t is kept only with keep_debug");
        return nodes_to_ref(*j, B->snap.mx, D, 3, out);
      case MPMGPU_N_F:
        if (!dbg) return fail(MPMGPU_ERR_STATE, "nodal f is kept only with keep_debug");
        return nodes_to_ref(*j, B->snap.f, D, 3, out);
      case MPMGPU_N_X_T: return nodes_to_ref(*j, B->V.vt, D, 3, out);
      case MPMGPU_N_DIFF_X_T: return nodes_to_ref(*j, B->V.dv, D, 3, out);
      case MPMGPU_N_U: {
        MPM_TRY(nodes_to_ref(*j, B->V.vt, D, 3, out));
        // moveGrid: u = dt * x_t (explicit_usl.cpp:252)
        for (int64_t i = 0; i < 3 * j->g.nnodes; i++) out[i] = j->sp.dt * out[i];
        return MPMGPU_OK;
      }
    }
    return fail(MPMGPU_ERR_ARG, "unknown node field");
  }

  mpmgpu_status download_contact(int job, int contact, int field, double* out) override {
    if (job < 0 || job >= (int)jobs_.size() || jobs_[(size_t)job].removed) return fail(MPMGPU_ERR_ARG, "no such job");
    HJob& j = jobs_[(size_t)job];
    if (contact < 0 || contact >= j.nc) return fail(MPMGPU_ERR_ARG, "no such contact");
    if (!keep_debug_) return fail(MPMGPU_ERR_STATE, "contact fields are kept only with keep_debug");
    if (field != MPMGPU_C_NORMAL && field != MPMGPU_C_FORCE) return fail(MPMGPU_ERR_ARG, "unknown contact field");
    MPM_TRY(synchronize());
    const Geom& g = j.g;
    double* src = (field == MPMGPU_C_NORMAL) ? j.normal_out[contact] : j.force_out[contact];
    std::vector<double> tmp;
    MPM_TRY(download(tmp, src, 3 * (size_t)g.nslots));
    std::vector<uint8_t> act((size_t)g.nblocks, 0);
    if (j.block_off >= 0) MPM_TRY(download(act, was_active_ + j.block_off, (size_t)g.nblocks));
    contact_host_to_ref(g, j.primed, act.data(), tmp.data(), field == MPMGPU_C_NORMAL, out);
    return MPMGPU_OK;
  }

  // ---- profiling ----

  mpmgpu_status profile(int enable) override {
    MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
    for (int s = 0; s < kStages; s++) {
      for (auto& pr : pending_[s]) {
        event_pool_.push_back(pr.first);
        event_pool_.push_back(pr.second);
      }
      pending_[s].clear();
      stage_launches_[s] = 0;
      stage_ms_[s] = 0.0;
    }
    profiling_ = enable != 0;
    return MPMGPU_OK;
  }

  mpmgpu_status profile_read(int stage, int64_t* launches, double* total_ms) override {
    if (stage < 0 || stage >= kStages) return fail(MPMGPU_ERR_ARG, "no such stage");
    MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
    for (int s = 0; s < kStages; s++) {
      for (auto& pr : pending_[s]) {
        float ms = 0.0f;
        MPM_CUDA_TRY(cudaEventElapsedTime(&ms, pr.first, pr.second));
        stage_ms_[s] += ms;
        stage_launches_[s]++;
        event_pool_.push_back(pr.first);
        event_pool_.push_back(pr.second);
      }
      pending_[s].clear();
    }
    if (launches) *launches = stage_launches_[stage];
    if (total_ms) *total_ms = stage_ms_[stage];
    return MPMGPU_OK;
  }

  // ---- autotuning ----

  // Tunes the launch shape on the current jobs, restoring their state after
  // every trial (the state after the call is the state before it): first
  // the points per work item (each available choice timed over `steps`
  // steps), then the re-binning interval (4, 8, 16, 32 steps, each timed
  // over 32 steps with its re-binnings), keeping the fastest of each.
  mpmgpu_status autotune(int steps, int* best_cap) override {
    if (steps < 1) return fail(MPMGPU_ERR_ARG, "autotune needs at least one step");
    MPM_TRY(commit());
    if (live_jobs_ == 0) return fail(MPMGPU_ERR_STATE, "no jobs to tune on");
    MPM_TRY(snapshot_save());
    const int original_cap = cap_, original_si = sort_interval_;
    cudaEvent_t e0, e1;
    MPM_CUDA_TRY(cudaEventCreate(&e0));
    MPM_CUDA_TRY(cudaEventCreate(&e1));
    // one trial: re-bin, 2 warm-up steps, `n` timed steps re-binning every
    // `si` steps; the state is restored afterwards
    auto trial = [&](int n, int si, float* ms) -> mpmgpu_status {
      drop_graphs();
      MPM_TRY(launch_sort());   // work items depend on the item size
      for (int w = 0; w < 2; w++) MPM_TRY(launch_step());
      cudaEventRecord(e0, stream_);
      int since = 0;
      for (int k = 0; k < n; k++) {
        MPM_TRY(launch_step());
        if (++since >= si) {
          MPM_TRY(launch_sort());
          since = 0;
        }
      }
      cudaEventRecord(e1, stream_);
      if (cudaEventSynchronize(e1) != cudaSuccess) return fail(MPMGPU_ERR_CUDA, "autotune timing failed");
      cudaEventElapsedTime(ms, e0, e1);
      return snapshot_restore();
    };
    mpmgpu_status st = MPMGPU_OK;
    const int original_form = form_;
    int best_c = original_cap, best_f = original_form, best_si = original_si;
    float best_ms = 1e30f;
    // kernel form and points per item
    const int cand[6][2] = {{kFormStaged, 256}, {kFormStaged, 512}, {kFormStaged, 1024},
                            {kFormLean, 128},   {kFormLean, 256},   {kFormLean, 512}};
    for (int ci = 0; ci < 6 && st == MPMGPU_OK; ci++) {
      const int f = cand[ci][0], c = cand[ci][1];
      if (!form_available(dim_, mixed(), det_, f, c) || (det_ && c != default_cap())) continue;
      form_ = f;
      cap_ = c;
      float ms = 0.0f;
      st = trial(steps, 1 << 30, &ms);
      if (st == MPMGPU_OK && ms < best_ms) {
        best_ms = ms;
        best_c = c;
        best_f = f;
      }
    }
    cap_ = best_c;
    form_ = best_f;
    best_ms = 1e30f;
    const int intervals[4] = {4, 8, 16, 32};
    for (int k = 0; k < 4 && st == MPMGPU_OK; k++) {
      float ms = 0.0f;
      st = trial(32, intervals[k], &ms);
      if (st == MPMGPU_OK && ms < best_ms) {
        best_ms = ms;
        best_si = intervals[k];
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cap_ = (st == MPMGPU_OK) ? best_c : original_cap;
    form_ = (st == MPMGPU_OK) ? best_f : original_form;
    sort_interval_ = (st == MPMGPU_OK) ? best_si : original_si;
    drop_graphs();
    snapshot_free();
    MPM_TRY(st);
    MPM_TRY(launch_sort());
    if (best_cap) *best_cap = cap_;
    return MPMGPU_OK;
  }

  int sort_interval() const override { return sort_interval_; }
  int kernel_form() const override { return form_; }

  mpmgpu_status set_kernel(int form, int cap) override {
    if (!form_available(dim_, mixed(), det_, form, cap) || (det_ && cap != default_cap()))
      return fail(MPMGPU_ERR_ARG, "kernel form " + std::to_string(form) + " with " + std::to_string(cap) +
                                      " points per item is not available for this batch");
    if (form == form_ && cap == cap_) return MPMGPU_OK;
    form_ = form;
    cap_ = cap;
    drop_graphs();
    // the work items depend on the item size: re-bin before the next step
    membership_dirty_ = true;
    return MPMGPU_OK;
  }

  void set_wait_limit(uint32_t polls) override {
    wait_polls_ = polls;
    drop_graphs();   // the limit travels in the launch arguments
  }

 private:
  // ---- allocation helpers ----

  template <typename T>
  mpmgpu_status alloc_raw(T** p, size_t count, std::vector<void*>& owner) {
    void* q = nullptr;
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return fail(MPMGPU_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    owner.push_back(q);
    e = cudaMemsetAsync(q, 0, bytes, stream_);
    if (e != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    *p = static_cast<T*>(q);
    scratch_bytes_ += (int64_t)bytes;
    return MPMGPU_OK;
  }

  template <typename T>
  // A job's array from the pool, zeroed, ordered on the copy stream (the
  // compute stream waits for it in finish_uploads).
  mpmgpu_status alloc_dev(T** p, size_t count, std::vector<void*>& owner, int64_t& bytes) {
    void* q = nullptr;
    const size_t nb = std::max<size_t>(count * sizeof(T), 16);
    cudaError_t e = cudaMallocFromPoolAsync(&q, nb, pool_, copy_stream_);
    if (e != cudaSuccess) return fail(MPMGPU_ERR_NOMEM, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
    owner.push_back(q);
    e = cudaMemsetAsync(q, 0, nb, copy_stream_);
    if (e != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    *p = static_cast<T*>(q);
    bytes += (int64_t)nb;
    return MPMGPU_OK;
  }

  // A body's arrays are carved out of one pool allocation: one allocation,
  // one clear and one release per body instead of one per array. The first
  // pass of a layout only sums the sizes (base null), the second hands out
  // 256-byte aligned sub-arrays.
  struct Arena {
    unsigned char* base = nullptr;
    size_t used = 0;
  };
  template <typename T>
  static void carve(Arena& a, T** p, size_t count) {
    const size_t nb = (std::max<size_t>(count * sizeof(T), 16) + 255) / 256 * 256;
    *p = a.base ? reinterpret_cast<T*>(a.base + a.used) : nullptr;
    a.used += nb;
  }
  template <typename F>
  mpmgpu_status alloc_arena(F&& layout, std::vector<void*>& owner, int64_t& bytes) {
    Arena a;
    layout(a);
    const size_t total = std::max<size_t>(a.used, 256);
    void* q = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&q, total, pool_, copy_stream_);
    if (e != cudaSuccess) return fail(MPMGPU_ERR_NOMEM, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
    owner.push_back(q);
    e = cudaMemsetAsync(q, 0, total, copy_stream_);
    if (e != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    Arena b;
    b.base = static_cast<unsigned char*>(q);
    layout(b);
    bytes += (int64_t)total;
    return MPMGPU_OK;
  }

  // Point arrays hold n entries plus 8 of padding: the fused kernel's bulk
  // copies round their windows out to 16-byte boundaries and may read up to
  // 3 entries past the last point.
  void layout_points(Arena& a, PointsT<PT>& P, int64_t n, int nstate) {
    P = PointsT<PT>{};
    P.n = n;
    const size_t na = (size_t)n + 8;
    for (int d = 0; d < 3; d++) {
      carve(a, &P.x[d], na);
      carve(a, &P.v[d], na);
      carve(a, &P.u[d], na);
    }
    for (int c = 0; c < 6; c++) carve(a, &P.s[c], na);
    carve(a, &P.vol, na);
    carve(a, &P.m, na);
    carve(a, &P.ext, na);
    carve(a, &P.active, na);
    carve(a, &P.pid, na);
    P.L = nullptr;
    if (keep_debug_ && !mixed()) carve(a, &P.L, (size_t)n * 9);
    for (int k = 0; k < nstate; k++) carve(a, &P.ms[k], na);
    if (mixed()) {
      for (int d = 0; d < 3; d++) {
        carve(a, &P.xl[d], na);
        carve(a, &P.vl[d], na);
      }
      carve(a, &P.ml, na);
    }
  }

  // Returns a job's arrays to the pool after the work already queued on the
  // compute stream.
  void free_job(HJob& j) {
    for (auto& b : j.bodies) {
      for (void* p : b.allocs) cudaFreeAsync(p, stream_);
      b.allocs.clear();
    }
    for (void* p : j.allocs) cudaFreeAsync(p, stream_);
    j.allocs.clear();
    j.bytes = 0;
  }

  // Uploads go through a pinned staging buffer on the copy stream, so they
  // overlap the steps already queued on the compute stream.
  mpmgpu_status stage_reserve(size_t bytes) {
    MPM_CUDA_TRY(cudaStreamSynchronize(copy_stream_));  // the staging buffer is free again
    stage_used_ = 0;
    if (bytes <= stage_cap_) return MPMGPU_OK;
    pinned_give(stage_, stage_cap_);
    stage_ = nullptr;
    // at least twice the old size: pinning pages is slow (about as slow as
    // the upload itself), so a batch that grows job by job reallocates only
    // a few times
    const size_t want = std::max<size_t>(std::max<size_t>(bytes, 2 * stage_cap_), (size_t)64 << 20);
    stage_cap_ = 0;
    size_t cap = 0;
    MPM_CUDA_TRY(pinned_take(want, &stage_, &cap));
    stage_cap_ = cap;
    return MPMGPU_OK;
  }

  // Runs body(a, b) over [0, n) in chunks on up to 8 host threads (one
  // thread below 2^18 entries).
  template <typename F>
  static void host_parallel(int64_t n, F&& body) {
    const int64_t per = (int64_t)1 << 18;
    const int hw = std::max(1, (int)std::thread::hardware_concurrency());
    const int nt = (int)std::min<int64_t>(std::min(8, hw), (n + per - 1) / per);
    if (nt <= 1) {
      body((int64_t)0, n);
      return;
    }
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back([&body, n, nt, t]() { body(n * t / nt, n * (t + 1) / nt); });
    body((int64_t)0, n / nt);
    for (auto& th : pool) th.join();
  }

  // Uploads n entries of a device array on the copy stream: fill(h, a, b)
  // writes entries a..b-1 of the host image straight into the pinned
  // staging buffer (reserved by stage_reserve), or into a pageable buffer
  // copied synchronously when the reservation is exceeded.
  template <typename T, typename F>
  mpmgpu_status upload_fill(T* dst, int64_t n, F&& fill) {
    if (n <= 0) return MPMGPU_OK;
    const size_t bytes = (size_t)n * sizeof(T);
    if (stage_used_ + bytes > stage_cap_) {
      std::vector<T> tmp((size_t)n);
      host_parallel(n, [&](int64_t a, int64_t b) { fill(tmp.data(), a, b); });
      MPM_CUDA_TRY(cudaMemcpyAsync(dst, tmp.data(), bytes, cudaMemcpyHostToDevice, copy_stream_));
      MPM_CUDA_TRY(cudaStreamSynchronize(copy_stream_));
      return MPMGPU_OK;
    }
    T* h = reinterpret_cast<T*>(static_cast<unsigned char*>(stage_) + stage_used_);
    host_parallel(n, [&](int64_t a, int64_t b) { fill(h, a, b); });
    stage_used_ += (bytes + 255) / 256 * 256;
    MPM_CUDA_TRY(cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, copy_stream_));
    return MPMGPU_OK;
  }

  // Orders the compute stream after the allocations and copies queued on
  // the copy stream, and waits for them (the staging buffer is reused).
  mpmgpu_status finish_uploads() {
    MPM_CUDA_TRY(cudaEventRecord(upload_ev_, copy_stream_));
    MPM_CUDA_TRY(cudaStreamWaitEvent(stream_, upload_ev_, 0));
    MPM_CUDA_TRY(cudaStreamSynchronize(copy_stream_));
    return MPMGPU_OK;
  }

  // Copies device arrays to pinned staging on the compute stream (after the
  // queued work) and waits once; checks the kernels' error flag like
  // synchronize(). h[k] points at item k's bytes until the next fetch.
  mpmgpu_status fetch(const std::vector<std::pair<const void*, size_t>>& items, std::vector<const unsigned char*>& h) {
    size_t total = 256;   // error flag first
    for (auto& it : items) total += (it.second + 255) / 256 * 256;
    if (total > dl_cap_) {
      MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
      pinned_give(dl_stage_, dl_cap_);
      dl_stage_ = nullptr;
      // twice the request: the next, larger download of the same jobs (the
      // stress after the positions) then fits without pinning pages again
      const size_t want = std::max<size_t>(2 * total, (size_t)16 << 20);
      dl_cap_ = 0;
      size_t cap = 0;
      MPM_CUDA_TRY(pinned_take(want, &dl_stage_, &cap));
      dl_cap_ = cap;
    }
    unsigned char* base = static_cast<unsigned char*>(dl_stage_);
    MPM_CUDA_TRY(cudaMemcpyAsync(base, err_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    size_t off = 256;
    h.clear();
    for (auto& it : items) {
      if (it.second > 0) MPM_CUDA_TRY(cudaMemcpyAsync(base + off, it.first, it.second, cudaMemcpyDeviceToHost, stream_));
      h.push_back(base + off);
      off += (it.second + 255) / 256 * 256;
    }
    MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
    int flag = 0;
    std::memcpy(&flag, base, sizeof(int));
    if (flag & kErrWideSpan) return fail(MPMGPU_ERR_DEVICE, "point corners span more than two cells (extent > cell size)");
    if (flag & kErrElemAlias) return fail(MPMGPU_ERR_DEVICE, "point within rounding of the upper domain face");
    if (flag & kErrWaitTimeout) return fail(MPMGPU_ERR_DEVICE, "a bulk copy did not complete within the wait limit");
    if (flag & kErrItemCap) return fail(MPMGPU_ERR_DEVICE, "a work item holds more points than the kernel takes");
    return MPMGPU_OK;
  }

  template <typename T>
  mpmgpu_status download(std::vector<T>& dst, const T* src, size_t n) {
    dst.resize(n);
    if (n == 0) return MPMGPU_OK;
    MPM_CUDA_TRY(cudaMemcpyAsync(dst.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, stream_));
    MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
    return MPMGPU_OK;
  }

  mpmgpu_status editable_job(int job, HJob** out) {
    if (job < 0 || job >= (int)jobs_.size() || jobs_[(size_t)job].removed) return fail(MPMGPU_ERR_ARG, "no such job");
    HJob& j = jobs_[(size_t)job];
    if (j.admitted) return fail(MPMGPU_ERR_STATE, "bodies and contacts must be added before the job starts");
    *out = &j;
    return MPMGPU_OK;
  }

  mpmgpu_status live_job(int job, HJob** out) {
    if (job < 0 || job >= (int)jobs_.size() || jobs_[(size_t)job].removed) return fail(MPMGPU_ERR_ARG, "no such job");
    *out = &jobs_[(size_t)job];
    return MPMGPU_OK;
  }

  mpmgpu_status readable_body(int job, int body, HJob** j, HBody** b) {
    MPM_TRY(live_job(job, j));
    if (body < 0 || body >= (int)(*j)->bodies.size()) return fail(MPMGPU_ERR_ARG, "no such body");
    *b = &(*j)->bodies[(size_t)body];
    return MPMGPU_OK;
  }

  int default_cap() const { return det_ && dim_ == 3 ? 256 : 512; }

  // Converts block-linear nodal arrays (comps SoA components, host copies)
  // to reference node order; nodes of blocks that were not active in the
  // last step read 0.
  static void nodes_host_to_ref(const Geom& g, const uint8_t* act, const double* const* arr, int comps, int width,
                                double* out) {
    for (int64_t i = 0; i < g.nnodes * width; i++) out[i] = 0.0;
    for (int d = 0; d < comps; d++)
      for (int k = 0; k < g.nn[2]; k++)
        for (int jj = 0; jj < g.nn[1]; jj++)
          for (int i = 0; i < g.nn[0]; i++) {
            const int64_t id = i + (int64_t)g.nn[0] * (jj + (int64_t)g.nn[1] * k);
            const bool on = act[(size_t)node_block(g, i, jj, k)] != 0;
            out[id * width + d] = on ? arr[d][(size_t)node_slot(g, i, jj, k)] : 0.0;
          }
  }

  // Copies a block-linear nodal array (comps SoA components) to reference
  // node order; nodes of blocks that were not active in the last step read 0.
  mpmgpu_status nodes_to_ref(HJob& j, double* const* arr, int comps, int width, double* out) {
    const Geom& g = j.g;
    std::vector<uint8_t> act;
    MPM_TRY(download(act, was_active_ + j.block_off, (size_t)g.nblocks));
    std::vector<std::vector<double>> tmp((size_t)comps);
    const double* host[3] = {};
    for (int d = 0; d < comps; d++) {
      MPM_TRY(download(tmp[(size_t)d], arr[d], (size_t)g.nslots));
      host[d] = tmp[(size_t)d].data();
    }
    nodes_host_to_ref(g, act.data(), host, comps, width, out);
    return MPMGPU_OK;
  }

  // Converts a contact's per-node output (3 per slot, host copy) to
  // reference node order.
  static void contact_host_to_ref(const Geom& g, bool primed, const uint8_t* act, const double* src, bool normal,
                                  double* out) {
    const double nan = std::nan("");
    for (int k = 0; k < g.nn[2]; k++)
      for (int jj = 0; jj < g.nn[1]; jj++)
        for (int i = 0; i < g.nn[0]; i++) {
          const int64_t id = i + (int64_t)g.nn[0] * (jj + (int64_t)g.nn[1] * k);
          const int64_t s = node_slot(g, i, jj, k);
          const bool on = primed && act[(size_t)node_block(g, i, jj, k)] != 0;
          for (int d = 0; d < 3; d++) {
            double v = src[(size_t)(3 * s + d)];
            // the reference normalises every node's normal; a zero normal gives 0 * (1/0)
            if (!on) v = normal ? (d < g.dim ? nan : 0.0) : 0.0;
            out[3 * id + d] = v;
          }
        }
  }

  // ---- block space (first-fit ranges, stable for a job's lifetime) ----

  int64_t block_alloc(int64_t len) {
    for (size_t i = 0; i < free_.size(); i++) {
      if (free_[i].second >= len) {
        const int64_t off = free_[i].first;
        free_[i].first += len;
        free_[i].second -= len;
        if (free_[i].second == 0) free_.erase(free_.begin() + (long)i);
        return off;
      }
    }
    // grow at the end (merging a free tail)
    int64_t off = block_end_;
    if (!free_.empty() && free_.back().first + free_.back().second == block_end_) {
      off = free_.back().first;
      free_.pop_back();
    }
    block_end_ = off + len;
    return off;
  }

  void block_free(int64_t off, int64_t len) {
    free_.push_back({off, len});
    std::sort(free_.begin(), free_.end());
    std::vector<std::pair<int64_t, int64_t>> merged;
    for (auto& r : free_) {
      if (!merged.empty() && merged.back().first + merged.back().second == r.first)
        merged.back().second += r.second;
      else
        merged.push_back(r);
    }
    free_ = merged;
  }

  // Grows a device array to at least `need` elements (doubling), keeping
  // the first `keep` elements; invalidates the graphs.
  template <typename T>
  mpmgpu_status grow(T** p, int64_t* cap, int64_t need, int64_t keep) {
    if (need <= *cap) return MPMGPU_OK;
    const int64_t ncap = std::max<int64_t>(need, std::max<int64_t>(2 * *cap, 1024));
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, (size_t)ncap * sizeof(T));
    if (e != cudaSuccess) return fail(MPMGPU_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    MPM_CUDA_TRY(cudaMemsetAsync(q, 0, (size_t)ncap * sizeof(T), stream_));
    if (*p != nullptr) {
      if (keep > 0) MPM_CUDA_TRY(cudaMemcpyAsync(q, *p, (size_t)keep * sizeof(T), cudaMemcpyDeviceToDevice, stream_));
      MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
      auto it = std::find(cap_allocs_.begin(), cap_allocs_.end(), (void*)*p);
      if (it != cap_allocs_.end()) cap_allocs_.erase(it);
      cudaFree(*p);
      scratch_bytes_ -= *cap * (int64_t)sizeof(T);
    }
    cap_allocs_.push_back(q);
    scratch_bytes_ += ncap * (int64_t)sizeof(T);
    *p = static_cast<T*>(q);
    *cap = ncap;
    drop_graphs();
    return MPMGPU_OK;
  }

  // ---- membership: tables, binning, priming ----

  // Applies joins and leaves at a step boundary: block ranges, tables,
  // re-binning of every body and the first scatter of joining bodies.
  mpmgpu_status commit() {
    if (!membership_dirty_ && !tables_dirty_) return MPMGPU_OK;
    const bool membership = membership_dirty_;
    if (membership) {
      for (auto& j : jobs_) {
        const bool want = j.admitted && !j.finished && !j.removed && j.steps_left > 0;
        if (j.admitted && !j.finished && j.steps_left <= 0) j.finished = true;
        if (want && !j.in_tables) {
          j.block_off = block_alloc(j.g.nblocks);
          if (!free_slots_.empty()) {
            j.slot = free_slots_.back();
            free_slots_.pop_back();
          } else {
            j.slot = next_slot_++;
          }
          j.fill_pending = true;
          j.in_tables = true;
        } else if (!want && j.in_tables) {
          j.in_tables = false;
          // its flags were set by its last scatter: clear them so no later
          // compaction lists its blocks (its stale block -> slot entries are
          // then never read)
          MPM_CUDA_TRY(cudaMemsetAsync(flags_ + j.block_off, 0, sizeof(uint32_t) * j.g.nblocks, stream_));
          block_free(j.block_off, j.g.nblocks);
          free_slots_.push_back(j.slot);
          j.slot = -1;
          j.block_off = j.removed ? -1 : j.block_off;
        }
      }
    }
    // table contents (the job table by stable slot, unused slots empty)
    std::vector<InstDev> insts((size_t)std::max(next_slot_, 1), InstDev{});
    std::vector<GridBody> gbodies;
    std::vector<BodyCtx<PT>> ctx;
    std::vector<int64_t> point_end, bin_end;
    std::vector<int32_t> item_off;
    int64_t points = 0, bins = 0, cells = 0, items = 0;
    live_jobs_ = 0;
    bool any_prime = false;
    for (auto& j : jobs_) {
      if (!j.in_tables) continue;
      InstDev I{};
      I.g = j.g;
      I.sp = j.sp;
      I.nb = (int)j.bodies.size();
      I.body0 = (int)ctx.size();
      I.nc = j.nc;
      for (int c = 0; c < j.nc; c++) {
        I.cb1[c] = j.cb1[c];
        I.cb2[c] = j.cb2[c];
        I.mu[c] = j.mu[c];
        I.reflected[c] = j.reflected[c];
        I.normal_out[c] = j.normal_out[c];
        I.force_out[c] = j.force_out[c];
      }
      I.block_off = j.block_off;
      insts[(size_t)j.slot] = I;
      for (auto& b : j.bodies) {
        GridBody G{};
        G.A = b.A;
        G.Ar = b.Ar;
        G.V = b.V;
        G.snap = b.snap;
        G.has_boundary = b.has_boundary;
        G.mu_f = b.mu_f;
        gbodies.push_back(G);
        BodyCtx<PT> c{};
        c.g = j.g;
        c.mc = j.mc;
        c.bg = j.bg;
        c.sp = j.sp;
        c.mat = b.mat;
        c.P = b.P;
        c.V = b.V;
        c.A = b.A;
        c.Ar = b.Ar;
        c.flags = flags_ + j.block_off;   // rebased after growth below
        c.needs_normal = b.needs_normal;
        c.prime = b.prime;
        any_prime = any_prime || b.prime;
        c.Palt = b.Palt;
        c.point_off = points;
        c.bin_off = bins;
        c.cell_off = cells;
        c.inst = j.slot;
        points += b.n;
        bins += j.bg.nbins + 1;
        cells += (int64_t)j.bg.nbins * j.bg.cells_per_bin + 1;
        item_off.push_back((int32_t)items);
        items += j.bg.nbins + b.n / kMinItemCap + 1;   // ceil(count / cap) summed over bins
        point_end.push_back(points);
        bin_end.push_back(bins);
        ctx.push_back(c);
      }
      live_jobs_++;
    }
    // capacities
    const int64_t nb = (int64_t)ctx.size(), ni = (int64_t)insts.size();
    MPM_TRY(grow(&insts_d_, &cap_insts_, std::max<int64_t>(ni, 1), 0));
    MPM_TRY(grow(&gbodies_d_, &cap_bodies_g_, std::max<int64_t>(nb, 1), 0));
    MPM_TRY(grow(&ctx_d_, &cap_bodies_c_, std::max<int64_t>(nb, 1), 0));
    MPM_TRY(grow(&point_end_d_, &cap_bodies_p_, std::max<int64_t>(nb, 1), 0));
    MPM_TRY(grow(&bin_end_d_, &cap_bodies_b_, std::max<int64_t>(nb, 1), 0));
    const int64_t old_blocks = cap_blocks_;
    MPM_TRY(grow(&flags_, &cap_blocks_, std::max<int64_t>(block_end_, 1), old_blocks));
    int64_t tmp_cap = old_blocks;
    MPM_TRY(grow(&was_active_, &tmp_cap, cap_blocks_, old_blocks));
    tmp_cap = old_blocks;
    MPM_TRY(grow(&blk_inst_, &tmp_cap, cap_blocks_, old_blocks));
    tmp_cap = old_blocks;
    MPM_TRY(grow(&list_, &tmp_cap, cap_blocks_, 0));
    MPM_TRY(grow(&key_, &cap_points_k_, std::max<int64_t>(points, 1), 0));
    MPM_TRY(grow(&rank_, &cap_points_r_, std::max<int64_t>(points, 1), 0));
    MPM_TRY(grow(&cell_count_, &cap_cells_, std::max<int64_t>(cells, 1), 0));
    MPM_TRY(grow(&cell_hist_, &cap_cells_h_, std::max<int64_t>(cells, 1), 0));
    MPM_TRY(grow(&crank_, &cap_points_c_, std::max<int64_t>(points, 1), 0));
    MPM_TRY(grow(&bin_scan_, &cap_bins_, bins + 2, 0));
    MPM_TRY(grow(&chunk_sum_, &cap_chunks_, cap_bins_ / kScanChunk + 2, 0));
    MPM_TRY(grow(&item_off_d_, &cap_bodies_i_, std::max<int64_t>(nb, 1), 0));
    if (det_) MPM_TRY(grow(&bounds_, &cap_bounds_, std::max<int64_t>(4 * nb, 4), 0));
    MPM_TRY(grow(&nwork_body_, &cap_bodies_w_, std::max<int64_t>(nb, 1), 0));
    MPM_TRY(grow(&work_end_body_, &cap_bodies_e_, std::max<int64_t>(nb, 1), 0));
    MPM_TRY(grow(&work_bin_, &cap_items_n_, std::max<int64_t>(items, 1), 0));
    MPM_TRY(grow(&work_start_, &cap_items_s_, std::max<int64_t>(items, 1), 0));
    MPM_TRY(grow(&work_end_, &cap_items_e_, std::max<int64_t>(items, 1), 0));
    MPM_TRY(grow(&flat_body_, &cap_items_fb_, std::max<int64_t>(items, 1), 0));
    MPM_TRY(grow(&flat_item_, &cap_items_fi_, std::max<int64_t>(items, 1), 0));
    for (size_t b = 0; b < ctx.size(); b++) ctx[b].flags = flags_ + insts[(size_t)ctx[b].inst].block_off;
    ctx_host_ = ctx;
    single_mode_ = ctx.size() <= (size_t)kSideStreams + 1;   // one launch per body, concurrent (one_body_launches)
    any_plain_ = any_normal_ = false;
    all_elastic_ = true;
    for (const auto& c : ctx) {
      (c.needs_normal ? any_normal_ : any_plain_) = true;
      if (c.mat.has_material && c.mat.kind != 0) all_elastic_ = false;
    }
    drop_graphs();   // one-body launches carry the table entries in their arguments
    // block -> job slot map: only the ranges of joining jobs change
    for (auto& j : jobs_) {
      if (!j.in_tables || !j.fill_pending) continue;
      const int64_t nbk = j.g.nblocks;
      k_fill_i32<<<(int)std::min<int64_t>((nbk + 255) / 256, 4096), 256, 0, stream_>>>(blk_inst_ + j.block_off, nbk,
                                                                                        j.slot);
      MPM_TRY(check_launch("k_fill_i32"));
      j.fill_pending = false;
    }
    BatchHdr hdr{};
    hdr.points = points;
    hdr.bins = bins;
    hdr.cells = cells;
    hdr.blocks = block_end_;
    hdr.nbodies = (int)nb;
    hdr.ninst = (int)ni;
    // the device tables change only between steps (stream order)
    MPM_TRY(upload_async(insts_d_, insts));
    MPM_TRY(upload_async(gbodies_d_, gbodies));
    MPM_TRY(upload_async(ctx_d_, ctx));
    MPM_TRY(upload_async(point_end_d_, point_end));
    MPM_TRY(upload_async(bin_end_d_, bin_end));
    MPM_TRY(upload_async(item_off_d_, item_off));
    MPM_CUDA_TRY(cudaMemcpyAsync(hdr_, &hdr, sizeof(hdr), cudaMemcpyHostToDevice, stream_));
    MPM_CUDA_TRY(cudaStreamSynchronize(stream_));  // host vectors go out of scope
    hdr_host_ = hdr;
    tables_dirty_ = false;
    membership_dirty_ = false;
    if (membership && live_jobs_ > 0) {
      MPM_TRY(launch_sort());
      if (any_prime) MPM_TRY(prime());
    }
    return MPMGPU_OK;
  }

  template <typename T>
  mpmgpu_status upload_async(T* dst, const std::vector<T>& src) {
    if (src.empty()) return MPMGPU_OK;
    MPM_CUDA_TRY(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, stream_));
    return MPMGPU_OK;
  }

  // First scatter of joining bodies (their nodal sums for the first step).
  mpmgpu_status prime() {
    if (det_) MPM_TRY(launch_bounds());
    MPM_TRY(launch_fused(1, det_ ? 2 : 3));
    // clear the prime flags in the host mirrors and the device table
    for (auto& j : jobs_) {
      if (!j.in_tables) continue;
      j.primed = true;
      for (auto& b : j.bodies) b.prime = 0;
    }
    for (auto& c : ctx_host_) c.prime = 0;
    MPM_TRY(launch_clear_prime());
    return MPMGPU_OK;
  }

  // ---- launches ----

  mpmgpu_status check_launch(const char* what) {
    launches_++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return MPMGPU_OK;
  }

  struct StageTimer {
    Batch* b;
    int stage;
    cudaEvent_t start = nullptr;
    StageTimer(Batch* bb, int s) : b(bb), stage(s) {
      if (!b->profiling_) return;
      start = b->take_event();
      cudaEventRecord(start, b->stream_);
    }
    ~StageTimer() {
      if (!b->profiling_ || !start) return;
      cudaEvent_t stop = b->take_event();
      cudaEventRecord(stop, b->stream_);
      b->pending_[stage].push_back({start, stop});
    }
  };
  cudaEvent_t take_event() {
    cudaEvent_t e = nullptr;
    if (!event_pool_.empty()) {
      e = event_pool_.back();
      event_pool_.pop_back();
    } else {
      cudaEventCreate(&e);
    }
    return e;
  }

  int stride_blocks(int threads) const { return sm_count_ * (2048 / threads); }

  template <int DIM, int CAP, bool NORMAL, bool SINGLE, bool DET>
  mpmgpu_status launch_fused_k(int prime_pass, int phases, int one_body, cudaStream_t st) {
    FusedLaunch<PT> fl{};
    if (SINGLE) fl.one = ctx_host_[(size_t)one_body];
    fl.one_body = SINGLE ? one_body : -1;
    fl.bodies = ctx_d_;
    fl.item_off = item_off_d_;
    fl.nwork_body = nwork_body_;
    fl.work_end_body = work_end_body_;
    fl.flat_body = flat_body_;
    fl.flat_item = flat_item_;
    fl.nbodies_cap = (int)ctx_host_.size();
    fl.work_bin = work_bin_;
    fl.work_start = work_start_;
    fl.work_end = work_end_;
    fl.nwork = nwork_;
    fl.err = err_;
    fl.drift = drift_;
    fl.prime_pass = prime_pass;
    fl.phases = phases;
    fl.bounds = bounds_;
    fl.wait_polls = wait_polls_;
    fl.queue = queue_;
    constexpr size_t smem = fused_smem_bytes<DIM, PT, CAP, NORMAL, DET>();
    auto kern = k_g2p2g<DIM, PT, CAP, NORMAL, SINGLE, DET>;
    // resident CTAs per SM, looked up once per kernel (before any capture)
    int& per_sm = fused_per_sm_[((CAP == 256 ? 0 : (CAP == 512 ? 1 : 2)) * 4 + (NORMAL ? 2 : 0) + (SINGLE ? 1 : 0)) * 2 +
                                (DET ? 1 : 0)];
    if (per_sm == 0) {
      MPM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      MPM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, fused_threads<PT, CAP>(), smem));
      if (per_sm < 1) return fail(MPMGPU_ERR_CUDA, "fused kernel does not fit on an SM");
    }
    const int blocks = per_sm * sm_count_;
    StageTimer timer(this, kStageFused);
    kern<<<blocks, fused_threads<PT, CAP>(), smem, st>>>(fl);
    return check_launch("k_g2p2g");
  }

  // One launch per body for small batches at the default item size (the
  // body's parameters then sit in the constant bank), else one launch per
  // kind of body (with or without the contact normal) over the table.
  template <int DIM, int CAP, bool DET>
  mpmgpu_status launch_fused_t(int prime_pass, int phases) {
    if constexpr (CAP == 512) {
      if (single_mode_) {
        return one_body_launches(prime_pass, [&](int b, cudaStream_t st) {
          if (ctx_host_[(size_t)b].needs_normal) return launch_fused_k<DIM, CAP, true, true, DET>(prime_pass, phases, b, st);
          return launch_fused_k<DIM, CAP, false, true, DET>(prime_pass, phases, b, st);
        });
      }
    }
    if (any_plain_) MPM_TRY((launch_fused_k<DIM, CAP, false, false, DET>(prime_pass, phases, -1, stream_)));
    if (any_normal_) MPM_TRY((launch_fused_k<DIM, CAP, true, false, DET>(prime_pass, phases, -1, stream_)));
    return MPMGPU_OK;
  }

  template <int NT, int PPT, bool NORMAL, bool SINGLE, int MAT>
  mpmgpu_status launch_lean_k(int prime_pass, int phases, int one_body, cudaStream_t st) {
    FusedLaunch<PT> fl{};
    if (SINGLE) fl.one = ctx_host_[(size_t)one_body];
    fl.one_body = SINGLE ? one_body : -1;
    fl.bodies = ctx_d_;
    fl.item_off = item_off_d_;
    fl.nwork_body = nwork_body_;
    fl.work_end_body = work_end_body_;
    fl.flat_body = flat_body_;
    fl.flat_item = flat_item_;
    fl.nbodies_cap = (int)ctx_host_.size();
    fl.work_bin = work_bin_;
    fl.work_start = work_start_;
    fl.work_end = work_end_;
    fl.nwork = nwork_;
    fl.err = err_;
    fl.drift = drift_;
    fl.prime_pass = prime_pass;
    fl.phases = phases;
    fl.bounds = nullptr;
    fl.wait_polls = wait_polls_;
    fl.queue = queue_;
    constexpr size_t smem = lean_smem_bytes<3, PT, NORMAL>();
    auto kern = k_g2p2g_lean<3, PT, NT, PPT, NORMAL, SINGLE, MAT>;
    int& per_sm =
        lean_per_sm_[(PPT == 2 ? 16 : 0) + (NT == 128 ? 8 : 0) + (NORMAL ? 4 : 0) + (SINGLE ? 2 : 0) + (MAT == 0 ? 1 : 0)];
    if (per_sm == 0) {
      MPM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      MPM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
      if (per_sm < 1) return fail(MPMGPU_ERR_CUDA, "fused kernel does not fit on an SM");
    }
    StageTimer timer(this, kStageFused);
    kern<<<per_sm * sm_count_, NT, smem, st>>>(fl);
    return check_launch("k_g2p2g_lean");
  }

  template <int NT, int PPT, bool NORMAL, bool SINGLE>
  mpmgpu_status launch_lean_s(int prime_pass, int phases, int one_body, bool elastic, cudaStream_t st) {
    if (elastic) return launch_lean_k<NT, PPT, NORMAL, SINGLE, 0>(prime_pass, phases, one_body, st);
    return launch_lean_k<NT, PPT, NORMAL, SINGLE, -1>(prime_pass, phases, one_body, st);
  }

  // points per item: 128 (CTAs of 128 threads), 256 (256 threads) or 512
  // (256 threads, two points each)
  template <bool NORMAL, bool SINGLE>
  mpmgpu_status launch_lean_m(int prime_pass, int phases, int one_body, bool elastic, cudaStream_t st) {
    if (cap_ == 128) return launch_lean_s<128, 1, NORMAL, SINGLE>(prime_pass, phases, one_body, elastic, st);
    if (cap_ == 512) return launch_lean_s<256, 2, NORMAL, SINGLE>(prime_pass, phases, one_body, elastic, st);
    return launch_lean_s<256, 1, NORMAL, SINGLE>(prime_pass, phases, one_body, elastic, st);
  }

  // The one-body launches of a stage, body by body (bodies still to prime
  // only, in a priming pass). The bodies are independent here (each gathers
  // from and scatters into its own nodal arrays), so the second to fourth
  // body's launch runs on a side stream forked from the step's stream and
  // joined back into it: its CTAs fill the SMs that the previous launch's
  // last round of items leaves idle (a 0.26 M-point body is 512 items for
  // 444 CTAs). A captured step graph holds the launches as parallel
  // branches. Profiled steps launch on the step's stream only, so that each
  // launch's stage time is its own.
  template <typename F>
  mpmgpu_status one_body_launches(int prime_pass, F&& launch_body) {
    int todo[kSideStreams + 1];
    int nt = 0;
    for (size_t b = 0; b < ctx_host_.size(); b++) {
      if (prime_pass && !ctx_host_[b].prime) continue;
      if (nt == kSideStreams + 1) return fail(MPMGPU_ERR_UNSUPPORTED, "too many bodies for one-body launches");
      todo[nt++] = (int)b;
    }
    const bool fork = !profiling_ && nt > 1;
    if (fork) MPM_CUDA_TRY(cudaEventRecord(fork_ev_, stream_));
    for (int i = 0; i < nt; i++) {
      cudaStream_t st = stream_;
      if (fork && i > 0) {
        st = side_[i - 1];
        MPM_CUDA_TRY(cudaStreamWaitEvent(st, fork_ev_, 0));
      }
      const mpmgpu_status r = launch_body(todo[i], st);
      if (fork && i > 0) MPM_CUDA_TRY(cudaEventRecord(join_ev_[i - 1], st));
      if (r != MPMGPU_OK) {
        for (int k = 1; fork && k <= i; k++) cudaStreamWaitEvent(stream_, join_ev_[k - 1], 0);
        return r;
      }
    }
    for (int i = 1; fork && i < nt; i++) MPM_CUDA_TRY(cudaStreamWaitEvent(stream_, join_ev_[i - 1], 0));
    return MPMGPU_OK;
  }

  mpmgpu_status launch_lean(int prime_pass, int phases) {
    if (single_mode_) {
      return one_body_launches(prime_pass, [&](int b, cudaStream_t st) {
        const BodyCtx<PT>& c = ctx_host_[(size_t)b];
        const bool el = !c.mat.has_material || c.mat.kind == 0;
        if (c.needs_normal) return launch_lean_m<true, true>(prime_pass, phases, b, el, st);
        return launch_lean_m<false, true>(prime_pass, phases, b, el, st);
      });
    }
    if (any_plain_) MPM_TRY((launch_lean_m<false, false>(prime_pass, phases, -1, all_elastic_, stream_)));
    if (any_normal_) MPM_TRY((launch_lean_m<true, false>(prime_pass, phases, -1, all_elastic_, stream_)));
    return MPMGPU_OK;
  }

  mpmgpu_status launch_fused(int prime_pass, int phases) {
    if (form_ != kFormStaged) return launch_lean(prime_pass, phases);
    if constexpr (sizeof(PT) == 8) {
      if (det_) {
        // the deterministic form: 256 points per item in 3D (two tile levels)
        if (dim_ == 3) return launch_fused_t<3, 256, true>(prime_pass, phases);
        return launch_fused_t<2, 512, true>(prime_pass, phases);
      }
    }
    if (dim_ == 3) {
      if (cap_ == 256) return launch_fused_t<3, 256, false>(prime_pass, phases);
      if constexpr (sizeof(PT) == 4) {
        if (cap_ == 1024) return launch_fused_t<3, 1024, false>(prime_pass, phases);
      }
      return launch_fused_t<3, 512, false>(prime_pass, phases);
    }
    return launch_fused_t<2, 512, false>(prime_pass, phases);
  }

  // Deterministic form: per-body bounds of the nodal contributions from the
  // updated point state (before the scatter that uses them).
  mpmgpu_status launch_bounds() {
    if constexpr (sizeof(PT) == 8) {
      MPM_CUDA_TRY(cudaMemsetAsync(bounds_, 0, sizeof(unsigned long long) * 4 * std::max<size_t>(ctx_host_.size(), 1),
                                   stream_));
      if (dim_ == 3)
        k_det_bounds<3><<<stride_blocks(256), 256, 0, stream_>>>(hdr_, ctx_d_, point_end_d_, bounds_);
      else
        k_det_bounds<2><<<stride_blocks(256), 256, 0, stream_>>>(hdr_, ctx_d_, point_end_d_, bounds_);
      return check_launch("k_det_bounds");
    }
    return MPMGPU_OK;
  }

  mpmgpu_status launch_clear_prime() {
    k_clear_prime<PT><<<1, 256, 0, stream_>>>(hdr_, ctx_d_);
    return check_launch("k_clear_prime");
  }

  mpmgpu_status launch_step_direct() {
    {
      StageTimer timer(this, kStageCompact);
      MPM_CUDA_TRY(cudaMemsetAsync(count_, 0, sizeof(unsigned long long), stream_));
      k_compact<<<stride_blocks(256), 256, 0, stream_>>>(hdr_, flags_, list_, count_, was_active_, active_nodes_);
      MPM_TRY(check_launch("k_compact"));
    }
    {
      StageTimer timer(this, kStageGrid);
      const int gb = sm_count_ * 32;
      if (dim_ == 3)
        k_grid<3><<<gb, 64, 0, stream_>>>(insts_d_, gbodies_d_, blk_inst_, list_, count_, active_nodes_);
      else
        k_grid<2><<<gb, 64, 0, stream_>>>(insts_d_, gbodies_d_, blk_inst_, list_, count_, active_nodes_);
      MPM_TRY(check_launch("k_grid"));
    }
    if (det_) {
      // update, bounds from the new state, then the scatter
      MPM_TRY(launch_fused(0, 1));
      MPM_TRY(launch_bounds());
      return launch_fused(0, 2);
    }
    return launch_fused(0, 3);
  }

  template <int DIM>
  mpmgpu_status launch_sort_direct_t() {
    const int sb = stride_blocks(256);
    k_sort_clear<<<sb, 256, 0, stream_>>>(hdr_, cell_count_, cell_hist_, nwork_body_);
    MPM_TRY(check_launch("k_sort_clear"));
    k_sort_count<DIM, PT><<<sb, 256, 0, stream_>>>(hdr_, ctx_d_, point_end_d_, key_, rank_, cell_count_, cell_hist_,
                                                   crank_);
    MPM_TRY(check_launch("k_sort_count"));
    k_bin_totals<PT><<<sb, 256, 0, stream_>>>(hdr_, ctx_d_, bin_end_d_, cell_count_, bin_scan_);
    MPM_TRY(check_launch("k_bin_totals"));
    const int chunks = (int)((cap_bins_ + kScanChunk - 1) / kScanChunk);
    k_scan_blocks<<<chunks, kScanChunk, 0, stream_>>>(hdr_, bin_scan_, chunk_sum_);
    MPM_TRY(check_launch("k_scan_blocks"));
    k_scan_small<<<1, 1024, 0, stream_>>>(chunk_sum_, chunks, nullptr);
    MPM_TRY(check_launch("k_scan_small"));
    k_scan_add<<<chunks, kScanChunk, 0, stream_>>>(hdr_, bin_scan_, chunk_sum_);
    MPM_TRY(check_launch("k_scan_add"));
    k_sort_scatter<DIM, PT><<<sb, 256, 0, stream_>>>(hdr_, ctx_d_, point_end_d_, key_, rank_, cell_count_, cell_hist_,
                                                     crank_, bin_scan_);
    MPM_TRY(check_launch("k_sort_scatter"));
    k_sort_flip<PT><<<std::max(1, (hdr_host_.nbodies + 255) / 256 + 1), 256, 0, stream_>>>(hdr_, ctx_d_);
    MPM_TRY(check_launch("k_sort_flip"));
    k_bin_work<PT><<<sb, 256, 0, stream_>>>(hdr_, ctx_d_, bin_end_d_, bin_scan_, item_off_d_, cap_, work_bin_,
                                            work_start_, work_end_, nwork_body_);
    MPM_TRY(check_launch("k_bin_work"));
    k_work_prefix<<<1, 1024, 0, stream_>>>(hdr_, nwork_body_, work_end_body_, nwork_);
    MPM_TRY(check_launch("k_work_prefix"));
    k_work_flat<<<sb, 256, 0, stream_>>>(hdr_, item_off_d_, nwork_body_, work_end_body_, nwork_, flat_body_,
                                         flat_item_);
    MPM_TRY(check_launch("k_work_flat"));
    return MPMGPU_OK;
  }

  mpmgpu_status launch_sort_direct() {
    StageTimer timer(this, kStageRebin);
    return dim_ == 3 ? launch_sort_direct_t<3>() : launch_sort_direct_t<2>();
  }

  // Host mirrors of the point buffers follow the device-side swap.
  void flip_mirrors() {
    for (auto& j : jobs_) {
      if (!j.in_tables) continue;
      for (auto& b : j.bodies) std::swap(b.P, b.Palt);
    }
    for (auto& c : ctx_host_) std::swap(c.P, c.Palt);
    flip_ ^= 1;
  }

  // Captures `body` into graph `g` on first use; launches it.
  template <typename F>
  mpmgpu_status run_graph(cudaGraphExec_t& g, bool& warm, int& kernels, F&& body) {
    // the first run of a launch sequence is direct (it also sets kernel
    // attributes, which cannot happen inside a capture); later runs replay
    // the captured graph
    if (!use_graph_ || profiling_ || !warm) {
      warm = true;
      return body();
    }
    if (g == nullptr) {
      cudaGraph_t graph = nullptr;
      MPM_CUDA_TRY(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      const int64_t before = launches_;
      mpmgpu_status st = body();
      cudaError_t e = cudaStreamEndCapture(stream_, &graph);
      kernels = (int)(launches_ - before);   // kernels the graph replays
      launches_ = before;
      if (st != MPMGPU_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
      }
      if (e != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      e = cudaGraphInstantiate(&g, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return fail(MPMGPU_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    MPM_CUDA_TRY(cudaGraphLaunch(g, stream_));
    launches_ += kernels;
    return MPMGPU_OK;
  }

  void drop_graphs() {
    for (int i = 0; i < 2; i++) {
      if (g_step_[i]) cudaGraphExecDestroy(g_step_[i]);
      g_step_[i] = nullptr;
      step_warm_[i] = false;
    }
    if (g_sort_) cudaGraphExecDestroy(g_sort_);
    g_sort_ = nullptr;
    sort_warm_ = false;
  }

  // The step graph depends on which point buffer is current (one-body
  // launches carry the pointers): one graph per buffer parity.
  mpmgpu_status launch_step() {
    return run_graph(g_step_[flip_], step_warm_[flip_], g_step_k_[flip_], [&] { return launch_step_direct(); });
  }

  mpmgpu_status launch_sort() {
    MPM_TRY(run_graph(g_sort_, sort_warm_, g_sort_k_, [&] { return launch_sort_direct(); }));
    flip_mirrors();
    steps_since_sort_ = 0;
    return MPMGPU_OK;
  }

  // ---- autotune snapshots ----

  std::vector<std::pair<void*, std::pair<void*, size_t>>> snap_;  // (saved copy, (live array, bytes))

  mpmgpu_status snap_one(void* live, size_t bytes) {
    if (!live || bytes == 0) return MPMGPU_OK;
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return fail(MPMGPU_ERR_NOMEM, "autotune snapshot: out of device memory");
    MPM_CUDA_TRY(cudaMemcpyAsync(q, live, bytes, cudaMemcpyDeviceToDevice, stream_));
    snap_.push_back({q, {live, bytes}});
    return MPMGPU_OK;
  }

  mpmgpu_status snapshot_save() {
    snapshot_free();
    for (auto& j : jobs_) {
      if (!j.in_tables) continue;
      const size_t ns = (size_t)j.g.nslots * sizeof(double);
      for (auto& b : j.bodies) {
        const size_t np = (size_t)(b.n + 8) * sizeof(PT), ni = (size_t)(b.n + 8) * sizeof(int32_t);
        // point buffers by role: the restore writes into whichever buffer
        // is current then (the trials re-bin and swap them)
        for (int d = 0; d < 3; d++) {
          MPM_TRY(snap_one(b.P.x[d], np));
          MPM_TRY(snap_one(b.P.v[d], np));
          MPM_TRY(snap_one(b.P.u[d], np));
        }
        for (int c = 0; c < 6; c++) MPM_TRY(snap_one(b.P.s[c], np));
        MPM_TRY(snap_one(b.P.vol, np));
        MPM_TRY(snap_one(b.P.m, np));
        MPM_TRY(snap_one(b.P.ext, np));
        MPM_TRY(snap_one(b.P.active, ni));
        MPM_TRY(snap_one(b.P.pid, ni));
        if (b.P.L) MPM_TRY(snap_one(b.P.L, (size_t)b.n * 9 * sizeof(double)));
        for (int k = 0; k < 9; k++)
          if (b.P.ms[k]) MPM_TRY(snap_one(b.P.ms[k], np));
        for (int d = 0; d < 3; d++) {
          MPM_TRY(snap_one(b.P.xl[d], np));
          MPM_TRY(snap_one(b.P.vl[d], np));
        }
        MPM_TRY(snap_one(b.P.ml, np));
        MPM_TRY(snap_one(b.A.m, ns));
        for (int d = 0; d < 3; d++) {
          MPM_TRY(snap_one(b.A.mx[d], ns));
          MPM_TRY(snap_one(b.A.f[d], ns));
          MPM_TRY(snap_one(b.A.nrm[d], ns));
          MPM_TRY(snap_one(b.V.vt[d], ns));
          MPM_TRY(snap_one(b.V.dv[d], ns));
        }
      }
    }
    MPM_TRY(snap_one(flags_, (size_t)cap_blocks_ * sizeof(uint32_t)));
    MPM_TRY(snap_one(was_active_, (size_t)cap_blocks_));
    snap_pbuf_.clear();
    for (auto& j : jobs_)
      for (auto& b : j.bodies) snap_pbuf_.push_back(b.P.x[0]);
    MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
    return MPMGPU_OK;
  }

  mpmgpu_status snapshot_restore() {
    // after the trial the current buffer may be the other one: restore the
    // saved point arrays into the buffer that was current at the save
    size_t k = 0;
    for (auto& j : jobs_)
      for (auto& b : j.bodies) {
        if (k < snap_pbuf_.size() && b.P.x[0] != snap_pbuf_[k]) std::swap(b.P, b.Palt);
        k++;
      }
    for (auto& s : snap_)
      MPM_CUDA_TRY(cudaMemcpyAsync(s.second.first, s.first, s.second.second, cudaMemcpyDeviceToDevice, stream_));
    // the table's point pointers must match the mirrors again
    tables_dirty_ = true;
    const bool m = membership_dirty_;
    MPM_TRY(commit());
    membership_dirty_ = m;
    MPM_CUDA_TRY(cudaStreamSynchronize(stream_));
    return MPMGPU_OK;
  }

  void snapshot_free() {
    for (auto& s : snap_) cudaFree(s.first);
    snap_.clear();
  }
  std::vector<void*> snap_pbuf_;

  // ---- state ----
  int dim_;
  int device_;
  bool keep_debug_;
  bool use_graph_;
  bool det_ = false;   // deterministic form: two-level exact nodal sums
  int sort_interval_ = 32;
  int cap_ = 512;
  int sm_count_ = 148;
  int fused_per_sm_[24] = {};
  cudaStream_t copy_stream_ = nullptr;
  cudaEvent_t upload_ev_ = nullptr;
  // one-body launches of the second to fourth body (one_body_launches)
  static constexpr int kSideStreams = 3;
  cudaStream_t side_[kSideStreams] = {};
  cudaEvent_t fork_ev_ = nullptr;
  cudaEvent_t join_ev_[kSideStreams] = {};
  cudaMemPool_t pool_ = nullptr;
  void* stage_ = nullptr;
  size_t stage_cap_ = 0, stage_used_ = 0;
  std::vector<BodyCtx<PT>> ctx_host_;   // host copy of the body table
  bool single_mode_ = false;
  bool any_plain_ = false, any_normal_ = false;
  // the frame in flight or last taken (frame_begin): field offsets (in
  // doubles) in its pinned copy
  struct Frame {
    int job = -1;
    bool pending = false;
    bool primed = false;
    int64_t nnodes = 0;
    double grav[3] = {0.0, 0.0, 0.0};
    std::vector<FramePointLayout> pts;
    std::vector<int64_t> npts;
    std::vector<FrameNodeLayout> nodes;
    std::vector<std::pair<int64_t, int64_t>> contact;   // normal, force
    const double* data = nullptr;
    const int* err = nullptr;
  } frame_;
  void* frame_stage_ = nullptr;   // pinned host copy
  size_t frame_cap_ = 0;
  void* frame_dev_ = nullptr;     // device staging in the reference layout
  size_t frame_dev_cap_ = 0;
  cudaEvent_t frame_ev_ = nullptr;

  mpmgpu_status frame_wait() {
    if (!frame_.pending) return MPMGPU_OK;
    frame_.pending = false;
    MPM_CUDA_TRY(cudaEventSynchronize(frame_ev_));
    const int flag = *frame_.err;
    if (flag & kErrWideSpan) return fail(MPMGPU_ERR_DEVICE, "point corners span more than two cells (extent > cell size)");
    if (flag & kErrElemAlias) return fail(MPMGPU_ERR_DEVICE, "point within rounding of the upper domain face");
    if (flag & kErrWaitTimeout) return fail(MPMGPU_ERR_DEVICE, "a bulk copy did not complete within the wait limit");
    if (flag & kErrItemCap) return fail(MPMGPU_ERR_DEVICE, "a work item holds more points than the kernel takes");
    return MPMGPU_OK;
  }

  mpmgpu_status frame_body(int job, int body, HBody** B) {
    if (job != frame_.job) return fail(MPMGPU_ERR_STATE, "no frame of this job was begun");
    HJob* j;
    MPM_TRY(readable_body(job, body, &j, B));
    if (body >= (int)frame_.pts.size()) return fail(MPMGPU_ERR_ARG, "no such body in the frame");
    return MPMGPU_OK;
  }
  bool all_elastic_ = true;              // every body IsotropicLinearElasticity (or no material)
  int form_ = kFormStaged;               // form of the fused kernel (cap_: its points per item)
  uint32_t wait_polls_ = kWaitPolls;     // poll limit of the fused kernels' first waits
  int lean_per_sm_[32] = {};
  int flip_ = 0;                        // point buffers swapped an odd number of times
  cudaStream_t stream_ = nullptr;
  std::vector<HJob> jobs_;
  int live_jobs_ = 0;
  bool membership_dirty_ = false;
  bool tables_dirty_ = false;
  int steps_since_sort_ = 0;
  int64_t launches_ = 0;
  int64_t scratch_bytes_ = 0;
  std::vector<void*> scratch_allocs_;
  std::vector<void*> cap_allocs_;
  // job slots
  std::vector<int> free_slots_;
  int next_slot_ = 0;
  // block space
  std::vector<std::pair<int64_t, int64_t>> free_;
  int64_t block_end_ = 0;
  // device tables and scratch
  BatchHdr* hdr_ = nullptr;
  BatchHdr hdr_host_{};
  unsigned long long* count_ = nullptr;
  int* err_ = nullptr;
  unsigned long long* drift_ = nullptr;
  int* queue_ = nullptr;   // the fused kernels' work queue (claim_item), zero between launches
  int32_t* nwork_ = nullptr;
  unsigned long long* active_nodes_ = nullptr;
  InstDev* insts_d_ = nullptr;
  int64_t cap_insts_ = 0;
  GridBody* gbodies_d_ = nullptr;
  int64_t cap_bodies_g_ = 0;
  BodyCtx<PT>* ctx_d_ = nullptr;
  int64_t cap_bodies_c_ = 0;
  int64_t* point_end_d_ = nullptr;
  int64_t cap_bodies_p_ = 0;
  int64_t* bin_end_d_ = nullptr;
  int64_t cap_bodies_b_ = 0;
  uint32_t* flags_ = nullptr;
  int64_t cap_blocks_ = 0;
  uint8_t* was_active_ = nullptr;
  int32_t* blk_inst_ = nullptr;
  int64_t* list_ = nullptr;
  int32_t* key_ = nullptr;
  int64_t cap_points_k_ = 0;
  int32_t* rank_ = nullptr;
  int64_t cap_points_r_ = 0;
  int32_t* cell_count_ = nullptr;
  int64_t cap_cells_ = 0;
  void* dl_stage_ = nullptr;   // pinned staging of downloads
  size_t dl_cap_ = 0;
  unsigned long long* cell_hist_ = nullptr;   // per cell: 8 class counts of 8 bits
  int64_t cap_cells_h_ = 0;
  int16_t* crank_ = nullptr;                  // per point: class << 8 | rank in class
  int64_t cap_points_c_ = 0;
  int32_t* bin_scan_ = nullptr;
  int64_t cap_bins_ = 0;
  int32_t* chunk_sum_ = nullptr;
  int64_t cap_chunks_ = 0;
  int32_t* flat_body_ = nullptr;
  int64_t cap_items_fb_ = 0;
  int32_t* flat_item_ = nullptr;
  int64_t cap_items_fi_ = 0;
  unsigned long long* bounds_ = nullptr;   // deterministic form: 4 per body
  int64_t cap_bounds_ = 0;
  int32_t* item_off_d_ = nullptr;
  int64_t cap_bodies_i_ = 0;
  int32_t* nwork_body_ = nullptr;
  int64_t cap_bodies_w_ = 0;
  int32_t* work_end_body_ = nullptr;
  int64_t cap_bodies_e_ = 0;
  int32_t* work_bin_ = nullptr;
  int64_t cap_items_n_ = 0;
  int32_t* work_start_ = nullptr;
  int64_t cap_items_s_ = 0;
  int32_t* work_end_ = nullptr;
  int64_t cap_items_e_ = 0;
  cudaGraphExec_t g_step_[2] = {nullptr, nullptr};
  int g_step_k_[2] = {0, 0};
  int g_sort_k_ = 0;
  cudaGraphExec_t g_sort_ = nullptr;
  bool step_warm_[2] = {false, false};
  bool sort_warm_ = false;
  // profiling
  bool profiling_ = false;
  std::vector<cudaEvent_t> event_pool_;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending_[kStages];
  int64_t stage_launches_[kStages] = {0, 0, 0, 0};
  double stage_ms_[kStages] = {0.0, 0.0, 0.0, 0.0};
};

}  // namespace mpmb200
