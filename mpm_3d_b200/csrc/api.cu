// Host side of the C ABI declared in include/mpm_b200.h.
//
// One step on the device (FP64 form):
//   compact   active node blocks flagged by the last scatter -> work list
//   grid      body force, contact, boundary, moveGrid on the active blocks
//   g2p2g     per bin of points: gather + point update (this step), map
//             build + scatter at the new positions (next step)
// plus, every sort_interval steps, a re-binning of the points. Before the
// first step a scatter-only pass of the fused kernel builds the first
// nodal sums.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "fused.cuh"
#include "kernels_fp64.cuh"
#include "sort.cuh"

using namespace mpmb200;

namespace {

struct BodyDev {
  int64_t n = 0;
  PointsDev P{};      // current storage order
  PointsDev Palt{};   // second buffer for re-binning
  NodesAcc A{};
  NodesVel V{};
  NodesAcc snap{};    // debug copies (m, mx, f) or null
  MaterialParams mat{};
  int has_boundary = 0;
  bool needs_normal = false;
  // binning
  int32_t* key = nullptr;
  int32_t* rank = nullptr;
  int32_t* cell_count = nullptr;  // nbins * cells_per_bin + 1
  int32_t* bin_start = nullptr;   // nbins + 2
  int32_t* work_bin = nullptr;
  int32_t* work_start = nullptr;
  int32_t* work_end = nullptr;
  int32_t* nwork = nullptr;
};

}  // namespace

struct mpmgpu_handle {
  mpmgpu_config cfg{};
  Geom g{};
  MapConst mc{};
  BinGeom bg{};
  StepParams sp{};
  cudaStream_t stream = nullptr;
  std::vector<BodyDev> bodies;
  ContactSet cs{};
  uint32_t* flags = nullptr;
  int64_t* list = nullptr;
  unsigned long long* count = nullptr;
  uint8_t* was_active = nullptr;
  int* err = nullptr;
  unsigned long long* drift = nullptr;
  std::vector<void*> allocs;
  std::string last_error;
  int64_t launches = 0;
  int sm_count = 148;
  bool stepped = false;
  bool primed = false;
  int steps_since_sort = 0;
  int sort_interval = 32;
  int fused_blocks = 0;
  // per-stage event timing (mpmgpu_profile)
  static constexpr int kStages = 4;
  bool profiling = false;
  std::vector<cudaEvent_t> event_pool;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[kStages];
  int64_t stage_launches[kStages] = {0, 0, 0, 0};
  double stage_ms[kStages] = {0.0, 0.0, 0.0, 0.0};
};

namespace {

mpmgpu_status fail(mpmgpu_handle* h, mpmgpu_status s, const std::string& msg) {
  if (h) h->last_error = msg;
  return s;
}

#define CUDA_TRY(h, expr)                                                                                     \
  do {                                                                                                        \
    cudaError_t e_ = (expr);                                                                                  \
    if (e_ != cudaSuccess) return fail((h), MPMGPU_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define TRY(expr)                   \
  do {                              \
    mpmgpu_status s_ = (expr);      \
    if (s_ != MPMGPU_OK) return s_; \
  } while (0)

template <typename T>
mpmgpu_status dev_alloc(mpmgpu_handle* h, T** p, size_t count) {
  void* q = nullptr;
  const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) return fail(h, MPMGPU_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  h->allocs.push_back(q);
  e = cudaMemsetAsync(q, 0, bytes, h->stream);
  if (e != cudaSuccess) return fail(h, MPMGPU_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
  *p = static_cast<T*>(q);
  return MPMGPU_OK;
}

int grid_blocks(const mpmgpu_handle* h, int64_t work, int threads) {
  int64_t b = (work + threads - 1) / threads;
  const int64_t cap = (int64_t)h->sm_count * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

mpmgpu_status check_launch(mpmgpu_handle* h, const char* what) {
  h->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, MPMGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return MPMGPU_OK;
}

// Stage timing: records a start event before and a stop event after the
// stage's launches when profiling is on.
struct StageTimer {
  mpmgpu_handle* h;
  int stage;
  cudaEvent_t start = nullptr;
  StageTimer(mpmgpu_handle* hh, int s) : h(hh), stage(s) {
    if (!h->profiling) return;
    start = take_event();
    cudaEventRecord(start, h->stream);
  }
  ~StageTimer() {
    if (!h->profiling || !start) return;
    cudaEvent_t stop = take_event();
    cudaEventRecord(stop, h->stream);
    h->pending[stage].push_back({start, stop});
  }
  cudaEvent_t take_event() {
    cudaEvent_t e = nullptr;
    if (!h->event_pool.empty()) {
      e = h->event_pool.back();
      h->event_pool.pop_back();
    } else {
      cudaEventCreate(&e);
    }
    return e;
  }
};

std::vector<double> column(const double* aos, int64_t n, int w, int d) {
  std::vector<double> out((size_t)n);
  for (int64_t i = 0; i < n; i++) out[(size_t)i] = aos[i * w + d];
  return out;
}

template <typename T>
mpmgpu_status upload(mpmgpu_handle* h, T* dst, const std::vector<T>& src) {
  if (src.empty()) return MPMGPU_OK;
  CUDA_TRY(h, cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return MPMGPU_OK;
}

template <typename T>
mpmgpu_status download(mpmgpu_handle* h, std::vector<T>& dst, const T* src, size_t n) {
  dst.resize(n);
  if (n == 0) return MPMGPU_OK;
  CUDA_TRY(h, cudaMemcpyAsync(dst.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return MPMGPU_OK;
}

// Point arrays hold n entries plus 8 of padding: the fused kernel's bulk
// copies round their windows out to 16-byte boundaries and may read up to 3
// entries past the last point.
mpmgpu_status alloc_points(mpmgpu_handle* h, PointsDev& P, int64_t n, bool with_L) {
  P.n = n;
  const size_t na = (size_t)n + 8;
  for (int d = 0; d < 3; d++) {
    TRY(dev_alloc(h, &P.x[d], na));
    TRY(dev_alloc(h, &P.v[d], na));
    TRY(dev_alloc(h, &P.u[d], na));
  }
  for (int c = 0; c < 6; c++) TRY(dev_alloc(h, &P.s[c], na));
  TRY(dev_alloc(h, &P.vol, na));
  TRY(dev_alloc(h, &P.m, na));
  TRY(dev_alloc(h, &P.ext, na));
  TRY(dev_alloc(h, &P.active, na));
  TRY(dev_alloc(h, &P.pid, na));
  P.L = nullptr;
  if (with_L) TRY(dev_alloc(h, &P.L, (size_t)n * 9));
  return MPMGPU_OK;
}

PointArrays point_arrays(const PointsDev& P) {
  PointArrays a{};
  a.nf = 0;
  for (int d = 0; d < 3; d++) a.f[a.nf++] = P.x[d];
  for (int d = 0; d < 3; d++) a.f[a.nf++] = P.v[d];
  for (int d = 0; d < 3; d++) a.f[a.nf++] = P.u[d];
  for (int c = 0; c < 6; c++) a.f[a.nf++] = P.s[c];
  a.f[a.nf++] = P.vol;
  a.f[a.nf++] = P.m;
  a.f[a.nf++] = P.ext;
  a.ni = 0;
  a.i[a.ni++] = P.active;
  a.i[a.ni++] = P.pid;
  a.L9 = P.L;
  return a;
}

// Re-bins the points of one body (counting sort by bin, rank-major within
// bins) and rebuilds the work list of non-empty bins.
template <int DIM>
mpmgpu_status sort_body(mpmgpu_handle* h, BodyDev& B) {
  cudaStream_t st = h->stream;
  const BinGeom& bg = h->bg;
  const int64_t ncells = (int64_t)bg.nbins * bg.cells_per_bin + 1;
  CUDA_TRY(h, cudaMemsetAsync(B.cell_count, 0, ncells * sizeof(int32_t), st));
  CUDA_TRY(h, cudaMemsetAsync(B.nwork, 0, sizeof(int32_t), st));
  if (B.n > 0) {
    k_sort_count<DIM><<<grid_blocks(h, B.n, 256), 256, 0, st>>>(h->g, bg, B.P, B.key, B.rank, B.cell_count);
    TRY(check_launch(h, "k_sort_count"));
  }
  k_bin_totals<<<(bg.nbins + 1 + 255) / 256, 256, 0, st>>>(bg, B.cell_count, B.bin_start);
  TRY(check_launch(h, "k_bin_totals"));
  k_scan_small<<<1, 1024, 0, st>>>(B.bin_start, bg.nbins + 1, B.bin_start + bg.nbins + 1);
  TRY(check_launch(h, "k_scan_small"));
  if (B.n > 0) {
    k_sort_scatter<<<grid_blocks(h, B.n, 256), 256, 0, st>>>(bg, B.n, B.key, B.rank, B.cell_count, B.bin_start,
                                                             point_arrays(B.P), point_arrays(B.Palt));
    TRY(check_launch(h, "k_sort_scatter"));
    std::swap(B.P, B.Palt);
  }
  k_bin_work<<<(bg.nbins + 255) / 256, 256, 0, st>>>(bg, B.bin_start, kCap, B.work_bin, B.work_start, B.work_end,
                                                      B.nwork);
  TRY(check_launch(h, "k_bin_work"));
  return MPMGPU_OK;
}

template <int DIM, int BB, bool NORMAL>
mpmgpu_status launch_fused(mpmgpu_handle* h, BodyDev& B, int do_g2p, int do_p2g) {
  FusedParams fp{};
  fp.g = h->g;
  fp.mc = h->mc;
  fp.bg = h->bg;
  fp.sp = h->sp;
  fp.mat = B.mat;
  fp.P = B.P;
  fp.V = B.V;
  fp.A = B.A;
  fp.work_bin = B.work_bin;
  fp.work_start = B.work_start;
  fp.work_end = B.work_end;
  fp.nwork = B.nwork;
  fp.flags = h->flags;
  fp.err = h->err;
  fp.drift = h->drift;
  fp.do_g2p = do_g2p;
  fp.do_p2g = do_p2g;
  const size_t smem = fused_smem_bytes<DIM, BB>(NORMAL);
  static bool configured = false;
  if (!configured) {
    CUDA_TRY(h, cudaFuncSetAttribute(k_g2p2g<DIM, BB, NORMAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = true;
  }
  int per_sm = 0;
  CUDA_TRY(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_g2p2g<DIM, BB, NORMAL>, kFusedThreads, smem));
  const int blocks = std::max(1, per_sm) * h->sm_count;
  StageTimer timer(h, 0);
  k_g2p2g<DIM, BB, NORMAL><<<blocks, kFusedThreads, smem, h->stream>>>(fp);
  return check_launch(h, "k_g2p2g");
}

template <int DIM>
mpmgpu_status fused(mpmgpu_handle* h, BodyDev& B, int do_g2p, int do_p2g) {
  constexpr int BB = DIM == 3 ? 4 : 8;
  if (B.needs_normal) return launch_fused<DIM, BB, true>(h, B, do_g2p, do_p2g);
  return launch_fused<DIM, BB, false>(h, B, do_g2p, do_p2g);
}

template <int DIM>
mpmgpu_status step_once(mpmgpu_handle* h) {
  const Geom& g = h->g;
  cudaStream_t st = h->stream;
  if (!h->primed) {
    for (BodyDev& B : h->bodies) TRY(sort_body<DIM>(h, B));
    for (BodyDev& B : h->bodies) TRY(fused<DIM>(h, B, 0, 1));
    h->primed = true;
    h->steps_since_sort = 0;
  }
  GridBodies GB{};
  GB.nb = (int)h->bodies.size();
  for (size_t b = 0; b < h->bodies.size(); b++) {
    GB.acc[b] = h->bodies[b].A;
    GB.vel[b] = h->bodies[b].V;
    GB.snap[b] = h->bodies[b].snap;
    GB.has_boundary[b] = h->bodies[b].has_boundary;
  }
  {
    StageTimer timer(h, 2);
    CUDA_TRY(h, cudaMemsetAsync(h->count, 0, sizeof(unsigned long long), st));
    k_compact<<<grid_blocks(h, g.nblocks, 256), 256, 0, st>>>(g.nblocks, h->flags, h->list, h->count, h->was_active);
    TRY(check_launch(h, "k_compact"));
  }
  {
    StageTimer timer(h, 1);
    const int gb = (int)std::min<int64_t>(std::max<int64_t>(g.nblocks, 1), (int64_t)h->sm_count * 32);
    k_grid<DIM><<<gb, 64, 0, st>>>(g, h->sp, GB, h->cs, h->list, h->count);
    TRY(check_launch(h, "k_grid"));
  }
  for (BodyDev& B : h->bodies) TRY(fused<DIM>(h, B, 1, 1));
  if (++h->steps_since_sort >= h->sort_interval) {
    StageTimer timer(h, 3);
    for (BodyDev& B : h->bodies) TRY(sort_body<DIM>(h, B));
    h->steps_since_sort = 0;
  }
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

const char* mpmgpu_last_error(const mpmgpu_handle* h) { return h ? h->last_error.c_str() : ""; }

mpmgpu_status mpmgpu_create(const mpmgpu_config* cfg, mpmgpu_handle** out) {
  if (!cfg || !out) return MPMGPU_ERR_ARG;
  *out = nullptr;
  if (cfg->dim != 2 && cfg->dim != 3) return MPMGPU_ERR_UNSUPPORTED;
  if (!(cfg->dt > 0)) return MPMGPU_ERR_ARG;
  if (cfg->cpdi_spec != 0 && cfg->cpdi_spec != 1) return MPMGPU_ERR_ARG;
  if (cfg->contact_spec != 0 && cfg->contact_spec != 1) return MPMGPU_ERR_ARG;
  if (cfg->mode != MPMGPU_MODE_FP64) return MPMGPU_ERR_UNSUPPORTED;
  if (cfg->sort_interval < 0) return MPMGPU_ERR_ARG;
  for (int d = 0; d < cfg->dim; d++)
    if (cfg->N[d] < 1 || !(cfg->L[d] > 0)) return MPMGPU_ERR_ARG;
  mpmgpu_handle* h = new mpmgpu_handle();
  h->cfg = *cfg;
  h->sort_interval = cfg->sort_interval > 0 ? cfg->sort_interval : 32;
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) {
    delete h;
    return MPMGPU_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, cfg->device);
  e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete h;
    return MPMGPU_ERR_CUDA;
  }
  Geom& g = h->g;
  g.dim = cfg->dim;
  g.cp = 1 << cfg->dim;
  g.nnodes = 1;
  for (int d = 0; d < 3; d++) {
    if (d < cfg->dim) {
      g.L[d] = cfg->L[d];
      g.N[d] = cfg->N[d];
      g.h[d] = cfg->L[d] / cfg->N[d];  // cartesian.cpp:40
      g.nn[d] = cfg->N[d] + 1;
      g.nnodes *= g.nn[d];
      h->mc.NL[d] = (double)cfg->N[d] / cfg->L[d];
      h->mc.invh[d] = 1.0 / g.h[d];
    } else {
      g.L[d] = 0.0;
      g.N[d] = 0;
      g.h[d] = 0.0;
      g.nn[d] = 1;
      h->mc.NL[d] = 0.0;
      h->mc.invh[d] = 0.0;
    }
  }
  if (cfg->dim == 3) {
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
  BinGeom& bg = h->bg;
  bg.B = cfg->dim == 3 ? 4 : 8;
  bg.cells_per_bin = cfg->dim == 3 ? 64 : 64;
  bg.nbx = (g.N[0] + bg.B - 1) / bg.B;
  bg.nby = (g.N[1] + bg.B - 1) / bg.B;
  bg.nbz = cfg->dim == 3 ? (g.N[2] + bg.B - 1) / bg.B : 1;
  bg.nbins = bg.nbx * bg.nby * bg.nbz;
  bg.T = bg.B + 3;
  bg.tile_nodes = cfg->dim == 3 ? bg.T * bg.T * bg.T : bg.T * bg.T;
  h->sp.dt = cfg->dt;
  h->sp.cpdi = cfg->cpdi_spec;
  h->sp.contact_spec = cfg->contact_spec;
  h->sp.keep_debug = cfg->keep_debug;
  // DefaultDriver gravity until set otherwise (default_driver.cpp:90-105)
  h->sp.grav[0] = h->sp.grav[1] = h->sp.grav[2] = 0.0;
  h->sp.grav[cfg->dim == 2 ? 1 : 2] = -9.81;
  mpmgpu_status s = MPMGPU_OK;
  if ((s = dev_alloc(h, &h->flags, (size_t)g.nblocks)) != MPMGPU_OK ||
      (s = dev_alloc(h, &h->list, (size_t)g.nblocks)) != MPMGPU_OK || (s = dev_alloc(h, &h->count, 1)) != MPMGPU_OK ||
      (s = dev_alloc(h, &h->was_active, (size_t)g.nblocks)) != MPMGPU_OK || (s = dev_alloc(h, &h->err, 1)) != MPMGPU_OK ||
      (s = dev_alloc(h, &h->drift, 1)) != MPMGPU_OK) {
    mpmgpu_destroy(h);
    return s;
  }
  *out = h;
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_add_body(mpmgpu_handle* h, const mpmgpu_body_desc* desc, int* body_id) {
  if (!h || !desc) return MPMGPU_ERR_ARG;
  if (h->stepped) return fail(h, MPMGPU_ERR_STATE, "bodies must be added before the first step");
  if ((int)h->bodies.size() >= kMaxBodies) return fail(h, MPMGPU_ERR_UNSUPPORTED, "too many bodies");
  if (desc->n < 0 || desc->n > (int64_t)INT32_MAX / 2 ||
      (desc->n > 0 && (!desc->m || !desc->v || !desc->x || !desc->x_t)))
    return fail(h, MPMGPU_ERR_ARG, "body arrays missing or too many points");
  const int D = h->g.dim;
  const int64_t n = desc->n;
  BodyDev B;
  B.n = n;
  TRY(alloc_points(h, B.P, n, h->cfg.keep_debug != 0));
  TRY(alloc_points(h, B.Palt, n, h->cfg.keep_debug != 0));
  if (n > 0) {
    for (int d = 0; d < D; d++) {
      TRY(upload(h, B.P.x[d], column(desc->x, n, 3, d)));
      TRY(upload(h, B.P.v[d], column(desc->x_t, n, 3, d)));
    }
    std::vector<double> tmp(desc->m, desc->m + n);
    TRY(upload(h, B.P.m, tmp));
    tmp.assign(desc->v, desc->v + n);
    TRY(upload(h, B.P.vol, tmp));
    // extent, default_points.cpp:49-57 (computed once, never updated)
    for (int64_t i = 0; i < n; i++) tmp[(size_t)i] = (D == 2) ? 0.5 * std::sqrt(desc->v[i]) : 0.5 * std::cbrt(desc->v[i]);
    TRY(upload(h, B.P.ext, tmp));
    if (desc->u)
      for (int d = 0; d < D; d++) TRY(upload(h, B.P.u[d], column(desc->u, n, 3, d)));
    if (desc->T) {
      // stored as xx yy zz xy yz xz (row-major 9 -> symmetric 6)
      static const int idx[6] = {0, 4, 8, 1, 5, 2};
      for (int c = 0; c < 6; c++) TRY(upload(h, B.P.s[c], column(desc->T, n, 9, idx[c])));
    }
    std::vector<int32_t> act((size_t)n, 1), pid((size_t)n);
    for (int64_t i = 0; i < n; i++) {
      if (desc->active) act[(size_t)i] = desc->active[i] != 0 ? 1 : 0;
      pid[(size_t)i] = (int32_t)i;
    }
    TRY(upload(h, B.P.active, act));
    TRY(upload(h, B.P.pid, pid));
  }
  const size_t ns = (size_t)h->g.nslots;
  TRY(dev_alloc(h, &B.A.m, ns));
  for (int d = 0; d < 3; d++) {
    TRY(dev_alloc(h, &B.A.mx[d], ns));
    TRY(dev_alloc(h, &B.A.f[d], ns));
    TRY(dev_alloc(h, &B.V.vt[d], ns));
    TRY(dev_alloc(h, &B.V.dv[d], ns));
    B.A.nrm[d] = nullptr;
  }
  if (h->cfg.keep_debug) {
    TRY(dev_alloc(h, &B.snap.m, ns));
    for (int d = 0; d < 3; d++) {
      TRY(dev_alloc(h, &B.snap.mx[d], ns));
      TRY(dev_alloc(h, &B.snap.f[d], ns));
      B.snap.nrm[d] = nullptr;
    }
  }
  const BinGeom& bg = h->bg;
  TRY(dev_alloc(h, &B.key, (size_t)n));
  TRY(dev_alloc(h, &B.rank, (size_t)n));
  TRY(dev_alloc(h, &B.cell_count, (size_t)bg.nbins * bg.cells_per_bin + 1));
  TRY(dev_alloc(h, &B.bin_start, (size_t)bg.nbins + 2));
  const size_t max_items = (size_t)bg.nbins + (size_t)n / kCap + 1;
  TRY(dev_alloc(h, &B.work_bin, max_items));
  TRY(dev_alloc(h, &B.work_start, max_items));
  TRY(dev_alloc(h, &B.work_end, max_items));
  TRY(dev_alloc(h, &B.nwork, 1));
  B.mat.has_material = desc->has_material;
  if (desc->has_material) {
    // isolin.cpp:34-38
    const double E = desc->E, nu = desc->nu;
    const double G = E / (2.0 * (1.0 + nu));
    const double K = E / (3.0 * (1.0 - 2 * nu));
    B.mat.G = G;
    B.mat.lambda = K - 2.0 * G / 3.0;
  }
  B.has_boundary = desc->has_boundary;
  h->bodies.push_back(B);
  if (body_id) *body_id = (int)h->bodies.size() - 1;
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_add_contact(mpmgpu_handle* h, int body1, int body2, double mu_f, int* contact_id) {
  if (!h) return MPMGPU_ERR_ARG;
  if (h->stepped) return fail(h, MPMGPU_ERR_STATE, "contacts must be added before the first step");
  if (body1 < 0 || body2 < 0 || body1 >= (int)h->bodies.size() || body2 >= (int)h->bodies.size() || body1 == body2)
    return fail(h, MPMGPU_ERR_ARG, "contact bodies out of range");
  if (h->cs.nc >= kMaxContacts) return fail(h, MPMGPU_ERR_UNSUPPORTED, "too many contacts");
  BodyDev& B1 = h->bodies[(size_t)body1];
  const size_t ns = (size_t)h->g.nslots;
  if (!B1.needs_normal) {
    for (int d = 0; d < 3; d++) TRY(dev_alloc(h, &B1.A.nrm[d], ns));
    B1.needs_normal = true;
  }
  const int c = h->cs.nc;
  h->cs.b1[c] = body1;
  h->cs.b2[c] = body2;
  h->cs.mu[c] = mu_f;
  h->cs.normal_out[c] = nullptr;
  h->cs.force_out[c] = nullptr;
  if (h->cfg.keep_debug) {
    TRY(dev_alloc(h, &h->cs.normal_out[c], 3 * ns));
    TRY(dev_alloc(h, &h->cs.force_out[c], 3 * ns));
  }
  h->cs.nc++;
  if (contact_id) *contact_id = c;
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_set_gravity(mpmgpu_handle* h, int use_vector, const double g[3]) {
  if (!h) return MPMGPU_ERR_ARG;
  for (int d = 0; d < 3; d++) h->sp.grav[d] = 0.0;
  if (use_vector) {
    if (!g) return fail(h, MPMGPU_ERR_ARG, "gravity vector missing");
    for (int d = 0; d < h->g.dim; d++) h->sp.grav[d] = g[d];
  } else {
    h->sp.grav[h->g.dim == 2 ? 1 : 2] = -9.81;
  }
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_step(mpmgpu_handle* h, int nsteps) {
  if (!h || nsteps < 0) return MPMGPU_ERR_ARG;
  if (h->bodies.empty()) return fail(h, MPMGPU_ERR_STATE, "no bodies");
  h->stepped = true;
  for (int s = 0; s < nsteps; s++) {
    mpmgpu_status r = (h->g.dim == 3) ? step_once<3>(h) : step_once<2>(h);
    if (r != MPMGPU_OK) return r;
  }
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_synchronize(mpmgpu_handle* h) {
  if (!h) return MPMGPU_ERR_ARG;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  int flag = 0;
  CUDA_TRY(h, cudaMemcpy(&flag, h->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag & kErrWideSpan) return fail(h, MPMGPU_ERR_DEVICE, "point corners span more than two cells (extent > cell size)");
  if (flag & kErrElemAlias) return fail(h, MPMGPU_ERR_DEVICE, "point within rounding of the upper domain face");
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_sizes(const mpmgpu_handle* h, int body, int64_t* n_points, int64_t* n_nodes) {
  if (!h || body < 0 || body >= (int)h->bodies.size()) return MPMGPU_ERR_ARG;
  if (n_points) *n_points = h->bodies[(size_t)body].n;
  if (n_nodes) *n_nodes = h->g.nnodes;
  return MPMGPU_OK;
}

int64_t mpmgpu_launch_count(const mpmgpu_handle* h) { return h ? h->launches : 0; }

void* mpmgpu_stream(const mpmgpu_handle* h) { return h ? (void*)h->stream : nullptr; }

mpmgpu_status mpmgpu_profile(mpmgpu_handle* h, int enable) {
  if (!h) return MPMGPU_ERR_ARG;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (int s = 0; s < mpmgpu_handle::kStages; s++) {
    for (auto& pr : h->pending[s]) {
      h->event_pool.push_back(pr.first);
      h->event_pool.push_back(pr.second);
    }
    h->pending[s].clear();
    h->stage_launches[s] = 0;
    h->stage_ms[s] = 0.0;
  }
  h->profiling = enable != 0;
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_profile_read(mpmgpu_handle* h, int stage, int64_t* launches, double* total_ms) {
  if (!h || stage < 0 || stage >= mpmgpu_handle::kStages) return MPMGPU_ERR_ARG;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (int s = 0; s < mpmgpu_handle::kStages; s++) {
    for (auto& pr : h->pending[s]) {
      float ms = 0.0f;
      CUDA_TRY(h, cudaEventElapsedTime(&ms, pr.first, pr.second));
      h->stage_ms[s] += ms;
      h->stage_launches[s]++;
      h->event_pool.push_back(pr.first);
      h->event_pool.push_back(pr.second);
    }
    h->pending[s].clear();
  }
  if (launches) *launches = h->stage_launches[stage];
  if (total_ms) *total_ms = h->stage_ms[stage];
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_download_points(mpmgpu_handle* h, int body, int field, double* out) {
  if (!h || !out || body < 0 || body >= (int)h->bodies.size()) return MPMGPU_ERR_ARG;
  TRY(mpmgpu_synchronize(h));
  BodyDev& B = h->bodies[(size_t)body];
  const int64_t n = B.n;
  const int D = h->g.dim;
  std::vector<int32_t> pid;
  TRY(download(h, pid, B.P.pid, (size_t)n));
  std::vector<double> tmp;
  auto vec3 = [&](double* const* arr) -> mpmgpu_status {
    for (int64_t i = 0; i < 3 * n; i++) out[i] = 0.0;
    for (int d = 0; d < D; d++) {
      TRY(download(h, tmp, arr[d], (size_t)n));
      for (int64_t i = 0; i < n; i++) out[3 * (int64_t)pid[(size_t)i] + d] = tmp[(size_t)i];
    }
    return MPMGPU_OK;
  };
  auto scal = [&](const double* arr) -> mpmgpu_status {
    TRY(download(h, tmp, arr, (size_t)n));
    for (int64_t i = 0; i < n; i++) out[pid[(size_t)i]] = tmp[(size_t)i];
    return MPMGPU_OK;
  };
  switch (field) {
    case MPMGPU_P_X: return vec3(B.P.x);
    case MPMGPU_P_U: return vec3(B.P.u);
    case MPMGPU_P_X_T: return vec3(B.P.v);
    case MPMGPU_P_MX_T: {
      TRY(vec3(B.P.v));
      std::vector<double> m;
      TRY(download(h, m, B.P.m, (size_t)n));
      // movePoints: mx_t = m * x_t (explicit_usl.cpp:295-297)
      for (int64_t i = 0; i < n; i++) {
        const int64_t q = pid[(size_t)i];
        for (int d = 0; d < D; d++) out[3 * q + d] = m[(size_t)i] * out[3 * q + d];
      }
      return MPMGPU_OK;
    }
    case MPMGPU_P_B:
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) out[3 * i + d] = h->sp.grav[d];
      return MPMGPU_OK;
    case MPMGPU_P_L:
      if (!B.P.L) return fail(h, MPMGPU_ERR_STATE, "L is kept only with keep_debug");
      TRY(download(h, tmp, B.P.L, (size_t)n * 9));
      for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 9; k++) out[9 * (int64_t)pid[(size_t)i] + k] = tmp[(size_t)(9 * i + k)];
      return MPMGPU_OK;
    case MPMGPU_P_T: {
      static const int idx[9] = {0, 3, 5, 3, 1, 4, 5, 4, 2};
      std::vector<std::vector<double>> s(6);
      for (int c = 0; c < 6; c++) TRY(download(h, s[(size_t)c], B.P.s[c], (size_t)n));
      for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 9; k++) out[9 * (int64_t)pid[(size_t)i] + k] = s[(size_t)idx[k]][(size_t)i];
      return MPMGPU_OK;
    }
    case MPMGPU_P_M: return scal(B.P.m);
    case MPMGPU_P_V: return scal(B.P.vol);
    case MPMGPU_P_EXTENT: return scal(B.P.ext);
    case MPMGPU_P_ACTIVE: {
      std::vector<int32_t> a;
      TRY(download(h, a, B.P.active, (size_t)n));
      // 2 = left the domain at the last move: still active until the next
      // map build deactivates it, as in the reference
      for (int64_t i = 0; i < n; i++) out[pid[(size_t)i]] = a[(size_t)i] != 0 ? 1.0 : 0.0;
      return MPMGPU_OK;
    }
  }
  return fail(h, MPMGPU_ERR_ARG, "unknown point field");
}

}  // extern "C"

namespace {

// Copies a block-linear nodal array (comps SoA components) to reference node
// order; nodes of blocks that were not active in the last step read `fill`.
mpmgpu_status nodes_to_ref(mpmgpu_handle* h, double* const* arr, int comps, int width, double* out, double fill) {
  const Geom& g = h->g;
  std::vector<uint8_t> act;
  TRY(download(h, act, h->was_active, (size_t)g.nblocks));
  for (int64_t i = 0; i < g.nnodes * width; i++) out[i] = 0.0;
  std::vector<double> tmp;
  for (int d = 0; d < comps; d++) {
    TRY(download(h, tmp, arr[d], (size_t)g.nslots));
    for (int k = 0; k < g.nn[2]; k++)
      for (int j = 0; j < g.nn[1]; j++)
        for (int i = 0; i < g.nn[0]; i++) {
          const int64_t id = i + (int64_t)g.nn[0] * (j + (int64_t)g.nn[1] * k);
          const bool on = act[(size_t)node_block(g, i, j, k)] != 0;
          out[id * width + d] = on ? tmp[(size_t)node_slot(g, i, j, k)] : fill;
        }
  }
  return MPMGPU_OK;
}

}  // namespace

extern "C" {

mpmgpu_status mpmgpu_download_nodes(mpmgpu_handle* h, int body, int field, double* out) {
  if (!h || !out || body < 0 || body >= (int)h->bodies.size()) return MPMGPU_ERR_ARG;
  TRY(mpmgpu_synchronize(h));
  BodyDev& B = h->bodies[(size_t)body];
  const int D = h->g.dim;
  const bool dbg = B.snap.m != nullptr;
  if (!h->primed) {
    for (int64_t i = 0; i < h->g.nnodes * (field == MPMGPU_N_M ? 1 : 3); i++) out[i] = 0.0;
    return MPMGPU_OK;
  }
  switch (field) {
    case MPMGPU_N_M:
      if (!dbg) return fail(h, MPMGPU_ERR_STATE, "nodal m is kept only with keep_debug");
      return nodes_to_ref(h, &B.snap.m, 1, 1, out, 0.0);
    case MPMGPU_N_MX_T:
      if (!dbg) return fail(h, MPMGPU_ERR_STATE, "nodal mx_t is kept only with keep_debug");
      return nodes_to_ref(h, B.snap.mx, D, 3, out, 0.0);
    case MPMGPU_N_F:
      if (!dbg) return fail(h, MPMGPU_ERR_STATE, "nodal f is kept only with keep_debug");
      return nodes_to_ref(h, B.snap.f, D, 3, out, 0.0);
    case MPMGPU_N_X_T: return nodes_to_ref(h, B.V.vt, D, 3, out, 0.0);
    case MPMGPU_N_DIFF_X_T: return nodes_to_ref(h, B.V.dv, D, 3, out, 0.0);
    case MPMGPU_N_U: {
      TRY(nodes_to_ref(h, B.V.vt, D, 3, out, 0.0));
      // moveGrid: u = dt * x_t (explicit_usl.cpp:252)
      for (int64_t i = 0; i < 3 * h->g.nnodes; i++) out[i] = h->sp.dt * out[i];
      return MPMGPU_OK;
    }
  }
  return fail(h, MPMGPU_ERR_ARG, "unknown node field");
}

mpmgpu_status mpmgpu_download_contact(mpmgpu_handle* h, int contact, int field, double* out) {
  if (!h || !out || contact < 0 || contact >= h->cs.nc) return MPMGPU_ERR_ARG;
  if (!h->cfg.keep_debug) return fail(h, MPMGPU_ERR_STATE, "contact fields are kept only with keep_debug");
  if (field != MPMGPU_C_NORMAL && field != MPMGPU_C_FORCE) return fail(h, MPMGPU_ERR_ARG, "unknown contact field");
  TRY(mpmgpu_synchronize(h));
  const Geom& g = h->g;
  double* src = (field == MPMGPU_C_NORMAL) ? h->cs.normal_out[contact] : h->cs.force_out[contact];
  std::vector<double> tmp;
  TRY(download(h, tmp, src, 3 * (size_t)g.nslots));
  std::vector<uint8_t> act;
  TRY(download(h, act, h->was_active, (size_t)g.nblocks));
  const double nan = std::nan("");
  for (int k = 0; k < g.nn[2]; k++)
    for (int j = 0; j < g.nn[1]; j++)
      for (int i = 0; i < g.nn[0]; i++) {
        const int64_t id = i + (int64_t)g.nn[0] * (j + (int64_t)g.nn[1] * k);
        const int64_t s = node_slot(g, i, j, k);
        const bool on = h->primed && act[(size_t)node_block(g, i, j, k)] != 0;
        for (int d = 0; d < 3; d++) {
          double v = tmp[(size_t)(3 * s + d)];
          // the reference normalises every node's normal; a zero normal gives 0 * (1/0)
          if (!on) v = (field == MPMGPU_C_NORMAL) ? (d < g.dim ? nan : 0.0) : 0.0;
          out[3 * id + d] = v;
        }
      }
  return MPMGPU_OK;
}

mpmgpu_status mpmgpu_dump_map(mpmgpu_handle* h, int body, int32_t* node, int32_t* point, double* s_val, double* grad,
                              int64_t* count) {
  if (!h || !count || body < 0 || body >= (int)h->bodies.size()) return MPMGPU_ERR_ARG;
  BodyDev& B = h->bodies[(size_t)body];
  const int cp = h->g.cp;
  const size_t slots = (size_t)B.n * cp * cp;
  int32_t* dnode = nullptr;
  double *ds = nullptr, *dg = nullptr;
  CUDA_TRY(h, cudaMalloc(&dnode, std::max<size_t>(slots, 1) * sizeof(int32_t)));
  CUDA_TRY(h, cudaMalloc(&ds, std::max<size_t>(slots, 1) * sizeof(double)));
  CUDA_TRY(h, cudaMalloc(&dg, std::max<size_t>(slots, 1) * 3 * sizeof(double)));
  if (B.n > 0) {
    if (h->g.dim == 3)
      k_export_map<3><<<grid_blocks(h, B.n, 128), 128, 0, h->stream>>>(h->g, h->sp.cpdi, B.P, dnode, ds, dg);
    else
      k_export_map<2><<<grid_blocks(h, B.n, 128), 128, 0, h->stream>>>(h->g, h->sp.cpdi, B.P, dnode, ds, dg);
  }
  mpmgpu_status st = check_launch(h, "k_export_map");
  std::vector<int32_t> hn(slots);
  std::vector<double> hs(slots), hg(3 * slots);
  if (st == MPMGPU_OK && slots > 0) {
    cudaError_t e = cudaMemcpyAsync(hn.data(), dnode, slots * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hs.data(), ds, slots * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hg.data(), dg, 3 * slots * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) st = fail(h, MPMGPU_ERR_CUDA, std::string("dump_map copy: ") + cudaGetErrorString(e));
  }
  cudaFree(dnode);
  cudaFree(ds);
  cudaFree(dg);
  if (st != MPMGPU_OK) return st;
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
  if (!h) return MPMGPU_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int s = 0; s < mpmgpu_handle::kStages; s++)
    for (auto& pr : h->pending[s]) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  for (cudaEvent_t e : h->event_pool) cudaEventDestroy(e);
  for (void* p : h->allocs) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return MPMGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free map export (mpmgpu_dump_map_noalloc).
//
// For callers that must not allocate device memory when they read the map
// (graph capture, caller-owned memory pools, real-time loops): the slot
// buffers that mpmgpu_dump_map takes from cudaMalloc live here in one static
// device array, and the compaction to the reference's triplet order runs on
// the device into the caller's arrays. Nothing is allocated on the host or
// the device by the call.
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

// Device address of the scratch array on `device`, looked up once per device
// with that device current (in host code the symbol is only a stand-in).
mpmgpu_status noalloc_scratch(mpmgpu_handle* h, int device, unsigned char** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return fail(h, MPMGPU_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_base[device] == nullptr) {
    int current = 0;
    CUDA_TRY(h, cudaGetDevice(&current));
    if (current != device) CUDA_TRY(h, cudaSetDevice(device));
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (current != device) CUDA_TRY(h, cudaSetDevice(current));
    if (e != cudaSuccess)
      return fail(h, MPMGPU_ERR_CUDA, std::string("cudaGetSymbolAddress(map scratch): ") + cudaGetErrorString(e));
    g_noalloc_base[device] = static_cast<unsigned char*>(p);
  }
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
  if (!h || !count || body < 0 || body >= (int)h->bodies.size()) return MPMGPU_ERR_ARG;
  if (capacity < 0 || (capacity > 0 && (!d_node || !d_point || !d_s || !d_grad)))
    return fail(h, MPMGPU_ERR_ARG, "output arrays missing");
  BodyDev& B = h->bodies[(size_t)body];
  const int per_point = h->g.cp * h->g.cp;
  const int64_t nslots = B.n * per_point;
  if (nslots > kNoAllocSlots)
    return fail(h, MPMGPU_ERR_ARG,
                "mpmgpu_dump_map_noalloc: body has " + std::to_string(B.n) + " points x " + std::to_string(per_point) +
                    " triplet slots = " + std::to_string(nslots) + " slots, above the static scratch limit of " +
                    std::to_string(kNoAllocSlots));
  unsigned char* base = nullptr;
  TRY(noalloc_scratch(h, h->cfg.device, &base));
  int32_t* node = reinterpret_cast<int32_t*>(base + kNoAllocOffNode);
  int32_t* pos = reinterpret_cast<int32_t*>(base + kNoAllocOffPos);
  int32_t* blk = reinterpret_cast<int32_t*>(base + kNoAllocOffBlk);
  double* s = reinterpret_cast<double*>(base + kNoAllocOffS);
  double* grad = reinterpret_cast<double*>(base + kNoAllocOffGrad);
  cudaStream_t st = h->stream;
  // every slot read below is written first by this call: nothing carries over
  if (B.n > 0) {
    if (h->g.dim == 3)
      k_export_map<3><<<grid_blocks(h, B.n, 128), 128, 0, st>>>(h->g, h->sp.cpdi, B.P, node, s, grad);
    else
      k_export_map<2><<<grid_blocks(h, B.n, 128), 128, 0, st>>>(h->g, h->sp.cpdi, B.P, node, s, grad);
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
  if (total > capacity) return fail(h, MPMGPU_ERR_ARG, "capacity below the triplet count");
  return MPMGPU_OK;
}
