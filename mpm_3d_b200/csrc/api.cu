// Host side of the C ABI declared in include/mpm_b200.h.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "kernels_fp64.cuh"

using namespace mpmb200;

namespace {

struct BodyDev {
  int64_t n = 0;
  PointsDev P{};
  NodesAcc A{};
  NodesVel V{};
  MaterialParams mat{};
  int has_boundary = 0;
  bool needs_normal = false;
};

}  // namespace

struct mpmgpu_handle {
  mpmgpu_config cfg{};
  Geom g{};
  StepParams sp{};
  cudaStream_t stream = nullptr;
  std::vector<BodyDev> bodies;
  ContactSet cs{};
  uint32_t* flags = nullptr;
  int64_t* list = nullptr;
  unsigned long long* count = nullptr;
  uint8_t* was_active = nullptr;
  int* err = nullptr;
  std::vector<void*> allocs;
  std::string last_error;
  int64_t launches = 0;
  int sm_count = 148;
  bool stepped = false;
};

namespace {

mpmgpu_status fail(mpmgpu_handle* h, mpmgpu_status s, const std::string& msg) {
  if (h) h->last_error = msg;
  return s;
}

#define CUDA_TRY(h, expr)                                                                               \
  do {                                                                                                  \
    cudaError_t e_ = (expr);                                                                            \
    if (e_ != cudaSuccess) return fail((h), MPMGPU_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
mpmgpu_status dev_alloc(mpmgpu_handle* h, T** p, size_t count, bool zero = true) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 1);
  if (e != cudaSuccess) return fail(h, MPMGPU_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  h->allocs.push_back(q);
  if (zero) {
    e = cudaMemsetAsync(q, 0, count * sizeof(T), h->stream);
    if (e != cudaSuccess) return fail(h, MPMGPU_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
  }
  *p = static_cast<T*>(q);
  return MPMGPU_OK;
}

#define TRY(expr)                       \
  do {                                  \
    mpmgpu_status s_ = (expr);          \
    if (s_ != MPMGPU_OK) return s_;     \
  } while (0)

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

// Host copy of a strided upload: column d of an AoS array of width w.
std::vector<double> column(const double* aos, int64_t n, int w, int d) {
  std::vector<double> out((size_t)n);
  for (int64_t i = 0; i < n; i++) out[(size_t)i] = aos[i * w + d];
  return out;
}

mpmgpu_status upload(mpmgpu_handle* h, double* dst, const std::vector<double>& src) {
  CUDA_TRY(h, cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return MPMGPU_OK;
}

mpmgpu_status download(mpmgpu_handle* h, std::vector<double>& dst, const double* src, size_t n) {
  dst.resize(n);
  CUDA_TRY(h, cudaMemcpyAsync(dst.data(), src, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
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
  for (int d = 0; d < cfg->dim; d++)
    if (cfg->N[d] < 1 || !(cfg->L[d] > 0)) return MPMGPU_ERR_ARG;
  mpmgpu_handle* h = new mpmgpu_handle();
  h->cfg = *cfg;
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
    } else {
      g.L[d] = 0.0;
      g.N[d] = 0;
      g.h[d] = 0.0;
      g.nn[d] = 1;
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
  h->sp.dt = cfg->dt;
  h->sp.cpdi = cfg->cpdi_spec;
  h->sp.contact_spec = cfg->contact_spec;
  h->sp.keep_debug = cfg->keep_debug;
  // DefaultDriver gravity until set otherwise (default_driver.cpp:90-105)
  h->sp.grav[0] = h->sp.grav[1] = h->sp.grav[2] = 0.0;
  h->sp.grav[cfg->dim == 2 ? 1 : 2] = -9.81;
  mpmgpu_status s = MPMGPU_OK;
  if ((s = dev_alloc(h, &h->flags, (size_t)g.nblocks)) != MPMGPU_OK ||
      (s = dev_alloc(h, &h->list, (size_t)g.nblocks)) != MPMGPU_OK ||
      (s = dev_alloc(h, &h->count, 1)) != MPMGPU_OK || (s = dev_alloc(h, &h->was_active, (size_t)g.nblocks)) != MPMGPU_OK ||
      (s = dev_alloc(h, &h->err, 1)) != MPMGPU_OK) {
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
  if (desc->n < 0 || (desc->n > 0 && (!desc->m || !desc->v || !desc->x || !desc->x_t)))
    return fail(h, MPMGPU_ERR_ARG, "body arrays missing");
  const int D = h->g.dim;
  const int64_t n = desc->n;
  BodyDev B;
  B.n = n;
  B.P.n = n;
  for (int d = 0; d < 3; d++) {
    TRY(dev_alloc(h, &B.P.x[d], (size_t)n));
    TRY(dev_alloc(h, &B.P.v[d], (size_t)n));
    TRY(dev_alloc(h, &B.P.u[d], (size_t)n));
  }
  for (int c = 0; c < 6; c++) TRY(dev_alloc(h, &B.P.s[c], (size_t)n));
  TRY(dev_alloc(h, &B.P.vol, (size_t)n));
  TRY(dev_alloc(h, &B.P.m, (size_t)n));
  TRY(dev_alloc(h, &B.P.ext, (size_t)n));
  TRY(dev_alloc(h, &B.P.active, (size_t)n));
  B.P.L = nullptr;
  if (h->cfg.keep_debug) TRY(dev_alloc(h, &B.P.L, (size_t)n * 9));
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
    std::vector<int32_t> act((size_t)n, 1);
    if (desc->active)
      for (int64_t i = 0; i < n; i++) act[(size_t)i] = desc->active[i] != 0 ? 1 : 0;
    CUDA_TRY(h, cudaMemcpyAsync(B.P.active, act.data(), act.size() * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
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

}  // extern "C"

namespace {

template <int DIM>
mpmgpu_status step_once(mpmgpu_handle* h) {
  const Geom& g = h->g;
  cudaStream_t st = h->stream;
  GridBodies GB{};
  GB.nb = (int)h->bodies.size();
  if (h->cfg.keep_debug) {
    // Debug form: nodal arrays are zeroed in full each step so downloads of
    // untouched nodes read zero, as the reference's full-grid arrays do.
    const size_t bytes = (size_t)g.nslots * sizeof(double);
    for (BodyDev& B : h->bodies) {
      CUDA_TRY(h, cudaMemsetAsync(B.A.m, 0, bytes, st));
      for (int d = 0; d < 3; d++) {
        CUDA_TRY(h, cudaMemsetAsync(B.A.mx[d], 0, bytes, st));
        CUDA_TRY(h, cudaMemsetAsync(B.A.f[d], 0, bytes, st));
        CUDA_TRY(h, cudaMemsetAsync(B.V.vt[d], 0, bytes, st));
        CUDA_TRY(h, cudaMemsetAsync(B.V.dv[d], 0, bytes, st));
        if (B.A.nrm[d]) CUDA_TRY(h, cudaMemsetAsync(B.A.nrm[d], 0, bytes, st));
      }
    }
    for (int c = 0; c < h->cs.nc; c++) {
      CUDA_TRY(h, cudaMemsetAsync(h->cs.force_out[c], 0, 3 * bytes, st));
      // untouched nodes have a 0/0 normal in the reference (contact_huang.cpp:93-96)
    }
  }
  for (size_t b = 0; b < h->bodies.size(); b++) {
    BodyDev& B = h->bodies[b];
    GB.acc[b] = B.A;
    GB.vel[b] = B.V;
    GB.has_boundary[b] = B.has_boundary;
    if (B.n == 0) continue;
    k_p2g<DIM><<<grid_blocks(h, B.n, 256), 256, 0, st>>>(g, h->sp, B.P, B.A, h->flags, h->err);
    TRY(check_launch(h, "k_p2g"));
  }
  CUDA_TRY(h, cudaMemsetAsync(h->count, 0, sizeof(unsigned long long), st));
  k_compact<<<grid_blocks(h, g.nblocks, 256), 256, 0, st>>>(g.nblocks, h->flags, h->list, h->count, h->was_active);
  TRY(check_launch(h, "k_compact"));
  const int gb = (int)std::min<int64_t>(g.nblocks, (int64_t)h->sm_count * 32);
  k_grid<DIM><<<gb, 64, 0, st>>>(g, h->sp, GB, h->cs, h->list, h->count);
  TRY(check_launch(h, "k_grid"));
  for (size_t b = 0; b < h->bodies.size(); b++) {
    BodyDev& B = h->bodies[b];
    if (B.n == 0) continue;
    k_g2p<DIM><<<grid_blocks(h, B.n, 256), 256, 0, st>>>(g, h->sp, B.P, B.V, B.mat, h->err);
    TRY(check_launch(h, "k_g2p"));
  }
  return MPMGPU_OK;
}

}  // namespace

extern "C" {

mpmgpu_status mpmgpu_step(mpmgpu_handle* h, int nsteps) {
  if (!h || nsteps < 0) return MPMGPU_ERR_ARG;
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

mpmgpu_status mpmgpu_download_points(mpmgpu_handle* h, int body, int field, double* out) {
  if (!h || !out || body < 0 || body >= (int)h->bodies.size()) return MPMGPU_ERR_ARG;
  TRY(mpmgpu_synchronize(h));
  BodyDev& B = h->bodies[(size_t)body];
  const int64_t n = B.n;
  const int D = h->g.dim;
  std::vector<double> tmp;
  auto vec3 = [&](double* const* arr) -> mpmgpu_status {
    for (int64_t i = 0; i < 3 * n; i++) out[i] = 0.0;
    for (int d = 0; d < D; d++) {
      TRY(download(h, tmp, arr[d], (size_t)n));
      for (int64_t i = 0; i < n; i++) out[3 * i + d] = tmp[(size_t)i];
    }
    return MPMGPU_OK;
  };
  auto scal = [&](const double* arr) -> mpmgpu_status {
    TRY(download(h, tmp, arr, (size_t)n));
    std::memcpy(out, tmp.data(), sizeof(double) * (size_t)n);
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
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < D; d++) out[3 * i + d] = m[(size_t)i] * out[3 * i + d];
      return MPMGPU_OK;
    }
    case MPMGPU_P_B:
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) out[3 * i + d] = h->sp.grav[d];
      return MPMGPU_OK;
    case MPMGPU_P_L:
      if (!B.P.L) return fail(h, MPMGPU_ERR_STATE, "L is kept only with keep_debug");
      TRY(download(h, tmp, B.P.L, (size_t)n * 9));
      std::memcpy(out, tmp.data(), sizeof(double) * 9 * (size_t)n);
      return MPMGPU_OK;
    case MPMGPU_P_T: {
      static const int idx[9] = {0, 3, 5, 3, 1, 4, 5, 4, 2};
      std::vector<std::vector<double>> s(6);
      for (int c = 0; c < 6; c++) TRY(download(h, s[(size_t)c], B.P.s[c], (size_t)n));
      for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 9; k++) out[9 * i + k] = s[(size_t)idx[k]][(size_t)i];
      return MPMGPU_OK;
    }
    case MPMGPU_P_M: return scal(B.P.m);
    case MPMGPU_P_V: return scal(B.P.vol);
    case MPMGPU_P_EXTENT: return scal(B.P.ext);
    case MPMGPU_P_ACTIVE: {
      std::vector<int32_t> a((size_t)n);
      CUDA_TRY(h, cudaMemcpy(a.data(), B.P.active, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < n; i++) out[i] = a[(size_t)i];
      return MPMGPU_OK;
    }
  }
  return fail(h, MPMGPU_ERR_ARG, "unknown point field");
}

}  // extern "C"

namespace {

// Copies a block-linear nodal array (width-component SoA) to reference node
// order; nodes of blocks that were not active in the last step read zero.
mpmgpu_status nodes_to_ref(mpmgpu_handle* h, double* const* arr, int comps, int width, double* out, bool mask_inactive,
                           double fill) {
  const Geom& g = h->g;
  std::vector<uint8_t> act((size_t)g.nblocks, 1);
  if (mask_inactive) CUDA_TRY(h, cudaMemcpy(act.data(), h->was_active, (size_t)g.nblocks, cudaMemcpyDeviceToHost));
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
  const bool dbg = h->cfg.keep_debug != 0;
  switch (field) {
    case MPMGPU_N_M:
      if (!dbg) return fail(h, MPMGPU_ERR_STATE, "nodal m is kept only with keep_debug");
      return nodes_to_ref(h, &B.A.m, 1, 1, out, false, 0.0);
    case MPMGPU_N_MX_T:
      if (!dbg) return fail(h, MPMGPU_ERR_STATE, "nodal mx_t is kept only with keep_debug");
      return nodes_to_ref(h, B.A.mx, D, 3, out, false, 0.0);
    case MPMGPU_N_F:
      if (!dbg) return fail(h, MPMGPU_ERR_STATE, "nodal f is kept only with keep_debug");
      return nodes_to_ref(h, B.A.f, D, 3, out, false, 0.0);
    case MPMGPU_N_X_T: return nodes_to_ref(h, B.V.vt, D, 3, out, !dbg, 0.0);
    case MPMGPU_N_DIFF_X_T: return nodes_to_ref(h, B.V.dv, D, 3, out, !dbg, 0.0);
    case MPMGPU_N_U: {
      TRY(nodes_to_ref(h, B.V.vt, D, 3, out, !dbg, 0.0));
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
  TRY(mpmgpu_synchronize(h));
  const Geom& g = h->g;
  double* src = (field == MPMGPU_C_NORMAL) ? h->cs.normal_out[contact] : h->cs.force_out[contact];
  if (field != MPMGPU_C_NORMAL && field != MPMGPU_C_FORCE) return fail(h, MPMGPU_ERR_ARG, "unknown contact field");
  std::vector<double> tmp;
  TRY(download(h, tmp, src, 3 * (size_t)g.nslots));
  std::vector<uint8_t> act((size_t)g.nblocks, 1);
  CUDA_TRY(h, cudaMemcpy(act.data(), h->was_active, (size_t)g.nblocks, cudaMemcpyDeviceToHost));
  const double nan = std::nan("");
  for (int k = 0; k < g.nn[2]; k++)
    for (int j = 0; j < g.nn[1]; j++)
      for (int i = 0; i < g.nn[0]; i++) {
        const int64_t id = i + (int64_t)g.nn[0] * (j + (int64_t)g.nn[1] * k);
        const int64_t s = node_slot(g, i, j, k);
        const bool on = act[(size_t)node_block(g, i, j, k)] != 0;
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
  for (void* p : h->allocs) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return MPMGPU_OK;
}

}  // extern "C"
