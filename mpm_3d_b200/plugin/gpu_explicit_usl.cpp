// GPUExplicitUSL: mpm_3d Solver plugin over the C ABI of include/mpm_b200.h.
// Compiled together with the reference's sources (registered as
// REGISTER(Solver, GPUExplicitUSL)); it uses only the reference's public
// object interface.
#include "gpu_explicit_usl.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <iostream>
#include <thread>
#include <vector>

#include "objects/bodies/bodies.hpp"
#include "objects/boundaries/boundaries.hpp"
#include "objects/contacts/contacts.hpp"
#include "objects/grids/grids.hpp"
#include "objects/materials/materials.hpp"
#include "objects/points/points.hpp"

namespace {

[[noreturn]] void unsupported(const std::string& what) {
  std::cerr << "GPUExplicitUSL: " << what << std::endl;
  exit(0);
}

}  // namespace

GPUExplicitUSL::~GPUExplicitUSL() {
  if (handle) mpmgpu_destroy(handle);
}

void GPUExplicitUSL::check(mpmgpu_status s, const char* what) {
  if (s == MPMGPU_OK) return;
  std::cerr << "GPUExplicitUSL: " << what << ": " << mpmgpu_status_string(s) << " ("
            << mpmgpu_last_error(handle) << ")" << std::endl;
  exit(0);
}

// explicit_usl.cpp:25-44, plus the optional write-back interval and form
// (0 FP64, 1 deterministic FP64, 2 mixed FP32/FP64; mpmgpu_mode).
void GPUExplicitUSL::init(Job* job) {
  if (int_props.size() >= 1) cpdi_spec = int_props[0];
  if (int_props.size() >= 2) contact_spec = int_props[1];
  if (int_props.size() >= 3) writeback_interval = int_props[2];
  if (int_props.size() >= 4) mode = int_props[3];
  if (int_props.size() >= 5) overlap = int_props[4];
  if (mode < 0 || mode > 2) {
    std::cerr << "GPUExplicitUSL: form " << mode << " is not 0 (FP64), 1 (deterministic) or 2 (mixed)." << std::endl;
    exit(0);
  }
  printf("Solver properties (cpdi_spec = %i, contact_spec = %i, writeback = %i, form = %i, overlap = %i).\n",
         cpdi_spec, contact_spec, writeback_interval, mode, overlap);
  std::cout << "Solver Initialized." << std::endl;
}

// Device set-up on the first step: Job::init runs solver->init before the
// grid and bodies exist (job.hpp:90-102).
void GPUExplicitUSL::setUp(Job* job) {
  CartesianLinear* grid = dynamic_cast<CartesianLinear*>(job->grid.get());
  if (!grid) unsupported("grid class " + job->grid->object_name + " (CartesianLinear only)");
  if (job->JOB_TYPE != Job::JOB_2D && job->JOB_TYPE != Job::JOB_3D)
    unsupported("job TYPE " + std::to_string(job->JOB_TYPE) + " (2 or 3 only)");
  const int dim = job->grid->GRID_DIM;
  mpmgpu_config cfg = {};
  cfg.dim = dim;
  for (int d = 0; d < dim; d++) {
    cfg.L[d] = grid->Lx(d);
    cfg.N[d] = grid->Nx(d);
  }
  cfg.dt = job->dt;
  cfg.cpdi_spec = cpdi_spec;
  cfg.contact_spec = contact_spec;
  cfg.mode = mode;
  cfg.device = 0;
  cfg.keep_debug = 1;  // node and contact fields are written in frames
  cfg.sort_interval = 0;
  check(mpmgpu_create(&cfg, &handle), "mpmgpu_create");

  gpu_body.assign(job->bodies.size(), -1);
  for (size_t b = 0; b < job->bodies.size(); b++) {
    if (job->activeBodies[b] == 0) continue;
    Body* body = job->bodies[b].get();
    if (!dynamic_cast<DefaultPoints*>(body->points.get()))
      unsupported("point class " + body->points->object_name + " (DefaultPoints only)");
    Points* pts = body->points.get();
    const int n = pts->x.size();
    std::vector<double> x(3 * (size_t)n), xt(3 * (size_t)n), u(3 * (size_t)n), T(9 * (size_t)n);
    std::vector<int32_t> active((size_t)n);
    for (int i = 0; i < n; i++) {
      for (int j = 0; j < 3; j++) {
        x[3 * i + j] = pts->x(i, j);
        xt[3 * i + j] = pts->x_t(i, j);
        u[3 * i + j] = pts->u(i, j);
      }
      for (int k = 0; k < 9; k++) T[9 * i + k] = pts->T[i][k];
      active[i] = pts->active(i);
    }
    mpmgpu_body_desc desc = {};
    desc.n = n;
    desc.m = pts->m.data();
    desc.v = pts->v.data();
    desc.x = x.data();
    desc.x_t = xt.data();
    desc.active = active.data();
    desc.u = u.data();
    desc.T = T.data();
    if (body->activeMaterial) {
      desc.has_material = 1;
      if (Sand_SachithLocal* sand = dynamic_cast<Sand_SachithLocal*>(body->material.get())) {
        // the properties as Sand_SachithLocal::init resolved them
        // (sand_sachithlocal.cpp:57-103)
        desc.material_kind = 2;
        desc.E = sand->E;
        desc.nu = sand->nu;
        const double props[6] = {sand->grains_d, sand->MU_S, sand->GRAINS_RHO,
                                 sand->RHO_CRITICAL, sand->MU_2, sand->I_0};
        for (int k = 0; k < 6; k++) desc.material_props[k] = props[k];
        desc.material_flags = sand->use_density_to_determine_pressure ? 1 : 0;
      } else {
        IsotropicLinearElasticity* mat = dynamic_cast<IsotropicLinearElasticity*>(body->material.get());
        if (!mat) unsupported("material class " + body->material->object_name);
        // CompressibleNeohookeanElasticity derives from IsotropicLinearElasticity
        desc.material_kind = dynamic_cast<CompressibleNeohookeanElasticity*>(mat) ? 1 : 0;
        desc.E = mat->E;
        desc.nu = mat->nu;
      }
    }
    if (body->activeBoundary) {
      Boundary* bc = body->boundary.get();
      if (dynamic_cast<CartesianBox*>(bc)) {
        desc.has_boundary = 1;
      } else if (dynamic_cast<CartesianSmoothBox*>(bc)) {
        desc.has_boundary = 2;
      } else if (CartesianFrictionalBox* fb = dynamic_cast<CartesianFrictionalBox*>(bc)) {
        desc.has_boundary = 3;
        desc.boundary_mu = fb->mu_f;   // set by CartesianFrictionalBox::init from boundary-props
      } else {
        unsupported("boundary class " + bc->object_name);
      }
    }
    int id = -1;
    check(mpmgpu_add_body(handle, &desc, &id), "mpmgpu_add_body");
    gpu_body[b] = id;
  }
  for (size_t c = 0; c < job->contacts.size(); c++) {
    if (job->activeContacts[c] == 0) continue;
    ContactHuang* ch = dynamic_cast<ContactHuang*>(job->contacts[c].get());
    if (!ch) unsupported("contact class " + job->contacts[c]->object_name);
    const int b1 = gpu_body[ch->bodyIDs[0]], b2 = gpu_body[ch->bodyIDs[1]];
    if (b1 < 0 || b2 < 0) unsupported("contact between inactive bodies");
    // ContactHuang_ReflectedBoundary derives from ContactHuang and differs in its normal
    if (dynamic_cast<ContactHuang_ReflectedBoundary*>(ch))
      check(mpmgpu_add_contact_reflected(handle, b1, b2, ch->mu_f, nullptr), "mpmgpu_add_contact_reflected");
    else
      check(mpmgpu_add_contact(handle, b1, b2, ch->mu_f, nullptr), "mpmgpu_add_contact");
  }
  // the driver has applied gravity to every point before the loop
  // (default_driver.cpp:58-60): take it from the points
  for (size_t b = 0; b < job->bodies.size(); b++) {
    if (gpu_body[b] < 0 || job->bodies[b]->points->b.size() == 0) continue;
    for (int d = 0; d < 3; d++) gravity[d] = job->bodies[b]->points->b(0, d);
    break;
  }
  check(mpmgpu_set_gravity(handle, 1, gravity), "mpmgpu_set_gravity");
  const std::string& sname = job->serializer->object_name;
  if ((sname == "DefaultVTK" || sname == "MinimalVTK" || sname == "AsyncVTK") && !job->serializer->fp64_props.empty())
    sample_rate = job->serializer->fp64_props[0];
}

// DefaultVTK::writeFrame writes when (t - t0) >= frames / rate or on its
// first call (default_vtk.cpp:121-124); the driver calls it right after
// step() with the same t (default_driver.cpp:65-80).
bool GPUExplicitUSL::frameDue(Job* job) {
  if (writeback_interval > 0) return steps % writeback_interval == 0;
  if (!(sample_rate > 0)) return true;
  if ((job->t - job->t0) >= (frames / sample_rate) || frames == 0) {
    frames++;
    return true;
  }
  return false;
}

// ExplicitUSL::step (explicit_usl.cpp:48-87) on the GPU.
void GPUExplicitUSL::step(Job* job) {
  if (!handle) setUp(job);
  if (queued_ahead)
    queued_ahead = false;   // queued behind the last frame's copies
  else
    check(mpmgpu_step(handle, 1), "mpmgpu_step");
  steps++;
  // explicit_usl.cpp:80-81: the driver sets the next step's body force
  job->driver->generateGravity(job);
  job->driver->applyGravity(job);
  for (size_t b = 0; b < job->bodies.size(); b++) {
    if (gpu_body[b] < 0 || job->bodies[b]->points->b.size() == 0) continue;
    double g[3];
    for (int d = 0; d < 3; d++) g[d] = job->bodies[b]->points->b(0, d);
    if (g[0] != gravity[0] || g[1] != gravity[1] || g[2] != gravity[2]) {
      for (int d = 0; d < 3; d++) gravity[d] = g[d];
      check(mpmgpu_set_gravity(handle, 1, gravity), "mpmgpu_set_gravity");
    }
    break;
  }
  if (frameDue(job)) writeBack(job);
}

namespace {

// Runs the tasks on up to `threads` host threads.
void run_tasks(std::vector<std::function<void()>>& tasks, unsigned threads) {
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    for (size_t k = next++; k < tasks.size(); k = next++) tasks[k]();
  };
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < threads && t < tasks.size(); t++) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
}

}  // namespace

// The host arrays the serializer reads at a frame (DefaultPoints::writeFrame,
// default_points.cpp:341-368; DefaultNodes::writeFrame,
// default_nodes.cpp:68-82; ContactHuang's contact arrays,
// contact_huang.cpp:202-206). The device writes every field in the
// reference's layout and order into one buffer and copies it to pinned host
// memory behind the step that just ran; with overlap on, the driver's next
// step is queued behind the copies (DefaultDriver::run calls step, then
// writeFrame, then advances t, default_driver.cpp:62-83, so that step comes
// next; its gravity is already set). The fields are then copied straight
// into the reference arrays' buffers (3 doubles per vector, 9 per tensor,
// mpm_vectorarray.hpp:29, mpm_tensorarray.hpp:31) on host threads while the
// GPU runs that step.
void GPUExplicitUSL::writeBack(Job* job) {
  check(mpmgpu_frame_begin(handle), "mpmgpu_frame_begin");
  if (overlap) {
    check(mpmgpu_step(handle, 1), "mpmgpu_step");
    queued_ahead = true;
  }
  std::vector<std::function<void()>> tasks;
  std::vector<std::vector<double>> bufs;   // fields whose reference storage is not double
  bool waited = false;
  // the first copy waits for the frame; the rest run in parallel
  auto add = [&](std::function<void()> run) {
    if (!waited) {
      run();
      waited = true;
    } else {
      tasks.push_back(std::move(run));
    }
  };
  auto point_field = [&](int id, int field, double* dst) {
    add([this, id, field, dst]() { check(mpmgpu_frame_points(handle, id, field, dst), "mpmgpu_frame_points"); });
  };
  auto node_field = [&](int id, int field, double* dst) {
    add([this, id, field, dst]() { check(mpmgpu_frame_nodes(handle, id, field, dst), "mpmgpu_frame_nodes"); });
  };
  for (size_t bi = 0; bi < job->bodies.size(); bi++) {
    const int id = gpu_body[bi];
    if (id < 0) continue;
    Points* pts = job->bodies[bi]->points.get();
    Nodes* nds = job->bodies[bi]->nodes.get();
    const int n = pts->x.size();
    point_field(id, MPMGPU_P_X, pts->x.data());
    point_field(id, MPMGPU_P_U, pts->u.data());
    point_field(id, MPMGPU_P_X_T, pts->x_t.data());
    point_field(id, MPMGPU_P_MX_T, pts->mx_t.data());
    // the velocity gradient is kept on the device in the FP64 forms only
    if (mode != MPMGPU_MODE_MIXED) point_field(id, MPMGPU_P_L, pts->L.data());
    point_field(id, MPMGPU_P_T, pts->T.data());
    point_field(id, MPMGPU_P_V, pts->v.data());
    bufs.emplace_back((size_t)n);
    double* ab = bufs.back().data();
    add([this, id, n, ab, pts]() {
      check(mpmgpu_frame_points(handle, id, MPMGPU_P_ACTIVE, ab), "mpmgpu_frame_points");
      for (int i = 0; i < n; i++) pts->active(i) = (int)ab[i];
    });
    Sand_SachithLocal* sand = job->bodies[bi]->activeMaterial
                                  ? dynamic_cast<Sand_SachithLocal*>(job->bodies[bi]->material.get())
                                  : nullptr;
    if (sand) {
      // the material's frame fields (Sand_SachithLocal::writeFrame)
      point_field(id, MPMGPU_P_GAMMAP, sand->gammap.data());
      point_field(id, MPMGPU_P_GAMMAP_DOT, sand->gammap_dot.data());
    }
    node_field(id, MPMGPU_N_M, nds->m.data());
    node_field(id, MPMGPU_N_MX_T, nds->mx_t.data());
    node_field(id, MPMGPU_N_F, nds->f.data());
    node_field(id, MPMGPU_N_X_T, nds->x_t.data());
    node_field(id, MPMGPU_N_U, nds->u.data());
    node_field(id, MPMGPU_N_DIFF_X_T, nds->diff_x_t.data());
  }
  int gc = 0;
  for (size_t c = 0; c < job->contacts.size(); c++) {
    if (job->activeContacts[c] == 0) continue;
    ContactHuang* ch = dynamic_cast<ContactHuang*>(job->contacts[c].get());
    double* nrm = ch->contact_normal.data();
    double* frc = ch->contact_force.data();
    add([this, gc, nrm]() { check(mpmgpu_frame_contact(handle, gc, MPMGPU_C_NORMAL, nrm), "mpmgpu_frame_contact"); });
    add([this, gc, frc]() { check(mpmgpu_frame_contact(handle, gc, MPMGPU_C_FORCE, frc), "mpmgpu_frame_contact"); });
    gc++;
  }
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  run_tasks(tasks, std::min(hw, 8u));
}

// As ExplicitUSL (explicit_usl.cpp:91-99): not implemented in the reference.
std::string GPUExplicitUSL::saveState(Job* job, Serializer* serializer, std::string filepath) { return "err"; }
int GPUExplicitUSL::loadState(Job* job, Serializer* serializer, std::string fullpath) { return 0; }
