// Harness around the reference solver's own hot-path sources (mpm_3d, compiled
// unmodified from their original location by oracle/Makefile).
//
// TEST INFRASTRUCTURE ONLY: this file is the CPU oracle's driver. It is linked
// only into oracle/_ref/libmpmref_*.so, which only tests, smoke() and the
// CPU-baseline / reference arm of bench.py load. Nothing in the product
// (mpm_3d_b200/) links or calls it.
//
// What it provides:
//   * Registry<T>::Registry() for all ten registries that Configurator builds
//     (include/config.hpp:23-32), restricted to the hot-path classes. The
//     reference's src/registry/registry.cpp cannot be compiled here: it pulls
//     in the FVM stack and Eigen's sparse/dense solvers.
//   * HarnessDriver: generateGravity/applyGravity restated from
//     src/objects/drivers/default_driver.cpp:90-119 (DefaultDriver) and the
//     gravity vector of src/objects/drivers/user_def_gravity_driver.cpp:24-45
//     (UserDefinedGravityDriver). drivers.hpp cannot be included because it
//     needs Eigen::SelfAdjointEigenSolver (drivers.hpp:186). The time loop of
//     DefaultDriver::run (default_driver.cpp:46-86) is replaced by ref_step(),
//     which runs an exact number of steps.
//   * NullSerializer: registered under the serializer class names so configs
//     that name DefaultVTK parse; it writes nothing (frames are read back with
//     the ref_get_* functions instead).
//   * A C ABI (ref_*) for ctypes: build a Job from a .cfg file with the
//     reference's own Configurator (src/config/config.cpp:176-213) and
//     Job::init (include/job.hpp:76-105), step it, and read every particle and
//     node field plus the per-body S / gradS triplet lists.
#include <cstring>
#include <string>
#include <unistd.h>
#include <vector>

#include "config.hpp"
#include "job.hpp"
#include "mpm_objects.hpp"
#include "registry.hpp"

#include "objects/bodies/bodies.hpp"
#include "objects/boundaries/boundaries.hpp"
#include "objects/contacts/contacts.hpp"
#include "objects/grids/grids.hpp"
#include "objects/materials/materials.hpp"
#include "objects/nodes/nodes.hpp"
#include "objects/points/points.hpp"
#include "objects/serializers/serializers.hpp"
#include "objects/solvers/solvers.hpp"

#include "async_vtk.hpp"

#ifdef MPM_WITH_GPU_PLUGIN
// Drop-in check: the GPU solver plugin registered next to ExplicitUSL, as a
// maintainer would add it to src/registry/registry.cpp.
#include "gpu_explicit_usl.hpp"
#endif

namespace {

class NullSerializer : public Serializer {
 public:
  NullSerializer() { object_name = "NullSerializer"; }
  void init(Job*) override {}
  std::string saveState(Job*) override { return "err"; }
  int loadState(Job*, std::string) override { return 0; }
  int writeFrame(Job*) override { return 0; }
  void writeDefaultPointHeader(Job*, Body*, std::ofstream&, int) override {}
  void writeDefaultNodeHeader(Job*, Body*, std::ofstream&, int) override {}
  void writeScalarArray(Eigen::VectorXd&, std::string) override {}
  void writeVectorArray(MPMVectorArray&, std::string) override {}
  void writeTensorArray(MPMTensorArray&, std::string) override {}
};

// Gravity handling of DefaultDriver / UserDefinedGravityDriver.
class HarnessDriver : public Driver {
 public:
  explicit HarnessDriver(bool user_defined) : user_defined_(user_defined) {
    object_name = user_defined ? "UserDefinedGravityDriver" : "DefaultDriver";
  }
  double stop_time = 0.0;
  KinematicVector gravity;

  // default_driver.cpp:24-43 / user_def_gravity_driver.cpp:24-45
  void init(Job* job) override {
    stop_time = fp64_props.empty() ? 0.0 : fp64_props[0];
    gravity = KinematicVector(job->JOB_TYPE);
    if (user_defined_) {
      gravity.setZero();
      for (int pos = 0; pos < job->DIM && pos + 1 < (int)fp64_props.size(); pos++) {
        gravity(pos) = fp64_props[1 + pos];
      }
    }
  }
  std::string saveState(Job*, Serializer*, std::string) override { return "error"; }
  int loadState(Job*, Serializer*, std::string) override { return 0; }
  void run(Job*) override {}

  // default_driver.cpp:90-105 (DefaultDriver); UserDefinedGravityDriver keeps
  // the vector read at init.
  void generateGravity(Job* job) override {
    if (user_defined_) return;
    double g = -9.81;
    gravity.setZero();
    if (job->JOB_TYPE == Job::JOB_1D) {
      gravity(0) = g;
    } else if (job->JOB_TYPE == Job::JOB_2D) {
      gravity(1) = g;
    } else if (job->JOB_TYPE == Job::JOB_3D) {
      gravity(2) = g;
    } else if (job->JOB_TYPE == Job::JOB_AXISYM) {
      gravity(1) = g;
    } else if (job->JOB_TYPE == Job::JOB_2D_OOP) {
      gravity(1) = g;
    }
  }

  // default_driver.cpp:109-119
  void applyGravity(Job* job) override {
    for (int b = 0; b < (int)job->bodies.size(); b++) {
      if (job->activeBodies[b] == 0) continue;
      for (int i = 0; i < job->bodies[b]->points->b.size(); i++) {
        job->bodies[b]->points->b(i) = gravity;
      }
    }
  }

 private:
  bool user_defined_;
};

template <typename Base, typename Derived>
std::unique_ptr<Base> make() {
  return std::unique_ptr<Base>(new Derived);
}
std::unique_ptr<Driver> make_default_driver() { return std::unique_ptr<Driver>(new HarnessDriver(false)); }
std::unique_ptr<Driver> make_user_gravity_driver() { return std::unique_ptr<Driver>(new HarnessDriver(true)); }

}  // namespace

// Registries restricted to the hot path (the reference's full list is
// src/registry/registry.cpp:61-201).
template <>
Registry<Serializer>::Registry() {
  object["DefaultVTK"] = &make<Serializer, NullSerializer>;
  object["MinimalVTK"] = &make<Serializer, NullSerializer>;
  object["NullSerializer"] = &make<Serializer, NullSerializer>;
  // the reference's own DefaultVTK under a harness name (configs naming
  // DefaultVTK keep the null serializer, so tests write no frames unless
  // they ask), and the AsyncVTK plugin as a maintainer would register it
  object["ReferenceDefaultVTK"] = &make<Serializer, DefaultVTK>;
  object["AsyncVTK"] = &make<Serializer, AsyncVTK>;
}
template <>
Registry<Driver>::Registry() {
  object["DefaultDriver"] = &make_default_driver;
  object["UserDefinedGravityDriver"] = &make_user_gravity_driver;
}
template <>
Registry<Solver>::Registry() {
  object["ExplicitUSL"] = &make<Solver, ExplicitUSL>;
  object["ParallelExplicitUSL"] = &make<Solver, ParallelExplicitUSL>;
  object["ThreadPoolExplicitUSL"] = &make<Solver, ThreadPoolExplicitUSL>;
#ifdef MPM_WITH_GPU_PLUGIN
  object["GPUExplicitUSL"] = &make<Solver, GPUExplicitUSL>;
#endif
}
template <>
Registry<Grid>::Registry() {
  object["CartesianLinear"] = &make<Grid, CartesianLinear>;
}
template <>
Registry<Body>::Registry() {
  object["DefaultBody"] = &make<Body, DefaultBody>;
}
template <>
Registry<Points>::Registry() {
  object["DefaultPoints"] = &make<Points, DefaultPoints>;
  object["ThreadPoolPoints"] = &make<Points, ThreadPoolPoints>;
}
template <>
Registry<Nodes>::Registry() {
  object["DefaultNodes"] = &make<Nodes, DefaultNodes>;
}
template <>
Registry<Contact>::Registry() {
  object["ContactHuang"] = &make<Contact, ContactHuang>;
  object["ContactHuang_ReflectedBoundary"] = &make<Contact, ContactHuang_ReflectedBoundary>;
}
template <>
Registry<Material>::Registry() {
  object["IsotropicLinearElasticity"] = &make<Material, IsotropicLinearElasticity>;
  object["CompressibleNeohookeanElasticity"] = &make<Material, CompressibleNeohookeanElasticity>;
  object["Sand_SachithLocal"] = &make<Material, Sand_SachithLocal>;
}
template <>
Registry<Boundary>::Registry() {
  object["CartesianBox"] = &make<Boundary, CartesianBox>;
  object["CartesianSmoothBox"] = &make<Boundary, CartesianSmoothBox>;
  object["CartesianFrictionalBox"] = &make<Boundary, CartesianFrictionalBox>;
}

namespace {

struct RefHandle {
  Job job;
  std::string error;
};

void copy_vec_array(const KinematicVectorArray& a, double* out) {
  for (int i = 0; i < a.size(); i++)
    for (int j = 0; j < 3; j++) out[3 * i + j] = a[i][j];
}
void copy_tensor_array_mat(const MaterialTensorArray& a, double* out) {
  for (int i = 0; i < a.size(); i++)
    for (int j = 0; j < 9; j++) out[9 * i + j] = a[i][j];
}
void copy_tensor_array_kin(const KinematicTensorArray& a, double* out) {
  for (int i = 0; i < a.size(); i++)
    for (int j = 0; j < 9; j++) out[9 * i + j] = a[i][j];
}
void copy_scalar(const Eigen::VectorXd& a, double* out) {
  for (int i = 0; i < a.rows(); i++) out[i] = a(i);
}

}  // namespace

extern "C" {

// Builds and initialises a Job from a .cfg file, then applies gravity once, as
// DefaultDriver::run does before its loop (default_driver.cpp:58-60).
// Relative point-file paths resolve against the config file's directory.
// Returns NULL on failure.
void* ref_create(const char* cfg_path) {
  std::string path(cfg_path);
  std::string dir = ".";
  std::string::size_type slash = path.rfind('/');
  if (slash != std::string::npos) dir = path.substr(0, slash);
  char cwd[4096];
  if (getcwd(cwd, sizeof(cwd)) == nullptr) return nullptr;
  RefHandle* h = new RefHandle();
  try {
    if (chdir(dir.c_str()) != 0) {
      delete h;
      return nullptr;
    }
    Configurator cfg;
    std::string base = (slash == std::string::npos) ? path : path.substr(slash + 1);
    cfg.init(base);
    if (cfg.configureJob(&h->job) != 1) {
      if (chdir(cwd) != 0) {
      }
      delete h;
      return nullptr;
    }
    h->job.init();
    if (chdir(cwd) != 0) {
    }
  } catch (...) {
    if (chdir(cwd) != 0) {
    }
    delete h;
    return nullptr;
  }
  h->job.driver->generateGravity(&h->job);
  h->job.driver->applyGravity(&h->job);
  return h;
}

void ref_destroy(void* hp) { delete static_cast<RefHandle*>(hp); }

// Runs n solver steps; t advances by dt per step (default_driver.cpp:63-80).
int ref_step(void* hp, int n) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  for (int s = 0; s < n; s++) {
    h->job.solver->step(&h->job);
    h->job.serializer->writeFrame(&h->job);  // default_driver.cpp:65-79
    h->job.t += h->job.dt;
  }
  return 0;
}

double ref_get_time(void* hp) { return static_cast<RefHandle*>(hp)->job.t; }
double ref_get_dt(void* hp) { return static_cast<RefHandle*>(hp)->job.dt; }
int ref_job_dim(void* hp) { return static_cast<RefHandle*>(hp)->job.DIM; }
int ref_num_bodies(void* hp) { return (int)static_cast<RefHandle*>(hp)->job.bodies.size(); }
int ref_num_contacts(void* hp) { return (int)static_cast<RefHandle*>(hp)->job.contacts.size(); }
int ref_num_points(void* hp, int b) { return static_cast<RefHandle*>(hp)->job.bodies[b]->points->x.size(); }
int ref_num_nodes(void* hp, int b) { return static_cast<RefHandle*>(hp)->job.bodies[b]->nodes->x.size(); }

// Point fields: x, u, x_t, mx_t, b (3 per point); L, T (9 per point);
// m, v, v0, extent, active, and gammap, gammap_dot of a Sand_SachithLocal
// body (1 per point). Returns the number of doubles per
// point, or -1 for an unknown name.
int ref_get_point_field(void* hp, int b, const char* name, double* out) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  Points* p = h->job.bodies[b]->points.get();
  std::string n(name);
  if (n == "x") return copy_vec_array(p->x, out), 3;
  if (n == "u") return copy_vec_array(p->u, out), 3;
  if (n == "x_t") return copy_vec_array(p->x_t, out), 3;
  if (n == "mx_t") return copy_vec_array(p->mx_t, out), 3;
  if (n == "b") return copy_vec_array(p->b, out), 3;
  if (n == "L") return copy_tensor_array_kin(p->L, out), 9;
  if (n == "T") return copy_tensor_array_mat(p->T, out), 9;
  if (n == "m") return copy_scalar(p->m, out), 1;
  if (n == "v") return copy_scalar(p->v, out), 1;
  if (n == "v0") return copy_scalar(p->v0, out), 1;
  if (n == "active") {
    for (int i = 0; i < p->active.rows(); i++) out[i] = p->active(i);
    return 1;
  }
  if (n == "extent") {
    DefaultPoints* dp = dynamic_cast<DefaultPoints*>(p);
    if (dp == nullptr) return -1;
    copy_scalar(dp->extent, out);
    return 1;
  }
  if (n == "gammap" || n == "gammap_dot") {
    // Sand_SachithLocal's per-point plastic shear strain and its rate
    // (the material's frame fields, sand_sachithlocal.cpp:118-122)
    Sand_SachithLocal* sand = dynamic_cast<Sand_SachithLocal*>(h->job.bodies[b]->material.get());
    if (sand == nullptr) return -1;
    copy_scalar(n == "gammap" ? sand->gammap : sand->gammap_dot, out);
    return 1;
  }
  return -1;
}

// Node fields: x, u, x_t, mx_t, f, diff_x_t (3 per node); m (1 per node).
int ref_get_node_field(void* hp, int b, const char* name, double* out) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  Nodes* nd = h->job.bodies[b]->nodes.get();
  std::string n(name);
  if (n == "x") return copy_vec_array(nd->x, out), 3;
  if (n == "u") return copy_vec_array(nd->u, out), 3;
  if (n == "x_t") return copy_vec_array(nd->x_t, out), 3;
  if (n == "mx_t") return copy_vec_array(nd->mx_t, out), 3;
  if (n == "f") return copy_vec_array(nd->f, out), 3;
  if (n == "diff_x_t") return copy_vec_array(nd->diff_x_t, out), 3;
  if (n == "m") return copy_scalar(nd->m, out), 1;
  return -1;
}

// Contact fields of contact c: "normal" and "force" (3 per node of body 1).
int ref_get_contact_field(void* hp, int c, const char* name, double* out) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  ContactHuang* ch = dynamic_cast<ContactHuang*>(h->job.contacts[c].get());
  if (ch == nullptr) return -1;
  std::string n(name);
  if (n == "normal") return copy_vec_array(ch->contact_normal, out), 3;
  if (n == "force") return copy_vec_array(ch->contact_force, out), 3;
  return -1;
}

// Triplet lists of the last map build of body b (S: node, point, value;
// gradS: node, point, 3-vector), in the order the reference built them.
int ref_map_size(void* hp, int b) { return static_cast<RefHandle*>(hp)->job.bodies[b]->S.size(); }
int ref_grad_map_size(void* hp, int b) { return static_cast<RefHandle*>(hp)->job.bodies[b]->gradS.size(); }
int ref_get_map(void* hp, int b, int* node, int* point, double* val) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  const MPMScalarSparseMatrix& S = h->job.bodies[b]->S;
  const std::vector<int>& iv = S.get_i_index_ref();
  const std::vector<int>& jv = S.get_j_index_ref();
  for (int k = 0; k < S.size(); k++) {
    node[k] = iv[k];
    point[k] = jv[k];
    val[k] = S.buffer[k];
  }
  return S.size();
}
int ref_get_grad_map(void* hp, int b, int* node, int* point, double* grad) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  const KinematicVectorSparseMatrix& G = h->job.bodies[b]->gradS;
  const std::vector<int>& iv = G.get_i_index_ref();
  const std::vector<int>& jv = G.get_j_index_ref();
  for (int k = 0; k < G.size(); k++) {
    node[k] = iv[k];
    point[k] = jv[k];
    for (int j = 0; j < 3; j++) grad[3 * k + j] = G.buffer[k][j];
  }
  return G.size();
}

// Rebuilds S/gradS for the current positions without stepping (the first
// stage of ExplicitUSL::step, explicit_usl.cpp:104-110).
int ref_build_map(void* hp) {
  RefHandle* h = static_cast<RefHandle*>(hp);
  ExplicitUSL* s = dynamic_cast<ExplicitUSL*>(h->job.solver.get());
  if (s == nullptr) return -1;
  for (int b = 0; b < (int)h->job.bodies.size(); b++) h->job.bodies[b]->generateMap(&h->job, s->cpdi_spec);
  return 0;
}

}  // extern "C"
