// Device-side state of one explicit MPM job: point arrays (SoA, FP64),
// nodal accumulators and nodal velocities (block-linear, FP64).
#pragma once

#include "geom.cuh"

namespace mpmb200 {

// Points of one body, structure of arrays. The Cauchy stress is stored as
// its 6 independent components (xx, yy, zz, xy, yz, xz): the reference's
// update (isolin.cpp:62-74) keeps T exactly symmetric when it starts
// symmetric, so the 9-component form carries no extra information.
struct PointsDev {
  int64_t n;
  double* x[3];
  double* v[3];     // x_t
  double* u[3];
  double* s[6];     // stress xx yy zz xy yz xz
  double* vol;
  double* m;
  double* ext;      // extent, default_points.cpp:40-57
  int32_t* active;   // 1 active, 0 inactive, 2 left the domain at the last
                     // move (inactive from the next map build on)
  int32_t* pid;      // original index of the point
  double* L;        // 9 per point when debug output is kept, else null
};

// Nodal accumulators of one body (the values mapPointsToNodes builds,
// explicit_usl.cpp:112-164): mass, momentum and force.
struct NodesAcc {
  double* m;
  double* mx[3];
  double* f[3];
  double* nrm[3];   // contact normal accumulator (gradS * m) or null
};

// Nodal velocity after moveGrid and the velocity increment diff_x_t
// (explicit_usl.cpp:233-264), read by the gather.
struct NodesVel {
  double* vt[3];
  double* dv[3];
};

struct GridBodies {
  int nb;
  NodesAcc acc[kMaxBodies];
  NodesVel vel[kMaxBodies];
  NodesAcc snap[kMaxBodies];  // debug copies of m, mx_t, f after the update (or null)
  int has_boundary[kMaxBodies];
};

struct ContactSet {
  int nc;
  int b1[kMaxContacts];
  int b2[kMaxContacts];
  double mu[kMaxContacts];
  double* normal_out[kMaxContacts];  // 3 * nslots or null (debug)
  double* force_out[kMaxContacts];   // 3 * nslots or null (debug)
};

struct StepParams {
  double dt;
  double grav[3];
  int cpdi;
  int contact_spec;
  int keep_debug;
};

struct MaterialParams {
  int has_material;
  double G;
  double lambda;
};

}  // namespace mpmb200
