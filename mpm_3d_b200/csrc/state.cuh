// Device-side state of a batch of explicit MPM jobs: point arrays (SoA, FP64
// or FP32), nodal accumulators and nodal velocities (block-linear, FP64
// always), and the per-job / per-body tables the kernels read.
#pragma once

#include "geom.cuh"

namespace mpmb200 {

// Points of one body, structure of arrays, in the point precision PT
// (double for the FP64 form, float for the mixed form). The Cauchy stress is
// stored as its 6 independent components (xx, yy, zz, xy, yz, xz). The
// reference's update (isolin.cpp:62-74) keeps T symmetric up to rounding: W T
// and T W are each other's negated transposes bit for bit, but their terms
// are added to the symmetric part in a different order for (i,j) and (j,i),
// so T_ij and T_ji can differ in the last bit. One stored value per pair is
// within the FP64 parity tolerance of either.
template <typename PT>
struct PointsT {
  int64_t n;
  PT* x[3];
  PT* v[3];     // x_t
  PT* u[3];
  PT* s[6];     // stress xx yy zz xy yz xz
  PT* vol;
  PT* m;
  PT* ext;      // extent, default_points.cpp:40-57
  int32_t* active;   // 1 active, 0 inactive, 2 left the domain at the last
                     // move (inactive from the next map build on)
  int32_t* pid;      // original index of the point
  double* L;         // 9 per point when debug output is kept (FP64 form), else null
  // Per-point state of the material, zero at the start, else null:
  // CompressibleNeohookeanElasticity keeps its deformation gradient as F - I
  // (ms[0..8], row-major; zero = identity,
  // CompressibleNeohookeanElasticity::init); Sand_SachithLocal its plastic
  // shear strain gammap (ms[0]) and rate gammap_dot (ms[1])
  // (sand_sachithlocal.cpp:98-101).
  PT* ms[9];
  // Mixed form only (null in the FP64 form): the low words of the
  // position, velocity and mass, whose values are hi + lo summed in double
  // (two FP32 words, 48 significant bits; the high words are x, v and m).
  // The dynamics of soft bodies amplify a perturbation of the state by up
  // to 1e5 over a few hundred steps, so storing x or x_t rounded to FP32
  // (relative error 6e-8 per step) moves a trajectory by up to 1e-2 of its
  // scale, while the stress, volume and displacement in one FP32 word stay
  // well inside the mixed form's 1e-4 bound.
  PT* xl[3];
  PT* vl[3];
  PT* ml;
};
using PointsDev = PointsT<double>;

// A two-word value (hi + lo in double; the FP64 form has no low word).
template <typename PT>
__host__ __device__ __forceinline__ double two_word(const PT* hi, const PT* lo, int64_t i) {
  return lo != nullptr ? (double)hi[i] + (double)lo[i] : (double)hi[i];
}

// Splits a double into a two-word FP32 value: hi = fl(v), lo = fl(v - hi).
__host__ __device__ __forceinline__ void split_two_word(double v, float& hi, float& lo) {
  hi = (float)v;
  lo = (float)(v - (double)hi);
}

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

struct StepParams {
  double dt;
  double grav[3];
  int cpdi;
  int contact_spec;
  int keep_debug;
};

struct MaterialParams {
  int has_material;
  int kind;          // 0 IsotropicLinearElasticity, 1 CompressibleNeohookeanElasticity,
                     // 2 Sand_SachithLocal
  double G;
  double lambda;     // K - 2G/3
  double K;          // E / (3 (1 - 2 nu))
  // Sand_SachithLocal properties (sand_sachithlocal.cpp:57-103)
  double grains_d, mu_s, grains_rho, rho_critical, mu_2, i_0;
  int use_density;   // USE_DENSITY_FOR_PRESSURE: pressure from the density
  int pad_;
};

// Per-point material state arrays of each material kind (PointsT::ms).
inline int material_state_arrays(int has_material, int kind) {
  return !has_material ? 0 : (kind == 1 ? 9 : (kind == 2 ? 2 : 0));
}

// One job (the reference's Job: one grid, its bodies and contacts). Bodies
// body0 .. body0+nb-1 of the body tables belong to it; contact body indices
// are local to the job.
struct InstDev {
  Geom g;
  StepParams sp;
  int nb;
  int body0;
  int nc;
  int cb1[kMaxContacts];
  int cb2[kMaxContacts];
  double mu[kMaxContacts];
  int reflected[kMaxContacts];       // ContactHuang_ReflectedBoundary normals
  double* normal_out[kMaxContacts];  // 3 * nslots or null (debug)
  double* force_out[kMaxContacts];   // 3 * nslots or null (debug)
  int64_t block_off;                 // first node block of the job in the batch's block space
};

// What the grid update needs of a body.
struct GridBody {
  NodesAcc A;
  NodesAcc Ar;       // deterministic form: level-1 (remainder) sums, else null
  NodesVel V;
  NodesAcc snap;     // debug copies of m, mx_t, f after the update (or null)
  int has_boundary;  // 0 none, 1 CartesianBox, 2 CartesianSmoothBox, 3 CartesianFrictionalBox
  double mu_f;       // CartesianFrictionalBox friction
};

// Sizes of the batch's index spaces, read by the kernels on the device so
// that captured graphs stay valid while jobs come and go.
struct BatchHdr {
  int64_t points;   // sum of body point counts (sort space)
  int64_t bins;     // sum of (nbins + 1) over bodies
  int64_t cells;    // sum of (nbins * cells_per_bin + 1) over bodies
  int64_t blocks;   // node-block space (jobs' ranges and free holes)
  int nbodies;
  int ninst;
};

}  // namespace mpmb200
