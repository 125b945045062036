// GPUExplicitUSL: an mpm_3d Solver plugin that runs ExplicitUSL's time step on
// a B200 through the C ABI of include/mpm_b200.h.
//
// Drop-in for ExplicitUSL (src/objects/solvers/solvers.hpp:41-68): a config
// that names it,
//
//   solver { class = "GPUExplicitUSL"  int-properties = {1, 1} }
//
// runs the same Job (grid, bodies, points, materials, boundaries, contacts,
// driver, serializer) with the step on the GPU. int-properties mirror
// ExplicitUSL::init (explicit_usl.cpp:25-44): {cpdi_spec, contact_spec}, plus
// optional entries: the host write-back interval in steps (0 = write back
// exactly when a DefaultVTK, MinimalVTK or AsyncVTK serializer is about to
// write a frame, and every step for other serializers), the form (0 FP64,
// 1 deterministic FP64, 2 mixed) and the overlap switch (1, the default:
// at a frame the driver's next step is queued on the GPU before the frame is
// converted on the host, so that the two run at the same time; 0: the step
// is queued when the driver asks for it).
//
// Supported objects on the path: CartesianLinear, DefaultBody with
// DefaultPoints/DefaultNodes, IsotropicLinearElasticity,
// CompressibleNeohookeanElasticity or Sand_SachithLocal, CartesianBox,
// CartesianSmoothBox or CartesianFrictionalBox, ContactHuang or
// ContactHuang_ReflectedBoundary. Anything else is reported on stderr and the
// run stops with exit(0), as the reference does for bad properties
// (cartesian.cpp:27-30).
#ifndef MPM_B200_GPU_EXPLICIT_USL_HPP
#define MPM_B200_GPU_EXPLICIT_USL_HPP

#include <string>

#include "job.hpp"
#include "mpm_b200.h"
#include "mpm_objects.hpp"

class GPUExplicitUSL : public Solver {
 public:
  GPUExplicitUSL() { object_name = "GPUExplicitUSL"; }
  ~GPUExplicitUSL() override;

  int cpdi_spec = 1;
  int contact_spec = Contact::IMPLICIT;
  int writeback_interval = 0;
  int mode = 0;  // mpmgpu_mode: 0 FP64, 1 deterministic FP64, 2 mixed
  int overlap = 1;

  void init(Job* job) override;
  void step(Job* job) override;
  std::string saveState(Job* job, Serializer* serializer, std::string filepath) override;
  int loadState(Job* job, Serializer* serializer, std::string fullpath) override;

  // Copies the GPU state of every body into the Job's host arrays.
  void writeBack(Job* job);

 private:
  void setUp(Job* job);
  bool frameDue(Job* job);
  void check(mpmgpu_status s, const char* what);

  mpmgpu_handle* handle = nullptr;
  std::vector<int> gpu_body;   // job body index -> handle body index (-1 inactive)
  double gravity[3] = {0.0, 0.0, 0.0};
  long steps = 0;
  long frames = 0;             // frames the serializer has written (mirrors DefaultVTK)
  bool queued_ahead = false;   // the next step was queued at the last frame
  double sample_rate = 0.0;    // DefaultVTK properties[0], 0 if unknown
};

#endif  // MPM_B200_GPU_EXPLICIT_USL_HPP
