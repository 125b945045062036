/*
 * mpm_b200: C ABI of the B200 (sm_100a) explicit MPM time step.
 *
 * This is the drop-in boundary for mpm_3d's ExplicitUSL solver. A host-side
 * Solver plugin (mpm_3d_b200/plugin/gpu_explicit_usl.cpp) owns one
 * mpmgpu_handle per Job and maps
 * the reference objects onto these calls:
 *
 *   Solver::init / lazy first step   -> mpmgpu_create, mpmgpu_add_body,
 *                                       mpmgpu_add_contact, mpmgpu_set_gravity
 *   Solver::step                     -> mpmgpu_step
 *   frame output / end of run        -> mpmgpu_frame_begin, mpmgpu_frame_points,
 *                                       mpmgpu_frame_nodes, mpmgpu_frame_contact
 *                                       (or mpmgpu_download_points / _nodes /
 *                                       _contact, one field at a time)
 *   Job teardown                     -> mpmgpu_destroy
 *
 * All pointers passed in are HOST pointers unless a function says otherwise;
 * sizes are element counts. Arrays of 3-vectors use the reference's AoS
 * layout (stride 3, mpm_vectorarray.hpp:29), 3x3 tensors are 9 doubles in
 * row-major order (mpm_tensorarray.hpp:31), points are in the order they
 * were added and nodes use the reference's node ids
 * (i + j*(Nx+1) + k*(Nx+1)*(Ny+1), cartesian.cpp:119-141).
 *
 * Every function returns an mpmgpu_status; none calls exit(). The reference
 * prints to stderr and calls exit(0) on bad properties (cartesian.cpp:27-30,
 * isolin.cpp:29-32); callers that want that behaviour do it themselves.
 */
#ifndef MPM_B200_H
#define MPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MPMGPU_OK = 0,
  MPMGPU_ERR_ARG = 1,         /* invalid argument (null, range, state) */
  MPMGPU_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  MPMGPU_ERR_NOMEM = 3,       /* device or host allocation failed */
  MPMGPU_ERR_UNSUPPORTED = 4, /* feature outside the implemented path */
  MPMGPU_ERR_STATE = 5,       /* call not valid in the handle's state */
  MPMGPU_ERR_DEVICE = 6       /* a kernel reported an error flag */
} mpmgpu_status;

/* Arithmetic forms of the step. */
typedef enum {
  /* FP64 throughout; nodal sums use atomics (order varies run to run). */
  MPMGPU_MODE_FP64 = 0,
  /* FP64 throughout; nodal sums exact in any order (two-level pre-rounded
   * contributions): bit-reproducible run to run, across re-binning
   * intervals and batch mixes. */
  MPMGPU_MODE_FP64_DETERMINISTIC = 1,
  /* FP32 particle state (position, velocity and mass as two FP32 words,
   * hi + lo), shape functions and stress; the stress update, the mass and
   * momentum contributions and the position and velocity updates in FP64
   * arithmetic; FP64 nodal mass, momentum and force sums, nodal division
   * and contact projection. */
  MPMGPU_MODE_MIXED = 2
} mpmgpu_mode;

/* Grid and solver settings: CartesianLinear (grids.hpp:58-97) properties,
 * the job's dt and TYPE, and ExplicitUSL's int-properties
 * (explicit_usl.cpp:25-44). */
typedef struct {
  int dim;          /* job TYPE: 2 (2D) or 3 (3D); GRID_DIM == dim */
  double L[3];      /* domain lengths Lx, Ly, Lz (unused axes ignored) */
  int N[3];         /* cells per axis Nx, Ny, Nz */
  double dt;        /* time step */
  int cpdi_spec;    /* 1: corner-sampled (GIMP) map, 0: point-sampled */
  int contact_spec; /* 1: IMPLICIT ContactHuang, 0: EXPLICIT */
  int mode;         /* mpmgpu_mode */
  int device;       /* CUDA device ordinal */
  int keep_debug;   /* 1: keep L, nodal m/mx_t/f and contact forces
                       readable after each step (costs extra traffic) */
  int sort_interval;/* steps between re-binning the points by cell
                       (0 = default 32); results do not depend on it */
} mpmgpu_config;

/* One DefaultBody: its points (DefaultPoints::readFromFile columns,
 * default_points.cpp:150-174), its material's E and nu (isolin.cpp:26-46)
 * and further properties, and its boundary: CartesianBox (cartesian_box.cpp),
 * CartesianSmoothBox (cartesian_smooth_box.cpp) or CartesianFrictionalBox
 * (cartesian_frictional_box.cpp, friction mu_f from its fp64 property). */
typedef struct {
  int64_t n;            /* number of points */
  const double* m;      /* n masses */
  const double* v;      /* n volumes */
  const double* x;      /* 3n positions (AoS) */
  const double* x_t;    /* 3n velocities (AoS) */
  const int32_t* active;/* n flags (nonzero = active); NULL = all active */
  int has_material;     /* 0: no Material (stress never updated) */
  double E, nu;
  int has_boundary;     /* 0: no Boundary, 1: CartesianBox, 2: CartesianSmoothBox,
                           3: CartesianFrictionalBox */
  const double* u;      /* 3n initial displacements (AoS) or NULL (zero) */
  const double* T;      /* 9n initial Cauchy stresses (row-major, symmetric)
                           or NULL (zero) */
  double boundary_mu;   /* CartesianFrictionalBox mu_f (boundary-props[0]) */
  int material_kind;    /* 0: IsotropicLinearElasticity (isolin.cpp),
                           1: CompressibleNeohookeanElasticity
                           (compressible_neohookean_elasticity.cpp: F from
                           the identity, neo-Hookean stress),
                           2: Sand_SachithLocal (sand_sachithlocal.cpp:
                           Jaumann trial stress, local mu(I) return,
                           gammap and gammap_dot from zero) */
  double material_props[6]; /* Sand_SachithLocal: grain diameter, mu_s,
                           grains_rho, rho_critical, mu_2, I_0 as its init
                           resolves them (sand_sachithlocal.cpp:57-103:
                           mu_2 = mu_s and I_0 = 1 when the config gives
                           six material-props) */
  int material_flags;   /* bit 0: USE_DENSITY_FOR_PRESSURE (Sand_SachithLocal
                           material-str-props) */
} mpmgpu_body_desc;

typedef struct mpmgpu_handle mpmgpu_handle;

/* Point fields, as named in DefaultPoints::writeFrame
 * (default_points.cpp:341-368). */
typedef enum {
  MPMGPU_P_X = 0,      /* 3 per point */
  MPMGPU_P_U = 1,      /* 3 */
  MPMGPU_P_X_T = 2,    /* 3 */
  MPMGPU_P_MX_T = 3,   /* 3 */
  MPMGPU_P_B = 4,      /* 3 */
  MPMGPU_P_L = 5,      /* 9, requires keep_debug */
  MPMGPU_P_T = 6,      /* 9 */
  MPMGPU_P_M = 7,      /* 1 */
  MPMGPU_P_V = 8,      /* 1 */
  MPMGPU_P_EXTENT = 9, /* 1 */
  MPMGPU_P_ACTIVE = 10, /* 1 (as double) */
  MPMGPU_P_GAMMAP = 11, /* 1, Sand_SachithLocal bodies: plastic shear
                           strain (sand_sachithlocal.cpp:118-122) */
  MPMGPU_P_GAMMAP_DOT = 12 /* 1, Sand_SachithLocal bodies: its rate */
} mpmgpu_point_field;

/* Node fields, as named in DefaultNodes::writeFrame
 * (default_nodes.cpp:68-82). m, mx_t and f require keep_debug. */
typedef enum {
  MPMGPU_N_M = 0,        /* 1 per node */
  MPMGPU_N_MX_T = 1,     /* 3 */
  MPMGPU_N_F = 2,        /* 3 */
  MPMGPU_N_X_T = 3,      /* 3 */
  MPMGPU_N_U = 4,        /* 3 */
  MPMGPU_N_DIFF_X_T = 5  /* 3 */
} mpmgpu_node_field;

/* ContactHuang fields (contact_huang.cpp:202-206); require keep_debug. */
typedef enum {
  MPMGPU_C_NORMAL = 0, /* 3 per node */
  MPMGPU_C_FORCE = 1   /* 3 per node */
} mpmgpu_contact_field;

const char* mpmgpu_status_string(mpmgpu_status s);
/* Message of the last failed call on h (empty if none). */
const char* mpmgpu_last_error(const mpmgpu_handle* h);

/* Replaces ExplicitUSL::init (explicit_usl.cpp:25-44) together with
 * CartesianLinear::init (cartesian.cpp:24-67). */
mpmgpu_status mpmgpu_create(const mpmgpu_config* cfg, mpmgpu_handle** out);

/* Replaces DefaultBody::init (default_body.cpp:24-40) with its Points,
 * Nodes, Material and Boundary init calls. Copies the arrays to the device. */
mpmgpu_status mpmgpu_add_body(mpmgpu_handle* h, const mpmgpu_body_desc* desc, int* body_id);

/* Replaces ContactHuang::init (contact_huang.cpp:24-75). */
mpmgpu_status mpmgpu_add_contact(mpmgpu_handle* h, int body1, int body2, double mu_f, int* contact_id);

/* Replaces ContactHuang_ReflectedBoundary::init
 * (contact_huang_reflected_boundary.cpp:25-84): ContactHuang whose normal
 * loses its components normal to the walls of the box at nodes where body1
 * has mass (generateRules, 90-114). */
mpmgpu_status mpmgpu_add_contact_reflected(mpmgpu_handle* h, int body1, int body2, double mu_f, int* contact_id);

/* Gravity as the driver applies it (Driver::generateGravity/applyGravity):
 * use_vector 0 = DefaultDriver (-9.81 along y in 2D, z in 3D,
 * default_driver.cpp:90-105), 1 = UserDefinedGravityDriver vector g. May be
 * called between steps; the new body force enters the next step's nodal
 * forces, as points->b set at the end of a step does in the reference
 * (explicit_usl.cpp:80-81). */
mpmgpu_status mpmgpu_set_gravity(mpmgpu_handle* h, int use_vector, const double g[3]);

/* Replaces nsteps calls of ExplicitUSL::step (explicit_usl.cpp:48-87).
 * Asynchronous with respect to the host; errors surface on the next
 * synchronizing call. */
mpmgpu_status mpmgpu_step(mpmgpu_handle* h, int nsteps);

/* Waits for all work queued on the handle's stream; checks device flags. */
mpmgpu_status mpmgpu_synchronize(mpmgpu_handle* h);

/* Copies one field of body b to host memory `out` (reference layout). */
mpmgpu_status mpmgpu_download_points(mpmgpu_handle* h, int body, int field, double* out);
mpmgpu_status mpmgpu_download_nodes(mpmgpu_handle* h, int body, int field, double* out);
mpmgpu_status mpmgpu_download_contact(mpmgpu_handle* h, int contact, int field, double* out);

/* The write-back behind a frame (DefaultPoints::writeFrame,
 * default_points.cpp:341-368; DefaultNodes::writeFrame,
 * default_nodes.cpp:68-82; the contact arrays of ContactHuang::writeFrame,
 * contact_huang.cpp:202-206) in two halves. mpmgpu_frame_begin queues, behind
 * the steps queued so far, copies of every body's point, node and contact
 * fields into pinned host memory, and returns without waiting; steps queued
 * after it run while the copies are converted. mpmgpu_frame_points / _nodes
 * / _contact then give one field in the layout of the mpmgpu_download_*
 * call of the same name, as it stood at mpmgpu_frame_begin (the first of
 * them waits for the copies). A frame stays readable until the next
 * mpmgpu_frame_begin. */
mpmgpu_status mpmgpu_frame_begin(mpmgpu_handle* h);
mpmgpu_status mpmgpu_frame_points(mpmgpu_handle* h, int body, int field, double* out);
mpmgpu_status mpmgpu_frame_nodes(mpmgpu_handle* h, int body, int field, double* out);
mpmgpu_status mpmgpu_frame_contact(mpmgpu_handle* h, int contact, int field, double* out);

/* Rebuilds the S / gradS maps of body b for the current positions (the
 * first stage of ExplicitUSL::step, DefaultPoints::generateMap,
 * default_points.cpp:196-330) with the reference's exact operation order,
 * and copies the triplets to host memory in the reference's order. With
 * node == NULL the call only reports the count. Buffers must hold at least
 * *count entries (3 doubles per entry for grad). Deactivates points outside
 * the domain, as generateMap does. */
mpmgpu_status mpmgpu_dump_map(mpmgpu_handle* h, int body, int32_t* node, int32_t* point, double* s_val,
                              double* grad, int64_t* count);

/* No counterpart in the reference: an allocation-free form of
 * mpmgpu_dump_map for callers that cannot allocate device memory when they
 * need the map, e.g. a host framework that owns all device memory through
 * its own pool, or a real-time loop that forbids cudaMalloc/cudaFree after
 * set-up.
 *
 * Writes the same triplets as mpmgpu_dump_map, in the same reference order,
 * into caller-provided DEVICE arrays: d_node[k], d_point[k] (int32),
 * d_s[k] and d_grad[3k..3k+2] (double), k < capacity. *count receives the
 * number of triplets; if it exceeds capacity the call writes the first
 * `capacity` triplets and returns MPMGPU_ERR_ARG.
 *
 * Scratch lives in one static device array of the library (20 MiB, held by
 * every GPU that loads the library until the process exits), so the call
 * allocates nothing, but it serves at most 524,288 triplet slots: points x
 * 4^dim (8,192 points in 3D, 32,768 in 2D); larger bodies are rejected with
 * MPMGPU_ERR_ARG. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), and so does the first call after the
 * device's context changed (a device reset). Every call reuses the same
 * array: calls that overlap on the GPU (from two handles or threads at once)
 * race and must be serialised by the caller. Returns after the triplets are
 * written (synchronises the handle's stream); while the handle's stream is
 * being captured into a CUDA graph the call queues nothing and returns
 * MPMGPU_ERR_UNSUPPORTED, leaving the capture intact. */
mpmgpu_status mpmgpu_dump_map_noalloc(mpmgpu_handle* h, int body, int32_t* d_node, int32_t* d_point, double* d_s,
                                      double* d_grad, int64_t capacity, int64_t* count);

/* Number of points of body b and nodes of the grid. */
mpmgpu_status mpmgpu_sizes(const mpmgpu_handle* h, int body, int64_t* n_points, int64_t* n_nodes);

/* Number of kernel launches issued since creation (for launch accounting). */
int64_t mpmgpu_launch_count(const mpmgpu_handle* h);

/* The CUDA stream (cudaStream_t) all of the handle's work is ordered on, so
 * a caller can record its own events around mpmgpu_step. (With two to four
 * bodies, a step runs the bodies' fused kernels on side streams forked from
 * this stream and joined back into it before the step's next kernel, so
 * events and waits on this stream see the whole step.) */
void* mpmgpu_stream(const mpmgpu_handle* h);

/* Nodes with mass (counted per body) in the last step's grid update, and
 * the number of point visits that found a point outside its bin's staged
 * tile since creation (drift between re-binnings). Synchronises. */
mpmgpu_status mpmgpu_active_nodes(mpmgpu_handle* h, int64_t* nodes, int64_t* drifted);

/* No counterpart in the reference. Poll limit of the device-side waits of
 * the fused kernel for the bulk copies of a work item (default 2^24 polls,
 * far beyond the microseconds a copy takes). A wait that runs out does not
 * hang the GPU: the kernel flags it, lets the copies in flight land and
 * returns, and the next mpmgpu_synchronize reports MPMGPU_ERR_DEVICE. After
 * that error the handle's simulation state is undefined (destroy it); the
 * device and other handles stay usable. A small limit is a way to exercise
 * that path without a fault. */
mpmgpu_status mpmgpu_set_wait_limit(mpmgpu_handle* h, uint32_t polls);

/* No counterpart in the reference. Forms of the fused gather / update /
 * scatter kernel; every form computes the same step (the parity tests run
 * each). */
typedef enum {
  /* point arrays of a work item staged in shared memory, the gather and
   * scatter phases apart: 256 or 512 points per item (3D FP64), 256, 512 or
   * 1024 (3D mixed), 512 (2D); the only form of 2D jobs and of the
   * deterministic form */
  MPMGPU_KERNEL_STAGED = 0,
  /* each thread takes its points from gather to scatter, point state read
   * from global memory: 128 points per item (CTAs of 128 threads), 256
   * (256 threads) or 512 (256 threads, two points each); 3D, not the
   * deterministic form */
  MPMGPU_KERNEL_POINT_PER_THREAD = 1
} mpmgpu_kernel_form;

/* Selects the fused kernel's form and points per work item (default: one
 * point per thread with 512 points in 3D outside the deterministic form,
 * else staged with 512); MPMGPU_ERR_ARG if the pair is not available for
 * the handle. Takes effect at the next step. */
mpmgpu_status mpmgpu_set_kernel(mpmgpu_handle* h, int form, int points_per_item);
mpmgpu_status mpmgpu_kernel(const mpmgpu_handle* h, int* form, int* points_per_item);
/* No counterpart in the reference. Tunes the handle's launch shape on its
 * own bodies as mpmgpu_batch_autotune does (every available kernel form and
 * points-per-item choice for `steps` steps, then the re-binning interval),
 * keeps the fastest and reports it in *form and *points_per_item (either
 * may be null). The simulation's state after the call is the state before
 * it. */
mpmgpu_status mpmgpu_autotune(mpmgpu_handle* h, int steps, int* form, int* points_per_item);

/* Per-stage device time accounting with CUDA events recorded on the
 * handle's stream around every launch of a stage. enable != 0 starts (and
 * resets) it, 0 stops it. Stages: 0 fused gather/scatter kernel, 1 grid
 * update, 2 active-block compaction, 3 point re-binning. */
mpmgpu_status mpmgpu_profile(mpmgpu_handle* h, int enable);
/* Waits for the stream, then reports launches and total milliseconds of a stage. */
mpmgpu_status mpmgpu_profile_read(mpmgpu_handle* h, int stage, int64_t* launches, double* total_ms);

/* Releases the handle. Its job memory returns to the process's pool for
 * the device, which keeps up to 48 GB reserved for later handles and
 * batches (the rest is returned to the device); pinned staging buffers are
 * kept for reuse likewise (up to 4 GB). */
mpmgpu_status mpmgpu_destroy(mpmgpu_handle* h);

/* ------------------------------------------------------------------------
 * Batch: many independent jobs advanced together.
 *
 * No counterpart in the reference, which runs one Job per process
 * (main.cpp:60-106). A batch holds jobs of one dimension and one arithmetic
 * form, each with its own grid, bodies, contacts, dt and step count; every
 * mpmgpu_batch_step advances all jobs that still have steps, with one
 * launch per stage for the whole batch (the step and the re-binning are
 * replayed from CUDA graphs). Jobs may be added while others run: they join
 * at the next step boundary; a job that has run its steps stops advancing
 * and stays readable until it is removed. Each job computes exactly what a
 * single-job handle with the same inputs computes (up to the order of the
 * nodal sums).
 * ---------------------------------------------------------------------- */

typedef struct mpmgpu_batch mpmgpu_batch;

typedef struct {
  int dim;             /* 2 or 3 for every job of the batch */
  int mode;            /* MPMGPU_MODE_FP64 or MPMGPU_MODE_MIXED */
  int device;          /* CUDA device ordinal */
  int sort_interval;   /* steps between re-binnings (0 = default 32) */
  int points_per_item; /* points per CTA work item: 0 = default (3D,
                          not deterministic: 512 on the point-per-thread
                          kernel; else 512 on the staged kernel); 128, 256
                          or 512 run on the point-per-thread kernel where
                          it applies, other sizes on the staged kernel
                          (1024 in the 3D mixed form, 512 in 2D); see
                          mpmgpu_set_kernel and mpmgpu_batch_autotune */
  int no_graph;        /* 1: launch stage by stage instead of graph replay */
  int keep_debug;      /* as mpmgpu_config.keep_debug */
} mpmgpu_batch_config;

/* One ContactHuang pair of a job (bodies are indices within the job);
 * reflected = 1 for ContactHuang_ReflectedBoundary. */
typedef struct {
  int body1, body2;
  double mu;
  int reflected;
} mpmgpu_contact_desc;

/* One job: grid / dt / cpdi_spec / contact_spec from `grid` (its mode,
 * device, keep_debug and sort_interval are the batch's), its bodies and
 * contacts, the driver gravity (as mpmgpu_set_gravity) and its step count. */
typedef struct {
  const mpmgpu_config* grid;
  int nbodies;
  const mpmgpu_body_desc* bodies;
  int ncontacts;
  const mpmgpu_contact_desc* contacts;
  int gravity_vector;   /* 0 = DefaultDriver, 1 = the vector below */
  double gravity[3];
  int64_t steps;
} mpmgpu_job_desc;

mpmgpu_status mpmgpu_batch_create(const mpmgpu_batch_config* cfg, mpmgpu_batch** out);
const char* mpmgpu_batch_last_error(const mpmgpu_batch* b);

/* Device bytes the job will hold once added (for admission control). */
mpmgpu_status mpmgpu_batch_footprint(const mpmgpu_batch* b, const mpmgpu_job_desc* job, int64_t* bytes);

/* Copies the job's arrays to the device; the job joins at the next step. */
mpmgpu_status mpmgpu_batch_add_job(mpmgpu_batch* b, const mpmgpu_job_desc* job, int* job_id);

/* nsteps steps of every job that still has steps (asynchronous). */
mpmgpu_status mpmgpu_batch_step(mpmgpu_batch* b, int nsteps);
mpmgpu_status mpmgpu_batch_synchronize(mpmgpu_batch* b);

/* Steps done and left of a job (host bookkeeping; no synchronisation). */
mpmgpu_status mpmgpu_batch_job_state(const mpmgpu_batch* b, int job, int64_t* steps_done, int64_t* steps_left);
mpmgpu_status mpmgpu_batch_sizes(const mpmgpu_batch* b, int job, int body, int64_t* n_points, int64_t* n_nodes);

/* As mpmgpu_download_points, for body `body` of job `job`. */
mpmgpu_status mpmgpu_batch_download_points(mpmgpu_batch* b, int job, int body, int field, double* out);
/* No counterpart in the reference. One point field of body `body` of each
 * of `count` jobs, outs[k] receiving jobs[k]'s (layout of
 * mpmgpu_download_points): the copies are queued together with one wait and
 * converted to the reference's order on up to `threads` host threads. */
mpmgpu_status mpmgpu_batch_download_points_many(mpmgpu_batch* b, int count, const int* jobs, int body, int field,
                                                double* const* outs, int threads);

/* Frees the job's device memory; it leaves the batch at the next step. */
mpmgpu_status mpmgpu_batch_remove_job(mpmgpu_batch* b, int job);

/* Jobs and points still stepping, and device bytes held by the batch. */
mpmgpu_status mpmgpu_batch_counts(const mpmgpu_batch* b, int* live_jobs, int64_t* live_points, int64_t* bytes_in_use);

/* Tunes the launch shape on the current jobs: times `steps` steps for every
 * available kernel form and points-per-item choice (staged 256, 512, 1024;
 * point per thread 128, 256, 512), then 32 steps for each re-binning
 * interval (4, 8, 16, 32),
 * restoring the jobs' state after each trial, and keeps the fastest of
 * each. The jobs' state after the call is the state before it. */
mpmgpu_status mpmgpu_batch_autotune(mpmgpu_batch* b, int steps, int* points_per_item);
int mpmgpu_batch_points_per_item(const mpmgpu_batch* b);
/* The fused kernel's form (mpmgpu_kernel_form) in use. */
int mpmgpu_batch_kernel_form(const mpmgpu_batch* b);
/* Selects the fused kernel's form and points per work item (as
 * mpmgpu_set_kernel); the jobs are re-binned before the next step. */
mpmgpu_status mpmgpu_batch_set_kernel(mpmgpu_batch* b, int form, int points_per_item);
int mpmgpu_batch_sort_interval(const mpmgpu_batch* b);

/* As mpmgpu_active_nodes, over every job of the batch. */
mpmgpu_status mpmgpu_batch_active_nodes(mpmgpu_batch* b, int64_t* nodes, int64_t* drifted);

/* Per-stage event timing, as mpmgpu_profile (launches stage by stage while
 * enabled). */
mpmgpu_status mpmgpu_batch_profile(mpmgpu_batch* b, int enable);
mpmgpu_status mpmgpu_batch_profile_read(mpmgpu_batch* b, int stage, int64_t* launches, double* total_ms);

void* mpmgpu_batch_stream(const mpmgpu_batch* b);
/* Kernel launches issued (a graph replay counts its kernels). */
int64_t mpmgpu_batch_launch_count(const mpmgpu_batch* b);
/* Releases the batch (memory as mpmgpu_destroy). */
mpmgpu_status mpmgpu_batch_destroy(mpmgpu_batch* b);

/* ------------------------------------------------------------------------
 * Server: continuous batching of simulation requests.
 *
 * No counterpart in the reference (its only run-time failure handling is
 * exit(0) on SIGINT, include/signal_handler.hpp:15-31). A server owns one
 * batch and a device memory budget. mpmgpu_server_submit admits a request
 * (one job) at once if its footprint (mpmgpu_batch_footprint) fits the
 * budget left by the requests still running; otherwise it returns
 * MPMGPU_ERR_STATE and the caller keeps the request queued and retries
 * after the next advance. A request whose footprint exceeds the whole budget
 * is rejected with MPMGPU_ERR_NOMEM (it could never run). Admitted requests join the running batch at the
 * next step boundary and step together with it; a request that has run its
 * steps has its final point state (x, u, x_t, T, v, active) copied to host
 * memory and its device memory released. Each request computes what it
 * would compute alone (up to the order of the nodal sums).
 * ---------------------------------------------------------------------- */

typedef struct mpmgpu_server mpmgpu_server;

/* cfg->points_per_item = 0 selects the batch default. */
mpmgpu_status mpmgpu_server_create(const mpmgpu_batch_config* cfg, int64_t budget_bytes, mpmgpu_server** out);
const char* mpmgpu_server_last_error(const mpmgpu_server* s);
/* Device bytes the request will reserve from the budget while it runs. */
mpmgpu_status mpmgpu_server_footprint(const mpmgpu_server* s, const mpmgpu_job_desc* job, int64_t* bytes);
mpmgpu_status mpmgpu_server_submit(mpmgpu_server* s, const mpmgpu_job_desc* job, int* request_id);
/* Queues `steps` steps of every running request. A request that runs its
 * last step here has its point state copied to pinned host memory and its
 * device memory released, both in stream order, without waiting; it is
 * reported finished by the next advance, which converts the copies while the
 * device runs that call's steps (advance waits for the previous call's
 * copies, never for the steps it queues). */
mpmgpu_status mpmgpu_server_advance(mpmgpu_server* s, int steps);
/* Ids of requests finished since the last poll (at most max_ids); returns
 * their number. */
int mpmgpu_server_poll(mpmgpu_server* s, int* ids, int max_ids);
/* State (1 running, 4 being copied out, 2 finished, 3 released, 5 cancelled),
 * admission and completion times on mpmgpu_server_clock, points and steps
 * of a request. */
mpmgpu_status mpmgpu_server_request(const mpmgpu_server* s, int id, int* state, double* t_admit, double* t_done,
                                    int64_t* points, int64_t* steps);
/* A finished request's final point field (MPMGPU_P_X, _U, _X_T, _T, _V or
 * _ACTIVE) of one body, in the layout of mpmgpu_download_points. */
mpmgpu_status mpmgpu_server_result(mpmgpu_server* s, int id, int body, int field, double* out);
/* Cancels a running request between advances: it leaves the batch at the
 * next step boundary and its device memory and budget share are freed; the
 * other requests are unaffected. MPMGPU_ERR_STATE if it is not running. */
mpmgpu_status mpmgpu_server_cancel(mpmgpu_server* s, int id);
/* Frees a finished request's host copy of its results. */
mpmgpu_status mpmgpu_server_release(mpmgpu_server* s, int id);
mpmgpu_status mpmgpu_server_stats(const mpmgpu_server* s, int* running, int64_t* reserved_bytes, int64_t* live_points,
                                  int64_t* particle_steps_done);
/* Seconds since the server was created (steady clock). */
double mpmgpu_server_clock(const mpmgpu_server* s);
mpmgpu_status mpmgpu_server_destroy(mpmgpu_server* s);

/* ---- .points files ----
 * Host-side reader of the DefaultPoints point files that the reference's
 * configs name (DefaultPoints::readFromFile, default_points.cpp:104-193):
 * a count line, then per point "m v x.. x_t.. active" separated by single
 * spaces, split and converted as the reference does (Parser::splitString,
 * std::stod). The lines are parsed on `threads` threads (0: all the host
 * offers); no GPU is used. Arrays come back in mpmgpu_body_desc's layout
 * (x and x_t AoS with stride 3, zero beyond dim), ready for
 * mpmgpu_add_body. A missing file or a malformed line (wrong column count,
 * a column that is not a number) gives MPMGPU_ERR_ARG and, where bad_line
 * is not NULL, the 1-based line number (0 for the file itself); the
 * reference prints an error there and keeps zeros for the remaining points.
 * mpmgpu_points_file_count reads the count line; _read requires n to equal
 * it. */
mpmgpu_status mpmgpu_points_file_count(const char* path, int64_t* n);
mpmgpu_status mpmgpu_points_file_read(const char* path, int dim, int64_t n, double* m, double* v, double* x,
                                      double* x_t, int32_t* active, int threads, int64_t* bad_line);

#ifdef __cplusplus
}
#endif

#endif /* MPM_B200_H */
