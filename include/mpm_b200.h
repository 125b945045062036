/*
 * mpm_b200: C ABI of the B200 (sm_100a) explicit MPM time step.
 *
 * This is the drop-in boundary for mpm_3d's ExplicitUSL solver. A host-side
 * Solver plugin owns one mpmgpu_handle per Job and maps
 * the reference objects onto these calls:
 *
 *   Solver::init / lazy first step   -> mpmgpu_create, mpmgpu_add_body,
 *                                       mpmgpu_add_contact, mpmgpu_set_gravity
 *   Solver::step                     -> mpmgpu_step
 *   frame output / end of run        -> mpmgpu_download_points,
 *                                       mpmgpu_download_nodes,
 *                                       mpmgpu_download_contact
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
  /* FP64 throughout; nodal sums in a fixed order: bit-reproducible. */
  MPMGPU_MODE_FP64_DETERMINISTIC = 1,
  /* FP32 particle state, shape functions and stress; FP64 nodal mass and
   * momentum sums, nodal division and contact projection. */
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
 * default_points.cpp:150-174), IsotropicLinearElasticity E and nu
 * (isolin.cpp:26-46) and whether a CartesianBox boundary is attached
 * (cartesian_box.cpp:23-60). */
typedef struct {
  int64_t n;            /* number of points */
  const double* m;      /* n masses */
  const double* v;      /* n volumes */
  const double* x;      /* 3n positions (AoS) */
  const double* x_t;    /* 3n velocities (AoS) */
  const int32_t* active;/* n flags (nonzero = active); NULL = all active */
  int has_material;     /* 0: no Material (stress never updated) */
  double E, nu;
  int has_boundary;     /* 0: no Boundary */
  const double* u;      /* 3n initial displacements (AoS) or NULL (zero) */
  const double* T;      /* 9n initial Cauchy stresses (row-major, symmetric)
                           or NULL (zero) */
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
  MPMGPU_P_ACTIVE = 10 /* 1 (as double) */
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
 * need the map, e.g. code running while a CUDA stream is being captured into
 * a graph, a host framework that owns all device memory through its own
 * pool, or a real-time loop that forbids cudaMalloc/cudaFree after set-up.
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
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture. Every call reuses the same array: calls that overlap on the GPU
 * (from two handles or threads at once) race and must be serialised by the
 * caller. Returns after the triplets are written (synchronises the handle's
 * stream). */
mpmgpu_status mpmgpu_dump_map_noalloc(mpmgpu_handle* h, int body, int32_t* d_node, int32_t* d_point, double* d_s,
                                      double* d_grad, int64_t capacity, int64_t* count);

/* Number of points of body b and nodes of the grid. */
mpmgpu_status mpmgpu_sizes(const mpmgpu_handle* h, int body, int64_t* n_points, int64_t* n_nodes);

/* Number of kernel launches issued since creation (for launch accounting). */
int64_t mpmgpu_launch_count(const mpmgpu_handle* h);

/* The CUDA stream (cudaStream_t) all of the handle's work is queued on, so
 * a caller can record its own events around mpmgpu_step. */
void* mpmgpu_stream(const mpmgpu_handle* h);

/* Per-stage device time accounting with CUDA events recorded on the
 * handle's stream around every launch of a stage. enable != 0 starts (and
 * resets) it, 0 stops it. Stages: 0 fused gather/scatter kernel, 1 grid
 * update, 2 active-block compaction, 3 point re-binning. */
mpmgpu_status mpmgpu_profile(mpmgpu_handle* h, int enable);
/* Waits for the stream, then reports launches and total milliseconds of a stage. */
mpmgpu_status mpmgpu_profile_read(mpmgpu_handle* h, int stage, int64_t* launches, double* total_ms);

mpmgpu_status mpmgpu_destroy(mpmgpu_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* MPM_B200_H */
