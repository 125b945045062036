/*
 * CPU restatement of mpm_3d's ExplicitUSL time step (the hot path), in C99.
 *
 * TEST INFRASTRUCTURE ONLY. This is the oracle: tests, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it (oracle/_ref/libmpm_oracle.so) to
 * check the CUDA path. Nothing in the product (mpm_3d_b200/) links or calls
 * it.
 *
 * Every floating-point operation follows the reference's own expression and
 * evaluation order, so that, compiled with -ffp-contract=off, its output is
 * bit-identical to the reference sources compiled the same way
 * (oracle/_ref/libmpmref_parity.so; checked by tests/test_oracle.py). The
 * reference's per-step COO triplet lists (S, gradS) are rebuilt here in the
 * reference's own order and every sparse product walks them in that order, so
 * even the summation order matches.
 *
 * Scope: JOB_TYPE 2 (2D) and 3 (3D) on CartesianLinear, DefaultBody /
 * DefaultPoints / DefaultNodes, IsotropicLinearElasticity, CartesianBox,
 * ContactHuang (IMPLICIT and EXPLICIT), DefaultDriver or user-defined
 * gravity. Axisymmetric, 1D and out-of-plane job types are not restated.
 *
 * Citations are file:line within the reference project (mpm_3d).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OC_MAX_BODIES 8
#define OC_MAX_CONTACTS 8

typedef struct {
  int n;                 /* points */
  double *x, *u, *x_t, *mx_t, *b; /* 3 per point (AoS, stride 3) */
  double *L, *T;         /* 9 per point (row-major 3x3) */
  double *m, *v, *v0, *extent;
  int *active;
  /* nodes: 3 per node unless noted */
  double *nx, *nu, *nx_t, *nmx_t, *nf, *ndiff, *nm /* 1 per node */;
  double *bc_mask;       /* the boundary's bcNodalMask, 3 per node */
  double *bc_force;      /* CartesianFrictionalBox bcNodalForce, 3 per node */
  double mu_f;           /* CartesianFrictionalBox friction */
  int has_material;
  int material_kind;     /* 0 IsotropicLinearElasticity, 1 CompressibleNeohookeanElasticity,
                            2 Sand_SachithLocal */
  double *F;             /* neo-Hookean deformation gradient, 9 per point (row-major) */
  double *gammap, *gammap_dot; /* Sand_SachithLocal plastic shear strain and rate, 1 per point */
  /* Sand_SachithLocal properties (sand_sachithlocal.cpp:57-103) */
  double grains_d, mu_s, grains_rho, rho_critical, mu_2, i_0;
  int use_density;       /* USE_DENSITY_FOR_PRESSURE */
  int has_boundary;      /* 0 none, 1 CartesianBox, 2 CartesianSmoothBox, 3 CartesianFrictionalBox */
  double E, nu_, G, K, lambda;
  /* COO triplets of the last map build */
  int nnz, gnnz, cap;
  int *S_i, *S_j;
  double *S_v;
  int *G_i, *G_j;
  double *G_v; /* 3 per triplet */
} oc_body;

typedef struct {
  int b1, b2;
  double mu_f;
  int reflected;          /* 1: ContactHuang_ReflectedBoundary */
  double *normal, *force; /* 3 per node */
} oc_contact;

typedef struct {
  int dim;               /* GRID_DIM == DIM for JOB_TYPE 2 and 3 */
  double Lx[3], hx[3];
  int Nx[3];
  int node_count, element_count, npe;
  double *x_n;           /* 3 per node */
  int *nodeIDs;          /* element_count x npe */
  int gridA[8][3];       /* cartesian.cpp:97-112 (0/1 offsets) */
  int pointA[8][3];      /* default_points.cpp:70-84 (-1/+1 corners) */
  double dt, t;
  int cpdi_spec, contact_spec;
  int user_gravity;
  double gravity[3];
  int nbodies, ncontacts;
  oc_body bodies[OC_MAX_BODIES];
  oc_contact contacts[OC_MAX_CONTACTS];
} oc_job;

/* ---- CartesianLinear (src/objects/grids/cartesian.cpp) ---- */

/* nodeIDToPosition, cartesian.cpp:258-274 */
static void node_position(const oc_job* J, int id, double out[3]) {
  int ijk[3] = {0, 0, 0};
  int tmp = id;
  for (int i = 0; i < J->dim; i++) {
    ijk[i] = tmp % (J->Nx[i] + 1);
    tmp = tmp / (J->Nx[i] + 1);
  }
  for (int i = 0; i < 3; i++) out[i] = 0.0;
  for (int i = 0; i < J->dim; i++) out[i] = J->hx[i] * ijk[i];
}

/* init + hiddenInit, cartesian.cpp:24-141 (volumes and surfaces unused) */
static int grid_init(oc_job* J) {
  J->node_count = 1;
  J->element_count = 1;
  J->npe = 1;
  for (int i = 0; i < J->dim; i++) {
    J->node_count *= (J->Nx[i] + 1);
    J->element_count *= J->Nx[i];
    J->npe *= 2;
  }
  J->x_n = (double*)malloc(sizeof(double) * 3 * (size_t)J->node_count);
  if (!J->x_n) return -1;
  for (int n = 0; n < J->node_count; n++) node_position(J, n, J->x_n + 3 * (size_t)n);
  int onoff[3] = {0, 0, 0};
  for (int n = 0; n < J->npe; n++) {
    for (int i = 0; i < J->dim; i++) J->gridA[n][i] = onoff[i];
    for (int i = 0; i < J->dim; i++) {
      if (onoff[i] == 0) {
        onoff[i] = 1;
        break;
      } else {
        onoff[i] = 0;
      }
    }
  }
  J->nodeIDs = (int*)calloc((size_t)J->element_count * J->npe, sizeof(int));
  if (!J->nodeIDs) return -1;
  for (int e = 0; e < J->element_count; e++) {
    int ijk[3] = {0, 0, 0};
    int tmp = e;
    for (int i = 0; i < J->dim; i++) {
      ijk[i] = tmp % J->Nx[i];
      tmp = tmp / J->Nx[i];
    }
    for (int n = 0; n < J->npe; n++) {
      int id = 0;
      for (int i = 0; i < J->dim; i++) {
        if (i == 0) id += (ijk[i] + J->gridA[n][i]);
        else if (i == 1) id += (ijk[i] + J->gridA[n][i]) * (J->Nx[i - 1] + 1);
        else id += (ijk[i] + J->gridA[n][i]) * (J->Nx[i - 1] + 1) * (J->Nx[i - 2] + 1);
      }
      J->nodeIDs[(size_t)e * J->npe + n] = id;
    }
  }
  return 0;
}

/* cartesianWhichElement, cartesian.cpp:219-240 */
static int which_element(const oc_job* J, const double x[3]) {
  int elementID = (int)floor(x[0] / J->Lx[0] * J->Nx[0]);
  for (int i = 0; i < J->dim; i++) {
    int in = (x[i] < J->Lx[i] && x[i] >= 0);
    if (!in) return -1;
    if (i == 1) {
      elementID = (int)(elementID + floor(x[i] / J->Lx[i] * J->Nx[i]) * (J->Nx[i - 1]));
    } else if (i == 2) {
      elementID = (int)(elementID + floor(x[i] / J->Lx[i] * J->Nx[i]) * (J->Nx[i - 1]) * (J->Nx[i - 2]));
    }
  }
  return elementID;
}

/* inDomain, cartesian.cpp:245-253 */
static int in_domain(const oc_job* J, const double x[3]) {
  for (int i = 0; i < J->dim; i++) {
    if (!(x[i] <= J->Lx[i] && x[i] >= 0)) return 0;
  }
  return 1;
}

/* evaluateBasisFnValue, cartesian.cpp:280-302. Appends up to npe entries. */
static int basis_value(const oc_job* J, const double x[3], int* nid, double* val) {
  int e = which_element(J, x);
  if (e < 0) return 0;
  for (int n = 0; n < J->npe; n++) {
    int node = J->nodeIDs[(size_t)e * J->npe + n];
    double tmp = 1.0;
    for (int i = 0; i < J->dim; i++) {
      double r = (x[i] - J->x_n[3 * (size_t)node + i]) / J->hx[i];
      tmp *= (1 - fabs(r));
    }
    nid[n] = node;
    val[n] = tmp;
  }
  return J->npe;
}

/* evaluateBasisFnGradient, cartesian.cpp:307-357 */
static int basis_gradient(const oc_job* J, const double x[3], int* nid, double* grad) {
  int e = which_element(J, x);
  if (e < 0) return 0;
  for (int n = 0; n < J->npe; n++) {
    int node = J->nodeIDs[(size_t)e * J->npe + n];
    double r[3] = {0, 0, 0};
    double tmp = 1.0;
    for (int i = 0; i < J->dim; i++) {
      r[i] = (x[i] - J->x_n[3 * (size_t)node + i]) / J->hx[i];
      tmp *= (1 - fabs(r[i]));
    }
    double g[3] = {0, 0, 0};
    for (int i = 0; i < J->dim; i++) {
      g[i] = -tmp / (1 - fabs(r[i])) * r[i] / fabs(r[i]) / J->hx[i];
      if (fabs(r[i]) >= 1) g[i] = 0.0;
    }
    nid[n] = node;
    for (int i = 0; i < 3; i++) grad[3 * n + i] = g[i];
  }
  return J->npe;
}

/* ---- DefaultPoints (src/objects/points/default_points.cpp) ---- */

static int body_reserve(oc_body* B, int need) {
  if (need <= B->cap) return 0;
  int cap = need;
  B->S_i = (int*)realloc(B->S_i, sizeof(int) * (size_t)cap);
  B->S_j = (int*)realloc(B->S_j, sizeof(int) * (size_t)cap);
  B->S_v = (double*)realloc(B->S_v, sizeof(double) * (size_t)cap);
  B->G_i = (int*)realloc(B->G_i, sizeof(int) * (size_t)cap);
  B->G_j = (int*)realloc(B->G_j, sizeof(int) * (size_t)cap);
  B->G_v = (double*)realloc(B->G_v, sizeof(double) * 3 * (size_t)cap);
  if (!B->S_i || !B->S_j || !B->S_v || !B->G_i || !B->G_j || !B->G_v) return -1;
  B->cap = cap;
  return 0;
}

/* generateMap, default_points.cpp:196-330 */
static int generate_map(oc_job* J, oc_body* B) {
  int cp = J->npe;
  if (body_reserve(B, B->n * cp * cp) != 0) return -1;
  B->nnz = 0;
  B->gnnz = 0;
  int nvec[64];
  double valvec[64];
  double gradvec[64 * 3];
  for (int i = 0; i < B->n; i++) {
    const double* xi = B->x + 3 * (size_t)i;
    int ith_cpdi = J->cpdi_spec;
    if (B->active[i] == 0) {
      continue;
    } else if (!in_domain(J, xi)) {
      B->active[i] = 0;
      continue;
    } else if (ith_cpdi == 1) {
      for (int c = 0; c < cp; c++) {
        double corner[3] = {0, 0, 0};
        for (int pos = 0; pos < J->dim; pos++) corner[pos] = xi[pos] + 0.5 * B->extent[i] * J->pointA[c][pos];
        if (!in_domain(J, corner)) {
          ith_cpdi = 0;
          break;
        }
      }
    }
    if (ith_cpdi == 0) {
      int cnt = basis_value(J, xi, nvec, valvec);
      for (int j = 0; j < cnt; j++) {
        B->S_i[B->nnz] = nvec[j];
        B->S_j[B->nnz] = i;
        B->S_v[B->nnz] = valvec[j];
        B->nnz++;
      }
      cnt = basis_gradient(J, xi, nvec, gradvec);
      for (int j = 0; j < cnt; j++) {
        B->G_i[B->gnnz] = nvec[j];
        B->G_j[B->gnnz] = i;
        for (int d = 0; d < 3; d++) B->G_v[3 * (size_t)B->gnnz + d] = gradvec[3 * j + d];
        B->gnnz++;
      }
    } else if (ith_cpdi == 1) {
      for (int c = 0; c < cp; c++) {
        double corner[3] = {0, 0, 0};
        for (int pos = 0; pos < J->dim; pos++) corner[pos] = xi[pos] + 0.5 * B->extent[i] * J->pointA[c][pos];
        int cnt = basis_value(J, corner, nvec, valvec);
        for (int j = 0; j < cnt; j++) {
          B->S_i[B->nnz] = nvec[j];
          B->S_j[B->nnz] = i;
          B->S_v[B->nnz] = valvec[j] / cp;
          B->nnz++;
        }
        /* gradient pass (default_points.cpp:290-324) evaluates the same
         * corner again; the values are identical, so they are reused. */
        for (int j = 0; j < cnt; j++) {
          double g[3] = {0, 0, 0};
          for (int pos = 0; pos < J->dim; pos++) g[pos] = valvec[j] / (cp * 0.5 * B->extent[i]) * J->pointA[c][pos];
          B->G_i[B->gnnz] = nvec[j];
          B->G_j[B->gnnz] = i;
          for (int d = 0; d < 3; d++) B->G_v[3 * (size_t)B->gnnz + d] = g[d];
          B->gnnz++;
        }
      }
    }
  }
  return 0;
}

/* ---- ExplicitUSL (src/objects/solvers/explicit_usl.cpp) ---- */

/* mapPointsToNodes, explicit_usl.cpp:112-164 */
static void map_points_to_nodes(oc_job* J, oc_body* B) {
  int N = J->node_count;
  memset(B->nm, 0, sizeof(double) * (size_t)N);
  memset(B->nmx_t, 0, sizeof(double) * 3 * (size_t)N);
  memset(B->nf, 0, sizeof(double) * 3 * (size_t)N);
  for (int k = 0; k < B->nnz; k++) B->nm[B->S_i[k]] += B->S_v[k] * B->m[B->S_j[k]];
  for (int p = 0; p < B->n; p++)
    for (int d = 0; d < 3; d++) B->mx_t[3 * (size_t)p + d] = (d < J->dim) ? B->m[p] * B->x_t[3 * (size_t)p + d] : B->x_t[3 * (size_t)p + d];
  for (int k = 0; k < B->nnz; k++) {
    int i = B->S_i[k], j = B->S_j[k];
    for (int d = 0; d < J->dim; d++) B->nmx_t[3 * (size_t)i + d] += B->S_v[k] * B->mx_t[3 * (size_t)j + d];
  }
  for (int i = 0; i < N; i++) {
    if (B->nm[i] > 0) {
      double inv = 1.0 / B->nm[i];
      for (int d = 0; d < J->dim; d++) B->nx_t[3 * (size_t)i + d] = B->nmx_t[3 * (size_t)i + d] * inv;
    } else {
      for (int d = 0; d < J->dim; d++) B->nx_t[3 * (size_t)i + d] = 0;
    }
  }
  /* f = S * (m b) */
  for (int k = 0; k < B->nnz; k++) {
    int i = B->S_i[k], j = B->S_j[k];
    for (int d = 0; d < J->dim; d++) B->nf[3 * (size_t)i + d] += B->S_v[k] * (B->m[j] * B->b[3 * (size_t)j + d]);
  }
  /* nvec = gradS.left_multiply_by_tensor(v T), mpm_sparse.cpp:691-706, with
   * MaterialTensor * KinematicVector from mpm_vector.hpp:816-824. */
  double* nvec = (double*)calloc(3 * (size_t)N, sizeof(double));
  for (int k = 0; k < B->gnnz; k++) {
    int i = B->G_i[k], j = B->G_j[k];
    const double* T = B->T + 9 * (size_t)j;
    const double* g = B->G_v + 3 * (size_t)k;
    double vj = B->v[j];
    for (int a = 0; a < 3; a++) {
      double tmp = 0;
      for (int c = 0; c < J->dim; c++) tmp += (T[3 * a + c] * vj) * g[c];
      nvec[3 * (size_t)i + a] += tmp;
    }
  }
  for (int i = 0; i < N; i++)
    for (int d = 0; d < J->dim; d++) B->nf[3 * (size_t)i + d] -= nvec[3 * (size_t)i + d];
  free(nvec);
}

/* ContactHuang::generateRules, contact_huang.cpp:80-99 */
static void contact_generate(oc_job* J, oc_contact* C) {
  oc_body* B = &J->bodies[C->b1];
  int N = J->node_count;
  memset(C->normal, 0, sizeof(double) * 3 * (size_t)N);
  for (int k = 0; k < B->gnnz; k++) {
    int i = B->G_i[k], j = B->G_j[k];
    for (int d = 0; d < J->dim; d++) C->normal[3 * (size_t)i + d] += B->G_v[3 * (size_t)k + d] * B->m[j];
  }
  if (!C->reflected) {
    for (int i = 0; i < N; i++) {
      double* n = C->normal + 3 * (size_t)i;
      double s = 0;
      for (int d = 0; d < J->dim; d++) s += n[d] * n[d];
      double inv = 1.0 / sqrt(s);
      for (int d = 0; d < J->dim; d++) n[d] *= inv;
    }
    return;
  }
  /* ContactHuang_ReflectedBoundary::generateRules
   * (contact_huang_reflected_boundary.cpp:90-114): at nodes where body 1 has
   * mass, the components normal to a wall of the box (Lx from init, 66-74)
   * are zeroed before the normalisation; other nodes keep the raw sum. */
  double Lmax[3] = {0, 0, 0};
  for (int i = 0; i < N; i++)
    for (int pos = 0; pos < J->dim; pos++)
      if (B->nx[3 * (size_t)i + pos] > Lmax[pos]) Lmax[pos] = B->nx[3 * (size_t)i + pos];
  for (int i = 0; i < N; i++) {
    if (!(B->nm[i] > 0)) continue;
    double* n = C->normal + 3 * (size_t)i;
    for (int pos = 0; pos < J->dim; pos++) {
      double xv = B->nx[3 * (size_t)i + pos];
      if (xv == 0 || xv == Lmax[pos]) n[pos] = 0;
    }
    double s = 0;
    for (int d = 0; d < J->dim; d++) s += n[d] * n[d];
    double inv = 1.0 / sqrt(s);
    for (int d = 0; d < J->dim; d++) n[d] *= inv;
  }
}

/* ContactHuang::applyRules, contact_huang.cpp:104-197 */
static void contact_apply(oc_job* J, oc_contact* C) {
  oc_body* B1 = &J->bodies[C->b1];
  oc_body* B2 = &J->bodies[C->b2];
  int D = J->dim;
  double dt = J->dt;
  for (int i = 0; i < J->node_count; i++) {
    double* fc_out = C->force + 3 * (size_t)i;
    if (B1->nm[i] > 0 && B2->nm[i] > 0) {
      double fcti[3] = {0, 0, 0};
      const double* normal = C->normal + 3 * (size_t)i;
      double m1 = B1->nm[i], m2 = B2->nm[i];
      double mv1[3] = {0, 0, 0}, mv2[3] = {0, 0, 0}, vcm[3] = {0, 0, 0};
      double* f1 = B1->nf + 3 * (size_t)i;
      double* f2 = B2->nf + 3 * (size_t)i;
      for (int d = 0; d < D; d++) {
        if (J->contact_spec == 1) {
          mv1[d] = B1->nmx_t[3 * (size_t)i + d] + dt * f1[d];
          mv2[d] = B2->nmx_t[3 * (size_t)i + d] + dt * f2[d];
        } else {
          mv1[d] = B1->nmx_t[3 * (size_t)i + d];
          mv2[d] = B2->nmx_t[3 * (size_t)i + d];
        }
      }
      double inv_m12 = 1.0 / (m1 + m2);
      for (int d = 0; d < D; d++) vcm[d] = (mv1[d] + mv2[d]) * inv_m12;
      double inv_m1 = 1.0 / m1;
      double test = 0;
      for (int d = 0; d < D; d++) test += (mv1[d] * inv_m1 - vcm[d]) * normal[d];
      if (test > 0) {
        double vcm_n = 0, mv1_n = 0;
        for (int d = 0; d < D; d++) vcm_n += vcm[d] * normal[d];
        for (int d = 0; d < D; d++) mv1_n += mv1[d] * normal[d];
        double fn1i = m1 / dt * (vcm_n - mv1_n / m1);
        double s1[3] = {0, 0, 0};
        double m1dt = m1 / dt;
        for (int d = 0; d < D; d++) s1[d] = m1dt * (vcm[d] - mv1[d] * inv_m1) - fn1i * normal[d];
        double ss = 0;
        for (int d = 0; d < D; d++) ss += s1[d] * s1[d];
        double ft1i = sqrt(ss);
        if (ft1i != 0) {
          double inv = 1.0 / ft1i;
          for (int d = 0; d < D; d++) s1[d] *= inv;
        }
        /* std::min(a, b) is (b < a) ? b : a */
        double a = (fn1i < 0.0) ? fn1i : 0.0;
        double mu_fn = C->mu_f * fabs(fn1i);
        double bb = (fabs(ft1i) < mu_fn) ? fabs(ft1i) : mu_fn;
        for (int d = 0; d < D; d++) fcti[d] = a * normal[d] + bb * s1[d];
        for (int d = 0; d < D; d++) f1[d] += fcti[d];
        for (int d = 0; d < D; d++) f2[d] -= fcti[d];
      }
      for (int d = 0; d < 3; d++) fc_out[d] = fcti[d];
    } else {
      for (int d = 0; d < 3; d++) fc_out[d] = 0;
    }
  }
}

/* Boundary masks: CartesianBox::init (cartesian_box.cpp:29-55) locks every
 * component of a node on any wall; CartesianSmoothBox::init
 * (cartesian_smooth_box.cpp:23-59) locks the wall-normal components;
 * CartesianFrictionalBox::init (cartesian_frictional_box.cpp:21-84) marks
 * lower (-1) and upper (1) walls per component and 2 for the other
 * components of a node on a wall. */
static void boundary_init(oc_job* J, oc_body* B) {
  double Lmax[3] = {0, 0, 0};
  for (int i = 0; i < J->node_count; i++)
    for (int pos = 0; pos < J->dim; pos++)
      if (B->nx[3 * (size_t)i + pos] > Lmax[pos]) Lmax[pos] = B->nx[3 * (size_t)i + pos];
  for (int i = 0; i < J->node_count; i++) {
    double* mk = B->bc_mask + 3 * (size_t)i;
    const double* xn = B->nx + 3 * (size_t)i;
    for (int d = 0; d < 3; d++) mk[d] = 0;
    if (B->has_boundary == 1) {
      for (int pos = 0; pos < J->dim; pos++) {
        if (xn[pos] == 0 || xn[pos] == Lmax[pos]) {
          for (int d = 0; d < J->dim; d++) mk[d] = 1;
          break;
        }
      }
    } else if (B->has_boundary == 2) {
      for (int pos = 0; pos < J->dim; pos++)
        if (xn[pos] == 0 || xn[pos] == Lmax[pos]) mk[pos] = 1;
    } else if (B->has_boundary == 3) {
      int is_edge = 0;
      for (int pos = 0; pos < J->dim; pos++) {
        if (xn[pos] == 0) {
          mk[pos] = -1;
          is_edge = 1;
        } else if (xn[pos] == Lmax[pos]) {
          mk[pos] = 1;
          is_edge = 1;
        }
      }
      for (int pos = 0; pos < J->dim; pos++)
        if (is_edge && mk[pos] != 1 && mk[pos] != -1) mk[pos] = 2;
    }
  }
}

/* std::min / std::max as the reference calls them */
static double std_min(double a, double b) { return (b < a) ? b : a; }
static double std_max(double a, double b) { return (a < b) ? b : a; }

static double vec_norm(const double* v, int dim) {
  double s = 0.0;
  for (int d = 0; d < dim; d++) s += v[d] * v[d];
  return sqrt(s);
}

/* CartesianBox::applyRules (cartesian_box.cpp:73-85) and
 * CartesianSmoothBox::applyRules (cartesian_smooth_box.cpp:69-83): locked
 * components of x_t, mx_t and f are zeroed. CartesianFrictionalBox::applyRules
 * (cartesian_frictional_box.cpp:94-143): the closing momentum of a wall
 * component (from the body force and stress divergence, bcNodalForce) gives
 * a normal force, the component is zeroed, and a friction force of at most
 * mu_f times the normal force opposes the remaining motion. */
static void boundary_apply(oc_job* J, oc_body* B) {
  const int dim = J->dim;
  const double dt = J->dt;
  for (int i = 0; i < J->node_count; i++) {
    const double* mk = B->bc_mask + 3 * (size_t)i;
    double* xt = B->nx_t + 3 * (size_t)i;
    double* mx = B->nmx_t + 3 * (size_t)i;
    double* f = B->nf + 3 * (size_t)i;
    if (B->has_boundary != 3) {
      for (int pos = 0; pos < dim; pos++)
        if (mk[pos] == 1) {
          xt[pos] = 0;
          mx[pos] = 0;
          f[pos] = 0;
        }
      continue;
    }
    const double* bf = B->bc_force + 3 * (size_t)i;
    double dmom[3] = {0, 0, 0};
    for (int pos = 0; pos < dim; pos++) {
      if (mk[pos] == -1) {
        dmom[pos] = -std_min(0.0, mx[pos] + dt * bf[pos]);
        xt[pos] = 0;
        mx[pos] = 0;
        f[pos] = 0;
      } else if (mk[pos] == 1) {
        dmom[pos] = -std_max(0.0, mx[pos] + dt * bf[pos]);
        xt[pos] = 0;
        mx[pos] = 0;
        f[pos] = 0;
      } else {
        dmom[pos] = 0;
      }
    }
    const double f_normal = vec_norm(dmom, dim) / dt;
    for (int pos = 0; pos < dim; pos++) dmom[pos] = mx[pos] + dt * f[pos];
    if (vec_norm(dmom, dim) > 0) {
      const double c = std_min(vec_norm(dmom, dim) / dt, f_normal * B->mu_f);
      /* vector / scalar multiplies by the reciprocal (mpm_vector.hpp:609-615) */
      const double inv = 1.0 / vec_norm(dmom, dim);
      for (int pos = 0; pos < dim; pos++) f[pos] -= (c * dmom[pos]) * inv;
    }
  }
}

/* moveGrid, explicit_usl.cpp:233-264 */
static void move_grid(oc_job* J, oc_body* B) {
  double dt = J->dt;
  int N = J->node_count;
  for (size_t k = 0; k < 3 * (size_t)N; k++) B->nmx_t[k] = B->nmx_t[k] + dt * B->nf[k];
  for (int i = 0; i < N; i++) {
    if (B->nm[i] > 0) {
      double inv = 1.0 / B->nm[i];
      for (int d = 0; d < J->dim; d++) B->nx_t[3 * (size_t)i + d] = B->nmx_t[3 * (size_t)i + d] * inv;
    } else {
      for (int d = 0; d < J->dim; d++) B->nx_t[3 * (size_t)i + d] = 0;
    }
  }
  for (size_t k = 0; k < 3 * (size_t)N; k++) B->nu[k] = dt * B->nx_t[k];
  for (int i = 0; i < N; i++) {
    if (B->nm[i] > 0) {
      double inv = 1.0 / B->nm[i];
      for (int d = 0; d < J->dim; d++) B->ndiff[3 * (size_t)i + d] = (dt * B->nf[3 * (size_t)i + d]) * inv;
    } else {
      for (int d = 0; d < J->dim; d++) B->ndiff[3 * (size_t)i + d] = 0;
    }
  }
}

/* movePoints, explicit_usl.cpp:266-300 (Sᵀ products, mpm_sparse.cpp:66-81) */
static void move_points(oc_job* J, oc_body* B) {
  size_t n3 = 3 * (size_t)B->n;
  double* tmp = (double*)calloc(n3, sizeof(double));
  double* tmp2 = (double*)calloc(n3, sizeof(double));
  for (int k = 0; k < B->nnz; k++) {
    int p = B->S_j[k], i = B->S_i[k];
    for (int d = 0; d < J->dim; d++) tmp[3 * (size_t)p + d] += B->S_v[k] * B->nu[3 * (size_t)i + d];
  }
  for (size_t k = 0; k < n3; k++) B->x[k] = B->x[k] + tmp[k];
  for (size_t k = 0; k < n3; k++) B->u[k] = B->u[k] + tmp[k];
  for (int k = 0; k < B->nnz; k++) {
    int p = B->S_j[k], i = B->S_i[k];
    for (int d = 0; d < J->dim; d++) tmp2[3 * (size_t)p + d] += B->S_v[k] * B->ndiff[3 * (size_t)i + d];
  }
  for (size_t k = 0; k < n3; k++) B->x_t[k] = B->x_t[k] + tmp2[k];
  for (int p = 0; p < B->n; p++)
    for (int d = 0; d < J->dim; d++) B->mx_t[3 * (size_t)p + d] = B->m[p] * B->x_t[3 * (size_t)p + d];
  free(tmp);
  free(tmp2);
}

/* calculateStrainRate, explicit_usl.cpp:302-330 (tensor_product_transpose,
 * mpm_sparse.cpp:673-688; KinematicVector::tensor, mpm_vector.hpp:684-700;
 * KinematicTensor::operator+=, mpm_tensor.hpp:698-712) */
static void strain_rate(oc_job* J, oc_body* B) {
  memset(B->L, 0, sizeof(double) * 9 * (size_t)B->n);
  int D = J->dim;
  for (int k = 0; k < B->gnnz; k++) {
    int p = B->G_j[k], i = B->G_i[k];
    const double* v = B->nx_t + 3 * (size_t)i;
    const double* g = B->G_v + 3 * (size_t)k;
    double* L = B->L + 9 * (size_t)p;
    for (int a = 0; a < D; a++)
      for (int c = 0; c < D; c++) L[3 * a + c] = L[3 * a + c] + v[a] * g[c];
  }
}

/* updateDensity, explicit_usl.cpp:332-345 */
static void update_density(oc_job* J, oc_body* B) {
  for (int p = 0; p < B->n; p++) {
    const double* L = B->L + 9 * (size_t)p;
    B->v[p] *= exp(J->dt * (L[0] + L[4] + L[8]));
  }
}

/* DefaultDriver::generateGravity/applyGravity, default_driver.cpp:90-119 */
static void apply_gravity(oc_job* J) {
  double g[3] = {0, 0, 0};
  if (J->user_gravity) {
    for (int d = 0; d < 3; d++) g[d] = J->gravity[d];
  } else if (J->dim == 2) {
    g[1] = -9.81;
  } else if (J->dim == 3) {
    g[2] = -9.81;
  }
  for (int bi = 0; bi < J->nbodies; bi++) {
    oc_body* B = &J->bodies[bi];
    for (int p = 0; p < B->n; p++)
      for (int d = 0; d < 3; d++) B->b[3 * (size_t)p + d] = g[d];
  }
}

/* IsotropicLinearElasticity::calculateStress, isolin.cpp:50-78, with the
 * MaterialTensor operators of mpm_tensor.hpp:964-1070. */
/* CompressibleNeohookeanElasticity::calculateStress
 * (compressible_neohookean_elasticity.cpp:44-62): F += (L F) dt, B = F F^T,
 * J = sqrt(det B), T = G/J (B - I) + (K - 2G/3) ln(J)/J I, with the 3x3
 * product and determinant of mpm_tensor.hpp (579-584, 1060-1070). */
static void update_stress_neohookean(oc_job* J, oc_body* B) {
  const double dt = J->dt;
  static const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int p = 0; p < B->n; p++) {
    if (B->active[p] == 0) continue;
    const double* L = B->L + 9 * (size_t)p;
    double* F = B->F + 9 * (size_t)p;
    double* T = B->T + 9 * (size_t)p;
    double LF[9], Bm[9];
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++)
        LF[3 * a + c] = L[3 * a + 0] * F[0 + c] + L[3 * a + 1] * F[3 + c] + L[3 * a + 2] * F[6 + c];
    for (int k = 0; k < 9; k++) F[k] = F[k] + LF[k] * dt;
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++)
        Bm[3 * a + c] = F[3 * a + 0] * F[3 * c + 0] + F[3 * a + 1] * F[3 * c + 1] + F[3 * a + 2] * F[3 * c + 2];
    const double da = Bm[0] * (Bm[4] * Bm[8] - Bm[7] * Bm[5]);
    const double db = Bm[1] * (Bm[3] * Bm[8] - Bm[6] * Bm[5]);
    const double dc = Bm[2] * (Bm[3] * Bm[7] - Bm[6] * Bm[4]);
    const double Jv = sqrt(da - db + dc);
    const double s1 = B->G / Jv;
    const double s2 = (B->K - 2.0 * B->G / 3.0) * log(Jv) / Jv;
    for (int k = 0; k < 9; k++) T[k] = s1 * (Bm[k] - I[k]) + s2 * I[k];
  }
}

/* Sand_SachithLocal::negative_root (sand_sachithlocal.cpp:44-53): the
 * smaller root of a x^2 + b x + c, in the form without cancellation. */
static double sand_negative_root(double a, double b, double c) {
  if (b > 0) return (-b - sqrt(b * b - 4 * a * c)) / (2 * a);
  return (2 * c) / (-b + sqrt(b * b - 4 * a * c));
}

/* Sand_SachithLocal::calculateStress (sand_sachithlocal.cpp:140-215) with
 * SPEC = UPDATE (explicit_usl.cpp:352) and cohesion c = 0: the Jaumann trial
 * stress s_tr = T + dt (2G D + lambda tr(D) I + W T - T W), its pressure
 * p_tr = -tr(s_tr)/3 (or K (rho/rho_c - 1) with USE_DENSITY_FOR_PRESSURE),
 * deviator t0 = s_tr + p_tr I and tau_tr = |t0|/sqrt(2). Below the critical
 * density or at p_tr <= 0 the stress is zero; inside the cone tau_tr <=
 * mu_s p_tr it is the trial stress; otherwise tau is the smaller root of
 * tau^2 - (S2 + tau_tr + alpha) tau + S2 tau_tr + S0 alpha and T = (tau /
 * tau_tr) t0 - p_tr I. gammap += nup dt, gammap_dot = nup with nup the
 * plastic shear rate. Tensor operations in the element order of
 * mpm_tensor.hpp (trace 564-567, norm 570-576). */
static void update_stress_sand(oc_job* J, oc_body* B) {
  const double dt = J->dt;
  const double c = 0;
  static const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int p = 0; p < B->n; p++) {
    if (B->active[p] == 0) continue;
    const double* L = B->L + 9 * (size_t)p;
    double* T = B->T + 9 * (size_t)p;
    double Lt[9], D[9], W[9];
    for (int a = 0; a < 3; a++)
      for (int k = 0; k < 3; k++) Lt[3 * a + k] = L[3 * k + a];
    for (int k = 0; k < 9; k++) D[k] = 0.5 * (L[k] + Lt[k]);
    for (int k = 0; k < 9; k++) W[k] = 0.5 * (L[k] - Lt[k]);
    const double trD = D[0] + D[4] + D[8];
    double WT[9], TW[9], tmp[9], s_tr[9], t0[9];
    for (int a = 0; a < 3; a++)
      for (int k = 0; k < 3; k++) {
        WT[3 * a + k] = W[3 * a + 0] * T[0 + k] + W[3 * a + 1] * T[3 + k] + W[3 * a + 2] * T[6 + k];
        TW[3 * a + k] = T[3 * a + 0] * W[0 + k] + T[3 * a + 1] * W[3 + k] + T[3 * a + 2] * W[6 + k];
      }
    const double twoG = 2 * B->G;
    const double ltr = B->lambda * trD;
    for (int k = 0; k < 9; k++) tmp[k] = ((twoG * D[k] + ltr * I[k]) + WT[k]) - TW[k];
    for (int k = 0; k < 9; k++) s_tr[k] = T[k] + dt * tmp[k];
    double p_tr = -(s_tr[0] + s_tr[4] + s_tr[8]) / 3.0;
    for (int k = 0; k < 9; k++) t0[k] = s_tr[k] + p_tr * I[k];
    double nn = 0;
    for (int k = 0; k < 9; k++) nn += t0[k] * t0[k];
    const double tau_tr = sqrt(nn) / sqrt(2.0);
    if (B->use_density) p_tr = B->K * ((B->m[p] / B->v[p] - B->rho_critical) / B->rho_critical);
    const int density_flag = (B->m[p] / B->v[p]) < B->rho_critical;
    double nup_tau;
    if (density_flag || p_tr <= c) {
      nup_tau = tau_tr / (B->G * dt);
      for (int k = 0; k < 9; k++) T[k] = 0.0;
    } else if (p_tr > c) {
      const double S0 = B->mu_s * p_tr;
      double tau_tau, scale_factor;
      if (tau_tr <= S0) {
        tau_tau = tau_tr;
        scale_factor = 1.0;
      } else {
        const double S2 = B->mu_2 * p_tr;
        const double alpha = B->G * B->i_0 * dt * sqrt(p_tr / B->grains_rho) / B->grains_d;
        const double Bq = -(S2 + tau_tr + alpha);
        const double Hq = S2 * tau_tr + S0 * alpha;
        tau_tau = sand_negative_root(1.0, Bq, Hq);
        scale_factor = (tau_tau / tau_tr);
      }
      nup_tau = ((tau_tr - tau_tau) / B->G) / dt;
      for (int k = 0; k < 9; k++) T[k] = scale_factor * t0[k] - p_tr * I[k];
    } else {
      nup_tau = 0; /* p_tr is NaN: T stays as it was */
    }
    B->gammap[p] += nup_tau * dt;
    B->gammap_dot[p] = nup_tau;
  }
}

static void update_stress(oc_job* J, oc_body* B) {
  if (B->material_kind == 1) {
    update_stress_neohookean(J, B);
    return;
  }
  if (B->material_kind == 2) {
    update_stress_sand(J, B);
    return;
  }
  double dt = J->dt;
  for (int p = 0; p < B->n; p++) {
    if (B->active[p] == 0) continue;
    const double* L = B->L + 9 * (size_t)p;
    double* T = B->T + 9 * (size_t)p;
    double Lt[9], D[9], W[9];
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++) Lt[3 * a + c] = L[3 * c + a];
    for (int k = 0; k < 9; k++) D[k] = 0.5 * (L[k] + Lt[k]);
    for (int k = 0; k < 9; k++) W[k] = 0.5 * (L[k] - Lt[k]);
    double trD = D[0] + D[4] + D[8];
    double WT[9], TW[9];
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++) {
        WT[3 * a + c] = W[3 * a + 0] * T[0 + c] + W[3 * a + 1] * T[3 + c] + W[3 * a + 2] * T[6 + c];
        TW[3 * a + c] = T[3 * a + 0] * W[0 + c] + T[3 * a + 1] * W[3 + c] + T[3 * a + 2] * W[6 + c];
      }
    double twoG = 2 * B->G;
    double ltr = B->lambda * trD;
    static const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double tmp[9];
    for (int k = 0; k < 9; k++) tmp[k] = ((twoG * D[k] + ltr * I[k]) + WT[k]) - TW[k];
    for (int k = 0; k < 9; k++) T[k] = T[k] + dt * tmp[k];
  }
}

/* ---- C ABI ---- */

void* oc_create(int dim, const double* L, const int* N, double dt, int cpdi_spec, int contact_spec) {
  oc_job* J = (oc_job*)calloc(1, sizeof(oc_job));
  if (!J) return NULL;
  J->dim = dim;
  for (int i = 0; i < 3; i++) {
    J->Lx[i] = (i < dim) ? L[i] : 0;
    J->Nx[i] = (i < dim) ? N[i] : 0;
    J->hx[i] = (i < dim) ? J->Lx[i] / J->Nx[i] : 0;
  }
  J->dt = dt;
  J->cpdi_spec = cpdi_spec;
  J->contact_spec = contact_spec;
  if (grid_init(J) != 0) return NULL;
  /* corner matrix of DefaultPoints::init, default_points.cpp:70-84 */
  int onoff[3] = {-1, -1, -1};
  for (int c = 0; c < J->npe; c++) {
    for (int i = 0; i < dim; i++) J->pointA[c][i] = onoff[i];
    for (int i = 0; i < dim; i++) {
      if (onoff[i] == -1) {
        onoff[i] = 1;
        break;
      } else {
        onoff[i] = -1;
      }
    }
  }
  return J;
}

/* Adds a body: n points with m, v (volume), x and x_t (3 per point, AoS),
 * active flags. Material E, nu (has_material); boundary kind (has_boundary: 0 none,
 * 1 CartesianBox, 2 CartesianSmoothBox, 3 CartesianFrictionalBox with mu_f =
 * boundary_mu).
 * Mirrors DefaultBody::init (default_body.cpp:24-40), DefaultPoints::init
 * (default_points.cpp:35-57), DefaultNodes::init (default_nodes.cpp:29-63),
 * IsotropicLinearElasticity::init (isolin.cpp:34-38). */
int oc_add_body(void* hp, int n, const double* m, const double* v, const double* x, const double* x_t,
                const int* active, int has_material, double E, double nu, int has_boundary, double boundary_mu,
                int material_kind) {
  oc_job* J = (oc_job*)hp;
  if (J->nbodies >= OC_MAX_BODIES) return -1;
  oc_body* B = &J->bodies[J->nbodies];
  memset(B, 0, sizeof(*B));
  size_t N = (size_t)J->node_count;
  B->n = n;
  B->x = (double*)calloc(3 * (size_t)n, sizeof(double));
  B->u = (double*)calloc(3 * (size_t)n, sizeof(double));
  B->x_t = (double*)calloc(3 * (size_t)n, sizeof(double));
  B->mx_t = (double*)calloc(3 * (size_t)n, sizeof(double));
  B->b = (double*)calloc(3 * (size_t)n, sizeof(double));
  B->L = (double*)calloc(9 * (size_t)n, sizeof(double));
  B->F = (double*)calloc(9 * (size_t)n, sizeof(double));
  for (int p = 0; p < n; p++) B->F[9 * (size_t)p] = B->F[9 * (size_t)p + 4] = B->F[9 * (size_t)p + 8] = 1.0;
  B->T = (double*)calloc(9 * (size_t)n, sizeof(double));
  B->gammap = (double*)calloc((size_t)n, sizeof(double));
  B->gammap_dot = (double*)calloc((size_t)n, sizeof(double));
  B->m = (double*)calloc((size_t)n, sizeof(double));
  B->v = (double*)calloc((size_t)n, sizeof(double));
  B->v0 = (double*)calloc((size_t)n, sizeof(double));
  B->extent = (double*)calloc((size_t)n, sizeof(double));
  B->active = (int*)calloc((size_t)n, sizeof(int));
  B->nx = (double*)calloc(3 * N, sizeof(double));
  B->nu = (double*)calloc(3 * N, sizeof(double));
  B->nx_t = (double*)calloc(3 * N, sizeof(double));
  B->nmx_t = (double*)calloc(3 * N, sizeof(double));
  B->nf = (double*)calloc(3 * N, sizeof(double));
  B->ndiff = (double*)calloc(3 * N, sizeof(double));
  B->nm = (double*)calloc(N, sizeof(double));
  B->bc_mask = (double*)calloc(3 * N, sizeof(double));
  B->bc_force = (double*)calloc(3 * N, sizeof(double));
  for (int p = 0; p < n; p++) {
    B->m[p] = m[p];
    B->v[p] = v[p];
    B->v0[p] = v[p];
    B->active[p] = active[p];
    for (int d = 0; d < J->dim; d++) {
      B->x[3 * (size_t)p + d] = x[3 * (size_t)p + d];
      B->x_t[3 * (size_t)p + d] = x_t[3 * (size_t)p + d];
    }
    B->extent[p] = (J->dim == 2) ? 0.5 * sqrt(v[p]) : 0.5 * cbrt(v[p]);
  }
  for (size_t i = 0; i < N; i++) node_position(J, (int)i, B->nx + 3 * i);
  B->has_material = has_material;
  B->material_kind = material_kind;
  B->has_boundary = has_boundary;
  B->mu_f = boundary_mu;
  B->E = E;
  B->nu_ = nu;
  B->G = E / (2.0 * (1.0 + nu));
  B->K = E / (3.0 * (1.0 - 2 * nu));
  B->lambda = B->K - 2.0 * B->G / 3.0;
  if (has_boundary) boundary_init(J, B);
  J->nbodies++;
  apply_gravity(J); /* DefaultDriver::run applies gravity before its loop */
  return J->nbodies - 1;
}

/* Sets a Sand_SachithLocal body's properties after E and nu, in the order of
 * its material-props (sand_sachithlocal.cpp:57-103): grain diameter, mu_s,
 * grains_rho, rho_critical and, when nprops >= 6, mu_2 and I_0 (otherwise
 * mu_2 = mu_s and I_0 = 1); use_density: the USE_DENSITY_FOR_PRESSURE
 * str-property. Returns -1 for a body of another material or too few
 * properties. */
int oc_set_sand(void* hp, int b, const double* props, int nprops, int use_density) {
  oc_job* J = (oc_job*)hp;
  if (b < 0 || b >= J->nbodies || nprops < 4) return -1;
  oc_body* B = &J->bodies[b];
  if (B->material_kind != 2) return -1;
  B->grains_d = props[0];
  B->mu_s = props[1];
  B->grains_rho = props[2];
  B->rho_critical = props[3];
  B->mu_2 = nprops >= 6 ? props[4] : B->mu_s;
  B->i_0 = nprops >= 6 ? props[5] : 1;
  B->use_density = use_density;
  return 0;
}

int oc_add_contact(void* hp, int b1, int b2, double mu_f, int reflected) {
  oc_job* J = (oc_job*)hp;
  if (J->ncontacts >= OC_MAX_CONTACTS) return -1;
  oc_contact* C = &J->contacts[J->ncontacts];
  C->b1 = b1;
  C->b2 = b2;
  C->mu_f = mu_f;
  C->reflected = reflected;
  C->normal = (double*)calloc(3 * (size_t)J->node_count, sizeof(double));
  C->force = (double*)calloc(3 * (size_t)J->node_count, sizeof(double));
  J->ncontacts++;
  return J->ncontacts - 1;
}

/* use_user: 0 = DefaultDriver gravity, 1 = UserDefinedGravityDriver vector */
void oc_set_gravity(void* hp, int use_user, const double* g) {
  oc_job* J = (oc_job*)hp;
  J->user_gravity = use_user;
  for (int d = 0; d < 3; d++) J->gravity[d] = (use_user && d < J->dim) ? g[d] : 0.0;
  apply_gravity(J);
}

/* ExplicitUSL::step, explicit_usl.cpp:48-87 */
int oc_step(void* hp, int nsteps) {
  oc_job* J = (oc_job*)hp;
  for (int s = 0; s < nsteps; s++) {
    for (int b = 0; b < J->nbodies; b++)
      if (generate_map(J, &J->bodies[b]) != 0) return -1;
    for (int b = 0; b < J->nbodies; b++) map_points_to_nodes(J, &J->bodies[b]);
    /* CartesianFrictionalBox::generateRules/applyRules recompute
     * S (m b) - gradS (V T) with the operations of mapPointsToNodes
     * (cartesian_frictional_box.cpp:86-108): the nodal force before contact */
    for (int b = 0; b < J->nbodies; b++)
      if (J->bodies[b].has_boundary == 3)
        memcpy(J->bodies[b].bc_force, J->bodies[b].nf, 3 * (size_t)J->node_count * sizeof(double));
    for (int c = 0; c < J->ncontacts; c++) contact_generate(J, &J->contacts[c]);
    for (int c = 0; c < J->ncontacts; c++) contact_apply(J, &J->contacts[c]);
    for (int b = 0; b < J->nbodies; b++)
      if (J->bodies[b].has_boundary) boundary_apply(J, &J->bodies[b]);
    for (int b = 0; b < J->nbodies; b++) move_grid(J, &J->bodies[b]);
    for (int b = 0; b < J->nbodies; b++) move_points(J, &J->bodies[b]);
    for (int b = 0; b < J->nbodies; b++) strain_rate(J, &J->bodies[b]);
    for (int b = 0; b < J->nbodies; b++) update_density(J, &J->bodies[b]);
    apply_gravity(J);
    for (int b = 0; b < J->nbodies; b++)
      if (J->bodies[b].has_material) update_stress(J, &J->bodies[b]);
    J->t += J->dt;
  }
  return 0;
}

/* Rebuilds the maps for the current positions without stepping. */
int oc_build_map(void* hp) {
  oc_job* J = (oc_job*)hp;
  for (int b = 0; b < J->nbodies; b++)
    if (generate_map(J, &J->bodies[b]) != 0) return -1;
  return 0;
}

int oc_num_nodes(void* hp) { return ((oc_job*)hp)->node_count; }

int oc_get_point_field(void* hp, int b, const char* name, double* out) {
  oc_job* J = (oc_job*)hp;
  oc_body* B = &J->bodies[b];
  size_t n = (size_t)B->n;
  if (!strcmp(name, "x")) return memcpy(out, B->x, 24 * n), 3;
  if (!strcmp(name, "u")) return memcpy(out, B->u, 24 * n), 3;
  if (!strcmp(name, "x_t")) return memcpy(out, B->x_t, 24 * n), 3;
  if (!strcmp(name, "mx_t")) return memcpy(out, B->mx_t, 24 * n), 3;
  if (!strcmp(name, "b")) return memcpy(out, B->b, 24 * n), 3;
  if (!strcmp(name, "L")) return memcpy(out, B->L, 72 * n), 9;
  if (!strcmp(name, "T")) return memcpy(out, B->T, 72 * n), 9;
  if (!strcmp(name, "m")) return memcpy(out, B->m, 8 * n), 1;
  if (!strcmp(name, "v")) return memcpy(out, B->v, 8 * n), 1;
  if (!strcmp(name, "v0")) return memcpy(out, B->v0, 8 * n), 1;
  if (!strcmp(name, "extent")) return memcpy(out, B->extent, 8 * n), 1;
  if (B->material_kind == 2 && !strcmp(name, "gammap")) return memcpy(out, B->gammap, 8 * n), 1;
  if (B->material_kind == 2 && !strcmp(name, "gammap_dot")) return memcpy(out, B->gammap_dot, 8 * n), 1;
  if (!strcmp(name, "active")) {
    for (size_t p = 0; p < n; p++) out[p] = B->active[p];
    return 1;
  }
  return -1;
}

int oc_get_node_field(void* hp, int b, const char* name, double* out) {
  oc_job* J = (oc_job*)hp;
  oc_body* B = &J->bodies[b];
  size_t N = (size_t)J->node_count;
  if (!strcmp(name, "x")) return memcpy(out, B->nx, 24 * N), 3;
  if (!strcmp(name, "u")) return memcpy(out, B->nu, 24 * N), 3;
  if (!strcmp(name, "x_t")) return memcpy(out, B->nx_t, 24 * N), 3;
  if (!strcmp(name, "mx_t")) return memcpy(out, B->nmx_t, 24 * N), 3;
  if (!strcmp(name, "f")) return memcpy(out, B->nf, 24 * N), 3;
  if (!strcmp(name, "diff_x_t")) return memcpy(out, B->ndiff, 24 * N), 3;
  if (!strcmp(name, "m")) return memcpy(out, B->nm, 8 * N), 1;
  return -1;
}

int oc_get_contact_field(void* hp, int c, const char* name, double* out) {
  oc_job* J = (oc_job*)hp;
  oc_contact* C = &J->contacts[c];
  size_t N = (size_t)J->node_count;
  if (!strcmp(name, "normal")) return memcpy(out, C->normal, 24 * N), 3;
  if (!strcmp(name, "force")) return memcpy(out, C->force, 24 * N), 3;
  return -1;
}

int oc_map_size(void* hp, int b) { return ((oc_job*)hp)->bodies[b].nnz; }
int oc_grad_map_size(void* hp, int b) { return ((oc_job*)hp)->bodies[b].gnnz; }
int oc_get_map(void* hp, int b, int* node, int* point, double* val) {
  oc_body* B = &((oc_job*)hp)->bodies[b];
  memcpy(node, B->S_i, sizeof(int) * (size_t)B->nnz);
  memcpy(point, B->S_j, sizeof(int) * (size_t)B->nnz);
  memcpy(val, B->S_v, sizeof(double) * (size_t)B->nnz);
  return B->nnz;
}
int oc_get_grad_map(void* hp, int b, int* node, int* point, double* grad) {
  oc_body* B = &((oc_job*)hp)->bodies[b];
  memcpy(node, B->G_i, sizeof(int) * (size_t)B->gnnz);
  memcpy(point, B->G_j, sizeof(int) * (size_t)B->gnnz);
  memcpy(grad, B->G_v, sizeof(double) * 3 * (size_t)B->gnnz);
  return B->gnnz;
}

void oc_destroy(void* hp) {
  oc_job* J = (oc_job*)hp;
  if (!J) return;
  for (int b = 0; b < J->nbodies; b++) {
    oc_body* B = &J->bodies[b];
    free(B->x); free(B->u); free(B->x_t); free(B->mx_t); free(B->b);
    free(B->L); free(B->F); free(B->T); free(B->gammap); free(B->gammap_dot); free(B->m); free(B->v); free(B->v0);
    free(B->extent); free(B->active); free(B->nx); free(B->nu); free(B->nx_t);
    free(B->nmx_t); free(B->nf); free(B->ndiff); free(B->nm); free(B->bc_mask); free(B->bc_force);
    free(B->S_i); free(B->S_j); free(B->S_v); free(B->G_i); free(B->G_j); free(B->G_v);
  }
  for (int c = 0; c < J->ncontacts; c++) {
    free(J->contacts[c].normal);
    free(J->contacts[c].force);
  }
  free(J->x_n);
  free(J->nodeIDs);
  free(J);
}
