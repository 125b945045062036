// Triplet-exact S / gradS rows in the reference's own operation order, for
// the connectivity export (mpmgpu_dump_map). Every floating-point operation
// is an explicit IEEE intrinsic, so nothing is contracted into an FMA and
// each value is bit-identical to the reference compiled without contraction.
#pragma once

#include "geom.cuh"

namespace mpmb200 {

// cartesianWhichElement, cartesian.cpp:219-240, including the integer
// accumulation of the per-axis floors.
template <int DIM>
__device__ __forceinline__ int which_element_exact(const Geom& g, const double* x) {
  int e = (int)floor(__dmul_rn(__ddiv_rn(x[0], g.L[0]), (double)g.N[0]));
#pragma unroll
  for (int i = 0; i < DIM; i++) {
    if (!(x[i] < g.L[i] && x[i] >= 0.0)) return -1;
    if (i == 1) {
      const double f = floor(__dmul_rn(__ddiv_rn(x[1], g.L[1]), (double)g.N[1]));
      e = (int)__dadd_rn((double)e, __dmul_rn(f, (double)g.N[0]));
    } else if (i == 2) {
      const double f = floor(__dmul_rn(__ddiv_rn(x[2], g.L[2]), (double)g.N[2]));
      e = (int)__dadd_rn((double)e, __dmul_rn(__dmul_rn(f, (double)g.N[1]), (double)g.N[0]));
    }
  }
  return e;
}

// nodeIDs(e, n) of hiddenInit, cartesian.cpp:114-141.
template <int DIM>
__device__ __forceinline__ int element_node(const Geom& g, int e, int n) {
  int ijk[3] = {0, 0, 0};
  int tmp = e;
#pragma unroll
  for (int i = 0; i < DIM; i++) {
    ijk[i] = tmp % g.N[i];
    tmp = tmp / g.N[i];
  }
  int id = 0;
#pragma unroll
  for (int i = 0; i < DIM; i++) {
    const int a = (n >> i) & 1;
    if (i == 0) id += ijk[0] + a;
    else if (i == 1) id += (ijk[1] + a) * (g.N[0] + 1);
    else id += (ijk[2] + a) * (g.N[1] + 1) * (g.N[0] + 1);
  }
  return id;
}

// nodeIDToPosition component d, cartesian.cpp:258-274.
template <int DIM>
__device__ __forceinline__ double node_coord(const Geom& g, int id, int d) {
  int tmp = id;
  int ijk = 0;
#pragma unroll
  for (int i = 0; i < DIM; i++) {
    const int v = tmp % (g.N[i] + 1);
    tmp = tmp / (g.N[i] + 1);
    if (i == d) ijk = v;
  }
  return __dmul_rn(g.h[d], (double)ijk);
}

// evaluateBasisFnValue, cartesian.cpp:280-302, for element e at position x:
// writes cp node ids and values.
template <int DIM>
__device__ __forceinline__ void element_values(const Geom& g, int e, const double* x, int* nid, double* val) {
  constexpr int npe = 1 << DIM;
#pragma unroll
  for (int n = 0; n < npe; n++) {
    const int id = element_node<DIM>(g, e, n);
    double tmp = 1.0;
#pragma unroll
    for (int i = 0; i < DIM; i++) {
      const double r = __ddiv_rn(__dsub_rn(x[i], node_coord<DIM>(g, id, i)), g.h[i]);
      tmp = __dmul_rn(tmp, __dsub_rn(1.0, fabs(r)));
    }
    nid[n] = id;
    val[n] = tmp;
  }
}

// Writes the triplets of one point (DefaultPoints::generateMap,
// default_points.cpp:211-324) into its cp*cp slots starting at `slot`, in
// the order the reference appends them. Unused slots get node -1.
// Returns -1 if the point is outside the domain (caller deactivates it).
template <int DIM>
__device__ int export_point(const Geom& g, int cpdi_spec, const double* x, double extent, int32_t* node_out,
                            double* s_out, double* g_out, int64_t slot) {
  constexpr int cp = 1 << DIM;
  for (int k = 0; k < cp * cp; k++) node_out[slot + k] = -1;
  if (!in_domain<DIM>(g, x)) return -1;
  int cpdi = cpdi_spec;
  const double half_ext = __dmul_rn(0.5, extent);
  if (cpdi == 1) {
    for (int c = 0; c < cp; c++) {
      double corner[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int d = 0; d < DIM; d++) corner[d] = __dadd_rn(x[d], __dmul_rn(half_ext, ((c >> d) & 1) ? 1.0 : -1.0));
      if (!in_domain<DIM>(g, corner)) {
        cpdi = 0;
        break;
      }
    }
  }
  int nid[8];
  double val[8];
  int64_t k = slot;
  if (cpdi == 0) {
    const int e = which_element_exact<DIM>(g, x);
    if (e < 0) return 0;
    element_values<DIM>(g, e, x, nid, val);
    for (int n = 0; n < cp; n++, k++) {
      double r[3] = {0.0, 0.0, 0.0};
      double tmp = 1.0;
#pragma unroll
      for (int i = 0; i < DIM; i++) {
        r[i] = __ddiv_rn(__dsub_rn(x[i], node_coord<DIM>(g, nid[n], i)), g.h[i]);
        tmp = __dmul_rn(tmp, __dsub_rn(1.0, fabs(r[i])));
      }
      node_out[k] = nid[n];
      s_out[k] = val[n];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        double gi = 0.0;
        if (i < DIM) {
          // -tmp / (1 - |r|) * r / |r| / h, cartesian.cpp:329-332
          gi = __ddiv_rn(__ddiv_rn(__dmul_rn(__ddiv_rn(-tmp, __dsub_rn(1.0, fabs(r[i]))), r[i]), fabs(r[i])), g.h[i]);
          if (fabs(r[i]) >= 1.0) gi = 0.0;
        }
        g_out[3 * k + i] = gi;
      }
    }
    return 1;
  }
  const double denom = __dmul_rn(__dmul_rn((double)cp, 0.5), extent);
  for (int c = 0; c < cp; c++) {
    double corner[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < DIM; d++) corner[d] = __dadd_rn(x[d], __dmul_rn(half_ext, ((c >> d) & 1) ? 1.0 : -1.0));
    const int e = which_element_exact<DIM>(g, corner);
    if (e < 0) continue;
    element_values<DIM>(g, e, corner, nid, val);
    for (int n = 0; n < cp; n++, k++) {
      node_out[k] = nid[n];
      s_out[k] = __ddiv_rn(val[n], (double)cp);
#pragma unroll
      for (int i = 0; i < 3; i++)
        g_out[3 * k + i] = (i < DIM) ? __dmul_rn(__ddiv_rn(val[n], denom), ((c >> i) & 1) ? 1.0 : -1.0) : 0.0;
    }
  }
  return 1;
}

}  // namespace mpmb200
