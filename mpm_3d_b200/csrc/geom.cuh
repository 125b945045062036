// Grid geometry, node storage layout and the per-point shape-function map of
// the explicit MPM step (CartesianLinear + DefaultPoints of mpm_3d).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mpmb200 {

constexpr int kMaxBodies = 8;
constexpr int kMaxContacts = 8;

// Device error flags (bit mask in one int).
constexpr int kErrWideSpan = 1;     // corner spread wider than one cell
constexpr int kErrElemAlias = 2;    // floor(x/L*N) == N for x < L (reference UB)
constexpr int kErrItemCap = 8;      // a work item larger than the kernel's points per item

// Uniform Cartesian grid (CartesianLinear, src/objects/grids/cartesian.cpp)
// and its node storage. Nodes are stored block-linear: blocks of
// 4x4x4 nodes (3D) or 8x8 nodes (2D), 64 nodes per block, each block
// contiguous in every nodal array, so a block of the grid update is one
// coalesced 512-byte segment per FP64 array.
struct Geom {
  int dim;
  double L[3];      // domain lengths
  double h[3];      // L/N, cartesian.cpp:40
  int N[3];         // cells per axis
  int nn[3];        // nodes per axis (N+1); 1 for an unused axis
  int bsh[3];       // log2 of block extent per axis
  int nb[3];        // blocks per axis
  int64_t nblocks;  // total node blocks
  int64_t nslots;   // nblocks * 64
  int cp;           // corners per point, 2^dim
  int64_t nnodes;   // reference node count, prod(N+1)
};

__host__ __device__ __forceinline__ int64_t node_slot(const Geom& g, int i, int j, int k) {
  const int bi = i >> g.bsh[0], bj = j >> g.bsh[1], bk = k >> g.bsh[2];
  const int li = (i & ((1 << g.bsh[0]) - 1)) | ((j & ((1 << g.bsh[1]) - 1)) << g.bsh[0]) |
                 ((k & ((1 << g.bsh[2]) - 1)) << (g.bsh[0] + g.bsh[1]));
  const int64_t blk = bi + (int64_t)g.nb[0] * (bj + (int64_t)g.nb[1] * bk);
  return blk * 64 + li;
}

__host__ __device__ __forceinline__ int64_t node_block(const Geom& g, int i, int j, int k) {
  return (i >> g.bsh[0]) + (int64_t)g.nb[0] * ((j >> g.bsh[1]) + (int64_t)g.nb[1] * (k >> g.bsh[2]));
}

// Inverse of node_slot: grid indices of local node li in block blk.
__host__ __device__ __forceinline__ void slot_ijk(const Geom& g, int64_t blk, int li, int& i, int& j, int& k) {
  const int bi = (int)(blk % g.nb[0]);
  const int64_t r = blk / g.nb[0];
  const int bj = (int)(r % g.nb[1]);
  const int bk = (int)(r / g.nb[1]);
  const int mx = (1 << g.bsh[0]) - 1, my = (1 << g.bsh[1]) - 1;
  i = (bi << g.bsh[0]) + (li & mx);
  j = (bj << g.bsh[1]) + ((li >> g.bsh[0]) & my);
  k = (bk << g.bsh[2]) + (li >> (g.bsh[0] + g.bsh[1]));
}

// One axis of a point's shape-function window: nodes base..base+span-1 with
// summed hat values W and signed sums G (R: double for the FP64 form, float
// for the mixed form).
template <typename R>
struct AxisMapT {
  int base;
  int span;
  R W[3];
  R G[3];
};

// The S / gradS rows of one point in separable form. For the corner-sampled
// map (CPDI_ON), the reference's S value of a (corner c, element node n)
// triplet is prod_d w_d(c,n) / cp and its gradient component d is
// (prod_d' w_d'(c,n)) / ((cp/2) * extent) * A(c,d)
// (default_points.cpp:264-324). Corners enumerate every lo/hi combination
// per axis and element nodes every 0/1 offset per axis, so the sum of all
// triplets that land on node k factorises exactly (in real arithmetic) into
//   S(k)      = sS * W_0[k_0] W_1[k_1] W_2[k_2]
//   dS/dx_d(k)= sG * G_d[k_d] prod_{d' != d} W_d'[k_d']
// with W and G the per-axis sums of hat values (G signed by the corner side).
// Point-sampled (CPDI_OFF) rows have the same form with W = hat values at x,
// G = -sign(r)/h (cartesian.cpp:307-357), sS = sG = 1.
template <typename R>
struct PointMapT {
  AxisMapT<R> ax[3];
  R sS;
  R sG;
};
using AxisMap = AxisMapT<double>;
using PointMap = PointMapT<double>;

// inDomain, cartesian.cpp:245-253 (closed interval).
template <int DIM>
__device__ __forceinline__ bool in_domain(const Geom& g, const double* x) {
#pragma unroll
  for (int d = 0; d < DIM; d++)
    if (!(x[d] <= g.L[d] && x[d] >= 0.0)) return false;
  return true;
}

// Per-axis element index of cartesianWhichElement, cartesian.cpp:226-236:
// floor(x / L * N) with explicit IEEE operations (no contraction).
__device__ __forceinline__ int axis_element(const Geom& g, int d, double c) {
  return (int)floor(__dmul_rn(__ddiv_rn(c, g.L[d]), (double)g.N[d]));
}

// Per-grid constants of the fast map.
struct MapConst {
  double NL[3];    // N / L: element index scale
  double invh[3];  // 1 / h
  float invhf[3];  // 1 / h in single precision (the mixed form's point-sampled gradients)
};

// Element index floor(x / L * N) without a division: the product x * (N/L)
// differs from the reference's two roundings by a few ulps, which can only
// change the floor when the value is within that distance of an integer; in
// that band the exact two-rounding form decides.
__device__ __forceinline__ int axis_element_fast(const Geom& g, const MapConst& mc, int d, double c) {
  const double t = c * mc.NL[d];
  const double f = floor(t);
  if (t - f < 1e-9 || (f + 1.0) - t < 1e-9) return axis_element(g, d, c);
  return (int)f;
}

// Builds the separable map of one point with the decisions of
// DefaultPoints::generateMap (default_points.cpp:211-236): corner-sampled
// unless a corner leaves the closed domain, no triplets for a corner (or
// point) without an element, deactivation outside the domain. Hat values are
// computed as (c - x_n) * (1/h), a different rounding of the reference's
// (c - x_n) / h; the element indices, and so the connectivity, are exact
// (axis_element_fast). Triplet-exact values come from exact_map.cuh.
// Returns -1 outside the domain (caller deactivates), 0 without triplets,
// 1 otherwise.
// The gradient scale of the corner-sampled map, 1 / ((cp/2) extent): it
// depends only on the point's extent, so a caller that builds two maps of
// one point computes it once and passes it in.
__device__ __forceinline__ double map_grad_scale(const Geom& g, double extent) {
  return 1.0 / ((g.cp * 0.5) * extent);
}
__device__ __forceinline__ float map_grad_scale(const Geom& g, float extent) {
  return 1.0f / (((float)g.cp * 0.5f) * extent);
}

template <int DIM>
__device__ __forceinline__ int build_map_fast(const Geom& g, const MapConst& mc, int cpdi_spec, const double* x,
                                              double extent, PointMap& pm, int* err, double sG) {
  if (!in_domain<DIM>(g, x)) return -1;
  int cpdi = cpdi_spec;
  const double a = 0.5 * extent;
  double clo[3], chi[3];
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    clo[d] = x[d] - a;
    chi[d] = x[d] + a;
  }
  if (cpdi == 1) {
#pragma unroll
    for (int d = 0; d < DIM; d++)
      if (!(clo[d] <= g.L[d] && clo[d] >= 0.0) || !(chi[d] <= g.L[d] && chi[d] >= 0.0)) cpdi = 0;
  }
  if (cpdi == 1) {
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      AxisMap& A = pm.ax[d];
      const int elo = axis_element_fast(g, mc, d, clo[d]);
      const bool hi_ok = chi[d] < g.L[d];
      const int ehi = hi_ok ? axis_element_fast(g, mc, d, chi[d]) : elo;
      if (elo >= g.N[d] || (hi_ok && ehi >= g.N[d])) {
        // element index rounded up to N for x < L: flagged, and no nodal
        // contributions (its nodes would lie outside the grid)
        atomicOr(err, kErrElemAlias);
        return 0;
      }
      const int delta = ehi - elo;
      if (delta > 1 || delta < 0) atomicOr(err, kErrWideSpan);
      A.base = elo;
      A.span = 2 + (hi_ok && delta == 1 ? 1 : 0);
      const double rl = (clo[d] - g.h[d] * (double)elo) * mc.invh[d];
      const double wl0 = 1.0 - fabs(rl), wl1 = 1.0 - fabs(rl - 1.0);
      double wh0 = 0.0, wh1 = 0.0;
      if (hi_ok) {
        const double rh = (chi[d] - g.h[d] * (double)ehi) * mc.invh[d];
        wh0 = 1.0 - fabs(rh);
        wh1 = 1.0 - fabs(rh - 1.0);
      }
      if (delta == 1) {
        A.W[0] = wl0;
        A.W[1] = wl1 + wh0;
        A.W[2] = wh1;
        A.G[0] = -wl0;
        A.G[1] = wh0 - wl1;
        A.G[2] = wh1;
      } else {
        A.W[0] = wl0 + wh0;
        A.W[1] = wl1 + wh1;
        A.W[2] = 0.0;
        A.G[0] = wh0 - wl0;
        A.G[1] = wh1 - wl1;
        A.G[2] = 0.0;
      }
    }
    pm.sS = 1.0 / (double)g.cp;
    pm.sG = sG;
    return 1;
  }
#pragma unroll
  for (int d = 0; d < DIM; d++)
    if (!(x[d] < g.L[d] && x[d] >= 0.0)) return 0;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    AxisMap& A = pm.ax[d];
    const int e = axis_element_fast(g, mc, d, x[d]);
    if (e >= g.N[d]) {
      atomicOr(err, kErrElemAlias);
      return 0;
    }
    A.base = e;
    A.span = 2;
#pragma unroll
    for (int o = 0; o < 2; o++) {
      const double r = (x[d] - g.h[d] * (double)(e + o)) * mc.invh[d];
      A.W[o] = 1.0 - fabs(r);
      A.G[o] = (fabs(r) >= 1.0) ? 0.0 : -(r / fabs(r)) * mc.invh[d];
    }
    A.W[2] = 0.0;
    A.G[2] = 0.0;
  }
  pm.sS = 1.0;
  pm.sG = 1.0;
  return 1;
}

// Map of the mixed form: the decisions of build_map_fast on the point's
// double position (the two-word value), so that its connectivity is the
// FP64 form's; each corner's offset from its element's first node is taken
// in double and rounded once, and the hat values and their sums are FP32
// arithmetic on it. (Offsets formed in FP32, x - h e with x ~ 1 and h ~
// 1/64, would keep only the bits of x below h: an error of about 4e-6 of a
// hat value per step.)
template <int DIM>
__device__ __forceinline__ int build_map_f32(const Geom& g, const MapConst& mc, int cpdi_spec, const double* x,
                                             float extent, PointMapT<float>& pm, int* err, float sG) {
  if (!in_domain<DIM>(g, x)) return -1;
  int cpdi = cpdi_spec;
  const double a = 0.5 * (double)extent;
  double clo[3], chi[3];
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    clo[d] = x[d] - a;
    chi[d] = x[d] + a;
  }
  if (cpdi == 1) {
#pragma unroll
    for (int d = 0; d < DIM; d++)
      if (!(clo[d] <= g.L[d] && clo[d] >= 0.0) || !(chi[d] <= g.L[d] && chi[d] >= 0.0)) cpdi = 0;
  }
  if (cpdi == 1) {
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      AxisMapT<float>& A = pm.ax[d];
      const int elo = axis_element_fast(g, mc, d, clo[d]);
      const bool hi_ok = chi[d] < g.L[d];
      const int ehi = hi_ok ? axis_element_fast(g, mc, d, chi[d]) : elo;
      if (elo >= g.N[d] || (hi_ok && ehi >= g.N[d])) {
        atomicOr(err, kErrElemAlias);
        return 0;
      }
      const int delta = ehi - elo;
      if (delta > 1 || delta < 0) atomicOr(err, kErrWideSpan);
      A.base = elo;
      A.span = 2 + (hi_ok && delta == 1 ? 1 : 0);
      const float rl = (float)((clo[d] - g.h[d] * (double)elo) * mc.invh[d]);
      const float wl0 = 1.0f - fabsf(rl), wl1 = 1.0f - fabsf(rl - 1.0f);
      float wh0 = 0.0f, wh1 = 0.0f;
      if (hi_ok) {
        const float rh = (float)((chi[d] - g.h[d] * (double)ehi) * mc.invh[d]);
        wh0 = 1.0f - fabsf(rh);
        wh1 = 1.0f - fabsf(rh - 1.0f);
      }
      if (delta == 1) {
        A.W[0] = wl0;
        A.W[1] = wl1 + wh0;
        A.W[2] = wh1;
        A.G[0] = -wl0;
        A.G[1] = wh0 - wl1;
        A.G[2] = wh1;
      } else {
        A.W[0] = wl0 + wh0;
        A.W[1] = wl1 + wh1;
        A.W[2] = 0.0f;
        A.G[0] = wh0 - wl0;
        A.G[1] = wh1 - wl1;
        A.G[2] = 0.0f;
      }
    }
    pm.sS = 1.0f / (float)g.cp;
    pm.sG = sG;
    return 1;
  }
#pragma unroll
  for (int d = 0; d < DIM; d++)
    if (!(x[d] < g.L[d] && x[d] >= 0.0)) return 0;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    AxisMapT<float>& A = pm.ax[d];
    const int e = axis_element_fast(g, mc, d, x[d]);
    if (e >= g.N[d]) {
      atomicOr(err, kErrElemAlias);
      return 0;
    }
    A.base = e;
    A.span = 2;
#pragma unroll
    for (int o = 0; o < 2; o++) {
      const float r = (float)((x[d] - g.h[d] * (double)(e + o)) * mc.invh[d]);
      A.W[o] = 1.0f - fabsf(r);
      A.G[o] = (fabsf(r) >= 1.0f) ? 0.0f : -(r / fabsf(r)) * mc.invhf[d];
    }
    A.W[2] = 0.0f;
    A.G[2] = 0.0f;
  }
  pm.sS = 1.0f;
  pm.sG = 1.0f;
  return 1;
}

// One map builder per point precision.
template <int DIM>
__device__ __forceinline__ int build_map(const Geom& g, const MapConst& mc, int cpdi, const double* x, double ext,
                                         PointMapT<double>& pm, int* err) {
  return build_map_fast<DIM>(g, mc, cpdi, x, ext, pm, err, map_grad_scale(g, ext));
}
template <int DIM>
__device__ __forceinline__ int build_map(const Geom& g, const MapConst& mc, int cpdi, const double* x, double ext,
                                         PointMapT<double>& pm, int* err, double sG) {
  return build_map_fast<DIM>(g, mc, cpdi, x, ext, pm, err, sG);
}
template <int DIM>
__device__ __forceinline__ int build_map(const Geom& g, const MapConst& mc, int cpdi, const double* x, float ext,
                                         PointMapT<float>& pm, int* err) {
  return build_map_f32<DIM>(g, mc, cpdi, x, ext, pm, err, map_grad_scale(g, ext));
}
template <int DIM>
__device__ __forceinline__ int build_map(const Geom& g, const MapConst& mc, int cpdi, const double* x, float ext,
                                         PointMapT<float>& pm, int* err, float sG) {
  return build_map_f32<DIM>(g, mc, cpdi, x, ext, pm, err, sG);
}

}  // namespace mpmb200
