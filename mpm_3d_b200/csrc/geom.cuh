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
// summed hat values W and signed sums G.
struct AxisMap {
  int base;
  int span;
  double W[3];
  double G[3];
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
struct PointMap {
  AxisMap ax[3];
  double sS;
  double sG;
};

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

// Hat value 1 - |(c - h*idx)/h| of cartesian.cpp:292-295.
__device__ __forceinline__ double hat(const Geom& g, int d, double c, int idx) {
  const double xn = __dmul_rn(g.h[d], (double)idx);
  const double r = __ddiv_rn(__dsub_rn(c, xn), g.h[d]);
  return __dsub_rn(1.0, fabs(r));
}

// Builds the separable map of one point, following the decisions of
// DefaultPoints::generateMap (default_points.cpp:211-236).
// Returns -1 if the point is outside the domain (the caller deactivates it),
// 0 if it has no triplets (whichElement fails), 1 otherwise.
template <int DIM>
__device__ __forceinline__ int build_map(const Geom& g, int cpdi_spec, const double* x, double extent, PointMap& pm,
                                         int* err) {
  if (!in_domain<DIM>(g, x)) return -1;
  int cpdi = cpdi_spec;
  const double a = __dmul_rn(0.5, extent);
  double clo[3], chi[3];
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    clo[d] = __dadd_rn(x[d], __dmul_rn(a, -1.0));
    chi[d] = __dadd_rn(x[d], __dmul_rn(a, 1.0));
  }
  if (cpdi == 1) {
#pragma unroll
    for (int d = 0; d < DIM; d++)
      if (!(clo[d] <= g.L[d] && clo[d] >= 0.0) || !(chi[d] <= g.L[d] && chi[d] >= 0.0)) cpdi = 0;
  }
  if (cpdi == 1) {
    // whichElement accepts x < L only; a hi corner exactly at L has no
    // element and contributes nothing (cartesian.cpp:228-230, 284-286).
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      AxisMap& A = pm.ax[d];
      const int elo = axis_element(g, d, clo[d]);
      const bool hi_ok = chi[d] < g.L[d];
      const int ehi = hi_ok ? axis_element(g, d, chi[d]) : elo;
      if (elo >= g.N[d] || (hi_ok && ehi >= g.N[d])) atomicOr(err, kErrElemAlias);
      const int delta = ehi - elo;
      if (delta > 1 || delta < 0) atomicOr(err, kErrWideSpan);
      A.base = elo;
      A.span = 2 + (hi_ok && delta == 1 ? 1 : 0);
      const double wl0 = hat(g, d, clo[d], elo), wl1 = hat(g, d, clo[d], elo + 1);
      A.W[0] = wl0;
      A.W[1] = wl1;
      A.W[2] = 0.0;
      A.G[0] = -wl0;
      A.G[1] = -wl1;
      A.G[2] = 0.0;
      if (hi_ok) {
        const double wh0 = hat(g, d, chi[d], ehi), wh1 = hat(g, d, chi[d], ehi + 1);
        const int o = (delta == 1) ? 1 : 0;
        A.W[o] += wh0;
        A.W[o + 1] += wh1;
        A.G[o] += wh0;
        A.G[o + 1] += wh1;
      }
    }
    pm.sS = 1.0 / (double)g.cp;
    pm.sG = 1.0 / ((g.cp * 0.5) * extent);
    return 1;
  }
  // CPDI_OFF: plain hat functions at x, evaluateBasisFnValue/Gradient.
#pragma unroll
  for (int d = 0; d < DIM; d++)
    if (!(x[d] < g.L[d] && x[d] >= 0.0)) return 0;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    AxisMap& A = pm.ax[d];
    const int e = axis_element(g, d, x[d]);
    if (e >= g.N[d]) atomicOr(err, kErrElemAlias);
    A.base = e;
    A.span = 2;
#pragma unroll
    for (int o = 0; o < 2; o++) {
      const double xn = __dmul_rn(g.h[d], (double)(e + o));
      const double r = __ddiv_rn(__dsub_rn(x[d], xn), g.h[d]);
      A.W[o] = __dsub_rn(1.0, fabs(r));
      // -sign(r)/h, NaN at r == 0 and 0 for |r| >= 1, as cartesian.cpp:329-332
      A.G[o] = (fabs(r) >= 1.0) ? 0.0 : -(r / fabs(r)) / g.h[d];
    }
    A.W[2] = 0.0;
    A.G[2] = 0.0;
  }
  pm.sS = 1.0;
  pm.sG = 1.0;
  return 1;
}

}  // namespace mpmb200
