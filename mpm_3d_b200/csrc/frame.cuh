// Frame conversion on the device: a body's point, node and contact fields
// written in the reference's layout and order (points by original index,
// 3 doubles per vector and 9 per tensor; nodes i + j (Nx+1) + k (Nx+1)(Ny+1))
// into one staging buffer, which the host then copies in one piece. The
// values are those of the one-field downloads (mpmgpu_download_*).
#pragma once

#include "geom.cuh"
#include "state.cuh"

namespace mpmb200 {

// Offsets (in doubles) of one body's point fields in a frame; -1 = absent.
struct FramePointLayout {
  int64_t x, u, xt, mxt, T, v, m, ext, active, L, gammap, gammap_dot;
};

// Offsets of one body's node fields; -1 = absent.
struct FrameNodeLayout {
  int64_t m, mxt, f, xt, u, dxt;
};

// One thread per stored point: the point's fields at its original index.
template <typename PT>
__global__ void k_frame_points(PointsT<PT> P, int dim, FramePointLayout o, double* out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P.n; p += stride) {
    const int64_t q = P.pid[p];
    // the mixed form's x, x_t and m are two-word values (hi + lo)
    const double m = two_word(P.m, P.ml, p);
    for (int d = 0; d < 3; d++) {
      const bool on = d < dim;
      const double x = on ? two_word(P.x[d], P.xl[d], p) : 0.0;
      const double xt = on ? two_word(P.v[d], P.vl[d], p) : 0.0;
      out[o.x + 3 * q + d] = x;
      out[o.u + 3 * q + d] = on ? (double)P.u[d][p] : 0.0;
      out[o.xt + 3 * q + d] = xt;
      // movePoints: mx_t = m * x_t (explicit_usl.cpp:295-297)
      out[o.mxt + 3 * q + d] = m * xt;
    }
    const int idx[9] = {0, 3, 5, 3, 1, 4, 5, 4, 2};   // row-major 3x3 from xx yy zz xy yz xz
    for (int k = 0; k < 9; k++) out[o.T + 9 * q + k] = (double)P.s[idx[k]][p];
    out[o.v + q] = (double)P.vol[p];
    out[o.m + q] = m;
    out[o.ext + q] = (double)P.ext[p];
    // 2 = left the domain at the last move: active until the next map build
    out[o.active + q] = P.active[p] != 0 ? 1.0 : 0.0;
    if (o.L >= 0)
      for (int k = 0; k < 9; k++) out[o.L + 9 * q + k] = P.L[9 * p + k];
    if (o.gammap >= 0) {
      out[o.gammap + q] = (double)P.ms[0][p];
      out[o.gammap_dot + q] = (double)P.ms[1][p];
    }
  }
}

// One thread per reference node: the body's nodal fields (zero in node
// blocks that were not active in the last step).
__global__ void k_frame_nodes(Geom g, double dt, const uint8_t* act, NodesAcc snap, NodesVel V, FrameNodeLayout o,
                              double* out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < g.nnodes; id += stride) {
    const int i = (int)(id % g.nn[0]);
    const int64_t r = id / g.nn[0];
    const int j = (int)(r % g.nn[1]);
    const int k = (int)(r / g.nn[1]);
    const bool on = act[node_block(g, i, j, k)] != 0;
    const int64_t s = node_slot(g, i, j, k);
    if (o.m >= 0) out[o.m + id] = on ? snap.m[s] : 0.0;
    for (int d = 0; d < 3; d++) {
      const bool dd = on && d < g.dim;
      if (o.mxt >= 0) out[o.mxt + 3 * id + d] = dd ? snap.mx[d][s] : 0.0;
      if (o.f >= 0) out[o.f + 3 * id + d] = dd ? snap.f[d][s] : 0.0;
      const double vt = dd ? V.vt[d][s] : 0.0;
      out[o.xt + 3 * id + d] = vt;
      // moveGrid: u = dt * x_t (explicit_usl.cpp:252)
      out[o.u + 3 * id + d] = dt * vt;
      out[o.dxt + 3 * id + d] = dd ? V.dv[d][s] : 0.0;
    }
  }
}

// One thread per reference node: a contact's normal or force (3 per slot on
// the device). The reference normalises every node's normal, so a node
// without mass reads 0 * (1/0) = NaN there in the grid's axes.
__global__ void k_frame_contact(Geom g, int primed, const uint8_t* act, const double* src, int normal,
                                double* out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < g.nnodes; id += stride) {
    const int i = (int)(id % g.nn[0]);
    const int64_t r = id / g.nn[0];
    const int j = (int)(r % g.nn[1]);
    const int k = (int)(r / g.nn[1]);
    const bool on = primed && act != nullptr && act[node_block(g, i, j, k)] != 0;
    const int64_t s = node_slot(g, i, j, k);
    for (int d = 0; d < 3; d++)
      out[3 * id + d] = on ? src[3 * s + d] : (normal ? (d < g.dim ? nan : 0.0) : 0.0);
  }
}

}  // namespace mpmb200
