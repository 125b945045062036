// Fused gather + point update + scatter kernel (G2P of step n, then the map
// build and P2G of step n+1), one pass over the points per step.
//
// A CTA works on one work item at a time: up to kCap points of one bin
// (B^dim cells). Per work item:
//   0. one thread issues bulk asynchronous copies (cp.async.bulk, completed
//      on an mbarrier) of the item's 19 point arrays into shared memory,
//      while the other threads stage the nodal velocities of the bin's node
//      tile ((B+3)^dim nodes) in shared memory;
//   1. every point gathers from the tile and updates its state (x, u, x_t,
//      V, stress); results go to global memory and back into the staged
//      copy;
//   2. the tile is cleared, every point builds its map at the new position
//      and adds its contributions with FP64 shared-memory atomics (points of
//      one warp lie in distinct cells: few same-address conflicts). Windows
//      of two nodes per axis inside the tile (the common case) take a
//      straight-line path with the force evaluated per window row;
//   3. the tile is added into the global nodal accumulators, one global
//      atomic per touched node and value.
// No phase waits on DRAM latency per point: the point state arrives in bulk
// and both phases read it from shared memory. Points whose window leaves the
// tile (drift since the last binning) use global memory and are counted.
#pragma once

#include "async_copy.cuh"
#include "geom.cuh"
#include "kernels_fp64.cuh"
#include "sort.cuh"
#include "state.cuh"

namespace mpmb200 {

struct FusedParams {
  Geom g;
  MapConst mc;
  BinGeom bg;
  StepParams sp;
  MaterialParams mat;
  PointsDev P;
  NodesVel V;
  NodesAcc A;
  const int32_t* work_bin;
  const int32_t* work_start;
  const int32_t* work_end;
  const int32_t* nwork;
  uint32_t* flags;
  int* err;
  unsigned long long* drift;
  int do_g2p;
  int do_p2g;
};

// Points per work item and the staged copy's row stride (slack for the
// alignment of the bulk copies: starts rounded down to 16 bytes).
constexpr int kCap = 512;
constexpr int kCapRow = kCap + 8;
// Staged point arrays: x0..2 v0..2 u0..2 s0..5 vol m ext (doubles), active.
constexpr int kFx = 0, kFv = 3, kFu = 6, kFs = 9, kFvol = 15, kFm = 16, kFext = 17, kNF = 18;

// Number of accumulated values per node: m, mx (3), f (3), contact normal (3).
__host__ __device__ constexpr int fused_nacc(bool normal) { return normal ? 10 : 7; }

template <int DIM, int B>
__host__ __device__ constexpr int fused_tile_nodes() {
  return DIM == 3 ? (B + 3) * (B + 3) * (B + 3) : (B + 3) * (B + 3);
}

// Shared memory layout: mbarrier | points [kNF][kCapRow] | active [kCapRow]
// | tile [max(6, NACC)][TN] | touched [TN].
constexpr size_t kOffPts = 16;
constexpr size_t kOffAct = kOffPts + sizeof(double) * kNF * kCapRow;
constexpr size_t kOffTile = kOffAct + sizeof(int32_t) * kCapRow;

template <int DIM, int B>
size_t fused_smem_bytes(bool normal) {
  constexpr int TN = fused_tile_nodes<DIM, B>();
  const int vals = fused_nacc(normal) > 6 ? fused_nacc(normal) : 6;
  return kOffTile + (size_t)vals * TN * sizeof(double) + (size_t)TN;
}

// Threads per CTA and minimum resident CTAs per SM of the fused kernel
// (2 CTAs of 256 threads: 128 registers per thread, ~105 KB shared each).
#ifndef MPMB200_FUSED_THREADS
#define MPMB200_FUSED_THREADS 256
#endif
#ifndef MPMB200_FUSED_MIN_CTAS
#define MPMB200_FUSED_MIN_CTAS 2
#endif
constexpr int kFusedThreads = MPMB200_FUSED_THREADS;

// Visits the window nodes of a point map: f(k0, k1, k2). Spans are 2 or 3
// per axis; the first two offsets of every axis are unconditional.
template <int DIM, typename F>
__device__ __forceinline__ void for_window(const PointMap& pm, F&& f) {
  constexpr int K2 = DIM == 3 ? 3 : 1;
#pragma unroll
  for (int k2 = 0; k2 < K2; k2++) {
    if (DIM == 3 && k2 == 2 && pm.ax[2].span < 3) break;
#pragma unroll
    for (int k1 = 0; k1 < 3; k1++) {
      if (k1 == 2 && pm.ax[1].span < 3) break;
#pragma unroll
      for (int k0 = 0; k0 < 3; k0++) {
        if (k0 == 2 && pm.ax[0].span < 3) break;
        f(k0, k1, k2);
      }
    }
  }
}

template <int DIM>
__device__ __forceinline__ bool window_in_tile(const PointMap& pm, const int* o, int T) {
  bool in = true;
#pragma unroll
  for (int d = 0; d < DIM; d++) in = in && pm.ax[d].base >= o[d] && pm.ax[d].base + pm.ax[d].span <= o[d] + T;
  return in;
}

// Gathered sums of one point: S^T x_t (du, before the dt factor), S^T
// diff_x_t (dv) and the velocity gradient L_ab = sum v_a dS/dx_b.
struct GatherSum {
  double du[3] = {0.0, 0.0, 0.0};
  double dv[3] = {0.0, 0.0, 0.0};
  double L[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
};

// The common window: two nodes per axis, inside the staged tile.
template <int DIM>
__device__ __forceinline__ bool regular_window(const PointMap& pm, const int* o, int T) {
  bool r = true;
#pragma unroll
  for (int d = 0; d < DIM; d++) r = r && pm.ax[d].span == 2 && pm.ax[d].base >= o[d] && pm.ax[d].base + 2 <= o[d] + T;
  return r;
}

// Gather over a regular (2^dim-node, in-tile) window: straight-line code.
template <int DIM, int T, int TN>
__device__ __forceinline__ GatherSum gather_regular(const PointMap& pm, const int* o, const double* tvel) {
  GatherSum gs;
  const int t0 = (pm.ax[0].base - o[0]) + T * ((pm.ax[1].base - o[1]) + (DIM == 3 ? T * (pm.ax[2].base - o[2]) : 0));
  const double W0s[2] = {pm.sS * pm.ax[0].W[0], pm.sS * pm.ax[0].W[1]};
  const double G0g[2] = {pm.sG * pm.ax[0].G[0], pm.sG * pm.ax[0].G[1]};
  const double W0g[2] = {pm.sG * pm.ax[0].W[0], pm.sG * pm.ax[0].W[1]};
  constexpr int K2 = DIM == 3 ? 2 : 1;
#pragma unroll
  for (int k2 = 0; k2 < K2; k2++) {
    const double wz = DIM == 3 ? pm.ax[2].W[k2] : 1.0;
    const double gz = DIM == 3 ? pm.ax[2].G[k2] : 0.0;
#pragma unroll
    for (int k1 = 0; k1 < 2; k1++) {
      const double W12 = pm.ax[1].W[k1] * wz;
      const double G1W2 = pm.ax[1].G[k1] * wz;
      const double W1G2 = pm.ax[1].W[k1] * gz;
#pragma unroll
      for (int k0 = 0; k0 < 2; k0++) {
        const int t = t0 + k0 + T * (k1 + T * k2);
        const double S = W0s[k0] * W12;
        const double gr0 = G0g[k0] * W12, gr1 = W0g[k0] * G1W2, gr2 = W0g[k0] * W1G2;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const double vt = tvel[d * TN + t];
          gs.du[d] += S * vt;
          gs.dv[d] += S * tvel[(3 + d) * TN + t];
          gs.L[d][0] += vt * gr0;
          gs.L[d][1] += vt * gr1;
          if (DIM == 3) gs.L[d][2] += vt * gr2;
        }
      }
    }
  }
  return gs;
}

// Gather over any window (three-node spans, nodes outside the tile).
template <int DIM, int T, int TN>
__device__ __forceinline__ GatherSum gather_general(const FusedParams& fp, const PointMap& pm, const int* o,
                                                    const double* tvel) {
  GatherSum gs;
  const Geom& g = fp.g;
  const bool in_tile = window_in_tile<DIM>(pm, o, T);
  if (!in_tile) atomicAdd(fp.drift, 1ull);
  const int t0 = (pm.ax[0].base - o[0]) + T * ((pm.ax[1].base - o[1]) + (DIM == 3 ? T * (pm.ax[2].base - o[2]) : 0));
  const double sS = pm.sS, sG = pm.sG;
  for_window<DIM>(pm, [&](int k0, int k1, int k2) {
    const double wz = DIM == 3 ? pm.ax[2].W[k2] : 1.0;
    const double gz = DIM == 3 ? pm.ax[2].G[k2] : 0.0;
    const double W12 = pm.ax[1].W[k1] * wz;
    const double S = sS * pm.ax[0].W[k0] * W12;
    const double gr0 = sG * pm.ax[0].G[k0] * W12;
    const double gw0 = sG * pm.ax[0].W[k0];
    const double gr1 = gw0 * (pm.ax[1].G[k1] * wz);
    const double gr2 = gw0 * (pm.ax[1].W[k1] * gz);
    double vt[3] = {0.0, 0.0, 0.0}, dv[3] = {0.0, 0.0, 0.0};
    if (in_tile) {
      const int t = t0 + k0 + T * (k1 + T * k2);
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        vt[d] = tvel[d * TN + t];
        dv[d] = tvel[(3 + d) * TN + t];
      }
    } else {
      const int64_t s = node_slot(g, pm.ax[0].base + k0, pm.ax[1].base + k1, DIM == 3 ? pm.ax[2].base + k2 : 0);
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        vt[d] = fp.V.vt[d][s];
        dv[d] = fp.V.dv[d][s];
      }
    }
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      gs.du[d] += S * vt[d];
      gs.dv[d] += S * dv[d];
      gs.L[d][0] += vt[d] * gr0;
      gs.L[d][1] += vt[d] * gr1;
      if (DIM == 3) gs.L[d][2] += vt[d] * gr2;
    }
  });
  return gs;
}

// Phase 1 for one point: gather, movePoints / calculateStrainRate /
// updateDensity / updateStress (explicit_usl.cpp:266-355). `sp` points at the
// point's column in the staged arrays (stride kCapRow).
template <int DIM, int T, int TN>
__device__ __forceinline__ void gather_update(const FusedParams& fp, int64_t p, double* sp, const int* o,
                                              const double* tvel) {
  const Geom& g = fp.g;
  const PointsDev& P = fp.P;
  const double dt = fp.sp.dt;
  double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < DIM; d++) x[d] = sp[(kFx + d) * kCapRow];
  PointMap pm;
  const int st = build_map_fast<DIM>(g, fp.mc, fp.sp.cpdi, x, sp[kFext * kCapRow], pm, fp.err);
  GatherSum gs;
  if (st > 0) {
    if (regular_window<DIM>(pm, o, T))
      gs = gather_regular<DIM, T, TN>(pm, o, tvel);
    else
      gs = gather_general<DIM, T, TN>(fp, pm, o, tvel);
  } else {
    gs = GatherSum{};
  }
  double* du = gs.du;
  double* dvel = gs.dv;
  auto& L = gs.L;
  // movePoints: u_node = dt * x_t_node; x += S^T u, u += S^T u,
  // x_t += S^T diff_x_t (explicit_usl.cpp:279-292)
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    const double dx = dt * du[d];
    const double xn = x[d] + dx;
    const double vn = sp[(kFv + d) * kCapRow] + dvel[d];
    sp[(kFx + d) * kCapRow] = xn;
    sp[(kFv + d) * kCapRow] = vn;
    P.x[d][p] = xn;
    P.v[d][p] = vn;
    P.u[d][p] = sp[(kFu + d) * kCapRow] + dx;
  }
  const double vol = sp[kFvol * kCapRow] * exp(dt * (L[0][0] + L[1][1] + L[2][2]));
  sp[kFvol * kCapRow] = vol;
  P.vol[p] = vol;
  if (fp.mat.has_material) {
    double s6[6];
#pragma unroll
    for (int c = 0; c < 6; c++) s6[c] = sp[(kFs + c) * kCapRow];
    jaumann_update<DIM>(L, s6, fp.mat.G, fp.mat.lambda, dt);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      sp[(kFs + c) * kCapRow] = s6[c];
      P.s[c][p] = s6[c];
    }
  }
  if (P.L != nullptr) {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) P.L[9 * p + 3 * a + b] = L[a][b];
  }
}

// Values a point adds to one tile node, in the order m, mx[0..DIM),
// f[0..DIM), normal[0..DIM); tile_field gives each one's tile row.
template <int DIM, bool NORMAL>
struct NodeVals {
  static constexpr int K = 1 + 2 * DIM + (NORMAL ? DIM : 0);
  double v[K];
};

template <int DIM>
__device__ __forceinline__ constexpr int tile_field(int i) {
  return i == 0 ? 0 : (i <= DIM ? i : (i <= 2 * DIM ? 4 + (i - 1 - DIM) : 7 + (i - 1 - 2 * DIM)));
}

// Adds one node's values to the shared tile (shared-memory FP64 atomics).
// Issuing the compare-and-swap steps of all values together was measured
// slower than the plain atomics (register pressure).
template <int DIM, bool NORMAL, int TN>
__device__ __forceinline__ void tile_add_node(double* tacc, int t, const NodeVals<DIM, NORMAL>& nv) {
#pragma unroll
  for (int i = 0; i < NodeVals<DIM, NORMAL>::K; i++) atomicAdd(tacc + tile_field<DIM>(i) * TN + t, nv.v[i]);
}

// Per-point scatter sources: m, m x_t and V sigma (symmetric 3x3).
struct ScatterSrc {
  double m;
  double mv[3];
  double V3[3][3];
};

// Scatter over a regular (2^dim-node, in-tile) window. The nodal force
// -V sigma . grad S is evaluated per row of the window as
// -(G0 A + W0 B) with A, B the row factors of the separable gradient.
template <int DIM, int T, int TN, bool NORMAL>
__device__ __forceinline__ void scatter_regular(const PointMap& pm, const int* o, const ScatterSrc& q, double* tacc,
                                                uint8_t* touched) {
  const int t0 = (pm.ax[0].base - o[0]) + T * ((pm.ax[1].base - o[1]) + (DIM == 3 ? T * (pm.ax[2].base - o[2]) : 0));
  const double W0s[2] = {pm.sS * pm.ax[0].W[0], pm.sS * pm.ax[0].W[1]};
  const double G0g[2] = {pm.sG * pm.ax[0].G[0], pm.sG * pm.ax[0].G[1]};
  const double W0g[2] = {pm.sG * pm.ax[0].W[0], pm.sG * pm.ax[0].W[1]};
  constexpr int K2 = DIM == 3 ? 2 : 1;
#pragma unroll
  for (int k2 = 0; k2 < K2; k2++) {
    const double wz = DIM == 3 ? pm.ax[2].W[k2] : 1.0;
    const double gz = DIM == 3 ? pm.ax[2].G[k2] : 0.0;
#pragma unroll
    for (int k1 = 0; k1 < 2; k1++) {
      const double W12 = pm.ax[1].W[k1] * wz;
      const double G1W2 = pm.ax[1].G[k1] * wz;
      const double W1G2 = pm.ax[1].W[k1] * gz;
      const double mrow = q.m * W12;
      double mvrow[3], A[3], Bf[3];
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        mvrow[d] = q.mv[d] * W12;
        A[d] = q.V3[d][0] * W12;
        Bf[d] = q.V3[d][1] * G1W2;
        if (DIM == 3) Bf[d] += q.V3[d][2] * W1G2;
      }
#pragma unroll
      for (int k0 = 0; k0 < 2; k0++) {
        const int t = t0 + k0 + T * (k1 + T * k2);
        touched[t] = 1;
        NodeVals<DIM, NORMAL> nv;
        nv.v[0] = W0s[k0] * mrow;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          nv.v[1 + d] = W0s[k0] * mvrow[d];
          nv.v[1 + DIM + d] = -(G0g[k0] * A[d] + W0g[k0] * Bf[d]);
        }
        if constexpr (NORMAL) {
          const double gr[3] = {G0g[k0] * W12, W0g[k0] * G1W2, W0g[k0] * W1G2};
#pragma unroll
          for (int d = 0; d < DIM; d++) nv.v[1 + 2 * DIM + d] = gr[d] * q.m;
        }
        tile_add_node<DIM, NORMAL, TN>(tacc, t, nv);
      }
    }
  }
}

// Scatter over any window (three-node spans, nodes outside the tile, which
// go straight to the global accumulators).
template <int DIM, int T, int TN, bool NORMAL>
__device__ __forceinline__ void scatter_general(const FusedParams& fp, const PointMap& pm, const int* o,
                                                const ScatterSrc& q, double* tacc, uint8_t* touched) {
  const Geom& g = fp.g;
  const bool in_tile = window_in_tile<DIM>(pm, o, T);
  if (!in_tile) {
    atomicAdd(fp.drift, 1ull);
    mark_blocks<DIM>(g, pm, fp.flags);
  }
  const int t0 = (pm.ax[0].base - o[0]) + T * ((pm.ax[1].base - o[1]) + (DIM == 3 ? T * (pm.ax[2].base - o[2]) : 0));
  const double sS = pm.sS, sG = pm.sG;
  for_window<DIM>(pm, [&](int k0, int k1, int k2) {
    const double wz = DIM == 3 ? pm.ax[2].W[k2] : 1.0;
    const double gz = DIM == 3 ? pm.ax[2].G[k2] : 0.0;
    const double W12 = pm.ax[1].W[k1] * wz;
    const double S = sS * pm.ax[0].W[k0] * W12;
    const double gw0 = sG * pm.ax[0].W[k0];
    const double gr[3] = {sG * pm.ax[0].G[k0] * W12, gw0 * (pm.ax[1].G[k1] * wz), gw0 * (pm.ax[1].W[k1] * gz)};
    double val[10];
    val[0] = S * q.m;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      val[1 + d] = S * q.mv[d];
      double fi = q.V3[d][0] * gr[0] + q.V3[d][1] * gr[1];
      if (DIM == 3) fi += q.V3[d][2] * gr[2];
      val[4 + d] = -fi;
      if (NORMAL) val[7 + d] = gr[d] * q.m;
    }
    if (in_tile) {
      const int t = t0 + k0 + T * (k1 + T * k2);
      touched[t] = 1;
      NodeVals<DIM, NORMAL> nv;
#pragma unroll
      for (int i = 0; i < NodeVals<DIM, NORMAL>::K; i++) nv.v[i] = val[tile_field<DIM>(i)];
      tile_add_node<DIM, NORMAL, TN>(tacc, t, nv);
    } else {
      const int64_t s = node_slot(g, pm.ax[0].base + k0, pm.ax[1].base + k1, DIM == 3 ? pm.ax[2].base + k2 : 0);
      atomicAdd(fp.A.m + s, val[0]);
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        atomicAdd(fp.A.mx[d] + s, val[1 + d]);
        atomicAdd(fp.A.f[d] + s, val[4 + d]);
        if (NORMAL) atomicAdd(fp.A.nrm[d] + s, val[7 + d]);
      }
    }
  });
}

// Phase 2 for one point: map build and scatter of mapPointsToNodes
// (explicit_usl.cpp:112-164) and the contact normal of
// ContactHuang::generateRules (contact_huang.cpp:91).
template <int DIM, int T, int TN, bool NORMAL>
__device__ __forceinline__ void map_scatter(const FusedParams& fp, int64_t p, const double* sp, const int* o,
                                            double* tacc, uint8_t* touched) {
  const Geom& g = fp.g;
  double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < DIM; d++) x[d] = sp[(kFx + d) * kCapRow];
  PointMap pm;
  const int st = build_map_fast<DIM>(g, fp.mc, fp.sp.cpdi, x, sp[kFext * kCapRow], pm, fp.err);
  if (st < 0) {
    // outside the domain: inactive from the next map build on
    // (default_points.cpp:217-219); before the first step, at once
    fp.P.active[p] = fp.do_g2p ? 2 : 0;
    return;
  }
  if (st == 0) return;
  const double m = sp[kFm * kCapRow];
  const double vol = sp[kFvol * kCapRow];
  double mv[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < DIM; d++) mv[d] = m * sp[(kFv + d) * kCapRow];
  // V * sigma as a symmetric 3x3 (stored xx yy zz xy yz xz)
  double vs[6];
#pragma unroll
  for (int c = 0; c < 6; c++) vs[c] = (DIM == 3 || c == 0 || c == 1 || c == 3) ? sp[(kFs + c) * kCapRow] * vol : 0.0;
  ScatterSrc src;
  src.m = m;
#pragma unroll
  for (int d = 0; d < 3; d++) src.mv[d] = mv[d];
  const double V3[3][3] = {{vs[0], vs[3], vs[5]}, {vs[3], vs[1], vs[4]}, {vs[5], vs[4], vs[2]}};
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) src.V3[a][b] = V3[a][b];
  if (regular_window<DIM>(pm, o, T))
    scatter_regular<DIM, T, TN, NORMAL>(pm, o, src, tacc, touched);
  else
    scatter_general<DIM, T, TN, NORMAL>(fp, pm, o, src, tacc, touched);
}

template <int DIM, int B, bool NORMAL>
__global__ void __launch_bounds__(MPMB200_FUSED_THREADS, MPMB200_FUSED_MIN_CTAS) k_g2p2g(FusedParams fp) {
  constexpr int T = B + 3;
  constexpr int TN = fused_tile_nodes<DIM, B>();
  constexpr int NACC = fused_nacc(NORMAL);
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  double* pts = reinterpret_cast<double*>(smem + kOffPts);
  int32_t* act = reinterpret_cast<int32_t*>(smem + kOffAct);
  double* tile = reinterpret_cast<double*>(smem + kOffTile);  // phase 1: vt0..2 dv0..2; phase 2: NACC values
  uint8_t* touched = reinterpret_cast<uint8_t*>(tile + (NACC > 6 ? NACC : 6) * TN);

  const Geom& g = fp.g;
  const PointsDev& P = fp.P;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  uint32_t parity = 0;
  const int nwork = *fp.nwork;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const int bin = fp.work_bin[w];
    const int64_t pstart = fp.work_start[w];
    const int n = fp.work_end[w] - (int)pstart;
    // bulk copy windows: 16-byte aligned starts, sizes rounded up to 16 bytes
    const int64_t s8 = pstart & ~(int64_t)1, s4 = pstart & ~(int64_t)3;
    const int off8 = (int)(pstart - s8), off4 = (int)(pstart - s4);
    const int n8 = (off8 + n + 1) & ~1, n4 = (off4 + n + 3) & ~3;
    if (threadIdx.x == 0) {
      const double* src[kNF] = {P.x[0], P.x[1], P.x[2], P.v[0], P.v[1], P.v[2], P.u[0], P.u[1], P.u[2],
                                P.s[0], P.s[1], P.s[2], P.s[3], P.s[4], P.s[5], P.vol, P.m, P.ext};
      fence_async_shared();
      mbar_arrive_expect_tx(bar, (uint32_t)(kNF * n8 * 8 + n4 * 4));
#pragma unroll 1
      for (int f = 0; f < kNF; f++) bulk_copy_g2s(pts + f * kCapRow, src[f] + s8, (uint32_t)(n8 * 8), bar);
      bulk_copy_g2s(act, P.active + s4, (uint32_t)(n4 * 4), bar);
    }
    int o[3] = {0, 0, 0};
    {
      const int bx = bin % fp.bg.nbx;
      const int r = bin / fp.bg.nbx;
      o[0] = bx * B - 1;
      o[1] = (r % fp.bg.nby) * B - 1;
      o[2] = DIM == 3 ? (r / fp.bg.nby) * B - 1 : 0;
    }
    if (fp.do_g2p) {
      for (int t = threadIdx.x; t < TN; t += blockDim.x) {
        const int i = o[0] + t % T, j = o[1] + (t / T) % T, k = DIM == 3 ? o[2] + t / (T * T) : 0;
        if (i < 0 || j < 0 || k < 0 || i >= g.nn[0] || j >= g.nn[1] || k >= g.nn[2]) continue;
        const int64_t s = node_slot(g, i, j, k);
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          tile[d * TN + t] = fp.V.vt[d][s];
          tile[(3 + d) * TN + t] = fp.V.dv[d][s];
        }
      }
    }
    const bool arrived = mbar_wait_bounded(bar, parity, fp.err);
    // one decision for the whole CTA (also the barrier after the tile loads)
    if (__syncthreads_or(arrived ? 0 : 1)) {
      if (!arrived) mbar_wait_bounded(bar, parity, fp.err);  // let copies in flight land before leaving
      return;
    }
    parity ^= 1u;
    if (fp.do_g2p) {
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int64_t p = pstart + j;
        const int a = act[off4 + j];
        if (a == 0) continue;
        if (a == 2) {
          // left the domain at the last move; generateMap deactivates it now
          P.active[p] = 0;
          act[off4 + j] = 0;
          continue;
        }
        gather_update<DIM, T, TN>(fp, p, pts + off8 + j, o, tile);
      }
      __syncthreads();
    }
    if (fp.do_p2g) {
      for (int t = threadIdx.x; t < NACC * TN; t += blockDim.x) tile[t] = 0.0;
      for (int t = threadIdx.x; t < TN; t += blockDim.x) touched[t] = 0;
      __syncthreads();
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        if (act[off4 + j] != 1) continue;
        map_scatter<DIM, T, TN, NORMAL>(fp, pstart + j, pts + off8 + j, o, tile, touched);
      }
      __syncthreads();
      for (int t = threadIdx.x; t < TN; t += blockDim.x) {
        if (!touched[t]) continue;
        const int i = o[0] + t % T, j = o[1] + (t / T) % T, k = DIM == 3 ? o[2] + t / (T * T) : 0;
        const int64_t s = node_slot(g, i, j, k);
        fp.flags[node_block(g, i, j, k)] = 1u;
        atomicAdd(fp.A.m + s, tile[t]);
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          atomicAdd(fp.A.mx[d] + s, tile[(1 + d) * TN + t]);
          atomicAdd(fp.A.f[d] + s, tile[(4 + d) * TN + t]);
          if (NORMAL) atomicAdd(fp.A.nrm[d] + s, tile[(7 + d) * TN + t]);
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace mpmb200
