// Fused gather + point update + scatter kernel (G2P of step n, then the map
// build and P2G of step n+1), one pass over the points per step.
//
// One CTA works on one bin (B^dim cells) at a time, in three phases that
// share one shared-memory node tile ((B+3)^dim nodes):
//   1. the tile holds the nodal velocities; every point of the bin gathers
//      from it, updates its state (x, u, x_t, V, stress) and writes it back;
//   2. the tile is cleared and every point builds its map at the new
//      position and adds its contributions with native FP64 shared-memory
//      atomics (points of one warp lie in distinct cells: no same-address
//      conflicts);
//   3. the tile is added into the global nodal accumulators with one global
//      atomic per touched node and value.
// Splitting the per-point work at the state write keeps the register
// footprint of each phase small; the bin's freshly written points are read
// back from L2 in phase 2. Points whose window leaves the tile (drift since
// the last binning) use global memory directly and are counted.
#pragma once

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

// Number of accumulated values per node: m, mx (3), f (3), contact normal (3).
__host__ __device__ constexpr int fused_nacc(bool normal) { return normal ? 10 : 7; }

template <int DIM, int B>
__host__ __device__ constexpr int fused_tile_nodes() {
  return DIM == 3 ? (B + 3) * (B + 3) * (B + 3) : (B + 3) * (B + 3);
}

template <int DIM, int B>
size_t fused_smem_bytes(bool normal) {
  constexpr int TN = fused_tile_nodes<DIM, B>();
  const int vals = fused_nacc(normal) > 6 ? fused_nacc(normal) : 6;
  return (size_t)vals * TN * sizeof(double) + (size_t)TN;
}

// Threads per CTA and minimum resident CTAs per SM of the fused kernel.
// 128 x 4 (128 registers per thread, 16 warps per SM) measured fastest on
// B200 among 256x1, 256x2, 128x3 and 128x4 for both 3D workloads.
#ifndef MPMB200_FUSED_THREADS
#define MPMB200_FUSED_THREADS 128
#endif
#ifndef MPMB200_FUSED_MIN_CTAS
#define MPMB200_FUSED_MIN_CTAS 4
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

// Phase 1 for one point: gather, movePoints / calculateStrainRate /
// updateDensity / updateStress (explicit_usl.cpp:266-355).
template <int DIM, int T, int TN>
__device__ __forceinline__ void gather_update(const FusedParams& fp, int64_t p, const int* o, const double* tvel) {
  const Geom& g = fp.g;
  const PointsDev& P = fp.P;
  const double dt = fp.sp.dt;
  double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < DIM; d++) x[d] = P.x[d][p];
  PointMap pm;
  const int st = build_map_fast<DIM>(g, fp.mc, fp.sp.cpdi, x, P.ext[p], pm, fp.err);
  double du[3] = {0.0, 0.0, 0.0}, dvel[3] = {0.0, 0.0, 0.0};
  double L[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  if (st > 0) {
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
        du[d] += S * vt[d];
        dvel[d] += S * dv[d];
        L[d][0] += vt[d] * gr0;
        L[d][1] += vt[d] * gr1;
        if (DIM == 3) L[d][2] += vt[d] * gr2;
      }
    });
  }
  // movePoints: u_node = dt * x_t_node; x += S^T u, u += S^T u,
  // x_t += S^T diff_x_t (explicit_usl.cpp:279-292)
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    const double dx = dt * du[d];
    P.x[d][p] = x[d] + dx;
    P.u[d][p] = P.u[d][p] + dx;
    P.v[d][p] = P.v[d][p] + dvel[d];
  }
  P.vol[p] = P.vol[p] * exp(dt * (L[0][0] + L[1][1] + L[2][2]));
  if (fp.mat.has_material) {
    double s6[6];
#pragma unroll
    for (int c = 0; c < 6; c++) s6[c] = P.s[c][p];
    jaumann_update<DIM>(L, s6, fp.mat.G, fp.mat.lambda, dt);
#pragma unroll
    for (int c = 0; c < 6; c++) P.s[c][p] = s6[c];
  }
  if (P.L != nullptr) {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) P.L[9 * p + 3 * a + b] = L[a][b];
  }
}

// Phase 2 for one point: map build and scatter of mapPointsToNodes
// (explicit_usl.cpp:112-164) and the contact normal of
// ContactHuang::generateRules (contact_huang.cpp:91).
template <int DIM, int T, int TN, bool NORMAL>
__device__ __forceinline__ void map_scatter(const FusedParams& fp, int64_t p, const int* o, double* tacc,
                                            uint8_t* touched) {
  const Geom& g = fp.g;
  const PointsDev& P = fp.P;
  double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < DIM; d++) x[d] = P.x[d][p];
  PointMap pm;
  const int st = build_map_fast<DIM>(g, fp.mc, fp.sp.cpdi, x, P.ext[p], pm, fp.err);
  if (st < 0) {
    // outside the domain: inactive from the next map build on
    // (default_points.cpp:217-219); before the first step, at once
    P.active[p] = fp.do_g2p ? 2 : 0;
    return;
  }
  if (st == 0) return;
  const double m = P.m[p];
  const double vol = P.vol[p];
  double mv[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < DIM; d++) mv[d] = m * P.v[d][p];
  // V * sigma as a symmetric 3x3 (stored xx yy zz xy yz xz)
  double vs[6];
#pragma unroll
  for (int c = 0; c < 6; c++) vs[c] = (DIM == 3 || c == 0 || c == 1 || c == 3) ? P.s[c][p] * vol : 0.0;
  const double V3[3][3] = {{vs[0], vs[3], vs[5]}, {vs[3], vs[1], vs[4]}, {vs[5], vs[4], vs[2]}};
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
    val[0] = S * m;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      val[1 + d] = S * mv[d];
      double fi = V3[d][0] * gr[0] + V3[d][1] * gr[1];
      if (DIM == 3) fi += V3[d][2] * gr[2];
      val[4 + d] = -fi;
      if (NORMAL) val[7 + d] = gr[d] * m;
    }
    if (in_tile) {
      const int t = t0 + k0 + T * (k1 + T * k2);
      touched[t] = 1;
      atomicAdd(tacc + t, val[0]);
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        atomicAdd(tacc + (1 + d) * TN + t, val[1 + d]);
        atomicAdd(tacc + (4 + d) * TN + t, val[4 + d]);
        if (NORMAL) atomicAdd(tacc + (7 + d) * TN + t, val[7 + d]);
      }
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

template <int DIM, int B, bool NORMAL>
__global__ void __launch_bounds__(MPMB200_FUSED_THREADS, MPMB200_FUSED_MIN_CTAS) k_g2p2g(FusedParams fp) {
  constexpr int T = B + 3;
  constexpr int TN = fused_tile_nodes<DIM, B>();
  constexpr int NACC = fused_nacc(NORMAL);
  constexpr int NVAL = NACC > 6 ? NACC : 6;
  extern __shared__ double smem[];
  double* tile = smem;  // phase 1: [6][TN] vt0 vt1 vt2 dv0 dv1 dv2; phase 2: [NACC][TN]
  uint8_t* touched = reinterpret_cast<uint8_t*>(tile + NVAL * TN);

  const Geom& g = fp.g;
  const PointsDev& P = fp.P;
  const int nwork = *fp.nwork;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const int bin = fp.work_bin[w];
    const int pstart = fp.work_start[w], pend = fp.work_end[w];
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
      __syncthreads();
      for (int p = pstart + threadIdx.x; p < pend; p += blockDim.x) {
        const int act = P.active[p];
        if (act == 0) continue;
        if (act == 2) {
          // left the domain at the last move; generateMap deactivates it now
          P.active[p] = 0;
          continue;
        }
        gather_update<DIM, T, TN>(fp, p, o, tile);
      }
      __syncthreads();
    }
    if (!fp.do_p2g) continue;
    for (int t = threadIdx.x; t < NACC * TN; t += blockDim.x) tile[t] = 0.0;
    for (int t = threadIdx.x; t < TN; t += blockDim.x) touched[t] = 0;
    __syncthreads();
    for (int p = pstart + threadIdx.x; p < pend; p += blockDim.x) {
      if (P.active[p] != 1) continue;
      map_scatter<DIM, T, TN, NORMAL>(fp, p, o, tile, touched);
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
    __syncthreads();
  }
}

}  // namespace mpmb200
