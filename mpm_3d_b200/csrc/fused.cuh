// Fused gather + point update + scatter kernel (G2P of step n, then the map
// build and P2G of step n+1), one pass over the points per step.
//
// One CTA works on one bin (B^dim cells) at a time: it stages the nodal
// velocities of the bin's node tile ((B+3)^dim nodes) in shared memory, runs
// the gather and point update for every point of the bin, builds the map at
// the new position and adds the point's contributions into a shared-memory
// accumulator tile (native FP64 shared atomics), then adds the tile into the
// global accumulators with one global atomic per touched node and value.
// Points whose window leaves the tile (drift since the last binning) use
// global memory directly and are counted, so the host can re-bin.
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
  return (size_t)(6 + fused_nacc(normal)) * TN * sizeof(double) + (size_t)TN;
}

template <int DIM, int B, bool NORMAL>
__global__ void __launch_bounds__(256) k_g2p2g(FusedParams fp) {
  constexpr int T = B + 3;
  constexpr int TN = fused_tile_nodes<DIM, B>();
  constexpr int NACC = fused_nacc(NORMAL);
  extern __shared__ double smem[];
  double* tvel = smem;              // [6][TN]: vt0 vt1 vt2 dv0 dv1 dv2
  double* tacc = smem + 6 * TN;     // [NACC][TN]: m mx0 mx1 mx2 f0 f1 f2 (n0 n1 n2)
  uint8_t* touched = reinterpret_cast<uint8_t*>(tacc + NACC * TN);

  const Geom& g = fp.g;
  const double dt = fp.sp.dt;
  const PointsDev& P = fp.P;
  const int nwork = *fp.nwork;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const int bin = fp.work_bin[w];
    const int pstart = fp.work_start[w], pend = fp.work_end[w];
    int o[3] = {0, 0, 0};
    {
      const int bx = bin % fp.bg.nbx;
      const int r = bin / fp.bg.nbx;
      const int by = r % fp.bg.nby;
      const int bz = r / fp.bg.nby;
      o[0] = bx * B - 1;
      o[1] = by * B - 1;
      o[2] = DIM == 3 ? bz * B - 1 : 0;
    }
    if (fp.do_g2p) {
      for (int t = threadIdx.x; t < TN; t += blockDim.x) {
        const int tx = t % T, ty = (t / T) % T, tz = DIM == 3 ? t / (T * T) : 0;
        const int i = o[0] + tx, j = o[1] + ty, k = o[2] + tz;
        if (i < 0 || j < 0 || k < 0 || i >= g.nn[0] || j >= g.nn[1] || k >= g.nn[2]) continue;
        const int64_t s = node_slot(g, i, j, k);
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          tvel[d * TN + t] = fp.V.vt[d][s];
          tvel[(3 + d) * TN + t] = fp.V.dv[d][s];
        }
      }
    }
    if (fp.do_p2g) {
      for (int t = threadIdx.x; t < NACC * TN; t += blockDim.x) tacc[t] = 0.0;
      for (int t = threadIdx.x; t < TN; t += blockDim.x) touched[t] = 0;
    }
    __syncthreads();

    for (int p = pstart + threadIdx.x; p < pend; p += blockDim.x) {
      int act = P.active[p];
      if (act == 0) continue;
      if (act == 2) {
        // left the domain at the last move; generateMap deactivates it now
        P.active[p] = 0;
        continue;
      }
      double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int d = 0; d < DIM; d++) x[d] = P.x[d][p];
      const double ext = P.ext[p];
      double vel[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int d = 0; d < DIM; d++) vel[d] = P.v[d][p];
      double s6[6];
      bool stress_loaded = false;

      if (fp.do_g2p) {
        PointMap pm;
        const int st = build_map_fast<DIM>(g, fp.mc, fp.sp.cpdi, x, ext, pm, fp.err);
        double du[3] = {0.0, 0.0, 0.0}, dvel[3] = {0.0, 0.0, 0.0};
        double L[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        if (st > 0) {
          bool in_tile = true;
#pragma unroll
          for (int d = 0; d < DIM; d++)
            in_tile = in_tile && pm.ax[d].base >= o[d] && pm.ax[d].base + pm.ax[d].span <= o[d] + T;
          if (!in_tile) atomicAdd(fp.drift, 1ull);
          const AxisMap& X = pm.ax[0];
          const AxisMap& Y = pm.ax[1];
          double W0s[3], G0g[3], W0g[3];
#pragma unroll
          for (int k = 0; k < 3; k++) {
            W0s[k] = pm.sS * X.W[k];
            G0g[k] = pm.sG * X.G[k];
            W0g[k] = pm.sG * X.W[k];
          }
          constexpr int K2 = DIM == 3 ? 3 : 1;
#pragma unroll
          for (int k2 = 0; k2 < K2; k2++) {
            if (DIM == 3 && k2 >= pm.ax[2].span) continue;
            const double wz = DIM == 3 ? pm.ax[2].W[k2] : 1.0;
            const double gz = DIM == 3 ? pm.ax[2].G[k2] : 0.0;
#pragma unroll
            for (int k1 = 0; k1 < 3; k1++) {
              if (k1 >= Y.span) continue;
              const double W12 = Y.W[k1] * wz;
              const double G1W2 = Y.G[k1] * wz;
              const double W1G2 = Y.W[k1] * gz;
#pragma unroll
              for (int k0 = 0; k0 < 3; k0++) {
                if (k0 >= X.span) continue;
                const double S = W0s[k0] * W12;
                const double gr[3] = {G0g[k0] * W12, W0g[k0] * G1W2, W0g[k0] * W1G2};
                double vt[3], dv[3];
                const int i = X.base + k0, j = Y.base + k1, k = DIM == 3 ? pm.ax[2].base + k2 : 0;
                if (in_tile) {
                  const int t = (i - o[0]) + T * ((j - o[1]) + (DIM == 3 ? T * (k - o[2]) : 0));
#pragma unroll
                  for (int d = 0; d < DIM; d++) {
                    vt[d] = tvel[d * TN + t];
                    dv[d] = tvel[(3 + d) * TN + t];
                  }
                } else {
                  const int64_t s = node_slot(g, i, j, k);
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
                }
#pragma unroll
                for (int a = 0; a < DIM; a++)
#pragma unroll
                  for (int b = 0; b < DIM; b++) L[a][b] += vt[a] * gr[b];
              }
            }
          }
        }
        // movePoints: u_node = dt * x_t_node, x += S^T u, u += S^T u,
        // x_t += S^T diff_x_t (explicit_usl.cpp:279-292)
        double uold[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const double dx = dt * du[d];
          x[d] = x[d] + dx;
          uold[d] = P.u[d][p] + dx;
          vel[d] = vel[d] + dvel[d];
          P.x[d][p] = x[d];
          P.u[d][p] = uold[d];
          P.v[d][p] = vel[d];
        }
        P.vol[p] = P.vol[p] * exp(dt * (L[0][0] + L[1][1] + L[2][2]));
#pragma unroll
        for (int c = 0; c < 6; c++) s6[c] = P.s[c][p];
        stress_loaded = true;
        if (fp.mat.has_material) {
          jaumann_update<DIM>(L, s6, fp.mat.G, fp.mat.lambda, dt);
#pragma unroll
          for (int c = 0; c < 6; c++) P.s[c][p] = s6[c];
        }
        if (P.L != nullptr) {
#pragma unroll
          for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) P.L[9 * (int64_t)p + 3 * a + b] = L[a][b];
        }
      }

      if (fp.do_p2g) {
        PointMap pm;
        const int st = build_map_fast<DIM>(g, fp.mc, fp.sp.cpdi, x, ext, pm, fp.err);
        if (st < 0) {
          // outside the domain: inactive from the next map build on
          // (default_points.cpp:217-219); before the first step, at once
          P.active[p] = fp.do_g2p ? 2 : 0;
          continue;
        }
        if (st == 0) continue;
        if (!stress_loaded) {
#pragma unroll
          for (int c = 0; c < 6; c++) s6[c] = P.s[c][p];
        }
        const double m = P.m[p];
        const double vol = P.vol[p];
        double mv[3] = {0.0, 0.0, 0.0}, vs[6];
#pragma unroll
        for (int d = 0; d < DIM; d++) mv[d] = m * vel[d];
#pragma unroll
        for (int c = 0; c < 6; c++) vs[c] = s6[c] * vol;
        // vs as a symmetric 3x3 (xx yy zz xy yz xz)
        const double V3[3][3] = {{vs[0], vs[3], vs[5]}, {vs[3], vs[1], vs[4]}, {vs[5], vs[4], vs[2]}};
        bool in_tile = true;
#pragma unroll
        for (int d = 0; d < DIM; d++)
          in_tile = in_tile && pm.ax[d].base >= o[d] && pm.ax[d].base + pm.ax[d].span <= o[d] + T;
        if (!in_tile) {
          atomicAdd(fp.drift, 1ull);
          mark_blocks<DIM>(g, pm, fp.flags);
        }
        const AxisMap& X = pm.ax[0];
        const AxisMap& Y = pm.ax[1];
        double W0s[3], G0g[3], W0g[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
          W0s[k] = pm.sS * X.W[k];
          G0g[k] = pm.sG * X.G[k];
          W0g[k] = pm.sG * X.W[k];
        }
        constexpr int K2 = DIM == 3 ? 3 : 1;
#pragma unroll
        for (int k2 = 0; k2 < K2; k2++) {
          if (DIM == 3 && k2 >= pm.ax[2].span) continue;
          const double wz = DIM == 3 ? pm.ax[2].W[k2] : 1.0;
          const double gz = DIM == 3 ? pm.ax[2].G[k2] : 0.0;
#pragma unroll
          for (int k1 = 0; k1 < 3; k1++) {
            if (k1 >= Y.span) continue;
            const double W12 = Y.W[k1] * wz;
            const double G1W2 = Y.G[k1] * wz;
            const double W1G2 = Y.W[k1] * gz;
#pragma unroll
            for (int k0 = 0; k0 < 3; k0++) {
              if (k0 >= X.span) continue;
              const double S = W0s[k0] * W12;
              const double gr[3] = {G0g[k0] * W12, W0g[k0] * G1W2, W0g[k0] * W1G2};
              double val[NACC];
              val[0] = S * m;
#pragma unroll
              for (int d = 0; d < 3; d++) {
                val[1 + d] = S * mv[d];
                double fi = 0.0;
#pragma unroll
                for (int e = 0; e < DIM; e++) fi += V3[d][e] * gr[e];
                val[4 + d] = -fi;
                if (NORMAL) val[7 + d] = gr[d] * m;
              }
              const int i = X.base + k0, j = Y.base + k1, k = DIM == 3 ? pm.ax[2].base + k2 : 0;
              if (in_tile) {
                const int t = (i - o[0]) + T * ((j - o[1]) + (DIM == 3 ? T * (k - o[2]) : 0));
                touched[t] = 1;
                atomicAdd(tacc + t, val[0]);
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                  atomicAdd(tacc + (1 + d) * TN + t, val[1 + d]);
                  atomicAdd(tacc + (4 + d) * TN + t, val[4 + d]);
                  if (NORMAL) atomicAdd(tacc + (7 + d) * TN + t, val[7 + d]);
                }
              } else {
                const int64_t s = node_slot(g, i, j, k);
                atomicAdd(fp.A.m + s, val[0]);
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                  atomicAdd(fp.A.mx[d] + s, val[1 + d]);
                  atomicAdd(fp.A.f[d] + s, val[4 + d]);
                  if (NORMAL) atomicAdd(fp.A.nrm[d] + s, val[7 + d]);
                }
              }
            }
          }
        }
      }
    }
    __syncthreads();
    if (fp.do_p2g) {
      for (int t = threadIdx.x; t < TN; t += blockDim.x) {
        if (!touched[t]) continue;
        const int tx = t % T, ty = (t / T) % T, tz = DIM == 3 ? t / (T * T) : 0;
        const int i = o[0] + tx, j = o[1] + ty, k = o[2] + tz;
        const int64_t s = node_slot(g, i, j, k);
        fp.flags[node_block(g, i, j, k)] = 1u;
        atomicAdd(fp.A.m + s, tacc[t]);
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          atomicAdd(fp.A.mx[d] + s, tacc[(1 + d) * TN + t]);
          atomicAdd(fp.A.f[d] + s, tacc[(4 + d) * TN + t]);
          if (NORMAL) atomicAdd(fp.A.nrm[d] + s, tacc[(7 + d) * TN + t]);
        }
      }
      __syncthreads();
    }
  }
}

}  // namespace mpmb200
