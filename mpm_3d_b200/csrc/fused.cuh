// Fused gather + point update + scatter kernel (G2P of step n, then the map
// build and P2G of step n+1), one pass over the points per step, for every
// body of every job in a batch in one launch.
//
// A CTA works on one work item at a time: up to CAP points of one bin
// (B^dim cells) of one body. Per work item:
//   0. the body's table entry is staged in shared memory; one thread issues
//      bulk asynchronous copies (cp.async.bulk, completed on an mbarrier) of
//      the item's 19 point arrays into shared memory, while the other
//      threads stage the nodal velocities of the bin's node tile ((B+3)^dim
//      nodes) in shared memory;
//   1. every point gathers from the tile and updates its state (x, u, x_t,
//      V, stress); results go to global memory and back into the staged
//      copy;
//   2. the tile is cleared, every point builds its map at the new position
//      and adds its contributions with FP64 shared-memory atomics (points of
//      one warp have distinct window bases: no same-address conflicts).
//      Windows inside the tile take a straight-line node box, the union of
//      the warp's window shapes, with the force evaluated per box row;
//   3. the tile is added into the global nodal accumulators, one global
//      atomic per touched node and value.
// No phase waits on DRAM latency per point: the point state arrives in bulk
// and both phases read it from shared memory. Points whose window leaves the
// tile (drift since the last binning) use global memory and are counted.
//
// PT is the point precision: double for the FP64 form, float for the mixed
// form (point state, shape functions and stress in FP32; nodal sums in
// FP64).
#pragma once

#include <cstddef>

#include "async_copy.cuh"
#include "geom.cuh"
#include "kernels_fp64.cuh"
#include "sort.cuh"
#include "state.cuh"

namespace mpmb200 {

// Launch arguments of the fused kernel. A launch covers either every body
// of the batch (entries read from the body table and staged in shared
// memory per work item) or one body whose entry travels in the launch
// arguments themselves (`one`, read through the constant bank): small
// batches launch once per body so that the hot loops read their
// parameters as constant operands.
template <typename PT>
struct FusedLaunch {
  BodyCtx<PT> one;      // the body of a one-body launch
  int one_body;         // its index in the body table (-1: every body)
  const BodyCtx<PT>* bodies;
  const int32_t* item_off;       // first item of each body's range
  const int32_t* nwork_body;     // items of each body
  const int32_t* work_end_body;  // inclusive prefix of nwork_body
  const int32_t* flat_body;      // flat index -> body (launches over every body)
  const int32_t* flat_item;      // flat index -> item
  const int32_t* work_bin;
  const int32_t* work_start;
  const int32_t* work_end;
  const int32_t* nwork;          // total items
  int nbodies_cap;               // bodies in the table (bound for the search)
  int* err;
  unsigned long long* drift;
  int prime_pass;   // 1: only bodies still to prime, scatter only
  int phases;       // 1: gather + point update, 2: map + scatter, 3: both
  const unsigned long long* bounds;  // deterministic form: 4 per body (k_det_bounds)
  // poll limit of the waits for a work item's bulk copies; a wait that runs
  // out flags kErrWaitTimeout and its CTA returns (after the copies in
  // flight have landed, waited for with the default limit)
  uint32_t wait_polls;
  // work queue of the launch (two counters, zero between launches; see
  // claim_item)
  int* queue;
};

// Dynamic distribution of the work items of a launch over the body table. A
// CTA's first item is its blockIdx.x; each later one is claimed from the
// launch's counter (items gridDim.x, gridDim.x + 1, ... in claim order), so
// that CTAs that drew small items take more of them: items differ in size by
// up to 8x where bins are cut by body surfaces, and a fixed stride left the
// slowest CTA with 5-17 % more than the mean of the work (measured 4 % and
// 7 % off the ensemble's FP64 and mixed kernels). A claim is made when the
// CTA starts its current item, one item ahead, to hide its latency. A
// one-body launch keeps the fixed stride: its items are few per CTA (one or
// two on a 0.5 M-point body), where claims made one item ahead crowd the
// last round onto fewer SMs than the stride does (measured 11 % slower on a
// two-body collision). queue[0] counts the claims, queue[1] the CTAs that
// finished; the last CTA to finish zeroes both, so the next launch over the
// table starts from zero (an engine issues those launches one after the
// other on its step stream; only one-body launches use side streams).
__device__ __forceinline__ int claim_item(int* queue) { return (int)gridDim.x + atomicAdd(queue, 1); }

// Called once per CTA by thread 0 after its last claim (every exit path).
__device__ __forceinline__ void queue_done(int* queue) {
  __threadfence();   // this CTA's claims precede its count of finished CTAs
  if (atomicAdd(queue + 1, 1) == (int)gridDim.x - 1) {
    atomicExch(queue, 0);
    atomicExch(queue + 1, 0);
  }
}

// Staged point arrays: x0..2 v0..2 u0..2 s0..5 vol m ext, then active.
constexpr int kFx = 0, kFv = 3, kFu = 6, kFs = 9, kFvol = 15, kFm = 16, kFext = 17, kNF = 18;

// Row stride of the staged copy: slack for the alignment of the bulk
// copies (starts rounded down, sizes rounded up to 16 bytes).
template <int CAP>
__host__ __device__ constexpr int cap_row() {
  return CAP + 8;
}

// Number of accumulated values per node: m, mx (3), f (3), contact normal (3).
__host__ __device__ constexpr int fused_nacc(bool normal) { return normal ? 10 : 7; }

// Slots of the node tile (T = B + 3 nodes per axis). In 3D the x-rows of
// four consecutive z planes share one y row of 4T slots: slot = x + 4T y +
// T (z mod 4) + 4T^2 (z div 4). A warp's lanes sit in distinct cells, x
// fastest: the 16 lanes of a half-warp (4 x 4 cells of one z plane) read
// and add at x + 4T y, which with 4T = 28 = 12 (mod 16) falls on 16
// distinct 8-byte bank pairs (rows of T = 7 slots put lanes two rows apart
// on the same banks). Slots with z >= T stay unused. 2D: x + T y.
template <int DIM, int T>
struct TileLayout {
  static constexpr int ZG = DIM == 3 ? 4 : 1;       // z planes per row
  static constexpr int RL = ZG * T;                 // slots per y row
  static constexpr int PG = RL * T;                 // slots per group of ZG planes
  static constexpr int N = DIM == 3 ? PG * ((T + ZG - 1) / ZG) : T * T;
  __host__ __device__ static constexpr int zoff(int z) { return DIM == 3 ? T * (z % ZG) + PG * (z / ZG) : 0; }
  __host__ __device__ static constexpr int slot(int x, int y, int z) { return x + RL * y + zoff(z); }
  // node of slot t (relative to the tile origin); false for unused slots
  __device__ static bool node(int t, int& x, int& y, int& z) {
    x = t % T;
    y = (t / RL) % T;
    z = DIM == 3 ? (t / T) % ZG + ZG * (t / PG) : 0;
    return z < (DIM == 3 ? T : 1);
  }
};

template <int DIM, int B>
__host__ __device__ constexpr int fused_tile_nodes() {
  return TileLayout<DIM, B + 3>::N;
}

template <int DIM>
__host__ __device__ constexpr int fused_bin() {
  return DIM == 3 ? 4 : 8;
}

// Shared memory layout: mbarriers (points, table entry slots 0 and 1) |
// body table entries [2] | points [kNF][row] | active [row] | tile [10][TN]
// doubles (two such levels in the deterministic form) | touched [TN].
template <typename PT>
__host__ __device__ constexpr size_t ctx_bytes() {
  return (offsetof(BodyCtx<PT>, Palt) + 15) / 16 * 16;
}
constexpr size_t kOffCtx = 32;
static_assert(ctx_bytes<double>() % 16 == 0 && ctx_bytes<float>() % 16 == 0, "bulk copies move 16-byte multiples");
static_assert(sizeof(BodyCtx<double>) % 16 == 0 && sizeof(BodyCtx<float>) % 16 == 0,
              "table entries start on 16-byte boundaries");
template <typename PT, int CAP>
__host__ __device__ constexpr size_t off_pts() {
  return kOffCtx + 2 * ctx_bytes<PT>();
}
template <typename PT, int CAP>
__host__ __device__ constexpr size_t off_act() {
  return off_pts<PT, CAP>() + (sizeof(PT) * kNF * cap_row<CAP>() + 15) / 16 * 16;
}
template <typename PT, int CAP>
__host__ __device__ constexpr size_t off_tile() {
  return off_act<PT, CAP>() + sizeof(int32_t) * cap_row<CAP>();
}
// The mixed form without contact normals keeps its FP32 velocity tile apart
// from its 7 accumulator rows (the bytes of 10 rows in all), so that a
// point can scatter while others still gather; the other kernels keep the
// velocity tile in the accumulator tile's space.
template <typename PT, bool NORMAL, bool DET>
__host__ __device__ constexpr bool split_tiles() {
  return sizeof(PT) == 4 && !NORMAL && !DET;
}
// Accumulator tile levels: 1, or 2 in the deterministic form; then the
// touched flags; then the separate velocity tile where there is one.
template <int DIM, typename PT, int CAP, bool NORMAL, bool DET>
__host__ __device__ constexpr size_t off_touched() {
  return off_tile<PT, CAP>() +
         sizeof(double) * (DET ? 20 : (split_tiles<PT, NORMAL, DET>() ? 7 : 10)) * fused_tile_nodes<DIM, fused_bin<DIM>()>();
}
template <int DIM, typename PT, int CAP, bool NORMAL, bool DET>
__host__ __device__ constexpr size_t off_tvel() {
  return (off_touched<DIM, PT, CAP, NORMAL, DET>() + fused_tile_nodes<DIM, fused_bin<DIM>()>() + 15) / 16 * 16;
}
template <int DIM, typename PT, int CAP, bool NORMAL, bool DET>
__host__ __device__ constexpr size_t fused_smem_bytes() {
  return split_tiles<PT, NORMAL, DET>()
             ? off_tvel<DIM, PT, CAP, NORMAL, DET>() + sizeof(PT) * 6 * fused_tile_nodes<DIM, fused_bin<DIM>()>()
             : off_touched<DIM, PT, CAP, NORMAL, DET>() + fused_tile_nodes<DIM, fused_bin<DIM>()>();
}

// Threads per CTA and the resident CTAs per SM the register budget is sized
// for (128 registers per thread either way): the mixed form runs 256-point
// items on 128-thread CTAs, four per SM, so that a barrier waits on fewer
// warps; larger items, and every FP64 item, run on 256-thread CTAs, two per
// SM (one point per thread for 256-point items: measured faster in FP64).
template <typename PT, int CAP>
__host__ __device__ constexpr int fused_threads() {
  return sizeof(PT) == 4 && CAP <= 256 ? 128 : 256;
}
template <typename PT, int CAP>
__host__ __device__ constexpr int fused_min_ctas() {
  return sizeof(PT) == 4 && CAP <= 256 ? 4 : 2;
}

// Entry k (0..2) of a 3-array without indexing it by a variable (which
// would move the array to local memory).
template <typename R>
__device__ __forceinline__ R sel3(const R* a, int k) {
  return k == 0 ? a[0] : (k == 1 ? a[1] : a[2]);
}

// Visits the window nodes of a point map: f(k0, k1, k2). Spans are 2 or 3
// per axis; the first two offsets of every axis are unconditional. Only the
// innermost axis is unrolled: the general windows are the rarer path, and a
// fully unrolled 3x3x3 visit inflates the kernel's instruction footprint.
template <int DIM, typename R, typename F>
__device__ __forceinline__ void for_window(const PointMapT<R>& pm, F&& f) {
  constexpr int K2 = DIM == 3 ? 3 : 1;
#pragma unroll 1
  for (int k2 = 0; k2 < K2; k2++) {
    if (DIM == 3 && k2 == 2 && pm.ax[2].span < 3) break;
#pragma unroll 1
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

template <int DIM, typename R>
__device__ __forceinline__ bool window_in_tile(const PointMapT<R>& pm, const int* o, int T) {
  bool in = true;
#pragma unroll
  for (int d = 0; d < DIM; d++) in = in && pm.ax[d].base >= o[d] && pm.ax[d].base + pm.ax[d].span <= o[d] + T;
  return in;
}

// Gathered sums of one point: S^T x_t (du, before the dt factor), S^T
// diff_x_t (dv) and the velocity gradient L_ab = sum v_a dS/dx_b.
template <typename R>
struct GatherSum {
  R du[3] = {R(0), R(0), R(0)};
  R dv[3] = {R(0), R(0), R(0)};
  R L[3][3] = {{R(0), R(0), R(0)}, {R(0), R(0), R(0)}, {R(0), R(0), R(0)}};
};

// Span bits of a window: bit d set when axis d spans three nodes.
template <int DIM, typename R>
__device__ __forceinline__ int span_bits(const PointMapT<R>& pm) {
  int b = 0;
#pragma unroll
  for (int d = 0; d < DIM; d++) b |= (pm.ax[d].span == 3 ? 1 : 0) << d;
  return b;
}

// Gather over a box of K0 x K1 (x K2) nodes from the window's base, all
// inside the staged tile: straight-line code. A warp runs the box of the
// union of its lanes' spans, so lanes whose window is narrower along an
// axis skip that axis' third node (their W and G there are zero anyway).
template <int DIM, int T, int TN, int K0, int K1, int K2, typename R>
__device__ __forceinline__ GatherSum<R> gather_box(const PointMapT<R>& pm, const int* o, const R* tvel) {
  GatherSum<R> gs;
  using TL = TileLayout<DIM, T>;
  const int txy = (pm.ax[0].base - o[0]) + TL::RL * (pm.ax[1].base - o[1]);
  const int bz = DIM == 3 ? pm.ax[2].base - o[2] : 0;
  const bool third0 = pm.ax[0].span == 3, third1 = pm.ax[1].span == 3, third2 = DIM == 3 && pm.ax[2].span == 3;
  constexpr int KZ = DIM == 3 ? K2 : 1;
  // sums over the unscaled separable products; the map's scales (sS on
  // values, sG on gradients) are applied once at the end
#pragma unroll
  for (int k2 = 0; k2 < KZ; k2++) {
    if (k2 == 2 && !third2) continue;
    const R wz = DIM == 3 ? pm.ax[2].W[k2] : R(1);
    const R gz = DIM == 3 ? pm.ax[2].G[k2] : R(0);
#pragma unroll
    for (int k1 = 0; k1 < K1; k1++) {
      if (k1 == 2 && !third1) continue;
      const R W12 = pm.ax[1].W[k1] * wz;
      const R G1W2 = pm.ax[1].G[k1] * wz;
      const R W1G2 = pm.ax[1].W[k1] * gz;
#pragma unroll
      for (int k0 = 0; k0 < K0; k0++) {
        if (k0 == 2 && !third0) continue;
        const int t = txy + k0 + TL::RL * k1 + TL::zoff(bz + k2);
        const R w0 = pm.ax[0].W[k0];
        const R S = w0 * W12;
        const R gr0 = pm.ax[0].G[k0] * W12, gr1 = w0 * G1W2, gr2 = w0 * W1G2;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const R vt = tvel[d * TN + t];
          gs.du[d] += S * vt;
          gs.dv[d] += S * tvel[(3 + d) * TN + t];
          gs.L[d][0] += vt * gr0;
          gs.L[d][1] += vt * gr1;
          if (DIM == 3) gs.L[d][2] += vt * gr2;
        }
      }
    }
  }
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    gs.du[d] *= pm.sS;
    gs.dv[d] *= pm.sS;
#pragma unroll
    for (int b = 0; b < DIM; b++) gs.L[d][b] *= pm.sG;
  }
  return gs;
}

// Gather over the union box of a warp with a three-node span on some axis:
// rolled loops over the y and z offsets (bounds from the warp's union mask),
// the x offsets unrolled, lanes skipping the third node of an axis they do
// not span. One compact loop for every such shape keeps the kernel's
// instruction footprint small (warps of different shapes run side by side).
template <int DIM, int T, int TN, typename R>
__device__ __forceinline__ GatherSum<R> gather_rolled(const PointMapT<R>& pm, const int* o, const R* tvel, int mask) {
  using TL = TileLayout<DIM, T>;
  GatherSum<R> gs;
  const int txy = (pm.ax[0].base - o[0]) + TL::RL * (pm.ax[1].base - o[1]);
  const int bz = DIM == 3 ? pm.ax[2].base - o[2] : 0;
  const bool third0 = pm.ax[0].span == 3, third1 = pm.ax[1].span == 3, third2 = DIM == 3 && pm.ax[2].span == 3;
  const int K1 = 2 + ((mask >> 1) & 1), K2 = DIM == 3 ? 2 + ((mask >> 2) & 1) : 1;
  const bool wide0 = (mask & 1) != 0;
#pragma unroll 1
  for (int k2 = 0; k2 < K2; k2++) {
    const bool on2 = k2 < 2 || third2;
    const R wz = DIM == 3 ? sel3(pm.ax[2].W, k2) : R(1);
    const R gz = DIM == 3 ? sel3(pm.ax[2].G, k2) : R(0);
    const int zo = TL::zoff(bz + k2);
#pragma unroll 1
    for (int k1 = 0; k1 < K1; k1++) {
      if (!on2 || (k1 == 2 && !third1)) continue;
      const R w1 = sel3(pm.ax[1].W, k1);
      const R W12 = w1 * wz;
      const R G1W2 = sel3(pm.ax[1].G, k1) * wz;
      const R W1G2 = w1 * gz;
      const int trow = txy + TL::RL * k1 + zo;
#pragma unroll
      for (int k0 = 0; k0 < 3; k0++) {
        if (k0 == 2 && !(wide0 && third0)) break;
        const int t = trow + k0;
        const R w0 = pm.ax[0].W[k0];
        const R S = w0 * W12;
        const R gr0 = pm.ax[0].G[k0] * W12, gr1 = w0 * G1W2, gr2 = w0 * W1G2;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const R vt = tvel[d * TN + t];
          gs.du[d] += S * vt;
          gs.dv[d] += S * tvel[(3 + d) * TN + t];
          gs.L[d][0] += vt * gr0;
          gs.L[d][1] += vt * gr1;
          if (DIM == 3) gs.L[d][2] += vt * gr2;
        }
      }
    }
  }
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    gs.du[d] *= pm.sS;
    gs.dv[d] *= pm.sS;
#pragma unroll
    for (int b = 0; b < DIM; b++) gs.L[d][b] *= pm.sG;
  }
  return gs;
}

// The warp's union box: straight-line code for two nodes per axis (the
// regular layouts' common shape), the rolled loop for every other shape.
template <int DIM, int T, int TN, typename R>
__device__ __forceinline__ GatherSum<R> gather_box_any(const PointMapT<R>& pm, const int* o, const R* tvel, int mask) {
  if (mask == 0) return gather_box<DIM, T, TN, 2, 2, 2>(pm, o, tvel);
  return gather_rolled<DIM, T, TN>(pm, o, tvel, mask);
}

// Gather over any window (three-node spans, nodes outside the tile).
template <int DIM, int T, int TN, typename PT, typename R>
__device__ __forceinline__ GatherSum<R> gather_general(const BodyCtx<PT>& c, unsigned long long* drift,
                                                       const PointMapT<R>& pm, const int* o, const R* tvel,
                                                       const double* vref) {
  GatherSum<R> gs;
  const Geom& g = c.g;
  const bool in_tile = window_in_tile<DIM>(pm, o, T);
  if (!in_tile) atomicAdd(drift, 1ull);
  using TL = TileLayout<DIM, T>;
  const int txy = (pm.ax[0].base - o[0]) + TL::RL * (pm.ax[1].base - o[1]);
  const int bz = DIM == 3 ? pm.ax[2].base - o[2] : 0;
  const R sS = pm.sS, sG = pm.sG;
  for_window<DIM>(pm, [&](int k0, int k1, int k2) {
    const R wz = DIM == 3 ? sel3(pm.ax[2].W, k2) : R(1);
    const R gz = DIM == 3 ? sel3(pm.ax[2].G, k2) : R(0);
    const R w1 = sel3(pm.ax[1].W, k1), g1 = sel3(pm.ax[1].G, k1);
    const R W12 = w1 * wz;
    const R S = sS * pm.ax[0].W[k0] * W12;
    const R gr0 = sG * pm.ax[0].G[k0] * W12;
    const R gw0 = sG * pm.ax[0].W[k0];
    const R gr1 = gw0 * (g1 * wz);
    const R gr2 = gw0 * (w1 * gz);
    R vt[3] = {R(0), R(0), R(0)}, dv[3] = {R(0), R(0), R(0)};
    if (in_tile) {
      const int t = txy + k0 + TL::RL * k1 + TL::zoff(bz + k2);
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        vt[d] = tvel[d * TN + t];
        dv[d] = tvel[(3 + d) * TN + t];
      }
    } else {
      const int64_t s = node_slot(g, pm.ax[0].base + k0, pm.ax[1].base + k1, DIM == 3 ? pm.ax[2].base + k2 : 0);
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        vt[d] = (R)(c.V.vt[d][s] - vref[d]);
        dv[d] = (R)c.V.dv[d][s];
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

// A staged point's position (k = kFx) or velocity (k = kFv) component in
// double: the FP64 form's value, or the mixed form's two-word value, its
// high word from the staged copy and its low word from global memory.
template <typename PT, int ROW>
__device__ __forceinline__ double staged_two(const PT* sp, const PointsT<PT>& P, int64_t p, int k, int d) {
  if constexpr (sizeof(PT) == 8) return sp[(k + d) * ROW];
  else return (double)sp[(k + d) * ROW] + (double)(k == kFx ? P.xl[d][p] : P.vl[d][p]);
}

// Stores a position or velocity component (the mixed form splits it into
// its two words).
template <typename PT, int ROW>
__device__ __forceinline__ void store_two(PT* sp, const PointsT<PT>& P, int64_t p, int k, int d, double v) {
  if constexpr (sizeof(PT) == 8) {
    sp[(k + d) * ROW] = v;
    (k == kFx ? P.x[d] : P.v[d])[p] = v;
  } else {
    float hi, lo;
    split_two_word(v, hi, lo);
    sp[(k + d) * ROW] = hi;
    (k == kFx ? P.x[d] : P.v[d])[p] = hi;
    (k == kFx ? P.xl[d] : P.vl[d])[p] = lo;
  }
}

// Phase 1 for one point: gather, movePoints / calculateStrainRate /
// updateDensity / updateStress (explicit_usl.cpp:266-355). `sp` points at the
// point's column in the staged arrays (stride ROW).
//
// The staged nodal velocities are relative to `vref` (zero in the FP64
// form; in the mixed form the velocity of the work item's first point,
// subtracted in FP64 before the conversion to FP32). Since the shape
// functions sum to one and their gradients to zero, S^T v = vref +
// S^T (v - vref) and the velocity gradient is that of v - vref: the same
// values in exact arithmetic, without the cancellation of a common
// translation against the velocity differences in FP32.
template <int DIM, int T, int TN, int ROW, bool DET, typename PT>
__device__ __forceinline__ void gather_update(const BodyCtx<PT>& c, int* err, unsigned long long* drift, int64_t p,
                                              PT* sp, const int* o, const PT* tvel, const double* vref) {
  using R = PT;
  const PointsT<PT>& P = c.P;
  const R dt = (R)c.sp.dt;
  double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < DIM; d++) x[d] = staged_two<PT, ROW>(sp, P, p, kFx, d);
  PointMapT<R> pm;
  const int st = build_map<DIM>(c.g, c.mc, c.sp.cpdi, x, sp[kFext * ROW], pm, err);
  GatherSum<R> gs;
  if (st > 0) {
    // windows inside the tile take the straight-line box of the union of
    // the warp's spans; the deterministic form takes one arithmetic for
    // every window (the straight-line path rounds differently, and whether
    // a window is inside the tile depends on the binning)
    const bool in = !DET && window_in_tile<DIM>(pm, o, T);
    const unsigned am = __activemask();
    const unsigned inm = __ballot_sync(am, in);
    if (in)
      gs = gather_box_any<DIM, T, TN>(pm, o, tvel, __reduce_or_sync(inm, span_bits<DIM>(pm)));
    else
      gs = gather_general<DIM, T, TN>(c, drift, pm, o, tvel, vref);
    if constexpr (sizeof(PT) == 4) {
#pragma unroll
      for (int d = 0; d < DIM; d++) gs.du[d] += (R)vref[d];
    }
  }
  // movePoints: u_node = dt * x_t_node; x += S^T u, u += S^T u,
  // x_t += S^T diff_x_t (explicit_usl.cpp:279-292); the mixed form adds
  // the increments to its two-word x and x_t in FP64
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    const R dx = dt * gs.du[d];
    const R un = sp[(kFu + d) * ROW] + dx;
    store_two<PT, ROW>(sp, P, p, kFx, d, x[d] + (double)dx);
    store_two<PT, ROW>(sp, P, p, kFv, d, staged_two<PT, ROW>(sp, P, p, kFv, d) + (double)gs.dv[d]);
    sp[(kFu + d) * ROW] = un;
    P.u[d][p] = un;
  }
  const R vol = sp[kFvol * ROW] * exp(dt * (gs.L[0][0] + gs.L[1][1] + gs.L[2][2]));
  sp[kFvol * ROW] = vol;
  P.vol[p] = vol;
  if (c.mat.has_material && c.mat.kind == 1) {
    R s6[6];
    neohookean_update<R>(P.ms, p, gs.L, s6, (R)c.mat.G, (R)c.mat.lambda, dt);
#pragma unroll
    for (int k = 0; k < 6; k++) {
      sp[(kFs + k) * ROW] = s6[k];
      P.s[k][p] = s6[k];
    }
  } else if (c.mat.has_material && c.mat.kind == 2) {
    R s6[6];
#pragma unroll
    for (int k = 0; k < 6; k++) s6[k] = sp[(kFs + k) * ROW];
    sand_update<DIM, R>(P.ms, p, gs.L, s6, (R)sp[kFm * ROW], vol, c.mat, dt);
#pragma unroll
    for (int k = 0; k < 6; k++) {
      sp[(kFs + k) * ROW] = s6[k];
      P.s[k][p] = s6[k];
    }
  } else if (c.mat.has_material) {
    R s6[6];
#pragma unroll
    for (int k = 0; k < 6; k++) s6[k] = sp[(kFs + k) * ROW];
    jaumann_point<DIM, R>(gs.L, s6, c.mat, c.sp.dt);
#pragma unroll
    for (int k = 0; k < 6; k++) {
      sp[(kFs + k) * ROW] = s6[k];
      P.s[k][p] = s6[k];
    }
  }
  if (P.L != nullptr) {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) P.L[9 * p + 3 * a + b] = (double)gs.L[a][b];
  }
}

// Values a point adds to one tile node, in the order m, mx[0..DIM),
// f[0..DIM), normal[0..DIM); tile_field gives each one's tile row. They
// are FP64 (the tile's type): the mixed form forms the mass and momentum
// contributions in FP64 from its two-word mass and velocity, and its force
// and normal contributions in FP32.
template <int DIM, bool NORMAL, typename R>
struct NodeVals {
  static constexpr int K = 1 + 2 * DIM + (NORMAL ? DIM : 0);
  double v[K];
};

template <int DIM>
__device__ __forceinline__ constexpr int tile_field(int i) {
  return i == 0 ? 0 : (i <= DIM ? i : (i <= 2 * DIM ? 4 + (i - 1 - DIM) : 7 + (i - 1 - 2 * DIM)));
}

// Adds one node's values to the shared FP64 tile (shared-memory FP64
// atomics). A hand-written variant that interleaved compare-and-swap loops
// over all of a node's values was measured slower (register pressure).
template <int DIM, bool NORMAL, int TN, bool DET, typename R>
__device__ __forceinline__ void tile_add_node(double* tacc, int t, const NodeVals<DIM, NORMAL, R>& nv,
                                              const Split2* ks) {
#pragma unroll
  for (int i = 0; i < NodeVals<DIM, NORMAL, R>::K; i++) {
    if constexpr (DET) {
      // deterministic form: two exactly summed levels (second tile behind the first)
      const int cls = i == 0 ? 0 : (i <= DIM ? 1 : (i <= 2 * DIM ? 2 : 3));
      double q0, q1;
      presplit(nv.v[i], ks[cls], q0, q1);
      atomicAdd(tacc + tile_field<DIM>(i) * TN + t, q0);
      atomicAdd(tacc + (10 + tile_field<DIM>(i)) * TN + t, q1);
    } else {
      atomicAdd(tacc + tile_field<DIM>(i) * TN + t, nv.v[i]);
    }
  }
}

// Per-point scatter sources: m, m x_t (FP64 in both forms: the mixed form's
// are its two-word values) and V sigma (symmetric 3x3, point precision).
template <typename R>
struct ScatterSrc {
  double m;
  double mv[3];
  R V3[3][3];
};

// Scatter over a box of K0 x K1 (x K2) nodes inside the tile (as
// gather_box). The nodal force -V sigma . grad S is formed per node from the
// node's gradient (measured 2 % faster on the column than row factors
// -(G0 A + W0 B) precomputed per box row, which hold 6 more values).
template <int DIM, int T, int TN, bool NORMAL, bool DET, int K0, int K1, int K2, typename R>
__device__ __forceinline__ void scatter_box(const PointMapT<R>& pm, const int* o, const ScatterSrc<R>& q,
                                            double* tacc, uint8_t* touched, const Split2* ks) {
  using TL = TileLayout<DIM, T>;
  const int txy = (pm.ax[0].base - o[0]) + TL::RL * (pm.ax[1].base - o[1]);
  const int bz = DIM == 3 ? pm.ax[2].base - o[2] : 0;
  const bool third0 = pm.ax[0].span == 3, third1 = pm.ax[1].span == 3, third2 = DIM == 3 && pm.ax[2].span == 3;
  constexpr int KZ = DIM == 3 ? K2 : 1;
  // the map's scales go into the point's sources once (sS on m and m x_t,
  // sG on V sigma and on m for the normal), the node loop uses the
  // unscaled axis factors
  const double sm = (double)pm.sS * q.m;
  const R gm = pm.sG * (R)q.m;
  double smv[3];
  R sV[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    smv[a] = (double)pm.sS * q.mv[a];
#pragma unroll
    for (int b = 0; b < 3; b++) sV[a][b] = pm.sG * q.V3[a][b];
  }
#pragma unroll
  for (int k2 = 0; k2 < KZ; k2++) {
    if (k2 == 2 && !third2) continue;
    const R wz = DIM == 3 ? pm.ax[2].W[k2] : R(1);
    const R gz = DIM == 3 ? pm.ax[2].G[k2] : R(0);
#pragma unroll
    for (int k1 = 0; k1 < K1; k1++) {
      if (k1 == 2 && !third1) continue;
      const R W12 = pm.ax[1].W[k1] * wz;
      const R G1W2 = pm.ax[1].G[k1] * wz;
      const R W1G2 = pm.ax[1].W[k1] * gz;
#pragma unroll
      for (int k0 = 0; k0 < K0; k0++) {
        if (k0 == 2 && !third0) continue;
        const int t = txy + k0 + TL::RL * k1 + TL::zoff(bz + k2);
        touched[t] = 1;
        const R w0 = pm.ax[0].W[k0], g0 = pm.ax[0].G[k0];
        const R S = w0 * W12, gr0 = g0 * W12, gr1 = w0 * G1W2, gr2 = w0 * W1G2;
        NodeVals<DIM, NORMAL, R> nv;
        nv.v[0] = (double)S * sm;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          nv.v[1 + d] = (double)S * smv[d];
          nv.v[1 + DIM + d] = (double)(-(sV[d][0] * gr0 + sV[d][1] * gr1 + (DIM == 3 ? sV[d][2] * gr2 : R(0))));
        }
        if constexpr (NORMAL) {
          const R gr[3] = {gr0, gr1, gr2};
#pragma unroll
          for (int d = 0; d < DIM; d++) nv.v[1 + 2 * DIM + d] = (double)(gr[d] * gm);
        }
        tile_add_node<DIM, NORMAL, TN, DET>(tacc, t, nv, ks);
      }
    }
  }
}

// Scatter over the union box of a warp with a three-node span on some axis
// (as gather_rolled).
template <int DIM, int T, int TN, bool NORMAL, bool DET, typename R>
__device__ __forceinline__ void scatter_rolled(const PointMapT<R>& pm, const int* o, const ScatterSrc<R>& q,
                                               double* tacc, uint8_t* touched, const Split2* ks, int mask) {
  using TL = TileLayout<DIM, T>;
  const int txy = (pm.ax[0].base - o[0]) + TL::RL * (pm.ax[1].base - o[1]);
  const int bz = DIM == 3 ? pm.ax[2].base - o[2] : 0;
  const bool third0 = pm.ax[0].span == 3, third1 = pm.ax[1].span == 3, third2 = DIM == 3 && pm.ax[2].span == 3;
  const int K1 = 2 + ((mask >> 1) & 1), K2 = DIM == 3 ? 2 + ((mask >> 2) & 1) : 1;
  const bool wide0 = (mask & 1) != 0;
  const double sm = (double)pm.sS * q.m;
  const R gm = pm.sG * (R)q.m;
  double smv[3];
  R sV[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    smv[a] = (double)pm.sS * q.mv[a];
#pragma unroll
    for (int b = 0; b < 3; b++) sV[a][b] = pm.sG * q.V3[a][b];
  }
#pragma unroll 1
  for (int k2 = 0; k2 < K2; k2++) {
    const bool on2 = k2 < 2 || third2;
    const R wz = DIM == 3 ? sel3(pm.ax[2].W, k2) : R(1);
    const R gz = DIM == 3 ? sel3(pm.ax[2].G, k2) : R(0);
    const int zo = TL::zoff(bz + k2);
#pragma unroll 1
    for (int k1 = 0; k1 < K1; k1++) {
      if (!on2 || (k1 == 2 && !third1)) continue;
      const R w1 = sel3(pm.ax[1].W, k1);
      const R W12 = w1 * wz;
      const R G1W2 = sel3(pm.ax[1].G, k1) * wz;
      const R W1G2 = w1 * gz;
      const int trow = txy + TL::RL * k1 + zo;
#pragma unroll
      for (int k0 = 0; k0 < 3; k0++) {
        if (k0 == 2 && !(wide0 && third0)) break;
        const int t = trow + k0;
        touched[t] = 1;
        const R w0 = pm.ax[0].W[k0], g0 = pm.ax[0].G[k0];
        const R S = w0 * W12, gr0 = g0 * W12, gr1 = w0 * G1W2, gr2 = w0 * W1G2;
        NodeVals<DIM, NORMAL, R> nv;
        nv.v[0] = (double)S * sm;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          nv.v[1 + d] = (double)S * smv[d];
          nv.v[1 + DIM + d] = (double)(-(sV[d][0] * gr0 + sV[d][1] * gr1 + (DIM == 3 ? sV[d][2] * gr2 : R(0))));
        }
        if constexpr (NORMAL) {
          const R gr[3] = {gr0, gr1, gr2};
#pragma unroll
          for (int d = 0; d < DIM; d++) nv.v[1 + 2 * DIM + d] = (double)(gr[d] * gm);
        }
        tile_add_node<DIM, NORMAL, TN, DET>(tacc, t, nv, ks);
      }
    }
  }
}

template <int DIM, int T, int TN, bool NORMAL, bool DET, typename R>
__device__ __forceinline__ void scatter_box_any(const PointMapT<R>& pm, const int* o, const ScatterSrc<R>& q,
                                                double* tacc, uint8_t* touched, const Split2* ks, int mask) {
  if (mask == 0) return scatter_box<DIM, T, TN, NORMAL, DET, 2, 2, 2>(pm, o, q, tacc, touched, ks);
  scatter_rolled<DIM, T, TN, NORMAL, DET>(pm, o, q, tacc, touched, ks, mask);
}

// Scatter over any window (three-node spans, nodes outside the tile, which
// go straight to the global accumulators).
template <int DIM, int T, int TN, bool NORMAL, bool DET, typename PT, typename R>
__device__ __forceinline__ void scatter_general(const BodyCtx<PT>& c, unsigned long long* drift,
                                                const PointMapT<R>& pm, const int* o, const ScatterSrc<R>& q,
                                                double* tacc, uint8_t* touched, const Split2* ks) {
  const Geom& g = c.g;
  const bool in_tile = window_in_tile<DIM>(pm, o, T);
  if (!in_tile) {
    atomicAdd(drift, 1ull);
    mark_blocks<DIM>(g, pm, c.flags);
  }
  using TL = TileLayout<DIM, T>;
  const int txy = (pm.ax[0].base - o[0]) + TL::RL * (pm.ax[1].base - o[1]);
  const int bz = DIM == 3 ? pm.ax[2].base - o[2] : 0;
  const R sS = pm.sS, sG = pm.sG;
  for_window<DIM>(pm, [&](int k0, int k1, int k2) {
    const R wz = DIM == 3 ? sel3(pm.ax[2].W, k2) : R(1);
    const R gz = DIM == 3 ? sel3(pm.ax[2].G, k2) : R(0);
    const R w1 = sel3(pm.ax[1].W, k1), g1 = sel3(pm.ax[1].G, k1);
    const R W12 = w1 * wz;
    const R S = sS * pm.ax[0].W[k0] * W12;
    const R gw0 = sG * pm.ax[0].W[k0];
    const R gr[3] = {sG * pm.ax[0].G[k0] * W12, gw0 * (g1 * wz), gw0 * (w1 * gz)};
    NodeVals<DIM, NORMAL, R> nv;
    nv.v[0] = (double)S * q.m;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      nv.v[1 + d] = (double)S * q.mv[d];
      R fi = q.V3[d][0] * gr[0] + q.V3[d][1] * gr[1];
      if (DIM == 3) fi += q.V3[d][2] * gr[2];
      nv.v[1 + DIM + d] = (double)(-fi);
      if constexpr (NORMAL) nv.v[1 + 2 * DIM + d] = (double)(gr[d] * (R)q.m);
    }
    if (in_tile) {
      const int t = txy + k0 + TL::RL * k1 + TL::zoff(bz + k2);
      touched[t] = 1;
      tile_add_node<DIM, NORMAL, TN, DET>(tacc, t, nv, ks);
    } else {
      const int64_t s = node_slot(g, pm.ax[0].base + k0, pm.ax[1].base + k1, DIM == 3 ? pm.ax[2].base + k2 : 0);
      // global accumulator of value i (m, mx, f, normal order of NodeVals)
      auto gadd = [&](double* a0, double* a1, int cls, double v) {
        if constexpr (DET) {
          double q0, q1;
          presplit(v, ks[cls], q0, q1);
          atomicAdd(a0 + s, q0);
          atomicAdd(a1 + s, q1);
        } else {
          atomicAdd(a0 + s, v);
        }
      };
      gadd(c.A.m, c.Ar.m, 0, nv.v[0]);
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        gadd(c.A.mx[d], c.Ar.mx[d], 1, nv.v[1 + d]);
        gadd(c.A.f[d], c.Ar.f[d], 2, nv.v[1 + DIM + d]);
        if constexpr (NORMAL) gadd(c.A.nrm[d], c.Ar.nrm[d], 3, nv.v[1 + 2 * DIM + d]);
      }
    }
  });
}

// Phase 2 for one point: map build and scatter of mapPointsToNodes
// (explicit_usl.cpp:112-164) and the contact normal of
// ContactHuang::generateRules (contact_huang.cpp:91).
template <int DIM, int T, int TN, int ROW, bool NORMAL, bool DET, typename PT>
__device__ __forceinline__ void map_scatter(const BodyCtx<PT>& c, int* err, unsigned long long* drift, int64_t p,
                                            const PT* sp, const int* o, int stepping, double* tacc, uint8_t* touched,
                                            const Split2* ks) {
  using R = PT;
  double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < DIM; d++) x[d] = staged_two<PT, ROW>(sp, c.P, p, kFx, d);
  PointMapT<R> pm;
  const int st = build_map<DIM>(c.g, c.mc, c.sp.cpdi, x, sp[kFext * ROW], pm, err);
  if (st < 0) {
    // outside the domain: inactive from the next map build on
    // (default_points.cpp:217-219); before the first step, at once
    c.P.active[p] = stepping ? 2 : 0;
    return;
  }
  if (st == 0) return;
  ScatterSrc<R> q;
  // the mixed form's two-word mass and velocity (momentum in FP64)
  q.m = sizeof(PT) == 8 ? (double)sp[kFm * ROW] : two_word(c.P.m, c.P.ml, p);
  const R vol = sp[kFvol * ROW];
#pragma unroll
  for (int d = 0; d < 3; d++) q.mv[d] = d < DIM ? q.m * staged_two<PT, ROW>(sp, c.P, p, kFv, d) : 0.0;
  // V * sigma as a symmetric 3x3 (stored xx yy zz xy yz xz)
  R vs[6];
#pragma unroll
  for (int k = 0; k < 6; k++) vs[k] = (DIM == 3 || k == 0 || k == 1 || k == 3) ? sp[(kFs + k) * ROW] * vol : R(0);
  const R V3[3][3] = {{vs[0], vs[3], vs[5]}, {vs[3], vs[1], vs[4]}, {vs[5], vs[4], vs[2]}};
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) q.V3[a][b] = V3[a][b];
  // as in gather_update: the union box of the warp for windows inside the
  // tile, the general path otherwise (and always in the deterministic form)
  const bool in = !DET && window_in_tile<DIM>(pm, o, T);
  const unsigned am = __activemask();
  const unsigned inm = __ballot_sync(am, in);
  if (in)
    scatter_box_any<DIM, T, TN, NORMAL, DET>(pm, o, q, tacc, touched, ks, __reduce_or_sync(inm, span_bits<DIM>(pm)));
  else
    scatter_general<DIM, T, TN, NORMAL, DET>(c, drift, pm, o, q, tacc, touched, ks);
}

// Phase 3: adds the touched nodes of the tile into the body's global
// accumulators (one global atomic per node and value) and flags their node
// blocks for the grid update.
template <int DIM, int T, int TN, bool NORMAL, bool DET, typename PT>
__device__ __forceinline__ void flush_tile(const BodyCtx<PT>& c, const Geom& g, const int* o, const double* tile,
                                           const uint8_t* touched) {
  for (int t = threadIdx.x; t < TN; t += blockDim.x) {
    if (!touched[t]) continue;
    int tx, ty, tz;
    TileLayout<DIM, T>::node(t, tx, ty, tz);
    const int i = o[0] + tx, j = o[1] + ty, k = o[2] + tz;
    const int64_t s = node_slot(g, i, j, k);
    c.flags[node_block(g, i, j, k)] = 1u;
    atomicAdd(c.A.m + s, tile[t]);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      atomicAdd(c.A.mx[d] + s, tile[(1 + d) * TN + t]);
      atomicAdd(c.A.f[d] + s, tile[(4 + d) * TN + t]);
      if (NORMAL) atomicAdd(c.A.nrm[d] + s, tile[(7 + d) * TN + t]);
    }
    if constexpr (DET) {
      const double* t1 = tile + 10 * TN;
      atomicAdd(c.Ar.m + s, t1[t]);
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        atomicAdd(c.Ar.mx[d] + s, t1[(1 + d) * TN + t]);
        atomicAdd(c.Ar.f[d] + s, t1[(4 + d) * TN + t]);
        if (NORMAL) atomicAdd(c.Ar.nrm[d] + s, t1[(7 + d) * TN + t]);
      }
    }
  }
}

template <int DIM, typename PT, int CAP, bool NORMAL, bool SINGLE, bool DET>
__global__ void __launch_bounds__(fused_threads<PT, CAP>(), fused_min_ctas<PT, CAP>())
    k_g2p2g(const __grid_constant__ FusedLaunch<PT> fl) {
  static_assert(!DET || sizeof(PT) == 8, "the deterministic form is FP64");
  __shared__ Split2 ksplit[4];   // deterministic form: per-field split of the item's body
  constexpr int B = fused_bin<DIM>();
  constexpr int T = B + 3;
  constexpr int TN = fused_tile_nodes<DIM, B>();
  constexpr int ROW = cap_row<CAP>();
  constexpr int AL = 16 / (int)sizeof(PT);   // elements per 16 bytes
  constexpr uint32_t kCtxBytes = (uint32_t)ctx_bytes<PT>();
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);          // point arrays
  uint64_t* bar_ctx = reinterpret_cast<uint64_t*>(smem + 8);  // table entry slots 0, 1
  // slot i holds the first ctx_bytes of a table entry (the fields up to
  // Palt); it is addressed by bytes, not as an array of whole entries
  auto slot_ctx = [&](int i) { return reinterpret_cast<BodyCtx<PT>*>(smem + kOffCtx + (size_t)i * kCtxBytes); };
  PT* pts = reinterpret_cast<PT*>(smem + off_pts<PT, CAP>());
  int32_t* act = reinterpret_cast<int32_t*>(smem + off_act<PT, CAP>());
  double* tile = reinterpret_cast<double*>(smem + off_tile<PT, CAP>());  // phase 2: NACC FP64 values
  // phase 1: nodal vt0..2 dv0..2 in the point precision (relative to the
  // reference velocity in the mixed form), in the accumulator tile's space
  constexpr bool SPLIT = split_tiles<PT, NORMAL, DET>();
  PT* tvel = SPLIT ? reinterpret_cast<PT*>(smem + off_tvel<DIM, PT, CAP, NORMAL, DET>()) : reinterpret_cast<PT*>(tile);
  // after the accumulator levels (two in the deterministic form)
  uint8_t* touched = smem + off_touched<DIM, PT, CAP, NORMAL, DET>();

  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init(bar_ctx, 1);
    mbar_init(bar_ctx + 1, 1);
    mbar_init_fence();
  }
  __syncthreads();
  uint32_t parity = 0;
  const int nwork = SINGLE ? fl.nwork_body[fl.one_body] : *fl.nwork;
  // launches over every body: the table entry of each work item arrives by
  // a bulk copy issued one item ahead (slot k & 1 for the CTA's k-th item)
  if (!SINGLE && threadIdx.x == 0 && (int)blockIdx.x < nwork) {
    mbar_arrive_expect_tx(bar_ctx, kCtxBytes);
    bulk_copy_g2s(slot_ctx(0), fl.bodies + fl.flat_body[blockIdx.x], kCtxBytes, bar_ctx);
  }
  // the CTA's next item (claim_item), slot k & 1 for its k-th item: written
  // by thread 0 before a barrier of the item, read by every thread after the
  // item's last barrier
  __shared__ int next_item[2];
  int k = 0;
  for (int w = blockIdx.x; w < nwork; w = SINGLE ? w + (int)gridDim.x : next_item[k & 1], k++) {
    // thread 0 claims the next item now and publishes it (and, over the
    // table, starts the copy of its entry) before the item's first barrier
    const int wn = !SINGLE && threadIdx.x == 0 ? claim_item(fl.queue) : 0;
    bool ahead = false;   // thread 0: the next entry's copy is in flight
    auto publish_next = [&]() {
      if (SINGLE || threadIdx.x != 0) return;
      next_item[k & 1] = wn;
      if (wn < nwork) {
        // the other slot was last read by the previous item (all threads
        // passed its closing barrier)
        const int other = (k & 1) ^ 1;
        fence_async_shared();
        mbar_arrive_expect_tx(bar_ctx + other, kCtxBytes);
        bulk_copy_g2s(slot_ctx(other), fl.bodies + fl.flat_body[wn], kCtxBytes, bar_ctx + other);
        ahead = true;
      }
    };
    int item, body_of_item;
    if (SINGLE) {
      body_of_item = fl.one_body;
      item = fl.item_off[fl.one_body] + w;
    } else {
      body_of_item = fl.flat_body[w];
      item = fl.flat_item[w];
      const int slot = k & 1;
      const bool got = mbar_wait_bounded(bar_ctx + slot, (uint32_t)((k >> 1) & 1), fl.err, fl.wait_polls);
      if (__syncthreads_or(got ? 0 : 1)) {
        // let the copy in flight land before leaving (the next entry's copy
        // is not issued yet)
        if (threadIdx.x == 0) {
          if (!got) mbar_wait_bounded(bar_ctx + slot, (uint32_t)((k >> 1) & 1), fl.err);
          queue_done(fl.queue);
        }
        return;
      }
    }
    const BodyCtx<PT>& c = SINGLE ? fl.one : *slot_ctx(k & 1);
    if (!SINGLE) {
      // items of the other kind (contact normal or not) belong to the other launch
      if ((c.needs_normal != 0) != NORMAL) {
        publish_next();
        __syncthreads();
        continue;
      }
    }
    const int prime = c.prime;
    if (fl.prime_pass && !prime) {
      publish_next();
      __syncthreads();   // every thread has read the staged entry
      continue;
    }
    const int do_g2p = (prime || !(fl.phases & 1)) ? 0 : 1;
    const bool do_p2g = (fl.phases & 2) != 0;
    const PointsT<PT>& P = c.P;
    const Geom& g = c.g;
    const int bin = fl.work_bin[item];
    const int64_t pstart = fl.work_start[item];
    const int n = fl.work_end[item] - (int)pstart;
    // bulk copy windows: 16-byte aligned starts, sizes rounded up to 16 bytes
    const int64_t sp0 = pstart & ~(int64_t)(AL - 1), s4 = pstart & ~(int64_t)3;
    const int offp = (int)(pstart - sp0), off4 = (int)(pstart - s4);
    const int np = (offp + n + AL - 1) & ~(AL - 1), n4 = (off4 + n + 3) & ~3;
    if (threadIdx.x == 0) {
      const PT* src[kNF] = {P.x[0], P.x[1], P.x[2], P.v[0], P.v[1], P.v[2], P.u[0], P.u[1], P.u[2],
                            P.s[0], P.s[1], P.s[2], P.s[3], P.s[4], P.s[5], P.vol, P.m, P.ext};
      fence_async_shared();
      mbar_arrive_expect_tx(bar, (uint32_t)(kNF * np * sizeof(PT) + n4 * 4));
#pragma unroll 1
      for (int f = 0; f < kNF; f++) bulk_copy_g2s(pts + f * ROW, src[f] + sp0, (uint32_t)(np * sizeof(PT)), bar);
      bulk_copy_g2s(act, P.active + s4, (uint32_t)(n4 * 4), bar);
    }
    int o[3] = {0, 0, 0};
    {
      const int bx = bin % c.bg.nbx;
      const int r = bin / c.bg.nbx;
      o[0] = bx * B - 1;
      o[1] = (r % c.bg.nby) * B - 1;
      o[2] = DIM == 3 ? (r / c.bg.nby) * B - 1 : 0;
    }
    // reference velocity of the mixed form: the item's first point (any
    // value is exact; one close to the item's velocities keeps the
    // differences small), read here from global memory (the same value the
    // staged copy receives)
    double vref[3] = {0.0, 0.0, 0.0};
    if (do_g2p) {
      if constexpr (sizeof(PT) == 4) {
#pragma unroll
        for (int d = 0; d < DIM; d++) vref[d] = (double)P.v[d][pstart];
      }
      // nodal velocities of the tile
      if constexpr (sizeof(PT) == 8) {
        for (int t = threadIdx.x; t < TN; t += blockDim.x) {
          int tx, ty, tz;
          if (!TileLayout<DIM, T>::node(t, tx, ty, tz)) continue;
          const int i = o[0] + tx, j = o[1] + ty, k = o[2] + tz;
          if (i < 0 || j < 0 || k < 0 || i >= g.nn[0] || j >= g.nn[1] || k >= g.nn[2]) continue;
          const int64_t s = node_slot(g, i, j, k);
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            tvel[d * TN + t] = c.V.vt[d][s];
            tvel[(3 + d) * TN + t] = c.V.dv[d][s];
          }
        }
      } else {
        // mixed form: every thread issues the loads of up to two nodes
        // before its first shared-memory store (one or two memory latencies
        // per item) and stores the values in FP32, relative to vref
        constexpr int NT = fused_threads<PT, CAP>();
        constexpr int ITER = (TN + NT - 1) / NT;
        constexpr int CH = ITER > 2 ? 2 : ITER;   // nodes per thread in flight (registers)
#pragma unroll 1
        for (int it0 = 0; it0 < ITER; it0 += CH) {
          double vv[CH][2 * DIM];
          int tt[CH];
#pragma unroll
          for (int ic = 0; ic < CH; ic++) {
            const int t = (int)threadIdx.x + (it0 + ic) * NT;
            tt[ic] = -1;
            int tx, ty, tz;
            if (t >= TN || !TileLayout<DIM, T>::node(t, tx, ty, tz)) continue;
            const int i = o[0] + tx, j = o[1] + ty, k = o[2] + tz;
            if (i < 0 || j < 0 || k < 0 || i >= g.nn[0] || j >= g.nn[1] || k >= g.nn[2]) continue;
            const int64_t s = node_slot(g, i, j, k);
            tt[ic] = t;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
              vv[ic][d] = c.V.vt[d][s];
              vv[ic][DIM + d] = c.V.dv[d][s];
            }
          }
#pragma unroll
          for (int ic = 0; ic < CH; ic++) {
            const int t = tt[ic];
            if (t < 0) continue;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
              tvel[d * TN + t] = (PT)(vv[ic][d] - vref[d]);
              tvel[(3 + d) * TN + t] = (PT)vv[ic][DIM + d];
            }
          }
        }
      }
    }
    if constexpr (SPLIT) {
      // the accumulators are cleared while the point arrays arrive
      if (do_p2g) {
        for (int t = threadIdx.x; t < 7 * TN; t += blockDim.x) tile[t] = 0.0;
        for (int t = threadIdx.x; t < TN; t += blockDim.x) touched[t] = 0;
      }
    }
    publish_next();
    const bool arrived = mbar_wait_bounded(bar, parity, fl.err, fl.wait_polls);
    // one decision for the whole CTA (also the barrier after the tile loads)
    if (__syncthreads_or(arrived ? 0 : 1)) {
      // let copies in flight land before leaving
      if (!arrived) mbar_wait_bounded(bar, parity, fl.err);
      if (threadIdx.x == 0) {
        if (ahead) mbar_wait_bounded(bar_ctx + ((k & 1) ^ 1), (uint32_t)(((k + 1) >> 1) & 1), fl.err);
        if (!SINGLE) queue_done(fl.queue);
      }
      return;
    }
    parity ^= 1u;
    if constexpr (SPLIT) {
      // each thread takes its points through gather, update, map and
      // scatter in one go
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int64_t p = pstart + j;
        const int a = act[off4 + j];
        if (a == 0) continue;
        if (do_g2p) {
          if (a == 2) {
            // left the domain at the last move; generateMap deactivates it now
            P.active[p] = 0;
            act[off4 + j] = 0;
            continue;
          }
          gather_update<DIM, T, TN, ROW, DET>(c, fl.err, fl.drift, p, pts + offp + j, o, tvel, vref);
        }
        if (do_p2g && a == 1)
          map_scatter<DIM, T, TN, ROW, NORMAL, DET>(c, fl.err, fl.drift, p, pts + offp + j, o, prime ? 0 : 1, tile,
                                                     touched, ksplit);
      }
      if (do_p2g) {
        __syncthreads();
        flush_tile<DIM, T, TN, NORMAL, DET>(c, g, o, tile, touched);
      }
      __syncthreads();
      continue;
    }
    if (do_g2p) {
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
        gather_update<DIM, T, TN, ROW, DET>(c, fl.err, fl.drift, p, pts + offp + j, o, tvel, vref);
      }
      __syncthreads();
    }
    if (do_p2g) {
      constexpr int NACC = fused_nacc(NORMAL);
      for (int t = threadIdx.x; t < NACC * TN; t += blockDim.x) tile[t] = 0.0;
      if constexpr (DET) {
        for (int t = threadIdx.x; t < NACC * TN; t += blockDim.x) tile[10 * TN + t] = 0.0;
        if (threadIdx.x < 4) {
          // split of each field from the body's bounds (k_det_bounds)
          const unsigned long long* bb = fl.bounds + 4 * (SINGLE ? fl.one_body : body_of_item);
          ksplit[threadIdx.x] = make_split(__longlong_as_double((long long)bb[threadIdx.x]), P.n);
        }
      }
      for (int t = threadIdx.x; t < TN; t += blockDim.x) touched[t] = 0;
      __syncthreads();
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        if (act[off4 + j] != 1) continue;
        // a point found outside the domain here is at a regular step's map
        // build (inactive from the next step on: state 2), or at the priming
        // map build before the first step (inactive at once)
        map_scatter<DIM, T, TN, ROW, NORMAL, DET>(c, fl.err, fl.drift, pstart + j, pts + offp + j, o, prime ? 0 : 1,
                                                   tile, touched, ksplit);
      }
      __syncthreads();
      flush_tile<DIM, T, TN, NORMAL, DET>(c, g, o, tile, touched);
    }
    __syncthreads();
  }
  if (!SINGLE && threadIdx.x == 0) queue_done(fl.queue);
}

}  // namespace mpmb200
