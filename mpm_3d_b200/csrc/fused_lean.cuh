// Lean form of the fused gather + point update + scatter kernel: each thread
// takes its points from gather to scatter, with no staged copy of the point
// arrays.
//
// A CTA of NT threads works on one work item at a time (at most PPT * NT
// points of one bin of one body, PPT points per thread):
//   0. the CTA stages the nodal velocities of the bin's node tile and clears
//      a separate FP64 accumulator tile;
//   1. one barrier; then each thread takes its points (global loads,
//      coalesced: consecutive threads, consecutive points) through gather,
//      state update (movePoints, calculateStrainRate, updateDensity,
//      updateStress), map build at the new position and scatter into the
//      accumulator tile, with no barrier between the phases;
//   2. one barrier; the touched tile nodes are added into the global
//      accumulators (one global atomic per node and value).
// Shared memory holds only the two tiles (about 41 KB in FP64, 31 KB in the
// mixed form), so residency is set by registers: the register budget (80 per
// thread in FP64, 64 in the mixed form) leaves room for 24 or 32 resident
// warps per SM, and was measured faster than 128 registers without spills
// at 16 warps. The material is a template parameter (MAT >= 0 compiles one
// constitutive model; -1 dispatches at run time), which keeps the other
// models' state out of the register budget. The arithmetic of every phase is
// the one of the staged kernel (fused.cuh), so both kernels give the same
// results up to the order of the nodal sums.
#pragma once

#include "fused.cuh"

namespace mpmb200 {

// Points per work item the autotuner chooses from: 128 (CTAs of 128
// threads), 256 (256 threads) and 512 (256 threads, two points each: one
// tile load, clear and flush for a whole 4x4x4 bin of 8 points per cell).
// 512 is the default: measured fastest on the column collapse and the
// block-drop ensemble in both forms (FP64 and mixed), 5 to 10 % ahead of
// 256 (a 128-thread variant with 96 registers and four points per thread
// was slower than both).
__host__ __device__ constexpr bool lean_size_ok(int cap) { return cap == 128 || cap == 256 || cap == 512; }
constexpr int kDefaultLeanCap = 512;

// Resident CTAs per SM the register budget is sized for: 80 registers per
// thread in FP64, 64 in the mixed form (measured: more resident warps beat
// the register spills this costs).
template <typename PT, int NT>
__host__ __device__ constexpr int lean_min_ctas() {
  return (sizeof(PT) == 4 ? 4 : 3) * (256 / NT);
}

// Shared memory: mbarriers (table entry slots 0 and 1) | table entry slots
// [2] | velocity tile [2 DIM][TN] in the point precision | accumulator tile
// [NACC][TN] FP64 | touched [TN].
template <int DIM, typename PT>
__host__ __device__ constexpr size_t lean_off_tvel() {
  return kOffCtx + 2 * ctx_bytes<PT>();
}
template <int DIM, typename PT>
__host__ __device__ constexpr size_t lean_off_tacc() {
  return (lean_off_tvel<DIM, PT>() + sizeof(PT) * 2 * DIM * fused_tile_nodes<DIM, fused_bin<DIM>()>() + 15) / 16 * 16;
}
template <int DIM, typename PT, bool NORMAL>
__host__ __device__ constexpr size_t lean_off_touched() {
  return lean_off_tacc<DIM, PT>() + sizeof(double) * fused_nacc(NORMAL) * fused_tile_nodes<DIM, fused_bin<DIM>()>();
}
template <int DIM, typename PT, bool NORMAL>
__host__ __device__ constexpr size_t lean_smem_bytes() {
  return lean_off_touched<DIM, PT, NORMAL>() + fused_tile_nodes<DIM, fused_bin<DIM>()>();
}

// Prefetch into L2: each thread asks for its own points' lines when its
// item starts, so that the update's loads of x_t, the stress and the
// volume, which come after the gather, find them in L2 rather than wait on
// DRAM (measured 3 to 6 % faster). A bulk prefetch of the CTA's next item
// by one thread, in addition or instead, was measured slower.
template <typename PT>
__device__ __forceinline__ void prefetch_point_l2(const PointsT<PT>& P, int64_t q) {
  const PT* arrs[kNF] = {P.x[0], P.x[1], P.x[2], P.v[0], P.v[1], P.v[2], P.u[0], P.u[1], P.u[2],
                         P.s[0], P.s[1], P.s[2], P.s[3], P.s[4], P.s[5], P.vol, P.m, P.ext};
#pragma unroll
  for (int f = 0; f < kNF; f++) prefetch_l2(arrs[f] + q);
  if constexpr (sizeof(PT) == 4) {
    const PT* lows[7] = {P.xl[0], P.xl[1], P.xl[2], P.vl[0], P.vl[1], P.vl[2], P.ml};
#pragma unroll
    for (int f = 0; f < 7; f++) prefetch_l2(lows[f] + q);
  }
}

// A position, velocity or mass in double: the FP64 form's value, or the
// mixed form's two words (hi + lo).
template <typename PT>
__device__ __forceinline__ double lean_two(const PT* hi, const PT* lo, int64_t p) {
  if constexpr (sizeof(PT) == 8) return hi[p];
  else return (double)hi[p] + (double)lo[p];
}

// Stores a position or velocity (the mixed form splits it into its two words).
template <typename PT>
__device__ __forceinline__ void lean_store_two(PT* hi, PT* lo, int64_t p, double v) {
  if constexpr (sizeof(PT) == 8) {
    hi[p] = v;
  } else {
    float h, l;
    split_two_word(v, h, l);
    hi[p] = h;
    lo[p] = l;
  }
}

// Stress update of one point for material MAT (-1: the body's kind at run
// time). s6 holds the stress before the step on entry, after it on exit.
template <int DIM, int MAT, typename R, typename PT>
__device__ __forceinline__ void lean_stress(const BodyCtx<PT>& c, int64_t p, const R L[3][3], R* s6, R m, R vol,
                                            R dt) {
  const PointsT<PT>& P = c.P;
  const int kind = MAT >= 0 ? MAT : c.mat.kind;
  if (kind == 1) {
    neohookean_update<R>(P.ms, p, L, s6, (R)c.mat.G, (R)c.mat.lambda, dt);
  } else if (kind == 2) {
    sand_update<DIM, R>(P.ms, p, L, s6, m, vol, c.mat, dt);
  } else {
    jaumann_point<DIM, R>(L, s6, c.mat, c.sp.dt);
  }
}

// One point through both phases. `a` is its active state (1 active, 2 left
// the domain at the last move). The arithmetic follows gather_update and
// map_scatter of the staged kernel.
template <int DIM, int T, int TN, bool NORMAL, int MAT, typename PT>
__device__ __forceinline__ void lean_point(const BodyCtx<PT>& c, int* err, unsigned long long* drift, int64_t p,
                                           int a, const int* o, const PT* tvel, const double* vref, double* tacc,
                                           uint8_t* touched, int do_g2p, bool do_p2g, int stepping) {
  using R = PT;
  const PointsT<PT>& P = c.P;
  const R dt = (R)c.sp.dt;
  const R ext = P.ext[p];
  const R sG = map_grad_scale(c.g, ext);
  // Register budget: values the later phases need are read back from the
  // point's arrays (L1/L2 hits) rather than kept across the gather and the
  // map builds: the position and displacement after the gather, the extent
  // for the second map, and the scatter's sources (the values the update
  // stored). Measured 6 to 9 % faster than keeping them (fewer spills). The
  // update issues its loads before its stores: the compiler cannot move a
  // load above a store to an array it may alias.
  // Position in double (the mixed form's two words), velocity vd.
  double x[3] = {0.0, 0.0, 0.0}, vd[3] = {0.0, 0.0, 0.0};
  R u[3] = {R(0), R(0), R(0)};
#pragma unroll
  for (int d = 0; d < DIM; d++) x[d] = lean_two(P.x[d], P.xl[d], p);
  R s6[6], vol;
  if (do_g2p) {
    if (a == 2) {
      // left the domain at the last move; generateMap deactivates it now
      P.active[p] = 0;
      return;
    }
    GatherSum<R> gs;
    {
      PointMapT<R> pm;
      const int st = build_map<DIM>(c.g, c.mc, c.sp.cpdi, x, ext, pm, err, sG);
      if (st > 0) {
        const bool in = window_in_tile<DIM>(pm, o, T);
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
    }
    // movePoints (explicit_usl.cpp:279-292); the mixed form adds the
    // increments to its two-word x and x_t in FP64
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const R dx = dt * gs.du[d];
      x[d] = lean_two(P.x[d], P.xl[d], p) + (double)dx;
      u[d] = P.u[d][p];
      vd[d] = lean_two(P.v[d], P.vl[d], p) + (double)gs.dv[d];
      u[d] = u[d] + dx;
      lean_store_two(P.x[d], P.xl[d], p, x[d]);
      lean_store_two(P.v[d], P.vl[d], p, vd[d]);
      P.u[d][p] = u[d];
    }
    vol = P.vol[p] * exp(dt * (gs.L[0][0] + gs.L[1][1] + gs.L[2][2]));
    P.vol[p] = vol;
#pragma unroll
    for (int k = 0; k < 6; k++) s6[k] = P.s[k][p];
    if (c.mat.has_material) {
      lean_stress<DIM, MAT, R>(c, p, gs.L, s6, MAT == 2 || MAT < 0 ? P.m[p] : R(0), vol, dt);
#pragma unroll
      for (int k = 0; k < 6; k++) P.s[k][p] = s6[k];
    }
    if (P.L != nullptr) {
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) P.L[9 * p + 3 * i + j] = (double)gs.L[i][j];
    }
  }
  if (!do_p2g || a != 1) return;
  // map build and scatter at the new position (mapPointsToNodes,
  // explicit_usl.cpp:112-164; contact normal, contact_huang.cpp:91)
  PointMapT<R> pm;
  const R ext2 = P.ext[p];
  const int st = build_map<DIM>(c.g, c.mc, c.sp.cpdi, x, ext2, pm, err, map_grad_scale(c.g, ext2));
  if (st < 0) {
    // outside the domain: inactive from the next map build on
    // (default_points.cpp:217-219); before the first step, at once
    P.active[p] = stepping ? 2 : 0;
    return;
  }
  if (st == 0) return;
  ScatterSrc<R> q;
  q.m = lean_two(P.m, P.ml, p);
#pragma unroll
  for (int d = 0; d < 3; d++) q.mv[d] = d < DIM ? q.m * lean_two(P.v[d], P.vl[d], p) : 0.0;
  const R vol_s = P.vol[p];
  R vs[6];
#pragma unroll
  for (int k = 0; k < 6; k++) vs[k] = (DIM == 3 || k == 0 || k == 1 || k == 3) ? P.s[k][p] * vol_s : R(0);
  const R V3[3][3] = {{vs[0], vs[3], vs[5]}, {vs[3], vs[1], vs[4]}, {vs[5], vs[4], vs[2]}};
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) q.V3[i][j] = V3[i][j];
  const bool in = window_in_tile<DIM>(pm, o, T);
  const unsigned am = __activemask();
  const unsigned inm = __ballot_sync(am, in);
  if (in)
    scatter_box_any<DIM, T, TN, NORMAL, false>(pm, o, q, tacc, touched, nullptr,
                                              __reduce_or_sync(inm, span_bits<DIM>(pm)));
  else
    scatter_general<DIM, T, TN, NORMAL, false>(c, drift, pm, o, q, tacc, touched, nullptr);
}

template <int DIM, typename PT, int NT, int PPT, bool NORMAL, bool SINGLE, int MAT>
__global__ void __launch_bounds__(NT, lean_min_ctas<PT, NT>())
    k_g2p2g_lean(const __grid_constant__ FusedLaunch<PT> fl) {
  constexpr int B = fused_bin<DIM>();
  constexpr int T = B + 3;
  constexpr int TN = fused_tile_nodes<DIM, B>();
  constexpr int NACC = fused_nacc(NORMAL);
  constexpr uint32_t kCtxBytes = (uint32_t)ctx_bytes<PT>();
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar_ctx = reinterpret_cast<uint64_t*>(smem + 8);   // table entry slots 0, 1
  auto slot_ctx = [&](int i) { return reinterpret_cast<BodyCtx<PT>*>(smem + kOffCtx + (size_t)i * kCtxBytes); };
  PT* tvel = reinterpret_cast<PT*>(smem + lean_off_tvel<DIM, PT>());
  double* tacc = reinterpret_cast<double*>(smem + lean_off_tacc<DIM, PT>());
  uint8_t* touched = smem + lean_off_touched<DIM, PT, NORMAL>();

  if (!SINGLE) {
    if (threadIdx.x == 0) {
      mbar_init(bar_ctx, 1);
      mbar_init(bar_ctx + 1, 1);
      mbar_init_fence();
    }
    __syncthreads();
  }
  const int nwork = SINGLE ? fl.nwork_body[fl.one_body] : *fl.nwork;
  // launches over every body: the table entry of each work item arrives by
  // a bulk copy issued one item ahead (slot k & 1 for the CTA's k-th item)
  if (!SINGLE && threadIdx.x == 0 && (int)blockIdx.x < nwork) {
    mbar_arrive_expect_tx(bar_ctx, kCtxBytes);
    bulk_copy_g2s(slot_ctx(0), fl.bodies + fl.flat_body[blockIdx.x], kCtxBytes, bar_ctx);
  }
  // the CTA's next item, slot k & 1 for its k-th item: written by thread 0
  // before a barrier of the item, read by every thread after the item's
  // last barrier (the slot is written again two items later)
  __shared__ int next_item[2];
  int k = 0;
  for (int w = blockIdx.x; w < nwork; w = SINGLE ? w + (int)gridDim.x : next_item[k & 1], k++) {
    // thread 0 claims the next item now and publishes it (and, over the
    // table, starts the copy of its entry) before the item's first barrier,
    // so that the claim's latency overlaps the tile loads
    const int wn = !SINGLE && threadIdx.x == 0 ? claim_item(fl.queue) : 0;
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
      }
    };
    int item;
    if (SINGLE) {
      item = fl.item_off[fl.one_body] + w;
    } else {
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
    if (n > PPT * NT && threadIdx.x == 0) atomicOr(fl.err, kErrItemCap);   // the work list was cut for another size
    // activity of the thread's points (coalesced loads issued before the tile work)
    int a[PPT];
#pragma unroll
    for (int r = 0; r < PPT; r++) {
      const int j = (int)threadIdx.x + r * NT;
      a[r] = j < n ? P.active[pstart + j] : 0;
      if (j < n) prefetch_point_l2(P, pstart + j);
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
    // differences small)
    double vref[3] = {0.0, 0.0, 0.0};
    if (do_g2p) {
      if constexpr (sizeof(PT) == 4) {
#pragma unroll
        for (int d = 0; d < DIM; d++) vref[d] = (double)P.v[d][pstart];
      }
      // nodal velocities of the tile: each thread issues the loads of up to
      // two nodes before its first shared-memory store
      constexpr int ITER = (TN + NT - 1) / NT;
      constexpr int CH = ITER > 2 ? 2 : ITER;
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
          const int i = o[0] + tx, jj = o[1] + ty, kk = o[2] + tz;
          if (i < 0 || jj < 0 || kk < 0 || i >= g.nn[0] || jj >= g.nn[1] || kk >= g.nn[2]) continue;
          const int64_t s = node_slot(g, i, jj, kk);
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
    if (do_p2g) {
      for (int t = threadIdx.x; t < NACC * TN; t += NT) tacc[t] = 0.0;
      for (int t = threadIdx.x; t < TN; t += NT) touched[t] = 0;
    }
    publish_next();
    __syncthreads();
#pragma unroll 1
    for (int r = 0; r < PPT; r++) {
      if (a[r] != 0)
        lean_point<DIM, T, TN, NORMAL, MAT>(c, fl.err, fl.drift, pstart + threadIdx.x + r * NT, a[r], o, tvel, vref,
                                            tacc, touched, do_g2p, do_p2g, prime ? 0 : 1);
    }
    if (do_p2g) {
      __syncthreads();
      flush_tile<DIM, T, TN, NORMAL, false>(c, g, o, tacc, touched);
    }
    __syncthreads();
  }
  if (!SINGLE && threadIdx.x == 0) queue_done(fl.queue);
}

}  // namespace mpmb200
