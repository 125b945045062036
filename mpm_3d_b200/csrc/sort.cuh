// Binning of points for the fused gather/scatter kernel.
//
// Points are kept grouped by bin: a block of B^dim cells (4x4x4 in 3D, 8x8
// in 2D). Within a bin they are laid out rank-major: first the first point
// of every cell (in cell order), then the second point of every cell, and so
// on. A warp of consecutive points therefore covers distinct cells, so the
// points of one warp never add into the same node at the same time in the
// shared-memory tile (same-address atomics serialise).
//
// The sort is a counting sort in three passes (count + rank, bin offsets,
// scatter); it is only run when points have drifted out of their bin's tile,
// because the fused kernel stays correct (slower) for drifted points.
#pragma once

#include "geom.cuh"

namespace mpmb200 {

// Bin layout for a grid.
struct BinGeom {
  int B;             // cells per bin per axis (4 in 3D, 8 in 2D)
  int cells_per_bin; // B^dim (64)
  int nbx, nby, nbz; // bins per axis
  int nbins;         // total bins (the inactive points use key nbins)
  int T;             // tile nodes per axis, B + 3
  int tile_nodes;    // T^dim
};

// Cell of a point for binning, clamped into the grid.
template <int DIM>
__device__ __forceinline__ void point_cell(const Geom& g, const double* x, int* c) {
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    int v = (int)floor(x[d] * (g.N[d] / g.L[d]));
    v = v < 0 ? 0 : (v >= g.N[d] ? g.N[d] - 1 : v);
    c[d] = v;
  }
}

template <int DIM>
__device__ __forceinline__ void bin_of(const BinGeom& bg, const int* c, int* bin, int* local) {
  const int bx = c[0] / bg.B, by = c[1] / bg.B, bz = DIM == 3 ? c[2] / bg.B : 0;
  *bin = bx + bg.nbx * (by + bg.nby * bz);
  const int lx = c[0] - bx * bg.B, ly = c[1] - by * bg.B, lz = DIM == 3 ? c[2] - bz * bg.B : 0;
  *local = lx + bg.B * (ly + bg.B * lz);
}

// Pass 1: key (bin * cells_per_bin + local cell) and rank within the cell.
// Inactive points go to the trailing key nbins * cells_per_bin.
template <int DIM>
__global__ void k_sort_count(Geom g, BinGeom bg, PointsDev P, int32_t* key, int32_t* rank, int32_t* cell_count) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P.n; p += stride) {
    int k;
    if (P.active[p] == 0) {
      k = bg.nbins * bg.cells_per_bin;
    } else {
      double xp[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int d = 0; d < DIM; d++) xp[d] = P.x[d][p];
      int c[3] = {0, 0, 0};
      point_cell<DIM>(g, xp, c);
      int b, l;
      bin_of<DIM>(bg, c, &b, &l);
      k = b * bg.cells_per_bin + l;
    }
    key[p] = k;
    rank[p] = atomicAdd(cell_count + k, 1);
  }
}

// Pass 2a: per-bin point counts (one thread per bin, sums its cells). The
// trailing inactive bin is bin index nbins.
__global__ void k_bin_totals(BinGeom bg, const int32_t* cell_count, int32_t* bin_total) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > bg.nbins) return;
  int s = 0;
  if (b < bg.nbins) {
    for (int l = 0; l < bg.cells_per_bin; l++) s += cell_count[b * bg.cells_per_bin + l];
  } else {
    s = cell_count[bg.nbins * bg.cells_per_bin];
  }
  bin_total[b] = s;
}

// Exclusive scan of n int32 values in place, one CTA of 1024 threads,
// in chunks (the bin count is at most a few hundred thousand).
__global__ void k_scan_small(int32_t* v, int n, int32_t* total) {
  __shared__ int32_t warp_sums[32];
  __shared__ int32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = 0; base < n; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int x = i < n ? v[i] : 0;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int ws = warp_sums[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, ws, o);
        if (lane >= o) ws += y;
      }
      warp_sums[lane] = ws;
    }
    __syncthreads();
    const int before = (wid > 0 ? warp_sums[wid - 1] : 0) + carry;
    if (i < n) v[i] = before + incl - x;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

// Pass 3: destination of each point inside its bin (rank-major order) and
// the permutation copy of every per-point array.
struct PointArrays {
  double* f[24];   // double arrays (x, v, u, s, vol, m, ext, ...)
  int nf;
  int32_t* i[4];   // int arrays (active, pid)
  int ni;
  double* L9;      // 9 doubles per point (debug velocity gradient) or null
};

__global__ void k_sort_scatter(BinGeom bg, int64_t n, const int32_t* key, const int32_t* rank, const int32_t* cell_count,
                               const int32_t* bin_start, PointArrays src, PointArrays dst) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += stride) {
    const int k = key[p];
    const int r = rank[p];
    const int b = k / bg.cells_per_bin;
    int64_t pos = bin_start[b];
    if (b < bg.nbins) {
      const int l = k - b * bg.cells_per_bin;
      const int32_t* cc = cell_count + (int64_t)b * bg.cells_per_bin;
      int below = 0, same_level = 0;
      for (int c = 0; c < bg.cells_per_bin; c++) {
        const int cnt = cc[c];
        below += cnt < r ? cnt : r;
        same_level += (c < l && cnt > r) ? 1 : 0;
      }
      pos += below + same_level;
    } else {
      pos += r;
    }
    for (int a = 0; a < src.nf; a++) dst.f[a][pos] = src.f[a][p];
    for (int a = 0; a < src.ni; a++) dst.i[a][pos] = src.i[a][p];
    if (src.L9 != nullptr)
      for (int a = 0; a < 9; a++) dst.L9[9 * pos + a] = src.L9[9 * p + a];
  }
}

// Work list: every non-empty bin split into items of at most `cap` points:
// bin id and [start, end) of the item's points. At most
// nonempty_bins + n / cap items.
__global__ void k_bin_work(BinGeom bg, const int32_t* bin_start, int cap, int32_t* work_bin, int32_t* work_start,
                           int32_t* work_end, int32_t* nwork) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bg.nbins) return;
  const int s = bin_start[b], e = bin_start[b + 1];
  if (e <= s) return;
  const int items = (e - s + cap - 1) / cap;
  const int first = atomicAdd(nwork, items);
  for (int i = 0; i < items; i++) {
    work_bin[first + i] = b;
    work_start[first + i] = s + i * cap;
    work_end[first + i] = min(e, s + (i + 1) * cap);
  }
}

}  // namespace mpmb200
