// Binning of points for the fused gather/scatter kernel, for every body of a
// batch in one set of launches.
//
// Points are kept grouped by bin: a block of B^dim cells (4x4x4 in 3D, 8x8
// in 2D). A point's cell here is the cell of its shape-function window's
// base node (the cell of the lower corner, x - extent/2), not the cell that
// contains x: the kernels visit a window as offsets from its base, so two
// points with the same base add into the same tile nodes in the same
// instruction, while points with distinct bases never collide. (Binning by
// the containing cell puts the two points of a cell along an axis on bases
// k-1 and k whenever the lower corner of one crosses a node, and neighbours
// then share bases.) Within a bin points are laid out rank-major: first the
// first point of every cell (in cell order), then the second point of every
// cell, and so on, so a warp of consecutive points covers distinct bases and
// its shared-memory atomics do not serialise on equal addresses. Within a
// cell, points are ranked by window class (the axes along which the window
// spans three nodes) before arrival order: in the regular layouts of a few
// points per cell the r-th point of every cell then has the same window
// shape, and a warp's node box (the union of its lanes' shapes) is its
// lanes' own.
//
// The sort is a counting sort over the batch's concatenated point space
// (count + rank, per-bin totals, one exclusive scan over all bodies' bins,
// scatter), then the work list of (body, bin, point range) items. It runs
// when jobs join or leave the batch and every sort_interval steps, because
// the fused kernel stays correct (slower) for points that drifted out of
// their bin's tile.
#pragma once

#include "geom.cuh"
#include "state.cuh"

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

// Per-body table entry. The first part (up to Palt) is what the fused
// kernel stages in shared memory for a work item.
template <typename PT>
struct alignas(16) BodyCtx {
  Geom g;
  MapConst mc;
  BinGeom bg;
  StepParams sp;
  MaterialParams mat;
  PointsT<PT> P;        // current storage order
  NodesVel V;
  NodesAcc A;
  NodesAcc Ar;          // deterministic form: level-1 (remainder) sums, else null
  uint32_t* flags;      // node-block flags of the body's job (its first block)
  int needs_normal;     // accumulate the contact normal (first body of a contact)
  int prime;            // 1 until the body's first scatter has run
  // sort side
  PointsT<PT> Palt;     // second buffer; swapped with P after a sort
  int64_t point_off;    // first point in the batch's point space
  int64_t bin_off;      // first entry in the batch's bin arrays (nbins + 1 per body)
  int64_t cell_off;     // first cell counter (nbins * cells_per_bin + 1 per body)
  int inst;
};

// Index of the entry whose [end[b-1], end[b]) range holds i (end: inclusive
// prefix sums, n entries).
template <typename I>
__device__ __forceinline__ int find_range(const I* end, int n, int64_t i) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (end[mid] > i) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Cell of a point for binning: the cell of its window's base, x - a with a
// half the point's extent (the lower corner of build_map), clamped into the
// grid. Windows then span base .. base+2, inside the bin's node tile (which
// starts one node below the bin) with one node to spare below.
// Also returns the point's window class: bit d set when the upper corner
// x + a lies in a later element than the lower one (a three-node span).
template <int DIM, typename PT>
__device__ __forceinline__ int point_cell(const Geom& g, const PT* x, double a, int* c) {
  int cls = 0;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    const double nl = g.N[d] / g.L[d];
    const double lo = floor(((double)x[d] - a) * nl);
    cls |= (floor(((double)x[d] + a) * nl) != lo ? 1 : 0) << d;
    int v = (int)lo;
    v = v < 0 ? 0 : (v >= g.N[d] ? g.N[d] - 1 : v);
    c[d] = v;
  }
  return cls;
}

template <int DIM>
__device__ __forceinline__ void bin_of(const BinGeom& bg, const int* c, int* bin, int* local) {
  const int bx = c[0] / bg.B, by = c[1] / bg.B, bz = DIM == 3 ? c[2] / bg.B : 0;
  *bin = bx + bg.nbx * (by + bg.nby * bz);
  const int lx = c[0] - bx * bg.B, ly = c[1] - by * bg.B, lz = DIM == 3 ? c[2] - bz * bg.B : 0;
  *local = lx + bg.B * (ly + bg.B * lz);
}

// Pass 0: clears the cell counters, the cells' class histograms and the
// per-body work-item counts.
__global__ void k_sort_clear(const BatchHdr* hdr, int32_t* cell_count, unsigned long long* cell_hist,
                             int32_t* nwork_body) {
  const int64_t n = hdr->cells;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    cell_count[i] = 0;
    cell_hist[i] = 0ull;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < hdr->nbodies; i += stride) nwork_body[i] = 0;
}

// Pass 1: key (bin * cells_per_bin + local cell, local to the body) and rank
// within the cell (arrival order). Inactive points go to the trailing key
// nbins * cells_per_bin. Active points also count in their cell's class
// histogram, eight 8-bit counts in one 64-bit word, and keep their class and
// their arrival rank within the class (crank = class << 8 | rank, the rank
// saturated at 255).
template <int DIM, typename PT>
__global__ void k_sort_count(const BatchHdr* hdr, const BodyCtx<PT>* bodies, const int64_t* point_end, int32_t* key,
                             int32_t* rank, int32_t* cell_count, unsigned long long* cell_hist, int16_t* crank) {
  const int64_t total = hdr->points;
  const int nb = hdr->nbodies;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += stride) {
    const BodyCtx<PT>& B = bodies[find_range(point_end, nb, q)];
    const int64_t p = q - B.point_off;
    int k;
    if (B.P.active[p] == 0) {
      k = B.bg.nbins * B.bg.cells_per_bin;
    } else {
      double xp[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int d = 0; d < DIM; d++) xp[d] = two_word(B.P.x[d], B.P.xl[d], p);   // the mixed form: hi + lo
      int c[3] = {0, 0, 0};
      const int cls = point_cell<DIM>(B.g, xp, 0.5 * (double)B.P.ext[p], c);
      int b, l;
      bin_of<DIM>(B.bg, c, &b, &l);
      k = b * B.bg.cells_per_bin + l;
      const unsigned long long old = atomicAdd(cell_hist + B.cell_off + k, 1ull << (8 * cls));
      const int rc = (int)((old >> (8 * cls)) & 0xffull);
      crank[q] = (int16_t)((cls << 8) | rc);
    }
    key[q] = k;
    rank[q] = atomicAdd(cell_count + B.cell_off + k, 1);
  }
}

// Pass 2: per-bin point counts (one thread per bin entry, summing its
// cells); entry nbins of a body counts its inactive points.
template <typename PT>
__global__ void k_bin_totals(const BatchHdr* hdr, const BodyCtx<PT>* bodies, const int64_t* bin_end,
                             const int32_t* cell_count, int32_t* bin_total) {
  const int64_t total = hdr->bins;
  const int nb = hdr->nbodies;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += stride) {
    const BodyCtx<PT>& B = bodies[find_range(bin_end, nb, i)];
    const int lb = (int)(i - B.bin_off);
    const int32_t* cc = cell_count + B.cell_off;
    int s = 0;
    if (lb < B.bg.nbins) {
      for (int l = 0; l < B.bg.cells_per_bin; l++) s += cc[lb * B.bg.cells_per_bin + l];
    } else {
      s = cc[B.bg.nbins * B.bg.cells_per_bin];
    }
    bin_total[i] = s;
  }
}

// Exclusive scan of n int32 values in place, one CTA of 1024 threads, in
// chunks (for short arrays: the block sums of k_scan_blocks).
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

// Multi-CTA exclusive scan of hdr->bins values: each CTA of 1024 threads
// scans its chunk in place and writes the chunk total; k_scan_small scans
// the totals; k_scan_add adds them back.
constexpr int kScanChunk = 1024;
// Smallest points-per-item any fused kernel uses (work item capacity).
constexpr int kMinItemCap = 128;

__device__ __forceinline__ int block_exclusive_scan_1024(int x, int* total) {
  __shared__ int32_t warp_sums[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
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
  *total = warp_sums[31];
  return (wid > 0 ? warp_sums[wid - 1] : 0) + incl - x;
}

__global__ void __launch_bounds__(kScanChunk) k_scan_blocks(const BatchHdr* hdr, int32_t* v, int32_t* chunk_sum) {
  const int64_t n = hdr->bins;
  const int64_t i = blockIdx.x * (int64_t)kScanChunk + threadIdx.x;
  const int x = i < n ? v[i] : 0;
  int tot = 0;
  const int ex = block_exclusive_scan_1024(x, &tot);
  if (i < n) v[i] = ex;
  if (threadIdx.x == 0) chunk_sum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanChunk) k_scan_add(const BatchHdr* hdr, int32_t* v, const int32_t* chunk_sum) {
  const int64_t n = hdr->bins;
  const int64_t i = blockIdx.x * (int64_t)kScanChunk + threadIdx.x;
  if (i < n) v[i] += chunk_sum[blockIdx.x];
}

// Pass 3: destination of each point inside its bin (rank-major order) and
// the permutation copy of every per-point array into the second buffer.
// The rank of a point within its cell is its class-order rank (points of
// lower classes first, then the class's arrival rank) when the cell's class
// histogram is exact, i.e. its counts sum to the cell's count (a class of
// 256 or more points in one cell would have carried into the next count);
// otherwise every point of that cell keeps its arrival rank. Either way the
// ranks of a cell are a permutation of 0 .. count-1.
template <int DIM, typename PT>
__global__ void k_sort_scatter(const BatchHdr* hdr, const BodyCtx<PT>* bodies, const int64_t* point_end,
                               const int32_t* key, const int32_t* rank, const int32_t* cell_count,
                               const unsigned long long* cell_hist, const int16_t* crank, const int32_t* bin_scan) {
  const int64_t total = hdr->points;
  const int nb = hdr->nbodies;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += stride) {
    const BodyCtx<PT>& B = bodies[find_range(point_end, nb, q)];
    const int64_t p = q - B.point_off;
    const int k = key[q];
    int r = rank[q];
    const int cpb = B.bg.cells_per_bin;
    const int b = k / cpb;
    const int32_t* bs = bin_scan + B.bin_off;
    int64_t pos = bs[b] - bs[0];
    if (b < B.bg.nbins) {
      const int l = k - b * cpb;
      const int32_t* cc = cell_count + B.cell_off + (int64_t)b * cpb;
      const unsigned long long h = cell_hist[B.cell_off + k];
      const int cr = crank[q];
      const int cls = cr >> 8;
      int sum = 0, lower = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int f = (int)((h >> (8 * j)) & 0xffull);
        sum += f;
        lower += j < cls ? f : 0;
      }
      if (sum == cc[l]) r = lower + (cr & 0xff);
      int below = 0, same_level = 0;
      for (int c = 0; c < cpb; c++) {
        const int cnt = cc[c];
        below += cnt < r ? cnt : r;
        same_level += (c < l && cnt > r) ? 1 : 0;
      }
      pos += below + same_level;
    } else {
      pos += r;
    }
    const PointsT<PT>& S = B.P;
    const PointsT<PT>& D = B.Palt;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      D.x[d][pos] = S.x[d][p];
      D.v[d][pos] = S.v[d][p];
      D.u[d][pos] = S.u[d][p];
    }
#pragma unroll
    for (int c = 0; c < 6; c++) D.s[c][pos] = S.s[c][p];
    D.vol[pos] = S.vol[p];
    D.m[pos] = S.m[p];
    D.ext[pos] = S.ext[p];
    D.active[pos] = S.active[p];
    D.pid[pos] = S.pid[p];
    if (S.L != nullptr)
      for (int a = 0; a < 9; a++) D.L[9 * pos + a] = S.L[9 * p + a];
#pragma unroll
    for (int a = 0; a < 9; a++)
      if (S.ms[a] != nullptr) D.ms[a][pos] = S.ms[a][p];
    if (S.ml != nullptr) {
#pragma unroll
      for (int d = 0; d < 3; d++) {
        D.xl[d][pos] = S.xl[d][p];
        D.vl[d][pos] = S.vl[d][p];
      }
      D.ml[pos] = S.ml[p];
    }
  }
}

// Swaps the two point buffers of every body after the scatter.
template <typename PT>
__global__ void k_sort_flip(const BatchHdr* hdr, BodyCtx<PT>* bodies) {
  const int nb = hdr->nbodies;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const PointsT<PT> t = bodies[b].P;
    bodies[b].P = bodies[b].Palt;
    bodies[b].Palt = t;
  }
}

// Bounds of the contributions of each body's points to one node, for the
// deterministic form's two-level split (make_split): bounds[4 b + k] (the
// bits of a non-negative double, so that an integer maximum orders them,
// and a maximum is the same whatever the order) for k = 0 mass (S m <= m),
// 1 momentum (m max_d |v_d|), 2 internal force (V 3 max|sigma| max|grad S|),
// 3 contact normal (m max|grad S|), with |grad S| <= max(2 / extent, 1 / h):
// 2 / extent for the corner-sampled map (sG times at most 2 x 2 x 2), 1 / h
// point-sampled.
template <int DIM>
__global__ void k_det_bounds(const BatchHdr* hdr, const BodyCtx<double>* bodies, const int64_t* point_end,
                             unsigned long long* bounds) {
  const int64_t total = hdr->points;
  const int nb = hdr->nbodies;
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  // a warp takes 32 consecutive points (mostly of one body) per round, so
  // that one atomic per field and warp carries the warp's maximum
  for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < total;
       base += warps * 32) {
    const int64_t q = base + lane;
    int b = -1;
    double c4[4] = {0.0, 0.0, 0.0, 0.0};
    if (q < total) {
      b = find_range(point_end, nb, q);
      const BodyCtx<double>& B = bodies[b];
      const int64_t p = q - B.point_off;
      if (B.P.active[p] != 0) {
        double hmin = B.g.h[0];
#pragma unroll
        for (int d = 1; d < DIM; d++) hmin = fmin(hmin, B.g.h[d]);
        const double gmax = fmax(2.0 / B.P.ext[p], 1.0 / hmin);
        const double m = B.P.m[p];
        double vmax = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) vmax = fmax(vmax, fabs(B.P.v[d][p]));
        double smax = 0.0;
#pragma unroll
        for (int c = 0; c < 6; c++) smax = fmax(smax, fabs(B.P.s[c][p]));
        c4[0] = m;
        c4[1] = m * vmax;
        c4[2] = B.P.vol[p] * 3.0 * smax * gmax;
        c4[3] = m * gmax;
      }
    }
    const int b0 = __shfl_sync(0xffffffffu, b, 0);
    const bool same = b == b0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      // non-negative doubles order like their bit patterns
      unsigned long long v = same ? (unsigned long long)__double_as_longlong(c4[k]) : 0ull;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
      }
      if (lane == 0 && b0 >= 0) atomicMax(bounds + 4 * b0 + k, v);
      if (!same && b >= 0) atomicMax(bounds + 4 * b + k, (unsigned long long)__double_as_longlong(c4[k]));
    }
  }
}

// Clears the prime flags of every body after the priming scatter.
template <typename PT>
__global__ void k_clear_prime(const BatchHdr* hdr, BodyCtx<PT>* bodies) {
  for (int b = threadIdx.x; b < hdr->nbodies; b += blockDim.x) bodies[b].prime = 0;
}

// Work list: every non-empty bin of every body split into items of at most
// `cap` points: bin and [start, end) of the item's points (local to the
// body). Each body's items fill its own range starting at item_off[body]
// (room for nbins + n / cap + 1 items), so that a launch over one body
// reads a contiguous range and CTAs share its items evenly.
template <typename PT>
__global__ void k_bin_work(const BatchHdr* hdr, const BodyCtx<PT>* bodies, const int64_t* bin_end,
                           const int32_t* bin_scan, const int32_t* item_off, int cap, int32_t* work_bin,
                           int32_t* work_start, int32_t* work_end, int32_t* nwork_body) {
  const int64_t total = hdr->bins;
  const int nb = hdr->nbodies;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += stride) {
    const int bi = find_range(bin_end, nb, i);
    const BodyCtx<PT>& B = bodies[bi];
    const int lb = (int)(i - B.bin_off);
    if (lb >= B.bg.nbins) continue;
    const int32_t base = bin_scan[B.bin_off];
    const int s = bin_scan[i] - base, e = bin_scan[i + 1] - base;
    if (e <= s) continue;
    // split evenly: a bin of 1.2 cap points becomes two items of 0.6 cap
    const int items = (e - s + cap - 1) / cap;
    const int first = item_off[bi] + atomicAdd(nwork_body + bi, items);
    const int cnt = e - s;
    for (int k = 0; k < items; k++) {
      work_bin[first + k] = lb;
      work_start[first + k] = s + (int)((int64_t)cnt * k / items);
      work_end[first + k] = s + (int)((int64_t)cnt * (k + 1) / items);
    }
  }
}

// Inclusive prefix of the per-body item counts (work_end_body[b]) and the
// total (one CTA; bodies are at most a few thousand).
__global__ void k_work_prefix(const BatchHdr* hdr, const int32_t* nwork_body, int32_t* work_end_body,
                              int32_t* nwork) {
  __shared__ int32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int nb = hdr->nbodies;
  for (int base = 0; base < nb; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int x = i < nb ? nwork_body[i] : 0;
    int tot = 0;
    const int ex = block_exclusive_scan_1024(x, &tot);
    if (i < nb) work_end_body[i] = carry + ex + x;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *nwork = carry;
}

// Flat work list for launches over every body: flat index w -> (body, item),
// body-major, so that consecutive CTAs take consecutive items.
__global__ void k_work_flat(const BatchHdr* hdr, const int32_t* item_off, const int32_t* nwork_body,
                            const int32_t* work_end_body, const int32_t* nwork, int32_t* flat_body,
                            int32_t* flat_item) {
  const int total = *nwork;
  const int nb = hdr->nbodies;
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < total; w += gridDim.x * blockDim.x) {
    const int b = find_range(work_end_body, nb, w);
    flat_body[w] = b;
    flat_item[w] = item_off[b] + (w - (work_end_body[b] - nwork_body[b]));
  }
}

}  // namespace mpmb200
