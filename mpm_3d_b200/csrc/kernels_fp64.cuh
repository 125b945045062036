// Kernels of the explicit step around the fused gather/scatter kernel (all
// nodal work is FP64 in every form): active-block compaction, grid update
// (contact, boundary, moveGrid), the Jaumann stress update and the exact
// triplet export.
#pragma once

#include "exact_map.cuh"
#include "geom.cuh"
#include "state.cuh"

namespace mpmb200 {

__device__ __forceinline__ double sym_at(const double* s6, int a, int b) {
  // xx yy zz xy yz xz
  if (a == b) return s6[a];
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  if (lo == 0 && hi == 1) return s6[3];
  if (lo == 1 && hi == 2) return s6[4];
  return s6[5];
}

// Marks the node blocks covered by a point's window.
template <int DIM, typename R>
__device__ __forceinline__ void mark_blocks(const Geom& g, const PointMapT<R>& pm, uint32_t* flags) {
  const int i0 = pm.ax[0].base >> g.bsh[0], i1 = (pm.ax[0].base + pm.ax[0].span - 1) >> g.bsh[0];
  const int j0 = pm.ax[1].base >> g.bsh[1], j1 = (pm.ax[1].base + pm.ax[1].span - 1) >> g.bsh[1];
  int k0 = 0, k1 = 0;
  if (DIM == 3) {
    k0 = pm.ax[2].base >> g.bsh[2];
    k1 = (pm.ax[2].base + pm.ax[2].span - 1) >> g.bsh[2];
  }
  for (int k = k0; k <= k1; k++)
    for (int j = j0; j <= j1; j++)
      for (int i = i0; i <= i1; i++) flags[i + (int64_t)g.nb[0] * (j + (int64_t)g.nb[1] * k)] = 1u;
}

// Sets n int32 values to v.
__global__ void k_fill_i32(int32_t* p, int64_t n, int32_t v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

// Compacts the flagged node blocks of the batch's block space into `list`,
// clears the flags and keeps the per-block activity of this step in
// `was_active`.
__global__ void k_compact(const BatchHdr* hdr, uint32_t* flags, int64_t* list, unsigned long long* count,
                          uint8_t* was_active, unsigned long long* active_nodes) {
  const int64_t nblocks = hdr->blocks;
  if (blockIdx.x == 0 && threadIdx.x == 0) *active_nodes = 0;   // counted by this step's grid update
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nblocks; base += stride) {
    const int64_t blk = base + threadIdx.x;
    const bool on = blk < nblocks && flags[blk] != 0u;
    if (blk < nblocks) {
      was_active[blk] = on ? 1 : 0;
      if (on) flags[blk] = 0u;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, on);
    if (mask == 0u) continue;
    unsigned long long first = 0;
    if (lane == 0) first = atomicAdd(count, (unsigned long long)__popc(mask));
    first = __shfl_sync(0xffffffffu, first, 0);
    if (on) list[first + __popc(mask & ((1u << lane) - 1u))] = blk;
  }
}

// Grid update over the active node blocks of every job in the batch:
// ContactHuang::generateRules normalisation and applyRules
// (contact_huang.cpp:80-197), CartesianBox (cartesian_box.cpp:73-85) and
// moveGrid (explicit_usl.cpp:233-264). One CTA of 64 threads per block, one
// thread per node; each node is owned by exactly one thread.
template <int DIM>
__global__ void __launch_bounds__(64) k_grid(const InstDev* insts, const GridBody* bodies, const int32_t* blk_inst,
                                             const int64_t* list, const unsigned long long* count,
                                             unsigned long long* active_nodes) {
  const int64_t cnt = (int64_t)*count;
  for (int64_t e = blockIdx.x; e < cnt; e += gridDim.x) {
    const int64_t gblk = list[e];
    const InstDev& I = insts[blk_inst[gblk]];
    const Geom& g = I.g;
    const StepParams& sp = I.sp;
    const double dt = sp.dt;
    const GridBody* GB = bodies + I.body0;
    const int64_t blk = gblk - I.block_off;
    const int li = threadIdx.x;
    int i, j, k;
    slot_ijk(g, blk, li, i, j, k);
    const bool inside = i < g.nn[0] && j < g.nn[1] && k < g.nn[2];
    const int64_t s = blk * 64 + li;
    {
      // nodes with mass, per body (the grid term of the step's traffic)
      int cnt = 0;
      if (inside)
        for (int b = 0; b < I.nb; b++) cnt += GB[b].A.m[s] > 0.0 ? 1 : 0;
      cnt = __reduce_add_sync(0xffffffffu, cnt);
      if ((threadIdx.x & 31) == 0 && cnt > 0) atomicAdd(active_nodes, (unsigned long long)cnt);
    }
    if (!inside) continue;
    if (GB[0].Ar.m != nullptr) {
      // deterministic form: each nodal value arrived as two exactly summed
      // parts (level 0 in A, level 1 in Ar); one fixed rounding joins them
      for (int b = 0; b < I.nb; b++) {
        const NodesAcc& A = GB[b].A;
        const NodesAcc& R = GB[b].Ar;
        A.m[s] = A.m[s] + R.m[s];
        R.m[s] = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          A.mx[d][s] = A.mx[d][s] + R.mx[d][s];
          A.f[d][s] = A.f[d][s] + R.f[d][s];
          R.mx[d][s] = 0.0;
          R.f[d][s] = 0.0;
          if (A.nrm[0] != nullptr) {
            A.nrm[d][s] = A.nrm[d][s] + R.nrm[d][s];
            R.nrm[d][s] = 0.0;
          }
        }
      }
    }
    // the scatter leaves out the body force; S * (m b) summed over points is
    // the nodal mass times g (explicit_usl.cpp:150-154, b uniform)
    for (int b = 0; b < I.nb; b++) {
      const NodesAcc& A = GB[b].A;
      const double m = A.m[s];
#pragma unroll
      for (int d = 0; d < DIM; d++)
        if (sp.grav[d] != 0.0) A.f[d][s] = A.f[d][s] + m * sp.grav[d];
    }
    // CartesianFrictionalBox reads the nodal force before contact
    // (bcNodalForce: S (m b) - gradS (V T), cartesian_frictional_box.cpp:86-108)
    double fpre[kMaxBodies][3];
    for (int b = 0; b < I.nb; b++)
      if (GB[b].has_boundary == 3)
#pragma unroll
        for (int d = 0; d < DIM; d++) fpre[b][d] = GB[b].A.f[d][s];
    for (int c = 0; c < I.nc; c++) {
      const NodesAcc& A1 = GB[I.cb1[c]].A;
      const NodesAcc& A2 = GB[I.cb2[c]].A;
      double n[3] = {0.0, 0.0, 0.0};
      double nn = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        n[d] = A1.nrm[d][s];
        nn += n[d] * n[d];
      }
      const double m1 = A1.m[s], m2 = A2.m[s];
      if (!I.reflected[c]) {
        const double inv_norm = 1.0 / sqrt(nn);
#pragma unroll
        for (int d = 0; d < DIM; d++) n[d] *= inv_norm;
      } else if (m1 > 0) {
        // ContactHuang_ReflectedBoundary (contact_huang_reflected_boundary.cpp:
        // 90-114): the components normal to a wall of the box are dropped
        // before the normalisation, at nodes where body 1 has mass
        nn = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const int cd = d == 0 ? i : (d == 1 ? j : k);
          if (cd == 0 || cd == g.N[d]) n[d] = 0.0;
          nn += n[d] * n[d];
        }
        const double inv_norm = 1.0 / sqrt(nn);
#pragma unroll
        for (int d = 0; d < DIM; d++) n[d] *= inv_norm;
      }
      double fc[3] = {0.0, 0.0, 0.0};
      if (m1 > 0 && m2 > 0) {
        double mv1[3], mv2[3], vcm[3];
        double f1[3], f2[3];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          f1[d] = A1.f[d][s];
          f2[d] = A2.f[d][s];
          if (sp.contact_spec == 1) {
            mv1[d] = A1.mx[d][s] + dt * f1[d];
            mv2[d] = A2.mx[d][s] + dt * f2[d];
          } else {
            mv1[d] = A1.mx[d][s];
            mv2[d] = A2.mx[d][s];
          }
        }
        const double inv_m12 = 1.0 / (m1 + m2);
        const double inv_m1 = 1.0 / m1;
        double test = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          vcm[d] = (mv1[d] + mv2[d]) * inv_m12;
          test += (mv1[d] * inv_m1 - vcm[d]) * n[d];
        }
        if (test > 0) {
          double vcm_n = 0.0, mv1_n = 0.0;
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            vcm_n += vcm[d] * n[d];
            mv1_n += mv1[d] * n[d];
          }
          const double fn = m1 / dt * (vcm_n - mv1_n / m1);
          const double m1dt = m1 / dt;
          double s1[3], ss = 0.0;
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            s1[d] = m1dt * (vcm[d] - mv1[d] * inv_m1) - fn * n[d];
            ss += s1[d] * s1[d];
          }
          const double ft = sqrt(ss);
          if (ft != 0) {
            const double inv = 1.0 / ft;
#pragma unroll
            for (int d = 0; d < DIM; d++) s1[d] *= inv;
          }
          const double a = (fn < 0.0) ? fn : 0.0;  // std::min(0.0, fn)
          const double mufn = I.mu[c] * fabs(fn);
          const double b = (fabs(ft) < mufn) ? fabs(ft) : mufn;  // std::min(mu|fn|, |ft|)
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            fc[d] = a * n[d] + b * s1[d];
            A1.f[d][s] = f1[d] + fc[d];
            A2.f[d][s] = f2[d] - fc[d];
          }
        }
      }
      if (I.normal_out[c] != nullptr) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
          I.normal_out[c][3 * s + d] = (d < DIM) ? n[d] : 0.0;
          I.force_out[c][3 * s + d] = fc[d];
        }
      }
    }
    const bool on_face = (i == 0 || i == g.N[0] || j == 0 || j == g.N[1] || (DIM == 3 && (k == 0 || k == g.N[2])));
    for (int b = 0; b < I.nb; b++) {
      const NodesAcc& A = GB[b].A;
      const NodesVel& V = GB[b].V;
      const double m = A.m[s];
      double mx[3], f[3];
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        mx[d] = A.mx[d][s];
        f[d] = A.f[d][s];
      }
      const int kind = GB[b].has_boundary;
      if (kind == 1 && on_face) {
        // CartesianBox (cartesian_box.cpp:73-85): every component of a node
        // on any wall
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          mx[d] = 0.0;
          f[d] = 0.0;
        }
      } else if (kind == 2 && on_face) {
        // CartesianSmoothBox (cartesian_smooth_box.cpp:69-83): the
        // wall-normal components only
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const int c = d == 0 ? i : (d == 1 ? j : k);
          if (c == 0 || c == g.N[d]) {
            mx[d] = 0.0;
            f[d] = 0.0;
          }
        }
      } else if (kind == 3 && on_face) {
        // CartesianFrictionalBox (cartesian_frictional_box.cpp:94-143): the
        // closing momentum of each wall component gives the normal force,
        // the component is zeroed, and friction of at most mu_f times the
        // normal force opposes the remaining motion (interior nodes: no
        // normal force, no change)
        double dmom[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const int c = d == 0 ? i : (d == 1 ? j : k);
          const double closing = mx[d] + dt * fpre[b][d];
          if (c == 0) {
            dmom[d] = -((closing < 0.0) ? closing : 0.0);   // -std::min(0.0, .)
            mx[d] = 0.0;
            f[d] = 0.0;
          } else if (c == g.N[d]) {
            dmom[d] = -((0.0 < closing) ? closing : 0.0);   // -std::max(0.0, .)
            mx[d] = 0.0;
            f[d] = 0.0;
          }
        }
        double nn = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) nn += dmom[d] * dmom[d];
        const double f_normal = sqrt(nn) / dt;
        double mm = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          dmom[d] = mx[d] + dt * f[d];
          mm += dmom[d] * dmom[d];
        }
        const double nrm = sqrt(mm);
        if (nrm > 0) {
          const double a = nrm / dt, bnd = f_normal * GB[b].mu_f;
          const double cf = (bnd < a) ? bnd : a;   // std::min(|dm| / dt, f_normal mu_f)
          // vector / scalar multiplies by the reciprocal (mpm_vector.hpp:609-615)
          const double inv = 1.0 / nrm;
#pragma unroll
          for (int d = 0; d < DIM; d++) f[d] = f[d] - (cf * dmom[d]) * inv;
        }
      }
      double inv = 0.0;
      if (m > 0) inv = 1.0 / m;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        mx[d] = mx[d] + dt * f[d];
        V.vt[d][s] = (m > 0) ? mx[d] * inv : 0.0;
        V.dv[d][s] = (m > 0) ? (dt * f[d]) * inv : 0.0;
      }
      const NodesAcc& Sn = GB[b].snap;
      if (Sn.m != nullptr) {
        Sn.m[s] = m;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          Sn.mx[d][s] = mx[d];
          Sn.f[d][s] = f[d];
        }
      }
      // the next step's scatter accumulates into zeroed arrays
      A.m[s] = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        A.mx[d][s] = 0.0;
        A.f[d][s] = 0.0;
        if (A.nrm[0] != nullptr) A.nrm[d][s] = 0.0;
      }
    }
  }
}

// Jaumann update of IsotropicLinearElasticity (isolin.cpp:62-74) on the 6
// stored components. For symmetric T and W = -W^T, (T W)_ab = -(W T)_ba, so
// W T - T W = (W T)_ab + (W T)_ba.
template <int DIM, typename R>
__device__ __forceinline__ void jaumann_update(const R L[3][3], R* s6, R G, R lambda, R dt) {
  R D[3][3], W[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      D[a][b] = R(0.5) * (L[a][b] + L[b][a]);
      W[a][b] = R(0.5) * (L[a][b] - L[b][a]);
    }
  const R trD = D[0][0] + D[1][1] + D[2][2];
  const R T[3][3] = {{s6[0], s6[3], s6[5]}, {s6[3], s6[1], s6[4]}, {s6[5], s6[4], s6[2]}};
  R WT[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) WT[a][b] = W[a][0] * T[0][b] + W[a][1] * T[1][b] + W[a][2] * T[2][b];
  const R twoG = R(2.0) * G;
  const R ltr = lambda * trD;
  const int ia[6] = {0, 1, 2, 0, 1, 0};
  const int ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int c = 0; c < 6; c++) {
    const int a = ia[c], b = ib[c];
    const R rate = ((twoG * D[a][b] + (a == b ? ltr : R(0.0))) + WT[a][b]) + WT[b][a];
    s6[c] = s6[c] + dt * rate;
  }
}

// The Jaumann update of one point in its form. The mixed form keeps its
// stress and velocity gradient in FP32 but runs the update in FP64 and
// rounds the result once (measured on the block-drop ensemble: the FP32
// update's rounding, amplified by a soft block's dynamics, reached 1.9e-4
// of the stress after 500 steps; in FP64 arithmetic 8.3e-5).
template <int DIM, typename R>
__device__ __forceinline__ void jaumann_point(const R L[3][3], R* s6, const MaterialParams& mp, double dt) {
  if constexpr (sizeof(R) == 4) {
    double Ld[3][3], sd[6];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) Ld[a][b] = (double)L[a][b];
#pragma unroll
    for (int k = 0; k < 6; k++) sd[k] = (double)s6[k];
    jaumann_update<DIM, double>(Ld, sd, mp.G, mp.lambda, dt);
#pragma unroll
    for (int k = 0; k < 6; k++) s6[k] = (R)sd[k];
  } else {
    jaumann_update<DIM, R>(L, s6, (R)mp.G, (R)mp.lambda, (R)dt);
  }
}

// CompressibleNeohookeanElasticity::calculateStress
// (compressible_neohookean_elasticity.cpp:44-62) for one point. The
// reference advances F += (L F) dt and sets T = G/J (B - I) + lambda ln(J)/J I
// with B = F F^T, J = sqrt(det B), lambda = K - 2G/3. Here the deformation
// gradient is kept as H = F - I (global memory, row-major components
// H[0..8]), so the same quantities come without the cancellation of B - I
// and ln J near the identity (which costs FP32 most of its digits at small
// strains): H += (L + L H) dt, B - I = H + H^T + H H^T,
// J - 1 = det(I + H) - 1 = tr H + ((tr H)^2 - tr(H H))/2 + det H, and
// ln J = log1p(J - 1). Returns the 6 stored stress components.
template <typename R, typename PT>
__device__ __forceinline__ void neohookean_update(PT* const* Hp, int64_t p, const R L[3][3], R* s6, R G, R lambda,
                                                  R dt) {
  R H[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) H[a][b] = (R)Hp[3 * a + b][p];
  R LH[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) LH[a][b] = L[a][0] * H[0][b] + L[a][1] * H[1][b] + L[a][2] * H[2][b];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      H[a][b] = H[a][b] + (L[a][b] + LH[a][b]) * dt;
      Hp[3 * a + b][p] = (PT)H[a][b];
    }
  const R trH = H[0][0] + H[1][1] + H[2][2];
  R trHH = R(0);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) trHH += H[a][b] * H[b][a];
  const R detH = H[0][0] * (H[1][1] * H[2][2] - H[2][1] * H[1][2]) - H[0][1] * (H[1][0] * H[2][2] - H[2][0] * H[1][2]) +
                 H[0][2] * (H[1][0] * H[2][1] - H[2][0] * H[1][1]);
  const R Jm1 = trH + R(0.5) * (trH * trH - trHH) + detH;
  const R J = R(1) + Jm1;
  const R s1 = G / J;
  const R s2 = lambda * log1p(Jm1) / J;
  const int ia[6] = {0, 1, 2, 0, 1, 0};
  const int ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int c = 0; c < 6; c++) {
    const int a = ia[c], b = ib[c];
    const R bmi = H[a][b] + H[b][a] + (H[a][0] * H[b][0] + H[a][1] * H[b][1] + H[a][2] * H[b][2]);
    s6[c] = s1 * bmi + (a == b ? s2 : R(0));
  }
}

// Sand_SachithLocal::calculateStress (sand_sachithlocal.cpp:140-215) for one
// point, cohesion 0, on the 6 stored components. The trial stress s_tr is
// the Jaumann update above; p_tr = -tr(s_tr)/3 (or K (rho/rho_c - 1) with
// USE_DENSITY_FOR_PRESSURE), t0 = s_tr + p_tr I, tau_tr = |t0|/sqrt(2) with
// |t0|^2 summed in the reference's row-major order. Below the critical
// density, or at p_tr <= 0, the stress is zero and the shear rate is
// tau_tr/(G dt). Inside the cone tau_tr <= mu_s p_tr the trial stress stays.
// Otherwise tau is the smaller root of tau^2 - (S2 + tau_tr + alpha) tau +
// S2 tau_tr + S0 alpha (S0 = mu_s p_tr, S2 = mu_2 p_tr, alpha = G I_0 dt
// sqrt(p_tr/grains_rho)/grains_d), taken as in negative_root (44-53), and
// T = (tau/tau_tr) t0 - p_tr I. A NaN p_tr leaves T as it was. gammap
// (st[0]) advances by the shear rate times dt and gammap_dot (st[1]) takes
// the rate. rho = m/V with V already updated this step (updateDensity runs
// before the stress, explicit_usl.cpp:332-352).
template <int DIM, typename R, typename PT>
__device__ __forceinline__ void sand_update(PT* const* st, int64_t p, const R L[3][3], R* s6, R m, R vol,
                                            const MaterialParams& mp, R dt) {
  R t0[6];
#pragma unroll
  for (int k = 0; k < 6; k++) t0[k] = s6[k];
  jaumann_update<DIM, R>(L, t0, (R)mp.G, (R)mp.lambda, dt);
  R p_tr = -((t0[0] + t0[1]) + t0[2]) / R(3.0);
#pragma unroll
  for (int k = 0; k < 3; k++) t0[k] = t0[k] + p_tr;
  // xx xy xz yx yy yz zx zy zz
  R nn = t0[0] * t0[0];
  nn += t0[3] * t0[3];
  nn += t0[5] * t0[5];
  nn += t0[3] * t0[3];
  nn += t0[1] * t0[1];
  nn += t0[4] * t0[4];
  nn += t0[5] * t0[5];
  nn += t0[4] * t0[4];
  nn += t0[2] * t0[2];
  const R tau_tr = sqrt(nn) / sqrt(R(2.0));
  const R G = (R)mp.G;
  const R rho = m / vol;
  const R rho_c = (R)mp.rho_critical;
  if (mp.use_density) p_tr = (R)mp.K * ((rho - rho_c) / rho_c);
  R nup;
  if (rho < rho_c || p_tr <= R(0)) {
    nup = tau_tr / (G * dt);
#pragma unroll
    for (int k = 0; k < 6; k++) s6[k] = R(0);
  } else if (p_tr > R(0)) {
    const R S0 = (R)mp.mu_s * p_tr;
    R tau = tau_tr, scale = R(1);
    if (!(tau_tr <= S0)) {
      const R S2 = (R)mp.mu_2 * p_tr;
      const R alpha = G * (R)mp.i_0 * dt * sqrt(p_tr / (R)mp.grains_rho) / (R)mp.grains_d;
      const R b = -(S2 + tau_tr + alpha);
      const R c = S2 * tau_tr + S0 * alpha;
      const R disc = sqrt(b * b - R(4) * c);
      tau = b > R(0) ? (-b - disc) / R(2) : (R(2) * c) / (-b + disc);
      scale = tau / tau_tr;
    }
    nup = ((tau_tr - tau) / G) / dt;
#pragma unroll
    for (int k = 0; k < 6; k++) s6[k] = scale * t0[k] - (k < 3 ? p_tr : R(0));
  } else {
    nup = R(0);
  }
  st[0][p] = (PT)((R)st[0][p] + nup * dt);
  st[1][p] = (PT)nup;
}

// Order-independent nodal sums of the deterministic form (pre-rounded
// two-level summation after Demmel and Nguyen, "Fast reproducible
// floating-point summation", ARITH 2013). With M bounding every partial sum
// of |contributions| to a node (n contributions of at most maxc each), a
// contribution x splits exactly into q0 + q1 + e: q0 is x rounded to a
// multiple of 2^(E0-52) with 2^E0 > 2M, q1 the remainder rounded to a
// multiple of 2^(E1-52) with E1 = E0 - 52 + L, 2^L > 2n, and |e| <
// 2^(E1-53). Sums of q0 (of q1) stay below 2^E0 (2^E1) in any order, so
// every addition is exact and the two sums are the same bits whatever the
// order; the nodal value is level0 + level1 rounded once.
struct Split2 {
  double s0;  // 1.5 * 2^E0
  double s1;  // 1.5 * 2^E1
};

__device__ __forceinline__ Split2 make_split(double maxc, int64_t n) {
  Split2 k{0.0, 0.0};
  if (!(maxc > 0.0) || n < 1) return k;  // all contributions are zero
  const int L = ilogb((double)n) + 2;
  const int E0 = ilogb(maxc) + L + 1;
  const int E1 = E0 - 52 + L;
  k.s0 = ldexp(1.5, E0);
  k.s1 = ldexp(1.5, E1);
  return k;
}

__device__ __forceinline__ void presplit(double x, const Split2& k, double& q0, double& q1) {
  q0 = __dsub_rn(__dadd_rn(k.s0, x), k.s0);
  const double r = __dsub_rn(x, q0);
  q1 = __dsub_rn(__dadd_rn(k.s1, r), k.s1);
}

// Exact triplet export (mpmgpu_dump_map).
template <int DIM>
__global__ void k_export_map(Geom g, int cpdi, PointsDev P, int32_t* node_out, double* s_out, double* g_out) {
  constexpr int cp = 1 << DIM;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P.n; p += stride) {
    // slots in original point order (P.pid), so the host reads triplets in
    // the reference's point-major order whatever the storage order
    const int64_t slot = (int64_t)P.pid[p] * cp * cp;
    if (!P.active[p]) {
      for (int k = 0; k < cp * cp; k++) node_out[slot + k] = -1;
      continue;
    }
    double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < DIM; d++) x[d] = P.x[d][p];
    if (export_point<DIM>(g, cpdi, x, P.ext[p], node_out, s_out, g_out, slot) < 0) P.active[p] = 0;
  }
}

}  // namespace mpmb200
