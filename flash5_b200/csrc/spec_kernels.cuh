// spec_kernels.cuh -- species and mass scalars of one unsplit hydro step,
// FLASH5's hy_fullSpecMsFluxHandling path (the default, unsplit/Config:
// 140-143).  They are passive: they read the hydro's face mass fluxes, the
// old cell velocities and flattening, the new density and, in 3D with the
// full CTU, where the hydro fell back to first order, and feed nothing back.
// So they run after the hydro direction kernels, in FP64 for every
// precision variant, compiled without FMA contraction in the expression
// order of the CPU oracle (bit-identical to it on the FP64 hydro path).
//
//   k_spec_sig   SpcSig of every box cell and direction: the entropy-wave
//                speed (the cell's normal velocity) times the upwind
//                difference (hy_DataReconstructNormalDir_PPM.F90:360-369,
//                hy_upwindTransverseFlux.F90:197-205 with speciesScalar)
//   k_spec_dir   per direction: PPM face values of the line cells
//                (hy_DataReconstructNormalDir_PPM.F90:289-301, 584-628),
//                transverse corrections (hy_dataReconstOneStep.F90:996-1014),
//                3D CTU cross terms or the first-order fallback
//                (hy_getRiemannState.F90:1053-1090 and y/z analogues,
//                fallbackToFirstOrder :1456-1475), upwind fluxes
//                F_dens * X (hy_getFaceFlux.F90:453-467) and the flux
//                divergence; the last direction updates
//                X = (X rho_old + dt sum (F_L - F_R)/dx) / rho_new
//                (updateSpeciesMassScalar, hy_unsplitUpdate.F90:1300-1318)
//                and renormalises the species (:850-859).
#pragma once
#include "hy_kernels.cuh"

namespace fhy {

// mass fraction q of the cell providing local cell (li, lj, lk) of block b
// (guard cells as Grid_fillGuardCells: periodic, zero gradient, mirrored
// without sign change)
template <int NDIM, int NX, int NY, int NZ>
__device__ __forceinline__ double load_spec(const DevParams &P, int b, int3 bc, int li, int lj, int lk, int q,
                                            size_t ncells) {
  if (P.sp_lh && !is_inside<NDIM, NX, NY, NZ>(li, lj, lk)) {   // AMR: the leaf's species guard cells
    using H = Halo<NDIM, NX, NY, NZ>;
    return P.sp_lh[((size_t)P.slot[b] * P.nsp + q) * H::n + H::idx(li, lj, lk)];
  }
  bool inside; int fx, fy, fz;
  const size_t o = cell_src<NDIM, NX, NY, NZ>(P, b, bc, li, lj, lk, inside, fx, fy, fz);
  return __ldg(P.sp_in + (size_t)q * ncells + o);
}

// velocity component d (0-based) of a cell, mirrored in reflecting guard cells
template <int NDIM, int NX, int NY, int NZ>
__device__ __forceinline__ double load_vel(const DevParams &P, int b, int3 bc, int li, int lj, int lk, int d) {
  if (P.lh && !is_inside<NDIM, NX, NY, NZ>(li, lj, lk)) {       // AMR: the leaf guard buffer (mirrored)
    using H = Halo<NDIM, NX, NY, NZ>;
    return P.lh[(size_t)P.slot[b] * 5 * H::n + (1 + d) * H::n + H::idx(li, lj, lk)];
  }
  bool inside; int f[3];
  const size_t o = cell_src<NDIM, NX, NY, NZ>(P, b, bc, li, lj, lk, inside, f[0], f[1], f[2]);
  const double v = __ldg(P.s_in[1 + d] + o);
  return f[d] ? -v : v;
}

// min / max as the CPU oracle takes them (a < b ? a : b), so that signed
// zeros come out the same
__device__ __forceinline__ double minmod_s(double a, double b) {     // hy_slopeLimiters.F90:56-60
  return .5 * (copysign(1., a) + copysign(1., b)) * rmin(fabs(a), fabs(b));
}

// Cells (N+2s)^d around a block's interior (s layers), staged in shared
// memory so that every guard-mapped cell is loaded once.
template <int NDIM, int NX, int NY, int NZ, int S>
struct Ext {
  static constexpr int ex = NX + 2 * S, ey = NDIM > 1 ? NY + 2 * S : 1, ez = NDIM > 2 ? NZ + 2 * S : 1;
  static constexpr int n = ex * ey * ez;
  __device__ static __forceinline__ int idx(int i, int j, int k) {
    return ((k + (NDIM > 2 ? S : 0)) * ey + (j + (NDIM > 1 ? S : 0))) * ex + (i + S);
  }
  __device__ static __forceinline__ void decode(int c, int &i, int &j, int &k) {
    i = c % ex - S;
    j = NDIM > 1 ? (c / ex) % ey - S : 0;
    k = NDIM > 2 ? c / (ex * ey) - S : 0;
  }
};

template <int NDIM, int NX, int NY, int NZ>
struct SigGeom {
  using B = Box<NDIM, NX, NY, NZ>;
  using E = Ext<NDIM, NX, NY, NZ, 2>;
  // velocities of the box cells, one species on the box plus one layer
  static constexpr size_t smem_bytes() { return ((size_t)3 * B::n + E::n) * sizeof(double); }
};

template <int NDIM, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256) k_spec_sig(const DevParams P, double *__restrict__ SSIG, size_t ncells) {
  using B = Box<NDIM, NX, NY, NZ>;
  using E = Ext<NDIM, NX, NY, NZ, 2>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sV = reinterpret_cast<double *>(smem_raw);     // [3][B::n]
  double *sX = sV + 3 * B::n;                            // [E::n]
  const int b = P.blk_list ? P.blk_list[blockIdx.x] : blockIdx.x;
  const int slot = P.slot ? P.slot[b] : (int)blockIdx.x;
  const int3 bc = blk_coords(P, b);
  for (int c = threadIdx.x; c < B::n; c += blockDim.x) {
    const int i = c % B::bx - 1, j = NDIM > 1 ? (c / B::bx) % B::by - 1 : 0;
    const int k = NDIM > 2 ? c / (B::bx * B::by) - 1 : 0;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) sV[d * B::n + c] = load_vel<NDIM, NX, NY, NZ>(P, b, bc, i, j, k, d);
  }
  for (int q = 0; q < P.nsp; ++q) {
    for (int c = threadIdx.x; c < E::n; c += blockDim.x) {
      int i, j, k;
      E::decode(c, i, j, k);
      sX[c] = load_spec<NDIM, NX, NY, NZ>(P, b, bc, i, j, k, q, ncells);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < B::n; c += blockDim.x) {
      const int i = c % B::bx - 1, j = NDIM > 1 ? (c / B::bx) % B::by - 1 : 0;
      const int k = NDIM > 2 ? c / (B::bx * B::by) - 1 : 0;
      const int e = E::idx(i, j, k);
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        const int st = d == 0 ? 1 : (d == 1 ? E::ex : E::ex * E::ey);
        const double lam = sV[d * B::n + c];
        const double sm = sX[e - st], s0 = sX[e], sp = sX[e + st];
        double g;
        if (lam > 0.) g = s0 - sm;
        else g = sp - s0;
        SSIG[(((size_t)slot * NDIM + d) * P.nsp + q) * B::n + c] = lam * g;
      }
    }
    __syncthreads();
  }
}

template <int NDIM, int NX, int NY, int NZ, int DIR>
struct SpecGeom {
  using L = DirGeom<NDIM, NX, NY, NZ, double, DIR>;
  // one species staged on the lines with 3 cells beyond the block along DIR
  static constexpr int sx = DIR == 1 ? NX + 6 : NX, sy = NDIM > 1 ? (DIR == 2 ? NY + 6 : NY) : 1,
                       sz = NDIM > 2 ? (DIR == 3 ? NZ + 6 : NZ) : 1;
  static constexpr int ns = sx * sy * sz;
  static constexpr int sstep = DIR == 1 ? 1 : (DIR == 2 ? sx : sx * sy);
  __device__ static __forceinline__ int sidx(int i, int j, int k) {
    return ((k + 3 * (DIR == 3)) * sy + (j + 3 * (DIR == 2))) * sx + (i + 3 * (DIR == 1));
  }
  // shared memory: per line cell the face values of one species (left,
  // right), the normal velocity, the flattening coefficient, the velocities
  // along the two CTU axes, the face flux and the fallback flag; the staged
  // species
  static constexpr size_t smem_bytes() { return (size_t)L::n * 7 * sizeof(double) + (size_t)ns * sizeof(double) + L::n; }
};

template <int NDIM, int NX, int NY, int NZ, int DIR, bool FIRST, bool LAST>
__global__ void __launch_bounds__(256) k_spec_dir(const DevParams P, const double *__restrict__ SSIG,
                                                  double *__restrict__ SACC, size_t ncells) {
  using L = DirGeom<NDIM, NX, NY, NZ, double, DIR>;
  using B = Box<NDIM, NX, NY, NZ>;
  constexpr int NCB = NX * NY * NZ;
  using SG = SpecGeom<NDIM, NX, NY, NZ, DIR>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sSl = reinterpret_cast<double *>(smem_raw);
  double *sSr = sSl + L::n;
  double *sU = sSr + L::n;            // normal velocity (lambda of the entropy wave)
  double *sFl = sU + L::n;            // flattening coefficient
  double *sA1 = sFl + L::n;           // velocities along the CTU axes A1, A2
  double *sA2 = sA1 + L::n;
  double *sFs = sA2 + L::n;           // species flux at the face left of each line cell
  double *sX = sFs + L::n;            // the staged species
  unsigned char *sFb = reinterpret_cast<unsigned char *>(sX + SG::ns);
  const int b = P.blk_list ? P.blk_list[blockIdx.x] : blockIdx.x;
  const int slot = P.slot ? P.slot[b] : (int)blockIdx.x;
  const int3 bc = blk_coords(P, b);
  const double dt = P.dt_dev ? *P.dt_dev : P.dt;
  double del[3];
  blk_deltas(P, b, del);                // the block's level
  const double delta = del[DIR - 1];
  const double hdtx = 0.5 * dt / del[0], hdty = 0.5 * dt / del[1], hdtz = 0.5 * dt / del[2];
  constexpr int A1 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1), S1 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2);
  constexpr int A2 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2), S2 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1);
  const bool ctu = NDIM == 3 && P.use_ctu;
  const size_t lb = sp_line_base<NDIM, NX, NY, NZ, DIR>(slot);
  const double *ssb = SSIG + (size_t)slot * NDIM * P.nsp * B::n;

  // ---- per line cell quantities shared by every species
  for (int t = threadIdx.x; t < L::n; t += blockDim.x) {
    int i, j, k;
    L::decode(t, i, j, k);
    sU[t] = load_vel<NDIM, NX, NY, NZ>(P, b, bc, i, j, k, DIR - 1);
    sFl[t] = P.use_flattening ? P.sp_flat[lb + t] : 0.;   // left by the hydro direction kernel
    if (ctu) {
      sA1[t] = load_vel<NDIM, NX, NY, NZ>(P, b, bc, i, j, k, A1 - 1);
      sA2[t] = load_vel<NDIM, NX, NY, NZ>(P, b, bc, i, j, k, A2 - 1);
      sFb[t] = P.sp_fb[lb + t];
    }
  }
  __syncthreads();

  const double dtn = dt / delta, hdtn = 0.5 * dtn;
  const double fac = dt * dt / (6. * (DIR == 1 ? del[1] : (DIR == 2 ? del[2] : del[0])) *
                                (DIR == 1 ? del[2] : (DIR == 2 ? del[0] : del[1])));
  for (int q = 0; q < P.nsp; ++q) {
    const double *sig = ssb + (size_t)q * B::n;           // + d * nsp * B::n for direction d
    const size_t dstr = (size_t)P.nsp * B::n;
    // ---- stage the species on the lines, 3 cells beyond the block along DIR
    for (int c = threadIdx.x; c < SG::ns; c += blockDim.x) {
      const int i = c % SG::sx - 3 * (DIR == 1), j = NDIM > 1 ? (c / SG::sx) % SG::sy - 3 * (DIR == 2) : 0;
      const int k = NDIM > 2 ? c / (SG::sx * SG::sy) - 3 * (DIR == 3) : 0;
      sX[c] = load_spec<NDIM, NX, NY, NZ>(P, b, bc, i, j, k, q, ncells);
    }
    __syncthreads();
    // ---- face values of the line cells
    for (int t = threadIdx.x; t < L::n; t += blockDim.x) {
      int i, j, k;
      L::decode(t, i, j, k);
      const int e = SG::sidx(i, j, k);
      double S[5];
#pragma unroll
      for (int s = -2; s <= 2; ++s) S[s + 2] = sX[e + s * SG::sstep];
      const double Smm = S[0], Sm = S[1], Sc = S[2], Sp = S[3], Spp = S[4];
      const double lam = sU[t];
      double dP = minmod_s(Sp - Sc, Spp - Sp);
      double d0 = minmod_s(Sc - Sm, Sp - Sc);
      double dN = minmod_s(Sm - Smm, Sc - Sm);
      double l = 0.5 * (Sc + Sm) - (d0 - dN) / 6.;
      double r = 0.5 * (Sc + Sp) - (dP - d0) / 6.;
      l = rmax(rmin(Sc, Sm), rmin(rmax(Sc, Sm), l));
      r = rmax(rmin(Sc, Sp), rmin(rmax(Sc, Sp), r));
      if ((r - Sc) * (Sc - l) <= 0.) { r = Sc; l = Sc; }
      if (6. * (r - l) * (Sc - 0.5 * (r + l)) > (r - l) * (r - l)) l = 3. * Sc - 2. * r;
      if (6. * (r - l) * (Sc - 0.5 * (r + l)) < -((r - l) * (r - l))) r = 3. * Sc - 2. * l;
      d0 = r - l;
      const double s6 = 6. * (Sc - 0.5 * (r + l));
      const double lm = rmin(lam, 0.), lp = rmax(lam, 0.);
      l = l - lm * hdtn * (d0 + (1. + lm * 4. / 3. * hdtn) * s6);
      r = r - lp * hdtn * (d0 - (1. - lp * 4. / 3. * hdtn) * s6);
      if (P.use_flattening) {
        const double f = sFl[t];
        l = f * Sc + (1.0 - f) * l;
        r = f * Sc + (1.0 - f) * r;
      }
      // transverse corrections with SpcSig of the other directions
      const int bi = B::idx(i, j, k);
      if (NDIM == 2) {
        if (DIR == 1) { const double g = sig[1 * dstr + bi]; l = l - hdty * g; r = r - hdty * g; }
        else          { const double g = sig[0 * dstr + bi]; l = l - hdtx * g; r = r - hdtx * g; }
      } else if (NDIM == 3) {
        const double gx = sig[0 * dstr + bi], gy = sig[1 * dstr + bi], gz = sig[2 * dstr + bi];
        if (DIR == 1)      { l = l - hdty * gy; r = r - hdty * gy; l = l - hdtz * gz; r = r - hdtz * gz; }
        else if (DIR == 2) { l = l - hdtx * gx; r = r - hdtx * gx; l = l - hdtz * gz; r = r - hdtz * gz; }
        else               { l = l - hdtx * gx - hdty * gy; r = r - hdtx * gx - hdty * gy; }
      }
      if (ctu) {
        if (sFb[t]) {
          l = Sc;
          r = Sc;
        } else {
          double T[2];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int ax = u ? A2 : A1, sd = u ? S2 : S1;
            const double lamA = u ? sA2[t] : sA1[t];
            const double *sg = sig + (size_t)(sd - 1) * dstr;
            const double gm = sg[B::idx(i - (ax == 1), j - (ax == 2), k - (ax == 3))];
            const double g0 = sg[bi];
            const double gp = sg[B::idx(i + (ax == 1), j + (ax == 2), k + (ax == 3))];
            const double g = lamA > 0. ? g0 - gm : gp - g0;
            T[u] = lamA * g;
          }
          r = r + (T[0] + T[1]) * fac;
          l = l + (T[0] + T[1]) * fac;
        }
      }
      sSl[t] = l;
      sSr[t] = r;
    }
    __syncthreads();
    // ---- upwind fluxes F_dens * X at the faces (the face left of line cell
    // t for along in [0, N]); on AMR hierarchies the fine/coarse faces
    // through the species flux register
    for (int t = threadIdx.x; t < L::n; t += blockDim.x) {
      int i, j, k;
      L::decode(t, i, j, k);
      if (L::along(i, j, k) < 0) continue;
      const double m = P.sp_mf[lb + t];
      if (m < 0.) sFs[t] = m * sSl[t];
      else sFs[t] = m * sSr[t - L::stride];
    }
    __syncthreads();
    if (P.sp_freg) {
      flux_register_v<NDIM, NX, NY, NZ, DIR>(P, b, bc, sFs, 0, [](int along, int t1, int t2) {
        const int i = DIR == 1 ? along : t1, j = DIR == 1 ? t1 : (DIR == 2 ? along : t2),
                  k = DIR == 3 ? along : (NDIM > 2 ? t2 : 0);
        return L::idx(i, j, k);
      }, P.sp_freg + (size_t)q * P.sp_freg_stride, 1);
      __syncthreads();
    }
    // ---- divergence
    for (int t = threadIdx.x; t < L::n; t += blockDim.x) {
      int i, j, k;
      L::decode(t, i, j, k);
      const int a = L::along(i, j, k);
      if (a < 0 || a >= L::nd) continue;
      const size_t off = (size_t)b * NCB + (size_t)((k * NY + j) * NX + i);
      const double FL = sFs[t], FR = sFs[t + L::stride];
      double acc = (FL - FR) / delta;
      if (!FIRST) acc = SACC[(size_t)q * ncells + off] + acc;
      if (!LAST) {
        SACC[(size_t)q * ncells + off] = acc;
      } else {
        const double X = P.sp_in[(size_t)q * ncells + off];
        P.sp_out[(size_t)q * ncells + off] = (X * P.s_in[0][off] + dt * acc) / P.s_out[0][off];
      }
    }
    __syncthreads();
  }
  // ---- species (not mass scalars) renormalised to a unit sum
  if (LAST && P.nspec > 0) {
    for (int c = threadIdx.x; c < NCB; c += blockDim.x) {
      const size_t off = (size_t)b * NCB + c;
      double sum = 0.;
      for (int q = 0; q < P.nspec; ++q) sum = sum + P.sp_out[(size_t)q * ncells + off];
      for (int q = 0; q < P.nspec; ++q) P.sp_out[(size_t)q * ncells + off] = P.sp_out[(size_t)q * ncells + off] / sum;
    }
  }
}

}  // namespace fhy
