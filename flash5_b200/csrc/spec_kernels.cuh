// spec_kernels.cuh -- species and mass scalars of one unsplit hydro step,
// FLASH5's hy_fullSpecMsFluxHandling path (the default, unsplit/Config:
// 140-143).  They are passive: they read the hydro's face mass fluxes, the
// old cell velocities and flattening, the new density and, in 3D with the
// full CTU, where the hydro fell back to first order, and feed nothing back.
// So they run after the hydro direction kernels, in FP64 for every
// precision variant, compiled without FMA contraction in the expression
// order of the CPU oracle (bit-identical to it on the FP64 hydro path).
//
//   k_spec_step  one CTA per block, all species and directions: PPM face
//                values of the line cells (hy_DataReconstructNormalDir_PPM.F90:
//                289-301, 584-628), transverse corrections with SpcSig, the
//                entropy-wave speed times the upwind difference
//                (hy_DataReconstructNormalDir_PPM.F90:360-369,
//                hy_upwindTransverseFlux.F90:197-205 with speciesScalar;
//                hy_dataReconstOneStep.F90:996-1014), 3D CTU cross terms or
//                the first-order fallback (hy_getRiemannState.F90:1053-1090
//                and y/z analogues, fallbackToFirstOrder :1456-1475), upwind
//                fluxes F_dens * X (hy_getFaceFlux.F90:453-467), the flux
//                divergence, the update
//                X = (X rho_old + dt sum (F_L - F_R)/dx) / rho_new
//                (updateSpeciesMassScalar, hy_unsplitUpdate.F90:1300-1318)
//                and the renormalisation of the species (:850-859).
// Every direction reads the old X (the step is unsplit), so one kernel stages
// a species once and keeps the divergence in registers across directions.
#pragma once
#include "hy_kernels.cuh"

namespace fhy {

// min / max as the CPU oracle takes them (a < b ? a : b), so that signed
// zeros come out the same
__device__ __forceinline__ double minmod_s(double a, double b) {     // hy_slopeLimiters.F90:56-60
  return .5 * (copysign(1., a) + copysign(1., b)) * rmin(fabs(a), fabs(b));
}

// Launch shape and shared memory of k_spec_step: the velocities on the box
// of one guard layer, one species on the cells the stencils read (the box
// plus, along each direction, three cells beyond the block on the lines of
// interior cells), and two face-flux arrays used by alternate directions.
template <int NDIM, int NX, int NY, int NZ>
struct SpecStep {
  using B = Box<NDIM, NX, NY, NZ>;
  using E = Ext<NDIM, NX, NY, NZ, 3>;
  static constexpr int n1 = DirGeom<NDIM, NX, NY, NZ, double, 1>::n;
  static constexpr int n2 = NDIM > 1 ? DirGeom<NDIM, NX, NY, NZ, double, 2>::n : 0;
  static constexpr int n3 = NDIM > 2 ? DirGeom<NDIM, NX, NY, NZ, double, 3>::n : 0;
  static constexpr int NL = n1 > n2 ? (n1 > n3 ? n1 : n3) : (n2 > n3 ? n2 : n3);   // line cells of a direction
  static constexpr int NCB = NX * NY * NZ;
  static constexpr int PER = (NL + 319) / 320;                     // line cells per thread
  static constexpr int NT = ((NL + PER - 1) / PER + 31) / 32 * 32;
  static constexpr int CPT = (NCB + NT - 1) / NT;                  // interior cells per thread
  static constexpr int MINB = NDIM > 2 ? 3 : 1;                     // CTAs per SM (3D: what shared memory allows)
  // staged cells: the box, then per direction two layers on either side of
  // the block on the lines of interior cells
  static constexpr int NPX = 4 * NY * (NDIM > 2 ? NZ : 1), NPY = NDIM > 1 ? 4 * NX * (NDIM > 2 ? NZ : 1) : 0,
                       NPZ = NDIM > 2 ? 4 * NX * NY : 0;
  static constexpr int NSTG = B::n + NPX + NPY + NPZ;
  static constexpr int NK = 16;                                    // CTA-wide constants
  static constexpr int NNB = NDIM > 2 ? 27 : 9;                    // neighbour blocks (uniform grids)
  static constexpr size_t smem_bytes() {
    return ((size_t)NDIM * B::n + E::n + 2 * NL + NK + 2 * NCB) * sizeof(double) +
           (size_t)NSTG * (sizeof(int) + sizeof(short)) + NNB * sizeof(int);
  }
  // staged cell u: its block-local coordinates
  __device__ static __forceinline__ void staged(int u, int &i, int &j, int &k) {
    if (u < B::n) {
      i = u % B::bx - 1;
      j = NDIM > 1 ? (u / B::bx) % B::by - 1 : 0;
      k = NDIM > 2 ? u / (B::bx * B::by) - 1 : 0;
      return;
    }
    int v = u - B::n, d = 0;
    if (v >= NPX) { v -= NPX; d = 1; if (v >= NPY) { v -= NPY; d = 2; } }
    const int w = v & 3, r = v >> 2;                                // layer: -3, -2, N+1, N+2
    const int n = d == 0 ? NX : (d == 1 ? NY : NZ);
    const int a = w < 2 ? w - 3 : n - 1 + w;
    const int n1 = d == 0 ? NY : NX;                                // first transverse extent
    const int t1 = NDIM > 1 ? r % n1 : 0, t2 = NDIM > 1 ? r / n1 : 0;
    if (d == 0) { i = a; j = t1; k = t2; }
    else if (d == 1) { i = t1; j = a; k = t2; }
    else { i = t1; j = t2; k = a; }
  }
};

// CTA-wide constants of k_spec_step in shared memory (computed once per block)
enum { SK_HDTX = 0, SK_HDTY, SK_HDTZ, SK_DIR0 };   // then per direction: delta, 1/delta, dtn/2, fac


// Face fluxes of one species along DIR: PPM face values of every line cell
// traced along the entropy wave and flattened, the transverse corrections
// with SpcSig of the other directions, the 3D CTU cross terms or the
// first-order fallback; each face takes F_dens * X from its upwind cell, so
// the cell on the upwind side writes it (sF[t] is the face left of line
// cell t).  SpcSig (the entropy-wave speed times the upwind difference) is
// taken from the staged velocities and species where it is read.
template <int NDIM, int NX, int NY, int NZ, int DIR>
__device__ __forceinline__ void spec_faces(const DevParams &P, int slot, const double *sV, const double *sX,
                                           double *sF, const double *sK) {
  using L = DirGeom<NDIM, NX, NY, NZ, double, DIR>;
  using B = Box<NDIM, NX, NY, NZ>;
  using E = Ext<NDIM, NX, NY, NZ, 3>;
  constexpr int es = DIR == 1 ? 1 : (DIR == 2 ? E::ex : E::ex * E::ey);
  constexpr int A1 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1), S1 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2);
  constexpr int A2 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2), S2 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1);
  const bool ctu = NDIM == 3 && P.use_ctu;
  const size_t lb = sp_line_base<NDIM, NX, NY, NZ, DIR>(slot);
  const double hdtx = sK[SK_HDTX], hdty = sK[SK_HDTY], hdtz = sK[SK_HDTZ];
  const double hdtn = sK[SK_DIR0 + 4 * (DIR - 1) + 2], fac = sK[SK_DIR0 + 4 * (DIR - 1) + 3];
  constexpr double r3 = 1. / 3., r6 = 1. / 6.;
  // SpcSig of direction d (0-based) at box cell (i, j, k)
  auto sig = [&](int d, int i, int j, int k) {
    const int st = d == 0 ? 1 : (d == 1 ? E::ex : E::ex * E::ey);
    const int e = E::idx(i, j, k);
    const double lam = sV[d * B::n + B::idx(i, j, k)];
    double g;
    if (lam > 0.) g = sX[e] - sX[e - st];
    else g = sX[e + st] - sX[e];
    return lam * g;
  };
  for (int t = threadIdx.x; t < L::n; t += blockDim.x) {
    int i, j, k;
    L::decode(t, i, j, k);
    // the hydro's per-line data first, so that its latency overlaps the stencil
    const int a = L::along(i, j, k);
    const double flat = P.use_flattening ? __ldg(P.sp_flat + lb + t) : 0.;
    const bool fb = ctu && __ldg(P.sp_fb + lb + t);
    const double mL = a >= 0 ? __ldg(P.sp_mf + lb + t) : 0.;
    const double mR = a < L::nd ? __ldg(P.sp_mf + lb + t + L::stride) : 0.;
    const int e = E::idx(i, j, k);
    const double Smm = sX[e - 2 * es], Sm = sX[e - es], Sc = sX[e], Sp = sX[e + es], Spp = sX[e + 2 * es];
    const int bi = B::idx(i, j, k);
    const double lam = sV[(DIR - 1) * B::n + bi];
    double dP = minmod_s(Sp - Sc, Spp - Sp);
    double d0 = minmod_s(Sc - Sm, Sp - Sc);
    double dN = minmod_s(Sm - Smm, Sc - Sm);
    double l = 0.5 * (Sc + Sm) - div_rn(d0 - dN, 6., r6);
    double r = 0.5 * (Sc + Sp) - div_rn(dP - d0, 6., r6);
    l = rmax(rmin(Sc, Sm), rmin(rmax(Sc, Sm), l));
    r = rmax(rmin(Sc, Sp), rmin(rmax(Sc, Sp), r));
    if ((r - Sc) * (Sc - l) <= 0.) { r = Sc; l = Sc; }
    if (6. * (r - l) * (Sc - 0.5 * (r + l)) > (r - l) * (r - l)) l = 3. * Sc - 2. * r;
    if (6. * (r - l) * (Sc - 0.5 * (r + l)) < -((r - l) * (r - l))) r = 3. * Sc - 2. * l;
    d0 = r - l;
    const double s6 = 6. * (Sc - 0.5 * (r + l));
    const double lm = rmin(lam, 0.), lp = rmax(lam, 0.);
    l = l - lm * hdtn * (d0 + (1. + div_rn(lm * 4., 3., r3) * hdtn) * s6);
    r = r - lp * hdtn * (d0 - (1. - div_rn(lp * 4., 3., r3) * hdtn) * s6);
    if (P.use_flattening) {                   // the coefficient left by the hydro direction kernel
      l = flat * Sc + (1.0 - flat) * l;
      r = flat * Sc + (1.0 - flat) * r;
    }
    // transverse corrections with SpcSig of the other directions
    if (NDIM == 2) {
      if (DIR == 1) { const double g = sig(1, i, j, k); l = l - hdty * g; r = r - hdty * g; }
      else          { const double g = sig(0, i, j, k); l = l - hdtx * g; r = r - hdtx * g; }
    } else if (NDIM == 3) {
      if (DIR == 1) {
        const double gy = sig(1, i, j, k), gz = sig(2, i, j, k);
        l = l - hdty * gy; r = r - hdty * gy; l = l - hdtz * gz; r = r - hdtz * gz;
      } else if (DIR == 2) {
        const double gx = sig(0, i, j, k), gz = sig(2, i, j, k);
        l = l - hdtx * gx; r = r - hdtx * gx; l = l - hdtz * gz; r = r - hdtz * gz;
      } else {
        const double gx = sig(0, i, j, k), gy = sig(1, i, j, k);
        l = l - hdtx * gx - hdty * gy; r = r - hdtx * gx - hdty * gy;
      }
    }
    if (ctu) {
      if (fb) {
        l = Sc;
        r = Sc;
      } else {
        double T[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int ax = u ? A2 : A1, sd = u ? S2 : S1;
          const double lamA = sV[(ax - 1) * B::n + bi];
          const double gm = sig(sd - 1, i - (ax == 1), j - (ax == 2), k - (ax == 3));
          const double g0 = sig(sd - 1, i, j, k);
          const double gp = sig(sd - 1, i + (ax == 1), j + (ax == 2), k + (ax == 3));
          const double g = lamA > 0. ? g0 - gm : gp - g0;
          T[u] = lamA * g;
        }
        r = r + (T[0] + T[1]) * fac;
        l = l + (T[0] + T[1]) * fac;
      }
    }
    if (a >= 0 && mL < 0.) sF[t] = mL * l;                // the face on the left: upwind if the mass flows left
    if (a < L::nd && !(mR < 0.)) sF[t + L::stride] = mR * r;   // the face on the right: upwind otherwise
  }
}

// The mixed path's face fluxes: the face values of spec_faces in FP32 on
// differences from the cell's mass fraction X_c (taken in FP64 and rounded:
// the delta form of the mixed hydro reconstruction, in which X_c is the
// origin, so 3 X_c - 2 r becomes -2 r and f X_c + (1 - f) l becomes
// (1 - f) l), SpcSig in FP32 on FP64 differences, and the upwind flux
// F_dens * (X_c + delta) in FP64.
template <int NDIM, int NX, int NY, int NZ, int DIR>
__device__ __forceinline__ void spec_faces_mx(const DevParams &P, int slot, const double *sV, const double *sX,
                                              double *sF, const double *sK) {
  using L = DirGeom<NDIM, NX, NY, NZ, double, DIR>;
  using B = Box<NDIM, NX, NY, NZ>;
  using E = Ext<NDIM, NX, NY, NZ, 3>;
  constexpr int es = DIR == 1 ? 1 : (DIR == 2 ? E::ex : E::ex * E::ey);
  constexpr int A1 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1), S1 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2);
  constexpr int A2 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2), S2 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1);
  const bool ctu = NDIM == 3 && P.use_ctu;
  const size_t lb = sp_line_base<NDIM, NX, NY, NZ, DIR>(slot);
  const float hdtx = float(sK[SK_HDTX]), hdty = float(sK[SK_HDTY]), hdtz = float(sK[SK_HDTZ]);
  const float hdtn = float(sK[SK_DIR0 + 4 * (DIR - 1) + 2]), fac = float(sK[SK_DIR0 + 4 * (DIR - 1) + 3]);
  auto sig = [&](int d, int i, int j, int k) -> float {
    const int st = d == 0 ? 1 : (d == 1 ? E::ex : E::ex * E::ey);
    const int e = E::idx(i, j, k);
    const double lam = sV[d * B::n + B::idx(i, j, k)];
    const double g = lam > 0. ? sX[e] - sX[e - st] : sX[e + st] - sX[e];
    return float(lam) * float(g);
  };
  auto minmod = [](float a, float b) { return a * b > 0.f ? copysignf(fminf(fabsf(a), fabsf(b)), a) : 0.f; };
  for (int t = threadIdx.x; t < L::n; t += blockDim.x) {
    int i, j, k;
    L::decode(t, i, j, k);
    const int a = L::along(i, j, k);
    const float flat = P.use_flattening ? float(__ldg(P.sp_flat + lb + t)) : 0.f;
    const bool fb = ctu && __ldg(P.sp_fb + lb + t);
    const double mL = a >= 0 ? __ldg(P.sp_mf + lb + t) : 0.;
    const double mR = a < L::nd ? __ldg(P.sp_mf + lb + t + L::stride) : 0.;
    const int e = E::idx(i, j, k);
    const double Xc = sX[e];
    const float Smm = float(sX[e - 2 * es] - Xc), Sm = float(sX[e - es] - Xc);
    const float Sp = float(sX[e + es] - Xc), Spp = float(sX[e + 2 * es] - Xc);
    const int bi = B::idx(i, j, k);
    const float lam = float(sV[(DIR - 1) * B::n + bi]);
    float dP = minmod(Sp, Spp - Sp);
    float d0 = minmod(-Sm, Sp);
    float dN = minmod(Sm - Smm, -Sm);
    float l = 0.5f * Sm - (d0 - dN) * (1.f / 6.f);
    float r = 0.5f * Sp - (dP - d0) * (1.f / 6.f);
    l = fmaxf(fminf(0.f, Sm), fminf(fmaxf(0.f, Sm), l));
    r = fmaxf(fminf(0.f, Sp), fminf(fmaxf(0.f, Sp), r));
    if (r * (-l) <= 0.f) { r = 0.f; l = 0.f; }
    if (6.f * (r - l) * (-0.5f * (r + l)) > (r - l) * (r - l)) l = -2.f * r;
    if (6.f * (r - l) * (-0.5f * (r + l)) < -((r - l) * (r - l))) r = -2.f * l;
    d0 = r - l;
    const float s6 = -3.f * (r + l);
    const float lm = fminf(lam, 0.f), lp = fmaxf(lam, 0.f);
    l = l - lm * hdtn * (d0 + (1.f + lm * (4.f / 3.f) * hdtn) * s6);
    r = r - lp * hdtn * (d0 - (1.f - lp * (4.f / 3.f) * hdtn) * s6);
    if (P.use_flattening) { l = (1.f - flat) * l; r = (1.f - flat) * r; }
    if (NDIM == 2) {
      const float c = DIR == 1 ? hdty * sig(1, i, j, k) : hdtx * sig(0, i, j, k);
      l -= c; r -= c;
    } else if (NDIM == 3) {
      const float c = DIR == 1 ? hdty * sig(1, i, j, k) + hdtz * sig(2, i, j, k)
                               : (DIR == 2 ? hdtx * sig(0, i, j, k) + hdtz * sig(2, i, j, k)
                                           : hdtx * sig(0, i, j, k) + hdty * sig(1, i, j, k));
      l -= c; r -= c;
    }
    if (ctu) {
      if (fb) {
        l = 0.f;
        r = 0.f;
      } else {
        float T = 0.f;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int ax = u ? A2 : A1, sd = u ? S2 : S1;
          const float lamA = float(sV[(ax - 1) * B::n + bi]);
          const float gm = sig(sd - 1, i - (ax == 1), j - (ax == 2), k - (ax == 3));
          const float g0 = sig(sd - 1, i, j, k);
          const float gp = sig(sd - 1, i + (ax == 1), j + (ax == 2), k + (ax == 3));
          T += lamA * (lamA > 0.f ? g0 - gm : gp - g0);
        }
        r += T * fac;
        l += T * fac;
      }
    }
    if (a >= 0 && mL < 0.) sF[t] = mL * (Xc + double(l));
    if (a < L::nd && !(mR < 0.)) sF[t + L::stride] = mR * (Xc + double(r));
  }
}

// one direction of k_spec_step: face fluxes, the species flux register at
// fine/coarse faces (AMR), and the flux divergence added, in the x, y, z
// order of the update, to the accumulators of the thread's interior cells
template <int NDIM, int NX, int NY, int NZ, int DIR, bool MX>
__device__ __forceinline__ void spec_dir(const DevParams &P, int b, int3 bc, int slot, int q, const double *sV,
                                         const double *sX, double *sF, const double *sK,
                                         double (&acc)[SpecStep<NDIM, NX, NY, NZ>::CPT]) {
  using L = DirGeom<NDIM, NX, NY, NZ, double, DIR>;
  using SS = SpecStep<NDIM, NX, NY, NZ>;
  if constexpr (MX) spec_faces_mx<NDIM, NX, NY, NZ, DIR>(P, slot, sV, sX, sF, sK);
  else spec_faces<NDIM, NX, NY, NZ, DIR>(P, slot, sV, sX, sF, sK);
  __syncthreads();
  if (P.sp_freg) {
    flux_register_v<NDIM, NX, NY, NZ, DIR>(P, b, bc, sF, 0, [](int along, int t1, int t2) {
      const int i = DIR == 1 ? along : t1, j = DIR == 1 ? t1 : (DIR == 2 ? along : t2),
                k = DIR == 3 ? along : (NDIM > 2 ? t2 : 0);
      return L::idx(i, j, k);
    }, P.sp_freg + (size_t)q * P.sp_freg_stride, 1);
    __syncthreads();
  }
  if (P.fmode == 1 || P.fmode == 2) {   // split step: keep the face fluxes
    constexpr int fx = NX + (DIR == 1), fy = NY + (DIR == 2), NF = (NX + 1) * NY * NZ;
    double *dst = P.sp_fstore + (((size_t)b * NDIM + (DIR - 1)) * P.nsp + q) * NF;
    for (int f = threadIdx.x; f < NF; f += blockDim.x) dst[f] = sF[L::idx(f % fx, (f / fx) % fy, f / (fx * fy))];
    if (P.fmode == 2) return;
  }
  const double delta = sK[SK_DIR0 + 4 * (DIR - 1)], rdelta = sK[SK_DIR0 + 4 * (DIR - 1) + 1];
#pragma unroll
  for (int u = 0; u < SS::CPT; ++u) {
    const int c = threadIdx.x + u * SS::NT;
    if (c < SS::NCB) {
      const int i = c % NX, j = (c / NX) % NY, k = c / (NX * NY);
      const int t = L::idx(i, j, k);
      const double d = div_rn(sF[t] - sF[t + L::stride], delta, rdelta);
      acc[u] = DIR == 1 ? d : acc[u] + d;
    }
  }
}

// The species pass of one step, one CTA per block: the velocities are staged
// once, then per species its cells, the three direction sweeps and
// X = (X rho_old + dt sum (F_L - F_R)/dx) / rho_new; last, the species (not
// the mass scalars) are renormalised to a unit sum.  The face arrays
// alternate between directions, so a direction's divergence and the next
// direction's faces need no barrier between them.
// MX: the mixed path's FP32 face values (spec_faces_mx)
template <int NDIM, int NX, int NY, int NZ, bool MX>
__global__ void __launch_bounds__(SpecStep<NDIM, NX, NY, NZ>::NT, SpecStep<NDIM, NX, NY, NZ>::MINB) k_spec_step(const DevParams P, size_t ncells) {
  using SS = SpecStep<NDIM, NX, NY, NZ>;
  using B = Box<NDIM, NX, NY, NZ>;
  using E = Ext<NDIM, NX, NY, NZ, 3>;
  constexpr int NCB = SS::NCB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sRo = reinterpret_cast<double *>(smem_raw);    // [NCB] old density (16-byte aligned)
  double *sRn = sRo + NCB;                               // [NCB] new density
  double *sV = sRn + NCB;                                // [NDIM][B::n]
  double *sX = sV + NDIM * B::n;                         // [E::n]
  double *sF0 = sX + E::n, *sF1 = sF0 + SS::NL;
  double *sK = sF1 + SS::NL;                             // [NK]
  int *tSrc = reinterpret_cast<int *>(sK + SS::NK);      // [NSTG] source of each staged cell
  int *sNb = tSrc + SS::NSTG;                            // [NNB] neighbour blocks
  short *tExt = reinterpret_cast<short *>(sNb + SS::NNB);   // [NSTG] its place in sX
  const int b = P.blk_list ? P.blk_list[blockIdx.x] : blockIdx.x;
  const int slot = P.slot ? P.slot[b] : (int)blockIdx.x;
  const int3 bc = blk_coords(P, b);
  const double dt = P.dt_dev ? *P.dt_dev : P.dt;
  const bool amr = P.sp_lh != nullptr;
  using H = Halo<NDIM, NX, NY, NZ>;
  // ---- the densities (contiguous per block), the constants, the neighbours
  for (int c = threadIdx.x; c < NCB / 2; c += SS::NT) {
    cp_async16(sRo + 2 * c, P.s_in[0] + (size_t)b * NCB + 2 * c);
    cp_async16(sRn + 2 * c, P.s_out[0] + (size_t)b * NCB + 2 * c);
  }
  if (threadIdx.x == 0) {
    double del[3];
    blk_deltas(P, b, del);                // the block's level
    sK[SK_HDTX] = 0.5 * dt / del[0];
    sK[SK_HDTY] = 0.5 * dt / del[1];
    sK[SK_HDTZ] = 0.5 * dt / del[2];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double da = d == 0 ? del[1] : (d == 1 ? del[2] : del[0]), db = d == 0 ? del[2] : (d == 1 ? del[0] : del[1]);
      sK[SK_DIR0 + 4 * d] = del[d];
      sK[SK_DIR0 + 4 * d + 1] = 1. / del[d];
      sK[SK_DIR0 + 4 * d + 2] = 0.5 * (dt / del[d]);
      sK[SK_DIR0 + 4 * d + 3] = dt * dt / (6. * da * db);
    }
  }
  if (!amr) neighbour_table<NDIM, NX, NY, NZ>(P, bc, sNb);
  __syncthreads();
  // ---- sources of the staged cells: offsets into a species of the state,
  // or (flagged in the sign bit) into the leaf's species guard buffer on AMR
  for (int u = threadIdx.x; u < SS::NSTG; u += SS::NT) {
    int i, j, k;
    SS::staged(u, i, j, k);
    tExt[u] = (short)E::idx(i, j, k);
    if (amr && !is_inside<NDIM, NX, NY, NZ>(i, j, k)) {
      tSrc[u] = (int)(0x80000000u | (unsigned)H::idx(i, j, k));
    } else if (amr) {
      tSrc[u] = (int)((size_t)b * NCB + (size_t)((k * NY + j) * NX + i));
    } else {
      int fx, fy, fz;
      tSrc[u] = (int)cell_src_nb<NDIM, NX, NY, NZ>(P, b, bc, sNb, i, j, k, fx, fy, fz);
    }
  }
  // ---- velocities of the box cells, mirrored in reflecting guard cells
  // (flip: the thread's cells whose component d changes sign, bit 3 r + d)
  constexpr int IB = (B::n + SS::NT - 1) / SS::NT;
  static_assert(3 * IB <= 32, "flip mask");
  unsigned flip = 0;
#pragma unroll
  for (int r = 0; r < IB; ++r) {
    const int c = threadIdx.x + r * SS::NT;
    if (c < B::n) {
      const int i = c % B::bx - 1, j = NDIM > 1 ? (c / B::bx) % B::by - 1 : 0;
      const int k = NDIM > 2 ? c / (B::bx * B::by) - 1 : 0;
      if (amr && !is_inside<NDIM, NX, NY, NZ>(i, j, k)) {     // the leaf guard buffer (mirrored)
        const double *h = P.lh + (size_t)slot * 5 * H::n + H::idx(i, j, k);
#pragma unroll
        for (int d = 0; d < NDIM; ++d) cp_async8(sV + d * B::n + c, h + (1 + d) * H::n);
      } else {
        int f[3] = {0, 0, 0};
        const size_t o = amr ? (size_t)b * NCB + (size_t)((k * NY + j) * NX + i)
                             : cell_src_nb<NDIM, NX, NY, NZ>(P, b, bc, sNb, i, j, k, f[0], f[1], f[2]);
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
          cp_async8(sV + d * B::n + c, P.s_in[1 + d] + o);
          if (f[d]) flip |= 1u << (3 * r + d);
        }
      }
    }
  }
  cp_async_wait_all();
  if (flip) {
#pragma unroll
    for (int r = 0; r < IB; ++r)
#pragma unroll
      for (int d = 0; d < NDIM; ++d)
        if (flip >> (3 * r + d) & 1u) {
          double *v = sV + d * B::n + threadIdx.x + r * SS::NT;
          *v = -*v;
        }
  }
  __syncthreads();
  const size_t lhb = amr ? (size_t)slot * P.nsp * H::n : 0;
  for (int q = 0; q < P.nsp; ++q) {
    const double *xin = P.sp_in + (size_t)q * ncells;
    const double *xlh = amr ? P.sp_lh + lhb + (size_t)q * H::n : xin;
    for (int u = threadIdx.x; u < SS::NSTG; u += SS::NT) {
      const int v = tSrc[u];
      cp_async8(sX + tExt[u], v >= 0 ? xin + v : xlh + (v & 0x7fffffff));
    }
    cp_async_wait_all();
    __syncthreads();
    double acc[SS::CPT];
    spec_dir<NDIM, NX, NY, NZ, 1, MX>(P, b, bc, slot, q, sV, sX, sF0, sK, acc);
    if constexpr (NDIM > 1) spec_dir<NDIM, NX, NY, NZ, 2, MX>(P, b, bc, slot, q, sV, sX, sF1, sK, acc);
    if constexpr (NDIM > 2) spec_dir<NDIM, NX, NY, NZ, 3, MX>(P, b, bc, slot, q, sV, sX, sF0, sK, acc);
    // the old mass fractions from the staged species; the barrier keeps the
    // next species' copies from overwriting them before every thread is done
    if (P.fmode != 2) {
#pragma unroll
    for (int u = 0; u < SS::CPT; ++u) {
      const int c = threadIdx.x + u * SS::NT;
      if (c < NCB) {
        const double X = sX[E::idx(c % NX, (c / NX) % NY, c / (NX * NY))];
        P.sp_out[(size_t)q * ncells + (size_t)b * NCB + c] =
            __ddiv_rn(__dadd_rn(__dmul_rn(X, sRo[c]), __dmul_rn(dt, acc[u])), sRn[c]);   // never contracted
      }
    }
    }
    __syncthreads();
  }
  if (P.fmode == 2) return;                // fluxes only: the state is not updated
  // ---- species (not mass scalars) renormalised to a unit sum; each thread
  // reads back only the cells it wrote
  if (P.nspec > 0) {
#pragma unroll
    for (int u = 0; u < SS::CPT; ++u) {
      const int c = threadIdx.x + u * SS::NT;
      if (c >= NCB) continue;
      const size_t off = (size_t)b * NCB + c;
      double sum = 0.;
      for (int q = 0; q < P.nspec; ++q) sum = sum + P.sp_out[(size_t)q * ncells + off];
      for (int q = 0; q < P.nspec; ++q) P.sp_out[(size_t)q * ncells + off] = P.sp_out[(size_t)q * ncells + off] / sum;
    }
  }
}

// The species update of the split step (flash_hy_update_solution) from the
// kept, possibly replaced face fluxes: the divergence in the x, y, z order
// and the update of k_spec_step, then the renormalisation.
template <int NDIM, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256) k_spec_update(const DevParams P, size_t ncells) {
  constexpr int NCB = NX * NY * NZ, NF = (NX + 1) * NY * NZ;
  const int b = P.blk_list ? P.blk_list[blockIdx.x] : blockIdx.x;
  const double dt = P.dt_dev ? *P.dt_dev : P.dt;
  double del[3];
  blk_deltas(P, b, del);
  const double rdel[3] = {1. / del[0], 1. / del[1], 1. / del[2]};
  for (int c = threadIdx.x; c < NCB; c += blockDim.x) {
    const int i = c % NX, j = (c / NX) % NY, k = c / (NX * NY);
    const size_t off = (size_t)b * NCB + c;
    const double ro = P.s_in[0][off], rn = P.s_out[0][off];
    for (int q = 0; q < P.nsp; ++q) {
      double acc = 0.;
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        const double *F = P.sp_fstore + (((size_t)b * NDIM + d) * P.nsp + q) * NF;
        const int fx = NX + (d == 0), fy = NY + (d == 1);
        const int fl = (k * fy + j) * fx + i, fr = fl + (d == 0 ? 1 : (d == 1 ? fx : fx * fy));
        const double dd = div_rn(F[fl] - F[fr], del[d], rdel[d]);
        acc = d == 0 ? dd : acc + dd;
      }
      P.sp_out[(size_t)q * ncells + off] =
          __ddiv_rn(__dadd_rn(__dmul_rn(P.sp_in[(size_t)q * ncells + off], ro), __dmul_rn(dt, acc)), rn);
    }
    if (P.nspec > 0) {
      double sum = 0.;
      for (int q = 0; q < P.nspec; ++q) sum = sum + P.sp_out[(size_t)q * ncells + off];
      for (int q = 0; q < P.nspec; ++q) P.sp_out[(size_t)q * ncells + off] = P.sp_out[(size_t)q * ncells + off] / sum;
    }
  }
}

}  // namespace fhy
