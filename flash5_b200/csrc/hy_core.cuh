// hy_core.cuh -- device arithmetic of the unsplit hydro update.
//
// Templated on the reconstruction/flux type R (double for the FP64 paths,
// float for the mixed path).  The expressions keep the evaluation order of
// the Fortran they restate (paths inside mbdevpl/FLASH5,
// source/physics/Hydro/HydroMain/unsplit unless stated), so that the FP64
// variant compiled without FMA contraction reproduces an IEEE evaluation of
// the reference arithmetic.  The hydro eigenvectors are sparse
// (OnlyHydro/hy_eigenVector.F90:114-151); the dot products below add only
// their non-zero terms, in index order, which gives the same values as the
// dense sums (the skipped terms are exact zeros).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "exact_rs.cuh"

namespace fhy {

// primitive slots of UHD.h:374-383 (HY_DENS..HY_EINT), 0-based
enum { HD = 0, HVX = 1, HVY = 2, HVZ = 3, HP = 4, HGC = 5, HGE = 6, HEI = 7 };
// flux slots of OnlyHydro/Config:6-13, 0-based
enum { FDENS = 0, FXMOM, FYMOM, FZMOM, FENER, FPRES, FEINT, FVOLU, NFLX = 8 };

// status bits (include/flash_hy.h)
constexpr unsigned ST_NEG_SOUND = 1u << 0;
constexpr unsigned ST_NEWTON = 1u << 2;
constexpr unsigned ST_NAN = 1u << 3;

struct DevParams {
  int ndim;
  int nbx, nby, nbz;          // blocks per axis of the uniform level
  int bc[6];
  int use_flattening, use_steepening, char_limiting, limiter, use_aux_eint, use_ctu;
  int riemann;                // 4 = HLLC, 100 = exact
  int learned;                // exact solver: MLP initial guess
  double lim_beta, gamma, gam1inv, ggprodinv, abar, smalle, smlrho, eswitch, tiny, cfl;
  double del[3];
  double dt;
  const double *dt_dev;       // when set, dt is read from device memory (graph-replayed steps)
  const int *blk_at;          // block index at block coordinates
  const int *blk_nbr;         // uniform grids: face neighbours of each block [b][x-, x+, y-, y+, z-, z+]
                              // (-1 beyond a non-periodic boundary or absent from the grid)
  const int *blk_coord;       // 3 ints per block
  const int *blk_list;        // optional list of blocks to update (NULL = all)
  const double *s_in[5];      // dens, velx, vely, velz, eint (block-major SoA)
  double *s_out[5];
  unsigned *status;
  const void *mlp;            // learned-guess network, xrs::MlpPacked (exact solver; NULL = off)
  double *harvest;            // optional face-state sample, [7][harvest_cap] (dl,ul,pl,dr,ur,pr,gamma)
  unsigned long long *harvest_n;
  long long harvest_cap;
  unsigned harvest_mask;      // a face is kept when its hash & mask == 0
  double rs_tol;              // exact solver: relative tolerance of p*
  int rs_max_iter;
  // AMR hierarchy (blk_level == NULL: one uniform level)
  const int *blk_level;       // level of each node
  const int *leaf;            // 1 for the leaves
  const int *parent;          // parent node, -1 on level 1
  const int *slot;            // leaf slot (guard buffer, sig scratch, flux register) / parent slot (halo)
  const int *at;              // node by (level, block coordinates), -1 where the level is not refined
  int at_off[17];
  int at_ext[17][3];
  double *lh;                 // leaf guard cells after the EOS: [slot][5][(N+8)^d]
  double *gp;                 // parent guard-inclusive blocks: [slot][6][(N+8)^d] (rho, v, e, E)
  double *pe;                 // parents' restricted specific total energy [node * NCB + cell]
  double *freg;               // fine-face fluxes at fine/coarse faces: [leaf slot][2 ndim][faces][8]
  // split step (hy_computeFluxes with Uout disassociated, hy_updateSolution):
  // 0 = fused step, 1 = store the fluxes and update, 2 = store the fluxes
  // only, 3 = update from the stored fluxes
  int fmode;
  double *fstore;             // [block][ndim][8 x faces (FLASH flx order) + n+1/2 pressure sum per cell]
  // species and mass scalars (nsp > 0; the first nspec are renormalised):
  // [nsp][ncells] block-major SoA interiors, double-buffered like s_in/s_out.
  // The hydro direction kernels leave for them, per launch slot and
  // direction in the line-cell order of DirGeom, the face mass flux
  // (sp_mf), whether the 3D CTU stage fell back to first order (sp_fb) and
  // the flattening coefficient (sp_flat).
  int nsp, nspec;
  const double *sp_in;
  double *sp_out;
  double *sp_mf;
  unsigned char *sp_fb;
  double *sp_flat;            // flattening coefficient of each line cell (same layout)
  // species on AMR hierarchies: guard cells of the leaves [leaf slot][nsp]
  // [halo], guard-inclusive copies of the parents [parent slot][nsp][halo],
  // the species flux register [nsp][leaf slot][2 ndim][faces]
  double *sp_lh, *sp_gp, *sp_freg;
  size_t sp_ncells;           // stride of the species arrays
  size_t sp_freg_stride;      // doubles per species in sp_freg
  // split step: species face fluxes F_dens * X per block, direction and
  // species, in the face order of the hydro flux store [block][dir][nsp][faces]
  double *sp_fstore;
  // the exact Riemann solver's gas constants (xrs::gas_of(gamma), host-side)
  xrs::Gas gas;
};

// Cell sizes of block b: level-1 deltas scaled by 2^(1-level) (exact).
__device__ __forceinline__ void blk_deltas(const DevParams &P, int b, double del[3]) {
  const double s = P.blk_level ? ldexp(1.0, 1 - P.blk_level[b]) : 1.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) del[d] = d < P.ndim ? P.del[d] * s : P.del[d];
}

__device__ __forceinline__ int at_node(const DevParams &P, int l, int x, int y, int z) {
  return P.at[P.at_off[l] + (z * P.at_ext[l][1] + y) * P.at_ext[l][0] + x];
}

template <class R> __device__ __forceinline__ R rmax(R a, R b) { return a > b ? a : b; }
template <class R> __device__ __forceinline__ R rmin(R a, R b) { return a < b ? a : b; }

// x / b rounded to nearest, from rb = RN(1 / b) (Markstein's theorem,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34 (1990): q0 = RN(x rb) is within an ulp of
// x / b, the remainder x - q0 b is exact with an FMA, and
// RN(q0 + (x - q0 b) rb) = RN(x / b)).  Outside the exponent range where
// the remainder cannot underflow or the product overflow (zeros,
// subnormals, infinities and NaN included) it divides.  Equal to x / b in
// every bit: a CPU test checks the method on random and special operands,
// and the FP64 GPU parity tests compare the kernels that use it with the
// oracle's divisions.
__device__ __forceinline__ double div_rn(double x, double b, double rb) {
  const double q0 = x * rb;
  const double a = fabs(q0), ax = fabs(x);
  if (a > 0x1p-960 && a < 0x1p1000 && ax > 0x1p-960 && ax < 0x1p1000) return fma(fma(-q0, b, x), rb, q0);
  return x / b;
}
__device__ __forceinline__ double rsign(double a, double b) { return copysign(fabs(a), b); }
__device__ __forceinline__ float rsign(float a, float b) { return copysignf(fabsf(a), b); }
__device__ __forceinline__ double rabs(double a) { return fabs(a); }
__device__ __forceinline__ float rabs(float a) { return fabsf(a); }
__device__ __forceinline__ double rsqrt_(double a) { return sqrt(a); }
__device__ __forceinline__ float rsqrt_(float a) { return sqrtf(a); }

// velocity slots of the normal / first / second transverse direction
// (hy_eigenVector.F90:75-89)
template <int DIR> struct Slots;
template <> struct Slots<1> { static constexpr int v1 = HVX, v2 = HVY, v3 = HVZ; };
template <> struct Slots<2> { static constexpr int v1 = HVY, v2 = HVZ, v3 = HVX; };
template <> struct Slots<3> { static constexpr int v1 = HVZ, v2 = HVX, v3 = HVY; };

// ---------------------------------------------------------------------------
// slope limiters, hy_slopeLimiters.F90:38-60; hy_TVDslope.F90:213-245
// ---------------------------------------------------------------------------
template <class R> __device__ __forceinline__ R lim_vanleer(R a, R b) {
  if (a * b <= R(0)) return R(0);
  return R(2) * a * b / (a + b);
}
template <class R> __device__ __forceinline__ R lim_mc(R a, R b) {
  R m = rabs(a), t = R(.25) * rabs(a + b);
  if (t < m) m = t;
  if (rabs(b) < m) m = rabs(b);
  return (rsign(R(1), a) + rsign(R(1), b)) * m;
}
template <class R> __device__ __forceinline__ R lim_minmod(R a, R b) {
  R m = rabs(a) < rabs(b) ? rabs(a) : rabs(b);
  return R(.5) * (rsign(R(1), a) + rsign(R(1), b)) * m;
}
template <class R> __device__ __forceinline__ R limit2(int lim, R beta, R d1, R d2) {
  switch (lim) {
    case 1: return lim_minmod(d1, d2);
    case 2: return lim_mc(d1, d2);
    case 4: return lim_vanleer(d1, d2);
    case 5:
      if (d2 > R(0)) return rmax(R(0), rmax(rmin(beta * d1, d2), rmin(d1, beta * d2)));
      return rmin(R(0), rmin(rmax(beta * d1, d2), rmax(d1, beta * d2)));
  }
  return R(0);
}

// ---------------------------------------------------------------------------
// eigen system in primitive variables: hy_eigenParameters.F90:71-89,
// hy_eigenValue.F90:46-50, OnlyHydro/hy_eigenVector.F90:95-152
// ---------------------------------------------------------------------------
template <class R> struct Eig {
  R lam[5];
  R cf, ahinv, a2inv, lp, rho, rp;
};

template <class R, int DIR>
__device__ __forceinline__ void eigen(const R *V, Eig<R> &e, unsigned &st) {
  constexpr int v1 = Slots<DIR>::v1;
  R un = V[v1];
  R a2 = V[HGC] * V[HP] / V[HD];
  if (a2 <= R(0)) st |= ST_NEG_SOUND;
  R cf = rsqrt_(a2);
  e.lam[0] = un - cf; e.lam[1] = un; e.lam[2] = un; e.lam[3] = un; e.lam[4] = un + cf;
  R dinv = R(1) / V[HD];
  R a2e = cf * cf;
  e.a2inv = R(1) / a2e;
  e.ahinv = R(0.5) / cf;
  R Na = R(0.5) * e.a2inv;
  e.lp = dinv * Na;
  e.rho = V[HD];
  e.rp = V[HD] * a2e;
  e.cf = cf;
}

// left eigenvector k (column k of LeftEigvec) dotted with d[0..4]
template <class R, int DIR>
__device__ __forceinline__ R ldot(const Eig<R> &e, int k, const R *d) {
  constexpr int v1 = Slots<DIR>::v1, v2 = Slots<DIR>::v2, v3 = Slots<DIR>::v3;
  switch (k) {
    case 0: return (-e.ahinv) * d[v1] + e.lp * d[HP];
    case 1: return d[v2];
    case 2: return d[HD] + (-e.a2inv) * d[HP];
    case 3: return d[v3];
    default: return e.ahinv * d[v1] + e.lp * d[HP];
  }
}

// right-eigenvector projection sum_k reig(v,k) db(k) (PPM.F90:528-570)
template <class R, int DIR>
__device__ __forceinline__ void rproject(const Eig<R> &e, const R db[5], R t[5]) {
  constexpr int v1 = Slots<DIR>::v1, v2 = Slots<DIR>::v2, v3 = Slots<DIR>::v3;
  t[HD] = e.rho * db[0] + db[2] + e.rho * db[4];
  t[v1] = (-e.cf) * db[0] + e.cf * db[4];
  t[v2] = db[1];
  t[v3] = db[3];
  t[HP] = e.rp * db[0] + e.rp * db[4];
}

// ---------------------------------------------------------------------------
// hy_TVDslope.F90:76-246; slots 5,6 (gamc, game) are never used downstream
// under FLASH_EOS_GAMMA (PPM.F90:733-736) and are not computed.
// ---------------------------------------------------------------------------
template <class R, int DIR>
__device__ __forceinline__ void tvd_slope_d(const DevParams &P, const R *dL, const R *dR, R dLe, R dRe,
                                            const Eig<R> &e, R db[8]) {
  const int lim = P.limiter;
  const R beta = R(P.lim_beta);
  if (P.char_limiting) {
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      R a = ldot<R, DIR>(e, k, dL), b = ldot<R, DIR>(e, k, dR);
      int lk = lim == 3 ? (k == 2 ? 2 : 1) : lim;
      db[k] = limit2(lk, beta, a, b);
    }
    db[HEI] = limit2(lim == 3 ? 2 : lim, beta, dLe, dRe);
    R t[5];
    rproject<R, DIR>(e, db, t);
#pragma unroll
    for (int n = 0; n < 5; ++n) db[n] = t[n];
  } else {
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      int lk = lim == 3 ? (k == HD ? 2 : 1) : lim;
      db[k] = limit2(lk, beta, dL[k], dR[k]);
    }
    db[HEI] = lim == 3 ? R(0) : limit2(lim, beta, dLe, dRe);   // hybrid: EINT is in neither case list, slope 0
  }
  db[HGC] = R(0); db[HGE] = R(0);
}

template <class R, int DIR>
__device__ __forceinline__ void tvd_slope(const DevParams &P, const R *VL, const R *V0, const R *VR,
                                          const Eig<R> &e, R db[8]) {
  R dL[5], dR[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) { dL[n] = V0[n] - VL[n]; dR[n] = VR[n] - V0[n]; }
  tvd_slope_d<R, DIR>(P, dL, dR, V0[HEI] - VL[HEI], VR[HEI] - V0[HEI], e, db);
}

// ---------------------------------------------------------------------------
// hy_upwindTransverseFlux.F90:75-207 (transOrder = 1), sparse reig terms
// ---------------------------------------------------------------------------
template <class R, int DIR>
__device__ __forceinline__ void upwind_tflux_d(const DevParams &P, const R *dl, const R *dr, R dle, R dre,
                                               const Eig<R> &e, R sig[8]) {
  constexpr int v1 = Slots<DIR>::v1, v2 = Slots<DIR>::v2, v3 = Slots<DIR>::v3;
  R dn[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) dn[n] = ldot<R, DIR>(e, n, e.lam[n] > R(0) ? dl : dr);
  const R *lam = e.lam;
  sig[HD] = (lam[0] * e.rho) * dn[0] + lam[2] * dn[2] + (lam[4] * e.rho) * dn[4];
  sig[v1] = (lam[0] * (-e.cf)) * dn[0] + (lam[4] * e.cf) * dn[4];
  sig[v2] = lam[1] * dn[1];
  sig[v3] = lam[3] * dn[3];
  sig[HP] = (lam[0] * e.rp) * dn[0] + (lam[4] * e.rp) * dn[4];
  sig[HGC] = R(0); sig[HGE] = R(0);
  sig[HEI] = P.use_aux_eint ? lam[2] * (lam[2] > R(0) ? dle : dre) : R(0);
}

// upwind differences dl = vc0 - vm1, dr = vp1 - vc0 of the three cells
template <class R, int DIR>
__device__ __forceinline__ void upwind_tflux(const DevParams &P, const R *vm1, const R *vc0, const R *vp1,
                                             const Eig<R> &e, R sig[8]) {
  R dl[5], dr[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) { dl[v] = vc0[v] - vm1[v]; dr[v] = vp1[v] - vc0[v]; }
  upwind_tflux_d<R, DIR>(P, dl, dr, vc0[HEI] - vm1[HEI], vp1[HEI] - vc0[HEI], e, sig);
}

// ---------------------------------------------------------------------------
// flattening of hy_getRiemannState.F90:356-454 for the cell at stencil
// position 3 of p[0..6] (pressures at c-3..c+3) and u[0..6] (normal vel.)
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ R flat_tilde(R pm2, R pm1, R pp1, R pp2, R um1, R up1) {
  R dp1 = (pp1 - pm1);
  R dp2 = (pp2 - pm2);
  R dv1 = up1 - um1;
  R Sp = rabs(dp2) > R(1.e-15) ? dp1 / dp2 - R(0.75) : R(0);
  R ft = rmax(R(0.0), rmin(R(1.0), R(10.0) * Sp));
  if ((rabs(dp1) / rmin(pm1, pp1) < R(1.) / R(3.)) || dv1 > R(0)) ft = R(0);
  return ft;
}
template <class R>
__device__ __forceinline__ R flat_coeff(const R *p, const R *u) {
  R t0 = flat_tilde(p[1], p[2], p[4], p[5], u[2], u[4]);
  R dp1 = (p[4] - p[2]);
  if (dp1 < R(0.0)) return rmax(t0, flat_tilde(p[2], p[3], p[5], p[6], u[3], u[5]));
  if (dp1 == R(0)) return t0;
  return rmax(t0, flat_tilde(p[0], p[1], p[3], p[4], u[1], u[3]));
}

// ---------------------------------------------------------------------------
// hy_DataReconstructNormalDir_PPM.F90:181-842 for one cell (HLL-type
// characteristic tracing).  V5: slots of c-2..c+2.  Outputs Wp (right face
// state) and Wm (left face state) for slots 0..7.
// ---------------------------------------------------------------------------
template <class R, int DIR>
__device__ __forceinline__ void ppm_cell(const DevParams &P, const R (*V5)[8], R flat, R dtn,
                                         R delta, R Wp[8], R Wm[8], unsigned &st) {
  constexpr int v1 = Slots<DIR>::v1, v2 = Slots<DIR>::v2, v3 = Slots<DIR>::v3;
  const R *Vmm = V5[0], *Vm = V5[1], *Vc = V5[2], *Vp = V5[3], *Vpp = V5[4];
  const R hdtn = R(0.5) * dtn;
  Eig<R> eN, e0, eP;
  eigen<R, DIR>(Vc, e0, st);
  eigen<R, DIR>(Vp, eP, st);
  eigen<R, DIR>(Vm, eN, st);
  R dbN[8], db0[8], dbP[8];
  tvd_slope<R, DIR>(P, Vmm, Vm, Vc, eN, dbN);
  tvd_slope<R, DIR>(P, Vm, Vc, Vp, e0, db0);
  tvd_slope<R, DIR>(P, Vc, Vp, Vpp, eP, dbP);
  const R Flattening = P.use_flattening ? flat : R(0);

  // slots reconstructed: 0..4 and EINT (7)
  constexpr int NS = 6;
  const int sl[NS] = {0, 1, 2, 3, 4, 7};
  R vecL[8], vecR[8];
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    int n = sl[q];
    vecL[n] = R(0.5) * (Vc[n] + Vm[n]) - (db0[n] - dbN[n]) / R(6.);
    vecR[n] = R(0.5) * (Vc[n] + Vp[n]) - (dbP[n] - db0[n]) / R(6.);
  }
  if (P.use_steepening) {                                     // PPM.F90:639-670
    const R eta1 = R(20.E0), eta2 = R(0.05E0), epsln = R(0.01E0), K0 = R(0.1E0);
    R temp1 = Vp[HD] - Vm[HD];
    if (rabs(temp1) > R(P.tiny)) {
      R del2rhoR = (Vpp[HD] - R(2.) * Vp[HD] + Vc[HD]) / (R(6.) * delta * delta);
      R del2rhoL = (Vc[HD] - R(2.) * Vm[HD] + Vmm[HD]) / (R(6.) * delta * delta);
      R eta_steep = (del2rhoL - del2rhoR) * (delta * delta) / temp1;
      if (del2rhoR * del2rhoL >= R(0)) eta_steep = R(0);
      if (epsln * rmin(Vp[HD], Vm[HD]) - rabs(Vp[HD] - Vm[HD]) >= R(0)) eta_steep = R(0);
      eta_steep = rmax(R(0), rmin(R(1), eta1 * (eta_steep - eta2)));
      R temp2 = rabs(Vp[HP] - Vm[HP]) / rmin(Vp[HP], Vm[HP]);
      R temp3 = rabs(Vp[HD] - Vm[HD]) / rmin(Vp[HD], Vm[HD]);
      if (Vc[HGE] * K0 * temp3 - temp2 < R(0.0)) eta_steep = R(0);
      vecL[HD] = vecL[HD] * (R(1) - eta_steep) + (Vm[HD] + R(0.5) * dbN[HD]) * eta_steep;
      vecR[HD] = vecR[HD] * (R(1) - eta_steep) + (Vp[HD] - R(0.5) * dbP[HD]) * eta_steep;
    }
  }
  if (P.use_flattening) {                                     // PPM.F90:676-679
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      int n = sl[q];
      vecL[n] = Flattening * Vc[n] + (R(1.0) - Flattening) * vecL[n];
      vecR[n] = Flattening * Vc[n] + (R(1.0) - Flattening) * vecR[n];
    }
  }
  R delW[8], W6[8];
#pragma unroll
  for (int q = 0; q < NS; ++q) {                               // PPM.F90:686-706
    int n = sl[q];
    if ((vecR[n] - Vc[n]) * (Vc[n] - vecL[n]) <= R(0)) { vecL[n] = Vc[n]; vecR[n] = Vc[n]; }
    if (R(6.) * (vecR[n] - vecL[n]) * (Vc[n] - R(0.5) * (vecL[n] + vecR[n])) > (vecR[n] - vecL[n]) * (vecR[n] - vecL[n]))
      vecL[n] = R(3.) * Vc[n] - R(2.) * vecR[n];
    if (R(6.) * (vecR[n] - vecL[n]) * (Vc[n] - R(0.5) * (vecL[n] + vecR[n])) < -((vecR[n] - vecL[n]) * (vecR[n] - vecL[n])))
      vecR[n] = R(3.) * Vc[n] - R(2.) * vecL[n];
    delW[n] = vecR[n] - vecL[n];
    W6[n] = R(6.) * (Vc[n] - R(0.5) * (vecR[n] + vecL[n]));
  }
  // EINT: entropy-wave traced initial guess (PPM.F90:715-727)
  {
    R lmax = rmax(e0.lam[2], R(0));
    Wp[HEI] = vecR[HEI] - lmax * hdtn * (delW[HEI] - (R(1.0) - lmax * hdtn * R(4.) / R(3.)) * W6[HEI]);
    R lmin = -rmin(e0.lam[2], R(0));
    Wm[HEI] = vecL[HEI] + lmin * hdtn * (delW[HEI] + (R(1.0) - lmin * hdtn * R(4.) / R(3.)) * W6[HEI]);
  }
  // characteristic tracing, all waves into both sides (PPM.F90:753-800)
  R mW6[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) mW6[n] = -W6[n];
  R sigL[5], sigR[5];
  const R f43 = R(4.) / R(3.);
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    R cA = ldot<R, DIR>(e0, n, delW);
    R cB = ldot<R, DIR>(e0, n, mW6);
    R lam = e0.lam[n];
    R x = dtn * lam;
    R AL = R(.5) * (R(-1.) - dtn * lam);
    R BL = R(.25) * (R(1.) + R(2.) * dtn * lam + f43 * (x * x));
    R AR = R(.5) * (R(1.) - dtn * lam);
    R BR = R(.25) * (R(1.) - R(2.) * dtn * lam + f43 * (x * x));
    // non-zero entries of column n of RightEigvec
    if (n == 0 || n == 4) {
      R rv = n == 0 ? -e0.cf : e0.cf;
      R tL_d = AL * e0.rho * cA + BL * e0.rho * cB, tR_d = AR * e0.rho * cA + BR * e0.rho * cB;
      R tL_v = AL * rv * cA + BL * rv * cB, tR_v = AR * rv * cA + BR * rv * cB;
      R tL_p = AL * e0.rp * cA + BL * e0.rp * cB, tR_p = AR * e0.rp * cA + BR * e0.rp * cB;
      if (n == 0) {
        sigL[HD] = tL_d; sigR[HD] = tR_d; sigL[v1] = tL_v; sigR[v1] = tR_v; sigL[HP] = tL_p; sigR[HP] = tR_p;
      } else {
        sigL[HD] = sigL[HD] + tL_d; sigR[HD] = sigR[HD] + tR_d;
        sigL[v1] = sigL[v1] + tL_v; sigR[v1] = sigR[v1] + tR_v;
        sigL[HP] = sigL[HP] + tL_p; sigR[HP] = sigR[HP] + tR_p;
      }
    } else {
      R tL = AL * cA + BL * cB, tR = AR * cA + BR * cB;       // reig entry 1
      if (n == 1) { sigL[v2] = tL; sigR[v2] = tR; }
      else if (n == 2) { sigL[HD] = sigL[HD] + tL; sigR[HD] = sigR[HD] + tR; }
      else { sigL[v3] = tL; sigR[v3] = tR; }
    }
  }
#pragma unroll
  for (int n = 0; n < 5; ++n) {                               // PPM.F90:841-842
    Wm[n] = Vc[n] + W6[n] / R(12.) + sigL[n];
    Wp[n] = Vc[n] + W6[n] / R(12.) + sigR[n];
  }
  Wp[HGC] = Vc[HGC]; Wp[HGE] = Vc[HGE];
  Wm[HGC] = Vc[HGC]; Wm[HGE] = Vc[HGE];
}

// ---------------------------------------------------------------------------
// hy_prim2con.F90:37-54, hy_prim2flx.F90:49-123, hy_HLLC.F90:94-311
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ void prim2con(const R *V, R CU[5]) {
  R u2 = V[HVX] * V[HVX] + V[HVY] * V[HVY] + V[HVZ] * V[HVZ];
  CU[0] = V[HD];
  CU[1] = V[HD] * V[HVX]; CU[2] = V[HD] * V[HVY]; CU[3] = V[HD] * V[HVZ];
  CU[4] = R(0.5) * V[HD] * u2 + V[HP] / (V[HGE] - R(1.)) + R(0.5) * R(0.);
}
template <class R, int DIR>
__device__ __forceinline__ void prim2flx(const R *V, R F[6]) {
  constexpr int v1 = Slots<DIR>::v1;
  R u2 = V[HVX] * V[HVX] + V[HVY] * V[HVY] + V[HVZ] * V[HVZ];
  R E = R(0.5) * V[HD] * u2 + V[HP] / (V[HGE] - R(1.));
  F[5] = V[HP];
  F[0] = V[HD] * V[v1];
  F[1] = F[0] * V[HVX];
  F[2] = F[0] * V[HVY];
  F[3] = F[0] * V[HVZ];
  F[DIR] = F[DIR] + R(1.0) * V[HP];            // hy_fPresInMomFlux = 1
  F[4] = (E + V[HP]) * V[v1];
}
template <class R, int DIR>
__device__ __forceinline__ void hllc(const DevParams &P, const R *Vm, const R *Vp, R Fs[6], unsigned &st) {
  constexpr int v1 = Slots<DIR>::v1;
  const R tiny = R(P.tiny);
  R velNL = Vm[v1], velNR = Vp[v1];
  R aL2 = Vm[HGC] * Vm[HP] / Vm[HD];
  R aR2 = Vp[HGC] * Vp[HP] / Vp[HD];
  if ((Vm[HD] < tiny && Vm[HD] > R(0)) || (Vp[HD] < tiny && Vp[HD] > R(0)) ||
      (Vm[HP] < tiny && Vm[HP] > R(0)) || (Vp[HP] < tiny && Vp[HP] > R(0))) {
#pragma unroll
    for (int n = 0; n < 6; ++n) Fs[n] = R(0);
    return;
  }
  if (aL2 < R(0) || aR2 < R(0)) {
    st |= ST_NEG_SOUND;
#pragma unroll
    for (int n = 0; n < 6; ++n) Fs[n] = R(0);
    return;
  }
  R cfL = rsqrt_(aL2), cfR = rsqrt_(aR2);
  R SL = rmin(velNL - cfL, velNR - cfR);
  R SR = rmax(velNL + cfL, velNR + cfR);
  R pL = Vm[HP], pR = Vp[HP];
  R UL[5], UR[5], FL[6], FR[6];
  prim2con(Vm, UL); prim2con(Vp, UR);
  prim2flx<R, DIR>(Vm, FL); prim2flx<R, DIR>(Vp, FR);
  R qStar = (Vp[HD] * velNR * (SR - velNR) - Vm[HD] * velNL * (SL - velNL) + pL - pR - R(0.) * R(0.) + R(0.) * R(0.));
  qStar = qStar / (Vp[HD] * (SR - velNR) - Vm[HD] * (SL - velNL));
  R numerL = SL - velNL, denomL = SL - qStar;
  R numerR = SR - velNR, denomR = SR - qStar;
  R pStar = Vm[HD] * numerL * (qStar - velNL) + pL;
  if (SL >= R(0)) {
#pragma unroll
    for (int n = 0; n < 6; ++n) Fs[n] = FL[n];
  } else if ((SL < R(0)) && (qStar >= R(0))) {
    R dStarL = UL[0] * numerL / denomL;
    R UC[5];
    UC[0] = dStarL;
    UC[4] = UL[4] * numerL / denomL + ((pStar * qStar - pL * velNL)) / denomL;
#pragma unroll
    for (int m = 1; m <= 3; ++m) UC[m] = (m == DIR) ? dStarL * qStar : UL[m] * numerL / denomL;
#pragma unroll
    for (int n = 0; n < 5; ++n) Fs[n] = FL[n] + SL * (UC[n] - UL[n]);
    Fs[5] = FL[5];
  } else if ((qStar < R(0)) && (SR >= R(0))) {
    R dStarR = UR[0] * numerR / denomR;
    R UC[5];
    UC[0] = dStarR;
    UC[4] = UR[4] * numerR / denomR + ((pStar * qStar - pR * velNR)) / denomR;
#pragma unroll
    for (int m = 1; m <= 3; ++m) UC[m] = (m == DIR) ? dStarR * qStar : UR[m] * numerR / denomR;
#pragma unroll
    for (int n = 0; n < 5; ++n) Fs[n] = FR[n] + SR * (UC[n] - UR[n]);
    Fs[5] = FR[5];
  } else {
#pragma unroll
    for (int n = 0; n < 6; ++n) Fs[n] = FR[n];
  }
}

}  // namespace fhy
