// exact_rs.cuh -- exact ideal-gas Riemann solver and the learned initial
// guess for its star pressure, shared by the isolated solver
// (riemann_exact.cu) and the hydro face fluxes (hy_kernels.cuh,
// hy_mixed.cuh).  FLASH5 has no exact solver on the unsplit path
// (hy_getFaceFlux.F90:324-372 dispatches Roe/HLL/HLLC/Marquina/LLF only).
//
// Method: E. F. Toro, "Riemann Solvers and Numerical Methods for Fluid
// Dynamics", 3rd ed., ch. 4 -- pressure functions f_K(p) (eqs. 4.6-4.7),
// two-rarefaction guess (eq. 4.46), Newton iteration on
// f(p) = f_L(p) + f_R(p) + (u_R - u_L) = 0, sampling of the self-similar
// solution at x/t = 0 (section 4.5) and the vacuum-generating case
// (section 4.6).  f is increasing and concave, so Newton from any point
// lands at or left of the root and then climbs monotonically; the iterate
// is still kept inside the bracket [pa, pb] built from the evaluated signs,
// so every solve terminates within max_iter.
//
// The learned guess is an 8-64-64-1 MLP with BF16 weights and activations
// and FP32 accumulation, evaluated with warp-level tensor-core mma.sync
// (m16n8k16) over the 32 interfaces of a warp.  It predicts ln(p*/p_TR)
// from eight scale-free features; Newton starts from p_TR*exp(y).
#pragma once
#include <cuda_bf16.h>
#include <float.h>
#include <stdint.h>

namespace xrs {

constexpr int NIN = 8, NH = 64;
// FP32 master parameter layout: W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NIN, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NH, NPARAM = OFF_B3 + 1;

// inference copy of the network: BF16 matrices in mma fragment order-ready
// row layout (W1 with K padded 8 -> 16), FP32 vectors; 16-byte multiple
struct MlpPacked {
  __nv_bfloat16 W1[NH][16];
  __nv_bfloat16 W2[NH][NH];
  float b1[NH], b2[NH], w3[NH];
  float b3, pad[3];
};
static_assert(sizeof(MlpPacked) % 16 == 0, "MlpPacked must be a multiple of 16 bytes");

// ---------------------------------------------------------------------------
// pressure functions, guess, Newton, star velocity
//
// Newton runs on w = p^z, z = (g-1)/(2g), not on p.  In w the rarefaction
// branch of f_K (Toro eq. 4.7) is linear, f_K = 2 c_K/(g-1) (w/w_K - 1), so
// the two-rarefaction guess (eq. 4.46) is the root of the linear part and
// the exact root where both waves are rarefactions.  For g <= 5/3 the
// shock branch (eq. 4.6) is convex in w, so Newton from the two-rarefaction
// guess, which lies at or right of the root, descends monotonically; for
// stiffer gases it is not convex near w_K and the bracket safeguards carry
// the iteration.  p = w^(1/z) with 1/z = 2 + 2/(g-1) is an integer power
// for g = 5/3, 7/5, 4/3, so the iteration needs no transcendental function
// there; w_K = p_K^z is taken once per side.
// ---------------------------------------------------------------------------
struct Side { double d, u, p, c, w; };              // w = p^z

// x^y for x > 0 as exp2(y log2 x): the relative error is a few ulp times
// |y log2 x|, far below the solver's tolerance, at a fraction of the cost
// of the correctly rounded FP64 pow
__device__ __forceinline__ double powp(double x, double y) { return exp2(y * log2(x)); }

// x^k by binary powering when k is an integer in [1, 16], else powp
__device__ __forceinline__ double pow_k(double x, double k) {
  const double kn = rint(k);
  if (fabs(k - kn) < 1e-9 && kn >= 1.0 && kn <= 16.0) {
    int e = (int)kn;
    double r = 1.0, b = x;
    while (e) {
      if (e & 1) r *= b;
      e >>= 1;
      if (e) b *= b;
    }
    return r;
  }
  return powp(x, k);
}

__host__ __device__ __forceinline__ double zexp(double g) { return (g - 1.0) / (2.0 * g); }

// p = w^n, n = 1/z = 2g/(g-1): unrolled for the integer exponents of
// g = 5/3, 7/5, 4/3 (5, 7, 8), else pow_k
struct PowN { int ni; double n; };
__host__ __device__ __forceinline__ PowN pown_of(double g) {
  const double n = 2.0 * g / (g - 1.0), r = rint(n);
  return PowN{(fabs(n - r) < 1e-9 && (r == 5.0 || r == 7.0 || r == 8.0)) ? (int)r : 0, n};
}
__device__ __forceinline__ double pow_n(double w, const PowN &e) {
  if (e.ni == 5) { const double w2 = w * w; return w2 * w2 * w; }
  if (e.ni == 7) { const double w2 = w * w, w4 = w2 * w2; return w4 * w2 * w; }
  if (e.ni == 8) { const double w2 = w * w, w4 = w2 * w2; return w4 * w4; }
  return pow_k(w, e.n);
}
// p = w^n and dp/dw = n w^(n-1), the latter from the same powers for the
// integer exponents (no division)
__device__ __forceinline__ double pow_n_d(double w, const PowN &e, double &dpdw) {
  if (e.ni == 5) { const double w2 = w * w, w4 = w2 * w2; dpdw = 5.0 * w4; return w4 * w; }
  if (e.ni == 7) { const double w2 = w * w, w6 = w2 * w2 * w2; dpdw = 7.0 * w6; return w6 * w; }
  if (e.ni == 8) { const double w2 = w * w, w4 = w2 * w2, w7 = w4 * w2 * w; dpdw = 8.0 * w7; return w7 * w; }
  const double p = pow_k(w, e.n);
  dpdw = e.n * p / w;
  return p;
}

// Constants of the gas, taken once per context on the host where the
// adiabatic index is uniform (the hydro kernels read them from their
// parameter block) and per solve in the isolated solver: z = (g-1)/(2g), p = w^n, and
// the coefficients of the pressure functions (Toro eqs. 4.6-4.7), the
// two-rarefaction guess and the sampling (section 4.5).
struct Gas {
  double g, z, gm1inv, k2, a2, g6, g2, hgm1;   // 1/(g-1), 2/(g-1), 2/(g+1), (g-1)/(g+1), (g+1)/(2g), (g-1)/2
  PowN e;
};
__host__ __device__ __forceinline__ Gas gas_of(double g) {
  Gas s;
  s.g = g;
  s.z = zexp(g);
  s.gm1inv = 1.0 / (g - 1.0);
  s.k2 = 2.0 / (g - 1.0);
  s.a2 = 2.0 / (g + 1.0);
  s.g6 = (g - 1.0) / (g + 1.0);
  s.g2 = (g + 1.0) / (2.0 * g);
  s.hgm1 = 0.5 * (g - 1.0);
  s.e = pown_of(g);
  return s;
}

__device__ __forceinline__ double p_of_w(double w, const Gas &G) { return pow_n(w, G.e); }
__device__ __forceinline__ Side make_side(double d, double u, double p, double c, const Gas &G) {
  return Side{d, u, p, c, powp(p, G.z)};
}

// Constants of one side's pressure function, taken once per solve: w_K,
// p_K, the rarefaction slope k = 2 c_K / ((g-1) w_K) and A_K, B_K of the
// shock branch.
struct SideK { double w, p, k, A, B; };
__device__ __forceinline__ SideK side_k(const Side &s, const Gas &G) {
  return SideK{s.w, s.p, G.k2 * s.c / s.w, G.a2 / s.d, G.g6 * s.p};
}

// f_K(w) and df_K/dw (Toro eqs. 4.6-4.7 with p = w^n, dp/dw = dpdw)
__device__ __forceinline__ void pres_fn(double w, double p, double dpdw, const SideK &s, double &f, double &fd) {
  if (w <= s.w) {                                   // rarefaction, Toro eq. 4.7
    f = s.k * (w - s.w);
    fd = s.k;
  } else {                                          // shock, Toro eq. 4.6
    const double r = 1.0 / (s.B + p);
    const double q = sqrt(s.A * r);
    f = (p - s.p) * q;
    fd = (1.0 - 0.5 * (p - s.p) * r) * q * dpdw;    // df/dp dp/dw
  }
}

// two-rarefaction guess in w (0 where the states generate vacuum), Toro
// eq. 4.46 with c_K/w_K = k_K (g-1)/2 from the sides' rarefaction slopes
__device__ __forceinline__ double tr_w(const Side &L, const Side &R, const SideK &kl, const SideK &kr, const Gas &G) {
  const double num = L.c + R.c - G.hgm1 * (R.u - L.u);
  return num > 0.0 ? num / (G.hgm1 * (kl.k + kr.k)) : 0.0;
}
__device__ __forceinline__ double tr_w(const Side &L, const Side &R, const Gas &G) {
  return tr_w(L, R, side_k(L, G), side_k(R, G), G);
}
__device__ __forceinline__ double tr_guess(const Side &L, const Side &R, const Gas &G) {
  return p_of_w(tr_w(L, R, G), G);
}

// vacuum generation test, Toro eq. 4.40
__device__ __forceinline__ bool vacuum(const Side &L, const Side &R, const Gas &G) {
  return G.k2 * (L.c + R.c) <= R.u - L.u;
}

// The two-rarefaction guess is the exact root when it does not exceed
// min(p_L, p_R) (both waves are rarefactions, Toro section 4.3.2).
__device__ __forceinline__ bool tr_exact(const Side &L, const Side &R, double ptr) { return ptr <= fmin(L.p, R.p); }

// Strong waves: the pressure range spanned by p_L, p_R and the PVRS
// estimate ppv covers a factor of two or more, and ppv lies above
// min(p_L, p_R).  Elsewhere the waves are weak or both are rarefactions
// (ppv <= pmin; Toro section 9.5.1), and Newton from the two-rarefaction
// guess converges in one to three evaluations: the network is consulted
// only for strong waves.
__device__ __forceinline__ bool strong_waves(const Side &L, const Side &R) {
  const double pmin = fmin(L.p, R.p), pmax = fmax(L.p, R.p);
  const double ppv = 0.5 * (L.p + R.p) - 0.125 * (R.u - L.u) * (L.d + R.d) * (L.c + R.c);
  return ppv > pmin && fmax(pmax, ppv) >= 2.0 * pmin;
}

// A single-precision screen for strong_waves on raw face states: true
// whenever the FP64 test can be true, so that the FP64 test (with the full
// sides) runs only on the faces that pass.  The comparisons carry margins of
// 1e-5 relative, and the PVRS estimate a margin of 1e-5 of the magnitude of
// its two terms (FP32 rounding of the handful of operations, cancellation
// included, stays below 1e-6 of it); NaN, infinities and values outside
// [1e-30, 1e30] pass, leaving the decision to the FP64 test.
__device__ __forceinline__ bool strong_screen(double dl, double ul, double pl, double dr, double ur, double pr,
                                              double g) {
  const float fdl = (float)dl, fpl = (float)pl, fdr = (float)dr, fpr = (float)pr, fg = (float)g;
  const float cl = sqrtf(fg * fpl / fdl), cr = sqrtf(fg * fpr / fdr);
  const float pa = 0.5f * (fpl + fpr), corr = 0.125f * ((float)ur - (float)ul) * (fdl + fdr) * (cl + cr);
  const float ppv = pa - corr, E = 1e-5f * (fabsf(pa) + fabsf(corr));
  const float pmin = fminf(fpl, fpr), pmax = fmaxf(fpl, fpr);
  if (!(pmin > 1e-30f && pmax < 1e30f && fminf(fdl, fdr) > 1e-30f && fmaxf(fdl, fdr) < 1e30f &&
        fabsf(ppv) < 1e30f && E < 1e30f))
    return true;
  return ppv + E > pmin * (1.f - 1e-5f) && fmaxf(pmax * (1.f + 1e-5f), ppv + E) >= 2.f * pmin * (1.f - 1e-5f);
}

// The star state of a solve: p*, u* and w* = p*^z (the sampling takes the
// rarefaction-side powers (p*/p_K)^z = w*/w_K from it).
struct Star { double p, u, w; };

// Newton on f(w) = f_L + f_R + (u_R - u_L) from w0 >= 0.  Converged when
// the step is below tol * z * w (a relative step of tol in p); once the
// last two steps show the quadratic regime, when the predicted next step
// |step|^3 / prev^2 is below a hundredth of that; or when the bracket
// [wa, wb] of evaluated signs is that narrow (near vacuum, where the
// rounding of f exceeds the tolerance on the step; the root is its
// midpoint).  A step that leaves the bracket is replaced by its midpoint
// (or a doubling while no upper end is known).  u* is f_L, f_R linearised
// from the last evaluation to the returned w*.  Returns the number of
// evaluations, or -max_iter when not converged.
__device__ __forceinline__ int newton(const Side &L, const Side &R, const SideK &kl, const SideK &kr, const Gas &G,
                                      double w0, double tol, int max_iter, Star &out) {
  const double du = R.u - L.u, ztol = G.z * tol;
  const PowN &e = G.e;
  double wa = 0.0, wb = DBL_MAX;
  double w = w0, prev = -1.0, p = 0.0;
  double fl = 0., fdl = 0., fr = 0., fdr = 0., we = w0;
  int evals = 0;
  for (; evals < max_iter;) {
    double dpdw;
    p = pow_n_d(w, e, dpdw);
    pres_fn(w, p, dpdw, kl, fl, fdl);
    pres_fn(w, p, dpdw, kr, fr, fdr);
    ++evals;
    we = w;
    const double f = fl + fr + du;
    if (f == 0.0) {
      out.w = w; out.p = p;
      out.u = 0.5 * (L.u + R.u) + 0.5 * (fr - fl);
      return evals;
    }
    if (f < 0.0) wa = w; else wb = w;
    if (wb - wa <= ztol * w) {
      out.w = 0.5 * (wa + wb);
      out.p = pow_n(out.w, e);
      const double dw = out.w - we;
      out.u = 0.5 * (L.u + R.u) + 0.5 * ((fr + fdr * dw) - (fl + fdl * dw));
      return evals;
    }
    const double step = f / (fdl + fdr);
    double wn = w - step;
    const double as = fabs(step);
    const bool inside = wn > wa && wn < wb;
    if (as <= ztol * w || (inside && prev > 0.0 && as < prev && as * (as / prev) * (as / prev) <= 0.01 * ztol * w)) {
      out.w = wn > 0.0 ? wn : w;
      out.p = pow_n(out.w, e);
      const double dw = out.w - we;
      out.u = 0.5 * (L.u + R.u) + 0.5 * ((fr + fdr * dw) - (fl + fdl * dw));
      return evals;
    }
    if (!inside) {
      wn = wb == DBL_MAX ? 2.0 * w : 0.5 * (wa + wb);
      prev = -1.0;
    } else {
      prev = as;
    }
    w = wn;
  }
  out.w = w; out.p = pow_n(w, e);
  const double dw = w - we;
  out.u = 0.5 * (L.u + R.u) + 0.5 * ((fr + fdr * dw) - (fl + fdl * dw));
  return -max_iter;
}

// ---------------------------------------------------------------------------
// the exact solution at x/t = 0 (Toro 4.5; vacuum generation 4.6)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void fan_left(const Side &L, const Gas &G, double &d, double &u, double &p) {
  const double c = G.a2 * (L.c + G.hgm1 * L.u);
  u = c;
  const double r = c / L.c;
  d = L.d * pow_k(r, G.k2);
  p = L.p * pow_n(r, G.e);
}
__device__ __forceinline__ void fan_right(const Side &R, const Gas &G, double &d, double &u, double &p) {
  const double c = G.a2 * (R.c - G.hgm1 * R.u);
  u = -c;
  const double r = c / R.c;
  d = R.d * pow_k(r, G.k2);
  p = R.p * pow_n(r, G.e);
}

// (d, u, p) at x/t = 0 and which side supplies the transverse velocities;
// behind a rarefaction (p*/p_K)^z = w*/w_K and rho*_K = rho_K (w*/w_K)^(2/(g-1))
__device__ __forceinline__ void sample0(const Side &L, const Side &R, const Gas &G, const Star &S, bool vac,
                                        double &d, double &u, double &p, bool &right) {
  if (vac) {
    const double sl = L.u + G.k2 * L.c, sr = R.u - G.k2 * R.c;
    if (0.0 <= L.u - L.c) { right = false; d = L.d; u = L.u; p = L.p; }
    else if (0.0 < sl) { right = false; fan_left(L, G, d, u, p); }
    else if (0.0 >= R.u + R.c) { right = true; d = R.d; u = R.u; p = R.p; }
    else if (0.0 > sr) { right = true; fan_right(R, G, d, u, p); }
    else { right = false; d = 0.0; u = 0.0; p = 0.0; }
    return;
  }
  const double ps = S.p, us = S.u;
  const double g1 = G.z, g2 = G.g2, g6 = G.g6, k = G.k2;
  if (0.0 <= us) {                                   // left of the contact
    right = false;
    if (ps > L.p) {                                  // left shock
      const double pr = ps / L.p;
      const double sl = L.u - L.c * sqrt(g2 * pr + g1);
      if (0.0 <= sl) { d = L.d; u = L.u; p = L.p; }
      else { d = L.d * (pr + g6) / (pr * g6 + 1.0); u = us; p = ps; }
    } else {                                         // left rarefaction
      if (0.0 <= L.u - L.c) { d = L.d; u = L.u; p = L.p; }
      else {
        const double q = S.w / L.w;
        const double cml = L.c * q;
        if (0.0 > us - cml) { d = L.d * pow_k(q, k); u = us; p = ps; }
        else fan_left(L, G, d, u, p);
      }
    }
  } else {                                           // right of the contact
    right = true;
    if (ps > R.p) {
      const double pr = ps / R.p;
      const double sr = R.u + R.c * sqrt(g2 * pr + g1);
      if (0.0 >= sr) { d = R.d; u = R.u; p = R.p; }
      else { d = R.d * (pr + g6) / (pr * g6 + 1.0); u = us; p = ps; }
    } else {
      if (0.0 >= R.u + R.c) { d = R.d; u = R.u; p = R.p; }
      else {
        const double q = S.w / R.w;
        const double cmr = R.c * q;
        if (0.0 <= us + cmr) { d = R.d * pow_k(q, k); u = us; p = ps; }
        else fan_right(R, G, d, u, p);
      }
    }
  }
}

// Godunov flux of the exact solution in the 6-slot layout of the HLLC
// solver (mass, three momenta, energy, pressure).  VL, VR are primitive
// states in the slot order dens, velx, vely, velz, pres, ...; DIR is the
// normal direction (1..3).
template <int DIR>
__device__ __forceinline__ void godunov_flux(const double *VL, const double *VR, const Side &L, const Side &R,
                                             const Gas &G, const Star &S, bool vac, double F[6]) {
  double d, u, p;
  bool right;
  sample0(L, R, G, S, vac, d, u, p, right);
  double v[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) v[m] = (m == DIR - 1) ? u : (right ? VR[1 + m] : VL[1 + m]);
  const double E = p * G.gm1inv + 0.5 * d * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  F[0] = d * u;
  F[1] = F[0] * v[0]; F[2] = F[0] * v[1]; F[3] = F[0] * v[2];
  F[DIR] += p;
  F[4] = (E + p) * u;
  F[5] = p;
}

// ---------------------------------------------------------------------------
// features (scale free, ~O(1)), computed in FP32; target = ln(p*/p_TR)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void features(const Side &L, const Side &R, double g, double ptr, float f[NIN]) {
  const float i4 = 1.0f / 9.2103404f, i3 = 1.0f / 6.9077553f;   // 1/ln(1e4), 1/ln(1e3)
  const float dl = float(L.d), dr = float(R.d), pl = float(L.p), pr = float(R.p);
  const float ul = float(L.u), ur = float(R.u), cl = float(L.c), cr = float(R.c), gf = float(g);
  const float du = ur - ul;
  // two-shock estimate (Toro eq. 4.47) around the PVRS pressure
  float ppv = fmaxf(0.5f * (pl + pr) - 0.125f * du * (dl + dr) * (cl + cr), 1e-6f * fminf(pl, pr));
  float gL = sqrtf(2.0f / ((gf + 1.0f) * dl) / (ppv + (gf - 1.0f) / (gf + 1.0f) * pl));
  float gR = sqrtf(2.0f / ((gf + 1.0f) * dr) / (ppv + (gf - 1.0f) / (gf + 1.0f) * pr));
  float pts = fmaxf((gL * pl + gR * pr - du) / (gL + gR), 1e-30f);
  float ptrf = float(ptr);
  f[0] = logf(pr / pl) * i4;
  f[1] = logf(dr / dl) * i3;
  f[2] = ul / cl * 0.2f;
  f[3] = ur / cr * 0.2f;
  f[4] = (gf - 1.5333333f) * 7.5f;
  f[5] = du / (cl + cr);
  f[6] = logf(ptrf / pl) * i4;
  f[7] = logf(pts / ptrf) * i4;
}

// ---------------------------------------------------------------------------
// tensor-core MLP inference for the 32 interfaces of a warp
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ uint32_t pick4(int q, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  return q == 0 ? a : (q == 1 ? b : (q == 2 ? c : d));
}

// y = MLP(f) for the interface of this lane.  All 32 lanes of the warp must
// call it together (inactive lanes pass any finite features).  Row m of the
// warp's 32 x 8 feature matrix is lane m's f; the A fragments of layer 1
// are gathered with shuffles, the layer-1 C fragments are reused as the
// layer-2 A fragments, layer 3 runs on the CUDA cores.
__device__ __forceinline__ float mlp_lane(const MlpPacked &M, const float f[NIN]) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, r = lane >> 2, q = lane & 3;
  const uint32_t w0 = pack_bf16(f[0], f[1]), w1 = pack_bf16(f[2], f[3]), w2 = pack_bf16(f[4], f[5]),
                 w3 = pack_bf16(f[6], f[7]);
  float yme = 0.f;
#pragma unroll
  for (int tile = 0; tile < 2; ++tile) {
    const int s0 = tile * 16 + r, s1 = s0 + 8;
    uint32_t a[4];
    {
      uint32_t x0 = __shfl_sync(FULL, w0, s0), x1 = __shfl_sync(FULL, w1, s0);
      uint32_t x2 = __shfl_sync(FULL, w2, s0), x3 = __shfl_sync(FULL, w3, s0);
      a[0] = pick4(q, x0, x1, x2, x3);
      x0 = __shfl_sync(FULL, w0, s1); x1 = __shfl_sync(FULL, w1, s1);
      x2 = __shfl_sync(FULL, w2, s1); x3 = __shfl_sync(FULL, w3, s1);
      a[1] = pick4(q, x0, x1, x2, x3);
      a[2] = 0u; a[3] = 0u;                       // K columns 8..15 are padding
    }
    // layer 1: [16 x 16] x [16 x 64], bias + relu
    float h1[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      uint32_t bb[2];
      bb[0] = *reinterpret_cast<const uint32_t *>(&M.W1[nt * 8 + r][2 * q]);
      bb[1] = *reinterpret_cast<const uint32_t *>(&M.W1[nt * 8 + r][2 * q + 8]);
      h1[nt][0] = h1[nt][1] = h1[nt][2] = h1[nt][3] = 0.f;
      mma_bf16(h1[nt], a, bb);
      const float c0 = M.b1[nt * 8 + 2 * q], c1 = M.b1[nt * 8 + 2 * q + 1];
      h1[nt][0] = fmaxf(h1[nt][0] + c0, 0.f); h1[nt][1] = fmaxf(h1[nt][1] + c1, 0.f);
      h1[nt][2] = fmaxf(h1[nt][2] + c0, 0.f); h1[nt][3] = fmaxf(h1[nt][3] + c1, 0.f);
    }
    // layer 2: [16 x 64] x [64 x 64]; k-step kk takes layer-1 n-tiles 2kk, 2kk+1
    float h2[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) h2[nt][0] = h2[nt][1] = h2[nt][2] = h2[nt][3] = 0.f;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      uint32_t a2[4];
      a2[0] = pack_bf16(h1[2 * kk][0], h1[2 * kk][1]);
      a2[1] = pack_bf16(h1[2 * kk][2], h1[2 * kk][3]);
      a2[2] = pack_bf16(h1[2 * kk + 1][0], h1[2 * kk + 1][1]);
      a2[3] = pack_bf16(h1[2 * kk + 1][2], h1[2 * kk + 1][3]);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        uint32_t bb[2];
        bb[0] = *reinterpret_cast<const uint32_t *>(&M.W2[nt * 8 + r][kk * 16 + 2 * q]);
        bb[1] = *reinterpret_cast<const uint32_t *>(&M.W2[nt * 8 + r][kk * 16 + 2 * q + 8]);
        mma_bf16(h2[nt], a2, bb);
      }
    }
    // layer 3: y = bf16(relu(h2 + b2)) . w3 + b3
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = nt * 8 + 2 * q;
      float v0 = __bfloat162float(__float2bfloat16(fmaxf(h2[nt][0] + M.b2[c], 0.f)));
      float v1 = __bfloat162float(__float2bfloat16(fmaxf(h2[nt][1] + M.b2[c + 1], 0.f)));
      float v2 = __bfloat162float(__float2bfloat16(fmaxf(h2[nt][2] + M.b2[c], 0.f)));
      float v3 = __bfloat162float(__float2bfloat16(fmaxf(h2[nt][3] + M.b2[c + 1], 0.f)));
      y0 += v0 * M.w3[c] + v1 * M.w3[c + 1];
      y1 += v2 * M.w3[c] + v3 * M.w3[c + 1];
    }
    y0 += __shfl_xor_sync(FULL, y0, 1); y0 += __shfl_xor_sync(FULL, y0, 2);
    y1 += __shfl_xor_sync(FULL, y1, 1); y1 += __shfl_xor_sync(FULL, y1, 2);
    // row m of this tile sits in the quad of lane 4 * (m & 7), in y0 (m < 8) or y1
    const float t0 = __shfl_sync(FULL, y0, 4 * (lane & 7)), t1 = __shfl_sync(FULL, y1, 4 * (lane & 7));
    if ((lane >> 4) == tile) yme = (lane & 8) ? t1 : t0;
  }
  return yme + M.b3;
}

// cooperative copy of the packed network into shared memory (caller syncs)
__device__ __forceinline__ void load_packed(MlpPacked &dst, const MlpPacked *__restrict__ src) {
  const int4 *s = reinterpret_cast<const int4 *>(src);
  int4 *d = reinterpret_cast<int4 *>(&dst);
  for (int t = threadIdx.x; t < (int)(sizeof(MlpPacked) / 16); t += blockDim.x) d[t] = s[t];
}

// FP32 master parameters -> inference copy (launch with one CTA)
static __global__ void k_pack_mlp(const float *__restrict__ w, MlpPacked *__restrict__ out) {
  for (int t = threadIdx.x; t < NH * 16; t += blockDim.x) {
    const int n = t / 16, k = t % 16;
    out->W1[n][k] = __float2bfloat16(k < NIN ? w[OFF_W1 + n * NIN + k] : 0.f);
  }
  for (int t = threadIdx.x; t < NH * NH; t += blockDim.x) out->W2[t / NH][t % NH] = __float2bfloat16(w[OFF_W2 + t]);
  for (int t = threadIdx.x; t < NH; t += blockDim.x) {
    out->b1[t] = w[OFF_B1 + t]; out->b2[t] = w[OFF_B2 + t]; out->w3[t] = w[OFF_W3 + t];
  }
  if (threadIdx.x == 0) { out->b3 = w[OFF_B3]; out->pad[0] = out->pad[1] = out->pad[2] = 0.f; }
}

}  // namespace xrs
