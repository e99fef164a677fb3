/*
 * oracle_exact.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * FP64 exact Riemann solver for the ideal-gas Euler equations, the CPU
 * checker of the project's exact solver.  FLASH5 has no exact solver on the
 * unsplit path (physics/Hydro/HydroMain/unsplit/hy_getFaceFlux.F90:324-372
 * dispatches Roe/HLL/HLLC/Marquina/LLF only), so parity for this part is
 * unpinned against the reference; the method is the published one of
 * E. F. Toro, "Riemann Solvers and Numerical Methods for Fluid Dynamics",
 * 3rd ed., ch. 4: the pressure functions f_K(p) (eqs. 4.6-4.8), the
 * two-rarefaction initial guess (eq. 4.46), Newton iteration on
 * f = f_L + f_R + du = 0 and sampling of the self-similar solution at
 * x/t = 0 (section 4.5).  The known answer shipped by the reference, the
 * Sod shock-tube secant solve of Simulation/SimulationMain/Sod/shocktube.pro
 * (lines 15-33, 90-120), is the cross-check used by the tests.
 *
 * Newton runs on w = p^z, z = (g-1)/(2g): there the rarefaction branch of
 * f_K is linear (so the two-rarefaction guess is the root of the linear
 * part) and, for g <= 5/3, the shock branch convex, so that Newton from the
 * two-rarefaction guess descends monotonically.  It is safeguarded by the bracket of
 * evaluated signs (see star_solve), so it always terminates within
 * max_iter.  The vacuum-generating case is sampled as in Toro section 4.6.
 * Powers are taken with pow(); the device solver takes the integer powers
 * p = w^(1/z) by multiplication, which agrees to rounding.
 */
#include <float.h>
#include <math.h>
#include <stddef.h>

typedef struct { double d, u, p, c, w; } side_t;    /* w = p^z */

static double zexp(double g) { return (g - 1.0) / (2.0 * g); }
static double p_of_w(double w, double g) { return pow(w, 2.0 * g / (g - 1.0)); }
static side_t make_side(double d, double u, double p, double g) {
  side_t s = {d, u, p, sqrt(g * p / d), pow(p, zexp(g))};
  return s;
}

/* f_K(w) and df_K/dw, Toro eqs. 4.6-4.7 with p = w^(1/z) */
static void pres_fn(double w, double p, const side_t *s, double g, double *f, double *fd) {
  if (w <= s->w) {                                   /* rarefaction: linear in w */
    double k = 2.0 * s->c / ((g - 1.0) * s->w);
    *f = k * (w - s->w);
    *fd = k;
  } else {                                           /* shock */
    double A = 2.0 / ((g + 1.0) * s->d);
    double B = (g - 1.0) / (g + 1.0) * s->p;
    double r = 1.0 / (B + p);
    double q = sqrt(A * r);
    *f = (p - s->p) * q;
    *fd = (1.0 - 0.5 * (p - s->p) * r) * q * (p / (zexp(g) * w));
  }
}

/* Two-rarefaction guess (Toro eq. 4.46) in w; 0 for vacuum-generating data */
static double tr_w(const side_t *L, const side_t *R, double g) {
  double num = L->c + R->c - 0.5 * (g - 1.0) * (R->u - L->u);
  return num > 0.0 ? num / (L->c / L->w + R->c / R->w) : 0.0;
}

double orc_two_rarefaction_guess(double dl, double ul, double pl, double dr, double ur, double pr, double g) {
  side_t L = make_side(dl, ul, pl, g), R = make_side(dr, ur, pr, g);
  return p_of_w(tr_w(&L, &R, g), g);
}

/* Strong waves (the network is consulted only there): the pressure range
 * of p_L, p_R and the PVRS estimate covers a factor of two or more, with
 * the PVRS estimate above min(p_L, p_R). */
int orc_strong_waves(double dl, double ul, double pl, double dr, double ur, double pr, double g) {
  double cl = sqrt(g * pl / dl), cr = sqrt(g * pr / dr);
  double pmin = fmin(pl, pr), pmax = fmax(pl, pr);
  double ppv = 0.5 * (pl + pr) - 0.125 * (ur - ul) * (dl + dr) * (cl + cr);
  return ppv > pmin && fmax(pmax, ppv) >= 2.0 * pmin;
}

/* Newton on f(w) from w0 >= 0.  The iterate is kept inside the bracket of
 * evaluated signs (wb = DBL_MAX until a positive f is seen): a step leaving
 * it is replaced by the bracket's midpoint (a doubling while no upper end is
 * known).  Converged when the step is below tol * z * w (a relative step of
 * tol in p), the predicted next step of the quadratic regime,
 * |step|^3/prev^2, is below a hundredth of that, or the bracket is that
 * narrow (near vacuum; the root is its midpoint).  u* uses f_L, f_R
 * linearised from the last evaluation to the returned w*.  Returns 0 on
 * convergence, 1 when max_iter evaluations were used. */
static int star_solve(const side_t *L, const side_t *R, double g, double w0, double tol, int max_iter,
                      double *pstar, double *ustar, double *wstar, int *iters) {
  double du = R->u - L->u, ztol = zexp(g) * tol;
  double fl = 0., fdl = 0., fr = 0., fdr = 0., p = 0.0;
  double wa = 0.0, wb = DBL_MAX, w = w0, we = w0, prev = -1.0;
  int evals = 0;
  *iters = 0;
  while (evals < max_iter) {
    p = p_of_w(w, g);
    pres_fn(w, p, L, g, &fl, &fdl);
    pres_fn(w, p, R, g, &fr, &fdr);
    *iters = ++evals;
    we = w;
    double f = fl + fr + du;
    if (f == 0.0) {
      *wstar = w; *pstar = p;
      *ustar = 0.5 * (L->u + R->u) + 0.5 * (fr - fl);
      return 0;
    }
    if (f < 0.0) wa = w; else wb = w;
    if (wb - wa <= ztol * w) {
      *wstar = 0.5 * (wa + wb);
      *pstar = p_of_w(*wstar, g);
      double dw = *wstar - we;
      *ustar = 0.5 * (L->u + R->u) + 0.5 * ((fr + fdr * dw) - (fl + fdl * dw));
      return 0;
    }
    double step = f / (fdl + fdr);
    double wn = w - step;
    double as = fabs(step);
    int inside = wn > wa && wn < wb;
    if (as <= ztol * w || (inside && prev > 0.0 && as < prev && as * (as / prev) * (as / prev) <= 0.01 * ztol * w)) {
      *wstar = wn > 0.0 ? wn : w;
      *pstar = p_of_w(*wstar, g);
      double dw = *wstar - we;
      *ustar = 0.5 * (L->u + R->u) + 0.5 * ((fr + fdr * dw) - (fl + fdl * dw));
      return 0;
    }
    if (!inside) { wn = wb == DBL_MAX ? 2.0 * w : 0.5 * (wa + wb); prev = -1.0; }
    else prev = as;
    w = wn;
  }
  *wstar = w;
  *pstar = p_of_w(w, g);
  double dw = w - we;
  *ustar = 0.5 * (L->u + R->u) + 0.5 * ((fr + fdr * dw) - (fl + fdl * dw));
  return 1;
}

/* Solve for p* and u*.  p0 > 0 is the initial guess; p0 <= 0 starts from
 * the two-rarefaction guess.  Returns 0 on convergence, 1 when max_iter
 * evaluations were used, 2 when the data generate vacuum (p* = 0).
 * *iters = pressure-function evaluations. */
int orc_star_state(double dl, double ul, double pl, double dr, double ur, double pr, double g,
                   double p0, double tol, int max_iter, double *pstar, double *ustar, int *iters) {
  side_t L = make_side(dl, ul, pl, g), R = make_side(dr, ur, pr, g);
  *iters = 0;
  /* vacuum generation test, Toro eq. 4.40 */
  if (2.0 * (L.c + R.c) / (g - 1.0) <= ur - ul) {
    *pstar = 0.0;
    *ustar = 0.5 * (ul + ur);
    return 2;
  }
  double ws, w0 = p0 > 0.0 ? pow(p0, zexp(g)) : tr_w(&L, &R, g);
  return star_solve(&L, &R, g, w0, tol, max_iter, pstar, ustar, &ws, iters);
}

/* Sample the exact solution at x/t = 0 (Toro section 4.5; vacuum
 * generation, section 4.6); returns the density, normal velocity and
 * pressure there and which side (0 = left, 1 = right) supplies the
 * transverse velocities.  Behind a rarefaction (p* / p_K)^z = w* / w_K. */
static void fan_left(const side_t *L, double g, double *d, double *u, double *p) {
  double c = 2.0 / (g + 1.0) * (L->c + 0.5 * (g - 1.0) * L->u);
  *u = c;
  double r = c / L->c;
  *d = L->d * pow(r, 2.0 / (g - 1.0));
  *p = L->p * pow(r, 2.0 * g / (g - 1.0));
}
static void fan_right(const side_t *R, double g, double *d, double *u, double *p) {
  double c = 2.0 / (g + 1.0) * (R->c - 0.5 * (g - 1.0) * R->u);
  *u = -c;
  double r = c / R->c;
  *d = R->d * pow(r, 2.0 / (g - 1.0));
  *p = R->p * pow(r, 2.0 * g / (g - 1.0));
}

static void sample0(const side_t *L, const side_t *R, double g, double ps, double us, double ws, int vac,
                    double *d, double *u, double *p, int *from_right) {
  if (vac) {
    double sl = L->u + 2.0 * L->c / (g - 1.0), sr = R->u - 2.0 * R->c / (g - 1.0);
    if (0.0 <= L->u - L->c) { *from_right = 0; *d = L->d; *u = L->u; *p = L->p; }
    else if (0.0 < sl) { *from_right = 0; fan_left(L, g, d, u, p); }
    else if (0.0 >= R->u + R->c) { *from_right = 1; *d = R->d; *u = R->u; *p = R->p; }
    else if (0.0 > sr) { *from_right = 1; fan_right(R, g, d, u, p); }
    else { *from_right = 0; *d = 0.0; *u = 0.0; *p = 0.0; }
    return;
  }
  double g1 = (g - 1.0) / (2.0 * g), g2 = (g + 1.0) / (2.0 * g), g6 = (g - 1.0) / (g + 1.0), k = 2.0 / (g - 1.0);
  if (0.0 <= us) {                                   /* left of the contact */
    *from_right = 0;
    if (ps > L->p) {                                 /* left shock */
      double pr = ps / L->p;
      double sl = L->u - L->c * sqrt(g2 * pr + g1);
      if (0.0 <= sl) { *d = L->d; *u = L->u; *p = L->p; }
      else { *d = L->d * (pr + g6) / (pr * g6 + 1.0); *u = us; *p = ps; }
    } else {                                         /* left rarefaction */
      if (0.0 <= L->u - L->c) { *d = L->d; *u = L->u; *p = L->p; }
      else {
        double q = ws / L->w;
        double cml = L->c * q;
        if (0.0 > us - cml) { *d = L->d * pow(q, k); *u = us; *p = ps; }
        else fan_left(L, g, d, u, p);
      }
    }
  } else {                                           /* right of the contact */
    *from_right = 1;
    if (ps > R->p) {
      double pr = ps / R->p;
      double sr = R->u + R->c * sqrt(g2 * pr + g1);
      if (0.0 >= sr) { *d = R->d; *u = R->u; *p = R->p; }
      else { *d = R->d * (pr + g6) / (pr * g6 + 1.0); *u = us; *p = ps; }
    } else {
      if (0.0 >= R->u + R->c) { *d = R->d; *u = R->u; *p = R->p; }
      else {
        double q = ws / R->w;
        double cmr = R->c * q;
        if (0.0 <= us + cmr) { *d = R->d * pow(q, k); *u = us; *p = ps; }
        else fan_right(R, g, d, u, p);
      }
    }
  }
}

/* Godunov flux of the exact solution in the 6-slot layout of the HLLC
 * oracle (mass, three momenta, energy, pressure).  VL, VR: primitive
 * states (dens, velx, vely, velz, pres); dir = 1..3.  Returns 1 when
 * Newton did not converge. */
int orc_exact_flux(int dir, const double *VL, const double *VR, double gamma, double tol,
                   int max_iter, double F[6], int *iters) {
  int n = dir;                                       /* normal velocity slot */
  side_t L = make_side(VL[0], VL[n], VL[4], gamma), R = make_side(VR[0], VR[n], VR[4], gamma);
  double ps = 0.0, us = 0.5 * (L.u + R.u), ws = 0.0;
  int vac = 2.0 * (L.c + R.c) / (gamma - 1.0) <= R.u - L.u;
  int st = 0;
  *iters = 0;
  if (!vac) st = star_solve(&L, &R, gamma, tr_w(&L, &R, gamma), tol, max_iter, &ps, &us, &ws, iters);
  double d, u, p;
  int fr;
  sample0(&L, &R, gamma, ps, us, ws, vac, &d, &u, &p, &fr);
  const double *Vt = fr ? VR : VL;
  double v[3] = {Vt[1], Vt[2], Vt[3]};
  v[dir - 1] = u;
  double E = p / (gamma - 1.0) + 0.5 * d * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  F[0] = d * u;
  F[1] = F[0] * v[0]; F[2] = F[0] * v[1]; F[3] = F[0] * v[2];
  F[dir] += p;
  F[4] = (E + p) * u;
  F[5] = p;
  return st;
}

/* Batched isolated solves (the N-interface star-pressure problem). */
void orc_star_batch(long n, const double *dl, const double *ul, const double *pl, const double *dr,
                    const double *ur, const double *pr, const double *gam, const double *p0,
                    double tol, int max_iter, double *pstar, double *ustar, int *iters, int *status) {
  #pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i)
    status[i] = orc_star_state(dl[i], ul[i], pl[i], dr[i], ur[i], pr[i], gam[i], p0 ? p0[i] : 0.0,
                               tol, max_iter, &pstar[i], &ustar[i], &iters[i]);
}
