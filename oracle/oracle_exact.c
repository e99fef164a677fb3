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
 * f(p) = f_L(p) + f_R(p) + du = 0 and sampling of the self-similar solution
 * at x/t = 0 (section 4.5).  The known answer shipped by the reference, the
 * Sod shock-tube secant solve of Simulation/SimulationMain/Sod/shocktube.pro
 * (lines 15-33, 90-120), is the cross-check used by the tests.
 *
 * Newton is safeguarded by the bracket of evaluated signs (see
 * orc_star_state), so it always terminates within max_iter.  The vacuum-
 * generating case is sampled as in Toro section 4.6.
 */
#include <float.h>
#include <math.h>
#include <stddef.h>

typedef struct { double d, u, p, c; } side_t;

/* Toro eq. 4.6-4.7 and their derivatives. */
/* qr = (p/pK)^((g-1)/2g) on the rarefaction branch, -1 on the shock branch */
static void pres_fn_q(double p, const side_t *s, double g, double *f, double *fd, double *qr) {
  if (p <= s->p) {                                   /* rarefaction */
    double prat = p / s->p;
    double ex = (g - 1.0) / (2.0 * g);
    double q = pow(prat, ex);
    *f = 2.0 * s->c / (g - 1.0) * (q - 1.0);
    *fd = q / (prat * s->d * s->c);                  /* (p/pK)^(-(g+1)/2g) / (dK cK) */
    *qr = q;
  } else {                                           /* shock */
    double A = 2.0 / ((g + 1.0) * s->d);
    double B = (g - 1.0) / (g + 1.0) * s->p;
    double q = sqrt(A / (B + p));
    *f = (p - s->p) * q;
    *fd = (1.0 - 0.5 * (p - s->p) / (B + p)) * q;
    *qr = -1.0;
  }
}
static void pres_fn(double p, const side_t *s, double g, double *f, double *fd) {
  double qr;
  pres_fn_q(p, s, g, f, fd, &qr);
}

/* The last evaluation of a Newton solve: its pressure and the rarefaction
 * branch powers (pe/pK)^((g-1)/2g) (-1 for a shock branch), which the
 * sampling carries to p* to first order. */
typedef struct { double pe, qL, qR; } last_eval_t;

/* Two-rarefaction guess, Toro eq. 4.46. */
double orc_two_rarefaction_guess(double dl, double ul, double pl, double dr, double ur, double pr, double g) {
  double cl = sqrt(g * pl / dl), cr = sqrt(g * pr / dr);
  double z = (g - 1.0) / (2.0 * g);
  double num = cl + cr - 0.5 * (g - 1.0) * (ur - ul);
  if (num <= 0.0) return 0.0;
  return pow(num / (cl / pow(pl, z) + cr / pow(pr, z)), 1.0 / z);
}

/* Strong waves (the network is consulted and the bracket probed only
 * there): the pressure range of p_L, p_R and the PVRS estimate covers a
 * factor of two or more, with the PVRS estimate above min(p_L, p_R). */
int orc_strong_waves(double dl, double ul, double pl, double dr, double ur, double pr, double g) {
  double cl = sqrt(g * pl / dl), cr = sqrt(g * pr / dr);
  double pmin = fmin(pl, pr), pmax = fmax(pl, pr);
  double ppv = 0.5 * (pl + pr) - 0.125 * (ur - ul) * (dl + dr) * (cl + cr);
  return ppv > pmin && fmax(pmax, ppv) >= 2.0 * pmin;
}

/* Solve for p* and u*.  p0 > 0 is the initial guess; p0 <= 0 starts from
 * the two-rarefaction guess and, for strong waves, first probes the bracket:
 * [pa, pb] = [p/4, p] with f(pb) > 0, from p = max(p_L, p_R) growing by 4,
 * and a start outside it is replaced by sqrt(pa * pb).  Returns 0 on
 * convergence, 1 when max_iter evaluations were used, 2 when the data
 * generate vacuum (p* = 0).  *iters = pressure-function evaluations.
 *
 * f is increasing and concave (Toro 4.3.1), so an iterate at or left of
 * the root stays there.  The iterate is kept inside the bracket of
 * evaluated signs (pb = DBL_MAX until a positive f is seen): a step leaving
 * it is replaced by a geometric bisection, a decimation towards zero
 * (pa = 0) or a growth by 4 (no upper end yet).  Converged when the step is
 * below tol * p or the predicted next step of the quadratic regime,
 * |step|^3/prev^2, is below tol * p / 100.  u* uses f_L, f_R linearised
 * from the last evaluation to the returned p*. */
static int star_solve(const side_t *Lp, const side_t *Rp, double g, double p, int probe, double tol, int max_iter,
                      double *pstar, double *ustar, int *iters, last_eval_t *le) {
  side_t L = *Lp, R = *Rp;
  double du = R.u - L.u;
  double fl = 0., fdl = 0., fr = 0., fdr = 0., qL = -1.0, qR = -1.0;
  double pa = 0.0, pb = DBL_MAX, pe = p, prev = -1.0;
  int evals = 0;
  le->pe = p; le->qL = -1.0; le->qR = -1.0;
  if (probe) {
    double q = fmax(L.p, R.p);
    for (int k = 0; k < 64 && evals < max_iter; ++k) {
      pres_fn(q, &L, g, &fl, &fdl); pres_fn(q, &R, g, &fr, &fdr);
      ++evals;
      if (fl + fr + du > 0.0) { pb = q; break; }
      pa = q;
      q *= 4.0;
    }
    if (!(p > pa && p < pb)) p = (pa > 0.0 && pb < DBL_MAX) ? sqrt(pa * pb) : (pb < DBL_MAX ? 0.5 * pb : 4.0 * pa);
  }
  *iters = evals;
  for (; evals < max_iter;) {
    pres_fn_q(p, &L, g, &fl, &fdl, &qL); pres_fn_q(p, &R, g, &fr, &fdr, &qR);
    ++evals;
    *iters = evals;
    pe = p;
    le->pe = pe; le->qL = qL; le->qR = qR;
    double f = fl + fr + du;
    if (f == 0.0) {
      *pstar = p;
      *ustar = 0.5 * (L.u + R.u) + 0.5 * (fr - fl);
      return 0;
    }
    if (f < 0.0) pa = p; else pb = p;
    double step = f / (fdl + fdr);
    double pn = p - step;
    double as = fabs(step);
    int inside = pn > pa && pn < pb;
    if (as <= tol * p || (inside && prev > 0.0 && as < prev && as * (as / prev) * (as / prev) <= 0.01 * tol * p)) {
      *pstar = pn > 0.0 ? pn : p;
      double dp = *pstar - pe;
      *ustar = 0.5 * (L.u + R.u) + 0.5 * ((fr + fdr * dp) - (fl + fdl * dp));
      return 0;
    }
    if (!inside) { pn = pb == DBL_MAX ? 4.0 * p : (pa > 0.0 ? sqrt(pa * pb) : 0.01 * pb); prev = -1.0; }
    else prev = as;
    p = pn;
  }
  *pstar = p;
  double dp = p - pe;
  *ustar = 0.5 * (L.u + R.u) + 0.5 * ((fr + fdr * dp) - (fl + fdl * dp));
  return 1;
}

int orc_star_state(double dl, double ul, double pl, double dr, double ur, double pr, double g,
                   double p0, double tol, int max_iter, double *pstar, double *ustar, int *iters) {
  side_t L = {dl, ul, pl, sqrt(g * pl / dl)}, R = {dr, ur, pr, sqrt(g * pr / dr)};
  *iters = 0;
  /* vacuum generation test, Toro eq. 4.40 */
  if (2.0 * (L.c + R.c) / (g - 1.0) <= ur - ul) {
    *pstar = 0.0;
    *ustar = 0.5 * (ul + ur);
    return 2;
  }
  int probe = p0 <= 0.0 && orc_strong_waves(dl, ul, pl, dr, ur, pr, g);
  double p = p0 > 0.0 ? p0 : orc_two_rarefaction_guess(dl, ul, pl, dr, ur, pr, g);
  last_eval_t le;
  return star_solve(&L, &R, g, p, probe, tol, max_iter, pstar, ustar, iters, &le);
}

/* Start of a hydro face solve: the two-rarefaction guess, with the bracket
 * probe for strong waves. */
static double face_start(double dl, double ul, double pl, double dr, double ur, double pr, double g, int *probe) {
  *probe = orc_strong_waves(dl, ul, pl, dr, ur, pr, g);
  return orc_two_rarefaction_guess(dl, ul, pl, dr, ur, pr, g);
}

/* Sample the exact solution at x/t = 0 (Toro section 4.5; vacuum
 * generation, section 4.6); returns the density, normal velocity and
 * pressure there and which side (0 = left, 1 = right) supplies the
 * transverse velocities. */
static void fan_left(const side_t *L, double g, double *d, double *u, double *p) {
  double c = 2.0 / (g + 1.0) * (L->c + 0.5 * (g - 1.0) * L->u);
  double r = c / L->c;
  *u = c;
  *d = L->d * pow(r, 2.0 / (g - 1.0));
  *p = L->p * pow(r, 2.0 * g / (g - 1.0));
}
static void fan_right(const side_t *R, double g, double *d, double *u, double *p) {
  double c = 2.0 / (g + 1.0) * (R->c - 0.5 * (g - 1.0) * R->u);
  double r = c / R->c;
  *u = -c;
  *d = R->d * pow(r, 2.0 / (g - 1.0));
  *p = R->p * pow(r, 2.0 * g / (g - 1.0));
}

/* pr^(1/g) from q = pr^((g-1)/2g): q^(2/(g-1)) by multiplications when
 * 2/(g-1) is an integer (g = 5/3: 3, g = 7/5: 5) */
static double pow_inv_gamma(double q, double pr, double g) {
  double k = 2.0 / (g - 1.0), kn = rint(k);
  if (fabs(k - kn) < 1e-9 && kn >= 1.0 && kn <= 16.0) {
    double r = q;
    for (int n = 1; n < (int)kn; ++n) r *= q;
    return r;
  }
  return pow(pr, 1.0 / g);
}
static double q_at(double ps, double pK, double g, double qe, double pe) {
  double ex = (g - 1.0) / (2.0 * g);
  return qe >= 0.0 ? qe * (1.0 + ex * (ps - pe) / pe) : pow(ps / pK, ex);
}

static void sample0(const side_t *L, const side_t *R, double g, double ps, double us, int vac,
                    double *d, double *u, double *p, int *from_right, const last_eval_t *le) {
  if (vac) {
    double sl = L->u + 2.0 * L->c / (g - 1.0), sr = R->u - 2.0 * R->c / (g - 1.0);
    if (0.0 <= L->u - L->c) { *from_right = 0; *d = L->d; *u = L->u; *p = L->p; }
    else if (0.0 < sl) { *from_right = 0; fan_left(L, g, d, u, p); }
    else if (0.0 >= R->u + R->c) { *from_right = 1; *d = R->d; *u = R->u; *p = R->p; }
    else if (0.0 > sr) { *from_right = 1; fan_right(R, g, d, u, p); }
    else { *from_right = 0; *d = 0.0; *u = 0.0; *p = 0.0; }
    return;
  }
  double g1 = (g - 1.0) / (2.0 * g), g2 = (g + 1.0) / (2.0 * g), g6 = (g - 1.0) / (g + 1.0);
  if (0.0 <= us) {                                   /* left of contact */
    *from_right = 0;
    if (ps > L->p) {                                 /* left shock */
      double pr = ps / L->p;
      double sl = L->u - L->c * sqrt(g2 * pr + g1);
      if (0.0 <= sl) { *d = L->d; *u = L->u; *p = L->p; }
      else { *d = L->d * (pr + g6) / (pr * g6 + 1.0); *u = us; *p = ps; }
    } else {                                         /* left rarefaction */
      if (0.0 <= L->u - L->c) { *d = L->d; *u = L->u; *p = L->p; }
      else {
        double pr = ps / L->p;
        double q = le ? q_at(ps, L->p, g, le->qL, le->pe) : pow(pr, g1);
        double cml = L->c * q;
        if (0.0 > us - cml) { *d = L->d * (le ? pow_inv_gamma(q, pr, g) : pow(pr, 1.0 / g)); *u = us; *p = ps; }
        else fan_left(L, g, d, u, p);
      }
    }
  } else {                                           /* right of contact */
    *from_right = 1;
    if (ps > R->p) {
      double pr = ps / R->p;
      double sr = R->u + R->c * sqrt(g2 * pr + g1);
      if (0.0 >= sr) { *d = R->d; *u = R->u; *p = R->p; }
      else { *d = R->d * (pr + g6) / (pr * g6 + 1.0); *u = us; *p = ps; }
    } else {
      if (0.0 >= R->u + R->c) { *d = R->d; *u = R->u; *p = R->p; }
      else {
        double pr = ps / R->p;
        double q = le ? q_at(ps, R->p, g, le->qR, le->pe) : pow(pr, g1);
        double cmr = R->c * q;
        if (0.0 <= us + cmr) { *d = R->d * (le ? pow_inv_gamma(q, pr, g) : pow(pr, 1.0 / g)); *u = us; *p = ps; }
        else fan_right(R, g, d, u, p);
      }
    }
  }
}

/* Godunov flux of the exact solution at a face, in the 6-slot layout of
 * hy_HLLC (mass, three momenta, energy, pressure).  VL/VR use the primitive
 * slots of UHD.h (dens, velx, vely, velz, pres, gamc, game, eint). */
int orc_exact_flux(int dir, const double *VL, const double *VR, double gamma, double tol,
                   int max_iter, double F[6], int *iters) {
  int n = dir;                                       /* normal velocity slot */
  side_t L = {VL[0], VL[n], VL[4], sqrt(gamma * VL[4] / VL[0])};
  side_t R = {VR[0], VR[n], VR[4], sqrt(gamma * VR[4] / VR[0])};
  double ps = 0.0, us = 0.5 * (L.u + R.u);
  int vac = 2.0 * (L.c + R.c) / (gamma - 1.0) <= R.u - L.u;
  int st = 0;
  last_eval_t le;
  *iters = 0;
  if (!vac) {
    int probe;
    double p0 = face_start(L.d, L.u, L.p, R.d, R.u, R.p, gamma, &probe);
    st = star_solve(&L, &R, gamma, p0, probe, tol, max_iter, &ps, &us, iters, &le);
  }
  double d, u, p;
  int fr;
  sample0(&L, &R, gamma, ps, us, vac, &d, &u, &p, &fr, vac ? NULL : &le);
  const double *Vt = fr ? VR : VL;
  double v[3] = {Vt[1], Vt[2], Vt[3]};
  v[dir - 1] = u;
  double E = p / (gamma - 1.0) + 0.5 * d * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  F[0] = d * u;
  F[1] = F[0] * v[0]; F[2] = F[0] * v[1]; F[3] = F[0] * v[2];
  F[dir] += p;
  F[4] = (E + p) * u;
  F[5] = p;
  return st == 1 ? 1 : 0;
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
