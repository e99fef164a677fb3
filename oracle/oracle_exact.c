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
 * Newton here is safeguarded by a bracket [pa, pb] with f(pa) < 0 < f(pb):
 * a step that leaves the bracket is replaced by a geometric bisection (or a
 * decimation towards zero while pa = 0), and the iteration stops when the
 * Newton step is below tol * p, so it always terminates within max_iter.
 */
#include <math.h>

typedef struct { double d, u, p, c; } side_t;

/* Toro eq. 4.6-4.7 and their derivatives. */
static void pres_fn(double p, const side_t *s, double g, double *f, double *fd) {
  if (p <= s->p) {                                   /* rarefaction */
    double prat = p / s->p;
    double ex = (g - 1.0) / (2.0 * g);
    *f = 2.0 * s->c / (g - 1.0) * (pow(prat, ex) - 1.0);
    *fd = (1.0 / (s->d * s->c)) * pow(prat, -(g + 1.0) / (2.0 * g));
  } else {                                           /* shock */
    double A = 2.0 / ((g + 1.0) * s->d);
    double B = (g - 1.0) / (g + 1.0) * s->p;
    double q = sqrt(A / (B + p));
    *f = (p - s->p) * q;
    *fd = (1.0 - 0.5 * (p - s->p) / (B + p)) * q;
  }
}

/* Two-rarefaction guess, Toro eq. 4.46. */
double orc_two_rarefaction_guess(double dl, double ul, double pl, double dr, double ur, double pr, double g) {
  double cl = sqrt(g * pl / dl), cr = sqrt(g * pr / dr);
  double z = (g - 1.0) / (2.0 * g);
  double num = cl + cr - 0.5 * (g - 1.0) * (ur - ul);
  if (num <= 0.0) return 0.0;
  return pow(num / (cl / pow(pl, z) + cr / pow(pr, z)), 1.0 / z);
}

/* Solve for p* and u*.  p0 > 0 is the initial guess (<= 0: two-rarefaction).
 * Returns 0 on convergence to |dp|/p < tol, 1 when max_iter was hit, 2 when
 * the data generate vacuum (p* = 0).  *iters = Newton/bisection steps. */
int orc_star_state(double dl, double ul, double pl, double dr, double ur, double pr, double g,
                   double p0, double tol, int max_iter, double *pstar, double *ustar, int *iters) {
  side_t L = {dl, ul, pl, sqrt(g * pl / dl)}, R = {dr, ur, pr, sqrt(g * pr / dr)};
  double du = ur - ul;
  *iters = 0;
  /* vacuum generation test, Toro eq. 4.40 */
  if (2.0 * (L.c + R.c) / (g - 1.0) <= du) {
    *pstar = 0.0;
    *ustar = 0.5 * (ul + ur);
    return 2;
  }
  double fl, fdl, fr, fdr;
  /* bracket: f is increasing in p; f(0+) < 0 here, find pb with f(pb) > 0 */
  double pa = 0.0, pb = fmax(pl, pr);
  for (int k = 0; k < 200; ++k) {
    pres_fn(pb, &L, g, &fl, &fdl); pres_fn(pb, &R, g, &fr, &fdr);
    if (fl + fr + du > 0.0) break;
    pa = pb;
    pb *= 4.0;
  }
  double p = p0 > 0.0 ? p0 : orc_two_rarefaction_guess(dl, ul, pl, dr, ur, pr, g);
  if (!(p > pa && p < pb)) p = pa > 0.0 ? sqrt(pa * pb) : 0.5 * pb;
  int status = 1;
  double prev = -1.0;
  for (int it = 0; it < max_iter; ++it) {
    pres_fn(p, &L, g, &fl, &fdl); pres_fn(p, &R, g, &fr, &fdr);
    double f = fl + fr + du;
    *iters = it + 1;
    if (f == 0.0) { status = 0; break; }
    if (f < 0.0) pa = p; else pb = p;
    double step = f / (fdl + fdr);
    double pn = p - step;
    double as = fabs(step);
    int inside = pn > pa && pn < pb;
    /* converged: step below tol, or the predicted next step of the
     * quadratic regime, |step|^3/prev^2, below tol/100 */
    if (as <= tol * p || (inside && prev > 0.0 && as < prev && as * (as / prev) * (as / prev) <= 0.01 * tol * p)) {
      if (pn > 0.0) p = pn;
      status = 0;
      break;
    }
    if (!inside) { pn = pa > 0.0 ? sqrt(pa * pb) : 0.01 * pb; prev = -1.0; }
    else prev = as;
    p = pn;
  }
  pres_fn(p, &L, g, &fl, &fdl); pres_fn(p, &R, g, &fr, &fdr);
  *pstar = p;
  *ustar = 0.5 * (ul + ur) + 0.5 * (fr - fl);
  return status;
}

/* Sample the exact solution at x/t = 0 (Toro section 4.5); returns the
 * density, normal velocity and pressure there and which side (0 = left,
 * 1 = right) supplies the transverse velocities. */
static void sample0(const side_t *L, const side_t *R, double g, double ps, double us,
                    double *d, double *u, double *p, int *from_right) {
  double g1 = (g - 1.0) / (2.0 * g), g2 = (g + 1.0) / (2.0 * g), g6 = (g - 1.0) / (g + 1.0);
  if (0.0 <= us) {                                   /* left of contact */
    *from_right = 0;
    if (ps > L->p) {                                 /* left shock */
      double sl = L->u - L->c * sqrt(g2 * ps / L->p + g1);
      if (0.0 <= sl) { *d = L->d; *u = L->u; *p = L->p; }
      else { *d = L->d * (ps / L->p + g6) / (ps / L->p * g6 + 1.0); *u = us; *p = ps; }
    } else {                                         /* left rarefaction */
      double shl = L->u - L->c;
      if (0.0 <= shl) { *d = L->d; *u = L->u; *p = L->p; }
      else {
        double cml = L->c * pow(ps / L->p, g1);
        double stl = us - cml;
        if (0.0 > stl) { *d = L->d * pow(ps / L->p, 1.0 / g); *u = us; *p = ps; }
        else {
          double c = 2.0 / (g + 1.0) * (L->c + 0.5 * (g - 1.0) * L->u);
          *u = c;
          *d = L->d * pow(c / L->c, 2.0 / (g - 1.0));
          *p = L->p * pow(c / L->c, 2.0 * g / (g - 1.0));
        }
      }
    }
  } else {                                           /* right of contact */
    *from_right = 1;
    if (ps > R->p) {
      double sr = R->u + R->c * sqrt(g2 * ps / R->p + g1);
      if (0.0 >= sr) { *d = R->d; *u = R->u; *p = R->p; }
      else { *d = R->d * (ps / R->p + g6) / (ps / R->p * g6 + 1.0); *u = us; *p = ps; }
    } else {
      double shr = R->u + R->c;
      if (0.0 >= shr) { *d = R->d; *u = R->u; *p = R->p; }
      else {
        double cmr = R->c * pow(ps / R->p, g1);
        double str = us + cmr;
        if (0.0 <= str) { *d = R->d * pow(ps / R->p, 1.0 / g); *u = us; *p = ps; }
        else {
          double c = 2.0 / (g + 1.0) * (R->c - 0.5 * (g - 1.0) * R->u);
          *u = -c;
          *d = R->d * pow(c / R->c, 2.0 / (g - 1.0));
          *p = R->p * pow(c / R->c, 2.0 * g / (g - 1.0));
        }
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
  double ps, us;
  int st = orc_star_state(VL[0], VL[n], VL[4], VR[0], VR[n], VR[4], gamma, 0.0, tol, max_iter,
                          &ps, &us, iters);
  side_t L = {VL[0], VL[n], VL[4], sqrt(gamma * VL[4] / VL[0])};
  side_t R = {VR[0], VR[n], VR[4], sqrt(gamma * VR[4] / VR[0])};
  double d, u, p;
  int fr;
  sample0(&L, &R, gamma, ps, us, &d, &u, &p, &fr);
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
