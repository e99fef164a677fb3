// amr_kernels.cuh -- guard cells of an AMR hierarchy in PARAMESH form, the
// device side of what Grid_fillGuardCells does before Hydro on PARAMESH
// (paramesh4/Grid_fillGuardCells.F90:227-569 with FLASH's native
// interpolation):
//   k_restrict    parent interiors = average of the 2^d children
//                 (amr_restrict_unk_genorder.F90, order 1), one level per
//                 launch, finest parents first;
//   k_parent_halo guard-inclusive copy of every parent (rho, v, e, E), one
//                 level per launch, coarsest first;
//   k_leaf_halo   guard cells of every leaf after the guard-cell EOS.
// A guard cell is copied from the node of the same level that owns it (a
// leaf, or a parent holding restricted data) or, where that level is not
// refined, linearly prolonged from the node's parent
// (amr_1blk_cc_prol_linear.F90 with the weights and indices of
// amr_prolong_cc_fun_init.F90).  Both restriction and prolongation act on
// per-volume values: velocities, e and E are multiplied by the density
// before and divided after (flash_convert_cc_hook.F90,
// flash_unconvert_cc_hook.F90).  Compiled without FMA contraction, in the
// expression order of the CPU oracle, so the FP64 path stays bit-identical.
#pragma once
#include "hy_kernels.cuh"

namespace fhy {

// specific total energy of a stored node cell: leaves keep E = e + ekin
// (the EOS identity), parents their restricted E
__device__ __forceinline__ double node_E(const DevParams &P, int m, size_t off, double e, double vx, double vy,
                                         double vz) {
  if (P.leaf[m]) {
    const double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
    return e + ekin;
  }
  return P.pe[off];
}

template <int NDIM, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256) k_restrict(DevParams P, double *st0, double *st1, double *st2, double *st3,
                                                  double *st4, const int *plist, double *sp, size_t ncells) {
  constexpr int NCB = NX * NY * NZ;
  const int b = plist[blockIdx.x];
  const int l = P.blk_level[b];
  const int3 pc = blk_coords(P, b);
  const double *const st[5] = {st0, st1, st2, st3, st4};
  constexpr int hx = NX / 2, hy = NY / 2, hz = NDIM > 2 ? NZ / 2 : 1;
  const double w = NDIM > 2 ? 0.125 : 0.25;
  for (int loc = threadIdx.x; loc < NCB; loc += blockDim.x) {
    const int i = loc % NX, j = (loc / NX) % NY, k = loc / (NX * NY);
    const int ox = i >= hx, oy = j >= hy, oz = NDIM > 2 ? k >= hz : 0;
    const int ch = at_node(P, l + 1, 2 * pc.x + ox, 2 * pc.y + oy, NDIM > 2 ? 2 * pc.z + oz : 0);
    const int fi = 2 * (i - ox * hx), fj = 2 * (j - oy * hy), fk = NDIM > 2 ? 2 * (k - oz * hz) : 0;
    double s[6] = {0., 0., 0., 0., 0., 0.};
    for (int kk = 0; kk <= (NDIM > 2 ? 1 : 0); ++kk)
      for (int jj = 0; jj <= 1; ++jj)
        for (int ii = 0; ii <= 1; ++ii) {
          const size_t off = (size_t)ch * NCB + (size_t)(((fk + kk) * NY + (fj + jj)) * NX + (fi + ii));
          const double rho = st[0][off], vx = st[1][off], vy = st[2][off], vz = st[3][off], e = st[4][off];
          const double E = node_E(P, ch, off, e, vx, vy, vz);
          s[0] = s[0] + w * rho;
          s[1] = s[1] + w * (rho * vx);
          s[2] = s[2] + w * (rho * vy);
          s[3] = s[3] + w * (rho * vz);
          s[4] = s[4] + w * (rho * e);
          s[5] = s[5] + w * (rho * E);
        }
    const size_t o = (size_t)b * NCB + loc;
    const double inv = 1. / s[0];
    st0[o] = s[0];
    st1[o] = inv * s[1];
    st2[o] = inv * s[2];
    st3[o] = inv * s[3];
    st4[o] = inv * s[4];
    P.pe[o] = inv * s[5];
    // species and mass scalars, per-mass like the velocities
    for (int q = 0; q < P.nsp; ++q) {
      double x = 0.;
      for (int kk = 0; kk <= (NDIM > 2 ? 1 : 0); ++kk)
        for (int jj = 0; jj <= 1; ++jj)
          for (int ii = 0; ii <= 1; ++ii) {
            const size_t off = (size_t)ch * NCB + (size_t)(((fk + kk) * NY + (fj + jj)) * NX + (fi + ii));
            x = x + w * (st[0][off] * sp[(size_t)q * ncells + off]);
          }
      sp[(size_t)q * ncells + o] = inv * x;
    }
  }
}

// Linear prolongation (amr_1blk_cc_prol_linear.F90 with the weights and
// indices of amr_prolong_cc_fun_init.F90) of child cell lp of the node at
// coordinates c from its parent's guard-inclusive copy gp ([6][Halo::n]:
// rho, vx, vy, vz, e, E), in per-volume form.
template <int NDIM, int NX, int NY, int NZ>
__device__ __forceinline__ void prolong_linear(const double *gp, const int c[3], const int lp[3], double out[6]) {
  using H = Halo<NDIM, NX, NY, NZ>;
  const int Nd[3] = {NX, NY, NZ};
  int i1[3] = {0, 0, 0};
  double wx[3] = {1., 1., 1.}, cx[3] = {0., 0., 0.};
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    const int N = Nd[d], ioff = (c[d] & 1) * (N / 2), ii = lp[d] + 1;
    i1[d] = (ii + 2 * N) / 2 - N + ioff - 1;
    wx[d] = fmod(0.75 + (double)(ii + 2 * N) * .5, 1.);
    cx[d] = 1. - wx[d];
  }
  double r[2][2][2][6];
  for (int kk = 0; kk <= (NDIM > 2 ? 1 : 0); ++kk)
    for (int jj = 0; jj <= 1; ++jj)
      for (int ii = 0; ii <= 1; ++ii) {
        const int h = H::idx(i1[0] + ii, i1[1] + jj, NDIM > 2 ? i1[2] + kk : 0);
        const double rho = gp[h];
        r[kk][jj][ii][0] = rho;
#pragma unroll
        for (int v = 1; v < 6; ++v) r[kk][jj][ii][v] = rho * gp[v * H::n + h];
      }
  double val[6];
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    const double plane0 = wx[1] * (wx[0] * r[0][0][0][v] + cx[0] * r[0][0][1][v]) +
                          cx[1] * (wx[0] * r[0][1][0][v] + cx[0] * r[0][1][1][v]);
    if (NDIM > 2) {
      const double plane1 = wx[1] * (wx[0] * r[1][0][0][v] + cx[0] * r[1][0][1][v]) +
                            cx[1] * (wx[0] * r[1][1][0][v] + cx[0] * r[1][1][1][v]);
      val[v] = wx[2] * plane0 + cx[2] * plane1;
    } else {
      val[v] = plane0;
    }
  }
  const double inv = 1. / val[0];
  out[0] = val[0];
#pragma unroll
  for (int v = 1; v < 6; ++v) out[v] = inv * val[v];
}

// (rho, vx, vy, vz, e, E) of guard cell (li, lj, lk) of node n, before the EOS
template <int NDIM, int NX, int NY, int NZ>
__device__ void amr_guard(const DevParams &P, const double *const st[5], int n, int li, int lj, int lk, double out[6]) {
  constexpr int NCB = NX * NY * NZ;
  using H = Halo<NDIM, NX, NY, NZ>;
  const int l = P.blk_level[n];
  const int3 c3 = blk_coords(P, n);
  const int c[3] = {c3.x, c3.y, c3.z}, Nd[3] = {NX, NY, NZ}, loc[3] = {li, lj, lk};
  int gl[3] = {0, 0, 0}, lp[3] = {0, 0, 0}, flip[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    const int tot = P.at_ext[l][d] * Nd[d], base = c[d] * Nd[d];
    int gc = base + loc[d];
    lp[d] = loc[d];
    if (gc < 0 || gc >= tot) {
      const int side = gc < 0 ? 2 * d : 2 * d + 1;
      if (P.bc[side] == -135) {
        gc = ((gc % tot) + tot) % tot;
      } else {
        gc = map_axis(gc, tot, P.bc[2 * d], P.bc[2 * d + 1], flip[d]);
        lp[d] = gc - base;
      }
    }
    gl[d] = gc;
  }
  const int m = at_node(P, l, gl[0] / NX, NDIM > 1 ? gl[1] / NY : 0, NDIM > 2 ? gl[2] / NZ : 0);
  if (m >= 0) {
    const size_t off = (size_t)m * NCB + (size_t)(((NDIM > 2 ? gl[2] % NZ : 0) * NY + (gl[1] % NY)) * NX + gl[0] % NX);
    out[0] = st[0][off]; out[1] = st[1][off]; out[2] = st[2][off]; out[3] = st[3][off]; out[4] = st[4][off];
    out[5] = node_E(P, m, off, out[4], out[1], out[2], out[3]);
  } else {
    // linear prolongation from the parent's guard-inclusive copy
    prolong_linear<NDIM, NX, NY, NZ>(P.gp + (size_t)P.slot[P.parent[n]] * 6 * H::n, c, lp, out);
  }
  if (flip[0]) out[1] = -out[1];
  if (flip[1]) out[2] = -out[2];
  if (flip[2]) out[3] = -out[3];
}

// Linear prolongation of one per-mass scalar x (a species) of child cell lp
// from the parent's guard-inclusive density gr and x gx: the arithmetic of
// prolong_linear on (rho, rho x).
template <int NDIM, int NX, int NY, int NZ>
__device__ __forceinline__ double prolong_scalar(const double *gr, const double *gx, const int c[3], const int lp[3]) {
  using H = Halo<NDIM, NX, NY, NZ>;
  const int Nd[3] = {NX, NY, NZ};
  int i1[3] = {0, 0, 0};
  double wx[3] = {1., 1., 1.}, cx[3] = {0., 0., 0.};
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    const int N = Nd[d], ioff = (c[d] & 1) * (N / 2), ii = lp[d] + 1;
    i1[d] = (ii + 2 * N) / 2 - N + ioff - 1;
    wx[d] = fmod(0.75 + (double)(ii + 2 * N) * .5, 1.);
    cx[d] = 1. - wx[d];
  }
  double r[2][2][2][2];
  for (int kk = 0; kk <= (NDIM > 2 ? 1 : 0); ++kk)
    for (int jj = 0; jj <= 1; ++jj)
      for (int ii = 0; ii <= 1; ++ii) {
        const int h = H::idx(i1[0] + ii, i1[1] + jj, NDIM > 2 ? i1[2] + kk : 0);
        const double rho = gr[h];
        r[kk][jj][ii][0] = rho;
        r[kk][jj][ii][1] = rho * gx[h];
      }
  double val[2];
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    const double plane0 = wx[1] * (wx[0] * r[0][0][0][v] + cx[0] * r[0][0][1][v]) +
                          cx[1] * (wx[0] * r[0][1][0][v] + cx[0] * r[0][1][1][v]);
    if (NDIM > 2) {
      const double plane1 = wx[1] * (wx[0] * r[1][0][0][v] + cx[0] * r[1][0][1][v]) +
                            cx[1] * (wx[0] * r[1][1][0][v] + cx[0] * r[1][1][1][v]);
      val[v] = wx[2] * plane0 + cx[2] * plane1;
    } else {
      val[v] = plane0;
    }
  }
  const double inv = 1. / val[0];
  return inv * val[1];
}

// species q of guard cell (li, lj, lk) of node n: from the node of the same
// level that owns the cell, or prolonged from n's parent (no sign change
// at reflecting boundaries)
template <int NDIM, int NX, int NY, int NZ>
__device__ double amr_guard_spec(const DevParams &P, size_t ncells, int n, int li, int lj, int lk, int q) {
  constexpr int NCB = NX * NY * NZ;
  using H = Halo<NDIM, NX, NY, NZ>;
  const int l = P.blk_level[n];
  const int3 c3 = blk_coords(P, n);
  const int c[3] = {c3.x, c3.y, c3.z}, Nd[3] = {NX, NY, NZ}, loc[3] = {li, lj, lk};
  int gl[3] = {0, 0, 0}, lp[3] = {0, 0, 0}, flip[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    const int tot = P.at_ext[l][d] * Nd[d], base = c[d] * Nd[d];
    int gc = base + loc[d];
    lp[d] = loc[d];
    if (gc < 0 || gc >= tot) {
      const int side = gc < 0 ? 2 * d : 2 * d + 1;
      if (P.bc[side] == -135) {
        gc = ((gc % tot) + tot) % tot;
      } else {
        gc = map_axis(gc, tot, P.bc[2 * d], P.bc[2 * d + 1], flip[d]);
        lp[d] = gc - base;
      }
    }
    gl[d] = gc;
  }
  const int m = at_node(P, l, gl[0] / NX, NDIM > 1 ? gl[1] / NY : 0, NDIM > 2 ? gl[2] / NZ : 0);
  if (m >= 0) {
    const size_t off = (size_t)m * NCB + (size_t)(((NDIM > 2 ? gl[2] % NZ : 0) * NY + (gl[1] % NY)) * NX + gl[0] % NX);
    return P.sp_in[(size_t)q * ncells + off];
  }
  const int p = P.parent[n];
  const size_t ps = (size_t)P.slot[p];
  return prolong_scalar<NDIM, NX, NY, NZ>(P.gp + ps * 6 * H::n, P.sp_gp + (ps * P.nsp + q) * H::n, c, lp);
}

template <int NDIM, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256) k_parent_halo(DevParams P, const double *st0, const double *st1,
                                                     const double *st2, const double *st3, const double *st4,
                                                     const int *plist) {
  constexpr int NCB = NX * NY * NZ;
  using H = Halo<NDIM, NX, NY, NZ>;
  const int b = plist[blockIdx.x];
  const double *const st[5] = {st0, st1, st2, st3, st4};
  double *gp = P.gp + (size_t)P.slot[b] * 6 * H::n;
  for (int h = threadIdx.x; h < H::n; h += blockDim.x) {
    const int li = h % H::hx - 4, lj = NDIM > 1 ? (h / H::hx) % H::hy - 4 : 0, lk = NDIM > 2 ? h / (H::hx * H::hy) - 4 : 0;
    double v[6];
    if (is_inside<NDIM, NX, NY, NZ>(li, lj, lk)) {
      const size_t off = (size_t)b * NCB + (size_t)((lk * NY + lj) * NX + li);
      v[0] = st0[off]; v[1] = st1[off]; v[2] = st2[off]; v[3] = st3[off]; v[4] = st4[off]; v[5] = P.pe[off];
    } else {
      amr_guard<NDIM, NX, NY, NZ>(P, st, b, li, lj, lk, v);
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) gp[q * H::n + h] = v[q];
  }
  if (P.sp_gp) {
    // species after the parent's own (rho, ...) copy: the prolongation from
    // the grandparent reads this level's parents only through their parent
    constexpr int NCB2 = NX * NY * NZ;
    const size_t ncells = P.sp_ncells;
    for (int qh = threadIdx.x; qh < P.nsp * H::n; qh += blockDim.x) {
      const int q = qh / H::n, h = qh % H::n;
      const int li = h % H::hx - 4, lj = NDIM > 1 ? (h / H::hx) % H::hy - 4 : 0, lk = NDIM > 2 ? h / (H::hx * H::hy) - 4 : 0;
      double x;
      if (is_inside<NDIM, NX, NY, NZ>(li, lj, lk))
        x = P.sp_in[(size_t)q * ncells + (size_t)b * NCB2 + (size_t)((lk * NY + lj) * NX + li)];
      else
        x = amr_guard_spec<NDIM, NX, NY, NZ>(P, ncells, b, li, lj, lk, q);
      P.sp_gp[((size_t)P.slot[b] * P.nsp + q) * H::n + h] = x;
    }
  }
}

// guard cells of the leaves, after the guard-cell EOS (Eos_getData.F90:80-96:
// e = E - ekin where that exceeds max(smalle, eintSwitch * ekin))
template <int NDIM, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256) k_leaf_halo(DevParams P, const double *st0, const double *st1,
                                                   const double *st2, const double *st3, const double *st4,
                                                   const int *llist) {
  using H = Halo<NDIM, NX, NY, NZ>;
  const int b = llist[blockIdx.x];
  const double *const st[5] = {st0, st1, st2, st3, st4};
  double *lh = P.lh + (size_t)P.slot[b] * 5 * H::n;
  for (int h = threadIdx.x; h < H::n; h += blockDim.x) {
    const int li = h % H::hx - 4, lj = NDIM > 1 ? (h / H::hx) % H::hy - 4 : 0, lk = NDIM > 2 ? h / (H::hx * H::hy) - 4 : 0;
    if (is_inside<NDIM, NX, NY, NZ>(li, lj, lk)) continue;
    double v[6];
    amr_guard<NDIM, NX, NY, NZ>(P, st, b, li, lj, lk, v);
    const double ekin = 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
    double eg = v[4];
    if (v[5] - ekin > rmax(P.smalle, P.eswitch * ekin)) eg = v[5] - ekin;
    lh[h] = v[0]; lh[H::n + h] = v[1]; lh[2 * H::n + h] = v[2]; lh[3 * H::n + h] = v[3]; lh[4 * H::n + h] = eg;
  }
  if (P.sp_lh) {
    for (int qh = threadIdx.x; qh < P.nsp * H::n; qh += blockDim.x) {
      const int q = qh / H::n, h = qh % H::n;
      const int li = h % H::hx - 4, lj = NDIM > 1 ? (h / H::hx) % H::hy - 4 : 0, lk = NDIM > 2 ? h / (H::hx * H::hy) - 4 : 0;
      if (is_inside<NDIM, NX, NY, NZ>(li, lj, lk)) continue;
      P.sp_lh[((size_t)P.slot[b] * P.nsp + q) * H::n + h] =
          amr_guard_spec<NDIM, NX, NY, NZ>(P, P.sp_ncells, b, li, lj, lk, q);
    }
  }
}

}  // namespace fhy
