// refine.cu -- the refinement criterion and the data movement of a regrid.
//
// k_estimate_error: gr_estimateBlkError (Grid/GridMain/AMR/
// gr_estimateBlkError.F90, Cartesian), Lohner's normalised second-derivative
// estimator of one variable, one CTA per block (leaves and parents).  The
// variable is staged with its 4 guard layers in shared memory (uniform grids:
// the in-kernel guard gather with the guard-cell EOS; AMR leaves: the leaf
// guard buffers; AMR parents: their guard-inclusive copies, the guard cells
// passed through the EOS rule of Eos_getData.F90:80-96), the first
// derivatives are taken on the fly, and the block error is the square root of
// the largest num/denom (an exact max reduction).  Compiled without FMA
// contraction, in the expression order of the CPU oracle.
#include "hy_launch.h"
#include "amr_kernels.cuh"

namespace fhy {

__device__ __forceinline__ double refvar(int var, double rho, double vx, double vy, double vz, double e, double gam1inv) {
  switch (var) {
    case FLASH_HY_REFVAR_DENS: return rho;
    case FLASH_HY_REFVAR_PRES: return rho * e * gam1inv;
    case FLASH_HY_REFVAR_VELX: return vx;
    case FLASH_HY_REFVAR_VELY: return vy;
    case FLASH_HY_REFVAR_VELZ: return vz;
    default: return e;
  }
}

template <int NDIM, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256) k_estimate_error(const DevParams P, int var, double filter, const int *list,
                                                        double *err) {
  using H = Halo<NDIM, NX, NY, NZ>;
  extern __shared__ __align__(16) double sV[];            // [H::n]
  __shared__ double wmax[8];
  __shared__ int whuge[8];
  const int b = list ? list[blockIdx.x] : blockIdx.x;
  const bool amr = P.leaf != nullptr;
  const bool parent = amr && !P.leaf[b];
  const int l = amr ? P.blk_level[b] : 1;
  const int3 bc = blk_coords(P, b);
  for (int h = threadIdx.x; h < H::n; h += blockDim.x) {
    const int li = h % H::hx - 4, lj = NDIM > 1 ? (h / H::hx) % H::hy - 4 : 0;
    const int lk = NDIM > 2 ? h / (H::hx * H::hy) - 4 : 0;
    double v;
    if (parent) {
      const double *g = P.gp + (size_t)P.slot[b] * 6 * H::n;
      const double rho = g[h], vx = g[H::n + h], vy = g[2 * H::n + h], vz = g[3 * H::n + h];
      double e = g[4 * H::n + h];
      if (!is_inside<NDIM, NX, NY, NZ>(li, lj, lk) && (var == FLASH_HY_REFVAR_PRES || var == FLASH_HY_REFVAR_EINT)) {
        const double E = g[5 * H::n + h];
        const double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
        if (E - ekin > rmax(P.smalle, P.eswitch * ekin)) e = E - ekin;
      }
      v = refvar(var, rho, vx, vy, vz, e, P.gam1inv);
    } else {
      double V[8];
      load_prim<NDIM, NX, NY, NZ, false>(P, b, bc, li, lj, lk, V);
      v = var == FLASH_HY_REFVAR_PRES ? V[HP] : refvar(var, V[HD], V[HVX], V[HVY], V[HVZ], V[HEI], P.gam1inv);
    }
    sV[h] = v;
  }
  __syncthreads();
  double delta[3], del[3] = {0., 0., 0.};
  blk_deltas(P, b, delta);
#pragma unroll
  for (int d = 0; d < NDIM; ++d) del[d] = 0.5e0 / delta[d];
  const int Nd[3] = {NX, NY, NZ}, cc[3] = {bc.x, bc.y, bc.z};
  int bs[3] = {0, 0, 0}, be[3] = {0, 0, 0}, len[3] = {1, 1, 1};
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    const int ext = amr ? P.at_ext[l][d] : (d == 0 ? P.nbx : (d == 1 ? P.nby : P.nbz));
    const bool lo = cc[d] == 0 && P.bc[2 * d] != FLASH_HY_BC_PERIODIC;
    const bool hi = cc[d] == ext - 1 && P.bc[2 * d + 1] != FLASH_HY_BC_PERIODIC;
    bs[d] = lo ? 0 : -2;
    be[d] = hi ? Nd[d] - 1 : Nd[d] + 1;
    len[d] = be[d] - bs[d] + 1;
  }
  const int st[3] = {1, H::hx, H::hx * H::hy};
  // (first-derivative axis, second-difference axis) in the order of the
  // estimator's delu2(1..SQNDIM)
  constexpr int NK = NDIM * NDIM;
  const int A[9][2] = {{0, 0}, {0, 1}, {1, 0}, {1, 1}, {0, 2}, {1, 2}, {2, 0}, {2, 1}, {2, 2}};
  double emax = 0.;
  int huge = 0;
  for (int q = threadIdx.x; q < len[0] * len[1] * len[2]; q += blockDim.x) {
    const int i = bs[0] + q % len[0], j = bs[1] + (q / len[0]) % len[1], k = bs[2] + q / (len[0] * len[1]);
    const int c0 = H::idx(i, j, k);
    double num = 0., denom = 0.;
#pragma unroll
    for (int kk = 0; kk < NK; ++kk) {
      const int a = A[kk][0], bb = A[kk][1];
      const int op = c0 + st[bb], om = c0 - st[bb];
      const double dup = (sV[op + st[a]] - sV[op - st[a]]) * del[a];
      const double dum = (sV[om + st[a]] - sV[om - st[a]]) * del[a];
      const double dap = (fabs(sV[op + st[a]]) + fabs(sV[op - st[a]])) * del[a];
      const double dam = (fabs(sV[om + st[a]]) + fabs(sV[om - st[a]])) * del[a];
      const double d2 = (dup - dum) * del[bb];
      const double d3 = (fabs(dup) + fabs(dum)) * del[bb];
      const double d4 = (dap + dam) * del[bb];
      num = num + d2 * d2;
      denom = denom + (d3 + (filter * d4)) * (d3 + (filter * d4));
    }
    if (denom == 0.0 && num != 0.0) huge = 1;
    else if (denom != 0.0) emax = rmax(emax, num / denom);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    emax = rmax(emax, __shfl_down_sync(0xffffffffu, emax, o));
    huge |= __shfl_down_sync(0xffffffffu, huge, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { wmax[w] = emax; whuge[w] = huge; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x + 31) / 32; ++q) { emax = rmax(emax, wmax[q]); huge |= whuge[q]; }
    err[b] = sqrt(huge ? DBL_MAX : emax);
  }
}

template <int NDIM, int NX, int NY, int NZ>
static int run_estimate(const ErrArgs &a) {
  using H = Halo<NDIM, NX, NY, NZ>;
  k_estimate_error<NDIM, NX, NY, NZ><<<a.n, 256, H::n * sizeof(double), a.stream>>>(a.P, a.var, a.filter, a.list,
                                                                                     a.err);
  return cudaGetLastError() == cudaSuccess ? 1 : -2;
}

int estimate_error(const ErrArgs &a, int ndim, int nx, int ny, int nz) {
  if (ndim == 2 && nx == 8 && ny == 8) return run_estimate<2, 8, 8, 1>(a);
  if (ndim == 2 && nx == 16 && ny == 16) return run_estimate<2, 16, 16, 1>(a);
  if (ndim == 3 && nx == 8 && ny == 8 && nz == 8) return run_estimate<3, 8, 8, 8>(a);
  return -1;
}

// ---------------------------------------------------------------------------
// data of a regridded hierarchy (gr_updateRefinement.F90:112-238)
// ---------------------------------------------------------------------------
// guard-inclusive copy (rho, v, e, E before the EOS) of the old leaves whose
// children are created, the data amr_prolong interpolates from
template <int NDIM, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256) k_node_halo(const DevParams P, const int *list, double *out) {
  constexpr int NCB = NX * NY * NZ;
  using H = Halo<NDIM, NX, NY, NZ>;
  const int b = list[blockIdx.x];
  const double *const st[5] = {P.s_in[0], P.s_in[1], P.s_in[2], P.s_in[3], P.s_in[4]};
  double *o = out + (size_t)blockIdx.x * (6 + P.nsp) * H::n;
  for (int h = threadIdx.x; h < H::n; h += blockDim.x) {
    const int li = h % H::hx - 4, lj = NDIM > 1 ? (h / H::hx) % H::hy - 4 : 0;
    const int lk = NDIM > 2 ? h / (H::hx * H::hy) - 4 : 0;
    double v[6];
    if (is_inside<NDIM, NX, NY, NZ>(li, lj, lk)) {
      const size_t off = (size_t)b * NCB + (size_t)((lk * NY + lj) * NX + li);
      v[0] = st[0][off]; v[1] = st[1][off]; v[2] = st[2][off]; v[3] = st[3][off]; v[4] = st[4][off];
      v[5] = node_E(P, b, off, v[4], v[1], v[2], v[3]);
    } else {
      amr_guard<NDIM, NX, NY, NZ>(P, st, b, li, lj, lk, v);
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) o[q * H::n + h] = v[q];
  }
  // species and mass scalars after the six state values
  for (int qh = threadIdx.x; qh < P.nsp * H::n; qh += blockDim.x) {
    const int q = qh / H::n, h = qh % H::n;
    const int li = h % H::hx - 4, lj = NDIM > 1 ? (h / H::hx) % H::hy - 4 : 0;
    const int lk = NDIM > 2 ? h / (H::hx * H::hy) - 4 : 0;
    o[(6 + q) * H::n + h] =
        is_inside<NDIM, NX, NY, NZ>(li, lj, lk)
            ? P.sp_in[(size_t)q * P.sp_ncells + (size_t)b * NCB + (size_t)((lk * NY + lj) * NX + li)]
            : amr_guard_spec<NDIM, NX, NY, NZ>(P, P.sp_ncells, b, li, lj, lk, q);
  }
}

// every new node: copy (how 0), derefined parent turned leaf (how 2) or new
// child prolonged from its old parent's copy (how 1); the EOS of
// Eos_wrapped(MODE_DENS_EI) on the leaves (Eos_getData.F90:80-96)
template <int NDIM, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256) k_regrid_fill(const RegridArgs a) {
  constexpr int NCB = NX * NY * NZ;
  using H = Halo<NDIM, NX, NY, NZ>;
  const int nb = blockIdx.x, o = a.src[nb], how = a.how[nb];
  const DevParams &Po = a.Po, &Pn = a.Pn;
  const bool leaf = Pn.leaf[nb];
  const int3 c3 = blk_coords(Pn, nb);
  const int cc[3] = {c3.x, c3.y, c3.z};
  for (int c = threadIdx.x; c < NCB; c += blockDim.x) {
    double v[6];
    const double *nh = a.nh + (size_t)(how == 1 ? a.slot[nb] : 0) * (6 + Pn.nsp) * H::n;
    const int lp[3] = {c % NX, (c / NX) % NY, c / (NX * NY)};
    if (how == 1) {
      prolong_linear<NDIM, NX, NY, NZ>(nh, cc, lp, v);
    } else {
      const size_t off = (size_t)o * NCB + c;
      v[0] = Po.s_in[0][off]; v[1] = Po.s_in[1][off]; v[2] = Po.s_in[2][off]; v[3] = Po.s_in[3][off];
      v[4] = Po.s_in[4][off];
      v[5] = node_E(Po, o, off, v[4], v[1], v[2], v[3]);
    }
    const size_t no = (size_t)nb * NCB + c;
    double e = v[4];
    if (leaf) {
      const double ekin = 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
      if (v[5] - ekin > rmax(Pn.smalle, Pn.eswitch * ekin)) e = v[5] - ekin;
    } else {
      Pn.pe[no] = v[5];
    }
    Pn.s_out[0][no] = v[0]; Pn.s_out[1][no] = v[1]; Pn.s_out[2][no] = v[2]; Pn.s_out[3][no] = v[3];
    Pn.s_out[4][no] = e;
    for (int q = 0; q < Pn.nsp; ++q)
      Pn.sp_out[(size_t)q * Pn.sp_ncells + no] =
          how == 1 ? prolong_scalar<NDIM, NX, NY, NZ>(nh, nh + (6 + q) * H::n, cc, lp)
                   : Po.sp_in[(size_t)q * Po.sp_ncells + (size_t)o * NCB + c];
  }
}

template <int NDIM, int NX, int NY, int NZ>
static int run_regrid(const RegridArgs &a) {
  using H = Halo<NDIM, NX, NY, NZ>;
  (void)sizeof(H);
  if (a.nref > 0) k_node_halo<NDIM, NX, NY, NZ><<<a.nref, 256, 0, a.stream>>>(a.Po, a.refl, a.nh);
  if (cudaGetLastError() != cudaSuccess) return -2;
  k_regrid_fill<NDIM, NX, NY, NZ><<<a.nnew, 256, 0, a.stream>>>(a);
  return cudaGetLastError() == cudaSuccess ? 2 : -2;
}

int regrid_fill(const RegridArgs &a, int ndim, int nx, int ny, int nz) {
  if (ndim == 2 && nx == 8 && ny == 8) return run_regrid<2, 8, 8, 1>(a);
  if (ndim == 2 && nx == 16 && ny == 16) return run_regrid<2, 16, 16, 1>(a);
  if (ndim == 3 && nx == 8 && ny == 8 && nz == 8) return run_regrid<3, 8, 8, 8>(a);
  return -1;
}

size_t halo_cells(int ndim, int nx, int ny, int nz) {
  return (size_t)(nx + 8) * (ndim > 1 ? ny + 8 : 1) * (ndim > 2 ? nz + 8 : 1);
}

}  // namespace fhy
