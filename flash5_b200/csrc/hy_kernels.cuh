// hy_kernels.cuh -- kernels of one unsplit hydro step on a uniform block grid.
//
// Device state: five block-major SoA arrays (dens, velx, vely, velz, eint) of
// the block interiors only.  Everything else FLASH keeps in UNK (PRES, GAMC,
// GAME, ENER, TEMP) is the gamma-law EOS of these five after every step
// (Eos_wrapped MODE_DENS_EI, eos_idealGamma.F90:323-335, Eos_putData.F90:
// 95-106), so it is recomputed where needed.  Guard cells are not stored: the
// kernels gather them from the neighbouring blocks (or the boundary
// condition) and apply the EOS to them, which is Grid_fillGuardCells with
// doEos (paramesh4/Grid_fillGuardCells.F90:227-569, Hydro.F90:121-123).
//
// One step = k_sig (transverse fluxes of every direction on the box of
// cells [-1, N]^d of every block) followed by one k_dir launch per direction
// (PPM + transverse + CTU corrections, HLLC, accumulation of the
// conservative update).  The last direction also finalises the update,
// applies hy_energyFix and the EOS, writes the new state and reduces the CFL
// time step per block.
#pragma once
#include "hy_core.cuh"
#include "exact_rs.cuh"
#include <float.h>

namespace fhy {

struct CflPart {          // per-block CFL reduction result
  double dt;              // cfl / max (|u_d| + c_s)/dx_d, DBL_MAX if 0
  int i, j, k, blk;       // 0-based interior cell of the winning cell
};

__device__ __forceinline__ int map_axis(int g, int n, int bclo, int bchi, int &flip) {
  if (g < 0) {
    if (bclo == -135) return ((g % n) + n) % n;
    if (bclo == -31) { flip = 1; return -1 - g; }
    return 0;
  }
  if (g >= n) {
    if (bchi == -135) return g % n;
    if (bchi == -31) { flip = 1; return 2 * n - 1 - g; }
    return n - 1;
  }
  return g;
}

// Offset of the stored cell that provides local cell (li,lj,lk) of block b.
template <int NDIM, int NX, int NY, int NZ>
__device__ __forceinline__ size_t cell_src(const DevParams &P, int b, int3 bc, int li, int lj, int lk,
                                           bool &inside, int &fx, int &fy, int &fz) {
  constexpr int NCB = NX * NY * NZ;
  inside = (li >= 0 && li < NX) && (NDIM < 2 || (lj >= 0 && lj < NY)) && (NDIM < 3 || (lk >= 0 && lk < NZ));
  fx = fy = fz = 0;
  if (inside) return (size_t)b * NCB + (size_t)((lk * NY + lj) * NX + li);
  int gx = map_axis(bc.x * NX + li, P.nbx * NX, P.bc[0], P.bc[1], fx);
  int gy = NDIM > 1 ? map_axis(bc.y * NY + lj, P.nby * NY, P.bc[2], P.bc[3], fy) : 0;
  int gz = NDIM > 2 ? map_axis(bc.z * NZ + lk, P.nbz * NZ, P.bc[4], P.bc[5], fz) : 0;
  int sb = P.blk_at[((gz / NZ) * P.nby + gy / NY) * P.nbx + gx / NX];
  return (size_t)sb * NCB + (size_t)(((gz % NZ) * NY + (gy % NY)) * NX + (gx % NX));
}

// Guard-inclusive box of a block (NGUARD = 4), the layout of the AMR guard
// buffers.
template <int NDIM, int NX, int NY, int NZ> struct Halo {
  static constexpr int hx = NX + 8, hy = NDIM > 1 ? NY + 8 : 1, hz = NDIM > 2 ? NZ + 8 : 1;
  static constexpr int n = hx * hy * hz;
  __device__ static __forceinline__ int idx(int li, int lj, int lk) {
    return ((lk + (NDIM > 2 ? 4 : 0)) * hy + (lj + (NDIM > 1 ? 4 : 0))) * hx + (li + 4);
  }
};

template <int NDIM, int NX, int NY, int NZ>
__device__ __forceinline__ bool is_inside(int li, int lj, int lk) {
  return (li >= 0 && li < NX) && (NDIM < 2 || (lj >= 0 && lj < NY)) && (NDIM < 3 || (lk >= 0 && lk < NZ));
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

// asynchronous 8- and 16-byte copies from global to shared memory
// (cp.async): a thread's copies are all in flight at once and hold no
// registers; cp.async.wait_all makes its own copies visible to it
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The source blocks of a block's guard cells on a uniform grid: entry
// (cz * 3 + cy) * 3 + cx for the side (0 below, 1 inside, 2 above) of each
// coordinate; threads 0..3^NDIM-1 write one entry each.
template <int NDIM, int NX, int NY, int NZ>
__device__ __forceinline__ void neighbour_table(const DevParams &P, int3 bc, int *nb) {
  constexpr int NNB = NDIM > 2 ? 27 : 9;
  if (threadIdx.x >= NNB) return;
  const int t = threadIdx.x, cx = t % 3, cy = (t / 3) % 3, cz = t / 9;
  int f;
  const int gx = map_axis(bc.x * NX + (cx == 0 ? -1 : (cx == 1 ? 0 : NX)), P.nbx * NX, P.bc[0], P.bc[1], f);
  const int gy = NDIM > 1 ? map_axis(bc.y * NY + (cy == 0 ? -1 : (cy == 1 ? 0 : NY)), P.nby * NY, P.bc[2], P.bc[3], f) : 0;
  const int gz = NDIM > 2 ? map_axis(bc.z * NZ + (cz == 0 ? -1 : (cz == 1 ? 0 : NZ)), P.nbz * NZ, P.bc[4], P.bc[5], f) : 0;
  nb[t] = P.blk_at[((gz / NZ) * P.nby + gy / NY) * P.nbx + gx / NX];
}

// Uniform grids: the cell that provides local cell (li, lj, lk), as cell_src,
// with the source block taken from the block's neighbour table nb (the
// source block depends only on whether each coordinate is below, inside or
// above the block: periodic wrap, mirror and clamp stay within one block).
template <int NDIM, int NX, int NY, int NZ>
__device__ __forceinline__ size_t cell_src_nb(const DevParams &P, int b, int3 bc, const int *nb, int li, int lj,
                                              int lk, int &fx, int &fy, int &fz) {
  constexpr int NCB = NX * NY * NZ;
  fx = fy = fz = 0;
  if (is_inside<NDIM, NX, NY, NZ>(li, lj, lk)) return (size_t)b * NCB + (size_t)((lk * NY + lj) * NX + li);
  const int gx = map_axis(bc.x * NX + li, P.nbx * NX, P.bc[0], P.bc[1], fx);
  const int gy = NDIM > 1 ? map_axis(bc.y * NY + lj, P.nby * NY, P.bc[2], P.bc[3], fy) : 0;
  const int gz = NDIM > 2 ? map_axis(bc.z * NZ + lk, P.nbz * NZ, P.bc[4], P.bc[5], fz) : 0;
  const int cx = li < 0 ? 0 : (li < NX ? 1 : 2), cy = NDIM > 1 ? (lj < 0 ? 0 : (lj < NY ? 1 : 2)) : 0;
  const int cz = NDIM > 2 ? (lk < 0 ? 0 : (lk < NZ ? 1 : 2)) : 0;
  return (size_t)nb[(cz * 3 + cy) * 3 + cx] * NCB + (size_t)(((gz % NZ) * NY + (gy % NY)) * NX + (gx % NX));
}


// Primitive slots of a cell as hy_getRiemannState sees it: interior cells
// straight from the state, guard cells after the guard-cell EOS.
template <int NDIM, int NX, int NY, int NZ, bool GAME = true>
__device__ __forceinline__ void load_prim(const DevParams &P, int b, int3 bc, int li, int lj, int lk, double V[8]) {
  if (P.lh && !is_inside<NDIM, NX, NY, NZ>(li, lj, lk)) {
    // AMR: the leaf guard buffer, filled (and passed through the EOS) by k_leaf_halo
    using H = Halo<NDIM, NX, NY, NZ>;
    const double *h = P.lh + (size_t)P.slot[b] * 5 * H::n + H::idx(li, lj, lk);
    const double rho = h[0], eg = h[4 * H::n];
    const double p = rho * eg * P.gam1inv;
    V[HD] = rho; V[HVX] = h[H::n]; V[HVY] = h[2 * H::n]; V[HVZ] = h[3 * H::n]; V[HP] = p;
    V[HGC] = P.gamma; V[HGE] = GAME ? p / (eg * rho) + 1 : 0.0; V[HEI] = eg;
    return;
  }
  bool inside; int fx, fy, fz;
  size_t o = cell_src<NDIM, NX, NY, NZ>(P, b, bc, li, lj, lk, inside, fx, fy, fz);
  double rho = __ldg(P.s_in[0] + o), vx = __ldg(P.s_in[1] + o), vy = __ldg(P.s_in[2] + o);
  double vz = __ldg(P.s_in[3] + o), e = __ldg(P.s_in[4] + o);
  if (fx) vx = -vx;
  if (fy) vy = -vy;
  if (fz) vz = -vz;
  double eg = e;
  if (!inside) {   // Eos_getData.F90:80-96 on ENER = eint + ekin of the source cell
    double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
    double ener = e + ekin;
    if (ener - ekin > rmax(P.smalle, P.eswitch * ekin)) eg = ener - ekin;
  }
  double p = rho * eg * P.gam1inv;
  V[HD] = rho; V[HVX] = vx; V[HVY] = vy; V[HVZ] = vz; V[HP] = p;
  // GAME (Eos_putData.F90:105-106) is only read for the cell's own face
  // states; stencil neighbours skip the division
  V[HGC] = P.gamma; V[HGE] = GAME ? p / (eg * rho) + 1 : 0.0; V[HEI] = eg;
}

template <int NDIM, int NX, int NY, int NZ> struct Box {
  static constexpr int bx = NX + 2, by = NDIM > 1 ? NY + 2 : 1, bz = NDIM > 2 ? NZ + 2 : 1;
  static constexpr int n = bx * by * bz;
  __device__ static __forceinline__ int idx(int i, int j, int k) {
    return ((k + (NDIM > 2)) * by + (j + (NDIM > 1))) * bx + (i + 1);
  }
};

__device__ __forceinline__ int3 blk_coords(const DevParams &P, int b) {
  return make_int3(P.blk_coord[3 * b], P.blk_coord[3 * b + 1], P.blk_coord[3 * b + 2]);
}

// Differences are taken in FP64 before any conversion to R, so the FP32
// path carries the relative precision of the differences, not of the values.
template <class R, int DIR>
__device__ __forceinline__ void sig_dir(const DevParams &P, const double *Vm, const double *Vc, const double *Vp,
                                        R sig[8], unsigned &st) {
  R c[8], dl[5], dr[5];
#pragma unroll
  for (int n = 0; n < 8; ++n) c[n] = R(Vc[n]);
#pragma unroll
  for (int n = 0; n < 5; ++n) { dl[n] = R(Vc[n] - Vm[n]); dr[n] = R(Vp[n] - Vc[n]); }
  Eig<R> e;
  eigen<R, DIR>(c, e, st);
  upwind_tflux_d<R, DIR>(P, dl, dr, R(Vc[HEI] - Vm[HEI]), R(Vp[HEI] - Vc[HEI]), e, sig);
}

// sig components kept in memory: dens, velx, vely, velz, pres, eint
__device__ __forceinline__ int sig_slot(int q) { return q < 5 ? q : HEI; }

// ---------------------------------------------------------------------------
// k_sig: transverse flux "sig" of every direction for the box cells
// (hy_DataReconstructNormalDir_PPM.F90:351-371 via hy_getRiemannState.F90:
// 471-637, which evaluates it for every cell of [lo-1, hi+1]^d).  The
// primitives of the box and of one layer beyond it along each axis are
// staged once in shared memory (cp.async through the neighbour table, then
// the guard cells' reflections and guard-cell EOS in place, the rules of
// load_prim); each box cell then reads its stencils from there.
// ---------------------------------------------------------------------------
// Stage rho, vx, vy, vz and e of the cells cell_of(c, i, j, k) selects
// (c in [0, n)) into sQ[5][n] as load_prim sees them: cp.async copies from
// the state (sources through the neighbour table nb; interior cells on AMR)
// or the leaf guard buffer (AMR, after the EOS), then, by the thread that
// issued them, the uniform grid's guard cells mirrored and passed through
// the guard-cell EOS (Eos_getData.F90:80-96 on ENER = eint + ekin of the
// source cell).  The caller synchronises before reading.
template <int NDIM, int NX, int NY, int NZ, class CellOf>
__device__ __forceinline__ void stage_prims(const DevParams &P, int b, int3 bc, int slot, const int *nb, double *sQ,
                                            int n, CellOf cell_of) {
  using H = Halo<NDIM, NX, NY, NZ>;
  constexpr int NCB = NX * NY * NZ;
  const bool amr = P.lh != nullptr;
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    int i, j, k;
    if (!cell_of(c, i, j, k)) continue;
    if (amr && !is_inside<NDIM, NX, NY, NZ>(i, j, k)) {
      const double *h = P.lh + (size_t)slot * 5 * H::n + H::idx(i, j, k);
#pragma unroll
      for (int v = 0; v < 5; ++v) cp_async8(sQ + v * n + c, h + v * H::n);
    } else {
      int fx, fy, fz;
      const size_t o = amr ? (size_t)b * NCB + (size_t)((k * NY + j) * NX + i)
                           : cell_src_nb<NDIM, NX, NY, NZ>(P, b, bc, nb, i, j, k, fx, fy, fz);
#pragma unroll
      for (int v = 0; v < 5; ++v) cp_async8(sQ + v * n + c, P.s_in[v] + o);
    }
  }
  cp_async_wait_all();
  if (amr) return;
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    int i, j, k;
    if (!cell_of(c, i, j, k) || is_inside<NDIM, NX, NY, NZ>(i, j, k)) continue;
    int f[3];
    cell_src_nb<NDIM, NX, NY, NZ>(P, b, bc, nb, i, j, k, f[0], f[1], f[2]);
    double vx = sQ[n + c], vy = sQ[2 * n + c], vz = sQ[3 * n + c];
    const double e = sQ[4 * n + c];
    if (f[0]) vx = -vx;
    if (f[1]) vy = -vy;
    if (f[2]) vz = -vz;
    double eg = e;
    const double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
    const double ener = e + ekin;
    if (ener - ekin > rmax(P.smalle, P.eswitch * ekin)) eg = ener - ekin;
    sQ[n + c] = vx; sQ[2 * n + c] = vy; sQ[3 * n + c] = vz; sQ[4 * n + c] = eg;
  }
}

// the primitive slots of load_prim<..., GAME> from the staged cell e
template <bool GAME = false>
__device__ __forceinline__ void staged_prim(const DevParams &P, const double *sQ, int n, int e, double V[8]) {
  const double rho = sQ[e], eg = sQ[4 * n + e];
  const double p = rho * eg * P.gam1inv;
  V[HD] = rho; V[HVX] = sQ[n + e]; V[HVY] = sQ[2 * n + e]; V[HVZ] = sQ[3 * n + e]; V[HP] = p;
  V[HGC] = P.gamma; V[HGE] = GAME ? p / (eg * rho) + 1 : 0.0; V[HEI] = eg;
}

// The lines of interior cells along DIR with four cells beyond the block on
// either side (the stencil of the FP64 direction kernel: PPM +-2, the
// flattening's pressures +-3 around line cells [-1, N]), in the thread
// order of the line cells.
template <int NDIM, int NX, int NY, int NZ, int DIR>
struct LineStage {
  static constexpr int sx = DIR == 1 ? NX + 8 : NX, sy = NDIM > 1 ? (DIR == 2 ? NY + 8 : NY) : 1,
                       sz = NDIM > 2 ? (DIR == 3 ? NZ + 8 : NZ) : 1;
  static constexpr int n = sx * sy * sz;
  static constexpr int step = DIR == 1 ? 1 : (DIR == 2 ? sx : sx * sy);
  __device__ static __forceinline__ int idx(int i, int j, int k) {
    return ((k + 4 * (DIR == 3)) * sy + (j + 4 * (DIR == 2))) * sx + (i + 4 * (DIR == 1));
  }
  __device__ static __forceinline__ void decode(int c, int &i, int &j, int &k) {
    i = c % sx - 4 * (DIR == 1);
    j = NDIM > 1 ? (c / sx) % sy - 4 * (DIR == 2) : 0;
    k = NDIM > 2 ? c / (sx * sy) - 4 * (DIR == 3) : 0;
  }
};

template <int NDIM, int NX, int NY, int NZ>
struct SigStage {
  using E = Ext<NDIM, NX, NY, NZ, 2>;
  static constexpr int NNB = NDIM > 2 ? 27 : 9;
  // rho, vx, vy, vz and e (after the guard-cell EOS) of the staged cells; the neighbour table
  static constexpr size_t smem_bytes() { return (size_t)5 * E::n * sizeof(double) + NNB * sizeof(int); }
  // staged: at most one coordinate outside the box [-1, N]
  __device__ static __forceinline__ bool needed(int i, int j, int k) {
    const int c[3] = {i, j, k}, n[3] = {NX, NY, NZ};
    int out = 0;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) out += c[d] < -1 || c[d] > n[d];
    return out <= 1;
  }
};

// 3D: three CTAs per SM where shared memory allows it (FP32 sig); the FP64
// kernel keeps two, which its registers need
template <int NDIM, int NX, int NY, int NZ, class R, int VAR>
__global__ void __launch_bounds__(320, NDIM > 2 ? (sizeof(R) == 4 ? 3 : 2) : 1) k_sig(const DevParams P,
                                                                                     R *__restrict__ SIG) {
  using B = Box<NDIM, NX, NY, NZ>;
  using SG = SigStage<NDIM, NX, NY, NZ>;
  using E = typename SG::E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sQ = reinterpret_cast<double *>(smem_raw);     // [5][E::n]
  int *sNb = reinterpret_cast<int *>(sQ + 5 * E::n);     // [NNB]
  const int b = P.blk_list ? P.blk_list[blockIdx.x] : blockIdx.x;
  const int3 bc = blk_coords(P, b);
  const int slot = P.slot ? P.slot[b] : (int)blockIdx.x;
  const bool amr = P.lh != nullptr;
  if (!amr) neighbour_table<NDIM, NX, NY, NZ>(P, bc, sNb);
  __syncthreads();
  stage_prims<NDIM, NX, NY, NZ>(P, b, bc, slot, sNb, sQ, E::n, [](int c, int &i, int &j, int &k) {
    E::decode(c, i, j, k);
    return SG::needed(i, j, k);
  });
  __syncthreads();
  unsigned st = 0;
  for (int t = threadIdx.x; t < B::n; t += blockDim.x) {
    int i = t % B::bx - 1, j = NDIM > 1 ? (t / B::bx) % B::by - 1 : 0, k = NDIM > 2 ? t / (B::bx * B::by) - 1 : 0;
    const int e = E::idx(i, j, k);
    double Vc[8], Vm[8], Vp[8];
    staged_prim(P, sQ, E::n, e, Vc);
#pragma unroll
    for (int d = 1; d <= NDIM; ++d) {
      const int es = d == 1 ? 1 : (d == 2 ? E::ex : E::ex * E::ey);
      staged_prim(P, sQ, E::n, e - es, Vm);
      staged_prim(P, sQ, E::n, e + es, Vp);
      R s[8];
      if (d == 1) sig_dir<R, 1>(P, Vm, Vc, Vp, s, st);
      else if (d == 2) sig_dir<R, 2>(P, Vm, Vc, Vp, s, st);
      else sig_dir<R, 3>(P, Vm, Vc, Vp, s, st);
      R *dst = SIG + ((size_t)(P.slot ? P.slot[b] : (int)blockIdx.x) * NDIM + (d - 1)) * 6 * B::n + t;
#pragma unroll
      for (int q = 0; q < 6; ++q) dst[(size_t)q * B::n] = s[sig_slot(q)];
    }
  }
  if (st) atomicOr(P.status, st);
}

__device__ __forceinline__ void load_sig(const float *p, size_t stride, float s[8]) {
#pragma unroll
  for (int q = 0; q < 6; ++q) s[sig_slot(q)] = p[q * stride];
  s[HGC] = 0.f; s[HGE] = 0.f;
}
__device__ __forceinline__ void load_sig(const double *p, size_t stride, double s[8]) {
#pragma unroll
  for (int q = 0; q < 6; ++q) s[sig_slot(q)] = p[q * stride];
  s[HGC] = 0.; s[HGE] = 0.;
}

// deterministic (max key, first index) reduction for the CFL step
struct CflCand { double key, val; int idx; };
__device__ __forceinline__ void cfl_merge(CflCand &a, const CflCand &b) {
  if (b.key > a.key || (b.key == a.key && b.idx < a.idx)) a = b;
}

template <int NX, int NY, int NZ>
__device__ void cfl_block_reduce(CflCand c, int blk, double cfl, CflPart *part) {
  __shared__ CflCand red[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    CflCand b;
    b.key = __shfl_down_sync(0xffffffffu, c.key, o);
    b.val = __shfl_down_sync(0xffffffffu, c.val, o);
    b.idx = __shfl_down_sync(0xffffffffu, c.idx, o);
    if (lane + o < 32) cfl_merge(c, b);
  }
  if (lane == 0) red[w] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    CflCand a = red[0];
    for (int q = 1; q < (int)(blockDim.x + 31) / 32; ++q) cfl_merge(a, red[q]);
    CflPart r;
    // Hydro_computeDt.F90:265-284: the winner is the first cell whose
    // dt_ltemp*cfl exceeds every earlier one; dt = cfl / dt_ltemp
    if (a.key > 0.0) {
      r.dt = cfl / a.val;
      r.i = a.idx % NX; r.j = (a.idx / NX) % NY; r.k = a.idx / (NX * NY);
    } else {
      r.dt = DBL_MAX; r.i = r.j = r.k = -1;
    }
    r.blk = blk;
    part[blk] = r;
  }
}

// ---------------------------------------------------------------------------
// exact Riemann face flux (no FLASH5 counterpart; Toro ch. 4, exact_rs.cuh)
// ---------------------------------------------------------------------------
__device__ __forceinline__ xrs::Side side_of(const double *V, int n, const xrs::Gas &G, unsigned &st) {
  const double c2 = G.g * V[HP] / V[HD];
  if (!(c2 > 0.0)) st |= ST_NEG_SOUND;
  return xrs::make_side(V[HD], V[n], V[HP], sqrt(c2), G);
}

// keep a hashed sample of the face states (two-rarefaction guess inexact) for
// training the learned guess
__device__ __forceinline__ void harvest_face(const DevParams &P, const xrs::Side &L, const xrs::Side &R, double g,
                                             unsigned key) {
  unsigned h = key * 2654435761u;
  h ^= h >> 15; h *= 2246822519u; h ^= h >> 13;
  if (h & P.harvest_mask) return;
  const unsigned long long k = atomicAdd(P.harvest_n, 1ull);
  if ((long long)k >= P.harvest_cap) return;
  const long long c = P.harvest_cap;
  double *S = P.harvest;
  S[k] = L.d; S[c + k] = L.u; S[2 * c + k] = L.p;
  S[3 * c + k] = R.d; S[4 * c + k] = R.u; S[5 * c + k] = R.p; S[6 * c + k] = g;
}

// Godunov flux from the exact solution, Newton from the two-rarefaction guess
template <int DIR>
__device__ __forceinline__ void exact_face(const DevParams &P, const xrs::Gas &G, const double *VL, const double *VR,
                                           double F[6], unsigned &st) {
  const xrs::Side L = side_of(VL, DIR, G, st), R = side_of(VR, DIR, G, st);
  const bool vac = xrs::vacuum(L, R, G);
  xrs::Star S{0.0, 0.5 * (L.u + R.u), 0.0};
  if (!vac) {
    const xrs::SideK kl = xrs::side_k(L, G), kr = xrs::side_k(R, G);
    if (xrs::newton(L, R, kl, kr, G, xrs::tr_w(L, R, kl, kr, G), P.rs_tol, P.rs_max_iter, S) < 0) st |= ST_NEWTON;
  }
  xrs::godunov_flux<DIR>(VL, VR, L, R, G, S, vac, F);
}

// ---------------------------------------------------------------------------
// AMR flux register (Grid_putFluxData / Grid_conserveFluxes with flux
// densities): a leaf whose neighbour across a DIR face is coarser stores its
// boundary face fluxes; a leaf whose neighbour there is a parent replaces
// its boundary face fluxes by the average of the touching fine leaves'
// stored fluxes.  Levels are launched finest first, so the fine fluxes are
// in place.  fidx(along, t1, t2) gives the position of a face in sF, t1/t2
// the tangential coordinates (y, z for x faces; x, z for y; x, y for z).
// ---------------------------------------------------------------------------
// The register of nv flux components per face: reg[(slot * 2 NDIM + face
// side) * NF * nv + face * nv + v]; the hydro's is P.freg with the NFLX
// fluxes, the species pass keeps one register per species.
template <int NDIM, int NX, int NY, int NZ, int DIR, class FaceIdx>
__device__ void flux_register_v(const DevParams &P, int b, int3 bc, double *sF, int fstride, FaceIdx fidx,
                                double *reg, int nv) {
  constexpr int N = DIR == 1 ? NX : (DIR == 2 ? NY : NZ);
  constexpr int n1 = DIR == 1 ? NY : NX;
  constexpr int n2 = NDIM > 2 ? (DIR == 3 ? NY : NZ) : 1;
  constexpr int NF = n1 * n2;
  constexpr int T1 = DIR == 1 ? 1 : 0, T2 = DIR == 3 ? 1 : 2;
  const int l = P.blk_level[b];
  for (int s = 0; s < 2; ++s) {
    int pos[3] = {bc.x, bc.y, NDIM > 2 ? bc.z : 0};
    pos[DIR - 1] += s ? 1 : -1;
    const int ext = P.at_ext[l][DIR - 1];
    if (pos[DIR - 1] < 0 || pos[DIR - 1] >= ext) {
      if (P.bc[2 * (DIR - 1) + s] != -135) continue;          // periodic only
      pos[DIR - 1] = (pos[DIR - 1] + ext) % ext;
    }
    const int m = at_node(P, l, pos[0], pos[1], pos[2]);
    const int along = s ? N : 0;
    if (m < 0) {
      double *dst = reg + ((size_t)P.slot[b] * 2 * NDIM + 2 * (DIR - 1) + s) * NF * nv;
      for (int q = threadIdx.x; q < NF * nv; q += blockDim.x) {
        const int face = q / nv, v = q % nv;
        dst[q] = sF[v * fstride + fidx(along, face % n1, face / n1)];
      }
    } else if (!P.leaf[m]) {
      const double w = NDIM > 2 ? 0.25 : 0.5;
      for (int q = threadIdx.x; q < NF * nv; q += blockDim.x) {
        const int face = q / nv, v = q % nv, q1 = face % n1, q2 = face / n1;
        int o[3] = {0, 0, 0};
        o[DIR - 1] = s ? 0 : 1;
        o[T1] = q1 >= n1 / 2;
        if (NDIM > 2) o[T2] = q2 >= n2 / 2;
        const int f = at_node(P, l + 1, 2 * pos[0] + o[0], 2 * pos[1] + o[1], NDIM > 2 ? 2 * pos[2] + o[2] : 0);
        const double *src = reg + ((size_t)P.slot[f] * 2 * NDIM + 2 * (DIR - 1) + (1 - s)) * NF * nv;
        double acc = 0.0;
        for (int r2 = 0; r2 <= (NDIM > 2 ? 1 : 0); ++r2)
          for (int r1 = 0; r1 <= 1; ++r1) {
            const int f1 = 2 * (q1 - o[T1] * (n1 / 2)) + r1, f2 = NDIM > 2 ? 2 * (q2 - o[T2] * (n2 / 2)) + r2 : 0;
            acc = acc + w * src[(f1 + n1 * f2) * nv + v];
          }
        sF[v * fstride + fidx(along, q1, q2)] = acc;
      }
    }
  }
}

template <int NDIM, int NX, int NY, int NZ, int DIR, class FaceIdx>
__device__ __forceinline__ void flux_register(const DevParams &P, int b, int3 bc, double *sF, int fstride,
                                              FaceIdx fidx) {
  flux_register_v<NDIM, NX, NY, NZ, DIR>(P, b, bc, sF, fstride, fidx, P.freg, NFLX);
}

// ---------------------------------------------------------------------------
// Stored fluxes of the split step: per block and direction the 8 flux
// components at the faces in FLASH's flx(var, i, j, k) face order (the
// DIR index runs over N+1 faces), stored component-major, then the n+1/2
// pressure sum (N05 + P05) of every interior cell.  fidx(along, t1, t2)
// gives a face's (or, with along in [0, N), a cell's) position in the
// kernel's shared arrays.
// ---------------------------------------------------------------------------
template <int NDIM, int NX, int NY, int NZ> struct FluxStore {
  static constexpr int NCB = NX * NY * NZ;
  static constexpr int NF = (NX + 1) * NY * NZ;            // square blocks: the same for every direction
  static constexpr int per_dir = NFLX * NF + NCB;
  __device__ static __forceinline__ double *base(const DevParams &P, int b, int dir) {
    return P.fstore + ((size_t)b * NDIM + (dir - 1)) * per_dir;
  }
};

template <int NDIM, int NX, int NY, int NZ, int DIR>
__device__ __forceinline__ void face_coords(int f, int &along, int &t1, int &t2) {
  constexpr int fx = NX + (DIR == 1), fy = NY + (DIR == 2);
  const int i = f % fx, j = (f / fx) % fy, k = f / (fx * fy);
  along = DIR == 1 ? i : (DIR == 2 ? j : k);
  t1 = DIR == 1 ? j : i;
  t2 = DIR == 3 ? j : k;
}

// store: sF faces and the cell pressure sums (sp(t) for a cell position t)
template <int NDIM, int NX, int NY, int NZ, int DIR, class T, class FaceIdx, class CellSp>
__device__ void flux_store(const DevParams &P, int b, const T *sF, int fstride, FaceIdx fidx, CellSp sp) {
  using FS = FluxStore<NDIM, NX, NY, NZ>;
  double *o = FS::base(P, b, DIR);
  for (int q = threadIdx.x; q < NFLX * FS::NF; q += blockDim.x) {
    const int v = q / FS::NF, f = q % FS::NF;
    int a, t1, t2;
    face_coords<NDIM, NX, NY, NZ, DIR>(f, a, t1, t2);
    o[q] = double(sF[v * fstride + fidx(a, t1, t2)]);
  }
  for (int c = threadIdx.x; c < FS::NCB; c += blockDim.x) {
    const int i = c % NX, j = (c / NX) % NY, k = c / (NX * NY);
    const int a = DIR == 1 ? i : (DIR == 2 ? j : k), t1 = DIR == 1 ? j : i, t2 = DIR == 3 ? j : k;
    o[NFLX * FS::NF + c] = sp(fidx(a, t1, t2));
  }
}

// ---------------------------------------------------------------------------
// k_dir: one direction of the unsplit update for one block per CTA.
//   phase 1: face states W-/W+ of the line cells (c_DIR in [-1, N], other
//            coordinates interior) -- PPM (hy_dataReconstOneStep.F90:485-
//            716), transverse corrections (:918-951), last negativity
//            check (:1120-1154), 3D full-CTU cross terms and positivity
//            fallback (hy_getRiemannState.F90:956-1313)
//   phase 2: HLLC (RS = 0) or the exact solver (RS = 1) at the N+1 faces
//            of every line plus the auxiliary
//            internal-energy and volume fluxes (hy_getFaceFlux.F90:283-442)
//   phase 3: accumulation of the conservative update in direction order
//            x, y, z (updateConservedVariable, hy_unsplitUpdate.F90:1187-
//            1242); the last direction finishes the cell: internal-energy
//            update with the n+1/2 pressure (:657-672, hy_getFaceFlux.F90:
//            551-557 and y/z analogues), hy_energyFix (:188-253), the EOS
//            and the CFL reduction (Hydro_computeDt.F90:186-290).
// ---------------------------------------------------------------------------
template <int NDIM, int NX, int NY, int NZ, class R, int DIR>
struct DirGeom {
  static constexpr int rx = DIR == 1 ? NX + 2 : NX;
  static constexpr int ry = NDIM > 1 ? (DIR == 2 ? NY + 2 : NY) : 1;
  static constexpr int rz = NDIM > 2 ? (DIR == 3 ? NZ + 2 : NZ) : 1;
  static constexpr int n = rx * ry * rz;
  static constexpr int stride = DIR == 1 ? 1 : (DIR == 2 ? rx : rx * ry);
  static constexpr int nd = DIR == 1 ? NX : (DIR == 2 ? NY : NZ);
  __device__ static __forceinline__ void decode(int t, int &i, int &j, int &k) {
    i = t % rx - (DIR == 1);
    j = NDIM > 1 ? (t / rx) % ry - (DIR == 2) : 0;
    k = NDIM > 2 ? t / (rx * ry) - (DIR == 3) : 0;
  }
  __device__ static __forceinline__ int along(int i, int j, int k) { return DIR == 1 ? i : (DIR == 2 ? j : k); }
  // line-cell index of cell (i, j, k), the inverse of decode
  __device__ static __forceinline__ int idx(int i, int j, int k) {
    return ((k + (DIR == 3)) * ry + (j + (DIR == 2))) * rx + (i + (DIR == 1));
  }
  static constexpr size_t smem_bytes() { return (size_t)n * (14 + NFLX) * sizeof(R); }
};
// per-slot offset of a direction's line cells in sp_mf / sp_fb
template <int NDIM, int NX, int NY, int NZ, int DIR>
__device__ __forceinline__ size_t sp_line_base(int slot) {
  using L = DirGeom<NDIM, NX, NY, NZ, double, DIR>;
  return ((size_t)slot * NDIM + (DIR - 1)) * L::n;
}

// slots stored for the face states: dens, velx, vely, velz, pres, game, eint
__device__ __forceinline__ int wslot(int q) { return q < 5 ? q : q + 1; }

template <int NDIM, int NX, int NY, int NZ, class R, int DIR, bool FIRST, bool LAST, int VAR, int RS>
__global__ void __launch_bounds__(320) k_dir(const DevParams P, const R *__restrict__ SIG, double *__restrict__ ACC,
                                             double *__restrict__ AUX, size_t ncells, CflPart *part) {
  using G = DirGeom<NDIM, NX, NY, NZ, R, DIR>;
  using B = Box<NDIM, NX, NY, NZ>;
  constexpr int NCB = NX * NY * NZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *sWp = reinterpret_cast<R *>(smem_raw);     // [7][n]
  R *sWm = sWp + 7 * G::n;                       // [7][n]
  R *sF = sWm + 7 * G::n;                        // [8][n]
  const int b = P.blk_list ? P.blk_list[blockIdx.x] : blockIdx.x;
  const int3 bc = blk_coords(P, b);
  unsigned st = 0;
  const double dt = P.dt_dev ? *P.dt_dev : P.dt;
  double del[3];
  blk_deltas(P, b, del);
  const double delta = del[DIR - 1];
  const R dtn = R(dt / delta);
  const R hdtx = R(0.5 * dt / del[0]), hdty = R(0.5 * dt / del[1]), hdtz = R(0.5 * dt / del[2]);
  const R *sigb = SIG + (size_t)(P.slot ? P.slot[b] : (int)blockIdx.x) * NDIM * 6 * B::n;

  auto fidx = [](int along, int t1, int t2) {
    const int i = DIR == 1 ? along : t1, j = DIR == 1 ? t1 : (DIR == 2 ? along : t2),
              k = DIR == 3 ? along : (NDIM > 2 ? t2 : 0);
    return ((k + (DIR == 3)) * G::ry + (j + (DIR == 2))) * G::rx + (i + (DIR == 1));
  };
  if (P.fmode != 3) {
  // ---------------- phase 0: the stencil of every line, staged once ---------
  // (in the flux array, unused until phase 2: 5 (N+8) <= 8 (N+2) for N >= 8)
  using LS = LineStage<NDIM, NX, NY, NZ, DIR>;
  static_assert(5 * LS::n <= NFLX * G::n, "line stage fits the flux array");
  __shared__ int sNb[NDIM > 2 ? 27 : 9];
  double *sQ = reinterpret_cast<double *>(sF);
  if (P.lh == nullptr) {
    neighbour_table<NDIM, NX, NY, NZ>(P, bc, sNb);
    __syncthreads();
  }
  stage_prims<NDIM, NX, NY, NZ>(P, b, bc, P.slot ? P.slot[b] : (int)blockIdx.x, sNb, sQ, LS::n,
                                [](int c, int &i, int &j, int &k) {
                                  LS::decode(c, i, j, k);
                                  return true;
                                });
  __syncthreads();
  // ---------------- phase 1: face states of the line cells ----------------
  for (int t = threadIdx.x; t < G::n; t += blockDim.x) {
    int i, j, k;
    G::decode(t, i, j, k);
    const int e0 = LS::idx(i, j, k);
    R V5[5][8];
    double Vd[8];
#pragma unroll
    for (int s = -2; s <= 2; ++s) {
      if (s == 0) staged_prim<true>(P, sQ, LS::n, e0, Vd);
      else staged_prim<false>(P, sQ, LS::n, e0 + s * LS::step, Vd);
#pragma unroll
      for (int n = 0; n < 8; ++n) V5[s + 2][n] = R(Vd[n]);
    }
    R flat = R(0);
    if (P.use_flattening) {
      R p7[7], u7[7];
      const int em = e0 - 3 * LS::step, ep = e0 + 3 * LS::step;
      p7[0] = R(sQ[em] * sQ[4 * LS::n + em] * P.gam1inv);
      p7[6] = R(sQ[ep] * sQ[4 * LS::n + ep] * P.gam1inv);
#pragma unroll
      for (int s = 0; s < 5; ++s) { p7[s + 1] = V5[s][HP]; u7[s + 1] = V5[s][Slots<DIR>::v1]; }
      u7[0] = R(0); u7[6] = R(0);
      flat = flat_coeff(p7, u7);
    }
    if (P.sp_flat) P.sp_flat[sp_line_base<NDIM, NX, NY, NZ, DIR>(P.slot ? P.slot[b] : (int)blockIdx.x) + t] = double(flat);
    R Wp[8], Wm[8];
    ppm_cell<R, DIR>(P, V5, flat, dtn, R(delta), Wp, Wm, st);
    const R *Vc = V5[2];
    // transverse corrections with the sig of the other directions (same cell)
    const int bi = B::idx(i, j, k);
    R sx[8], sy[8], sz[8];
    if (DIR != 1) load_sig(sigb + 0 * 6 * B::n + bi, B::n, sx);
    if (NDIM > 1 && DIR != 2) load_sig(sigb + 1 * 6 * B::n + bi, B::n, sy);
    if (NDIM > 2 && DIR != 3) load_sig(sigb + 2 * 6 * B::n + bi, B::n, sz);
    const int sl[6] = {0, 1, 2, 3, 4, 7};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      int n = sl[q];
      if (NDIM == 2) {
        if (DIR == 1) { Wm[n] = Wm[n] - hdty * sy[n]; Wp[n] = Wp[n] - hdty * sy[n]; }
        else          { Wm[n] = Wm[n] - hdtx * sx[n]; Wp[n] = Wp[n] - hdtx * sx[n]; }
      } else {
        if (DIR == 1)      { Wm[n] = Wm[n] - hdty * sy[n] - hdtz * sz[n]; Wp[n] = Wp[n] - hdty * sy[n] - hdtz * sz[n]; }
        else if (DIR == 2) { Wm[n] = Wm[n] - hdtx * sx[n] - hdtz * sz[n]; Wp[n] = Wp[n] - hdtx * sx[n] - hdtz * sz[n]; }
        else               { Wm[n] = Wm[n] - hdtx * sx[n] - hdty * sy[n]; Wp[n] = Wp[n] - hdtx * sx[n] - hdty * sy[n]; }
      }
    }
    if (Wm[HD] < R(0) || Wp[HD] < R(0) || Wm[HP] < R(0) || Wp[HP] < R(0)) {
#pragma unroll
      for (int n = 0; n < 8; ++n) { Wm[n] = Vc[n]; Wp[n] = Vc[n]; }
    }
    if (NDIM == 3 && P.use_ctu) {
      // axis / sig direction pairs of hy_getRiemannState.F90:999-1022,
      // 1101-1124, 1204-1227
      constexpr int A1 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1), S1 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2);
      constexpr int A2 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2), S2 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1);
      const double dA = del[A1 - 1], dB = del[A2 - 1];
      const R fac = R(dt * dt / (6. * (DIR == 1 ? del[1] : (DIR == 2 ? del[2] : del[0])) *
                                 (DIR == 1 ? del[2] : (DIR == 2 ? del[0] : del[1]))));
      (void)dA; (void)dB;
      R T1[8], T2[8];
      {
        R sm[8], s0[8], sp[8];
        const R *base = sigb + (size_t)(S1 - 1) * 6 * B::n;
        load_sig(base + B::idx(i - (A1 == 1), j - (A1 == 2), k - (A1 == 3)), B::n, sm);
        load_sig(base + bi, B::n, s0);
        load_sig(base + B::idx(i + (A1 == 1), j + (A1 == 2), k + (A1 == 3)), B::n, sp);
        Eig<R> e;
        eigen<R, A1>(Vc, e, st);
        upwind_tflux<R, A1>(P, sm, s0, sp, e, T1);
      }
      {
        R sm[8], s0[8], sp[8];
        const R *base = sigb + (size_t)(S2 - 1) * 6 * B::n;
        load_sig(base + B::idx(i - (A2 == 1), j - (A2 == 2), k - (A2 == 3)), B::n, sm);
        load_sig(base + bi, B::n, s0);
        load_sig(base + B::idx(i + (A2 == 1), j + (A2 == 2), k + (A2 == 3)), B::n, sp);
        Eig<R> e;
        eigen<R, A2>(Vc, e, st);
        upwind_tflux<R, A2>(P, sm, s0, sp, e, T2);
      }
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        int n = sl[q];
        Wp[n] = Wp[n] + (T1[n] + T2[n]) * fac;
        Wm[n] = Wm[n] + (T1[n] + T2[n]) * fac;
      }
      const bool fb = Wp[HD] <= R(0) || Wm[HD] <= R(0) || Wp[HP] <= R(0) || Wm[HP] <= R(0);
      if (fb) {
#pragma unroll
        for (int n = 0; n < 8; ++n) { Wm[n] = Vc[n]; Wp[n] = Vc[n]; }
      }
      if (P.sp_fb) P.sp_fb[sp_line_base<NDIM, NX, NY, NZ, DIR>(P.slot ? P.slot[b] : (int)blockIdx.x) + t] = fb;
    }
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      sWp[q * G::n + t] = Wp[wslot(q)];
      sWm[q * G::n + t] = Wm[wslot(q)];
    }
  }
  __syncthreads();

  // ---------------- phase 2: Riemann problems at the faces ----------------
  const R gam = R(P.gamma);
  for (int t = threadIdx.x; t < G::n; t += blockDim.x) {
    int i, j, k;
    G::decode(t, i, j, k);
    if (G::along(i, j, k) < 0) continue;
    R VL[8], VR[8];
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      VL[wslot(q)] = sWp[q * G::n + t - G::stride];
      VR[wslot(q)] = sWm[q * G::n + t];
    }
    VL[HGC] = gam; VR[HGC] = gam;
    R F[6];
    if constexpr (RS == 1) exact_face<DIR>(P, P.gas, VL, VR, F, st);
    else hllc<R, DIR>(P, VL, VR, F, st);
#pragma unroll
    for (int n = 0; n < 6; ++n) sF[n * G::n + t] = F[n];
    R fv = R(0), fe = R(0);
    if (P.use_aux_eint) {                         // hy_getFaceFlux.F90:433-442
      if (F[FDENS] > R(0)) { fv = F[FDENS] / VL[HD]; fe = F[FDENS] * VL[HEI]; }
      else { fv = F[FDENS] / VR[HD]; fe = F[FDENS] * VR[HEI]; }
    }
    sF[FEINT * G::n + t] = fe;
    sF[FVOLU * G::n + t] = fv;
    if (P.sp_mf) P.sp_mf[sp_line_base<NDIM, NX, NY, NZ, DIR>(P.slot ? P.slot[b] : (int)blockIdx.x) + t] = double(F[FDENS]);
  }
  __syncthreads();
  if constexpr (sizeof(R) == 8) {
    if (P.freg) {       // AMR: fine/coarse faces
      flux_register<NDIM, NX, NY, NZ, DIR>(P, b, bc, sF, G::n, [](int along, int t1, int t2) {
        const int i = DIR == 1 ? along : t1, j = DIR == 1 ? t1 : (DIR == 2 ? along : t2),
                  k = DIR == 3 ? along : (NDIM > 2 ? t2 : 0);
        return ((k + (DIR == 3)) * G::ry + (j + (DIR == 2))) * G::rx + (i + (DIR == 1));
      });
      __syncthreads();
    }
  }

  } else {
    // replay: the stored fluxes, and the stored pressure sums in place of
    // the face-state sum N05 + P05 of phase 3
    using FS = FluxStore<NDIM, NX, NY, NZ>;
    const double *src = FS::base(P, b, DIR);
    for (int q = threadIdx.x; q < NFLX * FS::NF; q += blockDim.x) {
      const int v = q / FS::NF, f = q % FS::NF;
      int a, t1, t2;
      face_coords<NDIM, NX, NY, NZ, DIR>(f, a, t1, t2);
      sF[v * G::n + fidx(a, t1, t2)] = R(src[q]);
    }
    for (int c = threadIdx.x; c < FS::NCB; c += blockDim.x) {
      const int i = c % NX, j = (c / NX) % NY, k = c / (NX * NY);
      const int t = fidx(DIR == 1 ? i : (DIR == 2 ? j : k), DIR == 1 ? j : i, DIR == 3 ? j : k);
      sWm[4 * G::n + t] = R(src[NFLX * FS::NF + c]);
      sWp[4 * G::n + t] = R(0);
    }
    __syncthreads();
  }
  if (P.fmode == 1 || P.fmode == 2) {
    flux_store<NDIM, NX, NY, NZ, DIR>(P, b, sF, G::n, fidx, [&](int t) {
      return double(sWm[4 * G::n + t]) + double(sWp[4 * G::n + t]);
    });
    if (P.fmode == 2) {
      if (st) atomicOr(P.status, st);
      return;
    }
  }

  // ---------------- phase 3: conservative update ----------------
  const double dtd = dt / delta;
  CflCand cand; cand.key = 0.0; cand.val = 0.0; cand.idx = 0x7fffffff;
  for (int t = threadIdx.x; t < G::n; t += blockDim.x) {
    int i, j, k;
    G::decode(t, i, j, k);
    int a = G::along(i, j, k);
    if (a < 0 || a >= G::nd) continue;
    const int loc = (k * NY + j) * NX + i;
    const size_t off = (size_t)b * NCB + loc;
    double FL[NFLX], FR[NFLX];
#pragma unroll
    for (int n = 0; n < NFLX; ++n) { FL[n] = double(sF[n * G::n + t]); FR[n] = double(sF[n * G::n + t + G::stride]); }
    double U[5];
    if (FIRST) {
      double rho = P.s_in[0][off], vx = P.s_in[1][off], vy = P.s_in[2][off], vz = P.s_in[3][off], e = P.s_in[4][off];
      double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
      U[0] = rho; U[1] = vx * rho; U[2] = vy * rho; U[3] = vz * rho; U[4] = rho * (e + ekin);
    } else {
#pragma unroll
      for (int n = 0; n < 5; ++n) U[n] = ACC[n * ncells + off];
    }
#pragma unroll
    for (int n = 0; n < 5; ++n) U[n] = U[n] - dtd * (FR[n] - FL[n]);
    const double ea = FL[FEINT] - FR[FEINT], eb = FL[FVOLU] - FR[FVOLU];
    const double sp = double(sWm[4 * G::n + t]) + double(sWp[4 * G::n + t]);   // N05 + P05
    if (!LAST) {
#pragma unroll
      for (int n = 0; n < 5; ++n) ACC[n * ncells + off] = U[n];
      double *ax = AUX + (size_t)(DIR - 1) * 3 * ncells;
      ax[off] = ea; ax[ncells + off] = eb; ax[2 * ncells + off] = sp;
    } else {
#pragma unroll
      for (int n = 0; n < 5; ++n) U[n] = U[n] + 0.0;       // + dt*(Sgeo + Sphys), both +0 here
      const double rho0 = P.s_in[0][off], e0 = P.s_in[4][off];
      double IntEner = 0.0;
      if (P.use_aux_eint) {
        // n+1/2 pressure: scrch_Ptr(1) of hy_getFaceFlux.F90:551-557 and the
        // y/z averages
        double pb;
        const double sx = AUX[2 * ncells + off];
        if (NDIM == 2) {
          pb = (0.5 * sx) * 0.5 + sp * 0.25;
        } else {
          const double sy = AUX[3 * ncells + 2 * ncells + off];
          pb = ((0.5 * sx) * 0.5 + sy * 0.25) * 4.0;
          pb = (pb + sp) / 6.0;
        }
        IntEner = rho0 * e0;
        {
          const double *ax = AUX;
          IntEner = IntEner + dt / del[0] * (ax[off] + pb * ax[ncells + off]);
        }
        if (NDIM == 2) {
          IntEner = IntEner + dt / del[1] * (ea + pb * eb);
        } else {
          const double *ay = AUX + 3 * ncells;
          IntEner = IntEner + dt / del[1] * (ay[off] + pb * ay[ncells + off]);
          IntEner = IntEner + dt / del[2] * (ea + pb * eb);
        }
        IntEner = IntEner + dt * 0.;
      }
      // hy_unsplitUpdate.F90:811-893
      double dens = rmax(U[0], P.smlrho);
      double vx = U[1] / dens, vy = U[2] / dens, vz = U[3] / dens;
      double ener = U[4] / dens;
      double eaux = IntEner / dens;
      // hy_energyFix.F90:188-253
      double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
      double eint = ener - ekin - 0.0;
      double newE;
      if (!P.use_aux_eint || eint > P.eswitch * (ekin + 0.0)) newE = rmax(P.smalle, eint);
      else newE = rmax(P.smalle, eaux);
      ener = newE + ekin;
      // Eos_wrapped(MODE_DENS_EI)
      double e = newE;
      if (ener - ekin > rmax(P.smalle, P.eswitch * ekin)) e = ener - ekin;
      P.s_out[0][off] = dens; P.s_out[1][off] = vx; P.s_out[2][off] = vy; P.s_out[3][off] = vz;
      P.s_out[4][off] = e;
      if (!(isfinite(dens) && isfinite(vx) && isfinite(vy) && isfinite(vz) && isfinite(e))) st |= ST_NAN;
      // CFL: Hydro_computeDt.F90:260-284 on the new state
      double pres = dens * e * P.gam1inv;
      double c2 = P.gamma * pres / dens;
      double cs = sqrt(c2);
      double dtl = (fabs(vx - 0.) + cs) * (1.0 / del[0]);
      if (NDIM > 1) dtl = rmax(dtl, (fabs(vy - 0.) + cs) * (1.0 / del[1]));
      if (NDIM > 2) dtl = rmax(dtl, (fabs(vz - 0.) + cs) * (1.0 / del[2]));
      CflCand c; c.key = dtl * P.cfl; c.val = dtl; c.idx = loc;
      cfl_merge(cand, c);
    }
  }
  if (LAST) cfl_block_reduce<NX, NY, NZ>(cand, b, P.cfl, part);
  if (st) atomicOr(P.status, st);
}

// CFL reduction of a stored state (Hydro_computeDt on its own).
template <int NDIM, int NX, int NY, int NZ>
__global__ void __launch_bounds__(320) k_cfl(const DevParams P, CflPart *part) {
  constexpr int NCB = NX * NY * NZ;
  const int b = blockIdx.x;
  if (P.leaf && !P.leaf[b]) {                 // AMR parents take no part in the time step
    if (threadIdx.x == 0) { CflPart r; r.dt = DBL_MAX; r.i = r.j = r.k = -1; r.blk = b; part[b] = r; }
    return;
  }
  double del[3];
  blk_deltas(P, b, del);
  CflCand cand; cand.key = 0.0; cand.val = 0.0; cand.idx = 0x7fffffff;
  for (int loc = threadIdx.x; loc < NCB; loc += blockDim.x) {
    size_t off = (size_t)b * NCB + loc;
    double dens = P.s_in[0][off], vx = P.s_in[1][off], vy = P.s_in[2][off], vz = P.s_in[3][off], e = P.s_in[4][off];
    double pres = dens * e * P.gam1inv;
    double cs = sqrt(P.gamma * pres / dens);
    double dtl = (fabs(vx - 0.) + cs) * (1.0 / del[0]);
    if (NDIM > 1) dtl = rmax(dtl, (fabs(vy - 0.) + cs) * (1.0 / del[1]));
    if (NDIM > 2) dtl = rmax(dtl, (fabs(vz - 0.) + cs) * (1.0 / del[2]));
    CflCand c; c.key = dtl * P.cfl; c.val = dtl; c.idx = loc;
    cfl_merge(cand, c);
  }
  cfl_block_reduce<NX, NY, NZ>(cand, b, P.cfl, part);
}

}  // namespace fhy
