// hy_mixed.cuh -- the mixed-precision direction kernel.
//
// Same algorithm as k_dir (PPM with characteristic limiting / flattening /
// steepening, transverse and 3D CTU corrections, HLLC, unsplit update), with
// three changes that do not exist in the FP64 parity path:
//  * the reconstruction runs in FP32 in "delta form": every quantity is an
//    increment relative to the cell value (differences of neighbours are
//    taken in FP64 and then rounded), and the face states are assembled as
//    W = V_cell (FP64) + dW (FP32).  FP32 rounding then scales with the
//    increments instead of the values, e.g. the 1e-3 pressure variations of
//    a p = 2.5 background keep ~1e-10 absolute precision instead of 1.5e-7;
//  * the primitive stencil of every line is staged once in shared memory
//    and the limited slopes of each cell are computed once and shared by
//    its neighbours (the reference recomputes three per cell,
//    hy_DataReconstructNormalDir_PPM.F90:438-441);
//  * the Riemann solve, the fluxes and the update run in FP64 (HLLC with
//    shared reciprocals instead of the reference's repeated divisions).
#pragma once
#include "hy_kernels.cuh"

namespace fhy {

// ---------------------------------------------------------------------------
// TMA staging of the direction kernels' line stencils (uniform 3D grids).
// Each state variable is described by tensor maps over its natural layout
// (x fastest, then y, then z of every block: dims 8 x 8 x 8*nblocks); one
// 3D tile copy brings a block's interior (box 8 x 8 x 8) and one a
// neighbour's 4-cell slab along the sweep direction (box 4 x 8 x 8,
// 8 x 4 x 8 or 8 x 8 x 4), straight into the staged layout below.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// one bounded poll of phase `parity`; true once it has completed
__device__ __forceinline__ bool mbar_try(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// 3D tile copy global -> shared through a tensor map (no multicast)
// L2 prefetch of [p, p + bytes) as one bulk request (16-byte aligned,
// bytes a multiple of 16)
__device__ __forceinline__ void bulk_prefetch_l2(const void *p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}
// fetch a tensor map into the descriptor cache ahead of its first copy
__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<unsigned long long>(map)) : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
// SM cycles (about a second) a CTA waits for its tile copies before it gives
// up (FLASH_HY_ERR_TIMEOUT)
constexpr long long kTmaWaitCycles = 1LL << 31;

// FP64 HLLC (hy_HLLC.F90:94-311) with one division per star state; igm1 =
// 1/(game - 1) of the cell the face state belongs to.
template <int DIR>
__device__ __forceinline__ void hllc_fp64(const DevParams &P, const double *Vm, const double *Vp, double igL,
                                          double igR, double Fs[6], unsigned &st) {
  constexpr int v1 = Slots<DIR>::v1;
  const double tiny = P.tiny;
  if ((Vm[HD] < tiny && Vm[HD] > 0.) || (Vp[HD] < tiny && Vp[HD] > 0.) || (Vm[HP] < tiny && Vm[HP] > 0.) ||
      (Vp[HP] < tiny && Vp[HP] > 0.)) {
#pragma unroll
    for (int n = 0; n < 6; ++n) Fs[n] = 0.;
    return;
  }
  const double uL = Vm[v1], uR = Vp[v1], dL = Vm[HD], dR = Vp[HD], pL = Vm[HP], pR = Vp[HP];
  const double aL2 = P.gamma * pL / dL, aR2 = P.gamma * pR / dR;
  if (aL2 < 0. || aR2 < 0.) {
    st |= ST_NEG_SOUND;
#pragma unroll
    for (int n = 0; n < 6; ++n) Fs[n] = 0.;
    return;
  }
  const double cL = sqrt(aL2), cR = sqrt(aR2);
  const double SL = fmin(uL - cL, uR - cR), SR = fmax(uL + cL, uR + cR);
  double qStar = (dR * uR * (SR - uR) - dL * uL * (SL - uL) + pL - pR) / (dR * (SR - uR) - dL * (SL - uL));
  // side whose flux (and star state) is used
  const bool useL = SL >= 0. || qStar >= 0.;
  const double *V = useL ? Vm : Vp;
  const double d = useL ? dL : dR, u = useL ? uL : uR, p = useL ? pL : pR, S = useL ? SL : SR;
  const double ig = useL ? igL : igR;
  const double u2 = V[HVX] * V[HVX] + V[HVY] * V[HVY] + V[HVZ] * V[HVZ];
  const double E = 0.5 * d * u2 + p * ig;
  double F[5], U[5];
  F[0] = d * u;
  F[1] = F[0] * V[HVX]; F[2] = F[0] * V[HVY]; F[3] = F[0] * V[HVZ];
  F[DIR] += p;
  F[4] = (E + p) * u;
  Fs[5] = p;
  const bool outside = useL ? (SL >= 0.) : (SR < 0.);
  if (outside) {
#pragma unroll
    for (int n = 0; n < 5; ++n) Fs[n] = F[n];
    return;
  }
  U[0] = d; U[1] = d * V[HVX]; U[2] = d * V[HVY]; U[3] = d * V[HVZ]; U[4] = E;
  const double num = S - u, rden = 1.0 / (S - qStar);
  const double r = num * rden;
  const double pStar = dL * (SL - uL) * (qStar - uL) + pL;
  double UC[5];
  UC[0] = d * r;
#pragma unroll
  for (int m = 1; m <= 3; ++m) UC[m] = (m == DIR) ? UC[0] * qStar : U[m] * r;
  UC[4] = U[4] * r + (pStar * qStar - p * u) * rden;
#pragma unroll
  for (int n = 0; n < 5; ++n) Fs[n] = F[n] + S * (UC[n] - U[n]);
}

// Per block, the K quarter candidates of a run step merged into the block's
// CFL result, as cfl_block_reduce writes it for a block handled whole
// (Hydro_computeDt.F90:265-284).
template <int NX, int NY, int K>
__global__ void k_cfl_runs(const CflCand *cq, int nblocks, double cfl, CflPart *part) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  CflCand a = cq[(size_t)b * K];
#pragma unroll
  for (int q = 1; q < K; ++q) cfl_merge(a, cq[(size_t)b * K + q]);
  CflPart r;
  if (a.key > 0.0) {
    r.dt = cfl / a.val;
    r.i = a.idx % NX; r.j = (a.idx / NX) % NY; r.k = a.idx / (NX * NY);
  } else {
    r.dt = DBL_MAX; r.i = r.j = r.k = -1;
  }
  r.blk = b;
  part[b] = r;
}

// Lines of a CTA: the block's lines along DIR (K = 1), or, with K > 1, a
// run of K blocks that follow one another along DIR, of which the CTA takes
// 1/K of the cross-section (quarter q of the slower transverse axis): the
// lines are K blocks long, so the stencil overlap along DIR (four guard
// cells on each side, recomputed slopes and face states at the ends) is
// paid once per run instead of once per block.
template <int NDIM, int NX, int NY, int NZ, int DIR, int RS = 0, int K = 1>
struct MxGeom {
  static constexpr int ND0 = DIR == 1 ? NX : (DIR == 2 ? NY : NZ);               // block extent along DIR
  static constexpr int ND = K * ND0;                                              // line interior
  static constexpr int T1 = DIR == 1 ? NY : NX;                                   // faster transverse axis
  static constexpr int T2 = DIR == 3 ? NY : NZ;                                   // slower one (split by K)
  static_assert(K == 1 || (NDIM == 3 && T2 % K == 0), "runs split the slower transverse axis");
  static constexpr int T2Q = T2 / K;
  static constexpr int C = T1 * T2Q;                                              // lines
  static constexpr int L4 = ND + 8, LS = ND + 4, LC = ND + 2;                      // staged, slope, line cells
  static constexpr int SA = L4 * C, SB = LS * C, SC = LC * C;
  // index of position x on line l in a space of length L with offset o
  __device__ static __forceinline__ int at(int x, int l, int L, int o) { return DIR == 1 ? l * L + (x + o) : (x + o) * C + l; }
  __device__ static __forceinline__ void dec(int s, int L, int o, int &x, int &l) {
    if (DIR == 1) { l = s / L; x = s % L - o; } else { l = s % C; x = s / C - o; }
  }
  static constexpr int step = DIR == 1 ? 1 : C;      // +1 along the line
  // staged stencil (positions x in [-4, ND + 3] of line l): the slab of the
  // neighbour below, the interior of each block of the run, the slab of the
  // neighbour above -- each in the natural x, y, z order of the block
  // store, so that each is one dense tile copy; along the sweep direction
  // the regions follow one another (DIR 3: plain along-major order)
  static constexpr int SLAB = 4 * C, LO = 0, MID = 4 * C, HI = (4 + ND) * C, MIDB = ND0 * C;
  __device__ static __forceinline__ int sidx(int x, int l) {
    if (DIR == 3) return (x + 4) * C + l;
    const int m = x < 0 ? 0 : (x >= ND ? K - 1 : x / ND0), xl = x - m * ND0;
    if (DIR == 1) return x < 0 ? l * 4 + (x + 4) : (x < ND ? MID + m * MIDB + l * ND0 + xl : HI + l * 4 + (x - ND));
    // DIR 2: line l = i + NX * k
    const int i = l % NX, k = l / NX;
    return x < 0 ? k * 4 * NX + (x + 4) * NX + i
                 : (x < ND ? MID + m * MIDB + (k * ND0 + xl) * NX + i : HI + k * 4 * NX + (x - ND) * NX + i);
  }
  // block of the run holding position x (the end blocks for the guard
  // positions) and x relative to that block
  __device__ static __forceinline__ int blk_of(int x, int &xl) {
    const int m = x < 0 ? 0 : (x >= ND ? K - 1 : x / ND0);
    xl = x - m * ND0;
    return m;
  }
  // block-local cell of block-relative position xl on line l of quarter q
  __device__ static __forceinline__ void cell(int xl, int l, int q, int &i, int &j, int &k) {
    const int t1 = l % T1, t2 = l / T1 + q * T2Q;
    if (DIR == 1) { i = xl; j = t1; k = t2; }
    else if (DIR == 2) { j = xl; i = t1; k = t2; }
    else { k = xl; i = t1; j = t2; }
    if (NDIM < 3) k = (DIR == 3) ? k : 0;
  }
  __device__ static __forceinline__ void cell(int x, int l, int &i, int &j, int &k) { cell(x, l, 0, i, j, k); }
  // shared memory: staged prims (FP64), then a region used first for the
  // reconstruction scratch and then for the face fluxes
  // (with the exact solver the slope scratch, dead during the Riemann
  // phase, also holds the learned-guess network, so it is at least that big)
  static constexpr size_t prim_bytes = (size_t)5 * SA * 8;
  static constexpr size_t slope_bytes = (size_t)SB * 4 + (size_t)SB * 6 * 4;
  static constexpr size_t wp_off =
      (RS == 1 && slope_bytes < sizeof(xrs::MlpPacked)) ? sizeof(xrs::MlpPacked) : slope_bytes;
  static constexpr size_t recon_bytes = wp_off + (size_t)2 * SC * 6 * 4 + (size_t)SC * 8;
  static constexpr size_t flux_bytes = (size_t)SC * 9 * 8;
  // + the CTA's face-state ranges (learned gate, 16 warps x 6 floats), the
  // staging barrier and the slack that aligns the tile destinations to 128
  // bytes
  static constexpr size_t red_bytes = 16 * 6 * 4;
  // runs (K > 1) and 2D blocks keep the face fluxes in their own region,
  // so that the Riemann phase writes them as it goes (the CTAs per SM that
  // the registers allow still fit); one 3D block per CTA lays them over the
  // reconstruction scratch and holds them in registers until that is dead
  static constexpr bool own_flux = K > 1 || NDIM == 2;
  static constexpr size_t flux_off = own_flux ? recon_bytes : 0;
  static constexpr size_t smem_bytes() {
    return prim_bytes + (own_flux ? recon_bytes + flux_bytes : (recon_bytes > flux_bytes ? recon_bytes : flux_bytes)) +
           red_bytes + 16 + 128;
  }
};

// threads per CTA of k_dir_mx: three compiled candidates per block shape,
// picked at run time (flash_hy_set_tuning / flash_hy_autotune); the middle
// one is the default.  3D 8^3: 640 line cells per direction and block (2
// CTAs per SM by shared memory), 544 on a run of four (576 slope cells,
// two per thread at 288 threads; the register file of each of the SM's four
// schedulers holds five warps of 96 registers a thread at 288 and 320);
// 2D 8^2: 80 faces; 2D 16^2: 288 faces.
template <int NDIM, int NX, int NY, int NZ> struct MxThreads {
  static constexpr int c0 = NDIM == 3 ? 288 : (NX == 8 ? 64 : 192);
  static constexpr int c1 = NDIM == 3 ? 320 : (NX == 8 ? 96 : 288);
  static constexpr int c2 = NDIM == 3 ? 384 : (NX == 8 ? 128 : 320);
  static constexpr int n = c1;
  static constexpr int pick(int sel) { return sel == 0 ? c0 : (sel == 1 ? c1 : c2); }
};

// Sweep order ORD of the mixed path: 0 = x, y, z (FLASH's SWEEP_XYZ), 1 =
// z, y, x (SWEEP_ZYX).  The directions accumulate the conservative update
// in that order; an earlier direction's internal-energy terms sit in AUX
// slot aux_slot (its position in the order), and the last direction
// gathers them per direction and applies the same x, y, z formula.
template <int NDIM, int ORD>
__host__ __device__ constexpr int aux_slot(int d) { return ORD == 0 ? d - 1 : NDIM - d; }

template <int NDIM, int NX, int NY, int NZ, int DIR, bool FIRST, bool LAST, int RS, int NT, int K = 1, int ORD = 0>
__global__ void __launch_bounds__(NT, NDIM == 3 ? 2 : 1)
k_dir_mx(const DevParams P, const float *__restrict__ SIG, double *__restrict__ ACC, double *__restrict__ AUX,
         size_t ncells, CflPart *part, const __grid_constant__ TmaLine tm) {
  static_assert(NT % 32 == 0, "threads per CTA must be a multiple of 32");
  using G = MxGeom<NDIM, NX, NY, NZ, DIR, RS, K>;
  using B = Box<NDIM, NX, NY, NZ>;
  constexpr int NCB = NX * NY * NZ;
  constexpr int NIT = (G::SC + NT - 1) / NT;
  constexpr int v1 = Slots<DIR>::v1;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  unsigned char *smem_raw =
      smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);          // tile destinations: 128-byte aligned
  double *sV = reinterpret_cast<double *>(smem_raw);                     // [5][SA]: rho,u,v,w,e (sidx order)
  unsigned char *reg = smem_raw + G::prim_bytes;
  float *sFlat = reinterpret_cast<float *>(reg);                          // [SB]
  float *sDb = sFlat + G::SB;                                             // [6][SB]
  float *sWp = reinterpret_cast<float *>(reg + G::wp_off);                // [6][SC] increments
  float *sWm = sWp + 6 * G::SC;                                           // [6][SC]
  double *sIg = reinterpret_cast<double *>(sWm + 6 * G::SC);              // [SC] 1/(game-1)
  double *sF = reinterpret_cast<double *>(reg + G::flux_off);            // [9][SC] face fluxes

  static_assert((6 * B::n * 4) % 16 == 0 && (NCB * 8) % 16 == 0, "bulk prefetch sizes must be multiples of 16 bytes");
  // the tile copies' descriptors load while the block's indices do
  if (NDIM == 3 && tm.on && threadIdx.x < 10) prefetch_tensormap(threadIdx.x < 5 ? &tm.intr[threadIdx.x] : &tm.slab[threadIdx.x - 5]);
  // the CTA's blocks: one (K = 1), or run blockIdx.x / K of K blocks that
  // follow one another along DIR (with the neighbours below and above the
  // run), of which the CTA takes quarter qtr = blockIdx.x % K
  int blk[K], nbs[2] = {-1, -1}, qtr = 0;
  if constexpr (K == 1) {
    blk[0] = P.blk_list ? P.blk_list[blockIdx.x] : blockIdx.x;
  } else {
    const int *run = tm.runs + (size_t)(blockIdx.x / K) * (K + 2);
    qtr = blockIdx.x % K;
#pragma unroll
    for (int m = 0; m < K; ++m) blk[m] = run[m];
    nbs[0] = run[K];
    nbs[1] = run[K + 1];
  }
  const int b = blk[0];
  const int3 bc = blk_coords(P, b);
  unsigned st = 0;
  double del[3];
  blk_deltas(P, b, del);
  const double dt = P.dt_dev ? *P.dt_dev : P.dt, delta = del[DIR - 1];
  const float dtn = float(dt / delta), hdtn = 0.5f * dtn;
  const float hdtx = float(0.5 * dt / del[0]), hdty = float(0.5 * dt / del[1]), hdtz = float(0.5 * dt / del[2]);
  const float *sigb = SIG + (size_t)(P.slot ? P.slot[b] : (int)blockIdx.x) * NDIM * 6 * B::n;
  // What the kernel reads from global memory after its staging -- the sig
  // of the other directions (face states), the accumulators of the earlier
  // directions and, in the last direction, their aux rows (update) -- is
  // prefetched into L2 at the start, one bulk request per contiguous range
  // (lanes of warp 0), so that the first touch overlaps the staging and the
  // slopes.
  // (On a run, CTA qtr prefetches the ranges of block qtr of the run: the run's
  // K CTAs together cover its K blocks.)
  if (threadIdx.x < 32) {
    const int ln = threadIdx.x;
    const int pb = K == 1 ? b : blk[qtr];
    const float *ps = K == 1 ? sigb : SIG + (size_t)pb * NDIM * 6 * B::n;
    if (ln < NDIM && ln != DIR - 1 && P.fmode != 3) bulk_prefetch_l2(ps + (size_t)ln * 6 * B::n, 6u * B::n * 4u);
    if (!FIRST && ln >= 4 && ln < 9) bulk_prefetch_l2(ACC + (ln - 4) * ncells + (size_t)pb * NCB, NCB * 8u);
    if (LAST && ln >= 12 && ln < 12 + 3 * (NDIM - 1))
      bulk_prefetch_l2(AUX + (ln - 12) * ncells + (size_t)pb * NCB, NCB * 8u);
  }

  auto fidx = [](int along, int t1, int t2) { return G::at(along, t1 + (DIR == 1 ? NY : NX) * t2, G::LC, 1); };
  if (P.fmode != 3) {
  // ---- A: stage the primitive stencil of every line (guard cells get the EOS)
  // Uniform 3D grids: the block's interior and the neighbours' slabs along
  // DIR by TMA tile copies (one thread issues 15, an mbarrier counts the
  // bytes), then the pressure and the guard cells' EOS in place; slabs
  // beyond a non-periodic boundary (mirror / copy rules) and all other
  // grids through load_prim.
  bool tma = NDIM == 3 && tm.on && P.lh == nullptr && P.blk_nbr != nullptr;   // always on runs (K > 1)
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(smem_raw + G::smem_bytes() - 16 - 128);
  float *sRed = reinterpret_cast<float *>(smem_raw + G::smem_bytes() - 16 - 128 - G::red_bytes);
  if (tma) {
    // the neighbours below / above along DIR (-1: load_prim) from the
    // block's face-neighbour row (one load, not dependent on the
    // coordinates), or from the run's row
    if constexpr (K == 1) {
      nbs[0] = P.blk_nbr[6 * b + 2 * (DIR - 1)];
      nbs[1] = P.blk_nbr[6 * b + 2 * (DIR - 1) + 1];
    }
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();                          // the barrier is initialised before anyone polls it
    // copies: the interior of each block of the run (quarter qtr of its
    // cross-section) and the slabs of the neighbours along DIR, five
    // variables; one thread issues them (K = 1) or the lanes of warp 0
    // issue one each
    constexpr int NOPS = 5 * (K + 2);
    const int q5[5] = {0, 1, 2, 3, 4};         // staged slots of dens, velx, vely, velz, eint
    const int qo = qtr * G::T2Q;                 // quarter offset on the slower transverse axis
    auto copy = [&](int o) {
      const int v = o / (K + 2), r = o % (K + 2);
      double *dst = sV + q5[v] * G::SA;
      if (r < K) {
        tma_load_3d(dst + G::MID + r * G::MIDB, &tm.intr[v], 0, DIR == 3 ? qo : 0, blk[r] * NZ + (DIR == 3 ? 0 : qo),
                    bar);
      } else if (r == K) {
        // the slab below: the neighbour's last four layers
        if (nbs[0] >= 0)
          tma_load_3d(dst + G::LO, &tm.slab[v], DIR == 1 ? NX - 4 : 0, DIR == 2 ? NY - 4 : (DIR == 3 ? qo : 0),
                      nbs[0] * NZ + (DIR == 3 ? NZ - 4 : qo), bar);
      } else if (nbs[1] >= 0) {
        // the slab above: its first four
        tma_load_3d(dst + G::HI, &tm.slab[v], 0, DIR == 3 ? qo : 0, nbs[1] * NZ + (DIR == 3 ? 0 : qo), bar);
      }
    };
    const unsigned slab_bytes = (unsigned)G::SLAB * 8u, mid_bytes = (unsigned)(K * G::MIDB) * 8u;
    if constexpr (K == 1) {
      if (threadIdx.x == 0) {
        mbar_expect_tx(bar, 5u * (mid_bytes + (nbs[0] >= 0 ? slab_bytes : 0u) + (nbs[1] >= 0 ? slab_bytes : 0u)));
#pragma unroll
        for (int o = 0; o < NOPS; ++o) copy(o);
      }
    } else {
      static_assert(NOPS <= 32, "one copy per lane of warp 0");
      if (threadIdx.x < 32) {
        if (threadIdx.x == 0)
          mbar_expect_tx(bar, 5u * (mid_bytes + (nbs[0] >= 0 ? slab_bytes : 0u) + (nbs[1] >= 0 ? slab_bytes : 0u)));
        __syncwarp();
        if (threadIdx.x < NOPS) copy(threadIdx.x);
      }
    }
  }
  // cells no tile copy covers
  for (int s = threadIdx.x; s < G::SA; s += NT) {
    int x, l, i, j, k;
    G::dec(s, G::L4, 4, x, l);
    if (tma && (x < 0 ? nbs[0] >= 0 : (x >= G::ND ? nbs[1] >= 0 : true))) continue;
    int xl;
    const int m = G::blk_of(x, xl);
    G::cell(xl, l, qtr, i, j, k);
    double V[8];
    if constexpr (K == 1) load_prim<NDIM, NX, NY, NZ, false>(P, b, bc, i, j, k, V);
    else load_prim<NDIM, NX, NY, NZ, false>(P, blk[m], blk_coords(P, blk[m]), i, j, k, V);
    const int q = G::sidx(x, l);
    sV[0 * G::SA + q] = V[HD]; sV[1 * G::SA + q] = V[HVX]; sV[2 * G::SA + q] = V[HVY];
    sV[3 * G::SA + q] = V[HVZ]; sV[4 * G::SA + q] = V[HEI];
  }
  if (tma) {
    // bounded wait for the tile copies; a CTA that gives up flags
    // FLASH_HY_ERR_TIMEOUT, waits (bounded) once more for its copies in
    // flight and leaves
    bool done = false;
    const long long t0 = clock64();
    while (!done && clock64() - t0 < kTmaWaitCycles) done = mbar_try(bar, 0);
    if (__syncthreads_or(!done)) {
      if (threadIdx.x == 0) atomicOr(P.status, (unsigned)FLASH_HY_ERR_TIMEOUT);
      const long long t1 = clock64();
      while (clock64() - t1 < kTmaWaitCycles && !mbar_try(bar, 0)) {
      }
      return;
    }
    // the copied guard cells' EOS (Eos_getData.F90:80-96 on ENER = eint +
    // ekin, as load_prim); the pressure is not staged (Vs below)
    for (int g = threadIdx.x; g < 8 * G::C; g += NT) {
      const int side = g >= 4 * G::C, r = g - side * 4 * G::C;
      if (nbs[side] < 0) continue;
      const int x = side ? G::ND + r / G::C : r / G::C - 4, l = r % G::C;
      const int q = G::sidx(x, l);
      const double e = sV[4 * G::SA + q];
      const double vx = sV[G::SA + q], vy = sV[2 * G::SA + q], vz = sV[3 * G::SA + q];
      const double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
      const double ener = e + ekin;
      if (ener - ekin > rmax(P.smalle, P.eswitch * ekin)) sV[4 * G::SA + q] = ener - ekin;
    }
  }
  __syncthreads();
  // q: 0..5 = rho, u, v, w, p, e; the pressure of the gamma law from the
  // staged rho and e, in the EOS's order (rho * e) * gam1inv
  const double gam1inv = P.gam1inv;
  auto Vs = [&](int q, int s) -> double {
    if (q == 4) return sV[s] * sV[4 * G::SA + s] * gam1inv;
    return sV[(q == 5 ? 4 : q) * G::SA + s];
  };

  // ---- B: limited slopes and flattening switches of cells [-2, N+1]
  for (int q = threadIdx.x; q < G::SB; q += NT) {
    int x, l;
    G::dec(q, G::LS, 2, x, l);
    const int s = G::sidx(x, l), sm = G::sidx(x - 1, l), sp = G::sidx(x + 1, l);
    float Vc[8], dL[5], dR[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      Vc[n] = float(Vs(n, s));
      dL[n] = float(Vs(n, s) - Vs(n, sm));
      dR[n] = float(Vs(n, sp) - Vs(n, s));
    }
    Vc[HGC] = float(P.gamma); Vc[HGE] = 0.f; Vc[HEI] = float(Vs(5, s));
    Eig<float> e;
    eigen<float, DIR>(Vc, e, st);
    float db[8];
    tvd_slope_d<float, DIR>(P, dL, dR, float(Vs(5, s) - Vs(5, sm)), float(Vs(5, sp) - Vs(5, s)), e, db);
#pragma unroll
    for (int n = 0; n < 5; ++n) sDb[n * G::SB + q] = db[n];
    sDb[5 * G::SB + q] = db[HEI];
    if (P.use_flattening) {
      const int smm = G::sidx(x - 2, l), spp = G::sidx(x + 2, l);
      float dp1 = float(Vs(4, sp) - Vs(4, sm));
      float dp2 = float(Vs(4, spp) - Vs(4, smm));
      float dv1 = float(Vs(v1, sp) - Vs(v1, sm));
      float pmin = float(fmin(Vs(4, sm), Vs(4, sp)));
      float Sp = fabsf(dp2) > 1.e-15f ? dp1 / dp2 - 0.75f : 0.f;
      float ft = fmaxf(0.f, fminf(1.f, 10.f * Sp));
      if ((fabsf(dp1) / pmin < 1.f / 3.f) || dv1 > 0.f) ft = 0.f;
      sFlat[q] = ft;
    }
  }
  __syncthreads();

  // ---- C: face states of the line cells [-1, N] as increments
  // (exact solver with a network: the ranges of the face states' pressure,
  // density and normal velocity over the CTA, for the learned gate's bound)
  float rg[6] = {3.0e38f, -3.0e38f, 3.0e38f, -3.0e38f, 3.0e38f, -3.0e38f};   // p, rho, u: min, max
  for (int t = threadIdx.x; t < G::SC; t += NT) {
    int x, l, i, j, k, xl;
    G::dec(t, G::LC, 1, x, l);
    const int mb = G::blk_of(x, xl);             // block of the run: its sig box covers xl in [-1, N]
    G::cell(xl, l, qtr, i, j, k);
    const float *sigc = K == 1 ? sigb : SIG + (size_t)blk[mb] * NDIM * 6 * B::n;
    const int s = G::sidx(x, l), sm = G::sidx(x - 1, l), sp = G::sidx(x + 1, l), q = G::at(x, l, G::LS, 2);
    const int qs = G::step;
    float Vc[8], dL[8], dR[8];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      Vc[n] = float(Vs(n, s));
      dL[n] = float(Vs(n, s) - Vs(n, sm));
      dR[n] = float(Vs(n, sp) - Vs(n, s));
    }
    Vc[HGC] = float(P.gamma); Vc[HEI] = float(Vs(5, s));
    dL[HEI] = float(Vs(5, s) - Vs(5, sm));
    dR[HEI] = float(Vs(5, sp) - Vs(5, s));
    Eig<float> e0;
    eigen<float, DIR>(Vc, e0, st);
    float flat = 0.f;
    if (P.use_flattening) {
      float t0 = sFlat[q];
      double dp1 = Vs(4, sp) - Vs(4, sm);
      if (dp1 < 0.) flat = fmaxf(t0, sFlat[q + qs]);
      else if (dp1 == 0.) flat = t0;
      else flat = fmaxf(t0, sFlat[q - qs]);
    }
    if (K == 1 && P.sp_flat)
      P.sp_flat[sp_line_base<NDIM, NX, NY, NZ, DIR>(P.slot ? P.slot[b] : (int)blockIdx.x) + DirGeom<NDIM, NX, NY, NZ, double, DIR>::idx(i, j, k)] =
          double(flat);
    const int sl[6] = {0, 1, 2, 3, 4, 7};
    float lft[8], rgt[8], delW[8], W6[8];
#pragma unroll
    for (int qq = 0; qq < 6; ++qq) {
      int n = sl[qq], m = qq < 5 ? qq : 5;
      float dbN = sDb[m * G::SB + q - qs], db0 = sDb[m * G::SB + q], dbP = sDb[m * G::SB + q + qs];
      lft[n] = -0.5f * dL[n] - (db0 - dbN) / 6.f;
      rgt[n] = 0.5f * dR[n] - (dbP - db0) / 6.f;
    }
    if (P.use_steepening) {
      const float eta1 = 20.f, eta2 = 0.05f, epsln = 0.01f, K0 = 0.1f;
      double rm = Vs(0, sm), rp = Vs(0, sp), rc = Vs(0, s);
      double rmm = Vs(0, G::sidx(x - 2, l)), rpp = Vs(0, G::sidx(x + 2, l));
      float temp1 = float(rp - rm);
      if (fabsf(temp1) > float(P.tiny)) {
        float dd = float(delta);
        float d2R = float((rpp - rp) - (rp - rc)) / (6.f * dd * dd);
        float d2L = float((rc - rm) - (rm - rmm)) / (6.f * dd * dd);
        float eta = (d2L - d2R) * (dd * dd) / temp1;
        if (d2R * d2L >= 0.f) eta = 0.f;
        if (epsln * float(fmin(rp, rm)) - fabsf(temp1) >= 0.f) eta = 0.f;
        eta = fmaxf(0.f, fminf(1.f, eta1 * (eta - eta2)));
        double pm = Vs(4, sm), pp = Vs(4, sp);
        float temp2 = float(fabs(pp - pm) / fmin(pp, pm));
        float temp3 = fabsf(temp1) / float(fmin(rp, rm));
        double game_c = Vs(4, s) / (Vs(5, s) * rc) + 1;
        if (float(game_c) * K0 * temp3 - temp2 < 0.f) eta = 0.f;
        float dbN = sDb[q - qs], dbP = sDb[q + qs];
        lft[HD] = lft[HD] * (1.f - eta) + (-dL[HD] + 0.5f * dbN) * eta;
        rgt[HD] = rgt[HD] * (1.f - eta) + (dR[HD] - 0.5f * dbP) * eta;
      }
    }
#pragma unroll
    for (int qq = 0; qq < 6; ++qq) {
      int n = sl[qq];
      if (P.use_flattening) { lft[n] = (1.f - flat) * lft[n]; rgt[n] = (1.f - flat) * rgt[n]; }
      if (rgt[n] * (-lft[n]) <= 0.f) { lft[n] = 0.f; rgt[n] = 0.f; }
      float dw = rgt[n] - lft[n];
      if (6.f * dw * (-0.5f * (lft[n] + rgt[n])) > dw * dw) lft[n] = -2.f * rgt[n];
      dw = rgt[n] - lft[n];
      if (6.f * dw * (-0.5f * (lft[n] + rgt[n])) < -(dw * dw)) rgt[n] = -2.f * lft[n];
      delW[n] = rgt[n] - lft[n];
      W6[n] = -3.f * (lft[n] + rgt[n]);
    }
    float dWp[8], dWm[8];
    {
      float lmax = fmaxf(e0.lam[2], 0.f);
      dWp[HEI] = rgt[HEI] - lmax * hdtn * (delW[HEI] - (1.f - lmax * hdtn * 4.f / 3.f) * W6[HEI]);
      float lmin = -fminf(e0.lam[2], 0.f);
      dWm[HEI] = lft[HEI] + lmin * hdtn * (delW[HEI] + (1.f - lmin * hdtn * 4.f / 3.f) * W6[HEI]);
    }
    {
      constexpr int u1 = Slots<DIR>::v1, u2 = Slots<DIR>::v2, u3 = Slots<DIR>::v3;
      float mW6[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) mW6[n] = -W6[n];
      float sL[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, sR[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        float cA = ldot<float, DIR>(e0, n, delW), cB = ldot<float, DIR>(e0, n, mW6);
        float lam = e0.lam[n], xx = dtn * lam;
        float AL = 0.5f * (-1.f - xx), BL = 0.25f * (1.f + 2.f * xx + (4.f / 3.f) * (xx * xx));
        float AR = 0.5f * (1.f - xx), BR = 0.25f * (1.f - 2.f * xx + (4.f / 3.f) * (xx * xx));
        float tL = AL * cA + BL * cB, tR = AR * cA + BR * cB;
        if (n == 0 || n == 4) {
          float rv = n == 0 ? -e0.cf : e0.cf;
          sL[HD] += e0.rho * tL; sR[HD] += e0.rho * tR;
          sL[u1] += rv * tL; sR[u1] += rv * tR;
          sL[HP] += e0.rp * tL; sR[HP] += e0.rp * tR;
        } else if (n == 1) { sL[u2] += tL; sR[u2] += tR; }
        else if (n == 2) { sL[HD] += tL; sR[HD] += tR; }
        else { sL[u3] += tL; sR[u3] += tR; }
      }
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        dWm[n] = W6[n] / 12.f + sL[n];
        dWp[n] = W6[n] / 12.f + sR[n];
      }
    }
    // transverse corrections
    const int bi = B::idx(i, j, k);
    float sx[8], sy[8], sz[8];
    if (DIR != 1) load_sig(sigc + 0 * 6 * B::n + bi, B::n, sx);
    if (NDIM > 1 && DIR != 2) load_sig(sigc + 1 * 6 * B::n + bi, B::n, sy);
    if (NDIM > 2 && DIR != 3) load_sig(sigc + 2 * 6 * B::n + bi, B::n, sz);
#pragma unroll
    for (int qq = 0; qq < 6; ++qq) {
      int n = sl[qq];
      float c = 0.f;
      if (NDIM == 2) c = DIR == 1 ? hdty * sy[n] : hdtx * sx[n];
      else c = DIR == 1 ? hdty * sy[n] + hdtz * sz[n] : (DIR == 2 ? hdtx * sx[n] + hdtz * sz[n] : hdtx * sx[n] + hdty * sy[n]);
      dWm[n] -= c;
      dWp[n] -= c;
    }
    const double rc = Vs(0, s), pc = Vs(4, s);
    if (rc + dWm[HD] < 0. || rc + dWp[HD] < 0. || pc + dWm[HP] < 0. || pc + dWp[HP] < 0.) {
#pragma unroll
      for (int n = 0; n < 8; ++n) { dWm[n] = 0.f; dWp[n] = 0.f; }
    }
    if (NDIM == 3 && P.use_ctu) {
      constexpr int A1 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1), S1 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2);
      constexpr int A2 = DIR == 1 ? 3 : (DIR == 2 ? 1 : 2), S2 = DIR == 1 ? 2 : (DIR == 2 ? 3 : 1);
      const float fac = float(dt * dt / (6. * (DIR == 1 ? del[1] : (DIR == 2 ? del[2] : del[0])) *
                                         (DIR == 1 ? del[2] : (DIR == 2 ? del[0] : del[1]))));
      float T1[8], T2[8];
      {
        float sm[8], s0[8], sp[8];
        const float *base = sigc + (size_t)(S1 - 1) * 6 * B::n;
        load_sig(base + B::idx(i - (A1 == 1), j - (A1 == 2), k - (A1 == 3)), B::n, sm);
        load_sig(base + bi, B::n, s0);
        load_sig(base + B::idx(i + (A1 == 1), j + (A1 == 2), k + (A1 == 3)), B::n, sp);
        Eig<float> e;
        eigen<float, A1>(Vc, e, st);
        upwind_tflux<float, A1>(P, sm, s0, sp, e, T1);
      }
      {
        float sm[8], s0[8], sp[8];
        const float *base = sigc + (size_t)(S2 - 1) * 6 * B::n;
        load_sig(base + B::idx(i - (A2 == 1), j - (A2 == 2), k - (A2 == 3)), B::n, sm);
        load_sig(base + bi, B::n, s0);
        load_sig(base + B::idx(i + (A2 == 1), j + (A2 == 2), k + (A2 == 3)), B::n, sp);
        Eig<float> e;
        eigen<float, A2>(Vc, e, st);
        upwind_tflux<float, A2>(P, sm, s0, sp, e, T2);
      }
#pragma unroll
      for (int qq = 0; qq < 6; ++qq) {
        int n = sl[qq];
        float c = (T1[n] + T2[n]) * fac;
        dWp[n] += c;
        dWm[n] += c;
      }
      const bool fb = rc + dWp[HD] <= 0. || rc + dWm[HD] <= 0. || pc + dWp[HP] <= 0. || pc + dWm[HP] <= 0.;
      if (fb) {
#pragma unroll
        for (int n = 0; n < 8; ++n) { dWm[n] = 0.f; dWp[n] = 0.f; }
      }
      if (K == 1 && P.sp_fb)
        P.sp_fb[sp_line_base<NDIM, NX, NY, NZ, DIR>(P.slot ? P.slot[b] : (int)blockIdx.x) + DirGeom<NDIM, NX, NY, NZ, double, DIR>::idx(i, j, k)] = fb;
    }
#pragma unroll
    for (int qq = 0; qq < 6; ++qq) {
      sWp[qq * G::SC + t] = dWp[sl[qq]];
      sWm[qq * G::SC + t] = dWm[sl[qq]];
    }
    // 1/(game-1) of the cell: game - 1 = p/(e rho) (Eos_putData.F90:105-106)
    sIg[t] = (Vs(5, s) * rc) / pc;
    if (RS == 1 && P.mlp) {
      const float fp = float(pc), fr = float(rc), fu = float(Vs(v1, s));
      const float q6[6] = {fp + dWm[HP], fp + dWp[HP], fr + dWm[HD], fr + dWp[HD], fu + dWm[v1], fu + dWp[v1]};
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        rg[2 * m] = fminf(rg[2 * m], fminf(q6[2 * m], q6[2 * m + 1]));
        rg[2 * m + 1] = fmaxf(rg[2 * m + 1], fmaxf(q6[2 * m], q6[2 * m + 1]));
        // NaN anywhere keeps the gate open
        if (q6[2 * m] != q6[2 * m] || q6[2 * m + 1] != q6[2 * m + 1]) rg[2 * m] = -3.0e38f;
      }
    }
  }
  if (RS == 1 && P.mlp) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        rg[2 * m] = fminf(rg[2 * m], __shfl_xor_sync(0xffffffffu, rg[2 * m], o));
        rg[2 * m + 1] = fmaxf(rg[2 * m + 1], __shfl_xor_sync(0xffffffffu, rg[2 * m + 1], o));
      }
    if ((threadIdx.x & 31) == 0)
#pragma unroll
      for (int m = 0; m < 6; ++m) sRed[(threadIdx.x >> 5) * 6 + m] = rg[m];
  }
  __syncthreads();

  // ---- D: Riemann problems at the faces, FP64
  double Fr[NIT][9];
  if constexpr (RS == 1) {
    // exact solver.  With a network attached, pass 1 evaluates its
    // tensor-core guess for the faces with strong waves (the network sits
    // over the slope scratch, dead from here on) and leaves the start value
    // w0 = p0^z in sP0 (over the unused 1/(game-1) array; negative = network
    // start, limited to three evaluations; 0 = two-rarefaction start); pass
    // 2 runs Newton and the Godunov flux.  Each thread reads back only its
    // own entries.
    double *sP0 = sIg;
    // The CTA-wide bound: every face has p_min >= P_lo, p_max <= P_hi and a
    // PVRS estimate ppv <= P_hi + 0.5 (U_hi - U_lo) rho_hi c_hi with c_hi =
    // sqrt(gamma P_hi / rho_lo); strong_waves needs max(p_max, ppv) >= 2
    // p_min, so below 2 P_lo (a 1e-4 margin covers the FP32 rounding) no
    // face of the CTA consults the network and the gate pass is skipped:
    // the same decisions, and results, as testing every face.
    bool learned = P.mlp != nullptr;
    if (learned) {
      float r[6] = {3.0e38f, -3.0e38f, 3.0e38f, -3.0e38f, 3.0e38f, -3.0e38f};
      for (int w = 0; w < NT / 32; ++w)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          r[2 * m] = fminf(r[2 * m], sRed[w * 6 + 2 * m]);
          r[2 * m + 1] = fmaxf(r[2 * m + 1], sRed[w * 6 + 2 * m + 1]);
        }
      const float chi = sqrtf(float(P.gamma) * r[1] / r[2]);
      const float bound = r[1] + 0.5f * (r[5] - r[4]) * r[3] * chi;
      const bool finite = r[0] > 1e-30f && r[1] < 1e30f && r[2] > 1e-30f && r[3] < 1e30f && r[4] > -1e30f &&
                          r[5] < 1e30f && bound < 1e30f;
      if (finite && bound < 2.f * r[0] * (1.f - 1e-4f)) learned = false;
    }
    const double g = P.gamma;
    const xrs::Gas &gas = P.gas;             // from the parameter block
    // s: staged index of the face's right cell, sl: of its left cell
    auto face = [&](int qq, bool left, int2 s, int t) -> double {
      return left ? Vs(qq, s.y) + double(sWp[qq * G::SC + t - G::step])
                  : Vs(qq, s.x) + double(sWm[qq * G::SC + t]);
    };
    // the two face states; w = p^z only with `with_w` (pass 1a tests for
    // strong waves without it)
    auto sides = [&](int2 s, int t, xrs::Side &L, xrs::Side &R, bool with_w = true) {
      const double dl = face(0, true, s, t), ul = face(DIR, true, s, t), pl = face(4, true, s, t);
      const double dr = face(0, false, s, t), ur = face(DIR, false, s, t), pr = face(4, false, s, t);
      const double c2l = g * pl / dl, c2r = g * pr / dr;
      if (!(c2l > 0.0) || !(c2r > 0.0)) st |= ST_NEG_SOUND;
      L = xrs::Side{dl, ul, pl, sqrt(c2l), 0.0};
      R = xrs::Side{dr, ur, pr, sqrt(c2r), 0.0};
      if (with_w) {
        L.w = xrs::powp(pl, gas.z);
        R.w = xrs::powp(pr, gas.z);
      }
    };
    if (learned) {
      // pass 1a: faces with strong waves and an inexact two-rarefaction
      // guess get sP0 = w_TR > 0, all others 0 (two-rarefaction start)
      int need = 0;
#pragma unroll
      for (int it = 0; it < NIT; ++it) {
        const int t = threadIdx.x + it * NT;
        if (t >= G::SC) break;
        int x, l;
        G::dec(t, G::LC, 1, x, l);
        if (x < 0) continue;
        const int2 s4 = make_int2(G::sidx(x, l), G::sidx(x - 1, l));
        double q = 0.0;
        // the FP32 screen first; the FP64 sides and tests only where it passes
        if (xrs::strong_screen(face(0, true, s4, t), face(DIR, true, s4, t), face(4, true, s4, t),
                               face(0, false, s4, t), face(DIR, false, s4, t), face(4, false, s4, t), g)) {
          xrs::Side L, R;
          sides(s4, t, L, R, false);
          if (!xrs::vacuum(L, R, gas) && xrs::strong_waves(L, R)) {
            L.w = xrs::powp(L.p, gas.z);
            R.w = xrs::powp(R.p, gas.z);
            const double wtr = xrs::tr_w(L, R, gas);
            if (!xrs::tr_exact(L, R, xrs::p_of_w(wtr, gas))) q = wtr;
          }
        }
        sP0[t] = q;
        need |= q > 0.0;
      }
      // pass 1b: the network's start for those faces (negative: limited to
      // three evaluations); skipped by CTAs and warps without such faces
      if (__syncthreads_or(need)) {
        xrs::MlpPacked *sM = reinterpret_cast<xrs::MlpPacked *>(reg);
        xrs::load_packed(*sM, static_cast<const xrs::MlpPacked *>(P.mlp));
        __syncthreads();
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
          const int t = threadIdx.x + it * NT;
          if (t - (int)(threadIdx.x & 31) >= G::SC) break;    // warp-uniform: NT is a multiple of 32
          int x = -1, l = 0;
          if (t < G::SC) G::dec(t, G::LC, 1, x, l);
          const double q = (t < G::SC && x >= 0) ? sP0[t] : 0.0;
          const bool net = q > 0.0;
          if (!__any_sync(0xffffffffu, net)) continue;
          xrs::Side L{1.0, 0.0, 1.0, 1.0, 1.0}, R{1.0, 0.0, 1.0, 1.0, 1.0};
          if (net) sides(make_int2(G::sidx(x, l), G::sidx(x - 1, l)), t, L, R);
          float f[xrs::NIN];
          if (net) xrs::features(L, R, g, xrs::p_of_w(q, gas), f);
          else {
#pragma unroll
            for (int k = 0; k < xrs::NIN; ++k) f[k] = 0.f;
          }
          const float y = fminf(fmaxf(xrs::mlp_lane(*sM, f), -20.f), 20.f);
          if (net) sP0[t] = -(q * (double)expf(float(gas.z) * y));    // (p*/p_TR)^z
        }
      }
    }
    // One copy of the face solve, looped over the thread's faces (not
    // unrolled: the solver and the sampling are large, and two copies of
    // them overflow the instruction cache); the results go to the
    // registers of face `it` by compile-time selection.
#pragma unroll 1
    for (int it = 0; it < NIT; ++it) {
      const int t = threadIdx.x + it * NT;
      if (t >= G::SC) break;
      int x, l;
      G::dec(t, G::LC, 1, x, l);
      if (x < 0) continue;
      const int2 s = make_int2(G::sidx(x, l), G::sidx(x - 1, l));
      xrs::Side L, R;
      sides(s, t, L, R);
      const bool vac = xrs::vacuum(L, R, gas);
      xrs::Star S{0.0, 0.5 * (L.u + R.u), 0.0};
      if (!vac) {
        const double q = learned ? sP0[t] : 0.0;
        const xrs::SideK kl = xrs::side_k(L, gas), kr = xrs::side_k(R, gas);
        const double w0 = q < 0.0 ? -q : xrs::tr_w(L, R, kl, kr, gas);
        // the network's start gets three evaluations; if they do not
        // converge, Newton restarts from the two-rarefaction guess
        int k;
#pragma unroll 1
        for (int attempt = 0;; ++attempt) {
          const bool net = attempt == 0 && q < 0.0;
          k = xrs::newton(L, R, kl, kr, gas, attempt == 0 ? w0 : xrs::tr_w(L, R, kl, kr, gas), P.rs_tol,
                          net ? 3 : P.rs_max_iter, S);
          if (k >= 0 || !net) break;
        }
        if (k < 0) st |= ST_NEWTON;
        if (P.harvest && (q < 0.0 || (xrs::strong_waves(L, R) && !xrs::tr_exact(L, R, xrs::p_of_w(w0, gas)))))
          harvest_face(P, L, R, g, (unsigned)(blockIdx.x * 4 + DIR) * 2048u + (unsigned)t);
      }
      double VL[8], VR[8];
#pragma unroll
      for (int qq = 0; qq < 6; ++qq) {
        const int n = qq < 5 ? qq : HEI;
        VL[n] = face(qq, true, s, t);
        VR[n] = face(qq, false, s, t);
      }
      double F[9];
      xrs::godunov_flux<DIR>(VL, VR, L, R, gas, S, vac, F);
      double fv = 0., fe = 0.;
      if (P.use_aux_eint) {
        if (F[FDENS] > 0.) { fv = F[FDENS] / VL[HD]; fe = F[FDENS] * VL[HEI]; }
        else { fv = F[FDENS] / VR[HD]; fe = F[FDENS] * VR[HEI]; }
      }
      F[FEINT] = fe;
      F[FVOLU] = fv;
      F[8] = (Vs(4, s.x) + double(sWm[4 * G::SC + t])) + (Vs(4, s.x) + double(sWp[4 * G::SC + t]));
      if constexpr (G::own_flux) {
#pragma unroll
        for (int n = 0; n < 9; ++n) sF[n * G::SC + t] = F[n];
      } else {
#pragma unroll
        for (int j = 0; j < NIT; ++j)
          if (j == it) {
#pragma unroll
            for (int n = 0; n < 9; ++n) Fr[j][n] = F[n];
          }
      }
    }
  } else {
#pragma unroll
  for (int it = 0; it < NIT; ++it) {
    const int t = threadIdx.x + it * NT;
    if (t >= G::SC) break;
    int x, l;
    G::dec(t, G::LC, 1, x, l);
    if (x < 0) continue;
    const int s = G::sidx(x, l);
    const int tl = t - G::step, sL = G::sidx(x - 1, l);
    double VL[8], VR[8];
#pragma unroll
    for (int qq = 0; qq < 6; ++qq) {
      int n = qq < 5 ? qq : HEI;
      VL[n] = Vs(qq, sL) + double(sWp[qq * G::SC + tl]);
      VR[n] = Vs(qq, s) + double(sWm[qq * G::SC + t]);
    }
    double F[9];
    hllc_fp64<DIR>(P, VL, VR, sIg[tl], sIg[t], F, st);
    double fv = 0., fe = 0.;
    if (P.use_aux_eint) {
      if (F[FDENS] > 0.) { fv = F[FDENS] / VL[HD]; fe = F[FDENS] * VL[HEI]; }
      else { fv = F[FDENS] / VR[HD]; fe = F[FDENS] * VR[HEI]; }
    }
    F[FEINT] = fe;
    F[FVOLU] = fv;
    // N05 + P05 of this cell (n+1/2 pressure sum)
    F[8] = (Vs(4, s) + double(sWm[4 * G::SC + t])) + (Vs(4, s) + double(sWp[4 * G::SC + t]));
#pragma unroll
    for (int n = 0; n < 9; ++n) {
      if constexpr (G::own_flux) sF[n * G::SC + t] = F[n];
      else Fr[it][n] = F[n];
    }
  }
  }
  if constexpr (!G::own_flux) {
    // the fluxes go over the reconstruction scratch once every thread is
    // done reading it
    __syncthreads();
#pragma unroll
    for (int it = 0; it < NIT; ++it) {
      const int t = threadIdx.x + it * NT;
      if (t >= G::SC) break;
      int x, l;
      G::dec(t, G::LC, 1, x, l);
      if (x < 0) continue;
#pragma unroll
      for (int n = 0; n < 9; ++n) sF[n * G::SC + t] = Fr[it][n];
    }
  }
  __syncthreads();
  if (K == 1 && P.freg) {         // AMR: fine/coarse faces
    flux_register<NDIM, NX, NY, NZ, DIR>(P, b, bc, sF, G::SC, [](int along, int t1, int t2) {
      return G::at(along, t1 + (DIR == 1 ? NY : NX) * t2, G::LC, 1);
    });
    __syncthreads();
  }
  if (K == 1 && P.sp_mf) {        // face mass fluxes for the species pass
    for (int t = threadIdx.x; t < G::SC; t += NT) {
      int x, l, i, j, k;
      G::dec(t, G::LC, 1, x, l);
      if (x < 0) continue;
      G::cell(x, l, i, j, k);
      P.sp_mf[sp_line_base<NDIM, NX, NY, NZ, DIR>(P.slot ? P.slot[b] : (int)blockIdx.x) + DirGeom<NDIM, NX, NY, NZ, double, DIR>::idx(i, j, k)] =
          sF[FDENS * G::SC + t];
    }
  }

  } else {
    // replay: the stored fluxes and pressure sums
    using FS = FluxStore<NDIM, NX, NY, NZ>;
    const double *src = FS::base(P, b, DIR);
    for (int q = threadIdx.x; q < NFLX * FS::NF; q += NT) {
      const int v = q / FS::NF, f = q % FS::NF;
      int a, t1, t2;
      face_coords<NDIM, NX, NY, NZ, DIR>(f, a, t1, t2);
      sF[v * G::SC + fidx(a, t1, t2)] = src[q];
    }
    for (int c = threadIdx.x; c < FS::NCB; c += NT) {
      const int i = c % NX, j = (c / NX) % NY, k = c / (NX * NY);
      sF[8 * G::SC + fidx(DIR == 1 ? i : (DIR == 2 ? j : k), DIR == 1 ? j : i, DIR == 3 ? j : k)] =
          src[NFLX * FS::NF + c];
    }
    __syncthreads();
  }
  if (K == 1 && (P.fmode == 1 || P.fmode == 2)) {
    flux_store<NDIM, NX, NY, NZ, DIR>(P, b, sF, G::SC, fidx, [&](int t) { return sF[8 * G::SC + t]; });
    if (P.fmode == 2) {
      if (st) atomicOr(P.status, st);
      return;
    }
  }

  // ---- E: conservative update
  const double dtd = dt / delta;
  CflCand cand[K];                         // per block of the run
#pragma unroll
  for (int m = 0; m < K; ++m) { cand[m].key = 0.0; cand[m].val = 0.0; cand[m].idx = 0x7fffffff; }
  for (int t = threadIdx.x; t < G::SC; t += NT) {
    int x, l, i, j, k, xl;
    G::dec(t, G::LC, 1, x, l);
    if (x < 0 || x >= G::ND) continue;
    const int mb = G::blk_of(x, xl);
    G::cell(xl, l, qtr, i, j, k);
    const int loc = (k * NY + j) * NX + i;
    const size_t off = (size_t)(K == 1 ? b : blk[mb]) * NCB + loc;
    double FL[NFLX], FR[NFLX];
#pragma unroll
    for (int n = 0; n < NFLX; ++n) { FL[n] = sF[n * G::SC + t]; FR[n] = sF[n * G::SC + t + G::step]; }
    const double sp = sF[8 * G::SC + t];
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
    if (!LAST) {
#pragma unroll
      for (int n = 0; n < 5; ++n) ACC[n * ncells + off] = U[n];
      double *ax = AUX + (size_t)aux_slot<NDIM, ORD>(DIR) * 3 * ncells;
      ax[off] = ea; ax[ncells + off] = eb; ax[2 * ncells + off] = sp;
    } else {
      const double rho0 = P.s_in[0][off], e0 = P.s_in[4][off];
      double IntEner = 0.0;
      if (P.use_aux_eint && ORD == 0) {
        double pb;
        const double sx = AUX[2 * ncells + off];
        if (NDIM == 2) {
          pb = (0.5 * sx) * 0.5 + sp * 0.25;
        } else {
          const double sy = AUX[5 * ncells + off];
          pb = (((0.5 * sx) * 0.5 + sy * 0.25) * 4.0 + sp) / 6.0;
        }
        IntEner = rho0 * e0 + dt / del[0] * (AUX[off] + pb * AUX[ncells + off]);
        if (NDIM == 2) {
          IntEner += dt / del[1] * (ea + pb * eb);
        } else {
          IntEner += dt / del[1] * (AUX[3 * ncells + off] + pb * AUX[4 * ncells + off]);
          IntEner += dt / del[2] * (ea + pb * eb);
        }
      } else if (P.use_aux_eint) {
        // the same formula for another order: each direction's (ea, eb,
        // speed), this direction's own, the earlier ones' from their slots
        double te[3], tb[3], ts[3];
#pragma unroll
        for (int d = 1; d <= NDIM; ++d) {
          if (d == DIR) { te[d - 1] = ea; tb[d - 1] = eb; ts[d - 1] = sp; continue; }
          const double *ad = AUX + (size_t)aux_slot<NDIM, ORD>(d) * 3 * ncells;
          te[d - 1] = ad[off]; tb[d - 1] = ad[ncells + off]; ts[d - 1] = ad[2 * ncells + off];
        }
        double pb;
        if (NDIM == 2) pb = (0.5 * ts[0]) * 0.5 + ts[1] * 0.25;
        else pb = (((0.5 * ts[0]) * 0.5 + ts[1] * 0.25) * 4.0 + ts[2]) / 6.0;
        IntEner = rho0 * e0 + dt / del[0] * (te[0] + pb * tb[0]);
        IntEner += dt / del[1] * (te[1] + pb * tb[1]);
        if (NDIM == 3) IntEner += dt / del[2] * (te[2] + pb * tb[2]);
      }
      double dens = fmax(U[0], P.smlrho);
      double rinv = 1.0 / dens;
      double vx = U[1] * rinv, vy = U[2] * rinv, vz = U[3] * rinv;
      double ener = U[4] * rinv;
      double eaux = IntEner * rinv;
      double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
      double eint = ener - ekin;
      double newE = (!P.use_aux_eint || eint > P.eswitch * ekin) ? fmax(P.smalle, eint) : fmax(P.smalle, eaux);
      ener = newE + ekin;
      double e = newE;
      if (ener - ekin > fmax(P.smalle, P.eswitch * ekin)) e = ener - ekin;
      P.s_out[0][off] = dens; P.s_out[1][off] = vx; P.s_out[2][off] = vy; P.s_out[3][off] = vz;
      P.s_out[4][off] = e;
      if (!(isfinite(dens) && isfinite(vx) && isfinite(vy) && isfinite(vz) && isfinite(e))) st |= ST_NAN;
      double pres = dens * e * P.gam1inv;
      double cs = sqrt(P.gamma * pres * rinv);
      double dtl = (fabs(vx) + cs) * (1.0 / del[0]);
      if (NDIM > 1) dtl = fmax(dtl, (fabs(vy) + cs) * (1.0 / del[1]));
      if (NDIM > 2) dtl = fmax(dtl, (fabs(vz) + cs) * (1.0 / del[2]));
      CflCand c; c.key = dtl * P.cfl; c.val = dtl; c.idx = loc;
#pragma unroll
      for (int m = 0; m < K; ++m)
        if (m == mb) cfl_merge(cand[m], c);
    }
  }
  if constexpr (LAST) {
    if constexpr (K == 1) {
      cfl_block_reduce<NX, NY, NZ>(cand[0], b, P.cfl, part);
    } else {
      // the CTA's candidate for each block of the run; k_cfl_runs merges
      // the K quarters of every block (the same max / first-index rule, so
      // the result equals a reduction over the whole block)
      // (one barrier: every warp reduces its K candidates, then thread m
      // merges the warps' candidates of block m)
      __shared__ CflCand red[32][K];
      const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
      for (int m = 0; m < K; ++m) {
        CflCand c = cand[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          CflCand o2;
          o2.key = __shfl_down_sync(0xffffffffu, c.key, o);
          o2.val = __shfl_down_sync(0xffffffffu, c.val, o);
          o2.idx = __shfl_down_sync(0xffffffffu, c.idx, o);
          if (lane + o < 32) cfl_merge(c, o2);
        }
        if (lane == 0) red[w][m] = c;
      }
      __syncthreads();
      if (threadIdx.x < K) {
        const int m = threadIdx.x;
        CflCand a = red[0][m];
        for (int q = 1; q < NT / 32; ++q) cfl_merge(a, red[q][m]);
        const int bm = tm.runs[(size_t)(blockIdx.x / K) * (K + 2) + m];   // blk[m] (not indexed at run time)
        static_cast<CflCand *>(tm.cflq)[(size_t)bm * K + qtr] = a;
      }
    }
  }
  if (st) atomicOr(P.status, st);
}

}  // namespace fhy
