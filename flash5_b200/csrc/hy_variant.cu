// hy_variant.cu -- instantiates the step kernels for one arithmetic variant.
// Compiled once per variant (see flash5_b200/build.py):
//   FHY_VARIANT=1  FP64, no FMA contraction (--fmad=false): the parity path
//   FHY_VARIANT=2  FP64 with FMA contraction
//   FHY_VARIANT=3  FP32 reconstruction / Riemann solve, FP64 update; compiled
//                  once per threads-per-CTA candidate of the direction
//                  kernels (FHY_MXSEL = 0, 1, 2), the transverse-flux pass
//                  and the dispatcher only in unit 0
#include <string.h>
#include "hy_launch.h"
#include "../../include/flash_hy.h"
#if FHY_VARIANT == 3
#include "hy_mixed.cuh"
#endif

#if FHY_VARIANT == 3
#ifndef FHY_MXSEL
#define FHY_MXSEL 0
#endif
#define FHY_PASTE2(a, b) a##b
#define FHY_PASTE(a, b) FHY_PASTE2(a, b)
typedef float Real;
#define FHY_ENTRY FHY_PASTE(step_mixed_nt, FHY_MXSEL)
#elif FHY_VARIANT == 2
typedef double Real;
#define FHY_ENTRY step_fp64_fma
#else
typedef double Real;
#define FHY_ENTRY step_fp64_exact
#endif

namespace fhy {

// the mixed direction kernels take runs of kMxRun blocks (full uniform 3D
// grids with run maps, the plain step)
static bool use_runs(const StepArgs &a) {
  return FHY_VARIANT == 3 && a.tma_run && a.nlev == 0 && a.P.blk_list == nullptr && a.P.fmode == 0 &&
         a.nlaunch == a.nblocks;
}

// ORD: sweep order of the mixed path (0 = x, y, z; 1 = z, y, x); the FP64
// variants always run x, y, z
template <int NDIM, int NX, int NY, int NZ, int DIR, bool FIRST, bool LAST, int RS, int ORD = 0>
static bool launch_dir_one(const StepArgs &a) {
#if FHY_VARIANT == 3
  using G = MxGeom<NDIM, NX, NY, NZ, DIR, RS>;
  constexpr int NT = MxThreads<NDIM, NX, NY, NZ>::pick(FHY_MXSEL);
  auto kern = k_dir_mx<NDIM, NX, NY, NZ, DIR, FIRST, LAST, RS, NT, 1, ORD>;
  const int threads = NT;
#else
  static_assert(ORD == 0, "the FP64 variants sweep x, y, z");
  using G = DirGeom<NDIM, NX, NY, NZ, Real, DIR>;
  auto kern = k_dir<NDIM, NX, NY, NZ, Real, DIR, FIRST, LAST, FHY_VARIANT, RS>;
  const int threads = a.dir_threads;
#endif
  const size_t smem = G::smem_bytes();
  if (a.set_attr && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return false;
#if FHY_VARIANT == 3
  TmaLine tl;
  memset(&tl, 0, sizeof tl);
  if constexpr (NDIM == 3) {
    // full uniform grid: runs of kMxRun blocks along the sweep
    if (use_runs(a)) {
      using GR = MxGeom<NDIM, NX, NY, NZ, DIR, RS, kMxRun>;
      auto kr = k_dir_mx<NDIM, NX, NY, NZ, DIR, FIRST, LAST, RS, NT, kMxRun, ORD>;
      const size_t smr = GR::smem_bytes();
      if (a.set_attr && cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr) != cudaSuccess)
        return false;
      tl = a.tma_run[DIR - 1];
      kr<<<a.nlaunch, threads, smr, a.stream>>>(a.P, (const Real *)a.sig, a.acc, a.aux, a.ncells, a.part, tl);
      if (LAST)
        k_cfl_runs<NX, NY, kMxRun><<<(a.nblocks + 255) / 256, 256, 0, a.stream>>>(
            static_cast<const CflCand *>(tl.cflq), a.nblocks, a.P.cfl, a.part);
      return cudaGetLastError() == cudaSuccess;
    }
  }
  if (NDIM == 3 && a.tma && a.nlev == 0) tl = a.tma[DIR - 1];
  kern<<<a.nlaunch, threads, smem, a.stream>>>(a.P, (const Real *)a.sig, a.acc, a.aux, a.ncells, a.part, tl);
#else
  kern<<<a.nlaunch, threads, smem, a.stream>>>(a.P, (const Real *)a.sig, a.acc, a.aux, a.ncells, a.part);
#endif
  return cudaGetLastError() == cudaSuccess;
}

// one direction: a single launch, or on an AMR hierarchy one launch per
// level, finest first
template <int NDIM, int NX, int NY, int NZ, int DIR, bool FIRST, bool LAST, int RS, int ORD = 0>
static bool launch_dir(const StepArgs &a) {
  if (a.nlev == 0) return launch_dir_one<NDIM, NX, NY, NZ, DIR, FIRST, LAST, RS, ORD>(a);
  StepArgs b = a;
  for (int l = a.nlev; l >= 1; --l) {
    if (a.lev_count[l] == 0) continue;
    b.P.blk_list = a.lev_list[l];
    b.nlaunch = a.lev_count[l];
    if (!launch_dir_one<NDIM, NX, NY, NZ, DIR, FIRST, LAST, RS, ORD>(b)) return false;
    b.set_attr = false;
  }
  return true;
}

// the transverse-flux pass (all leaves on an AMR hierarchy)
#if FHY_VARIANT != 3 || FHY_MXSEL == 0
template <int NDIM, int NX, int NY, int NZ>
static bool launch_sig(const StepArgs &a) {
  auto kern = k_sig<NDIM, NX, NY, NZ, Real, FHY_VARIANT>;
  const size_t smem = SigStage<NDIM, NX, NY, NZ>::smem_bytes();
  if (a.set_attr && smem > 48 * 1024 &&
      (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
       cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared) !=
           cudaSuccess))
    return false;
  if (a.nlev == 0) {
    kern<<<a.nlaunch, a.threads, smem, a.stream>>>(a.P, (Real *)a.sig);
  } else {
    DevParams P = a.P;
    P.blk_list = a.leaves;
    kern<<<a.nleaves, a.threads, smem, a.stream>>>(P, (Real *)a.sig);
  }
  return cudaGetLastError() == cudaSuccess;
}
#if FHY_VARIANT == 3
bool sig_mixed(const StepArgs &a, int ndim, int nx, int ny, int nz) {
  if (ndim == 2 && nx == 8 && ny == 8) return launch_sig<2, 8, 8, 1>(a);
  if (ndim == 2 && nx == 16 && ny == 16) return launch_sig<2, 16, 16, 1>(a);
  if (ndim == 3 && nx == 8 && ny == 8 && nz == 8) return launch_sig<3, 8, 8, 8>(a);
  return false;
}
#endif
#else
template <int NDIM, int NX, int NY, int NZ>
static bool launch_sig(const StepArgs &a) { return sig_mixed(a, NDIM, NX, NY, NZ); }
#endif

// RS: 0 = HLLC, 1 = exact Riemann solver
template <int NDIM, int NX, int NY, int NZ, int RS>
static int run_rs(const StepArgs &a) {
  if (!a.no_sig && !launch_sig<NDIM, NX, NY, NZ>(a)) return -2;
  int nl = 1;
  const int nsig = a.no_sig ? 0 : 1;
  if (a.nlev > 0) {
    nl = 0;
    for (int l = 1; l <= a.nlev; ++l) nl += a.lev_count[l] > 0;
  }
  // z, y, x on the mixed path when asked (the plain step and AMR; the split
  // step's flux modes keep x, y, z).  The middle direction of 3D has the
  // same AUX slot in both orders, so it shares the x, y, z kernel.
  bool ok;
  if constexpr (FHY_VARIANT == 3) {
    if (a.sweep == 1 && a.P.fmode == 0) {
      if constexpr (NDIM == 2)
        ok = launch_dir<NDIM, NX, NY, NZ, 2, true, false, RS, 1>(a) &&
             launch_dir<NDIM, NX, NY, NZ, 1, false, true, RS, 1>(a);
      else
        ok = launch_dir<NDIM, NX, NY, NZ, 3, true, false, RS, 1>(a) &&
             launch_dir<NDIM, NX, NY, NZ, 2, false, false, RS>(a) &&
             launch_dir<NDIM, NX, NY, NZ, 1, false, true, RS, 1>(a);
      return ok ? nsig + NDIM * nl + (NDIM == 3 && use_runs(a) ? 1 : 0) : -2;
    }
  }
  if constexpr (NDIM == 2) {
    ok = launch_dir<NDIM, NX, NY, NZ, 1, true, false, RS>(a) && launch_dir<NDIM, NX, NY, NZ, 2, false, true, RS>(a);
    return ok ? nsig + 2 * nl : -2;
  } else {
    ok = launch_dir<NDIM, NX, NY, NZ, 1, true, false, RS>(a) &&
         launch_dir<NDIM, NX, NY, NZ, 2, false, false, RS>(a) &&
         launch_dir<NDIM, NX, NY, NZ, 3, false, true, RS>(a);
    return ok ? nsig + 3 * nl + (use_runs(a) ? 1 : 0) : -2;   // + the CFL merge of the runs
  }
}

template <int NDIM, int NX, int NY, int NZ>
static int run(const StepArgs &a) {
  return a.P.riemann == FLASH_HY_RS_EXACT ? run_rs<NDIM, NX, NY, NZ, 1>(a) : run_rs<NDIM, NX, NY, NZ, 0>(a);
}

int FHY_ENTRY(const StepArgs &a, int ndim, int nx, int ny, int nz) {
  if (ndim == 2 && nx == 8 && ny == 8) return run<2, 8, 8, 1>(a);
  if (ndim == 2 && nx == 16 && ny == 16) return run<2, 16, 16, 1>(a);
  if (ndim == 3 && nx == 8 && ny == 8 && nz == 8) return run<3, 8, 8, 8>(a);
  return -1;
}

#if FHY_VARIANT == 3 && FHY_MXSEL == 0
int step_mixed(const StepArgs &a, int ndim, int nx, int ny, int nz) {
  switch (a.mx_sel) {
    case 0: return step_mixed_nt0(a, ndim, nx, ny, nz);
    case 2: return step_mixed_nt2(a, ndim, nx, ny, nz);
    default: return step_mixed_nt1(a, ndim, nx, ny, nz);
  }
}
int mx_threads_of(int sel, int ndim, int nx) {
  if (ndim == 3) return MxThreads<3, 8, 8, 8>::pick(sel);
  return nx == 8 ? MxThreads<2, 8, 8, 1>::pick(sel) : MxThreads<2, 16, 16, 1>::pick(sel);
}
#endif

#if FHY_VARIANT == 1
template <int NDIM, int NX, int NY, int NZ>
static int run_cfl(const StepArgs &a) {
  k_cfl<NDIM, NX, NY, NZ><<<a.nlaunch, a.threads, 0, a.stream>>>(a.P, a.part);
  return cudaGetLastError() == cudaSuccess ? 1 : -2;
}
int cfl_state(const StepArgs &a, int ndim, int nx, int ny, int nz) {
  if (ndim == 2 && nx == 8 && ny == 8) return run_cfl<2, 8, 8, 1>(a);
  if (ndim == 2 && nx == 16 && ny == 16) return run_cfl<2, 16, 16, 1>(a);
  if (ndim == 3 && nx == 8 && ny == 8 && nz == 8) return run_cfl<3, 8, 8, 8>(a);
  return -1;
}
size_t sig_bytes_per_block(int ndim, int nx, int ny, int nz, int real_bytes) {
  size_t box = (size_t)(nx + 2) * (ndim > 1 ? ny + 2 : 1) * (ndim > 2 ? nz + 2 : 1);
  return box * 6 * ndim * real_bytes;
}
#endif

}  // namespace fhy
