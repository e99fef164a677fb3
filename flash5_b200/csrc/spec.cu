// spec.cu -- the species / mass-scalar pass of a hydro step (spec_kernels.cuh),
// FP64 without FMA contraction for every precision variant.
#include "hy_launch.h"
#include "spec_kernels.cuh"

namespace fhy {

template <int NDIM, int NX, int NY, int NZ, int DIR, bool FIRST, bool LAST>
static bool launch_spec_dir(const SpecArgs &a) {
  const size_t smem = SpecGeom<NDIM, NX, NY, NZ, DIR>::smem_bytes();
  if (a.nlev == 0) {
    k_spec_dir<NDIM, NX, NY, NZ, DIR, FIRST, LAST><<<a.nlaunch, 256, smem, a.stream>>>(a.P, a.ssig, a.sacc, a.ncells);
    return cudaGetLastError() == cudaSuccess;
  }
  DevParams P = a.P;
  for (int l = a.nlev; l >= 1; --l) {          // finest first: the fine species fluxes go to the register
    if (a.lev_count[l] == 0) continue;
    P.blk_list = a.lev_list[l];
    k_spec_dir<NDIM, NX, NY, NZ, DIR, FIRST, LAST><<<a.lev_count[l], 256, smem, a.stream>>>(P, a.ssig, a.sacc,
                                                                                         a.ncells);
    if (cudaGetLastError() != cudaSuccess) return false;
  }
  return true;
}

template <int NDIM, int NX, int NY, int NZ>
static int run_spec(const SpecArgs &a) {
  DevParams P = a.P;
  int n0 = a.nlaunch;
  if (a.nlev > 0) { P.blk_list = a.leaves; n0 = a.nleaves; }
  k_spec_sig<NDIM, NX, NY, NZ><<<n0, 256, SigGeom<NDIM, NX, NY, NZ>::smem_bytes(), a.stream>>>(P, a.ssig, a.ncells);
  if (cudaGetLastError() != cudaSuccess) return -2;
  int nl = 1;
  if (a.nlev > 0) {
    nl = 0;
    for (int l = 1; l <= a.nlev; ++l) nl += a.lev_count[l] > 0;
  }
  if constexpr (NDIM == 2) {
    const bool ok = launch_spec_dir<NDIM, NX, NY, NZ, 1, true, false>(a) &&
                    launch_spec_dir<NDIM, NX, NY, NZ, 2, false, true>(a);
    return ok ? 1 + 2 * nl : -2;
  } else {
    const bool ok = launch_spec_dir<NDIM, NX, NY, NZ, 1, true, false>(a) &&
                    launch_spec_dir<NDIM, NX, NY, NZ, 2, false, false>(a) &&
                    launch_spec_dir<NDIM, NX, NY, NZ, 3, false, true>(a);
    return ok ? 1 + 3 * nl : -2;
  }
}

int spec_step(const SpecArgs &a, int ndim, int nx, int ny, int nz) {
  if (ndim == 2 && nx == 8 && ny == 8) return run_spec<2, 8, 8, 1>(a);
  if (ndim == 2 && nx == 16 && ny == 16) return run_spec<2, 16, 16, 1>(a);
  if (ndim == 3 && nx == 8 && ny == 8 && nz == 8) return run_spec<3, 8, 8, 8>(a);
  return -2;
}

}  // namespace fhy
