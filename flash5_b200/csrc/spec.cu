// spec.cu -- the species / mass-scalar pass of a hydro step (spec_kernels.cuh).
// Compiled twice: FP64 without FMA contraction (every precision variant's
// updates, the FP64 paths' face values; spec_step), and with
// FHY_SPEC_MIXED and contraction for the mixed path's FP32 face values
// (spec_step_mx).  Each unit instantiates its own kernels only.
#include "hy_launch.h"
#include "spec_kernels.cuh"

namespace fhy {

template <int NDIM, int NX, int NY, int NZ, bool MX>
static int run_spec(const SpecArgs &a) {
  using SS = SpecStep<NDIM, NX, NY, NZ>;
  const size_t smem = SS::smem_bytes();
  if (smem > 48 * 1024 &&
      (cudaFuncSetAttribute(k_spec_step<NDIM, NX, NY, NZ, MX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
           cudaSuccess ||
       cudaFuncSetAttribute(k_spec_step<NDIM, NX, NY, NZ, MX>, cudaFuncAttributePreferredSharedMemoryCarveout,
                            cudaSharedmemCarveoutMaxShared) != cudaSuccess))
    return -2;
  if constexpr (!MX) {
    if (a.P.fmode == 3) {                    // split step: the update from the kept fluxes (uniform grids)
      k_spec_update<NDIM, NX, NY, NZ><<<a.nlaunch, 256, 0, a.stream>>>(a.P, a.ncells);
      return cudaGetLastError() == cudaSuccess ? 1 : -2;
    }
  }
  if (a.nlev == 0) {
    k_spec_step<NDIM, NX, NY, NZ, MX><<<a.nlaunch, SS::NT, smem, a.stream>>>(a.P, a.ncells);
    return cudaGetLastError() == cudaSuccess ? 1 : -2;
  }
  DevParams P = a.P;
  int n = 0;
  for (int l = a.nlev; l >= 1; --l) {          // finest first: the fine species fluxes go to the register
    if (a.lev_count[l] == 0) continue;
    P.blk_list = a.lev_list[l];
    k_spec_step<NDIM, NX, NY, NZ, MX><<<a.lev_count[l], SS::NT, smem, a.stream>>>(P, a.ncells);
    if (cudaGetLastError() != cudaSuccess) return -2;
    ++n;
  }
  return n;
}

template <bool MX>
static int spec_step_t(const SpecArgs &a, int ndim, int nx, int ny, int nz) {
  if (ndim == 2 && nx == 8 && ny == 8) return run_spec<2, 8, 8, 1, MX>(a);
  if (ndim == 2 && nx == 16 && ny == 16) return run_spec<2, 16, 16, 1, MX>(a);
  if (ndim == 3 && nx == 8 && ny == 8 && nz == 8) return run_spec<3, 8, 8, 8, MX>(a);
  return -2;
}

#ifdef FHY_SPEC_MIXED
int spec_step_mx(const SpecArgs &a, int ndim, int nx, int ny, int nz) { return spec_step_t<true>(a, ndim, nx, ny, nz); }
#else
int spec_step(const SpecArgs &a, int ndim, int nx, int ny, int nz) {
  if (a.mixed && a.P.fmode != 3) return spec_step_mx(a, ndim, nx, ny, nz);
  return spec_step_t<false>(a, ndim, nx, ny, nz);
}
#endif

}  // namespace fhy
