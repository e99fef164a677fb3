// spec.cu -- the species / mass-scalar pass of a hydro step (spec_kernels.cuh),
// FP64 without FMA contraction for every precision variant.
#include "hy_launch.h"
#include "spec_kernels.cuh"

namespace fhy {

template <int NDIM, int NX, int NY, int NZ>
static int run_spec(const SpecArgs &a) {
  using SS = SpecStep<NDIM, NX, NY, NZ>;
  const size_t smem = SS::smem_bytes();
  if (smem > 48 * 1024 &&
      (cudaFuncSetAttribute(k_spec_step<NDIM, NX, NY, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
           cudaSuccess ||
       cudaFuncSetAttribute(k_spec_step<NDIM, NX, NY, NZ>, cudaFuncAttributePreferredSharedMemoryCarveout,
                            cudaSharedmemCarveoutMaxShared) != cudaSuccess))
    return -2;
  if (a.P.fmode == 3) {                      // split step: the update from the kept fluxes (uniform grids)
    k_spec_update<NDIM, NX, NY, NZ><<<a.nlaunch, 256, 0, a.stream>>>(a.P, a.ncells);
    return cudaGetLastError() == cudaSuccess ? 1 : -2;
  }
  if (a.nlev == 0) {
    k_spec_step<NDIM, NX, NY, NZ><<<a.nlaunch, SS::NT, smem, a.stream>>>(a.P, a.ncells);
    return cudaGetLastError() == cudaSuccess ? 1 : -2;
  }
  DevParams P = a.P;
  int n = 0;
  for (int l = a.nlev; l >= 1; --l) {          // finest first: the fine species fluxes go to the register
    if (a.lev_count[l] == 0) continue;
    P.blk_list = a.lev_list[l];
    k_spec_step<NDIM, NX, NY, NZ><<<a.lev_count[l], SS::NT, smem, a.stream>>>(P, a.ncells);
    if (cudaGetLastError() != cudaSuccess) return -2;
    ++n;
  }
  return n;
}

int spec_step(const SpecArgs &a, int ndim, int nx, int ny, int nz) {
  if (ndim == 2 && nx == 8 && ny == 8) return run_spec<2, 8, 8, 1>(a);
  if (ndim == 2 && nx == 16 && ny == 16) return run_spec<2, 16, 16, 1>(a);
  if (ndim == 3 && nx == 8 && ny == 8 && nz == 8) return run_spec<3, 8, 8, 8>(a);
  return -2;
}

}  // namespace fhy
