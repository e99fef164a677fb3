// cfl_noalloc.cu -- the CFL time-step reduction for callers that cannot
// allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc: a Fortran code whose
// device memory is owned by another framework's pool allocator (so a second
// allocator would fragment or overcommit it), or a run inside an allocation
// budget fixed at start-up.  For them
// flash_hy_compute_dt_noalloc computes the same time step as
// flash_hy_compute_dt (Hydro_computeDt + the MINLOC reduction) from state
// arrays the caller already owns, without any context and without
// allocating.
//
// Its only scratch is the file-scope array g_cfl_part below, one entry per
// block for at most FLASH_HY_NOALLOC_MAX_BLOCKS blocks (1.5 MiB), plus one
// result slot.  Every GPU that loads this library holds that memory until the
// process exits.  Host code never uses the symbol itself as a device
// address: the first call in each CUDA context (the device's primary context,
// or a driver-API context the caller made current) resolves the addresses
// with cudaGetSymbolAddress and caches them under the context's unique ID
// (cuCtxGetId), since module globals belong to a context, not to a device
// number; that first call should come before any stream capture.  The call
// returns dt on the host, so it synchronises the stream it is given.  Every
// call overwrites every entry it reads, so nothing has to be cleared between
// calls, but all calls share the one array: calls that overlap on the GPU
// (different streams, or threads of the same process) race and must be
// serialised by the caller.
#include <cuda.h>
#include <cuda_runtime.h>
#include <float.h>
#include <mutex>
#include <stdio.h>
#include "../../include/flash_hy.h"
#include "hy_launch.h"

using namespace fhy;

namespace {

struct NoallocResult {
  double dt;
  int i, j, k, blk;
};

static __device__ __align__(256) CflPart g_cfl_part[FLASH_HY_NOALLOC_MAX_BLOCKS];
static __device__ __align__(256) NoallocResult g_cfl_result;

// scratch addresses per CUDA context, keyed by the context's unique ID
struct ScratchAddr {
  unsigned long long ctx_id;
  void *part, *result;
};
constexpr int kMaxContexts = 64;
std::mutex g_mutex;
ScratchAddr g_addr[kMaxContexts];
int g_naddr = 0, g_next = 0;
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// unique ID of the calling thread's current CUDA context (binding the
// current device's primary context first when none is current, as the
// runtime's first call would); false when the driver cannot tell.  Called
// with g_mutex held.
bool current_context_id(unsigned long long *id) {
  if (!g_ctx_get_current || !g_ctx_get_id) {
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void **)&g_ctx_get_current, cudaEnableDefault, &q1) !=
            cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", (void **)&g_ctx_get_id, cudaEnableDefault, &q2) != cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess) {
      g_ctx_get_current = nullptr;
      g_ctx_get_id = nullptr;
      return false;
    }
  }
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return false;
  if (!ctx) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess) return false;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
  }
  return g_ctx_get_id(ctx, id) == CUDA_SUCCESS;
}

// minimum dt over the per-block results, ties to the lowest block index
__global__ void k_noalloc_reduce(const CflPart *part, int nblocks, NoallocResult *out) {
  __shared__ double sdt[256];
  __shared__ int sb[256];
  double best = DBL_MAX;
  int bb = 0x7fffffff;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    double d = part[b].dt;
    if (d < best || (d == best && b < bb)) { best = d; bb = b; }
  }
  sdt[threadIdx.x] = best;
  sb[threadIdx.x] = bb;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      double d = sdt[threadIdx.x + s];
      int q = sb[threadIdx.x + s];
      if (d < sdt[threadIdx.x] || (d == sdt[threadIdx.x] && q < sb[threadIdx.x])) { sdt[threadIdx.x] = d; sb[threadIdx.x] = q; }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    NoallocResult r;
    r.dt = sdt[0];
    int b = sb[0];
    if (b >= 0 && b < nblocks && part[b].i >= 0) { r.i = part[b].i; r.j = part[b].j; r.k = part[b].k; r.blk = b; }
    else { r.i = r.j = r.k = -1; r.blk = -1; }
    *out = r;
  }
}

}  // namespace

extern "C" int flash_hy_compute_dt_noalloc(const double *d_dens, const double *d_velx, const double *d_vely,
                                           const double *d_velz, const double *d_eint, int ndim, int nxb, int nyb,
                                           int nzb, int nblocks, const double deltas[3], double gamma, double cfl,
                                           void *stream, double *dt_out, int minloc_out[5]) {
  if (!d_dens || !d_velx || !d_vely || !d_velz || !d_eint || !deltas || !dt_out || !minloc_out)
    return FLASH_HY_ERR_BAD_ARG;
  if (nblocks <= 0 || nblocks > FLASH_HY_NOALLOC_MAX_BLOCKS) {
    fprintf(stderr,
            "flash_hy_compute_dt_noalloc: %d blocks requested, the fixed scratch holds at most %d "
            "(FLASH_HY_NOALLOC_MAX_BLOCKS); use flash_hy_compute_dt for larger grids\n",
            nblocks, FLASH_HY_NOALLOC_MAX_BLOCKS);
    return FLASH_HY_ERR_BAD_ARG;
  }
  if (!(gamma > 1.0) || !(cfl > 0.0)) return FLASH_HY_ERR_BAD_ARG;
  void *part_addr = nullptr, *result_addr = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    unsigned long long id = 0;
    if (!current_context_id(&id)) return FLASH_HY_ERR_CUDA;
    for (int q = 0; q < g_naddr; ++q)
      if (g_addr[q].ctx_id == id) { part_addr = g_addr[q].part; result_addr = g_addr[q].result; }
    if (!part_addr) {
      // one-time set-up in this context: device addresses of the scratch
      if (cudaGetSymbolAddress(&part_addr, g_cfl_part) != cudaSuccess ||
          cudaGetSymbolAddress(&result_addr, g_cfl_result) != cudaSuccess)
        return FLASH_HY_ERR_CUDA;
      const int slot = g_naddr < kMaxContexts ? g_naddr++ : (g_next++ % kMaxContexts);
      g_addr[slot] = ScratchAddr{id, part_addr, result_addr};
    }
  }
  StepArgs a;
  memset(&a, 0, sizeof a);
  a.P.ndim = ndim;
  a.P.gamma = gamma;
  a.P.gam1inv = 1. / (1.0 / (gamma - 1.0));    // as eos_idealGamma: 1/eos_gammam1
  a.P.cfl = cfl;
  for (int d = 0; d < 3; ++d) a.P.del[d] = d < ndim ? deltas[d] : 1.0;
  a.P.s_in[0] = d_dens; a.P.s_in[1] = d_velx; a.P.s_in[2] = d_vely; a.P.s_in[3] = d_velz; a.P.s_in[4] = d_eint;
  a.part = static_cast<CflPart *>(part_addr);
  a.nlaunch = nblocks;
  a.threads = 320;
  a.stream = static_cast<cudaStream_t>(stream);
  a.set_attr = true;
  int n = cfl_state(a, ndim, nxb, ndim > 1 ? nyb : 1, ndim > 2 ? nzb : 1);
  if (n == -1) return FLASH_HY_ERR_UNSUPPORTED;
  if (n < 0) return FLASH_HY_ERR_CUDA;
  k_noalloc_reduce<<<1, 256, 0, a.stream>>>(static_cast<const CflPart *>(part_addr), nblocks,
                                              static_cast<NoallocResult *>(result_addr));
  if (cudaGetLastError() != cudaSuccess) return FLASH_HY_ERR_CUDA;
  NoallocResult h;
  if (cudaMemcpyAsync(&h, result_addr, sizeof h, cudaMemcpyDeviceToHost, a.stream) != cudaSuccess ||
      cudaStreamSynchronize(a.stream) != cudaSuccess)
    return FLASH_HY_ERR_CUDA;
  *dt_out = h.dt;
  const int NG = 4;
  if (h.blk >= 0) {
    minloc_out[0] = h.i + NG + 1;
    minloc_out[1] = ndim > 1 ? h.j + NG + 1 : 1;
    minloc_out[2] = ndim > 2 ? h.k + NG + 1 : 1;
    minloc_out[3] = 1;
    minloc_out[4] = h.blk;
  } else {
    for (int q = 0; q < 5; ++q) minloc_out[q] = 0;
    minloc_out[4] = -1;
  }
  return h.dt > 0.0 ? 0 : FLASH_HY_ERR_NONPOS_DT;
}
