// flash_hy.cu -- the C ABI of include/flash_hy.h: context, device block
// store, UNK upload/download, the Hydro step and the CFL time step.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>
#include "../../include/flash_hy.h"
#include "hy_launch.h"
#include "amr_kernels.cuh"

using namespace fhy;

struct DtInfo {
  double dt;
  int i, j, k, level, blk;
};

struct flash_hy_ctx {
  flash_hy_params p;
  int ndim, nx, ny, nz, nblocks, nbx, nby, nbz, bc[6];
  double del[3];
  size_t ncb, ncells;
  int device;
  cudaStream_t stream;
  double *state[2][5];
  int cur;
  double *acc, *aux;
  void *sig;
  int *d_blk_at, *d_blk_coord, *d_list;
  int *d_blk_nbr;             // uniform grids: [nblocks][6] face neighbours
  fhy::TmaLine *tma_run;      // run kernels' maps (2 state buffers x 3 directions), or NULL
  int *d_runs[3];             // per direction: [nblocks / kMxRun][kMxRun + 2]
  void *d_cflq;               // [nblocks][kMxRun] CFL candidates of the run quarters
  int list_cap;
  int *h_list;               // 0-based copy of a caller's 1-based block list
  int h_list_cap;
  int mesh_me;               // hy_meshMe: the rank reported in the dt minloc
  fhy::TmaLine *tma_maps;    // [2 state buffers][3 directions]: TMA staging of k_dir_mx, or NULL
  struct XferPool *xfer;     // host threads, streams and pinned slots of upload / download
  CflPart *d_part;
  DtInfo *d_dt, *h_dt;
  unsigned *d_status, *h_status;
  unsigned char *d_stage;
  size_t stage_bytes;
  int dt_valid;
  int launches;
  int threads;         // threads per CTA: transverse-flux and CFL passes
  int dir_threads;     // FP64 direction kernels
  int mx_sel;          // mixed direction kernels: candidate 0, 1, 2
  int mx_runs;         // mixed 3D direction kernels: blocks per CTA along the sweep (1 or kMxRun)
  int mx_sweep;        // mixed direction kernels: FLASH_HY_SWEEP_XYZ or FLASH_HY_SWEEP_ZYX
  int host_ng;         // guard layers of the caller's UNK arrays
  float *d_wmaster;    // learned guess: FP32 master weights
  void *d_mlp;         // learned guess: packed BF16 inference copy (xrs::MlpPacked)
  int mlp_set;
  double *d_harvest;   // [7][harvest_cap] face states kept for training
  unsigned long long *d_harvest_n;
  long long harvest_cap;
  unsigned harvest_mask;
  // graph replay of flash_hy_step: one executable graph per state-buffer
  // parity (the step reads buffer cur and writes 1 - cur); dt is written to
  // d_stepdt by a one-thread kernel launched before the replay
  bool use_graph;
  cudaGraphExec_t gexec[2];
  int glaunches[2];
  int plain_steps[2];
  double *d_stepdt;
  // AMR hierarchy (max_level > 1): node tables, level lists, guard buffers
  int amr, nlev;
  int *d_level, *d_leaf, *d_parent, *d_slot, *d_at;
  int at_off[17], at_ext[17][3];
  int *d_leaves, nleaves;
  int *d_lev_leaves[17], lev_leaves[17];
  int *d_lev_parents[17], lev_parents[17];
  int nparents;
  double *d_lh, *d_gp, *d_pe, *d_freg;
  // a rank's share of a sharded grid: owned blocks and the ghost exchange
  bool partial;
  int *h_blk_at;               // host copy of the block table (uniform grids)
  int *d_owned, n_owned;       // blocks the step advances
  int *d_owned_mask;           // 1 for owned blocks (dt reduction)
  int *h_owned, *h_recv;       // host copies of the owned and received (ghost) lists
  int n_recv_h;
  int *d_inner, n_inner;       // owned blocks whose guard cells come from owned blocks only
  int *d_edge, n_edge;         // the other owned blocks (they read ghost blocks)
  int phase_pending;           // flash_hy_step_phase: phase 1 enqueued, phase 2 due
  double phase_dt;
  int *d_send, n_send, *d_recv, n_recv;  // blocks packed for / unpacked from other ranks
  double *d_fstore;            // stored fluxes of the split step
  double *d_sp_fstore;         // and their species fluxes
  // species and mass scalars: state [2][nsp][ncells]; face mass fluxes,
  // fallback flags and flattening left by the hydro direction kernels
  int nsp, nspec;
  double *spec[2], *sp_mf, *sp_flat;
  unsigned char *sp_fb;
  double *sp_lh, *sp_gp, *sp_freg;   // AMR: species guard cells, parent copies, flux register
  size_t sp_freg_stride;
  double *d_err;               // refinement criterion per block
  char err[512];
};

// ---------------------------------------------------------------------------
// device memory of the contexts: a per-device cache of freed blocks.  An AMR
// regrid creates a context for the new tree and closes the old one every few
// steps; cudaMalloc and cudaFree of a context's buffers cost ~12 ms there
// (cudaFree synchronises the device) against 0.5 ms for the data movement.
// Blocks are rounded to a power of two up to 2 MiB (at least 256 B) and to
// a multiple of 2 MiB above; a request takes the smallest cached block of
// its device that holds it and is at most twice its size, else cudaMalloc
// (after releasing the device's cache if that fails).  At most 32 GiB stay
// cached; flash_hy_release_memory frees them.  Pointers that did not come
// from ctx_alloc are freed directly.
// ---------------------------------------------------------------------------
namespace {
struct CachedBlock { void *p; size_t bytes; int device; };
std::mutex g_mem_mu;
std::vector<CachedBlock> g_cached;
std::unordered_map<void *, CachedBlock> g_live;
size_t g_cached_bytes = 0;
constexpr size_t kGranule = (size_t)2 << 20, kCacheCap = (size_t)32 << 30;

void release_cached_locked(int device) {
  for (size_t q = 0; q < g_cached.size();) {
    if (device < 0 || g_cached[q].device == device) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(g_cached[q].device);
      cudaFree(g_cached[q].p);
      cudaSetDevice(cur);
      g_cached_bytes -= g_cached[q].bytes;
      g_cached[q] = g_cached.back();
      g_cached.pop_back();
    } else {
      ++q;
    }
  }
}
}  // namespace

// on the current device
static cudaError_t ctx_alloc(void **p, size_t bytes) {
  int device = 0;
  cudaGetDevice(&device);
  size_t r = 256;
  if (bytes > kGranule) r = (bytes + kGranule - 1) / kGranule * kGranule;
  else while (r < bytes) r <<= 1;
  std::lock_guard<std::mutex> lk(g_mem_mu);
  int best = -1;
  for (int q = 0; q < (int)g_cached.size(); ++q) {
    const CachedBlock &b = g_cached[q];
    if (b.device == device && b.bytes >= r && b.bytes <= 2 * r && (best < 0 || b.bytes < g_cached[best].bytes)) best = q;
  }
  if (best >= 0) {
    const CachedBlock b = g_cached[best];
    g_cached[best] = g_cached.back();
    g_cached.pop_back();
    g_cached_bytes -= b.bytes;
    g_live[b.p] = b;
    *p = b.p;
    return cudaSuccess;
  }
  cudaError_t e = cudaMalloc(p, r);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    release_cached_locked(device);
    e = cudaMalloc(p, r);
  }
  if (e == cudaSuccess) g_live[*p] = CachedBlock{*p, r, device};
  return e;
}

static void ctx_free(void *p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_mem_mu);
  auto it = g_live.find(p);
  if (it == g_live.end()) {
    cudaFree(p);
    return;
  }
  const CachedBlock b = it->second;
  g_live.erase(it);
  if (g_cached_bytes + b.bytes > kCacheCap) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(b.device);
    cudaFree(b.p);
    cudaSetDevice(cur);
    return;
  }
  g_cached.push_back(b);
  g_cached_bytes += b.bytes;
}

extern "C" int flash_hy_release_memory(int device) {
  std::lock_guard<std::mutex> lk(g_mem_mu);
  release_cached_locked(device);
  return 0;
}

// Tensor maps of the mixed direction kernels' TMA staging (uniform 3D
// grids of 8^3 blocks): for both state buffers, each variable and each
// sweep direction, the interior box and the slab box along the direction,
// over the block store's natural layout (dims 8, 8, 8 * nblocks; FP64).
// cuTensorMapEncodeTiled comes from the driver through the runtime, so the
// library needs no link-time dependency on libcuda.  Returns NULL when the
// driver offers no encoder (the kernels then stage through load_prim).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static_assert(fhy::kMxRun == FLASH_HY_MX_RUN, "the run length of the header and the kernels agree");
static fhy::TmaLine *make_tma_maps(flash_hy_ctx *c, int K = 1) {
  if (c->ndim != 3 || c->nx != 8 || c->ny != 8 || c->nz != 8) return nullptr;
  static EncodeTiledFn encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return nullptr;
    encode = (EncodeTiledFn)fn;
  }
  void *mem = nullptr;
  if (posix_memalign(&mem, 64, 6 * sizeof(fhy::TmaLine)) != 0) return nullptr;
  fhy::TmaLine *m = static_cast<fhy::TmaLine *>(mem);
  memset(m, 0, 6 * sizeof(fhy::TmaLine));
  const cuuint64_t dims[3] = {8, 8, (cuuint64_t)c->nblocks * 8};
  const cuuint64_t strides[2] = {8 * sizeof(double), 64 * sizeof(double)};
  const cuuint32_t one[3] = {1, 1, 1};
  // runs (K > 1): 1/K of the slower transverse axis (z for the x and y
  // sweeps, y for the z sweep)
  const cuuint32_t q = (cuuint32_t)(8 / K);
  const cuuint32_t box_in[3][3] = {{8, 8, q}, {8, 8, q}, {8, q, 8}};
  const cuuint32_t box_slab[3][3] = {{4, 8, q}, {8, 4, q}, {8, q, 4}};
  for (int par = 0; par < 2; ++par)
    for (int d = 0; d < 3; ++d) {
      fhy::TmaLine &t = m[par * 3 + d];
      for (int v = 0; v < 5; ++v) {
        if (encode(&t.intr[v], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, c->state[par][v], dims, strides, box_in[d], one,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
            encode(&t.slab[v], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, c->state[par][v], dims, strides, box_slab[d], one,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
          free(m);
          return nullptr;
        }
      }
      t.on = 1;
    }
  return m;
}

static void drop_graphs(flash_hy_ctx *c) {
  for (int q = 0; q < 2; ++q) {
    if (c->gexec[q]) cudaGraphExecDestroy(c->gexec[q]);
    c->gexec[q] = nullptr;
  }
}

__global__ void k_set_dt(double *d, double dt) { *d = dt; }

static int amr_restrict_all(flash_hy_ctx *c);

static int fail(flash_hy_ctx *c, int code, const char *fmt, const char *detail) {
  if (c) snprintf(c->err, sizeof c->err, fmt, detail ? detail : "");
  return code;
}
#define CUDA_OK(c, call)                                                             \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) return fail((c), FLASH_HY_ERR_CUDA, "CUDA: %s", cudaGetErrorString(e_)); \
  } while (0)

static bool shape_supported(int ndim, int nx, int ny, int nz) {
  return (ndim == 2 && ((nx == 8 && ny == 8) || (nx == 16 && ny == 16))) ||
         (ndim == 3 && nx == 8 && ny == 8 && nz == 8);
}

static void fill_devparams(const flash_hy_ctx *c, DevParams &P) {
  memset(&P, 0, sizeof P);
  P.ndim = c->ndim;
  P.nbx = c->nbx; P.nby = c->nby; P.nbz = c->nbz;
  for (int f = 0; f < 6; ++f) P.bc[f] = c->bc[f];
  P.use_flattening = c->p.use_flattening;
  P.use_steepening = c->p.use_steepening;
  P.char_limiting = c->p.char_limiting;
  P.limiter = c->p.slope_limiter;
  P.use_aux_eint = c->p.use_aux_eint;
  P.use_ctu = c->p.use_3d_full_ctu;
  P.riemann = c->p.riemann_solver;
  P.learned = c->p.learned_guess;
  P.mlp = (c->p.learned_guess && c->mlp_set) ? c->d_mlp : nullptr;
  P.rs_tol = 1e-12;
  P.rs_max_iter = 50;
  if (c->harvest_cap > 0) {
    P.harvest = c->d_harvest;
    P.harvest_n = c->d_harvest_n;
    P.harvest_cap = c->harvest_cap;
    P.harvest_mask = c->harvest_mask;
  }
  P.lim_beta = c->p.limited_slope_beta;
  P.gamma = c->p.gamma;
  P.gas = xrs::gas_of(c->p.gamma);
  double gammam1 = 1.0 / (c->p.gamma - 1.0);            // eos_initGamma.F90:32
  P.gam1inv = 1. / gammam1;                             // eos_idealGamma.F90:323-326
  P.ggprodinv = 1. / (gammam1 * c->p.gas_constant);     // eos_idealGamma.F90:262
  P.abar = c->p.single_species_a;
  P.smalle = c->p.smalle;
  P.smlrho = c->p.smlrho;
  P.eswitch = c->p.eint_switch;
  P.tiny = c->p.tiny;
  P.cfl = c->p.cfl;
  for (int d = 0; d < 3; ++d) P.del[d] = c->del[d];
  P.blk_at = c->d_blk_at;
  P.blk_nbr = c->d_blk_nbr;
  P.blk_coord = c->d_blk_coord;
  P.status = c->d_status;
  for (int v = 0; v < 5; ++v) {
    P.s_in[v] = c->state[c->cur][v];
    P.s_out[v] = c->state[1 - c->cur][v];
  }
  if (c->nsp > 0) {
    P.nsp = c->nsp;
    P.nspec = c->nspec;
    P.sp_in = c->spec[c->cur];
    P.sp_out = c->spec[1 - c->cur];
    P.sp_mf = c->sp_mf;
    P.sp_fb = c->sp_fb;
    P.sp_flat = c->sp_flat;
    P.sp_ncells = c->ncells;
    P.sp_fstore = c->d_sp_fstore;
    if (c->amr) {
      P.sp_lh = c->sp_lh;
      P.sp_gp = c->sp_gp;
      P.sp_freg = c->sp_freg;
      P.sp_freg_stride = c->sp_freg_stride;
    }
  }
  if (c->amr) {
    P.blk_level = c->d_level;
    P.leaf = c->d_leaf;
    P.parent = c->d_parent;
    P.slot = c->d_slot;
    P.at = c->d_at;
    for (int l = 0; l < 17; ++l) {
      P.at_off[l] = c->at_off[l];
      for (int d = 0; d < 3; ++d) P.at_ext[l][d] = c->at_ext[l][d];
    }
    P.lh = c->d_lh;
    P.gp = c->d_gp;
    P.pe = c->d_pe;
    P.freg = c->d_freg;
  }
}

// Level tables of an AMR hierarchy given as all its tree nodes: a complete
// level 1, every other node's parent present, all 2^d children of a parent
// present.  2:1 balance across faces, edges and corners is the caller's
// contract (the guard fill and the flux register rely on it).
static int amr_tables(const flash_hy_grid_desc *g, std::vector<int> &at, int off[17], int ext[17][3],
                      std::vector<int> &parent, std::vector<int> &leaf) {
  const int L = g->max_level;
  if (L < 2 || L > 16 || !g->block_level) return FLASH_HY_ERR_BAD_ARG;
  long tot = 0;
  for (int l = 0; l < 17; ++l) {
    off[l] = (int)tot;
    for (int d = 0; d < 3; ++d) ext[l][d] = (l >= 1 && d < g->ndim) ? g->nblk_l1[d] << (l - 1) : 1;
    if (l >= 1 && l <= L) tot += (long)ext[l][0] * ext[l][1] * ext[l][2];
    if (tot > (1L << 30)) return FLASH_HY_ERR_UNSUPPORTED;
  }
  at.assign(tot, -1);
  auto node = [&](int l, int x, int y, int z) -> int {
    if (l < 1 || l > L || x < 0 || y < 0 || z < 0 || x >= ext[l][0] || y >= ext[l][1] || z >= ext[l][2]) return -1;
    return at[off[l] + ((long)z * ext[l][1] + y) * ext[l][0] + x];
  };
  for (int b = 0; b < g->nblocks; ++b) {
    int l = g->block_level[b];
    const int *cc = &g->block_coords[3 * b];
    int x = cc[0], y = g->ndim > 1 ? cc[1] : 0, z = g->ndim > 2 ? cc[2] : 0;
    if (l < 1 || l > L || x < 0 || y < 0 || z < 0 || x >= ext[l][0] || y >= ext[l][1] || z >= ext[l][2])
      return FLASH_HY_ERR_BAD_ARG;
    long q = off[l] + ((long)z * ext[l][1] + y) * ext[l][0] + x;
    if (at[q] >= 0) return FLASH_HY_ERR_BAD_ARG;
    at[q] = b;
  }
  for (long q = off[1]; q < off[1] + (long)ext[1][0] * ext[1][1] * ext[1][2]; ++q)
    if (at[q] < 0) return FLASH_HY_ERR_BAD_ARG;
  parent.assign(g->nblocks, -1);
  leaf.assign(g->nblocks, 0);
  const int nch_all = 1 << g->ndim;
  for (int b = 0; b < g->nblocks; ++b) {
    int l = g->block_level[b];
    const int *cc = &g->block_coords[3 * b];
    int x = cc[0], y = g->ndim > 1 ? cc[1] : 0, z = g->ndim > 2 ? cc[2] : 0;
    if (l > 1) {
      parent[b] = node(l - 1, x / 2, y / 2, z / 2);
      if (parent[b] < 0) return FLASH_HY_ERR_BAD_ARG;
    }
    int nch = 0;
    for (int o = 0; o < nch_all; ++o)
      nch += node(l + 1, 2 * x + (o & 1), g->ndim > 1 ? 2 * y + ((o >> 1) & 1) : 0, g->ndim > 2 ? 2 * z + (o >> 2) : 0) >= 0;
    if (nch != 0 && nch != nch_all) return FLASH_HY_ERR_BAD_ARG;
    leaf[b] = nch == 0;
  }
  return 0;
}

extern "C" int flash_hy_create(const flash_hy_params *params, const flash_hy_grid_desc *g, int device,
                               flash_hy_ctx **out) {
  if (!params || !g || !out) return FLASH_HY_ERR_BAD_ARG;
  *out = nullptr;
  if (params->order != 3 ||
      (params->riemann_solver != FLASH_HY_RS_HLLC && params->riemann_solver != FLASH_HY_RS_EXACT) ||
      params->f_pres_in_mom_flux != 1.0 || params->precision < 0 || params->precision > 2)
    return FLASH_HY_ERR_UNSUPPORTED;
  // the learned guess belongs to the exact solver and to the mixed path
  if (params->learned_guess &&
      (params->riemann_solver != FLASH_HY_RS_EXACT || params->precision != FLASH_HY_PREC_MIXED))
    return FLASH_HY_ERR_UNSUPPORTED;
  if (params->gamma <= 1.0 || params->cfl <= 0.0) return FLASH_HY_ERR_BAD_ARG;
  if (params->nspecies < 0 || params->nmass_scalars < 0 ||
      params->nspecies + params->nmass_scalars > FLASH_HY_MAX_SPECIES)
    return FLASH_HY_ERR_BAD_ARG;
  int nz = g->ndim > 2 ? g->nzb : 1, ny = g->ndim > 1 ? g->nyb : 1;
  if (!shape_supported(g->ndim, g->nxb, ny, nz)) return FLASH_HY_ERR_UNSUPPORTED;
  if (g->nblocks <= 0 || !g->block_coords || g->nguard < 0) return FLASH_HY_ERR_BAD_ARG;
  // the species pass addresses the cells of one species with 31-bit offsets
  if (params->nspecies + params->nmass_scalars > 0 && (double)g->nblocks * g->nxb * ny * nz > 2147483647.0)
    return FLASH_HY_ERR_UNSUPPORTED;
  int nbx = g->nblk_l1[0], nby = g->ndim > 1 ? g->nblk_l1[1] : 1, nbz = g->ndim > 2 ? g->nblk_l1[2] : 1;
  const bool amr = g->max_level > 1;
  std::vector<int> amr_at, amr_parent, amr_leaf;
  int amr_off[17], amr_ext[17][3];
  if (amr) {
    if (params->precision != FLASH_HY_PREC_FP64 && params->precision != FLASH_HY_PREC_MIXED) return FLASH_HY_ERR_UNSUPPORTED;
    if (nbx <= 0 || nby <= 0 || nbz <= 0) return FLASH_HY_ERR_BAD_ARG;
    int rc0 = amr_tables(g, amr_at, amr_off, amr_ext, amr_parent, amr_leaf);
    if (rc0) return rc0;
  } else if (nbx <= 0 || nby <= 0 || nbz <= 0 || (long)nbx * nby * nbz < g->nblocks) {
    return FLASH_HY_ERR_BAD_ARG;
  }
  // fewer blocks than positions: a rank's share of a grid (owned + ghost
  // blocks); such a context steps only the owned blocks it is given
  const bool partial = !amr && (long)nbx * nby * nbz > g->nblocks;
  std::vector<int> at(amr ? 0 : (size_t)nbx * nby * nbz, -1), coords(3 * (size_t)g->nblocks);
  for (int b = 0; b < g->nblocks && amr; ++b) {
    coords[3 * b] = g->block_coords[3 * b];
    coords[3 * b + 1] = g->ndim > 1 ? g->block_coords[3 * b + 1] : 0;
    coords[3 * b + 2] = g->ndim > 2 ? g->block_coords[3 * b + 2] : 0;
  }
  for (int b = 0; b < g->nblocks && !amr; ++b) {
    int x = g->block_coords[3 * b], y = g->ndim > 1 ? g->block_coords[3 * b + 1] : 0,
        z = g->ndim > 2 ? g->block_coords[3 * b + 2] : 0;
    if (x < 0 || x >= nbx || y < 0 || y >= nby || z < 0 || z >= nbz) return FLASH_HY_ERR_BAD_ARG;
    size_t a = ((size_t)z * nby + y) * nbx + x;
    if (at[a] >= 0) return FLASH_HY_ERR_BAD_ARG;
    at[a] = b;
    coords[3 * b] = x; coords[3 * b + 1] = y; coords[3 * b + 2] = z;
  }
  for (int f = 0; f < 2 * g->ndim; ++f)
    if (g->bc[f] != FLASH_HY_BC_OUTFLOW && g->bc[f] != FLASH_HY_BC_PERIODIC && g->bc[f] != FLASH_HY_BC_REFLECTING)
      return FLASH_HY_ERR_UNSUPPORTED;
  for (int d = 0; d < g->ndim; ++d)
    if ((g->bc[2 * d] == FLASH_HY_BC_PERIODIC) != (g->bc[2 * d + 1] == FLASH_HY_BC_PERIODIC)) return FLASH_HY_ERR_BAD_ARG;

  flash_hy_ctx *c = (flash_hy_ctx *)calloc(1, sizeof(flash_hy_ctx));
  c->p = *params;
  c->ndim = g->ndim; c->nx = g->nxb; c->ny = ny; c->nz = nz;
  c->nblocks = g->nblocks; c->nbx = nbx; c->nby = nby; c->nbz = nbz;
  c->partial = partial;
  if (!amr) {
    c->h_blk_at = (int *)malloc(at.size() * sizeof(int));
    memcpy(c->h_blk_at, at.data(), at.size() * sizeof(int));
  }
  for (int f = 0; f < 6; ++f) c->bc[f] = f < 2 * g->ndim ? g->bc[f] : FLASH_HY_BC_OUTFLOW;
  int nb[3] = {g->nxb, ny, nz}, nbl[3] = {nbx, nby, nbz};
  for (int d = 0; d < 3; ++d)
    c->del[d] = d < g->ndim ? (g->domain_hi[d] - g->domain_lo[d]) / (double)(nbl[d] * nb[d]) : 1.0;
  c->ncb = (size_t)g->nxb * ny * nz;
  c->ncells = c->ncb * g->nblocks;
  c->device = device;
  c->threads = g->ndim == 3 ? 320 : (g->nxb == 8 ? 96 : 288);  // line cells split evenly
  c->dir_threads = c->threads;
  c->mx_sel = 1;
  c->mx_runs = 1;
  c->mx_sweep = FLASH_HY_SWEEP_XYZ;
  c->host_ng = g->nguard;
  c->nspec = params->nspecies;
  c->nsp = params->nspecies + params->nmass_scalars;
  *out = c;
  int rc = 0;
#define ALLOC(ptr, bytes)                                                           \
  do {                                                                              \
    cudaError_t e_ = ctx_alloc((void **)&(ptr), (bytes));                           \
    if (e_ != cudaSuccess) { rc = fail(c, FLASH_HY_ERR_CUDA, "cudaMalloc: %s", cudaGetErrorString(e_)); goto bad; } \
  } while (0)
  if (cudaSetDevice(device) != cudaSuccess) { rc = fail(c, FLASH_HY_ERR_CUDA, "cudaSetDevice%s", ""); goto bad; }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    rc = fail(c, FLASH_HY_ERR_CUDA, "stream%s", ""); goto bad;
  }
  for (int s = 0; s < 2; ++s)
    for (int v = 0; v < 5; ++v) ALLOC(c->state[s][v], c->ncells * sizeof(double));
  ALLOC(c->acc, 5 * c->ncells * sizeof(double));
  if (g->ndim > 1) ALLOC(c->aux, (size_t)(g->ndim - 1) * 3 * c->ncells * sizeof(double));
  if (!amr) c->tma_maps = make_tma_maps(c);
  if (amr) {
    c->amr = 1;
    c->nlev = g->max_level;
    std::vector<int> slot(g->nblocks, -1), leaves;
    std::vector<std::vector<int>> lev_leaves(17), lev_parents(17);
    for (int b = 0; b < g->nblocks; ++b) {
      int l = g->block_level[b];
      if (amr_leaf[b]) { slot[b] = (int)leaves.size(); leaves.push_back(b); lev_leaves[l].push_back(b); }
    }
    int np = 0;
    for (int b = 0; b < g->nblocks; ++b)
      if (!amr_leaf[b]) { slot[b] = np++; lev_parents[g->block_level[b]].push_back(b); }
    c->nleaves = (int)leaves.size();
    c->nparents = np;
    for (int l = 0; l < 17; ++l) {
      c->at_off[l] = amr_off[l];
      for (int d = 0; d < 3; ++d) c->at_ext[l][d] = amr_ext[l][d];
    }
    const size_t hn = (size_t)(g->nxb + 8) * (g->ndim > 1 ? ny + 8 : 1) * (g->ndim > 2 ? nz + 8 : 1);
    const size_t nf = g->ndim == 2 ? (size_t)(g->nxb > ny ? g->nxb : ny) : (size_t)g->nxb * ny;
    int rb = params->precision == FLASH_HY_PREC_MIXED ? 4 : 8;
    ALLOC(c->sig, sig_bytes_per_block(g->ndim, g->nxb, ny, nz, rb) * c->nleaves);
    ALLOC(c->d_lh, (size_t)c->nleaves * 5 * hn * sizeof(double));
    if (np > 0) ALLOC(c->d_gp, (size_t)np * 6 * hn * sizeof(double));
    ALLOC(c->d_pe, c->ncells * sizeof(double));
    ALLOC(c->d_freg, (size_t)c->nleaves * 2 * g->ndim * nf * NFLX * sizeof(double));
    ALLOC(c->d_level, g->nblocks * sizeof(int));
    ALLOC(c->d_leaf, g->nblocks * sizeof(int));
    ALLOC(c->d_parent, g->nblocks * sizeof(int));
    ALLOC(c->d_slot, g->nblocks * sizeof(int));
    ALLOC(c->d_at, amr_at.size() * sizeof(int));
    ALLOC(c->d_leaves, leaves.size() * sizeof(int));
    bool ok = cudaMemcpy(c->d_level, g->block_level, g->nblocks * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_leaf, amr_leaf.data(), g->nblocks * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_parent, amr_parent.data(), g->nblocks * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_slot, slot.data(), g->nblocks * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_at, amr_at.data(), amr_at.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c->d_leaves, leaves.data(), leaves.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
    for (int l = 1; l <= c->nlev && ok; ++l) {
      c->lev_leaves[l] = (int)lev_leaves[l].size();
      c->lev_parents[l] = (int)lev_parents[l].size();
      if (c->lev_leaves[l]) {
        ALLOC(c->d_lev_leaves[l], lev_leaves[l].size() * sizeof(int));
        ok = cudaMemcpy(c->d_lev_leaves[l], lev_leaves[l].data(), lev_leaves[l].size() * sizeof(int),
                        cudaMemcpyHostToDevice) == cudaSuccess;
      }
      if (ok && c->lev_parents[l]) {
        ALLOC(c->d_lev_parents[l], lev_parents[l].size() * sizeof(int));
        ok = cudaMemcpy(c->d_lev_parents[l], lev_parents[l].data(), lev_parents[l].size() * sizeof(int),
                        cudaMemcpyHostToDevice) == cudaSuccess;
      }
    }
    if (!ok) { rc = fail(c, FLASH_HY_ERR_CUDA, "AMR table copies%s", ""); goto bad; }
  } else {
    int rb = params->precision == FLASH_HY_PREC_MIXED ? 4 : 8;
    ALLOC(c->sig, sig_bytes_per_block(g->ndim, g->nxb, ny, nz, rb) * g->nblocks);
  }
  if (c->nsp > 0) {
    // per-slot scratch: a slot per block, or per leaf on an AMR hierarchy
    const size_t nslot = amr ? (size_t)c->nleaves : (size_t)g->nblocks;
    const size_t lines = (size_t)(g->nxb + 2) * (g->ndim > 1 ? ny : 1) * (g->ndim > 2 ? nz : 1);
    for (int s = 0; s < 2; ++s) ALLOC(c->spec[s], (size_t)c->nsp * c->ncells * sizeof(double));
    ALLOC(c->sp_mf, nslot * g->ndim * lines * sizeof(double));
    ALLOC(c->sp_fb, nslot * g->ndim * lines);
    ALLOC(c->sp_flat, nslot * g->ndim * lines * sizeof(double));
    if (amr) {
      const size_t hn = (size_t)(g->nxb + 8) * (g->ndim > 1 ? ny + 8 : 1) * (g->ndim > 2 ? nz + 8 : 1);
      const size_t nf = g->ndim == 2 ? (size_t)(g->nxb > ny ? g->nxb : ny) : (size_t)g->nxb * ny;
      ALLOC(c->sp_lh, (size_t)c->nleaves * c->nsp * hn * sizeof(double));
      if (c->nparents > 0) ALLOC(c->sp_gp, (size_t)c->nparents * c->nsp * hn * sizeof(double));
      c->sp_freg_stride = (size_t)c->nleaves * 2 * g->ndim * nf;
      ALLOC(c->sp_freg, (size_t)c->nsp * c->sp_freg_stride * sizeof(double));
    }
  }
  if (!amr) ALLOC(c->d_blk_at, at.size() * sizeof(int));
  if (!amr) ALLOC(c->d_blk_nbr, (size_t)g->nblocks * 6 * sizeof(int));
  ALLOC(c->d_blk_coord, coords.size() * sizeof(int));
  ALLOC(c->d_part, g->nblocks * sizeof(CflPart));
  ALLOC(c->d_dt, sizeof(DtInfo));
  ALLOC(c->d_status, sizeof(unsigned));
  ALLOC(c->d_stepdt, sizeof(double));
  {
    const char *e = getenv("FLASH_HY_GRAPH");
    c->use_graph = !(e && e[0] == '0');
  }
  if (cudaMallocHost((void **)&c->h_dt, sizeof(DtInfo)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_status, sizeof(unsigned)) != cudaSuccess) {
    rc = fail(c, FLASH_HY_ERR_CUDA, "cudaMallocHost%s", ""); goto bad;
  }
  c->h_dt->dt = 0.0;
  c->h_dt->blk = -1;
  // face neighbours of every block, as the direction kernels look them up
  // (periodic wrap; -1 beyond other boundaries or for a block absent from
  // a rank's share)
  if (!amr) {
    std::vector<int> nbr((size_t)g->nblocks * 6, -1);
    for (int b = 0; b < g->nblocks; ++b)
      for (int d = 0; d < 3; ++d)
        for (int side = 0; side < 2; ++side) {
          int cc[3] = {coords[3 * b], coords[3 * b + 1], coords[3 * b + 2]};
          cc[d] += side ? 1 : -1;
          if (cc[d] < 0 || cc[d] >= nbl[d]) {
            if (d >= g->ndim || c->bc[2 * d + side] != FLASH_HY_BC_PERIODIC) continue;
            cc[d] = (cc[d] + nbl[d]) % nbl[d];
          }
          nbr[(size_t)6 * b + 2 * d + side] = at[((size_t)cc[2] * nby + cc[1]) * nbx + cc[0]];
        }
    if (cudaMemcpy(c->d_blk_nbr, nbr.data(), nbr.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = fail(c, FLASH_HY_ERR_CUDA, "init copies%s", ""); goto bad;
    }
    // runs of the mixed direction kernels: on a full grid whose block
    // counts divide by kMxRun, every block with coordinate = 0 mod kMxRun
    // along the sweep starts a run of kMxRun blocks (+ its neighbours below
    // and above the run); the species pass keeps one block per CTA
    constexpr int K = fhy::kMxRun;
    if (c->tma_maps && !partial && c->nsp == 0 && nbx % K == 0 && nby % K == 0 && nbz % K == 0) {
      bool ok = true;
      for (int d = 0; d < 3 && ok; ++d) {
        std::vector<int> runs;
        runs.reserve((size_t)g->nblocks / K * (K + 2));
        for (int b = 0; b < g->nblocks; ++b) {
          if (coords[3 * b + d] % K != 0) continue;
          int cur = b;
          for (int m = 0; m < K; ++m) {
            runs.push_back(cur);
            if (m < K - 1) cur = nbr[(size_t)6 * cur + 2 * d + 1];
            if (cur < 0) ok = false;
          }
          runs.push_back(nbr[(size_t)6 * b + 2 * d]);
          runs.push_back(nbr[(size_t)6 * runs[runs.size() - 2] + 2 * d + 1]);
          if (!ok) break;
        }
        if (!ok || runs.size() != (size_t)g->nblocks / K * (K + 2)) { ok = false; break; }
        ALLOC(c->d_runs[d], runs.size() * sizeof(int));
        if (cudaMemcpy(c->d_runs[d], runs.data(), runs.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
          rc = fail(c, FLASH_HY_ERR_CUDA, "init copies%s", ""); goto bad;
        }
      }
      if (ok) {
        ALLOC(c->d_cflq, (size_t)g->nblocks * K * sizeof(fhy::CflCand));
        c->tma_run = make_tma_maps(c, K);
        if (c->tma_run)
          for (int t = 0; t < 6; ++t) {
            c->tma_run[t].runs = c->d_runs[t % 3];
            c->tma_run[t].cflq = c->d_cflq;
          }
        if (c->tma_run) c->mx_runs = K;
      }
    }
  }
  if ((!amr && cudaMemcpy(c->d_blk_at, at.data(), at.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(c->d_blk_coord, coords.data(), coords.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(c->d_status, 0, sizeof(unsigned)) != cudaSuccess) {
    rc = fail(c, FLASH_HY_ERR_CUDA, "init copies%s", ""); goto bad;
  }
  return 0;
bad:
  return rc;
#undef ALLOC
}

static void xfer_free(flash_hy_ctx *c);

extern "C" int flash_hy_destroy(flash_hy_ctx *c) {
  if (!c) return FLASH_HY_ERR_BAD_ARG;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int s = 0; s < 2; ++s)
    for (int v = 0; v < 5; ++v) ctx_free(c->state[s][v]);
  ctx_free(c->acc); ctx_free(c->aux); ctx_free(c->sig);
  ctx_free(c->d_blk_at); ctx_free(c->d_blk_nbr); ctx_free(c->d_blk_coord); ctx_free(c->d_list);
  ctx_free(c->d_part); ctx_free(c->d_dt); ctx_free(c->d_status); ctx_free(c->d_stage);
  ctx_free(c->d_wmaster); ctx_free(c->d_mlp); ctx_free(c->d_harvest); ctx_free(c->d_harvest_n);
  drop_graphs(c);
  ctx_free(c->d_stepdt);
  ctx_free(c->d_level); ctx_free(c->d_leaf); ctx_free(c->d_parent); ctx_free(c->d_slot); ctx_free(c->d_at);
  ctx_free(c->d_leaves); ctx_free(c->d_lh); ctx_free(c->d_gp); ctx_free(c->d_pe); ctx_free(c->d_freg);
  for (int l = 0; l < 17; ++l) { ctx_free(c->d_lev_leaves[l]); ctx_free(c->d_lev_parents[l]); }
  ctx_free(c->d_owned); ctx_free(c->d_owned_mask); ctx_free(c->d_send); ctx_free(c->d_recv);
  ctx_free(c->d_inner); ctx_free(c->d_edge);
  free(c->h_owned); free(c->h_recv);
  ctx_free(c->d_fstore);
  ctx_free(c->d_sp_fstore);
  for (int s = 0; s < 2; ++s) ctx_free(c->spec[s]);
  ctx_free(c->sp_mf); ctx_free(c->sp_fb); ctx_free(c->sp_flat);
  ctx_free(c->d_err);
  ctx_free(c->sp_lh); ctx_free(c->sp_gp); ctx_free(c->sp_freg);
  free(c->h_blk_at);
  free(c->h_list);
  free(c->tma_maps);
  free(c->tma_run);
  for (int d = 0; d < 3; ++d) ctx_free(c->d_runs[d]);
  ctx_free(c->d_cflq);
  xfer_free(c);
  if (c->h_dt) cudaFreeHost(c->h_dt);
  if (c->h_status) cudaFreeHost(c->h_status);
  if (c->stream) cudaStreamDestroy(c->stream);
  free(c);
  return 0;
}

// ---------------------------------------------------------------------------
// UNK <-> device block store
//
// Only the variables the device needs (upload) or the state it owns
// (download) cross PCIe, packed as SoA [variable][cell] over the interiors:
// host threads gather them from the caller's UNK (either layout, with or
// without guard cells) into pinned buffers and the copy engine moves one
// sub-chunk while the next is gathered; downloads run the other way (device
// pack, copy, host scatter into the owned variables only; guard cells and
// variables the device does not own keep the caller's values).  A device
// kernel converts between the packed copy and the state (the upload's EOS;
// on AMR hierarchies the download's Eos_putData outputs, which on uniform
// grids the host derives from the five state variables).
// ---------------------------------------------------------------------------
struct HostLayout {
  int layout, nunk, ng[3], nt[3];
  int v_dens, v_eint, v_ener, v_gamc, v_game, v_pres, v_temp, v_velx, v_vely, v_velz;  // 0-based, -1 absent
  int v_spec;           // first species (0-based); species and mass scalars follow
};

static inline size_t unk_index(const HostLayout &L, size_t b, int i, int j, int k, int v) {
  if (L.layout == FLASH_HY_LAYOUT_VAR_FASTEST)
    return ((((size_t)b * L.nt[2] + k) * L.nt[1] + j) * L.nt[0] + i) * L.nunk + v;
  return ((((size_t)b * L.nunk + v) * L.nt[2] + k) * L.nt[1] + j) * L.nt[0] + i;
}

// the packed variables of a transfer: UNK indices (0-based) in packed order
struct PackList {
  int n;
  int unk[10 + FLASH_HY_MAX_SPECIES];
  // positions in the packed order (-1 absent): upload dens, velx, vely, velz, eint, ener,
  // species; download dens, velx, vely, velz, eint, pres, temp, gamc, game, ener, species
  int at[10], spec;
};

// The packed copy is chunked SoA: chunk c holds cells [c S, c S + n_c)
// (n_c = S but for the last chunk) as [variable][cell], one contiguous
// copy per chunk.
__device__ __forceinline__ size_t chunk_off(size_t t, size_t S, int nv, size_t ncells, int q) {
  const size_t c = t / S, c0 = c * S;
  const size_t n = ncells - c0 < S ? ncells - c0 : S;
  return c0 * nv + (size_t)q * n + (t - c0);
}

// upload: dens, velx, vely, velz, eint, ener (as mapped), species
__global__ void k_unpack_soa(const double *__restrict__ st, PackList pl, DevParams P, size_t ncells, size_t S) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= ncells) return;
  auto get = [&](int q) { return q < 0 ? 0.0 : st[chunk_off(t, S, pl.n, ncells, q)]; };
  double rho = get(pl.at[0]), vx = get(pl.at[1]), vy = get(pl.at[2]), vz = get(pl.at[3]);
  // Eos_getData.F90:80-96 then MODE_DENS_EI keeps eint (Grid_initDomain's EOS)
  double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
  double eint = pl.at[4] >= 0 ? get(pl.at[4]) : get(pl.at[5]) - ekin;
  if (pl.at[5] >= 0) {
    double ener = get(pl.at[5]);
    if (ener - ekin > rmax(P.smalle, P.eswitch * ekin)) eint = ener - ekin;
  }
  P.s_out[0][t] = rho; P.s_out[1][t] = vx; P.s_out[2][t] = vy; P.s_out[3][t] = vz; P.s_out[4][t] = eint;
  for (int q = 0; q < P.nsp; ++q) P.sp_out[(size_t)q * ncells + t] = get(pl.spec + q);
}

// download: Eos_putData.F90:95-106 of the gamma law for the owned variables
__global__ void k_pack_soa(double *__restrict__ st, PackList pl, DevParams P, int ncb, size_t ncells, size_t S) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= ncells) return;
  const size_t b = t / ncb;
  double rho = P.s_in[0][t], vx = P.s_in[1][t], vy = P.s_in[2][t], vz = P.s_in[3][t], e = P.s_in[4][t];
  double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
  double pres = rho * e * P.gam1inv;
  double temp = e * P.ggprodinv * P.abar;
  auto put = [&](int q, double x) { if (q >= 0) st[chunk_off(t, S, pl.n, ncells, q)] = x; };
  put(pl.at[0], rho); put(pl.at[1], vx); put(pl.at[2], vy); put(pl.at[3], vz);
  put(pl.at[4], e); put(pl.at[5], pres); put(pl.at[6], temp); put(pl.at[7], P.gamma);
  put(pl.at[8], pres / (e * rho) + 1); put(pl.at[9], (P.leaf && !P.leaf[b]) ? P.pe[t] : e + ekin);
  for (int q = 0; q < P.nsp; ++q) put(pl.spec + q, P.sp_in[(size_t)q * ncells + t]);
}

static int make_layout(flash_hy_ctx *c, int layout, int nunk, const flash_hy_varmap *vm, int nguard, HostLayout &L) {
  if (layout != FLASH_HY_LAYOUT_VAR_FASTEST && layout != FLASH_HY_LAYOUT_XYZ_FASTEST) return FLASH_HY_ERR_BAD_ARG;
  if (nunk <= 0 || !vm) return FLASH_HY_ERR_BAD_ARG;
  L.layout = layout; L.nunk = nunk;
  int nb[3] = {c->nx, c->ny, c->nz};
  for (int d = 0; d < 3; ++d) {
    L.ng[d] = d < c->ndim ? nguard : 0;
    L.nt[d] = nb[d] + 2 * L.ng[d];
  }
  const int *m = &vm->dens;
  int *o = &L.v_dens;
  for (int q = 0; q < 10; ++q) {
    if (m[q] < 0 || m[q] > nunk) return FLASH_HY_ERR_BAD_ARG;
    o[q] = m[q] - 1;
  }
  if (L.v_dens < 0 || L.v_velx < 0 || (L.v_eint < 0 && L.v_ener < 0)) return FLASH_HY_ERR_BAD_ARG;
  L.v_spec = -1;
  if (c->nsp > 0) {
    if (vm->species < 1 || vm->species - 1 + c->nsp > nunk) return FLASH_HY_ERR_BAD_ARG;
    L.v_spec = vm->species - 1;
  }
  return 0;
}

static PackList pack_list(const flash_hy_ctx *c, const HostLayout &L, bool upload) {
  PackList pl;
  pl.n = 0;
  auto add = [&](int v) { if (v < 0) return -1; pl.unk[pl.n] = v; return pl.n++; };
  for (int q = 0; q < 10; ++q) pl.at[q] = -1;
  if (upload) {
    const int vs[6] = {L.v_dens, L.v_velx, L.v_vely, L.v_velz, L.v_eint, L.v_ener};
    for (int q = 0; q < 6; ++q) pl.at[q] = add(vs[q]);
  } else {
    const int vs[10] = {L.v_dens, L.v_velx, L.v_vely, L.v_velz, L.v_eint,
                        L.v_pres, L.v_temp, L.v_gamc, L.v_game, L.v_ener};
    for (int q = 0; q < 10; ++q) pl.at[q] = add(vs[q]);
  }
  pl.spec = -1;
  for (int q = 0; q < c->nsp; ++q) {
    const int k = add(L.v_spec + q);
    if (q == 0) pl.spec = k;
  }
  return pl;
}

static int ensure_stage(flash_hy_ctx *c, size_t bytes) {
  if (c->stage_bytes >= bytes) return 0;
  if (c->d_stage) { cudaStreamSynchronize(c->stream); cudaFree(c->d_stage); c->d_stage = nullptr; c->stage_bytes = 0; }
  CUDA_OK(c, cudaMalloc((void **)&c->d_stage, bytes));
  c->stage_bytes = bytes;
  return 0;
}

// Per-context transfer workers: a stream, two pinned slots and their
// events per host thread (created on first use, kept until destroy).
struct XferPool {
  int nthreads;
  size_t slot_cells;                     // cells per sub-chunk (whole blocks)
  size_t slot_doubles;                   // slot_cells x the most packed variables
  cudaStream_t st[64];
  cudaEvent_t ev[64][2], done[64];
  double *pinned;                        // [nthreads][2][slot_doubles]
  cudaEvent_t start;                     // recorded on the context's stream
};

static void xfer_release(XferPool *x) {
  for (int t = 0; t < x->nthreads; ++t) {
    if (x->st[t]) cudaStreamDestroy(x->st[t]);
    for (int q = 0; q < 2; ++q) if (x->ev[t][q]) cudaEventDestroy(x->ev[t][q]);
    if (x->done[t]) cudaEventDestroy(x->done[t]);
  }
  if (x->start) cudaEventDestroy(x->start);
  if (x->pinned) cudaFreeHost(x->pinned);
  free(x);
}

static int xfer_pool(flash_hy_ctx *c, XferPool *&out) {
  if (c->xfer) { out = c->xfer; return 0; }
  XferPool *x = (XferPool *)calloc(1, sizeof(XferPool));
  if (!x) return fail(c, FLASH_HY_ERR_CUDA, "host allocation%s", "");
  const size_t per_block = c->ncb;
  const size_t blocks_per_slot = per_block >= 65536 ? 1 : 65536 / per_block;
  x->slot_cells = blocks_per_slot * per_block;
  x->slot_doubles = x->slot_cells * (10 + c->nsp);
  const int hw = (int)std::thread::hardware_concurrency();
  const size_t slots = (c->ncells + x->slot_cells - 1) / x->slot_cells;
  int n = hw > 0 ? hw : 1;
  if (n > 64) n = 64;
  if ((size_t)n > slots) n = (int)slots;
  x->nthreads = n;
  cudaError_t e = cudaEventCreateWithFlags(&x->start, cudaEventDisableTiming);
  for (int t = 0; t < n && e == cudaSuccess; ++t) {
    e = cudaStreamCreateWithFlags(&x->st[t], cudaStreamNonBlocking);
    for (int q = 0; q < 2 && e == cudaSuccess; ++q) e = cudaEventCreateWithFlags(&x->ev[t][q], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x->done[t], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaMallocHost((void **)&x->pinned, (size_t)n * 2 * x->slot_doubles * sizeof(double));
  if (e != cudaSuccess) {
    xfer_release(x);
    return fail(c, FLASH_HY_ERR_CUDA, "transfer buffers: %s", cudaGetErrorString(e));
  }
  c->xfer = x;
  out = x;
  return 0;
}

static void xfer_free(flash_hy_ctx *c) {
  if (c->xfer) xfer_release(c->xfer);
  c->xfer = nullptr;
}

// Run worker(t, first_chunk, end_chunk) on the pool's threads, the chunks
// (slot_cells cells each, whole blocks) split evenly into contiguous ranges;
// returns the first CUDA error any worker saw.
template <class F>
static cudaError_t run_workers(flash_hy_ctx *c, XferPool *x, F worker) {
  std::vector<cudaError_t> err(x->nthreads, cudaSuccess);
  const size_t nch = (c->ncells + x->slot_cells - 1) / x->slot_cells;
  auto body = [&](int t) {
    const size_t b0 = nch * t / x->nthreads, b1 = nch * (t + 1) / x->nthreads;
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = worker(t, b0, b1);
    err[t] = e;
  };
  if (x->nthreads == 1) {
    body(0);
  } else {
    std::vector<std::thread> th;
    th.reserve(x->nthreads);
    for (int t = 0; t < x->nthreads; ++t) th.emplace_back(body, t);
    for (auto &h : th) h.join();
  }
  for (cudaError_t e : err)
    if (e != cudaSuccess) return e;
  return cudaSuccess;
}

// gather (upload) or scatter (download) the packed variables of blocks
// [b0, b1) between the caller's UNK and a pinned slot laid out [var][cell]
// (non-temporal stores into the slot were measured slower: 232 vs 149 ms
// for the 512^3 upload)
static void host_gather(const flash_hy_ctx *c, const HostLayout &L, const PackList &pl, const double *unk, size_t b0,
                        size_t b1, double *slot) {
  const size_t n = (b1 - b0) * c->ncb;
  size_t t = 0;
  for (size_t b = b0; b < b1; ++b)
    for (int k = 0; k < c->nz; ++k)
      for (int j = 0; j < c->ny; ++j)
        for (int i = 0; i < c->nx; ++i, ++t) {
          const size_t base = unk_index(L, b, i + L.ng[0], j + L.ng[1], k + L.ng[2], 0);
          const size_t vstride = L.layout == FLASH_HY_LAYOUT_VAR_FASTEST
                                     ? 1
                                     : (size_t)L.nt[0] * L.nt[1] * L.nt[2];
          for (int q = 0; q < pl.n; ++q) slot[(size_t)q * n + t] = unk[base + (size_t)pl.unk[q] * vstride];
        }
}
static void host_scatter(const flash_hy_ctx *c, const HostLayout &L, const PackList &pl, double *unk, size_t b0,
                         size_t b1, const double *slot) {
  const size_t n = (b1 - b0) * c->ncb;
  size_t t = 0;
  for (size_t b = b0; b < b1; ++b)
    for (int k = 0; k < c->nz; ++k)
      for (int j = 0; j < c->ny; ++j)
        for (int i = 0; i < c->nx; ++i, ++t) {
          const size_t base = unk_index(L, b, i + L.ng[0], j + L.ng[1], k + L.ng[2], 0);
          const size_t vstride = L.layout == FLASH_HY_LAYOUT_VAR_FASTEST
                                     ? 1
                                     : (size_t)L.nt[0] * L.nt[1] * L.nt[2];
          for (int q = 0; q < pl.n; ++q) unk[base + (size_t)pl.unk[q] * vstride] = slot[(size_t)q * n + t];
        }
}

// Download of a uniform grid: only the five state variables (and the
// species) cross PCIe; the host writes them and the gamma-law EOS outputs
// of Eos_putData.F90:95-106 -- PRES, TEMP, GAMC, GAME, ENER -- with the same
// IEEE double operations, in the same order, as k_pack_soa (bit-identical:
// the host code has no FMA contraction).
static void host_scatter_eos(const flash_hy_ctx *c, const HostLayout &L, const DevParams &P, double *unk, size_t b0,
                             size_t b1, const double *slot, int nsp) {
  const size_t n = (b1 - b0) * c->ncb;
  const size_t vstride = L.layout == FLASH_HY_LAYOUT_VAR_FASTEST ? 1 : (size_t)L.nt[0] * L.nt[1] * L.nt[2];
  const double gam1inv = P.gam1inv, ggprodinv = P.ggprodinv, abar = P.abar, gamma = P.gamma;
  size_t t = 0;
  for (size_t b = b0; b < b1; ++b)
    for (int k = 0; k < c->nz; ++k)
      for (int j = 0; j < c->ny; ++j)
        for (int i = 0; i < c->nx; ++i, ++t) {
          const size_t base = unk_index(L, b, i + L.ng[0], j + L.ng[1], k + L.ng[2], 0);
          const double rho = slot[t], vx = slot[n + t], vy = slot[2 * n + t], vz = slot[3 * n + t],
                       e = slot[4 * n + t];
          const double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
          const double pres = rho * e * gam1inv;
          auto put = [&](int v, double val) { if (v >= 0) unk[base + (size_t)v * vstride] = val; };
          put(L.v_dens, rho); put(L.v_velx, vx); put(L.v_vely, vy); put(L.v_velz, vz); put(L.v_eint, e);
          put(L.v_pres, pres); put(L.v_temp, e * ggprodinv * abar); put(L.v_gamc, gamma);
          put(L.v_game, pres / (e * rho) + 1); put(L.v_ener, e + ekin);
          for (int q = 0; q < nsp; ++q) put(L.v_spec + q, slot[(size_t)(5 + q) * n + t]);
        }
}

extern "C" int flash_hy_upload(flash_hy_ctx *c, const double *unk, int layout, int nunk, const flash_hy_varmap *vm) {
  if (!c || !unk) return FLASH_HY_ERR_BAD_ARG;
  HostLayout L;
  int rc = make_layout(c, layout, nunk, vm, c->host_ng, L);
  if (rc) return fail(c, rc, "bad UNK layout or variable map%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  const PackList pl = pack_list(c, L, true);
  if ((rc = ensure_stage(c, (size_t)(10 + c->nsp) * c->ncells * sizeof(double)))) return rc;
  XferPool *x = nullptr;
  if ((rc = xfer_pool(c, x))) return rc;
  double *st = (double *)c->d_stage;
  CUDA_OK(c, cudaEventRecord(x->start, c->stream));   // earlier users of the stage buffer
  const size_t spb = x->slot_cells / c->ncb;           // blocks per chunk
  cudaError_t e = run_workers(c, x, [&](int t, size_t k0, size_t k1) -> cudaError_t {
    cudaError_t r = cudaStreamWaitEvent(x->st[t], x->start, 0);
    int s = 0;
    for (size_t k = k0; k < k1 && r == cudaSuccess; ++k, s ^= 1) {
      const size_t a = k * spb, a1 = a + spb < (size_t)c->nblocks ? a + spb : (size_t)c->nblocks;
      const size_t n = (a1 - a) * c->ncb;
      double *slot = x->pinned + ((size_t)t * 2 + s) * x->slot_doubles;
      r = cudaEventSynchronize(x->ev[t][s]);        // the slot's previous copy is done
      if (r != cudaSuccess) break;
      host_gather(c, L, pl, unk, a, a1, slot);
      r = cudaMemcpyAsync(st + a * c->ncb * pl.n, slot, n * pl.n * sizeof(double), cudaMemcpyHostToDevice, x->st[t]);
      if (r == cudaSuccess) r = cudaEventRecord(x->ev[t][s], x->st[t]);
    }
    if (r == cudaSuccess) r = cudaEventRecord(x->done[t], x->st[t]);
    return r;
  });
  if (e != cudaSuccess) return fail(c, FLASH_HY_ERR_CUDA, "upload copies: %s", cudaGetErrorString(e));
  for (int t = 0; t < x->nthreads; ++t) CUDA_OK(c, cudaStreamWaitEvent(c->stream, x->done[t], 0));
  DevParams P;
  fill_devparams(c, P);
  for (int v = 0; v < 5; ++v) P.s_out[v] = c->state[c->cur][v];
  if (c->nsp > 0) P.sp_out = c->spec[c->cur];
  k_unpack_soa<<<(unsigned)((c->ncells + 255) / 256), 256, 0, c->stream>>>(st, pl, P, c->ncells, x->slot_cells);
  CUDA_OK(c, cudaGetLastError());
  // the pinned slots are reused by the next transfer only after its event waits
  c->dt_valid = 0;
  return 0;
}

extern "C" int flash_hy_download(flash_hy_ctx *c, double *unk, int layout, int nunk, const flash_hy_varmap *vm) {
  if (!c || !unk) return FLASH_HY_ERR_BAD_ARG;
  HostLayout L;
  int rc = make_layout(c, layout, nunk, vm, c->host_ng, L);
  if (rc) return fail(c, rc, "bad UNK layout or variable map%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  // uniform grids: the five state variables and the species cross, the host
  // derives the EOS outputs; AMR hierarchies: the ten owned variables (a
  // parent's ENER is not eint + ekin)
  const bool derive = !c->amr;
  PackList pl = pack_list(c, L, false);
  if (derive) {
    pl.n = 5 + c->nsp;
    for (int q = 0; q < 10; ++q) pl.at[q] = q < 5 ? q : -1;
    pl.spec = c->nsp > 0 ? 5 : -1;
  }
  if ((rc = ensure_stage(c, (size_t)(10 + c->nsp) * c->ncells * sizeof(double)))) return rc;
  XferPool *x = nullptr;
  if ((rc = xfer_pool(c, x))) return rc;
  if (c->amr && amr_restrict_all(c)) return fail(c, FLASH_HY_ERR_CUDA, "restriction launch%s", "");
  double *st = (double *)c->d_stage;
  DevParams P;
  fill_devparams(c, P);
  k_pack_soa<<<(unsigned)((c->ncells + 255) / 256), 256, 0, c->stream>>>(st, pl, P, (int)c->ncb, c->ncells,
                                                                         x->slot_cells);
  CUDA_OK(c, cudaGetLastError());
  CUDA_OK(c, cudaEventRecord(x->start, c->stream));
  const size_t spb = x->slot_cells / c->ncb;
  const size_t nb = (size_t)c->nblocks;
  cudaError_t e = run_workers(c, x, [&](int t, size_t k0, size_t k1) -> cudaError_t {
    cudaError_t r = cudaStreamWaitEvent(x->st[t], x->start, 0);
    // copy chunk k + 1 while chunk k is scattered
    auto issue = [&](size_t k, int s) -> cudaError_t {
      const size_t a = k * spb, a1 = a + spb < nb ? a + spb : nb, n = (a1 - a) * c->ncb;
      double *slot = x->pinned + ((size_t)t * 2 + s) * x->slot_doubles;
      const cudaError_t q2 = cudaMemcpyAsync(slot, st + a * c->ncb * pl.n, n * pl.n * sizeof(double),
                                             cudaMemcpyDeviceToHost, x->st[t]);
      return q2 == cudaSuccess ? cudaEventRecord(x->ev[t][s], x->st[t]) : q2;
    };
    int s = 0;
    if (r == cudaSuccess && k0 < k1) r = issue(k0, 0);
    for (size_t k = k0; k < k1 && r == cudaSuccess; ++k, s ^= 1) {
      if (k + 1 < k1) r = issue(k + 1, s ^ 1);
      if (r == cudaSuccess) r = cudaEventSynchronize(x->ev[t][s]);
      if (r != cudaSuccess) break;
      const size_t a = k * spb, a1 = a + spb < nb ? a + spb : nb;
      const double *slot = x->pinned + ((size_t)t * 2 + s) * x->slot_doubles;
      if (derive) host_scatter_eos(c, L, P, unk, a, a1, slot, c->nsp);
      else host_scatter(c, L, pl, unk, a, a1, slot);
    }
    return r;
  });
  if (e != cudaSuccess) return fail(c, FLASH_HY_ERR_CUDA, "download copies: %s", cudaGetErrorString(e));
  return 0;
}

// ---------------------------------------------------------------------------
// step
// ---------------------------------------------------------------------------
// AMR: restriction (finest parents first), parent halos (coarsest first),
// leaf guard cells; returns the number of launches, or -1 on a launch error
template <int NDIM, int NX, int NY, int NZ>
static int amr_guard_fill(flash_hy_ctx *c, const DevParams &P) {
  double *const *st = c->state[c->cur];
  int n = 0;
  for (int l = c->nlev - 1; l >= 1; --l) {
    if (!c->lev_parents[l]) continue;
    k_restrict<NDIM, NX, NY, NZ><<<c->lev_parents[l], 256, 0, c->stream>>>(P, st[0], st[1], st[2], st[3], st[4],
                                                                          c->d_lev_parents[l],
                                                                          c->nsp ? c->spec[c->cur] : nullptr,
                                                                          c->ncells);
    ++n;
  }
  for (int l = 1; l < c->nlev; ++l) {
    if (!c->lev_parents[l]) continue;
    k_parent_halo<NDIM, NX, NY, NZ><<<c->lev_parents[l], 256, 0, c->stream>>>(P, st[0], st[1], st[2], st[3], st[4],
                                                                             c->d_lev_parents[l]);
    ++n;
  }
  k_leaf_halo<NDIM, NX, NY, NZ><<<c->nleaves, 256, 0, c->stream>>>(P, st[0], st[1], st[2], st[3], st[4], c->d_leaves);
  ++n;
  return cudaGetLastError() == cudaSuccess ? n : -1;
}

static int amr_prepare(flash_hy_ctx *c, const DevParams &P) {
  if (c->ndim == 2 && c->nx == 8) return amr_guard_fill<2, 8, 8, 1>(c, P);
  if (c->ndim == 2 && c->nx == 16) return amr_guard_fill<2, 16, 16, 1>(c, P);
  if (c->ndim == 3) return amr_guard_fill<3, 8, 8, 8>(c, P);
  return -1;
}

// parents = restriction of the current leaves (before a download)
static int amr_restrict_all(flash_hy_ctx *c) {
  DevParams P;
  fill_devparams(c, P);
  double *const *st = c->state[c->cur];
  double *sp = c->nsp ? c->spec[c->cur] : nullptr;
  for (int l = c->nlev - 1; l >= 1; --l) {
    if (!c->lev_parents[l]) continue;
    if (c->ndim == 2 && c->nx == 8)
      k_restrict<2, 8, 8, 1><<<c->lev_parents[l], 256, 0, c->stream>>>(P, st[0], st[1], st[2], st[3], st[4], c->d_lev_parents[l],
                                                               sp, c->ncells);
    else if (c->ndim == 2)
      k_restrict<2, 16, 16, 1><<<c->lev_parents[l], 256, 0, c->stream>>>(P, st[0], st[1], st[2], st[3], st[4], c->d_lev_parents[l],
                                                               sp, c->ncells);
    else
      k_restrict<3, 8, 8, 8><<<c->lev_parents[l], 256, 0, c->stream>>>(P, st[0], st[1], st[2], st[3], st[4], c->d_lev_parents[l],
                                                               sp, c->ncells);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

static int enqueue_step(flash_hy_ctx *c, double dt, const int *d_list, int nlaunch, const double *dt_dev = nullptr,
                        bool set_attr = true, int fmode = 0) {
  StepArgs a;
  fill_devparams(c, a.P);
  a.P.dt = dt;
  a.P.dt_dev = dt_dev;
  a.P.fmode = fmode;
  a.P.fstore = c->d_fstore;
  a.no_sig = fmode == 3;
  a.set_attr = set_attr;
  a.P.blk_list = d_list;
  a.sig = c->sig;
  a.acc = c->acc;
  a.aux = c->aux;
  a.ncells = c->ncells;
  a.part = c->d_part;
  a.nlaunch = nlaunch;
  a.threads = c->threads;
  a.dir_threads = c->dir_threads;
  a.mx_sel = c->mx_sel;
  a.sweep = c->p.precision == FLASH_HY_PREC_MIXED && c->mx_sweep == FLASH_HY_SWEEP_ZYX ? 1 : 0;
  a.stream = c->stream;
  a.tma = c->tma_maps ? c->tma_maps + 3 * c->cur : nullptr;
  a.tma_run = c->tma_run && c->mx_runs > 1 ? c->tma_run + 3 * c->cur : nullptr;
  a.nblocks = c->nblocks;
  a.nlev = 0;
  int pre = 0;
  if (c->amr) {
    pre = amr_prepare(c, a.P);
    if (pre < 0) return fail(c, FLASH_HY_ERR_CUDA, "AMR guard-cell launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    a.nlev = c->nlev;
    a.leaves = c->d_leaves;
    a.nleaves = c->nleaves;
    for (int l = 0; l < 17; ++l) { a.lev_list[l] = c->d_lev_leaves[l]; a.lev_count[l] = c->lev_leaves[l]; }
  }
  int n;
  switch (c->p.precision) {
    case FLASH_HY_PREC_FP64_FMA: n = step_fp64_fma(a, c->ndim, c->nx, c->ny, c->nz); break;
    case FLASH_HY_PREC_MIXED: n = step_mixed(a, c->ndim, c->nx, c->ny, c->nz); break;
    default: n = step_fp64_exact(a, c->ndim, c->nx, c->ny, c->nz); break;
  }
  if (n == -1) return fail(c, FLASH_HY_ERR_UNSUPPORTED, "unsupported block shape%s", "");
  if (n < 0) return fail(c, FLASH_HY_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  if (c->nsp > 0) {
    SpecArgs sa;
    sa.P = a.P;
    sa.mixed = c->p.precision == FLASH_HY_PREC_MIXED;
    sa.P.sp_fstore = c->d_sp_fstore;
    sa.ncells = c->ncells;
    sa.nlaunch = nlaunch;
    sa.stream = c->stream;
    sa.nlev = a.nlev;
    for (int l = 0; l < 17; ++l) { sa.lev_list[l] = a.lev_list[l]; sa.lev_count[l] = a.lev_count[l]; }
    const int ns = spec_step(sa, c->ndim, c->nx, c->ny, c->nz);
    if (ns < 0) return fail(c, FLASH_HY_ERR_CUDA, "species launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    n += ns;
  }
  c->launches = n + pre;
  return 0;
}

extern "C" int flash_hy_step(flash_hy_ctx *c, double simTime, double dt, double dtOld, int sweepOrder) {
  (void)simTime; (void)dtOld; (void)sweepOrder;
  if (!c) return FLASH_HY_ERR_BAD_ARG;
  if (!(dt > 0.0)) return fail(c, FLASH_HY_ERR_NONPOS_DT, "dt must be positive%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  if (c->partial && c->n_owned == 0)
    return fail(c, FLASH_HY_ERR_UNSUPPORTED, "a partial grid needs its owned blocks (flash_hy_set_owned_blocks)%s", "");
  const int *step_list = c->n_owned ? c->d_owned : nullptr;
  const int step_n = c->n_owned ? c->n_owned : c->nblocks;
  if (!c->use_graph) {
    int rc = enqueue_step(c, dt, step_list, step_n);
    if (rc) return rc;
  } else {
    const int q = c->cur;
    k_set_dt<<<1, 1, 0, c->stream>>>(c->d_stepdt, dt);
    CUDA_OK(c, cudaGetLastError());
    if (!c->gexec[q] && c->plain_steps[q] == 0) {
      // first step of this parity runs uncaptured (it also sets the kernels'
      // shared-memory attributes, which are not stream work)
      int rc = enqueue_step(c, dt, step_list, step_n, c->d_stepdt, true);
      if (rc) return rc;
      c->plain_steps[q]++;
      c->launches = c->launches + 1;
    } else {
      if (!c->gexec[q]) {
        cudaGraph_t g = nullptr;
        CUDA_OK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(c, dt, step_list, step_n, c->d_stepdt, false);
        cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (ec != cudaSuccess) return fail(c, FLASH_HY_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ec));
        ec = cudaGraphInstantiate(&c->gexec[q], g, 0);
        cudaGraphDestroy(g);
        if (ec != cudaSuccess) {
          c->gexec[q] = nullptr;
          return fail(c, FLASH_HY_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ec));
        }
        c->glaunches[q] = c->launches;
      }
      CUDA_OK(c, cudaGraphLaunch(c->gexec[q], c->stream));
      c->launches = c->glaunches[q] + 1;
    }
  }
  c->cur = 1 - c->cur;
  c->dt_valid = 1;
  return 0;
}

extern "C" int flash_hy_step_phase(flash_hy_ctx *c, double simTime, double dt, double dtOld, int phase) {
  (void)simTime; (void)dtOld;
  if (!c || (phase != 1 && phase != 2)) return FLASH_HY_ERR_BAD_ARG;
  if (c->n_owned == 0)
    return fail(c, FLASH_HY_ERR_UNSUPPORTED, "step_phase needs a rank's owned blocks (flash_hy_set_owned_blocks)%s", "");
  if (!(dt > 0.0)) return fail(c, FLASH_HY_ERR_NONPOS_DT, "dt must be positive%s", "");
  if (phase == 2 && (!c->phase_pending || dt != c->phase_dt))
    return fail(c, FLASH_HY_ERR_BAD_ARG, "step_phase 2 must follow phase 1 with the same dt%s", "");
  if (phase == 1 && c->phase_pending)
    return fail(c, FLASH_HY_ERR_BAD_ARG, "step_phase 1 twice without phase 2%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  const int *list = phase == 1 ? c->d_inner : c->d_edge;
  const int n = phase == 1 ? c->n_inner : c->n_edge;
  if (n > 0) {
    const int rc = enqueue_step(c, dt, list, n);
    if (rc) return rc;
  }
  if (phase == 1) {
    c->phase_pending = 1;
    c->phase_dt = dt;
  } else {
    c->phase_pending = 0;
    c->cur = 1 - c->cur;
    c->dt_valid = 1;
  }
  return 0;
}

// device copy of a caller's block list (kept in the context): FLASH's
// 1-based block IDs (blockList(1:blockCount)), stored 0-based
static int upload_list(flash_hy_ctx *c, int n, const int *list) {
  if (n > c->h_list_cap) {
    int *p = (int *)realloc(c->h_list, (size_t)n * sizeof(int));
    if (!p) return fail(c, FLASH_HY_ERR_CUDA, "host allocation of the block list%s", "");
    c->h_list = p;
    c->h_list_cap = n;
  }
  for (int q = 0; q < n; ++q) {
    if (list[q] < 1 || list[q] > c->nblocks)
      return fail(c, FLASH_HY_ERR_BAD_ARG, "block ID %s outside 1..nblocks (FLASH's 1-based blockList)",
                  std::to_string(list[q]).c_str());
    c->h_list[q] = list[q] - 1;
  }
  if (n > c->list_cap) {
    cudaStreamSynchronize(c->stream);
    cudaFree(c->d_list);
    c->d_list = nullptr;
    CUDA_OK(c, cudaMalloc((void **)&c->d_list, n * sizeof(int)));
    c->list_cap = n;
  }
  if (n > 0) {
    CUDA_OK(c, cudaMemcpyAsync(c->d_list, c->h_list, n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUDA_OK(c, cudaStreamSynchronize(c->stream));   // h_list is reused by the next call
  }
  return 0;
}

// blocks outside a list keep their state in the buffer the step writes
static int carry_state(flash_hy_ctx *c) {
  for (int v = 0; v < 5; ++v)
    CUDA_OK(c, cudaMemcpyAsync(c->state[1 - c->cur][v], c->state[c->cur][v], c->ncells * sizeof(double),
                               cudaMemcpyDeviceToDevice, c->stream));
  if (c->nsp > 0)
    CUDA_OK(c, cudaMemcpyAsync(c->spec[1 - c->cur], c->spec[c->cur], (size_t)c->nsp * c->ncells * sizeof(double),
                               cudaMemcpyDeviceToDevice, c->stream));
  return 0;
}

extern "C" int flash_hy_step_blocks(flash_hy_ctx *c, int blockCount, const int *blockList, double timeEndAdv,
                                    double dt, double dtOld, int sweepOrder) {
  (void)timeEndAdv; (void)dtOld; (void)sweepOrder;
  if (!c || blockCount < 0 || (blockCount > 0 && !blockList)) return FLASH_HY_ERR_BAD_ARG;
  if (c->amr) return fail(c, FLASH_HY_ERR_UNSUPPORTED, "block lists on an AMR hierarchy%s", "");
  if (!(dt > 0.0)) return fail(c, FLASH_HY_ERR_NONPOS_DT, "dt must be positive%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  int rc = upload_list(c, blockCount, blockList);
  if (rc) return rc;
  if ((rc = carry_state(c))) return rc;
  if (blockCount > 0) {
    rc = enqueue_step(c, dt, c->d_list, blockCount);
    if (rc) return rc;
  }
  c->cur = 1 - c->cur;
  c->dt_valid = 0;
  return 0;
}

// ---------------------------------------------------------------------------
// split step: fluxes, then the update (hy_computeFluxes / hy_updateSolution)
// ---------------------------------------------------------------------------
static int ensure_fstore(flash_hy_ctx *c) {
  if (c->d_fstore) return 0;
  const size_t nf = (size_t)(c->nx + 1) * c->ny * c->nz;
  const size_t per = (size_t)NFLX * nf + c->ncb;
  CUDA_OK(c, cudaMalloc((void **)&c->d_fstore, (size_t)c->nblocks * c->ndim * per * sizeof(double)));
  if (c->nsp > 0)
    CUDA_OK(c, cudaMalloc((void **)&c->d_sp_fstore, (size_t)c->nblocks * c->ndim * c->nsp * nf * sizeof(double)));
  return 0;
}

extern "C" int flash_hy_compute_fluxes(flash_hy_ctx *c, int blockCount, const int *blockList, double dt, int flags) {
  if (!c || blockCount < 0 || (blockCount > 0 && !blockList)) return FLASH_HY_ERR_BAD_ARG;
  if (flags != FLASH_HY_UPDATE_NONE && flags != FLASH_HY_UPDATE_ALL) return fail(c, FLASH_HY_ERR_BAD_ARG, "flags%s", "");
  if (c->amr) return fail(c, FLASH_HY_ERR_UNSUPPORTED, "split step on an AMR hierarchy%s", "");
  if (!(dt > 0.0)) return fail(c, FLASH_HY_ERR_NONPOS_DT, "dt must be positive%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  int rc = ensure_fstore(c);
  if (rc) return rc;
  if ((rc = upload_list(c, blockCount, blockList))) return rc;
  if (flags == FLASH_HY_UPDATE_ALL && (rc = carry_state(c))) return rc;
  if (blockCount > 0) {
    rc = enqueue_step(c, dt, c->d_list, blockCount, nullptr, true, flags == FLASH_HY_UPDATE_ALL ? 1 : 2);
    if (rc) return rc;
  }
  if (flags == FLASH_HY_UPDATE_ALL) {
    c->cur = 1 - c->cur;
    c->dt_valid = 0;
  }
  return 0;
}

extern "C" int flash_hy_update_solution(flash_hy_ctx *c, int blockCount, const int *blockList, double dt) {
  if (!c || blockCount < 0 || (blockCount > 0 && !blockList)) return FLASH_HY_ERR_BAD_ARG;
  if (c->amr) return fail(c, FLASH_HY_ERR_UNSUPPORTED, "split step on an AMR hierarchy%s", "");
  if (!c->d_fstore) return fail(c, FLASH_HY_ERR_BAD_ARG, "no stored fluxes (flash_hy_compute_fluxes first)%s", "");
  if (!(dt > 0.0)) return fail(c, FLASH_HY_ERR_NONPOS_DT, "dt must be positive%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  int rc = upload_list(c, blockCount, blockList);
  if (rc) return rc;
  if ((rc = carry_state(c))) return rc;
  if (blockCount > 0) {
    rc = enqueue_step(c, dt, c->d_list, blockCount, nullptr, true, 3);
    if (rc) return rc;
  }
  c->cur = 1 - c->cur;
  c->dt_valid = 0;
  return 0;
}

// blk: 0-based block (the entry points take FLASH's 1-based blockID)
static int flux_span(flash_hy_ctx *c, int blk, int dir, size_t &off, size_t &nf) {
  if (blk < 0 || blk >= c->nblocks || dir < 1 || dir > c->ndim) return FLASH_HY_ERR_BAD_ARG;
  if (!c->d_fstore) return FLASH_HY_ERR_BAD_ARG;
  nf = (size_t)(c->nx + 1) * c->ny * c->nz;
  const size_t per = (size_t)NFLX * nf + c->ncb;
  off = ((size_t)blk * c->ndim + (dir - 1)) * per;
  return 0;
}

// species fluxes of a block and direction in the species flux store
static size_t sp_flux_off(const flash_hy_ctx *c, int blk, int dir, size_t nf) {
  return ((size_t)blk * c->ndim + (dir - 1)) * c->nsp * nf;
}

extern "C" int flash_hy_get_fluxes(flash_hy_ctx *c, int blockID, int dir, double *flx) {
  if (!c || !flx) return FLASH_HY_ERR_BAD_ARG;
  const int blk = blockID - 1;
  size_t off, nf;
  if (flux_span(c, blk, dir, off, nf)) return fail(c, FLASH_HY_ERR_BAD_ARG, "get_fluxes: %s", "bad block/direction");
  CUDA_OK(c, cudaSetDevice(c->device));
  const int nfl = NFLX + c->nsp;
  std::vector<double> h(NFLX * nf), hs((size_t)c->nsp * nf);
  CUDA_OK(c, cudaMemcpyAsync(h.data(), c->d_fstore + off, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (c->nsp > 0)
    CUDA_OK(c, cudaMemcpyAsync(hs.data(), c->d_sp_fstore + sp_flux_off(c, blk, dir, nf), hs.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  for (size_t f = 0; f < nf; ++f) {
    for (int v = 0; v < NFLX; ++v) flx[f * nfl + v] = h[v * nf + f];
    for (int q = 0; q < c->nsp; ++q) flx[f * nfl + NFLX + q] = hs[q * nf + f];
  }
  return 0;
}

extern "C" int flash_hy_put_fluxes(flash_hy_ctx *c, int blockID, int dir, const double *flx) {
  if (!c || !flx) return FLASH_HY_ERR_BAD_ARG;
  const int blk = blockID - 1;
  size_t off, nf;
  if (flux_span(c, blk, dir, off, nf)) return fail(c, FLASH_HY_ERR_BAD_ARG, "put_fluxes: %s", "bad block/direction");
  CUDA_OK(c, cudaSetDevice(c->device));
  const int nfl = NFLX + c->nsp;
  std::vector<double> h(NFLX * nf), hs((size_t)c->nsp * nf);
  for (size_t f = 0; f < nf; ++f) {
    for (int v = 0; v < NFLX; ++v) h[v * nf + f] = flx[f * nfl + v];
    for (int q = 0; q < c->nsp; ++q) hs[q * nf + f] = flx[f * nfl + NFLX + q];
  }
  CUDA_OK(c, cudaMemcpyAsync(c->d_fstore + off, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (c->nsp > 0)
    CUDA_OK(c, cudaMemcpyAsync(c->d_sp_fstore + sp_flux_off(c, blk, dir, nf), hs.data(), hs.size() * sizeof(double),
                               cudaMemcpyHostToDevice, c->stream));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  return 0;
}

__global__ void k_dt_reduce(const CflPart *part, int nblocks, const int *blk_level, const int *leaf, int ndim,
                            DtInfo *out) {
  __shared__ double sdt[1024];
  __shared__ int sb[1024];
  double best = DBL_MAX;
  int bb = 0x7fffffff;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    if (leaf && !leaf[b]) continue;
    double d = part[b].dt;
    if (d < best || (d == best && b < bb)) { best = d; bb = b; }
  }
  sdt[threadIdx.x] = best; sb[threadIdx.x] = bb;
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
    DtInfo r;
    r.dt = sdt[0];
    int b = sb[0];
    if (b >= 0 && b < nblocks && part[b].i >= 0) {
      const int NG = 4;
      r.i = part[b].i + NG + 1;
      r.j = ndim > 1 ? part[b].j + NG + 1 : 1;
      r.k = ndim > 2 ? part[b].k + NG + 1 : 1;
      r.level = blk_level ? blk_level[b] : 1;
      r.blk = b;
    } else {
      r.i = r.j = r.k = 0; r.level = 0; r.blk = -1;
    }
    *out = r;
  }
}

extern "C" int flash_hy_compute_dt(flash_hy_ctx *c, double *dt_out, int minloc_out[5]) {
  if (!c || !dt_out) return FLASH_HY_ERR_BAD_ARG;
  CUDA_OK(c, cudaSetDevice(c->device));
  if (!c->dt_valid) {
    StepArgs a;
    fill_devparams(c, a.P);
    a.part = c->d_part;
    a.nlaunch = c->nblocks;
    a.threads = c->threads;
    a.dir_threads = c->dir_threads;
    a.mx_sel = c->mx_sel;
    a.stream = c->stream;
    a.tma = nullptr;
    a.set_attr = true;
    if (cfl_state(a, c->ndim, c->nx, c->ny, c->nz) < 0) return fail(c, FLASH_HY_ERR_CUDA, "cfl launch%s", "");
    c->dt_valid = 1;
  }
  k_dt_reduce<<<1, 1024, 0, c->stream>>>(c->d_part, c->nblocks, c->amr ? c->d_level : nullptr,
                                         c->amr ? c->d_leaf : (c->n_owned ? c->d_owned_mask : nullptr), c->ndim,
                                         c->d_dt);
  CUDA_OK(c, cudaGetLastError());
  CUDA_OK(c, cudaMemcpyAsync(c->h_dt, c->d_dt, sizeof(DtInfo), cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(c, cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  *dt_out = c->h_dt->dt;
  if (minloc_out) {
    minloc_out[0] = c->h_dt->i; minloc_out[1] = c->h_dt->j; minloc_out[2] = c->h_dt->k;
    minloc_out[3] = c->h_dt->level; minloc_out[4] = c->mesh_me;
  }
  int st = (int)*c->h_status;
  if (!(c->h_dt->dt > 0.0)) st |= FLASH_HY_ERR_NONPOS_DT;
  return st;
}

extern "C" int flash_hy_set_mesh_me(flash_hy_ctx *c, int rank) {
  if (!c || rank < 0) return FLASH_HY_ERR_BAD_ARG;
  c->mesh_me = rank;
  return 0;
}

extern "C" int flash_hy_dt_block(flash_hy_ctx *c, int *blockID) {
  if (!c || !blockID) return FLASH_HY_ERR_BAD_ARG;
  // h_dt holds the result of the last flash_hy_compute_dt (synchronised)
  *blockID = c->h_dt->blk >= 0 ? c->h_dt->blk + 1 : 0;
  return 0;
}

// ---------------------------------------------------------------------------
// launch shapes and the autotuner
// ---------------------------------------------------------------------------
static int thread_candidates(const flash_hy_ctx *c, int *v) {
  if (c->ndim == 3) { const int s[] = {128, 192, 256, 320}; memcpy(v, s, sizeof(s)); return 4; }
  if (c->nx == 8) { const int s[] = {64, 96, 128}; memcpy(v, s, sizeof(s)); return 3; }
  const int s[] = {128, 192, 256, 288, 320};
  memcpy(v, s, sizeof(s));
  return 5;
}
static int index_of(const int *v, int n, int x) {
  for (int q = 0; q < n; ++q)
    if (v[q] == x) return q;
  return -1;
}

extern "C" int flash_hy_tuning_candidates(flash_hy_ctx *c, int *sig, int *n_sig, int *dir, int *n_dir, int *mx,
                                          int *n_mx) {
  if (!c || !sig || !n_sig || !dir || !n_dir || !mx || !n_mx) return FLASH_HY_ERR_BAD_ARG;
  *n_sig = thread_candidates(c, sig);
  *n_dir = thread_candidates(c, dir);
  *n_mx = 3;
  for (int q = 0; q < 3; ++q) mx[q] = mx_threads_of(q, c->ndim, c->nx);
  return 0;
}

extern "C" int flash_hy_get_tuning(flash_hy_ctx *c, flash_hy_tuning *out) {
  if (!c || !out) return FLASH_HY_ERR_BAD_ARG;
  out->sig_threads = c->threads;
  out->dir_threads = c->dir_threads;
  out->mx_threads = mx_threads_of(c->mx_sel, c->ndim, c->nx);
  out->mx_runs = c->mx_runs;
  out->mx_sweep = c->mx_sweep;
  return 0;
}

extern "C" int flash_hy_set_tuning(flash_hy_ctx *c, const flash_hy_tuning *t) {
  if (!c || !t) return FLASH_HY_ERR_BAD_ARG;
  int cand[FLASH_HY_TUNE_MAX];
  const int n = thread_candidates(c, cand);
  int sel = -1;
  for (int q = 0; q < 3; ++q)
    if (mx_threads_of(q, c->ndim, c->nx) == t->mx_threads) sel = q;
  if (index_of(cand, n, t->sig_threads) < 0 || index_of(cand, n, t->dir_threads) < 0 || sel < 0)
    return fail(c, FLASH_HY_ERR_BAD_ARG, "set_tuning: %s", "not a candidate launch shape of this block shape");
  if (t->mx_runs != 1 && !(t->mx_runs == fhy::kMxRun && c->tma_run))
    return fail(c, FLASH_HY_ERR_BAD_ARG, "set_tuning: %s", "mx_runs is 1 or FLASH_HY_MX_RUN where runs are offered");
  if (t->mx_sweep != FLASH_HY_SWEEP_XYZ &&
      !(t->mx_sweep == FLASH_HY_SWEEP_ZYX && c->p.precision == FLASH_HY_PREC_MIXED))
    return fail(c, FLASH_HY_ERR_BAD_ARG, "set_tuning: %s",
                "mx_sweep is FLASH_HY_SWEEP_XYZ, or FLASH_HY_SWEEP_ZYX on the mixed-precision path");
  if (t->sig_threads != c->threads || t->dir_threads != c->dir_threads || sel != c->mx_sel ||
      t->mx_runs != c->mx_runs || t->mx_sweep != c->mx_sweep) {
    CUDA_OK(c, cudaSetDevice(c->device));
    CUDA_OK(c, cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->plain_steps[0] = c->plain_steps[1] = 0;
  }
  c->threads = t->sig_threads;
  c->dir_threads = t->dir_threads;
  c->mx_sel = sel;
  c->mx_runs = t->mx_runs;
  c->mx_sweep = t->mx_sweep;
  return 0;
}

extern "C" int flash_hy_autotune(flash_hy_ctx *c, double dt, int steps, flash_hy_tuning *best,
                                 flash_hy_tuning *table, float *table_ms, int cap, int *n_trials) {
  if (!c || !(dt > 0.0) || steps < 1 || steps > 1000 || cap < 0 || (cap > 0 && (!table || !table_ms)))
    return FLASH_HY_ERR_BAD_ARG;
  if (c->partial && c->n_owned == 0)
    return fail(c, FLASH_HY_ERR_UNSUPPORTED, "a partial grid needs its owned blocks (flash_hy_set_owned_blocks)%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  const int *step_list = c->n_owned ? c->d_owned : nullptr;
  const int step_n = c->n_owned ? c->n_owned : c->nblocks;
  const int cur0 = c->cur;
  const size_t vbytes = c->ncells * sizeof(double);
  const int nkeep = 5 + c->nsp;       // state variables, then species and mass scalars
  unsigned saved_status = 0;
  CUDA_OK(c, cudaMemcpy(&saved_status, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  double *keep = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = 0, nt = 0;
  const int sig0 = c->threads, dir0 = c->dir_threads, sel0 = c->mx_sel, runs0 = c->mx_runs, sweep0 = c->mx_sweep;
  int cand[FLASH_HY_TUNE_MAX];
  const int ncand = thread_candidates(c, cand);
  const bool mixed = c->p.precision == FLASH_HY_PREC_MIXED;
  auto restore = [&]() -> cudaError_t {
    for (int v = 0; v < nkeep; ++v) {
      double *dst = v < 5 ? c->state[cur0][v] : c->spec[cur0] + (size_t)(v - 5) * c->ncells;
      cudaError_t e = cudaMemcpyAsync(dst, keep + (size_t)v * c->ncells, vbytes, cudaMemcpyDeviceToDevice, c->stream);
      if (e != cudaSuccess) return e;
    }
    c->cur = cur0;
    return cudaSuccess;
  };
  // one trial: untimed step, then `steps` timed steps, from the kept state
  auto trial = [&](float &ms) -> int {
    if (restore() != cudaSuccess) return fail(c, FLASH_HY_ERR_CUDA, "autotune: %s", "state restore");
    for (int s = 0; s <= steps; ++s) {
      if (s == 1 && cudaEventRecord(e0, c->stream) != cudaSuccess)
        return fail(c, FLASH_HY_ERR_CUDA, "autotune: %s", "event");
      const int r = enqueue_step(c, dt, step_list, step_n, nullptr, true);
      if (r) return r;
      c->cur = 1 - c->cur;
    }
    if (cudaEventRecord(e1, c->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
      return fail(c, FLASH_HY_ERR_CUDA, "autotune: %s", "event");
    if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) return fail(c, FLASH_HY_ERR_CUDA, "autotune: %s", "event");
    ms /= (float)steps;
    return 0;
  };
  auto record = [&](float ms) {
    if (nt < cap) {
      table[nt].sig_threads = c->threads;
      table[nt].dir_threads = c->dir_threads;
      table[nt].mx_threads = mx_threads_of(c->mx_sel, c->ndim, c->nx);
      table[nt].mx_runs = c->mx_runs;
      table[nt].mx_sweep = c->mx_sweep;
      table_ms[nt] = ms;
    }
    ++nt;
  };
  drop_graphs(c);
  c->plain_steps[0] = c->plain_steps[1] = 0;
  if (cudaMalloc((void **)&keep, nkeep * vbytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, FLASH_HY_ERR_CUDA, "autotune: %s", "no room for the state copy");
  }
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    rc = fail(c, FLASH_HY_ERR_CUDA, "autotune: %s", "event");
    goto done;
  }
  for (int v = 0; v < nkeep; ++v)
    if (cudaMemcpyAsync(keep + (size_t)v * c->ncells,
                        v < 5 ? c->state[cur0][v] : c->spec[cur0] + (size_t)(v - 5) * c->ncells, vbytes,
                        cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess) {
      rc = fail(c, FLASH_HY_ERR_CUDA, "autotune: %s", "state copy");
      goto done;
    }
  {
    // direction kernels first (the step's bulk), then the transverse pass
    float best_ms = 3.4e38f;
    int best_dir = mixed ? sel0 : dir0;
    const int ndir = mixed ? 3 : ncand;
    for (int q = 0; q < ndir && !rc; ++q) {
      if (mixed) c->mx_sel = q; else c->dir_threads = cand[q];
      float ms = 0.f;
      rc = trial(ms);
      if (rc) break;
      record(ms);
      if (ms < best_ms) { best_ms = ms; best_dir = mixed ? q : cand[q]; }
    }
    if (!rc) {
      if (mixed) c->mx_sel = best_dir; else c->dir_threads = best_dir;
      // runs of blocks along the sweep, where offered: the other setting
      if (mixed && c->tma_run) {
        const int other = c->mx_runs > 1 ? 1 : fhy::kMxRun;
        const int keep_runs = c->mx_runs;
        c->mx_runs = other;
        float ms = 0.f;
        rc = trial(ms);
        if (!rc) {
          record(ms);
          if (ms < best_ms) best_ms = ms;
          else c->mx_runs = keep_runs;
        }
      }
      // the other sweep order of the mixed path
      if (mixed && !rc) {
        const int keep_sweep = c->mx_sweep;
        c->mx_sweep = keep_sweep == FLASH_HY_SWEEP_ZYX ? FLASH_HY_SWEEP_XYZ : FLASH_HY_SWEEP_ZYX;
        float ms = 0.f;
        rc = trial(ms);
        if (!rc) {
          record(ms);
          if (!(ms < best_ms)) c->mx_sweep = keep_sweep;
        }
      }
    }
    if (!rc) {
      int best_sig = sig0;
      best_ms = 3.4e38f;
      for (int q = 0; q < ncand && !rc; ++q) {
        c->threads = cand[q];
        float ms = 0.f;
        rc = trial(ms);
        if (rc) break;
        record(ms);
        if (ms < best_ms) { best_ms = ms; best_sig = cand[q]; }
      }
      c->threads = best_sig;
    }
  }
done:
  if (keep) {
    if (restore() != cudaSuccess && !rc) rc = fail(c, FLASH_HY_ERR_CUDA, "autotune: %s", "state restore");
    cudaStreamSynchronize(c->stream);
    cudaFree(keep);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (rc) { c->threads = sig0; c->dir_threads = dir0; c->mx_sel = sel0; c->mx_runs = runs0; c->mx_sweep = sweep0; }
  cudaMemcpy(c->d_status, &saved_status, sizeof(unsigned), cudaMemcpyHostToDevice);
  c->dt_valid = 0;
  drop_graphs(c);
  c->plain_steps[0] = c->plain_steps[1] = 0;
  if (n_trials) *n_trials = nt;
  if (best) flash_hy_get_tuning(c, best);
  return rc;
}

// ---------------------------------------------------------------------------
// refinement criterion (gr_estimateError)
// ---------------------------------------------------------------------------
// the estimator of one variable for every node into the device array d_out
static int estimate_into(flash_hy_ctx *c, int var, double refine_filter, double *d_out) {
  CUDA_OK(c, cudaMemsetAsync(d_out, 0, (size_t)c->nblocks * sizeof(double), c->stream));
  ErrArgs a;
  fill_devparams(c, a.P);
  if (c->amr && amr_prepare(c, a.P) < 0)
    return fail(c, FLASH_HY_ERR_CUDA, "AMR guard-cell launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  a.var = var;
  a.filter = refine_filter;
  a.list = c->n_owned ? c->d_owned : nullptr;
  a.n = c->n_owned ? c->n_owned : c->nblocks;
  a.err = d_out;
  a.stream = c->stream;
  if (estimate_error(a, c->ndim, c->nx, c->ny, c->nz) < 0)
    return fail(c, FLASH_HY_ERR_CUDA, "estimator launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return 0;
}

extern "C" int flash_hy_mark_refine_tree(flash_hy_ctx *c, int nvar, const int *vars, double refine_filter,
                                         const double *refine_cutoff, const double *derefine_cutoff, int max_refine,
                                         int min_level, int cap, int *new_n, int *new_levels, int *new_coords,
                                         int *new_parent, int *src, int *how) {
  if (!c || nvar < 1 || nvar > 16 || !vars || !refine_cutoff || !derefine_cutoff || !new_n) return FLASH_HY_ERR_BAD_ARG;
  if (!c->amr) return fail(c, FLASH_HY_ERR_UNSUPPORTED, "mark_refine_tree needs an AMR hierarchy%s", "");
  if (c->nlev > 15) return fail(c, FLASH_HY_ERR_UNSUPPORTED, "mark_refine_tree: at most 15 levels%s", "");
  for (int v = 0; v < nvar; ++v)
    if (vars[v] < FLASH_HY_REFVAR_DENS || vars[v] > FLASH_HY_REFVAR_EINT) return FLASH_HY_ERR_BAD_ARG;
  CUDA_OK(c, cudaSetDevice(c->device));
  double *d_err = nullptr, *d_cut = nullptr;
  int rc = 0, trc = 0;
  if (cudaMalloc((void **)&d_err, (size_t)nvar * c->nblocks * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void **)&d_cut, 2 * (size_t)nvar * sizeof(double)) != cudaSuccess) {
    cudaFree(d_err);
    return fail(c, FLASH_HY_ERR_CUDA, "mark_refine_tree allocation%s", "");
  }
  for (int v = 0; v < nvar && !rc; ++v) rc = estimate_into(c, vars[v], refine_filter, d_err + (size_t)v * c->nblocks);
  if (!rc) {
    std::vector<double> cut(2 * (size_t)nvar);
    for (int v = 0; v < nvar; ++v) { cut[v] = refine_cutoff[v]; cut[nvar + v] = derefine_cutoff[v]; }
    if (cudaMemcpyAsync(d_cut, cut.data(), cut.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream) !=
        cudaSuccess)
      rc = fail(c, FLASH_HY_ERR_CUDA, "mark_refine_tree copies%s", "");
    else {
      TreeArgs a;
      a.err = d_err; a.nvar = nvar; a.nblocks = c->nblocks; a.ndim = c->ndim; a.L = c->nlev;
      a.rc = d_cut; a.dc = d_cut + nvar;
      a.max_refine = max_refine; a.min_level = min_level;
      a.level = c->d_level; a.coord = c->d_blk_coord; a.leaf = c->d_leaf; a.parent = c->d_parent; a.old_at = c->d_at;
      for (int l = 0; l < 17; ++l) {
        a.at_off[l] = c->at_off[l];
        for (int d = 0; d < 3; ++d) a.at_ext[l][d] = c->at_ext[l][d];
      }
      for (int d = 0; d < 3; ++d) a.periodic[d] = d < c->ndim && c->bc[2 * d] == FLASH_HY_BC_PERIODIC;
      a.stream = c->stream; a.cap = cap;
      a.new_n = new_n; a.new_levels = new_levels; a.new_coords = new_coords; a.new_parent = new_parent;
      a.src = src; a.how = how;
      if (cap > 0 && (!new_levels || !new_coords || !new_parent || !src || !how)) trc = -4;
      else trc = tree_update_dev(a);
      if (trc == -2) rc = fail(c, FLASH_HY_ERR_CUDA, "mark_refine_tree: %s", cudaGetErrorString(cudaGetLastError()));
      else if (trc == -4) rc = fail(c, FLASH_HY_ERR_BAD_ARG, "mark_refine_tree: %s", "cap too small");
      else if (trc) rc = fail(c, FLASH_HY_ERR_UNSUPPORTED, "mark_refine_tree: %s", "the tree rules did not settle");
    }
  }
  cudaStreamSynchronize(c->stream);
  cudaFree(d_err);
  cudaFree(d_cut);
  return rc;
}

extern "C" int flash_hy_estimate_error(flash_hy_ctx *c, int var, double refine_filter, double *err) {
  if (!c || !err || var < FLASH_HY_REFVAR_DENS || var > FLASH_HY_REFVAR_EINT || c->ndim < 2)
    return FLASH_HY_ERR_BAD_ARG;
  if (c->partial && c->n_owned == 0)
    return fail(c, FLASH_HY_ERR_UNSUPPORTED, "a partial grid needs its owned blocks (flash_hy_set_owned_blocks)%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  if (!c->d_err) CUDA_OK(c, cudaMalloc((void **)&c->d_err, (size_t)c->nblocks * sizeof(double)));
  CUDA_OK(c, cudaMemsetAsync(c->d_err, 0, (size_t)c->nblocks * sizeof(double), c->stream));
  ErrArgs a;
  fill_devparams(c, a.P);
  if (c->amr && amr_prepare(c, a.P) < 0)
    return fail(c, FLASH_HY_ERR_CUDA, "AMR guard-cell launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  a.var = var;
  a.filter = refine_filter;
  // a rank's share: its owned blocks only (ghost blocks lack their neighbours)
  a.list = c->n_owned ? c->d_owned : nullptr;
  a.n = c->n_owned ? c->n_owned : c->nblocks;
  a.err = c->d_err;
  a.stream = c->stream;
  if (estimate_error(a, c->ndim, c->nx, c->ny, c->nz) < 0)
    return fail(c, FLASH_HY_ERR_CUDA, "estimator launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  CUDA_OK(c, cudaMemcpyAsync(err, c->d_err, (size_t)c->nblocks * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  return 0;
}

// ---------------------------------------------------------------------------
// regrid: data of a new hierarchy from an old one (gr_updateRefinement)
// ---------------------------------------------------------------------------
extern "C" int flash_hy_regrid(flash_hy_ctx *old, flash_hy_ctx *nw, int n, const int *src, const int *how) {
  if (!old || !nw || !src || !how || old == nw) return FLASH_HY_ERR_BAD_ARG;
  if (!old->amr || !nw->amr || old->device != nw->device || old->ndim != nw->ndim || old->nx != nw->nx ||
      old->ny != nw->ny || old->nz != nw->nz || n != nw->nblocks || old->nsp != nw->nsp)
    return fail(nw, FLASH_HY_ERR_BAD_ARG, "regrid: %s", "contexts of different shapes or not AMR hierarchies");
  std::vector<int> refl, slot(n, -1), of(old->nblocks, -1);
  std::vector<int> oleaf(old->nblocks);
  CUDA_OK(old, cudaSetDevice(old->device));
  CUDA_OK(old, cudaMemcpy(oleaf.data(), old->d_leaf, old->nblocks * sizeof(int), cudaMemcpyDeviceToHost));
  for (int q = 0; q < n; ++q) {
    if (src[q] < 0 || src[q] >= old->nblocks || how[q] < 0 || how[q] > 2 || (how[q] == 1 && !oleaf[src[q]]))
      return fail(nw, FLASH_HY_ERR_BAD_ARG, "regrid: %s", "bad source block or kind");
    if (how[q] == 1) {
      if (of[src[q]] < 0) { of[src[q]] = (int)refl.size(); refl.push_back(src[q]); }
      slot[q] = of[src[q]];
    }
  }
  CUDA_OK(nw, cudaStreamSynchronize(nw->stream));
  RegridArgs a;
  fill_devparams(old, a.Po);
  if (amr_prepare(old, a.Po) < 0)
    return fail(old, FLASH_HY_ERR_CUDA, "AMR guard-cell launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  fill_devparams(nw, a.Pn);
  for (int v = 0; v < 5; ++v) a.Pn.s_out[v] = nw->state[nw->cur][v];
  if (nw->nsp) a.Pn.sp_out = nw->spec[nw->cur];
  a.nref = (int)refl.size();
  a.nnew = n;
  a.stream = old->stream;
  int *d_idx = nullptr;
  double *d_nh = nullptr;
  const size_t hn = halo_cells(old->ndim, old->nx, old->ny, old->nz);
  int rc = 0;
  if (cudaMalloc((void **)&d_idx, (3 * (size_t)n + refl.size() + 1) * sizeof(int)) != cudaSuccess ||
      (a.nref && cudaMalloc((void **)&d_nh, (size_t)a.nref * (6 + old->nsp) * hn * sizeof(double)) != cudaSuccess)) {
    cudaGetLastError();
    rc = fail(nw, FLASH_HY_ERR_CUDA, "regrid: %s", "scratch allocation");
  } else {
    int *d_src = d_idx, *d_how = d_idx + n, *d_slot = d_idx + 2 * n, *d_refl = d_idx + 3 * n;
    if (cudaMemcpyAsync(d_src, src, n * sizeof(int), cudaMemcpyHostToDevice, a.stream) != cudaSuccess ||
        cudaMemcpyAsync(d_how, how, n * sizeof(int), cudaMemcpyHostToDevice, a.stream) != cudaSuccess ||
        cudaMemcpyAsync(d_slot, slot.data(), n * sizeof(int), cudaMemcpyHostToDevice, a.stream) != cudaSuccess ||
        (a.nref && cudaMemcpyAsync(d_refl, refl.data(), refl.size() * sizeof(int), cudaMemcpyHostToDevice,
                                   a.stream) != cudaSuccess)) {
      rc = fail(nw, FLASH_HY_ERR_CUDA, "regrid: %s", "index copies");
    } else {
      a.src = d_src; a.how = d_how; a.slot = d_slot; a.refl = d_refl; a.nh = d_nh;
      if (regrid_fill(a, old->ndim, old->nx, old->ny, old->nz) < 0)
        rc = fail(nw, FLASH_HY_ERR_CUDA, "regrid launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    // the copies read pageable host vectors: finish before they go away
    if (cudaStreamSynchronize(a.stream) != cudaSuccess && !rc) rc = fail(nw, FLASH_HY_ERR_CUDA, "regrid: %s", "sync");
  }
  cudaFree(d_idx);
  cudaFree(d_nh);
  nw->dt_valid = 0;
  drop_graphs(nw);
  nw->plain_steps[0] = nw->plain_steps[1] = 0;
  return rc;
}

extern "C" int flash_hy_sync(flash_hy_ctx *c) {
  if (!c) return FLASH_HY_ERR_BAD_ARG;
  CUDA_OK(c, cudaSetDevice(c->device));
  CUDA_OK(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(c, cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  return (int)*c->h_status;
}

extern "C" void *flash_hy_stream(flash_hy_ctx *c) { return c ? (void *)c->stream : nullptr; }

extern "C" int flash_hy_export_state(flash_hy_ctx *c, double *d_out) {
  if (!c || !d_out) return FLASH_HY_ERR_BAD_ARG;
  CUDA_OK(c, cudaSetDevice(c->device));
  for (int v = 0; v < 5; ++v)
    CUDA_OK(c, cudaMemcpyAsync(d_out + (size_t)v * c->ncells, c->state[c->cur][v], c->ncells * sizeof(double),
                               cudaMemcpyDeviceToDevice, c->stream));
  return 0;
}

extern "C" int flash_hy_last_error(flash_hy_ctx *c, char *buf, int len) {
  if (!c || !buf || len <= 0) return FLASH_HY_ERR_BAD_ARG;
  snprintf(buf, len, "%s", c->err);
  return 0;
}

extern "C" int flash_hy_last_launch_count(flash_hy_ctx *c) { return c ? c->launches : -1; }

// ---------------------------------------------------------------------------
// exact Riemann solver: learned initial guess and face-state harvesting
// ---------------------------------------------------------------------------
extern "C" int flash_hy_set_guess_weights(flash_hy_ctx *c, const float *w, int n) {
  if (!c || !w || n != xrs::NPARAM) return fail(c, FLASH_HY_ERR_BAD_ARG, "set_guess_weights: %s", "bad arguments");
  CUDA_OK(c, cudaSetDevice(c->device));
  if (!c->d_wmaster) {
    CUDA_OK(c, cudaMalloc((void **)&c->d_wmaster, xrs::NPARAM * sizeof(float)));
    CUDA_OK(c, cudaMalloc(&c->d_mlp, sizeof(xrs::MlpPacked)));
  }
  CUDA_OK(c, cudaMemcpyAsync(c->d_wmaster, w, xrs::NPARAM * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  xrs::k_pack_mlp<<<1, 256, 0, c->stream>>>(c->d_wmaster, static_cast<xrs::MlpPacked *>(c->d_mlp));
  CUDA_OK(c, cudaGetLastError());
  CUDA_OK(c, cudaStreamSynchronize(c->stream));     // the host copy may go away after return
  c->mlp_set = 1;
  drop_graphs(c);                                   // captured steps hold the old kernel parameters
  return 0;
}

extern "C" int flash_hy_harvest(flash_hy_ctx *c, long long cap, int keep_log2) {
  if (!c || cap < 0 || keep_log2 < 0 || keep_log2 > 30) return fail(c, FLASH_HY_ERR_BAD_ARG, "harvest: %s", "bad arguments");
  if (c->p.riemann_solver != FLASH_HY_RS_EXACT || c->p.precision != FLASH_HY_PREC_MIXED)
    return fail(c, FLASH_HY_ERR_UNSUPPORTED, "harvest: %s", "needs the exact solver on the mixed path");
  CUDA_OK(c, cudaSetDevice(c->device));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  cudaFree(c->d_harvest); c->d_harvest = nullptr;
  c->harvest_cap = 0;
  drop_graphs(c);
  if (cap == 0) return 0;
  CUDA_OK(c, cudaMalloc((void **)&c->d_harvest, (size_t)7 * cap * sizeof(double)));
  if (!c->d_harvest_n) CUDA_OK(c, cudaMalloc((void **)&c->d_harvest_n, sizeof(unsigned long long)));
  CUDA_OK(c, cudaMemsetAsync(c->d_harvest_n, 0, sizeof(unsigned long long), c->stream));
  c->harvest_cap = cap;
  c->harvest_mask = (1u << keep_log2) - 1u;
  return 0;
}

extern "C" int flash_hy_harvest_fetch(flash_hy_ctx *c, double *d_states, long long n_max, long long *n_out) {
  if (!c || !n_out || n_max < 0) return fail(c, FLASH_HY_ERR_BAD_ARG, "harvest_fetch: %s", "bad arguments");
  *n_out = 0;
  if (c->harvest_cap == 0) return 0;
  CUDA_OK(c, cudaSetDevice(c->device));
  unsigned long long h = 0;
  CUDA_OK(c, cudaMemcpyAsync(&h, c->d_harvest_n, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  long long n = (long long)h < c->harvest_cap ? (long long)h : c->harvest_cap;
  if (!d_states) { *n_out = n; return 0; }       // query only
  if (n > n_max) n = n_max;
  for (int k = 0; k < 7 && n > 0; ++k)
    CUDA_OK(c, cudaMemcpyAsync(d_states + (size_t)k * n, c->d_harvest + (size_t)k * c->harvest_cap, n * sizeof(double),
                               cudaMemcpyDeviceToDevice, c->stream));
  CUDA_OK(c, cudaMemsetAsync(c->d_harvest_n, 0, sizeof(unsigned long long), c->stream));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  *n_out = n;
  return 0;
}

// ---------------------------------------------------------------------------
// sharded grids: owned blocks and the ghost-block exchange
// ---------------------------------------------------------------------------
// Split the owned blocks into those whose 26 neighbours (boundary rules
// applied) are all owned -- their step may run while the ghost blocks are in
// transit -- and the others, which read a received ghost block.
static int split_owned(flash_hy_ctx *c) {
  cudaFree(c->d_inner); cudaFree(c->d_edge);
  c->d_inner = c->d_edge = nullptr;
  c->n_inner = c->n_edge = 0;
  if (!c->n_owned) return 0;
  std::vector<char> ghost(c->nblocks, 0);
  for (int q = 0; q < c->n_recv_h; ++q) ghost[c->h_recv[q]] = 1;
  std::vector<int> coords(3 * (size_t)c->nblocks), inner, edge;
  CUDA_OK(c, cudaMemcpy(coords.data(), c->d_blk_coord, coords.size() * sizeof(int), cudaMemcpyDeviceToHost));
  const int nbl[3] = {c->nbx, c->nby, c->nbz};
  for (int q = 0; q < c->n_owned; ++q) {
    const int b = c->h_owned[q];
    const int *cc = &coords[3 * (size_t)b];
    bool touches = false;
    for (int o = 0; o < 27 && !touches; ++o) {
      int off[3] = {o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1}, p[3];
      bool ok = true;
      for (int d = 0; d < 3; ++d) {
        if (d >= c->ndim) { if (off[d]) ok = false; p[d] = 0; continue; }
        p[d] = cc[d] + off[d];
        if (p[d] < 0 || p[d] >= nbl[d]) {
          if (c->bc[2 * d] != FLASH_HY_BC_PERIODIC) { p[d] = cc[d]; continue; }
          p[d] = (p[d] + nbl[d]) % nbl[d];
        }
      }
      if (!ok) continue;
      const int nb = c->h_blk_at ? c->h_blk_at[((size_t)p[2] * c->nby + p[1]) * c->nbx + p[0]] : -1;
      if (nb >= 0 && ghost[nb]) touches = true;
    }
    (touches ? edge : inner).push_back(b);
  }
  if (!inner.empty()) {
    CUDA_OK(c, cudaMalloc((void **)&c->d_inner, inner.size() * sizeof(int)));
    CUDA_OK(c, cudaMemcpy(c->d_inner, inner.data(), inner.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  if (!edge.empty()) {
    CUDA_OK(c, cudaMalloc((void **)&c->d_edge, edge.size() * sizeof(int)));
    CUDA_OK(c, cudaMemcpy(c->d_edge, edge.data(), edge.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  c->n_inner = (int)inner.size();
  c->n_edge = (int)edge.size();
  return 0;
}

extern "C" int flash_hy_set_owned_blocks(flash_hy_ctx *c, int n, const int *list) {
  if (!c || n <= 0 || !list || c->amr) return fail(c, FLASH_HY_ERR_BAD_ARG, "set_owned_blocks: %s", "bad arguments");
  std::vector<int> mask(c->nblocks, 0);
  for (int q = 0; q < n; ++q) {
    if (list[q] < 0 || list[q] >= c->nblocks || mask[list[q]])
      return fail(c, FLASH_HY_ERR_BAD_ARG, "set_owned_blocks: %s", "block out of range or repeated");
    mask[list[q]] = 1;
  }
  if (c->partial) {
    // every block an owned block reads guard cells from must be present
    std::vector<int> coords(3 * (size_t)c->nblocks);
    CUDA_OK(c, cudaSetDevice(c->device));
    CUDA_OK(c, cudaMemcpy(coords.data(), c->d_blk_coord, coords.size() * sizeof(int), cudaMemcpyDeviceToHost));
    const int nbl[3] = {c->nbx, c->nby, c->nbz};
    for (int q = 0; q < n; ++q) {
      const int *cc = &coords[3 * list[q]];
      for (int o = 0; o < 27; ++o) {
        int off[3] = {o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1}, p[3];
        bool ok = true;
        for (int d = 0; d < 3; ++d) {
          if (d >= c->ndim) { if (off[d]) ok = false; p[d] = 0; continue; }
          p[d] = cc[d] + off[d];
          if (p[d] < 0 || p[d] >= nbl[d]) {
            if (c->bc[2 * d] != FLASH_HY_BC_PERIODIC) { p[d] = cc[d]; continue; }   // boundary: own cells
            p[d] = (p[d] + nbl[d]) % nbl[d];
          }
        }
        if (!ok) continue;
        if (c->h_blk_at[((size_t)p[2] * c->nby + p[1]) * c->nbx + p[0]] < 0)
          return fail(c, FLASH_HY_ERR_BAD_ARG, "set_owned_blocks: %s", "a neighbour of an owned block is absent");
      }
    }
  }
  CUDA_OK(c, cudaSetDevice(c->device));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  cudaFree(c->d_owned); cudaFree(c->d_owned_mask);
  c->d_owned = nullptr; c->d_owned_mask = nullptr; c->n_owned = 0;
  CUDA_OK(c, cudaMalloc((void **)&c->d_owned, n * sizeof(int)));
  CUDA_OK(c, cudaMalloc((void **)&c->d_owned_mask, c->nblocks * sizeof(int)));
  CUDA_OK(c, cudaMemcpy(c->d_owned, list, n * sizeof(int), cudaMemcpyHostToDevice));
  CUDA_OK(c, cudaMemcpy(c->d_owned_mask, mask.data(), c->nblocks * sizeof(int), cudaMemcpyHostToDevice));
  c->n_owned = n;
  free(c->h_owned);
  c->h_owned = (int *)malloc((size_t)n * sizeof(int));
  if (!c->h_owned) return fail(c, FLASH_HY_ERR_CUDA, "host allocation%s", "");
  memcpy(c->h_owned, list, (size_t)n * sizeof(int));
  c->dt_valid = 0;
  c->phase_pending = 0;
  drop_graphs(c);
  return split_owned(c);
}

extern "C" int flash_hy_set_exchange(flash_hy_ctx *c, int nsend, const int *send, int nrecv, const int *recv) {
  if (!c || nsend < 0 || nrecv < 0 || (nsend && !send) || (nrecv && !recv))
    return fail(c, FLASH_HY_ERR_BAD_ARG, "set_exchange: %s", "bad arguments");
  for (int q = 0; q < nsend; ++q)
    if (send[q] < 0 || send[q] >= c->nblocks) return fail(c, FLASH_HY_ERR_BAD_ARG, "set_exchange: %s", "send block");
  for (int q = 0; q < nrecv; ++q)
    if (recv[q] < 0 || recv[q] >= c->nblocks) return fail(c, FLASH_HY_ERR_BAD_ARG, "set_exchange: %s", "recv block");
  CUDA_OK(c, cudaSetDevice(c->device));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  cudaFree(c->d_send); cudaFree(c->d_recv);
  c->d_send = c->d_recv = nullptr;
  c->n_send = c->n_recv = 0;
  if (nsend) {
    CUDA_OK(c, cudaMalloc((void **)&c->d_send, nsend * sizeof(int)));
    CUDA_OK(c, cudaMemcpy(c->d_send, send, nsend * sizeof(int), cudaMemcpyHostToDevice));
  }
  if (nrecv) {
    CUDA_OK(c, cudaMalloc((void **)&c->d_recv, nrecv * sizeof(int)));
    CUDA_OK(c, cudaMemcpy(c->d_recv, recv, nrecv * sizeof(int), cudaMemcpyHostToDevice));
  }
  c->n_send = nsend;
  c->n_recv = nrecv;
  free(c->h_recv);
  c->h_recv = (int *)malloc((size_t)(nrecv > 0 ? nrecv : 1) * sizeof(int));
  if (!c->h_recv) return fail(c, FLASH_HY_ERR_CUDA, "host allocation%s", "");
  if (nrecv) memcpy(c->h_recv, recv, (size_t)nrecv * sizeof(int));
  c->n_recv_h = nrecv;
  c->phase_pending = 0;
  return split_owned(c);
}

// buf[i][v][cell] <-> state[v][list[i] * ncb + cell], one CTA per listed block
// one record per listed block: the 5 state variables, then the species and
// mass scalars, ncb values each
__global__ void k_blocks_to_buf(const double *s0, const double *s1, const double *s2, const double *s3,
                                const double *s4, const double *sp, int nsp, size_t ncells, const int *list, int ncb,
                                double *buf) {
  const double *st[5] = {s0, s1, s2, s3, s4};
  const size_t b = (size_t)list[blockIdx.x];
  const int nv = 5 + nsp;
  double *dst = buf + (size_t)blockIdx.x * nv * ncb;
  for (int t = threadIdx.x; t < nv * ncb; t += blockDim.x) {
    const int v = t / ncb, c = t % ncb;
    dst[t] = v < 5 ? st[v][b * ncb + c] : sp[(size_t)(v - 5) * ncells + b * ncb + c];
  }
}
__global__ void k_buf_to_blocks(double *s0, double *s1, double *s2, double *s3, double *s4, double *sp, int nsp,
                                size_t ncells, const int *list, int ncb, const double *buf) {
  double *st[5] = {s0, s1, s2, s3, s4};
  const size_t b = (size_t)list[blockIdx.x];
  const int nv = 5 + nsp;
  const double *src = buf + (size_t)blockIdx.x * nv * ncb;
  for (int t = threadIdx.x; t < nv * ncb; t += blockDim.x) {
    const int v = t / ncb, c = t % ncb;
    if (v < 5) st[v][b * ncb + c] = src[t];
    else sp[(size_t)(v - 5) * ncells + b * ncb + c] = src[t];
  }
}

extern "C" int flash_hy_pack(flash_hy_ctx *c, double *d_buf) {
  if (!c || (c->n_send && !d_buf)) return FLASH_HY_ERR_BAD_ARG;
  if (!c->n_send) return 0;
  CUDA_OK(c, cudaSetDevice(c->device));
  double *const *st = c->state[c->cur];
  k_blocks_to_buf<<<c->n_send, 256, 0, c->stream>>>(st[0], st[1], st[2], st[3], st[4], c->spec[c->cur], c->nsp,
                                                    c->ncells, c->d_send, (int)c->ncb, d_buf);
  CUDA_OK(c, cudaGetLastError());
  return 0;
}

extern "C" int flash_hy_unpack(flash_hy_ctx *c, const double *d_buf) {
  if (!c || (c->n_recv && !d_buf)) return FLASH_HY_ERR_BAD_ARG;
  if (!c->n_recv) return 0;
  CUDA_OK(c, cudaSetDevice(c->device));
  double *const *st = c->state[c->cur];
  k_buf_to_blocks<<<c->n_recv, 256, 0, c->stream>>>(st[0], st[1], st[2], st[3], st[4], c->spec[c->cur], c->nsp,
                                                    c->ncells, c->d_recv, (int)c->ncb, d_buf);
  CUDA_OK(c, cudaGetLastError());
  c->dt_valid = 0;
  return 0;
}
