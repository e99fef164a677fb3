// flash_hy.cu -- the C ABI of include/flash_hy.h: context, device block
// store, UNK upload/download, the Hydro step and the CFL time step.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <string>
#include <vector>
#include "../../include/flash_hy.h"
#include "hy_launch.h"

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
  int list_cap;
  CflPart *d_part;
  DtInfo *d_dt, *h_dt;
  unsigned *d_status, *h_status;
  unsigned char *d_stage;
  size_t stage_bytes;
  int dt_valid;
  int launches;
  int threads;
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
  char err[512];
};

static void drop_graphs(flash_hy_ctx *c) {
  for (int q = 0; q < 2; ++q) {
    if (c->gexec[q]) cudaGraphExecDestroy(c->gexec[q]);
    c->gexec[q] = nullptr;
  }
}

__global__ void k_set_dt(double *d, double dt) { *d = dt; }

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
  P.blk_coord = c->d_blk_coord;
  P.status = c->d_status;
  for (int v = 0; v < 5; ++v) {
    P.s_in[v] = c->state[c->cur][v];
    P.s_out[v] = c->state[1 - c->cur][v];
  }
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
  int nz = g->ndim > 2 ? g->nzb : 1, ny = g->ndim > 1 ? g->nyb : 1;
  if (!shape_supported(g->ndim, g->nxb, ny, nz)) return FLASH_HY_ERR_UNSUPPORTED;
  if (g->max_level > 1) return FLASH_HY_ERR_UNSUPPORTED;
  if (g->nblocks <= 0 || !g->block_coords || g->nguard < 0) return FLASH_HY_ERR_BAD_ARG;
  int nbx = g->nblk_l1[0], nby = g->ndim > 1 ? g->nblk_l1[1] : 1, nbz = g->ndim > 2 ? g->nblk_l1[2] : 1;
  if (nbx <= 0 || nby <= 0 || nbz <= 0 || (long)nbx * nby * nbz != g->nblocks) return FLASH_HY_ERR_BAD_ARG;
  std::vector<int> at((size_t)nbx * nby * nbz, -1), coords(3 * (size_t)g->nblocks);
  for (int b = 0; b < g->nblocks; ++b) {
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
  for (int f = 0; f < 6; ++f) c->bc[f] = f < 2 * g->ndim ? g->bc[f] : FLASH_HY_BC_OUTFLOW;
  int nb[3] = {g->nxb, ny, nz}, nbl[3] = {nbx, nby, nbz};
  for (int d = 0; d < 3; ++d)
    c->del[d] = d < g->ndim ? (g->domain_hi[d] - g->domain_lo[d]) / (double)(nbl[d] * nb[d]) : 1.0;
  c->ncb = (size_t)g->nxb * ny * nz;
  c->ncells = c->ncb * g->nblocks;
  c->device = device;
  c->threads = g->ndim == 3 ? 320 : (g->nxb == 8 ? 96 : 288);  // line cells split evenly
  c->host_ng = g->nguard;
  *out = c;
  int rc = 0;
#define ALLOC(ptr, bytes)                                                           \
  do {                                                                              \
    cudaError_t e_ = cudaMalloc((void **)&(ptr), (bytes));                          \
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
  {
    int rb = params->precision == FLASH_HY_PREC_MIXED ? 4 : 8;
    ALLOC(c->sig, sig_bytes_per_block(g->ndim, g->nxb, ny, nz, rb) * g->nblocks);
  }
  ALLOC(c->d_blk_at, at.size() * sizeof(int));
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
  if (cudaMemcpy(c->d_blk_at, at.data(), at.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_blk_coord, coords.data(), coords.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(c->d_status, 0, sizeof(unsigned)) != cudaSuccess) {
    rc = fail(c, FLASH_HY_ERR_CUDA, "init copies%s", ""); goto bad;
  }
  return 0;
bad:
  return rc;
#undef ALLOC
}

extern "C" int flash_hy_destroy(flash_hy_ctx *c) {
  if (!c) return FLASH_HY_ERR_BAD_ARG;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int s = 0; s < 2; ++s)
    for (int v = 0; v < 5; ++v) cudaFree(c->state[s][v]);
  cudaFree(c->acc); cudaFree(c->aux); cudaFree(c->sig);
  cudaFree(c->d_blk_at); cudaFree(c->d_blk_coord); cudaFree(c->d_list);
  cudaFree(c->d_part); cudaFree(c->d_dt); cudaFree(c->d_status); cudaFree(c->d_stage);
  cudaFree(c->d_wmaster); cudaFree(c->d_mlp); cudaFree(c->d_harvest); cudaFree(c->d_harvest_n);
  drop_graphs(c);
  cudaFree(c->d_stepdt);
  if (c->h_dt) cudaFreeHost(c->h_dt);
  if (c->h_status) cudaFreeHost(c->h_status);
  if (c->stream) cudaStreamDestroy(c->stream);
  free(c);
  return 0;
}

// ---------------------------------------------------------------------------
// UNK <-> device block store
// ---------------------------------------------------------------------------
struct HostLayout {
  int layout, nunk, ng[3], nt[3];
  int v_dens, v_eint, v_ener, v_gamc, v_game, v_pres, v_temp, v_velx, v_vely, v_velz;  // 0-based, -1 absent
};

__device__ __forceinline__ size_t unk_index(const HostLayout &L, int b, int i, int j, int k, int v) {
  if (L.layout == FLASH_HY_LAYOUT_VAR_FASTEST)
    return ((((size_t)b * L.nt[2] + k) * L.nt[1] + j) * L.nt[0] + i) * L.nunk + v;
  return ((((size_t)b * L.nunk + v) * L.nt[2] + k) * L.nt[1] + j) * L.nt[0] + i;
}

__global__ void k_unpack(const double *__restrict__ stage, HostLayout L, DevParams P, int nx, int ny, int nz,
                         size_t ncells) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= ncells) return;
  size_t ncb = (size_t)nx * ny * nz;
  int b = (int)(t / ncb), loc = (int)(t % ncb);
  int i = loc % nx, j = (loc / nx) % ny, k = loc / (nx * ny);
  int hi = i + L.ng[0], hj = j + L.ng[1], hk = k + L.ng[2];
  auto get = [&](int v) { return v < 0 ? 0.0 : stage[unk_index(L, b, hi, hj, hk, v)]; };
  double rho = get(L.v_dens), vx = get(L.v_velx), vy = get(L.v_vely), vz = get(L.v_velz);
  // Eos_getData.F90:80-96 then MODE_DENS_EI keeps eint (Grid_initDomain's EOS)
  double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
  double eint = L.v_eint >= 0 ? get(L.v_eint) : get(L.v_ener) - ekin;
  if (L.v_ener >= 0) {
    double ener = get(L.v_ener);
    if (ener - ekin > rmax(P.smalle, P.eswitch * ekin)) eint = ener - ekin;
  }
  P.s_out[0][t] = rho; P.s_out[1][t] = vx; P.s_out[2][t] = vy; P.s_out[3][t] = vz; P.s_out[4][t] = eint;
}

__global__ void k_pack(double *__restrict__ stage, HostLayout L, DevParams P, int nx, int ny, int nz, size_t ncells) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= ncells) return;
  size_t ncb = (size_t)nx * ny * nz;
  int b = (int)(t / ncb), loc = (int)(t % ncb);
  int i = loc % nx, j = (loc / nx) % ny, k = loc / (nx * ny);
  int hi = i + L.ng[0], hj = j + L.ng[1], hk = k + L.ng[2];
  double rho = P.s_in[0][t], vx = P.s_in[1][t], vy = P.s_in[2][t], vz = P.s_in[3][t], e = P.s_in[4][t];
  // Eos_putData.F90:95-106 of the gamma law
  double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
  double pres = rho * e * P.gam1inv;
  double temp = e * P.ggprodinv * P.abar;
  auto put = [&](int v, double x) { if (v >= 0) stage[unk_index(L, b, hi, hj, hk, v)] = x; };
  put(L.v_dens, rho); put(L.v_velx, vx); put(L.v_vely, vy); put(L.v_velz, vz);
  put(L.v_pres, pres); put(L.v_temp, temp); put(L.v_gamc, P.gamma); put(L.v_eint, e);
  put(L.v_ener, e + ekin); put(L.v_game, pres / (e * rho) + 1);
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
  return 0;
}

static int ensure_stage(flash_hy_ctx *c, size_t bytes) {
  if (c->stage_bytes >= bytes) return 0;
  if (c->d_stage) { cudaStreamSynchronize(c->stream); cudaFree(c->d_stage); c->d_stage = nullptr; c->stage_bytes = 0; }
  CUDA_OK(c, cudaMalloc((void **)&c->d_stage, bytes));
  c->stage_bytes = bytes;
  return 0;
}

extern "C" int flash_hy_upload(flash_hy_ctx *c, const double *unk, int layout, int nunk, const flash_hy_varmap *vm) {
  if (!c || !unk) return FLASH_HY_ERR_BAD_ARG;
  HostLayout L;
  int rc = make_layout(c, layout, nunk, vm, c->host_ng, L);
  if (rc) return fail(c, rc, "bad UNK layout or variable map%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  size_t bytes = (size_t)c->nblocks * L.nt[0] * L.nt[1] * L.nt[2] * nunk * sizeof(double);
  if ((rc = ensure_stage(c, bytes))) return rc;
  CUDA_OK(c, cudaMemcpyAsync(c->d_stage, unk, bytes, cudaMemcpyHostToDevice, c->stream));
  DevParams P;
  fill_devparams(c, P);
  for (int v = 0; v < 5; ++v) P.s_out[v] = c->state[c->cur][v];
  k_unpack<<<(unsigned)((c->ncells + 255) / 256), 256, 0, c->stream>>>((const double *)c->d_stage, L, P, c->nx, c->ny,
                                                                       c->nz, c->ncells);
  CUDA_OK(c, cudaGetLastError());
  c->dt_valid = 0;
  return 0;
}

extern "C" int flash_hy_download(flash_hy_ctx *c, double *unk, int layout, int nunk, const flash_hy_varmap *vm) {
  if (!c || !unk) return FLASH_HY_ERR_BAD_ARG;
  HostLayout L;
  int rc = make_layout(c, layout, nunk, vm, c->host_ng, L);
  if (rc) return fail(c, rc, "bad UNK layout or variable map%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  size_t bytes = (size_t)c->nblocks * L.nt[0] * L.nt[1] * L.nt[2] * nunk * sizeof(double);
  if ((rc = ensure_stage(c, bytes))) return rc;
  bool full = (L.ng[0] == 0) && (L.v_dens >= 0);
  // Variables we do not own (and guard cells) keep the caller's values.
  int owned = 0;
  for (int q = 0; q < 10; ++q) owned += (&L.v_dens)[q] >= 0;
  if (!(full && owned == nunk)) CUDA_OK(c, cudaMemcpyAsync(c->d_stage, unk, bytes, cudaMemcpyHostToDevice, c->stream));
  DevParams P;
  fill_devparams(c, P);
  k_pack<<<(unsigned)((c->ncells + 255) / 256), 256, 0, c->stream>>>((double *)c->d_stage, L, P, c->nx, c->ny, c->nz,
                                                                     c->ncells);
  CUDA_OK(c, cudaGetLastError());
  CUDA_OK(c, cudaMemcpyAsync(unk, c->d_stage, bytes, cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  return 0;
}

// ---------------------------------------------------------------------------
// step
// ---------------------------------------------------------------------------
static int enqueue_step(flash_hy_ctx *c, double dt, const int *d_list, int nlaunch, const double *dt_dev = nullptr,
                        bool set_attr = true) {
  StepArgs a;
  fill_devparams(c, a.P);
  a.P.dt = dt;
  a.P.dt_dev = dt_dev;
  a.set_attr = set_attr;
  a.P.blk_list = d_list;
  a.sig = c->sig;
  a.acc = c->acc;
  a.aux = c->aux;
  a.ncells = c->ncells;
  a.part = c->d_part;
  a.nlaunch = nlaunch;
  a.threads = c->threads;
  a.stream = c->stream;
  int n;
  switch (c->p.precision) {
    case FLASH_HY_PREC_FP64_FMA: n = step_fp64_fma(a, c->ndim, c->nx, c->ny, c->nz); break;
    case FLASH_HY_PREC_MIXED: n = step_mixed(a, c->ndim, c->nx, c->ny, c->nz); break;
    default: n = step_fp64_exact(a, c->ndim, c->nx, c->ny, c->nz); break;
  }
  if (n == -1) return fail(c, FLASH_HY_ERR_UNSUPPORTED, "unsupported block shape%s", "");
  if (n < 0) return fail(c, FLASH_HY_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  c->launches = n;
  return 0;
}

extern "C" int flash_hy_step(flash_hy_ctx *c, double simTime, double dt, double dtOld, int sweepOrder) {
  (void)simTime; (void)dtOld; (void)sweepOrder;
  if (!c) return FLASH_HY_ERR_BAD_ARG;
  if (!(dt > 0.0)) return fail(c, FLASH_HY_ERR_NONPOS_DT, "dt must be positive%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  if (!c->use_graph) {
    int rc = enqueue_step(c, dt, nullptr, c->nblocks);
    if (rc) return rc;
  } else {
    const int q = c->cur;
    k_set_dt<<<1, 1, 0, c->stream>>>(c->d_stepdt, dt);
    CUDA_OK(c, cudaGetLastError());
    if (!c->gexec[q] && c->plain_steps[q] == 0) {
      // first step of this parity runs uncaptured (it also sets the kernels'
      // shared-memory attributes, which are not stream work)
      int rc = enqueue_step(c, dt, nullptr, c->nblocks, c->d_stepdt, true);
      if (rc) return rc;
      c->plain_steps[q]++;
      c->launches = c->launches + 1;
    } else {
      if (!c->gexec[q]) {
        cudaGraph_t g = nullptr;
        CUDA_OK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(c, dt, nullptr, c->nblocks, c->d_stepdt, false);
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

extern "C" int flash_hy_step_blocks(flash_hy_ctx *c, int blockCount, const int *blockList, double timeEndAdv,
                                    double dt, double dtOld, int sweepOrder) {
  (void)timeEndAdv; (void)dtOld; (void)sweepOrder;
  if (!c || blockCount < 0 || (blockCount > 0 && !blockList)) return FLASH_HY_ERR_BAD_ARG;
  if (!(dt > 0.0)) return fail(c, FLASH_HY_ERR_NONPOS_DT, "dt must be positive%s", "");
  for (int q = 0; q < blockCount; ++q)
    if (blockList[q] < 0 || blockList[q] >= c->nblocks) return fail(c, FLASH_HY_ERR_BAD_ARG, "block id out of range%s", "");
  CUDA_OK(c, cudaSetDevice(c->device));
  if (blockCount > c->list_cap) {
    cudaStreamSynchronize(c->stream);
    cudaFree(c->d_list);
    c->d_list = nullptr;
    CUDA_OK(c, cudaMalloc((void **)&c->d_list, blockCount * sizeof(int)));
    c->list_cap = blockCount;
  }
  // blocks outside the list keep their state
  for (int v = 0; v < 5; ++v)
    CUDA_OK(c, cudaMemcpyAsync(c->state[1 - c->cur][v], c->state[c->cur][v], c->ncells * sizeof(double),
                               cudaMemcpyDeviceToDevice, c->stream));
  if (blockCount > 0) {
    CUDA_OK(c, cudaMemcpyAsync(c->d_list, blockList, blockCount * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUDA_OK(c, cudaStreamSynchronize(c->stream));   // blockList is caller memory
    int rc = enqueue_step(c, dt, c->d_list, blockCount);
    if (rc) return rc;
  }
  c->cur = 1 - c->cur;
  c->dt_valid = 0;
  return 0;
}

__global__ void k_dt_reduce(const CflPart *part, int nblocks, const int *blk_level, int ndim, DtInfo *out) {
  __shared__ double sdt[1024];
  __shared__ int sb[1024];
  double best = DBL_MAX;
  int bb = 0x7fffffff;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
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
      r.level = 1;
      r.blk = b;
    } else {
      r.i = r.j = r.k = 0; r.level = 0; r.blk = -1;
    }
    (void)blk_level;
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
    a.stream = c->stream;
    a.set_attr = true;
    if (cfl_state(a, c->ndim, c->nx, c->ny, c->nz) < 0) return fail(c, FLASH_HY_ERR_CUDA, "cfl launch%s", "");
    c->dt_valid = 1;
  }
  k_dt_reduce<<<1, 1024, 0, c->stream>>>(c->d_part, c->nblocks, nullptr, c->ndim, c->d_dt);
  CUDA_OK(c, cudaGetLastError());
  CUDA_OK(c, cudaMemcpyAsync(c->h_dt, c->d_dt, sizeof(DtInfo), cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(c, cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
  CUDA_OK(c, cudaStreamSynchronize(c->stream));
  *dt_out = c->h_dt->dt;
  if (minloc_out) {
    minloc_out[0] = c->h_dt->i; minloc_out[1] = c->h_dt->j; minloc_out[2] = c->h_dt->k;
    minloc_out[3] = c->h_dt->level; minloc_out[4] = c->h_dt->blk;
  }
  int st = (int)*c->h_status;
  if (!(c->h_dt->dt > 0.0)) st |= FLASH_HY_ERR_NONPOS_DT;
  return st;
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
