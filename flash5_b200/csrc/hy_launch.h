// hy_launch.h -- interface between the C-ABI (flash_hy.cu) and the kernel
// variants (hy_variant.cu, compiled once per arithmetic variant).
#pragma once
#include <cuda.h>
#include "hy_kernels.cuh"
#include "../../include/flash_hy.h"

namespace fhy {

// Blocks per run of the mixed direction kernels on full uniform 3D grids:
// a CTA stages kMxRun blocks that follow one another along the sweep and
// 1/kMxRun of their cross-section.
constexpr int kMxRun = 4;

// Tensor maps of the step's input state for the mixed direction kernels'
// TMA staging (k_dir_mx, uniform 3D grids): per state variable the block
// interior (box 8 x 8 x 8) and the neighbour slab along the sweep direction
// (box 4 x 8 x 8, 8 x 4 x 8 or 8 x 8 x 4) over the natural block layout;
// for runs, the same boxes cut to 1/kMxRun of the slower transverse axis.
struct TmaLine {
  CUtensorMap intr[5];        // dens, velx, vely, velz, eint
  CUtensorMap slab[5];
  int on;                     // 0: the stencil is staged by load_prim
  const int *runs;            // runs: [nblocks / kMxRun][kMxRun + 2] blocks along the sweep, neighbours below / above
  void *cflq;                 // runs, last direction: [nblocks][kMxRun] CflCand of the quarters
};

struct StepArgs {
  DevParams P;
  void *sig;          // transverse-flux scratch, sizeof(R) * 6 * ndim * box * nlaunch
  double *acc;        // [5][ncells] conservative-update accumulator
  double *aux;        // [ndim-1][3][ncells] eint-update terms of the earlier directions
  size_t ncells;
  CflPart *part;      // per-block CFL results
  int nlaunch;        // CTAs (blocks updated)
  int threads;        // threads per CTA of the transverse-flux and CFL passes
  int dir_threads;    // threads per CTA of the FP64 direction kernels
  int mx_sel;         // candidate (0, 1, 2) of the mixed direction kernels' threads per CTA
  int sweep = 0;      // mixed path: 0 = directions x, y, z; 1 = z, y, x
  cudaStream_t stream;
  bool set_attr;      // raise the kernels' dynamic shared-memory limit (not while capturing a graph)
  // AMR (nlev > 0): k_sig over all leaves, then per direction one launch per
  // level, finest first (the flux register needs the fine fluxes first)
  bool no_sig;        // update from stored fluxes: the transverse-flux pass is not needed
  int nlev;
  const int *leaves;  // all leaves (device)
  int nleaves;
  const int *lev_list[17];  // leaves of each level (device), 1-based levels
  int lev_count[17];
  const TmaLine *tma; // [3] (directions x, y, z) for the input state, or NULL
  const TmaLine *tma_run = nullptr;  // [3] maps of the run kernels (full uniform 3D grids), or NULL
  int nblocks = 0;    // blocks of the grid (run kernels: the CFL merge)
};

// the species / mass-scalar pass after the hydro direction kernels
struct SpecArgs {
  DevParams P;        // the step's parameters (species buffers, mass fluxes, flags)
  bool mixed;         // the mixed path: FP32 face values (spec_step_mx)
  size_t ncells;
  int nlaunch;
  cudaStream_t stream;
  // AMR (nlev > 0): one launch per level, finest first (the species flux
  // register)
  int nlev;
  const int *lev_list[17];
  int lev_count[17];
};
// launches k_spec_step (once, or once per level); returns the launch count or -2
int spec_step(const SpecArgs &a, int ndim, int nx, int ny, int nz);
int spec_step_mx(const SpecArgs &a, int ndim, int nx, int ny, int nz);

// the refinement criterion of every listed block (all blocks without a list)
struct ErrArgs {
  DevParams P;
  int var;            // FLASH_HY_REFVAR_*
  double filter;      // refine_filter
  const int *list;
  int n;
  double *err;        // device, indexed by block
  cudaStream_t stream;
};
int estimate_error(const ErrArgs &a, int ndim, int nx, int ny, int nz);

// data movement of a regrid from an old AMR context to a new one
struct RegridArgs {
  DevParams Po;            // old context after its guard fill (s_in = its state)
  DevParams Pn;            // new context (s_out = the state to fill, pe, leaf)
  const int *refl;         // old leaves whose children are created
  int nref;
  double *nh;              // [nref][6][halo] their guard-inclusive copies
  const int *src, *how, *slot;  // per new node; slot = index into refl (how 1)
  int nnew;
  cudaStream_t stream;
};
int regrid_fill(const RegridArgs &a, int ndim, int nx, int ny, int nz);
size_t halo_cells(int ndim, int nx, int ny, int nz);

// marking and the tree of a regrid on the device (tree_dev.cu): errors of
// nvar refinement variables [nvar][nblocks] (device), the old tree's tables
// (device), the new node arrays (host, capacity cap).  Returns 0, -2 (CUDA),
// -3 (a rule did not settle), -4 (cap too small; *new_n says what is needed)
// or -5 (the tree would need a node two levels below the old tree).
struct TreeArgs {
  const double *err;
  int nvar, nblocks, ndim, L;
  const double *rc, *dc;       // per-variable cutoffs (device)
  int max_refine, min_level;
  const int *level, *coord, *leaf, *parent, *old_at;
  int at_off[17];
  int at_ext[17][3];
  int periodic[3];
  cudaStream_t stream;
  int cap;
  int *new_n, *new_levels, *new_coords, *new_parent, *src, *how;
};
int tree_update_dev(const TreeArgs &a);

// Enqueue one hydro step; returns the number of kernel launches, or -1 for an
// unsupported block shape, or -2 for a launch error.
int step_fp64_exact(const StepArgs &a, int ndim, int nx, int ny, int nz);
int step_fp64_fma(const StepArgs &a, int ndim, int nx, int ny, int nz);
int step_mixed(const StepArgs &a, int ndim, int nx, int ny, int nz);
int step_mixed_nt0(const StepArgs &a, int ndim, int nx, int ny, int nz);
int step_mixed_nt1(const StepArgs &a, int ndim, int nx, int ny, int nz);
int step_mixed_nt2(const StepArgs &a, int ndim, int nx, int ny, int nz);
bool sig_mixed(const StepArgs &a, int ndim, int nx, int ny, int nz);
// threads per CTA of mixed candidate `sel` for a block shape
int mx_threads_of(int sel, int ndim, int nx);
// CFL reduction of the stored state (one launch).
int cfl_state(const StepArgs &a, int ndim, int nx, int ny, int nz);
size_t sig_bytes_per_block(int ndim, int nx, int ny, int nz, int real_bytes);

}  // namespace fhy
