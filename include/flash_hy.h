/*
 * flash_hy.h -- C ABI of the B200 unsplit-hydro block update.
 *
 * Drop-in boundary for FLASH5's directionally unsplit hydro step over the leaf
 * blocks of a block-structured grid.  Every entry point takes plain pointers
 * and sizes, returns an int status (0 = OK, otherwise FLASH_HY_ERR_* bit
 * flags) and never aborts the process.  The library owns device memory; the
 * caller owns host memory.  One context per GPU; calls on one context are not
 * thread-safe.
 *
 * Reference interfaces replaced (paths inside mbdevpl/FLASH5):
 *   Hydro(simTime, dt, dtOld, sweepOrder)
 *       source/physics/Hydro/Hydro_interface.F90:52-57,
 *       source/physics/Hydro/HydroMain/unsplit/Hydro.F90:6-343
 *   Hydro_init            source/physics/Hydro/HydroMain/unsplit/Hydro_init.F90:60-688
 *   Hydro_computeDt       source/physics/Hydro/Hydro_interface.F90:12-32,
 *                         source/physics/Hydro/HydroMain/unsplit/Hydro_computeDt.F90:63-328
 *   hy_computeFluxes / hy_updateSolution (per-block API)
 *                         source/physics/Hydro/localAPI/hy_interface.F90:969,982
 *   Grid UNK ownership    source/Grid/GridMain/UG/gr_createDomain.F90:127-147,
 *                         source/Grid/GridMain/AMR/paramesh/Grid_tile.F90:157-182
 */
#ifndef FLASH_HY_H
#define FLASH_HY_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status bits (0 = success) --------------------------------------- */
#define FLASH_HY_OK                 0
#define FLASH_HY_ERR_NEG_SOUNDSPEED (1 << 0) /* a^2 <= 0 (hy_eigenParameters.F90:83-86, hy_HLLC.F90:125-127) */
#define FLASH_HY_ERR_NONPOS_DT      (1 << 1) /* Hydro_computeDt.F90:321-323 */
#define FLASH_HY_ERR_NEWTON_NOCONV  (1 << 2) /* exact Riemann solver gave up */
#define FLASH_HY_ERR_NAN            (1 << 3) /* non-finite value in the updated state */
#define FLASH_HY_ERR_TIMEOUT        (1 << 4) /* a bounded device wait expired */
#define FLASH_HY_ERR_BAD_ARG        (1 << 5)
#define FLASH_HY_ERR_CUDA           (1 << 6)
#define FLASH_HY_ERR_UNSUPPORTED    (1 << 7)

/* ---- enumerations (numeric values follow FLASH's own headers) ---------- */
/* Riemann solvers: UHD.h:366-372 numbering; EXACT has no FLASH counterpart */
#define FLASH_HY_RS_HLLC   4
#define FLASH_HY_RS_EXACT  100
/* slope limiters: UHD.h:15-19 */
#define FLASH_HY_LIM_MINMOD  1
#define FLASH_HY_LIM_MC      2
#define FLASH_HY_LIM_HYBRID  3
#define FLASH_HY_LIM_VANLEER 4
#define FLASH_HY_LIM_LIMITED 5
/* boundary conditions: source/Simulation/constants.h:62-64 */
#define FLASH_HY_BC_REFLECTING (-31)
#define FLASH_HY_BC_OUTFLOW    (-32)
#define FLASH_HY_BC_PERIODIC   (-135)
/* arithmetic of the reconstruction + flux stage */
#define FLASH_HY_PREC_FP64   0  /* FP64 everywhere, no FMA contraction   */
#define FLASH_HY_PREC_FP64_FMA 1 /* FP64 everywhere, FMA contraction on  */
#define FLASH_HY_PREC_MIXED  2  /* FP32 reconstruction/flux, FP64 update */
/* host UNK layouts: default FLASH unk(var,i,j,k,blk) and --index-reorder
 * unk(i,j,k,var,blk) (gr_createDomain.F90:133-135, bin/Readme.Reorder) */
#define FLASH_HY_LAYOUT_VAR_FASTEST 0
#define FLASH_HY_LAYOUT_XYZ_FASTEST 1
/* update modes of hy_computeFluxes (UHD.h:24-27) */
#define FLASH_HY_UPDATE_NONE 0
#define FLASH_HY_UPDATE_ALL  3

/* ---- variable map: 1-based *_VAR indices of the caller's UNK ---------- */
/* FLASH sorts VARIABLE declarations alphabetically (bin/unitCfg.py:713-714);
 * for +uhd with the gamma EOS: DENS=1 EINT=2 ENER=3 GAMC=4 GAME=5 PRES=6
 * SHOK=7 TEMP=8 VELX=9 VELY=10 VELZ=11.  0 = variable absent.           */
typedef struct flash_hy_varmap {
  int dens, eint, ener, gamc, game, pres, temp, velx, vely, velz;
  int species;   /* first species (SPECIES_BEGIN); the nspecies species and
                    the nmass_scalars mass scalars are consecutive from it
                    (SPECIES_BEGIN .. MASS_SCALARS_END); 0 when there are none */
} flash_hy_varmap;

/* ---- runtime parameters (names follow unsplit/Config:105-159) ---------- */
typedef struct flash_hy_params {
  int    order;            /* 3 = PPM (the only order on this path)       */
  int    riemann_solver;   /* FLASH_HY_RS_*                               */
  int    slope_limiter;    /* FLASH_HY_LIM_*                              */
  int    char_limiting;    /* charLimiting                                */
  int    use_flattening;   /* use_flattening                              */
  int    use_steepening;   /* use_steepening                              */
  int    use_aux_eint;     /* use_auxEintEqn                              */
  int    use_3d_full_ctu;  /* use_3dFullCTU                               */
  int    precision;        /* FLASH_HY_PREC_*                             */
  int    learned_guess;    /* exact solver: seed Newton with the MLP      */
  double limited_slope_beta;  /* LimitedSlopeBeta                         */
  double f_pres_in_mom_flux;  /* hy_fPresInMomFlux                        */
  double cfl;
  double eint_switch;      /* eintSwitch                                  */
  double smlrho, smallp, smalle, tiny;
  double gamma;            /* eos_gamma                                   */
  double gas_constant;     /* eos_gasConstant (PhysicalConstants "ideal gas constant") */
  double single_species_a; /* eos_singleSpeciesA                          */
  /* species and mass scalars advected with hy_fullSpecMsFluxHandling
   * (the default, unsplit/Config:140-143): PPM face values, upwind fluxes
   * F_dens * X, the conservative update and, for species only, the
   * renormalisation to a unit sum (hy_unsplitUpdate.F90:827-859).  At most
   * FLASH_HY_MAX_SPECIES in all.  Uniform grids and AMR hierarchies (the
   * species are restricted, prolonged in per-mass form into the guard cells
   * and corrected at fine/coarse faces like the mass flux), in the fused
   * and in the split step. */
  int nspecies;            /* NSPECIES                                     */
  int nmass_scalars;       /* NMASS_SCALARS                                */
} flash_hy_params;
#define FLASH_HY_MAX_SPECIES 16

/* ---- grid descriptor ---------------------------------------------------
 * Blocks of nxb x nyb x nzb interior cells.  FLASH keeps NGUARD=4 guard
 * layers (unsplit/Config:209-211); the device keeps none and fills halos
 * inside the kernels.  Block b sits at integer block coordinates
 * block_coords[3*b .. 3*b+2] of its refinement level block_level[b]
 * (1-based, as tileDesc%level); level L has 2^(L-1) times the level-1 block
 * count per axis (nblk_l1[]).  A uniform grid uses one level.           */
typedef struct flash_hy_grid_desc {
  int ndim;
  int nxb, nyb, nzb;
  int nguard;              /* guard layers of the host UNK arrays (0 or 4) */
  int nblocks;
  int nblk_l1[3];          /* level-1 blocks per axis                       */
  int max_level;
  const int *block_coords; /* [3*nblocks]                                   */
  const int *block_level;  /* [nblocks]                                     */
  double domain_lo[3], domain_hi[3];
  int bc[6];               /* xl, xr, yl, yr, zl, zr: FLASH_HY_BC_*         */
} flash_hy_grid_desc;

typedef struct flash_hy_ctx flash_hy_ctx;

/* Hydro_init + Grid block storage allocation.  device: CUDA ordinal. */
int flash_hy_create(const flash_hy_params *params, const flash_hy_grid_desc *grid,
                    int device, flash_hy_ctx **ctx_out);
int flash_hy_destroy(flash_hy_ctx *ctx);
/* Device memory of destroyed contexts is kept per device (at most 32 GiB)
 * and reused by later contexts, so that an AMR regrid -- a context for the
 * new tree, the old one destroyed -- costs no cudaMalloc/cudaFree round trip.
 * release_memory frees the kept blocks of a device (all devices: -1). */
int flash_hy_release_memory(int device);

/* Copy the caller's UNK (host memory, nunk variables per cell, guard layers
 * as grid->nguard) into the device block store and apply the gamma-law EOS
 * in MODE_DENS_EI to every interior cell, as Grid_initDomain does after
 * Simulation_initBlock (GridMain/UG/Grid_initDomain.F90:85).             */
int flash_hy_upload(flash_hy_ctx *ctx, const double *unk, int layout, int nunk,
                    const flash_hy_varmap *vars);
/* Write the device state back into the caller's UNK interiors: DENS, VEL*,
 * EINT plus the EOS outputs PRES, TEMP, GAMC, GAME, ENER
 * (Eos_putData semantics).  Guard cells are left untouched.             */
int flash_hy_download(flash_hy_ctx *ctx, double *unk, int layout, int nunk,
                      const flash_hy_varmap *vars);

/* Hydro(simTime, dt, dtOld, sweepOrder): guard-cell fill (with EOS on the
 * guard cells), reconstruction, Riemann solve, conservative update, energy
 * fix and EOS on every leaf block, one launch sequence on the context's
 * stream.  sweepOrder is accepted and ignored, as in the unsplit solver
 * (unsplit/Hydro.F90:45-48).  The CFL reduction of the new state is fused
 * into the update and cached for flash_hy_compute_dt.                    */
int flash_hy_step(flash_hy_ctx *ctx, double simTime, double dt, double dtOld,
                  int sweepOrder);
/* FLASH4-style Hydro(blockCount, blockList, timeEndAdv, dt, dtOld,
 * sweepOrder) / hy_uhd_unsplit: update only the listed blocks.  blockList
 * holds FLASH's 1-based block IDs (blockList(1:blockCount) as FLASH passes
 * it, localAPI/hy_biermannSource.F90:9-24): block b of the descriptor is ID
 * b + 1.  IDs outside 1..nblocks give FLASH_HY_ERR_BAD_ARG.  The same
 * 1-based IDs are taken by compute_fluxes / update_solution (blockList) and
 * get_fluxes / put_fluxes (blockID, as Grid_getFluxData).               */
int flash_hy_step_blocks(flash_hy_ctx *ctx, int blockCount, const int *blockList,
                         double timeEndAdv, double dt, double dtOld, int sweepOrder);
/* The step split in two, as hy_computeFluxes / hy_updateSolution
 * (localAPI/hy_interface.F90:969,982) and unsplit/Hydro.F90:186-230 use it
 * around a caller's own flux correction (Grid_putFluxData,
 * Grid_conserveFluxes): compute_fluxes computes and keeps the face fluxes
 * of the listed blocks (1-based block IDs) (flags = FLASH_HY_UPDATE_NONE: Uout disassociated,
 * the state is unchanged; FLASH_HY_UPDATE_ALL: also updates, as
 * flash_hy_step_blocks); get/put_fluxes read or replace one block's fluxes
 * in one direction (1..ndim) in FLASH's flux-array layout flx(NFLUXES, i,
 * j, k) over the faces (the dir index runs over nb+1 faces; host memory),
 * NFLUXES = 8 + nspecies + nmass_scalars: the species and mass-scalar
 * fluxes F_dens * X follow the 8 hydro fluxes (xflux(HY_END_FLUX + isph),
 * hy_getFaceFlux.F90:453-467); update_solution applies the kept (possibly
 * replaced) fluxes to the listed blocks, species and mass scalars included
 * (hy_unsplitUpdate.F90:478-491, 827-859).  Uniform grids only.          */
int flash_hy_compute_fluxes(flash_hy_ctx *ctx, int blockCount, const int *blockList, double dt, int flags);
int flash_hy_get_fluxes(flash_hy_ctx *ctx, int blockID, int dir, double *flx);
int flash_hy_put_fluxes(flash_hy_ctx *ctx, int blockID, int dir, const double *flx);
int flash_hy_update_solution(flash_hy_ctx *ctx, int blockCount, const int *blockList, double dt);

/* Hydro_computeDt + the MPI_MINLOC reduction of Driver_computeDt.F90:376-377:
 * dt_out = cfl / max_cells max_d (|u_d| + c_s)/dx_d; minloc_out = (i, j, k,
 * level, meshMe) as FLASH's dtMinLoc (Hydro_computeDt.F90:266-270): 1-based
 * guard-inclusive cell indices, the block's refinement level and the rank
 * set by flash_hy_set_mesh_me (hy_meshMe; 0 by default).  Across ranks the
 * caller reduces as Driver_computeDt does (MINLOC, then a broadcast from the
 * winning rank).                                                         */
int flash_hy_compute_dt(flash_hy_ctx *ctx, double *dt_out, int minloc_out[5]);
/* The rank this context reports in minloc_out[4] (hy_meshMe, the MPI rank
 * of the process owning the context's blocks).                           */
int flash_hy_set_mesh_me(flash_hy_ctx *ctx, int rank);
/* FLASH's 1-based block ID of the cell that set the last flash_hy_compute_dt
 * (0 when none did); FLASH's dtMinLoc does not carry it.                 */
int flash_hy_dt_block(flash_hy_ctx *ctx, int *blockID);

/* Device-side access for callers that keep the state resident. */
int flash_hy_sync(flash_hy_ctx *ctx);
void *flash_hy_stream(flash_hy_ctx *ctx);        /* cudaStream_t of the context */
/* Enqueue (on the context's stream) a copy of the device state into the
 * caller's DEVICE buffer d_out: [5][nblocks * nzb * nyb * nxb] doubles --
 * dens, velx, vely, velz, eint of every block's interior, block-major.
 * No FLASH counterpart (FLASH's state lives in host UNK). */
int flash_hy_export_state(flash_hy_ctx *ctx, double *d_out);
int flash_hy_last_error(flash_hy_ctx *ctx, char *buf, int len);
/* Number of kernel launches issued by the last flash_hy_step call. */
int flash_hy_last_launch_count(flash_hy_ctx *ctx);

/* ---- exact solver inside the hydro step (riemann_solver = FLASH_HY_RS_EXACT)
 * No counterpart in FLASH5 (see the exact-solver section below).  With
 * learned_guess = 1 (mixed precision only) the face solves start Newton
 * from the network's estimate of p* once weights are attached; until then,
 * and wherever the network's start does not converge within three
 * evaluations, they start from the two-rarefaction guess, so the converged
 * fluxes do not depend on the network.  w = FP32 master weights in the
 * layout of flash_hy_rsolver_get_weights (n = flash_hy_rsolver_num_params()),
 * host memory.                                                          */
int flash_hy_set_guess_weights(flash_hy_ctx *ctx, const float *w, int n);
/* Keep a hashed sample (about one face in 2^keep_log2 where the
 * two-rarefaction guess is not exact) of the face states the mixed exact
 * path solves, up to cap states, as training data for the guess; cap = 0
 * stops.  fetch copies the states kept so far into the DEVICE array
 * d_states as SoA [7][n] (rho_L, u_L, p_L, rho_R, u_R, p_R, gamma; u normal
 * to the face), n = min(kept, n_max), and starts a new sample; d_states =
 * NULL only reports the count.                                          */
int flash_hy_harvest(flash_hy_ctx *ctx, long long cap, int keep_log2);
int flash_hy_harvest_fetch(flash_hy_ctx *ctx, double *d_states, long long n_max, long long *n_out);

/* ---- sharded grids (one context per GPU / MPI rank) ----------------------
 * FLASH distributes blocks over MPI ranks (PARAMESH Morton order, UG process
 * grid) and fills guard cells from other ranks' blocks in
 * Grid_fillGuardCells (UG gr_shiftData.F90:100-173); the dt reduction is the
 * MPI_MINLOC of Driver_computeDt.F90:376-377.  A rank's context is created
 * from its share of the grid: its owned blocks plus ghost blocks (copies of
 * other ranks' blocks touching an owned block), all with global block
 * coordinates and the global nblk_l1.  set_owned_blocks names the blocks
 * flash_hy_step advances and flash_hy_compute_dt reduces over (local
 * indices; every block an owned block reads guard cells from must be
 * present); set_exchange names the local blocks packed for other ranks and
 * those unpacked from them; pack / unpack copy the 5 state variables of
 * those blocks (nblocks x (5 + nspecies + nmass_scalars) x nxb*nyb*nzb
 * doubles: the state variables, then the species; DEVICE buffers) on the
 * context's stream.  Ghost blocks are not advanced: unpack fresh copies
 * before every step.                                                     */
int flash_hy_set_owned_blocks(flash_hy_ctx *ctx, int n, const int *blocks);
int flash_hy_set_exchange(flash_hy_ctx *ctx, int nsend, const int *send_blocks, int nrecv,
                          const int *recv_blocks);
int flash_hy_pack(flash_hy_ctx *ctx, double *d_buf);
int flash_hy_unpack(flash_hy_ctx *ctx, const double *d_buf);
/* The step of a rank's share in two phases, so that the ghost exchange
 * overlaps the step (gr_shiftData.F90:100-173 exchanges first, then FLASH
 * steps): phase 1 advances the owned blocks whose guard cells all lie in
 * owned blocks and may run while the ghost blocks are in transit; phase 2,
 * after flash_hy_unpack, advances the other owned blocks and completes the
 * step (the state advances, the CFL reduction covers all owned blocks).
 * Phase 2 must follow phase 1 with the same dt.  Results equal
 * flash_hy_step on the same share bit for bit.                          */
int flash_hy_step_phase(flash_hy_ctx *ctx, double simTime, double dt, double dtOld, int phase);

/* ---- refinement criterion ------------------------------------------------
 * gr_estimateError / gr_estimateBlkError (Grid/GridMain/AMR/
 * gr_estimateBlkError.F90, Cartesian): Lohner's normalised second-derivative
 * estimator of one variable for every block, leaves and parents (FLASH's
 * ACTIVE_BLKS), after the guard-cell fill with EOS that
 * Grid_markRefineDerefine.F90 performs.  err (HOST, nblocks doubles)
 * receives sqrt(max over the cells of num / denom) per block; HUGE where a
 * cell has denom = 0 and num != 0.  The pressure is (gamma-1) rho e of each
 * cell (parents: of their restricted state).  Uniform grids and AMR
 * hierarchies.                                                          */
#define FLASH_HY_REFVAR_DENS 1
#define FLASH_HY_REFVAR_PRES 2
#define FLASH_HY_REFVAR_VELX 3
#define FLASH_HY_REFVAR_VELY 4
#define FLASH_HY_REFVAR_VELZ 5
#define FLASH_HY_REFVAR_EINT 6
int flash_hy_estimate_error(flash_hy_ctx *ctx, int var, double refine_filter, double *err);

/* ---- regrid --------------------------------------------------------------
 * gr_updateRefinement (Grid/GridMain/AMR/paramesh/gr_updateRefinement.F90:
 * 112-238) after the host has marked blocks (gr_markRefineDerefine) and
 * built the new tree: fills the state of context new_ctx (created for the
 * new hierarchy) from old_ctx.  For every new node q: how[q] = 0 copies old
 * node src[q] (a kept node, or a refined leaf that becomes a parent); 2
 * turns old parent src[q] into a leaf with its restricted data
 * (derefinement); 1 prolongs new child q from old leaf src[q]
 * (amr_prolong: linear prolongation in per-volume form from the old leaf
 * with its guard cells in the old hierarchy).  Then the EOS on every leaf,
 * as FLASH does after a grid change.  Both contexts must be AMR
 * hierarchies of the same block shape on the same device.               */
int flash_hy_regrid(flash_hy_ctx *old_ctx, flash_hy_ctx *new_ctx, int n, const int *src, const int *how);

/* The tree of a regrid (PARAMESH amr_refine_derefine, restated): from the
 * grid descriptor of an AMR hierarchy and per-node marks (refine, derefine:
 * 0/1 bytes, leaves only), the marked leaves below max_level are split,
 * refinement spreads until every leaf's neighbours (diagonals included) are
 * within one level, and a parent at level >= min_level loses its children
 * when all of them are unrefined leaves marked for derefinement and no
 * neighbour's child touching it stays refined.  Writes the new node count
 * to *new_n and, when it fits in cap, the new nodes ordered by level and
 * Morton index: new_levels[n], new_coords[3n], new_parent[n] (-1 on level
 * 1), and src / how for flash_hy_regrid.  FLASH_HY_ERR_BAD_ARG when cap is
 * too small (*new_n says how much is needed) or the tree is incomplete. */
int flash_hy_refine_tree(const flash_hy_grid_desc *grid, const unsigned char *refine, const unsigned char *derefine,
                         int min_level, int cap, int *new_n, int *new_levels, int *new_coords, int *new_parent,
                         int *src, int *how);

/* Grid_markRefineDerefine + the tree of Grid_updateRefinement on the device:
 * the estimator of each of the nvar variables vars[] (FLASH_HY_REFVAR_*,
 * refine_filter as flash_hy_estimate_error), FLASH's marks with the
 * per-variable cutoffs refine_cutoff[v] / derefine_cutoff[v] and max_refine
 * (gr_markRefineDerefine.F90: per variable, a leaf is marked for
 * derefinement when it is not marked to refine or stay and both its error
 * and its parent's are at or below the derefine cutoff; any node above the
 * refine cutoff is marked to refine, not at or above max_refine; only leaves
 * keep their marks), then the tree rules of flash_hy_refine_tree, all as
 * kernels over a dense table of block positions per level.  The outputs are
 * those of flash_hy_refine_tree for the same marks, in HOST arrays (the new
 * context is created from them): new_n, new_levels, new_coords, new_parent,
 * src, how.  AMR hierarchies of at most 15 levels.                     */
int flash_hy_mark_refine_tree(flash_hy_ctx *ctx, int nvar, const int *vars, double refine_filter,
                              const double *refine_cutoff, const double *derefine_cutoff, int max_refine,
                              int min_level, int cap, int *new_n, int *new_levels, int *new_coords, int *new_parent,
                              int *src, int *how);

/* ---- launch shapes and their autotuner ----------------------------------
 * No FLASH5 counterpart (FLASH picks no launch shapes; its block loop is
 * Hydro.F90:156-229).  Threads per CTA of the step's kernels: the
 * transverse-flux and CFL passes (sig_threads), the FP64 direction kernels
 * (dir_threads; FLASH_HY_PREC_FP64 and _FP64_FMA) and the mixed-precision
 * direction kernels (mx_threads; FLASH_HY_PREC_MIXED, three compiled
 * candidates per block shape).  Every face and cell is computed by one
 * thread and the CFL reduction is order independent, so sig_threads and
 * dir_threads leave results bit-identical; the mx_threads candidates are
 * separately compiled FMA-contracted kernels and agree to rounding.
 * set_tuning refuses values that are not
 * candidates of the context's block shape (FLASH_HY_ERR_BAD_ARG);
 * tuning_candidates lists them (arrays of FLASH_HY_TUNE_MAX entries).
 * autotune times `steps` steps of dt, after one untimed step, for every
 * candidate of the direction kernels (then, on the mixed path, the other
 * mx_runs setting where runs are offered and the other sweep order) and
 * then of the transverse-flux pass
 * (coordinate search: the two are separate launches), each trial from a
 * copy of the current state; it restores the state, keeps the fastest
 * shape, and writes every trial (shape, ms per step) to table / table_ms
 * (capacity cap; *n_trials = their number).  Status bits raised by the
 * trials are dropped; the next flash_hy_compute_dt recomputes dt from the
 * restored state.                                                         */
#define FLASH_HY_TUNE_MAX 8
/* mx_runs: blocks a CTA of the mixed-precision 3D direction kernels
 * stages along the sweep -- 1, or FLASH_HY_MX_RUN where the context offers
 * runs (a full uniform grid of 8^3 blocks whose block counts divide by it,
 * no species): the CTA then takes runs of FLASH_HY_MX_RUN blocks and
 * 1/FLASH_HY_MX_RUN of their cross-section, which shares the stencil
 * overlap along the sweep.  The two are separately compiled FMA-contracted
 * kernels, like the mx_threads candidates, and agree to rounding.  The
 * default is FLASH_HY_MX_RUN where offered; autotune tries both.        */
#define FLASH_HY_MX_RUN 4
/* mx_sweep: the order in which the mixed-precision direction kernels
 * accumulate the conservative update -- FLASH_HY_SWEEP_XYZ (the default)
 * or FLASH_HY_SWEEP_ZYX, FLASH's SWEEP_XYZ / SWEEP_ZYX values
 * (source/Simulation/constants.h:359-360).  Each direction's face states
 * and fluxes come from the same old state either way (the step is
 * unsplit), so the two orders agree to rounding; the FP64 paths keep
 * x, y, z, the order of FLASH's update expression, and accept only
 * FLASH_HY_SWEEP_XYZ; the split step (flash_hy_compute_fluxes /
 * flash_hy_update_solution) runs x, y, z whatever is set.  autotune tries
 * both on the mixed path.                                               */
#define FLASH_HY_SWEEP_XYZ 1
#define FLASH_HY_SWEEP_ZYX 2
typedef struct {
  int sig_threads;
  int dir_threads;
  int mx_threads;
  int mx_runs;
  int mx_sweep;
} flash_hy_tuning;
int flash_hy_get_tuning(flash_hy_ctx *ctx, flash_hy_tuning *out);
int flash_hy_set_tuning(flash_hy_ctx *ctx, const flash_hy_tuning *t);
int flash_hy_tuning_candidates(flash_hy_ctx *ctx, int *sig, int *n_sig, int *dir, int *n_dir, int *mx,
                               int *n_mx);
int flash_hy_autotune(flash_hy_ctx *ctx, double dt, int steps, flash_hy_tuning *best, flash_hy_tuning *table,
                      float *table_ms, int cap, int *n_trials);

/* ---- CFL time step without any device allocation ------------------------
 * No counterpart in the reference: FLASH5's Hydro_computeDt runs on host
 * arrays.  This entry point is for callers that cannot call cudaMalloc
 * (device memory owned by another framework's pool, or a fixed allocation
 * budget set at start-up).  It
 * computes the time step of flash_hy_compute_dt from caller-owned DEVICE
 * arrays (block-major SoA: dens, velx, vely, velz, eint of the interiors,
 * nblocks x nzb x nyb x nxb each, all EOS-consistent) and writes dt and the
 * minloc (i, j, k, level, block) to HOST memory.  Its scratch is a fixed
 * file-scope device array of FLASH_HY_NOALLOC_MAX_BLOCKS entries (1.5 MiB,
 * held by every GPU that loads the library until exit); larger grids are
 * rejected with FLASH_HY_ERR_BAD_ARG.  The first call in each CUDA context
 * (per device, or per driver-API context) resolves the scratch address and
 * should precede any stream capture.  The result is returned on the host, so
 * the call synchronises `stream` (NULL: the default stream).  All calls share
 * the scratch: calls that overlap on the GPU race, and the caller serialises
 * them.  minloc_out[4] is the 0-based block (the arrays carry no rank).  */
#define FLASH_HY_NOALLOC_MAX_BLOCKS 65536
int flash_hy_compute_dt_noalloc(const double *d_dens, const double *d_velx, const double *d_vely,
                                const double *d_velz, const double *d_eint, int ndim, int nxb, int nyb, int nzb,
                                int nblocks, const double deltas[3], double gamma, double cfl, void *stream,
                                double *dt_out, int minloc_out[5]);

/* ---- exact Riemann solver with a learned star-pressure guess ----------
 * No counterpart in FLASH5 (its unsplit solvers are approximate:
 * source/physics/Hydro/HydroMain/unsplit/hy_getFaceFlux.F90:324-372); the
 * hydro step uses it when riemann_solver = FLASH_HY_RS_EXACT.  Arrays are
 * DEVICE pointers.  states = SoA [7][n] of (rho_L, u_L, p_L, rho_R, u_R,
 * p_R, gamma) with u the face-normal velocity; star = SoA [2][n] (p*, u*);
 * iters[n] = Newton iterations (fallback included); flags[n]: bit 0 fell
 * back to the two-rarefaction guess, bit 1 vacuum, bit 2 not converged,
 * bit 3 the network was consulted (learned solves with strong waves).   */
typedef struct flash_hy_rsolver flash_hy_rsolver;
int flash_hy_rsolver_create(int device, flash_hy_rsolver **out);
int flash_hy_rsolver_destroy(flash_hy_rsolver *r);
void *flash_hy_rsolver_stream(flash_hy_rsolver *r);
int flash_hy_rsolver_generate(flash_hy_rsolver *r, unsigned long long seed, long n, double *d_states);
int flash_hy_rsolver_solve(flash_hy_rsolver *r, const double *d_states, long n, double *d_star,
                           unsigned char *d_iters, unsigned char *d_flags, int learned, double tol, int max_iter);
/* network output: the estimate of ln(pstar / p_TR) per interface (d_y[n] floats) */
int flash_hy_rsolver_predict(flash_hy_rsolver *r, const double *d_states, long n, float *d_y);
int flash_hy_rsolver_make_samples(flash_hy_rsolver *r, const double *d_states, const double *d_star, long n,
                                  float *d_x, float *d_t, long cap, long *count_out);
int flash_hy_rsolver_grad(flash_hy_rsolver *r, const float *d_x, const float *d_t, const int *d_idx, int nb,
                          float *h_grad, float *h_loss);
int flash_hy_rsolver_train(flash_hy_rsolver *r, const float *d_x, const float *d_t, long ns, int epochs, int batch,
                           float lr, float *loss_out);
int flash_hy_rsolver_get_weights(flash_hy_rsolver *r, float *h_w, int n);
int flash_hy_rsolver_set_weights(flash_hy_rsolver *r, const float *h_w, int n);
int flash_hy_rsolver_num_params(void);
int flash_hy_rsolver_sync(flash_hy_rsolver *r);
/* Where the batched solves and predict run the network: on the tcgen05
 * tensor cores, 128 interfaces per MMA tile with the accumulator in TMEM
 * (FLASH_HY_INFER_TCGEN05, the default), or per warp on mma.sync
 * (FLASH_HY_INFER_WARP_MMA, the form the hydro kernels use inline).  Both
 * give the same converged p*; the network outputs agree to rounding (the
 * tcgen05 form takes the FP32 biases and output weights as two BF16 parts
 * and accumulates in another order).  Other values give
 * FLASH_HY_ERR_BAD_ARG.                                                 */
#define FLASH_HY_INFER_TCGEN05  0
#define FLASH_HY_INFER_WARP_MMA 1
int flash_hy_rsolver_set_inference(flash_hy_rsolver *r, int mode);

#ifdef __cplusplus
}
#endif
#endif /* FLASH_HY_H */
