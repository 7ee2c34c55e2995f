/*
 * rgpu.h -- C ABI of the B200 Godunov level step (librgpu.so).
 *
 * The library replaces the CPU hydro hot path of RAMSES-CPP,
 * HydroSolver::godunov_fine(ilevel, dt, dx) and the calls around it in
 * Simulation::amr_step, for a host application that keeps owning its AmrGrid.
 * Every entry point takes plain pointers and sizes; no C++ or torch type
 * crosses the boundary.  Every function that can fail returns an int status
 * (RG_OK == 0, negative on error) and never throws or aborts; the message of
 * the last failure is returned by rg_last_error().
 *
 * Reference interfaces replaced (paths relative to the RAMSES-CPP tree):
 *   include/ramses/solvers/hydro/HydroSolver.hpp:19   godunov_fine
 *   include/ramses/solvers/hydro/HydroSolver.hpp:20   set_uold
 *   include/ramses/solvers/hydro/HydroSolver.hpp:21   set_unew
 *   include/ramses/solvers/hydro/HydroSolver.hpp:22   compute_courant_step
 *   include/ramses/core/AmrGrid.hpp:26-31,104-107     grid arrays and uold layout
 *
 * Data layout is the reference's own (AmrGrid.hpp:104-107): the state is
 * [nvar][ncell] doubles, variable-major; cell ids are 1-based,
 * icell = ncoarse + (ic-1)*ngridmax + igrid (AmrGrid.cpp:279).
 *
 * Threading: one host thread per rg_ctx; calls are not re-entrant.  All device
 * work is queued on the context's own stream; rg_download_state and
 * rg_synchronize are the synchronisation points.
 */
#ifndef RGPU_H
#define RGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RG_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
enum {
    RG_OK = 0,
    RG_ERR_ARG = -1,         /* invalid argument (null pointer, bad size, bad level)   */
    RG_ERR_CUDA = -2,        /* a CUDA runtime call failed (message has the CUDA error) */
    RG_ERR_UNSUPPORTED = -3, /* configuration outside what the GPU path implements      */
    RG_ERR_TOPOLOGY = -4,    /* inconsistent tree arrays (list cycle, bad index)        */
    RG_ERR_STATE = -5,       /* call made before the data it needs was provided         */
    RG_ERR_TIMEOUT = -6,     /* a bounded device-side wait gave up                      */
    RG_ERR_DEVICE = -7,      /* a device-side check set the error word (see message)    */
    RG_ERR_NOMEM = -8        /* device allocation failed                                */
};

/* ---- Riemann solver selection (hydro_params/riemann) -------------------- */
/* The reference resolves the string at HydroSolver.cpp:456-461; any string it
 * does not know falls back to LLF, and rg_riemann_from_string does the same. */
enum {
    RG_RIEMANN_LLF = 0,
    RG_RIEMANN_HLL = 1,
    RG_RIEMANN_HLLC = 2,
    RG_RIEMANN_EXACT = 3,
    RG_RIEMANN_ACOUSTIC = 4
};

/* Exact-solver Newton initial guess. */
enum {
    RG_GUESS_TWO_SHOCK = 0, /* RiemannSolver.cpp:215 (the reference's guess)          */
    RG_GUESS_LEARNED = 1    /* MLP prediction (rg_mlp_*), two-shock as the fallback   */
};

/* Solver knobs, read once per call instead of per interface
 * (HydroSolver.cpp:55,62,216-217,456 look them up by string inside the loop). */
typedef struct rg_params {
    int ndim;            /* 1 or 3 (compile-time NDIM of the host build)              */
    int nvar;            /* ndim+2 plus passive scalars; non-thermal energies unsupported */
    int slope_type;      /* hydro_params/slope_type, 0..8 (SlopeLimiter.cpp:7-60)     */
    int riemann;         /* RG_RIEMANN_*                                               */
    int interpol_type;   /* refine_params/interpol_type (ghost-cell slopes)            */
    int interpol_var;    /* refine_params/interpol_var                                 */
    double gamma;        /* AmrGrid::gamma                                             */
    double courant_factor;
    int exact_niter;     /* Newton iteration cap; reference value 10 (RiemannSolver.cpp:198) */
    double exact_tol;    /* stop when |dp/(p+1e-10)| < tol; reference 1e-6 (:234)      */
    int exact_guess;     /* RG_GUESS_*                                                 */
    double boxlen;       /* amr_params/boxlen; only sets the CFL start value (HydroSolver.cpp:880) */
    int flags;           /* reserved, must be 0                                        */
} rg_params;

/* Borrowed view of the host AmrGrid arrays (AmrGrid.hpp:15-31).  The library
 * copies what it needs during rg_sync_topology and keeps no host pointer. */
typedef struct rg_grid_view {
    int ncoarse, ngridmax, ncell, nvar;
    int nx, ny, nz;
    int ncpu, nboundary, nlevelmax;
    const int* son;        /* [ncell]                                   */
    const int* father;     /* [ngridmax]                                */
    const int* nbor;       /* [6*ngridmax]: father cell of each neighbour oct */
    const int* next;       /* [ngridmax]: level / free linked lists     */
    const int* headl;      /* [(ncpu+nboundary)*(nlevelmax+1)] (headl_vec) */
    const int* bound_type; /* [nbound_type] or NULL                     */
    int nbound_type;
} rg_grid_view;

typedef struct rg_ctx rg_ctx;

/* ---- lifecycle ----------------------------------------------------------- */
/* Replaces HydroSolver::HydroSolver (HydroSolver.hpp:16).  device < 0 picks the
 * current CUDA device.  Returns NULL only when allocation of the host-side
 * context itself fails; a context whose set-up failed reports it through
 * rg_last_error and returns errors from every later call. */
rg_ctx* rg_create(const rg_params* params, int device);
void rg_destroy(rg_ctx* ctx);
const char* rg_last_error(const rg_ctx* ctx);
int rg_set_params(rg_ctx* ctx, const rg_params* params);
int rg_riemann_from_string(const char* name);
const char* rg_version(void);

/* ---- grid mirror ---------------------------------------------------------- */
/* Upload the tree arrays.  Must be called after every host change of the tree
 * (TreeUpdater) or of ngridmax (AmrGrid::resize_grids, AmrGrid.cpp:118-238);
 * it invalidates every cached level plan and CUDA graph. */
int rg_sync_topology(rg_ctx* ctx, const rg_grid_view* grid);
/* Copy host state [nvar][ncell] to the device; either pointer may be NULL. */
int rg_upload_state(rg_ctx* ctx, const double* uold, const double* unew);
/* Copy device state back to host [nvar][ncell]; either pointer may be NULL.
 * Synchronises the context stream. */
int rg_download_state(rg_ctx* ctx, double* uold, double* unew);
/* Device addresses of the resident state (for callers that keep data on the
 * GPU between steps).  Valid until the next rg_sync_topology. */
int rg_device_state(rg_ctx* ctx, double** uold_dev, double** unew_dev);

/* ---- the level step ------------------------------------------------------- */
/* HydroSolver::set_unew (HydroSolver.cpp:575-590): unew <- uold on level. */
int rg_set_unew(rg_ctx* ctx, int ilevel);
/* HydroSolver::set_uold (HydroSolver.cpp:592-611): uold <- unew, son==0 only. */
int rg_set_uold(rg_ctx* ctx, int ilevel);
/* HydroSolver::godunov_fine (HydroSolver.cpp:18-573), including the reflux
 * into coarser and same-level neighbour cells in the reference's order. */
int rg_godunov_level(rg_ctx* ctx, int ilevel, double dt, double dx);
/* HydroSolver::compute_courant_step (HydroSolver.cpp:878-977).  With
 * pressure_cap != 0 the reference formula is used as is (p <= 100 rho);
 * with 0 the cap is left out (the stable variant for strong blasts).
 * Synchronises and writes the minimum to *dt_out. */
int rg_courant_step(rg_ctx* ctx, int ilevel, double dx, double courant_factor,
                    int pressure_cap, double* dt_out);
/* One device-resident level substep: dt from the on-device CFL reduction
 * (rg_courant_step semantics, no host round trip), then set_unew,
 * godunov_fine and set_uold.  With use_graph != 0 the sequence is captured in
 * a CUDA graph on first use and replayed afterwards.  *dt_used (may be NULL)
 * receives the dt of this substep after an implicit synchronisation only when
 * dt_used is non-NULL. */
int rg_level_substep(rg_ctx* ctx, int ilevel, double dx, int pressure_cap,
                     int use_graph, double* dt_used);
int rg_synchronize(rg_ctx* ctx);
/* Run the context's work on a caller-owned cudaStream_t (passed as void*,
 * NULL restores the context's own stream), or read the stream in use, so a
 * host application can order the level step with its own work and time it
 * with its own events.  Changing the stream drops captured graphs. */
int rg_set_stream(rg_ctx* ctx, void* stream);
int rg_get_stream(rg_ctx* ctx, void** stream);

/* A single-level run: the host loop
 *     t = t_start; n = 0;
 *     while (t < t_end && n < max_steps) { rg_level_substep(.., &dt); t += dt; ++n; }
 * (Simulation's time loop when levelmin == levelmax, Simulation.cpp:366-430)
 * as ONE CUDA graph launch: a WHILE conditional node repeats the substep and
 * a clock kernel that adds dt on the device and sets the loop condition, so
 * no dt travels to the host between substeps.  Same state bits, t and step
 * count as the host loop.  Levels of at most 1024 cells run the whole loop
 * in one single-block kernel instead (block barriers between the phases of
 * a substep, no launch per substep).  Levels without refined cells whose
 * stencils stay inside them (uniform periodic grids), one box; max_steps
 * bounds the loop, and each launch runs at most 65,536 substeps (the host
 * relaunches until t_end or max_steps), so no launch runs for long. */
int rg_level_run(rg_ctx* ctx, int ilevel, double dx, int pressure_cap, double t_start, double t_end,
                 int64_t max_steps, double* t_out, int64_t* steps_out);

/* ---- exact solver and its learned Newton start ----------------------------- */
/* Exact two-shock Newton solves (RiemannSolver::solve_godunov_nr,
 * RiemannSolver.cpp:194-307) of n independent interfaces.  Device arrays:
 * ql/qr [ndim+2][n] rotated primitives (rho, u_n, u_t..., p), gamma [n] or
 * NULL (params.gamma), outputs flux [ndim+2][n], pstar [n], iters [n] (Newton
 * updates), each may be NULL.  guess: RG_GUESS_TWO_SHOCK (the reference's
 * :215) or RG_GUESS_LEARNED.  niter/tol: 10/1e-6 reproduce the reference;
 * a tol of 1e-14 with a larger cap is the converged mode. */
int rg_exact_batch(rg_ctx* ctx, int n, const double* ql_dev, const double* qr_dev, const double* gamma_dev,
                   double* flux_dev, double* pstar_dev, int* iters_dev, int guess, int niter, double tol);
/* The exact solver's stress workload, seeded: density ratios log-uniform to
 * 1e4, pressure ratios to 1e6, 30 % strong double rarefactions, gamma 5/3 or
 * 1.4 per interface; layout as rg_exact_batch. */
int rg_stress_states(rg_ctx* ctx, int n, uint64_t seed, double* ql_dev, double* qr_dev, double* gamma_dev);
/* Learned Newton start (no reference counterpart): an 8-64-64-1 SiLU MLP
 * predicting log(pstar / base), base = Toro's two-shock estimate (the plain
 * guess's formula with the wave mass fluxes evaluated at the plain guess),
 * from the interface states, trained on the GPU
 * (BF16 tensor-core forward/backward, FP32 master weights, Adam) on nsamples
 * stress states labelled by the converged Newton root.  Used by
 * rg_exact_batch and by the level step when params.exact_guess ==
 * RG_GUESS_LEARNED; the two-shock guess is kept whenever the prediction is not
 * a finite positive number or lies within the gate band of it (near-linear
 * waves, where the linearised start is already exact).  *loss_out: mean
 * squared error (standardised target) over the last epoch. */
int rg_mlp_train(rg_ctx* ctx, int nsamples, int epochs, int batch, float lr, uint64_t seed, float* loss_out);
int rg_mlp_nparam(void);
/* Parameter block of rg_mlp_nparam() floats: W1[64][8], b1, W2[64][64], b2,
 * w3, b3, feature means and scales [8]+[8], target mean and scale, gate
 * (|log(prediction / two-shock guess)| below which the two-shock guess is
 * kept; 0.2 after training). */
int rg_mlp_get(rg_ctx* ctx, float* params);
int rg_mlp_set(rg_ctx* ctx, const float* params);
/* Gradient check: loss (sum of squared errors) and gradients of the mean
 * squared error w.r.t. the first 4801 parameters for n samples of
 * standardised features x [8][n] and targets t [n] (host arrays), computed by
 * the training kernel without updating the weights. */
int rg_mlp_grad(rg_ctx* ctx, int n, const float* x, const float* t, float* grad, float* loss);

/* Level step on state held in host memory: the drop-in form of
 * HydroSolver::godunov_fine (HydroSolver.cpp:18-573) for callers whose
 * AmrGrid keeps uold/unew on the host between calls.  Uploads uold only at
 * the cells the step reads (the level's cells and the stencil cells outside
 * it) and unew only at its update targets, runs the step, and writes back
 * unew at the targets alone; every other host value is left untouched, as
 * the reference leaves it.  uold/unew: host arrays of nvar*ncell doubles in
 * AmrGrid's layout.  Synchronises the context stream before returning. */
int rg_godunov_level_host(rg_ctx* ctx, int ilevel, double dt, double dx, const double* uold, double* unew);
/* Level-wise transfers for a host application that keeps the state resident
 * on the device between its hydro calls and touches it on the host in between
 * (the reference's TreeUpdater reads uold, restrict_fine writes the refined
 * cells' uold, make_grid_fine writes the new cells' uold and unew; none reads
 * unew).  rg_upload_level: the cells a level step of ilevel reads -- the
 * level's cells, refined ones included, and the coarser cells of its ghost
 * stencils -- from host uold (nvar*ncell doubles, AmrGrid's layout).
 * rg_download_level: every cell of the level from the device uold and unew
 * into host arrays (either may be null); synchronises.  No reference
 * counterpart: they replace the host-resident vectors of AmrGrid.hpp:104-107
 * around HydroSolver::set_unew / set_uold (HydroSolver.cpp:575-611). */
int rg_upload_level(rg_ctx* ctx, int ilevel, const double* uold);
int rg_download_level(rg_ctx* ctx, int ilevel, double* uold, double* unew);

/* Snapshot records of level ilevel from the device state, as
 * RamsesWriter::write_hydro (src/io/RamsesWriter.cpp:145-226) writes them:
 * out[((ic-1)*nvar + iv-1)*noct + k] for child slot ic, variable iv (density
 * floored at 1e-10, velocities, pressure) and the level's k-th oct in list
 * order.  cap: doubles available at out (needs 2^ndim * nvar * noct).
 * Synchronises the context stream. */
int rg_level_output(rg_ctx* ctx, int ilevel, double* out, int64_t cap);

/* One substep (rg_level_substep) of a level without refined cells on state
 * held in host memory: uploads uold only at the cells the substep reads, runs
 * it, and writes back uold (and unew, if not null) at the level's update
 * targets only.  For callers that keep the state on the host between
 * substeps.  Synchronises the context stream before returning. */
int rg_level_substep_host(rg_ctx* ctx, int ilevel, double dx, int pressure_cap, double* uold, double* unew,
                          double* dt_used);

/* ---- allocation-free variant ---------------------------------------------- */
/* No counterpart in the reference.  The same level step as rg_godunov_level
 * for callers that must not allocate device memory once set-up is over (a
 * device-memory budget committed at start-up, a framework allocator that owns
 * the free memory, a time loop that may not call cudaMalloc/cudaFree because
 * they synchronise): it calls no allocating routine.  State comes from the
 * caller's device buffers, [nvar][ncell] like the grid, on the context's
 * device and at least nvar*ncell doubles long (checked; RG_ERR_ARG otherwise):
 * uold_dev is read; unew_dev must already hold the level's starting unew --
 * normally a copy of uold_dev, as rg_set_unew makes it -- since the fold adds
 * the flux updates to it, and only the level's update targets (its cells and
 * the coarser cells that take refluxes) are written.  The flux scratch is a 64 MiB static device
 * array inside the library (levels of at most 279,620 cells in 3D, 1,398,101
 * in 1D; larger levels return RG_ERR_ARG); every GPU that loads the library
 * keeps those 64 MiB until exit.  The level's plan must already exist (one
 * earlier rg_godunov_level or rg_set_unew call for the level after
 * rg_sync_topology, or after a change of the device-resident tree, builds
 * it), else RG_ERR_STATE; RG_ERR_STATE too for the learned Newton start
 * without a network, as rg_godunov_level.  The first call on each
 * device resolves the scratch address with cudaGetSymbolAddress, so make that
 * first call before any stream capture.  All calls share the one scratch
 * array: calls whose kernels overlap on the GPU race and must be ordered by
 * the caller; nothing in it needs to start at zero. */
int rg_godunov_level_noalloc(rg_ctx* ctx, int ilevel, double dt, double dx, const double* uold_dev,
                             double* unew_dev);

/* ---- introspection (integer parity checks, profiling) ---------------------- */
/* Oct ids (1-based) of level ilevel in linked-list order.  *n_out gets the
 * count; at most cap entries are written. */
int rg_level_octs(rg_ctx* ctx, int ilevel, int* octs_out, int cap, int* n_out);
/* Neighbour cell ids per level cell, the result of AmrGrid::get_nbor_cells
 * (AmrGrid.cpp:402-444): out[(k*2^ndim + ic-1)*6 + j], j = 2*idim+side. */
int rg_level_nbor_cells(rg_ctx* ctx, int ilevel, int* out, int cap);
/* Sizes of a level's step plan (built on demand): the level's cells, the
 * update targets (those cells plus the coarser cells that receive
 * refluxes, HydroSolver.cpp:476-482), the ordered update events, the coarser
 * cells read by ghost stencils, and the targets with more than 16 updates,
 * which the fold hands one warp each. */
typedef struct rg_plan_info {
    int ncells, ntarg, nevents, nextra_prim, nlong;
} rg_plan_info;
int rg_level_plan_info(rg_ctx* ctx, int ilevel, rg_plan_info* out);
/* Number of cell updates (son==0 cells) the last rg_godunov_level or
 * rg_level_substep of this level processed. */
int64_t rg_level_cell_updates(rg_ctx* ctx, int ilevel);
/* Milliseconds of device time of the last godunov kernels (CUDA events on the
 * context stream); per-kernel breakdown in out[0..n) (prim, face, fold; in a
 * fused leaf substep "prim" covers the CFL + primitive pass). */
int rg_last_kernel_ms(rg_ctx* ctx, float* out, int n);
/* Device memory of the context's stream-ordered pool, which every device
 * array of the context comes from: bytes the pool holds from the driver
 * (reserved) and bytes handed out (used).  No reference counterpart. */
int rg_pool_usage(rg_ctx* ctx, uint64_t* reserved, uint64_t* used);
/* Enable (on != 0) or disable the per-kernel CUDA events read by
 * rg_last_kernel_ms; they are recorded by rg_godunov_level and by eager
 * (use_graph == 0) rg_level_substep calls (captured graphs carry no events).  The RG_TIMING=1 environment variable sets the
 * initial value. */
int rg_set_timing(rg_ctx* ctx, int on);
/* With rg_set_timing(ctx, 2) every level step (rg_godunov_level and the level
 * steps inside rg_amr_coarse_step) records its own events: this returns the
 * summed device milliseconds of its three phases (ms[0] primitives, ms[1]
 * face kernel, ms[2] fold), the cells the face kernels processed and the
 * number of level steps since the last reset (reset != 0 clears them).
 * Synchronises the context stream.  No reference counterpart. */
int rg_kernel_ms_totals(rg_ctx* ctx, double* ms, int64_t* cells, int64_t* steps, int reset);
/* Exact-solver statistics accumulated by the face kernels: Newton updates
 * and Riemann solves since the last reset (reset != 0 clears them). */
int rg_exact_stats(rg_ctx* ctx, int64_t* iters, int64_t* calls, int reset);
/* The face kernel's launch shape (tiles per block, register cap, batch of
 * tiles per queue grab) is timed on the first substep of each level of 2^17
 * cells or more and the fastest kept; a smaller 3-D level takes the default
 * shape, or, when its tiles of 32 cells outnumber the default's 8 resident
 * blocks per SM, the one with 9 or 10 that holds them in one wave.  on == 0
 * keeps the default shape. */
int rg_set_autotune(rg_ctx* ctx, int on);
/* ---- ensembles of independent boxes (no reference counterpart) ----------
 * Many independent periodic boxes, each a uniform grid the reference would
 * run as its own simulation, stepped together: the host merges their trees
 * into one forest whose level list `ilevel` chains every box's leaf octs,
 * box after box (so each box keeps the oct order, hence the update order, it
 * has alone), and tells the library which list positions belong to which
 * box.  rg_level_substep then computes one CFL step per box (the reference
 * formula with that box's dx) and advances every box by its own dt in the
 * same launches.  first_oct[nbox+1]: box b owns level-list positions
 * [first_oct[b], first_oct[b+1]); dx[nbox]: the dx the reference passes for
 * that box's level (boxlen / (nx 2^level)).  The level must have no refined
 * cell.  The table is dropped when rg_sync_topology rebuilds the plans.
 * rg_godunov_level, rg_courant_step and the allocation-free entry point
 * refuse a level with boxes (they take one dt for the whole level). */
int rg_set_level_boxes(rg_ctx* ctx, int ilevel, int nbox, const int* first_oct, const double* dx);
/* Optional, after rg_set_level_boxes: each box is one periodic lattice of
 * extent[3b..3b+2] cells (multiples of 8); lat_id / lat_p give, for every
 * site of every box (box after box, x fastest), its cell id and its position
 * p = (ic-1)*noct + k in the level (k = position of its oct in the level
 * list).  The library checks every site against the level's neighbours,
 * ghost stencils and interface kinds before it uses the brick face kernel on
 * the boxes; a mismatch returns RG_ERR_ARG and changes nothing. */
int rg_set_level_lattices(rg_ctx* ctx, int ilevel, int nbox, const int* extent, const int* lat_id,
                          const int* lat_p);
/* dt of every box in the last substep (nbox must equal the level's count);
 * rg_level_substep's dt_used reports the smallest of them. */
int rg_level_box_dt(rg_ctx* ctx, int ilevel, double* dt_out, int nbox);

/* No reference counterpart, measurement only: the device's FP64 throughput
 * in TFLOP/s (independent fused multiply-add chains on every SM, best of 5
 * timed launches), the peak the face kernel's compute roofline is reported
 * against. */
int rg_measure_fp64_peak(rg_ctx* ctx, double* tflops);

/* Shape chosen for a level: variant index, batch, and its timed ms. */
int rg_face_config(rg_ctx* ctx, int ilevel, int* variant, int* batch, float* ms);
/* Pin the face-kernel shape of a level (variant 0..10, batch >= 1; 7 and 8
 * select the software-pipelined kernel on levels above level 0 in 2D/3D,
 * 9 and 10 the brick kernel on levels that form one complete periodic
 * lattice; elsewhere those ids run the default shape). */
int rg_set_face_config(rg_ctx* ctx, int ilevel, int variant, int batch);

/* ---- device-resident tree maintenance (TreeUpdater on the GPU) -------------
 * The reference rebuilds its AMR tree on the host between hydro steps
 * (TreeUpdater, src/core/TreeUpdater.cpp:27-636).  After rg_tree_attach the
 * tree lives on the device and these calls replace the TreeUpdater methods
 * of the same names with the same arguments and the same results, bit for
 * bit (flags, oct ids from the FIFO free list, level and free-list links,
 * coordinates, prolonged and restricted states), so a whole coarse step
 * (Simulation::amr_step, src/core/Simulation.cpp:522-635) runs without the
 * host touching the tree.  Scope: 3D hydro (nvar 5), ncpu 1, no boundary
 * patches, levels above the coarse level (ilevel >= 2; the coarse level is
 * refined at initialisation, on the host).  When make_grid_fine needs more
 * octs than the free list holds, ngridmax doubles (as often as needed) with
 * the reference's relayout of every array (AmrGrid::resize_grids,
 * AmrGrid.cpp:117-248, called from get_free_grid, :259-261): ncell and the
 * cell ids change, so size the host arrays by rg_tree_sizes before
 * rg_tree_fetch or rg_download_state.  Not reproduced: the debug printf of
 * each flagged cell (TreeUpdater.cpp:519). */
typedef struct rg_tree_arrays {
    int* son;      /* [ncell]      (rg_tree_fetch writes; attach reads the grid view's) */
    int* father;   /* [ngridmax]                                                      */
    int* nbor;     /* [6*ngridmax]                                                    */
    int* next;     /* [ngridmax]                                                      */
    int* prev;     /* [ngridmax]   AmrGrid::prev                                      */
    int* headl;    /* [(ncpu+nboundary)*(nlevelmax+1)] headl_vec                      */
    int* taill;    /* same shape: taill_vec                                           */
    int* numbl;    /* same shape: numbl_vec                                           */
    int* flag1;    /* [ncell]                                                         */
    int* flag2;    /* [ncell]                                                         */
    int* cpu_map;  /* [ncell]                                                         */
    double* xg;    /* [3*ngridmax] oct centres                                        */
    double* uold;  /* [nvar*ncell]                                                    */
    double* unew;  /* [nvar*ncell]                                                    */
    int headf, tailf, numbf; /* AmrGrid free list                                     */
} rg_tree_arrays;
/* Take over the tree: rg_sync_topology(g) plus the state and every other
 * tree array of t (its son/father/nbor/next/headl are not read: the view's
 * are).  levelmin: amr_params/levelmin, read by flag_fine.  A later
 * rg_sync_topology hands the tree back to the host. */
int rg_tree_attach(rg_ctx* ctx, const rg_grid_view* g, const rg_tree_arrays* t, int levelmin);
/* Copy the device-resident tree and state back into t (NULL arrays are
 * skipped); headf/tailf/numbf are filled in. */
int rg_tree_fetch(rg_ctx* ctx, rg_tree_arrays* t);
/* TreeUpdater::flag_fine (TreeUpdater.cpp:327-575) with its smooth_fine,
 * test_flag and ensure_ref_rules; err_grad_b2 > 0 is RG_ERR_UNSUPPORTED
 * (MHD only).  Neither this call nor rg_restrict_fine waits for the device:
 * a consistency check their kernels fail is returned by the next call that
 * synchronises (rg_make_grid_fine, rg_remove_grid_fine, rg_courant_step,
 * rg_synchronize, ...). */
int rg_flag_fine(rg_ctx* ctx, int ilevel, double err_grad_d, double err_grad_p, double err_grad_u,
                 double err_grad_b2, int nexpand, int icount, int nsubcycle);
/* TreeUpdater::make_grid_fine (TreeUpdater.cpp:27-149): new octs for
 * flagged unrefined cells of level ilevel, state prolonged by interpol_hydro
 * (HydroSolver.cpp:734-876, params.interpol_var / interpol_type). */
int rg_make_grid_fine(rg_ctx* ctx, int ilevel);
/* TreeUpdater::remove_grid_fine (TreeUpdater.cpp:151-186). */
int rg_remove_grid_fine(rg_ctx* ctx, int ilevel);
/* TreeUpdater::restrict_fine (TreeUpdater.cpp:188-207): uold of level
 * ilevel's refined cells from their children. */
int rg_restrict_fine(rg_ctx* ctx, int ilevel);
/* AmrGrid::count_grids_at_level (AmrGrid.cpp:304-308) of the resident tree. */
int rg_count_grids(rg_ctx* ctx, int ilevel, int* n);
/* AmrGrid::ngridmax and ::ncell of the context's tree (they grow when
 * rg_make_grid_fine runs out of free octs).  Either pointer may be NULL. */
int rg_tree_sizes(rg_ctx* ctx, int* ngridmax, int* ncell);

/* One coarse step of the resident run: Simulation::run's step
 * (Simulation.cpp:366-397) with Simulation::amr_step (:522-635), every grid
 * and hydro call on the device, sub-cycling 2 from levelmin on.  The clock
 * carries Simulation's dtnew_/dtold_, time, step count and the hydro cell
 * updates from one call to the next (zero it before the first). */
typedef struct rg_amr_config {
    int levelmin;          /* amr_params/levelmin                                   */
    int nexpand;           /* amr_params/nexpand                                    */
    double courant_factor; /* hydro_params/courant_factor                           */
    double err_grad_d;     /* refine_params; <= 0 switches a criterion off          */
    double err_grad_p;
    double err_grad_u;
    int pressure_cap;      /* 1: compute_courant_step as the reference (p <= 100 rho
                              cap); 0: the same formula without the cap             */
    double boxlen;         /* amr_params/boxlen                                     */
} rg_amr_config;
typedef struct rg_amr_clock {
    double dtnew[33], dtold[33]; /* per level                                          */
    double t;
    int64_t nstep;
    int64_t cell_updates;        /* son == 0 cells processed by godunov_fine           */
} rg_amr_clock;
int rg_amr_coarse_step(rg_ctx* ctx, const rg_amr_config* cfg, rg_amr_clock* clock);
/* No reference counterpart.  Between tree changes rg_amr_coarse_step replays
 * its level steps as CUDA graphs: the segments between two of the host's
 * waits (the change probes) form a run, captured whole at its first visit at
 * a topology (after the plans and other caches it reads are prepared) and
 * replayed until the tree changes.  on > 0 / on == 0 switches
 * that on or off (on < 0 leaves it; the RG_AMR_GRAPHS=0 environment variable
 * sets the initial value off); *captured and *replayed (either may be null)
 * get the context's counts of captured and replayed runs.  Changing the
 * parameters, the face shapes, the autotuning or the network drops the
 * captured runs. */
int rg_amr_graphs(rg_ctx* ctx, int on, int64_t* captured, int64_t* replayed);

#ifdef __cplusplus
}
#endif

#endif /* RGPU_H */
