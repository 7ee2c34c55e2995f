// rg_internal.cuh -- device data model of the B200 Godunov level step.
//
// The host application owns the AmrGrid (RAMSES-CPP include/ramses/core/
// AmrGrid.hpp); the library mirrors the tree and the state in HBM and keeps,
// per refinement level, a "level plan": the integer work of
// HydroSolver::godunov_fine (src/solvers/hydro/HydroSolver.cpp:18-115) done
// once per topology instead of once per call:
//   - the level's oct list in linked-list order (HydroSolver.cpp:43-47),
//     from a pointer-jumping list ranking of next[];
//   - the six neighbour cells of every level cell (AmrGrid::get_nbor_cells,
//     AmrGrid.cpp:402-444) and, per interface, the two neighbours of that
//     neighbour along the interface normal (the ghost-branch stencil,
//     HydroSolver.cpp:179-191);
//   - the interface kind (refined -> zero flux, ghost, same-level, boundary)
//     and whether it refluxes into its neighbour (HydroSolver.cpp:125-162,476);
//   - per target cell, the ordered list of updates it receives (refluxes from
//     neighbours and its own flux-sum update), sorted by the CPU loop key
//     (oct position, ic, idim, side), so the GPU fold applies them in the
//     reference's order without atomics.
// Cell storage index inside a plan: p = (ic-1)*noct + k (k = oct position);
// for fixed ic consecutive k touch consecutive octs, which keeps the state
// reads of a warp coalesced when octs are allocated in list order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <array>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/rgpu.h"

namespace rg {

enum Kind : int8_t { K_NONE = 0, K_ZERO = 1, K_GHOST = 2, K_SAME = 3, K_BOUND = 4 };
constexpr int KIND_MASK = 7;
constexpr int KIND_REFLUX = 8;   // interface refluxes into its neighbour
constexpr int KIND_REFLECT = 16; // boundary branch with btype == 1 (velocity flip)
constexpr int OWN_SLOT = 7;      // event slot of a cell's own update

// device error word: first error wins; info carries an index for the message
enum DevErr : int { DE_NONE = 0, DE_TOPO_CYCLE = 1, DE_LIST = 2, DE_SAME_OUTSIDE = 3, DE_NBOR_DEPTH = 4,
                    DE_EVENT_OVERFLOW = 5, DE_BAD_INDEX = 6 };

struct DevStatus {
    int err;
    int info;
    unsigned long long dtmin_bits;  // CFL min-reduction scratch
    double dt, dx, dtdx;            // values of the current step (read by kernels)
    unsigned long long cell_updates;
    double inv_dx;                  // 1/dx, used only when dx_pow2 != 0
    int dx_pow2;
    unsigned int face_next, face_done;  // persistent face-kernel work queue
    unsigned long long exact_iters, exact_calls;  // exact-solver Newton statistics
    double run_t;                                 // rg_level_run: the level's time and
    long long run_steps;                          // substeps, advanced on the device,
    long long run_limit;                          // and the step count this launch stops at
    unsigned int cfl_done, cfl_pad;               // blocks of a CFL pass done (its clock update)
};

// The resident AMR step's clock update after a level's CFL pass
// (Simulation.cpp:552-554, 600-607): on the device clock ck (dtnew[0..32],
// dtold[0..32], t), dtold = dtnew; dtnew = the CFL word, capped by the
// coarser level's dtnew over its sub-cycles (nsub_coarser > 0 above
// levelmin); the word re-armed at dt_start for the next pass; on a level
// without finer octs the time update follows (finer = 1: no finer octs below
// nlevelmax, the finer level's steps become this one's over its nsub
// sub-cycles; finer = 2 at nlevelmax).  ck == nullptr: no update.
constexpr int kClockLevels = 33, kClockDtOld = kClockLevels, kClockTime = 2 * kClockLevels;
struct ClockStep {
    double* ck = nullptr;
    int il = 0, nsub_coarser = 0, finer = 0, nsub = 1;
    double dt_start = 0.0;
    // set_step: the level's step values (dt, dx, dt/dx) are set from the new
    // dtnew right away (a level whose godunov step follows its CFL pass)
    int set_step = 0;
    double dx = 0.0;
};

// word: the CFL word as the pass left it
__device__ __forceinline__ void clock_step_apply(const ClockStep& cs, DevStatus* st, unsigned long long word) {
    double* ck = cs.ck;
    const int il = cs.il;
    ck[kClockDtOld + il] = ck[il];
    double d = __longlong_as_double((long long)word);
    st->dtmin_bits = (unsigned long long)__double_as_longlong(cs.dt_start);
    if (cs.nsub_coarser > 0) {
        const double cand = ck[il - 1] / (double)cs.nsub_coarser;
        d = cand < d ? cand : d;  // std::min(d, cand)
    }
    ck[il] = d;
    if (cs.finer == 1) {
        const double v = ck[il] / (double)cs.nsub;
        ck[kClockDtOld + il + 1] = v;
        ck[il + 1] = v;
    }
    if (cs.finer) ck[kClockTime] += ck[il];
}

// Step values of one box of an ensemble level (independent periodic boxes
// whose leaf octs share one level list, each with its own dx and CFL step):
// the box's CFL min-reduction word and the values derived from it.
struct BoxStep {
    unsigned long long dtmin_bits;
    double dt, dx, dtdx, inv_dx;
    int dx_pow2, pad;
};

// Read-only view of the mirrored tree handed to kernels.
struct TreeView {
    int ncoarse, ngridmax, ncell, nx, ny, nz;
    int nbound_type;
    const int* son;
    const int* father;
    const int* nbor;
    const int* bound_type;
    const int* cell_level;  // [ncell+1] HydroSolver.cpp:22-38
};

// Per-level plan arrays (device).  NS = 2*ndim interface slots.
struct PlanView {
    int ilevel, level0, noct, ncells, ntarg, nextra_prim;
    const int* octs;       // [noct] (level > 0)
    const int* icn;        // [NS][ncells]
    const int* stc;        // [NS][2][ncells]
    const int8_t* kind;    // [NS][ncells]
    const int* toff;       // [ntarg+1]
    const int* tev;        // [toff[ntarg]] event keys: (cpu_pos*8 + slot)
    const int* textra;     // [ntarg-ncells] cell ids of extra (coarser) targets
    const int* xprim;      // [nextra_prim] cells outside the level needing primitives
    const int* obox;       // [noct] box of each oct position (ensemble levels), else nullptr
    BoxStep* boxes;        // [nbox] per-box step values (ensemble levels), else nullptr
};

// Box of level cell p (ensemble levels only).
__device__ __forceinline__ int box_of(const PlanView& P, int p) { return P.obox[p % P.noct]; }

// A target with more updates than this is folded by a whole warp (fold_long).
constexpr int kLongEvents = 16;

struct Plan {
    bool valid = false;
    int ilevel = -1, level0 = 0, noct = 0, ncells = 0, ntarg = 0, nextra_prim = 0, nevents = 0;
    long long nactive = 0;
    int *octs = nullptr, *icn = nullptr, *stc = nullptr, *toff = nullptr, *tev = nullptr, *textra = nullptr,
        *xprim = nullptr;
    int8_t* kind = nullptr;
    cudaGraphExec_t graph = nullptr;  // substep graph (set_unew..set_uold)
    int graph_cap = -1;
    double graph_dx = 0.0, graph_cfl = 0.0;
    int face_variant = -1, face_batch = 4;  // autotuned face-kernel shape (-1: not tuned yet)
    float face_ms = 0.f;
    int substeps_run = 0;
    int lattice = 0;           // the level is one complete periodic lattice (rg_lattice.cu)
    int lat_e[3] = {0, 0, 0};  // its extent
    int lat_kind = 0;          // the (single) interface kind of its faces
    int* lat_id = nullptr;     // [ex*ey*ez] cell id of each lattice site (x fastest)
    int* lat_p = nullptr;      // [ex*ey*ez] plan position of each site
    // ensemble levels whose boxes are each one periodic lattice: per box its
    // extent, its first site in lat_id/lat_p and its first brick
    int box_lattice = 0;
    int* bl_ext = nullptr;        // [3*nbox]
    int* bl_off = nullptr;        // [nbox]
    int* bl_brick_off = nullptr;  // [nbox+1]
    int bl_nbricks = 0;
    bool ids_ready = false;    // level-sparse host transfer: cell ids read / written
    int* read_ids = nullptr;   // [ncells + nextra_prim] then targ_ids [ntarg] (one allocation)
    int* targ_ids = nullptr;
    std::vector<int> h_read, h_targ;
    std::vector<int> h_cells;  // the level's own cells (the first ncells read ids)
    // the same cells as runs of consecutive cell ids (first id, count): few on
    // a uniform level (one per child slot), so transfers are plain copies
    std::vector<std::pair<int, int>> read_runs, targ_runs, cell_runs;
    // targets with more than kLongEvents updates (coarse cells taking the
    // refluxes of many finer faces), folded one warp each by k_fold's first
    // blocks and skipped by its others
    int nlong = 0;
    int* tlong = nullptr;      // [nlong] target indices
    int nbox = 0;              // ensemble level: number of boxes (0: one grid)
    int* obox = nullptr;       // [noct]
    BoxStep* boxes = nullptr;  // [nbox]
    PlanView view() const {
        return PlanView{ilevel, level0, noct, ncells, ntarg, nextra_prim, octs, icn, stc, kind, toff, tev, textra,
                        xprim, obox, boxes};
    }
};

// Face-kernel shape chosen for a level, kept across plan rebuilds (an AMR run
// rebuilds its plans whenever the tree changes) and reused while the level's
// cell count stays within a factor eight of the one it was tuned on.
struct TunedShape {
    int variant = -1, batch = 1, ncells = 0;
    float ms = 0.f;
};

// A captured run of the resident AMR coarse step (rg_amr.cu: the level-step
// segments between two of the host's waits), valid for the topology version,
// scratch buffers and configuration it was captured with.
struct RunGraph {
    cudaGraphExec_t exec = nullptr;
    long long topo = -1, warm = -1, failed = -1;
    const void* flux = nullptr;
    const void* tscr = nullptr;
    rg_amr_config cfg{};
};

struct Tuning {
    int face_block = 128;
    int face_blocks_per_sm = 0;  // 0 = plain grid covering all work
    int fold_block = 256;
};

}  // namespace rg

struct rg_ctx {
    rg_params params{};
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;      // stream in use
    cudaStream_t own_stream = nullptr;  // created by rg_create
    cudaMemPool_t pool = nullptr;       // every device array of the context (dev_alloc)
    std::string err;
    bool broken = false;

    // mirrored tree
    int ncoarse = 0, ngridmax = 0, ncell = 0, nvar = 0, nx = 1, ny = 1, nz = 1, ncpu = 1, nboundary = 0,
        nlevelmax = 0, nbound_type = 0;
    size_t cap_cell = 0, cap_grid = 0, cap_headl = 0;
    int *d_son = nullptr, *d_father = nullptr, *d_nbor = nullptr, *d_next = nullptr, *d_bound = nullptr;
    int *d_jump = nullptr, *d_dist = nullptr, *d_jump2 = nullptr, *d_dist2 = nullptr;
    int* d_cell_level = nullptr;
    int *d_cpos = nullptr, *d_tmap = nullptr, *d_pmark = nullptr;  // [ncell+1] plan-build scratch
    std::vector<int> h_headl;
    bool have_topology = false, ranked = false;
    long long topo_version = 0;

    // state
    size_t cap_state = 0;
    double *d_uold = nullptr, *d_unew = nullptr, *d_prim = nullptr;
    bool have_state = false;

    // scratch shared by all levels (levels run one after another on the stream)
    size_t cap_flux = 0;
    double* d_flux = nullptr;
    size_t cap_scan = 0;
    int* d_scan = nullptr;

    rg::DevStatus* d_status = nullptr;
    rg::DevStatus* h_status = nullptr;  // pinned mirror

    std::vector<rg::Plan> plans;
    std::vector<rg::TunedShape> tuned;  // per level
    // the CFL word and primitives the last fused fold prepared: valid for the
    // next substep of this level with these arguments, until any call that
    // touches the state or the CFL word
    int next_level = -1, next_cap = 0;
    double next_dx = 0.0, next_cfl = 0.0;
    rg::Tuning tuning;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    float last_ms[3] = {0, 0, 0};
    bool timing = false;
    // rg_set_timing(ctx, 2): every level step (launch_godunov) records its
    // own four events from this pool and its cell count, summed by
    // rg_kernel_ms_totals, so a whole AMR coarse step can be timed per kernel
    bool timing_acc = false;
    std::vector<std::array<cudaEvent_t, 4>> acc_ev;
    std::vector<long long> acc_cells;
    size_t acc_n = 0;
    bool no_autotune = false;
    double* h_stage = nullptr;  // pinned staging of level-sparse host transfers
    size_t cap_hstage = 0;
    double* d_stage = nullptr;
    size_t cap_dstage = 0;
    float* d_mlp = nullptr;  // learned Newton start: parameters + Adam state
    bool mlp_valid = false;
    std::vector<long long> cell_updates;

    // device-resident tree (rg_tree_attach, rg_tree.cu): the arrays only the
    // tree operations need, the free list as a FIFO ring of oct ids (device
    // d_fq, host mirror h_fq, entries fq_head .. fq_head + numbf - 1 modulo
    // ngridmax) and the level lists' tails and counts (heads: h_headl)
    int *d_prev = nullptr, *d_flag1 = nullptr, *d_flag2 = nullptr, *d_cpu_map = nullptr, *d_fq = nullptr;
    double* d_xg = nullptr;
    int* d_tscr = nullptr;  // tree-operation scratch
    size_t cap_tscr = 0;
    std::vector<int> h_taill, h_numbl, h_fq;
    int fq_head = 0, numbf = 0, levelmin = 1;
    bool tree_resident = false;
    // each level's oct list in list order for the tree operations, kept while
    // the topology version it was built at is current (rg_plan.cu
    // level_octs_cached): a coarse step calls the tree operations about 35
    // times on unchanged lists
    std::vector<int*> lvl_octs;
    std::vector<int> lvl_cap, lvl_n;
    std::vector<long long> lvl_ver;
    // rg_amr_coarse_step: the clock buffer (kept so captured graphs can name
    // it) and the captured runs by their index in the coarse step, replayed
    // while the topology is unchanged
    double* d_clock = nullptr;
    // page-locked copy of the clock the device holds (valid when clock_known):
    // a coarse step called with that clock uploads nothing
    double* h_clock = nullptr;
    bool clock_known = false;
    std::map<int, rg::RunGraph> amr_graphs;
    bool amr_graphs_on = true;
    long long amr_captured = 0, amr_replayed = 0;
    bool tree_dirty = false;  // links changed on the device: ranks, cell levels and plans are stale
    // the levels whose plans (bit L) and oct lists a tree change since the
    // last refresh may have changed: the next refresh drops only those (bits
    // above 63 stand for themselves: such levels always count as changed)
    uint64_t plans_dirty = ~0ull, lists_dirty = ~0ull;
    // authorize_fine (flag2 = cpu_map == myid over every cell) has an effect:
    // false while flag2 == (cpu_map == 1) holds everywhere, which only
    // attaching, refining (new cells' cpu_map), removing (freed cells' flag2)
    // and the coarse flags below levelmin (coarse cpu_map) can break
    bool auth_dirty = true;
};

namespace rg {
// host-side helpers shared by the translation units
int set_error(rg_ctx* c, int code, const std::string& msg);
int check_cuda(rg_ctx* c, cudaError_t e, const char* what);
int check_device_status(rg_ctx* c);  // synchronises
int build_plan(rg_ctx* c, int ilevel, Plan& plan);
void free_plan(rg_ctx* c, Plan& plan);
// Device arrays of a context come from its own stream-ordered memory pool:
// allocated and freed in order on the context's stream, freed memory kept by
// the pool for reuse.  Plans are rebuilt after every tree change; plain
// cudaMalloc / cudaFree cost milliseconds per call (a free waits for the whole
// device) with stalls of hundreds of milliseconds under that churn, the pool
// microseconds.
int create_pool(rg_ctx* c);
cudaError_t dev_alloc(rg_ctx* c, void** p, size_t bytes);
template <class T>
cudaError_t dev_alloc(rg_ctx* c, T** p, size_t bytes) {
    return dev_alloc(c, (void**)p, bytes);
}
void dev_free(rg_ctx* c, void* p);
int rank_lists(rg_ctx* c);
// Exclusive scan of n ints on the context stream; *total gets the sum (synchronises).
int exclusive_scan(rg_ctx* c, const int* in, int* out, int n, int* total);
// the same, enqueue only: the total stays in device memory (*total_dev, or
// the scan scratch when total_dev is null; *total_at gets where)
int exclusive_scan_dev(rg_ctx* c, const int* in, int* out, int n, int* total_dev, int** total_at = nullptr);
// Octs of level list `ilevel` in linked-list order, from the list ranks, into the
// device array out[cap]; *noct gets the count (synchronises).
int level_oct_list(rg_ctx* c, int ilevel, int* out, int cap, int* noct);
// The same list of a device-resident tree from a per-level cache, rebuilt
// only when the topology changed since it was built; *octs stays valid until
// the next tree change.
int level_octs_cached(rg_ctx* c, int ilevel, const int** octs, int* noct);
// what a level step needs before it can be captured: the plan, the flux
// scratch, the face shape of a level too small to be timed (*ready becomes
// false, nothing else done, for a level whose shape waits for timing or an
// ensemble level)
int prepare_level_step(rg_ctx* c, int ilevel, bool* ready);
// after device tree operations changed links: drop plans, re-rank the lists,
// recompute cell levels (no-op when nothing changed)
int refresh_tree(rg_ctx* c);
// rg_level_run on a level of at most kRunBlockCells cells (two per thread of
// the block): the whole loop in one single-block kernel (rg_step.cu); the clock
// in DevStatus run_t/run_steps.  Larger levels are faster spread over the GPU.
constexpr int kRunBlockCells = 1024;
int launch_run_block(rg_ctx* c, const Plan& P, double dx, int pressure_cap, double t_end, long long max_steps);
// TreeUpdater operations on the device-resident tree (rg_tree.cu)
int tree_flag_fine(rg_ctx* c, int ilevel, double ed, double ep, double ev, double eb2, int nexp, int icount,
                   int nsub);
// `changed` (optional): the number of octs created / freed
int tree_make_grid_fine(rg_ctx* c, int ilevel, int* changed = nullptr);
int tree_remove_grid_fine(rg_ctx* c, int ilevel, int* changed = nullptr);
int tree_restrict_fine(rg_ctx* c, int ilevel);
// flag_fine(il) for il = lmin-1..1 and, with `restrictions`, restrict_fine(il)
// for il = lmin-1..0 as two launches; *done false when not applicable
int tree_tail_below_min(rg_ctx* c, int lmin, bool restrictions, bool* done);
// Which of make_grid_fine(L) and remove_grid_fine(L), for the levels L whose
// bit is set in `levels` (bit L; L = 1 is the coarse cells, which only
// make_grid_fine looks at), can change the resident tree?  One pass over those
// levels (after the authorisation the first make_grid_fine would run) and one
// read-back.  Bit L of `refine` is clear when no cell of level list L is a
// refinement candidate, bit L of `kill` when no oct of it is a removal
// candidate; bits of levels not probed stay set.  A clear bit holds until a
// call changes the tree: make_grid_fine(L) can make cells of list L + 1
// candidates (the new octs' cells keep the flags their slots held), and
// remove_grid_fine(L + 1) octs of list L.
struct TreeChanges {
    uint64_t refine = ~0ull, kill = ~0ull;
    bool any(uint64_t levels) const { return ((refine | kill) & levels) != 0; }
};
int tree_changes_pending(rg_ctx* c, uint64_t levels, TreeChanges* out);
inline uint64_t level_bits(int lo, int hi) {  // bits lo..hi, 1 <= lo, hi <= 63
    uint64_t m = 0;
    for (int L = lo < 1 ? 1 : lo; L <= hi && L <= 63; ++L) m |= 1ull << L;
    return m;
}
Plan* existing_plan(rg_ctx* c, int ilevel);  // built plan or nullptr; never builds
// forget the captured AMR coarse-step runs (they bake in the solver constants,
// face shapes and network pointer)
void drop_amr_graphs(rg_ctx* c);
int compute_cell_levels(rg_ctx* c);
// step launchers (enqueue only)
int launch_set_unew(rg_ctx* c, const Plan& p);
int launch_set_uold(rg_ctx* c, const Plan& p);
// set_unew: also HydroSolver::set_unew of the level in the same pass;
// armed: the CFL word already holds its start value (no arming launch)
// clock (optional): the AMR clock update, done by the pass's last block
// with_prim: the pass also writes the primitives of the level's cells and its
// extra (ghost-stencil) cells, the godunov step's first pass
int launch_courant(rg_ctx* c, const Plan& p, double dx, int pressure_cap, double courant_factor,
                   bool set_unew = false, bool armed = false, const ClockStep* clock = nullptr, bool with_prim = false);
// the step values (dt, dt/dx, 1/dx) from a dt in device memory
int launch_set_dt_device(rg_ctx* c, const double* dt, double dx);
// rg_courant_step without reading the step back: the CFL word holds it
int courant_step_device(rg_ctx* c, int ilevel, double dx, double courant_factor, int pressure_cap,
                        bool set_unew = false, bool armed = false, const ClockStep* clock = nullptr,
                        bool with_prim = false);
// rg_godunov_level with its dt read by the device from dt_dev
// set_uold: HydroSolver::set_uold of the level folded into the fold kernels
// prim_ready: the primitives and step values are in place (the CFL pass with
// with_prim and set_step), so the primitive pass is not launched
int godunov_level_device_dt(rg_ctx* c, int ilevel, const double* dt_dev, double dx, bool set_uold = false,
                            bool prim_ready = false);
int launch_set_dt_host(rg_ctx* c, double dt, double dx);
int launch_finalize_dt(rg_ctx* c, double dx);
// dt_dev != nullptr: the primitive pass also sets the step values from it
int launch_godunov(rg_ctx* c, const Plan& p, bool set_uold = false, const double* dt_dev = nullptr,
                   double dx = 0.0, bool prim_ready = false);
// the four events a level step records its kernel boundaries into: the
// context's last-call set, or in accumulating mode the next set of the pool
cudaEvent_t* step_events(rg_ctx* c, long long ncells);
int launch_leaf_prefix(rg_ctx* c, const Plan& p, double dx, int pressure_cap, double courant_factor);
int launch_leaf_core(rg_ctx* c, const Plan& p, double dx, int pressure_cap, double courant_factor);
// a leaf level whose stencils and updates stay inside it: its fold can prepare
// the next substep
inline bool leaf_fusable(const Plan& P) { return P.nextra_prim == 0 && P.ntarg == P.ncells && !P.level0; }
int launch_godunov_ext(rg_ctx* c, const Plan& p, const double* uold, double* unew, double* prim, double* flux);
TreeView tree_view(const rg_ctx* c);
void remember_shape(rg_ctx* c, const Plan& P);
int build_lattice(rg_ctx* c, Plan& P);
int launch_level_output(rg_ctx* c, const Plan& P, double* out_dev);
int set_box_lattices(rg_ctx* c, Plan& P, const int* ext, const int* lat_id, const int* lat_p);
// unew may be null (only uold's read cells are uploaded)
int upload_level_host(rg_ctx* c, Plan& P, const double* uold, const double* unew);
// the level's targets of src_dev (default: the device unew) into host array dst
int download_level_host(rg_ctx* c, Plan& P, double* dst, const double* src_dev = nullptr);
// every cell of the level (refined ones too) of the device uold / unew into
// host arrays (either may be null); synchronises
int download_level_cells(rg_ctx* c, Plan& P, double* uold, double* unew);
int mlp_ensure(rg_ctx* c);
int mlp_train(rg_ctx* c, int nsamples, int epochs, int batch, float lr, unsigned long long seed, float* loss_out);
int mlp_grad(rg_ctx* c, int n, const float* x_host, const float* t_host, float* grad_host, float* loss_host);
int launch_exact_batch(rg_ctx* c, int n, const double* ql, const double* qr, const double* gam, double* flux,
                       double* pstar, int* iters, const float* mlp, int niter, double tol);
int launch_stress_states(rg_ctx* c, int n, unsigned long long seed, double* ql, double* qr, double* gam);
}  // namespace rg
