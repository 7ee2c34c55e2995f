"""GPU level step (librgpu.so through its C ABI) against the oracle and the
reference's golden vectors.  Bit-exact for integer work and for the
HLLC/HLL/LLF/acoustic solvers; the exact solver differs only through pow()
(CUDA vs glibc) and is held to 3e-12 relative (the path's stated tolerance)."""
import numpy as np
import pytest

import rg_tree
import rgpu
from refsupport import GridArrays, make_params

pytestmark = pytest.mark.gpu

RIEMANN_NAMES = ["llf", "hll", "hllc", "exact", "acoustic"]
EXACT_RTOL = 3e-12


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


def close_rel(a, b, rtol=EXACT_RTOL):
    """|a-b| <= rtol * max(|a|, |b|, floor) per entry; floor avoids 0/0 near zero."""
    scale = np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-300)
    return bool(np.all(np.abs(a - b) <= rtol * scale + 1e-300))


def ga_of(g):
    return GridArrays(ncoarse=g.ncoarse, ngridmax=g.ngridmax, ncell=g.ncell, nvar=g.nvar, nx=g.nx, ny=g.ny,
                      nz=g.nz, ncpu=1, nboundary=0, nlevelmax=g.nlevelmax, son=g.son, father=g.father, nbor=g.nbor,
                      next=g.next, headl=g.headl)


@pytest.fixture(scope="module")
def ctx_factory(rgpu_lib):
    made = []

    def make(params):
        c = rgpu.Context(params, 0)
        made.append(c)
        return c
    yield make
    for c in made:
        c.close()


@pytest.mark.parametrize("riem,slope,itype", [("hllc", 2, 1), ("hllc", 1, 2), ("llf", 8, 3), ("hll", 4, 1),
                                              ("acoustic", 7, 4), ("hllc", 5, 0), ("llf", 6, 1), ("hllc", 0, 2),
                                              ("exact", 2, 1)])
def test_uniform_3d_matches_oracle(ctx_factory, oracle, riem, slope, itype):
    L = 5
    g = rg_tree.build_uniform(3, L)
    ga = ga_of(g)
    params = make_params(3, slope_type=slope, riemann=riem, interpol_type=itype)
    ctx = ctx_factory(params)
    ctx.sync_topology(g)
    uold = rg_tree.random_state(g, L, seed=slope * 11 + itype)
    unew = uold.copy()
    ctx.upload_state(uold, unew)
    dx = 1.0 / 2 ** L
    for step in range(3):
        dt = 0.4 * oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, uold, pressure_cap=False)
        oracle.set_unew(ga, 3, 5, L, uold, unew)
        oracle.godunov_fine(ga, params, L, dt, dx, uold, unew)
        ctx.set_unew(L)
        ctx.godunov_level(L, dt, dx)
        got = np.empty_like(unew)
        ctx.download_state(unew=got)
        if riem == "exact":
            assert close_rel(got, unew), f"step {step}"
            ctx.upload_state(unew=unew)  # continue from the oracle state
        else:
            assert bits_equal(got, unew), f"step {step}: {np.count_nonzero(got != unew)} values differ"
        oracle.set_uold(ga, 3, 5, L, uold, unew)
        ctx.set_uold(L)
    got_old = np.empty_like(uold)
    ctx.download_state(uold=got_old)
    assert close_rel(got_old, uold) if riem == "exact" else bits_equal(got_old, uold)


def test_golden_uniform_cases(ctx_factory, golden):
    d = golden("uniform")
    keys = sorted({k.split("_")[0] for k in d.files})
    for key in keys:
        ndim, L, slope, riem, itype = (int(x) for x in d[f"{key}_meta"])
        g = rg_tree.build_uniform(ndim, L)
        params = make_params(ndim, slope_type=slope, riemann=RIEMANN_NAMES[riem], interpol_type=itype)
        ctx = ctx_factory(params)
        ctx.sync_topology(g)
        dt, dx = (float(x) for x in d[f"{key}_dtdx"])
        u0 = d[f"{key}_uold"]
        ctx.upload_state(u0, u0)
        ctx.godunov_level(L, dt, dx)
        got = np.empty_like(u0)
        ctx.download_state(unew=got)
        want = d[f"{key}_unew"]
        if RIEMANN_NAMES[riem] == "exact":
            assert close_rel(got, want), key
        else:
            assert bits_equal(got, want), key


@pytest.mark.parametrize("fixture,variant", [("amr3d", None), ("amr1d", None), ("amr3d", 7), ("amr3d", 8),
                                             ("amr1d", 7)])
def test_golden_amr_calls(ctx_factory, golden, fixture, variant):
    """godunov_fine calls recorded from a sub-cycled AMR run of the reference:
    coarse-fine ghost states and reflux into coarser cells, bit-exact; also
    with the software-pipelined face kernel forced on every level (its
    coarse-fine faces load the neighbour's inner stencil cell directly)."""
    d = golden(fixture)
    ndim, slope, riem = (int(x) for x in d["params"])
    params = make_params(ndim, slope_type=slope, riemann=RIEMANN_NAMES[riem])
    for k in sorted({k.split("_")[0] for k in d.files if k.startswith("L")}):
        ncoarse, ngm, ncell, nvar, nx, ny, nz, nlevelmax, il = (int(x) for x in d[f"{k}_meta"])
        g = GridArrays(ncoarse=ncoarse, ngridmax=ngm, ncell=ncell, nvar=nvar, nx=nx, ny=ny, nz=nz, ncpu=1,
                       nboundary=0, nlevelmax=nlevelmax, son=d[f"{k}_son"], father=d[f"{k}_father"],
                       nbor=d[f"{k}_nbor"], next=d[f"{k}_next"], headl=d[f"{k}_headl"])
        ctx = ctx_factory(params)
        ctx.sync_topology(g)
        dt, dx = (float(x) for x in d[f"{k}_dtdx"])
        if variant is not None:
            ctx.set_face_config(il, variant, 1)
        ctx.upload_state(d[f"{k}_uold"], d[f"{k}_unew_in"])
        ctx.godunov_level(il, dt, dx)
        got = np.empty(nvar * ncell)
        ctx.download_state(unew=got)
        assert bits_equal(got, d[f"{k}_unew_out"]), f"{fixture} {k}: {np.count_nonzero(got != d[f'{k}_unew_out'])}"


@pytest.mark.parametrize("fixture", ["amr3d", "amr1d"])
def test_golden_amr_calls_host_sparse(ctx_factory, golden, fixture):
    """rg_godunov_level_host on host arrays: moves only the cells the step reads
    and writes, gives the reference's bits at the targets and leaves every other
    host value as it was."""
    d = golden(fixture)
    ndim, slope, riem = (int(x) for x in d["params"])
    params = make_params(ndim, slope_type=slope, riemann=RIEMANN_NAMES[riem])
    ctx = ctx_factory(params)
    for k in sorted({k.split("_")[0] for k in d.files if k.startswith("L")}):
        ncoarse, ngm, ncell, nvar, nx, ny, nz, nlevelmax, il = (int(x) for x in d[f"{k}_meta"])
        g = GridArrays(ncoarse=ncoarse, ngridmax=ngm, ncell=ncell, nvar=nvar, nx=nx, ny=ny, nz=nz, ncpu=1,
                       nboundary=0, nlevelmax=nlevelmax, son=d[f"{k}_son"], father=d[f"{k}_father"],
                       nbor=d[f"{k}_nbor"], next=d[f"{k}_next"], headl=d[f"{k}_headl"])
        ctx.sync_topology(g)
        dt, dx = (float(x) for x in d[f"{k}_dtdx"])
        unew = np.array(d[f"{k}_unew_in"], dtype=np.float64)
        ctx.godunov_level_host(il, dt, dx, np.array(d[f"{k}_uold"], dtype=np.float64), unew)
        assert bits_equal(unew, d[f"{k}_unew_out"]), f"{fixture} {k}: {np.count_nonzero(unew != d[f'{k}_unew_out'])}"


def test_level_index_matches_oracle(ctx_factory, oracle, golden):
    """Oct order (level linked list) and neighbour cells (get_nbor_cells): exact."""
    d = golden("amr3d")
    for k in ("L3", "L4", "L5"):
        ncoarse, ngm, ncell, nvar, nx, ny, nz, nlevelmax, il = (int(x) for x in d[f"{k}_meta"])
        g = GridArrays(ncoarse=ncoarse, ngridmax=ngm, ncell=ncell, nvar=nvar, nx=nx, ny=ny, nz=nz, ncpu=1,
                       nboundary=0, nlevelmax=nlevelmax, son=d[f"{k}_son"], father=d[f"{k}_father"],
                       nbor=d[f"{k}_nbor"], next=d[f"{k}_next"], headl=d[f"{k}_headl"])
        ctx = ctx_factory(make_params(3, slope_type=2, riemann="hllc"))
        ctx.sync_topology(g)
        octs = ctx.level_octs(il)
        assert np.array_equal(octs, g.level_octs(il))
        icn = ctx.level_nbor_cells(il, len(octs) * 8)
        want = np.array([oracle.nbor_cells(g, 3, int(ig), ic) for ig in octs for ic in range(1, 9)])
        assert np.array_equal(icn, want)


def test_courant_matches_oracle(ctx_factory, oracle):
    L = 5
    g = rg_tree.build_uniform(3, L)
    ga = ga_of(g)
    ctx = ctx_factory(make_params(3))
    ctx.sync_topology(g)
    u = rg_tree.random_state(g, L, seed=5, p_range=(-3, 5))
    ctx.upload_state(u, u)
    dx = 1.0 / 2 ** L
    for cap in (True, False):
        assert ctx.courant_step(L, dx, 0.8, cap) == oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, u, pressure_cap=cap)


@pytest.mark.parametrize("use_graph", [False, True])
def test_device_substep_sedov(ctx_factory, oracle, use_graph):
    """rg_level_substep (on-device CFL, set_unew, godunov, set_uold; optionally a
    CUDA graph) against the oracle sequence with the same uncapped CFL."""
    L = 6
    g = rg_tree.build_uniform(3, L)
    ga = ga_of(g)
    params = make_params(3, slope_type=2, riemann="hllc")
    ctx = ctx_factory(params)
    ctx.sync_topology(g)
    uold = rg_tree.sedov_state(g, L)
    unew = uold.copy()
    ctx.upload_state(uold, unew)
    dx = 1.0 / 2 ** L
    for step in range(6):
        dt = oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, uold, pressure_cap=False)
        oracle.set_unew(ga, 3, 5, L, uold, unew)
        oracle.godunov_fine(ga, params, L, dt, dx, uold, unew)
        oracle.set_uold(ga, 3, 5, L, uold, unew)
        dt_gpu = ctx.level_substep(L, dx, pressure_cap=False, use_graph=use_graph, want_dt=True)
        assert dt_gpu == dt, step
    got = np.empty_like(uold)
    ctx.download_state(uold=got)
    assert bits_equal(got, uold)
    assert ctx.cell_updates(L) == 32 ** 3


def test_sod_1d_matches_golden(ctx_factory, golden):
    d = golden("sod1d")
    ndim, L = (int(x) for x in d["meta"])
    g = rg_tree.build_uniform(ndim, L)
    ctx = ctx_factory(make_params(1, slope_type=1, riemann="hllc"))
    ctx.sync_topology(g)
    ctx.upload_state(d["uold0"], d["uold0"])
    dx = 1.0 / 2 ** L
    for dt_ref in d["dts"]:
        dt = ctx.courant_step(L, dx, 0.8, True)
        assert dt == dt_ref
        ctx.set_unew(L)
        ctx.godunov_level(L, dt, dx)
        ctx.set_uold(L)
    got = np.empty_like(d["uold0"])
    ctx.download_state(uold=got)
    assert bits_equal(got, d["uold_final"])


def test_full_size_128_cubed_step_matches_oracle(ctx_factory, oracle):
    """One step at the benchmark size (128^3, reference level 8) from a
    developed Sedov state, bit-exact against the oracle."""
    L = 8
    g = rg_tree.build_uniform(3, L)
    ga = ga_of(g)
    params = make_params(3, slope_type=2, riemann="hllc")
    ctx = ctx_factory(params)
    ctx.sync_topology(g)
    u0 = rg_tree.sedov_state(g, L)
    ctx.upload_state(u0, u0)
    dx = 1.0 / 2 ** L
    for _ in range(10):
        ctx.level_substep(L, dx, pressure_cap=False, use_graph=True)
    uold = np.empty_like(u0)
    unew = np.empty_like(u0)
    ctx.download_state(uold, unew)
    dt = oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, uold, pressure_cap=False)
    assert ctx.level_substep(L, dx, pressure_cap=False, use_graph=True, want_dt=True) == dt
    oracle.set_unew(ga, 3, 5, L, uold, unew)
    oracle.godunov_fine(ga, params, L, dt, dx, uold, unew)
    oracle.set_uold(ga, 3, 5, L, uold, unew)
    got = np.empty_like(u0)
    ctx.download_state(uold=got)
    assert bits_equal(got, uold)


def test_topology_errors_are_reported(ctx_factory):
    """Host-side fault injection: corrupt tree arrays give error codes, and the
    context stays usable afterwards (no device fault)."""
    L = 4
    g = rg_tree.build_uniform(3, L)
    ctx = ctx_factory(make_params(3))
    bad = rg_tree.build_uniform(3, L)
    octs = bad.level_octs[L]
    bad.next[octs[-1] - 1] = octs[0]  # the level list becomes a cycle
    with pytest.raises(rgpu.RGError) as e:
        ctx.sync_topology(bad)
    assert e.value.code == rgpu.RG_ERR_TOPOLOGY
    ctx.sync_topology(g)
    with pytest.raises(rgpu.RGError) as e:
        ctx.godunov_level(L, 1e-3, 1.0 / 2 ** L)
    assert e.value.code == rgpu.RG_ERR_STATE
    u = rg_tree.random_state(g, L)
    ctx.upload_state(u, u)
    with pytest.raises(rgpu.RGError) as e:
        ctx.godunov_level(L + 5, 1e-3, 0.1)
    assert e.value.code == rgpu.RG_ERR_ARG
    ctx.godunov_level(L, 1e-3, 1.0 / 2 ** L)
    ctx.synchronize()


@pytest.mark.parametrize("variant", list(range(11)))
def test_every_face_kernel_shape_is_bit_identical(ctx_factory, oracle, variant):
    """The autotuner may pick any shape: each must give the oracle's bits."""
    L = 5
    g = rg_tree.build_uniform(3, L)
    ga = ga_of(g)
    params = make_params(3, slope_type=2, riemann="hllc")
    ctx = ctx_factory(params)
    ctx.sync_topology(g)
    u = rg_tree.random_state(g, L, seed=variant)
    want = u.copy()
    dx = 1.0 / 2 ** L
    dt = 0.3 * oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, u, pressure_cap=False)
    oracle.godunov_fine(ga, params, L, dt, dx, u.copy(), want)
    for batch in (1, 3, 16):
        ctx.set_face_config(L, variant, batch)
        ctx.upload_state(u, u)
        ctx.godunov_level(L, dt, dx)
        got = np.empty_like(u)
        ctx.download_state(unew=got)
        assert bits_equal(got, want), (variant, batch)


def test_autotuner_picks_a_shape_and_exact_stats_count(ctx_factory):
    L = 7  # 64^3 = 2^18 cells: timed (levels below 2^17 cells are not)
    g = rg_tree.build_uniform(3, L)
    ctx = ctx_factory(make_params(3, slope_type=2, riemann="exact"))
    ctx.sync_topology(g)
    u = rg_tree.sedov_state(g, L)
    ctx.upload_state(u, u)
    dx = 1.0 / 2 ** L
    ctx.level_substep(L, dx, use_graph=True)  # eager first substep + autotune
    v, b, ms = ctx.face_config(L)
    assert 0 <= v <= 10 and b >= 1 and ms > 0
    ctx.exact_stats(reset=True)
    ctx.level_substep(L, dx, use_graph=True)
    ctx.synchronize()
    iters, calls = ctx.exact_stats()
    assert calls == 6 * 64 ** 3 and iters >= calls


def test_empty_level_is_a_no_op(ctx_factory):
    """A level list with no octs (headl = 0): every entry point returns OK and
    leaves the state as it was."""
    g = rg_tree.build_uniform(3, 4, nlevelmax=6)
    ctx = ctx_factory(make_params(3, slope_type=2, riemann="hllc"))
    ctx.sync_topology(g)
    u = rg_tree.random_state(g, 4, seed=3)
    ctx.upload_state(u, u)
    for il in (5, 6):
        ctx.set_unew(il)
        ctx.godunov_level(il, 1e-3, 1.0 / 2 ** il)
        ctx.set_uold(il)
        ctx.level_substep(il, 1.0 / 2 ** il, use_graph=False)
        unew = u.copy()
        ctx.godunov_level_host(il, 1e-3, 1.0 / 2 ** il, u, unew)
        assert bits_equal(unew, u)
        assert ctx.cell_updates(il) == 0
    a, b = np.empty_like(u), np.empty_like(u)
    ctx.download_state(uold=a, unew=b)
    assert bits_equal(a, u) and bits_equal(b, u)


@pytest.mark.parametrize("variant", [1, 9])
def test_nx3_grid_with_non_power_of_two_dx(ctx_factory, oracle, variant):
    """3x3x3 coarse cells refined to 24^3 (dx = 1/48, not a power of two: true
    divisions in the slopes and traces); tiled and brick kernels."""
    L = 4
    g = rg_tree.build_uniform(3, L, nx=3, ny=3, nz=3)
    ga = ga_of(g)
    params = make_params(3, slope_type=2, riemann="hllc")
    ctx = ctx_factory(params)
    ctx.sync_topology(g)
    u = rg_tree.random_state(g, L, seed=21)
    dx = 1.0 / (3 * 2 ** L)
    dt = 0.3 * oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, u, pressure_cap=False)
    want = u.copy()
    oracle.godunov_fine(ga, params, L, dt, dx, u.copy(), want)
    ctx.set_face_config(L, variant, 1)
    ctx.upload_state(u, u)
    ctx.godunov_level(L, dt, dx)
    got = np.empty_like(u)
    ctx.download_state(unew=got)
    assert bits_equal(got, want)
    assert ctx.courant_step(L, dx, 0.8, pressure_cap=False) == oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, u,
                                                                               pressure_cap=False)


@pytest.mark.parametrize("riem,slope,itype", [("llf", 1, 1), ("hll", 8, 3), ("hllc", 2, 2), ("acoustic", 7, 4),
                                              ("exact", 2, 1), ("hllc", 5, 0)])
def test_brick_kernel_every_solver(ctx_factory, oracle, riem, slope, itype):
    """The brick face kernel (forced) on a 16^3 lattice level, every Riemann
    solver, slope and interpolation family: the oracle's bits (exact: 3e-12)."""
    L = 5
    g = rg_tree.build_uniform(3, L)
    ga = ga_of(g)
    params = make_params(3, slope_type=slope, riemann=riem, interpol_type=itype)
    ctx = ctx_factory(params)
    ctx.sync_topology(g)
    ctx.set_face_config(L, 10, 1)
    u = rg_tree.random_state(g, L, seed=slope * 7 + itype)
    dx = 1.0 / 2 ** L
    dt = 0.4 * oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, u, pressure_cap=False)
    want = u.copy()
    oracle.godunov_fine(ga, params, L, dt, dx, u.copy(), want)
    ctx.upload_state(u, u)
    ctx.godunov_level(L, dt, dx)
    got = np.empty_like(u)
    ctx.download_state(unew=got)
    assert close_rel(got, want) if riem == "exact" else bits_equal(got, want)


def test_substep_sequence_with_interruptions(ctx_factory, oracle):
    """Consecutive substeps reuse the CFL word and primitives the previous fused
    fold prepared; a state upload, a change of the pressure cap, a manual
    godunov_level and graph/eager switches must each be seen (oracle bits and
    dt at every step)."""
    L = 5
    g = rg_tree.build_uniform(3, L)
    ga = ga_of(g)
    params = make_params(3, slope_type=2, riemann="hllc")
    ctx = ctx_factory(params)
    ctx.sync_topology(g)
    uold = rg_tree.sedov_state(g, L)
    unew = uold.copy()
    ctx.upload_state(uold, unew)
    dx = 1.0 / 2 ** L
    plan = [(False, True), (False, True), (False, False), ("upload", None), (False, True), (True, True),
            (True, False), (False, True), ("godunov", None), (False, True), (False, False)]
    for step, (cap, graph) in enumerate(plan):
        if cap == "upload":
            uold = rg_tree.random_state(g, L, seed=step)
            unew = uold.copy()
            ctx.upload_state(uold, unew)
            continue
        if cap == "godunov":
            # a direct level step between substeps (the reference's godunov_fine)
            dt = 0.5 * oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, uold, pressure_cap=False)
            oracle.godunov_fine(ga, params, L, dt, dx, uold, unew)
            ctx.godunov_level(L, dt, dx)
            continue
        dt = oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, uold, pressure_cap=cap)
        oracle.set_unew(ga, 3, 5, L, uold, unew)
        oracle.godunov_fine(ga, params, L, dt, dx, uold, unew)
        oracle.set_uold(ga, 3, 5, L, uold, unew)
        dt_gpu = ctx.level_substep(L, dx, pressure_cap=cap, use_graph=graph, want_dt=True)
        assert dt_gpu == dt, step
        got = np.empty_like(uold)
        ctx.download_state(uold=got)
        assert bits_equal(got, uold), step


@pytest.mark.parametrize("key", ["L3", "L4", "L5"])
def test_substep_on_amr_levels(ctx_factory, oracle, golden, key):
    """rg_level_substep on the levels of a sub-cycled AMR tree (coarse levels
    with refined cells take the unfused path: CFL, set_unew, godunov_fine,
    set_uold; the finest level the leaf path), two substeps each, against the
    oracle's sequence with the same uncapped CFL."""
    d = golden("amr3d")
    ndim, slope, riem = (int(x) for x in d["params"])
    params = make_params(ndim, slope_type=slope, riemann=RIEMANN_NAMES[riem])
    ncoarse, ngm, ncell, nvar, nx, ny, nz, nlevelmax, il = (int(x) for x in d[f"{key}_meta"])
    g = GridArrays(ncoarse=ncoarse, ngridmax=ngm, ncell=ncell, nvar=nvar, nx=nx, ny=ny, nz=nz, ncpu=1,
                   nboundary=0, nlevelmax=nlevelmax, son=d[f"{key}_son"], father=d[f"{key}_father"],
                   nbor=d[f"{key}_nbor"], next=d[f"{key}_next"], headl=d[f"{key}_headl"])
    ctx = ctx_factory(params)
    ctx.sync_topology(g)
    uold = np.array(d[f"{key}_uold"], dtype=np.float64)
    unew = np.array(d[f"{key}_unew_in"], dtype=np.float64)
    ctx.upload_state(uold, unew)
    dx = 1.0 / (nx * 2 ** il)
    for step in range(2):
        dt = oracle.courant(g, ndim, nvar, il, dx, 1.4, 0.8, uold, pressure_cap=False)
        oracle.set_unew(g, ndim, nvar, il, uold, unew)
        oracle.godunov_fine(g, params, il, dt, dx, uold, unew)
        oracle.set_uold(g, ndim, nvar, il, uold, unew)
        dt_gpu = ctx.level_substep(il, dx, pressure_cap=False, use_graph=(step == 1), want_dt=True)
        assert dt_gpu == dt, (key, step)
    a, b = np.empty_like(uold), np.empty_like(unew)
    ctx.download_state(uold=a, unew=b)
    assert bits_equal(a, uold) and bits_equal(b, unew)


@pytest.mark.parametrize("memory", ["pageable", "pinned"])
def test_host_substeps_move_only_the_level(ctx_factory, oracle, memory):
    """rg_level_substep_host on a host array: oracle bits and dt each substep,
    and cells outside the level (the coarse levels) keep their host values.
    pageable: numpy arrays (gathered run by run into pinned staging); pinned:
    page-locked arrays (one DMA per run of consecutive cell ids)."""
    L = 5
    g = rg_tree.build_uniform(3, L)
    ga = ga_of(g)
    params = make_params(3, slope_type=2, riemann="hllc")
    ctx = ctx_factory(params)
    ctx.sync_topology(g)
    uold = rg_tree.sedov_state(g, L)
    unew = uold.copy()
    if memory == "pinned":
        torch = pytest.importorskip("torch")
        t_host = torch.from_numpy(uold.copy()).pin_memory()
        t_unew = torch.full((uold.size,), 7.0, dtype=torch.float64).pin_memory()
        host, host_unew = t_host.numpy(), t_unew.numpy()  # views of the page-locked buffers
    else:
        host = uold.copy()
        host_unew = np.full_like(uold, 7.0)
    outside = np.setdiff1d(np.arange(1, g.ncell + 1), g.cell_ids(L))
    before = host.reshape(5, -1)[:, outside - 1].copy()
    dx = 1.0 / 2 ** L
    for step in range(3):
        dt = oracle.courant(ga, 3, 5, L, dx, 1.4, 0.8, uold, pressure_cap=False)
        oracle.set_unew(ga, 3, 5, L, uold, unew)
        oracle.godunov_fine(ga, params, L, dt, dx, uold, unew)
        oracle.set_uold(ga, 3, 5, L, uold, unew)
        dt_gpu = ctx.level_substep_host_ptr(L, dx, host.ctypes.data, host_unew.ctypes.data)
        assert dt_gpu == dt, step
        ids = g.cell_ids(L)
        assert bits_equal(host.reshape(5, -1)[:, ids - 1], uold.reshape(5, -1)[:, ids - 1]), step
        assert bits_equal(host_unew.reshape(5, -1)[:, ids - 1], unew.reshape(5, -1)[:, ids - 1]), step
    assert bits_equal(host.reshape(5, -1)[:, outside - 1], before)
    assert np.all(host_unew.reshape(5, -1)[:, outside - 1] == 7.0)


@pytest.mark.parametrize("case", ["sod1d", "sedov3d_small", "sedov3d"])
def test_level_run_matches_host_loop(ctx_factory, case):
    """rg_level_run against the host loop `while t < t_end: t += level_substep()`:
    same state bits, same time, same step count.  sod1d (1024 cells, the Sod
    run of config 1 to t = 0.245) and sedov3d_small (8^3 = 512 cells) take the
    single-block kernel; sedov3d (32^3) the graph with a device-side WHILE loop."""
    if case == "sedov3d_small":
        ndim, L, params, cap, t_end = 3, 3, make_params(3, slope_type=2, riemann="hllc"), False, 0.3
        g = rg_tree.build_uniform(3, L)
        u0 = rg_tree.sedov_state(g, L)
    elif case == "sod1d":
        ndim, L, params, cap, t_end = 1, 11, make_params(1, slope_type=1, riemann="hllc"), True, 0.245
        g = rg_tree.build_uniform(1, L)
        u0 = rg_tree.sod_state(g, L, 1.4)
    else:
        ndim, L, params, cap, t_end = 3, 5, make_params(3, slope_type=2, riemann="hllc"), False, 1.5e-2
        g = rg_tree.build_uniform(3, L)
        u0 = rg_tree.sedov_state(g, L)
    dx = 1.0 / 2 ** L
    out = []
    for mode in ("host", "run"):
        ctx = ctx_factory(params)
        ctx.sync_topology(g)
        ctx.upload_state(u0, u0)
        if mode == "host":
            t, n = 0.0, 0
            while t < t_end:
                t += ctx.level_substep(L, dx, pressure_cap=cap, use_graph=True, want_dt=True)
                n += 1
        else:
            t, n = ctx.level_run(L, dx, t_end, pressure_cap=cap)
        u = np.empty_like(u0)
        ctx.download_state(uold=u)
        out.append((t, n, u))
    (t0, n0, u0h), (t1, n1, u1) = out
    assert n0 > 10 and n1 == n0 and t1 == t0
    assert bits_equal(u1, u0h)


def test_level_run_stops_at_max_steps(ctx_factory):
    L = 11
    g = rg_tree.build_uniform(1, L)
    u0 = rg_tree.sod_state(g, L, 1.4)
    ctx = ctx_factory(make_params(1, slope_type=1, riemann="hllc"))
    ctx.sync_topology(g)
    ctx.upload_state(u0, u0)
    t, n = ctx.level_run(L, 1.0 / 2 ** L, 10.0, pressure_cap=True, max_steps=37)
    assert n == 37 and 0.0 < t < 10.0
    t2, n2 = ctx.level_run(L, 1.0 / 2 ** L, 10.0, t_start=t, pressure_cap=True, max_steps=3)
    assert n2 == 3 and t2 > t
    assert ctx.level_run(L, 1.0 / 2 ** L, 0.0, t_start=1.0) == (1.0, 0)  # t_start >= t_end: no substep


def test_fp64_peak_probe(ctx_factory):
    """rg_measure_fp64_peak: the FP64 throughput the face kernel's compute
    roofline is reported against; a B200 lands in the tens of TFLOP/s."""
    ctx = ctx_factory(make_params(3))
    v = ctx.measure_fp64_peak()
    assert 5.0 < v < 200.0, v
