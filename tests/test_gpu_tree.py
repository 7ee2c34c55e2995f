"""AMR tree maintenance on the GPU (rg_tree.cu) against the reference's own
TreeUpdater (src/core/TreeUpdater.cpp), run through the compiled reference
harness on the same tree.

- every operation, level by level, on a sub-cycled Sedov tree after a coarse
  step: flag_fine (with smooth_fine, test_flag and ensure_ref_rules),
  make_grid_fine (oct ids from the FIFO free list, neighbours, coordinates,
  interpol_hydro for each interpol_var), remove_grid_fine (unlinking, freed
  ids appended to the free list) and restrict_fine: every tree array, the
  list heads / tails / counts, the free list and the state equal bit for bit;
- a run that outgrows its free list: ngridmax doubled and every array
  relabelled as the reference's resize_grids does;
- whole coarse steps with the tree resident on the device (rg_amr.DeviceAmrRun,
  through the native rg_amr_coarse_step and call by call) against the
  reference's run (refsupport.AmrRun): same tree, same state, same time, same
  cell-update count after each step.
"""
import numpy as np
import pytest

import rgpu
from rg_amr import DeviceAmrRun
from refsupport import AmrRun, RefHarness, namelist, sedov_ic

pytestmark = pytest.mark.gpu

LMIN, LMAX, GAMMA, ED, EP = 4, 7, 1.4, 0.1, 0.1


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


def reference_run(steps, interpol_var=0, interpol_type=1):
    nml = namelist(slope_type=2, riemann="hllc", interpol_type=interpol_type, interpol_var=interpol_var,
                   levelmin=LMIN, levelmax=LMAX, err_grad_d=ED, err_grad_p=EP)
    h = RefHarness(3).create(nml, ngridmax=30000, levelmin=LMIN, nlevelmax=LMAX, gamma=GAMMA)
    r = AmrRun(h, LMIN, LMAX, GAMMA, ed=ED, ep=EP)
    r.initialize(sedov_ic(3, LMIN))
    for _ in range(steps):
        r.coarse_step()
    return h, r


def device_ctx(h, interpol_var=0, interpol_type=1):
    params = rgpu.make_params(3, slope_type=2, riemann="hllc", interpol_type=interpol_type,
                              interpol_var=interpol_var, gamma=GAMMA)
    ctx = rgpu.Context(params, 0)
    ctx.tree_attach(h.grid(), h.tree_arrays(), LMIN)
    return ctx


def assert_same_tree(h, ctx, what):
    want = h.tree_arrays()
    got = ctx.tree_fetch(want)
    for k in rgpu.TREE_INT_ARRAYS:
        bad = np.flatnonzero(got[k] != want[k])
        assert bad.size == 0, f"{what}: {k} differs at {bad[:5]} (got {got[k][bad[:5]]}, want {want[k][bad[:5]]})"
    for k in rgpu.TREE_F64_ARRAYS:
        assert bits_equal(got[k], want[k]), f"{what}: {k} differs"
    for k in ("headf", "tailf", "numbf"):
        assert got[k] == want[k], f"{what}: {k} {got[k]} != {want[k]}"


@pytest.mark.parametrize("interpol_var", [0, 1, 2])
def test_each_tree_operation_matches_reference(rgpu_lib, interpol_var):
    itype = 4 if interpol_var == 2 else 1  # type 4 mixes central and moncen slopes
    h, _ = reference_run(1, interpol_var, itype)
    ctx = device_ctx(h, interpol_var, itype)
    try:
        assert_same_tree(h, ctx, "attach")
        made = killed = 0
        for il in range(LMAX, LMIN - 1, -1):
            for icount in (1, 2):
                h.flag_fine(il, ED, EP, -1.0, -1.0, 1, icount, 2)
                ctx.flag_fine(il, ED, EP, -1.0, -1.0, 1, icount, 2)
                assert_same_tree(h, ctx, f"flag_fine({il}, icount={icount})")
        for il in range(LMIN, LMAX + 1):
            n0 = h.count_grids(il + 1)
            h.make_grid_fine(il)
            ctx.make_grid_fine(il)
            made += h.count_grids(il + 1) - n0
            assert_same_tree(h, ctx, f"make_grid_fine({il})")
            assert ctx.count_grids(il + 1) == h.count_grids(il + 1)
        # re-flag each level with thresholds nothing exceeds and without the
        # sub-cycle rules: only fathers of refined octs keep their flags, so the
        # finest octs are removed
        for il in range(LMAX, LMIN, -1):
            h.flag_fine(il - 1, 1e30, 1e30, -1.0, -1.0, 0, 2, 2)
            ctx.flag_fine(il - 1, 1e30, 1e30, -1.0, -1.0, 0, 2, 2)
            n0 = h.count_grids(il)
            h.remove_grid_fine(il)
            ctx.remove_grid_fine(il)
            killed += n0 - h.count_grids(il)
            assert_same_tree(h, ctx, f"remove_grid_fine({il})")
        for il in range(LMAX, -1, -1):
            h.restrict_fine(il)
            ctx.restrict_fine(il)
        assert_same_tree(h, ctx, "restrict_fine")
        assert made > 0, "the sequence refined nothing"
        assert killed > 0, "the sequence removed nothing"
    finally:
        ctx.close()


@pytest.mark.parametrize("native", [True, False])
def test_device_resident_amr_run_matches_reference(rgpu_lib, native):
    """native: rg_amr_coarse_step; else the same sequence call by call."""
    h, r = reference_run(0)
    ctx = device_ctx(h)
    try:
        d = DeviceAmrRun(ctx, nx=1, levelmin=LMIN, nlevelmax=LMAX, ed=ED, ep=EP, native=native)
        headf0 = h.tree_arrays()["headf"]
        for step in range(3):
            r.coarse_step()
            d.coarse_step()
            assert_same_tree(h, ctx, f"coarse step {step}")
            assert d.t == r.t and d.cell_updates == r.cell_updates
        assert sum(h.count_grids(il) for il in range(LMIN + 1, LMAX + 1)) > 0
        assert h.tree_arrays()["headf"] != headf0, "no oct was allocated during the run"
        # the run's folds included targets with more than 16 updates (one warp each)
        assert max(ctx.plan_info(il)["nlong"] for il in range(LMIN, LMAX + 1)) > 0
    finally:
        ctx.close()


def test_tree_calls_report_misuse(rgpu_lib):
    """Errors instead of undefined behaviour: no attached tree, an inconsistent
    free list, and a single-level run on a level that has refined cells."""
    h, _ = reference_run(0)
    params = rgpu.make_params(3, slope_type=2, riemann="hllc", gamma=GAMMA)
    ctx = rgpu.Context(params, 0)
    try:
        with pytest.raises(rgpu.RGError) as e:
            ctx.make_grid_fine(LMIN)
        assert e.value.code == rgpu.RG_ERR_STATE
        bad = dict(h.tree_arrays())
        bad["numbf"] = int(bad["numbf"]) + 1
        with pytest.raises(rgpu.RGError) as e:
            ctx.tree_attach(h.grid(), bad, LMIN)
        assert e.value.code == rgpu.RG_ERR_TOPOLOGY
        ctx.tree_attach(h.grid(), h.tree_arrays(), LMIN)
        with pytest.raises(rgpu.RGError) as e:
            ctx.level_run(LMIN, 1.0 / 2 ** LMIN, 1.0)  # level LMIN has refined cells after initialisation
        assert e.value.code == rgpu.RG_ERR_UNSUPPORTED
        assert ctx.count_grids(LMAX + 5) == 0
    finally:
        ctx.close()


def test_free_list_growth_matches_reference(rgpu_lib):
    """A run whose refinements outgrow the free list.  The reference doubles
    ngridmax in get_free_grid whenever the list runs dry (AmrGrid.cpp:259-261,
    resize_grids :117-248), relabelling every cell id, several times within
    one make_grid_fine here; the device grows the same way, and after each
    coarse step the sizes, every tree array, the free list and the state are
    equal."""
    nml = namelist(slope_type=2, riemann="hllc", levelmin=LMIN, levelmax=LMAX, err_grad_d=ED, err_grad_p=EP)
    probe = RefHarness(3).create(nml, ngridmax=30000, levelmin=LMIN, nlevelmax=LMAX, gamma=GAMMA)
    AmrRun(probe, LMIN, LMAX, GAMMA, ed=ED, ep=EP).initialize(sedov_ic(3, LMIN))
    ngm0 = probe.get("ngridmax") - probe.get("numbf") + 8  # the initialised tree plus 8 free octs
    probe.close()
    h = RefHarness(3).create(nml, ngridmax=ngm0, levelmin=LMIN, nlevelmax=LMAX, gamma=GAMMA)
    r = AmrRun(h, LMIN, LMAX, GAMMA, ed=ED, ep=EP)
    r.initialize(sedov_ic(3, LMIN))
    assert h.get("ngridmax") == ngm0, "the reference grew during initialisation: the case tests nothing"
    ctx = device_ctx(h)
    try:
        d = DeviceAmrRun(ctx, nx=1, levelmin=LMIN, nlevelmax=LMAX, ed=ED, ep=EP)
        for step in range(3):
            r.coarse_step()
            d.coarse_step()
            assert ctx.tree_sizes() == (h.get("ngridmax"), h.get("ncell")), f"coarse step {step}"
            assert_same_tree(h, ctx, f"coarse step {step}")
            assert d.t == r.t and d.cell_updates == r.cell_updates
        assert h.get("ngridmax") >= 4 * ngm0, "the run did not outgrow the free list twice"
    finally:
        ctx.close()
        h.close()


@pytest.mark.parametrize("lmin,lmax,ngm", [(LMIN, LMAX, 30000), (5, 8, 60000)])
def test_device_initialisation_matches_reference(rgpu_lib, lmin, lmax, ngm):
    """rg_amr.initialize: the uniform grid built on the host (rg_tree), then
    Simulation::initialize's rounds (initial condition, flag_fine and
    make_grid_fine of every level, until a level stays empty) by the device
    kernels, against the reference's own initialisation of the same Sedov run:
    every tree array, the free list and the state equal; then two coarse steps
    from each stay equal, time and cell-update counts included."""
    import rg_amr
    nml = namelist(slope_type=2, riemann="hllc", levelmin=lmin, levelmax=lmax, err_grad_d=ED, err_grad_p=EP)
    h = RefHarness(3).create(nml, ngridmax=ngm, levelmin=lmin, nlevelmax=lmax, gamma=GAMMA)
    r = AmrRun(h, lmin, lmax, GAMMA, ed=ED, ep=EP)
    r.initialize(sedov_ic(3, lmin))
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc", interpol_type=1, gamma=GAMMA), 0)
    try:
        rg_amr.initialize(ctx, 3, lmin, lmax, ngm, rg_amr.sedov_primitives(3, lmin, GAMMA), GAMMA, ed=ED, ep=EP)
        assert ctx.tree_sizes() == (h.get("ngridmax"), h.get("ncell"))
        assert_same_tree(h, ctx, "after initialisation")
        d = DeviceAmrRun(ctx, nx=1, levelmin=lmin, nlevelmax=lmax, ed=ED, ep=EP)
        for step in range(2):
            r.coarse_step()
            d.coarse_step()
            assert_same_tree(h, ctx, f"coarse step {step}")
            assert d.t == r.t and d.cell_updates == r.cell_updates
    finally:
        ctx.close()
        h.close()


@pytest.mark.parametrize("graphs", [True, False])
def test_replayed_level_steps_match_reference(rgpu_lib, graphs):
    """Twelve coarse steps at Courant 0.25 (the tree settles, so the native
    step captures its level steps as graphs and replays them between tree
    changes) against the reference after every step; and the same with the
    graphs switched off."""
    nml = namelist(slope_type=2, riemann="hllc", levelmin=LMIN, levelmax=LMAX, err_grad_d=ED, err_grad_p=EP)
    h = RefHarness(3).create(nml, ngridmax=30000, levelmin=LMIN, nlevelmax=LMAX, gamma=GAMMA)
    r = AmrRun(h, LMIN, LMAX, GAMMA, cfl=0.25, ed=ED, ep=EP)
    r.initialize(sedov_ic(3, LMIN))
    ctx = device_ctx(h)
    try:
        ctx.amr_graphs(graphs)
        d = DeviceAmrRun(ctx, nx=1, levelmin=LMIN, nlevelmax=LMAX, cfl=0.25, ed=ED, ep=EP)
        for step in range(12):
            r.coarse_step()
            d.coarse_step()
            assert_same_tree(h, ctx, f"coarse step {step}")
            assert d.t == r.t and d.cell_updates == r.cell_updates
        captured, replayed = ctx.amr_graphs()
        if graphs:
            assert captured > 0 and replayed > 0, (captured, replayed)
        else:
            assert captured == 0 and replayed == 0
    finally:
        ctx.close()


def test_captured_runs_follow_parameter_changes(rgpu_lib):
    """Runs captured as graphs bake in the solver constants and the step's
    configuration: after rg_set_params (here the Riemann solver) and after a
    new Courant factor in the coarse step's configuration, the replayed steps
    must match steps issued eagerly (graphs off) bit for bit."""
    import rg_amr
    out = []
    for graphs in (True, False):
        ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc", gamma=GAMMA), 0)
        try:
            ctx.amr_graphs(graphs)
            rg_amr.initialize(ctx, 3, LMIN, LMAX, 30000, rg_amr.sedov_primitives(3, LMIN, GAMMA), GAMMA, ed=ED, ep=EP)
            d = DeviceAmrRun(ctx, nx=1, levelmin=LMIN, nlevelmax=LMAX, cfl=0.25, ed=ED, ep=EP)
            for _ in range(6):
                d.coarse_step()
            before = ctx.amr_graphs()
            ctx.set_params(rgpu.make_params(3, slope_type=2, riemann="llf", gamma=GAMMA))
            for _ in range(3):
                d.coarse_step()
            d.cfg.courant_factor = 0.2
            for _ in range(3):
                d.coarse_step()
            a = ctx.tree_fetch(level_list_like())
            out.append((a["uold"].copy(), a["son"].copy(), d.t, d.cell_updates, before, ctx.amr_graphs()))
        finally:
            ctx.close()
    (u1, s1, t1, n1, b1, e1), (u2, s2, t2, n2, _, e2) = out
    assert b1[1] > 0, b1  # runs were replayed before the changes
    assert e1[0] > b1[0], (b1, e1)  # and captured again after them
    assert e2 == (0, 0)
    assert t1 == t2 and n1 == n2
    assert np.array_equal(s1, s2) and bits_equal(u1, u2)


def level_list_like():
    """Level-list arrays of the right lengths for Context.tree_fetch on a tree
    that rg_amr.initialize built on the device."""
    import rg_tree
    arrays = rg_tree.tree_arrays(rg_tree.build_uniform(3, LMIN, ngridmax=30000, nlevelmax=LMAX))
    return {k: arrays[k] for k in ("headl", "taill", "numbl")}
