"""rg_godunov_level_noalloc: the level step for callers that may not allocate
device memory after set-up (a committed memory budget, a framework allocator
that owns the free memory, a time loop where cudaMalloc's implicit
synchronisation is not allowed).  Its flux scratch is a static 64 MiB array
inside the library and its state comes from the caller's own device buffers.

Checked through the C ABI against the allocating entry point rg_godunov_level,
bit for bit (the tolerance every parity test of these solvers uses), on two
calls in a row with different states, so the second call also shows that what
the first call left in the shared array does not leak into the result; on a
sub-cycled AMR level whose coarser neighbours take up to ~180 refluxes each
(the warp fold of long targets) with the LLF and the exact solver; and that
the calls allocate nothing: the context's memory pool keeps its reserved and
used bytes, and the device's free memory does not move (after the first call,
which loads the library's kernels and its static array on a lazily loading
runtime).  This file is named to be collected last and creates everything it
uses, so it passes alone in a fresh process as well as after the other
tests."""
import numpy as np
import pytest

import rg_tree
import rgpu

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


def _reference_step(ctx, level, dt, dx, uold, unew):
    ctx.upload_state(uold, unew)
    ctx.godunov_level(level, dt, dx)
    out = np.empty_like(unew)
    ctx.download_state(unew=out)
    return out


def _noalloc_call(torch, ctx, level, dt, dx, uold_dev, unew_dev, check_free):
    """One allocation-free call; asserts the pool and (check_free) the
    device's free memory are the same after it as before."""
    torch.cuda.synchronize()
    pool0 = ctx.pool_usage()
    free0 = torch.cuda.mem_get_info()[0]
    ctx.godunov_level_noalloc(level, dt, dx, uold_dev.data_ptr(), unew_dev.data_ptr())
    ctx.synchronize()
    assert ctx.pool_usage() == pool0, "the context's memory pool changed"
    if check_free:
        assert torch.cuda.mem_get_info()[0] == free0, "device free memory changed across the call"


@pytest.mark.parametrize("ndim,level,riemann,slope", [(3, 5, "hllc", 2), (1, 9, "hllc", 1)])
def test_noalloc_matches_allocating_entry_point_on_two_calls(ndim, level, riemann, slope):
    torch = pytest.importorskip("torch")
    g = rg_tree.build_uniform(ndim, level)
    ctx = rgpu.Context(rgpu.make_params(ndim, slope_type=slope, riemann=riemann), 0)
    try:
        ctx.sync_topology(g)
        dx = 1.0 / 2 ** level
        states = [rg_tree.random_state(g, level, seed=11), rg_tree.sedov_state(g, level)]
        # the first allocating call builds the level plan the allocation-free call needs
        ref = [_reference_step(ctx, level, dt, dx, u, u) for dt, u in zip((2e-4, 3e-7), states)]
        bufs = [torch.from_numpy(u).to("cuda:0") for u in states]
        news = [b.clone() for b in bufs]  # the starting unew: a copy of uold, as rg_set_unew makes it
        for call, dt in enumerate((2e-4, 3e-7)):
            _noalloc_call(torch, ctx, level, dt, dx, bufs[call], news[call], check_free=call > 0)
            got = news[call].cpu().numpy()
            assert bits_equal(got, ref[call]), f"call {call + 1}: {np.count_nonzero(got != ref[call])} values differ"
            assert bits_equal(bufs[call].cpu().numpy(), states[call]), "uold_dev must be read only"
        # a third call on the first state: the device's free memory stays put too
        again = bufs[0].clone()
        _noalloc_call(torch, ctx, level, 2e-4, dx, bufs[0], again, check_free=True)
        assert bits_equal(again.cpu().numpy(), ref[0])
    finally:
        ctx.close()


def _sedov_amr(steps):
    from refsupport import AmrRun, RefHarness, namelist, sedov_ic
    nml = namelist(slope_type=2, riemann="hllc", levelmin=4, levelmax=7, err_grad_d=0.1, err_grad_p=0.1)
    h = RefHarness(3).create(nml, ngridmax=30000, levelmin=4, nlevelmax=7, gamma=1.4)
    r = AmrRun(h, 4, 7, 1.4, ed=0.1, ep=0.1)
    r.initialize(sedov_ic(3, 4))
    for _ in range(steps):
        r.coarse_step()
    return h, r


@pytest.mark.parametrize("riemann", ["llf", "exact"])
def test_noalloc_on_an_amr_level_with_long_reflux_targets(riemann):
    """Level 7 of a sub-cycled Sedov run (levels 4..7, three coarse steps):
    ghost states from coarser cells, refluxes into them, and coarse targets
    with more than 16 updates, each folded by one warp."""
    torch = pytest.importorskip("torch")
    h, _ = _sedov_amr(3)
    try:
        g = h.grid()
        a = h.arrays()
        uold, unew_in = a["uold"].copy(), a["unew"].copy()
        params = rgpu.make_params(3, slope_type=2, riemann=riemann, interpol_type=1)
        ctx = rgpu.Context(params, 0)
        try:
            ctx.sync_topology(g)
            for il, dt in ((7, 1.1e-5), (6, 2.3e-5)):
                dx = 1.0 / 2 ** il
                ref = _reference_step(ctx, il, dt, dx, uold, unew_in)
                if il == 7:
                    assert ctx.plan_info(il)["nlong"] > 0, "the case must reach the warp fold of long targets"
                uold_dev = torch.from_numpy(uold).to("cuda:0")
                unew_dev = torch.from_numpy(unew_in).to("cuda:0")
                for call in range(2):
                    out = unew_dev.clone()
                    _noalloc_call(torch, ctx, il, dt, dx, uold_dev, out, check_free=call > 0)
                    got = out.cpu().numpy()
                    assert bits_equal(got, ref), f"level {il} call {call + 1}: {np.count_nonzero(got != ref)} differ"
        finally:
            ctx.close()
    finally:
        h.close()


def test_noalloc_rejects_missing_plan_and_oversized_levels():
    torch = pytest.importorskip("torch")
    small = rg_tree.build_uniform(3, 4)
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc"), 0)
    try:
        ctx.sync_topology(small)
        buf = torch.zeros(small.nvar * small.ncell, dtype=torch.float64, device="cuda:0")
        with pytest.raises(rgpu.RGError) as e:  # no plan yet: building one would allocate
            ctx.godunov_level_noalloc(4, 1e-4, 1.0 / 16, buf.data_ptr(), buf.data_ptr())
        assert e.value.code == rgpu.RG_ERR_STATE
        big = rg_tree.build_uniform(3, 8)  # 128^3 cells: 63 M scratch doubles > 8 M
        ctx.sync_topology(big)
        u = rg_tree.sedov_state(big, 8)
        ctx.upload_state(u, u)
        ctx.set_unew(8)  # builds the plan
        big_buf = torch.from_numpy(u).to("cuda:0")
        with pytest.raises(rgpu.RGError) as e:
            ctx.godunov_level_noalloc(8, 1e-7, 1.0 / 256, big_buf.data_ptr(), big_buf.data_ptr())
        assert e.value.code == rgpu.RG_ERR_ARG and "static scratch holds" in str(e.value)
    finally:
        ctx.close()


def _cuda_malloc(nbytes):
    """A device allocation of exactly nbytes from the CUDA runtime itself (a
    caching allocator would hand out a slice of a larger segment)."""
    import ctypes as C
    rt = C.CDLL("libcudart.so.12")
    p = C.c_void_p()
    assert rt.cudaMalloc(C.byref(p), C.c_size_t(nbytes)) == 0
    return p.value, lambda: rt.cudaFree(p)


def test_noalloc_rejects_short_or_host_buffers_and_learned_start_without_network():
    torch = pytest.importorskip("torch")
    level = 6  # a 12 MB state: half of it is well past any rounding of the allocation size
    g = rg_tree.build_uniform(3, level)
    u = rg_tree.sedov_state(g, level)
    dx = 1.0 / 2 ** level
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc"), 0)
    try:
        ctx.sync_topology(g)
        ctx.upload_state(u, u)
        ctx.set_unew(level)
        full = torch.from_numpy(u).to("cuda:0")
        short, free_short = _cuda_malloc(u.nbytes // 2)
        try:
            with pytest.raises(rgpu.RGError) as e:
                ctx.godunov_level_noalloc(level, 1e-6, dx, full.data_ptr(), short)
            assert e.value.code == rgpu.RG_ERR_ARG and "nvar*ncell" in str(e.value)
        finally:
            torch.cuda.synchronize()
            free_short()
        host = np.ascontiguousarray(u)
        with pytest.raises(rgpu.RGError) as e:
            ctx.godunov_level_noalloc(level, 1e-6, dx, host.ctypes.data, full.data_ptr())
        assert e.value.code == rgpu.RG_ERR_ARG and "device memory" in str(e.value)
    finally:
        ctx.close()
    g = rg_tree.build_uniform(3, 4)
    u = rg_tree.sedov_state(g, 4)
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="exact", exact_guess=1), 0)
    try:
        ctx.sync_topology(g)
        ctx.upload_state(u, u)
        ctx.set_unew(4)
        full = torch.from_numpy(u).to("cuda:0")
        with pytest.raises(rgpu.RGError) as e:
            ctx.godunov_level_noalloc(4, 1e-4, 1.0 / 16, full.data_ptr(), full.clone().data_ptr())
        assert e.value.code == rgpu.RG_ERR_STATE and "network" in str(e.value)
    finally:
        ctx.close()


def test_noalloc_rejects_a_plan_made_stale_by_a_tree_change():
    """After make_grid_fine changed the device-resident tree, the level plans
    describe the old tree: the allocation-free call refuses until one
    allocating call for the level has rebuilt them."""
    torch = pytest.importorskip("torch")
    changed = False
    for steps in (1, 2, 3):
        h, _ = _sedov_amr(steps)
        try:
            ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc", interpol_type=1), 0)
            try:
                ctx.tree_attach(h.grid(), h.tree_arrays(), 4)
                ctx.set_unew(4)  # plan of level 4 on the attached tree
                before = [ctx.count_grids(il) for il in range(4, 8)]
                for il in range(4, 7):  # the refinements amr_step(levelmin) starts with
                    ctx.make_grid_fine(il + 1)
                if [ctx.count_grids(il) for il in range(4, 8)] == before:
                    continue
                changed = True
                ngm, ncell = ctx.tree_sizes()
                buf = torch.zeros(5 * ncell, dtype=torch.float64, device="cuda:0")
                with pytest.raises(rgpu.RGError) as e:
                    ctx.godunov_level_noalloc(4, 1e-6, 1.0 / 16, buf.data_ptr(), buf.clone().data_ptr())
                # the tree operations either left the plans marked stale or
                # already dropped them: refused either way, nothing launched
                assert e.value.code == rgpu.RG_ERR_STATE
                assert "tree changed" in str(e.value) or "no level plan" in str(e.value)
                ctx.set_unew(4)  # an allocating call rebuilds the plans; the call is accepted again
                uold_dev, unew_dev = ctx.device_state()
                ctx.godunov_level_noalloc(4, 1e-6, 1.0 / 16, uold_dev, unew_dev)
                ctx.synchronize()
            finally:
                ctx.close()
        finally:
            h.close()
        if changed:
            break
    assert changed, "no refinement changed the tree within three coarse steps"
