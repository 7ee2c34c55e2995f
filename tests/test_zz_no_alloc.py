"""rg_godunov_level_noalloc: the level step for callers that may not allocate
device memory after set-up (a committed memory budget, a framework allocator
that owns the free memory, a time loop where cudaMalloc's implicit
synchronisation is not allowed).  Its flux scratch is a static 64 MiB array
inside the library and its state comes from the caller's own device buffers.

Checked through the C ABI against the allocating entry point rg_godunov_level,
bit for bit (the tolerance every HLLC parity test here uses), on two calls in
a row with different states, so the second call also shows that what the
first call left in the shared array does not leak into the result.  This file
is named to be collected last and creates everything it uses, so it passes
alone in a fresh process as well as after the other tests."""
import numpy as np
import pytest

import rg_tree
import rgpu

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


def _reference_step(ctx, level, dt, dx, u):
    ctx.upload_state(u, u)
    ctx.godunov_level(level, dt, dx)
    out = np.empty_like(u)
    ctx.download_state(unew=out)
    return out


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
        ref = [_reference_step(ctx, level, dt, dx, u) for dt, u in zip((2e-4, 3e-7), states)]
        for call, (dt, u) in enumerate(zip((2e-4, 3e-7), states)):
            uold_dev = torch.from_numpy(u).to("cuda:0")
            unew_dev = uold_dev.clone()
            torch.cuda.synchronize()
            ctx.godunov_level_noalloc(level, dt, dx, uold_dev.data_ptr(), unew_dev.data_ptr())
            ctx.synchronize()
            got = unew_dev.cpu().numpy()
            assert bits_equal(got, ref[call]), f"call {call + 1}: {np.count_nonzero(got != ref[call])} values differ"
            assert bits_equal(uold_dev.cpu().numpy(), u), "uold_dev must be read only"
    finally:
        ctx.close()


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
