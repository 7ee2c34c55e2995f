"""Snapshot hydro files written from the device state are byte-identical to
the reference's RamsesWriter::write_hydro on the same tree and state
(src/io/RamsesWriter.cpp:145-226): a uniform 3D grid and a sub-cycled AMR
Sedov run in 3D and 1D."""
import numpy as np
import pytest

import rgpu
import rg_snapshot
from refsupport import AmrRun, RefHarness, namelist, sedov_ic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_reference(rgpu_lib, reference_available):
    if not reference_available:
        pytest.skip("needs the reference build")


def _ctx_from_harness(h, ndim, gamma):
    a = h.arrays()
    ctx = rgpu.Context(rgpu.make_params(ndim, gamma=gamma), 0)
    ctx.sync_topology(h.grid())
    ctx.upload_state(np.array(a["uold"]), np.array(a["unew"]))
    return ctx


@pytest.mark.parametrize("ndim,lmin,lmax,ngm,steps", [(3, 4, 4, 800, 0), (3, 3, 5, 800, 2), (1, 5, 7, 200, 4)])
def test_hydro_file_matches_reference_writer(tmp_path, ndim, lmin, lmax, ngm, steps):
    nml = namelist(slope_type=2, riemann="hllc", levelmin=lmin, levelmax=lmax, err_grad_d=0.1, err_grad_p=0.1)
    h = RefHarness(ndim).create(nml, ngridmax=ngm, levelmin=lmin, nlevelmax=lmax, gamma=1.4)
    run = AmrRun(h, lmin, lmax, 1.4, ed=0.1, ep=0.1)
    run.initialize(sedov_ic(ndim, lmin))
    for _ in range(steps):
        run.coarse_step()
    ref_path, gpu_path = tmp_path / "ref.out", tmp_path / "gpu.out"
    h.write_hydro(ref_path)
    ctx = _ctx_from_harness(h, ndim, 1.4)
    try:
        rg_snapshot.write_hydro(gpu_path, ctx, ndim, ndim + 2, lmax, 1.4)
    finally:
        ctx.close()
        h.close()
    a, b = ref_path.read_bytes(), gpu_path.read_bytes()
    assert len(a) == len(b) and a == b


def test_hydro_file_of_a_device_resident_run(tmp_path):
    """The tree resident on the device (rg_tree_attach + rg_amr_coarse_step):
    after two coarse steps on both sides, the hydro file written from the
    device's own tree and state equals the reference writer's bytes after the
    reference's two coarse steps, with no copy of the tree back to the host."""
    from rg_amr import DeviceAmrRun
    lmin, lmax = 3, 5
    nml = namelist(slope_type=2, riemann="hllc", levelmin=lmin, levelmax=lmax, err_grad_d=0.1, err_grad_p=0.1)
    h = RefHarness(3).create(nml, ngridmax=4000, levelmin=lmin, nlevelmax=lmax, gamma=1.4)
    run = AmrRun(h, lmin, lmax, 1.4, ed=0.1, ep=0.1)
    run.initialize(sedov_ic(3, lmin))
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc", gamma=1.4), 0)
    try:
        ctx.tree_attach(h.grid(), h.tree_arrays(), lmin)
        d = DeviceAmrRun(ctx, nx=1, levelmin=lmin, nlevelmax=lmax, ed=0.1, ep=0.1)
        for _ in range(2):
            run.coarse_step()
            d.coarse_step()
        ref_path, gpu_path = tmp_path / "ref.out", tmp_path / "gpu.out"
        h.write_hydro(ref_path)
        rg_snapshot.write_hydro(gpu_path, ctx, 3, 5, lmax, 1.4)
    finally:
        ctx.close()
        h.close()
    a, b = ref_path.read_bytes(), gpu_path.read_bytes()
    assert len(a) == len(b) and a == b
