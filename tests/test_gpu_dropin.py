"""The drop-in: the reference's own AmrGrid / TreeUpdater / HydroSolver API
with the GpuHydroSolver patch (ramses-cpp_b200/host/GpuHydroSolver.cpp)
supplied through create_hydro_solver, against the unmodified reference, on
the same inputs.  Whole runs, tree included, must stay bit-identical."""
import numpy as np
import pytest

from refsupport import ORACLE_DIR, AmrRun, RefHarness, namelist, sedov_ic

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


@pytest.fixture(scope="module", autouse=True)
def need_dropin(rgpu_lib):
    if not (ORACLE_DIR / "_ref" / "libref_harness_gpu3d.so").exists():
        from refsupport import ensure_built
        if not ensure_built("dropin"):
            pytest.skip("drop-in build needs the reference sources")


def _pair(ndim, nml, **kw):
    return RefHarness(ndim).create(nml, **kw), RefHarness(ndim, "gpu").create(nml, **kw)


@pytest.mark.parametrize("ndim,lmin,lmax,ngm,slope,riem,steps", [
    (3, 3, 5, 800, 2, "hllc", 3),
    (3, 4, 5, 1200, 1, "llf", 2),
    (1, 5, 7, 200, 1, "hllc", 6),
    (1, 6, 8, 400, 2, "hll", 4),
])
def test_amr_run_dropin_matches_reference(ndim, lmin, lmax, ngm, slope, riem, steps):
    nml = namelist(slope_type=slope, riemann=riem, levelmin=lmin, levelmax=lmax, err_grad_d=0.1, err_grad_p=0.1)
    kw = dict(ngridmax=ngm, levelmin=lmin, nlevelmax=lmax, gamma=1.4)
    ref, gpu = _pair(ndim, nml, **kw)
    runs = [AmrRun(h, lmin, lmax, 1.4, ed=0.1, ep=0.1) for h in (ref, gpu)]
    for r in runs:
        r.initialize(sedov_ic(ndim, lmin))
    for step in range(steps):
        for r in runs:
            r.coarse_step()
        a, b = ref.arrays(), gpu.arrays()
        for k in ("son", "father", "nbor", "next", "headl"):
            assert np.array_equal(a[k], b[k]), f"step {step}: tree array {k} differs"
        assert bits_equal(a["uold"], b["uold"]), f"step {step}: {np.count_nonzero(a['uold'] != b['uold'])} uold values differ"
        assert bits_equal(a["unew"], b["unew"]), f"step {step}: unew differs"
        assert runs[0].t == runs[1].t
    assert runs[1].cell_updates > 0
    ref.close()
    gpu.close()
