"""The host side of the device-resident AMR run, on CPU: rg_amr.DeviceAmrRun's
call-by-call path (native=False) driven against a context stand-in that
forwards every call to the reference harness (the reference's own
TreeUpdater and HydroSolver, compiled here) must leave the same tree, state,
time and cell-update count as refsupport.AmrRun, the replay of
Simulation::run / amr_step (src/core/Simulation.cpp:366-397, 522-635).  This
checks the coarse-step loop's control flow (which level steps, in which order, with
which icount / nsubcycle arguments) without a GPU; the device operations
themselves are checked against the reference in tests/test_gpu_tree.py."""
import numpy as np

from rg_amr import DeviceAmrRun
from refsupport import AmrRun, Oracle, RefHarness, namelist, sedov_ic

LMIN, LMAX, GAMMA, ED, EP = 3, 5, 1.4, 0.1, 0.1


class HarnessContext:
    """The rgpu.Context calls DeviceAmrRun makes, answered by a reference harness."""

    def __init__(self, h):
        self.h, self.oracle = h, Oracle()
        self.calls = []

    def count_grids(self, il):
        return self.h.count_grids(il)

    def make_grid_fine(self, il):
        self.calls.append(("make", il))
        self.h.make_grid_fine(il)

    def remove_grid_fine(self, il):
        self.calls.append(("remove", il))
        self.h.remove_grid_fine(il)

    def restrict_fine(self, il):
        self.calls.append(("restrict", il))
        self.h.restrict_fine(il)

    def flag_fine(self, il, ed, ep, ev, eb2, nexp, icount, nsub):
        self.calls.append(("flag", il, icount, nsub))
        self.h.flag_fine(il, ed, ep, ev, eb2, nexp, icount, nsub)

    def courant_step(self, il, dx, cfl, pressure_cap=False):
        return self.oracle.courant(self.h.grid(), self.h.ndim, self.h.nvar, il, dx, GAMMA, cfl,
                                   self.h.arrays()["uold"], pressure_cap=pressure_cap)

    def set_unew(self, il):
        self.h.set_unew(il)

    def set_uold(self, il):
        self.h.set_uold(il)

    def godunov_level(self, il, dt, dx):
        self.calls.append(("godunov", il))
        self.last = il
        self.h.godunov_fine(il, dt, dx)

    def cell_updates(self, il):
        return self.oracle.cell_updates(self.h.grid(), self.h.ndim, il)


def make_run():
    nml = namelist(slope_type=2, riemann="hllc", levelmin=LMIN, levelmax=LMAX, err_grad_d=ED, err_grad_p=EP)
    h = RefHarness(3).create(nml, ngridmax=4000, levelmin=LMIN, nlevelmax=LMAX, gamma=GAMMA)
    r = AmrRun(h, LMIN, LMAX, GAMMA, ed=ED, ep=EP)
    r.initialize(sedov_ic(3, LMIN))
    return h, r


def test_device_run_driver_replays_the_reference_step():
    h_ref, r = make_run()
    h_dev, _ = make_run()
    ctx = HarnessContext(h_dev)
    d = DeviceAmrRun(ctx, nx=1, levelmin=LMIN, nlevelmax=LMAX, ed=ED, ep=EP, native=False)
    for _ in range(2):
        r.coarse_step()
        d.coarse_step()
    a, b = h_ref.tree_arrays(), h_dev.tree_arrays()
    for k in ("son", "father", "nbor", "next", "prev", "headl", "flag1", "cpu_map"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["uold"].view(np.int64), b["uold"].view(np.int64))
    assert d.t == r.t and d.cell_updates == r.cell_updates and d.nstep == r.nstep
    # the step visited the finer levels with sub-cycling
    levels = [c[1] for c in ctx.calls if c[0] == "godunov"]
    assert set(levels) >= {LMIN, LMIN + 1} and levels.count(LMIN + 1) == 2 * levels.count(LMIN)
