"""A whole AMR run with the tree and the state resident on the GPU.

`DeviceAmrRun` runs Simulation::amr_step and the coarse step around it
(RAMSES-CPP src/core/Simulation.cpp:366-397, 522-635) on one rgpu.Context
after `Context.tree_attach`: the tree operations (flag_fine, make_grid_fine,
remove_grid_fine, restrict_fine; rg_tree.cu), the CFL step
(compute_courant_step, HydroSolver.cpp:878-977), set_unew / godunov_fine /
set_uold all run on the device.  Same call sequence as the reference's
step, so the tree, every oct id and the state come out bit for bit as the
reference's own run leaves them; when a refinement needs more octs than the
free list holds, ngridmax doubles as in the reference (Context.tree_sizes
gives the new sizes).

By default a coarse step is one native call (rg_amr_coarse_step, rg_amr.cu),
whose clock (each level's dt and the time) stays on the device until the
step ends; `native=False` issues the same sequence call by call from Python
through the per-operation entry points, reading each level's dt back, which
the tests use to check both paths.

The CFL step takes the reference formula with or without its p <= 100 rho
cap (`pressure_cap`); the sub-cycled Sedov runs use it without the cap, which
makes the blast unstable at these resolutions.
"""


import rgpu


class DeviceAmrRun:
    def __init__(self, ctx, nx, levelmin, nlevelmax, cfl=0.8, ed=-1.0, ep=-1.0, ev=-1.0, nexpand=1,
                 pressure_cap=False, boxlen=1.0, native=True):
        self.ctx, self.nx, self.lmin, self.lmax = ctx, nx, levelmin, nlevelmax
        self.native = native
        self.cfg = rgpu.rg_amr_config(levelmin, nexpand, cfl, ed, ep, ev, 1 if pressure_cap else 0, boxlen)
        self.clock = rgpu.rg_amr_clock()
        self.cfl, self.ed, self.ep, self.ev, self.nexp = cfl, ed, ep, ev, nexpand
        self.pressure_cap, self.boxlen = pressure_cap, boxlen
        self.nsub = [1] * 33
        for i in range(levelmin, 33):
            self.nsub[i] = 2
        self.dtnew = [0.0] * 33
        self.dtold = [0.0] * 33
        self.t = 0.0
        self.nstep = 0
        self.cell_updates = 0

    def amr_step(self, il, icount):
        c = self.ctx
        if il > self.lmax:
            return
        if il > 0 and c.count_grids(il) == 0:
            return
        if self.lmin < self.lmax and (il == self.lmin or icount > 1):
            for i in range(il, self.lmax + 1):
                c.make_grid_fine(i + 1)
            for i in range(self.lmax, il - 1, -1):
                c.remove_grid_fine(i + 1)
        dx = self.boxlen / (self.nx * 2 ** il)
        self.dtold[il] = self.dtnew[il]
        self.dtnew[il] = c.courant_step(il, dx, self.cfl, pressure_cap=self.pressure_cap)
        if il > self.lmin:
            cand = self.dtnew[il - 1] / self.nsub[il - 1]
            self.dtnew[il] = cand if cand < self.dtnew[il] else self.dtnew[il]
        dt = self.dtnew[il]
        c.set_unew(il)
        nsub = self.nsub[il]
        if il < self.lmax:
            if c.count_grids(il + 1) > 0:
                for i in range(1, nsub + 1):
                    self.amr_step(il + 1, i)
            else:
                self.dtold[il + 1] = self.dtnew[il] / nsub
                self.dtnew[il + 1] = self.dtnew[il] / nsub
                self.t += dt
                self.nstep += 1
        else:
            self.t += dt
            self.nstep += 1
        c.godunov_level(il, dt, dx)
        self.cell_updates += c.cell_updates(il)
        c.set_uold(il)
        if il < self.lmax:
            c.restrict_fine(il)
        c.flag_fine(il + 1, self.ed, self.ep, self.ev, -1.0, self.nexp, icount,
                    self.nsub[il - 1] if il > 0 else 1)

    def coarse_step(self):
        if self.native:
            self.ctx.amr_coarse_step(self.cfg, self.clock)
            self.t, self.nstep, self.cell_updates = self.clock.t, self.clock.nstep, self.clock.cell_updates
            return
        c = self.ctx
        if self.lmin < self.lmax:
            for il in range(1, self.lmin):
                c.make_grid_fine(il)
        self.amr_step(self.lmin, 1)
        for il in range(self.lmin, 0, -1):
            c.flag_fine(il, self.ed, self.ep, self.ev, -1.0, self.nexp, 2, 2)
        if self.lmin < self.lmax:
            for il in range(self.lmin - 1, -1, -1):
                c.restrict_fine(il)
