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


import numpy as np

import rg_tree
import rgpu


def sedov_primitives(ndim, base_level, gamma=1.4, rho0=1.0, p0=1e-5, e_blast=1.0, nx=1):
    """The Sedov blast initial condition as a function of cell centres: density
    rho0 and pressure p0 everywhere at rest, except the central 2^ndim cells of
    ``base_level`` (|x - 0.5| < dx_base on every axis), which share the energy
    e_blast as pressure (gamma-1) e_blast / (2 dx_base)^ndim."""
    dxb = 1.0 / (nx * 2 ** (base_level - 1))
    p_blast = (gamma - 1.0) * e_blast / (2 * dxb) ** ndim

    def fn(xc):
        inside = np.all(np.abs(xc[:, :ndim] - 0.5) < dxb, axis=1)
        n = len(xc)
        return np.full(n, rho0), [np.zeros(n)] * ndim, np.where(inside, p_blast, p0)
    return fn


def _cell_centres(a, ncoarse, ngridmax, nx, ndim, level, octs):
    """AmrGrid::get_cell_center (AmrGrid.cpp:331-365) of the cells of level
    list ``level`` (oct ids ``octs``), or of the coarse cells for level 0;
    boxlen 1."""
    if level == 0:
        idx = np.arange(ncoarse)
        out = np.full((ncoarse, 3), 0.5)
        dxc = 1.0 / nx
        xyz = [idx % nx, (idx % (nx * nx)) // nx, idx // (nx * nx)]
        for d in range(ndim):
            out[:, d] = (xyz[d] + 0.5) * dxc
        return out
    ttd = 1 << ndim
    dx = 1.0 / (nx * (2.0 ** (level - 1)))
    scale = 1.0 / nx
    out = np.full((len(octs), ttd, 3), 0.5)
    for ic in range(ttd):
        for d in range(ndim):
            bit = (ic >> d) & 1
            out[:, ic, d] = a["xg"][d * ngridmax + octs - 1] * scale + (bit - 0.5) * dx
    return out.reshape(-1, 3)


def init_flow(ctx, like, ndim, nx, nlevelmax, ic_fn, gamma):
    """Simulation::init_flow on the resident tree: the primitive initial
    condition ic_fn(centres) -> (rho, [v], p) written as conservative
    variables into uold of the coarse cells and of every level's cells, unew
    made a copy of uold, then restrict_fine from nlevelmax-1 down to 0."""
    a = ctx.tree_fetch(like)
    ngm, ncell = ctx.tree_sizes()
    ncoarse = nx ** ndim if ndim == 3 else nx
    nvar = ndim + 2
    u = a["uold"].reshape(nvar, ncell)
    ttd = 1 << ndim
    for L in range(0, nlevelmax + 1):
        if L == 0:
            ids = np.arange(1, ncoarse + 1)
            octs = None
        else:
            octs = ctx.level_octs(L).astype(np.int64) if ctx.count_grids(L) > 0 else np.zeros(0, np.int64)
            if len(octs) == 0:
                continue
            ic = np.arange(1, ttd + 1)
            ids = (ncoarse + (ic[None, :] - 1) * ngm + octs[:, None]).reshape(-1)
        xc = _cell_centres(a, ncoarse, ngm, nx, ndim, L, octs)
        rho, vel, p = ic_fn(xc)
        u[0, ids - 1] = rho
        for d in range(ndim):
            u[1 + d, ids - 1] = rho * vel[d]
        u[ndim + 1, ids - 1] = p / (gamma - 1.0) + 0.5 * rho * sum(vel[d] ** 2 for d in range(ndim))
    uold = np.ascontiguousarray(u.reshape(-1))
    ctx.upload_state(uold, uold.copy())
    for il in range(nlevelmax - 1, -1, -1):
        ctx.restrict_fine(il)


def initialize(ctx, ndim, levelmin, nlevelmax, ngridmax, ic_fn, gamma, ed=-1.0, ep=-1.0, ev=-1.0, nexpand=1):
    """Simulation::initialize (src/core/Simulation.cpp:226-296) with the tree
    on the device: the uniform grid to ``levelmin`` built on the host
    (rg_tree.build_uniform, the arrays the reference's uniform refinement
    leaves), attached to the context, then for each finer level the
    reference's rounds -- initial condition, flag_fine and make_grid_fine of
    every level -- until a level stays empty, and the initial condition once
    more; all tree work by the device kernels.  nx = 1."""
    g = rg_tree.build_uniform(ndim, levelmin, ngridmax=ngridmax, nlevelmax=nlevelmax)
    arrays = rg_tree.tree_arrays(g)
    ctx.tree_attach(g, arrays, levelmin)
    like = {"headl": arrays["headl"], "taill": arrays["taill"], "numbl": arrays["numbl"]}
    for il_ref in range(levelmin + 1, nlevelmax + 1):
        init_flow(ctx, like, ndim, 1, nlevelmax, ic_fn, gamma)
        for il in range(1, nlevelmax + 1):
            ctx.flag_fine(il, ed, ep, ev, -1.0, nexpand, 1)
            ctx.make_grid_fine(il)
        if ctx.count_grids(il_ref) == 0:
            break
    init_flow(ctx, like, ndim, 1, nlevelmax, ic_fn, gamma)


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
