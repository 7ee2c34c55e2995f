"""Host-side builders of AmrGrid tree arrays and of the synthetic workloads.

``build_uniform`` reproduces, with vectorised numpy, the arrays the reference
produces for a uniform grid (levelmin == levelmax): Simulation::initialize
(RAMSES-CPP src/core/Simulation.cpp:226-234) flags every cell below levelmin
and TreeUpdater::make_grid_fine (src/core/TreeUpdater.cpp:27-150) refines
them level by level, popping octs off the free list (AmrGrid.cpp:259-268) in
level-list order and appending them to the next level list
(AmrGrid.cpp:289-302).  So octs are numbered breadth first, children of the
q-th oct of a level and child slot ic get id base + 2^ndim*q + ic; nbor[]
holds the coarse periodic neighbours for level-2 octs
(TreeUpdater.cpp:79-83) and the parent cell's neighbour cells deeper
(TreeUpdater.cpp:91-95); xg follows TreeUpdater.cpp:84-100 (exact dyadic
arithmetic, so equal to the reference's doubles).

Levels use the reference's numbering: level list L holds octs whose cells
are 2^(L-1)*nx per side (the Fortran RAMSES level L-1).
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Grid:
    ndim: int
    nx: int
    ny: int
    nz: int
    ngridmax: int
    nlevelmax: int
    nvar: int
    levelmin: int
    boxlen: float = 1.0
    ncpu: int = 1
    nboundary: int = 0
    son: np.ndarray = None
    father: np.ndarray = None
    nbor: np.ndarray = None
    next: np.ndarray = None
    headl: np.ndarray = None
    xg: np.ndarray = None
    level_octs: dict = field(default_factory=dict)

    @property
    def ncoarse(self):
        return self.nx * self.ny * self.nz

    @property
    def ncell(self):
        return self.ncoarse + (1 << self.ndim) * self.ngridmax

    def cell_ids(self, level):
        octs = self.level_octs.get(level, np.zeros(0, np.int64))
        ic = np.arange(1, (1 << self.ndim) + 1)
        return (self.ncoarse + (ic[None, :] - 1) * self.ngridmax + octs[:, None]).reshape(-1)

    def cell_centers(self, level):
        """Centres of the cells of level list ``level`` (get_cell_center, AmrGrid.cpp:331-365)."""
        octs = self.level_octs[level]
        ttd = 1 << self.ndim
        dx = self.boxlen / (self.nx * (1 << (level - 1)))
        scale = self.boxlen / self.nx
        out = np.full((len(octs), ttd, 3), 0.5 * self.boxlen)
        for ic in range(ttd):
            bits = [(ic >> d) & 1 for d in range(3)]
            for d in range(self.ndim):
                out[:, ic, d] = self.xg[d * self.ngridmax + octs - 1] * scale + (bits[d] - 0.5) * dx
        return out.reshape(-1, 3)

    def empty_state(self):
        return np.zeros(self.nvar * self.ncell, dtype=np.float64)


def _coarse_nbor(nx, ny, nz, cells, idim, side):
    idx = cells - 1
    iz = idx // (nx * ny)
    rem = idx % (nx * ny)
    iy = rem // nx
    ix = rem % nx
    c = [ix, iy, iz]
    n = [nx, ny, nz]
    c[idim] = (c[idim] + (-1 if side == 0 else 1) + n[idim]) % n[idim]
    return c[2] * nx * ny + c[1] * nx + c[0] + 1


def build_uniform(ndim, levelmin, nx=1, ny=1, nz=1, ngridmax=None, nlevelmax=None, nvar=None, boxlen=1.0):
    """Tree arrays of a uniform grid refined to level list ``levelmin``."""
    ttd = 1 << ndim
    ncoarse = nx * ny * nz
    counts = {L: ncoarse * ttd ** (L - 2) for L in range(2, levelmin + 1)}
    total = sum(counts.values())
    ngridmax = ngridmax or max(total, 1)
    if ngridmax < total:
        raise ValueError("ngridmax below the oct count (the reference would resize the grid)")
    nlevelmax = nlevelmax or levelmin
    g = Grid(ndim=ndim, nx=nx, ny=ny, nz=nz, ngridmax=ngridmax, nlevelmax=nlevelmax, nvar=nvar or ndim + 2,
             levelmin=levelmin, boxlen=boxlen)
    ncell = g.ncell
    son = np.zeros(ncell, np.int32)
    father = np.zeros(ngridmax, np.int32)
    nbor = np.zeros(6 * ngridmax, np.int32)
    nxt = np.zeros(ngridmax, np.int32)
    xg = np.zeros(3 * ngridmax, np.float64)
    headl = np.zeros((nlevelmax + 1), np.int32)
    base = 0
    parents = None  # octs of the previous level, list order
    for L in range(2, levelmin + 1):
        n = counts[L]
        ids = np.arange(base + 1, base + n + 1, dtype=np.int64)
        if L == 2:
            cells = np.arange(1, ncoarse + 1, dtype=np.int64)
            father[ids - 1] = cells
            son[cells - 1] = ids
            for idim in range(3):
                for side in range(2):
                    nbor[(idim * 2 + side) * ngridmax + ids - 1] = _coarse_nbor(nx, ny, nz, cells, idim, side)
            idx = cells - 1
            xyz = [idx % nx, (idx % (nx * ny)) // nx, idx // (nx * ny)]
            for d in range(ndim):
                xg[d * ngridmax + ids - 1] = xyz[d] + 0.5
        else:
            npar = len(parents)
            # child of (parent q, slot ic) has id base + ttd*q + ic (1-based ic)
            q = np.repeat(np.arange(npar), ttd)
            icx = np.tile(np.arange(ttd), npar)
            par = parents[q]
            pcell = ncoarse + icx * ngridmax + par
            father[ids - 1] = pcell
            son[pcell - 1] = ids
            dxl = 1.0 / (1 << (L - 2))
            for d in range(ndim):
                bit = (icx >> d) & 1
                xg[d * ngridmax + ids - 1] = xg[d * ngridmax + par - 1] + (bit - 0.5) * dxl
            # parent cell neighbours (same level, uniform): get_nbor_cells of the parent cell
            for idim in range(ndim):
                for side in range(2):
                    bit = (icx >> idim) & 1
                    inward = (bit == 1) if side == 0 else (bit == 0)
                    icp = icx ^ (1 << idim)
                    slot = 2 * idim + side
                    nb_father = nbor[slot * ngridmax + par - 1]
                    nb_oct = np.where(inward, par, son[np.maximum(nb_father, 1) - 1])
                    nbor[slot * ngridmax + ids - 1] = ncoarse + icp * ngridmax + nb_oct
        nxt[ids - 1] = ids + 1
        nxt[ids[-1] - 1] = 0
        headl[L] = base + 1
        g.level_octs[L] = ids
        parents = ids
        base += n
    if total < ngridmax:
        free = np.arange(total + 1, ngridmax + 1)
        nxt[free - 1] = free + 1
        nxt[ngridmax - 1] = 0
    g.son, g.father, g.nbor, g.next, g.headl, g.xg = son, father, nbor, nxt, headl, xg
    return g


def tree_arrays(g):
    """Every array and scalar of the AmrGrid tree (AmrGrid.hpp:26-31) as the
    reference's uniform refinement leaves it, for ``rg_tree_attach``: the
    arrays of ``build_uniform`` plus
    - flag1 = 1 on the refined cells (the ones flag_fine marked before
      make_grid_fine split them), 0 elsewhere;
    - flag2 = cpu_map = 1 on every cell (one process owns the whole domain);
    - prev = each oct's predecessor in its level list, and in the free list
      (AmrGrid.cpp:259-302 keep both lists doubly linked);
    - the level lists' tails and counts, and the free list: the octs after the
      last used one, in id order (headf, tailf, numbf);
    - uold = unew = 0 (the initial conditions come after).
    The level-list arrays are indexed like headl: ilevel * (ncpu + nboundary)."""
    ngm, ncell = g.ngridmax, g.ncell
    nh = len(g.headl)
    prev = np.zeros(ngm, np.int32)
    taill = np.zeros(nh, np.int32)
    numbl = np.zeros(nh, np.int32)
    used = 0
    for L, ids in g.level_octs.items():
        if len(ids) == 0:
            continue
        prev[ids[1:] - 1] = ids[:-1]
        taill[L] = ids[-1]
        numbl[L] = len(ids)
        used = max(used, int(ids[-1]))
    free = np.arange(used + 1, ngm + 1)
    if len(free):
        prev[free[1:] - 1] = free[:-1]
    return {"son": g.son, "father": g.father, "nbor": g.nbor, "next": g.next, "prev": prev, "headl": g.headl,
            "taill": taill, "numbl": numbl, "flag1": (g.son > 0).astype(np.int32),
            "flag2": np.ones(ncell, np.int32), "cpu_map": np.ones(ncell, np.int32), "xg": g.xg,
            "uold": np.zeros(g.nvar * ncell), "unew": np.zeros(g.nvar * ncell),
            "headf": int(free[0]) if len(free) else 0, "tailf": int(free[-1]) if len(free) else 0,
            "numbf": int(len(free))}


# ------------------------------------------------------------------ workloads

def sedov_state(g, level, gamma=1.4, rho0=1.0, p0=1e-5, e_blast=1.0, base_level=None):
    """Sedov blast: background (rho0, 0, p0); energy e_blast spread over the
    central 2^ndim cells of ``base_level`` (|x_c - 0.5| < dx_base on every axis)."""
    base_level = base_level or level
    u = g.empty_state().reshape(g.nvar, g.ncell)
    dxb = g.boxlen / (g.nx * (1 << (base_level - 1)))
    vol = (2 * dxb) ** g.ndim
    p_blast = (gamma - 1.0) * e_blast / vol
    for L in range(2, level + 1):
        ids = g.cell_ids(L)
        xc = g.cell_centers(L)
        inside = np.all(np.abs(xc[:, :g.ndim] - 0.5 * g.boxlen) < dxb, axis=1)
        p = np.where(inside, p_blast, p0)
        u[0, ids - 1] = rho0
        u[g.ndim + 1, ids - 1] = p / (gamma - 1.0)
    return u.reshape(-1)


def sod_state(g, level, gamma=1.4, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1), x0=0.5):
    """1D (or planar along x) shock tube: primitive (rho, u, p) left/right of x0."""
    u = g.empty_state().reshape(g.nvar, g.ncell)
    for L in range(2, level + 1):
        ids = g.cell_ids(L)
        xc = g.cell_centers(L)
        lft = xc[:, 0] < x0
        for (rho, vel, p), m in ((left, lft), (right, ~lft)):
            u[0, ids[m] - 1] = rho
            u[1, ids[m] - 1] = rho * vel
            u[g.ndim + 1, ids[m] - 1] = p / (gamma - 1.0) + 0.5 * rho * vel * vel
    return u.reshape(-1)


def planar_riemann_state(g, level, normal, left, right, gamma=5.0 / 3.0):
    """Planar discontinuity through the box centre with unit ``normal``;
    ``left``/``right`` = (rho, u_normal, p); tangential velocity zero."""
    u = g.empty_state().reshape(g.nvar, g.ncell)
    nrm = np.asarray(normal, dtype=np.float64)[:g.ndim]
    for L in range(2, level + 1):
        ids = g.cell_ids(L)
        xc = g.cell_centers(L)[:, :g.ndim] - 0.5 * g.boxlen
        side = xc @ nrm < 0.0
        for (rho, un, p), m in ((left, side), (right, ~side)):
            u[0, ids[m] - 1] = rho
            for d in range(g.ndim):
                u[1 + d, ids[m] - 1] = rho * un * nrm[d]
            u[g.ndim + 1, ids[m] - 1] = p / (gamma - 1.0) + 0.5 * rho * un * un
    return u.reshape(-1)


def random_state(g, level, seed=0, gamma=1.4, rho_range=(-1, 1), p_range=(-1, 1), vmax=1.0):
    """Log-uniform density and pressure, uniform velocity, on every level <= ``level``."""
    rng = np.random.default_rng(seed)
    u = g.empty_state().reshape(g.nvar, g.ncell)
    for L in range(2, level + 1):
        ids = g.cell_ids(L)
        n = len(ids)
        rho = 10 ** rng.uniform(*rho_range, n)
        v = rng.uniform(-vmax, vmax, (g.ndim, n))
        p = 10 ** rng.uniform(*p_range, n)
        u[0, ids - 1] = rho
        u[1:1 + g.ndim, ids - 1] = rho * v
        u[g.ndim + 1, ids - 1] = p / (gamma - 1.0) + 0.5 * rho * (v ** 2).sum(0)
    return u.reshape(-1)
