"""Ensembles of independent periodic boxes stepped together on one GPU.

Each box is a uniform 3D grid that the reference (RAMSES-CPP) would run as a
simulation of its own: levelmin = levelmax, periodic, one CFL step per
substep (Simulation::amr_step, src/core/Simulation.cpp:522-635, with the
level's dx = boxlen / (nx 2^level), :548).  To step hundreds of uneven boxes
in the same launches, their trees are merged into one forest:

- coarse cells, octs and cells of box b are renumbered into one id space
  (the reference's cell numbering icell = ncoarse + (ic-1) ngridmax + igrid,
  AmrGrid.cpp:279, over the summed ncoarse and ngridmax), so every son /
  father / nbor entry keeps pointing inside its own box: boxes never see each
  other;
- one level list (``Forest.level``) chains the leaf octs of every box, box
  after box, each box in its own list order, so the level plan's update order
  inside a box -- and therefore every bit of the result -- is the one the box
  has alone;
- ``first_oct`` tells the library which list positions belong to which box;
  the step then takes a CFL step per box with that box's dx
  (rg_set_level_boxes in include/rgpu.h).

The workload generator follows the ensemble configuration: edges drawn
uniformly from {16, 24, 32, 48, 64} (24 and 48 are nx = 3 coarse grids:
edge = nx 2^(level-1) in the reference's level numbering), a planar Riemann
problem through the centre with a normal uniform on the sphere, rho
log-uniform in [1e-3, 1e3], p log-uniform in [1e-4, 1e4], normal velocity
uniform in [-3, 3], gamma 5/3.
"""
from dataclasses import dataclass

import numpy as np

import rg_tree

# edge -> (nx, reference level list of the leaf octs)
EDGE_LAYOUT = {16: (1, 5), 24: (3, 4), 32: (1, 6), 48: (3, 5), 64: (1, 7)}
ENSEMBLE_SEED = 20261203


@dataclass
class BoxSpec:
    index: int
    edge: int
    nx: int
    level: int
    normal: tuple
    left: tuple   # (rho, u_normal, p)
    right: tuple

    @property
    def cells(self):
        return self.edge ** 3

    @property
    def dx(self):
        """dx the reference passes to godunov_fine for this box's level (boxlen 1)."""
        return 1.0 / (self.nx * (1 << self.level))


def box_specs(n=512, seed=ENSEMBLE_SEED, edges=(16, 24, 32, 48, 64)):
    """The seeded ensemble: ``n`` boxes with uneven edges and planar Riemann problems."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n):
        edge = int(edges[rng.integers(len(edges))])
        nx, level = EDGE_LAYOUT[edge]
        v = rng.normal(size=3)
        normal = tuple(v / np.linalg.norm(v))
        states = []
        for _ in range(2):
            rho = 10.0 ** rng.uniform(-3.0, 3.0)
            un = rng.uniform(-3.0, 3.0)
            p = 10.0 ** rng.uniform(-4.0, 4.0)
            states.append((rho, un, p))
        out.append(BoxSpec(b, edge, nx, level, normal, states[0], states[1]))
    return out


def shard_boxes(specs, world):
    """Partition boxes over ``world`` ranks, balanced by cell count (largest
    first onto the least loaded rank).  Boxes are independent, so a rank steps
    its shard with no exchange at all.  Returns one list of specs per rank,
    each in ascending box index."""
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for s in sorted(specs, key=lambda s: (-s.cells, s.index)):
        r = min(range(world), key=lambda i: (loads[i], i))
        parts[r].append(s)
        loads[r] += s.cells
    return [sorted(p, key=lambda s: s.index) for p in parts]


class Forest:
    """Merged tree arrays of a list of boxes (see the module docstring)."""

    def __init__(self, specs, gamma=5.0 / 3.0):
        self.specs = list(specs)
        self.gamma = gamma
        self.ndim = 3
        ttd = 8
        self.boxes = [rg_tree.build_uniform(3, s.level, nx=s.nx, ny=s.nx, nz=s.nx) for s in self.specs]
        self.coarse_off = np.cumsum([0] + [g.ncoarse for g in self.boxes])
        self.oct_off = np.cumsum([0] + [g.ngridmax for g in self.boxes])
        NC, NG = int(self.coarse_off[-1]), int(self.oct_off[-1])
        self.level = max(s.level for s in self.specs)
        V = self.level
        g = rg_tree.Grid(ndim=3, nx=NC, ny=1, nz=1, ngridmax=NG, nlevelmax=V, nvar=5, levelmin=V)
        ncell = g.ncell
        son = np.zeros(ncell, np.int32)
        father = np.zeros(NG, np.int32)
        nbor = np.zeros(6 * NG, np.int32)
        nxt = np.zeros(NG, np.int32)
        headl = np.zeros(V + 1, np.int32)
        for b, gb in enumerate(self.boxes):
            og = int(self.oct_off[b])
            ngm = gb.ngridmax
            cells = np.arange(1, gb.ncell + 1, dtype=np.int64)
            s = gb.son.astype(np.int64)
            son[self.map_cells(b, cells) - 1] = np.where(s > 0, s + og, 0)
            father[og:og + ngm] = self.map_cells(b, gb.father.astype(np.int64))
            for k in range(6):
                nbor[k * NG + og:k * NG + og + ngm] = self.map_cells(b, gb.nbor[k * ngm:(k + 1) * ngm].astype(np.int64))
        # level lists: every box's leaf octs in list V; shallower octs in the
        # list of their depth (box after box in both)
        lists = {L: [] for L in range(2, V + 1)}
        for b, (sp, gb) in enumerate(zip(self.specs, self.boxes)):
            og = int(self.oct_off[b])
            for L in range(2, sp.level):
                lists[L].append(gb.level_octs[L] + og)
            lists[V].append(gb.level_octs[sp.level] + og)
        for L, parts in lists.items():
            if not parts:
                continue
            ids = np.concatenate(parts).astype(np.int64)
            nxt[ids[:-1] - 1] = ids[1:]
            nxt[ids[-1] - 1] = 0
            headl[L] = ids[0]
            g.level_octs[L] = ids
        g.son, g.father, g.nbor, g.next, g.headl = son, father, nbor, nxt, headl
        g.xg = np.zeros(3 * NG)
        self.grid = g
        leaf_counts = [len(gb.level_octs[sp.level]) for sp, gb in zip(self.specs, self.boxes)]
        self.first_oct = np.cumsum([0] + leaf_counts).astype(np.int32)
        self.dx = np.array([s.dx for s in self.specs], dtype=np.float64)

    @property
    def nbox(self):
        return len(self.specs)

    @property
    def cells(self):
        return int(sum(s.cells for s in self.specs))

    def map_cells(self, b, ids):
        """Forest ids of box ``b``'s cell ids (values <= 0 are kept)."""
        gb = self.boxes[b]
        ids = np.asarray(ids, dtype=np.int64)
        ncb, ngm = gb.ncoarse, gb.ngridmax
        NC, NG = int(self.coarse_off[-1]), int(self.oct_off[-1])
        j = ids - ncb - 1
        fine = NC + (j // ngm) * NG + int(self.oct_off[b]) + (j % ngm) + 1
        out = np.where(ids <= ncb, int(self.coarse_off[b]) + ids, fine)
        return np.where(ids > 0, out, ids).astype(np.int32)

    def box_state(self, b):
        """Initial conservative state of box ``b`` in its own layout."""
        sp, gb = self.specs[b], self.boxes[b]
        return rg_tree.planar_riemann_state(gb, sp.level, sp.normal, sp.left, sp.right, self.gamma)

    def initial_state(self):
        u = self.grid.empty_state().reshape(5, self.grid.ncell)
        for b, gb in enumerate(self.boxes):
            ub = self.box_state(b).reshape(5, gb.ncell)
            cells = np.arange(1, gb.ncell + 1)
            u[:, self.map_cells(b, cells) - 1] = ub
        return u.reshape(-1)

    def lattices(self):
        """Per box: its periodic lattice of cells (x fastest) as forest cell ids and as
        positions p = (ic-1)*noct + k in the leaf level (k = oct position in the level
        list), concatenated box after box, with the extents [nbox][3]."""
        noct = int(self.first_oct[-1])
        ids_all, p_all, ext = [], [], []
        for b, (sp, gb) in enumerate(zip(self.specs, self.boxes)):
            E = sp.edge
            octs = gb.level_octs[sp.level]
            ids = gb.cell_ids(sp.level)                       # oct-major, ic minor
            ijk = np.rint(gb.cell_centers(sp.level) * E - 0.5).astype(np.int64)
            site = ijk[:, 0] + E * (ijk[:, 1] + E * ijk[:, 2])
            k = np.repeat(np.arange(len(octs)), 8) + int(self.first_oct[b])
            icx = np.tile(np.arange(8), len(octs))
            lat_id = np.zeros(E ** 3, np.int32)
            lat_p = np.full(E ** 3, -1, np.int32)
            lat_id[site] = self.map_cells(b, ids)
            lat_p[site] = icx * noct + k
            ids_all.append(lat_id)
            p_all.append(lat_p)
            ext.append((E, E, E))
        return np.array(ext, np.int32), np.concatenate(ids_all), np.concatenate(p_all)

    def extract(self, u, b):
        """Leaf-cell state of box ``b`` from a forest state, as [nvar][leaf cells] in the
        box's own cell order (Grid.cell_ids of its leaf level)."""
        sp, gb = self.specs[b], self.boxes[b]
        ids = gb.cell_ids(sp.level)
        return np.asarray(u).reshape(5, self.grid.ncell)[:, self.map_cells(b, ids) - 1]
