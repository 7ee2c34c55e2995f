"""ctypes bindings to the parity checkers (test infrastructure only).

- ``RefHarness``: the RAMSES-CPP reference compiled from its own sources into
  ``oracle/_ref/libref_harness{1,3}d.so`` (see ``oracle/Makefile``), driven
  through its AmrGrid / TreeUpdater / HydroSolver API.
- ``Oracle``: the C restatement ``oracle/rg_oracle.c`` built into
  ``oracle/_build/liboracle.so``.

Both operate on the reference data layout: state ``[nvar][ncell]`` doubles,
1-based cell ids (``AmrGrid.hpp:104-107``).
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"


def reference_dir():
    """Where the RAMSES-CPP sources are: RG_REFERENCE_DIR, else the default of
    the oracle's build recipe (``make -C oracle refdir``)."""
    env = os.environ.get("RG_REFERENCE_DIR")
    if env:
        return Path(env)
    r = subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "refdir"], capture_output=True, text=True)
    return Path(r.stdout.strip()) if r.returncode == 0 and r.stdout.strip() else Path("reference-not-configured")


REF_SRC = reference_dir()

I32P = C.POINTER(C.c_int)
F64P = C.POINTER(C.c_double)


# The ABI structs of include/rgpu.h, shared with the GPU binding.
import sys as _sys  # noqa: E402
_sys.path.insert(0, str(ROOT / "ramses-cpp_b200"))
from rgpu import RIEMANN, make_params, rg_grid_view, rg_params  # noqa: E402,F401


def _ptr(a, t):
    return a.ctypes.data_as(t)


def ensure_built(target):
    """Build oracle targets on demand (``oracle`` always; ``ref`` needs the reference tree)."""
    lib = {"oracle": ORACLE_DIR / "_build" / "liboracle.so",
           "ref": ORACLE_DIR / "_ref" / "libref_harness3d.so",
           "dropin": ORACLE_DIR / "_ref" / "libref_harness_gpu3d.so"}[target]
    if lib.exists():
        return True
    if target in ("ref", "dropin") and not REF_SRC.exists():
        return False
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), target, f"REF={REF_SRC}", "-j8"], check=True)
    return lib.exists()


class GridArrays:
    """numpy copies of the tree arrays + a matching ``rg_grid_view``."""

    def __init__(self, **kw):
        self.__dict__.update(kw)
        self._keep = []
        v = rg_grid_view()
        for k in ("ncoarse", "ngridmax", "ncell", "nvar", "nx", "ny", "nz", "ncpu", "nboundary", "nlevelmax"):
            setattr(v, k, int(kw[k]))
        for k in ("son", "father", "nbor", "next", "headl"):
            a = np.ascontiguousarray(kw[k], dtype=np.int32)
            setattr(self, k, a)
            setattr(v, k, _ptr(a, I32P))
        v.bound_type = None
        v.nbound_type = 0
        self.view = v

    def level_octs(self, ilevel):
        octs = []
        ig = int(self.headl[ilevel * (self.ncpu + self.nboundary)]) if 0 <= ilevel <= self.nlevelmax else 0
        while ig > 0:
            octs.append(ig)
            ig = int(self.next[ig - 1])
        return np.array(octs, dtype=np.int32)

    def cell_ids(self, ilevel, ndim):
        octs = self.level_octs(ilevel)
        ttd = 1 << ndim
        ic = np.arange(1, ttd + 1)
        return (self.ncoarse + (ic[None, :] - 1) * self.ngridmax + octs[:, None]).reshape(-1)


class RefHarness:
    """The reference driven through its own API.  variant="gpu" loads the
    drop-in build whose HydroSolver is the GpuHydroSolver patch."""

    def __init__(self, ndim, variant="cpu"):
        target = "dropin" if variant == "gpu" else "ref"
        assert ensure_built(target), "reference sources unavailable"
        self.ndim = ndim
        name = f"libref_harness_gpu{ndim}d.so" if variant == "gpu" else f"libref_harness{ndim}d.so"
        self.lib = C.CDLL(str(ORACLE_DIR / "_ref" / name))
        L = self.lib
        L.rh_create.restype = C.c_void_p
        L.rh_create.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_double, C.c_double]
        L.rh_destroy.argtypes = [C.c_void_p]
        L.rh_get.restype = C.c_longlong
        L.rh_get.argtypes = [C.c_void_p, C.c_char_p]
        L.rh_ptr.restype = C.c_void_p
        L.rh_ptr.argtypes = [C.c_void_p, C.c_char_p]
        L.rh_count_grids.argtypes = [C.c_void_p, C.c_int]
        L.rh_cell_center.argtypes = [C.c_void_p, C.c_int, F64P]
        L.rh_flag_fine.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_int, C.c_int, C.c_int]
        for n in ("rh_make_grid_fine", "rh_remove_grid_fine", "rh_restrict_fine", "rh_set_unew", "rh_set_uold"):
            getattr(L, n).argtypes = [C.c_void_p, C.c_int]
        L.rh_godunov_fine.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.rh_courant.restype = C.c_double
        L.rh_courant.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double]
        L.rh_riemann.argtypes = [C.c_char_p, F64P, F64P, F64P, C.c_double]
        L.rh_slope.restype = C.c_double
        L.rh_slope.argtypes = [C.c_double] * 3 + [C.c_int, C.c_double, C.c_double]
        L.rh_interpol_hydro.argtypes = [C.c_void_p, F64P, F64P]
        L.rh_write_hydro.argtypes = [C.c_void_p, C.c_char_p]
        self.h = None

    # -- construction -----------------------------------------------------------
    def create(self, nml, nx=1, ny=1, nz=1, ngridmax=1000, nvar=None, levelmin=1, nlevelmax=1,
               gamma=1.4, boxlen=1.0):
        nvar = nvar or self.ndim + 2
        self.h = self.lib.rh_create(nml.encode(), nx, ny, nz, ngridmax, nvar, levelmin, nlevelmax, gamma, boxlen)
        assert self.h, "rh_create failed"
        self.nvar = nvar
        self.levelmin, self.nlevelmax = levelmin, nlevelmax
        return self

    def write_hydro(self, path):
        """The reference's RamsesWriter::write_hydro of the current state."""
        self.lib.rh_write_hydro(self.h, str(path).encode())

    def close(self):
        if self.h:
            self.lib.rh_destroy(self.h)
            self.h = None

    def get(self, name):
        return int(self.lib.rh_get(self.h, name.encode()))

    def _arr(self, name, n, dtype):
        p = self.lib.rh_ptr(self.h, name.encode())
        ct = C.c_double if dtype == np.float64 else C.c_int
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(n,))

    def arrays(self):
        """Live numpy views of the reference's vectors (invalid after a resize)."""
        ncell, ngm, nvar = self.get("ncell"), self.get("ngridmax"), self.nvar
        return dict(uold=self._arr("uold", nvar * ncell, np.float64), unew=self._arr("unew", nvar * ncell, np.float64),
                    son=self._arr("son", ncell, np.int32), father=self._arr("father", ngm, np.int32),
                    nbor=self._arr("nbor", 6 * ngm, np.int32), next=self._arr("next", ngm, np.int32),
                    headl=self._arr("headl", self.get("headl_size"), np.int32),
                    xg=self._arr("xg", 3 * ngm, np.float64), flag1=self._arr("flag1", ncell, np.int32))

    def tree_arrays(self):
        """Every array and scalar of the reference's tree (AmrGrid.hpp:26-30): the
        hydro arrays plus prev, flag2, cpu_map, the level-list tails and counts
        and the free list (headf, tailf, numbf)."""
        a = self.arrays()
        ncell, ngm, nh = self.get("ncell"), self.get("ngridmax"), self.get("headl_size")
        a.update(prev=self._arr("prev", ngm, np.int32), flag2=self._arr("flag2", ncell, np.int32),
                 cpu_map=self._arr("cpu_map", ncell, np.int32), taill=self._arr("taill", nh, np.int32),
                 numbl=self._arr("numbl", nh, np.int32))
        a.update(headf=self.get("headf"), tailf=self.get("tailf"), numbf=self.get("numbf"))
        return a

    def grid(self):
        a = self.arrays()
        return GridArrays(ncoarse=self.get("ncoarse"), ngridmax=self.get("ngridmax"), ncell=self.get("ncell"),
                          nvar=self.nvar, nx=self.get("nx"), ny=self.get("ny"), nz=self.get("nz"),
                          ncpu=self.get("ncpu"), nboundary=self.get("nboundary"), nlevelmax=self.get("nlevelmax"),
                          son=a["son"].copy(), father=a["father"].copy(), nbor=a["nbor"].copy(),
                          next=a["next"].copy(), headl=a["headl"].copy())

    def cell_centers(self, ids):
        out = np.zeros((len(ids), 3))
        buf = (C.c_double * 3)()
        for i, c in enumerate(ids):
            self.lib.rh_cell_center(self.h, int(c), buf)
            out[i] = buf[:]
        return out

    def count_grids(self, il):
        return self.lib.rh_count_grids(self.h, il)

    # -- tree operations (reference TreeUpdater) ------------------------------------
    def flag_fine(self, il, ed=-1.0, ep=-1.0, ev=-1.0, eb2=-1.0, nexp=1, icount=1, nsub=2):
        self.lib.rh_flag_fine(self.h, il, ed, ep, ev, eb2, nexp, icount, nsub)

    def make_grid_fine(self, il):
        self.lib.rh_make_grid_fine(self.h, il)

    def remove_grid_fine(self, il):
        self.lib.rh_remove_grid_fine(self.h, il)

    def restrict_fine(self, il):
        self.lib.rh_restrict_fine(self.h, il)

    def refine_uniform(self, levelmin, nexpand=1):
        """Base refinement loop of Simulation::initialize (Simulation.cpp:226-234)."""
        for _ in range(1, levelmin + 1):
            for il in range(1, self.nlevelmax + 1):
                self.flag_fine(il, -1, -1, -1, -1, nexpand, 1)
                self.make_grid_fine(il)

    # -- hydro ------------------------------------------------------------------------
    def set_unew(self, il):
        self.lib.rh_set_unew(self.h, il)

    def set_uold(self, il):
        self.lib.rh_set_uold(self.h, il)

    def godunov_fine(self, il, dt, dx):
        self.lib.rh_godunov_fine(self.h, il, dt, dx)

    def courant(self, il, dx, gamma, cfl):
        return self.lib.rh_courant(self.h, il, dx, gamma, cfl)

    def riemann(self, name, ql, qr, gamma):
        ql = np.ascontiguousarray(ql, dtype=np.float64)
        qr = np.ascontiguousarray(qr, dtype=np.float64)
        f = np.zeros(20)
        self.lib.rh_riemann(name.encode(), _ptr(ql, F64P), _ptr(qr, F64P), _ptr(f, F64P), gamma)
        return f

    def slope(self, ql, qc, qr, t, theta=1.5, nu=0.0):
        return self.lib.rh_slope(ql, qc, qr, t, theta, nu)


def namelist(slope_type=2, riemann="hllc", interpol_type=1, interpol_var=0, levelmin=1, levelmax=1,
             err_grad_d=-1.0, err_grad_p=-1.0, nexpand=1, extra=""):
    return (f"&AMR_PARAMS\nlevelmin={levelmin}\nlevelmax={levelmax}\nnexpand={nexpand}\n/\n"
            f"&HYDRO_PARAMS\nslope_type={slope_type}\nriemann='{riemann}'\n/\n"
            f"&REFINE_PARAMS\ninterpol_type={interpol_type}\ninterpol_var={interpol_var}\n"
            f"err_grad_d={err_grad_d}\nerr_grad_p={err_grad_p}\n/\n{extra}")


class Oracle:
    def __init__(self):
        ensure_built("oracle")
        self.lib = L = C.CDLL(str(ORACLE_DIR / "_build" / "liboracle.so"))
        GV = C.POINTER(rg_grid_view)
        PP = C.POINTER(rg_params)
        L.orc_godunov_fine.argtypes = [GV, PP, C.c_int, C.c_double, C.c_double, F64P, F64P,
                                       C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.orc_set_unew.argtypes = [GV, C.c_int, C.c_int, C.c_int, F64P, F64P]
        L.orc_set_uold.argtypes = [GV, C.c_int, C.c_int, C.c_int, F64P, F64P]
        L.orc_courant_step.restype = C.c_double
        L.orc_courant_step.argtypes = [GV, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_int, F64P]
        L.orc_level_cell_updates.restype = C.c_longlong
        L.orc_level_cell_updates.argtypes = [GV, C.c_int, C.c_int]
        L.orc_get_nbor_cells.argtypes = [GV, C.c_int, I32P, C.c_int, I32P, C.c_int]
        L.orc_get_nbor_grids.argtypes = [GV, C.c_int, I32P]
        for n in ("orc_solve_llf", "orc_solve_hll", "orc_solve_hllc", "orc_solve_acoustic"):
            getattr(L, n).argtypes = [F64P, F64P, F64P, C.c_double, C.c_int]
        L.orc_solve_exact.argtypes = [F64P, F64P, F64P, C.c_double, C.c_int, C.c_int, C.c_double, C.c_double,
                                      I32P, F64P]
        L.orc_compute_slope.restype = C.c_double
        L.orc_compute_slope.argtypes = [C.c_double] * 3 + [C.c_int, C.c_double, C.c_double]

    def godunov_fine(self, grid, params, il, dt, dx, uold, unew):
        it, calls = C.c_longlong(0), C.c_longlong(0)
        rc = self.lib.orc_godunov_fine(C.byref(grid.view), C.byref(params), il, dt, dx, _ptr(uold, F64P),
                                       _ptr(unew, F64P), C.byref(it), C.byref(calls))
        assert rc == 0, f"orc_godunov_fine rc={rc}"
        return it.value, calls.value

    def set_unew(self, grid, ndim, nvar, il, uold, unew):
        assert self.lib.orc_set_unew(C.byref(grid.view), ndim, nvar, il, _ptr(uold, F64P), _ptr(unew, F64P)) == 0

    def set_uold(self, grid, ndim, nvar, il, uold, unew):
        assert self.lib.orc_set_uold(C.byref(grid.view), ndim, nvar, il, _ptr(uold, F64P), _ptr(unew, F64P)) == 0

    def courant(self, grid, ndim, nvar, il, dx, gamma, cfl, uold, pressure_cap=True, boxlen=1.0):
        return self.lib.orc_courant_step(C.byref(grid.view), ndim, nvar, il, dx, gamma, cfl, boxlen,
                                         1 if pressure_cap else 0, _ptr(uold, F64P))

    def cell_updates(self, grid, ndim, il):
        return self.lib.orc_level_cell_updates(C.byref(grid.view), ndim, il)

    def nbor_cells(self, grid, ndim, igrid, ic):
        ign = (C.c_int * 7)()
        self.lib.orc_get_nbor_grids(C.byref(grid.view), igrid, ign)
        icn = (C.c_int * 6)()
        self.lib.orc_get_nbor_cells(C.byref(grid.view), ndim, ign, ic, icn, igrid)
        return list(icn)

    def riemann(self, name, ql, qr, gamma, ndim, niter=10, tol=1e-6, p0=-1.0):
        ql = np.ascontiguousarray(ql, dtype=np.float64)
        qr = np.ascontiguousarray(qr, dtype=np.float64)
        f = np.zeros(20)
        if name == "exact":
            it = C.c_int(0)
            ps = C.c_double(0)
            self.lib.orc_solve_exact(_ptr(ql, F64P), _ptr(qr, F64P), _ptr(f, F64P), gamma, ndim, niter, tol, p0,
                                     C.byref(it), C.byref(ps))
            return f
        getattr(self.lib, f"orc_solve_{name}")(_ptr(ql, F64P), _ptr(qr, F64P), _ptr(f, F64P), gamma, ndim)
        return f

    def slope(self, ql, qc, qr, t, theta=1.5, nu=0.0):
        return self.lib.orc_compute_slope(ql, qc, qr, t, theta, nu)

    def exact_pstar(self, ql, qr, gamma, ndim, niter, tol, p0=-1.0):
        """The exact solver's flux (nvar entries) and converged p*."""
        ql = np.ascontiguousarray(ql, dtype=np.float64)
        qr = np.ascontiguousarray(qr, dtype=np.float64)
        f = np.zeros(20)
        it, ps = C.c_int(0), C.c_double(0)
        self.lib.orc_solve_exact(_ptr(ql, F64P), _ptr(qr, F64P), _ptr(f, F64P), gamma, ndim, niter, tol, p0,
                                 C.byref(it), C.byref(ps))
        return f[:ndim + 2].copy(), ps.value


# ------------------------------------------------------------------ AMR replay

def harness_cell_centers(h, ids):
    """Cell centres computed like AmrGrid::get_cell_center, vectorised over ids."""
    a = h.arrays()
    ncoarse, ngm, nx, ndim = h.get("ncoarse"), h.get("ngridmax"), h.get("nx"), h.ndim
    ny, nz = h.get("ny"), h.get("nz")
    ids = np.asarray(ids, dtype=np.int64)
    out = np.full((len(ids), 3), 0.5)
    coarse = ids <= ncoarse
    if coarse.any():
        idx = ids[coarse] - 1
        dxc = 1.0 / max(nx, ny, nz)
        xyz = [idx % nx, (idx % (nx * ny)) // nx, idx // (nx * ny)]
        for d in range(ndim):
            out[coarse, d] = (xyz[d] + 0.5) * dxc
    fine = ~coarse
    if fine.any():
        rel = ids[fine] - ncoarse - 1
        ig = rel % ngm + 1
        icx = rel // ngm
        level = np.ones(len(ig), np.int64)
        curr = ig.copy()
        father = a["father"]
        for _ in range(64):
            fc = father[curr - 1]
            step = (curr > 0) & (fc > ncoarse)
            if not step.any():
                break
            curr = np.where(step, (fc - ncoarse - 1) % ngm + 1, curr)
            level += step
        dx = 1.0 / (nx * (2.0 ** level))
        scale = 1.0 / nx
        xg = a["xg"]
        for d in range(ndim):
            bit = (icx >> d) & 1
            out[fine, d] = xg[d * ngm + ig - 1] * scale + (bit - 0.5) * dx
    return out


def all_level_cells(h, nlevelmax):
    g = h.grid()
    ids = [np.arange(1, g.ncoarse + 1)]
    for L in range(1, nlevelmax + 1):
        c = g.cell_ids(L, h.ndim)
        if len(c):
            ids.append(c)
    return np.concatenate(ids)


def apply_ic(h, nlevelmax, ic_fn, gamma):
    """Write primitive ICs rho, v, p = ic_fn(xc) into uold (and unew) of every cell."""
    ids = all_level_cells(h, nlevelmax)
    xc = harness_cell_centers(h, ids)
    rho, vel, p = ic_fn(xc)
    a = h.arrays()
    nvar, ncell, ndim = h.nvar, h.get("ncell"), h.ndim
    u = a["uold"].reshape(nvar, ncell)
    u[0, ids - 1] = rho
    for d in range(ndim):
        u[1 + d, ids - 1] = rho * vel[d]
    u[ndim + 1, ids - 1] = p / (gamma - 1.0) + 0.5 * rho * sum(vel[d] ** 2 for d in range(ndim))
    a["unew"][:] = a["uold"]


def sedov_ic(ndim, base_level, gamma=1.4, rho0=1.0, p0=1e-5, e_blast=1.0, nx=1):
    dxb = 1.0 / (nx * 2 ** (base_level - 1))
    p_blast = (gamma - 1.0) * e_blast / (2 * dxb) ** ndim

    def fn(xc):
        inside = np.all(np.abs(xc[:, :ndim] - 0.5) < dxb, axis=1)
        n = len(xc)
        return np.full(n, rho0), [np.zeros(n)] * ndim, np.where(inside, p_blast, p0)
    return fn


class AmrRun:
    """Replay of Simulation::initialize / run / amr_step (src/core/Simulation.cpp:42-296,
    366-397, 522-635) on the reference harness, with the CFL step computed by the
    reference formula without its p <= 100 rho cap (that cap makes the Sedov blast
    unstable) and an optional hook around every hydro call."""

    def __init__(self, h, levelmin, nlevelmax, gamma, cfl=0.8, ed=-1.0, ep=-1.0, ev=-1.0, nexpand=1,
                 oracle=None, on_godunov=None):
        self.h, self.lmin, self.lmax, self.gamma, self.cfl = h, levelmin, nlevelmax, gamma, cfl
        self.ed, self.ep, self.ev, self.nexp = ed, ep, ev, nexpand
        self.nsub = [1] * 33
        for i in range(levelmin, 33):
            self.nsub[i] = 2
        self.dtnew = [0.0] * 33
        self.dtold = [0.0] * 33
        self.t = 0.0
        self.nstep = 0
        self.oracle = oracle or Oracle()
        self.on_godunov = on_godunov
        self.cell_updates = 0

    def initialize(self, ic_fn):
        h = self.h
        h.refine_uniform(self.lmin, self.nexp)
        for il_ref in range(self.lmin + 1, self.lmax + 1):
            self.init_flow(ic_fn)
            for il in range(1, self.lmax + 1):
                h.flag_fine(il, self.ed, self.ep, self.ev, -1.0, self.nexp, 1)
                h.make_grid_fine(il)
            if h.count_grids(il_ref) == 0:
                break
        self.init_flow(ic_fn)

    def init_flow(self, ic_fn):
        apply_ic(self.h, self.lmax, ic_fn, self.gamma)
        for il in range(self.lmax - 1, -1, -1):
            self.h.restrict_fine(il)

    def courant(self, il, dx):
        g = self.h.grid()
        a = self.h.arrays()
        return self.oracle.courant(g, self.h.ndim, self.h.nvar, il, dx, self.gamma, self.cfl, a["uold"],
                                   pressure_cap=False)

    def godunov(self, il, dt, dx):
        if self.on_godunov:
            self.on_godunov(self, il, dt, dx)
        else:
            self.h.godunov_fine(il, dt, dx)
        self.cell_updates += self.oracle.cell_updates(self.h.grid(), self.h.ndim, il)

    def amr_step(self, il, icount):
        h = self.h
        if il > self.lmax:
            return
        if h.count_grids(il) == 0 and il > 0:
            return
        if self.lmin < self.lmax and (il == self.lmin or icount > 1):
            for i in range(il, self.lmax + 1):
                h.make_grid_fine(i + 1)
            for i in range(self.lmax, il - 1, -1):
                h.remove_grid_fine(i + 1)
        dx = 1.0 / (h.get("nx") * 2 ** il)
        self.dtold[il] = self.dtnew[il]
        self.dtnew[il] = self.courant(il, dx)
        if il > self.lmin:
            cand = self.dtnew[il - 1] / self.nsub[il - 1]
            self.dtnew[il] = cand if cand < self.dtnew[il] else self.dtnew[il]
        dt = self.dtnew[il]
        h.set_unew(il)
        nsub = self.nsub[il]
        if il < self.lmax:
            if h.count_grids(il + 1) > 0:
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
        self.godunov(il, dt, dx)
        h.set_uold(il)
        if il < self.lmax:
            h.restrict_fine(il)
        h.flag_fine(il + 1, self.ed, self.ep, self.ev, -1.0, self.nexp, icount, self.nsub[il - 1] if il > 0 else 1)

    def coarse_step(self):
        h = self.h
        if self.lmin < self.lmax:
            for il in range(1, self.lmin):
                h.make_grid_fine(il)
        self.amr_step(self.lmin, 1)
        for il in range(self.lmin, 0, -1):
            h.flag_fine(il, self.ed, self.ep, self.ev, -1.0, self.nexp, 2, 2)
        if self.lmin < self.lmax:
            for il in range(self.lmin - 1, -1, -1):
                h.restrict_fine(il)
