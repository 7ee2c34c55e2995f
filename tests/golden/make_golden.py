"""Generate the golden vectors in tests/golden/ from the RAMSES-CPP reference.

    python tests/golden/make_golden.py          (needs the reference sources)

The reference is compiled from its own sources by oracle/Makefile and driven
through its public API by oracle/ref_harness.cpp; nothing here computes an
expected value itself.  The fixtures pin the C oracle and the GPU library on
machines where the reference tree is not available.
"""
import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parents[1] / "ramses-cpp_b200"))

from refsupport import (AmrRun, Oracle, RefHarness, make_params, namelist, sedov_ic)  # noqa: E402
import rg_tree  # noqa: E402

SEED = 20261203


def rand_states(rng, n, ndim, hard=False):
    """Rotated primitive states [rho, u_n, u_t..., p]."""
    nv = ndim + 2
    q = np.zeros((n, nv))
    lo, hi = (-3, 3) if hard else (-1, 1)
    q[:, 0] = 10 ** rng.uniform(lo, hi, n)
    q[:, 1:1 + ndim] = rng.uniform(-3 if hard else -1, 3 if hard else 1, (n, ndim))
    q[:, ndim + 1] = 10 ** rng.uniform(lo - 1, hi + 1, n)
    return q


def riemann_vectors(out):
    rng = np.random.default_rng(SEED)
    data = {}
    for ndim in (1, 3):
        h = RefHarness(ndim)
        for hard in (False, True):
            n = 256
            ql, qr = rand_states(rng, n, ndim, hard), rand_states(rng, n, ndim, hard)
            # a few degenerate pairs: identical states, vacuum-ish, strong rarefaction
            ql[:4], qr[:4] = ql[4:8], ql[4:8]
            qr[8:12, 1] = ql[8:12, 1] + 20.0
            tag = f"{ndim}d_{'hard' if hard else 'soft'}"
            data[f"ql_{tag}"], data[f"qr_{tag}"] = ql, qr
            for name in ("llf", "hll", "hllc", "acoustic", "exact"):
                for gamma in (1.4, 5.0 / 3.0):
                    f = np.array([h.riemann(name, ql[i], qr[i], gamma)[:ndim + 2] for i in range(n)])
                    data[f"flux_{name}_{tag}_g{gamma:.4f}"] = f
    np.savez_compressed(out, **data)


def slope_vectors(out):
    rng = np.random.default_rng(SEED + 1)
    h = RefHarness(3)
    n = 400
    ql, qc, qr = rng.normal(size=n), rng.normal(size=n), rng.normal(size=n)
    ql[:20] = qc[:20]  # flat left side
    nu = rng.uniform(-0.9, 0.9, n)
    data = dict(ql=ql, qc=qc, qr=qr, nu=nu)
    for t in range(9):
        data[f"slope_{t}"] = np.array([h.slope(ql[i], qc[i], qr[i], t, 1.5, nu[i]) for i in range(n)])
    np.savez_compressed(out, **data)


def uniform_cases(out):
    """godunov_fine on small uniform grids from random and Sedov states."""
    data = {}
    rng = np.random.default_rng(SEED + 2)
    cases = [(3, 4, 2, "hllc", 1), (3, 4, 1, "llf", 1), (3, 4, 3, "hll", 2), (3, 4, 7, "acoustic", 3),
             (3, 4, 8, "exact", 1), (1, 7, 1, "hllc", 1), (1, 7, 2, "llf", 2), (1, 7, 4, "exact", 3)]
    for ci, (ndim, L, slope, riem, itype) in enumerate(cases):
        g = rg_tree.build_uniform(ndim, L)
        h = RefHarness(ndim).create(namelist(slope_type=slope, riemann=riem, interpol_type=itype, levelmin=L,
                                             levelmax=L), ngridmax=g.ngridmax, levelmin=L, nlevelmax=L)
        h.refine_uniform(L)
        a = h.arrays()
        u0 = rg_tree.random_state(g, L, seed=int(rng.integers(1 << 30)))
        a["uold"][:] = u0
        a["unew"][:] = u0
        dx = 1.0 / 2 ** L
        dt = 0.5 * h.courant(L, dx, 1.4, 0.8)
        h.set_unew(L)
        h.godunov_fine(L, dt, dx)
        key = f"c{ci}"
        data[f"{key}_meta"] = np.array([ndim, L, slope, ["llf", "hll", "hllc", "exact", "acoustic"].index(riem), itype])
        data[f"{key}_dtdx"] = np.array([dt, dx])
        data[f"{key}_uold"] = u0
        data[f"{key}_unew"] = a["unew"].copy()
        h.close()
    np.savez_compressed(out, **data)


def sod_run(out, nsteps=20):
    """1D Sod tube (64 cells), MinMod + HLLC, the reference's own CFL."""
    ndim, L, gamma = 1, 7, 1.4
    g = rg_tree.build_uniform(ndim, L)
    h = RefHarness(ndim).create(namelist(slope_type=1, riemann="hllc", levelmin=L, levelmax=L), ngridmax=g.ngridmax,
                                levelmin=L, nlevelmax=L)
    h.refine_uniform(L)
    a = h.arrays()
    u0 = rg_tree.sod_state(g, L, gamma)
    a["uold"][:] = u0
    a["unew"][:] = u0
    dx = 1.0 / 2 ** L
    dts = []
    for _ in range(nsteps):
        dt = h.courant(L, dx, gamma, 0.8)
        dts.append(dt)
        h.set_unew(L)
        h.godunov_fine(L, dt, dx)
        h.set_uold(L)
    np.savez_compressed(out, uold0=u0, uold_final=a["uold"].copy(), dts=np.array(dts), meta=np.array([ndim, L]))


def amr_calls(out, ndim, lmin, lmax, ngridmax, ncoarse_steps, slope, riem, keep_levels):
    """Record godunov_fine calls of a sub-cycled AMR Sedov run: tree + state in, unew out."""
    gamma = 1.4
    h = RefHarness(ndim).create(namelist(slope_type=slope, riemann=riem, levelmin=lmin, levelmax=lmax,
                                         err_grad_d=0.1, err_grad_p=0.1), ngridmax=ngridmax, levelmin=lmin,
                                nlevelmax=lmax, gamma=gamma)
    rec = {}
    seen = set()

    def hook(run, il, dt, dx):
        a = run.h.arrays()
        want = il in keep_levels and il not in seen and run.nstep >= 2
        if want:
            g = run.h.grid()
            k = f"L{il}"
            for name in ("son", "father", "nbor", "next", "headl"):
                rec[f"{k}_{name}"] = getattr(g, name).copy()
            rec[f"{k}_uold"] = a["uold"].copy()
            rec[f"{k}_unew_in"] = a["unew"].copy()
            rec[f"{k}_meta"] = np.array([g.ncoarse, g.ngridmax, g.ncell, g.nvar, g.nx, g.ny, g.nz, g.nlevelmax, il])
            rec[f"{k}_dtdx"] = np.array([dt, dx])
        run.h.godunov_fine(il, dt, dx)
        if want:
            rec[f"L{il}_unew_out"] = run.h.arrays()["unew"].copy()
            seen.add(il)

    run = AmrRun(h, lmin, lmax, gamma, ed=0.1, ep=0.1, on_godunov=hook)
    run.initialize(sedov_ic(ndim, lmin, gamma))
    for _ in range(ncoarse_steps):
        run.coarse_step()
    rec["params"] = np.array([ndim, slope, ["llf", "hll", "hllc", "exact", "acoustic"].index(riem)])
    np.savez_compressed(out, **rec)
    h.close()


def tree_digests(out):
    rows = []
    for ndim, L, nx in [(3, 5, 1), (3, 4, 3), (1, 8, 1), (1, 6, 4)]:
        ny = nx if ndim > 1 else 1
        nz = nx if ndim > 2 else 1
        g = rg_tree.build_uniform(ndim, L, nx=nx, ny=ny, nz=nz)
        h = RefHarness(ndim).create(namelist(levelmin=L, levelmax=L), nx=nx, ny=ny, nz=nz, ngridmax=g.ngridmax,
                                    levelmin=L, nlevelmax=L)
        h.refine_uniform(L)
        a = h.arrays()
        dig = hashlib.sha256(b"".join(np.ascontiguousarray(a[k]).tobytes()
                                      for k in ("son", "father", "nbor", "next", "headl", "xg"))).hexdigest()
        rows.append(f"{ndim} {L} {nx} {g.ngridmax} {dig}")
        h.close()
    (out).write_text("\n".join(rows) + "\n")


if __name__ == "__main__":
    riemann_vectors(HERE / "riemann.npz")
    slope_vectors(HERE / "slopes.npz")
    uniform_cases(HERE / "uniform.npz")
    sod_run(HERE / "sod1d.npz")
    amr_calls(HERE / "amr3d.npz", 3, 3, 5, 600, 3, 2, "hllc", {3, 4, 5})
    amr_calls(HERE / "amr1d.npz", 1, 5, 7, 200, 4, 1, "hllc", {5, 6, 7})
    tree_digests(HERE / "tree_digests.txt")
    for p in sorted(HERE.iterdir()):
        print(f"{p.name:22s} {p.stat().st_size:9d} B")
