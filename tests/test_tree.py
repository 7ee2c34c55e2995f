"""Host-side tree builder (ramses-cpp_b200/rg_tree.py) against the reference:
integer arrays of the uniform grid must be bit-identical."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

import rg_tree

GOLDEN = Path(__file__).resolve().parent / "golden" / "tree_digests.txt"


def _digest(g):
    return hashlib.sha256(b"".join(np.ascontiguousarray(getattr(g, k)).tobytes()
                                   for k in ("son", "father", "nbor", "next", "headl", "xg"))).hexdigest()


def test_uniform_tree_matches_reference_digests():
    rows = [r.split() for r in GOLDEN.read_text().splitlines() if r.strip()]
    assert len(rows) >= 4
    for ndim, L, nx, ngm, dig in rows:
        ndim, L, nx, ngm = int(ndim), int(L), int(nx), int(ngm)
        g = rg_tree.build_uniform(ndim, L, nx=nx, ny=nx if ndim > 1 else 1, nz=nx if ndim > 2 else 1)
        assert g.ngridmax == ngm
        assert _digest(g) == dig, (ndim, L, nx)


def test_uniform_tree_matches_reference_live(reference_available):
    if not reference_available:
        pytest.skip("reference sources not present")
    from refsupport import RefHarness, namelist
    for ndim, L, nx, extra in [(3, 4, 1, 0), (3, 3, 2, 17), (1, 7, 1, 5), (1, 5, 3, 0)]:
        ny, nz = (nx if ndim > 1 else 1), (nx if ndim > 2 else 1)
        g0 = rg_tree.build_uniform(ndim, L, nx=nx, ny=ny, nz=nz)
        g = rg_tree.build_uniform(ndim, L, nx=nx, ny=ny, nz=nz, ngridmax=g0.ngridmax + extra)
        h = RefHarness(ndim).create(namelist(levelmin=L, levelmax=L), nx=nx, ny=ny, nz=nz, ngridmax=g.ngridmax,
                                    levelmin=L, nlevelmax=L)
        h.refine_uniform(L)
        a = h.arrays()
        for k in ("son", "father", "nbor", "next", "headl", "xg"):
            assert np.array_equal(a[k], getattr(g, k)), (ndim, L, nx, k)
        ids = g.cell_ids(L)
        assert np.array_equal(h.cell_centers(ids[:64]), g.cell_centers(L)[:64])
        h.close()


def test_cell_counts_and_layout():
    g = rg_tree.build_uniform(3, 5)
    assert len(g.level_octs[5]) == 8 ** 3 and len(g.cell_ids(5)) == 16 ** 3
    c = g.cell_centers(5)
    assert np.allclose(np.sort(np.unique(c[:, 0])), (np.arange(16) + 0.5) / 16)
