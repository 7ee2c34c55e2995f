"""Ensembles of independent boxes merged into one forest (rg_ensemble).

CPU: the merge keeps every box closed (ids point inside the box) and the
oracle's level step over the forest's leaf list, with one dt for all boxes,
equals bit for bit the oracle's step of each box alone; the sharding over
ranks covers every box once, and two gloo ranks stepping their shards after a
min-reduction of the CFL step give the one-rank forest's bits (world size 2).
GPU: one substep sequence over a mixed ensemble (edges 16, 24, 32; nx = 1
and 3) through rg_set_level_boxes equals, per box, the oracle run of that box
alone with its own CFL step: same dt bits, same state bits.
"""
import os

import numpy as np
import pytest

import rg_ensemble as ens
from refsupport import GridArrays, Oracle, make_params


def ga_of(g):
    return GridArrays(ncoarse=g.ncoarse, ngridmax=g.ngridmax, ncell=g.ncell, nvar=g.nvar, nx=g.nx, ny=g.ny,
                      nz=g.nz, ncpu=1, nboundary=0, nlevelmax=g.nlevelmax, son=g.son, father=g.father, nbor=g.nbor,
                      next=g.next, headl=g.headl)


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


def specs_of(edges, seed=7):
    pool = ens.box_specs(64, seed=seed)
    out = []
    for e in edges:
        s = next(s for s in pool if s.edge == e and s not in out)
        out.append(s)
    return out


def test_box_specs_follow_the_ensemble_distribution():
    specs = ens.box_specs(512)
    assert len(specs) == 512
    edges = np.array([s.edge for s in specs])
    assert set(edges) == {16, 24, 32, 48, 64}
    for s in specs:
        assert s.edge == s.nx * 2 ** (s.level - 1)
        assert abs(np.linalg.norm(s.normal) - 1) < 1e-12
        for rho, un, p in (s.left, s.right):
            assert 1e-3 <= rho <= 1e3 and 1e-4 <= p <= 1e4 and -3 <= un <= 3
    assert ens.box_specs(512)[17] == specs[17]  # seeded


def test_forest_keeps_boxes_closed():
    f = ens.Forest(specs_of([16, 24, 32, 16]))
    g = f.grid
    V = f.level
    leaf = g.level_octs[V]
    assert len(leaf) == f.first_oct[-1] == sum(len(b.level_octs[s.level]) for s, b in zip(f.specs, f.boxes))
    for b in range(f.nbox):
        lo, hi = f.oct_off[b], f.oct_off[b + 1]
        octs = leaf[f.first_oct[b]:f.first_oct[b + 1]]
        assert np.all((octs > lo) & (octs <= hi))
        # neighbours' father cells stay inside the box: coarse range or the box's octs
        nb = np.stack([g.nbor[k * g.ngridmax + octs - 1] for k in range(6)])
        fine = nb > g.ncoarse
        assert np.all(nb > 0)
        assert np.all((nb[~fine] > f.coarse_off[b]) & (nb[~fine] <= f.coarse_off[b + 1]))
        ig = (nb[fine] - g.ncoarse - 1) % g.ngridmax + 1
        assert np.all((ig > lo) & (ig <= hi))
    # son / father are inverse
    octs = np.arange(1, g.ngridmax + 1)
    assert np.all(g.son[g.father[octs - 1] - 1] == octs)


def test_box_lattices_are_permutations_of_the_level():
    f = ens.Forest(specs_of([16, 24, 32]))
    ext, lat_id, lat_p = f.lattices()
    g = f.grid
    noct = int(f.first_oct[-1])
    assert len(lat_p) == len(lat_id) == noct * 8 == int((ext.prod(axis=1)).sum())
    assert np.array_equal(np.sort(lat_p), np.arange(noct * 8))
    leaf = g.level_octs[f.level]
    icx, k = lat_p // noct, lat_p % noct
    assert np.array_equal(lat_id, g.ncoarse + icx * g.ngridmax + leaf[k])
    # x neighbours inside a box are the +x lattice sites (periodic)
    E = int(ext[0, 0])
    box0 = lat_id[:E ** 3].reshape(E, E, E)  # [z][y][x]
    cid = box0[0, 0, 0]
    ig, ic = (cid - g.ncoarse - 1) % g.ngridmax + 1, (cid - g.ncoarse - 1) // g.ngridmax
    assert ic & 1 == 0 and box0[0, 0, 1] == cid + g.ngridmax  # same oct, x bit set


@pytest.mark.parametrize("edges", [[16, 16, 16], [24, 24]])
def test_forest_step_equals_each_box_alone(edges):
    """Same dx across the forest (the oracle takes one dx per call): the forest's
    leaf-list step with one dt gives every box the bits it gets alone."""
    f = ens.Forest(specs_of(edges, seed=3))
    orc = Oracle()
    params = make_params(3, slope_type=2, riemann="hllc", gamma=f.gamma)
    dx = float(f.dx[0])
    assert np.all(f.dx == dx)
    u0 = f.initial_state()
    ga = ga_of(f.grid)
    dt = 0.5 * min(orc.courant(ga_of(b), 3, 5, s.level, dx, f.gamma, 0.8, f.box_state(i), pressure_cap=False)
                   for i, (s, b) in enumerate(zip(f.specs, f.boxes)))
    uold, unew = u0.copy(), u0.copy()
    orc.godunov_fine(ga, params, f.level, dt, dx, uold, unew)
    for i, (s, b) in enumerate(zip(f.specs, f.boxes)):
        ub = f.box_state(i)
        ubn = ub.copy()
        orc.godunov_fine(ga_of(b), params, s.level, dt, dx, ub, ubn)
        want = ubn.reshape(5, b.ncell)[:, b.cell_ids(s.level) - 1]
        assert bits_equal(f.extract(unew, i), want), i


def _shard_worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    specs = ens.box_specs(512)
    mine = ens.shard_boxes(specs, world)[rank]
    idx = torch.zeros(512, dtype=torch.int64)
    idx[[s.index for s in mine]] = 1
    load = torch.tensor([sum(s.cells for s in mine)], dtype=torch.int64)
    dist.all_reduce(idx)
    loads = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(loads, load)
    if rank == 0:
        np.save(os.path.join(out_dir, "cover.npy"), idx.numpy())
        np.save(os.path.join(out_dir, "loads.npy"), np.array([int(x) for x in loads]))
    dist.destroy_process_group()


def test_sharding_covers_every_box_once_gloo(tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_shard_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    cover = np.load(tmp_path / "cover.npy")
    loads = np.load(tmp_path / "loads.npy")
    assert np.all(cover == 1)
    assert abs(int(loads[0]) - int(loads[1])) <= 64 ** 3
    assert loads.sum() == sum(s.cells for s in ens.box_specs(512))


def _step_forest(f, dt, steps):
    """`steps` oracle level steps of a same-dx forest with one dt; the level
    state of each box (box index -> array) afterwards."""
    orc = Oracle()
    params = make_params(3, slope_type=2, riemann="hllc", gamma=f.gamma)
    ga = ga_of(f.grid)
    dx = float(f.dx[0])
    uold = f.initial_state()
    unew = uold.copy()
    for _ in range(steps):
        orc.set_unew(ga, 3, 5, f.level, uold, unew)
        orc.godunov_fine(ga, params, f.level, dt, dx, uold, unew)
        orc.set_uold(ga, 3, 5, f.level, uold, unew)
    return {s.index: f.extract(uold, i) for i, s in enumerate(f.specs)}


def _forest_dt(f):
    orc = Oracle()
    dx = float(f.dx[0])
    return min(orc.courant(ga_of(b), 3, 5, s.level, dx, f.gamma, 0.8, f.box_state(i), pressure_cap=False)
               for i, (s, b) in enumerate(zip(f.specs, f.boxes)))


def _sharded_step_worker(rank, world, port, out_dir, idx):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    specs = [s for s in ens.box_specs(64, seed=7) if s.index in idx]
    mine = ens.Forest(ens.shard_boxes(specs, world)[rank])
    # the one exchange of the step: the CFL step, min over every rank's boxes
    dt = torch.tensor([_forest_dt(mine)], dtype=torch.float64)
    dist.all_reduce(dt, op=dist.ReduceOp.MIN)
    res = _step_forest(mine, float(dt.item()), 2)
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    if rank == 0:
        merged = {}
        for part in gathered:
            assert not set(part) & set(merged), "a box was stepped on two ranks"
            merged.update(part)
        np.savez(os.path.join(out_dir, "sharded.npz"), dt=float(dt.item()),
                 **{f"b{k}": v for k, v in merged.items()})
    dist.destroy_process_group()


def test_sharded_forest_steps_equal_the_one_rank_forest_gloo(tmp_path):
    """Boxes partitioned over two gloo ranks: each rank steps its shard with the
    oracle after a min-reduction of the CFL step over the ranks; the boxes
    gathered on rank 0 equal, bit for bit, the same boxes stepped as one forest
    on one rank, and the reduced dt equals the one-rank forest's."""
    import socket

    import torch.multiprocessing as mp
    pool = ens.box_specs(64, seed=7)
    idx = [s.index for s in pool if s.edge == 16][:6]  # same dx: the oracle takes one dx per level step
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_sharded_step_worker, args=(2, port, str(tmp_path), idx), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(tmp_path / "sharded.npz")
    whole = ens.Forest([s for s in pool if s.index in idx])
    dt = _forest_dt(whole)
    assert float(got["dt"]) == dt
    want = _step_forest(whole, dt, 2)
    assert sorted(int(k[1:]) for k in got.files if k.startswith("b")) == sorted(want)
    for k, v in want.items():
        assert bits_equal(got[f"b{k}"], v), k


@pytest.mark.gpu
@pytest.mark.parametrize("bricks", [False, True])
def test_ensemble_substeps_match_each_box_alone(rgpu_lib, bricks):
    """Tiled face kernel, or (bricks) the brick kernel over the boxes' lattices."""
    import rgpu
    specs = specs_of([16, 24, 32, 16, 24, 32, 16], seed=11)
    f = ens.Forest(specs)
    orc = Oracle()
    gamma = f.gamma
    params = rgpu.make_params(3, slope_type=2, riemann="hllc", gamma=gamma, courant_factor=0.8)
    ctx = rgpu.Context(params, 0)
    try:
        ctx.sync_topology(f.grid)
        u0 = f.initial_state()
        ctx.upload_state(u0, u0)
        ctx.set_level_boxes(f.level, f.first_oct, f.dx)
        if bricks:
            ctx.set_level_lattices(f.level, *f.lattices())
            ctx.set_face_config(f.level, 9, 1)
        nsteps = 3
        dts = []
        for k in range(nsteps):
            ctx.level_substep(f.level, 0.0, pressure_cap=False, use_graph=(k > 0))
            dts.append(ctx.level_box_dt(f.level, f.nbox))
        got = np.empty_like(u0)
        ctx.download_state(uold=got)
    finally:
        ctx.close()
    op = make_params(3, slope_type=2, riemann="hllc", gamma=gamma)
    for i, (s, b) in enumerate(zip(f.specs, f.boxes)):
        ga = ga_of(b)
        uold = f.box_state(i)
        unew = uold.copy()
        for k in range(nsteps):
            dt = orc.courant(ga, 3, 5, s.level, s.dx, gamma, 0.8, uold, pressure_cap=False)
            assert dt == dts[k][i], (i, k, dt, dts[k][i])
            orc.set_unew(ga, 3, 5, s.level, uold, unew)
            orc.godunov_fine(ga, op, s.level, dt, s.dx, uold, unew)
            orc.set_uold(ga, 3, 5, s.level, uold, unew)
        want = uold.reshape(5, b.ncell)[:, b.cell_ids(s.level) - 1]
        assert bits_equal(f.extract(got, i), want), i


@pytest.mark.gpu
def test_wrong_lattice_map_is_rejected(rgpu_lib):
    import rgpu
    f = ens.Forest(specs_of([16, 24], seed=5))
    ctx = rgpu.Context(rgpu.make_params(3, slope_type=2, riemann="hllc", gamma=f.gamma), 0)
    try:
        ctx.sync_topology(f.grid)
        u0 = f.initial_state()
        ctx.upload_state(u0, u0)
        ctx.set_level_boxes(f.level, f.first_oct, f.dx)
        ext, lat_id, lat_p = f.lattices()
        bad_p = lat_p.copy()
        bad_p[[5, 6]] = bad_p[[6, 5]]          # two sites swapped: positions no longer hold their cells
        with pytest.raises(rgpu.RGError) as e:
            ctx.set_level_lattices(f.level, ext, lat_id, bad_p)
        assert e.value.code == rgpu.RG_ERR_ARG
        bad_id = lat_id.copy()
        bad_id[:16 ** 3] = np.roll(bad_id[:16 ** 3].reshape(16, 16, 16), 1, axis=2).reshape(-1)
        with pytest.raises(rgpu.RGError):
            ctx.set_level_lattices(f.level, ext, bad_id, lat_p)
        ctx.set_level_lattices(f.level, ext, lat_id, lat_p)  # the right maps are still accepted
        ctx.level_substep(f.level, 0.0, use_graph=False)
        ctx.synchronize()
    finally:
        ctx.close()
