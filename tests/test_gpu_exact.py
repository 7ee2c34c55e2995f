"""Exact Riemann solver and its learned Newton start on the GPU.

- reference mode (10 iterations, 1e-6) against the oracle on the stress
  workload: fluxes within 3e-12 (pow() differs by ulps between libm and CUDA);
- the tensor-core training kernel's gradients against an FP64 CPU mirror of
  the same network with the same BF16 roundings;
- training is reproducible: two contexts trained with the same seed hold the
  same parameter bits (the gradient is reduced in a fixed order);
- the learned start reaches the same converged root (|dp|/p <= 1e-13) with
  fewer Newton updates on the stress workload, and does not add updates
  where the two-shock start is already exact (the level step on Sedov).
"""
import numpy as np
import pytest

import rg_tree
import rgpu
from refsupport import make_params

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx(rgpu_lib):
    c = rgpu.Context(rgpu.make_params(3, riemann="exact"), 0)
    s = torch.cuda.Stream()
    c.set_stream(s.cuda_stream)
    yield c
    c.close()


def stress(ctx, n, seed):
    ql = torch.empty(5 * n, dtype=torch.float64, device="cuda")
    qr = torch.empty_like(ql)
    g = torch.empty(n, dtype=torch.float64, device="cuda")
    ctx.stress_states(n, seed, ql.data_ptr(), qr.data_ptr(), g.data_ptr())
    ctx.synchronize()
    return ql, qr, g


def solve(ctx, n, ql, qr, g, learned, niter, tol):
    f = torch.empty(5 * n, dtype=torch.float64, device="cuda")
    ps = torch.empty(n, dtype=torch.float64, device="cuda")
    it = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.exact_batch(n, ql.data_ptr(), qr.data_ptr(), g.data_ptr(), f.data_ptr(), ps.data_ptr(), it.data_ptr(),
                    learned=learned, niter=niter, tol=tol)
    ctx.synchronize()
    return f.cpu().numpy().reshape(5, n), ps.cpu().numpy(), it.cpu().numpy()


def test_reference_mode_matches_oracle(ctx, oracle):
    n = 4096
    ql, qr, g = stress(ctx, n, 99)
    f, ps, it = solve(ctx, n, ql, qr, g, False, 10, 1e-6)
    a, b, gam = ql.cpu().numpy().reshape(5, n), qr.cpu().numpy().reshape(5, n), g.cpu().numpy()
    want = np.array([oracle.riemann("exact", a[:, i], b[:, i], gam[i], 3)[:5] for i in range(n)]).T
    scale = np.maximum(np.abs(want), 1e-300)
    rel = np.abs(f - want) / scale
    ok = (rel <= 3e-12) | (np.abs(f - want) <= 3e-12 * np.abs(want).max(axis=0, keepdims=True) * 1e-6)
    assert ok.mean() > 0.9999, f"{np.count_nonzero(~ok)} of {ok.size} flux entries beyond 3e-12"
    assert np.isfinite(f).all()


def _bf16(a):
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def cpu_grads(p, x, t):
    """FP64 mirror of the training kernel (same BF16 roundings, same loss)."""
    W1 = p[0:512].reshape(64, 8)
    b1 = p[512:576]
    W2 = p[576:4672].reshape(64, 64)
    b2 = p[4672:4736]
    w3 = p[4736:4800]
    b3 = p[4800]
    n = len(t)
    xb = _bf16(x.T)
    W1b, W2b = _bf16(W1), _bf16(W2)
    Z1 = xb @ W1b.T + b1
    H1b = _bf16(_silu(Z1))
    Z2 = H1b @ W2b.T + b2
    H2 = _silu(Z2)
    y = H2 @ w3 + b3
    e = y - t
    dy = 2 * e / n
    dZ2 = dy[:, None] * w3[None, :] * _dsilu(Z2)
    dH1 = _bf16(dZ2) @ W2b
    dZ1 = dH1 * _dsilu(Z1)
    g = np.concatenate([(dZ1.T @ xb).ravel(), dZ1.sum(0), (dZ2.T @ H1b).ravel(), dZ2.sum(0), H2.T @ dy, [dy.sum()]])
    return g, float((e ** 2).sum())


def test_training_gradients_match_fp64_cpu(ctx):
    rng = np.random.default_rng(5)
    nparam = 4820
    p = np.zeros(nparam, dtype=np.float32)
    p[:4801] = rng.normal(0, 0.3, 4801)
    p[4801 + 8:4801 + 16] = 1.0  # feature scales
    p[4818] = 1.0                # target scale
    p[4819] = 0.2                # gate
    ctx.mlp_set(p)
    n = 1000  # not a multiple of the 64-sample tile: exercises the masking
    x = rng.normal(0, 1, (8, n)).astype(np.float32)
    t = rng.normal(0, 1, n).astype(np.float32)
    g_gpu, loss_gpu = ctx.mlp_grad(x, t)
    g_cpu, loss_cpu = cpu_grads(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss_gpu - loss_cpu) <= 2e-3 * loss_cpu
    blocks = {"W1": (0, 512), "b1": (512, 576), "W2": (576, 4672), "b2": (4672, 4736), "w3": (4736, 4800),
              "b3": (4800, 4801)}
    for name, (a, b) in blocks.items():
        gg, gc = g_gpu[a:b].astype(np.float64), g_cpu[a:b]
        err = np.linalg.norm(gg - gc) / max(np.linalg.norm(gc), 1e-30)
        cos = gg @ gc / max(np.linalg.norm(gg) * np.linalg.norm(gc), 1e-30)
        assert err < 2e-2 and cos > 0.9995, f"{name}: rel err {err:.2e}, cosine {cos:.6f}"


def test_training_is_reproducible(ctx):
    ws = []
    for _ in range(2):
        c = rgpu.Context(rgpu.make_params(3, riemann="exact"), 0)
        try:
            c.mlp_train(nsamples=1 << 20, epochs=2, seed=9)
            ws.append(c.mlp_get())
        finally:
            c.close()
    assert np.array_equal(ws[0].view(np.int32), ws[1].view(np.int32))


def test_converged_mode_matches_oracle(ctx, oracle):
    """Converged mode (100 updates, 1e-14) against the C oracle's same
    bracketed iteration and polish: same root to 1e-13 on every pair, no pair
    at the cap; fluxes within 3e-12 (the cube and pow() differ by ulps
    between libm and CUDA)."""
    n = 4096
    ql, qr, g = stress(ctx, n, 77)
    f, ps, it = solve(ctx, n, ql, qr, g, False, 100, 1e-14)
    a, b, gam = ql.cpu().numpy().reshape(5, n), qr.cpu().numpy().reshape(5, n), g.cpu().numpy()
    want_p = np.empty(n)
    want_f = np.empty((5, n))
    for i in range(n):
        want_f[:, i], want_p[i] = oracle.exact_pstar(a[:, i], b[:, i], gam[i], 3, 100, 1e-14)
    assert it.max() < 100, "a pair reached the iteration cap"
    rel = np.abs(ps - want_p) / np.maximum(np.abs(want_p), 1e-300)
    assert rel.max() <= 1e-13, rel.max()
    scale = np.maximum(np.abs(want_f), 1e-300)
    frel = np.abs(f - want_f) / scale
    assert np.mean(frel <= 3e-12) > 0.9999, np.count_nonzero(frel > 3e-12)


def test_learned_start_same_root_fewer_iterations(ctx):
    """Converged mode: from the plain and from the learned start every pair
    converges inside the cap, to the same p* bits and the same flux bits (the
    polish from the root's 30 leading bits takes the start out of the
    result), with fewer Newton updates from the learned start."""
    loss = ctx.mlp_train(seed=3)
    assert np.isfinite(loss) and loss < 0.02
    n = 1 << 20
    ql, qr, g = stress(ctx, n, 2026)  # held out: another seed than training
    f0, p0, i0 = solve(ctx, n, ql, qr, g, False, 100, 1e-14)
    f1, p1, i1 = solve(ctx, n, ql, qr, g, True, 100, 1e-14)
    assert i0.max() < 100 and i1.max() < 100, "a pair reached the iteration cap"
    assert i1.mean() < 0.8 * i0.mean(), (i0.mean(), i1.mean())
    rel = np.abs(p1 - p0) / np.maximum(np.abs(p0), 1e-300)
    assert np.count_nonzero(rel > 1e-13) == 0, rel.max()
    frel = np.abs(f1 - f0) / np.maximum(np.abs(f0), 1e-300)
    assert np.count_nonzero(frel > 1e-12) == 0, frel.max()


def test_level_step_with_learned_start(ctx):
    """Sedov 32^3 with the exact solver in converged mode: the learned start
    changes the Newton path, not the result (1e-12).  Almost every Sedov
    interface is a weak wave whose two-shock start is already exact, so the
    gate must keep that start and the update count must not grow."""
    ctx.mlp_train(seed=4)
    w = ctx.mlp_get()
    L = 6
    g = rg_tree.build_uniform(3, L)
    u = rg_tree.sedov_state(g, L)
    dx = 1.0 / 2 ** L
    out, its = {}, {}
    for learned in (False, True):
        c = rgpu.Context(make_params(3, slope_type=2, riemann="exact", exact_niter=100, exact_tol=1e-14,
                                     exact_guess=1 if learned else 0), 0)
        if learned:
            c.mlp_set(w)
        c.sync_topology(g)
        c.upload_state(u, u)
        c.exact_stats(reset=True)
        for _ in range(3):
            c.godunov_level(L, 1e-5, dx)
        c.synchronize()
        its[learned] = c.exact_stats()
        r = np.empty_like(u)
        c.download_state(unew=r)
        out[learned] = r
        c.close()
    a, b = out[False], out[True]
    rel = np.abs(a - b) / np.maximum(np.abs(a), 1e-300)
    assert rel.max() < 1e-12
    (i0, c0), (i1, c1) = its[False], its[True]
    # near-uniform Sedov interfaces keep their (exact) two-shock start
    assert c0 == c1 and i1 <= 1.02 * i0
