"""Weighted PageRank and its implicit adjoint (no reference counterpart).

Checked against: the FP64 restatement (oracle), a dense FP64 solve of (I - d P^T) r = (1-d) w
and (I - d P) lambda = c at small scale, and FP64 central finite differences of the GPU
forward on random edges.  Tolerance 1e-6 relative for gradients.  The forward/adjoint pair is
also wrapped in a torch.autograd.Function here (and only here) for torch.autograd.gradcheck and
autograd gradients against the dense solve.
"""
import numpy as np
import pytest

import graphine_b200.gre as G
import oracle as O
from conftest import rel_l1

pytestmark = pytest.mark.gpu
D = 0.85


def weighted_graph(scale, seed, directed=False, reorder=False):
    n, off, col = G.rmat_host(scale, 16, seed, not directed)
    rng = np.random.default_rng(seed)
    w = np.exp(rng.standard_normal(len(col)))  # lognormal(0, 1) per arc
    g = G.Graph.from_csr(n, off, col, dir=G.InOut if not directed else G.Out, symmetric=not directed, reorder=reorder)
    g.set_weights_f64(w)
    return n, off, col, w, g


def dense_P(n, off, col, w):
    P = np.zeros((n, n))
    src = np.repeat(np.arange(n), np.diff(off.astype(np.int64)))
    np.add.at(P, (src, col.astype(np.int64)), w)
    s = P.sum(axis=1)
    nz = s > 0
    P[nz] /= s[nz][:, None]
    return P


@pytest.mark.parametrize("reorder", [False, True], ids=["plain", "relabelled"])
def test_weighted_forward_and_adjoint_vs_dense_solve(reorder):
    """The differentiation config's dense check: a directed RMAT-12 graph (4096 vertices) with
    lognormal weights, forward and adjoint against LU solves of the dense FP64 systems."""
    n, off, col, w, g = weighted_graph(12, 3, directed=True, reorder=reorder)
    rng = np.random.default_rng(1)
    pers = rng.random(n) + 0.5
    c = rng.standard_normal(n)
    r, st, status = G.pagerank_weighted(g, D, pers, tol=1e-15, max_iters=2000)
    assert status == G.GRE_SUCCESS
    P = dense_P(n, off, col, w)
    I = np.eye(n)
    r_ref = np.linalg.solve(I - D * P.T, (1 - D) * pers)
    assert rel_l1(r, r_ref) <= 1e-10
    lam, gp, gw, st, status = G.pagerank_adjoint(g, r, c, D, tol=1e-15, max_iters=2000)
    lam_ref = np.linalg.solve(I - D * P, c)
    assert rel_l1(lam, lam_ref) <= 1e-10
    assert rel_l1(gp, (1 - D) * lam_ref) <= 1e-10
    src = np.repeat(np.arange(n), np.diff(off.astype(np.int64)))
    s = np.bincount(src, weights=w, minlength=n)
    pl = P @ lam_ref
    gw_ref = D * r_ref[src] / s[src] * (lam_ref[col] - pl[src])
    assert rel_l1(gw, gw_ref) <= 1e-8


@pytest.mark.parametrize("reorder", [False, True], ids=["plain", "relabelled"])
def test_adjoint_vs_oracle_restatement(reorder):
    n, off, col, w, g = weighted_graph(12, 5, reorder=reorder)
    rng = np.random.default_rng(2)
    pers = np.ones(n)
    c = rng.standard_normal(n)
    R = O.Restatement.from_csr(n, off, col)
    r_ref = R.pagerank_weighted(w, pers, D, 400)
    r, _, _ = G.pagerank_weighted(g, D, None, tol=1e-15, max_iters=2000)
    assert rel_l1(r, r_ref) <= 1e-9
    lam_ref, gp_ref, gw_ref = R.pagerank_adjoint(w, r_ref, c, D, 400)
    lam, gp, gw, _, _ = G.pagerank_adjoint(g, r, c, D, tol=1e-15, max_iters=2000)
    assert rel_l1(lam, lam_ref) <= 1e-9
    assert rel_l1(gp, gp_ref) <= 1e-9
    assert rel_l1(gw, gw_ref) <= 1e-6


def test_adjoint_vs_central_differences():
    n, off, col, w, g = weighted_graph(12, 9)
    rng = np.random.default_rng(4)
    c = rng.standard_normal(n)
    r, _, _ = G.pagerank_weighted(g, D, None, tol=1e-15, max_iters=3000)
    lam, gp, gw, _, _ = G.pagerank_adjoint(g, r, c, D, tol=1e-15, max_iters=3000)
    h = 1e-6
    edges = rng.choice(len(col), size=40, replace=False)
    fd = []
    for a in edges:
        vals = []
        for sgn in (+1, -1):
            w2 = w.copy()
            w2[a] += sgn * h
            g.set_weights_f64(w2)
            r2, _, _ = G.pagerank_weighted(g, D, None, tol=1e-16, max_iters=3000)
            vals.append(float(c @ r2))
        fd.append((vals[0] - vals[1]) / (2 * h))
    g.set_weights_f64(w)
    fd = np.array(fd)
    err = np.abs(fd - gw[edges]).max() / max(np.abs(gw[edges]).max(), 1e-300)
    assert err <= 1e-4, err  # FD noise ~ eps*|L|/h dominates below this
    # personalisation gradient: L is linear in pers, dL/dpers = (1-d) lambda exactly
    e = int(rng.integers(n))
    p1 = np.ones(n)
    p1[e] += 1.0
    r1, _, _ = G.pagerank_weighted(g, D, p1, tol=1e-16, max_iters=3000)
    assert abs(float(c @ r1) - float(c @ r) - gp[e]) <= 1e-9 * max(1.0, abs(gp[e]))


def _pagerank_function():
    """The adjoint behind a torch.autograd.Function (gradient-check harness only): forward sets
    the arc weights and solves the weighted PageRank on the GPU, backward solves the transposed
    fixed point with the incoming gradient as c (gre_pagerank_adjoint)."""
    import torch

    class WeightedPageRank(torch.autograd.Function):
        @staticmethod
        def forward(ctx, w, pers, g):
            wd = w.detach().cpu().contiguous()
            g.set_weights_f64(wd.numpy())
            r, _, _ = G.pagerank_weighted(g, D, pers.detach().cpu().numpy(), tol=1e-16, max_iters=5000)
            ctx.g = g
            ctx.save_for_backward(wd.clone(), torch.from_numpy(r.copy()))
            return torch.from_numpy(r.copy())

        @staticmethod
        def backward(ctx, grad_r):
            wd, r = ctx.saved_tensors
            ctx.g.set_weights_f64(wd.numpy())  # other forward calls may have changed the graph's weights
            _, gp, gw, _, _ = G.pagerank_adjoint(ctx.g, r.numpy(), grad_r.contiguous().numpy(), D, tol=1e-16,
                                                 max_iters=5000)
            return torch.from_numpy(gw.copy()), torch.from_numpy(gp.copy()), None

    return WeightedPageRank


def test_autograd_function_gradcheck():
    """torch.autograd.gradcheck of the wrapped forward/adjoint pair (FP64 central differences on
    every arc weight and personalisation entry of a small weighted graph)."""
    import torch

    n, off, col, w, g = weighted_graph(5, 13, directed=True)
    fn = _pagerank_function()
    wt = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    pers = torch.tensor(np.random.default_rng(3).random(n) + 0.5, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda a, b: fn.apply(a, b, g), (wt, pers), eps=1e-6, atol=1e-7, rtol=1e-5)


def test_autograd_function_matches_dense_gradient():
    import torch

    n, off, col, w, g = weighted_graph(9, 21)
    fn = _pagerank_function()
    rng = np.random.default_rng(8)
    c = torch.tensor(rng.standard_normal(n))
    wt = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    pers = torch.ones(n, dtype=torch.float64, requires_grad=True)
    loss = (c * fn.apply(wt, pers, g)).sum()
    gw, gp = torch.autograd.grad(loss, (wt, pers))
    P = dense_P(n, off, col, w)
    I = np.eye(n)
    r_ref = np.linalg.solve(I - D * P.T, (1 - D) * np.ones(n))
    lam = np.linalg.solve(I - D * P, c.numpy())
    src = np.repeat(np.arange(n), np.diff(off.astype(np.int64)))
    s = np.bincount(src, weights=w, minlength=n)
    gw_ref = D * r_ref[src] / s[src] * (lam[col] - (P @ lam)[src])
    assert rel_l1(gw.numpy(), gw_ref) <= 1e-6
    assert rel_l1(gp.numpy(), (1 - D) * lam) <= 1e-6


def test_adjoint_vs_central_differences_s20_1000_edges():
    """The differentiation config as stated: RMAT-20 (EF16, symmetric, relabelled) with lognormal
    (0, 1) arc weights, L = c . r with c ~ N(0, 1); dL/dW on 1000 random arcs against FP64 central
    differences with h = 1e-6.

    The gradient comes from converged solves (tol = 0, 230 Jacobi steps: 0.85^230 < 1e-16).  Both
    solves of a difference run the same fixed 150 steps, so they take the same summation path
    (the 150-step map's derivative differs from the fixed point's by about 150 * 0.85^150 < 1e-8
    relative), and
    L(w+h) - L(w-h) is formed as c . (r+ - r-) so that no large sum cancels.  What is left is
    rounding noise in r (a few ulps per vertex, uncorrelated between vertices) carried into the
    difference quotient: noise ~ eps * ||c * r||_2 / h.  The per-arc tolerance is 64x that floor
    plus 1e-5 relative (the O(h^2) truncation term is below 1e-10 relative here)."""
    import torch

    n, off, col = G.rmat_host(20, 16, 41, True)
    rng = np.random.default_rng(41)
    w = np.exp(rng.standard_normal(len(col)))
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True, reorder=True)
    dev = torch.device("cuda", 0)
    wd = torch.tensor(w, dtype=torch.float64, device=dev)
    g.set_weights_f64(wd)
    c = rng.standard_normal(n)
    steps, fd_steps = 230, 150
    r = torch.empty(n, dtype=torch.float64, device=dev)
    G.pagerank_weighted(g, D, None, tol=0.0, max_iters=steps, out=r)
    r_h = r.cpu().numpy()
    _, _, gw, _, _ = G.pagerank_adjoint(g, r_h, c, D, tol=0.0, max_iters=steps)
    h = 1e-6
    arcs = rng.choice(len(col), size=1000, replace=False)
    ct = torch.tensor(c, dtype=torch.float64, device=dev)
    rp, rm = torch.empty_like(r), torch.empty_like(r)
    fd = np.empty(len(arcs))
    for i, a in enumerate(arcs):
        a = int(a)
        base = float(w[a])
        wd[a] = base + h
        g.set_weights_f64(wd)
        G.pagerank_weighted(g, D, None, tol=0.0, max_iters=fd_steps, out=rp)
        wd[a] = base - h
        g.set_weights_f64(wd)
        G.pagerank_weighted(g, D, None, tol=0.0, max_iters=fd_steps, out=rm)
        wd[a] = base
        fd[i] = float(torch.dot(ct, rp - rm)) / (2 * h)
    g.set_weights_f64(wd)
    eps = np.finfo(np.float64).eps
    floor = eps * float(np.linalg.norm(c * r_h)) / h
    tol = 64 * floor + 1e-5 * np.abs(gw[arcs])
    err = np.abs(fd - gw[arcs])
    assert np.all(err <= tol), (float(err.max()), float(floor), int(np.argmax(err / tol)))
    assert rel_l1(fd, gw[arcs]) <= 1e-4, rel_l1(fd, gw[arcs])
