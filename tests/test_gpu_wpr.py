"""Differentiable weighted PageRank: forward/backward C-ABI pair, wrapped in a
torch.autograd.Function here (the harness only), checked against the FP64
oracle, an FP64 dense solve and FP64 central finite differences on scale-10
instances of the generator."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
ALPHA = 0.85
ITERS = 160


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def ob():
    import olive_b200
    return olive_b200


def make_problem(scale, seed):
    rp, cl = oracle.rmat_csr(scale, 16, seed)
    rng = np.random.default_rng(seed)
    E, V = len(cl), len(rp) - 1
    w = rng.lognormal(0.0, 1.0, E).astype(np.float32)
    p = rng.exponential(1.0, V)
    p = (p / p.sum()).astype(np.float32)          # Dirichlet(1)
    g = rng.standard_normal(V).astype(np.float32)
    return rp, cl, w, p, g


def wpr_function(torch):
    class WeightedPageRank(torch.autograd.Function):
        """r = WPR(w, p); backward through olv_wpr_backward (implicit adjoint)."""

        @staticmethod
        def forward(ctx, w, p, graph, iters):
            r = torch.empty(graph.V, dtype=torch.float32, device="cuda")
            graph.wpr_forward(p.contiguous(), w=w.contiguous(), alpha=ALPHA, max_it=iters,
                              out=r)
            ctx.graph, ctx.iters = graph, iters
            return r

        @staticmethod
        def backward(ctx, grad_r):
            g = ctx.graph
            dw = torch.empty(g.E, dtype=torch.float32, device="cuda")
            dp = torch.empty(g.V, dtype=torch.float32, device="cuda")
            g.wpr_backward(grad_r.contiguous(), max_it=ctx.iters, dw_out=dw, dp_out=dp)
            return dw, dp, None, None

    return WeightedPageRank


def rel_inf(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


# Gradient tolerance.  Normwise: max|d| / max|ref| and ||d||_2 / ||ref||_2 both
# below 1e-5.  Per element: |d_e| <= 1e-5 (|ref_e| + s_e) + 1e-7 max|ref|, where
# s_e is the size of the terms whose difference the entry is: for dL/dw_uv =
# alpha r_u (lambda_v - t_u) / W_u it is alpha r_u (|lambda_v| + |t_u|) / W_u,
# for dL/dp_v = (1 - alpha) lambda_v = (1 - alpha)(g_v + alpha t_v) it is
# (1 - alpha)(|g_v| + alpha |t_v|) (t = P lambda).  The s_e term covers entries
# that cancel exactly in FP64 (a row with one out-edge has t_u = lambda_v) and
# are left with FP32 rounding of the two terms; the 1e-7 max|ref| floor (under
# two FP32 units of roundoff at the largest entry's scale) covers entries whose
# error comes from the rounding of their neighbours' adjoints.  An FP32
# emulation of the solver puts 99.7-99.9% of the entries within 1e-5 relative
# with neither term.
GRAD_RTOL = 1e-5
GRAD_FLOOR = 1e-7


def operand_scales(rp, cl, w, r, g, lam):
    """s_e for dL/dw (per CSR edge) and dL/dp (per vertex), from FP64 r and lambda."""
    V = len(rp) - 1
    src = np.repeat(np.arange(V), np.diff(rp.astype(np.int64)))
    w64 = np.asarray(w, np.float64)
    W = np.bincount(src, w64, V)
    t = np.bincount(src, w64 * lam[cl], V) / np.where(W > 0, W, 1.0)
    s_w = ALPHA * r[src] * (np.abs(lam[cl]) + np.abs(t[src])) / W[src]
    s_p = (1 - ALPHA) * (np.abs(np.asarray(g, np.float64)) + ALPHA * np.abs(t))
    return s_w, s_p


def assert_grad_close(got, ref, what, scale=None):
    got = np.asarray(got, np.float64)
    assert rel_inf(got, ref) < GRAD_RTOL, (what, rel_inf(got, ref))
    assert np.linalg.norm(got - ref) < GRAD_RTOL * np.linalg.norm(ref), what
    d = np.abs(got - ref)
    tol = GRAD_RTOL * (np.abs(ref) + (0.0 if scale is None else scale)) + \
        GRAD_FLOOR * np.max(np.abs(ref))
    bad = np.flatnonzero(d > tol)
    assert len(bad) == 0, (what, len(bad), bad[:5], d[bad[:5]], ref[bad[:5]])


@pytest.mark.parametrize("seed", [1, 2])
def test_forward_backward_vs_fp64_oracle(ob, seed):
    rp, cl, w, p, g = make_problem(10, seed)
    with ob.Graph.from_csr(rp, cl) as G:
        r = G.wpr_forward(p, w=w, alpha=ALPHA, max_it=ITERS)
        r_ref = oracle.wpr_forward(rp, cl, w.astype(np.float64), p.astype(np.float64), ALPHA,
                                   ITERS)
        assert rel_inf(r.astype(np.float64), r_ref) < 1e-5
        dw, dp = G.wpr_backward(g, max_it=ITERS)
        lam, dw_ref, dp_ref = oracle.wpr_backward(rp, cl, w.astype(np.float64), r_ref,
                                                  g.astype(np.float64), ALPHA, ITERS)
        s_w, s_p = operand_scales(rp, cl, w, r_ref, g, lam)
        assert_grad_close(dw, dw_ref, "dw", s_w)
        assert_grad_close(dp, dp_ref, "dp", s_p)


def test_dense_solve_and_finite_differences(ob):
    rp, cl, w, p, g = make_problem(10, 3)
    V, E = len(rp) - 1, len(cl)
    deg = np.diff(rp.astype(np.int64))
    src = np.repeat(np.arange(V), deg)
    w64 = w.astype(np.float64)
    W = np.zeros(V)
    np.add.at(W, src, w64)
    P = np.zeros((V, V))
    np.add.at(P, (src, cl.astype(np.int64)), w64 / W[src])
    r_dense = np.linalg.solve(np.eye(V) - ALPHA * P.T, (1 - ALPHA) * p.astype(np.float64))
    lam_dense = np.linalg.solve(np.eye(V) - ALPHA * P, g.astype(np.float64))
    Plam = P @ lam_dense
    dw_dense = ALPHA * r_dense[src] * (lam_dense[cl] - Plam[src]) / W[src]
    with ob.Graph.from_csr(rp, cl) as G:
        r = G.wpr_forward(p, w=w, alpha=ALPHA, max_it=ITERS)
        dw, dp = G.wpr_backward(g, max_it=ITERS)
    assert rel_inf(r.astype(np.float64), r_dense) < 1e-5
    s_w, s_p = operand_scales(rp, cl, w, r_dense, g, lam_dense)
    assert_grad_close(dw, dw_dense, "dw vs dense solve", s_w)
    assert_grad_close(dp, (1 - ALPHA) * lam_dense, "dp vs dense solve", s_p)
    # FP64 central differences of L(w) = g . r(w) on the largest gradients
    for e in np.argsort(-np.abs(dw_dense))[:6]:
        h = 1e-5 * w64[e]
        wp_, wm_ = w64.copy(), w64.copy()
        wp_[e] += h
        wm_[e] -= h
        rp_ = np.linalg.solve(np.eye(V) - ALPHA * _P(src, cl, wp_, V).T, (1 - ALPHA) * p)
        rm_ = np.linalg.solve(np.eye(V) - ALPHA * _P(src, cl, wm_, V).T, (1 - ALPHA) * p)
        fd = (g.astype(np.float64) @ (rp_ - rm_)) / (2 * h)
        assert abs(dw[e] - fd) <= 1e-4 * abs(fd) + 1e-9, (e, dw[e], fd)


def _P(src, cl, w, V):
    W = np.zeros(V)
    np.add.at(W, src, w)
    P = np.zeros((V, V))
    np.add.at(P, (src, cl.astype(np.int64)), w / W[src])
    return P


def test_autograd_function(torch, ob):
    rp, cl, w, p, g = make_problem(10, 4)
    Fn = wpr_function(torch)
    with ob.Graph.from_csr(rp, cl) as G:
        wt = torch.tensor(w, device="cuda", requires_grad=True)
        pt = torch.tensor(p, device="cuda", requires_grad=True)
        gt = torch.tensor(g, device="cuda")
        r = Fn.apply(wt, pt, G, ITERS)
        loss = (gt * r).sum()
        loss.backward()
        r_ref = oracle.wpr_forward(rp, cl, w.astype(np.float64), p.astype(np.float64), ALPHA,
                                   ITERS)
        lam, dw_ref, dp_ref = oracle.wpr_backward(rp, cl, w.astype(np.float64), r_ref,
                                                  g.astype(np.float64), ALPHA, ITERS)
        s_w, s_p = operand_scales(rp, cl, w, r_ref, g, lam)
        assert_grad_close(wt.grad.cpu().numpy(), dw_ref, "autograd dw", s_w)
        assert_grad_close(pt.grad.cpu().numpy(), dp_ref, "autograd dp", s_p)
        assert abs(loss.item() - float(g.astype(np.float64) @ r_ref)) < 1e-5 * abs(loss.item()) + 1e-7


def test_deterministic_and_dangling_rows(ob):
    # a graph with dangling vertices (rows without out-edges)
    rp, cl = oracle.grid_csr(8, 8)
    rp = rp.copy()
    keep = np.ones(len(cl), bool)
    keep[rp[5]:rp[6]] = False          # vertex 5 has no out-edges
    cl2 = cl[keep]
    deg = np.diff(rp.astype(np.int64))
    deg[5] = 0
    rp2 = np.concatenate([[0], np.cumsum(deg)]).astype(np.uint32)
    rng = np.random.default_rng(0)
    w = rng.lognormal(0, 1, len(cl2)).astype(np.float32)
    p = np.full(64, 1 / 64, np.float32)
    g = rng.standard_normal(64).astype(np.float32)
    with ob.Graph.from_csr(rp2, cl2) as G:
        r1 = G.wpr_forward(p, w=w, max_it=ITERS)
        d1 = G.wpr_backward(g, max_it=ITERS)
        r2 = G.wpr_forward(p, w=w, max_it=ITERS)
        d2 = G.wpr_backward(g, max_it=ITERS)
    assert r1.tobytes() == r2.tobytes() and d1[0].tobytes() == d2[0].tobytes()
    r_ref = oracle.wpr_forward(rp2, cl2, w.astype(np.float64), p.astype(np.float64), ALPHA, ITERS)
    assert rel_inf(r1.astype(np.float64), r_ref) < 1e-5
    lam, dw_ref, dp_ref = oracle.wpr_backward(rp2, cl2, w.astype(np.float64), r_ref,
                                              g.astype(np.float64), ALPHA, ITERS)
    s_w, _ = operand_scales(rp2, cl2, w, r_ref, g, lam)
    assert_grad_close(d1[0], dw_ref, "dw with dangling rows", s_w)


def test_rmat18_gradient_vs_oracle(ob):
    """RMAT-18: a power-law graph with long rows (segments) in both directions."""
    rp, cl, w, p, g = make_problem(18, 5)
    with ob.Graph.from_csr(rp, cl) as G:
        r = G.wpr_forward(p, w=w, max_it=ITERS)
        dw, dp = G.wpr_backward(g, max_it=ITERS)
    r_ref = oracle.wpr_forward(rp, cl, w.astype(np.float64), p.astype(np.float64), ALPHA, ITERS)
    lam, dw_ref, dp_ref = oracle.wpr_backward(rp, cl, w.astype(np.float64), r_ref,
                                              g.astype(np.float64), ALPHA, ITERS)
    assert rel_inf(r.astype(np.float64), r_ref) < 1e-5
    assert np.max(np.abs(r - r_ref) / r_ref) < 1e-5       # every rank (all positive)
    s_w, s_p = operand_scales(rp, cl, w, r_ref, g, lam)
    assert_grad_close(dw, dw_ref, "dw rmat18", s_w)
    assert_grad_close(dp, dp_ref, "dp rmat18", s_p)
