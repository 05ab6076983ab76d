"""olv_ppr_batch: K personalised PageRank vectors on a general graph (pull over
the reverse graph, 128-byte rows of K contributions), against the FP64 oracle
after the same number of iterations: every vector within 1e-6 relative
(normwise, max|d| / max|ref|), every entry within 1e-5 relative, exact zeros
where the seed does not reach."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ob():
    import torch
    assert torch.cuda.is_available()
    import olive_b200
    return olive_b200


def check(got, ref):
    got = got.astype(np.float64)
    for k in range(ref.shape[1]):
        r, g = ref[:, k], got[:, k]
        assert np.max(np.abs(g - r)) <= 1e-6 * np.max(np.abs(r)), k
        nz = r > 0
        assert np.all(g[~nz] == 0), k
        assert np.max(np.abs(g[nz] - r[nz]) / r[nz]) < 1e-5, (k, np.max(np.abs(g[nz] - r[nz]) / r[nz]))


@pytest.mark.parametrize("scale,seed,K", [(10, 1, 32), (14, 3, 32), (16, 5, 7), (18, 2, 32)])
def test_ppr_rmat_vs_oracle(ob, scale, seed, K):
    with ob.Graph.rmat(scale, 16, seed) as g:
        rp, cl, _ = g.csr()
        deg = np.diff(rp.astype(np.int64))
        rng = np.random.default_rng(scale)
        seeds = rng.choice(g.V, K, replace=False).astype(np.uint32)
        seeds[0] = int(np.argmax(deg))                  # the hub
        seeds[-1] = int(np.flatnonzero(deg == 0)[0])    # a dangling seed
        out = g.ppr(seeds, 0.85, 50, 1e-7)
        it = g.last_stats.iterations
        ref, it_ref = oracle.ppr(rp, cl, seeds, 0.85, it, 0.0)
        assert it_ref == it and it >= 2
        check(out, ref)


def test_ppr_fixed_iterations_duplicates_and_determinism(ob):
    import torch
    rp, cl = oracle.grid_csr(40, 30)
    with ob.Graph.from_csr(rp, cl) as g:
        seeds = np.array([0, 17, 17, 1199, 600], np.uint32)
        a = g.ppr(seeds, 0.85, 30, 0.0)
        assert g.last_stats.iterations == 30
        ref, _ = oracle.ppr(rp, cl, seeds, 0.85, 30, 0.0)
        check(a, ref)
        np.testing.assert_array_equal(a[:, 1], a[:, 2])
        dev = torch.empty((g.V, 5), dtype=torch.float32, device="cuda")
        g.ppr(torch.from_numpy(seeds.astype(np.int32)).cuda(), 0.85, 30, 0.0, out=dev)
        assert dev.cpu().numpy().tobytes() == a.tobytes()


def test_ppr_matches_batch_kernel_instances(ob):
    """The general-graph PPR and the block-diagonal batch kernel agree with the
    same oracle on an ER instance."""
    sizes = oracle.er_batch_sizes(1, 2000, 3000, 9)
    lrp, lcl = oracle.er_batch_instance(0, int(sizes[0]), 8, 9)
    seeds = np.random.default_rng(2).integers(0, len(lrp) - 1, 32).astype(np.uint32)
    ref, _ = oracle.ppr(lrp, lcl, seeds, 0.85, 25, 0.0)
    with ob.Graph.from_csr(lrp, lcl) as g:
        check(g.ppr(seeds, 0.85, 25, 0.0), ref)


def test_ppr_bad_arguments(ob):
    rp, cl = oracle.grid_csr(4, 4)
    with ob.Graph.from_csr(rp, cl) as g:
        with pytest.raises(ob.OliveError):
            g.ppr(np.arange(33, dtype=np.uint32) % 16)
        with pytest.raises(ob.OliveError):
            g.ppr(np.array([16], np.uint32))
        with pytest.raises(ob.OliveError):
            g.ppr(np.array([], np.uint32))
