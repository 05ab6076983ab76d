"""CPU model of the SSSP superstep schedule (olive_b200/csrc/sssp.cu), checked
against Dijkstra.

The device solve orders the atomicMin relaxation of SSSP.cu:54-76 as
delta-stepping with a near queue, a far pile and light/heavy edges, and
relaxes a settled bucket's heavy edges either by push (every heavy out-edge
of the bucket) or by pull (every in-edge of every vertex at or above the
threshold whose source is settled).  It collects the settled bucket either
densely or from the list of the bucket's relax inputs.  This model runs the
same schedule synchronously in numpy, choosing push or pull with the
kernel's rule, and checks that both choices and both collects give Dijkstra's
distances, that a pull never lowers a vertex below the threshold, and that
the bucket list covers every settled vertex; and that the run on vertices
renumbered by in-degree, mapped back, gives the same distances.  No GPU
needed.
"""
import numpy as np
import pytest

from oracle import oracle

INF = 0x7fffffff


def _expand(rp, deg, sel, us):
    """(u, e) for every edge of rows us whose position passes sel."""
    cnt = deg[us]
    tot = int(cnt.sum())
    if tot == 0:
        return np.empty(0, np.int64), np.empty(0, np.int64)
    u = np.repeat(us, cnt)
    off = np.arange(tot) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    e = rp[u] + off
    m = sel[e]
    return u[m], e[m]


def _lower(dist, v, nd):
    """Apply candidate distances; return the improved vertices and values."""
    imp = nd < dist[v]
    v, nd = v[imp], nd[imp]
    o = np.lexsort((nd, v))
    v, nd = v[o], nd[o]
    first = np.ones(len(v), bool)
    first[1:] = v[1:] != v[:-1]
    v, nd = v[first], nd[first]
    dist[v] = nd
    return v, nd


def schedule(rp, col, w, src, delta, pull_mode, list_collect, sub=0, nsub=1, tail=0):
    """pull_mode: 'never', 'always' or 'rule' (the kernel's choice:
    E - settled in-edges + V/2 < heavy out-edges of the bucket).  sub > 0:
    the light phase of the first nsub heavy buckets runs in sub-buckets of
    width sub (the far pile is split at each sub-bucket's end; the heavy step
    follows the last one).  tail > delta: the buckets after the first are
    tail wide and relax every edge in-bucket, with no heavy step."""
    rp = rp.astype(np.int64)
    col = col.astype(np.int64)
    w = w.astype(np.int64)
    V, E = len(rp) - 1, len(col)
    deg = np.diff(rp)
    row = np.repeat(np.arange(V), deg)
    order = np.argsort(col, kind="stable")
    cptr = np.zeros(V + 1, np.int64)
    np.add.at(cptr, col + 1, 1)
    cptr = np.cumsum(cptr)
    indeg = np.diff(cptr)
    csrc, cw = row[order], w[order]
    light = w <= delta
    hdeg = np.bincount(row[~light], minlength=V)
    dist = np.full(V, INF, np.int64)
    dist[src] = 0
    far = np.zeros(V, bool)
    q = np.array([src])
    sw = sub if 0 < sub < delta else delta
    hb = 0
    lo, bend = 0, delta
    hi = min(sw if nsub > 0 else delta, bend)
    settled_in, pulls = 0, 0
    wide = False
    every = np.ones(E, bool)
    while True:
        blist = []
        while True:
            while len(q):                       # relax supersteps: light (or all) edges
                blist.append(q)
                u, e = _expand(rp, deg, every if wide else light, q)
                v, nd = _lower(dist, col[e], np.minimum(dist[u] + w[e], INF))
                far[v[nd >= hi]] = True
                q = v[nd < hi]
            fv = np.flatnonzero(far)
            fv = fv[dist[fv] >= hi]
            if not wide and hi < bend and len(fv) and dist[fv].min() < bend:   # next sub-bucket
                hi = min(max(hi, int(dist[fv].min())) + sw, bend)
                far[:] = False
                far[fv] = True
                q = fv[dist[fv] < hi]
                far[q] = False
                continue
            break
        in_bucket = np.flatnonzero((dist >= lo) & (dist < hi))
        if wide:   # every edge of the bucket was relaxed: no heavy step
            fv = np.flatnonzero(far)
            fv = fv[dist[fv] >= hi]
            far[:] = False
            far[fv] = True
            if len(fv) == 0:
                return dist, pulls
            lo = max(hi, int(dist[fv].min()))
            hi = bend = lo + tail
            q = fv[dist[fv] < hi]
            far[q] = False
            continue
        if list_collect:
            listed = np.unique(np.concatenate(blist)) if blist else np.empty(0, np.int64)
            listed = listed[(dist[listed] >= lo) & (dist[listed] < hi)]
            np.testing.assert_array_equal(listed, in_bucket)   # the list covers the bucket
        hw = int(hdeg[in_bucket].sum())
        settled_in += int(indeg[in_bucket].sum())
        pull = {"never": False, "always": True,
                "rule": (E - settled_in) + V // 2 < hw}[pull_mode]
        if pull:
            pulls += 1
            uns = np.flatnonzero(dist >= hi)
            cnt = indeg[uns]
            vv = np.repeat(uns, cnt)
            off = np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt)
            ce = cptr[vv] + off
            du = dist[csrc[ce]]
            ok = du < hi
            v, nd = _lower(dist, vv[ok], np.minimum(du[ok] + cw[ce][ok], INF))
        else:
            u, e = _expand(rp, deg, ~light, in_bucket)
            v, nd = _lower(dist, col[e], np.minimum(dist[u] + w[e], INF))
        assert (nd >= hi).all()          # heavy relaxations land at or above the threshold
        far[v] = True
        fv = np.flatnonzero(far)
        fv = fv[dist[fv] >= hi]
        far[:] = False
        far[fv] = True
        if len(fv) == 0:
            return dist, pulls
        wide = tail > delta
        # a pull followed by wide buckets opens the next bucket at the
        # threshold itself (it routes every vertex; no split pass)
        lo = hi if (wide and pull) else max(hi, int(dist[fv].min()))
        hb += 1
        if wide:
            hi = bend = lo + tail
        else:
            bend = lo + delta
            hi = min(lo + (sw if hb < nsub else delta), bend)
        q = fv[dist[fv] < hi]
        far[q] = False


@pytest.mark.parametrize("scale,seed,delta", [(11, 1, 64), (12, 2, 16), (12, 3, 200)])
@pytest.mark.parametrize("pull_mode", ["never", "always", "rule"])
def test_schedule_matches_dijkstra_rmat(scale, seed, delta, pull_mode):
    rp, col = oracle.rmat_csr(scale, 16, seed)
    w = oracle.uint_weights(len(col), seed + 10)
    deg = np.diff(rp.astype(np.int64))
    hub = int(np.argmax(deg))
    ref = oracle.dijkstra(rp, col, w, hub)[0].astype(np.int64)
    dist, pulls = schedule(rp, col, w, hub, delta, pull_mode, list_collect=True)
    np.testing.assert_array_equal(dist, ref)
    if pull_mode == "rule" and delta == 64:
        assert pulls >= 1   # from the hub the first bucket's heavy edges go by pull


def test_schedule_matches_dijkstra_random_and_unit_weights():
    rng = np.random.default_rng(3)
    V, E = 2000, 12000
    src = np.sort(rng.integers(0, V, E))
    dst = rng.integers(0, V, E)
    rp = np.zeros(V + 1, np.int64)
    np.add.at(rp, src + 1, 1)
    rp = np.cumsum(rp).astype(np.uint32)
    col = dst.astype(np.uint32)
    for w in (rng.integers(1, 1000, E).astype(np.uint32), np.ones(E, np.uint32)):
        ref = oracle.dijkstra(rp, col, w, 0)[0].astype(np.int64)
        for mode in ("never", "always"):
            dist, _ = schedule(rp, col, w, 0, 32, mode, list_collect=True)
            np.testing.assert_array_equal(dist, ref)


def renumber_by_in_degree(rp, col, w):
    """The renumbering the device solve runs on: vertices in descending
    in-degree, ties in id order (a stable sort); rows keep their entry order.
    Returns (perm, newid, rp', col', w')."""
    rp = rp.astype(np.int64)
    V = len(rp) - 1
    indeg = np.bincount(col.astype(np.int64), minlength=V)
    perm = np.argsort(-indeg, kind="stable")
    newid = np.empty(V, np.int64)
    newid[perm] = np.arange(V)
    deg = np.diff(rp)[perm]
    nrp = np.concatenate([[0], np.cumsum(deg)])
    rows = np.concatenate([np.arange(rp[v], rp[v + 1]) for v in perm]) if V else np.empty(0, int)
    return perm, newid, nrp.astype(np.uint32), newid[col[rows]].astype(np.uint32), w[rows]


@pytest.mark.parametrize("scale,seed", [(10, 1), (11, 4)])
def test_schedule_on_renumbered_graph(scale, seed):
    rp, col = oracle.rmat_csr(scale, 16, seed)
    w = oracle.uint_weights(len(col), seed + 10)
    perm, newid, nrp, ncol, nw = renumber_by_in_degree(rp, col, w)
    indeg = np.bincount(col.astype(np.int64), minlength=len(rp) - 1)
    assert (np.diff(indeg[perm]) <= 0).all()          # highest in-degree first
    deg = np.diff(rp.astype(np.int64))
    for src in (int(np.argmax(deg)), int(np.flatnonzero(deg > 0)[2])):
        ref = oracle.dijkstra(rp, col, w, src)[0].astype(np.int64)
        dnew, _ = schedule(nrp, ncol, nw, int(newid[src]), 64, "rule", list_collect=True)
        np.testing.assert_array_equal(dnew[newid], ref)   # mapped back: out[v] = dnew[newid[v]]


@pytest.mark.parametrize("sub,nsub", [(8, 1), (4, 2), (16, 1), (1, 3)])
@pytest.mark.parametrize("pull_mode", ["never", "rule"])
def test_schedule_with_sub_buckets(sub, nsub, pull_mode):
    """The first heavy buckets' light phase in sub-buckets: same distances,
    and the bucket list still covers each heavy bucket."""
    for scale, seed in ((11, 1), (12, 5)):
        rp, col = oracle.rmat_csr(scale, 16, seed)
        w = oracle.uint_weights(len(col), seed + 10)
        hub = int(np.argmax(np.diff(rp.astype(np.int64))))
        ref = oracle.dijkstra(rp, col, w, hub)[0].astype(np.int64)
        dist, _ = schedule(rp, col, w, hub, 64, pull_mode, list_collect=True, sub=sub, nsub=nsub)
        np.testing.assert_array_equal(dist, ref)


@pytest.mark.parametrize("tail", [65, 128, 256, 1 << 20])
@pytest.mark.parametrize("pull_mode", ["never", "rule"])
def test_schedule_with_wide_tail_buckets(tail, pull_mode):
    """Buckets after the first relaxing every edge in-bucket (width tail, no
    heavy step): Dijkstra's distances from the hub and from a low-degree
    vertex, and from random weights on a random graph."""
    rp, col = oracle.rmat_csr(12, 16, 7)
    w = oracle.uint_weights(len(col), 17)
    deg = np.diff(rp.astype(np.int64))
    for src in (int(np.argmax(deg)), int(np.flatnonzero(deg == 1)[0])):
        ref = oracle.dijkstra(rp, col, w, src)[0].astype(np.int64)
        dist, _ = schedule(rp, col, w, src, 64, pull_mode, list_collect=True, tail=tail)
        np.testing.assert_array_equal(dist, ref)
    rng = np.random.default_rng(5)
    V, E = 1500, 9000
    s = np.sort(rng.integers(0, V, E))
    rp = np.zeros(V + 1, np.int64)
    np.add.at(rp, s + 1, 1)
    rp = np.cumsum(rp).astype(np.uint32)
    col = rng.integers(0, V, E).astype(np.uint32)
    w = rng.integers(1, 1000, E).astype(np.uint32)
    ref = oracle.dijkstra(rp, col, w, 0)[0].astype(np.int64)
    dist, _ = schedule(rp, col, w, 0, 32, pull_mode, list_collect=True, tail=tail)
    np.testing.assert_array_equal(dist, ref)
