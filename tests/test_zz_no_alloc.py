"""olv_bfs_noalloc: the BFS entry point that allocates nothing, for callers that
own all device memory themselves (a host application's memory pool, a
memory-capped plugin) and may not call cudaMalloc.  Called through the C ABI
with caller-owned device buffers and compared with olv_bfs, twice in a row
(the second call reuses the shared fixed scratch).  This file is collected last
on purpose."""
import ctypes

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


def _call(L, rp, cl, V, E, src, out, stream=None):
    rc = L.olv_bfs_noalloc(ctypes.c_void_p(rp.data_ptr()), ctypes.c_void_p(cl.data_ptr()),
                           V, E, src, ctypes.c_void_p(out.data_ptr()), stream, None)
    return rc


def test_noalloc_bfs_matches_olv_bfs_twice():
    import torch
    import olive_b200 as ob
    assert torch.cuda.is_available()
    L = ob.lib()
    with ob.Graph.rmat(16, 16, 9) as g:
        rp_h, cl_h, _ = g.csr()
        hub, _ = g.max_degree_vertex()
        rp = torch.from_numpy(rp_h.astype(np.int32)).cuda()
        cl = torch.from_numpy(cl_h.astype(np.int32)).cuda()
        out = torch.empty(g.V, dtype=torch.int32, device="cuda")
        deg = np.diff(rp_h.astype(np.int64))
        other = int(np.flatnonzero(deg > 0)[7])
        for src in (hub, other):      # two calls in a row share the scratch
            rc = _call(L, rp, cl, g.V, g.E, src, out)
            assert rc == 0, L.olv_last_error()
            torch.cuda.synchronize()
            want = g.bfs(src)        # the existing entry point
            np.testing.assert_array_equal(out.cpu().numpy(), want)   # levels: exact


def test_noalloc_bfs_commits_no_memory_and_takes_a_stream():
    """After a first call (which may load the device code), further calls leave
    the device's free memory unchanged; a caller's own stream works."""
    import torch
    import olive_b200 as ob
    L = ob.lib()
    rp_h, cl_h = oracle.rmat_csr(14, 16, 5)
    V, E = len(rp_h) - 1, len(cl_h)
    rp = torch.from_numpy(rp_h.astype(np.int32)).cuda()
    cl = torch.from_numpy(cl_h.astype(np.int32)).cuda()
    out = torch.empty(V, dtype=torch.int32, device="cuda")
    want, _ = oracle.bfs(rp_h, cl_h, 3)
    assert _call(L, rp, cl, V, E, 3, out) == 0, L.olv_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert _call(L, rp, cl, V, E, 3, out) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    s = torch.cuda.Stream()
    out2 = torch.full((V,), -5, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert _call(L, rp, cl, V, E, 3, out2, ctypes.c_void_p(s.cuda_stream)) == 0
    s.synchronize()
    np.testing.assert_array_equal(out2.cpu().numpy(), want)


def test_noalloc_bfs_reference_fixture_and_limits():
    import torch
    import olive_b200 as ob
    L = ob.lib()
    rp_h, cl_h = oracle.grid_csr(128, 128)
    rp = torch.from_numpy(rp_h.astype(np.int32)).cuda()
    cl = torch.from_numpy(cl_h.astype(np.int32)).cuda()
    out = torch.empty(len(rp_h) - 1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        assert _call(L, rp, cl, len(rp_h) - 1, len(cl_h), 0, out) == 0
        np.testing.assert_array_equal(out.cpu().numpy(), oracle.bfs(rp_h, cl_h, 0)[0])
    # sizes beyond the fixed scratch are rejected before any work
    assert _call(L, rp, cl, (1 << 20) + 1, len(cl_h), 0, out) == -6
    assert b"exceeds the fixed scratch" in L.olv_last_error()
    # an invalid CSR is caught by the device-side check, not by a fault
    bad = cl.clone()
    bad[5] = 1 << 30
    assert _call(L, rp, bad, len(rp_h) - 1, len(cl_h), 0, out) == -1
    assert b"invalid CSR" in L.olv_last_error()
    # host memory is not the current device's memory: rejected before any launch
    host_out = torch.empty(len(rp_h) - 1, dtype=torch.int32).pin_memory()
    assert _call(L, rp, cl, len(rp_h) - 1, len(cl_h), 0, host_out) == -1
    assert b"device memory of the current device" in L.olv_last_error()
