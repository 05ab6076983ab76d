"""GPU output writer (olv_write_text) against the C library's own printf on
the same values, byte for byte: "%d\\n", "%u\\n" and "%f\\n" (the formats of the
reference apps' print() methods), from host and device buffers, across the
chunk boundary; and the binary CSR dump round trip (olv_graph_save /
olv_graph_load)."""
import ctypes
import ctypes.util
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
_libc = ctypes.CDLL(ctypes.util.find_library("c"))


def printf_lines(fmt, values, cast):
    buf = ctypes.create_string_buffer(512)
    out = []
    for v in values:
        n = _libc.snprintf(buf, 512, fmt, cast(v))
        out.append(buf.raw[:n])
    return b"".join(out)


@pytest.fixture(scope="module")
def ob():
    import torch
    assert torch.cuda.is_available()
    import olive_b200
    return olive_b200


def _read(p):
    with open(p, "rb") as f:
        return f.read()


def test_int32_and_uint32(ob, tmp_path):
    rng = np.random.default_rng(1)
    a = np.concatenate([rng.integers(-2**31, 2**31, 5000),
                        [0, -1, 1, 2**31 - 1, -2**31, 10, 9, 99, 100]]).astype(np.int32)
    p = str(tmp_path / "a.txt")
    n = ob.write_text(p, a)
    want = printf_lines(b"%d\n", a.tolist(), ctypes.c_int)
    assert _read(p) == want and n == len(want)
    u = np.concatenate([rng.integers(0, 2**32, 3000), [0, 2**32 - 1, 2**31]]).astype(np.uint32)
    ob.write_text(p, u)
    assert _read(p) == printf_lines(b"%u\n", u.tolist(), ctypes.c_uint)


def _doubles(rng):
    tie = 15625.0 * np.array([1, 3, 5, 7, 9, 1001]) / 128.0          # x * 1e6 ends in .5
    vals = [0.0, -0.0, 1.0, -1.0, 0.5, 1e-7, -1e-7, 4.9999995e-7, 5e-7, 5.000001e-7,
            0.1, 0.2, 0.3, 1 / 3, 2 / 3, 123456.7890125, 2.0 ** 53, 2.0 ** 53 + 2,
            1e20, -1e20, 2.0 ** 100, 5e-324, 2.2250738585072014e-308,
            float("inf"), -float("inf")]
    vals += list(tie) + list(-tie)
    vals += list(rng.random(2000))                                 # ranks
    vals += list(rng.random(1000) * 10.0 ** rng.integers(-12, 15, 1000))
    vals += list(-rng.random(500) * 10.0 ** rng.integers(-9, 9, 500))
    return np.array(vals, np.float64)


def test_double_fixed6_matches_printf(ob, tmp_path):
    d = _doubles(np.random.default_rng(2))
    p = str(tmp_path / "d.txt")
    ob.write_text(p, d)
    assert _read(p) == printf_lines(b"%f\n", d.tolist(), ctypes.c_double)


def test_nan_and_float32_and_device_input(ob, tmp_path):
    import torch
    d = np.array([float("nan"), -float("nan"), 1.5], np.float64)
    p = str(tmp_path / "n.txt")
    ob.write_text(p, d)
    assert _read(p) == printf_lines(b"%f\n", d.tolist(), ctypes.c_double)
    f = np.random.default_rng(3).random(3000).astype(np.float32) * 7 - 2
    ob.write_text(p, torch.from_numpy(f).cuda())
    assert _read(p) == printf_lines(b"%f\n", f.astype(np.float64).tolist(), ctypes.c_double)


def test_chunks_and_large_output(ob, tmp_path):
    n = (1 << 24) + 12345
    a = (np.arange(n, dtype=np.int64) * 2654435761 % 4000000007 - 2000000000).astype(np.int32)
    p = str(tmp_path / "big.txt")
    b = ob.write_text(p, a)
    want = ("\n".join(map(str, a.tolist())) + "\n").encode()
    assert b == len(want) and _read(p) == want
    os.unlink(p)


def test_value_out_of_range_is_rejected(ob, tmp_path):
    with pytest.raises(ob.OliveError, match="2\\^107"):
        ob.write_text(str(tmp_path / "x.txt"), np.array([1.0, 2.0 ** 110], np.float64))


def test_graph_binary_dump_round_trip(ob, tmp_path):
    p = str(tmp_path / "g.bin")
    with ob.Graph.rmat(12, 16, 4, weights=True, wseed=5) as g:
        rp, cl, w = g.csr()
        g.save(p)
        hub, _ = g.max_degree_vertex()
        d = g.sssp(hub)
    with ob.Graph.load(p) as g2:
        rp2, cl2, w2 = g2.csr()
        np.testing.assert_array_equal(rp2, rp)
        np.testing.assert_array_equal(cl2, cl)
        np.testing.assert_array_equal(w2, w)
        np.testing.assert_array_equal(g2.sssp(hub), d)
