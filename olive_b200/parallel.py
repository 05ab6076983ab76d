"""Multi-process plumbing for running the engine on several GPUs of one node.

Two ways to use several GPUs:
  * replicas (what bench.py --gpus N measures): one process per GPU, launched
    by torch.distributed.run, each owning whole work units -- its own sources
    for multi-source BFS, its own instances of a batch, or a full replica of
    a single-source run; nothing crosses GPUs on the data path, the only
    collectives are the timing and counting reductions below;
  * a 1-D vertex partition of one graph (PartitionedGraph, at the end of this
    file): each rank owns a vertex range and the in-edges of its vertices;
    BFS and PageRank supersteps exchange one bitmap or vector slice per rank
    (NCCL all-gathers between GPUs, gloo on CPU in the tests).
"""
import datetime
import os


def rank_world():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def init(backend="nccl", timeout_s=120, device=None):
    """Join the process group named by the torchrun environment (no-op alone)."""
    import torch.distributed as dist
    _, world, _ = rank_world()
    if world > 1 and not dist.is_initialized():
        kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if device is not None:
            kw["device_id"] = device
        dist.init_process_group(backend, **kw)
    return world


def shard(items, rank, world):
    """Contiguous, balanced split of a sequence: shard r of `world`."""
    n = len(items)
    lo = n * rank // world
    hi = n * (rank + 1) // world
    return items[lo:hi]


def _reduce(x, op, device):
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, device="cpu"):
    """Largest value over all ranks (the job time of a multi-GPU step)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x, device="cpu"):
    """Sum over all ranks (work units processed by the whole job)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM, device)


def finish():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------- 1-D vertex partition --
# A graph split across ranks by contiguous vertex ranges (the reference's
# intended multi-GPU engine, olive.h:61-199 with the edge-cut of
# partitionStrategy.h:58-62, never built).  Each rank owns vertices [lo, hi)
# -- lo a multiple of 64, ranges balanced by in-edges -- and holds their
# in-edges (rows lo..hi-1 of the reverse graph, global source ids).  Every
# superstep is local work on the owned rows (olv_part_* kernels on the GPU)
# followed by one exchange:
#   BFS        all-gather of each rank's words of the next-frontier bitmap
#              (V/8 bytes in all: 2 MB at 2^24 vertices) and a sum of the
#              vertices found;
#   PageRank   all-gather of the owned contributions r/outdeg (4 B per
#              vertex) and sums of |r' - r| and of the dangling ranks.
# Remote data lands in each GPU's own memory (NCCL collectives); no kernel
# reads another GPU's memory.


def partition_ranges(colptr, world):
    """Contiguous [lo, hi) per rank, lo a multiple of 64, about E/world
    in-edges each (colptr: the reverse graph's row offsets)."""
    import numpy as np
    colptr = np.asarray(colptr, np.int64)
    V, E = len(colptr) - 1, int(colptr[-1])
    cuts = [0]
    for r in range(1, world):
        v = int(np.searchsorted(colptr, E * r // world, side="left"))
        v = min(max((v // 64) * 64, cuts[-1]), V)
        cuts.append(v)
    cuts.append(V)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def reverse_csr(rowptr, col):
    """(colptr, rowidx): in-edges grouped by destination, sources in CSR order."""
    import numpy as np
    rowptr = np.asarray(rowptr, np.int64)
    V = len(rowptr) - 1
    src = np.repeat(np.arange(V, dtype=np.uint32), np.diff(rowptr))
    order = np.argsort(np.asarray(col, np.int64), kind="stable")
    colptr = np.zeros(V + 1, np.int64)
    np.add.at(colptr, np.asarray(col, np.int64) + 1, 1)
    return np.cumsum(colptr).astype(np.uint32), src[order]


class GpuPartStep:
    """The local work of one part on the current GPU (olv_part_* kernels)."""

    def __init__(self, V, lo, hi, colptr, rowidx, outdeg, stream=None):
        import ctypes
        import numpy as np
        from . import _check, _ptr, lib
        self.V, self.lo, self.hi = V, lo, hi
        self._h = ctypes.c_void_p()
        cp = np.ascontiguousarray(colptr, np.uint32)
        ri = np.ascontiguousarray(rowidx, np.uint32)
        od = np.ascontiguousarray(outdeg, np.uint32)
        _check(lib().olv_part_create(V, lo, hi, _ptr(cp), _ptr(ri) if len(ri) else None, _ptr(od),
                                     ctypes.byref(self._h)), "olv_part_create")
        if stream is not None:
            _check(lib().olv_part_set_stream(self._h, getattr(stream, "cuda_stream", stream)),
                   "olv_part_set_stream")

    def bfs(self, frontier, level, next_level, next_words):
        import ctypes
        from . import _U64, _check, lib
        found = _U64()
        _check(lib().olv_part_bfs_step(self._h, frontier.data_ptr(), level.data_ptr(), next_level,
                                       next_words.data_ptr(), ctypes.byref(found)),
               "olv_part_bfs_step")
        return found.value

    def pagerank(self, contrib, base, alpha, rank, contrib_out):
        import ctypes
        from . import _check, lib
        sums = (ctypes.c_double * 2)()
        _check(lib().olv_part_pr_step(self._h, contrib.data_ptr(), base, alpha, rank.data_ptr(),
                                      contrib_out.data_ptr(), sums), "olv_part_pr_step")
        return sums[0], sums[1]

    def close(self):
        from . import lib
        if self._h:
            lib().olv_part_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DistComm:
    """Exchange among the ranks of the default process group (NCCL between
    GPUs, gloo on CPU): every rank holds one part."""

    def gather(self, slices, pad):
        import torch
        import torch.distributed as dist
        (t,) = slices
        buf = torch.zeros(pad, dtype=t.dtype, device=t.device)
        buf[:len(t)] = t
        out = [torch.empty_like(buf) for _ in range(dist.get_world_size())]
        dist.all_gather(out, buf)
        return out

    def sum(self, x, device):
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        dist.all_reduce(t)
        return float(t.item())


class LocalComm:
    """All parts in this process (one GPU or the CPU): the exchange is a
    concatenation.  Used to run a partitioned solve on fewer GPUs than parts."""

    def gather(self, slices, pad):
        return list(slices)

    def sum(self, x, device):
        return float(x)


class PartitionedGraph:
    """A graph split into parts by vertex ranges.  `ranges` lists every
    part's [lo, hi); this process holds the parts `mine` (indices into
    ranges) with their `steps` (GpuPartStep, or any object with the same
    bfs / pagerank methods) and exchanges through `comm`."""

    def __init__(self, V, outdeg, ranges, mine, steps, comm, device):
        import numpy as np
        self.V, self.ranges, self.mine, self.steps = V, ranges, mine, steps
        self.comm, self.device = comm, device
        self.outdeg = np.asarray(outdeg, np.uint32)
        self.words = (V + 63) // 64
        self.pad_words = max((hi - lo + 63) // 64 for lo, hi in ranges)
        self.pad_rows = max(hi - lo for lo, hi in ranges)

    @classmethod
    def build(cls, rowptr, col, world, rank=None, device="cuda", step_factory=None):
        """Split the CSR into `world` parts.  rank=None keeps every part in this
        process (LocalComm); otherwise this process is part `rank` of the
        default process group (DistComm)."""
        import numpy as np
        V = len(rowptr) - 1
        outdeg = np.diff(np.asarray(rowptr, np.int64)).astype(np.uint32)
        colptr, rowidx = reverse_csr(rowptr, col)
        ranges = partition_ranges(colptr, world)
        mine = list(range(world)) if rank is None else [rank]
        factory = step_factory or (lambda V_, lo, hi, cp, ri, od: GpuPartStep(V_, lo, hi, cp, ri,
                                                                              od))
        steps = []
        for r in mine:
            lo, hi = ranges[r]
            cp = (colptr[lo:hi + 1].astype(np.int64) - int(colptr[lo])).astype(np.uint32)
            ri = rowidx[int(colptr[lo]):int(colptr[hi])]
            steps.append(factory(V, lo, hi, cp, ri, outdeg[lo:hi]))
        comm = LocalComm() if rank is None else DistComm()
        return cls(V, outdeg, ranges, mine, steps, comm, device)

    def _assemble_words(self, gathered):
        import torch
        full = torch.zeros(self.words, dtype=torch.int64, device=self.device)
        for r, g in enumerate(gathered):
            lo, hi = self.ranges[r]
            nw = (hi - lo + 63) // 64
            full[lo // 64:lo // 64 + nw] |= g[:nw]
        return full

    def bfs(self, src):
        """BFS levels from src (int32, 0x7fffffff unreached), as numpy."""
        import numpy as np
        import torch
        dev = self.device
        frontier = torch.zeros(self.words, dtype=torch.int64, device=dev)
        frontier[src // 64] = 1 << (src % 64) if src % 64 < 63 else -(1 << 63)
        levels = []
        for (lo, hi) in (self.ranges[r] for r in self.mine):
            lv = torch.full((hi - lo,), 0x7FFFFFFF, dtype=torch.int32, device=dev)
            if lo <= src < hi:
                lv[src - lo] = 0
            levels.append(lv)
        nxt = [torch.zeros(self.pad_words, dtype=torch.int64, device=dev) for _ in self.mine]
        level = 0
        while True:
            found = sum(st.bfs(frontier, lv, level + 1, nx)
                        for st, lv, nx in zip(self.steps, levels, nxt))
            if self.comm.sum(found, dev) == 0:
                break
            frontier = self._assemble_words(self.comm.gather(nxt, self.pad_words))
            level += 1
        return self._assemble_rows(levels, np.int32)

    def _assemble_rows(self, parts, dtype):
        import numpy as np
        import torch
        gathered = self.comm.gather([self._padded(p) for p in parts], self.pad_rows)
        out = np.empty(self.V, dtype)
        for r, g in enumerate(gathered):
            lo, hi = self.ranges[r]
            out[lo:hi] = g[:hi - lo].cpu().numpy()
        return out

    def _padded(self, t):
        import torch
        if len(t) == self.pad_rows:
            return t
        buf = torch.zeros(self.pad_rows, dtype=t.dtype, device=t.device)
        buf[:len(t)] = t
        return buf

    def pagerank(self, alpha=0.85, max_it=50, tol=1e-7, dangling="uniform"):
        """PageRank (PageRank.cu semantics, dangling mass redistributed
        uniformly or dropped): (ranks as numpy, iterations, last residual)."""
        import numpy as np
        import torch
        dev, V = self.device, self.V
        r0 = np.float32(1.0) / np.float32(V)
        ranks, conts = [], []
        dang = 0.0
        for (lo, hi) in (self.ranges[r] for r in self.mine):
            ranks.append(torch.full((hi - lo,), float(r0), dtype=torch.float32, device=dev))
            od = torch.from_numpy(self.outdeg[lo:hi].astype(np.float32)).to(dev)
            conts.append(torch.where(od > 0, float(r0) / od.clamp(min=1), torch.zeros_like(od)))
            dang += float(r0) * float((self.outdeg[lo:hi] == 0).sum())
        dang = self.comm.sum(dang, dev)
        contrib = self._assemble_floats(conts)
        it, res = 0, 0.0
        while it < max_it:
            base = (1 - alpha) / V + (alpha * dang / V if dangling == "uniform" else 0.0)
            new_conts = [torch.empty_like(c) for c in conts]
            res_l, dang_l = 0.0, 0.0
            for st, rk, nc in zip(self.steps, ranks, new_conts):
                a, d = st.pagerank(contrib, base, alpha, rk, nc)
                res_l += a
                dang_l += d
            res = self.comm.sum(res_l, dev)
            dang = self.comm.sum(dang_l, dev)
            conts = new_conts
            contrib = self._assemble_floats(conts)
            it += 1
            if res < tol:
                break
        return self._assemble_rows(ranks, np.float32), it, res

    def _assemble_floats(self, parts):
        import torch
        gathered = self.comm.gather([self._padded(p) for p in parts], self.pad_rows)
        full = torch.empty(self.V, dtype=torch.float32, device=self.device)
        for r, g in enumerate(gathered):
            lo, hi = self.ranges[r]
            full[lo:hi] = g[:hi - lo]
        return full

    def close(self):
        for st in self.steps:
            if hasattr(st, "close"):
                st.close()
