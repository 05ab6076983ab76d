// Load-balanced frontier advance for sm_100a.
//
// Replaces edgeFilterKernel (oliverKernel.h:45-83), which gave every queued
// source a fixed group of 1..32 threads (hubs serialised, lanes idle on short
// rows).  Here a CTA takes a chunk of kBlock queued sources, scans their
// out-degrees in shared memory and lets all kBlock threads walk the chunk's
// edges in order, so column indices are read as contiguous runs.  Rows longer
// than Tuning::hub_degree are cut into pieces of Tuning::piece edges that a
// second kernel spreads over all warps of the GPU.  Destinations are appended
// to the output queue with one atomic per warp.
//
// An Op supplies the per-edge work, split so that a thread can keep several
// edges' loads in flight before it issues their atomics:
//   void begin(TravCtl *c)                          load per-superstep values
//   SV src_value(uint32_t u)                        value carried from the source
//   Pre prepare(SV sv, uint32_t e, uint32_t v)      plain loads for one edge
//   void apply_n<N>(const Pre (&p)[N], const uint32_t (&v)[N], int (&act)[N])
//                                                   the atomics of a thread's N edges
//                                                   (all issued before any result is
//                                                   used); act[j] becomes 0: nothing,
//                                                   1: push v to the output queue,
//                                                   2: push to the secondary (far) queue
//   kPacked, Pre prepare_packed(SV sv, uint32_t val, uint32_t v)
//                                                   ops that set kPacked read (column,
//                                                   value) pairs from AdvanceArgs::cw
//                                                   and get the value here instead
//   bool on_input(uint32_t u)                       once per input queue entry;
//                                                   false: skip its edges now
//   void on_push(bool pushed, uint32_t v)           after each warp-wide push
//   void flush(unsigned long long relaxed)          once per thread at the end
//   kEpilogue, bool epilogue_on() / void epilogue(TravCtl *c)
//                                                   optional: when epilogue_on(),
//                                                   one thread of the last CTA of
//                                                   k_advance_pieces to finish runs
//                                                   epilogue(c) after every CTA's
//                                                   updates are visible (the
//                                                   superstep's control step, with
//                                                   no launch of its own)
#pragma once
#include <type_traits>

#include "olv_travctl.cuh"

namespace olv {

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// Append v (where p) to q with one atomic per warp.  All 32 lanes must call.
__device__ __forceinline__ void warp_push(bool p, uint32_t v, uint32_t *__restrict__ q,
                                          uint32_t *__restrict__ qsize) {
    const unsigned m = __ballot_sync(0xffffffffu, p);
    if (!m) return;
    const uint32_t lane = lane_id();
    const uint32_t leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(qsize, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (p) q[base + __popc(m & ((1u << lane) - 1u))] = v;
}

// Append the v[j] with act[j] == want (j < N) to q with one atomic per warp.
template <int N>
__device__ __forceinline__ void warp_push_n(const int (&act)[N], const uint32_t (&v)[N], int want,
                                            uint32_t *__restrict__ q, uint32_t *__restrict__ qsize) {
    unsigned m[N];
    uint32_t tot = 0;
#pragma unroll
    for (int j = 0; j < N; j++) {
        m[j] = __ballot_sync(0xffffffffu, act[j] == want);
        tot += __popc(m[j]);
    }
    if (!tot) return;
    const uint32_t lane = lane_id();
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(qsize, tot);
    base = __shfl_sync(0xffffffffu, base, 0);
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < N; j++) {
        if (act[j] == want) q[base + __popc(m[j] & lt)] = v[j];
        base += __popc(m[j]);
    }
}

// Pushes are staged in shared memory and moved to the global queue in bulk,
// so the queue's tail counter sees one atomic per CTA chunk (or per warp
// buffer) instead of one per warp per round: a single counter hit by every
// warp serialises at its L2 slice.
constexpr uint32_t kStage = 2048;   // staged entries per CTA and queue
constexpr uint32_t kWarpStage = 512;  // staged entries per warp and queue (pieces)

// Warp appends its entries with act[j] == want to a staging buffer (shared
// atomics).  A batch that does not fit goes straight to the global queue and
// records its reservation start in *s_lim: reservations are ordered, so every
// batch staged before it lies below that position, and the buffer's valid
// entries are [0, min(*s_n, *s_lim)).
template <int N>
__device__ __forceinline__ void stage_push_n(const int (&act)[N], const uint32_t (&v)[N], int want,
                                             uint32_t *s_buf, uint32_t *s_n, uint32_t *s_lim,
                                             uint32_t cap, uint32_t *__restrict__ q,
                                             uint32_t *qsize) {
    unsigned m[N];
    uint32_t tot = 0;
#pragma unroll
    for (int j = 0; j < N; j++) {
        m[j] = __ballot_sync(0xffffffffu, act[j] == want);
        tot += __popc(m[j]);
    }
    if (!tot) return;
    const uint32_t lane = lane_id();
    uint32_t pos = 0;
    if (lane == 0) {
        pos = atomicAdd(s_n, tot);
        if (pos + tot > cap) {               // does not fit: global queue instead
            atomicMin(s_lim, pos);
            pos = 0x80000000u | atomicAdd(qsize, tot);
        }
    }
    pos = __shfl_sync(0xffffffffu, pos, 0);
    uint32_t *dst = s_buf;
    if (pos & 0x80000000u) {
        dst = q;
        pos &= 0x7fffffffu;
    }
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < N; j++) {
        if (act[j] == want) dst[pos + __popc(m[j] & lt)] = v[j];
        pos += __popc(m[j]);
    }
}

// Whole CTA: move the staged entries to the global queue with one atomic.
__device__ __forceinline__ void stage_flush(uint32_t *s_buf, uint32_t *s_n, uint32_t *s_lim,
                                            uint32_t *s_base, uint32_t *__restrict__ q,
                                            uint32_t *qsize) {
    __syncthreads();
    const uint32_t n = min(*s_n, *s_lim);
    if (threadIdx.x == 0) *s_base = n ? atomicAdd(qsize, n) : 0;
    __syncthreads();
    const uint32_t base = *s_base;
    for (uint32_t i = threadIdx.x; i < n; i += kBlock) q[base + i] = s_buf[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        *s_n = 0;
        *s_lim = kStage;
    }
}

// One warp: move its staged entries to the global queue with one atomic.
__device__ __forceinline__ void warp_stage_flush(uint32_t *s_buf, uint32_t *s_n, uint32_t *s_lim,
                                                 uint32_t *__restrict__ q, uint32_t *qsize) {
    __syncwarp();
    const uint32_t n = min(*s_n, *s_lim);
    uint32_t base = 0;
    if (lane_id() == 0 && n) base = atomicAdd(qsize, n);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (uint32_t i = lane_id(); i < n; i += 32) q[base + i] = s_buf[i];
    __syncwarp();
    if (lane_id() == 0) {
        *s_n = 0;
        *s_lim = kWarpStage;
    }
    __syncwarp();
}

// Warp sum of a 64-bit value added to *dst by lane 0.  All lanes must call.
__device__ __forceinline__ void warp_add64(unsigned long long x, unsigned long long *dst) {
#pragma unroll
    for (int o = 16; o; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane_id() == 0 && x) atomicAdd(dst, x);
}

// Exclusive scan over the CTA (blockDim.x == kBlock).  s_warp holds 33 words.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t *total,
                                                         uint32_t *s_warp) {
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        constexpr int NW = kBlock / 32;
        uint32_t t = lane < NW ? s_warp[lane] : 0;
        uint32_t ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= (uint32_t)o) ti += y;
        }
        if (lane < NW) s_warp[lane] = ti - t;
        if (lane == NW - 1) s_warp[32] = ti;
    }
    __syncthreads();
    const uint32_t r = s_warp[wid] + incl - x;
    *total = s_warp[32];
    __syncthreads();
    return r;
}

#ifndef OLV_ITEMS
#define OLV_ITEMS 8
#endif
constexpr int kItems = OLV_ITEMS;   // edges per thread kept in flight

struct AdvanceArgs {
    const uint32_t *rbeg = nullptr;   // row u's edges are [rbeg[u], rend[u]) (CSR: rowptr, rowptr+1)
    const uint32_t *rend = nullptr;
    const uint2 *rng = nullptr;       // or, when set, [rng[u].x, rng[u].y) (one 8-byte load)
    const uint32_t *col = nullptr;
    const uint2 *cw = nullptr;        // Op::kPacked: (column, edge value) per edge
    TravCtl *ctl = nullptr;
    uint32_t *q0 = nullptr, *q1 = nullptr;       // queue buffers; ctl->cur selects the input
    uint32_t *far0 = nullptr, *far1 = nullptr;   // secondary queues; ctl->far_cur selects
    uint2 *pieces = nullptr;          // (row, piece index) of split hub rows
    uint32_t hub_degree = 0;
    uint32_t piece = 0;
    uint32_t want_mode = 0;           // kernel runs only when ctl->mode == want_mode ...
    const uint32_t *rbeg2 = nullptr;  // ... or, with these row ranges, when it is want_mode2
    const uint32_t *rend2 = nullptr;
    const uint2 *rng2 = nullptr;
    uint32_t want_mode2 = 0xffffffffu;   // 0xffffffff: no second mode
    const uint32_t *rbeg3 = nullptr;  // ... or, with these, when it is want_mode3
    const uint32_t *rend3 = nullptr;
    const uint2 *rng3 = nullptr;
    uint32_t want_mode3 = 0xffffffffu;   // 0xffffffff: no third mode
};

// Row ranges of the current mode.
struct RowRanges {
    const uint32_t *beg, *end;
    const uint2 *rng;
    __device__ __forceinline__ uint2 of(uint32_t u) const {
        if (rng) return __ldg(&rng[u]);
        return make_uint2(__ldg(&beg[u]), __ldg(&end[u]));
    }
};

// Row ranges for the current mode, or false when the kernel has nothing to do.
__device__ __forceinline__ bool advance_ranges(const AdvanceArgs &a, const TravCtl *c,
                                               RowRanges &r) {
    if (c->done) return false;
    const uint32_t m = c->mode;
    if (m == a.want_mode) {
        r = RowRanges{a.rbeg, a.rend, a.rng};
        return true;
    }
    if (m == a.want_mode2) {
        r = RowRanges{a.rbeg2, a.rend2, a.rng2};
        return true;
    }
    if (m == a.want_mode3) {
        r = RowRanges{a.rbeg3, a.rend3, a.rng3};
        return true;
    }
    return false;
}

// Column (and, for packed ops, the edge value) of edge e, streamed once.
template <class Op>
__device__ __forceinline__ uint32_t load_edge(const AdvanceArgs &a, uint32_t e, uint32_t &val) {
    if constexpr (Op::kPacked) {
        const uint2 x = __ldcs(&a.cw[e]);   // evict first
        val = x.y;
        return x.x;
    } else {
        val = 0;
        return __ldcs(&a.col[e]);
    }
}

template <class Op>
__device__ __forceinline__ typename Op::Pre prepare_edge(Op &op, typename Op::SV sv, uint32_t e,
                                                         uint32_t v, uint32_t val) {
    if constexpr (Op::kPacked)
        return op.prepare_packed(sv, val, v);
    else
        return op.prepare(sv, e, v);
}

// Per-superstep chunk expansion over the input queue.  A chunk is kBlock * S
// queued sources (S per thread): with short rows (a few edges per source, as
// in SSSP's light phase) a larger S spreads the scan and the barriers of a
// chunk over more edges.
template <class Op, uint32_t S = 1>
__global__ void __launch_bounds__(kBlock, Op::kMinBlocks) k_advance_chunks(AdvanceArgs a, Op op) {
    static_assert(S == 1 || S == 2 || S == 4 || S == 8, "sources per thread: 1, 2, 4 or 8");
    constexpr uint32_t kChunk = kBlock * S;   // queued sources per chunk
    constexpr uint32_t kRound = kBlock * kItems;   // edge slots per round
    TravCtl *c = a.ctl;
    RowRanges rr;
    if (!advance_ranges(a, c, rr)) return;
    op.begin(c);
    const uint32_t cur = c->cur;
    const uint32_t n = c->qsize[cur];
    const uint32_t *__restrict__ qin = cur ? a.q1 : a.q0;
    uint32_t *__restrict__ qout = cur ? a.q0 : a.q1;
    uint32_t *qout_size = &c->qsize[cur ^ 1];
    uint32_t *__restrict__ far = c->far_cur ? a.far1 : a.far0;
    uint32_t *far_size = &c->far_size[c->far_cur];

    using SV = typename Op::SV;
    __shared__ uint32_t s_beg[kChunk];
    __shared__ uint32_t s_off[kChunk];
    __shared__ SV s_val[kChunk];
    __shared__ uint32_t s_warp[33];
    constexpr uint32_t kFarStage = Op::kHasFar ? kStage : 1;
    __shared__ uint32_t s_q[kStage], s_f[kFarStage];
    __shared__ uint32_t s_qn, s_fn, s_qlim, s_flim, s_base;
    if (threadIdx.x == 0) {
        s_qn = 0;
        s_fn = 0;
        s_qlim = kStage;
        s_flim = kStage;
    }

    unsigned long long relaxed = 0;
    for (uint64_t c0 = (uint64_t)blockIdx.x * kChunk; c0 < n; c0 += (uint64_t)gridDim.x * kChunk) {
        // thread t takes the S consecutive entries c0 + t*S .. c0 + t*S + S-1;
        // the row range and the source value of every entry are loaded
        // together, before on_input's test (a value read early is at worst
        // older: an input whose value drops this superstep is queued again)
        uint32_t beg[S], deg[S], tdeg = 0, u[S];
        SV sv0[S];
        uint2 r[S];
#pragma unroll
        for (uint32_t s = 0; s < S; s++) {
            const uint64_t i = c0 + threadIdx.x * S + s;
            u[s] = i < n ? qin[i] : 0xffffffffu;
        }
#pragma unroll
        for (uint32_t s = 0; s < S; s++) {
            r[s] = make_uint2(0u, 0u);
            sv0[s] = 0;
            if (u[s] != 0xffffffffu) {
                r[s] = rr.of(u[s]);
                sv0[s] = op.src_value(u[s]);
            }
        }
#pragma unroll
        for (uint32_t s = 0; s < S; s++) {
            beg[s] = r[s].x;
            deg[s] = r[s].y - r[s].x;
            if (u[s] != 0xffffffffu && !op.on_input(u[s])) deg[s] = 0;
            if (deg[s] > a.hub_degree) {
                const uint32_t np = (deg[s] + a.piece - 1) / a.piece;
                const uint32_t b = atomicAdd(&c->npieces, np);
                for (uint32_t p = 0; p < np; p++) a.pieces[b + p] = make_uint2(u[s], p);
                relaxed += deg[s];
                deg[s] = 0;
            }
            relaxed += deg[s];
            tdeg += deg[s];
        }
        uint32_t total;
        uint32_t off = block_exclusive_scan(tdeg, &total, s_warp);
#pragma unroll
        for (uint32_t s = 0; s < S; s++) {
            s_beg[threadIdx.x * S + s] = beg[s];
            s_off[threadIdx.x * S + s] = off;
            s_val[threadIdx.x * S + s] = sv0[s];
            off += deg[s];
        }
        __syncthreads();
        for (uint32_t base = 0; base < total; base += kRound) {
            uint32_t e[kItems], v[kItems];
            SV sv[kItems];
            int act[kItems];
#pragma unroll
            for (int j = 0; j < kItems; j++) {
                const uint32_t k = base + j * kBlock + threadIdx.x;
                act[j] = k < total;
                e[j] = 0;
                sv[j] = 0;
                v[j] = 0;
                if (act[j]) {
                    // the last entry whose offset is <= k owns edge slot k
                    uint32_t lo = 0;
#pragma unroll
                    for (uint32_t step = kChunk / 2; step > 0; step >>= 1)
                        if (s_off[lo + step] <= k) lo += step;
                    e[j] = s_beg[lo] + (k - s_off[lo]);
                    sv[j] = s_val[lo];
                }
            }
            uint32_t ev[kItems];
#pragma unroll
            for (int j = 0; j < kItems; j++)
                if (act[j]) v[j] = load_edge<Op>(a, e[j], ev[j]);
            typename Op::Pre pre[kItems];
#pragma unroll
            for (int j = 0; j < kItems; j++)
                if (act[j]) pre[j] = prepare_edge(op, sv[j], e[j], v[j], ev[j]);
            op.template apply_n<kItems>(pre, v, act);
            stage_push_n<kItems>(act, v, 1, s_q, &s_qn, &s_qlim, kStage, qout, qout_size);
            if (Op::kHasFar)
                stage_push_n<kItems>(act, v, 2, s_f, &s_fn, &s_flim, kStage, far, far_size);
#pragma unroll
            for (int j = 0; j < kItems; j++) op.on_push(act[j] == 1, v[j]);
        }
        // the staging buffers are emptied once half full, and at the end:
        // most chunks then pay no flush (three barriers and an atomic each)
        __syncthreads();
        if (min(s_qn, s_qlim) >= kStage / 2) stage_flush(s_q, &s_qn, &s_qlim, &s_base, qout, qout_size);
        if (Op::kHasFar && min(s_fn, s_flim) >= kStage / 2)
            stage_flush(s_f, &s_fn, &s_flim, &s_base, far, far_size);
        __syncthreads();
    }
    stage_flush(s_q, &s_qn, &s_qlim, &s_base, qout, qout_size);
    if (Op::kHasFar) stage_flush(s_f, &s_fn, &s_flim, &s_base, far, far_size);
    op.flush(relaxed);
}

template <class Op, class = void>
struct op_epilogue : std::false_type {};
template <class Op>
struct op_epilogue<Op, std::void_t<decltype(Op::kEpilogue)>>
    : std::integral_constant<bool, Op::kEpilogue> {};

template <class Op>
__device__ __forceinline__ void advance_pieces_body(const AdvanceArgs &a, Op &op, TravCtl *c,
                                                    const RowRanges &rr, uint32_t np);

// Hub pieces: one warp per piece of up to a.piece edges.
template <class Op>
__global__ void __launch_bounds__(kBlock, Op::kMinBlocks) k_advance_pieces(AdvanceArgs a, Op op) {
    TravCtl *c = a.ctl;
    RowRanges rr;
    if (advance_ranges(a, c, rr)) {
        const uint32_t np = c->npieces;
        if (np) advance_pieces_body(a, op, c, rr, np);
    }
    if constexpr (op_epilogue<Op>::value) {
        if (!op.epilogue_on()) return;   // kernel argument: the same in every CTA
        __shared__ uint32_t s_last;
        __threadfence();   // this thread's updates are visible before the CTA counts itself
        __syncthreads();
        if (threadIdx.x == 0) {
            s_last = atomicAdd(&c->end_arrive, 1u) == gridDim.x - 1;
            if (s_last) {
                __threadfence();   // every other CTA's updates are visible from here
                c->end_arrive = 0;
                op.epilogue(c);
            }
        }
    }
}

template <class Op>
__device__ __forceinline__ void advance_pieces_body(const AdvanceArgs &a, Op &op, TravCtl *c,
                                                    const RowRanges &rr, uint32_t np) {
    op.begin(c);
    const uint32_t cur = c->cur;
    uint32_t *__restrict__ qout = cur ? a.q0 : a.q1;
    uint32_t *qout_size = &c->qsize[cur ^ 1];
    uint32_t *__restrict__ far = c->far_cur ? a.far1 : a.far0;
    uint32_t *far_size = &c->far_size[c->far_cur];
    const uint32_t lane = lane_id();
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    constexpr uint32_t kFarW = Op::kHasFar ? kWarpStage : 1;
    __shared__ uint32_t s_q[kBlock / 32][kWarpStage], s_f[kBlock / 32][kFarW];
    __shared__ uint32_t s_qn[kBlock / 32], s_fn[kBlock / 32];
    __shared__ uint32_t s_qlim[kBlock / 32], s_flim[kBlock / 32];
    const uint32_t wl = threadIdx.x >> 5;
    if (lane == 0) {
        s_qn[wl] = 0;
        s_fn[wl] = 0;
        s_qlim[wl] = kWarpStage;
        s_flim[wl] = kWarpStage;
    }
    __syncwarp();
    for (uint32_t p = warp; p < np; p += nwarps) {
        const uint2 pc = a.pieces[p];
        const uint32_t u = pc.x;
        const uint2 r = rr.of(u);
        const uint32_t rb = r.x, re = r.y;
        const uint32_t b = rb + pc.y * a.piece;
        const uint32_t e_end = min(re, b + a.piece);
        const typename Op::SV sv = op.src_value(u);
        for (uint32_t base = b; base < e_end; base += 32 * kItems) {
            uint32_t e[kItems], v[kItems], ev[kItems];
            int act[kItems];
#pragma unroll
            for (int j = 0; j < kItems; j++) {
                e[j] = base + j * 32 + lane;
                act[j] = e[j] < e_end;
                v[j] = act[j] ? load_edge<Op>(a, e[j], ev[j]) : 0;
            }
            typename Op::Pre pre[kItems];
#pragma unroll
            for (int j = 0; j < kItems; j++)
                if (act[j]) pre[j] = prepare_edge(op, sv, e[j], v[j], ev[j]);
            op.template apply_n<kItems>(pre, v, act);
            // flush before a round could overflow the warp's buffers (the
            // counts were last written by lane 0's shared atomics)
            __syncwarp();
            if (s_qn[wl] + 32 * kItems > kWarpStage)
                warp_stage_flush(s_q[wl], &s_qn[wl], &s_qlim[wl], qout, qout_size);
            stage_push_n<kItems>(act, v, 1, s_q[wl], &s_qn[wl], &s_qlim[wl], kWarpStage, qout,
                                 qout_size);
            if (Op::kHasFar) {
                if (s_fn[wl] + 32 * kItems > kWarpStage)
                    warp_stage_flush(s_f[wl], &s_fn[wl], &s_flim[wl], far, far_size);
                stage_push_n<kItems>(act, v, 2, s_f[wl], &s_fn[wl], &s_flim[wl], kWarpStage, far,
                                     far_size);
            }
#pragma unroll
            for (int j = 0; j < kItems; j++) op.on_push(act[j] == 1, v[j]);
        }
    }
    warp_stage_flush(s_q[wl], &s_qn[wl], &s_qlim[wl], qout, qout_size);
    if (Op::kHasFar) warp_stage_flush(s_f[wl], &s_fn[wl], &s_flim[wl], far, far_size);
    op.flush(0);
}

// ------------------------------------------------------------------ pull --
// Pull over in-edge rows (the reverse graph): every row r in [0, n) that the
// Op wants reduces the contributions of its in-edges whose source passes the
// Op's test, and is listed once when it got at least one.  Load-balanced like
// the push: a CTA takes kBlock consecutive rows, scans their in-degrees and
// lets all threads walk the chunk's in-edges in order, reducing into a
// per-row slot in shared memory; each row's owner then stores the slot and
// lists the row.  Rows over hub_degree in-edges go to pieces of `piece` edges
// that k_pull_pieces spreads over all warps; they reduce straight into the
// global accumulator.  An Op supplies:
//   using Acc                                     accumulator type
//   static constexpr int kMinBlocks
//   static constexpr bool kFirstHit               a row stops at its first contribution
//   bool row_wanted(uint32_t r)
//   Acc acc_load(uint32_t r)                      the row's current (reset) value
//   bool contributes(uint32_t u, uint32_t e, Acc &x)   source u over in-edge e
//   void reduce_slot(Acc &slot, const Acc &x)     into shared memory
//   void reduce_row(uint32_t r, const Acc &x)     into the global accumulator
//   void store(uint32_t r, const Acc &slot)
//   bool mark(uint32_t r)                         true when r is newly marked
// and, optionally, for the first-hit kernels (kFirstHit):
//   bool passes(uint32_t u)                       source u would contribute (a plain
//                                                 load: several are kept in flight)
//   Acc contribution(uint32_t u, uint32_t e)      its contribution (u passes)
struct PullArgs {
    const uint32_t *colptr = nullptr;   // in-edges of r: [colptr[r], colptr[r+1])
    const uint32_t *rowidx = nullptr;   // their sources
    TravCtl *ctl = nullptr;             // runs only when ctl->mode == want_mode
    uint32_t want_mode = 0;
    uint32_t n = 0;                     // rows
    uint2 *pieces = nullptr;            // (row, piece) of hub rows; count in ctl->npieces
    uint32_t hub_degree = 0;
    uint32_t piece = 0;
    uint32_t *qout = nullptr;           // rows with a contribution; count in ctl->qsize[1]
    // first-hit pulls: per row, the in-neighbour to probe before the others
    // (kNoFirst: no in-edges) and that in-edge's position; null: no probe
    const uint32_t *first = nullptr;
    const uint32_t *firstpos = nullptr;
};

constexpr uint32_t kNoFirst = 0xffffffffu;

template <class Op>
__global__ void __launch_bounds__(kBlock, Op::kMinBlocks) k_pull_chunks(PullArgs a, Op op) {
    TravCtl *c = a.ctl;
    if (c->done || c->mode != a.want_mode) return;
    using Acc = typename Op::Acc;
    __shared__ uint32_t s_beg[kBlock], s_off[kBlock], s_warp[33];
    __shared__ int s_hit[kBlock];
    __shared__ __align__(16) unsigned char s_acc_raw[kBlock * sizeof(Acc)];
    Acc *s_acc = reinterpret_cast<Acc *>(s_acc_raw);
    uint32_t *qsize = &c->qsize[1];
    for (uint64_t base_row = (uint64_t)blockIdx.x * kBlock; base_row < a.n;
         base_row += (uint64_t)gridDim.x * kBlock) {
        const uint32_t r = (uint32_t)(base_row + threadIdx.x);
        uint32_t beg = 0, deg = 0;
        if (r < a.n && op.row_wanted(r)) {
            beg = __ldg(&a.colptr[r]);
            deg = __ldg(&a.colptr[r + 1]) - beg;
            if (deg > a.hub_degree) {
                const uint32_t np = (deg + a.piece - 1) / a.piece;
                const uint32_t b = atomicAdd(&c->npieces, np);
                for (uint32_t p = 0; p < np; p++) a.pieces[b + p] = make_uint2(r, p);
                deg = 0;
            }
        }
        if (deg) s_acc[threadIdx.x] = op.acc_load(r);
        s_hit[threadIdx.x] = 0;
        uint32_t total;
        const uint32_t off = block_exclusive_scan(deg, &total, s_warp);
        s_beg[threadIdx.x] = beg;
        s_off[threadIdx.x] = off;
        __syncthreads();
        for (uint32_t base = 0; base < total; base += kBlock * kItems) {
            uint32_t lo[kItems], u[kItems], e[kItems];
            bool act[kItems];
#pragma unroll
            for (int j = 0; j < kItems; j++) {
                const uint32_t k = base + j * kBlock + threadIdx.x;
                act[j] = k < total;
                lo[j] = 0;
                u[j] = 0;
                e[j] = 0;
                if (act[j]) {
                    uint32_t l = 0;
#pragma unroll
                    for (uint32_t step = kBlock / 2; step > 0; step >>= 1)
                        if (s_off[l + step] <= k) l += step;
                    lo[j] = l;
                    e[j] = s_beg[l] + (k - s_off[l]);
                    if (Op::kFirstHit && s_hit[l]) act[j] = false;
                }
            }
#pragma unroll
            for (int j = 0; j < kItems; j++)
                if (act[j]) u[j] = __ldcs(&a.rowidx[e[j]]);   // streamed once: evict first
#pragma unroll
            for (int j = 0; j < kItems; j++) {
                Acc x;
                if (act[j] && op.contributes(u[j], e[j], x)) {
                    op.reduce_slot(s_acc[lo[j]], x);
                    s_hit[lo[j]] = 1;
                }
            }
        }
        __syncthreads();
        bool newly = false;
        if (deg && s_hit[threadIdx.x]) {
            op.store(r, s_acc[threadIdx.x]);
            newly = op.mark(r);
        }
        warp_push(newly, r, a.qout, qsize);
        __syncthreads();   // the shared arrays are rewritten by the next chunk
    }
}

// Hub rows of the pull: one warp per piece, contributions reduced into the
// global accumulator.
template <class Op>
__global__ void __launch_bounds__(kBlock, Op::kMinBlocks) k_pull_pieces(PullArgs a, Op op) {
    TravCtl *c = a.ctl;
    if (c->done || c->mode != a.want_mode) return;
    const uint32_t np = c->npieces;
    if (np == 0) return;
    using Acc = typename Op::Acc;
    const uint32_t lane = lane_id();
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t p = warp; p < np; p += nwarps) {
        const uint2 pc = a.pieces[p];
        const uint32_t r = pc.x;
        const uint32_t rb = __ldg(&a.colptr[r]), re = __ldg(&a.colptr[r + 1]);
        const uint32_t b = rb + pc.y * a.piece;
        const uint32_t e_end = min(re, b + a.piece);
        bool hit = false;
        for (uint32_t base = b; base < e_end; base += 32 * kItems) {
            uint32_t u[kItems], e[kItems];
#pragma unroll
            for (int j = 0; j < kItems; j++) {
                e[j] = base + j * 32 + lane;
                u[j] = e[j] < e_end ? __ldcs(&a.rowidx[e[j]]) : 0;
            }
#pragma unroll
            for (int j = 0; j < kItems; j++) {
                Acc x;
                if (e[j] < e_end && op.contributes(u[j], e[j], x)) {
                    op.reduce_row(r, x);
                    hit = true;
                }
            }
            if (Op::kFirstHit && __any_sync(0xffffffffu, hit)) break;
        }
        const bool any = __any_sync(0xffffffffu, hit);
        bool newly = false;
        if (any && lane == 0) newly = op.mark(r);
        warp_push(newly, r, a.qout, &c->qsize[1]);
    }
}

// First-contribution pull (Ops with kFirstHit: any single contribution is
// enough, as for BFS levels): a bottom-up step that stops each row at a
// contributing in-edge.  k_pull_first_rows gives every wanted row to one
// thread.  With a.first set, the thread probes one in-edge, the row's
// likeliest parent (a.first[r], a.firstpos[r]: coalesced loads), and lists
// the row for k_pull_first_long when the probe fails and the row has more
// in-edges.  Without it, a row with at most kFirstLight in-edges reads them
// four at a time and stops at the first source that passes (CSC order);
// longer rows are listed.  The list lives in a.pieces (count in
// ctl->npieces): k_pull_first_long gives each listed row a group of 8 lanes
// that scans its in-edges from the start, 32 per step, and stops at the
// first passing one in CSC order.  Ops with passes() / contribution() test a
// step's sources with all their loads in flight and gather only the first
// passing one; Ops with mark_warp() flag a warp's rows with one call.
#ifndef OLV_FIRST_LIGHT
#define OLV_FIRST_LIGHT 32
#endif
constexpr uint32_t kFirstLight = OLV_FIRST_LIGHT;
constexpr uint32_t kFirstGroup = 8;   // lanes per long row

template <class Op, class = void>
struct op_has_passes : std::false_type {};
template <class Op>
struct op_has_passes<Op, std::void_t<decltype(std::declval<Op &>().passes(0u))>>
    : std::true_type {};

// The first of n (<= 4) sources u[0..n) that contributes, in order: its index
// (or -1) and its contribution in x.
template <class Op>
__device__ __forceinline__ int first_contribution(Op &op, const uint32_t (&u)[4], uint32_t e0,
                                                  uint32_t n, typename Op::Acc &x) {
    if constexpr (op_has_passes<Op>::value) {
        bool p[4];
#pragma unroll
        for (int j = 0; j < 4; j++) p[j] = (uint32_t)j < n && op.passes(u[j]);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (p[j]) {
                x = op.contribution(u[j], e0 + j);
                return j;
            }
        return -1;
    } else {
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((uint32_t)j < n && op.contributes(u[j], e0 + j, x)) return j;
        return -1;
    }
}

template <class Op, class = void>
struct op_has_mark_warp : std::false_type {};
template <class Op>
struct op_has_mark_warp<Op, std::void_t<decltype(std::declval<Op &>().mark_warp(0u, 0u))>>
    : std::true_type {};

// The rows of this warp's lanes that hit (r = r0 + lane, r0 a multiple of 32)
// flagged by the Op: one mark_warp call for the warp when the Op has it, else
// mark() per row.  True for the rows whose flag this call set.
template <class Op>
__device__ __forceinline__ bool mark_rows(Op &op, bool hit, uint32_t r) {
    if constexpr (op_has_mark_warp<Op>::value) {
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        const uint32_t lane = lane_id();
        uint32_t set = 0;
        if (m && lane == 0) set = op.mark_warp(r, m);
        set = __shfl_sync(0xffffffffu, set, 0);
        return (set >> lane) & 1u;
    } else {
        return hit && op.mark(r);
    }
}

template <class Op>
__global__ void __launch_bounds__(kBlock, Op::kMinBlocks) k_pull_first_rows(PullArgs a, Op op) {
    TravCtl *c = a.ctl;
    if (c->done || c->mode != a.want_mode) return;
    using Acc = typename Op::Acc;
    // both lists staged in shared memory (one counter atomic per flush, not
    // per warp and row block: every warp of the grid appends to them)
    __shared__ uint32_t s_q[kStage], s_l[kStage];
    __shared__ uint32_t s_qn, s_qlim, s_ln, s_llim, s_base;
    uint32_t *lrows = reinterpret_cast<uint32_t *>(a.pieces);
    if (threadIdx.x == 0) {
        s_qn = 0;
        s_qlim = kStage;
        s_ln = 0;
        s_llim = kStage;
    }
    __syncthreads();
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < a.n;
         base += (uint64_t)gridDim.x * kBlock) {
        const uint32_t r = (uint32_t)(base + threadIdx.x);
        bool hit = false, is_long = false;
        if (r < a.n && op.row_wanted(r)) {
            if (a.first) {
                // one probe of the row's likeliest parent (coalesced loads);
                // a row it fails with more in-edges goes to the group kernel
                const uint32_t u = __ldg(&a.first[r]);
                if (u != kNoFirst) {
                    Acc x;
                    bool p;
                    if constexpr (op_has_passes<Op>::value) {
                        p = op.passes(u);
                        if (p) x = op.contribution(u, __ldg(&a.firstpos[r]));
                    } else {
                        p = op.contributes(u, __ldg(&a.firstpos[r]), x);
                    }
                    if (p) {
                        op.reduce_row(r, x);
                        hit = true;
                    } else {
                        is_long = __ldg(&a.colptr[r + 1]) - __ldg(&a.colptr[r]) > 1;
                    }
                }
            } else {
                const uint32_t b = __ldg(&a.colptr[r]), e = __ldg(&a.colptr[r + 1]);
                if (e - b > kFirstLight) {
                    is_long = true;
                } else {
                    for (uint32_t i = b; i < e; i += 4) {
                        const uint32_t n = min(4u, e - i);
                        uint32_t u[4];
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            u[j] = (uint32_t)j < n ? __ldcs(&a.rowidx[i + j]) : 0;
                        Acc x;
                        if (first_contribution(op, u, i, n, x) >= 0) {
                            op.reduce_row(r, x);
                            hit = true;
                            break;
                        }
                    }
                }
            }
        }
        const bool newly = mark_rows(op, hit, r);
        const uint32_t vr[1] = {r};
        const int aq[1] = {newly ? 1 : 0}, al[1] = {is_long ? 1 : 0};
        stage_push_n<1>(aq, vr, 1, s_q, &s_qn, &s_qlim, kStage, a.qout, &c->qsize[1]);
        stage_push_n<1>(al, vr, 1, s_l, &s_ln, &s_llim, kStage, lrows, &c->npieces);
        __syncthreads();
        if (min(s_qn, s_qlim) >= kStage / 2)
            stage_flush(s_q, &s_qn, &s_qlim, &s_base, a.qout, &c->qsize[1]);
        if (min(s_ln, s_llim) >= kStage / 2)
            stage_flush(s_l, &s_ln, &s_llim, &s_base, lrows, &c->npieces);
        __syncthreads();
    }
    stage_flush(s_q, &s_qn, &s_qlim, &s_base, a.qout, &c->qsize[1]);
    stage_flush(s_l, &s_ln, &s_llim, &s_base, lrows, &c->npieces);
}

// Listed rows, a group of 8 lanes per row (four rows per warp): each step
// reads the row's next 32 in-edges, lane s of the group taking positions
// s, s+8, s+16, s+24 (every load instruction reads one 32-byte sector per
// group), and the row stops at its first passing in-edge in CSC order.
template <class Op>
__global__ void __launch_bounds__(kBlock, Op::kMinBlocks) k_pull_first_long(PullArgs a, Op op) {
    TravCtl *c = a.ctl;
    if (c->done || c->mode != a.want_mode) return;
    using Acc = typename Op::Acc;
    constexpr uint32_t kGroups = 32 / kFirstGroup;
    constexpr uint32_t kStep = kFirstGroup * 4;   // in-edges per group step
    const uint32_t nl = c->npieces;
    const uint32_t *rows = reinterpret_cast<const uint32_t *>(a.pieces);
    const uint32_t lane = lane_id();
    const uint32_t grp = lane / kFirstGroup, sub = lane % kFirstGroup;
    // found rows staged per warp, one counter atomic per flush
    const uint32_t wl = threadIdx.x >> 5;
    __shared__ uint32_t s_q[kBlock / 32][kWarpStage];
    __shared__ uint32_t s_qn[kBlock / 32], s_qlim[kBlock / 32];
    if (lane == 0) {
        s_qn[wl] = 0;
        s_qlim[wl] = kWarpStage;
    }
    __syncwarp();
    const uint32_t gshift = grp * kFirstGroup;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t k0 = warp * kGroups; k0 < nl; k0 += nwarps * kGroups) {
        const uint32_t k = k0 + grp;
        uint32_t r = 0, i = 0, e = 0;
        if (k < nl) {
            r = rows[k];
            i = __ldg(&a.colptr[r]);
            e = __ldg(&a.colptr[r + 1]);
        }
        bool found = false;
        // every lane stays in the loop until all four groups are done (warp votes)
        while (__any_sync(0xffffffffu, !found && i < e)) {
            const bool active = !found && i < e;
            uint32_t u[4];
            bool p[4];
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const uint32_t j = i + t * kFirstGroup + sub;
                u[t] = active && j < e ? __ldcs(&a.rowidx[j]) : 0;
            }
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const uint32_t j = i + t * kFirstGroup + sub;
                if constexpr (op_has_passes<Op>::value) {
                    p[t] = active && j < e && op.passes(u[t]);
                } else {
                    Acc y;
                    p[t] = active && j < e && op.contributes(u[t], j, y);
                }
            }
            // the first passing position of the step: lowest t, then lowest lane
            int tw = -1;
            uint32_t gw = 0;
#pragma unroll
            for (int t = 3; t >= 0; t--) {
                const uint32_t gm =
                    (__ballot_sync(0xffffffffu, p[t]) >> gshift) & ((1u << kFirstGroup) - 1u);
                if (gm) {
                    tw = t;
                    gw = gm;
                }
            }
            if (active && tw >= 0) {
                if (sub == (uint32_t)(__ffs(gw) - 1)) {
                    uint32_t uw = u[0];
#pragma unroll
                    for (int t = 1; t < 4; t++)
                        if (t == tw) uw = u[t];
                    const uint32_t j = i + (uint32_t)tw * kFirstGroup + sub;
                    Acc x;
                    if constexpr (op_has_passes<Op>::value)
                        x = op.contribution(uw, j);
                    else
                        op.contributes(uw, j, x);
                    op.reduce_row(r, x);
                }
                found = true;
            }
            i += kStep;
        }
        const bool newly = found && sub == 0 && op.mark(r);
        const uint32_t vr[1] = {r};
        const int aq[1] = {newly ? 1 : 0};
        __syncwarp();
        if (s_qn[wl] + 32 > kWarpStage)
            warp_stage_flush(s_q[wl], &s_qn[wl], &s_qlim[wl], a.qout, &c->qsize[1]);
        stage_push_n<1>(aq, vr, 1, s_q[wl], &s_qn[wl], &s_qlim[wl], kWarpStage, a.qout,
                        &c->qsize[1]);
    }
    warp_stage_flush(s_q[wl], &s_qn[wl], &s_qlim[wl], a.qout, &c->qsize[1]);
}

}  // namespace olv
