// Host generator of a batch of Erdos-Renyi digraphs packed block-diagonally
// in one CSR (no reference counterpart; it builds the batched workload).
//
// Instance i has V_i = vmin + h(seed, i) mod (vmax - vmin + 1) vertices and
// exactly deg * V_i edges drawn uniformly without self-loops or duplicates:
// candidate j of instance i is (u, v) = (h(s_i, 2j) mod V_i, h(s_i, 2j+1) mod V_i),
// self-loops are rejected and a repeated pair keeps its first draw, until
// deg * V_i edges are kept.  Vertex ids are offset by the instance's start;
// rows are sorted by destination.  Instances are generated in parallel on the
// host threads.
#include <algorithm>
#include <thread>
#include <vector>

#include "olv_internal.cuh"
#include "olv_rng.cuh"

namespace olv {

static void er_instance(uint64_t seed, uint32_t n, uint64_t m, std::vector<uint64_t> &edges) {
    const uint64_t possible = (uint64_t)n * (n - 1);
    if (m > possible) m = possible;
    edges.clear();
    std::vector<std::pair<uint64_t, uint64_t>> cand;   // (key, draw index)
    uint64_t j = 0;
    std::vector<uint64_t> kept;
    while (kept.size() < m) {
        const uint64_t want = (m - kept.size()) + (m - kept.size()) / 8 + 64;
        cand.clear();
        for (const uint64_t k : kept) cand.push_back({k, 0});   // already kept: earlier draws
        for (uint64_t t = 0; t < want; t++, j++) {
            const uint32_t u = (uint32_t)(hash64(seed, 2 * j) % n);
            const uint32_t v = (uint32_t)(hash64(seed, 2 * j + 1) % n);
            if (u == v) continue;
            cand.push_back({((uint64_t)u << 32) | v, j + 1});
        }
        std::sort(cand.begin(), cand.end());
        std::vector<std::pair<uint64_t, uint64_t>> uniq;   // first draw of each pair
        for (size_t i = 0; i < cand.size(); i++)
            if (i == 0 || cand[i].first != cand[i - 1].first) uniq.push_back(cand[i]);
        std::sort(uniq.begin(), uniq.end(),
                  [](const std::pair<uint64_t, uint64_t> &a, const std::pair<uint64_t, uint64_t> &b) {
                      return a.second < b.second;
                  });
        kept.clear();
        for (size_t i = 0; i < uniq.size() && kept.size() < m; i++) kept.push_back(uniq[i].first);
    }
    edges = kept;
    std::sort(edges.begin(), edges.end());
}

uint32_t er_instance_size(uint64_t seed, int i, uint32_t vmin, uint32_t vmax) {
    return vmin + (uint32_t)(hash64(seed ^ 0xa5a5a5a5ULL, (uint64_t)i) % (uint64_t)(vmax - vmin + 1));
}

int build_er_batch(int count, uint32_t vmin, uint32_t vmax, uint32_t deg, uint64_t seed,
                   std::vector<uint32_t> &offsets, std::vector<uint32_t> &rowptr,
                   std::vector<uint32_t> &col) {
    offsets.assign(count + 1, 0);
    for (int i = 0; i < count; i++)
        offsets[i + 1] = offsets[i] + er_instance_size(seed, i, vmin, vmax);
    std::vector<std::vector<uint64_t>> inst(count);
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++)
        th.emplace_back([&, t]() {
            for (int i = (int)t; i < count; i += (int)nt) {
                const uint32_t n = offsets[i + 1] - offsets[i];
                er_instance(hash64(seed, 1000003ULL + i), n, (uint64_t)deg * n, inst[i]);
            }
        });
    for (auto &x : th) x.join();
    const uint64_t V = offsets[count];
    uint64_t E = 0;
    for (auto &x : inst) E += x.size();
    if (E > 0xffffffffULL || V > 0xffffffffULL) return OLV_ERR_LIMIT;
    rowptr.assign(V + 1, 0);
    col.resize(E);
    uint64_t pos = 0;
    for (int i = 0; i < count; i++) {
        const uint32_t base = offsets[i];
        for (const uint64_t k : inst[i]) {
            rowptr[base + (uint32_t)(k >> 32) + 1]++;
            col[pos++] = base + (uint32_t)k;
        }
    }
    for (uint64_t v = 0; v < V; v++) rowptr[v + 1] += rowptr[v];
    return OLV_OK;
}

}  // namespace olv

using namespace olv;

extern "C" int olv_graph_create_er_batch(int count, uint32_t vmin, uint32_t vmax,
                                         uint32_t avg_degree, uint64_t seed,
                                         uint32_t *inst_offsets, olv_graph **out) {
    OLV_CHECK_ARG(out && inst_offsets, "olv_graph_create_er_batch: null pointer");
    OLV_CHECK_ARG(count >= 1, "olv_graph_create_er_batch: count must be >= 1");
    OLV_CHECK_ARG(vmin >= 2 && vmax >= vmin, "olv_graph_create_er_batch: need 2 <= vmin <= vmax");
    OLV_CHECK_ARG(avg_degree >= 1, "olv_graph_create_er_batch: avg_degree must be >= 1");
    std::vector<uint32_t> offsets, rowptr, col;
    int r = build_er_batch(count, vmin, vmax, avg_degree, seed, offsets, rowptr, col);
    if (r != OLV_OK) {
        set_error("olv_graph_create_er_batch: batch exceeds uint32 ids");
        return r;
    }
    memcpy(inst_offsets, offsets.data(), (count + 1) * sizeof(uint32_t));
    return olv_graph_create(rowptr.data(), col.data(), nullptr, OLV_W_NONE,
                            (uint32_t)(rowptr.size() - 1), col.size(), out);
}
