/*
 * olive_b200 source-compatible header layer: CsrGraph<VertexValue,EdgeValue>
 * with the reference's public members and loaders (csrGraph.h:55-285).
 *
 * fromEdgeListFile reads "V E" then "src dst [value]" lines ('#' lines are
 * comments, csrGraph.h:106-171).  Differences, on purpose:
 *   - tuples are stably sorted by source before the CSR is built; the
 *     reference assumed src-sorted input (its sort, csrGraph.h:149, is
 *     commented out) and attached out-of-order tuples to the wrong row;
 *   - an optional third column is stored in edgeValues (the reference
 *     parsed a constant 1 and never stored it);
 *   - the file is parsed from one buffered read instead of fscanf per line;
 *     ids >= V are reported and dropped instead of writing out of bounds;
 *   - a file that starts with the 8 bytes "OLVCSR1\n" is a binary CSR dump
 *     (no reference counterpart; text files of 10^8+ edges take minutes to
 *     parse): uint64 V, uint64 E, uint64 flags (bit 0: uint32 edge values
 *     follow), uint32 rowptr[V+1], uint32 col[E], [uint32 values[E]], all
 *     little-endian.  The rows are taken as stored.  olv_graph_save and
 *     olive_b200.write_csr_binary write it.
 * fromDimacsFile follows csrGraph.h:177-236: header "V E" with E undirected
 * (stored edges = 2E), then one line of 1-based neighbour ids per vertex;
 * '#' and '%' lines are comments; extra header fields are ignored.
 */
#ifndef OLIVE_CSR_GRAPH_H
#define OLIVE_CSR_GRAPH_H

#include <algorithm>
#include <cmath>
#include <cstring>
#include <iostream>
#include <vector>

#include "common.h"
#include "edgeTuple.h"
#include "logging.h"
#include "timer.h"
#include "utils.h"

namespace olive_detail {

struct FileBuf {
    std::vector<char> data;
    bool ok = false;
    explicit FileBuf(const char *path) {
        FILE *f = fopen(path, "rb");
        if (!f) return;
        fseek(f, 0, SEEK_END);
        long n = ftell(f);
        fseek(f, 0, SEEK_SET);
        data.resize(n > 0 ? (size_t)n + 1 : 1);
        size_t got = n > 0 ? fread(data.data(), 1, (size_t)n, f) : 0;
        data.resize(got + 1);
        data[got] = '\0';
        fclose(f);
        ok = true;
    }
};

// Parse an unsigned decimal at p (skipping blanks); returns false at end of line.
inline bool next_uint(const char *&p, unsigned long long &x) {
    while (*p == ' ' || *p == '\t' || *p == '\r') p++;
    if (*p < '0' || *p > '9') return false;
    unsigned long long v = 0;
    while (*p >= '0' && *p <= '9') v = v * 10 + (unsigned long long)(*p++ - '0');
    x = v;
    return true;
}

inline void skip_line(const char *&p) {
    while (*p && *p != '\n') p++;
    if (*p == '\n') p++;
}

}  // namespace olive_detail

template <typename VertexValue, typename EdgeValue>
class CsrGraph {
public:
    VertexId vertexCount;
    EdgeId edgeCount;
    EdgeId *vertices;
    VertexId *edges;
    EdgeValue *edgeValues;
    VertexValue *vertexValues;

    CsrGraph()
        : vertexCount(0), edgeCount(0), vertices(NULL), edges(NULL), edgeValues(NULL),
          vertexValues(NULL) {}

    ~CsrGraph() { release(); }

    void release() {
        delete[] vertices;
        delete[] edges;
        delete[] edgeValues;
        delete[] vertexValues;
        vertices = NULL;
        edges = NULL;
        edgeValues = NULL;
        vertexValues = NULL;
    }

    void initGraph(VertexId V, EdgeId E) {
        release();
        vertexCount = V;
        edgeCount = E;
        vertices = new EdgeId[(size_t)V + 1];
        edges = new VertexId[E ? E : 1];
        edgeValues = new EdgeValue[E ? E : 1]();
        vertexValues = new VertexValue[V ? V : 1]();
    }

    void fromEdgeListFile(const char *path) {
        using namespace olive_detail;
        FileBuf fb(path);
        if (!fb.ok) {
            LOG(ERROR) << "Can not open graph file: " << path;
            return;
        }
        Stopwatch sw;
        sw.start();
        if (fromBinary(fb, path)) {
            LOG(INFO) << "It took " << sw.getElapsedMillis()
                      << "ms to load the binary CSR graph.";
            return;
        }
        const char *p = fb.data.data();
        unsigned long long V = 0, E = 0;
        bool header = false;
        std::vector<VertexId> src, dst;
        std::vector<EdgeValue> val;
        size_t dropped = 0;
        while (*p) {
            if (*p == '#' || *p == '\n' || *p == '\r') {
                skip_line(p);
                continue;
            }
            unsigned long long a, b, c;
            const char *q = p;
            if (!next_uint(q, a) || !next_uint(q, b)) {
                skip_line(p);
                continue;
            }
            if (!header) {
                V = a;
                E = b;
                header = true;
                LOG(INFO) << "Parsing graph: " << V << " nodes, " << E << " edges";
                assert(V > 0);
                src.reserve(E);
                dst.reserve(E);
                val.reserve(E);
            } else if (src.size() < E) {
                bool has = next_uint(q, c);
                if (a >= V || b >= V) {
                    dropped++;
                } else {
                    src.push_back((VertexId)a);
                    dst.push_back((VertexId)b);
                    val.push_back(has ? (EdgeValue)c : EdgeValue(1));
                }
            }
            p = q;
            skip_line(p);
        }
        if (dropped) LOG(ERROR) << dropped << " edges with ids >= " << V << " dropped";
        if (src.size() != E)
            LOG(WARNING) << "header says " << E << " edges, parsed " << src.size();
        LOG(INFO) << "It took " << sw.getElapsedMillis() << "ms to parse " << src.size()
                  << " edge tuples.";
        buildFromTuples((VertexId)V, src, dst, val);
        LOG(INFO) << "It took " << sw.getElapsedMillis()
                  << "ms to generate the CSR graph from edge list file.";
    }

    void fromDimacsFile(const char *path) {
        using namespace olive_detail;
        FileBuf fb(path);
        if (!fb.ok) {
            LOG(ERROR) << "Can not open graph file: " << path;
            return;
        }
        Stopwatch sw;
        sw.start();
        const char *p = fb.data.data();
        unsigned long long V = 0, E = 0;
        while (*p && (*p == '#' || *p == '%')) skip_line(p);
        const char *q = p;
        if (!next_uint(q, V) || !next_uint(q, E)) {
            LOG(ERROR) << "bad DIMACS header in " << path;
            return;
        }
        skip_line(p);
        initGraph((VertexId)V, (EdgeId)(E * 2));
        LOG(INFO) << "Parsing graph: " << V << " nodes, " << E << " (bi)edges";
        unsigned long long parsed = 0;
        VertexId v = 0;
        while (*p && v < V) {
            if (*p == '#' || *p == '%') {
                skip_line(p);
                continue;
            }
            vertices[v] = (EdgeId)parsed;
            unsigned long long x;
            while (next_uint(p, x)) {
                if (parsed < E * 2 && x >= 1 && x <= V) edges[parsed] = (VertexId)(x - 1);
                parsed++;
            }
            skip_line(p);
            v++;
        }
        for (; v <= V; v++) vertices[v] = (EdgeId)std::min<unsigned long long>(parsed, E * 2);
        if (parsed != E * 2) {
            LOG(ERROR) << parsed << "!=" << E * 2;
            assert(0);
        }
        LOG(INFO) << "It took " << sw.getElapsedMillis()
                  << "ms to generate the CSR graph from Dimacs file.";
    }

    /** Degree histogram in powers of two (csrGraph.h:241-285). */
    void print(bool verbose = false) const {
        if (verbose)
            for (VertexId v = 0; v < vertexCount; v++) {
                printf("[%u] ", v);
                for (EdgeId e = vertices[v]; e < vertices[v + 1]; e++) printf(" ->%u", edges[e]);
                printf("\n");
            }
        size_t hist[33] = {0};
        int top = 0;
        for (VertexId v = 0; v < vertexCount; v++) {
            EdgeId d = vertices[v + 1] - vertices[v];
            int slot = 0;
            while (d) {
                d >>= 1;
                slot++;
            }
            top = std::max(top, slot);
            hist[slot]++;
        }
        printf("deg[0]: 0\t%zu\t%.2f%%\n", hist[0], (float)hist[0] / vertexCount * 100);
        for (int i = 1; i <= top; i++)
            printf("deg[%d]: (%d, %d]\t%zu\t%.2f%%\n", i, i >= 2 ? 1 << (i - 2) : 0, 1 << (i - 1),
                   hist[i], (float)hist[i] / vertexCount * 100);
    }

private:
    // Binary CSR dump (see the file comment); false when the file is text.
    bool fromBinary(const olive_detail::FileBuf &fb, const char *path) {
        const size_t n = fb.data.size() - 1;   // FileBuf appends a terminator
        const char *b = fb.data.data();
        if (n < 32 || memcmp(b, "OLVCSR1\n", 8) != 0) return false;
        unsigned long long hdr[3];
        memcpy(hdr, b + 8, sizeof hdr);
        const unsigned long long V = hdr[0], E = hdr[1], flags = hdr[2];
        const unsigned long long need = 32 + 4 * (V + 1) + 4 * E * ((flags & 1) ? 2 : 1);
        if (V >= 0xffffffffULL || E > 0xffffffffULL || n < need) {
            LOG(ERROR) << "truncated or oversized binary CSR file: " << path;
            return true;
        }
        initGraph((VertexId)V, (EdgeId)E);
        memcpy(vertices, b + 32, 4 * (V + 1));
        memcpy(edges, b + 32 + 4 * (V + 1), 4 * E);
        if (flags & 1) {
            const uint32_t *vals = reinterpret_cast<const uint32_t *>(b + 32 + 4 * (V + 1) + 4 * E);
            for (unsigned long long e = 0; e < E; e++) edgeValues[e] = (EdgeValue)vals[e];
        } else {
            for (unsigned long long e = 0; e < E; e++) edgeValues[e] = EdgeValue(1);
        }
        bool ok = vertices[0] == 0 && vertices[V] == E;
        for (unsigned long long v = 0; ok && v < V; v++) ok = vertices[v] <= vertices[v + 1];
        for (unsigned long long e = 0; ok && e < E; e++) ok = edges[e] < V;
        if (!ok) {
            LOG(ERROR) << "invalid CSR in binary file " << path;
            release();
            vertexCount = 0;
            edgeCount = 0;
        } else {
            LOG(INFO) << "Loaded binary CSR: " << V << " nodes, " << E << " edges";
        }
        return true;
    }

    void buildFromTuples(VertexId V, const std::vector<VertexId> &src,
                         const std::vector<VertexId> &dst, const std::vector<EdgeValue> &val) {
        const size_t E = src.size();
        initGraph(V, (EdgeId)E);
        std::fill(vertices, vertices + (size_t)V + 1, 0);
        for (size_t i = 0; i < E; i++) vertices[src[i] + 1]++;
        for (VertexId v = 0; v < V; v++) vertices[v + 1] += vertices[v];
        std::vector<EdgeId> cur(vertices, vertices + V);
        for (size_t i = 0; i < E; i++) {   // stable: file order within a row
            EdgeId pos = cur[src[i]]++;
            edges[pos] = dst[i];
            edgeValues[pos] = val[i];
        }
    }
};

#endif  // OLIVE_CSR_GRAPH_H
