/*
 * olive_b200 source-compatible header layer: COO edge triple and its
 * comparators (edgeTuple.h:42-67).
 */
#ifndef OLIVE_EDGE_TUPLE_H
#define OLIVE_EDGE_TUPLE_H

#include "common.h"

template <typename EdgeValue>
class EdgeTuple {
public:
    VertexId srcId;
    VertexId dstId;
    EdgeValue value;
    EdgeTuple() : srcId(0), dstId(0), value() {}
    EdgeTuple(VertexId s, VertexId d, EdgeValue v) : srcId(s), dstId(d), value(v) {}
};

template <typename EdgeTuple>
bool edgeTupleSrcCompare(EdgeTuple a, EdgeTuple b) { return a.srcId < b.srcId; }

template <typename EdgeTuple>
bool edgeTupleDstCompare(EdgeTuple a, EdgeTuple b) { return a.dstId < b.dstId; }

#endif  // OLIVE_EDGE_TUPLE_H
