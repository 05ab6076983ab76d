/*
 * olive_b200 source-compatible header layer: Olive<VertexValue, EdgeValue,
 * AccumValue>, the class name the reference's README documents
 * (README.md:49-68).  The reference's multi-GPU Olive<V,A> (olive.h:51-461)
 * never built (it includes a missing flexible.h); here the name is the
 * single-GPU engine, i.e. one partition with no inter-GPU messaging.
 */
#ifndef OLIVE_H
#define OLIVE_H

#include "oliver.h"

template <typename VertexValue, typename EdgeValue, typename AccumValue>
class Olive : public Oliver<VertexValue, EdgeValue, AccumValue> {
public:
    using Oliver<VertexValue, EdgeValue, AccumValue>::Oliver;
};

#endif  // OLIVE_H
