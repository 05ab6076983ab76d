// Superstep loops as CUDA graphs: a while-conditional node whose body is the
// kernel chain of one superstep.  The last kernel of the chain decides, on the
// device, whether the body runs again (cudaGraphSetConditional), so a whole
// traversal or solve is one cudaGraphLaunch with no host round trip.  The
// reference instead synchronised the host after every primitive
// (oliver.h:82,112,140,169) and copied the frontier size back each superstep
// (vertexSubset.h:100-103).
#pragma once
#include <cuda_runtime.h>

#include "olv_internal.cuh"

namespace olv {

struct WhileGraph {
    cudaGraph_t graph = nullptr;
    cudaGraph_t body = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle handle = 0;
    cudaGraphNode_t last = nullptr;
    bool ready = false;

    int begin() {
        destroy();
        OLV_CUDA(cudaGraphCreate(&graph, 0));
        OLV_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        OLV_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
        body = cp.conditional.phGraph_out[0];
        last = nullptr;
        return OLV_OK;
    }

    int add(const void *func, dim3 grid, dim3 block, void **args) {
        cudaKernelNodeParams kp = {};
        kp.func = const_cast<void *>(func);
        kp.gridDim = grid;
        kp.blockDim = block;
        kp.sharedMemBytes = 0;
        kp.kernelParams = args;
        cudaGraphNode_t n;
        OLV_CUDA(cudaGraphAddKernelNode(&n, body, last ? &last : nullptr, last ? 1 : 0, &kp));
        last = n;
        return OLV_OK;
    }

    int finish() {
        OLV_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        ready = true;
        return OLV_OK;
    }

    int launch(cudaStream_t s) {
        OLV_CUDA(cudaGraphLaunch(exec, s));
        return OLV_OK;
    }

    void destroy() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        body = nullptr;
        ready = false;
    }
};

}  // namespace olv
