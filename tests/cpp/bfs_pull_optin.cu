// BFS on the source-compatible Oliver API (include/olive/) with the functor
// opt-ins of the header layer's pull: the edge functor declares
// pullCandidate() (only unvisited vertices pull) and pullFirstHit (one parent
// is enough), which makes the engine's generic pull a bottom-up BFS step.
// Otherwise the program follows the reference's BFS.cu: the same vertex,
// edge and init functors, the same loop, levels written to BFS.txt with
// "%d\n", "iterations: N, time: T ms" logged.  Built by olive_b200/dropin.py.
#include "oliver.h"

FILE *outputFile;

struct Vtx {
    int level;
    inline void print() { fprintf(outputFile, "%d\n", level); }
};

struct EdgeF {
    __device__ inline int gather(Vtx src, EdgeId, Dump_Edge) { return src.level + 1; }
    __device__ inline void reduce(int &acc, int x) { acc = x; }
    __device__ inline bool pullCandidate(const Vtx &v) const { return v.level == 0x7fffffff; }
    static constexpr bool pullFirstHit = true;
};

struct VertF {
    int inf;
    explicit VertF(int i) : inf(i) {}
    __device__ inline void update(Vtx &v, int acc) { v.level = acc; }
    __device__ inline bool cond(Vtx v, int) { return v.level == inf; }
};

struct InitF {
    int level;
    explicit InitF(int l) : level(l) {}
    __device__ inline void operator()(Vtx &v, int) { v.level = level; }
};

int main(int argc, char **argv) {
    CommandLine cl(argc, argv, "<inFile> [-s 0] [-round 100] [-dimacs]");
    char *inFile = cl.getArgument(0);
    VertexId source = cl.getOptionIntValue("-s", 0);
    int max_rounds = cl.getOptionIntValue("-round", 100);
    CsrGraph<int, int> graph;
    if (cl.getOption("-dimacs"))
        graph.fromDimacsFile(inFile);
    else
        graph.fromEdgeListFile(inFile);
    const int inf = 0x7fffffff;
    Oliver<Vtx, Dump_Edge, int> ol;
    ol.readGraph(graph);
    VertexSubset all(graph.vertexCount, true);
    ol.vertexMap<InitF>(all, InitF(inf));
    all.del();
    VertexSubset frontier(graph.vertexCount, source);
    ol.vertexMap<InitF>(frontier, InitF(0));
    VertexSubset edgeFrontier(graph.vertexCount, false);
    double start = getTimeMillis();
    int iterations = 0;
    while (1) {
        int size = frontier.size();
        ol.edgeFilter<EdgeF>(edgeFrontier, frontier, EdgeF());
        ol.vertexFilter<VertF>(frontier, edgeFrontier, VertF(inf));
        if (size == 0 || iterations == max_rounds) break;
        iterations++;
    }
    double totalTime = getTimeMillis() - start;
    LOG(INFO) << "iterations: " << iterations << ", time: " << totalTime << "ms";
    outputFile = fopen("BFS.txt", "w");
    ol.printVertices();
    fclose(outputFile);
    frontier.del();
    edgeFrontier.del();
    return 0;
}
