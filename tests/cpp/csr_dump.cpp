// Loads a graph file with the source-compatible CsrGraph (include/olive/csrGraph.h)
// and prints "V E", then one line per vertex: its out-neighbours in CSR order.
// Used by tests/test_loaders.py; built with g++ on the host.
#include <cstdio>

#include "commandLine.h"
#include "csrGraph.h"

int main(int argc, char **argv) {
    CommandLine cl(argc, argv, "<inFile> [-dimacs]");
    char *path = cl.getArgument(0);
    Logging::ReportingLevel() = ERROR;
    CsrGraph<int, int> g;
    if (cl.getOption("-dimacs"))
        g.fromDimacsFile(path);
    else
        g.fromEdgeListFile(path);
    printf("%u %u\n", g.vertexCount, g.edgeCount);
    for (VertexId v = 0; v < g.vertexCount; v++) {
        for (EdgeId e = g.vertices[v]; e < g.vertices[v + 1]; e++)
            printf(e == g.vertices[v] ? "%u" : " %u", g.edges[e]);
        printf("\n");
    }
    return 0;
}
