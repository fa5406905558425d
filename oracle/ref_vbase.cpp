// Test infrastructure (never linked by the product): calls Grappolo's
// vBaseRedistribution (Coloring/vBase.cpp:6-168) from a copy of its source
// that oracle/Makefile patches into oracle/_ref/patched/ with the one line the
// function lacks: it is declared int and falls off its end without a return,
// which g++ turns into a trap.  Nothing else of the function changes, so its
// results pin balanced recolouring wherever the function's first-fit scan
// (vBase.cpp:113-116, which reads one element past freq when no colour
// qualifies) finds a colour; the callers (tests/golden/make_golden.py) keep
// only such cases for type 0.
#include <cstdlib>
#include <omp.h>
#include "defs.h"
#include "coloring.h"

static graph *vb_graph(long nv, const long *ptr, const long *tail, const double *w) {
    graph *G = (graph *)malloc(sizeof(graph));
    G->numVertices = nv;
    G->sVertices = nv;
    G->numEdges = ptr[nv] / 2;
    G->edgeListPtrs = (long *)malloc(sizeof(long) * (nv + 1));
    G->edgeList = (edge *)malloc(sizeof(edge) * (ptr[nv] ? ptr[nv] : 1));
    for (long i = 0; i <= nv; i++) G->edgeListPtrs[i] = ptr[i];
    for (long i = 0; i < nv; i++)
        for (long j = ptr[i]; j < ptr[i + 1]; j++) {
            G->edgeList[j].head = i;
            G->edgeList[j].tail = tail[j];
            G->edgeList[j].weight = w[j];
        }
    return G;
}

extern "C" int ref_vbase(long nv, const long *ptr, const long *tail, const double *w, int *color,
                         int ncolors, int type) {
    omp_set_num_threads(1);  // its loops are OpenMP loops; one thread is the order pinned
    graph *G = vb_graph(nv, ptr, tail, w);
    const int r = vBaseRedistribution(G, color, ncolors, type);
    free(G->edgeListPtrs);
    free(G->edgeList);
    free(G);
    return r;
}
