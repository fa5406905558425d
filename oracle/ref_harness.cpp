// Harness around Grappolo's own hot-path functions.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's unmodified sources (Utility/, Coloring/,
// BasicCommunitiesDetection/, FullSyncOptimization/, InputsOutput/) into
// oracle/_ref/libgrappolo_ref.so.  It converts the SoA CSR that the tests use
// into the reference's `graph`/`edge` structs (DefineStructure/defs.h:78-92),
// calls the reference function named in each wrapper, and copies results
// back.  It is what pins the C restatement in louvain_oracle.c, generates the
// golden fixtures, and is the CPU baseline that bench.py times.
#include <cstdio>
#include <omp.h>
#include <cstdlib>
#include <cstring>
#include <map>
#include <unistd.h>
#include <vector>

#include "defs.h"
#include "basic_comm.h"
#include "basic_util.h"
#include "color_comm.h"
#include "coloring.h"
#include "input_output.h"
#include "sync_comm.h"
#include "utilityClusteringFunctions.h"

static int g_quiet = 0;
static int g_saved_fd = -1;

static void quiet_begin() {
    if (!g_quiet) return;
    fflush(stdout);
    g_saved_fd = dup(1);
    FILE *devnull = fopen("/dev/null", "w");
    dup2(fileno(devnull), 1);
    fclose(devnull);
}

static void quiet_end() {
    if (!g_quiet || g_saved_fd < 0) return;
    fflush(stdout);
    dup2(g_saved_fd, 1);
    close(g_saved_fd);
    g_saved_fd = -1;
}

static graph *make_graph(long nv, const long *ptr, const long *tail, const double *w) {
    graph *G = (graph *)malloc(sizeof(graph));
    long nnz = ptr[nv];
    G->numVertices = nv;
    G->sVertices = nv;
    long loops = 0;
    G->edgeListPtrs = (long *)malloc(sizeof(long) * (nv + 1));
    G->edgeList = (edge *)malloc(sizeof(edge) * (nnz ? nnz : 1));
    memcpy(G->edgeListPtrs, ptr, sizeof(long) * (nv + 1));
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : loops)
    for (long i = 0; i < nv; i++) {
        for (long j = ptr[i]; j < ptr[i + 1]; j++) {
            G->edgeList[j].head = i;
            G->edgeList[j].tail = tail[j];
            G->edgeList[j].weight = w[j];
            if (tail[j] == i) loops++;
        }
    }
    G->numEdges = (nnz - loops) / 2 + loops;
    return G;
}

static void free_graph(graph *G) {
    free(G->edgeListPtrs);
    free(G->edgeList);
    free(G);
}

extern "C" {

void ref_set_quiet(int q) { g_quiet = q; }

// Coloring/coloringDistanceOne.cpp:50 algoDistanceOneVertexColoringOpt,
// colours initialised to -1 as runMultiPhaseColoring.cpp:61-65 does.
int ref_color(long nv, const long *ptr, const long *tail, const double *w, int *color,
              int nthreads, double *totTime) {
    graph *G = make_graph(nv, ptr, tail, w);
    for (long i = 0; i < nv; i++) color[i] = -1;
    quiet_begin();
    int mc = algoDistanceOneVertexColoringOpt(G, color, nthreads, totTime);
    quiet_end();
    free_graph(G);
    return mc;
}

// Coloring/coloringMultiHashMaxMin.cpp:59 algoColoringMultiHashMaxMin; its
// random values come from the C library's rand().
int ref_color_mhash(long nv, const long *ptr, const long *tail, const double *w, int nHash,
                    int nItrs, int *color, int nthreads) {
    graph *G = make_graph(nv, ptr, tail, w);
    double t = 0;
    quiet_begin();
    int mc = algoColoringMultiHashMaxMin(G, color, nthreads, &t, nHash, nItrs);
    quiet_end();
    free_graph(G);
    return mc;
}

// Coloring/parallelLouvainWithColoring.cpp:47 algoLouvainWithDistOneColoring
double ref_coloring_phase(long nv, const long *ptr, const long *tail, const double *w,
                          long *C, int *color, int numColor, double Lower, double thresh,
                          int nthreads, int *numItr, double *totTime) {
    graph *G = make_graph(nv, ptr, tail, w);
    quiet_begin();
    double q = algoLouvainWithDistOneColoring(G, C, nthreads, color, numColor, Lower, thresh,
                                              totTime, numItr);
    quiet_end();
    free_graph(G);
    return q;
}

// BasicCommunitiesDetection/parallelLouvainMethod.cpp:65 parallelLouvianMethod
double ref_basic_phase(long nv, const long *ptr, const long *tail, const double *w, long *C,
                       double Lower, double thresh, int nthreads, int *numItr,
                       double *totTime) {
    graph *G = make_graph(nv, ptr, tail, w);
    quiet_begin();
    double q = parallelLouvianMethod(G, C, nthreads, Lower, thresh, totTime, numItr);
    quiet_end();
    free_graph(G);
    return q;
}

// Utility/buildNextPhase.cpp:48 renumberClustersContiguously
long ref_renumber(long *C, long n) {
    quiet_begin();
    long r = renumberClustersContiguously(C, n);
    quiet_end();
    return r;
}

// Utility/buildNextPhase.cpp:83 buildNextLevelGraphOpt.  Returns the output
// nnz; arrays are malloc'd here and released with ref_free.  Fails (-1) if an
// output record's head does not match its row.
long ref_build_next_level(long nv, const long *ptr, const long *tail, const double *w,
                          long *C, long ncl, int nthreads, long **optr, long **otail,
                          double **ow, long *numEdges) {
    graph *G = make_graph(nv, ptr, tail, w);
    graph *Gout = (graph *)malloc(sizeof(graph));
    quiet_begin();
    buildNextLevelGraphOpt(G, Gout, C, ncl, nthreads);
    quiet_end();
    long onv = Gout->numVertices;
    long onnz = Gout->edgeListPtrs[onv];
    long *p = (long *)malloc(sizeof(long) * (onv + 1));
    long *t = (long *)malloc(sizeof(long) * (onnz ? onnz : 1));
    double *ww = (double *)malloc(sizeof(double) * (onnz ? onnz : 1));
    memcpy(p, Gout->edgeListPtrs, sizeof(long) * (onv + 1));
    long bad = 0;
    for (long i = 0; i < onv; i++)
        for (long j = p[i]; j < p[i + 1]; j++) {
            t[j] = Gout->edgeList[j].tail;
            ww[j] = Gout->edgeList[j].weight;
            if (Gout->edgeList[j].head != i) bad++;
        }
    *numEdges = Gout->numEdges;
    free_graph(Gout);
    free_graph(G);
    *optr = p; *otail = t; *ow = ww;
    return bad ? -1 : onnz;
}

// Utility/vertexFollowing.cpp:46 vertexFollowing: C and the count to fix.
long ref_vertex_following(long nv, const long *ptr, const long *tail, const double *w, long *C,
                          int nthreads) {
    graph *G = make_graph(nv, ptr, tail, w);
    omp_set_num_threads(nthreads);
    quiet_begin();
    long r = vertexFollowing(G, C);
    quiet_end();
    free_graph(G);
    return r;
}

// Utility/vertexFollowing.cpp:91 buildNewGraphVF, output as ref_build_next_level.
long ref_build_new_graph_vf(long nv, const long *ptr, const long *tail, const double *w,
                            long *C, long ncl, int nthreads, long **optr, long **otail,
                            double **ow, long *numEdges) {
    graph *G = make_graph(nv, ptr, tail, w);
    graph *Gout = (graph *)malloc(sizeof(graph));
    omp_set_num_threads(nthreads);
    quiet_begin();
    buildNewGraphVF(G, Gout, C, ncl);
    quiet_end();
    long onv = Gout->numVertices;
    long onnz = Gout->edgeListPtrs[onv];
    long *p = (long *)malloc(sizeof(long) * (onv + 1));
    long *t = (long *)malloc(sizeof(long) * (onnz ? onnz : 1));
    double *ww = (double *)malloc(sizeof(double) * (onnz ? onnz : 1));
    memcpy(p, Gout->edgeListPtrs, sizeof(long) * (onv + 1));
    long bad = 0;
    for (long i = 0; i < onv; i++)
        for (long j = p[i]; j < p[i + 1]; j++) {
            t[j] = Gout->edgeList[j].tail;
            ww[j] = Gout->edgeList[j].weight;
            if (Gout->edgeList[j].head != i) bad++;
        }
    *numEdges = Gout->numEdges;
    free_graph(Gout);
    free_graph(G);
    *optr = p; *otail = t; *ow = ww;
    return bad ? -1 : onnz;
}

void ref_free(void *p) { free(p); }

// Persistent graphs for repeated timing of one input (the AoS copy is built
// once, in parallel).
void *ref_graph_create(long nv, const long *ptr, const long *tail, const double *w) {
  return make_graph(nv, ptr, tail, w);
}

void ref_graph_free(void *G) { free_graph((graph *)G); }

int ref_color_g(void *Gv, int *color, int nthreads, double *totTime) {
  graph *G = (graph *)Gv;
  for (long i = 0; i < G->numVertices; i++) color[i] = -1;
  quiet_begin();
  int mc = algoDistanceOneVertexColoringOpt(G, color, nthreads, totTime);
  quiet_end();
  return mc;
}

double ref_coloring_phase_g(void *Gv, long *C, int *color, int numColor, double Lower,
                            double thresh, int nthreads, int *numItr, double *totTime) {
  quiet_begin();
  double q = algoLouvainWithDistOneColoring((graph *)Gv, C, nthreads, color, numColor, Lower,
                                            thresh, totTime, numItr);
  quiet_end();
  return q;
}

// Per-vertex move decision through the reference's own primitives, set up as
// the colour sweep does (parallelLouvainWithColoring.cpp:181-188):
// own community first with Counter 0, buildLocalMapCounter
// (utilityClusteringFunctions.cpp:172), then max() (:226).
void ref_decide_batch(long nv, const long *ptr, const long *tail, const double *w,
                      const long *C, const double *vDeg, const double *cDeg,
                      const long *cSize, double constant, long nverts, const long *verts,
                      long *targets) {
    graph *G = make_graph(nv, ptr, tail, w);
    Comm *cInfo = (Comm *)malloc(sizeof(Comm) * (nv ? nv : 1));
    for (long i = 0; i < nv; i++) { cInfo[i].size = cSize[i]; cInfo[i].degree = cDeg[i]; }
    long *Cm = (long *)malloc(sizeof(long) * (nv ? nv : 1));
    memcpy(Cm, C, sizeof(long) * nv);
    for (long k = 0; k < nverts; k++) {
        long i = verts[k];
        long adj1 = ptr[i], adj2 = ptr[i + 1];
        if (adj1 == adj2) { targets[k] = -1; continue; }
        std::map<long, long> clusterLocalMap;
        std::vector<double> Counter;
        clusterLocalMap[Cm[i]] = 0;
        Counter.push_back(0);
        double selfLoop = buildLocalMapCounter(adj1, adj2, clusterLocalMap, Counter,
                                               G->edgeList, Cm, i);
        targets[k] = max(clusterLocalMap, Counter, selfLoop, cInfo, vDeg[i], Cm[i], constant);
    }
    free(Cm);
    free(cInfo);
    free_graph(G);
}

// Utility/utilityClusteringFunctions.cpp:70,89 sumVertexDegree +
// calConstantForSecondTerm.
double ref_vertex_degrees(long nv, const long *ptr, const long *tail, const double *w,
                          double *vDeg) {
    graph *G = make_graph(nv, ptr, tail, w);
    Comm *cInfo = (Comm *)malloc(sizeof(Comm) * (nv ? nv : 1));
    sumVertexDegree(G->edgeList, G->edgeListPtrs, vDeg, nv, cInfo);
    double c = calConstantForSecondTerm(vDeg, nv);
    free(cInfo);
    free_graph(G);
    return c;
}

// Coloring/runMultiPhaseColoring.cpp:51 and
// BasicCommunitiesDetection/runMultiPhaseBasic.cpp:52.  They print their
// results; stdout is captured into `log` (NUL-terminated, truncated to cap).
static long run_captured(char *log, long cap, void (*fn)(void *), void *arg) {
    fflush(stdout);
    int saved = dup(1);
    FILE *tmp = tmpfile();
    dup2(fileno(tmp), 1);
    fn(arg);
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    long n = 0;
    if (log && cap > 0) {
        fseek(tmp, 0, SEEK_END);
        long size = ftell(tmp);
        long keep = size < cap - 1 ? size : cap - 1;
        fseek(tmp, size - keep, SEEK_SET);
        n = (long)fread(log, 1, keep, tmp);
        log[n] = 0;
    }
    fclose(tmp);
    return n;
}

struct mp_args {
    graph *G; long *C_orig; int coloring, numColors, replaceMap, basicOpt;
    long minGraphSize; double threshold, C_threshold; int nthreads;
};

static void call_coloring(void *p) {
    mp_args *a = (mp_args *)p;
    runMultiPhaseColoring(a->G, a->C_orig, a->coloring, a->numColors, a->replaceMap,
                          a->minGraphSize, a->threshold, a->C_threshold, a->nthreads, 1);
}

static void call_basic(void *p) {
    mp_args *a = (mp_args *)p;
    runMultiPhaseBasic(a->G, a->C_orig, a->basicOpt, a->minGraphSize, a->threshold,
                       a->C_threshold, a->nthreads, 1);
}

long ref_run_multiphase_coloring(long nv, const long *ptr, const long *tail, const double *w,
                                 long *C_orig, int coloring, int numColors, int replaceMap,
                                 long minGraphSize, double threshold, double C_threshold,
                                 int nthreads, char *log, long cap) {
    mp_args a;
    a.G = make_graph(nv, ptr, tail, w);  // freed by the reference
    a.C_orig = C_orig; a.coloring = coloring; a.numColors = numColors;
    a.replaceMap = replaceMap; a.basicOpt = 0; a.minGraphSize = minGraphSize;
    a.threshold = threshold; a.C_threshold = C_threshold; a.nthreads = nthreads;
    for (long i = 0; i < nv; i++) C_orig[i] = -1;
    return run_captured(log, cap, call_coloring, &a);
}

// FullSyncOptimization/runMultiPhaseSyncType.cpp:48 (syncType 3: the
// early-termination Louvain of parallelLouvainMethodEarlyTerminate.cpp).
static void call_sync(void *p) {
    mp_args *a = (mp_args *)p;
    runMultiPhaseSyncType(a->G, a->C_orig, a->basicOpt, a->minGraphSize, a->threshold,
                          a->C_threshold, a->nthreads, 1);
}

long ref_run_multiphase_sync(long nv, const long *ptr, const long *tail, const double *w,
                             long *C_orig, int syncType, long minGraphSize, double threshold,
                             double C_threshold, int nthreads, char *log, long cap) {
    mp_args a;
    a.G = make_graph(nv, ptr, tail, w);  // freed by the reference
    a.C_orig = C_orig; a.coloring = 0; a.numColors = 0; a.replaceMap = 0;
    a.basicOpt = syncType; a.minGraphSize = minGraphSize; a.threshold = threshold;
    a.C_threshold = C_threshold; a.nthreads = nthreads;
    for (long i = 0; i < nv; i++) C_orig[i] = -1;
    return run_captured(log, cap, call_sync, &a);
}

long ref_run_multiphase_basic(long nv, const long *ptr, const long *tail, const double *w,
                              long *C_orig, int basicOpt, long minGraphSize, double threshold,
                              double C_threshold, int nthreads, char *log, long cap) {
    mp_args a;
    a.G = make_graph(nv, ptr, tail, w);
    a.C_orig = C_orig; a.coloring = 0; a.numColors = 0; a.replaceMap = 0;
    a.basicOpt = basicOpt; a.minGraphSize = minGraphSize; a.threshold = threshold;
    a.C_threshold = C_threshold; a.nthreads = nthreads;
    for (long i = 0; i < nv; i++) C_orig[i] = -1;
    return run_captured(log, cap, call_basic, &a);
}

static edge *make_edges(long n, const long *h, const long *t, const double *w) {
    edge *e = (edge *)malloc(sizeof(edge) * (n ? n : 1));
    for (long i = 0; i < n; i++) { e[i].head = h[i]; e[i].tail = t[i]; e[i].weight = w[i]; }
    return e;
}

static void take_edges(long n, const edge *e, long *h, long *t, double *w) {
    for (long i = 0; i < n; i++) { h[i] = e[i].head; t[i] = e[i].tail; w[i] = e[i].weight; }
}

// Utility/utilityFunctions.cpp:416 removeEdges; all NE entries written back.
long ref_remove_edges(long nv, long ne, long *h, long *t, double *w) {
    edge *e = make_edges(ne, h, t, w);
    quiet_begin();
    long nge = removeEdges(nv, ne, e);
    quiet_end();
    take_edges(ne, e, h, t, w);
    free(e);
    return nge;
}

// Utility/utilityFunctions.cpp:463 SortEdgesUndirected; ptrs holds NV+2 entries.
void ref_sort_edges_undirected(long nv, long ne, const long *h, const long *t, const double *w,
                               long *ptrs, long *oh, long *ot, double *ow) {
    edge *e1 = make_edges(ne, h, t, w);
    edge *e2 = (edge *)malloc(sizeof(edge) * (2 * ne ? 2 * ne : 1));
    SortEdgesUndirected(nv, ne, e1, e2, ptrs);
    take_edges(2 * ne, e2, oh, ot, ow);
    free(e1); free(e2);
}

// Utility/utilityFunctions.cpp:501 SortNodeEdgesByIndex, rows in place.
void ref_sort_node_edges(long nv, const long *ptrs, long *h, long *t, double *w) {
    long nnz = ptrs[nv];
    edge *e1 = make_edges(nnz, h, t, w);
    edge *e2 = (edge *)malloc(sizeof(edge) * (nnz ? nnz : 1));
    SortNodeEdgesByIndex(nv, e1, e2, (long *)ptrs);
    take_edges(nnz, e1, h, t, w);
    free(e1); free(e2);
}

// InputsOutput/writeBinary.cpp:2 writeGraphBinaryFormatNew.
void ref_write_binary(long nv, const long *ptr, const long *tail, const double *w, long numEdges,
                      long weighted, const char *path) {
    graph *G = make_graph(nv, ptr, tail, w);
    G->numEdges = numEdges;
    quiet_begin();
    writeGraphBinaryFormatNew(G, (char *)path, weighted);
    quiet_end();
    free_graph(G);
}

// InputsOutput/loadBinary.cpp:6 parse_EdgeListBinaryNew -> SoA CSR (malloc'd).
long ref_load_binary(const char *path, long **optr, long **ohead, long **otail, double **ow,
                     long *numEdges) {
    graph G;
    quiet_begin();
    parse_EdgeListBinaryNew(&G, (char *)path);
    quiet_end();
    long nv = G.numVertices, nnz = 2 * G.numEdges;
    long *p = (long *)malloc(sizeof(long) * (nv + 1));
    long *hh = (long *)malloc(sizeof(long) * (nnz ? nnz : 1));
    long *t = (long *)malloc(sizeof(long) * (nnz ? nnz : 1));
    double *ww = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
    memcpy(p, G.edgeListPtrs, sizeof(long) * (nv + 1));
    take_edges(nnz, G.edgeList, hh, t, ww);
    free(G.edgeListPtrs);
    free(G.edgeList);
    *optr = p; *ohead = hh; *otail = t; *ow = ww; *numEdges = G.numEdges;
    return nv;
}

// Utility/utilityClusterComparisonMetrics.cpp:50 computeCommunityComparisons;
// the relabelled arrays are written back, the printed statistics go to log.
long ref_compare(long *C1, long *C2, long n, int nthreads, char *log, long cap) {
    struct Args { long *C1, *C2, n; int nthreads; } a{C1, C2, n, nthreads};
    return run_captured(log, cap, [](void *p) {
        Args *a = (Args *)p;
        omp_set_num_threads(a->nthreads);
        std::vector<long> v1(a->C1, a->C1 + a->n), v2(a->C2, a->C2 + a->n);
        computeCommunityComparisons(v1, a->n, v2, a->n);
        memcpy(a->C1, v1.data(), sizeof(long) * a->n);
        memcpy(a->C2, v2.data(), sizeof(long) * a->n);
    }, &a);
}

// utilityClusterComparisonMetrics.cpp:310 computeGiniCoefficient (sorts sizes).
double ref_gini(long *size, int n) {
    quiet_begin();
    double g = computeGiniCoefficient(size, n);
    quiet_end();
    return g;
}

// InputsOutput/loadMetis.cpp:19 loadMetisFileFormat -> SoA CSR (malloc'd).
long ref_load_metis(const char *path, long **optr, long **otail, double **ow) {
    graph G;
    quiet_begin();
    loadMetisFileFormat(&G, path);
    quiet_end();
    long nv = G.numVertices;
    long nnz = G.edgeListPtrs[nv];
    long *p = (long *)malloc(sizeof(long) * (nv + 1));
    long *t = (long *)malloc(sizeof(long) * (nnz ? nnz : 1));
    double *ww = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
    memcpy(p, G.edgeListPtrs, sizeof(long) * (nv + 1));
    for (long j = 0; j < nnz; j++) { t[j] = G.edgeList[j].tail; ww[j] = G.edgeList[j].weight; }
    free(G.edgeListPtrs);
    free(G.edgeList);
    *optr = p; *otail = t; *ow = ww;
    return nv;
}

}  // extern "C"
