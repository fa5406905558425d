// Grappolo's C++ entry points (include/grappolo_compat.h) over the C ABI.
#include <cstdio>
#include <vector>
#include <cstdlib>
#include <cstring>

#include "grappolo_b200.h"
#include "grappolo_compat.h"

static_assert(sizeof(edge) == sizeof(glv_edge), "edge layout");
static_assert(sizeof(graph) == sizeof(glv_graph), "graph layout");

static int mode_for(int nThreads) {
  const char *env = getenv("GRAPPOLO_B200_MODE");
  if (env && !strcmp(env, "verify")) return GLV_MODE_VERIFY;
  if (env && !strcmp(env, "fast")) return GLV_MODE_FAST;
  return nThreads <= 1 ? GLV_MODE_VERIFY : GLV_MODE_FAST;
}

static void die(const char *where, int rc) {
  fprintf(stderr, "%s: grappolo_b200 error %d: %s\n", where, rc, glv_last_error());
  exit(1);
}

static void print_summary(const glv_run_stats &s, int coloring, int numThreads) {
  printf("********************************************\n");
  printf("*********    Compact Summary   *************\n");
  printf("********************************************\n");
  printf("Number of threads              : %d\n", numThreads);
  printf("Total number of phases         : %d\n", s.phases);
  printf("Total number of iterations     : %d\n", s.total_iterations);
  printf("Final number of clusters       : %ld\n", s.final_clusters);
  printf("Final modularity               : %lf\n", s.final_modularity);
  printf("Total time for clustering      : %lf\n", s.time_clustering);
  printf("Total time for building phases : %lf\n", s.time_building);
  if (coloring) printf("Total time for coloring        : %lf\n", s.time_coloring);
  printf("********************************************\n");
  printf("TOTAL TIME                     : %lf\n",
         s.time_clustering + s.time_building + s.time_coloring);
  printf("********************************************\n");
}

static void free_graph(graph *G) {
  if (!G) return;
  free(G->edgeListPtrs);
  free(G->edgeList);
  free(G);
}

void runMultiPhaseColoring(graph *G, long *C_orig, int coloring, int numColors, int replaceMap,
                           long minGraphSize, double threshold, double C_threshold,
                           int numThreads, int threadsOpt) {
  (void)threadsOpt;
  printf("Within runMultiPhaseColoring()\n");
  glv_run_stats *s = (glv_run_stats *)calloc(1, sizeof(glv_run_stats));
  int rc = glv_run_multiphase_coloring((const glv_graph *)G, C_orig, coloring, numColors,
                                       replaceMap, minGraphSize, threshold, C_threshold,
                                       mode_for(numThreads), s);
  if (rc != GLV_OK) die("runMultiPhaseColoring", rc);
  print_summary(*s, coloring != 0, numThreads);
  free(s);
  free_graph(G);  // the reference consumes G (runMultiPhaseColoring.cpp:226-232)
}

void runMultiPhaseBasic(graph *G, long *C_orig, int basicOpt, long minGraphSize,
                        double threshold, double C_threshold, int numThreads, int threadsOpt) {
  (void)threadsOpt;
  glv_run_stats *s = (glv_run_stats *)calloc(1, sizeof(glv_run_stats));
  int rc = glv_run_multiphase_basic((const glv_graph *)G, C_orig, basicOpt, minGraphSize,
                                    threshold, C_threshold, mode_for(numThreads), s);
  if (rc != GLV_OK) die("runMultiPhaseBasic", rc);
  print_summary(*s, 0, numThreads);
  free(s);
  free_graph(G);
}

double algoLouvainWithDistOneColoring(graph *G, long *C, int nThreads, int *color, int numColor,
                                      double Lower, double thresh, double *totTime, int *numItr) {
  printf("Within algoLouvainWithDistOneColoring(#colors= %d)\n", numColor);
  double q = 0;
  int rc = glv_louvain_coloring_phase((const glv_graph *)G, C, color, numColor, Lower, thresh,
                                      mode_for(nThreads), &q, numItr, totTime);
  if (rc != GLV_OK) die("algoLouvainWithDistOneColoring", rc);
  return q;
}

double parallelLouvianMethod(graph *G, long *C, int nThreads, double Lower, double thresh,
                             double *totTime, int *numItr) {
  printf("Within parallelLouvianMethod()\n");
  double q = 0;
  int rc = glv_louvain_basic_phase((const glv_graph *)G, C, Lower, thresh, mode_for(nThreads),
                                   &q, numItr, totTime);
  if (rc != GLV_OK) die("parallelLouvianMethod", rc);
  return q;
}

int algoDistanceOneVertexColoringOpt(graph *G, int *vtxColor, int nThreads, double *totTime) {
  int mc = -1;
  int rc = glv_distance_one_coloring((const glv_graph *)G, vtxColor, mode_for(nThreads), &mc,
                                     totTime);
  if (rc != GLV_OK) die("algoDistanceOneVertexColoringOpt", rc);
  return mc;
}

int algoColoringMultiHashMaxMin(graph *G, int *vtxColor, int nThreads, double *totTime, int nHash,
                                int nItrs) {
  (void)nThreads;
  int mc = -1;
  int rc = glv_color_multihash((const glv_graph *)G, vtxColor, nHash, nItrs, &mc, totTime);
  if (rc != GLV_OK) die("algoColoringMultiHashMaxMin", rc);
  return mc;
}

long removeEdges(long NV, long NE, edge *edgeList) {
  long n = 0;
  int rc = glv_remove_edges(NV, NE, (glv_edge *)edgeList, &n);
  if (rc != GLV_OK) die("removeEdges", rc);
  return n;
}

void SortEdgesUndirected(long NV, long NE, edge *list1, edge *list2, long *ptrs) {
  int rc = glv_sort_edges_undirected(NV, NE, (const glv_edge *)list1, (glv_edge *)list2, ptrs);
  if (rc != GLV_OK) die("SortEdgesUndirected", rc);
}

void SortNodeEdgesByIndex(long NV, edge *list1, edge *list2, long *ptrs) {
  int rc = glv_sort_node_edges_by_index(NV, (glv_edge *)list1, (glv_edge *)list2, ptrs);
  if (rc != GLV_OK) die("SortNodeEdgesByIndex", rc);
}

void parse_EdgeListBinaryNew(graph *G, char *fileName) {
  printf("Parsing a file in binary format...\n");
  int rc = glv_load_binary(fileName, (glv_graph *)G);
  if (rc != GLV_OK) die("parse_EdgeListBinaryNew", rc);
}

void writeGraphBinaryFormatNew(graph *G, char *filename, long weighted) {
  int rc = glv_write_binary((const glv_graph *)G, filename, weighted);
  if (rc != GLV_OK) die("writeGraphBinaryFormatNew", rc);
  printf("Graph has been stored in file: %s\n", filename);
}

void computeCommunityComparisons(std::vector<long> &C1, long N1, std::vector<long> &C2, long N2) {
  glv_comparison r;
  int rc = glv_compare_communities(C1.data(), N1, C2.data(), N2, &r);
  if (rc != GLV_OK) die("computeCommunityComparisons", rc);
  printf("*******************************************\n");
  printf("Cluster comparison statistics: \n");
  printf("*******************************************\n");
  printf("|C1| (truth)          : %ld\n", r.n1);
  printf("Num communities in C1 : %ld\n", r.num_communities1);
  printf("|C2| (output)         : %ld\n", r.n2);
  printf("Num communities in C2 : %ld\n", r.num_communities2);
  printf("-------------------------------------------\n");
  printf("Same-Same (True positive)  : %ld\n", r.same_same);
  printf("Same-Diff (False negative) : %ld\n", r.same_diff);
  printf("Diff-Same (False positive) : %ld\n", r.diff_same);
  printf("-------------------------------------------\n");
  printf("Precision             :  %lf (%3.2lf%%)\n", r.precision, r.precision * 100);
  printf("Recall                :  %lf (%3.2lf%%)\n", r.recall, r.recall * 100);
  printf("F-score               :  %lf\n", r.f_score);
  printf("-------------------------------------------\n");
  printf("Gini coefficient, C1  :  %lf \n", r.gini1);
  printf("Gini coefficient, C2  :  %lf \n", r.gini2);
  printf("*******************************************\n");
}

double computeGiniCoefficient(long *colorSize, int numColors) {
  double g = 0;
  int rc = glv_gini_coefficient(colorSize, numColors, &g);
  if (rc != GLV_OK) die("computeGiniCoefficient", rc);
  return g;
}

int vBaseRedistribution(graph *G, int *vtxColor, int ncolors, int type) {
  long moves = 0;
  int rc = glv_vbase_redistribution((const glv_graph *)G, vtxColor, ncolors, type, &moves);
  if (rc != GLV_OK) die("vBaseRedistribution", rc);
  return (int)moves;
}

long renumberClustersContiguously(long *C, long size) {
  long n = 0;
  int rc = glv_renumber_clusters(C, size, &n);
  if (rc != GLV_OK) die("renumberClustersContiguously", rc);
  return n;
}

long vertexFollowing(graph *G, long *C) {
  long n = 0;
  int rc = glv_vertex_following((const glv_graph *)G, C, &n);
  if (rc != GLV_OK) die("vertexFollowing", rc);
  return n;
}

double buildNewGraphVF(graph *Gin, graph *Gout, long *C, long numUniqueClusters) {
  double t = 0;
  int rc = glv_build_new_graph_vf((const glv_graph *)Gin, (glv_graph *)Gout, C, numUniqueClusters,
                                  &t);
  if (rc != GLV_OK) die("buildNewGraphVF", rc);
  return t;
}

double buildNextLevelGraphOpt(graph *Gin, graph *Gout, long *C, long numUniqueClusters,
                              int nThreads) {
  double t = 0;
  int rc = glv_build_next_level((const glv_graph *)Gin, (glv_graph *)Gout, C, numUniqueClusters,
                                mode_for(nThreads), &t);
  if (rc != GLV_OK) die("buildNextLevelGraphOpt", rc);
  return t;
}
