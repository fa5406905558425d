/*
 * Grappolo's own C++ API for the clustering path, served by the B200 engine.
 *
 * The declarations repeat the reference's prototypes (and its `edge`/`graph`
 * structs) exactly, so code written against Grappolo — e.g. its
 * driverForGraphClustering.cpp — links against libgrappolo_b200.so instead of
 * the reference's Coloring/, BasicCommunitiesDetection/ and Utility/ objects.
 * The symbols have C++ linkage, as in the reference.
 *
 * Behaviour follows the reference: the multiphase drivers free the input graph
 * and print their summary; phases return the modularity and report time and
 * iteration counts through pointers; errors print a message and exit(1)
 * (the reference asserts/exits).  nThreads == 1 selects the reference's
 * one-thread results bit for bit; larger values select the fast schedule
 * (GRAPPOLO_B200_MODE=verify|fast overrides).
 */
#ifndef GRAPPOLO_COMPAT_H
#define GRAPPOLO_COMPAT_H

/* DefineStructure/defs.h:78-92 */
typedef struct {
  long head;
  long tail;
  double weight;
} edge;

typedef struct {
  long numVertices;
  long sVertices;
  long numEdges;
  long *edgeListPtrs;
  edge *edgeList;
} graph;

/* DefineStructure/color_comm.h:7-8 */
void runMultiPhaseColoring(graph *G, long *C_orig, int coloring, int numColors, int replaceMap,
                           long minGraphSize, double threshold, double C_threshold,
                           int numThreads, int threadsOpt);
/* DefineStructure/color_comm.h:10-11 */
double algoLouvainWithDistOneColoring(graph *G, long *C, int nThreads, int *color, int numColor,
                                      double Lower, double thresh, double *totTime, int *numItr);
/* DefineStructure/basic_comm.h:5-6 */
void runMultiPhaseBasic(graph *G, long *C_orig, int basicOpt, long minGraphSize,
                        double threshold, double C_threshold, int numThreads, int threadsOpt);
/* DefineStructure/basic_comm.h:21-22 */
double parallelLouvianMethod(graph *G, long *C, int nThreads, double Lower, double thresh,
                             double *totTime, int *numItr);
/* DefineStructure/coloring.h:8 */
int algoDistanceOneVertexColoringOpt(graph *G, int *vtxColor, int nThreads, double *totTime);
/* DefineStructure/coloring.h:15 (Coloring/vBase.cpp); returns the vertices moved */
int vBaseRedistribution(graph *G, int *vtxColor, int ncolors, int type);
/* DefineStructure/coloring.h:12 (Coloring/coloringMultiHashMaxMin.cpp) */
int algoColoringMultiHashMaxMin(graph *G, int *vtxColor, int nThreads, double *totTime, int nHash,
                                int nItrs);
/* DefineStructure/basic_util.h:5-6 */
long renumberClustersContiguously(long *C, long size);
double buildNextLevelGraphOpt(graph *Gin, graph *Gout, long *C, long numUniqueClusters,
                              int nThreads);
/* DefineStructure/basic_util.h:14-15 (Utility/vertexFollowing.cpp) */
long vertexFollowing(graph *G, long *C);
double buildNewGraphVF(graph *Gin, graph *Gout, long *C, long numUniqueClusters);

/* DefineStructure/input_output.h:5-6, utilityClusteringFunctions.h:83
 * (Utility/utilityFunctions.cpp:416-531), computed on the GPU */
long removeEdges(long NV, long NE, edge *edgeList);
void SortEdgesUndirected(long NV, long NE, edge *list1, edge *list2, long *ptrs);
void SortNodeEdgesByIndex(long NV, edge *list1, edge *list2, long *ptrs);
/* DefineStructure/input_output.h:15,25 (InputsOutput/loadBinary.cpp, writeBinary.cpp) */
void parse_EdgeListBinaryNew(graph *G, char *fileName);
void writeGraphBinaryFormatNew(graph *G, char *filename, long weighted);

/* DefineStructure/utilityClusteringFunctions.h:71,73
 * (Utility/utilityClusterComparisonMetrics.cpp), computed on the GPU */
#include <vector>
void computeCommunityComparisons(std::vector<long> &C1, long N1, std::vector<long> &C2, long N2);
double computeGiniCoefficient(long *colorSize, int numColors);

#endif /* GRAPPOLO_COMPAT_H */
