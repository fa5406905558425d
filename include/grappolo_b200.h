/*
 * grappolo_b200 — C ABI of the B200 Louvain engine.
 *
 * Plain pointers and sizes only; every entry point returns a status code
 * (GLV_OK on success) and never aborts the process.  Host-buffer entry points
 * copy their inputs to the GPU and their results back before returning; the
 * glv_dev_* entry points take device pointers and run on the given CUDA stream.
 *
 * Each entry point names the reference interface it replaces
 * (Grappolo, DefineStructure/*.h).  The reference's C++ signatures themselves
 * are exported by the same library (include/grappolo_compat.h) as thin
 * wrappers over these functions.
 */
#ifndef GRAPPOLO_B200_H
#define GRAPPOLO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as Grappolo's `edge` and `graph` (DefineStructure/defs.h:78-92). */
typedef struct glv_edge {
  long head;
  long tail;
  double weight;
} glv_edge;

typedef struct glv_graph {
  long numVertices;
  long sVertices;
  long numEdges;       /* undirected edges, self-loops counted once */
  long *edgeListPtrs;  /* [numVertices+1] row offsets */
  glv_edge *edgeList;  /* [edgeListPtrs[numVertices]] entries */
} glv_graph;

enum {
  GLV_OK = 0,
  GLV_ERR_ARG = 1,        /* invalid argument (sizes, ids out of range, NULL) */
  GLV_ERR_CUDA = 2,       /* a CUDA call failed */
  GLV_ERR_OOM = 3,        /* device or host allocation failed */
  GLV_ERR_COLORS = 4,     /* a colouring needed >= 4096 colours (coloringUtils.cpp:57-60) */
  GLV_ERR_TOO_LARGE = 5,  /* numVertices >= 2^31 (ids are int32 on the device) */
  GLV_ERR_UNSUPPORTED = 6,/* option outside this engine's scope (e.g. replaceMap = 1) */
  GLV_ERR_NO_DEVICE = 7,  /* no CUDA device */
  GLV_ERR_LIMIT = 8,      /* a size exceeds a fixed limit of the entry point */
  GLV_ERR_IO = 9          /* a graph file could not be opened, read or written */
};

/* Execution modes.
 * GLV_MODE_VERIFY reproduces the reference's one-thread schedule: sequential
 *   greedy colouring in vertex order, community totals and coarse weights
 *   folded in the reference's order.  Results are bit-identical to the
 *   reference run with OMP_NUM_THREADS=1.
 * GLV_MODE_FAST uses hash-priority colouring and atomic accumulation, like the
 *   reference run with many threads: results are valid Louvain results but not
 *   bit-identical (final modularity agrees to about 1e-3).
 * With integral edge weights (total < 2^53) every accumulation is exact in any
 * order, so the modes differ only in the colouring. */
enum { GLV_MODE_VERIFY = 0, GLV_MODE_FAST = 1, GLV_MODE_LEARNED = 2 };
/* GLV_MODE_LEARNED is GLV_MODE_FAST plus the learned move gate in the colour
 * phases: from the second sweep of a phase on, a small MLP (glv_gate_set)
 * predicts from the previous sweep which vertices will move and only those
 * are evaluated.  A phase still ends only after a full, ungated sweep gains
 * less than its threshold.  No counterpart in the reference (it replaces the
 * early-termination heuristic of
 * FullSyncOptimization/parallelLouvainMethodEarlyTerminate.cpp:116-195). */

#define GLV_MAX_PHASES 256
#define GLV_KERNEL_SLOTS 11

typedef struct glv_phase_stats {
  long num_vertices;   /* level graph */
  long nnz;            /* CSR entries of the level graph */
  int colored;         /* 1: colour-class sweep phase, 0: Jacobi phase */
  int recolored;       /* colouring computed for this level (0: reused) */
  int num_colors;
  int iterations;
  double modularity;   /* value the phase returned */
  long clusters;       /* after renumbering */
  double time_sweep;   /* s, local moving + modularity */
  double time_color;   /* s */
  double time_coarsen; /* s, renumbering + next-level build */
  double edges_swept;  /* CSR entries evaluated by local moving */
} glv_phase_stats;

typedef struct glv_run_stats {
  int phases;               /* reference's phase counter at exit */
  int total_iterations;
  long final_clusters;      /* reference's "Final number of clusters" */
  double final_modularity;  /* reference's "Final modularity" (prevMod at exit) */
  double time_total;        /* s, whole call incl. transfers */
  double time_clustering;   /* s */
  double time_coloring;     /* s */
  double time_building;     /* s */
  double time_transfer;     /* s, host<->device copies */
  double edges_swept;       /* sum over phases */
  long kernel_launches;     /* kernels this call launched */
  /* With glv_set_profiling(1): device time of the local-moving sweep kernels
   * (CUDA events around every class's sweep launches, on the engine's stream)
   * and their algorithmic bytes, 16 B per CSR entry + 36 B per vertex
   * (tail 4 + weight 8 + C[tail] 4; offset 8 + C 4 + degree 8 + own total 8
   * + member id 4 + decision 4) per full sweep. */
  double sweep_kernel_time; /* s */
  double sweep_bytes;
  long sweep_steps;         /* (class, sublevel) steps timed */
  /* With glv_set_profiling(2) and the per-class launch schedule: device time
   * per launch kind — the nine degree bins of the sweep (rows of 0-4, 5-8,
   * 9-16, 17-32, 33-127, 128-511, 512-1023, 1024-2047 entries and larger hubs),
   * the community-total update, the modularity pass. */
  double kernel_time[GLV_KERNEL_SLOTS]; /* s */
  int nphase;               /* entries filled in phase[] */
  glv_phase_stats phase[GLV_MAX_PHASES];
  /* The autotuner's choice for this run's first colour phase (0 = not tuned:
   * small level, Jacobi-only run, or GRAPPOLO_B200_AUTOTUNE=0): the degree
   * above which rows are hubs, the entries per hub chunk, and 1 when the
   * choice came from the process's cache of earlier runs on the same graph. */
  int tuned_block_max;
  int tuned_hub_chunk;
  int tuned_from_cache;
  /* Blocks per thread-block cluster of the hub rows in the first colour
   * phase (0: every hub row as chunks over global tables). */
  int hub_cluster;
} glv_run_stats;

/* ---- graph construction and files ---------------------------------------- */

/* Replaces removeEdges (Utility/utilityFunctions.cpp:416-460, input_output.h:5):
 * drops self-loops and every repeat of a (head, tail) pair (the first stays),
 * compacting in place as the reference does: the first *numGoodEdges entries
 * are the kept edges in the reference's order; entries past them are left as
 * they were.  Runs on the GPU. */
int glv_remove_edges(long NV, long NE, glv_edge *edgeList, long *numGoodEdges);

/* Replaces SortEdgesUndirected (utilityFunctions.cpp:463-498, input_output.h:6):
 * list2[2*NE] receives every edge in the rows of both its ends, in list order;
 * ptrs[NV+2] the row offsets (ptrs[NV+1] = 2*NE, as the reference leaves it). */
int glv_sort_edges_undirected(long NV, long NE, const glv_edge *list1, glv_edge *list2,
                              long *ptrs);

/* Replaces SortNodeEdgesByIndex (utilityFunctions.cpp:501-531,
 * utilityClusteringFunctions.h:83): each row of list1 sorted by tail, equal
 * tails in the order the reference's merge sort leaves them (later entry
 * first).  list2 is not written (the reference uses it as scratch). */
int glv_sort_node_edges_by_index(long NV, glv_edge *list1, glv_edge *list2, const long *ptrs);

/* Edge list to CSR in one call, as the reference's loaders do it
 * (e.g. InputsOutput/loadPajekFormat.cpp:94-150): GLV_CSR_REMOVE_EDGES first
 * applies removeEdges; every edge is then stored in the rows of both ends in
 * list order; GLV_CSR_SORT_ROWS then applies SortNodeEdgesByIndex.  Gout's
 * arrays are malloc'd (free with free()); Gout->numEdges = kept edges. */
#define GLV_CSR_REMOVE_EDGES 1
#define GLV_CSR_SORT_ROWS 2
int glv_build_csr(long NV, long NE, const glv_edge *edges, int flags, glv_graph *Gout);

/* Device-resident form of glv_build_csr: int64 heads / tails and double
 * weights (NULL: all 1.0) on the device; d_ptr[NV+1] int64, d_tail_out and
 * d_weight_out must hold 2*NE entries (int32 / double); *nnz receives the
 * entries written.  Ordered on `stream` (a cudaStream_t, NULL = legacy
 * default stream); returns after it has finished. */
int glv_dev_build_csr(long NV, long NE, const long *d_head, const long *d_tail,
                      const double *d_weight, int flags, long *d_ptr, int *d_tail_out,
                      double *d_weight_out, long *nnz, void *stream);

/* Grappolo's binary graph file (InputsOutput/loadBinary.cpp:6-48,
 * writeBinary.cpp:2-29, input_output.h:15,25): NV, NE, weighted as three
 * longs, edgeListPtrs[NV+1], then 2*NE glv_edge records.  glv_load_binary
 * replaces parse_EdgeListBinaryNew (arrays malloc'd); glv_write_binary
 * replaces writeGraphBinaryFormatNew (G->edgeList must hold 2*numEdges
 * entries). */
int glv_binary_header(const char *path, long *numVertices, long *numEdges, long *weighted);
int glv_load_binary(const char *path, glv_graph *G);
int glv_write_binary(const glv_graph *G, const char *path, long weighted);

/* Streams a binary graph file straight into device memory: d_ptr[NV+1]
 * int64, d_tail[2*NE] int32, d_weight[2*NE] double (sizes from
 * glv_binary_header; nnz = 2*NE).  The file is read in chunks through two
 * pinned buffers while earlier chunks are copied and split on `stream`;
 * tails are checked against NV.  Returns after the stream has finished. */
int glv_dev_load_binary(const char *path, long numVertices, long nnz, long *d_ptr, int *d_tail,
                        double *d_weight, void *stream);

/* ---- comparing community assignments -------------------------------------- */

typedef struct {
  long n1, n2;                /* vertices labelled by C1 (truth) and C2 (output) */
  long num_communities1;      /* nC1 and nC2 as the reference counts them */
  long num_communities2;
  long same_same;             /* pairs together in both (true positives) */
  long same_diff;             /* together in C1, apart in C2 (false negatives) */
  long diff_same;             /* apart in C1, together in C2 (false positives) */
  double precision, recall, f_score;
  double gini1, gini2;        /* Gini coefficient of each side's community sizes */
} glv_comparison;

/* Replaces computeCommunityComparisons
 * (Utility/utilityClusterComparisonMetrics.cpp:50-307,
 * utilityClusteringFunctions.h:71): C1 is the truth.  Ids may be 0- or
 * 1-based; -1 entries are relabelled in place as the reference does (C1: a
 * new community; C2: N2 + 1).  The pair counts come from the contingency
 * table of the two labellings on the GPU, equal to the reference's pair
 * enumeration.  N1 must equal N2. */
int glv_compare_communities(long *C1, long N1, long *C2, long N2, glv_comparison *out);

/* Device form: int64 label arrays in device memory (relabelled in place). */
int glv_dev_compare_communities(long n, long *d_C1, long *d_C2, glv_comparison *out,
                                void *stream);

/* Replaces computeGiniCoefficient (utilityClusterComparisonMetrics.cpp:310-330,
 * basic_util.h:18): sorts colorSize[numColors] ascending in place and returns
 * the coefficient through *gini.  Sums are exact 64-bit integers (the
 * reference's FP64 sums agree while they stay below 2^53). */
int glv_gini_coefficient(long *colorSize, int numColors, double *gini);

/* ---- multiphase drivers ------------------------------------------------- */

/* Replaces runMultiPhaseColoring (Coloring/runMultiPhaseColoring.cpp:51-238,
 * declared DefineStructure/color_comm.h:7-8).  coloring = 1 is the distance-1
 * colouring; coloring = 3 the incomplete multi-hash max/min colouring
 * (Coloring/coloringMultiHashMaxMin.cpp:59-228) with two hashes and
 * max(1, numColors / 4) iterations, its random values drawn from the C
 * library's rand() exactly as the reference draws them (seed with srand() to
 * reproduce a reference run).  coloring = 2 applies glv_vbase_redistribution
 * (type 0) after each distance-1 colouring; other values are GLV_ERR_ARG.
 * replaceMap must be 0.  C_orig[numVertices] receives the
 * final community of every input vertex (-1 for isolated vertices).  Unlike the
 * reference, G is not freed.  `stats` may be NULL. */
int glv_run_multiphase_coloring(const glv_graph *G, long *C_orig, int coloring, int numColors,
                                int replaceMap, long minGraphSize, double threshold,
                                double C_threshold, int mode, glv_run_stats *stats);

/* Replaces runMultiPhaseBasic (BasicCommunitiesDetection/runMultiPhaseBasic.cpp:52-170,
 * basic_comm.h:5-6) for basicOpt = 0. */
int glv_run_multiphase_basic(const glv_graph *G, long *C_orig, int basicOpt, long minGraphSize,
                             double threshold, double C_threshold, int mode,
                             glv_run_stats *stats);

/* Struct-of-arrays host variant of glv_run_multiphase_coloring: ptr int64[nv+1],
 * tail int64[nnz], weight f64[nnz]. */
int glv_run_multiphase_coloring_csr(long nv, const long *ptr, const long *tail,
                                    const double *weight, long *C_orig, long minGraphSize,
                                    double threshold, double C_threshold, int mode,
                                    glv_run_stats *stats);

int glv_run_multiphase_basic_csr(long nv, const long *ptr, const long *tail, const double *weight,
                                 long *C_orig, double threshold, int mode, glv_run_stats *stats);

/* Device-resident variant: d_ptr int64[nv+1], d_tail int32[nnz], d_weight
 * f64[nnz] and d_C_orig int32[nv] are device pointers; `stream` is a
 * cudaStream_t (NULL = legacy default stream).  The input graph is not
 * modified.  `coloring` = 1 runs the colouring driver, 0 the basic one. */
int glv_dev_run_multiphase(long nv, const long *d_ptr, const int *d_tail, const double *d_weight,
                           int *d_C_orig, int coloring, long minGraphSize, double threshold,
                           double C_threshold, int mode, void *stream, glv_run_stats *stats);

/* Replaces vertexFollowing (Utility/vertexFollowing.cpp:46-88, basic_util.h:14):
 * C[i] = i, -1 for an isolated vertex, its neighbour for a degree-one vertex
 * whose neighbour has degree > 1 (or a lower id).  *numVtxToFix = isolated +
 * following vertices. */
int glv_vertex_following(const glv_graph *G, long *C, long *numVtxToFix);

/* Replaces buildNewGraphVF (Utility/vertexFollowing.cpp:91-255, basic_util.h:15):
 * the graph of the (renumbered) clusters C, without the zero self-loops of
 * buildNextLevelGraphOpt and with every weight cast to long before it is
 * summed, as the reference does.  Gout's arrays are malloc'd (free() them).
 * Rows are sorted by tail (the reference's one-thread order). */
int glv_build_new_graph_vf(const glv_graph *Gin, glv_graph *Gout, const long *C,
                           long numUniqueClusters, double *totTime);

/* ---- batches of independent graphs --------------------------------------
 * No reference counterpart as one call: a batch runs
 * runMultiPhaseColoring (Coloring/runMultiPhaseColoring.cpp:51-238) or, with
 * coloring = 0, runMultiPhaseBasic (BasicCommunitiesDetection/runMultiPhaseBasic.cpp:52-170)
 * on every graph of the batch, each graph with its own modularity constant,
 * phase tests and phase count, in one level holding all graphs.  Graph g owns
 * vertices [vertex_offsets[g], vertex_offsets[g+1]) of one CSR; tails are
 * global vertex ids and must stay inside their row's graph (GLV_ERR_ARG
 * otherwise); every graph needs at least one vertex.  C_out receives each
 * vertex's community as a graph-local id (-1 = isolated).  mode: GLV_MODE_VERIFY
 * (integral weights only; results equal per-graph runs) or GLV_MODE_FAST. */
typedef struct {
  /* per graph: caller-owned arrays of num_graphs entries, each may be NULL */
  double *final_modularity; /* the phase loop's "Final modularity" (prevMod) */
  int *phases;
  int *iterations;
  long *clusters;
  double *done_seconds;     /* time from the start of the run until the graph finished */
  /* whole batch (filled by the call) */
  int rounds;               /* phase rounds of the batch loop */
  double time_total, time_clustering, time_coloring, time_building, time_transfer;
  double edges_swept;
  long kernel_launches;
} glv_batch_stats;

int glv_run_batch_csr(int num_graphs, const long *vertex_offsets, const long *ptr,
                      const long *tail, const double *weight, long *C_out, int coloring,
                      long minGraphSize, double threshold, double C_threshold, int mode,
                      glv_batch_stats *stats);

/* Device-resident batch: d_ptr int64[nv+1], d_tail int32[nnz], d_weight f64[nnz],
 * d_C int32[nv] on the device; vertex_offsets stays a host array. */
int glv_dev_run_batch(int num_graphs, const long *vertex_offsets, const long *d_ptr,
                      const int *d_tail, const double *d_weight, int *d_C, int coloring,
                      long minGraphSize, double threshold, double C_threshold, int mode,
                      void *stream, glv_batch_stats *stats);

/* ---- single phases and primitives (host buffers) ------------------------ */

/* Replaces algoLouvainWithDistOneColoring (Coloring/parallelLouvainWithColoring.cpp:47-286,
 * color_comm.h:10-11).  C[numVertices] is overwritten with the state after the
 * last sweep; *mod receives the returned prevMod. */
int glv_louvain_coloring_phase(const glv_graph *G, long *C, const int *color, int numColor,
                               double Lower, double thresh, int mode, double *mod, int *numItr,
                               double *totTime);

/* Replaces parallelLouvianMethod (BasicCommunitiesDetection/parallelLouvainMethod.cpp:65-326,
 * basic_comm.h:21-22). */
int glv_louvain_basic_phase(const glv_graph *G, long *C, double Lower, double thresh, int mode,
                            double *mod, int *numItr, double *totTime);

/* Replaces algoDistanceOneVertexColoringOpt (Coloring/coloringDistanceOne.cpp:50-233,
 * coloring.h:8).  *maxColor receives the largest colour (the reference's
 * return value). */
int glv_distance_one_coloring(const glv_graph *G, int *vtxColor, int mode, int *maxColor,
                              double *totTime);

/* Replaces vBaseRedistribution (Coloring/vBase.cpp:6-168, coloring.h:15):
 * rebalances a proper colouring with ncolors colours in place.  Classes above
 * avg = ceil(NV / ncolors) give vertices, in vertex order, to colours below
 * avg that were not above it and that no neighbour has: the first such
 * colour (type 0) or the least used (type 1).  The result stays proper.
 * Where no colour qualifies the vertex keeps its colour (the reference's
 * type 0 reads past its frequency array there).  *moves (may be NULL)
 * receives the number of vertices recoloured (the reference returns nothing). */
int glv_vbase_redistribution(const glv_graph *G, int *vtxColor, int ncolors, int type,
                             long *moves);

/* Replaces algoColoringMultiHashMaxMin (Coloring/coloringMultiHashMaxMin.cpp:59-228,
 * coloring.h:12): the incomplete colouring with nHash hashes and nItrs
 * iterations.  Random values come from the C library's rand(), drawn as the
 * reference draws them; vertices left uncoloured hold *maxColor (the
 * reference's return value).  GLV_ERR_COLORS when 2 * nHash * nItrs + 1
 * reaches 4096. */
int glv_color_multihash(const glv_graph *G, int *vtxColor, int nHash, int nItrs,
                        int *maxColor, double *totTime);

/* Replaces renumberClustersContiguously (Utility/buildNextPhase.cpp:48-79,
 * basic_util.h:5). */
int glv_renumber_clusters(long *C, long size, long *numClusters);

/* Replaces buildNextLevelGraphOpt (Utility/buildNextPhase.cpp:83-255,
 * basic_util.h:6).  Gout->edgeListPtrs and Gout->edgeList are malloc'd and
 * owned by the caller (release with free()). */
int glv_build_next_level(const glv_graph *Gin, glv_graph *Gout, const long *C,
                         long numUniqueClusters, int mode, double *totTime);

/* Modularity of an assignment over a graph: the formula of
 * Coloring/parallelLouvainWithColoring.cpp:226-249, standing in for the
 * unimplemented computeModularity (Utility/utilityClusterComparisonMetrics.cpp:409-411). */
int glv_modularity(const glv_graph *G, const long *C, double *mod);

/* Move decisions of a vertex list against one fixed state — the unit
 * buildLocalMapCounter + max compute for one vertex
 * (Utility/utilityClusteringFunctions.cpp:172-194,226-259).  Host buffers
 * (SoA CSR, int64 ids).  targets[k] receives the decision for verts[k]. */
int glv_decide_batch(long nv, const long *ptr, const long *tail, const double *weight,
                     const long *C, const double *vDeg, const double *cDeg, const long *cSize,
                     double constant, long nverts, const long *verts, long *targets);

/* Modularity of an assignment on the device without allocating anything.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * during their run: code whose device memory is all handed out by a host
 * framework's caching allocator (a foreign cudaMalloc can fail on a
 * fragmented or full device and implicitly synchronises it), or code running
 * under a memory budget fixed at start-up.  Inputs and the output are the
 * caller's device buffers: d_ptr int64[nv+1], d_tail int32[nnz],
 * d_weight f64[nnz], d_C int32[nv] (-1 = in no community: such a vertex's
 * entries add nothing to e_xx), d_cDeg f64[nv] (total weighted degree of each
 * community id), `constant` = 1 / (sum of all weighted degrees).  d_out f64[3]
 * receives {Q, e_xx, a2_x}: e_xx is the sum of w over entries (i, t) with
 * C[t] == C[i] >= 0, a2_x the sum of d_cDeg[c]^2 over all ids c < nv, and
 * Q = e_xx*constant - a2_x*constant^2.
 * Scratch is a 1 MiB static device array compiled into the library, which
 * bounds nv to 16,777,216 (larger nv returns GLV_ERR_LIMIT without touching the
 * GPU).  Every GPU that loads the library holds that array until the process
 * exits.  The first call on a device looks up the array's address (once per
 * device, with that device current); make that first call before any stream
 * capture.  The address is kept for the life of the process: after a
 * cudaDeviceReset of that device the entry must not be called again.
 * Without a GPU it returns GLV_ERR_NO_DEVICE.  The work is queued on `stream` (cudaStream_t, NULL = legacy
 * default stream) and is complete when the stream reaches it.  All calls on a
 * device share the one array: calls that overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller. */
int glv_dev_modularity_static(long nv, const long *d_ptr, const int *d_tail,
                              const double *d_weight, const int *d_C, const double *d_cDeg,
                              double constant, double *d_out, void *stream);

/* Device memory: the engine allocates from its own stream-ordered pool per
 * device, keeps the blocks a call frees for the next call (blocks a call does
 * not reuse go back to the pool when it ends), and runs all its work on one
 * internal stream per device (calls from several host threads on one device
 * are serialised).  Between calls the engine therefore still holds up to one
 * call's peak of device memory.  This returns the cached blocks and the
 * pool's unused memory to the driver, e.g. before handing the device to
 * another allocator. */
void glv_release_cached_memory(void);

/* ---- learned move gate (no counterpart in the reference) ---------------- */
#define GLV_GATE_PARAMS 4673   /* W1[64][6] b1[64] W2[64][64] b2[64] W3[64] b3 */
#define GLV_GATE_FEATURES 6

/* Process-wide gate used by GLV_MODE_LEARNED: FP32 master parameters (rounded
 * to BF16 on the device) and the keep threshold on the predicted move
 * probability. */
int glv_gate_set(const float *params, float tau);

/* Move probabilities of n feature rows (device pointers d_feat[n][6],
 * d_prob[n]) with the parameters of glv_gate_set; runs the tensor-core
 * inference kernel on `stream` and synchronises it. */
int glv_gate_infer(long n, const float *d_feat, float *d_prob, void *stream);

/* One forward/backward pass of the weighted binary cross-entropy (mean over
 * the rows) on host arrays x[n][6], y[n] (0/1), w[n]; grad[GLV_GATE_PARAMS]
 * and *loss receive the result.  The gradient-check entry point. */
int glv_gate_grad(long n, const float *x, const float *y, const float *w, const float *params,
                  float *grad, double *loss);

/* Adam training on host arrays (copied to the device once): `epochs` passes
 * in mini-batches of `batch` rows, learning rate `lr`; params is read as the
 * initial value and receives the result; *loss the last epoch's mean loss. */
int glv_gate_train(long n, const float *x, const float *y, const float *w, int epochs,
                   long batch, float lr, unsigned seed, float *params, double *loss);

/* Trace capture for training: while on, every plain colour sweep from the
 * second of a phase appends (features before the sweep, moved 0/1) for a
 * hashed sample `rate` of the non-isolated vertices, up to `capacity` rows. */
int glv_trace_begin(long capacity, double rate);
/* Copies up to cap rows (x[cap][6], y[cap]) to the host; returns rows held. */
long glv_trace_fetch(float *x, float *y, long cap);
int glv_trace_end(void);

/* ---- library information ------------------------------------------------ */
/* Process-wide switch for the following calls: 0 off; 1 time each colour
 * class's sweep with CUDA events (sweep_kernel_time / sweep_bytes); 2 also
 * time every launch by kind (kernel_time). */
void glv_set_profiling(int on);
const char *glv_version(void);
const char *glv_last_error(void);
/* Kernel launches issued by this library since load (all entry points). */
long glv_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* GRAPPOLO_B200_H */
