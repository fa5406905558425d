/*
 * CPU oracle for the multiphase-Louvain-with-colouring path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file; it is used by tests/, by __graft_entry__.smoke() and by
 * bench.py's cpu_baseline leg, and only as the checker.
 *
 * Each function restates, in plain C, what Grappolo's own code computes when it
 * runs on one OpenMP thread (the deterministic schedule), citing the reference
 * file:line it follows.  The restatement is pinned against the reference itself:
 * oracle/Makefile compiles the reference's sources into oracle/_ref/ and
 * tests/test_oracle_vs_reference.py compares the two bit for bit; the golden
 * fixtures under tests/golden/ were generated by the compiled reference.
 *
 * Conventions: vertex ids and offsets are int64 (`long`), weights FP64, CSR
 * rows as in DefineStructure/defs.h:85-92 (every undirected edge stored in both
 * directions, self-loops once).  All FP expressions are written in the
 * reference's evaluation order and the file is compiled with
 * -ffp-contract=off so no FMA contraction changes a rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define LVO_MAX_COLORS 4096 /* Coloring/coloringUtils.h: #define MaxDegree 4096 */

/* ------------------------------------------------------------------------ */
/* A per-vertex community -> weight map.  The reference uses std::map plus a
 * Counter vector (Utility/utilityClusteringFunctions.cpp:172-194).  The move
 * decision it feeds (max(), :226-259) does not depend on iteration order, so
 * an open-addressing table with insertion-ordered slots is equivalent.       */
typedef struct {
    long cap;        /* power of two */
    long *keys;      /* -2 = empty   */
    long *slot;      /* index into val[] */
    double *val;
    long *order;     /* keys in insertion order */
    long n;
} lvo_map;

static void map_init(lvo_map *m, long max_entries) {
    long cap = 16;
    while (cap < 2 * (max_entries + 1)) cap <<= 1;
    m->cap = cap;
    m->keys = (long *)malloc(sizeof(long) * cap);
    m->slot = (long *)malloc(sizeof(long) * cap);
    m->val = (double *)malloc(sizeof(double) * (max_entries + 1));
    m->order = (long *)malloc(sizeof(long) * (max_entries + 1));
    for (long i = 0; i < cap; i++) m->keys[i] = -2;
    m->n = 0;
}

static void map_free(lvo_map *m) {
    free(m->keys); free(m->slot); free(m->val); free(m->order);
}

static void map_clear(lvo_map *m) {
    for (long k = 0; k < m->n; k++) {
        long key = m->order[k];
        uint64_t h = ((uint64_t)key * 0x9E3779B97F4A7C15ull) & (uint64_t)(m->cap - 1);
        while (m->keys[h] != key) h = (h + 1) & (uint64_t)(m->cap - 1);
        m->keys[h] = -3; /* tombstone during clear */
    }
    for (long k = 0; k < m->n; k++) {
        long key = m->order[k];
        uint64_t h = ((uint64_t)key * 0x9E3779B97F4A7C15ull) & (uint64_t)(m->cap - 1);
        while (m->keys[h] != -3) h = (h + 1) & (uint64_t)(m->cap - 1);
        m->keys[h] = -2;
    }
    m->n = 0;
}

/* Returns the value index of `key`, inserting it with value `init` if absent. */
static long map_find_or_insert(lvo_map *m, long key, double init, int *inserted) {
    uint64_t h = ((uint64_t)key * 0x9E3779B97F4A7C15ull) & (uint64_t)(m->cap - 1);
    while (1) {
        if (m->keys[h] == key) { *inserted = 0; return m->slot[h]; }
        if (m->keys[h] == -2) {
            m->keys[h] = key;
            m->slot[h] = m->n;
            m->val[m->n] = init;
            m->order[m->n] = key;
            *inserted = 1;
            return m->n++;
        }
        h = (h + 1) & (uint64_t)(m->cap - 1);
    }
}

static long max_degree(long nv, const long *ptr) {
    long md = 0;
    for (long i = 0; i < nv; i++)
        if (ptr[i + 1] - ptr[i] > md) md = ptr[i + 1] - ptr[i];
    return md;
}

/* ------------------------------------------------------------------------ */
/* Utility/utilityClusteringFunctions.cpp:70-87 (sumVertexDegree) and :89-96
 * (calConstantForSecondTerm): CSR-order degree sums; 1 / sequential sum.      */
double lvo_vertex_degrees(long nv, const long *ptr, const double *w, double *vDeg) {
    double total = 0;
    for (long i = 0; i < nv; i++) {
        double s = 0;
        for (long j = ptr[i]; j < ptr[i + 1]; j++) s += w[j];
        vDeg[i] = s;
    }
    for (long i = 0; i < nv; i++) total += vDeg[i];
    return (double)1 / total;
}

/* One vertex's move decision against a given state:
 * Coloring/parallelLouvainWithColoring.cpp:181-191 builds the map with the own
 * community first at 0 (:183-184), buildLocalMapCounter
 * (utilityClusteringFunctions.cpp:172-194) sums weights per neighbouring
 * community in CSR order and the self-loop weight; max() (:226-259) takes the
 * strictly positive best gain, ties to the lower id, with swap protection.
 * Returns -1 for an empty row.  *own_w receives Counter[own] (the Jacobi phase
 * adds it to clusterWeightInternal, parallelLouvainMethod.cpp:215).          */
static long decide(long i, const long *ptr, const long *tail, const double *w,
                   const long *C, const double *vDeg, const double *cDeg,
                   const long *cSize, double constant, lvo_map *m, double *own_w) {
    long adj1 = ptr[i], adj2 = ptr[i + 1];
    if (adj1 == adj2) { *own_w = 0; return -1; }
    long sc = C[i];
    int ins;
    map_clear(m);
    map_find_or_insert(m, sc, 0.0, &ins);
    double selfLoop = 0;
    for (long j = adj1; j < adj2; j++) {
        long t = tail[j];
        if (t == i) selfLoop += w[j];
        long k = map_find_or_insert(m, C[t], w[j], &ins);
        if (!ins) m->val[k] += w[j];
    }
    double degree = vDeg[i];
    long maxIndex = sc;
    double curGain = 0, maxGain = 0;
    double eix = m->val[0] - selfLoop;
    double ax = cDeg[sc] - degree;
    for (long k = 1; k < m->n; k++) {
        long y = m->order[k];
        if (y == sc) continue;
        double ay = cDeg[y];
        double eiy = m->val[k];
        curGain = 2 * (eiy - eix) - 2 * degree * (ay - ax) * constant;
        if ((curGain > maxGain) || ((curGain == maxGain) && (curGain != 0) && (y < maxIndex))) {
            maxGain = curGain;
            maxIndex = y;
        }
    }
    if (cSize[maxIndex] == 1 && cSize[sc] == 1 && maxIndex > sc) maxIndex = sc;
    *own_w = m->val[0];
    return maxIndex;
}

/* Move decisions for a list of vertices against one fixed state (no updates).
 * This is the per-step unit the GPU sweep is compared on.                    */
void lvo_decide_batch(long nv, const long *ptr, const long *tail, const double *w,
                      const long *C, const double *vDeg, const double *cDeg,
                      const long *cSize, double constant, long nverts,
                      const long *verts, long *targets) {
    lvo_map m;
    map_init(&m, max_degree(nv, ptr));
    for (long k = 0; k < nverts; k++) {
        double own;
        targets[k] = decide(verts[k], ptr, tail, w, C, vDeg, cDeg, cSize, constant, &m, &own);
    }
    map_free(&m);
}

/* ------------------------------------------------------------------------ */
/* Coloring/coloringDistanceOne.cpp:50-233 at one thread: the speculative pass
 * (:137-150) visits v = 0..NV-1 in order and takes the first colour not used by
 * an already coloured neighbour (coloringUtils.cpp:44-67, self-loops skipped);
 * the conflict pass then finds nothing.  Input colours must be -1 (the callers
 * initialise them so, runMultiPhaseColoring.cpp:61-65,174-177).
 * Returns the largest colour, or -2 when a colour reaches MaxDegree (the
 * reference exits there, coloringUtils.cpp:57-60).                          */
int lvo_color_greedy(long nv, const long *ptr, const long *tail, int *color) {
    unsigned char *mark = (unsigned char *)calloc(LVO_MAX_COLORS + 1, 1);
    int maxc = -1;
    for (long v = 0; v < nv; v++) color[v] = -1;
    for (long v = 0; v < nv; v++) {
        int mc = -1;
        for (long k = ptr[v]; k < ptr[v + 1]; k++) {
            long t = tail[k];
            if (t == v) continue;
            int c = color[t];
            if (c >= 0) {
                if (c >= LVO_MAX_COLORS) { free(mark); return -2; }
                mark[c] = 1;
                if (c > mc) mc = c;
            }
        }
        int my;
        for (my = 0; my <= mc; my++) if (!mark[my]) break;
        color[v] = my;
        if (my > maxc) maxc = my;
        for (long k = ptr[v]; k < ptr[v + 1]; k++) {
            long t = tail[k];
            if (t != v && color[t] >= 0) mark[color[t]] = 0;
        }
    }
    free(mark);
    return maxc;
}

/* Coloring/coloringMultiHashMaxMin.cpp:59-228 (incomplete colouring) at one
 * thread.  Draws nHash x nv values from the C library's rand(), hash after
 * hash (:45-57, :95-101); every vertex starts at maxColor = 2*nHash*nItrs
 * (:106-110).  In pass (itr, ihash) an uncoloured vertex takes colour
 * cur = 2*itr*nHash + 2*ihash when its value is above that of every
 * neighbour still at a colour >= cur, cur + 1 when below all of them
 * (:117-155).  An iteration that colours nothing after all vertices are
 * coloured lowers maxColor to 2*(itr-1)*nHash + 2*nHash + 1 (:160-168).
 * Returns maxColor; uncoloured vertices keep it.                           */
int lvo_color_mhash(long nv, const long *ptr, const long *tail, int nHash, int nItrs,
                    int *color) {
    double *rnd = (double *)malloc(sizeof(double) * (size_t)nHash * (nv ? nv : 1));
    for (int h = 0; h < nHash; h++)
        for (long v = 0; v < nv; v++) rnd[(size_t)h * nv + v] = (double)rand();
    int maxColor = 2 * nHash * nItrs;
    for (long v = 0; v < nv; v++) color[v] = maxColor;
    long totalColored = 0, iterFreq = 0;
    for (int itr = 0; itr < nItrs; itr++) {
        for (int h = 0; h < nHash; h++) {
            const int cur = 2 * itr * nHash + 2 * h;
            const double *r = rnd + (size_t)h * nv;
            for (long v = 0; v < nv; v++) {
                if (color[v] != maxColor) continue;
                int isMax = 1, isMin = 1;
                for (long k = ptr[v]; k < ptr[v + 1]; k++) {
                    long u = tail[k];
                    if (u == v || color[u] < cur) continue;
                    if (r[v] <= r[u]) isMax = 0;
                    if (r[v] >= r[u]) isMin = 0;
                }
                if (isMax) { color[v] = cur; iterFreq++; }
                else if (isMin) { color[v] = cur + 1; iterFreq++; }
            }
        }
        totalColored += iterFreq;
        if (iterFreq == 0) {
            if (totalColored == nv) {
                maxColor = 2 * (itr - 1) * nHash + 2 * nHash + 1;
                break;
            }
        } else {
            iterFreq = 0;
        }
    }
    free(rnd);
    return maxColor;
}

/* vBaseRedistribution (Coloring/vBase.cpp:6-168) at one thread; type 0 takes
 * the first qualifying colour, type 1 the least used (lowest on ties).  avg = ceil(NV / ncolors); a class is oversized when it holds more
 * than avg vertices (:78-90).  In vertex order, a vertex of an oversized class
 * whose class still holds more than avg moves to the smallest colour that no
 * neighbour has, that holds fewer than avg and that was not oversized
 * (:94-134).  When no colour below ncolors qualifies, type 0 in the reference
 * reads one entry past its frequency arrays (:113-116); here the vertex stays
 * (what type 1 does, and what the reference's checks of myColor != ncolors
 * at :128-130 expect), and
 * *stuck (may be NULL) counts those vertices.  Moves are sequential, so the
 * colouring stays proper and the conflict pass (:137-141) finds nothing.
 * Returns the number of moves.                                              */
long lvo_vbase(long nv, const long *ptr, const long *tail, int *color, int ncolors, int type,
               long *stuck) {
    long *freq = (long *)calloc(ncolors + 1, sizeof(long));
    unsigned char *over = (unsigned char *)calloc(ncolors + 1, 1);
    unsigned char *mark = (unsigned char *)calloc(ncolors + 1, 1);
    long *base = (long *)malloc(sizeof(long) * (nv ? nv : 1));
    for (long v = 0; v < nv; v++) { base[v] = color[v]; freq[color[v]]++; }
    long avg = (long)ceil((double)nv / (double)ncolors);
    for (int c = 0; c < ncolors; c++) over[c] = freq[c] > avg;
    long moves = 0;
    for (long v = 0; v < nv; v++) {
        if (!over[base[v]]) continue;
        if (color[v] != -1 && freq[color[v]] <= avg) continue;
        for (long k = ptr[v]; k < ptr[v + 1]; k++) {
            long u = tail[k];
            if (u != v && color[u] >= 0 && color[u] < ncolors) mark[color[u]] = 1;
        }
        int my = -1;
        for (int c = 0; c < ncolors; c++) {
            if (mark[c] || freq[c] >= avg || over[c]) continue;
            if (type == 0) { my = c; break; }                /* first fit (:112-117) */
            if (my == -1 || freq[my] > freq[c]) my = c;       /* least used (:118-126) */
        }
        for (long k = ptr[v]; k < ptr[v + 1]; k++) {
            long u = tail[k];
            if (u != v && color[u] >= 0 && color[u] < ncolors) mark[color[u]] = 0;
        }
        if (my >= 0) {
            freq[my]++;
            freq[color[v]]--;
            color[v] = my;
            moves++;
        } else if (stuck) {
            (*stuck)++;
        }
    }
    free(freq); free(over); free(mark); free(base);
    return moves;
}

/* Modularity pieces shared by both sweeps: Q = e_xx*c - a2_x*c*c
 * (parallelLouvainWithColoring.cpp:222-249, parallelLouvainMethod.cpp:244-255). */
static double modularity_from(long nv, const double *cWI, const double *cDeg, double c) {
    double e_xx = 0, a2_x = 0;
    for (long i = 0; i < nv; i++) {
        e_xx += cWI[i];
        a2_x += cDeg[i] * cDeg[i];
    }
    return e_xx * c - a2_x * c * c;
}

/* Coloring/parallelLouvainWithColoring.cpp:47-286 at one thread.
 * `C` is overwritten (input ignored, :105-108); classes are swept in colour
 * order with members in ascending id (:113-141), each class deciding against
 * the community totals from the class start and writing C in place
 * (:158-218); the totals take the class's deltas, accumulated from zero in
 * member order, at the class end.  Returns prevMod (:284); C holds the state
 * after the last sweep.  `trace_q` (may be NULL) receives each iteration's Q. */
double lvo_coloring_phase(long nv, const long *ptr, const long *tail, const double *w,
                          long *C, const int *color, int numColor, double Lower,
                          double thresh, int *numItr, double *trace_q, int trace_cap) {
    double *vDeg = (double *)malloc(sizeof(double) * (nv ? nv : 1));
    double *cDeg = (double *)malloc(sizeof(double) * (nv ? nv : 1));
    long *cSize = (long *)malloc(sizeof(long) * (nv ? nv : 1));
    double *uDeg = (double *)calloc(nv ? nv : 1, sizeof(double));
    long *uSize = (long *)calloc(nv ? nv : 1, sizeof(long));
    long *touched = (long *)malloc(sizeof(long) * (2 * nv + 1));
    double *cWI = (double *)malloc(sizeof(double) * (nv ? nv : 1));
    double constant = lvo_vertex_degrees(nv, ptr, w, vDeg);
    for (long i = 0; i < nv; i++) { cDeg[i] = vDeg[i]; cSize[i] = 1; C[i] = i; }

    long *colorPtr = (long *)calloc(numColor + 1, sizeof(long));
    long *colorIndex = (long *)malloc(sizeof(long) * (nv ? nv : 1));
    long *added = (long *)calloc(numColor + 1, sizeof(long));
    for (long i = 0; i < nv; i++) colorPtr[color[i] + 1]++;
    for (long i = 0; i < numColor; i++) colorPtr[i + 1] += colorPtr[i];
    for (long i = 0; i < nv; i++) {
        long tc = color[i];
        colorIndex[colorPtr[tc] + added[tc]++] = i;
    }

    lvo_map m;
    map_init(&m, max_degree(nv, ptr));
    double prevMod = Lower, currMod = -1;
    int itr = 0;
    while (1) {
        itr++;
        for (long ci = 0; ci < numColor; ci++) {
            long nt = 0;
            for (long K = colorPtr[ci]; K < colorPtr[ci + 1]; K++) {
                long i = colorIndex[K];
                double own;
                long target = decide(i, ptr, tail, w, C, vDeg, cDeg, cSize, constant, &m, &own);
                if (target != C[i] && target != -1) {
                    uDeg[target] += vDeg[i]; uSize[target] += 1;
                    uDeg[C[i]] -= vDeg[i]; uSize[C[i]] -= 1;
                    touched[nt++] = target; touched[nt++] = C[i];
                }
                C[i] = target;
            }
            /* cInfo += cUpdate (:213-217); untouched entries add 0.0, a no-op */
            for (long k = 0; k < nt; k++) {
                long c = touched[k];
                if (uSize[c] != 0 || uDeg[c] != 0 || 1) {
                    cSize[c] += uSize[c]; cDeg[c] += uDeg[c];
                    uSize[c] = 0; uDeg[c] = 0;
                }
            }
        }
        for (long i = 0; i < nv; i++) {
            double s = 0;
            for (long j = ptr[i]; j < ptr[i + 1]; j++)
                if (C[tail[j]] == C[i]) s += w[j];
            cWI[i] = s;
        }
        currMod = modularity_from(nv, cWI, cDeg, constant);
        if (trace_q && itr <= trace_cap) trace_q[itr - 1] = currMod;
        if ((currMod - prevMod) < thresh) break;
        prevMod = currMod;
    }
    *numItr = itr;
    map_free(&m);
    free(vDeg); free(cDeg); free(cSize); free(uDeg); free(uSize); free(touched); free(cWI);
    free(colorPtr); free(colorIndex); free(added);
    return prevMod;
}

/* BasicCommunitiesDetection/parallelLouvainMethod.cpp:65-326 at one thread:
 * synchronous (Jacobi) moves; Q is taken on the state before the moves
 * (:244-255); on exit C = the last accepted state (:304-307) and the return
 * value is max(Q_prev, Lower) (:271-273).                                      */
double lvo_basic_phase(long nv, const long *ptr, const long *tail, const double *w,
                       long *C, double Lower, double thresh, int *numItr,
                       double *trace_q, int trace_cap) {
    long n1 = nv ? nv : 1;
    double *vDeg = (double *)malloc(sizeof(double) * n1);
    double *cDeg = (double *)malloc(sizeof(double) * n1);
    long *cSize = (long *)malloc(sizeof(long) * n1);
    double *uDeg = (double *)malloc(sizeof(double) * n1);
    long *uSize = (long *)malloc(sizeof(long) * n1);
    double *cWI = (double *)malloc(sizeof(double) * n1);
    long *past = (long *)malloc(sizeof(long) * n1);
    long *curr = (long *)malloc(sizeof(long) * n1);
    long *target = (long *)malloc(sizeof(long) * n1);
    double constant = lvo_vertex_degrees(nv, ptr, w, vDeg);
    for (long i = 0; i < nv; i++) { cDeg[i] = vDeg[i]; cSize[i] = 1; past[i] = i; curr[i] = i; }
    lvo_map m;
    map_init(&m, max_degree(nv, ptr));
    double prevMod = -1, currMod = -1;
    int itr = 0;
    while (1) {
        itr++;
        for (long i = 0; i < nv; i++) { cWI[i] = 0; uDeg[i] = 0; uSize[i] = 0; }
        for (long i = 0; i < nv; i++) {
            double own = 0;
            if (ptr[i] != ptr[i + 1]) {
                target[i] = decide(i, ptr, tail, w, curr, vDeg, cDeg, cSize, constant, &m, &own);
                cWI[i] += own;
            } else {
                target[i] = -1;
            }
            if (target[i] != curr[i] && target[i] != -1) {
                uDeg[target[i]] += vDeg[i]; uSize[target[i]] += 1;
                uDeg[curr[i]] -= vDeg[i]; uSize[curr[i]] -= 1;
            }
        }
        currMod = modularity_from(nv, cWI, cDeg, constant);
        if (trace_q && itr <= trace_cap) trace_q[itr - 1] = currMod;
        if ((currMod - prevMod) < thresh) break;
        prevMod = currMod;
        if (prevMod < Lower) prevMod = Lower;
        for (long i = 0; i < nv; i++) { cSize[i] += uSize[i]; cDeg[i] += uDeg[i]; }
        long *tmp = past; past = curr; curr = target; target = tmp;
    }
    *numItr = itr;
    for (long i = 0; i < nv; i++) C[i] = past[i];
    map_free(&m);
    free(vDeg); free(cDeg); free(cSize); free(uDeg); free(uSize); free(cWI);
    free(past); free(curr); free(target);
    return prevMod;
}

/* Utility/buildNextPhase.cpp:48-79: ids in order of first occurrence scanning
 * i = 0..size-1; negative entries are left alone.                             */
long lvo_renumber(long *C, long size) {
    long maxc = -1;
    for (long i = 0; i < size; i++) if (C[i] > maxc) maxc = C[i];
    long *map = (long *)malloc(sizeof(long) * (maxc + 2));
    for (long k = 0; k <= maxc; k++) map[k] = -1;
    long n = 0;
    for (long i = 0; i < size; i++) {
        if (C[i] >= 0) {
            if (map[C[i]] < 0) map[C[i]] = n++;
            C[i] = map[C[i]];
        }
    }
    free(map);
    return n;
}

/* Utility/buildNextPhase.cpp:83-255 at one thread.  Every cluster gets a
 * self-loop entry seeded with 0.0 (:119-123); an entry i->t with C[i] >= C[t]
 * adds its weight to cluster pair (C[i], C[t]) in (i, j) order, a new pair
 * starting at the weight (:145-174); row a then lists its pairs (a, b<=a) in
 * ascending b followed by the mirrored pairs (a, b>a) in ascending b
 * (:205-223).  Returns the output nnz; *numEdges_out = NE_out + NV_out
 * (:234-239).  Output arrays are malloc'd (release with lvo_free).           */
long lvo_build_next_level(long nv, const long *ptr, const long *tail, const double *w,
                          const long *C, long ncl, long **optr, long **otail,
                          double **ow, long *numEdges_out) {
    long nnz = ptr[nv];
    /* pair table keyed by a*ncl+b (b <= a) */
    long cap = 16;
    while (cap < 2 * (nnz + ncl + 1)) cap <<= 1;
    long *keys = (long *)malloc(sizeof(long) * cap);
    long *slot = (long *)malloc(sizeof(long) * cap);
    for (long k = 0; k < cap; k++) keys[k] = -1;
    long maxpairs = nnz + ncl + 1;
    long *pa = (long *)malloc(sizeof(long) * maxpairs);
    long *pb = (long *)malloc(sizeof(long) * maxpairs);
    double *pw = (double *)malloc(sizeof(double) * maxpairs);
    long np = 0;
#define PAIR_FIND(A, B, INIT, IDX, NEW)                                               \
    do {                                                                              \
        long key_ = (A) * ncl + (B);                                                  \
        uint64_t h_ = ((uint64_t)key_ * 0x9E3779B97F4A7C15ull) & (uint64_t)(cap - 1); \
        NEW = 0;                                                                      \
        while (1) {                                                                   \
            if (keys[h_] == key_) { IDX = slot[h_]; break; }                          \
            if (keys[h_] == -1) {                                                     \
                keys[h_] = key_; slot[h_] = np; pa[np] = (A); pb[np] = (B);           \
                pw[np] = (INIT); IDX = np++; NEW = 1; break;                          \
            }                                                                         \
            h_ = (h_ + 1) & (uint64_t)(cap - 1);                                      \
        }                                                                             \
    } while (0)
    long idx; int isnew;
    for (long a = 0; a < ncl; a++) { PAIR_FIND(a, a, 0.0, idx, isnew); }
    for (long i = 0; i < nv; i++) {
        for (long j = ptr[i]; j < ptr[i + 1]; j++) {
            long a = C[i], b = C[tail[j]];
            if (a >= b) {
                PAIR_FIND(a, b, w[j], idx, isnew);
                if (!isnew) pw[idx] += w[j];
            }
        }
    }
#undef PAIR_FIND
    /* row sizes: pair (a,b): row a gets one, row b one more if a > b */
    long *rp = (long *)calloc(ncl + 1, sizeof(long));
    long ne_off = 0;
    for (long p = 0; p < np; p++) {
        rp[pa[p] + 1]++;
        if (pa[p] > pb[p]) { rp[pb[p] + 1]++; ne_off++; }
    }
    for (long a = 0; a < ncl; a++) rp[a + 1] += rp[a];
    long onnz = rp[ncl];
    long *ot = (long *)malloc(sizeof(long) * (onnz ? onnz : 1));
    double *owt = (double *)malloc(sizeof(double) * (onnz ? onnz : 1));
    /* sort pairs by (a, b): counting sort on b then stable on a */
    long *ord = (long *)malloc(sizeof(long) * (np ? np : 1));
    long *tmp = (long *)malloc(sizeof(long) * (np ? np : 1));
    long *cnt = (long *)calloc(ncl + 1, sizeof(long));
    for (long p = 0; p < np; p++) cnt[pb[p] + 1]++;
    for (long k = 0; k < ncl; k++) cnt[k + 1] += cnt[k];
    for (long p = 0; p < np; p++) tmp[cnt[pb[p]]++] = p;
    memset(cnt, 0, sizeof(long) * (ncl + 1));
    for (long p = 0; p < np; p++) cnt[pa[p] + 1]++;
    for (long k = 0; k < ncl; k++) cnt[k + 1] += cnt[k];
    for (long q = 0; q < np; q++) { long p = tmp[q]; ord[cnt[pa[p]]++] = p; }
    /* rows in processing order: cluster i = 0.. emits its pairs ascending;
       the mirror goes to row b at its next free slot (:205-223)             */
    long *fill = (long *)calloc(ncl + 1, sizeof(long));
    for (long q = 0; q < np; q++) {
        long p = ord[q];
        long a = pa[p], b = pb[p];
        long where = rp[a] + fill[a]++;
        ot[where] = b; owt[where] = pw[p];
        if (a != b) {
            where = rp[b] + fill[b]++;
            ot[where] = a; owt[where] = pw[p];
        }
    }
    free(fill); free(cnt); free(tmp); free(ord);
    free(keys); free(slot); free(pa); free(pb); free(pw);
    *optr = rp; *otail = ot; *ow = owt;
    *numEdges_out = ne_off + ncl;
    return onnz;
}

/* Utility/vertexFollowing.cpp:46-88 vertexFollowing.  C[i] = i; an isolated
 * vertex gets -1; a degree-one vertex i with neighbour t follows it (C[i] = t)
 * when t has degree > 1 or i > t (so of two degree-one partners the higher id
 * follows).  Returns the number of isolated plus following vertices.       */
long lvo_vertex_following(long nv, const long *ptr, const long *tail, long *C) {
    long num = 0;
    for (long i = 0; i < nv; i++) C[i] = i;
    for (long i = 0; i < nv; i++) {
        long d = ptr[i + 1] - ptr[i];
        if (d == 0) { num++; C[i] = -1; continue; }
        if (d == 1) {
            long t = tail[ptr[i]];
            if ((ptr[t + 1] - ptr[t]) > 1 || i > t) { num++; C[i] = t; }
        }
    }
    return num;
}

/* Utility/vertexFollowing.cpp:91-255 buildNewGraphVF at one thread.  Like
 * lvo_build_next_level but with no zero self-loop seeds and with each entry's
 * weight cast to long before it is added (:150-152: `(long)weight`), the sums
 * kept in long (:113 map<long,long>).  Rows come out sorted by tail: cluster
 * i's map (keys b <= i, ascending) fills row i, and each mirror goes to row b
 * after b's own entries (:190-210).  *numEdges_out = NE_out + NE_self.      */
long lvo_build_new_graph_vf(long nv, const long *ptr, const long *tail, const double *w,
                            const long *C, long ncl, long **optr, long **otail, double **ow,
                            long *numEdges_out) {
    long nnz = ptr[nv];
    long cap = 16;
    while (cap < 2 * (nnz + 1)) cap <<= 1;
    long *keys = (long *)malloc(sizeof(long) * cap);
    long *slot = (long *)malloc(sizeof(long) * cap);
    for (long k = 0; k < cap; k++) keys[k] = -1;
    long *pa = (long *)malloc(sizeof(long) * (nnz + 1));
    long *pb = (long *)malloc(sizeof(long) * (nnz + 1));
    long *pw = (long *)malloc(sizeof(long) * (nnz + 1));
    long np = 0;
    for (long i = 0; i < nv; i++) {
        if (C[i] < 0 || C[i] > ncl) continue;
        for (long j = ptr[i]; j < ptr[i + 1]; j++) {
            long a = C[i], b = C[tail[j]];
            if (a < b) continue;
            long key = a * ncl + b;
            uint64_t h = ((uint64_t)key * 0x9E3779B97F4A7C15ull) & (uint64_t)(cap - 1);
            while (1) {
                if (keys[h] == key) { pw[slot[h]] += (long)w[j]; break; }
                if (keys[h] == -1) {
                    keys[h] = key; slot[h] = np;
                    pa[np] = a; pb[np] = b; pw[np] = (long)w[j]; np++;
                    break;
                }
                h = (h + 1) & (uint64_t)(cap - 1);
            }
        }
    }
    long *rp = (long *)calloc(ncl + 1, sizeof(long));
    long ne_out = 0, ne_self = 0;
    for (long p = 0; p < np; p++) {
        rp[pa[p] + 1]++;
        if (pa[p] > pb[p]) { rp[pb[p] + 1]++; ne_out++; } else ne_self++;
    }
    for (long a = 0; a < ncl; a++) rp[a + 1] += rp[a];
    long onnz = rp[ncl];
    long *ot = (long *)malloc(sizeof(long) * (onnz ? onnz : 1));
    double *owt = (double *)malloc(sizeof(double) * (onnz ? onnz : 1));
    /* pairs sorted by (a, b) (counting sorts), then emitted cluster by cluster */
    long *ord = (long *)malloc(sizeof(long) * (np ? np : 1));
    long *tmp = (long *)malloc(sizeof(long) * (np ? np : 1));
    long *cnt = (long *)calloc(ncl + 1, sizeof(long));
    for (long p = 0; p < np; p++) cnt[pb[p] + 1]++;
    for (long k = 0; k < ncl; k++) cnt[k + 1] += cnt[k];
    for (long p = 0; p < np; p++) tmp[cnt[pb[p]]++] = p;
    memset(cnt, 0, sizeof(long) * (ncl + 1));
    for (long p = 0; p < np; p++) cnt[pa[p] + 1]++;
    for (long k = 0; k < ncl; k++) cnt[k + 1] += cnt[k];
    for (long q = 0; q < np; q++) { long p = tmp[q]; ord[cnt[pa[p]]++] = p; }
    long *fill = (long *)calloc(ncl + 1, sizeof(long));
    for (long q = 0; q < np; q++) {
        long p = ord[q];
        long a = pa[p], b = pb[p];
        long where = rp[a] + fill[a]++;
        ot[where] = b; owt[where] = (double)pw[p];
        if (a != b) {
            where = rp[b] + fill[b]++;
            ot[where] = a; owt[where] = (double)pw[p];
        }
    }
    free(fill); free(cnt); free(tmp); free(ord);
    free(keys); free(slot); free(pa); free(pb); free(pw);
    *optr = rp; *otail = ot; *ow = owt;
    *numEdges_out = ne_out + ne_self;
    return onnz;
}

/* ---- edge-list preprocessing (Utility/utilityFunctions.cpp:416-531) ---- */

static const long *g_key_head, *g_key_tail;
static int cmp_pair_then_index(const void *a, const void *b) {
    long i = *(const long *)a, j = *(const long *)b;
    if (g_key_head[i] != g_key_head[j]) return g_key_head[i] < g_key_head[j] ? -1 : 1;
    if (g_key_tail[i] != g_key_tail[j]) return g_key_tail[i] < g_key_tail[j] ? -1 : 1;
    return i < j ? -1 : (i > j);
}

/* removeEdges (utilityFunctions.cpp:416-460) on SoA arrays, in place.  An
 * edge is kept when it is not a self-loop and no earlier edge has the same
 * (head, tail) (:428-446).  The compaction (:448-455) fills the dropped slots
 * below NGE, in ascending order, with the kept edges at positions >= NGE
 * taken from the top down; positions >= NGE are left as they were.
 * Returns NGE.                                                              */
long lvo_remove_edges(long nv, long ne, long *head, long *tail, double *w) {
    (void)nv;
    long *idx = (long *)malloc(sizeof(long) * (ne ? ne : 1));
    unsigned char *good = (unsigned char *)calloc(ne ? ne : 1, 1);
    for (long i = 0; i < ne; i++) idx[i] = i;
    g_key_head = head; g_key_tail = tail;
    qsort(idx, ne, sizeof(long), cmp_pair_then_index);
    long nge = 0;
    for (long s = 0; s < ne; s++) {
        long i = idx[s];
        int first = s == 0 || head[idx[s - 1]] != head[i] || tail[idx[s - 1]] != tail[i];
        if (first && head[i] != tail[i]) { good[i] = 1; nge++; }
    }
    long top = ne - 1;
    for (long k = 0; k < nge; k++) {
        if (good[k]) continue;
        while (!good[top]) top--;
        head[k] = head[top]; tail[k] = tail[top]; w[k] = w[top];
        top--;
    }
    free(idx); free(good);
    return nge;
}

/* SortEdgesUndirected (utilityFunctions.cpp:463-498): every edge i, in list
 * order, is appended to its head's row as head->tail and then to its tail's
 * row as tail->head.  ptrs[0..NV] is the CSR offset array and ptrs[NV+1]
 * = 2*NE, as the reference's shifted histogram leaves it.                 */
void lvo_sort_edges_undirected(long nv, long ne, const long *head, const long *tail,
                               const double *w, long *ptrs, long *ohead, long *otail,
                               double *ow) {
    long *fill = (long *)calloc(nv + 1, sizeof(long));
    for (long i = 0; i <= nv + 1; i++) ptrs[i] = 0;
    for (long i = 0; i < ne; i++) { ptrs[head[i] + 1]++; ptrs[tail[i] + 1]++; }
    for (long v = 0; v < nv; v++) ptrs[v + 1] += ptrs[v];
    ptrs[nv + 1] = 2 * ne;
    for (long v = 0; v < nv; v++) fill[v] = ptrs[v];
    for (long i = 0; i < ne; i++) {
        long a = fill[head[i]]++;
        ohead[a] = head[i]; otail[a] = tail[i]; ow[a] = w[i];
        long b = fill[tail[i]]++;
        ohead[b] = tail[i]; otail[b] = head[i]; ow[b] = w[i];
    }
    free(fill);
}

static const long *g_row_tail;
static int cmp_tail_then_later(const void *a, const void *b) {
    long i = *(const long *)a, j = *(const long *)b;
    if (g_row_tail[i] != g_row_tail[j]) return g_row_tail[i] < g_row_tail[j] ? -1 : 1;
    return i > j ? -1 : (i < j);
}

/* SortNodeEdgesByIndex (utilityFunctions.cpp:501-531): each row sorted by
 * tail.  Its bottom-up merge takes the right run's element on equal tails
 * (:517-518), and two entries of one row first meet when the higher-placed
 * one is in the right run, so equal tails end in descending position.     */
void lvo_sort_node_edges(long nv, const long *ptrs, long *head, long *tail, double *w) {
    long nnz = ptrs[nv];
    long *idx = (long *)malloc(sizeof(long) * (nnz ? nnz : 1));
    long *th = (long *)malloc(sizeof(long) * (nnz ? nnz : 1));
    long *tt = (long *)malloc(sizeof(long) * (nnz ? nnz : 1));
    double *tw = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
    memcpy(th, head, sizeof(long) * nnz); memcpy(tt, tail, sizeof(long) * nnz);
    memcpy(tw, w, sizeof(double) * nnz);
    for (long j = 0; j < nnz; j++) idx[j] = j;
    g_row_tail = tt;
    for (long v = 0; v < nv; v++)
        qsort(idx + ptrs[v], ptrs[v + 1] - ptrs[v], sizeof(long), cmp_tail_then_later);
    for (long j = 0; j < nnz; j++) { head[j] = th[idx[j]]; tail[j] = tt[idx[j]]; w[j] = tw[idx[j]]; }
    free(idx); free(th); free(tt); free(tw);
}

/* ---- comparing community assignments (utilityClusterComparisonMetrics.cpp) */

static int cmp_long(const void *a, const void *b) {
    long x = *(const long *)a, y = *(const long *)b;
    return x < y ? -1 : (x > y);
}

/* computeGiniCoefficient (:310-330): sizes sorted ascending in place. */
double lvo_gini(long *size, int n) {
    qsort(size, n, sizeof(long), cmp_long);
    double num = 0.0, den = 0.0;
    for (long i = 0; i < n; i++) {
        num = num + ((i + 1) * size[i]);
        den = den + size[i];
    }
    return ((2 * num) / (n * den)) - ((double)(n + 1) / (double)n);
}

/* Members of each community (0-based index ids[i] in [0, nc)), in vertex order. */
static void group(long n, const long *ids, long nc, long **ptr_out, long **idx_out) {
    long *ptr = (long *)calloc(nc + 1, sizeof(long));
    long *idx = (long *)malloc(sizeof(long) * (n ? n : 1));
    long *fill = (long *)calloc(nc, sizeof(long));
    for (long i = 0; i < n; i++) ptr[ids[i] + 1]++;
    for (long c = 0; c < nc; c++) ptr[c + 1] += ptr[c];
    for (long i = 0; i < n; i++) idx[ptr[ids[i]] + fill[ids[i]]++] = i;
    free(fill);
    *ptr_out = ptr; *idx_out = idx;
}

/* computeCommunityComparisons (:50-307) at one thread.  C1, C2 are
 * relabelled in place as the reference does: C1's -1 entries become the
 * community count, which then grows by one (:63-87); C2's become N + 1
 * (:89-113).  Ids are 0-based when 0 occurs, else 1-based.  Pairs are
 * enumerated inside each community of C1 (:203-225) and of C2 (:228-251).
 * res: SameSame, SameDiff, DiffSame, nC1, nC2; dres: precision, recall,
 * F-score, Gini C1, Gini C2.  Returns -1 when an id is below -1.            */
int lvo_compare_communities(long *C1, long *C2, long n, long *res, double *dres) {
    long nC1 = -1, nC2 = -1;
    int z1 = 0, z2 = 0, m1 = 0;
    for (long i = 0; i < n; i++) {
        if (C1[i] < -1 || C2[i] < -1) return -1;
        if (C1[i] == 0) z1 = 1;
        if (C1[i] == -1) m1 = 1;
        if (C1[i] > nC1) nC1 = C1[i];
        if (C2[i] == -1) C2[i] = n + 1;
        if (C2[i] == 0) z2 = 1;
        if (C2[i] > nC2) nC2 = C2[i];
    }
    if (z1) nC1++;
    if (m1) {
        for (long i = 0; i < n; i++) if (C1[i] == -1) C1[i] = nC1;
        nC1++;
    }
    if (z2) nC2++;
    long *t1 = (long *)malloc(sizeof(long) * n), *t2 = (long *)malloc(sizeof(long) * n);
    for (long i = 0; i < n; i++) { t1[i] = C1[i] - (z1 ? 0 : 1); t2[i] = C2[i] - (z2 ? 0 : 1); }
    long *p1, *i1, *p2, *i2;
    group(n, t1, nC1, &p1, &i1);
    group(n, t2, nC2, &p2, &i2);
    long ss = 0, sd = 0, ds = 0, agree = 0;
    for (long c = 0; c < nC1; c++)
        for (long a = p1[c]; a < p1[c + 1]; a++)
            for (long b = a + 1; b < p1[c + 1]; b++) {
                if (C2[i1[a]] == C2[i1[b]]) ss++; else sd++;
            }
    for (long c = 0; c < nC2; c++)
        for (long a = p2[c]; a < p2[c + 1]; a++)
            for (long b = a + 1; b < p2[c + 1]; b++) {
                if (C1[i2[a]] == C1[i2[b]]) agree++; else ds++;
            }
    double precision = (double)ss / (double)(ss + ds);
    double recall = (double)ss / (double)(ss + sd);
    long *s1 = (long *)malloc(sizeof(long) * nC1), *s2 = (long *)malloc(sizeof(long) * nC2);
    for (long c = 0; c < nC1; c++) s1[c] = p1[c + 1] - p1[c];
    for (long c = 0; c < nC2; c++) s2[c] = p2[c + 1] - p2[c];
    res[0] = ss; res[1] = sd; res[2] = ds; res[3] = nC1; res[4] = nC2;
    dres[0] = precision; dres[1] = recall;
    dres[2] = 2 * ((precision * recall) / (precision + recall));
    dres[3] = lvo_gini(s1, (int)nC1);
    dres[4] = lvo_gini(s2, (int)nC2);
    free(t1); free(t2); free(p1); free(i1); free(p2); free(i2); free(s1); free(s2);
    return 0;
}

void lvo_free(void *p) { free(p); }

/* Q of a final assignment over the original graph.  The reference's
 * computeModularity (Utility/utilityClusterComparisonMetrics.cpp:409-411) is an
 * unimplemented stub; this restates the formula its sweeps use
 * (parallelLouvainWithColoring.cpp:226-249) with per-community degree sums:
 * e_xx = sum_i sum_{j: C[t]==C[i]} w,  a2_x = sum_c (sum_{i in c} k_i)^2.
 * Vertices with C < 0 contribute nothing.                                     */
double lvo_modularity(long nv, const long *ptr, const long *tail, const double *w,
                      const long *C) {
    double *vDeg = (double *)malloc(sizeof(double) * (nv ? nv : 1));
    double c = lvo_vertex_degrees(nv, ptr, w, vDeg);
    long maxc = -1;
    for (long i = 0; i < nv; i++) if (C[i] > maxc) maxc = C[i];
    double *cd = (double *)calloc(maxc + 2, sizeof(double));
    double e_xx = 0, a2_x = 0;
    for (long i = 0; i < nv; i++) {
        if (C[i] < 0) continue;
        cd[C[i]] += vDeg[i];
        double s = 0;
        for (long j = ptr[i]; j < ptr[i + 1]; j++)
            if (C[tail[j]] == C[i]) s += w[j];
        e_xx += s;
    }
    for (long k = 0; k <= maxc; k++) a2_x += cd[k] * cd[k];
    free(vDeg); free(cd);
    return e_xx * c - a2_x * c * c;
}

/* ------------------------------------------------------------------------ */
/* Per-phase record of a multiphase run (what the reference prints per phase). */
typedef struct {
    long nv, nnz;         /* level graph */
    int colored;          /* 1 = colour sweep, 0 = Jacobi sweep */
    int recolored;        /* colouring computed for this level (else stale) */
    int num_colors;
    int iterations;
    double mod;           /* value returned by the phase */
    long clusters;        /* after renumbering */
} lvo_phase;

typedef struct {
    int phases;           /* reference's `phase` counter at exit */
    int total_iterations;
    long final_clusters;
    double final_mod;     /* printed "Final modularity" = prevMod at exit */
    int nrec;             /* entries filled in rec[] */
} lvo_summary;

static void free_graph(long *ptr, long *tail, double *w, int owned) {
    if (owned) { free(ptr); free(tail); free(w); }
}

/* Coloring/runMultiPhaseColoring.cpp:51-238 at one thread, coloring = 1, 2
 * or 3 (2: lvo_vbase after the distance-1 colouring, :67-73, :180-186;
 * 3: lvo_color_mhash with two hashes and max(1, numColors / 4) iterations,
 * :76-86, :187-196).
 * Later phases recolour only when NV > minGraphSize and still colouring
 * (:173); otherwise the first NV entries of the previous colouring are reused
 * with the previous colour count (:61-66,113-115).  The first colour phase
 * that fails to gain switches to Jacobi phases on the same graph (:199-206).
 * C_orig is composed after every phase, before the gain test (:128-144).     */
/* Vertices of the last multiphase run for which no colour qualified in a
 * coloring = 2 recolouring (where type 0 of the reference is undefined). */
static long vbase_stuck_total = 0;

long lvo_last_vbase_stuck(void) { return vbase_stuck_total; }

static int color_for(int coloring, int numColors, long nv, const long *ptr, const long *tail,
                     int *colors) {
    if (coloring == 3) {
        int nItrs = numColors / 4;
        if (nItrs <= 0) nItrs = 1;
        return lvo_color_mhash(nv, ptr, tail, 2, nItrs, colors);
    }
    for (long i = 0; i < nv; i++) colors[i] = -1;
    int mc = lvo_color_greedy(nv, ptr, tail, colors);
    /* coloring = 2 balances the colouring (runMultiPhaseColoring.cpp:67-73) */
    if (coloring == 2 && mc >= 0) lvo_vbase(nv, ptr, tail, colors, mc + 1, 0, &vbase_stuck_total);
    return mc;
}

int lvo_run_multiphase_coloring(long nv, const long *ptr0, const long *tail0,
                                const double *w0, long *C_orig, int coloring, int numColors,
                                long minGraphSize, double threshold, double C_threshold,
                                lvo_summary *sum, lvo_phase *rec, int rec_cap) {
    long *ptr = (long *)ptr0, *tail = (long *)tail0;
    double *w = (double *)w0;
    int owned = 0;
    long NV = nv, gnv = nv;
    vbase_stuck_total = 0;
    int *colors = (int *)malloc(sizeof(int) * (nv ? nv : 1));
    int nColors = color_for(coloring, numColors, gnv, ptr, tail, colors);
    if (nColors == -2) { free(colors); return -1; }
    nColors += 1;
    int recolored = 1;
    double prevMod = -1, currMod = -1;
    long phase = 1;
    long *C = (long *)malloc(sizeof(long) * (nv ? nv : 1));
    for (long i = 0; i < nv; i++) C[i] = -1;
    int nonColor = 0, totItr = 0, nrec = 0;
    long numClusters = 0;
    while (1) {
        prevMod = currMod;
        int itr = 0;
        int usedColor = !nonColor;
        if (!nonColor) {
            currMod = lvo_coloring_phase(gnv, ptr, tail, w, C, colors, nColors, currMod,
                                         C_threshold, &itr, NULL, 0);
        } else {
            currMod = lvo_basic_phase(gnv, ptr, tail, w, C, currMod, threshold, &itr, NULL, 0);
        }
        totItr += itr;
        numClusters = lvo_renumber(C, gnv);
        if (rec && nrec < rec_cap) {
            lvo_phase *r = &rec[nrec];
            r->nv = gnv; r->nnz = ptr[gnv]; r->colored = usedColor;
            r->recolored = usedColor ? recolored : 0;
            r->num_colors = usedColor ? nColors : 0;
            r->iterations = itr; r->mod = currMod; r->clusters = numClusters;
        }
        nrec++;
        if (phase == 1) {
            for (long i = 0; i < NV; i++) C_orig[i] = C[i];
        } else {
            for (long i = 0; i < NV; i++)
                if (C_orig[i] >= 0) C_orig[i] = C[C_orig[i]];
        }
        if ((phase > 200) || (totItr > 10000)) break;
        if ((currMod - prevMod) > threshold) {
            long *np_, *nt_; double *nw_; long ne_;
            lvo_build_next_level(gnv, ptr, tail, w, C, numClusters, &np_, &nt_, &nw_, &ne_);
            free_graph(ptr, tail, w, owned);
            ptr = np_; tail = nt_; w = nw_; owned = 1;
            gnv = numClusters;
            free(C);
            C = (long *)malloc(sizeof(long) * (gnv ? gnv : 1));
            for (long i = 0; i < gnv; i++) C[i] = -1;
            phase++;
            recolored = 0;
            if ((gnv > minGraphSize) && !nonColor) {
                int mc = color_for(coloring, numColors, gnv, ptr, tail, colors);
                if (mc == -2) { free(colors); free(C); free_graph(ptr, tail, w, owned); return -1; }
                nColors = mc + 1;
                recolored = 1;
            }
        } else {
            if (!nonColor) nonColor = 1;
            else break;
        }
    }
    sum->phases = (int)phase;
    sum->total_iterations = totItr;
    sum->final_clusters = numClusters;
    sum->final_mod = prevMod;
    sum->nrec = nrec;
    free(C); free(colors);
    free_graph(ptr, tail, w, owned);
    return 0;
}

/* BasicCommunitiesDetection/runMultiPhaseBasic.cpp:52-170 (basicOpt 0,
 * threadsOpt 1: parallelLouvianMethod every phase, cap totItr > 100000).      */
int lvo_run_multiphase_basic(long nv, const long *ptr0, const long *tail0,
                             const double *w0, long *C_orig, double threshold,
                             lvo_summary *sum, lvo_phase *rec, int rec_cap) {
    long *ptr = (long *)ptr0, *tail = (long *)tail0;
    double *w = (double *)w0;
    int owned = 0;
    long NV = nv, gnv = nv;
    double prevMod = -1, currMod = -1;
    long phase = 1;
    long *C = (long *)malloc(sizeof(long) * (nv ? nv : 1));
    for (long i = 0; i < nv; i++) C[i] = -1;
    int totItr = 0, nrec = 0;
    long numClusters = 0;
    while (1) {
        prevMod = currMod;
        int itr = 0;
        currMod = lvo_basic_phase(gnv, ptr, tail, w, C, currMod, threshold, &itr, NULL, 0);
        totItr += itr;
        numClusters = lvo_renumber(C, gnv);
        if (rec && nrec < rec_cap) {
            lvo_phase *r = &rec[nrec];
            r->nv = gnv; r->nnz = ptr[gnv]; r->colored = 0; r->recolored = 0;
            r->num_colors = 0; r->iterations = itr; r->mod = currMod; r->clusters = numClusters;
        }
        nrec++;
        if (phase == 1) {
            for (long i = 0; i < NV; i++) C_orig[i] = C[i];
        } else {
            for (long i = 0; i < NV; i++)
                if (C_orig[i] >= 0) C_orig[i] = C[C_orig[i]];
        }
        if ((phase > 200) || (totItr > 100000)) break;
        if ((currMod - prevMod) > threshold) {
            long *np_, *nt_; double *nw_; long ne_;
            lvo_build_next_level(gnv, ptr, tail, w, C, numClusters, &np_, &nt_, &nw_, &ne_);
            free_graph(ptr, tail, w, owned);
            ptr = np_; tail = nt_; w = nw_; owned = 1;
            gnv = numClusters;
            free(C);
            C = (long *)malloc(sizeof(long) * (gnv ? gnv : 1));
            for (long i = 0; i < gnv; i++) C[i] = -1;
            phase++;
        } else {
            break;
        }
    }
    sum->phases = (int)phase;
    sum->total_iterations = totItr;
    sum->final_clusters = numClusters;
    sum->final_mod = prevMod;
    sum->nrec = nrec;
    free(C);
    free_graph(ptr, tail, w, owned);
    return 0;
}
