"""Seeded synthetic graphs and Grappolo's binary graph format.

Every generator returns a :class:`CSRGraph` in the layout Grappolo's loaders
produce (``DefineStructure/defs.h:85-92``): ``ptr`` int64[NV+1] row offsets,
``tail`` int64[nnz] column ids and ``weight`` float64[nnz], undirected graphs
stored twice (once per direction), rows sorted by tail, no duplicate entries.

The generators stand in for the inputs the reference is run on (there is no
dataset in the reference tree); each one names its shape, sizes and seed.
"""
from __future__ import annotations

import dataclasses
import struct

import numpy as np


@dataclasses.dataclass
class CSRGraph:
    ptr: np.ndarray      # int64[NV+1]
    tail: np.ndarray     # int64[nnz]
    weight: np.ndarray   # float64[nnz]

    @property
    def num_vertices(self) -> int:
        return int(self.ptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.tail.shape[0])

    @property
    def num_edges(self) -> int:
        """Grappolo's ``numEdges``: undirected edges, self-loops counted once."""
        nv = self.num_vertices
        heads = np.repeat(np.arange(nv, dtype=np.int64), np.diff(self.ptr))
        loops = int(np.count_nonzero(heads == self.tail))
        return (self.nnz - loops) // 2 + loops

    def heads(self) -> np.ndarray:
        return np.repeat(np.arange(self.num_vertices, dtype=np.int64), np.diff(self.ptr))


def csr_from_undirected(nv: int, u: np.ndarray, v: np.ndarray,
                        w: np.ndarray | None = None) -> CSRGraph:
    """Symmetrise an undirected edge list (u, v, w) into a deduplicated CSR.

    Self-loops are dropped. When a pair appears more than once the first
    occurrence's weight is kept, so each undirected edge has one weight that is
    stored in both directions.
    """
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    if w is None:
        w = np.ones(u.shape[0], dtype=np.float64)
    keep = u != v
    u, v, w = u[keep], v[keep], np.asarray(w, dtype=np.float64)[keep]
    lo = np.minimum(u, v)
    hi = np.maximum(u, v)
    key = lo * nv + hi
    _, first = np.unique(key, return_index=True)
    lo, hi, w = lo[first], hi[first], w[first]
    src = np.concatenate([lo, hi])
    dst = np.concatenate([hi, lo])
    ww = np.concatenate([w, w])
    order = np.lexsort((dst, src))
    src, dst, ww = src[order], dst[order], ww[order]
    ptr = np.zeros(nv + 1, dtype=np.int64)
    np.cumsum(np.bincount(src, minlength=nv), out=ptr[1:])
    return CSRGraph(ptr, dst.astype(np.int64), ww.astype(np.float64))


def planted_partition(num_blocks: int = 1000, block_size: int = 100,
                      intra_degree: float = 12.0, inter_degree: float = 4.0,
                      seed: int = 1) -> CSRGraph:
    """Planted-partition graph with equal blocks and unit weights.

    Inside a block every pair is an edge with probability
    ``intra_degree / (block_size - 1)``; on top of that
    ``inter_degree * NV / 2`` edges join uniform random endpoints in different
    blocks. Default: 100,000 vertices in 1,000 blocks of 100, intra degree 12,
    inter degree 4 (the plain-Louvain parity workload).
    """
    rng = np.random.default_rng(seed)
    nv = num_blocks * block_size
    p = intra_degree / (block_size - 1)
    iu, ju = np.triu_indices(block_size, k=1)
    pick = rng.random((num_blocks, iu.shape[0])) < p
    blk, pair = np.nonzero(pick)
    u_in = blk * block_size + iu[pair]
    v_in = blk * block_size + ju[pair]
    m_out = int(round(inter_degree * nv / 2))
    uo = rng.integers(0, nv, size=m_out, dtype=np.int64)
    vo = rng.integers(0, nv, size=m_out, dtype=np.int64)
    cross = (uo // block_size) != (vo // block_size)
    u = np.concatenate([u_in, uo[cross]])
    v = np.concatenate([v_in, vo[cross]])
    return csr_from_undirected(nv, u, v)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
         c: float = 0.19, seed: int = 1, weighted: bool = True) -> CSRGraph:
    """R-MAT graph (Chakrabarti et al.) on 2**scale vertices.

    ``edge_factor * 2**scale`` edges are drawn by recursive quadrant choice with
    probabilities (a, b, c, 1-a-b-c); the result is symmetrised with self-loops
    and duplicates removed. Weights are uniform in (0, 1] when ``weighted``.
    Vertex ids are not permuted, so low ids are the hubs.
    """
    rng = np.random.default_rng(seed)
    nv = 1 << scale
    m = edge_factor * nv
    u = np.zeros(m, dtype=np.int64)
    v = np.zeros(m, dtype=np.int64)
    ab, abc = a + b, a + b + c
    for _ in range(scale):
        r = rng.random(m)
        u = (u << 1) | (r >= ab)
        v = (v << 1) | (((r >= a) & (r < ab)) | (r >= abc))
    w = (1.0 - rng.random(m)) if weighted else None
    return csr_from_undirected(nv, u, v, w)


def random_weights(g: CSRGraph, seed: int = 7) -> CSRGraph:
    """Same topology, FP64 weights uniform in (0, 1], symmetric per edge."""
    rng = np.random.default_rng(seed)
    heads = g.heads()
    lo = np.minimum(heads, g.tail)
    hi = np.maximum(heads, g.tail)
    key = lo * g.num_vertices + hi
    uniq, inv = np.unique(key, return_inverse=True)
    wu = 1.0 - rng.random(uniq.shape[0])
    return CSRGraph(g.ptr.copy(), g.tail.copy(), wu[inv].astype(np.float64))


def from_edges(nv: int, edges, weights=None, keep_self_loops: bool = True) -> CSRGraph:
    """Small hand-built graphs: undirected (u, v[, w]) list, self-loops kept once."""
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    w = np.ones(e.shape[0]) if weights is None else np.asarray(weights, dtype=np.float64)
    loops = e[:, 0] == e[:, 1]
    g = csr_from_undirected(nv, e[~loops, 0], e[~loops, 1], w[~loops])
    if keep_self_loops and loops.any():
        heads = np.concatenate([g.heads(), e[loops, 0]])
        tails = np.concatenate([g.tail, e[loops, 1]])
        ws = np.concatenate([g.weight, w[loops]])
        order = np.lexsort((tails, heads))
        ptr = np.zeros(nv + 1, dtype=np.int64)
        np.cumsum(np.bincount(heads, minlength=nv), out=ptr[1:])
        g = CSRGraph(ptr, tails[order], ws[order])
    return g


def load_metis(path: str) -> CSRGraph:
    """Unweighted METIS adjacency file (1-based neighbour lists), as in karate.graph."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines() if not ln.startswith('%')]
    nv = int(lines[0].split()[0])
    heads, tails = [], []
    for i in range(nv):
        toks = lines[1 + i].split() if 1 + i < len(lines) else []
        for t in toks:
            heads.append(i)
            tails.append(int(t) - 1)
    heads = np.asarray(heads, dtype=np.int64)
    tails = np.asarray(tails, dtype=np.int64)
    order = np.lexsort((tails, heads))
    ptr = np.zeros(nv + 1, dtype=np.int64)
    np.cumsum(np.bincount(heads, minlength=nv), out=ptr[1:])
    return CSRGraph(ptr, tails[order], np.ones(heads.shape[0]))


# Grappolo binary format (InputsOutput/loadBinary.cpp:6-48, writeBinary.cpp:2-29):
# int64 NV, int64 NE, int64 weighted, int64[NV+1] offsets, then 2*NE records of
# {int64 head, int64 tail, float64 weight}.
_EDGE = np.dtype([('head', '<i8'), ('tail', '<i8'), ('weight', '<f8')])


def write_binary(g: CSRGraph, path: str, weighted: int = 1) -> None:
    rec = np.empty(g.nnz, dtype=_EDGE)
    rec['head'] = g.heads()
    rec['tail'] = g.tail
    rec['weight'] = g.weight
    with open(path, 'wb') as f:
        f.write(struct.pack('<qqq', g.num_vertices, g.nnz // 2, weighted))
        f.write(g.ptr.astype('<i8').tobytes())
        f.write(rec.tobytes())


def read_binary(path: str) -> CSRGraph:
    with open(path, 'rb') as f:
        nv, ne, _ = struct.unpack('<qqq', f.read(24))
        ptr = np.frombuffer(f.read(8 * (nv + 1)), dtype='<i8').copy()
        rec = np.frombuffer(f.read(_EDGE.itemsize * 2 * ne), dtype=_EDGE)
    return CSRGraph(ptr, rec['tail'].astype(np.int64), rec['weight'].astype(np.float64))


def rmat_edges_device(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
                      c: float = 0.19, seed: int = 1, device='cuda'):
    """The raw R-MAT edge list, as an edge-list file would hold it: 2^scale
    vertices, edge_factor * 2^scale edges with their repeats and self-loops,
    weights uniform in (0, 1].  Returns device tensors (head int64, tail
    int64, weight float64), drawn from torch's device generator."""
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    m = edge_factor << scale
    u = torch.zeros(m, dtype=torch.int64, device=device)
    v = torch.zeros(m, dtype=torch.int64, device=device)
    ab, abc = a + b, a + b + c
    for _ in range(scale):
        r = torch.rand(m, generator=gen, device=device)
        u = (u << 1) | (r >= ab).to(torch.int64)
        v = (v << 1) | (((r >= a) & (r < ab)) | (r >= abc)).to(torch.int64)
        del r
    w = 1.0 - torch.rand(m, generator=gen, device=device, dtype=torch.float64)
    return u, v, w


def rmat_edges(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
               c: float = 0.19, seed: int = 1):
    """Host (numpy) counterpart of :func:`rmat_edges_device` (a different
    stream of random numbers): raw (head, tail, weight) arrays."""
    rng = np.random.default_rng(seed)
    m = edge_factor << scale
    u = np.zeros(m, dtype=np.int64)
    v = np.zeros(m, dtype=np.int64)
    ab, abc = a + b, a + b + c
    for _ in range(scale):
        r = rng.random(m)
        u = (u << 1) | (r >= ab)
        v = (v << 1) | (((r >= a) & (r < ab)) | (r >= abc))
    return u, v, 1.0 - rng.random(m)


def rmat_device(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
                c: float = 0.19, seed: int = 1, device='cuda', weighted: bool = True):
    """R-MAT graph built directly in device memory with torch (large inputs).

    Same construction as :func:`rmat` (recursive quadrant choice, symmetrised,
    self-loops and duplicates removed, weights uniform in (0, 1]) but drawn from
    torch's device generator, so the graph differs from the numpy one of the
    same seed.  Returns device tensors (ptr int64[NV+1], tail int32[nnz],
    weight float64[nnz]).
    """
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    nv = 1 << scale
    m = edge_factor * nv
    u = torch.zeros(m, dtype=torch.int64, device=device)
    v = torch.zeros(m, dtype=torch.int64, device=device)
    ab, abc = a + b, a + b + c
    for _ in range(scale):
        r = torch.rand(m, generator=gen, device=device)
        u = (u << 1) | (r >= ab).to(torch.int64)
        v = (v << 1) | (((r >= a) & (r < ab)) | (r >= abc)).to(torch.int64)
        del r
    keep = u != v
    u, v = u[keep], v[keep]
    key = torch.minimum(u, v) * nv + torch.maximum(u, v)
    del u, v, keep
    key = torch.unique(key)
    lo, hi = key // nv, key % nv
    del key
    if weighted:
        w = 1.0 - torch.rand(lo.numel(), generator=gen, device=device, dtype=torch.float64)
    else:
        w = torch.ones(lo.numel(), device=device, dtype=torch.float64)
    src = torch.cat([lo, hi])
    dst = torch.cat([hi, lo])
    ww = torch.cat([w, w])
    del lo, hi, w
    order = torch.argsort(src * nv + dst)
    src, dst, ww = src[order], dst[order], ww[order]
    del order
    ptr = torch.zeros(nv + 1, dtype=torch.int64, device=device)
    ptr[1:] = torch.cumsum(torch.bincount(src, minlength=nv), 0)
    return ptr, dst.to(torch.int32), ww


def planted_partition_mixed(nv: int, block_size: int, mu: float, mean_degree: float,
                            seed: int = 1) -> CSRGraph:
    """Planted partition with mixing fraction `mu` and expected degree `mean_degree`.

    Vertices fall into consecutive blocks of `block_size` (the last may be
    smaller).  Each block gets (1-mu)*d*|B|/2 uniform intra pairs and the graph
    mu*d*NV/2 uniform pairs between different blocks; duplicates and
    self-loops are dropped.  Unit weights.  This is the graph family of the
    batched workload (sizes, block sizes, mu and degree drawn per graph).
    """
    rng = np.random.default_rng(seed)
    block = np.arange(nv, dtype=np.int64) // block_size
    starts = np.arange(0, nv, block_size, dtype=np.int64)
    sizes = np.minimum(block_size, nv - starts)
    m_in = rng.poisson((1.0 - mu) * mean_degree * sizes / 2.0)
    bidx = np.repeat(np.arange(starts.shape[0]), m_in)
    u = starts[bidx] + (rng.random(bidx.shape[0]) * sizes[bidx]).astype(np.int64)
    v = starts[bidx] + (rng.random(bidx.shape[0]) * sizes[bidx]).astype(np.int64)
    m_out = int(rng.poisson(mu * mean_degree * nv / 2.0))
    uo = rng.integers(0, nv, size=m_out, dtype=np.int64)
    vo = rng.integers(0, nv, size=m_out, dtype=np.int64)
    cross = block[uo] != block[vo]
    return csr_from_undirected(nv, np.concatenate([u, uo[cross]]), np.concatenate([v, vo[cross]]))


def _powerlaw_ints(rng, n, exponent, lo, hi):
    """n integers from a discrete power law p(k) ~ k^-exponent on [lo, hi]."""
    a = 1.0 - exponent
    r = rng.random(n)
    x = ((hi ** a - lo ** a) * r + lo ** a) ** (1.0 / a)
    return np.clip(np.floor(x).astype(np.int64), lo, hi)


def planted_powerlaw(nv: int, degree_exp: float = 2.5, mean_degree: float = 20.0,
                     max_degree: int = 5000, community_exp: float = 1.5, community_min: int = 20,
                     community_max: int = 20000, mu: float = 0.3, seed: int = 1) -> CSRGraph:
    """Planted power-law community graph (LFR-style benchmark shape).

    Community sizes follow a power law (exponent `community_exp`, sizes in
    [community_min, community_max]); degrees a power law (exponent
    `degree_exp`, at most `max_degree`) whose lower cut-off is chosen to give
    `mean_degree`.  A vertex keeps a fraction 1-mu of its stubs inside its
    community and mu outside; stubs are paired at random (configuration model)
    within communities and across the graph, then duplicates, self-loops and
    intra-community pairs among the outside stubs are dropped.  Unit weights.
    """
    rng = np.random.default_rng(seed)
    sizes = []
    total = 0
    while total < nv:
        s = int(_powerlaw_ints(rng, 1, community_exp, community_min, community_max)[0])
        s = min(s, nv - total)
        sizes.append(s)
        total += s
    sizes = np.asarray(sizes, dtype=np.int64)
    comm = np.repeat(np.arange(sizes.shape[0]), sizes)
    rng.shuffle(comm)
    # lower degree cut-off giving the requested mean
    lo = 1
    for cand in range(1, 200):
        d = _powerlaw_ints(np.random.default_rng(seed + 1), 200000, degree_exp, cand, max_degree)
        if d.mean() >= mean_degree:
            lo = cand
            break
    deg = _powerlaw_ints(rng, nv, degree_exp, lo, max_degree)
    csize = sizes[comm]
    k_in = np.minimum(np.rint((1.0 - mu) * deg).astype(np.int64), csize - 1)
    k_out = deg - k_in
    # intra-community stubs: sort by (community, random) and pair neighbours
    su = np.repeat(np.arange(nv, dtype=np.int64), k_in)
    key = comm[su].astype(np.float64) + rng.random(su.shape[0])
    su = su[np.argsort(key, kind='stable')]
    cs = comm[su]
    even = su.shape[0] - (su.shape[0] % 2)
    pu, pv = su[0:even:2], su[1:even:2]
    same = cs[0:even:2] == cs[1:even:2]
    # outside stubs: global random pairing, intra pairs dropped
    so = np.repeat(np.arange(nv, dtype=np.int64), k_out)
    rng.shuffle(so)
    even2 = so.shape[0] - (so.shape[0] % 2)
    qu, qv = so[0:even2:2], so[1:even2:2]
    cross = comm[qu] != comm[qv]
    return csr_from_undirected(nv, np.concatenate([pu[same], qu[cross]]),
                               np.concatenate([pv[same], qv[cross]]))


def batch_specs(num_graphs: int = 4096, seed: int = 3, nv_range=(500, 200000),
                block_range=(20, 2000), mu_range=(0.1, 0.6), degree_range=(6.0, 32.0)):
    """Per-graph parameters of the batched workload: vertex counts and block
    sizes log-uniform, mixing fraction and mean degree uniform.  Returns an
    (num_graphs, 4) float64 array of (nv, block_size, mu, mean_degree)."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(nv_range[0]), np.log(nv_range[1])
    nv = np.floor(np.exp(rng.uniform(lo, hi, num_graphs))).astype(np.int64)
    blo, bhi = np.log(block_range[0]), np.log(block_range[1])
    bs = np.floor(np.exp(rng.uniform(blo, bhi, num_graphs))).astype(np.int64)
    bs = np.minimum(bs, nv)
    mu = rng.uniform(mu_range[0], mu_range[1], num_graphs)
    deg = rng.uniform(degree_range[0], degree_range[1], num_graphs)
    return np.stack([nv, bs, mu, deg], axis=1).astype(np.float64)


def planted_batch_device(specs, seed: int = 3, device='cuda', group_pairs: int = 200_000_000):
    """The graphs of `specs` (rows of :func:`batch_specs`) as one device CSR laid
    end to end, built with torch on the device: the construction of
    :func:`planted_partition_mixed` graph by graph (Poisson intra-block pair
    counts, uniform inter-block pairs, duplicates and self-loops dropped, unit
    weights), drawn from torch's generator, so a graph differs from the numpy
    one.  Graphs are built in groups of about `group_pairs` candidate pairs to
    bound the scratch memory.  Returns (vertex_offsets int64 numpy[G+1],
    ptr int64[NV+1], tail int32[nnz], weight float64[nnz]) on the device."""
    import torch
    specs = np.asarray(specs, dtype=np.float64)
    G = specs.shape[0]
    nv = specs[:, 0].astype(np.int64)
    bs = specs[:, 1].astype(np.int64)
    mu, deg = specs[:, 2], specs[:, 3]
    voff = np.zeros(G + 1, dtype=np.int64)
    np.cumsum(nv, out=voff[1:])
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    expect = (deg * nv / 2.0).astype(np.int64) + 1  # candidate pairs per graph
    ptr_parts, tail_parts = [], []
    g0 = 0
    while g0 < G:
        g1 = g0 + 1
        tot = expect[g0]
        while g1 < G and tot + expect[g1] <= group_pairs:
            tot += expect[g1]
            g1 += 1
        base = voff[g0]
        n_loc = int(voff[g1] - base)
        # blocks of the group (host), intra-block pair counts per block
        bstart, bsize, m_in = [], [], []
        for g in range(g0, g1):
            st = np.arange(0, nv[g], bs[g], dtype=np.int64)
            sz = np.minimum(bs[g], nv[g] - st)
            bstart.append(st + (voff[g] - base))
            bsize.append(sz)
            m_in.append(rng.poisson((1.0 - mu[g]) * deg[g] * sz / 2.0))
        bstart = torch.from_numpy(np.concatenate(bstart)).to(device)
        bsize = torch.from_numpy(np.concatenate(bsize)).to(device)
        m_in = torch.from_numpy(np.concatenate(m_in).astype(np.int64)).to(device)
        bid = torch.repeat_interleave(torch.arange(bstart.numel(), device=device), m_in)
        u = bstart[bid] + (torch.rand(bid.numel(), generator=gen, device=device,
                                      dtype=torch.float64) * bsize[bid]).to(torch.int64)
        v = bstart[bid] + (torch.rand(bid.numel(), generator=gen, device=device,
                                      dtype=torch.float64) * bsize[bid]).to(torch.int64)
        del bid
        # inter-block pairs per graph
        m_out = torch.from_numpy(rng.poisson(mu[g0:g1] * deg[g0:g1] * nv[g0:g1] / 2.0)
                                 .astype(np.int64)).to(device)
        gst = torch.from_numpy(voff[g0:g1] - base).to(device)
        gnv = torch.from_numpy(nv[g0:g1]).to(device)
        gbs = torch.from_numpy(bs[g0:g1]).to(device)
        gi = torch.repeat_interleave(torch.arange(g1 - g0, device=device), m_out)
        uo = (torch.rand(gi.numel(), generator=gen, device=device, dtype=torch.float64)
              * gnv[gi]).to(torch.int64)
        vo = (torch.rand(gi.numel(), generator=gen, device=device, dtype=torch.float64)
              * gnv[gi]).to(torch.int64)
        cross = (uo // gbs[gi]) != (vo // gbs[gi])
        uo = (uo + gst[gi])[cross]
        vo = (vo + gst[gi])[cross]
        del gi, cross
        u = torch.cat([u, uo])
        v = torch.cat([v, vo])
        del uo, vo
        keep = u != v
        key = torch.minimum(u, v)[keep] * n_loc + torch.maximum(u, v)[keep]
        del u, v, keep
        key = torch.unique(key)
        lo, hi = key // n_loc, key % n_loc
        del key
        src = torch.cat([lo, hi])
        dst = torch.cat([hi, lo])
        del lo, hi
        order = torch.argsort(src * n_loc + dst)
        src, dst = src[order], dst[order]
        del order
        cnt = torch.bincount(src, minlength=n_loc)
        del src
        ptr_parts.append(cnt)
        tail_parts.append((dst + base).to(torch.int32))
        del dst
        g0 = g1
    cnt = torch.cat(ptr_parts)
    del ptr_parts
    ptr = torch.zeros(voff[-1] + 1, dtype=torch.int64, device=device)
    ptr[1:] = torch.cumsum(cnt, 0)
    del cnt
    tail = torch.cat(tail_parts)
    del tail_parts
    w = torch.ones(tail.numel(), dtype=torch.float64, device=device)
    return voff, ptr, tail, w


def rmat_device_lean(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
                     c: float = 0.19, seed: int = 1, device='cuda', chunk: int = 1 << 27):
    """R-MAT in device memory for scales whose edge lists are tens of GB
    (scale 26 and up): the construction of :func:`rmat_device` with bounded
    scratch.  Edges are drawn in chunks into one key array, deduplicated by
    one sort, and the CSR is filled by counting (rows sorted by tail) instead
    of sorting the symmetric list.  Weights are U(0,1] from a hash of the
    undirected edge, so both directions carry the same weight.  Returns
    (ptr int64[NV+1], tail int32[nnz], weight float64[nnz]) on the device."""
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    nv = 1 << scale
    m = edge_factor * nv
    keys = torch.empty(m, dtype=torch.int64, device=device)
    n = 0
    ab, abc = a + b, a + b + c
    for s0 in range(0, m, chunk):
        k = min(chunk, m - s0)
        u = torch.zeros(k, dtype=torch.int64, device=device)
        v = torch.zeros(k, dtype=torch.int64, device=device)
        for _ in range(scale):
            r = torch.rand(k, generator=gen, device=device)
            u = (u << 1) | (r >= ab).to(torch.int64)
            v = (v << 1) | (((r >= a) & (r < ab)) | (r >= abc)).to(torch.int64)
            del r
        keep = u != v
        kk = torch.minimum(u, v)[keep] * nv + torch.maximum(u, v)[keep]
        keys[n:n + kk.numel()] = kk
        n += kk.numel()
        del u, v, keep, kk
    keys = keys[:n]
    keys, _ = torch.sort(keys)
    keys = torch.unique_consecutive(keys)
    ne = keys.numel()
    lo = (keys // nv).to(torch.int32)
    hi = (keys % nv).to(torch.int32)
    # weight of each undirected edge: top 53 bits of a multiplicative hash
    h = keys * (-7046029254386353131)  # 0x9E3779B97F4A7C15 as int64, wraps
    del keys
    wu = 1.0 - ((h >> 11) & ((1 << 53) - 1)).to(torch.float64) * (2.0 ** -53)
    del h
    cnt_lo = torch.bincount(lo, minlength=nv)
    cnt_hi = torch.bincount(hi, minlength=nv)
    ptr = torch.zeros(nv + 1, dtype=torch.int64, device=device)
    ptr[1:] = torch.cumsum(cnt_lo + cnt_hi, 0)
    nnz = int(ptr[-1])
    tail = torch.empty(nnz, dtype=torch.int32, device=device)
    w = torch.empty(nnz, dtype=torch.float64, device=device)
    # row r = [tails below r (edges (x, r), x ascending)] then [tails above r]
    first_lo = torch.zeros(nv + 1, dtype=torch.int64, device=device)
    first_lo[1:] = torch.cumsum(cnt_lo, 0)
    first_hi = torch.zeros(nv + 1, dtype=torch.int64, device=device)
    first_hi[1:] = torch.cumsum(cnt_hi, 0)
    # upper part: the key order is (lo, hi), so each lo's edges are a run
    for s0 in range(0, ne, chunk):
        i = torch.arange(s0, min(ne, s0 + chunk), device=device, dtype=torch.int64)
        r = lo[i].to(torch.int64)
        at = ptr[r] + cnt_hi[r] + (i - first_lo[r])
        tail[at] = hi[i]
        w[at] = wu[i]
        del i, r, at
    # lower part: a stable sort by hi keeps each hi's edges in ascending lo
    hs, perm = torch.sort(hi, stable=True)
    del hs
    for s0 in range(0, ne, chunk):
        kx = torch.arange(s0, min(ne, s0 + chunk), device=device, dtype=torch.int64)
        p = perm[kx]
        r = hi[p].to(torch.int64)
        at = ptr[r] + (kx - first_hi[r])
        tail[at] = lo[p]
        w[at] = wu[p]
        del kx, p, r, at
    del perm, lo, hi, wu, cnt_lo, cnt_hi, first_lo, first_hi
    return ptr, tail, w
