#!/usr/bin/env python
"""Benchmark: plain multiphase Louvain (distance-1 colouring) on an R-MAT graph.

Workload: R-MAT scale 24 (16.7M vertices, edge factor 16, a=.57 b=.19 c=.19),
symmetrised, self-loops and duplicates removed, FP64 weights uniform in (0,1],
seeded and generated on the device; coloring=1, threshold 1e-6, C_thresh 1e-4,
minGraphSize 1000 (the reference's runMultiPhaseColoring configuration).

A step is one full multiphase run (colouring, colour-class sweeps, modularity,
renumbering, coarsening, every phase) with the graph resident in HBM.  The
metric is local-move edges/s: CSR entries evaluated by the local-moving sweeps
over the whole run, divided by the run's device time.  The graph (several GB)
is larger than L2, so no flush is needed between steps.

--impl reference times Grappolo's own OpenMP code (oracle/_ref, compiled from
its sources with its shipped flags) on all host cores for the same metric,
one sweep iteration of phase 1 per step (a bounded sample of the workload).

Multi-GPU (torchrun): the single-graph path does not shard, so every rank runs
an independent replica (weak scaling); value = all ranks' edges / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'local-move edges/s'
UNIT = 'edges/s'


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=5)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', choices=['ours', 'reference'], default='ours')
    p.add_argument('--scale', type=int, default=24)
    p.add_argument('--mode', choices=['fast', 'verify', 'learned'], default='fast')
    p.add_argument('--no-e2e', action='store_true')
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--no-learned', action='store_true',
                   help='rmat workload: skip the learned-gate comparison runs')
    p.add_argument('--full-run-scale', type=int, default=20,
                   help='R-MAT scale of the reference full-run sample in cpu_baseline')
    p.add_argument('--profile-level', type=int, default=1,
                   help='1: time each class sweep (roofline); 2: time every launch by kind')
    p.add_argument('--workload', choices=['rmat', 'powerlaw', 'batch', 'csr', 'compare'],
                   default='rmat',
                   help='rmat: one R-MAT graph (default); batch: 4,096 planted-partition '
                        'graphs run as batches; csr: edge list to CSR (removeEdges, both '
                        'directions, rows sorted) of a raw R-MAT edge list; compare: '
                        'community-comparison metrics of two labellings of 2^scale vertices')
    p.add_argument('--powerlaw-vertices', type=int, default=4_000_000,
                   help='powerlaw workload: vertices of the planted power-law graph')
    p.add_argument('--gate-tau', type=float, default=None,
                   help='learned mode: keep threshold of the move gate (default: the trained one)')
    p.add_argument('--csr-sample-scale', type=int, default=16,
                   help='csr workload: R-MAT scale of the reference\'s CPU sample')
    p.add_argument('--batch-graphs', type=int, default=4096)
    p.add_argument('--batch-sample', type=int, default=24,
                   help='batch workload: graphs the reference runs for cpu_baseline')
    p.add_argument('--wave-pairs', type=float, default=3.5e8,
                   help='batch workload: expected undirected pairs per batched run')
    return p.parse_args()


def workload_config(args, nv, nnz, extra=None):
    kind = 'learned-gated' if args.mode == 'learned' else 'plain'
    if args.workload == 'powerlaw':
        cfg = {'workload': f'{kind} multiphase Louvain (coloring=1) on a planted power-law '
                           f'community graph of {nv} vertices',
               'graph': f'planted power-law, {nv} vertices, degree exponent 2.5 (mean 20, max '
                        f'5000), community-size exponent 1.5 (20 to 20000), mu 0.3, unit FP64 '
                        f'weights, seed 1 (host generator)',
               'num_vertices': nv, 'nnz': nnz, 'threshold': 1e-6, 'C_threshold': 1e-4,
               'minGraphSize': 1000, 'parallelism': f'replicas x{args.gpus}',
               'l2': 'inputs larger than L2 (no flush)'}
        if args.mode == 'learned':
            cfg['gate_tau'] = args.gate_tau
        if extra:
            cfg.update(extra)
        return cfg
    gen = ('bounded-scratch device builder, weights from an edge hash' if args.scale >= 26
           else 'device builder')
    cfg = {'workload': f'{kind} multiphase Louvain (coloring=1) on R-MAT scale {args.scale}',
           'graph': f'R-MAT scale {args.scale}, edge factor 16, a=0.57 b=0.19 c=0.19, '
                    f'symmetrised, dedup, no self-loops, FP64 weights U(0,1], seed 1 ({gen})',
           'num_vertices': nv, 'nnz': nnz, 'threshold': 1e-6, 'C_threshold': 1e-4,
           'minGraphSize': 1000, 'parallelism': f'replicas x{args.gpus}',
           'l2': 'inputs larger than L2 (no flush)'}
    if extra:
        cfg.update(extra)
    return cfg


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile('w+', suffix='.csv', delete=False)
        q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
        try:
            self.p = subprocess.Popen(['nvidia-smi', f'--query-gpu={q}', '--format=csv,noheader,nounits',
                                       '-i', str(index), '-lms', '200'], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(',') for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, r[5:9]):
                if val.lower() == 'active':
                    reasons.add(name)
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': mx,
                'reasons': sorted(reasons), 'samples': len(sm)}


def measured_peak():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            return float(json.load(f)['hbm_gbs']), 'measured'
    except (OSError, KeyError, ValueError):
        return 6650.0, 'fallback'


def profiled_traffic_ratio():
    """DRAM bytes per algorithmic byte of the sweep kernels, from the committed ncu summary."""
    path = os.path.join(ROOT, 'profiles', 'sweep_iteration_rmat24.txt')
    try:
        with open(path) as f:
            for line in f:
                if line.startswith('traffic_per_algorithmic_byte'):
                    return float(line.split('=')[1])
    except OSError:
        pass
    return None


def aggregate(seconds, edges, dist=None, device=None):
    """Whole-job figures over replicas: max time over ranks, edges summed."""
    if dist is None or not dist.is_initialized():
        return seconds, edges
    import torch
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    e = torch.tensor([edges], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t), float(e)


# --------------------------------------------------------------------- reference arm
def run_reference(args, rank):
    if rank != 0:
        return 0
    if args.workload == 'csr':
        return run_csr_reference(args)
    if args.workload == 'compare':
        return run_compare_reference(args)
    import numpy as np
    import torch
    from grappolo_b200 import graphs
    from oracle import Reference
    dev = torch.device('cuda:0') if torch.cuda.is_available() else torch.device('cpu')
    if args.workload == 'powerlaw':
        g = graphs.planted_powerlaw(args.powerlaw_vertices, seed=1)
    else:
        ptr, tail, w = graphs.rmat_device(args.scale, device=dev)
        g = graphs.CSRGraph(ptr.cpu().numpy(), tail.cpu().numpy().astype(np.int64),
                            w.cpu().numpy())
        del ptr, tail, w
    if dev.type == 'cuda':
        torch.cuda.empty_cache()
    cores = os.cpu_count() or 1
    R = Reference(fast=True)
    h = R.graph(g)
    col, mc, tcol = R.color_g(h, g.num_vertices, cores)
    vals = []
    for k in range(args.warmup + args.steps):
        _, _, itr, tt = R.coloring_phase_g(h, g.num_vertices, col, mc + 1, -1.0, float('inf'),
                                           cores)
        if k >= args.warmup:
            vals.append(g.nnz * itr / tt)
    R.free_graph(h)
    value = statistics.median(vals)
    sample = (f'phase-1 colour-class sweep iteration (+modularity) of the reference '
              f'algoLouvainWithDistOneColoring on the full graph, {cores} OpenMP threads, '
              f'-Ofast build; its own iteration timer; colouring ({mc + 1} colours, '
              f'{tcol:.2f} s) done once before')
    line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'impl': 'reference',
            'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': 1e3 * g.nnz / value, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': workload_config(args, g.num_vertices, g.nnz),
            'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': cores, 'kind': 'reference',
                             'sample': sample},
            'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)
    return 0


CSR_METRIC = 'CSR build input edges/s'
CSR_UNIT = 'edges/s'


def csr_config(args, nv, ne, nnz=None, extra=None):
    cfg = {'workload': f'edge list to CSR (removeEdges, every edge in both rows, rows sorted by '
                       f'tail) of a raw R-MAT scale {args.scale} edge list',
           'graph': f'R-MAT scale {args.scale}, edge factor 16, a=0.57 b=0.19 c=0.19, raw '
                    f'(repeats and self-loops kept), FP64 weights U(0,1], seed 1',
           'num_vertices': nv, 'num_input_edges': ne, 'nnz': nnz,
           'parallelism': f'replicas x{args.gpus}', 'l2': 'inputs larger than L2 (no flush)'}
    if extra:
        cfg.update(extra)
    return cfg


def csr_cpu_sample(scale):
    """The reference's removeEdges + SortEdgesUndirected + SortNodeEdgesByIndex
    (Utility/utilityFunctions.cpp:416-531; sequential code, one core) on a raw
    R-MAT edge list of the given scale.  Returns (edges/s, seconds, edges)."""
    from grappolo_b200 import graphs
    from oracle import Reference
    R = Reference(fast=True)
    h, t, w = graphs.rmat_edges(scale, seed=1)
    nv = 1 << scale
    t0 = time.perf_counter()
    rh, rt, rw, n = R.remove_edges(nv, h, t, w)
    ptrs, sh, st, sw = R.sort_edges_undirected(nv, rh[:n], rt[:n], rw[:n])
    R.sort_node_edges(nv, ptrs, sh, st, sw)
    dt = time.perf_counter() - t0
    return len(h) / dt, dt, len(h)


def csr_sample_text(scale, dt, ne):
    return (f'reference removeEdges + SortEdgesUndirected + SortNodeEdgesByIndex (sequential, '
            f'-Ofast build) on a raw R-MAT scale {scale} edge list ({ne} edges, {dt:.1f} s); '
            f'removeEdges walks a per-head list, so its time grows with the square of the '
            f'largest degree and larger samples do not finish in minutes')


def run_csr_reference(args):
    vals = []
    for k in range(args.warmup + args.steps):
        v, dt, ne = csr_cpu_sample(args.csr_sample_scale)
        if k >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    nv = 1 << args.scale
    line = {'metric': CSR_METRIC, 'value': value, 'unit': CSR_UNIT, 'impl': 'reference',
            'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': 1e3 * (16 << args.scale) / value, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'int64', 'data': 'synthetic',
            'config': csr_config(args, nv, 16 << args.scale),
            'cpu_baseline': {'value': value, 'unit': CSR_UNIT, 'cores': 1, 'kind': 'reference',
                             'sample': csr_sample_text(args.csr_sample_scale, dt, ne)},
            'e2e': {'value': value, 'unit': CSR_UNIT, 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)
    return 0


CMP_METRIC = 'labelled vertices compared/s'
CMP_UNIT = 'vertices/s'
CMP_BLOCK = 1000


def compare_labels(n, seed=7):
    """Truth: consecutive blocks of CMP_BLOCK vertices; output: the truth with
    20% of the vertices moved to random labels and 0.05% of either side -1."""
    import numpy as np
    rng = np.random.default_rng(seed)
    C1 = np.arange(n, dtype=np.int64) // CMP_BLOCK
    C2 = C1.copy()
    flip = rng.random(n) < 0.2
    C2[flip] = rng.integers(0, 2 * max(1, n // CMP_BLOCK), int(flip.sum()))
    C1[rng.integers(0, n, n // 2000)] = -1
    C2[rng.integers(0, n, n // 2000)] = -1
    return C1, C2


def compare_config(args, n):
    return {'workload': f'computeCommunityComparisons (pair counts, precision, recall, F-score, '
                        f'Gini) of two labellings of 2^{args.scale} vertices',
            'labels': f'truth: blocks of {CMP_BLOCK}; output: 20% of vertices relabelled at '
                      f'random, 0.05% of each side -1; seed 7',
            'num_vertices': n, 'parallelism': f'replicas x{args.gpus}',
            'l2': 'inputs larger than L2 (no flush)' if n >= (1 << 24) else 'inputs in L2'}


def compare_cpu_sample(scale):
    """The reference's computeCommunityComparisons on one sample of 2^scale
    vertices, at one thread: its pair loops sit in an `omp parallel for`
    nested inside an `omp parallel` region, so with T threads every thread
    runs every pair (T times the work, and counts T times too large).
    Returns (vertices/s, seconds, n, threads)."""
    from oracle import Reference
    n = 1 << scale
    C1, C2 = compare_labels(n)
    cores = 1
    R = Reference(fast=True)
    t0 = time.perf_counter()
    R.compare(C1, C2, nthreads=cores)
    dt = time.perf_counter() - t0
    return n / dt, dt, n, cores


def run_compare_reference(args):
    vals = []
    for k in range(args.warmup + args.steps):
        v, dt, n, cores = compare_cpu_sample(min(args.scale, 20))
        if k >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    line = {'metric': CMP_METRIC, 'value': value, 'unit': CMP_UNIT, 'impl': 'reference',
            'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': 1e3 * (1 << args.scale) / value, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'int64', 'data': 'synthetic',
            'config': compare_config(args, 1 << args.scale),
            'cpu_baseline': {'value': value, 'unit': CMP_UNIT, 'cores': cores,
                             'kind': 'reference',
                             'sample': f'reference computeCommunityComparisons, one thread (its '
                                       f'nested OpenMP regions repeat all work per thread), '
                                       f'-Ofast build, on {n} vertices ({dt:.2f} s)'},
            'e2e': {'value': value, 'unit': CMP_UNIT, 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_compare_workload(args, world, rank, local):
    """A step compares two device-resident labellings (glv_dev_compare_communities);
    e2e: glv_compare_communities from host arrays, relabelled arrays copied back."""
    import torch
    from grappolo_b200 import louvain, _lib
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    L = _lib.lib()
    n = 1 << args.scale
    C1, C2 = compare_labels(n)
    d1, d2 = torch.tensor(C1, device=dev), torch.tensor(C2, device=dev)
    w1, w2 = d1.clone(), d2.clone()
    stream = torch.cuda.current_stream().cuda_stream

    def step():
        w1.copy_(d1)  # the call relabels in place; every step starts from the inputs
        w2.copy_(d2)
        return louvain.compare_communities_device(w1, w2, stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    l0 = L.glv_kernel_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        st = step()
    ev1.record()
    torch.cuda.synchronize()
    launches = L.glv_kernel_launch_count() - l0
    if dist:
        dist.barrier()
    clk = clocks.stop()
    t = ev0.elapsed_time(ev1) * 1e-3
    t_max, n_all = aggregate(t, float(n * args.steps), dist, dev)
    # algorithmic bytes: both labellings read once (8 B each per vertex)
    alg = 16 * n
    peak, peak_kind = measured_peak()
    achieved = alg / (t / args.steps) / 1e9
    roofline = {'bound': 'hbm', 'kernel': 'the whole comparison (our kernels, the CUB radix sort '
                                          'and run-length encode), per step',
                'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                'peak_kind': peak_kind, 'traffic': None, 'algorithmic_bytes_per_launch': alg,
                'avg_launch_s': t / args.steps}
    e2e = None
    if not args.no_e2e:
        h1 = torch.from_numpy(C1).pin_memory()
        h2 = torch.from_numpy(C2).pin_memory()
        import numpy as np
        a, b = h1.numpy(), h2.numpy()

        def e2e_step():
            a[:] = C1
            b[:] = C2
            r = _lib.GlvComparison()
            import ctypes as ct
            lp = lambda x: ct.cast(x.data_ptr(), ct.POINTER(ct.c_long))  # noqa: E731
            _lib.check(L.glv_compare_communities(lp(h1), n, lp(h2), n, ct.byref(r)))
            return r

        e2e_step()
        e0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        et = time.perf_counter() - e0
        et, ee = aggregate(et, float(n * args.steps), dist, dev)
        e2e = {'value': ee / et, 'unit': CMP_UNIT, 'h2d_bytes_per_step': 16 * n,
               'd2h_bytes_per_step': 16 * n, 'seconds_per_step': et / args.steps,
               'note': 'timed on the host clock; includes resetting the pinned inputs'}
        del np
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cv, cdt, cn, cores = compare_cpu_sample(min(args.scale, 20))
        cpu = {'value': cv, 'unit': CMP_UNIT, 'cores': cores, 'kind': 'reference',
               'sample': f'reference computeCommunityComparisons, one thread (its nested '
                         f'OpenMP regions repeat all work per thread), -Ofast build, on {cn} '
                         f'vertices ({cdt:.2f} s)'}
    extra = {'f_score': st['f_score'], 'same_same': st['same_same']}
    line = {'metric': CMP_METRIC, 'value': n_all / t_max, 'unit': CMP_UNIT, 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * t / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'int64',
            'data': 'synthetic (seeded labellings)',
            'config': dict(compare_config(args, n), **extra), 'roofline': roofline,
            'cpu_baseline': cpu, 'e2e': e2e, 'gpu_launches': launches, 'clocks': clk}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


# --------------------------------------------------------------------------- our arm
def run_csr_workload(args, world, rank, local):
    """A step builds the CSR of a raw R-MAT edge list resident in HBM with
    glv_dev_build_csr (removeEdges, both directions of every kept edge in list
    order, rows sorted by tail: the reference loaders' result).  e2e: the same
    build through glv_build_csr from a pinned host edge list to a host CSR."""
    import ctypes as ct
    import torch
    from grappolo_b200 import graphs, _lib
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    L = _lib.lib()
    u, v, w = graphs.rmat_edges_device(args.scale, seed=1, device=dev)
    nv, ne = 1 << args.scale, u.numel()
    ptr = torch.empty(nv + 1, dtype=torch.int64, device=dev)
    tail = torch.empty(2 * ne, dtype=torch.int32, device=dev)
    wout = torch.empty(2 * ne, dtype=torch.float64, device=dev)
    flags = _lib.GLV_CSR_REMOVE_EDGES | _lib.GLV_CSR_SORT_ROWS
    stream = torch.cuda.current_stream().cuda_stream
    nnz = ct.c_long(0)

    def step():
        _lib.check(L.glv_dev_build_csr(nv, ne, u.data_ptr(), v.data_ptr(), w.data_ptr(), flags,
                                       ptr.data_ptr(), tail.data_ptr(), wout.data_ptr(),
                                       ct.byref(nnz), stream))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    l0 = L.glv_kernel_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    launches = L.glv_kernel_launch_count() - l0
    if dist:
        dist.barrier()
    clk = clocks.stop()
    t = ev0.elapsed_time(ev1) * 1e-3
    t_max, e_all = aggregate(t, float(ne * args.steps), dist, dev)
    value = e_all / t_max
    out_nnz = nnz.value
    # algorithmic bytes: read every input edge (24 B), write the CSR (12 B per
    # entry + the row offsets)
    alg = 24 * ne + 12 * out_nnz + 8 * (nv + 1)
    peak, peak_kind = measured_peak()
    achieved = alg / (t / args.steps) / 1e9
    roofline = {'bound': 'hbm', 'kernel': 'the whole build (our kernels and the CUB radix sorts '
                                          'and scans between them), per step',
                'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                'peak_kind': peak_kind, 'traffic': None,
                'algorithmic_bytes_per_launch': alg, 'avg_launch_s': t / args.steps}
    e2e = None
    if not args.no_e2e:
        aos = torch.empty((ne, 3), dtype=torch.int64, pin_memory=True)
        aos.copy_(torch.stack([u, v, w.view(torch.int64)], dim=1))
        libc = ct.CDLL(None)

        def e2e_step():
            out = _lib.GlvGraph()
            _lib.check(L.glv_build_csr(nv, ne, ct.cast(aos.data_ptr(), ct.POINTER(_lib.GlvEdge)),
                                       flags, ct.byref(out)))
            libc.free(ct.cast(out.edgeListPtrs, ct.c_void_p))
            libc.free(ct.cast(out.edgeList, ct.c_void_p))
            return out.numEdges

        e2e_step()
        if dist:
            dist.barrier()
        e0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        et = time.perf_counter() - e0
        et, ee = aggregate(et, float(ne * args.steps), dist, dev)
        e2e = {'value': ee / et, 'unit': CSR_UNIT, 'h2d_bytes_per_step': 24 * ne,
               'd2h_bytes_per_step': 24 * out_nnz + 8 * (nv + 1),
               'seconds_per_step': et / args.steps}
        del aos
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cv, cdt, cne = csr_cpu_sample(args.csr_sample_scale)
        cpu = {'value': cv, 'unit': CSR_UNIT, 'cores': 1, 'kind': 'reference',
               'sample': csr_sample_text(args.csr_sample_scale, cdt, cne)}
    line = {'metric': CSR_METRIC, 'value': value, 'unit': CSR_UNIT, 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * t / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'int64',
            'data': 'synthetic (seeded raw R-MAT edge list generated on the device)',
            'config': csr_config(args, nv, ne, out_nnz,
                                 {'kept_edges': out_nnz // 2,
                                  'flags': 'GLV_CSR_REMOVE_EDGES | GLV_CSR_SORT_ROWS'}),
            'roofline': roofline, 'cpu_baseline': cpu, 'e2e': e2e, 'gpu_launches': launches,
            'clocks': clk}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def run_batch_workload(args, world, rank, local):
    """Many planted-partition graphs (vertex counts log-U[500, 200k], block sizes
    log-U[20, 2000], mu U[0.1, 0.6], mean degree U[6, 32], unit weights),
    generated on the device and run as batched multiphase Louvain (coloring=1).
    Graphs are split into consecutive waves of about --wave-pairs expected
    pairs; each wave is one batched run.  A step runs every wave once; the
    metric is graphs/s over the whole set, with per-graph finishing times
    (from the start of its wave) as p50/p99.  On N GPUs the set is split into
    N shards of about equal expected entries (grappolo_b200.sharding), each
    rank runs its shard and the per-graph results are gathered on the host
    (strong scaling: the whole set is the job)."""
    import numpy as np
    import torch
    from grappolo_b200 import graphs, louvain, _lib
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=900),
                                device_id=dev)
    mode = _lib.GLV_MODE_FAST if args.mode == 'fast' else _lib.GLV_MODE_VERIFY
    from grappolo_b200 import sharding
    all_specs = graphs.batch_specs(args.batch_graphs, seed=3)
    mine = sharding.shard_by_work(all_specs[:, 0] * all_specs[:, 3], world)[rank]
    specs = all_specs[mine]
    pairs = specs[:, 0] * specs[:, 3] / 2.0
    waves, g0 = [], 0
    while g0 < len(specs):
        g1, tot = g0 + 1, pairs[g0]
        while g1 < len(specs) and tot + pairs[g1] <= args.wave_pairs:
            tot += pairs[g1]
            g1 += 1
        waves.append((g0, g1))
        g0 = g1
    data = []
    for k, (a, b) in enumerate(waves):
        voff, ptr, tail, w = graphs.planted_batch_device(specs[a:b], seed=1000 + 7919 * rank + k,
                                                         device=dev)
        C = torch.empty(ptr.numel() - 1, dtype=torch.int32, device=dev)
        data.append((voff, ptr, tail, w, C))
    torch.cuda.synchronize()
    nnz_total = sum(d[2].numel() for d in data)
    nv_total = sum(d[1].numel() - 1 for d in data)
    stream = torch.cuda.current_stream().cuda_stream

    def step():
        out = []
        for voff, ptr, tail, w, C in data:
            out.append(louvain.run_batch_device(voff, ptr.data_ptr(), tail.data_ptr(),
                                                w.data_ptr(), C.data_ptr(), coloring=True,
                                                mode=mode, stream=stream))
        return out

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    runs = [step() for _ in range(args.steps)]
    ev1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    t = ev0.elapsed_time(ev1) * 1e-3
    graphs_done = args.steps * len(specs)
    t_max, g_all = aggregate(t, graphs_done, dist, dev)
    last = runs[-1]
    # per-graph results of every shard, in the batch's graph order
    per = sharding.gather_results(
        mine, np.stack([np.concatenate([r['done_seconds'] for r in last]),
                        np.concatenate([r['final_modularity'] for r in last])], axis=1),
        len(all_specs), dist)
    done, q = per[:, 0], per[:, 1]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = batch_cpu_baseline(data[0], args.batch_sample)
    edges = sum(r['edges_swept'] for run in runs for r in run)
    launches = sum(r['kernel_launches'] for run in runs for r in run)
    line = {'metric': 'batched Louvain graphs/s', 'value': g_all / t_max, 'unit': 'graphs/s',
            'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': 1e3 * t / args.steps, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic (seeded planted-partition graphs generated on the device)',
            'config': {'workload': f'batched plain multiphase Louvain (coloring=1) on '
                                   f'{len(all_specs)} planted-partition graphs',
                       'graphs': len(all_specs), 'graphs_this_rank': len(specs),
                       'num_vertices_this_rank': int(nv_total), 'nnz_this_rank': int(nnz_total),
                       'waves': len(waves), 'wave_pairs': args.wave_pairs, 'mode': args.mode,
                       'threshold': 1e-6, 'C_threshold': 1e-4, 'minGraphSize': 1000,
                       'per_graph_done_s_p50': float(np.percentile(done, 50)),
                       'per_graph_done_s_p99': float(np.percentile(done, 99)),
                       'modularity_mean': float(q.mean()), 'modularity_min': float(q.min()),
                       'local_move_edges_per_s': edges / t,
                       'rounds_per_wave': [r['rounds'] for r in last],
                       'parallelism': (f'{world} shards of about equal expected entries, '
                                       f'per-graph results gathered on the host')
                       if world > 1 else 'one GPU',
                       'l2': 'inputs larger than L2 (no flush)'},
            'gpu_launches': launches, 'clocks': clk, 'cpu_baseline': cpu, 'e2e': None}
    if world > 1:
        line['scaling'] = 'strong'
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def batch_cpu_baseline(wave, sample):
    """The reference's runMultiPhaseColoring (oracle/_ref, shipped -Ofast flags,
    all host cores) on the first `sample` graphs of the first wave, one call per
    graph: graphs/s on that subset."""
    import numpy as np
    from grappolo_b200 import graphs
    from oracle import Reference
    voff, ptr, tail, w, _ = wave
    hptr, htail, hw = ptr.cpu().numpy(), tail.cpu().numpy(), w.cpu().numpy()
    cores = os.cpu_count() or 1
    R = Reference(fast=True)
    n = min(sample, len(voff) - 1)
    secs, ents = 0.0, 0
    for k in range(n):
        v0, v1 = int(voff[k]), int(voff[k + 1])
        e0, e1 = int(hptr[v0]), int(hptr[v1])
        g = graphs.CSRGraph(hptr[v0:v1 + 1] - e0, htail[e0:e1].astype(np.int64) - v0, hw[e0:e1])
        t0 = time.perf_counter()
        R.run_multiphase_coloring(g, nthreads=cores)
        secs += time.perf_counter() - t0
        ents += g.nnz
    return {'value': n / secs, 'unit': 'graphs/s', 'cores': cores, 'kind': 'reference',
            'sample': f'reference runMultiPhaseColoring (-Ofast build, {cores} OpenMP threads) '
                      f'on the first {n} graphs of the first wave, one call per graph '
                      f'({ents} CSR entries, {secs:.1f} s)'}


def main():
    args = parse_args()
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        return run_reference(args, rank)
    if args.workload == 'batch':
        return run_batch_workload(args, world, rank, local)
    if args.workload == 'csr':
        return run_csr_workload(args, world, rank, local)
    if args.workload == 'compare':
        return run_compare_workload(args, world, rank, local)
    if args.workload == 'rmat' and args.scale >= 26:
        # graphs of tens of GB: torch's allocator maps pages as needed and
        # unmaps the builder's freed scratch on empty_cache(), so none of it
        # stays reserved beside the graph (the engine allocates from its own
        # pool; with whole segments ~33 GB stayed reserved at scale 27)
        os.environ.setdefault('PYTORCH_CUDA_ALLOC_CONF', 'expandable_segments:True')
    import numpy as np
    import torch
    from grappolo_b200 import graphs, louvain, _lib
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    L = _lib.lib()
    mode = {'fast': _lib.GLV_MODE_FAST, 'verify': _lib.GLV_MODE_VERIFY,
            'learned': _lib.GLV_MODE_LEARNED}[args.mode]
    if args.mode == 'learned':
        from grappolo_b200 import gate
        params, tau = gate.load_default()
        if args.gate_tau is None:
            args.gate_tau = tau
        gate.set_gate(params, args.gate_tau)

    if args.workload == 'powerlaw':
        g = graphs.planted_powerlaw(args.powerlaw_vertices, seed=1)
        ptr = torch.from_numpy(g.ptr).to(dev)
        tail = torch.from_numpy(g.tail.astype(np.int32)).to(dev)
        w = torch.from_numpy(g.weight).to(dev)
        del g
    elif args.scale >= 26:  # edge lists of tens of GB: the bounded-scratch builder
        ptr, tail, w = graphs.rmat_device_lean(args.scale, device=dev)
        torch.cuda.empty_cache()  # hand torch's freed scratch back for the engine's pool
    else:
        ptr, tail, w = graphs.rmat_device(args.scale, device=dev)
    nv, nnz = ptr.numel() - 1, tail.numel()
    C = torch.empty(nv, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()

    def step(profile=False):
        L.glv_set_profiling(args.profile_level if profile else 0)
        st = louvain.run_multiphase_device(nv, ptr.data_ptr(), tail.data_ptr(), w.data_ptr(),
                                           C.data_ptr(), coloring=True, mode=mode,
                                           stream=torch.cuda.current_stream().cuda_stream)
        L.glv_set_profiling(0)
        return st

    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    ev0.record()
    for _ in range(args.steps):
        stats.append(step(profile=True))
    ev1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    t = ev0.elapsed_time(ev1) * 1e-3
    edges = sum(s['edges_swept'] for s in stats)
    launches = sum(s['kernel_launches'] for s in stats)
    sweep_t = sum(s['sweep_kernel_time'] for s in stats)
    sweep_b = sum(s['sweep_bytes'] for s in stats)
    t, edges_all = aggregate(t, edges, dist, dev)
    value = edges_all / t

    # end to end through the reference-facing API: host AoS graph (pinned),
    # host->device copy and C_orig read-back inside every step
    e2e = None
    if not args.no_e2e:
        if args.scale >= 26:  # the engine's cached blocks back to the device for torch
            L.glv_release_cached_memory()
            torch.cuda.empty_cache()
        # the AoS edge records (head, tail, weight) in pinned host memory, built on the
        # device a chunk of entries at a time (R-MAT 27 holds 101 GB of them)
        aos = torch.empty((nnz, 3), dtype=torch.int64, pin_memory=True)
        chunk = 1 << 27
        for b in range(0, nnz, chunk):
            e = min(nnz, b + chunk)
            pos = torch.arange(b, e, device=dev, dtype=torch.int64)
            heads = torch.searchsorted(ptr, pos, right=True) - 1
            aos[b:e].copy_(torch.stack([heads, tail[b:e].to(torch.int64),
                                        w[b:e].view(torch.int64)], dim=1))
            del pos, heads
        hptr = ptr.cpu().pin_memory()
        hC = torch.empty(nv, dtype=torch.int64, pin_memory=True)
        import ctypes as ct
        gstruct = _lib.GlvGraph(nv, nv, nnz // 2, ct.cast(hptr.data_ptr(), ct.POINTER(ct.c_long)),
                                ct.cast(aos.data_ptr(), ct.POINTER(_lib.GlvEdge)))

        def e2e_step():
            st = _lib.GlvRunStats()
            _lib.check(L.glv_run_multiphase_coloring(
                ct.byref(gstruct), ct.cast(hC.data_ptr(), ct.POINTER(ct.c_long)), 1, 16, 0,
                1000, 1e-6, 1e-4, mode, ct.byref(st)))
            return st.to_dict()

        e2e_step()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = time.perf_counter()
        est = [e2e_step() for _ in range(args.steps)]
        et = time.perf_counter() - e0
        et, ee = aggregate(et, sum(s['edges_swept'] for s in est), dist, dev)
        e2e = {'value': ee / et, 'unit': UNIT, 'h2d_bytes_per_step': 24 * nnz + 8 * (nv + 1),
               'd2h_bytes_per_step': 8 * nv,
               'seconds_per_step': et / args.steps,
               'transfer_s_per_step': statistics.mean(s['time_transfer'] for s in est)}
        del aos, hptr, hC

    # time-to-modularity, learned gate vs plain, on the same graph
    learned_cmp = None
    if args.mode == 'fast' and args.workload == 'rmat' and not args.no_learned:
        learned_cmp = learned_vs_plain(L, nv, ptr, tail, w, C, stats, t / args.steps,
                                       args.steps, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(ptr, tail, w)
        if args.workload == 'rmat':
            cpu['full_run'] = reference_full_run(args.full_run_scale)

    peak, peak_kind = measured_peak()
    achieved = (sweep_b / sweep_t) / 1e9 if sweep_t > 0 else None
    ratio = profiled_traffic_ratio()
    steps_timed = sum(s['sweep_steps'] for s in stats)
    roofline = {'bound': 'hbm',
                'kernel': 'k_sweep_iteration (one Louvain iteration: every colour class and the '
                          'modularity; 32 B per CSR entry + 48 B per vertex with a full '
                          'modularity pass, 16 B per entry + 44 B per vertex when e_xx is '
                          'carried from the moves)',
                'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                'frac': (achieved / peak) if achieved else None, 'peak_kind': peak_kind,
                'traffic': (ratio * sweep_b / steps_timed) if (ratio and steps_timed) else None,
                'traffic_source': 'ncu dram__bytes_read.sum + dram__bytes_write.sum over the '
                                  'algorithmic bytes of one k_sweep_iteration launch on this '
                                  'R-MAT scale 24 graph (phase 1, iteration 2), times the '
                                  'average launch\'s algorithmic bytes',
                'algorithmic_bytes_per_launch': sweep_b / steps_timed if steps_timed else None,
                'avg_launch_s': sweep_t / steps_timed if steps_timed else None}
    s0 = stats[-1]
    extra = {'final_modularity': s0['final_modularity'], 'phases': s0['phases'],
             'iterations': s0['total_iterations'], 'final_clusters': s0['final_clusters'],
             'colors_phase1': s0['phase'][0]['num_colors'] if s0['phase'] else None,
             'mode': args.mode, 'time_to_modularity_s': t / args.steps,
             'kernel_time_per_step_s': dict(zip(
                 ['bin_deg0-4', 'bin_deg5-8', 'bin_deg9-16', 'bin_deg17-32', 'bin_deg33-127',
                  'bin_deg128-511', 'bin_deg512-1023', 'bin_deg1024-2047', 'bin_hubs', 'apply',
                  'modularity'],
                 [sum(s['kernel_time'][k] for s in stats) / args.steps for k in range(11)]))
             if args.profile_level >= 2 else None,
             'time_split_s': {'sweep+modularity': s0['time_clustering'],
                              'coloring': s0['time_coloring'],
                              'renumber+coarsen': s0['time_building'],
                              'other': s0['time_total'] - s0['time_clustering']
                              - s0['time_coloring'] - s0['time_building']},
             'learned': learned_cmp,
             'autotune': {'block_max': s0['tuned_block_max'], 'hub_chunk': s0['tuned_hub_chunk'],
                          'hub_cluster': s0['hub_cluster'],
                          'from_cache': bool(s0['tuned_from_cache'])},
             'step_totals_s': [round(s['time_total'], 4) for s in stats],
             'step_splits_s': [[round(s[k], 4) for k in ('time_clustering', 'time_coloring',
                                                         'time_building')] for s in stats]}
    line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * t / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic (seeded R-MAT generated on the device)',
            'config': workload_config(args, nv, nnz, extra), 'roofline': roofline,
            'cpu_baseline': cpu, 'e2e': e2e, 'gpu_launches': launches, 'clocks': clk}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def learned_vs_plain(L, nv, ptr, tail, w, C, plain_stats, plain_s, steps, dev):
    """The learned gate (shipped parameters) on the same graph as the plain
    timed runs: device time per full run, final Q and entries evaluated."""
    import torch
    from grappolo_b200 import _lib, gate, louvain
    params, tau = gate.load_default()
    gate.set_gate(params, tau)

    def run():
        return louvain.run_multiphase_device(nv, ptr.data_ptr(), tail.data_ptr(), w.data_ptr(),
                                             C.data_ptr(), coloring=True,
                                             mode=_lib.GLV_MODE_LEARNED,
                                             stream=torch.cuda.current_stream().cuda_stream)
    run()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    st = [run() for _ in range(steps)]
    ev1.record()
    torch.cuda.synchronize()
    lt = ev0.elapsed_time(ev1) * 1e-3 / steps
    q_plain = statistics.median(s['final_modularity'] for s in plain_stats)
    q_learned = statistics.median(s['final_modularity'] for s in st)
    return {'gate_tau': tau, 'plain_s_per_run': plain_s, 'learned_s_per_run': lt,
            'time_ratio_learned_over_plain': lt / plain_s,
            'q_plain_median': q_plain, 'q_learned_median': q_learned,
            'dq': q_learned - q_plain,
            'entries_plain_per_run': statistics.mean(s['edges_swept'] for s in plain_stats),
            'entries_learned_per_run': statistics.mean(s['edges_swept'] for s in st),
            'iterations_plain': plain_stats[-1]['total_iterations'],
            'iterations_learned': st[-1]['total_iterations']}


def _reference_basic_and_early_termination(path, cores):
    """Child process of reference_full_run: the reference's plain Jacobi
    multiphase run and its early-termination run on the graph saved at path."""
    import numpy as np
    from grappolo_b200 import graphs
    from oracle import Reference
    z = np.load(path)
    g = graphs.CSRGraph(z['ptr'], z['tail'], z['weight'])
    _, sb, _ = Reference(fast=True).run_multiphase_basic(g, nthreads=cores)
    _, se, _ = Reference(fast=True).run_multiphase_sync(g, 3, nthreads=cores)
    return sb, se


def reference_full_run(scale):
    """Time to modularity of the reference itself: Grappolo's
    runMultiPhaseColoring (oracle/_ref, shipped -Ofast flags, all host cores;
    Coloring/runMultiPhaseColoring.cpp:51-238) on the seeded numpy R-MAT graph
    of the given scale, beside this engine's fast mode on the same graph."""
    from grappolo_b200 import _lib, graphs, louvain
    from oracle import Reference
    g = graphs.rmat(scale, seed=1)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    _, s, _ = Reference(fast=True).run_multiphase_coloring(g, nthreads=cores)
    ref_wall = time.perf_counter() - t0
    # the heuristic the learned gate stands in for, run by the reference
    # itself beside the plain method it modifies: runMultiPhaseBasic and
    # runMultiPhaseSyncType(3), the early-termination Louvain
    # (FullSyncOptimization/parallelLouvainMethodEarlyTerminate.cpp:116-195),
    # in a child process, so that a failure of that code costs only its record
    import numpy as np
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, 'graph.npz')
        np.savez(path, ptr=g.ptr, tail=g.tail, weight=g.weight)
        try:
            with ProcessPoolExecutor(1, mp_context=mp.get_context('spawn')) as ex:
                sb, se = ex.submit(_reference_basic_and_early_termination, path, cores).result()
        except Exception as e:  # noqa: BLE001 - the record says what happened
            sb = se = {'error': f'{type(e).__name__}: {e}'}
    louvain.run_multiphase_csr(g, coloring=True, mode=_lib.GLV_MODE_FAST)  # warm
    t0 = time.perf_counter()
    _, st = louvain.run_multiphase_csr(g, coloring=True, mode=_lib.GLV_MODE_FAST)
    gpu_wall = time.perf_counter() - t0

    def arm(x):
        if 'error' in x:
            return {'error': x['error']}
        return {'total_time_s': x.get('total_time'), 'final_modularity': x.get('final_mod'),
                'phases': x.get('phases'), 'iterations': x.get('total_iterations')}
    return {'graph': f'R-MAT scale {scale}, edge factor 16, a=0.57 b=0.19 c=0.19, FP64 '
                     f'weights U(0,1], numpy seed 1 ({g.num_vertices} vertices, {g.nnz} '
                     f'CSR entries)',
            'reference': {'threads': cores, 'total_time_s': s.get('total_time'),
                          'wall_s': ref_wall, 'final_modularity': s.get('final_mod'),
                          'phases': s.get('phases'),
                          'iterations': s.get('total_iterations')},
            'gpu_fast': {'wall_s_host_csr_in': gpu_wall,
                         'engine_total_s': st['time_total'],
                         'final_modularity': st['final_modularity'],
                         'phases': st['phases'], 'iterations': st['total_iterations']},
            'time_ratio_reference_over_gpu': (s.get('total_time') or ref_wall) / gpu_wall,
            'reference_basic': arm(sb),
            'reference_early_termination': arm(se),
            'early_termination_time_over_basic':
                (se['total_time'] / sb['total_time'])
                if se.get('total_time') and sb.get('total_time') else None}


def cpu_baseline(ptr, tail, w):
    """The reference (oracle/_ref, shipped -Ofast flags) on all host cores: one phase-1
    colour sweep iteration of the same graph (a bounded sample)."""
    import numpy as np
    from grappolo_b200 import graphs
    from oracle import Reference
    g = graphs.CSRGraph(ptr.cpu().numpy(), tail.cpu().numpy().astype(np.int64), w.cpu().numpy())
    cores = os.cpu_count() or 1
    R = Reference(fast=True)
    h = R.graph(g)
    col, mc, tcol = R.color_g(h, g.num_vertices, cores)
    _, _, itr, tt = R.coloring_phase_g(h, g.num_vertices, col, mc + 1, -1.0, float('inf'), cores)
    R.free_graph(h)
    return {'value': g.nnz * itr / tt, 'unit': UNIT, 'cores': cores, 'kind': 'reference',
            'sample': f'one phase-1 colour-class sweep iteration (+modularity) of the '
                      f'reference algoLouvainWithDistOneColoring on the same graph '
                      f'({g.nnz} CSR entries, {mc + 1} colours), {cores} OpenMP threads, '
                      f'-Ofast build, its own iteration timer ({tt:.2f} s)'}


if __name__ == '__main__':
    sys.exit(main())
