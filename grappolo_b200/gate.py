"""Learned move gate: host-side training pipeline and parameter I/O.

The plain method generates its own training data: with trace capture on,
every plain colour sweep records, for a hashed sample of vertices, the six
features the gate sees (from the previous sweep) and whether the sweep moved
the vertex.  The MLP is trained on the GPU by the library's own forward and
backward kernels (glv_gate_train) with class-balanced weights, and the keep
threshold tau is the largest one that keeps a target share of the moves on
held-out traces.  Trained parameters live in gate_params.npz beside this file.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

from . import _lib, graphs, louvain

HERE = os.path.dirname(os.path.abspath(__file__))
PARAMS_PATH = os.path.join(HERE, 'gate_params.npz')
NPARAMS = 4673
_fp = ct.POINTER(ct.c_float)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised parameters (layout W1[64][6] b1 W2[64][64] b2 W3[64] b3)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, dtype=np.float32)
    p[0:384] = rng.standard_normal(384) * np.sqrt(2.0 / 6)
    p[448:4544] = rng.standard_normal(4096) * np.sqrt(2.0 / 64)
    p[4608:4672] = rng.standard_normal(64) * np.sqrt(1.0 / 64)
    return p


def set_gate(params, tau: float) -> None:
    p = _f32(params)
    _lib.check(_lib.lib().glv_gate_set(p.ctypes.data_as(_fp), float(tau)))


def load_default():
    """(params, tau) from gate_params.npz, or None."""
    if not os.path.exists(PARAMS_PATH):
        return None
    z = np.load(PARAMS_PATH)
    return z['params'].astype(np.float32), float(z['tau'])


def grad(x, y, w, params):
    x, y, w, p = _f32(x), _f32(y), _f32(w), _f32(params)
    g = np.zeros(NPARAMS, dtype=np.float32)
    loss = ct.c_double(0)
    _lib.check(_lib.lib().glv_gate_grad(x.shape[0], x.ctypes.data_as(_fp), y.ctypes.data_as(_fp),
                                        w.ctypes.data_as(_fp), p.ctypes.data_as(_fp),
                                        g.ctypes.data_as(_fp), ct.byref(loss)))
    return loss.value, g


def train(x, y, w, params=None, epochs: int = 8, batch: int = 16384, lr: float = 2e-3,
          seed: int = 0):
    x, y, w = _f32(x), _f32(y), _f32(w)
    p = _f32(init_params(seed) if params is None else params).copy()
    loss = ct.c_double(0)
    _lib.check(_lib.lib().glv_gate_train(x.shape[0], x.ctypes.data_as(_fp), y.ctypes.data_as(_fp),
                                         w.ctypes.data_as(_fp), epochs, batch, lr, seed,
                                         p.ctypes.data_as(_fp), ct.byref(loss)))
    return p, loss.value


def infer(x, params):
    """Move probabilities of host feature rows via the tensor-core kernel."""
    import torch
    set_gate(params, 0.5)
    dev = torch.device('cuda')
    xd = torch.from_numpy(_f32(x)).to(dev)
    pd = torch.empty(xd.shape[0], dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    _lib.check(_lib.lib().glv_gate_infer(xd.shape[0], xd.data_ptr(), pd.data_ptr(),
                                         ct.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return pd.cpu().numpy()


def balanced_weights(y):
    y = np.asarray(y)
    pos = max(float(y.mean()), 1e-6)
    return np.where(y > 0.5, 0.5 / pos, 0.5 / max(1.0 - pos, 1e-6)).astype(np.float32)


def collect_traces(graph_list, rate: float = 0.25, capacity: int = 4_000_000):
    """Run the plain fast method on each graph with trace capture on."""
    L = _lib.lib()
    _lib.check(L.glv_trace_begin(capacity, rate))
    try:
        for g in graph_list:
            louvain.run_multiphase_csr(g, coloring=True, mode=_lib.GLV_MODE_FAST)
        n = L.glv_trace_fetch(None, None, 0)
        x = np.zeros((n, 6), dtype=np.float32)
        y = np.zeros(n, dtype=np.float32)
        L.glv_trace_fetch(x.ctypes.data_as(_fp), y.ctypes.data_as(_fp), n)
    finally:
        L.glv_trace_end()
    return x, y


def training_graphs(count: int, seed: int = 100):
    """Graphs of the batched-workload family (log-uniform sizes and block
    sizes, mu ~ U[0.1, 0.6], mean degree ~ U[6, 32]), capped at 60k vertices."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        nv = int(np.exp(rng.uniform(np.log(2000), np.log(60000))))
        block = int(np.exp(rng.uniform(np.log(20), np.log(2000))))
        mu = float(rng.uniform(0.1, 0.6))
        d = float(rng.uniform(6, 32))
        out.append(graphs.planted_partition_mixed(nv, block, mu, d, seed=seed + 1 + k))
    return out


def choose_tau(prob, y, keep_recall: float = 0.97):
    """Largest threshold that keeps `keep_recall` of the held-out moves."""
    pos = np.sort(prob[y > 0.5])
    if pos.size == 0:
        return 0.5
    k = int(np.floor((1.0 - keep_recall) * pos.size))
    return float(min(max(pos[k], 1e-4), 0.999))


def fit_default(n_graphs: int = 48, seed: int = 100, out: str = PARAMS_PATH):
    """Collect traces, train, choose tau on a held-out split, save."""
    x, y = collect_traces(training_graphs(n_graphs, seed))
    rng = np.random.default_rng(seed)
    idx = rng.permutation(x.shape[0])
    cut = int(0.8 * idx.size)
    tr, va = idx[:cut], idx[cut:]
    p, loss = train(x[tr], y[tr], balanced_weights(y[tr]), epochs=10, seed=seed)
    prob = infer(x[va], p)
    tau = choose_tau(prob, y[va])
    keep = prob >= tau
    stats = dict(rows=int(x.shape[0]), moved=float(y.mean()), loss=float(loss), tau=tau,
                 kept=float(keep.mean()), recall=float(keep[y[va] > 0.5].mean()))
    np.savez(out, params=p, tau=np.float32(tau),
             **{k: np.float64(v) for k, v in stats.items() if k != 'tau'})
    return p, tau, stats


if __name__ == '__main__':
    import json
    import sys
    path = sys.argv[1] if len(sys.argv) > 1 else PARAMS_PATH
    _, _, st = fit_default(out=path)
    print(json.dumps(st))
