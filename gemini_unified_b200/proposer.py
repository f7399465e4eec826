"""Learned step/order proposer of the FK solver: training data, training, weights.

The network (3 x 64, tanh; csrc/proposer.cu) predicts for each (item, phase)
the work of the phase's integrations when the step-size control aims at
attempt 5 and at attempt 7, relative to the reference's 6, and the factor that
brings the initial step of the initial-value formulas to the step the control
settles on.  The labels come from step logs of the integrator run with order
targets 5, 6 and 7 on a training workload; the features are the ones the
inference kernel computes (dumped by the library).  Training runs on the GPU
with the library's own forward, backward and Adam kernels.

    python -m gemini_unified_b200.proposer --workload global_small --out <file.npz>
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os

import numpy as np

from . import configs, model as M
from .fk import GeminiFK, GEM_BACKEND_GPU_FAST, lib

NF, NO = 11, 3
NPARAM = 5123
USE_ORDER, USE_STEP = 1, 2
SEQDIV = np.array([2, 4, 6, 8, 12, 16, 24])
ATTEMPT_WORK = np.cumsum(SEQDIV + 1)   # substeps through attempt j, the closing one included
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "proposer_global_small.npz")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _bind():
    L = lib()
    vp = ctypes.c_void_p
    L.gem_proposer_set.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_float]
    L.gem_proposer_dump.argtypes = [vp, ctypes.c_int]
    L.gem_proposer_dump_read.argtypes = [vp, vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
    L.gem_prop_grad.argtypes = [vp] * 4 + [ctypes.c_int, vp, vp]
    L.gem_prop_train.argtypes = [vp] * 4 + [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint,
                                            vp]
    return L


def step_work(rec) -> np.ndarray:
    """Work of each logged step attempt: attempts 1..j when it converged at j, 1..7 when rejected."""
    r = rec["result"].astype(np.int64)
    return np.where(r > 0, ATTEMPT_WORK[np.clip(r, 1, 7) - 1], ATTEMPT_WORK[6]).astype(np.float64)


def collect(workload: str, jf: tuple | None = None, kopts=(5, 6, 7), capacity: int = 30_000_000):
    """Features [3 n][11] and labels, masks [3 n][3] of every (phase, item) of a workload slab."""
    L = _bind()
    w = configs.WORKLOADS[workload]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    lo, hi = jf if jf else (g.nf1, g.nf2)
    fk = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST)
    n = int(g.nwn[lo - 1: hi].sum())
    work, hfirst, hset, feats = {}, None, None, None
    for k in kopts:
        fk.order_target(k)
        fk.steplog(capacity)
        if feats is None:
            fk._check(L.gem_proposer_dump(fk._h, 1))
        fk.run(w.params, jre, lo, hi, f32=False, f64=False)
        if feats is None:
            feats = np.zeros(3 * n * NF, np.float32)
            cnt = ctypes.c_longlong()
            fk._check(L.gem_proposer_dump_read(fk._h, _p(feats), feats.size, ctypes.byref(cnt)))
            feats = feats.reshape(3 * n, NF)
            fk._check(L.gem_proposer_dump(fk._h, 0))
        rec = fk.steplog_read(capacity)
        key = rec["phase"].astype(np.int64) * n + rec["k"]
        work[k] = np.bincount(key, weights=step_work(rec), minlength=3 * n)
        if k == 6:
            hfirst, hset = initial_steps(rec, key, 3 * n)
    fk.steplog(0)
    y = np.zeros((3 * n, NO), np.float32)
    mask = np.zeros((3 * n, NO), np.float32)
    ok = work[6] > 0
    for q, k in enumerate((5, 7)):
        if k in work:
            good = ok & (work[k] > 0)
            y[good, q] = np.log(work[k][good] / work[6][good])
            mask[good, q] = 1.0
    good = (hfirst > 0) & (hset > 0)
    y[good, 2] = np.clip(np.log(hset[good] / hfirst[good]), -1.4, 1.4)
    mask[good, 2] = 1.0
    return feats, y, mask, {int(k): float(v.sum()) for k, v in work.items()}


def initial_steps(rec, key, nkey):
    """|h| of the first step of each (phase, item) and the median |h| of its accepted steps 3..8."""
    order = np.lexsort((np.arange(len(key)), key))
    ks = key[order]
    hs = np.abs(rec["h"][order])
    acc = rec["result"][order] > 0
    first_idx = np.r_[0, np.nonzero(ks[1:] != ks[:-1])[0] + 1]
    hfirst = np.zeros(nkey)
    hfirst[ks[first_idx]] = hs[first_idx]
    hset = np.zeros(nkey)
    pos = np.arange(len(ks)) - np.repeat(first_idx, np.diff(np.r_[first_idx, len(ks)]))
    sel = acc & (pos >= 2) & (pos < 8)
    fk_, v_ = ks[sel], hs[sel]
    if len(fk_):
        o = np.lexsort((v_, fk_))
        fk_, v_ = fk_[o], v_[o]
        starts = np.r_[0, np.nonzero(fk_[1:] != fk_[:-1])[0] + 1]
        cnt = np.diff(np.r_[starts, len(fk_)])
        keep = cnt >= 4
        hset[fk_[starts[keep]]] = v_[starts + cnt // 2][keep]
    return hfirst, hset


def standardise(x):
    mu = x.mean(0)
    sd = x.std(0)
    sd = np.where(sd > 1e-6, sd, 1.0)
    return mu.astype(np.float32), sd.astype(np.float32)


def init_weights(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, 1 / np.sqrt(NF), 64 * NF), np.zeros(64), rng.normal(0, 1 / np.sqrt(64), 64 * 64),
             np.zeros(64), rng.normal(0, 1 / np.sqrt(64), NO * 64) * 0.1, np.zeros(NO)]
    return np.concatenate(parts).astype(np.float32)


def gradient(w, x, y, mask):
    """Loss and gradient of the masked MSE from the library's training kernel."""
    L = _bind()
    grad = np.zeros(NPARAM, np.float32)
    loss = np.zeros(1, np.float32)
    a = [np.ascontiguousarray(v, np.float32) for v in (w, x, y, mask)]
    if L.gem_prop_grad(*[_p(v) for v in a], len(a[1]), _p(grad), _p(loss)) != 0:
        raise RuntimeError("gem_prop_grad failed")
    return float(loss[0]), grad


def train(x, y, mask, epochs=300, batch=2048, lr=3e-3, seed=0):
    """Train on the GPU with the library's kernels; returns (weights, norm, loss history)."""
    L = _bind()
    mu, sd = standardise(x)
    xs = np.ascontiguousarray((x - mu) / sd, np.float32)
    w = init_weights(seed)
    hist = np.zeros(epochs, np.float32)
    rc = L.gem_prop_train(_p(w), _p(xs), _p(np.ascontiguousarray(y, np.float32)),
                          _p(np.ascontiguousarray(mask, np.float32)), len(xs), epochs, batch, lr, seed, _p(hist))
    if rc != 0:
        raise RuntimeError("gem_prop_train failed")
    return w, np.concatenate([mu, sd]).astype(np.float32), hist


def save(path, w, norm, meta):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, w=w, norm=norm, meta=json.dumps(meta))


def load(path=WEIGHTS):
    d = np.load(path)
    return d["w"].astype(np.float32), d["norm"].astype(np.float32)


def enable(fk: GeminiFK, path=WEIGHTS, use: int = USE_ORDER | USE_STEP, margin: float = 0.1):
    """Switch the proposer on for a context (fast backend)."""
    w, norm = load(path)
    fk._check(_bind().gem_proposer_set(fk._h, _p(w), _p(norm), int(use), float(margin)))


def disable(fk: GeminiFK):
    fk._check(_bind().gem_proposer_set(fk._h, None, None, 0, 0.0))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="global_small")
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--epochs", type=int, default=300)
    a = ap.parse_args(argv)
    x, y, mask, work = collect(a.workload)
    w, norm, hist = train(x, y, mask, epochs=a.epochs)
    meta = {"workload": a.workload, "samples": int(len(x)), "epochs": a.epochs, "loss_first": float(hist[0]),
            "loss_last": float(hist[-1]), "work_by_order_target": work}
    save(a.out, w, norm, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
