"""Training data and training of the expansion-order network, on the GPU.

The data are made by the FMM itself (no counterpart in the reference, which
takes p from the caller): for each synthetic problem the library's evaluate is
run at every order of a p sweep, in FP64 and in mixed precision, and its
relative L2 error against the FP64 direct sum on 256 sampled targets (the
referee of test.py:11-18) is recorded, together with the evaluate time at each
leaf size. Labels for any tolerance are then read off the error curves
(``learned.label_p``), so one sweep yields a sample per tolerance.

    python -m hfmm_b200.train_order generate --problems 120 --out sweep.npz
    python -m hfmm_b200.train_order train --data sweep.npz --out order_net.npz

Problems: N log-uniform in [5e4, 5e5]; uniform in the unit cube or 1-16
Gaussian clusters with sigma in [0.01, 0.1] (clipped to the cube); the eight
cube corners are added so that the domain extent is exactly 1 and the decode
factors repeat across problems of the same k (they are cached);
k from a grid in [1, 24]; complex N(0, 1) charges.
"""
import argparse
import math
import time

import numpy as np
import torch

from . import learned, operators
from .learned import N_FEATURES, LEAVES, TOL_MIXED, label_p

K_GRID = (1.0, 1.5, 2.0, 3.0, 4.0, 6.0, 8.0, 12.0, 16.0, 24.0)
P_SWEEP = tuple(range(4, 15))
TOLS = tuple(10.0 ** (-e) for e in np.arange(3.0, 8.01, 0.5))


def make_problem(rng):
    n = int(math.exp(rng.uniform(math.log(5e4), math.log(5e5))))
    if rng.random() < 1 / 3:
        kind, x = "uniform", rng.random((n, 3))
    else:
        nc = int(rng.integers(1, 17))
        sig = float(rng.uniform(0.01, 0.1))
        kind = f"clusters{nc}"
        c = rng.uniform(0.1, 0.9, (nc, 3))
        x = np.clip(c[rng.integers(0, nc, n)] + sig * rng.standard_normal((n, 3)), 0.0, 1.0)
    corners = np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], np.float64)
    x = np.vstack([x, corners])
    k = float(rng.choice(K_GRID))
    q = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    return x, k, q, kind


class _DecodeCache:
    """Memoises operators.level_decodes while the sweep runs (same extent and k
    give the same factors); cleared whenever k changes."""

    def __init__(self):
        self.orig = operators.level_decodes
        self.k = None
        self.memo = {}

    def __call__(self, p, level, extent, k, imaginary, eps_rel):
        if k != self.k:
            self.memo.clear()
            self.k = k
        key = (p, level, extent, imaginary, eps_rel)
        if key not in self.memo:
            self.memo[key] = self.orig(p, level, extent, k, imaginary, eps_rel)
        return self.memo[key]


def _time_eval(hf, st, q_re, q_im, phi, E, prec, reps=1, warmup=0):
    for _ in range(warmup):
        hf.evaluate_into(st, q_re, q_im, phi, E, prec)
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(reps):
        hf.evaluate_into(st, q_re, q_im, phi, E, prec)
    b.record(s)
    b.synchronize()
    hf.check_errors(st)
    return a.elapsed_time(b) / reps


def generate(n_problems, seed=0, n_check=256, verbose=True):
    import hfmm_b200 as hf
    rng = np.random.default_rng(seed)
    probs = [make_problem(np.random.default_rng([seed, i])) for i in range(n_problems)]
    order = sorted(range(n_problems), key=lambda i: probs[i][1])   # group by k for the cache
    cache = _DecodeCache()
    hf.level_decodes = cache      # the name _load_tables calls
    out = dict(feats=[], err64=[], errmx=[], t64=[], tmx=[], leaf_t=[], leaf_p=[], n=[], k=[],
               kind=[])
    dev = torch.device("cuda", torch.cuda.current_device())
    try:
        for j, i in enumerate(order):
            x, k, q, kind = probs[i]
            t0 = time.time()
            f = learned.features_for(x, k, 1.0, dev)
            f[0] = 0.0                                  # tolerance slot, filled per sample
            q_re = torch.as_tensor(q.real.copy()).to(dev)
            q_im = torch.as_tensor(q.imag.copy()).to(dev)
            tg = np.sort(rng.choice(len(x), n_check, replace=False)).astype(np.int32)
            tg_d = torch.as_tensor(tg).to(dev)
            e64, emx, t64, tmx = [], [], [], []
            ref = None
            for p in P_SWEEP:
                st = hf.setup(x, k, p=p, N_max=learned.FEATURE_LEAF, device=dev)
                if ref is None:
                    r_phi, r_E = hf.direct_at(st, q_re, q_im, tg_d, field=True)
                    ref = (r_phi.cpu().numpy(), r_E.cpu().numpy())
                phi = torch.empty(st.n, dtype=torch.complex128, device=dev)
                E = torch.empty((st.n, 3), dtype=torch.complex128, device=dev)
                for prec, errs, ts in ((hf.PREC_FP64, e64, t64), (hf.PREC_MIXED, emx, tmx)):
                    if prec == hf.PREC_MIXED and p < 5:
                        errs.append(np.inf)
                        ts.append(np.nan)
                        continue
                    ts.append(_time_eval(hf, st, q_re, q_im, phi, E, prec))
                    errs.append(max(learned._rel_l2(phi[tg_d].cpu().numpy(), ref[0]),
                                    learned._rel_l2(E[tg_d].cpu().numpy(), ref[1])))
                st.close()
                del phi, E
            # leaf timing at the order the mixed path needs for 1e-6
            lp = int(min(learned.P_MAX, max(5, math.ceil(label_p(P_SWEEP, emx, TOL_MIXED)))))
            lt = []
            for leaf in LEAVES:
                st = hf.setup(x, k, p=lp, N_max=leaf, device=dev)
                phi = torch.empty(st.n, dtype=torch.complex128, device=dev)
                E = torch.empty((st.n, 3), dtype=torch.complex128, device=dev)
                lt.append(_time_eval(hf, st, q_re, q_im, phi, E, hf.PREC_MIXED, reps=2, warmup=1))
                st.close()
                del phi, E
            for key, val in (("feats", f), ("err64", e64), ("errmx", emx), ("t64", t64),
                             ("tmx", tmx), ("leaf_t", lt), ("leaf_p", lp), ("n", len(x)),
                             ("k", k), ("kind", kind)):
                out[key].append(val)
            if verbose:
                print(f"[{j + 1}/{n_problems}] N={len(x)} k={k} {kind}: "
                      f"err64={np.array2string(np.array(e64), precision=1)} "
                      f"leaf_p={lp} leaf_ms={np.round(lt, 2)} ({time.time() - t0:.1f} s)",
                      flush=True)
    finally:
        hf.level_decodes = cache.orig
    res = {k: np.asarray(v) for k, v in out.items()}
    res["ps"] = np.asarray(P_SWEEP)
    return res


def samples(data, tols=TOLS):
    """Training pairs (X, T): one per (problem, tolerance)."""
    X, T = [], []
    ps = data["ps"]
    for i in range(len(data["feats"])):
        leaf_best = math.log2(LEAVES[int(np.argmin(data["leaf_t"][i]))])
        for tol in tols:
            errs = data["errmx"][i] if tol >= TOL_MIXED else data["err64"][i]
            f = np.array(data["feats"][i], np.float32)
            f[0] = math.log10(tol)
            X.append(f)
            T.append((label_p(ps, errs, tol), leaf_best))
    return np.asarray(X, np.float32), np.asarray(T, np.float32)


def train(data, steps=4000, lr=2e-3, seed=0, holdout=0.2, verbose=True, device=None):
    """Train on the sweep data with a problem-level holdout; returns (net, stats)."""
    n = len(data["feats"])
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n)
    n_val = int(round(holdout * n))
    val, trn = perm[:n_val], perm[n_val:]
    sub = lambda idx: {k: (v[idx] if k != "ps" else v) for k, v in data.items()}
    Xt, Tt = samples(sub(trn))
    net = learned.OrderNet.init(Xt, Tt, seed=seed, device=device)
    hist = []
    chunk = 500
    for s in range(0, steps, chunk):
        loss = net.train(Xt, Tt, min(chunk, steps - s), lr)
        hist.append(loss)
        if verbose:
            print(f"step {min(s + chunk, steps)}: normalised loss {loss:.4g}", flush=True)
    stats = dict(train_loss=hist[-1], n_train=len(Xt))
    if n_val:
        Xv, Tv = samples(sub(val))
        Y = net.predict(Xv)
        stats.update(val_p_mae=float(np.mean(np.abs(Y[:, 0] - Tv[:, 0]))),
                     val_leaf_mae=float(np.mean(np.abs(Y[:, 1] - Tv[:, 1]))), n_val=len(Xv))
    return net, stats


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sp = ap.add_subparsers(dest="cmd", required=True)
    g = sp.add_parser("generate")
    g.add_argument("--problems", type=int, default=120)
    g.add_argument("--seed", type=int, default=0)
    g.add_argument("--out", required=True)
    t = sp.add_parser("train")
    t.add_argument("--data", required=True)
    t.add_argument("--steps", type=int, default=4000)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    if a.cmd == "generate":
        res = generate(a.problems, a.seed)
        np.savez_compressed(a.out, **res)
    else:
        data = dict(np.load(a.data, allow_pickle=False))
        net, stats = train(data, a.steps, a.lr)
        print(stats)
        net.save(a.out, **{k: np.float64(v) for k, v in stats.items()})


if __name__ == "__main__":
    main()
