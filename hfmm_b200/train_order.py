"""Training data and training of the expansion-order network, on the GPU.

The data are made by the FMM itself (no counterpart in the reference, which
takes p from the caller): for each synthetic problem the library's evaluate is
run at every order of a p sweep, in FP64 and in mixed precision (with the
low-rank M2L the front doors use, ``learned.compress_for``), and its
relative L2 error against the FP64 direct sum on 256 sampled targets (the
referee of test.py:11-18) is recorded, together with the evaluate time at each
leaf size. Labels for any tolerance are then read off the error curves
(``learned.label_p``), so one sweep yields a sample per tolerance.

    python -m hfmm_b200.train_order generate --problems 120 --out sweep.npz
    python -m hfmm_b200.train_order generate --high-k --problems 24 --seed 1 --out high.npz
    python -m hfmm_b200.train_order merge sweep.npz high.npz --out all.npz
    python -m hfmm_b200.train_order train --data all.npz --out order_net.npz

Problems: N log-uniform in [5e4, 5e5]; uniform in the unit cube or 1-16
Gaussian clusters with sigma in [0.01, 0.1] (clipped to the cube); the eight
cube corners are added so that the domain extent is exactly 1 and the decode
factors repeat across problems of the same k (they are cached);
k from a grid in [1, 24] (p swept 4..14), or, for the high-frequency sweep, from
{32, 40, 50} (p swept 6..16); complex N(0, 1) charges.
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
# the high-frequency sweep (k x extent 32..50, the 8M-point clustered workload's 44
# among them): orders up to the clamp P_MAX = 16, starting at 6
K_GRID_HIGH = (32.0, 40.0, 50.0)
P_SWEEP_HIGH = tuple(range(6, 17))
# tolerances the network is trained for: 1e-3 .. 10^-6.5 in quarter decades. Below
# about 2e-7 the FP64 method itself stalls (the cos component's eps_rel = 1e-7
# damping, HFMM.py:75-77), most problems cannot meet the tolerance at any swept p,
# and the certified front door uses the conservative order there instead.
TOLS = tuple(10.0 ** (-e) for e in np.arange(3.0, 6.51, 0.25))


def make_problem(rng, k_grid=K_GRID):
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
    k = float(rng.choice(k_grid))
    q = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    return x, k, q, kind


class _DecodeCache:
    """Memoises operators.level_decodes while the sweep runs (same extent and k
    give the same factors); cleared whenever k changes."""

    def __init__(self):
        self.orig = operators.level_decodes
        self.k = None
        self.memo = {}

    def __call__(self, p, level, extent, k, imaginary, eps_rel, kind="helmholtz"):
        if k != self.k:
            self.memo.clear()
            self.k = k
        key = (p, level, extent, imaginary, eps_rel, kind)
        if key not in self.memo:
            self.memo[key] = self.orig(p, level, extent, k, imaginary, eps_rel, kind)
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


def generate(n_problems, seed=0, n_check=256, verbose=True, k_grid=K_GRID, p_sweep=P_SWEEP):
    import hfmm_b200 as hf
    rng = np.random.default_rng(seed)
    probs = [make_problem(np.random.default_rng([seed, i]), k_grid) for i in range(n_problems)]
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
            cmp = learned.compress_for(1e-6, hf.PREC_MIXED)
            for p in p_sweep:
                st = hf.setup(x, k, p=p, N_max=learned.FEATURE_LEAF, device=dev,
                              m2l_compress=cmp if p >= 5 else None)
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
            lp = int(min(learned.P_MAX, max(5, math.ceil(label_p(p_sweep, emx, TOL_MIXED)))))
            lt = []
            for leaf in LEAVES:
                st = hf.setup(x, k, p=lp, N_max=leaf, device=dev, m2l_compress=cmp)
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
    res["ps"] = np.asarray(p_sweep)
    return res


def merge(datasets):
    """One training set from sweeps over different orders: every problem's error and
    time curves are laid on the union of the swept orders, NaN where its sweep did not
    run that order (label_p leaves those out)."""
    ps = np.unique(np.concatenate([d["ps"] for d in datasets]))
    out = {}
    for d in datasets:
        idx = np.searchsorted(ps, d["ps"])
        for key, v in d.items():
            if key == "ps":
                continue
            if key in ("err64", "errmx", "t64", "tmx"):
                w = np.full((v.shape[0], len(ps)), np.nan)
                w[:, idx] = v
                v = w
            out.setdefault(key, []).append(v)
    res = {k: np.concatenate(v) for k, v in out.items()}
    res["ps"] = ps
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


def _fit(X, T, steps, lr, seed, device):
    net = learned.OrderNet.init(X, T, seed=seed, device=device)
    net.train(X, T, steps, lr)
    return net


def cross_validate(data, steps_list=(200, 400, 600, 1000), lr=1e-3, folds=5, seed=0,
                   margins=(0.25, 0.5, 0.75), device=None):
    """k-fold cross-validation over problems (every sample of a problem in one fold),
    training with the GPU kernels. Returns {steps: stats} with the mean absolute p
    error, the leaf accuracy, and per margin the share of held-out samples whose
    chosen p falls below the label (a certification miss) and the mean overshoot."""
    n = len(data["feats"])
    perm = np.random.default_rng(seed).permutation(n)
    sub = lambda idx: {k: (v[idx] if k != "ps" else v) for k, v in data.items()}
    preds = {s: [] for s in steps_list}
    for f in range(folds):
        val = perm[f::folds]
        trn = np.setdiff1d(perm, val)
        Xt, Tt = samples(sub(trn))
        Xv, Tv = samples(sub(val))
        net = learned.OrderNet.init(Xt, Tt, seed=seed + f, device=device)
        done = 0
        for st in steps_list:
            net.train(Xt, Tt, st - done, lr)
            done = st
            preds[st].append((net.predict(Xv), Tv))
    out = {}
    for st in steps_list:
        Y = np.concatenate([a for a, _ in preds[st]])
        T = np.concatenate([b for _, b in preds[st]])
        r = {"p_mae": float(np.mean(np.abs(Y[:, 0] - T[:, 0]))),
             "leaf_acc": float(np.mean(np.abs(np.round(Y[:, 1]) - T[:, 1]) < 0.5))}
        for mg in margins:
            pc = np.ceil(Y[:, 0] + mg)
            r[f"under@{mg}"] = float(np.mean(pc < T[:, 0] - 1e-9))
            r[f"over@{mg}"] = float(np.mean(pc - T[:, 0]))
        out[st] = r
    return out


def train(data, steps=None, lr=1e-3, seed=0, verbose=True, device=None):
    """Choose the step count by cross-validation (unless given), then train on every
    problem; returns (net, stats)."""
    cvs = cross_validate(data, lr=lr, seed=seed, device=device)
    if verbose:
        for st, r in cvs.items():
            print(f"cv steps {st}: " + ", ".join(f"{k} {v:.3f}" for k, v in r.items()), flush=True)
    if steps is None:
        steps = min(cvs, key=lambda st: cvs[st]["p_mae"])
    X, T = samples(data)
    net = _fit(X, T, steps, lr, seed, device)
    Y = net.predict(X)
    stats = dict(steps=steps, lr=lr, n_train=len(X), n_problems=len(data["feats"]),
                 train_p_mae=float(np.mean(np.abs(Y[:, 0] - T[:, 0]))),
                 **{f"cv_{k}": v for k, v in cvs[steps].items()})
    return net, stats


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sp = ap.add_subparsers(dest="cmd", required=True)
    g = sp.add_parser("generate")
    g.add_argument("--problems", type=int, default=120)
    g.add_argument("--seed", type=int, default=0)
    g.add_argument("--out", required=True)
    g.add_argument("--high-k", action="store_true",
                   help="the high-frequency sweep: k in K_GRID_HIGH, p in P_SWEEP_HIGH")
    m = sp.add_parser("merge")
    m.add_argument("inputs", nargs="+")
    m.add_argument("--out", required=True)
    t = sp.add_parser("train")
    t.add_argument("--data", required=True)
    t.add_argument("--steps", type=int, default=None, help="default: chosen by cross-validation")
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    if a.cmd == "generate":
        kw = dict(k_grid=K_GRID_HIGH, p_sweep=P_SWEEP_HIGH) if a.high_k else {}
        res = generate(a.problems, a.seed, **kw)
        np.savez_compressed(a.out, **res)
    elif a.cmd == "merge":
        res = merge([dict(np.load(f, allow_pickle=False)) for f in a.inputs])
        np.savez_compressed(a.out, **res)
    else:
        data = dict(np.load(a.data, allow_pickle=False))
        net, stats = train(data, a.steps, a.lr)
        print(stats)
        net.save(a.out, **{k: np.float64(v) for k, v in stats.items()})


if __name__ == "__main__":
    main()
