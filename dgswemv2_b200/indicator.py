"""Learned troubled-cell indicator: training data, training and evaluation through the library's kernels.

The network (18 -> 64 -> 64 -> 1, ReLU, sigmoid) predicts whether the Cockburn-Shu limiter changes a cell
(the reference limiter's own decision, CS_slope_limiter_serial,
source/problem/SWE/problem_slope_limiter/swe_CS_sl_serial.hpp:9-23). Training data come from
Problem.stage_record (features of the state each limiter pass sees, and that pass's decisions) on
config-3-style bowls with seeded Gaussian humps; training runs the library's FP32 gradient and Adam
kernels (dgsw_mlp_grad, dgsw_mlp_adam); inference inside the step runs on the tensor cores. torch is
used only to hold device buffers and to shuffle/gather minibatches.

    python -m dgswemv2_b200.indicator train --compare-raw --report record.json   # data + training on cuda:0
"""
import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import Problem, _lib, configs

N_PARAM = _lib.DGSW_MLP_NPARAM
N_FEAT = _lib.DGSW_MLP_NFEATURES
N_H = 64
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "indicator_p1.f32")


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the indicator kernels need a CUDA device")
    return torch


def init_params(seed):
    """He-uniform weights, zero biases."""
    rng = np.random.default_rng(seed)
    P = np.zeros(N_PARAM, np.float32)
    o1 = N_H * N_FEAT
    P[:o1] = rng.uniform(-1, 1, o1) * math.sqrt(6.0 / N_FEAT)
    o2 = o1 + N_H
    P[o2:o2 + N_H * N_H] = rng.uniform(-1, 1, N_H * N_H) * math.sqrt(6.0 / N_H)
    o3 = o2 + N_H * N_H + N_H
    P[o3:o3 + N_H] = rng.uniform(-1, 1, N_H) * math.sqrt(6.0 / N_H)
    return P


def load_weights(path=WEIGHTS):
    P = np.fromfile(path, np.float32)
    if P.size != N_PARAM:
        raise ValueError("%s holds %d values, expected %d" % (path, P.size, N_PARAM))
    return P


def forward(x, params, tensor_cores=True):
    """p = MLP(x) for a device tensor x [n][18] (FP32); params a device tensor [5441]."""
    torch = _torch()
    p = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
    _lib.check(_lib.load().dgsw_mlp_forward(C.c_void_p(x.data_ptr()), x.shape[0], C.c_void_p(params.data_ptr()),
                                            C.c_void_p(p.data_ptr()), int(tensor_cores),
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return p


class Trainer:
    """Adam on the FP32 master parameters with the library's gradient and update kernels."""

    def __init__(self, params, lr=2e-3, betas=(0.9, 0.999), eps=1e-8, max_batch=1 << 16):
        torch = _torch()
        self.torch = torch
        self.P = torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda()
        self.m = torch.zeros_like(self.P)
        self.v = torch.zeros_like(self.P)
        self.g = torch.zeros_like(self.P)
        self.loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        self.work = torch.empty(int(_lib.load().dgsw_mlp_grad_work_floats(max_batch)), dtype=torch.float32,
                                device="cuda")
        self.max_batch = max_batch
        self.lr, self.betas, self.eps = lr, betas, eps
        self.t = 0

    def grad(self, x, y, pos_weight):
        assert x.shape[0] <= self.max_batch
        lib = _lib.load()
        s = C.c_void_p(self.torch.cuda.current_stream().cuda_stream)
        _lib.check(lib.dgsw_mlp_grad(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.shape[0],
                                     C.c_void_p(self.P.data_ptr()), float(pos_weight), C.c_void_p(self.g.data_ptr()),
                                     C.c_void_p(self.work.data_ptr()), self.work.numel(),
                                     C.c_void_p(self.loss.data_ptr()), s))
        return self.g

    def step(self, x, y, pos_weight):
        self.grad(x, y, pos_weight)
        self.t += 1
        s = C.c_void_p(self.torch.cuda.current_stream().cuda_stream)
        _lib.check(_lib.load().dgsw_mlp_adam(C.c_void_p(self.P.data_ptr()), C.c_void_p(self.m.data_ptr()),
                                             C.c_void_p(self.v.data_ptr()), C.c_void_p(self.g.data_ptr()), self.t,
                                             self.lr, self.betas[0], self.betas[1], self.eps, s))

    def params(self):
        return self.P.cpu().numpy().copy()


def record(nq=256, seeds=range(8), steps=400, every=4, keep=0.035, dt=0.25, precision="fp32", seed=0,
           feature_sets=(0,)):
    """Features and labels of the cells the limiter looks at, from bowl runs with random Gaussian humps:
    every `every`-th stage of `steps` SSP-RK2 steps, a random `keep` fraction of those cells. With several
    feature sets, one run per set steps in lockstep (the runs are deterministic: identical states and
    labels) and each gives its features for the same cells. Returns ([X per feature set], y)."""
    torch = _torch()
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    Xs, ys = [[] for _ in feature_sets], []
    for sd in seeds:
        mesh, cfg = configs.bowl_humps(nq=nq, seed=int(sd), dt=dt, precision=precision)
        runs = []
        for fs in feature_sets:
            P = Problem(cfg, mesh)
            P.set_indicator_features(fs)
            runs.append((P, torch.empty((P.ne, N_FEAT), dtype=torch.float32, device="cuda"),
                         torch.empty(P.ne, dtype=torch.uint8, device="cuda")))
        ne = runs[0][0].ne
        for st in range(steps * cfg.rk_nstages):
            for P, feat, lab in runs:
                P.stage_record(feat.data_ptr(), lab.data_ptr())
            if st % every:
                continue
            lab = runs[0][2]
            for _, _, other in runs[1:]:
                assert torch.equal(other, lab), "lockstep runs diverged"
            sel = (lab != 255) & (torch.rand(ne, generator=g, device="cuda") < keep)
            for i, (_, feat, _) in enumerate(runs):
                Xs[i].append(feat[sel].clone())
            ys.append(lab[sel].clone())
        for P, _, _ in runs:
            P.close()
    return [torch.cat(x) for x in Xs], torch.cat(ys)


def normalisation(X):
    """Per-feature mean and standard deviation of a training set (FP64 sums; 1 for a constant feature)."""
    torch = _torch()
    Xd = X.double()
    mu, sd = Xd.mean(0), Xd.std(0)
    sd = torch.where(sd > 0, sd, torch.ones_like(sd))
    return mu.float(), sd.float()


def fold_normalisation(params, mu, sd):
    """A network trained on (x - mu) / sd as a network on x: W1' = W1 / sd, b1' = b1 - W1' mu."""
    P = np.asarray(params, np.float64).copy()
    W1 = P[:N_H * N_FEAT].reshape(N_H, N_FEAT)
    b1 = P[N_H * N_FEAT:N_H * N_FEAT + N_H]
    mu = np.asarray(mu, np.float64)
    sd = np.asarray(sd, np.float64)
    W1n = W1 / sd[None, :]
    P[:N_H * N_FEAT] = W1n.ravel()
    P[N_H * N_FEAT:N_H * N_FEAT + N_H] = b1 - W1n @ mu
    return P.astype(np.float32)


def metrics(p, y, confidence=0.9):
    """Gate statistics at a confidence: fraction of cells sent to the limiter, miss rate (limited cells
    the gate skips, over all limited cells), accuracy at 0.5."""
    skip = p < (1.0 - confidence)
    pos = y == 1
    npos = int(pos.sum())
    return {
        "cells": int(y.numel()),
        "positive_fraction": npos / max(1, int(y.numel())),
        "sent_fraction": float((~skip).float().mean()),
        "miss_rate": int((skip & pos).sum()) / max(1, npos),
        "accuracy": float(((p >= 0.5) == pos).float().mean()),
    }


def train(X, y, Xv=None, yv=None, epochs=8, batch=8192, lr=2e-3, seed=0, log=print):
    torch = _torch()
    n = X.shape[0]
    npos = int((y == 1).sum())
    pos_weight = float(min(20.0, max(1.0, (n - npos) / max(1, npos))))
    T = Trainer(init_params(seed), lr=lr, max_batch=batch)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    steps_per_epoch = n // batch
    hist = []
    t0 = time.time()
    for ep in range(epochs):
        # cosine learning-rate decay over the run
        perm = torch.randperm(n, generator=g, device="cuda")
        for b in range(steps_per_epoch):
            k = ep * steps_per_epoch + b
            T.lr = lr * 0.5 * (1.0 + math.cos(math.pi * k / (epochs * steps_per_epoch)))
            idx = perm[b * batch:(b + 1) * batch]
            T.step(X[idx].contiguous(), y[idx].contiguous(), pos_weight)
        rec = {"epoch": ep, "loss": float(T.loss.item()), "seconds": time.time() - t0}
        if Xv is not None:
            Pd = T.P
            rec.update(metrics(forward(Xv, Pd, tensor_cores=True), yv))
        hist.append(rec)
        log(json.dumps(rec))
    return T.params(), {"pos_weight": pos_weight, "history": hist, "train_cells": n}


def evaluate(params, nq=1024, steps=200, dt=0.06, confidence=0.9, precision="fp32", warmup=3, feature_set=0):
    """Config-4 inference: Thacker bowl on nq x nq quads (2 nq^2 triangles), p = 1, SSP-RK2, wetting and
    drying. Runs the same `steps` from t = 0 with no limiter, the plain limiter, the MLP-gated limiter and
    the shadow mode (plain decisions, gate misses counted); reports device time per step after `warmup`
    steps, the L2 error against the analytic solution, the miss rate and the fraction of cells sent to
    the limiter."""
    mesh, cfg = configs.config3(nq=nq, dt=dt, precision=precision)
    out = {"elements": mesh.n_elems, "steps": steps, "dt": dt, "confidence": confidence, "precision": precision}
    for name, lim, mode in (("no_limiter", False, 0), ("plain", True, 0), ("gated", True, 1), ("shadow", True, 2)):
        cfg.slope_limiting = lim
        P = Problem(cfg, mesh)
        if mode:
            P.set_indicator_features(feature_set)
            P.set_indicator(params, confidence=confidence, mode=mode)
        P.step_serial(warmup)
        if mode:
            P.indicator_stats(reset=True)
        P.step_serial(steps - warmup)
        ms, launches = P.last_step_timing()
        r = {"ms_per_step": ms / (steps - warmup), "l2_error": P.compute_residual_L2(), "launches": launches}
        if mode:
            considered, sent, limited, missed = P.indicator_stats()
            r.update({"considered": considered, "sent": sent, "limited": limited, "missed": missed,
                      "sent_fraction": sent / max(1, considered)})
            if mode == 2:
                r["miss_rate"] = missed / max(1, limited + missed)
        out[name] = r
        P.close()
    base = out["no_limiter"]["ms_per_step"]
    out["limiter_ms_plain"] = out["plain"]["ms_per_step"] - base
    out["limiter_ms_gated"] = out["gated"]["ms_per_step"] - base
    out["l2_added_by_gate"] = out["gated"]["l2_error"] / out["plain"]["l2_error"] - 1.0
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--nq", type=int, default=256)
    ap.add_argument("--runs", type=int, default=17)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--epochs", type=int, default=16)
    ap.add_argument("--keep", type=float, default=0.035)
    ap.add_argument("--report", default=None)
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--eval-nq", type=int, default=1024)
    ap.add_argument("--eval-steps", type=int, default=200)
    ap.add_argument("--compare-raw", action="store_true",
                    help="also train on the raw feature set (same cells) and report both")
    a = ap.parse_args()
    if a.cmd == "evaluate":
        print(json.dumps(evaluate(load_weights(a.weights), nq=a.eval_nq, steps=a.eval_steps)), flush=True)
        return
    torch = _torch()
    sets = (0, 1) if a.compare_raw else (0,)
    t0 = time.time()
    Xs, y = record(nq=a.nq, seeds=range(a.runs), steps=a.steps, keep=a.keep, feature_sets=sets)
    Xvs, yv = record(nq=a.nq, seeds=range(1000, 1002), steps=a.steps, keep=a.keep, seed=1, feature_sets=sets)
    rep = {"train_cells": int(y.numel()), "val_cells": int(yv.numel()), "record_seconds": time.time() - t0}
    print(json.dumps(rep), flush=True)
    for fs, X, Xv in zip(sets, Xs, Xvs):
        name = "characteristic" if fs == 0 else "raw"
        if fs == 1:
            # the raw set is trained on standardised inputs; the standardisation is then folded into the
            # first layer so that the network reads the raw features
            mu, sd = normalisation(X)
            P, info = train((X - mu) / sd, y, (Xv - mu) / sd, yv, epochs=a.epochs)
            P = fold_normalisation(P, mu.cpu().numpy(), sd.cpu().numpy())
        else:
            P, info = train(X, y, Xv, yv, epochs=a.epochs)
        Pd = torch.from_numpy(P).cuda()
        info["validation_fp32"] = metrics(forward(Xv, Pd, tensor_cores=False), yv)
        info["validation_tensor_cores"] = metrics(forward(Xv, Pd, tensor_cores=True), yv)
        rep[name] = info
        out = a.out if fs == 0 else a.out.replace(".f32", "_raw.f32")
        os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
        P.astype(np.float32).tofile(out)
        rep[name]["weights"] = os.path.basename(out)
        rep[name]["config4"] = evaluate(P, nq=a.eval_nq, steps=a.eval_steps, feature_set=fs)
        print(json.dumps({name: {k: rep[name][k] for k in ("validation_fp32", "validation_tensor_cores")}}), flush=True)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
