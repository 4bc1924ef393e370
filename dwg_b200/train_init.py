"""Train and evaluate the learned normal initialiser on the GPU.

Training data are DWG-converged leaf normals: each seeded procedural cloud
(sphere, torus, superquadric unions, with noise and outliers) is reconstructed
by the plain pipeline (Gauss-map start, an even number of iterations, so that
the converged normals keep the start's orientation convention), and the
network learns to map the covariance features of each leaf to its converged
normal.  Forward, backward and Adam steps are the library's own kernels.

Usage::

    python -m dwg_b200.train_init --shapes 2000 --min-points 50000 \\
        --max-points 500000 --out dwg_b200/weights/normal_init.bin

``--shapes`` sets how many clouds are generated (the full recipe is 2000).
``evaluate()`` measures how many DWG iterations the plain and the learned
start need to bring the winding field within a tolerance of the plain
method's converged field.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "normal_init.bin")


def _torch():
    import torch
    return torch


def converged_leaves(P, grid, iters, dev):
    """Leaf positions and DWG-converged leaf normals of cloud P (host)."""
    from . import turbo
    torch = _torch()
    assert iters % 2 == 0, "an even iteration count keeps the start's orientation"
    Pd = torch.from_numpy(np.ascontiguousarray(P, np.float32)).to(dev)
    d = turbo.TurboDWG(Pd, None, grid_reso=grid, final_reso=grid, total_iter=iters, use_graph=1)
    try:
        d.TurboScreenedDWGLaunch(iters)
        pos = torch.from_numpy(d.get("leaf_pos")).to(dev)
        nrm = torch.from_numpy(d.get("leaf_nrm")).to(dev)
    finally:
        d.close()
    return pos, nrm


def make_dataset(shapes, lo, hi, grid, iters, seed, dev, log=print):
    """Features [M x 12] and targets [M x 3] (device) of `shapes` clouds."""
    from . import datasets as D
    from .turbo import LearnedNormalInit
    torch = _torch()
    rng = np.random.default_rng(seed)
    feats, tgts, sizes = [], [], []
    t0 = time.time()
    for i in range(shapes):
        c = D.random_cloud(rng, lo, hi, kinds=4)
        P, _, _ = D.normalize(c["points"])
        pos, nrm = converged_leaves(P.astype(np.float32), grid, iters, dev)
        F = LearnedNormalInit.features(pos)
        ok = torch.isfinite(F).all(1) & (nrm.norm(dim=1) > 0.5)
        feats.append(F[ok])
        tgts.append(nrm[ok])
        sizes.append(int(ok.sum()))
        if (i + 1) % max(1, shapes // 10) == 0:
            log(f"  shape {i + 1}/{shapes}: {sum(sizes)} leaves, {time.time() - t0:.0f} s")
    return torch.cat(feats), torch.cat(tgts), sizes


def train(model, X, Y, epochs, batch, lr, seed, log=print, Xv=None, Yv=None):
    """Adam on minibatches, cosine-decayed learning rate; returns the history."""
    torch = _torch()
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    M = X.shape[0]
    steps = epochs * math.ceil(M / batch)
    hist, k = [], 0
    for ep in range(epochs):
        perm = torch.randperm(M, device=X.device, generator=g)
        tot, cnt = 0.0, 0
        for b0 in range(0, M, batch):
            idx = perm[b0:b0 + batch]
            if idx.numel() < 2:
                continue
            lr_k = lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * k / max(1, steps))))
            loss = model.train_step(X[idx].contiguous(), Y[idx].contiguous(), lr_k)
            tot += loss * idx.numel()
            cnt += idx.numel()
            k += 1
        rec = {"epoch": ep, "train_loss": tot / max(cnt, 1)}
        if Xv is not None and Xv.shape[0]:
            rec["val_loss"] = val_loss(model, Xv, Yv)
        hist.append(rec)
        log("  " + json.dumps(rec))
    return hist


def val_loss(model, X, Y):
    torch = _torch()
    y = model.forward(X)
    yh = y / (y.norm(dim=1, keepdim=True) + 1e-12)
    return float((1 - (yh * Y).sum(1)).mean())


def _rms_sign(w, ref):
    """RMS distance of w to +ref or -ref (orientation flips between iterations)."""
    a = float(np.sqrt(np.mean((w - ref) ** 2)))
    b = float(np.sqrt(np.mean((w + ref) ** 2)))
    return min(a, b)


def evaluate(P, model, grid=256, iters=40, tol=1e-4, dev="cuda", precision=1):
    """Iterations and device time the plain (Gauss map) and the learned start
    need before the iteration grid field is within RMS `tol` of the plain
    method's field after `iters` iterations (sign-matched).  Returns a dict."""
    from . import turbo
    torch = _torch()
    Pd = torch.from_numpy(np.ascontiguousarray(P, np.float32)).to(dev)
    flags = dict(grid_reso=grid, final_reso=grid, total_iter=iters, use_graph=1, precision=precision)
    ref = turbo.TurboDWG(Pd, None, **flags)
    ref.TurboScreenedDWGLaunch(iters)
    w_ref = ref.get("field")
    ref.close()
    out = {"tol": tol, "iters_ref": iters, "grid": grid, "points": int(len(P))}
    for name, m in (("plain", None), ("learned", model)):
        d = turbo.TurboDWG(Pd, None, init_model=m, **flags)
        errs = []
        for t in range(iters):
            d.TurboScreenedDWGLaunch(1)
            errs.append(_rms_sign(d.get("field"), w_ref))
        d.close()
        conv = next((t + 1 for t, e in enumerate(errs) if e <= tol), None)
        # device time of create + conv iterations, without host reads
        ms = None
        if conv is not None:
            s = torch.cuda.current_stream()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            d = turbo.TurboDWG(Pd, None, init_model=m, **flags)
            d.TurboScreenedDWGLaunch(conv)
            e1.record(s)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            d.close()
        out[name] = {"iters_to_tol": conv, "ms_to_tol": ms, "rms_err": errs}
    p, l = out["plain"], out["learned"]
    if p["iters_to_tol"] and l["iters_to_tol"]:
        out["iter_ratio"] = p["iters_to_tol"] / l["iters_to_tol"]
        out["time_ratio"] = p["ms_to_tol"] / l["ms_to_tol"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--shapes", type=int, default=2000)
    ap.add_argument("--min-points", type=int, default=50000)
    ap.add_argument("--max-points", type=int, default=500000)
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--iters", type=int, default=30)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=32768)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--val-frac", type=float, default=0.05)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--report", default=None, help="write the training history (JSON) here")
    ap.add_argument("--eval-points", type=int, default=0, help="held-out superquadric union size (0: skip)")
    ap.add_argument("--eval-grid", type=int, default=256)
    ap.add_argument("--eval-iters", type=int, default=40)
    a = ap.parse_args(argv)

    from . import build, datasets as D
    from .turbo import LearnedNormalInit
    build.build()
    torch = _torch()
    dev = torch.device("cuda")
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731

    t0 = time.time()
    log(f"generating {a.shapes} shapes ({a.min_points}-{a.max_points} points, grid {a.grid}, {a.iters} iters)")
    X, Y, sizes = make_dataset(a.shapes, a.min_points, a.max_points, a.grid, a.iters, a.seed, dev, log)
    t_data = time.time() - t0
    nv = int(round(len(sizes) * a.val_frac))
    cut = sum(sizes[: len(sizes) - nv])
    Xt, Yt, Xv, Yv = X[:cut], Y[:cut], X[cut:], Y[cut:]
    log(f"{X.shape[0]} samples ({Xt.shape[0]} train, {Xv.shape[0]} validation), {t_data:.0f} s")
    model = LearnedNormalInit(seed=a.seed)
    base = val_loss(model, Xv, Yv) if Xv.shape[0] else None
    # the Gauss map's loss on the validation set, for scale
    t1 = time.time()
    hist = train(model, Xt, Yt, a.epochs, a.batch, a.lr, a.seed, log, Xv, Yv)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    model.save(a.out)
    rep = {"shapes": a.shapes, "points": [a.min_points, a.max_points], "grid": a.grid, "iters": a.iters,
           "samples": int(X.shape[0]), "epochs": a.epochs, "batch": a.batch, "lr": a.lr, "seed": a.seed,
           "val_loss_untrained": base, "history": hist, "data_s": t_data, "train_s": t_train, "out": a.out}
    if a.eval_points:
        P, _ = D.superquadric_union(a.eval_points, seed=10_000 + a.seed)
        P, _, _ = D.normalize(P)
        rep["eval"] = evaluate(P.astype(np.float32), model, a.eval_grid, a.eval_iters)
        e = rep["eval"]
        log(f"eval: plain {e['plain']['iters_to_tol']} iters / {e['plain']['ms_to_tol']} ms, "
            f"learned {e['learned']['iters_to_tol']} iters / {e['learned']['ms_to_tol']} ms")
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f, indent=1)
    print(json.dumps({k: v for k, v in rep.items() if k not in ("history", "eval")}))


if __name__ == "__main__":
    main()
