"""Seeded synthetic point clouds with the shapes of the benchmark configurations.

The reference's README names no dataset; every workload here is procedural:

* ``sphere``   -- points uniform on the unit sphere, isotropic Gaussian noise.
* ``torus``    -- torus (R, r) sampled by area with density 1 + 0.8 sin(3 theta)
                  (theta = toroidal angle), noise along the true normal.
* ``superquadric_union`` -- union of seeded superquadrics (exponents, semi-axes,
                  rotations, centres random); only points outside every other
                  solid are kept; optional uniform outliers in the bbox.
* ``batch``    -- many clouds of log-uniform size drawn from the three families.

Positions are returned as float32 arrays of shape (n, 3) together with the
true outward normals (float32), and are NOT normalised: ``normalize`` applies
the reference's reader normalisation (include/DWGProcess.h:53-97).
"""
from __future__ import annotations

import numpy as np


def normalize(P):
    """Centre on the mean and divide by max_ij 2|x_ij| (include/DWGProcess.h:53-97).

    Carried in float64 like the reference reader, returned as float32."""
    P = np.asarray(P, np.float64)
    c = P.mean(axis=0)
    Q = P - c
    scale = float(np.max(2.0 * np.abs(Q))) if len(Q) else 1.0
    if scale == 0.0:
        scale = 1.0
    return (Q / scale).astype(np.float32), c, scale


def sphere(n, noise=0.002, seed=0):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    P = d + noise * rng.standard_normal((n, 3))
    return P.astype(np.float32), d.astype(np.float32)


def torus(n, R=1.0, r=0.35, noise=0.003, seed=0):
    """Area-uniform (Jacobian R + r cos phi) times density 1 + 0.8 sin(3 theta),
    by rejection; Gaussian noise of sigma ``noise`` along the true normal."""
    rng = np.random.default_rng(seed)
    out_p, out_n, have = [], [], 0
    wmax = (R + r) * 1.8
    while have < n:
        m = max(1024, 2 * (n - have) * 3)
        th = rng.uniform(0, 2 * np.pi, m)
        ph = rng.uniform(0, 2 * np.pi, m)
        w = (R + r * np.cos(ph)) * (1.0 + 0.8 * np.sin(3 * th))
        keep = rng.uniform(0, wmax, m) < w
        th, ph = th[keep], ph[keep]
        nrm = np.stack([np.cos(ph) * np.cos(th), np.cos(ph) * np.sin(th), np.sin(ph)], 1)
        ctr = np.stack([R * np.cos(th), R * np.sin(th), np.zeros_like(th)], 1)
        p = ctr + r * nrm + noise * rng.standard_normal((len(th), 1)) * nrm
        out_p.append(p)
        out_n.append(nrm)
        have += len(th)
    P = np.concatenate(out_p)[:n]
    N = np.concatenate(out_n)[:n]
    return P.astype(np.float32), N.astype(np.float32)


def _rand_rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def _sq_params(rng, k):
    return [dict(e1=rng.uniform(0.3, 3.0), e2=rng.uniform(0.3, 3.0),
                 a=rng.uniform(0.05, 1.0, 3), R=_rand_rotation(rng),
                 c=rng.uniform(-1.0, 1.0, 3)) for _ in range(k)]


def _sq_surface(rng, p, m):
    """m samples on one superquadric surface, approximately area-uniform:
    oversample the parametric surface and keep by local area element."""
    def fexp(x, e):
        return np.sign(x) * np.abs(x) ** e
    M = 4 * m
    eta = rng.uniform(-np.pi / 2, np.pi / 2, M)
    om = rng.uniform(-np.pi, np.pi, M)
    a, e1, e2 = p["a"], p["e1"], p["e2"]

    def X(eta, om):
        return np.stack([a[0] * fexp(np.cos(eta), e1) * fexp(np.cos(om), e2),
                         a[1] * fexp(np.cos(eta), e1) * fexp(np.sin(om), e2),
                         a[2] * fexp(np.sin(eta), e1)], 1)
    h = 1e-4
    x0 = X(eta, om)
    de = (X(eta + h, om) - x0) / h
    do = (X(eta, om + h) - x0) / h
    dA = np.linalg.norm(np.cross(de, do), axis=1)
    dA = np.nan_to_num(dA, nan=0.0, posinf=0.0)
    cap = np.quantile(dA, 0.99) + 1e-12
    keep = rng.uniform(0, cap, M) < np.minimum(dA, cap)
    x0 = x0[keep][:m]
    nrm = np.cross(de[keep][:m], do[keep][:m])
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True) + 1e-30
    out = x0 @ p["R"].T + p["c"]
    nrm = nrm @ p["R"].T
    # orient away from the solid: flip where a small step along n goes inside
    ins_plus = _sq_inside(out + 1e-3 * nrm, p) < 1.0
    nrm[ins_plus] *= -1
    return out, nrm


def _sq_inside(x, p, local=False):
    """Superquadric inside-outside function F(x) (< 1 inside)."""
    if not local:
        x = (x - p["c"]) @ p["R"]
    a, e1, e2 = p["a"], p["e1"], p["e2"]
    t = (np.abs(x[:, 0] / a[0]) ** (2 / e2) + np.abs(x[:, 1] / a[1]) ** (2 / e2)) ** (e2 / e1)
    return t + np.abs(x[:, 2] / a[2]) ** (2 / e1)


def superquadric_union(n, k=12, outlier_frac=0.01, noise=0.0, seed=0):
    """``n`` surface points of the union of ``k`` seeded superquadrics plus
    ``round(n * outlier_frac)`` uniform outliers in the bounding box."""
    rng = np.random.default_rng(seed)
    sq = _sq_params(rng, k)
    areas = []
    for p in sq:
        a = p["a"]
        # ellipsoid surface area, Knud Thomsen's approximation (p = 1.6)
        areas.append(4 * np.pi * (((a[0] * a[1]) ** 1.6 + (a[0] * a[2]) ** 1.6 + (a[1] * a[2]) ** 1.6) / 3)
                     ** (1 / 1.6))
    areas = np.array(areas)
    outP, outN, have = [], [], 0
    while have < n:
        need = n - have
        per = np.maximum(1, np.round(2.0 * need * areas / areas.sum()).astype(int))
        for i, p in enumerate(sq):
            x, nr = _sq_surface(rng, p, int(per[i]))
            keep = np.ones(len(x), bool)
            for j, q in enumerate(sq):
                if j != i:
                    keep &= _sq_inside(x, q) >= 1.0
            x, nr = x[keep], nr[keep]
            if noise > 0:
                x = x + noise * rng.standard_normal((len(x), 1)) * nr
            outP.append(x)
            outN.append(nr)
            have += len(x)
    P = np.concatenate(outP)
    N = np.concatenate(outN)
    sel = rng.permutation(len(P))[:n]
    P, N = P[sel], N[sel]
    no = int(round(n * outlier_frac))
    if no:
        lo, hi = P.min(0), P.max(0)
        O = rng.uniform(lo, hi, (no, 3))
        On = rng.standard_normal((no, 3))
        On /= np.linalg.norm(On, axis=1, keepdims=True)
        P = np.concatenate([P, O])
        N = np.concatenate([N, On])
    return P.astype(np.float32), N.astype(np.float32)


def random_cloud(rng, lo, hi, kinds=3):
    """One cloud of log-uniform size in [lo, hi] from {sphere, torus,
    3-superquadric union} (``kinds=4`` adds unions of 4-12 superquadrics with
    1% outliers), noise sigma uniform in [0.001, 0.01]."""
    n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    kind = int(rng.integers(0, kinds))
    sig = float(rng.uniform(0.001, 0.01))
    s = int(rng.integers(0, 2**31))
    if kind == 0:
        P, N = sphere(n, noise=sig, seed=s)
    elif kind == 1:
        P, N = torus(n, noise=sig, seed=s)
    elif kind == 2:
        P, N = superquadric_union(n, k=3, outlier_frac=0.0, noise=sig, seed=s)
    else:
        k = int(rng.integers(4, 13))
        m = int(round(n / 1.01))
        P, N = superquadric_union(m, k=k, outlier_frac=0.01, noise=sig, seed=s)
    return dict(points=P, normals=N, kind=kind, noise=sig)


def batch(count=64, lo=2000, hi=200000, seed=0):
    """Clouds of log-uniform size from {sphere, torus, 3-superquadric union},
    noise sigma uniform in [0.001, 0.01]; per-cloud grid resolution
    clamp(round(128 (n/2000)^(1/3)), 128, 256)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        c = random_cloud(rng, lo, hi)
        n = len(c["points"])
        c["grid_reso"] = int(np.clip(round(128 * (n / 2000.0) ** (1 / 3)), 128, 256))
        out.append(c)
    return out


def random_normals(n, seed=0):
    """GetRandomNs (include/DWGProcess.h:264-281) with a seed: u, v uniform in
    [0, 2 pi), n = (sin u cos v, sin u sin v, cos u)."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(0, 2 * np.pi, n)
    v = rng.uniform(0, 2 * np.pi, n)
    return np.stack([np.sin(u) * np.cos(v), np.sin(u) * np.sin(v), np.cos(u)], 1).astype(np.float32)


CONFIGS = {
    "c1_sphere_10k": dict(kind="sphere", n=10_000, noise=0.002, grid_reso=128, final_reso=128,
                          total_iter=30),
    "c2_torus_100k": dict(kind="torus", n=100_000, noise=0.003, grid_reso=256, final_reso=256,
                          total_iter=30),
    "c3_sq_union_1m": dict(kind="sq_union", n=1_000_000, grid_reso=256, final_reso=256,
                           total_iter=30),
}


def make(config, seed=0):
    c = CONFIGS[config]
    if c["kind"] == "sphere":
        return sphere(c["n"], c["noise"], seed)
    if c["kind"] == "torus":
        return torus(c["n"], noise=c["noise"], seed=seed)
    return superquadric_union(c["n"], seed=seed)
