"""CPU oracle of the learned normal initialiser (test infrastructure only).

The reference has no learned part: the initialiser replaces the Gauss map of
``TurboNormalInitialization::GaussMapInit`` (src/TurboNormalInit.cu:3-44) as
the source of the leaves' initial normals, so this module restates the
library's own definition of it in FP64 NumPy and is pinned by central finite
differences of its own loss, not by reference fixtures (parity unpinned by the
reference, which has no such component).

Definition restated (the CUDA side is dwg_b200/csrc/mlp.cu):
  features (12): eigenvalues l1 >= l2 >= l3 of the covariance of the 16
    nearest points (self included) over l1+l2+l3; the eigenvector of l3 and of
    l1, each with a non-negative dot product with the unit direction from the
    bounding-box centre to the point; (centroid_w - point) / spread_w over the
    wide neighbourhood: the 64 nearest points of the subsample S = P[::4],
    spread_w their RMS distance to centroid_w.
  network: 12 (padded 16) -> 128 -> 128 -> 128 -> 3 (padded 8), GELU with erf
    after the hidden layers.  Inputs, weights and hidden activations are
    rounded to BF16 (round to nearest even) where they feed a product; the
    products accumulate exactly here (FP32 on the GPU).
  loss: mean over the batch of 1 - <y/(|y|+1e-12), t>.
  backward: dY rounded to BF16; the bias gradient of a hidden layer sums the
    unrounded dZ, its weight gradient uses dZ rounded to BF16; dH = dZ_bf16 @
    W_bf16^T.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

IN, IN_PAD, HID, OUT, OUT_PAD = 12, 16, 128, 3, 8
DIN = (IN_PAD, HID, HID, HID)
DOUT = (HID, HID, HID, OUT_PAD)
FEATURE_K = 16


def param_count() -> int:
    return sum(a * b + b for a, b in zip(DIN, DOUT))


def unflatten(flat):
    """flat -> [(W [din x dout], b [dout])] in float64."""
    flat = np.asarray(flat, np.float64)
    out, o = [], 0
    for din, dout in zip(DIN, DOUT):
        W = flat[o:o + din * dout].reshape(din, dout)
        o += din * dout
        b = flat[o:o + dout]
        o += dout
        out.append((W, b))
    assert o == flat.size
    return out


def flatten(layers):
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in layers])


def bf16(x):
    """Round to BF16 (nearest even) through FP32, as __float2bfloat16_rn."""
    x32 = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    u = x32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def _round(x, on):
    return bf16(x) if on else np.asarray(x, np.float64)


def forward(flat, F, rounding=True):
    """Raw outputs [n x 3] and the cache of the backward pass."""
    layers = unflatten(flat)
    n = F.shape[0]
    X = np.zeros((n, IN_PAD))
    X[:, :IN] = F
    X = _round(X, rounding)
    acts, zs = [X], []
    h = X
    for l, (W, b) in enumerate(layers):
        z = h @ _round(W, rounding) + b
        zs.append(z)
        if l < len(layers) - 1:
            h = _round(gelu(z), rounding)
            acts.append(h)
    return zs[-1][:, :OUT], (layers, acts, zs)


def loss_and_grads(flat, F, T, rounding=True):
    """(loss, flat gradient) of mean(1 - cos) as the GPU computes them."""
    y, (layers, acts, zs) = forward(flat, F, rounding)
    n = F.shape[0]
    nn = np.sqrt((y * y).sum(1)) + 1e-12
    yh = y / nn[:, None]
    c = (yh * T).sum(1)
    loss = float(np.mean(1.0 - c))
    dy = np.zeros((n, OUT_PAD))
    dy[:, :OUT] = -(T - c[:, None] * yh) / nn[:, None] / n
    dzb = _round(dy, rounding)
    dz = dzb
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        gb = dz.sum(0)
        gW = acts[l].T @ dzb
        grads[l] = (gW, gb)
        if l == 0:
            break
        dh = dzb @ _round(W, rounding).T
        dz = dh * gelu_grad(zs[l - 1])
        dzb = _round(dz, rounding)
    return loss, flatten(grads)


def init_params(seed: int):
    """A random parameter vector with zero padding (test inputs only)."""
    rng = np.random.default_rng(seed)
    layers = []
    real_in = (IN, HID, HID, HID)
    real_out = (HID, HID, HID, OUT)
    for l, (din, dout) in enumerate(zip(DIN, DOUT)):
        W = np.zeros((din, dout))
        lim = np.sqrt(6.0 / real_in[l])
        W[:real_in[l], :real_out[l]] = rng.uniform(-lim, lim, (real_in[l], real_out[l]))
        b = np.zeros(dout)
        b[:real_out[l]] = rng.uniform(-0.1, 0.1, real_out[l])
        layers.append((W, b))
    return flatten(layers).astype(np.float32)


WIDE_K, WIDE_STRIDE = 64, 4


def features(P, nb, nbw=None):
    """Features [n x 12] of points P [n x 3] from neighbour ids nb [n x k]
    and wide-neighbourhood ids nbw [n x kw] into P[::4] (None: the
    16-neighbourhood itself, for the known-answer tests)."""
    P = np.asarray(P, np.float64)
    lo = np.asarray(P.min(0), np.float32).astype(np.float64)
    hi = np.asarray(P.max(0), np.float32).astype(np.float64)
    centre = 0.5 * (lo + hi)
    Q = P[nb]                                    # n x k x 3
    cen = Q.mean(1)
    D = Q - cen[:, None, :]
    cov = np.einsum("nki,nkj->nij", D, D) / nb.shape[1]
    lam, vec = np.linalg.eigh(cov)               # ascending
    g = P - centre
    gn = np.linalg.norm(g, axis=1, keepdims=True)
    g = np.where(gn > 0, g / np.where(gn > 0, gn, 1), np.array([0.0, 0.0, 1.0]))
    v3 = vec[:, :, 0]
    v1 = vec[:, :, 2]
    v3 = np.where(((v3 * g).sum(1) < 0)[:, None], -v3, v3)
    v1 = np.where(((v1 * g).sum(1) < 0)[:, None], -v1, v1)
    s = np.maximum(lam.sum(1), 1e-30)
    out = np.empty((P.shape[0], IN))
    out[:, 0] = np.maximum(lam[:, 2], 0) / s
    out[:, 1] = np.maximum(lam[:, 1], 0) / s
    out[:, 2] = np.maximum(lam[:, 0], 0) / s
    out[:, 3:6] = v3
    out[:, 6:9] = v1
    if nbw is None:
        out[:, 9:12] = (cen - P) / np.sqrt(s)[:, None]
    else:
        S = P[::WIDE_STRIDE]
        W = S[nbw]
        cw = W.mean(1)
        sw = np.sqrt(np.maximum(((W - cw[:, None, :]) ** 2).sum(2).mean(1), 1e-30))
        out[:, 9:12] = (cw - P) / sw[:, None]
    return out, lam, g
