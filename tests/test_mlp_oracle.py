"""CPU checks of the learned-initialiser oracle: its backward pass against
central finite differences of its own loss (FP64, no BF16 rounding), the BF16
rounding helper, and the feature definition on a known answer."""
import numpy as np

from oracle import mlp as M


def test_param_count_matches_layout():
    assert M.param_count() == 16 * 128 + 128 + 2 * (128 * 128 + 128) + 128 * 8 + 8


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -2.5, 0.0], np.float64)
    r = M.bf16(x)
    # 1 + 2^-9 is a tie between 1 and 1 + 2^-7 -> even (1.0)
    assert r[3] == 1.0
    assert r[1] == 1.0  # 1 + 2^-8 rounds down (below the halfway point of 2^-7 steps)
    assert r[2] == 1.0 + 2 ** -7
    assert r[4] == -2.5 and r[5] == 0.0


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    flat = M.init_params(7).astype(np.float64)
    F = rng.normal(size=(24, M.IN))
    T = rng.normal(size=(24, 3))
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    loss, g = M.loss_and_grads(flat, F, T, rounding=False)
    assert np.isfinite(loss)
    # probe a spread of real (non-padding) parameters in every layer
    layers = M.unflatten(np.arange(M.param_count(), dtype=np.float64))
    probes = []
    for l, (W, b) in enumerate(layers):
        rin = M.IN if l == 0 else M.HID
        rout = M.OUT if l == 3 else M.HID
        for _ in range(6):
            probes.append(int(W[rng.integers(rin), rng.integers(rout)]))
        probes.append(int(b[rng.integers(rout)]))
    h = 1e-6
    for i in probes:
        e = np.zeros_like(flat)
        e[i] = h
        lp, _ = M.loss_and_grads(flat + e, F, T, rounding=False)
        lm, _ = M.loss_and_grads(flat - e, F, T, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_padding_gradients_are_zero():
    rng = np.random.default_rng(4)
    flat = M.init_params(1).astype(np.float64)
    F = rng.normal(size=(16, M.IN))
    T = rng.normal(size=(16, 3))
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    _, g = M.loss_and_grads(flat, F, T)
    gl = M.unflatten(g)
    assert np.all(gl[0][0][M.IN:, :] == 0)       # padded inputs
    assert np.all(gl[3][0][:, M.OUT:] == 0)      # padded outputs
    assert np.all(gl[3][1][M.OUT:] == 0)


def test_features_of_a_plane_patch():
    # points on the plane z = 0.2: smallest eigenvalue 0, its eigenvector +-z,
    # eigenvalue fractions summing to 1
    rng = np.random.default_rng(5)
    xy = rng.uniform(-0.05, 0.05, size=(64, 2)) + 0.1
    P = np.column_stack([xy, np.full(64, 0.2)])
    d = ((P[:, None, :] - P[None, :, :]) ** 2).sum(-1)
    nb = np.argsort(d, axis=1, kind="stable")[:, :M.FEATURE_K]
    f, lam, g = M.features(P, nb)
    assert np.allclose(f[:, 2], 0, atol=1e-12)
    assert np.allclose(np.abs(f[:, 5]), 1, atol=1e-9)
    assert np.allclose(f[:, :3].sum(1), 1, atol=1e-12)
    # eigenvectors point away from the bounding-box centre
    assert np.all((f[:, 3:6] * g).sum(1) >= 0) and np.all((f[:, 6:9] * g).sum(1) >= 0)
