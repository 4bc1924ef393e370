"""GPU tests of the learned normal initialiser through the C ABI: features,
forward pass and gradients against the FP64 oracle with BF16 rounding points,
training, parameter files, and the pipeline's use of it."""
import ctypes as C
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import capi, datasets as D  # noqa: E402
from oracle import mlp as M  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda"


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def new_mlp(lib, seed=0):
    h = C.c_void_p()
    capi.check(lib.dwg_mlp_create(seed, None, C.byref(h)))
    return h


def set_params(lib, h, flat):
    flat = np.ascontiguousarray(flat, np.float32)
    capi.check(lib.dwg_mlp_set_params(h, flat.ctypes.data, flat.size))


def get_params(lib, h):
    out = np.empty(lib.dwg_mlp_param_count(), np.float32)
    capi.check(lib.dwg_mlp_get_params(h, out.ctypes.data, out.size))
    return out


def noisy_cloud(n=4000, seed=2):
    P, _ = D.torus(n, seed=seed)
    Pn, _, _ = D.normalize(P)
    return Pn.astype(np.float32)


def gpu_features(lib, P):
    F = torch.empty((len(P), M.IN), dtype=torch.float32, device=DEV)
    Pd = cu(P)
    capi.check(lib.dwg_mlp_features(capi.ptr(Pd), len(P), capi.ptr(F), None))
    torch.cuda.synchronize()
    return F.cpu().numpy()


def test_features_match_oracle(dwg_lib, oracle_lib):
    P = noisy_cloud()
    Fg = gpu_features(dwg_lib, P)
    nb = oracle_lib.knn(P, P, M.FEATURE_K)
    nbw = oracle_lib.knn(P[::M.WIDE_STRIDE], P, M.WIDE_K)
    Fo, lam, g = M.features(P, nb, nbw)
    assert np.isfinite(Fg).all()
    # eigenvalue fractions and centroid offsets: FP64 on both sides
    assert np.abs(Fg[:, :3] - Fo[:, :3]).max() < 2e-5
    assert np.abs(Fg[:, 9:] - Fo[:, 9:]).max() < 2e-5
    # eigenvectors where they are well defined: separated eigenvalues and a
    # clear orientation against the bounding-box centre
    s = lam.sum(1)
    gap3 = (lam[:, 1] - lam[:, 0]) / s
    gap1 = (lam[:, 2] - lam[:, 1]) / s
    ok3 = (gap3 > 1e-2) & (np.abs((Fo[:, 3:6] * g).sum(1)) > 1e-2)
    ok1 = (gap1 > 1e-2) & (np.abs((Fo[:, 6:9] * g).sum(1)) > 1e-2)
    assert ok3.mean() > 0.8 and ok1.mean() > 0.5
    assert np.abs(Fg[ok3, 3:6] - Fo[ok3, 3:6]).max() < 1e-4
    assert np.abs(Fg[ok1, 6:9] - Fo[ok1, 6:9]).max() < 1e-4


def batch(n, seed):
    rng = np.random.default_rng(seed)
    F = rng.normal(size=(n, M.IN)).astype(np.float32)
    T = rng.normal(size=(n, 3))
    T = (T / np.linalg.norm(T, axis=1, keepdims=True)).astype(np.float32)
    return F, T


def test_forward_matches_oracle(dwg_lib):
    flat = M.init_params(11)
    h = new_mlp(dwg_lib)
    try:
        set_params(dwg_lib, h, flat)
        F, _ = batch(5000, 1)
        out = torch.empty((len(F), 3), dtype=torch.float32, device=DEV)
        Fd = cu(F)
        capi.check(dwg_lib.dwg_mlp_forward(h, capi.ptr(Fd), len(F), capi.ptr(out), None))
        yg = out.cpu().numpy().astype(np.float64)
        yo, _ = M.forward(flat, F)
        scale = np.abs(yo).max()
        # FP32 accumulation order and rare one-ulp BF16 flips of activations
        assert np.abs(yg - yo).max() <= 2e-3 * scale
        assert np.sqrt(np.mean((yg - yo) ** 2)) <= 2e-4 * scale
    finally:
        dwg_lib.dwg_mlp_destroy(h)


@pytest.mark.parametrize("n", [64, 3000, 70000])
def test_gradients_match_oracle(dwg_lib, n):
    flat = M.init_params(5)
    h = new_mlp(dwg_lib)
    try:
        set_params(dwg_lib, h, flat)
        F, T = batch(n, n)
        Fd, Td = cu(F), cu(T)
        grads = np.empty(M.param_count(), np.float32)
        loss = C.c_float()
        capi.check(dwg_lib.dwg_mlp_gradients(h, capi.ptr(Fd), capi.ptr(Td), n, C.byref(loss),
                                             grads.ctypes.data, grads.size, None))
        lo, go = M.loss_and_grads(flat, F, T)
        assert abs(loss.value - lo) <= 1e-5 * max(1.0, abs(lo))
        gl, ol = M.unflatten(grads), M.unflatten(go)
        for l in range(4):
            for a, b in zip(gl[l], ol[l]):
                err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
                assert err < 5e-3, (l, err)
        # padding stays exactly zero
        assert np.all(gl[0][0][M.IN:, :] == 0) and np.all(gl[3][0][:, M.OUT:] == 0)
        assert np.all(gl[3][1][M.OUT:] == 0)
    finally:
        dwg_lib.dwg_mlp_destroy(h)


def test_training_reduces_loss(dwg_lib):
    P = noisy_cloud(6000, seed=4)
    F = gpu_features(dwg_lib, P)
    # target: the smallest-eigenvector feature turned by a fixed rotation, a
    # function of the features the network can learn
    c, s = np.cos(0.7), np.sin(0.7)
    R = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], np.float32)
    T = (F[:, 3:6] @ R.T).astype(np.float32)
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    Fd, Td = cu(F), cu(T)
    h = new_mlp(dwg_lib, seed=3)
    try:
        loss = C.c_float()
        losses = []
        for _ in range(300):
            capi.check(dwg_lib.dwg_mlp_train_step(h, capi.ptr(Fd), capi.ptr(Td), len(F), 2e-3, C.byref(loss), None))
            losses.append(loss.value)
        assert np.isfinite(losses).all()
        assert losses[-1] < 0.2 * losses[0], (losses[0], losses[-1])
        assert losses[-1] < 0.1
    finally:
        dwg_lib.dwg_mlp_destroy(h)


def test_param_file_round_trip(dwg_lib, tmp_path):
    h1, h2 = new_mlp(dwg_lib, 1), new_mlp(dwg_lib, 2)
    try:
        path = str(tmp_path / "w.bin").encode()
        capi.check(dwg_lib.dwg_mlp_save(h1, path))
        capi.check(dwg_lib.dwg_mlp_load(h2, path))
        assert np.array_equal(get_params(dwg_lib, h1), get_params(dwg_lib, h2))
        bad = str(tmp_path / "bad.bin").encode()
        with open(bad, "wb") as f:
            f.write(b"DWGMLP01" + np.int64(5).tobytes() + np.zeros(5, np.float32).tobytes())
        assert dwg_lib.dwg_mlp_load(h2, bad) == capi.DWG_ERR_INVALID
        assert dwg_lib.dwg_mlp_set_params(h2, get_params(dwg_lib, h1).ctypes.data, 7) == capi.DWG_ERR_INVALID
    finally:
        dwg_lib.dwg_mlp_destroy(h1)
        dwg_lib.dwg_mlp_destroy(h2)


def test_zero_network_falls_back_to_gauss_map(dwg_lib):
    P = noisy_cloud(3000)
    h = new_mlp(dwg_lib)
    try:
        set_params(dwg_lib, h, np.zeros(M.param_count(), np.float32))
        Pd = cu(P)
        Nl = torch.empty_like(Pd)
        Ng = torch.empty_like(Pd)
        capi.check(dwg_lib.dwg_mlp_init_normals(h, capi.ptr(Pd), len(P), capi.ptr(Nl), None))
        capi.check(dwg_lib.dwg_gauss_map_init(capi.ptr(Pd), len(P), capi.ptr(Ng), None))
        torch.cuda.synchronize()
        assert torch.equal(Nl, Ng)
    finally:
        dwg_lib.dwg_mlp_destroy(h)


def test_learned_pipeline_with_zero_network_equals_plain(dwg_lib):
    P = noisy_cloud(20000, seed=6)
    Pd = cu(P)
    h = new_mlp(dwg_lib)
    set_params(dwg_lib, h, np.zeros(M.param_count(), np.float32))
    res = {}
    try:
        for mode in (3, 4):
            prm = capi.default_params(grid_reso=64, final_reso=64, total_iter=4, in_normal=mode, use_graph=1)
            p = C.c_void_p()
            if mode == 3:
                capi.check(dwg_lib.dwg_pipeline_create(capi.ptr(Pd), None, len(P), C.byref(prm), None, C.byref(p)))
            else:
                capi.check(dwg_lib.dwg_pipeline_create_learned(capi.ptr(Pd), len(P), C.byref(prm), h, None,
                                                               C.byref(p)))
            try:
                capi.check(dwg_lib.dwg_pipeline_iterate(p, 4))
                L = C.c_longlong()
                capi.check(dwg_lib.dwg_pipeline_size(p, b"leaves", C.byref(L)))
                nrm = np.empty((L.value, 3), np.float32)
                capi.check(dwg_lib.dwg_pipeline_get(p, b"leaf_nrm", nrm.ctypes.data))
                res[mode] = nrm
            finally:
                dwg_lib.dwg_pipeline_destroy(p)
        assert np.array_equal(res[3], res[4])
        # in_normal 4 without a network is refused
        prm = capi.default_params(in_normal=4)
        p = C.c_void_p()
        assert dwg_lib.dwg_pipeline_create(capi.ptr(Pd), None, len(P), C.byref(prm), None,
                                           C.byref(p)) == capi.DWG_ERR_INVALID
    finally:
        dwg_lib.dwg_mlp_destroy(h)
