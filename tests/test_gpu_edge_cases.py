"""Edge cases of the GPU path: non-finite and degenerate inputs, empty query
sets, clouds too small for the neighbour counts, duplicated and flat clouds
(the last two against the oracle)."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import capi, datasets as D, turbo  # noqa: E402

pytestmark = pytest.mark.gpu

SMALL = dict(grid_reso=40, final_reso=40, total_iter=3, max_depth=7)


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_non_finite_points_are_rejected(dwg_lib):
    P, _ = D.sphere(2000, seed=3)
    for bad in (np.nan, np.inf):
        Q = P.astype(np.float32).copy()
        Q[777, 1] = bad
        with pytest.raises(capi.DwgError, match="non-finite"):
            turbo.TurboLibiGWN(cu(Q), max_depth=8)
        with pytest.raises(capi.DwgError, match="non-finite"):
            turbo.KnnIndex(cu(Q))
        with pytest.raises(capi.DwgError, match="non-finite"):
            turbo.reconstruct(cu(Q), **SMALL)


def test_empty_query_sets(dwg_lib):
    P, N = D.sphere(3000, seed=4)
    Pd, Nd = cu(P.astype(np.float32)), cu(N.astype(np.float32))
    A = torch.full((len(P),), 2e-6, device="cuda")
    t = turbo.TurboLibiGWN(Pd, max_depth=8, areas=A)
    t.UpdateMassNormals(Nd, A)
    empty = torch.empty((0, 3), dtype=torch.float32, device="cuda")
    assert t.TurboLibiScreenedGWNLaunch(empty).numel() == 0
    assert turbo.KnnIndex(Pd).query(empty, 10).shape == (0, 10)
    # a field that never crosses the iso value has no triangles
    res = np.array([9, 8, 7], np.int32)
    field = torch.zeros(int(np.prod(res)), device="cuda")
    cap = 1000
    tris = torch.empty((cap, 9), device="cuda")
    T = turbo.TurboMC().TurboMarchingCubes(field, None, 9, 8, 7, 0.5, origin=np.zeros(3, np.float32), spacing=0.1,
                                           tris=tris, capacity=cap)
    assert T == 0


def test_cloud_smaller_than_the_neighbour_counts(dwg_lib):
    rng = np.random.default_rng(5)
    P = rng.uniform(-0.5, 0.5, (12, 3)).astype(np.float32)
    with pytest.raises(capi.DwgError, match="neighbours"):
        turbo.reconstruct(cu(P), **SMALL)


@pytest.mark.parametrize("kind", ["duplicated", "flat"])
def test_degenerate_clouds_track_oracle(oracle_lib, kind):
    if kind == "duplicated":
        # every point three times: multi-point leaves, exact kNN ties
        P, _ = D.sphere(2000, noise=0.002, seed=6)
        P = np.repeat(P, 3, axis=0)
    else:
        # a flat disc: no extent in z
        rng = np.random.default_rng(7)
        r, a = np.sqrt(rng.random(6000)), rng.random(6000) * 2 * np.pi
        P = np.stack([r * np.cos(a), r * np.sin(a), np.zeros_like(r)], 1)
    Pn, _, _ = D.normalize(P)
    ref = oracle_lib.reconstruct(Pn, **SMALL)
    got = turbo.reconstruct(cu(Pn), **SMALL)
    assert np.array_equal(got["leaf_pos"], ref["leaf_pos"])
    for k in ("leaf_nrm", "iso", "tris"):
        assert np.all(np.isfinite(got[k])), k
    assert np.allclose(got["iso"][:1], ref["iso"][:1], rtol=1e-4, atol=1e-9)
    assert abs(len(got["tris"]) - len(ref["tris"])) <= 0.01 * len(ref["tris"]) + 4
