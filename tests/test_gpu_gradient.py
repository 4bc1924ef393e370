"""Gradients of the winding-number sums and the FP64 sums on the GPU
(dwg_gwn_points_grad / _grid_grad / _points_fp64 / _grid_fp64) against the
FP64 oracle with the same opening decisions.  The oracle's gradient itself is
checked against central differences in tests/test_oracle.py."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import datasets as D, turbo  # noqa: E402

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def case(oracle_lib):
    P, N = D.torus(20000, seed=21)
    Pn, _, _ = D.normalize(P)
    rng = np.random.default_rng(3)
    A = rng.uniform(1e-6, 3e-6, len(Pn)).astype(np.float32)
    R = rng.uniform(0.001, 0.004, len(Pn)).astype(np.float32)
    Q = np.concatenate([Pn[:4000] + rng.normal(0, 0.01, (4000, 3)),
                        rng.uniform(-0.55, 0.55, (6000, 3))]).astype(np.float32)
    return Pn, N.astype(np.float32), A, R, Q


@pytest.mark.parametrize("screened,sigma,radii", [(True, 20.0, False), (True, 10.0, True), (False, 0.0, False)])
def test_fp64_sums_and_gradients_match_oracle(oracle_lib, case, screened, sigma, radii):
    Pn, N, A, R, Q = case
    tree = turbo.TurboLibiGWN(cu(Pn), max_depth=8, areas=cu(A))
    Rd = cu(R) if radii else None
    tree.UpdateMassNormals(cu(N), cu(A))
    w64, g64 = tree.value_and_gradient(cu(Q), i_Normals=cu(N), i_As=cu(A), i_radii=Rd, beta=2.3, sigma=sigma,
                                       screened=screened, fp64=True)
    w32, g32 = tree.value_and_gradient(cu(Q), i_Normals=cu(N), i_As=cu(A), i_radii=Rd, beta=2.3, sigma=sigma,
                                       screened=screened)
    assert tree.status() == 0
    ot = oracle_lib.Octree(Pn, 8)
    wo, go = ot.gwn_grad(Pn, N, A, Q, beta=2.3, sigma=sigma, screened=screened, radii=R if radii else None)
    w64, g64 = w64.cpu().numpy(), g64.cpu().numpy()
    w32, g32 = w32.cpu().numpy().astype(np.float64), g32.cpu().numpy().astype(np.float64)
    sw, sg = np.abs(wo).max(), np.abs(go).max()
    # FP64 on the GPU = the oracle's FP64 sums up to the order of the additions
    assert np.abs(w64 - wo).max() <= 1e-11 * sw, np.abs(w64 - wo).max() / sw
    assert np.abs(g64 - go).max() <= 1e-11 * sg, np.abs(g64 - go).max() / sg
    # FP32 terms summed in FP64: FP32 rounding of each term
    ew, eg = np.abs(w32 - wo), np.abs(g32 - go)
    assert ew.max() <= 1e-5 * sw and np.sqrt(np.mean(ew ** 2)) <= 1e-6 * sw, (ew.max() / sw)
    assert eg.max() <= 1e-4 * sg and np.sqrt(np.mean(eg ** 2)) <= 1e-5 * sg, (eg.max() / sg)
    # the values equal the warp kernels' sums to FP32 rounding
    if not radii:
        out = torch.empty(len(Q), dtype=torch.float32, device="cuda")
        if screened:
            tree.TurboLibiScreenedGWNLaunch(cu(Q), None, len(Q), None, None, None, 2.3, sigma, out)
        else:
            tree.TurboLibiGWNLaunch(cu(Q), None, len(Q), None, None, 2.3, out)
        wk = out.cpu().numpy().astype(np.float64)
        assert np.abs(wk - wo).max() <= 1e-5 * sw


def test_grid_fp64_and_gradient_match_points(oracle_lib, case):
    Pn, N, A, R, Q = case
    tree = turbo.TurboLibiGWN(cu(Pn), max_depth=8, areas=cu(A))
    tree.UpdateMassNormals(cu(N), cu(A))
    res, org, h = np.array([23, 19, 11], np.int32), np.array([-0.55, -0.5, -0.2], np.float32), np.float32(0.045)
    wg, gg = tree.value_and_gradient(grid=(res, org, h), beta=2.3, sigma=20.0, fp64=True)
    z, y, x = np.meshgrid(np.arange(res[2]), np.arange(res[1]), np.arange(res[0]), indexing="ij")
    G = np.stack([org[0] + x.astype(np.float32) * h, org[1] + y.astype(np.float32) * h,
                  org[2] + z.astype(np.float32) * h], -1).reshape(-1, 3).astype(np.float32)
    wp, gp = tree.value_and_gradient(cu(G), beta=2.3, sigma=20.0, fp64=True)
    assert np.array_equal(wg.cpu().numpy(), wp.cpu().numpy())
    assert np.array_equal(gg.cpu().numpy(), gp.cpu().numpy())
    # and the FP32 grid sums of the warp kernels sit within FP32 rounding of them
    w32 = tree.grid(res, org, h, sigma=20.0).cpu().numpy().astype(np.float64)
    w64 = wg.cpu().numpy()
    assert np.abs(w32 - w64).max() <= 1e-5 * np.abs(w64).max()
