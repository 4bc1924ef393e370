"""The iteration grid's field at the benchmark configurations, against the
FP64 oracle with the same opening decisions.

C2 (nonuniform torus, 100k points) and C3 (12 superquadrics + 1 % outliers,
1.01 M points), both at 256^3: after five DWG iterations the pipeline's
leaves and leaf normals are read, the sixth iteration (sigma 10, summed from
the screening weights that iteration 4 kept) computes the grid field, and
20,000 seeded grid samples of it are compared with the oracle's Barnes-Hut
sums over the same leaves and normals in FP64 (src/TurboLibiGWN.cu:328-836,
restated in oracle/dwg_oracle.c).  The oracle is fed the GPU octree's
moments, so the discrete opening decisions are taken on identical inputs.
"""
import numpy as np
import pytest
import torch

from dwg_b200 import datasets as D, turbo

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _match_nodes(gpu, ot):
    """GPU node index -> oracle node index, by (depth, first sorted point)"""
    ost = ot.dfs_starts()
    key = {(int(d), int(s)): i for i, (d, s, c) in enumerate(zip(ot.depth, ost, ot.counts)) if c > 0}
    return np.array([key[(int(d), int(s))] for d, s in zip(gpu["depth"], gpu["pt_start"])])


@pytest.mark.parametrize("config", ["c2_torus_100k", "c3_sq_union_1m"])
def test_iteration_field_matches_fp64_oracle(oracle_lib, config):
    P, _ = D.make(config, seed=1000)
    Pn, _, _ = D.normalize(P)
    Pd = torch.from_numpy(np.ascontiguousarray(Pn, np.float32)).to(DEV)
    dwg = turbo.TurboDWG(Pd, None, grid_reso=256, final_reso=256, total_iter=30)
    dwg.TurboScreenedDWGLaunch(5)
    L = dwg.get("leaf_pos")
    N = dwg.get("leaf_nrm")
    dwg.TurboScreenedDWGLaunch(1)  # iteration 5: sigma 10 from the kept weights
    field = dwg.get("field")
    res = dwg.get("grid_res").astype(np.int64)
    org = dwg.get("grid_origin")
    del dwg
    # the grid samples the kernels evaluate: origin + index x spacing in FP32
    rng = np.random.default_rng(5)
    sel = np.sort(rng.choice(int(np.prod(res)), 20000, replace=False))
    ix, iy, iz = sel % res[0], (sel // res[0]) % res[1], sel // (res[0] * res[1])
    h = np.float32(org[3])
    Q = np.stack([org[0] + ix.astype(np.float32) * h, org[1] + iy.astype(np.float32) * h,
                  org[2] + iz.astype(np.float32) * h], 1).astype(np.float32)
    # the leaf octree with the pipeline's areas (2e-6 each: no outlier filter)
    A = np.full(len(L), 2e-6, np.float32)
    gt = turbo.TurboLibiGWN(torch.from_numpy(L).to(DEV), max_depth=10, areas=torch.from_numpy(A).to(DEV))
    gt.UpdateMassNormals(torch.from_numpy(N).to(DEV), torch.from_numpy(A).to(DEV))
    torch.cuda.synchronize()
    g = gt.export()
    ot = oracle_lib.Octree(L, 10)
    idx = _match_nodes(g, ot)
    M = ot.num_nodes
    CM, R, EC = np.zeros((M, 3)), np.zeros(M), np.zeros((M, 3))
    CM[idx], R[idx], EC[idx] = g["cm"], g["radius"], g["ec"]
    w_ref, terms = ot.gwn(L, N, A, Q, beta=2.3, sigma=10.0, screened=True, moments=(CM, R, EC))
    assert terms.min() > 0
    err = np.abs(field[sel].astype(np.float64) - w_ref)
    wmax = np.abs(w_ref).max()
    # FP32 terms summed in FP64 against FP64 terms: the floor is the FP32
    # rounding of the inputs, ~1e-7 of the field scale
    print(f"{config}: max err / max |w| {err.max() / wmax:.2e}, rms err / max |w| "
          f"{np.sqrt((err ** 2).mean()) / wmax:.2e}, mean terms {terms.mean():.0f}")
    assert err.max() < 1e-5 * wmax, err.max() / wmax
    assert np.sqrt((err ** 2).mean()) < 1e-6 * wmax
