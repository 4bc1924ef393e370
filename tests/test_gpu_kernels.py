"""GPU parity tests: every CUDA kernel against the CPU oracle on the same
seeded inputs, called through the C ABI (ctypes)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import capi, datasets as D, turbo  # noqa: E402

pytestmark = pytest.mark.gpu

DEV = "cuda"


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def cloud(n=20000, kind="torus", seed=1):
    if kind == "torus":
        P, N = D.torus(n, seed=seed)
    else:
        P, N = D.sphere(n, seed=seed)
    Pn, _, _ = D.normalize(P)
    return Pn, N.astype(np.float32)


def match_nodes(gpu, ot):
    """map GPU node index -> oracle node index by (depth, first sorted point)"""
    ost = ot.dfs_starts()
    key = {(int(d), int(s)): i for i, (d, s, c) in enumerate(zip(ot.depth, ost, ot.counts)) if c > 0}
    return np.array([key[(int(d), int(s))] for d, s in zip(gpu["depth"], gpu["pt_start"])])


@pytest.fixture(scope="module")
def torus_tree(dwg_lib, oracle_lib):
    P, N = cloud(20000)
    A = np.full(len(P), 2e-6, np.float32)
    P_d, N_d, A_d = cu(P), cu(N), cu(A)
    gt = turbo.TurboLibiGWN(P_d, max_depth=8, areas=A_d)
    gt.UpdateMassNormals(N_d, A_d)
    torch.cuda.synchronize()
    ot = oracle_lib.Octree(P, 8)
    return P, N, A, gt, ot


def test_octree_topology_matches_octreeDWG(torus_tree):
    P, N, A, gt, ot = torus_tree
    g = gt.export()
    # sorted point order == depth-first order of octreeDWG
    assert np.array_equal(g["perm"], ot.dfs_order())
    # same set of non-empty nodes with the same depth / point range / count
    idx = match_nodes(g, ot)
    assert len(idx) == int((ot.counts > 0).sum())
    assert np.array_equal(g["pt_count"], ot.counts[idx])
    # leaves are the same nodes
    leaf_o = ot.children[idx, 0] == -1
    leaf_g = (g["skip"] == np.arange(len(idx)) + 1)
    assert np.array_equal(leaf_o, leaf_g)
    # pre-order: every subtree is a contiguous node range
    assert np.all(g["skip"] > np.arange(len(idx)))
    assert g["skip"][0] == len(idx)


def test_octree_moments_fp64(torus_tree):
    P, N, A, gt, ot = torus_tree
    g = gt.export()
    idx = match_nodes(g, ot)
    CM, R, EC = ot.moments(P, N, A)
    assert np.allclose(g["cm"], CM[idx], rtol=0, atol=1e-14)
    assert np.allclose(g["radius"], R[idx], rtol=0, atol=1e-14)
    assert np.allclose(g["ec"], EC[idx], rtol=1e-12, atol=1e-18)


def _oracle_gwn_with_gpu_moments(ot, g, idx, P, N, A, Q, **kw):
    """oracle traversal fed the GPU's moments (so that the discrete opening
    decisions are taken on identical float inputs)"""
    M = ot.num_nodes
    CM = np.zeros((M, 3))
    R = np.zeros(M)
    EC = np.zeros((M, 3))
    CM[idx], R[idx], EC[idx] = g["cm"], g["radius"], g["ec"]
    return ot.gwn(P, N, A, Q, moments=(CM, R, EC), **kw)


@pytest.mark.parametrize("screened,sigma", [(True, 20.0), (True, 10.0), (False, 0.0)])
@pytest.mark.parametrize("precision", [0, 1, 2, 3])
def test_gwn_points_same_sums_as_oracle(torus_tree, screened, sigma, precision, dwg_lib):
    import ctypes as C
    P, N, A, gt, ot = torus_tree
    g = gt.export()
    idx = match_nodes(g, ot)
    rng = np.random.default_rng(7)
    Q = np.concatenate([P[rng.choice(len(P), 3000, replace=False)],
                        rng.uniform(-0.6, 0.6, (3000, 3)).astype(np.float32)])
    w_ref, t_ref = _oracle_gwn_with_gpu_moments(ot, g, idx, P, N, A, Q, beta=2.3, sigma=sigma,
                                                screened=screened)
    out = torch.empty(len(Q), dtype=torch.float32, device=DEV)
    terms = torch.empty(len(Q), dtype=torch.int32, device=DEV)
    p = capi.gwn_params(beta=2.3, sigma=sigma, screened=screened, precision=precision)
    Q_d = cu(Q)
    capi.check(dwg_lib.dwg_gwn_points_counted(gt._h, None, None, None, capi.ptr(Q_d), len(Q), C.byref(p),
                                              capi.ptr(out), capi.ptr(terms), None))
    torch.cuda.synchronize()
    assert gt.status() == 0
    # identical opening decisions: the same number of terms per query
    assert np.array_equal(terms.cpu().numpy(), t_ref)
    w = out.cpu().numpy().astype(np.float64)
    err = np.abs(w - w_ref)
    wmax = np.abs(w_ref).max()
    # FP32 sums vs the FP64 oracle of the same terms: the floor is the FP32
    # rounding of the inputs (p - q, float moments), ~1e-7 of the field scale
    assert err.max() < 1e-5 * wmax, (precision, err.max() / wmax)
    assert np.sqrt((err ** 2).mean()) < 1e-6 * wmax


def test_gwn_grid_matches_oracle(torus_tree, oracle_lib):
    P, N, A, gt, ot = torus_tree
    g = gt.export()
    idx = match_nodes(g, ot)
    res = np.array([21, 18, 13], np.int32)
    org = np.array([-0.55, -0.5, -0.2], np.float32)
    h = np.float32(0.05)
    Q = oracle_lib.grid_points(res, org, h)
    w_ref, _ = _oracle_gwn_with_gpu_moments(ot, g, idx, P, N, A, Q, beta=2.3, sigma=20.0, screened=True)
    terms = torch.zeros(1, dtype=torch.int64, device=DEV)
    w = gt.grid(res, org, h, beta=2.3, sigma=20.0, precision=1, terms=terms).cpu().numpy()
    assert gt.status() == 0
    assert np.max(np.abs(w - w_ref)) < 2e-5 * max(1e-3, np.abs(w_ref).max())
    _, t_ref = _oracle_gwn_with_gpu_moments(ot, g, idx, P, N, A, Q, beta=2.3, sigma=20.0, screened=True)
    assert int(terms.item()) == int(t_ref.sum())


def test_marching_cubes_bit_exact(oracle_lib):
    rng = np.random.default_rng(3)
    res = np.array([37, 29, 33], np.int32)
    org = np.array([-0.7, -0.5, -0.6], np.float32)
    h = np.float32(0.037)
    G = oracle_lib.grid_points(res, org, h)
    f = np.zeros(len(G))
    for _ in range(6):
        c = rng.uniform(-0.5, 0.5, 3)
        f += np.exp(-((G - c) ** 2).sum(1) / 0.02)
    f = f.astype(np.float32)
    iso = np.float32(0.37)
    ref = oracle_lib.marching_cubes(f, res, org, h, iso)
    T = ref["T"]
    assert T > 1000
    mc = turbo.TurboMC()
    tris = torch.empty((T + 10, 9), dtype=torch.float32, device=DEV)
    cen = torch.empty((T + 10, 3), dtype=torch.float32, device=DEV)
    nrm = torch.empty((T + 10, 3), dtype=torch.float32, device=DEV)
    n = mc.TurboMarchingCubes(cu(f), None, *res.tolist(), iso, mid_points=cen, mid_normals=nrm, tris=tris,
                              origin=org, spacing=h, capacity=T + 10)
    assert n == T
    assert np.array_equal(tris[:T].cpu().numpy(), ref["tris"])
    assert np.array_equal(cen[:T].cpu().numpy(), ref["centroids"])
    assert np.array_equal(nrm[:T].cpu().numpy(), ref["normals"])


def test_marching_cubes_overflow_reported(oracle_lib, dwg_lib):
    import ctypes as C
    res = np.array([16, 16, 16], np.int32)
    org = np.zeros(3, np.float32)
    G = oracle_lib.grid_points(res, org, np.float32(1 / 15))
    f = (0.4 - np.linalg.norm(G - 0.5, axis=1)).astype(np.float32)
    T_ref = oracle_lib.marching_cubes(f, res, org, np.float32(1 / 15), 0.0)["T"]
    cap = T_ref // 2
    cen = torch.empty((cap, 3), dtype=torch.float32, device=DEV)
    T = C.c_longlong()
    f_d = cu(f)
    rc = dwg_lib.dwg_marching_cubes(capi.ptr(f_d), res.ctypes.data, None, org.ctypes.data, float(1 / 15), 0.0,
                                    None, capi.ptr(cen), None, cap, None, C.byref(T), None)
    assert rc == capi.DWG_ERR_OVERFLOW and T.value == T_ref


def test_knn_matches_bruteforce_with_ties(oracle_lib):
    rng = np.random.default_rng(4)
    P = (rng.integers(0, 12, (3000, 3)) * 0.01).astype(np.float32)  # lattice: exact ties
    Q = np.concatenate([(rng.integers(0, 12, (500, 3)) * 0.01 + 0.005).astype(np.float32),
                        rng.uniform(-0.05, 0.16, (500, 3)).astype(np.float32)])
    for k in (1, 10, 15, 16, 20, 64):
        ref = oracle_lib.knn(P, Q, k)
        ix = turbo.KnnIndex(cu(P))
        got = ix.query(cu(Q), k).cpu().numpy()
        assert np.array_equal(got, ref), k


def test_knn_surface_cloud(oracle_lib):
    P, _ = cloud(20000)
    rng = np.random.default_rng(5)
    Q = P[rng.choice(len(P), 2000, replace=False)] + rng.normal(0, 0.003, (2000, 3)).astype(np.float32)
    ref = oracle_lib.knn(P, Q, 15)
    got = turbo.KnnIndex(cu(P)).query(cu(Q), 15).cpu().numpy()
    assert np.array_equal(got, ref)


def test_knn_far_queries(oracle_lib):
    # queries offset from the surface by up to ~25 grid cells, and outside the
    # points' bounding box: the search continues over the occupancy pyramid
    P, N = cloud(30000)
    rng = np.random.default_rng(8)
    sel = rng.choice(len(P), 3000, replace=False)
    off = rng.uniform(-0.3, 0.3, (3000, 1)).astype(np.float32)
    Q = np.concatenate([P[sel] + off * N[sel], rng.uniform(-0.8, 0.8, (500, 3)).astype(np.float32)])
    Q = np.ascontiguousarray(Q, np.float32)
    ix = turbo.KnnIndex(cu(P))
    for k in (1, 10, 15, 40):
        ref = oracle_lib.knn(P, Q, k)
        got = ix.query(cu(Q), k).cpu().numpy()
        assert np.array_equal(got, ref), k


def test_diffusion_and_zero_repair_bit_exact(oracle_lib, dwg_lib):
    rng = np.random.default_rng(6)
    L, T, k = 4000, 9000, 15
    Lpos = rng.uniform(-0.5, 0.5, (L, 3)).astype(np.float32)
    knn = rng.integers(0, L // 2, (T, k)).astype(np.int32)  # upper half never hit -> zero normals
    tn = rng.standard_normal((T, 3)).astype(np.float32)
    tn /= np.linalg.norm(tn, axis=1, keepdims=True)
    N0 = rng.standard_normal((L, 3)).astype(np.float32)
    ref_n, ref_z, ref_c = oracle_lib.diffuse_normals(knn, tn, N0)
    # device tensors stay referenced until the kernels have run
    knn_d, tn_d, n_dev, pos_d = cu(knn), cu(tn), cu(N0), cu(Lpos)
    isz = torch.zeros(L, dtype=torch.uint8, device=DEV)
    zc = torch.zeros(1, dtype=torch.int32, device=DEV)
    capi.check(dwg_lib.dwg_diffuse_normals(capi.ptr(knn_d), capi.ptr(tn_d), T, k, L, capi.ptr(n_dev),
                                           capi.ptr(isz), capi.ptr(zc), None))
    torch.cuda.synchronize()
    assert int(zc.item()) == ref_c and ref_c > 10
    assert np.array_equal(isz.cpu().numpy().astype(bool), ref_z)
    assert np.array_equal(n_dev.cpu().numpy(), ref_n)
    rep = oracle_lib.zero_repair(Lpos, ref_n, ref_z, 10)
    ix = turbo.KnnIndex(pos_d)
    capi.check(dwg_lib.dwg_zero_repair(ix._h, capi.ptr(n_dev), capi.ptr(isz), capi.ptr(zc), 10, 10, None))
    torch.cuda.synchronize()
    assert np.array_equal(n_dev.cpu().numpy(), rep)


def test_gauss_map_load_normals_radii_bit_exact(oracle_lib, dwg_lib):
    P, _ = cloud(5000, kind="sphere")
    P_d = cu(P)
    out = torch.empty((len(P), 3), dtype=torch.float32, device=DEV)
    turbo.TurboNormalInitialization().GaussMapInit(P_d, out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), oracle_lib.gauss_map(P))
    nb = oracle_lib.knn(P, P, 10)
    nb_d = cu(nb)
    got = torch.empty(len(P), dtype=torch.float32, device=DEV)
    capi.check(dwg_lib.dwg_radii(capi.ptr(P_d), len(P), capi.ptr(nb_d), 10, capi.ptr(got), None))
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), oracle_lib.radii(P, nb))
    LN = oracle_lib.gauss_map(P)
    LN_d = cu(LN)
    ln = torch.empty((len(P), 3), dtype=torch.float32, device=DEV)
    capi.check(dwg_lib.dwg_load_normals(capi.ptr(nb_d), 10, len(P), capi.ptr(LN_d), capi.ptr(ln), None))
    torch.cuda.synchronize()
    assert np.array_equal(ln.cpu().numpy(), oracle_lib.load_normals(nb, LN))


def test_voxel_grid_matches_oracle(oracle_lib):
    P, _ = cloud(3000)
    for s in (16, 128, 257):
        res, org, h = turbo.voxel_grid(cu(P), 0.05, s)
        r2, o2, h2 = oracle_lib.voxel_grid(P, 0.05, s)
        assert np.array_equal(res, r2) and np.array_equal(org, o2) and h == h2


def _lattice_cloud(n=20000, cells=128, seed=6):
    """octree-leaf-like input: a torus snapped to a lattice (many cocircular
    neighbourhoods), duplicates removed"""
    P, _ = cloud(n, kind="torus", seed=seed)
    Q = np.unique(np.round(P * cells), axis=0) / cells
    return Q.astype(np.float32)


@pytest.mark.parametrize("kind", ["scattered", "lattice"])
def test_pca_normals_and_point_areas_bit_exact(oracle_lib, kind):
    # --com_As 1 inputs on the same neighbour rows: both sides run the same
    # FP64 Jacobi sequence and exact Delaunay predicates
    P = cloud(20000, kind="torus", seed=5)[0] if kind == "scattered" else _lattice_cloud()
    P_d = cu(P)
    nb10 = oracle_lib.knn(P, P, 10)
    view = ((P.max(0) + P.min(0)) / np.float32(2)).astype(np.float32)
    ref_n = oracle_lib.pca_normals(P, nb10, view)
    got_n = turbo.pca_normals(P_d, cu(nb10), view)
    torch.cuda.synchronize()
    assert np.array_equal(got_n.cpu().numpy(), ref_n)
    nb15 = oracle_lib.knn(P, P, 15)
    ref_a = oracle_lib.point_areas(P, nb15, ref_n)
    got_a = turbo.point_areas(P_d, cu(nb15), cu(ref_n))
    torch.cuda.synchronize()
    assert np.array_equal(got_a.cpu().numpy(), ref_a)
    assert ref_a.min() >= 0 and np.mean(ref_a > 0) > 0.99
    # the rows only need self first: a shorter k gives a finite answer too
    got3 = turbo.point_areas(P_d, cu(nb15[:, :3].copy()), cu(ref_n))
    assert torch.isfinite(got3).all()
    with pytest.raises(capi.DwgError):
        turbo.point_areas(cu(P[:2000]), cu(oracle_lib.knn(P[:2000], P[:2000], 33)), cu(ref_n[:2000]))


@pytest.mark.parametrize("order", [1, 2])
def test_fwn_expansion_matches_oracle(torus_tree, order, dwg_lib, oracle_lib):
    # igl::fast_winding_number's far field of orders 1 and 2 on the plain sum
    import ctypes as C
    P, N, A, gt, ot = torus_tree
    g = gt.export()
    idx = match_nodes(g, ot)
    CM, R, EC = ot.moments(P, N, A)
    HO_ref = ot.expansion(P, N, A, CM)[idx]
    HO = gt.expansion()
    # FP64 coefficients: the GPU shifts children's sums to the parent's
    # centre, the oracle sums each node's points directly
    mass = g["pt_count"][:, None] * 2e-6
    tol1 = 1e-11 * mass * g["radius"][:, None]
    tol2 = 1e-11 * mass * g["radius"][:, None] ** 2
    assert np.all(np.abs(HO[:, :9] - HO_ref[:, :9]) <= tol1 + 1e-30)
    assert np.all(np.abs(HO[:, 9:] - HO_ref[:, 9:]) <= tol2 + 1e-30)
    # the sums, with the oracle fed the GPU's moments (identical decisions)
    M = ot.num_nodes
    full = [np.zeros((M, 3)), np.zeros(M), np.zeros((M, 3)), np.zeros((M, 36))]
    full[0][idx], full[1][idx], full[2][idx], full[3][idx] = g["cm"], g["radius"], g["ec"], HO
    rng = np.random.default_rng(9)
    Q = np.concatenate([P[rng.choice(len(P), 2000, replace=False)],
                        rng.uniform(-0.6, 0.6, (4000, 3)).astype(np.float32)])
    w_ref, t_ref = ot.fwn(P, N, A, Q, order, beta=2.0, moments=full)
    out = torch.empty(len(Q), dtype=torch.float32, device=DEV)
    terms = torch.empty(len(Q), dtype=torch.int32, device=DEV)
    p = capi.gwn_params(beta=2.0, sigma=0.0, screened=False, precision=1, order=order)
    Q_d = cu(Q)
    capi.check(dwg_lib.dwg_gwn_points_counted(gt._h, None, None, None, capi.ptr(Q_d), len(Q), C.byref(p),
                                              capi.ptr(out), capi.ptr(terms), None))
    torch.cuda.synchronize()
    assert gt.status() == 0
    assert np.array_equal(terms.cpu().numpy(), t_ref)
    w = out.cpu().numpy().astype(np.float64)
    err = np.abs(w - w_ref)
    wmax = np.abs(w_ref).max()
    assert err.max() < 1e-5 * wmax and np.sqrt((err ** 2).mean()) < 1e-6 * wmax
    # the grid path evaluates the same terms
    res = np.array([17, 15, 9], np.int32)
    org = np.array([-0.55, -0.5, -0.2], np.float32)
    h = np.float32(0.06)
    Qg = oracle_lib.grid_points(res, org, h)
    wg_ref, _ = ot.fwn(P, N, A, Qg, order, beta=2.0, moments=full)
    wg = gt.grid(res, org, h, beta=2.0, sigma=0.0, screened=False, precision=1, order=order).cpu().numpy()
    assert np.max(np.abs(wg - wg_ref)) < 2e-5 * max(1e-3, np.abs(wg_ref).max())
    # screened sums take order 0 only
    with pytest.raises(capi.DwgError):
        gt.grid(res, org, h, beta=2.0, sigma=10.0, screened=True, order=order)


def test_fwn_order2_closer_to_exact_on_gpu(oracle_lib):
    # a closed sphere: order-2 far field, as in igl::fast_winding_number's
    # default, is several times closer to the exact sum than order 0
    rng = np.random.default_rng(0)
    n = 20000
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    P = (v * 0.4).astype(np.float32)
    N = v.astype(np.float32)
    A = np.full(n, 4 * np.pi * 0.16 / n, np.float32)
    Q = rng.uniform(-0.6, 0.6, (4000, 3)).astype(np.float32)
    exact = oracle_lib.gwn_exact(P, N, A, Q, screened=False)
    P_d, N_d, A_d, Q_d = cu(P), cu(N), cu(A), cu(Q)
    gt = turbo.TurboLibiGWN(P_d, max_depth=8, areas=A_d)
    gt.UpdateMassNormals(N_d, A_d)
    rms = []
    for order in (0, 2):
        w = gt.TurboLibiGWNLaunch(Q_d, beta=2.0, order=order).cpu().numpy()
        rms.append(np.sqrt(np.mean((w - exact) ** 2)))
    assert rms[1] < rms[0] / 3


def test_zero_repair_large_grid_bit_exact(oracle_lib, dwg_lib):
    # a grid above 2^22 cells: the subset index bounds only the queried cells
    # (radius-3 blocks, the rest to the per-thread search); a flagged cap of
    # the sphere leaves its centre far from any unflagged point
    rng = np.random.default_rng(12)
    L = 600000
    v = rng.standard_normal((L, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    Lpos = (0.45 * v).astype(np.float32)
    N0 = rng.standard_normal((L, 3)).astype(np.float32)
    N0 /= np.linalg.norm(N0, axis=1, keepdims=True)
    isz = (v[:, 2] > 0.995) | (rng.random(L) < 0.002)
    ref = oracle_lib.zero_repair(Lpos, N0, isz, 10)
    pos_d, n_dev = cu(Lpos), cu(N0)
    isz_d = cu(isz.astype(np.uint8))
    zc = torch.tensor([int(isz.sum())], dtype=torch.int32, device=DEV)
    ix = turbo.KnnIndex(pos_d)
    capi.check(dwg_lib.dwg_zero_repair(ix._h, capi.ptr(n_dev), capi.ptr(isz_d), capi.ptr(zc), 10, 10, None))
    torch.cuda.synchronize()
    assert np.array_equal(n_dev.cpu().numpy(), ref)


@pytest.mark.parametrize("k", [10, 16])
def test_zero_repair_far_queries_bit_exact(oracle_lib, dwg_lib, k):
    # a grid above 2^22 cells with the cap z > 0.8 of the sphere flagged: the
    # flagged points near the pole lie ~50 cells from every unflagged point,
    # so their per-thread walk runs past its visit budget and the warp-per-
    # query search over the pyramid finishes them
    rng = np.random.default_rng(13)
    L = 420000
    v = rng.standard_normal((L, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    Lpos = (0.45 * v).astype(np.float32)
    N0 = rng.standard_normal((L, 3)).astype(np.float32)
    N0 /= np.linalg.norm(N0, axis=1, keepdims=True)
    isz = v[:, 2] > 0.8
    ref = oracle_lib.zero_repair(Lpos, N0, isz, k)
    pos_d, n_dev = cu(Lpos), cu(N0)
    isz_d = cu(isz.astype(np.uint8))
    zc = torch.tensor([int(isz.sum())], dtype=torch.int32, device=DEV)
    ix = turbo.KnnIndex(pos_d)
    capi.check(dwg_lib.dwg_zero_repair(ix._h, capi.ptr(n_dev), capi.ptr(isz_d), capi.ptr(zc), k, 10, None))
    torch.cuda.synchronize()
    assert np.array_equal(n_dev.cpu().numpy(), ref)


@pytest.mark.parametrize("L,k", [(420000, 10), (60000, 16)])
def test_zero_repair_seeded_repeats_bit_exact(oracle_lib, dwg_lib, L, k):
    # repairs on one index start each flagged point's search from its
    # neighbours of the previous repair where those are still unflagged.  A
    # flagged polar cap that grows (recorded neighbours become flagged: no
    # seed), shrinks (seeds valid but no longer the nearest) and stays (seeds
    # exact), with scattered flags that change each time; every repair must
    # equal the oracle's repair from scratch.  420k points: a grid above 2^22
    # cells (bounds of the queried cells only; far queries through the
    # per-thread walk and the warp search), 60k: the whole-grid bound
    rng = np.random.default_rng(14)
    v = rng.standard_normal((L, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    Lpos = (0.45 * v).astype(np.float32)
    N0 = rng.standard_normal((L, 3)).astype(np.float32)
    N0 /= np.linalg.norm(N0, axis=1, keepdims=True)
    ix = turbo.KnnIndex(cu(Lpos))
    for cap, seed in ((0.8, 1), (0.75, 2), (0.85, 3), (0.85, 3)):
        isz = (v[:, 2] > cap) | (np.random.default_rng(seed).random(L) < 0.002)
        ref = oracle_lib.zero_repair(Lpos, N0, isz, k)
        n_dev, isz_d = cu(N0), cu(isz.astype(np.uint8))
        zc = torch.tensor([int(isz.sum())], dtype=torch.int32, device=DEV)
        capi.check(dwg_lib.dwg_zero_repair(ix._h, capi.ptr(n_dev), capi.ptr(isz_d), capi.ptr(zc), k, 10, None))
        torch.cuda.synchronize()
        assert np.array_equal(n_dev.cpu().numpy(), ref), cap


@pytest.mark.parametrize("tile", [0, 2])
def test_gwn_grid_lists_bit_identical(tile):
    # dwg_gwn_grid with lists records the grid's interaction lists on its first
    # call and replays them afterwards; lists=2 also keeps the screening
    # weights of two sigmas.  Same sums and term counts as the traversal, bit
    # for bit: after the normals change, for a sigma without a slot, on a
    # second grid
    P, N = cloud(20000, seed=9)
    A = np.full(len(P), 2e-6, np.float32)
    gt = turbo.TurboLibiGWN(cu(P), max_depth=8, areas=cu(A))
    gt.UpdateMassNormals(cu(N), cu(A))
    rng = np.random.default_rng(4)
    N2 = rng.normal(size=N.shape).astype(np.float32)
    N2 /= np.linalg.norm(N2, axis=1, keepdims=True)
    for res, org, h in (([40, 36, 30], [-0.55, -0.5, -0.2], 0.03), ([23, 29, 17], [-0.6, -0.55, -0.25], 0.05)):
        res = np.array(res, np.int32)
        org = np.array(org, np.float32)
        runs = {}
        for lists in (0, 2, 1):
            gt.UpdateMassNormals(cu(N), cu(A))
            runs[lists] = []
            # slots: 20 written, read; 10 written; both read; 5 has no slot
            for sigma, nrm in ((20.0, None), (20.0, None), (10.0, None), (20.0, N2), (10.0, None), (5.0, None),
                               (10.0, N)):
                if nrm is not None:
                    gt.UpdateMassNormals(cu(nrm), cu(A))
                t = torch.zeros(1, dtype=torch.int64, device=DEV)
                w = gt.grid(res, org, h, sigma=sigma, tile=tile, terms=t, lists=lists).cpu().numpy()
                assert gt.status() == 0
                runs[lists].append((w, int(t.item())))
            if lists:  # the list kept for this grid, and its weight slots
                entries, slots = gt.list_size()
                assert entries > 0 and slots == (2 if lists == 2 else 0), (lists, entries, slots)
        for lists in (1, 2):
            for step, ((w0, t0), (w, t)) in enumerate(zip(runs[0], runs[lists])):
                assert t0 > 0
                assert np.array_equal(w0, w), (tuple(res), lists, step)
                assert t == t0, (tuple(res), lists, step)


def test_gwn_grid_kept_weights_follow_new_radii():
    # With use_radii the screening weights depend on the points' radii:
    # dwg_gwn_grid drops the kept weights whenever radii are passed, so a call
    # with new radii and the same sigma sums with the new radii (lists 2 equal
    # to the traversal, bit for bit)
    P, N = cloud(20000, seed=9)
    A = np.full(len(P), 2e-6, np.float32)
    rng = np.random.default_rng(12)
    R1 = rng.uniform(0.001, 0.004, len(P)).astype(np.float32)
    R2 = (R1 * 1.7).astype(np.float32)
    res, org, h = np.array([40, 36, 30], np.int32), np.array([-0.55, -0.5, -0.2], np.float32), 0.03
    runs = {}
    for lists in (0, 2):
        gt = turbo.TurboLibiGWN(cu(P), max_depth=8, areas=cu(A))
        gt.UpdateMassNormals(cu(N), cu(A))
        runs[lists] = [gt.grid(res, org, h, sigma=20.0, lists=lists, i_radii=cu(R)).cpu().numpy()
                       for R in (R1, R1, R2, R2)]
        assert gt.status() == 0
    assert not np.array_equal(runs[0][0], runs[0][2])  # the radii matter
    for step, (w0, w2) in enumerate(zip(runs[0], runs[2])):
        assert np.array_equal(w0, w2), step


def test_compensated_fp32_sums_are_as_close_to_fp64_as_fp64_sums(torus_tree):
    # precision 3 keeps each query's sum in FP32 with Neumaier compensation:
    # its error against the FP64 oracle (same terms) is that of precision 1
    # (FP32 terms summed in FP64), below that of plain FP32 sums
    P, N, A, gt, ot = torus_tree
    g = gt.export()
    idx = match_nodes(g, ot)
    rng = np.random.default_rng(17)
    Q = np.concatenate([P[rng.choice(len(P), 4000, replace=False)],
                        rng.uniform(-0.6, 0.6, (4000, 3)).astype(np.float32)])
    w_ref, _ = _oracle_gwn_with_gpu_moments(ot, g, idx, P, N, A, Q, beta=2.3, sigma=20.0, screened=True)
    err = {}
    for prec in (0, 1, 3):
        w = gt.TurboLibiScreenedGWNLaunch(cu(Q), None, len(Q), None, None, None, 2.3, 20.0,
                                          precision=prec).cpu().numpy().astype(np.float64)
        err[prec] = float(np.sqrt(np.mean((w - w_ref) ** 2)))
    print("RMS error vs FP64 (same terms): fp32 sum %.3g, fp64 sum %.3g, compensated fp32 sum %.3g"
          % (err[0], err[1], err[3]))
    assert err[3] <= 1.1 * err[1] + 1e-12, err
    assert err[3] <= 1.02 * err[0], err


@pytest.mark.parametrize("k", [10, 15])
def test_knn_cell_grouped_queries_dense_and_sparse(oracle_lib, k):
    # the pipeline's k (10: zero repair, 10 slots per lane; 15: triangles) on
    # many queries per cell and on a few per cell: exact either way
    P, N = cloud(20000, seed=13)
    rng = np.random.default_rng(21)
    sel = rng.choice(len(P), 40000)
    off = rng.uniform(-0.05, 0.05, (40000, 1)).astype(np.float32)
    Q = np.ascontiguousarray(P[sel] + off * N[sel], np.float32)
    ix = turbo.KnnIndex(cu(P))
    dense = ix.query(cu(Q), k).cpu().numpy()
    sparse = ix.query(cu(Q[:5000]), k).cpu().numpy()
    assert np.array_equal(dense[:5000], sparse)
    assert np.array_equal(sparse, oracle_lib.knn(P, Q[:5000], k))
