"""CPU tests of the oracle: pinned to the reference's marching-cubes table
(fixture derived from src/TurboMC.cu) and to analytic known answers."""
import json
import os

import numpy as np
import pytest

from dwg_b200 import datasets as D

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "mc_reference_loops.json")


def oriented_loops(row):
    tris = [tuple(int(x) for x in row[i:i + 3]) for i in range(0, 16, 3) if row[i] >= 0]
    de = {}
    for t in tris:
        for k in range(3):
            de[(t[k], t[(k + 1) % 3])] = 1
    bnd = [e for e in de if (e[1], e[0]) not in de]
    nx = {a: b for a, b in bnd}
    loops, seen = [], set()
    for a in sorted(nx):
        if a in seen:
            continue
        loop, c = [a], nx[a]
        seen.add(a)
        while c != a:
            loop.append(c)
            seen.add(c)
            c = nx[c]
        i = loop.index(min(loop))
        loops.append(loop[i:] + loop[:i])
    return sorted(loops), len(tris)


def check_table_against_fixture(et, tt):
    g = json.load(open(GOLDEN))
    assert len(g["cases"]) == 256
    for case in g["cases"]:
        ci = case["case"]
        loops, ntri = oriented_loops(tt[ci])
        assert ntri == case["tri_count"], ci
        assert loops == case["loops"], ci
        # edge mask: an edge is cut iff its corners differ
        mask = 0
        for e in range(12):
            a = e & 7
            b = ((e + 1) & 3) if e < 4 else (4 + ((e - 3) & 3) if e < 8 else e - 4)
            if ((ci >> a) & 1) != ((ci >> b) & 1):
                mask |= 1 << e
        assert et[ci] == mask


def reference_triangles():
    g = json.load(open(GOLDEN))
    tt = np.full((256, 16), -1, np.int8)
    for c in g["cases"]:
        flat = [e for t in c["tris"] for e in t]
        tt[c["case"], : len(flat)] = flat
    return tt


def test_oracle_mc_table_matches_reference_fixture(oracle_lib):
    # the oracle's own polygons from the cube geometry are the reference's ...
    et, tp = oracle_lib.mc_polygons()
    check_table_against_fixture(et, tp)
    # ... and it triangulates them with the reference's triangles
    et2, tt = oracle_lib.mc_tables()
    assert np.array_equal(et, et2)
    assert np.array_equal(tt, reference_triangles())
    check_table_against_fixture(et2, tt)


def test_oracle_sphere_gwn_known_answer(oracle_lib):
    """Plain GWN of a closed, well-sampled sphere with true normals and areas
    4 pi / N: ~1 inside, ~0 outside (exact all-pairs)."""
    n = 6000
    P, N = D.sphere(n, noise=0.0, seed=3)
    A = np.full(n, 4 * np.pi / n, np.float32)
    Q = np.array([[0, 0, 0], [0.3, -0.2, 0.1], [1.8, 0, 0], [0, -2.5, 1.0]], np.float32)
    w = oracle_lib.gwn_exact(P, N, A, Q, screened=False)
    assert abs(w[0] - 1) < 2e-3 and abs(w[1] - 1) < 5e-3
    assert abs(w[2]) < 5e-3 and abs(w[3]) < 5e-3
    # Barnes-Hut at beta=2.3 (order 0) stays within a few percent
    t = oracle_lib.Octree(P, 10)
    wb, terms = t.gwn(P, N, A, Q, beta=2.3, screened=False)
    assert np.all(np.abs(wb - w) < 0.05)
    assert np.all(terms < n)  # far field actually used
    # beta = 0 opens nothing far: Barnes-Hut equals the exact sum
    w0, t0 = t.gwn(P, N, A, Q, beta=0.0, screened=False)
    # (beta=0 makes every node with R>0 far; use a huge beta instead)
    wbig, tbig = t.gwn(P, N, A, Q, beta=1e30, screened=False)
    assert np.allclose(wbig, w, rtol=1e-12, atol=1e-12)
    assert np.all(tbig == n)


def test_oracle_octree_topology_rules(oracle_lib):
    P, _ = D.torus(3000, seed=1)
    Pn, _, _ = D.normalize(P)
    t = oracle_lib.Octree(Pn, 6)
    ch, cnt, dep = t.children, t.counts, t.depth
    for v in range(t.num_nodes):
        internal = ch[v, 0] != -1
        if internal:
            assert cnt[v] > 1 and dep[v] < 6
            assert cnt[ch[v]].sum() == cnt[v]
            assert np.all(dep[ch[v]] == dep[v] + 1)
        else:
            assert cnt[v] <= 1 or dep[v] == 6
    # depth-first order is a permutation
    perm = t.dfs_order()
    assert sorted(perm.tolist()) == list(range(len(Pn)))


def test_oracle_knn_order_and_ties(oracle_lib):
    rng = np.random.default_rng(0)
    P = rng.integers(0, 4, (200, 3)).astype(np.float32)  # lattice: many exact ties
    Q = rng.integers(0, 4, (50, 3)).astype(np.float32) + 0.5
    k = 7
    got = oracle_lib.knn(P, Q, k)
    for qi in range(len(Q)):
        d2 = ((P - Q[qi]) ** 2).sum(1).astype(np.float32)
        order = np.lexsort((np.arange(len(P)), d2))[:k]
        assert got[qi].tolist() == order.tolist()


def test_oracle_marching_cubes_sphere_sdf(oracle_lib):
    """Cases of an analytic field are exactly the corner-sign bits; every
    vertex lies on a cut edge; normals are unit."""
    res = np.array([24, 20, 22], np.int32)
    org = np.array([-1.1, -1.0, -1.05], np.float32)
    h = np.float32(0.1)
    G = oracle_lib.grid_points(res, org, h)
    f = (0.8 - np.linalg.norm(G, axis=1)).astype(np.float32)
    m = oracle_lib.marching_cubes(f, res, org, h, 0.0)
    F = f.reshape(res[2], res[1], res[0])
    corners = [(0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1), (0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)]
    cases = np.zeros((res[2] - 1, res[1] - 1, res[0] - 1), np.int64)
    for c, (ox, oy, oz) in enumerate(corners):
        v = F[oz:oz + res[2] - 1, oy:oy + res[1] - 1, ox:ox + res[0] - 1]
        cases |= (v > 0).astype(np.int64) << c
    assert np.array_equal(m["cases"], cases.reshape(-1).astype(np.uint8))
    et, tt = oracle_lib.mc_tables()
    ntri = np.array([(tt[i] >= 0).sum() // 3 for i in range(256)])
    assert m["T"] == int(ntri[cases.reshape(-1)].sum())
    # |n| = |c| / (|c| + 1e-8): below 1 for small (sliver) triangles
    nn = np.linalg.norm(m["normals"], axis=1)
    assert np.all(nn <= 1 + 1e-6) and np.mean(nn > 0.999) > 0.98
    r = np.linalg.norm(m["tris"].reshape(-1, 3), axis=1)
    assert np.all(np.abs(r - 0.8) < 0.02)


def test_oracle_voxel_grid_shape():
    import oracle
    P, _ = D.sphere(2000, seed=0)
    Pn, _, _ = D.normalize(P)
    res, org, h = oracle.voxel_grid(Pn, 0.05, 64)
    assert max(res) == 64 and min(res) >= 60
    top = org + (res - 1) * h
    mn, mx = Pn.min(0) - 0.05, Pn.max(0) + 0.05
    # the padded grid covers the box with one sample of pad on the long axis
    assert np.all(org <= mn + 1e-6) and np.all(top >= mx - 1e-6)


def test_oracle_diffusion_fixed_point_order_independent():
    import oracle
    rng = np.random.default_rng(2)
    L, T, k = 300, 2000, 15
    knn = rng.integers(0, L, (T, k)).astype(np.int32)
    tn = rng.standard_normal((T, 3)).astype(np.float32)
    tn /= np.linalg.norm(tn, axis=1, keepdims=True)
    N0 = np.zeros((L, 3), np.float32)
    a, za, ca = oracle.diffuse_normals(knn, tn, N0)
    perm = rng.permutation(T)
    b, zb, cb = oracle.diffuse_normals(knn[perm], tn[perm], N0)
    assert np.array_equal(a, b) and np.array_equal(za, zb) and ca == cb


@pytest.mark.slow
def test_oracle_reconstruct_small_sphere():
    import oracle
    P, N = D.sphere(1500, noise=0.002, seed=5)
    Pn, _, _ = D.normalize(P)
    r = oracle.reconstruct(Pn, grid_reso=40, final_reso=40, total_iter=4, max_depth=7)
    assert r["L"] > 100 and r["T"] > 100
    assert np.all(r["tri_count"] > 0)
    nrm = np.linalg.norm(r["leaf_nrm"], axis=1)
    assert np.allclose(nrm, 1, atol=1e-4)
    # The marching-cubes normals point towards the corners above the iso
    # value, so the orientation flips every iteration; after an even number
    # of iterations the Gauss-map (outward) orientation is back.  The inner
    # iso-shell of the screened field flips a minority of leaves; the final
    # point normals (mean of 10 leaves) agree.
    s = np.sign((r["leaf_nrm"] * r["leaf_pos"]).sum(1))
    assert s.mean() > 0.7
    sp = np.sign((r["point_nrm"] * Pn).sum(1))
    assert sp.mean() > 0.98


def test_oracle_outlier_filter_known_answer(oracle_lib):
    A = np.array([1, 3, 3, 2, 5, 5, 0.5], np.float32)
    # ceil(7 * 0.4) = 3 largest: the two 5s, then the first 3 (index order on ties)
    got = oracle_lib.outlier_filter(A, 0.4)
    want = A.copy()
    want[[4, 5, 1]] /= 1000.0
    assert np.array_equal(got, want)
    assert np.array_equal(oracle_lib.outlier_filter(A, 0.0), A)


def _embed(xy, z=0.3, seed=0):
    """planar 2-D points placed on a rotated plane in 3-D"""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    P = np.c_[xy, np.full(len(xy), z)] @ q.T
    return P.astype(np.float32), q[:, 2].astype(np.float32)


def test_oracle_point_areas_known_answers(oracle_lib):
    # centre of a regular hexagon of side 1: six equilateral Delaunay
    # triangles, a third of each => sqrt(3)/2 (the hexagonal Voronoi cell)
    ang = np.arange(6) * np.pi / 3
    xy = np.r_[[[0.0, 0.0]], np.c_[np.cos(ang), np.sin(ang)]]
    P, nrm = _embed(xy)
    N = np.tile(nrm, (len(P), 1))
    knn = np.arange(7, dtype=np.int32)[None, :]
    a = oracle_lib.point_areas(P, np.repeat(knn, 7, 0), N)
    assert abs(a[0] - np.sqrt(3) / 2) < 1e-5
    # one triangle, obtuse at the point itself: half of its area (0.2 * 0.5)
    P2, nrm2 = _embed(np.array([[0.0, 0.0], [-1.0, 0.2], [1.0, 0.2]]), seed=1)
    N2 = np.tile(nrm2, (3, 1))
    a2 = oracle_lib.point_areas(P2, np.array([[0, 1, 2]] * 3, np.int32), N2)
    assert abs(a2[0] - 0.1) < 1e-6
    # centre of a square lattice: every square around it is cocircular; one
    # triangulation per square (not both diagonals) => the unit Voronoi cell
    g = np.array([[x, y] for x in (-1.0, 0.0, 1.0) for y in (-1.0, 0.0, 1.0)])
    g = np.r_[[[0.0, 0.0]], g[np.any(g != 0, axis=1)]]
    P4, nrm4 = _embed(g, seed=4)
    a4 = oracle_lib.point_areas(P4, np.arange(9, dtype=np.int32)[None, :].repeat(9, 0), np.tile(nrm4, (9, 1)))
    assert abs(a4[0] - 1.0) < 1e-5
    # a neighbour whose normal disagrees is dropped: 2 left -> area 0
    N3 = N2.copy()
    N3[2] *= -1
    a3 = oracle_lib.point_areas(P2, np.array([[0, 1, 2]] * 3, np.int32), N3)
    assert a3[0] == 0.0


def test_oracle_pca_normals_face_the_viewpoint(oracle_lib):
    rng = np.random.default_rng(3)
    P, nrm = _embed(rng.uniform(-1, 1, (200, 2)), seed=2)
    knn = oracle_lib.knn(P, P, 10)
    centre = P.mean(0)
    for s in (1.0, -1.0):
        view = (centre + s * 5 * nrm).astype(np.float32)
        N = oracle_lib.pca_normals(P, knn, view)
        assert np.allclose(N, s * nrm[None, :], atol=1e-5)


def test_oracle_fwn_expansion_converges(oracle_lib):
    # igl::fast_winding_number's far-field expansion: on one cluster of
    # dipoles the error against the direct sum falls with the order and with
    # the distance (order p: ~ r^-(3+p))
    rng = np.random.default_rng(1)
    n = 200
    P = (rng.normal(size=(n, 3)) * 0.05).astype(np.float32)
    N = rng.normal(size=(n, 3))
    N = (N / np.linalg.norm(N, axis=1, keepdims=True)).astype(np.float32)
    A = rng.uniform(0.5, 1.5, n).astype(np.float32)
    t = oracle_lib.Octree(P, 4)
    CM, R, EC = t.moments(P, N, A)
    dirs = rng.normal(size=(40, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    errs = {}
    for dist in (0.6, 2.4):
        Q = (CM[0] + dist * dirs).astype(np.float32)
        exact = oracle_lib.gwn_exact(P, N, A, Q, screened=False)
        # beta small against the query distances over R: the root's children
        # (internal nodes) are far and take the expansion
        for order in (0, 1, 2):
            w, _ = t.fwn(P, N, A, Q, order, beta=0.5)
            errs[(dist, order)] = np.abs(w - exact).mean()
    for dist in (0.6, 2.4):
        assert errs[(dist, 2)] < errs[(dist, 1)] < errs[(dist, 0)]
    for order in (0, 1, 2):
        assert errs[(2.4, order)] < errs[(0.6, order)] / 4 ** (1 + order)


def test_oracle_fwn_sphere_order2_beats_order0(oracle_lib):
    rng = np.random.default_rng(0)
    n = 20000
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    P = (v * 0.4).astype(np.float32)
    N = v.astype(np.float32)
    A = np.full(n, 4 * np.pi * 0.16 / n, np.float32)
    Q = rng.uniform(-0.6, 0.6, (2000, 3)).astype(np.float32)
    t = oracle_lib.Octree(P, 8)
    exact = oracle_lib.gwn_exact(P, N, A, Q, screened=False)
    w0, t0 = t.fwn(P, N, A, Q, 0, beta=2.0)
    w2, t2 = t.fwn(P, N, A, Q, 2, beta=2.0)
    assert np.array_equal(t0, t2)  # same traversal, richer far terms
    rms0 = np.sqrt(np.mean((w0 - exact) ** 2))
    rms2 = np.sqrt(np.mean((w2 - exact) ** 2))
    assert rms2 < rms0 / 3


@pytest.mark.parametrize("screened,sigma", [(True, 20.0), (False, 0.0)])
def test_oracle_gradient_matches_central_differences(oracle_lib, screened, sigma):
    """The oracle's analytic gradient of the exact sum (beta = 1e30 opens every
    node, so no decision moves under the perturbation) against central
    differences of its value, at h = 1e-5 (the error falls as h^2)."""
    P, N = D.torus(3000, seed=3)
    Pn, _, _ = D.normalize(P)
    A = np.full(len(Pn), 2e-6, np.float32)
    rng = np.random.default_rng(1)
    Q = (Pn[:50] + rng.normal(0, 0.02, (50, 3))).astype(np.float64)
    t = oracle_lib.Octree(Pn, 8)
    w, g = t.gwn_grad(Pn, N, A, Q.astype(np.float32), beta=1e30, sigma=sigma, screened=screened)
    w0, _ = t.gwn(Pn, N, A, Q.astype(np.float32), beta=1e30, sigma=sigma, screened=screened)
    assert np.array_equal(w, w0)
    fd = np.zeros_like(g)
    for d in range(3):
        e = np.zeros(3)
        e[d] = 1e-5
        qp, qm = (Q + e).astype(np.float32), (Q - e).astype(np.float32)
        wp, _ = t.gwn(Pn, N, A, qp, beta=1e30, sigma=sigma, screened=screened)
        wm, _ = t.gwn(Pn, N, A, qm, beta=1e30, sigma=sigma, screened=screened)
        fd[:, d] = (wp - wm) / (qp[:, d].astype(np.float64) - qm[:, d])
    assert np.abs(fd - g).max() <= 2e-5 * np.abs(g).max()
