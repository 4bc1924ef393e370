"""The product against the reference's OWN GPU code, compiled unchanged from
its sources (src/TurboLibiGWN.cu, src/TurboMC.cu, src/TurboDWG.cu,
src/TurboNormalInit.cu, src/KNN_GWN.cu) into oracle/_ref/libref_dwg.so by
oracle/ref_dwg.mk, and against the FP64 oracle on the same inputs.

* GWN sums: TurboLibiGWN (screened at sigma 20 and 10, plain) vs dwg_gwn_*.
  The reference computes in FP32 with --use_fast_math; the FP64 oracle with the
  same opening decisions as the product is the third arm.
* Marching cubes: TurboMC on identical fields; the same triangle count and
  the same triangles (matched one to one, vertices to rounding).
* The whole DWG run at BASELINE config 1 (10k noisy sphere, 128^3, 30
  iterations): the reference's TurboDWG loop and final pass vs the product's
  pipeline and the oracle's reconstruction, each measured against the
  reference's own run-to-run spread (a second reference run).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import datasets as D, turbo  # noqa: E402
from oracle import ref_dwg  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    if not ref_dwg.available():
        pytest.skip("reference comparator not built (oracle/ref_dwg.mk needs the reference checkout)")
    return ref_dwg


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rms(x):
    return float(np.sqrt(np.mean(np.square(x, dtype=np.float64))))


@pytest.fixture(scope="module")
def torus_case(oracle_lib):
    P, N = D.torus(20000, seed=3)
    Pn, _, _ = D.normalize(P)
    rng = np.random.default_rng(5)
    A = rng.uniform(1e-6, 3e-6, len(Pn)).astype(np.float32)
    Q = np.concatenate([Pn, rng.uniform(-0.55, 0.55, (20000, 3))]).astype(np.float32)
    return Pn, N.astype(np.float32), A, Q


@pytest.mark.parametrize("screened,sigma", [(True, 20.0), (True, 10.0), (False, 0.0)])
def test_gwn_sums_match_reference_turbolibigwn(ref, oracle_lib, torus_case, screened, sigma):
    Pn, N, A, Q = torus_case
    depth = 8
    rg = ref.RefGWN(Pn, depth, A=A)
    w_ref = rg.eval(N, A, Q, beta=2.3, sigma=sigma, screened=screened).astype(np.float64)
    rg.close()
    tree = turbo.TurboLibiGWN(cu(Pn), max_depth=depth, areas=cu(A))
    Nd, Ad, Qd = cu(N), cu(A), cu(Q)
    tree.UpdateMassNormals(Nd, Ad)
    out = torch.empty(len(Q), dtype=torch.float32, device="cuda")
    if screened:
        tree.TurboLibiScreenedGWNLaunch(Qd, None, len(Q), Nd, Ad, None, 2.3, sigma, out)
    else:
        tree.TurboLibiGWNLaunch(Qd, None, len(Q), Nd, Ad, 2.3, out)
    torch.cuda.synchronize()
    w_gpu = out.cpu().numpy().astype(np.float64)
    ot = oracle_lib.Octree(Pn, depth)
    w64, _ = ot.gwn(Pn, N, A, Q, beta=2.3, sigma=sigma, screened=screened)
    scale = np.abs(w64).max()
    d = np.abs(w_gpu - w_ref)
    # Both FP32; the reference uses fast-math exp / divide and a sequential FP32
    # sum, and decides "near/far" in fast-math FP32, so a borderline node can
    # open in one and not the other.  Bounds (of the field's max magnitude):
    assert rms(d) <= 2e-5 * scale, (rms(d) / scale)
    assert np.quantile(d, 0.999) <= 2e-4 * scale, (np.quantile(d, 0.999) / scale)
    # The product is at least as close to the FP64 sums as the reference.
    e_gpu, e_ref = rms(w_gpu - w64), rms(w_ref - w64)
    assert e_gpu <= e_ref * 1.05 + 1e-9 * scale, (e_gpu / scale, e_ref / scale)


@pytest.mark.parametrize("kind", ["gwn_torus", "sphere_sdf_plateau"])
def test_marching_cubes_matches_reference_turbomc(ref, oracle_lib, torus_case, kind):
    if kind == "gwn_torus":
        Pn, N, A, _ = torus_case
        res, org, h = oracle_lib.voxel_grid(Pn, 0.05, 72)
        G = oracle_lib.grid_points(res, org, h)
        ot = oracle_lib.Octree(Pn, 8)
        field, _ = ot.gwn(Pn, N, A, G, beta=2.3, sigma=10.0, screened=True)
        field = field.astype(np.float32)
        isos = [float(np.float32(np.mean(field))), float(np.float32(np.mean(field) * 0.5))]
    else:
        res = np.array([61, 53, 47], np.int32)
        org = np.float32([-0.5, -0.45, -0.4])
        h = np.float32(1 / 60)
        G = oracle_lib.grid_points(res, org, h)
        r = np.linalg.norm(G.astype(np.float64), axis=1)
        field = np.round((0.3 - r) * 64).astype(np.float32) / 64  # plateaus: many samples exactly at iso
        isos = [0.0, 1 / 64]
    for iso in isos:
        tris_r, cen_r, nrm_r = ref.marching_cubes(field, G, res, iso)
        cap = max(int(np.prod(res.astype(np.int64))) // 2, 1000000)
        mp = torch.empty((cap, 3), dtype=torch.float32, device="cuda")
        mn = torch.empty((cap, 3), dtype=torch.float32, device="cuda")
        mt = torch.empty((cap, 9), dtype=torch.float32, device="cuda")
        T = turbo.TurboMC().TurboMarchingCubes(cu(field), None, int(res[0]), int(res[1]), int(res[2]), iso,
                                               mid_points=mp, mid_normals=mn, origin=org, spacing=float(h),
                                               tris=mt)
        cen_m = mp[:T].cpu().numpy()
        nrm_m = mn[:T].cpu().numpy()
        tris_m = mt[:T].cpu().numpy()
        # identical triangle count (the case index of every cell decides it)
        assert len(cen_m) == len(cen_r) == len(tris_r) > 0, (len(cen_m), len(cen_r), len(tris_r))
        # Triangle for triangle: the reference appends a cell's triangles at an
        # atomicAdd slot, the product in cell order, so match every reference
        # triangle to the product triangle with the nearest centroid; the
        # matching must be one-to-one and the three vertices (in order) equal
        # to rounding.  The reference forms a vertex as P1 - l (P2 - P1)
        # contracted to one FMA and divides with fast-math; the product rounds
        # each operation (<= 2 ulp apart at coordinates below 0.6).
        from scipy.spatial import cKDTree
        dist, j = cKDTree(cen_m.astype(np.float64)).query(cen_r.astype(np.float64))
        assert len(np.unique(j)) == len(j)
        assert dist.max() <= 3e-7, dist.max()
        dv = np.abs(tris_m[j] - tris_r).max()
        assert dv <= 2.5e-7, dv
        # normals: -cross / (|cross| + 1e-8) of the same vertices; a sliver's
        # cross product is the difference of nearly equal products, so its
        # direction carries the rounding of the vertices (fast-math vs
        # correctly rounded): bound the normals of all but slivers
        # of a triangle by up to dv moves its unit normal by about
        # dv (|e1| + |e2|) / |e1 x e2|: bound every triangle by that
        v = tris_r.astype(np.float64).reshape(-1, 3, 3)
        e1, e2 = v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]
        cr_len = np.linalg.norm(np.cross(e1, e2), axis=1)
        lever = (np.linalg.norm(e1, axis=1) + np.linalg.norm(e2, axis=1)) / np.maximum(cr_len, 1e-30)
        dn = np.abs(nrm_m[j] - nrm_r).max(1)
        bound = 4 * max(float(dv), 1e-7) * lever + 2e-6
        assert np.all(dn <= bound), (dn / bound).max()


# BASELINE config 1.  as_thres: the reference's default 0 makes OutlierFilter
# launch AsFiltertoZero with zero blocks (src/TurboDWG.cu:1001-1008); the
# pending launch error then makes its next thrust::reduce throw under CUDA
# 12.9's thrust and the run ends.  1e-7 divides the area of exactly one leaf
# (and of one point in the final pass) by 1000 in all three arms.
C1 = dict(grid_reso=128, final_reso=128, total_iter=30, as_thres=1e-7)


@pytest.fixture(scope="module")
def c1_runs(ref, oracle_lib):
    P, _ = D.make("c1_sphere_10k", seed=0)
    Pn, _, _ = D.normalize(P)
    r = ref.reconstruct_isolated(Pn, **C1)
    r2 = ref.reconstruct_isolated(Pn, **C1)  # the reference's run-to-run spread (float atomics)
    got = turbo.reconstruct(cu(Pn), **C1)
    orc = oracle_lib.reconstruct(Pn, **C1)
    return Pn, r, got, orc, r2


def _match_rows(a, b):
    """Index of each row of b in a (rows are float32 positions present in both)."""
    key = {row.tobytes(): i for i, row in enumerate(np.ascontiguousarray(a, np.float32))}
    return np.array([key[row.tobytes()] for row in np.ascontiguousarray(b, np.float32)])


def _chamfer(ta, tb):
    from scipy.spatial import cKDTree
    a = ta.reshape(-1, 3, 3).mean(1)
    b = tb.reshape(-1, 3, 3).mean(1)
    return cKDTree(b).query(a)[0].mean() + cKDTree(a).query(b)[0].mean()


def test_c1_leaf_set_equals_reference(c1_runs):
    Pn, r, got, _, _ = c1_runs
    assert len(r["leaf_pos"]) == len(got["leaf_pos"])
    idx = _match_rows(got["leaf_pos"], r["leaf_pos"])
    assert len(np.unique(idx)) == len(idx)


def _leaf_agreement(a_pos, a_nrm, b_pos, b_nrm):
    idx = _match_rows(a_pos, b_pos)
    return float((np.sum(a_nrm[idx] * b_nrm, 1) > 0).mean())


def _point_normals(r):
    """The reference writes the final points in kd order: back to input order."""
    out = np.empty_like(r["point_nrm"])
    out[r["perm"]] = r["point_nrm"]
    return out


def _ref_iso(r):
    t = np.arange(C1["total_iter"])
    return r["w_mean"] * np.where((t % 5 == 0) & (t != 0), 0.5, 1.0)


def test_c1_iso_and_triangle_counts_track_reference(c1_runs):
    Pn, r, got, orc, r2 = c1_runs
    ref_iso = _ref_iso(r)
    d_iso = np.abs(got["iso"] - ref_iso)
    d_iso_o = np.abs(orc["iso"] - ref_iso)
    d_iso_r = np.abs(_ref_iso(r2) - ref_iso)
    rel = np.abs(got["tri_count"] - r["tri_count"]) / r["tri_count"]
    rel_o = np.abs(orc["tri_count"] - r["tri_count"]) / r["tri_count"]
    rel_r = np.abs(r2["tri_count"] - r["tri_count"]) / r["tri_count"]
    print(f"C1 vs reference: |d iso| first two {d_iso[:2]}, max {d_iso.max():.3g} "
          f"(oracle {d_iso_o.max():.3g}, reference rerun {d_iso_r.max():.3g}); triangle counts rel diff "
          f"first two {rel[:2]}, mean {rel.mean():.3g}, max {rel.max():.3g} (oracle mean {rel_o.mean():.3g}, "
          f"reference rerun mean {rel_r.mean():.3g})")
    # The mean winding number is a small difference of O(1) field values: its
    # error is absolute (the reference sums in fast-math FP32).  Iterations 0
    # and 1 start from the same Gauss map and the same polygons.
    assert d_iso[:2].max() <= 2e-6, d_iso[:2]
    assert rel[:2].max() <= 2e-3, rel[:2]
    # Later iterations drift as rounding moves single cells across the iso
    # value; the product stays as close to the reference as the FP64 oracle
    assert d_iso.max() <= max(5e-5, 2 * d_iso_o.max()), d_iso.max()
    assert rel.mean() <= max(1e-2, 1.5 * rel_o.mean()), rel


def test_c1_orientation_agrees_with_reference(c1_runs):
    Pn, r, got, orc, r2 = c1_runs
    ag = _leaf_agreement(got["leaf_pos"], got["leaf_nrm"], r["leaf_pos"], r["leaf_nrm"])
    ag_o = _leaf_agreement(orc["leaf_pos"], orc["leaf_nrm"], r["leaf_pos"], r["leaf_nrm"])
    ag_r = _leaf_agreement(r2["leaf_pos"], r2["leaf_nrm"], r["leaf_pos"], r["leaf_nrm"])
    ag_go = _leaf_agreement(got["leaf_pos"], got["leaf_nrm"], orc["leaf_pos"], orc["leaf_nrm"])
    pn_ref = _point_normals(r)
    pa = float((np.sum(got["point_nrm"] * pn_ref, 1) > 0).mean())
    pa_o = float((np.sum(orc["point_nrm"] * pn_ref, 1) > 0).mean())
    pa_r = float((np.sum(_point_normals(r2) * pn_ref, 1) > 0).mean())
    print(f"C1 leaf orientation agreement: product-reference {ag:.5f}, oracle-reference {ag_o:.5f}, "
          f"reference-rerun {ag_r:.5f}, product-oracle {ag_go:.5f}; points: product-reference {pa:.5f}, "
          f"oracle-reference {pa_o:.5f}, reference-rerun {pa_r:.5f}")
    assert ag > 0.97 and pa > 0.97, (ag, pa)
    assert ag >= min(ag_o, ag_r) - 0.005 and pa >= min(pa_o, pa_r) - 0.005


def test_c1_final_mesh_close_to_reference(c1_runs):
    Pn, r, got, orc, r2 = c1_runs
    cell = 1.1 / (C1["final_reso"] - 1)
    T_ref, T_got = len(r["tris"]), len(got["tris"])
    ch = _chamfer(got["tris"], r["tris"]) / cell
    ch_o = _chamfer(orc["tris"], r["tris"]) / cell
    ch_r = _chamfer(r2["tris"], r["tris"]) / cell
    ch_go = _chamfer(got["tris"], orc["tris"]) / cell
    print(f"C1 final mesh: triangles product {T_got}, reference {T_ref}, rerun {len(r2['tris'])}, oracle "
          f"{len(orc['tris'])}; Chamfer in cells product-reference {ch:.4f}, oracle-reference {ch_o:.4f}, "
          f"reference-rerun {ch_r:.4f}, product-oracle {ch_go:.4f}; reference device seconds {r['secs']}")
    assert abs(T_got - T_ref) <= 0.02 * T_ref, (T_got, T_ref)
    # Two runs of the reference itself differ by a fraction of a cell (its
    # float atomics sum in a different order each run and the loop amplifies
    # it); the product must be no farther from the reference than that spread
    # or the FP64 oracle's distance, with a 20 % margin.
    assert ch <= 1.2 * max(ch_o, ch_r), (ch, ch_o, ch_r)
