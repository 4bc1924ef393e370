"""GPU pipeline (full DWG reconstruction) against the oracle's reconstruction
on the same seeded cloud; and size-independent properties at larger sizes."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import datasets as D, turbo  # noqa: E402

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


SMALL = dict(grid_reso=40, final_reso=40, total_iter=6, max_depth=7)


@pytest.fixture(scope="module")
def small_runs(oracle_lib):
    P, N = D.sphere(3000, noise=0.002, seed=11)
    Pn, _, _ = D.normalize(P)
    ref = oracle_lib.reconstruct(Pn, **SMALL)
    got = turbo.reconstruct(cu(Pn), **SMALL)
    return Pn, ref, got


def test_pipeline_leaves_identical(small_runs):
    Pn, ref, got = small_runs
    assert np.array_equal(got["leaf_pos"], ref["leaf_pos"])


def test_pipeline_iso_and_counts_track_oracle(small_runs):
    Pn, ref, got = small_runs
    # FP32 terms (FP64 sums) vs the FP64 oracle: the first iterations agree to ~1e-6;
    # later ones drift a little as single-precision ties flip a few cells
    assert np.allclose(got["iso"][:2], ref["iso"][:2], rtol=1e-5, atol=1e-10)
    assert np.allclose(got["iso"], ref["iso"], rtol=2e-2, atol=1e-8)
    # triangle counts: identical unless a grid value sits within rounding of the iso
    assert np.all(np.abs(got["tri_count"] - ref["tri_count"]) <= 0.002 * ref["tri_count"] + 4)


def test_pipeline_normals_agree_with_oracle(small_runs):
    Pn, ref, got = small_runs
    agree = np.sign((got["leaf_nrm"] * ref["leaf_nrm"]).sum(1))
    assert agree.mean() > 0.99
    pa = np.sign((got["point_nrm"] * ref["point_nrm"]).sum(1))
    assert pa.mean() > 0.99


def test_pipeline_mesh_close_to_oracle(small_runs):
    Pn, ref, got = small_runs
    a = got["tris"].reshape(-1, 3, 3).mean(1)
    b = ref["tris"].reshape(-1, 3, 3).mean(1)
    assert abs(len(a) - len(b)) <= 0.01 * len(b) + 4
    from scipy.spatial import cKDTree
    d1 = cKDTree(b).query(a)[0]
    d2 = cKDTree(a).query(b)[0]
    chamfer = d1.mean() + d2.mean()
    h = 1.1 / 39
    assert chamfer < 0.05 * h


def test_pipeline_graph_replay_equals_eager(oracle_lib):
    P, _ = D.torus(4000, seed=2)
    Pn, _, _ = D.normalize(P)
    a = turbo.reconstruct(cu(Pn), use_graph=1, **SMALL)
    b = turbo.reconstruct(cu(Pn), use_graph=0, **SMALL)
    for k in ("leaf_nrm", "iso", "tri_count", "zero_count", "tris", "point_nrm"):
        assert np.array_equal(a[k], b[k]), k


def test_pipeline_input_normals_mode(oracle_lib):
    P, N = D.torus(4000, seed=3)
    Pn, _, _ = D.normalize(P)
    cfg = dict(SMALL, in_normal=1, total_iter=2)
    ref = oracle_lib.reconstruct(Pn, normals=N, **cfg)
    Pd, Nd = cu(Pn), cu(N)
    got = turbo.reconstruct(Pd, Nd, **cfg)
    assert np.array_equal(got["leaf_pos"], ref["leaf_pos"])
    assert np.allclose(got["iso"], ref["iso"], rtol=1e-4, atol=1e-10)


def test_pipeline_outlier_filter_tracks_oracle(oracle_lib):
    # --As_thres: the largest ceil(n * thr) areas (here all equal: the first in
    # canonical order) are divided by 1000 before the iterations and the final pass
    P, _ = D.sphere(3000, noise=0.002, seed=12)
    Pn, _, _ = D.normalize(P)
    cfg = dict(SMALL, total_iter=2, as_thres=0.3)
    ref = oracle_lib.reconstruct(Pn, **cfg)
    got = turbo.reconstruct(cu(Pn), **cfg)
    plain = turbo.reconstruct(cu(Pn), **dict(cfg, as_thres=0.0))
    assert np.array_equal(got["leaf_pos"], ref["leaf_pos"])
    assert np.allclose(got["iso"], ref["iso"], rtol=1e-5, atol=1e-10)
    # the final pass follows the iterations' normals, which FP32 vs FP64 sums
    # move slightly (as in the unfiltered comparison above)
    assert np.allclose(got["final_iso"], ref["final_iso"], rtol=2e-2, atol=1e-10)
    # the filter changes the sums (30 % of the areas divided by 1000)
    assert not np.allclose(got["iso"], plain["iso"], rtol=1e-2)
    assert abs(got["final_iso"] - plain["final_iso"]) > 0.1 * abs(plain["final_iso"])


@pytest.mark.parametrize("in_normal", [0, 2, 3])
def test_pipeline_com_as_tracks_oracle(oracle_lib, in_normal):
    # --com_As 1: PCA normals replace the input, leaf areas by point_areas
    # before the moments, point areas again in the final pass; in_normal 2
    # starts from the seeded random leaf normals
    P, _ = D.torus(4000, seed=21)
    Pn, _, _ = D.normalize(P)
    cfg = dict(SMALL, total_iter=2, com_as=1, in_normal=in_normal)
    ref = oracle_lib.reconstruct(Pn, **cfg)
    got = turbo.reconstruct(cu(Pn), **cfg)
    plain = turbo.reconstruct(cu(Pn), **dict(SMALL, total_iter=2, in_normal=3))
    assert np.array_equal(got["leaf_pos"], ref["leaf_pos"])
    # the areas are bit-identical; the sums differ by FP32 terms vs FP64
    # rounding (relative to the terms, so more where the mean cancels)
    assert np.allclose(got["iso"], ref["iso"], rtol=2e-4, atol=1e-10)
    assert np.all(np.abs(got["tri_count"] - ref["tri_count"]) <= 0.002 * ref["tri_count"] + 4)
    assert np.allclose(got["final_iso"], ref["final_iso"], rtol=1e-3, atol=1e-10)
    # the computed areas change the field (constant 2e-6 otherwise)
    assert not np.allclose(got["iso"], plain["iso"], rtol=1e-2)


def test_pipeline_com_as_random_start_matches_oracle(oracle_lib):
    # with no iterations the leaf normals are the seeded random start itself
    P, _ = D.sphere(3000, noise=0.002, seed=22)
    Pn, _, _ = D.normalize(P)
    cfg = dict(SMALL, total_iter=0, com_as=1, in_normal=2, use_leaves_generate=1)
    got = turbo.reconstruct(cu(Pn), **cfg)
    want = oracle_lib.random_normals(len(got["leaf_pos"]))
    assert np.allclose(got["leaf_nrm"], want, atol=1e-7)


def test_write_stl_device_matches_host_writer(tmp_path):
    import ctypes as C
    from dwg_b200 import capi
    lib = capi.load()
    P, _ = D.torus(4000, seed=5)
    Pn, _, _ = D.normalize(P)
    got = turbo.reconstruct(cu(Pn), **dict(SMALL, total_iter=2))
    tris = np.ascontiguousarray(got["tris"], np.float32)
    # more than one 2^20-triangle chunk of the device writer
    big = np.tile(tris, (int(np.ceil(2.5 * (1 << 20) / len(tris))), 1))[: int(2.5 * (1 << 20))]
    for t in (tris, big):
        fh, fd = tmp_path / "h.stl", tmp_path / "d.stl"
        assert lib.dwg_write_stl(str(fh).encode(), t.ctypes.data, len(t)) == 0
        td = cu(t)
        capi.check(lib.dwg_write_stl_device(str(fd).encode(), capi.ptr(td), len(t), None))
        assert fh.read_bytes() == fd.read_bytes()


@pytest.mark.parametrize("com_as", [0, 1])
def test_dwg_cuda_cli_end_to_end(tmp_path, com_as):
    # the DWG_CUDA command line (src/main.cpp flags): read .xyz, reconstruct,
    # write the binary STL (device packer) and the oriented .xyz
    import os
    import subprocess
    import struct
    exe = os.path.join(os.path.dirname(turbo.__file__), "bin", "DWG_CUDA")
    P, N = D.torus(3000, seed=8)
    with open(tmp_path / "t.xyz", "w") as fh:
        for p, n in zip(P, N):
            fh.write(f"{p[0]:.7f} {p[1]:.7f} {p[2]:.7f} {n[0]:.6f} {n[1]:.6f} {n[2]:.6f}\n")
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([exe, "--in_path", str(tmp_path), "--in_name", "t.xyz", "--out_path", str(out),
                        "--grid_reso", "40", "--final_reso", "40", "--total_iter", "2", "--max_depth", "7",
                        "--output_mode", "3", "--com_As", str(com_as)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    stl = out / "t_md_7_gr_40_iter_2.stl"
    b = stl.read_bytes()
    T = struct.unpack("<I", b[80:84])[0]
    assert T > 100 and len(b) == 84 + 50 * T
    xyz = np.loadtxt(out / "t_md_7_gr_40_iter_2.xyz")
    assert xyz.shape == (3000, 6)
    assert np.allclose(np.linalg.norm(xyz[:, 3:], axis=1), 1, atol=1e-3)


@pytest.mark.parametrize("tile", [0, 2])
def test_interaction_lists_replay_bit_identical(tile):
    # the recorded interaction lists replay exactly the traversal's terms
    P, _ = D.torus(5000, seed=41)
    Pn, _, _ = D.normalize(P)
    cfg = dict(SMALL, total_iter=9, tile=tile)
    b = turbo.reconstruct(cu(Pn), grid_lists=0, **cfg)
    for lists in (1, 2):  # 2: screening weights kept per sigma (20, then 10)
        a = turbo.reconstruct(cu(Pn), grid_lists=lists, **cfg)
        for k in ("leaf_nrm", "iso", "tri_count", "zero_count", "terms", "tris", "point_nrm", "final_iso"):
            assert np.array_equal(a[k], b[k]), (lists, k)
