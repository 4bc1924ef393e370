"""CPU tests of the C ABI: the library loads, exports every symbol the header
declares, rejects bad arguments before touching the GPU, generates the
reference-pinned case table, and reads/writes the reference's file formats."""
import ctypes as C
import os
import re
import struct

import numpy as np
import pytest

from dwg_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dwg_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(dwg_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(dwg_lib):
    names = declared_functions()
    assert len(names) > 30
    for n in names:
        assert hasattr(dwg_lib, n), n
    # and the binding covers them all
    assert set(names) <= set(capi.exported_symbols())
    assert dwg_lib.dwg_version().startswith(b"dwg_b200")


def test_mc_table_matches_reference_fixture_and_oracle(dwg_lib, oracle_lib):
    """Edge masks from the cube geometry; triangles per case equal to the
    reference's (the fixture read from src/TurboMC.cu), which the library
    checks against the polygons the geometry gives."""
    from tests.test_oracle import check_table_against_fixture, reference_triangles
    et = np.zeros(256, np.int32)
    tt = np.zeros(256 * 16, np.int8)
    assert dwg_lib.dwg_mc_tables(et.ctypes.data, tt.ctypes.data) == 0
    tt = tt.reshape(256, 16)
    check_table_against_fixture(et, tt)
    assert np.array_equal(tt, reference_triangles())
    oet, ott = oracle_lib.mc_tables()
    assert np.array_equal(et, oet) and np.array_equal(tt, ott)


def test_invalid_arguments_are_rejected(dwg_lib):
    L = dwg_lib
    h = C.c_void_p()
    assert L.dwg_octree_build(None, 10, 8, None, None, C.byref(h)) == capi.DWG_ERR_INVALID
    assert b"null" in L.dwg_last_error()
    assert L.dwg_octree_build(1, 10, 8, None, None, None) == capi.DWG_ERR_INVALID
    assert L.dwg_knn(1, 5, 1, 3, 0, 1, None) == capi.DWG_ERR_INVALID          # k = 0
    assert L.dwg_knn(1, 5, 1, 3, 6, 1, None) == capi.DWG_ERR_INVALID          # k > n
    assert b"k=6" in L.dwg_last_error()
    assert L.dwg_pipeline_create(1, None, 100, None, None, C.byref(h)) == capi.DWG_ERR_INVALID
    p = capi.default_params()
    assert L.dwg_pipeline_create(None, None, 100, C.byref(p), None, C.byref(h)) == capi.DWG_ERR_INVALID
    p.in_normal = 1  # needs input normals
    assert L.dwg_pipeline_create(1, None, 100, C.byref(p), None, C.byref(h)) == capi.DWG_ERR_INVALID
    assert L.dwg_mc_tables(None, None) == capi.DWG_ERR_INVALID


def test_default_params_match_dwg_cuda_flags(dwg_lib):
    # src/main.cpp:19-39 and the hard-coded constants of the reference
    p = capi.default_params()
    assert (p.in_normal, p.grid_reso, p.final_reso, p.kw, p.final_kw, p.normal_kw, p.max_depth) == \
        (3, 400, 500, 10, 10, 10, 10)
    assert p.lambda_ == 10.0 and p.min_num == 0 and p.use_radii == 0 and p.total_iter == 40
    assert abs(p.offset_1 - 0.05) < 1e-7 and abs(p.offset_2 - 0.01) < 1e-7
    assert abs(p.beta - 2.3) < 1e-6 and abs(p.area - 2e-6) < 1e-12 and abs(p.screen - 0.0015) < 1e-9
    assert (p.knn_tri, p.knn_zero) == (15, 10)
    # this library's own switches: CUDA graphs on, FP32 terms summed in FP64,
    # interaction lists with kept screening weights
    assert (p.use_graph, p.precision, p.grid_lists, p.com_as) == (1, 1, 2, 0)


def test_ctypes_structs_match_the_header():
    # field names and order of the ctypes mirrors follow include/dwg_b200.h
    import re
    hdr = open(os.path.join(ROOT, "include", "dwg_b200.h")).read()

    def fields(struct):
        body = re.search(r"typedef struct\s*\{([^{}]*)\}\s*" + struct + r"\s*;", hdr).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        decls = re.findall(r"\b(?:int|float|double|long long)\s+([\w\s,]+);", body)
        return [n.strip() for d in decls for n in d.split(",")]

    assert [f for f, _ in capi.GwnParams._fields_] == fields("dwg_gwn_params")
    assert [f.rstrip("_") for f, _ in capi.Params._fields_] == fields("dwg_params")


def test_read_xyz_normalises_like_the_reference(dwg_lib, tmp_path):
    rng = np.random.default_rng(0)
    P = rng.uniform(-3, 7, (50, 3))
    N = rng.standard_normal((50, 3))
    f = tmp_path / "c.xyz"
    with open(f, "w") as fh:
        for p, n in zip(P, N):
            fh.write(" ".join(f"{v:.9f}" for v in (*p, *n)) + "\n")
    pts = C.POINTER(C.c_float)()
    nrm = C.POINTER(C.c_float)()
    n = C.c_int()
    assert dwg_lib.dwg_read_xyz(str(f).encode(), 1, C.byref(pts), C.byref(nrm), C.byref(n)) == 0
    got = np.ctypeslib.as_array(pts, (n.value, 3)).copy()
    gotn = np.ctypeslib.as_array(nrm, (n.value, 3)).copy()
    dwg_lib.dwg_free_host(C.cast(pts, C.c_void_p))
    dwg_lib.dwg_free_host(C.cast(nrm, C.c_void_p))
    Pr = np.array([[float(f"{v:.9f}") for v in p] for p in P])
    c = Pr.mean(0)
    scale = np.max(2 * np.abs(Pr - c))
    assert np.allclose(got, ((Pr - c) / scale).astype(np.float32), atol=1e-7)
    assert np.abs(got).max() <= 0.5 + 1e-6
    assert np.allclose(gotn, N, atol=1e-6)


def test_read_xyz_rejects_malformed(dwg_lib, tmp_path):
    f = tmp_path / "bad.xyz"
    f.write_text("1 2 3\n4 5\n")
    pts = C.POINTER(C.c_float)()
    n = C.c_int()
    assert dwg_lib.dwg_read_xyz(str(f).encode(), 1, C.byref(pts), None, C.byref(n)) == capi.DWG_ERR_INVALID
    assert b"line 2" in dwg_lib.dwg_last_error()
    f.write_text("1 2 nan\n")
    assert dwg_lib.dwg_read_xyz(str(f).encode(), 1, C.byref(pts), None, C.byref(n)) == capi.DWG_ERR_INVALID
    assert dwg_lib.dwg_read_xyz(b"/nonexistent/x.xyz", 1, C.byref(pts), None, C.byref(n)) == capi.DWG_ERR_INVALID


def test_write_stl_binary_format(dwg_lib, tmp_path):
    tris = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0], [0, 0, 0, 0, 0, 1, 1, 0, 0]], np.float32)
    f = tmp_path / "m.stl"
    assert dwg_lib.dwg_write_stl(str(f).encode(), tris.ctypes.data, 2) == 0
    b = f.read_bytes()
    assert len(b) == 80 + 4 + 2 * 50
    assert struct.unpack("<I", b[80:84])[0] == 2
    rec = struct.unpack("<12fH", b[84:134])
    assert rec[:3] == (0.0, 0.0, 1.0)  # cross((1,0,0),(0,1,0))
    assert rec[3:12] == tuple(tris[0])


def test_write_xyz(dwg_lib, tmp_path):
    P = np.array([[0.5, 1, 2]], np.float32)
    N = np.array([[0, 0, 1]], np.float32)
    f = tmp_path / "o.xyz"
    assert dwg_lib.dwg_write_xyz(str(f).encode(), P.ctypes.data, N.ctypes.data, 1) == 0
    assert [float(x) for x in f.read_text().split()] == [0.5, 1, 2, 0, 0, 1]


def test_read_xyz_chunked_parse_matches_python(dwg_lib, tmp_path):
    # a file large enough to be parsed in several newline-aligned chunks:
    # mixed 3/6-column lines, blank lines, signs, exponents, CRLF endings;
    # every value must be the correctly rounded double (as %lf / float())
    rng = np.random.default_rng(5)
    rows, want_p, want_n = [], [], []
    for i in range(60000):
        if i % 997 == 0:
            rows.append("")
        p = rng.uniform(-50, 50, 3)
        toks = [f"{x:+.7e}" if i % 3 == 0 else repr(float(x)) for x in p]
        if i % 2:
            nn = rng.standard_normal(3)
            toks += [f"{x:.6f}" for x in nn]
            want_n.append([float(t) for t in toks[3:]])
        else:
            want_n.append([0.0, 0.0, 0.0])
        want_p.append([float(t) for t in toks[:3]])
        rows.append(" \t".join(toks) + ("\r" if i % 5 == 0 else ""))
    f = tmp_path / "big.xyz"
    f.write_text("\n".join(rows) + "\n")
    assert f.stat().st_size > 3 << 20
    pts = C.POINTER(C.c_float)()
    nrm = C.POINTER(C.c_float)()
    n = C.c_int()
    assert dwg_lib.dwg_read_xyz(str(f).encode(), 0, C.byref(pts), C.byref(nrm), C.byref(n)) == 0
    got = np.ctypeslib.as_array(pts, (n.value, 3)).copy()
    gotn = np.ctypeslib.as_array(nrm, (n.value, 3)).copy()
    dwg_lib.dwg_free_host(C.cast(pts, C.c_void_p))
    dwg_lib.dwg_free_host(C.cast(nrm, C.c_void_p))
    assert n.value == len(want_p)
    assert np.array_equal(got, np.array(want_p).astype(np.float32))
    assert np.array_equal(gotn, np.array(want_n).astype(np.float32))
    # an error far into the file is reported with its line number
    rows2 = list(rows)
    rows2[50001] = "1.0 2.0"
    f.write_text("\n".join(rows2) + "\n")
    assert dwg_lib.dwg_read_xyz(str(f).encode(), 0, C.byref(pts), None, C.byref(n)) == capi.DWG_ERR_INVALID
    assert b"line 50002 " in dwg_lib.dwg_last_error()


def test_write_stl_many_triangles_threaded(dwg_lib, tmp_path):
    rng = np.random.default_rng(2)
    T = 300000
    tris = rng.uniform(-1, 1, (T, 9)).astype(np.float32)
    tris[7, 3:6] = tris[7, 0:3]  # degenerate: zero normal
    f = tmp_path / "m.stl"
    assert dwg_lib.dwg_write_stl(str(f).encode(), tris.ctypes.data, T) == 0
    b = f.read_bytes()
    assert len(b) == 84 + 50 * T
    rec = np.frombuffer(b[84:], dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]))
    assert np.array_equal(rec["v"], tris) and not rec["a"].any()
    e1, e2 = tris[:, 3:6] - tris[:, 0:3], tris[:, 6:9] - tris[:, 0:3]
    c = np.cross(e1, e2)
    with np.errstate(invalid="ignore"):
        nn = c / np.linalg.norm(c, axis=1, keepdims=True)
    ok = np.isfinite(nn).all(1)
    assert np.allclose(rec["n"][ok], nn[ok], atol=1e-6)
    assert not rec["n"][7].any()
