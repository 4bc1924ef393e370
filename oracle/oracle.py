"""ctypes front end of ``libdwg_oracle.so`` (the FP64 CPU restatement).

TEST INFRASTRUCTURE ONLY: this is the checker the CUDA path is compared
against.  Each wrapper names the reference function it restates; the C source
(``oracle/dwg_oracle.c``) cites file:line for every step.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdwg_oracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc)."""
    src = os.path.join(_HERE, "dwg_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class Params(C.Structure):
    _fields_ = [
        ("in_normal", C.c_int), ("grid_reso", C.c_int), ("final_reso", C.c_int),
        ("kw", C.c_int), ("final_kw", C.c_int), ("normal_kw", C.c_int), ("max_depth", C.c_int),
        ("lambda_", C.c_float), ("min_num", C.c_int), ("use_radii", C.c_int),
        ("offset_1", C.c_float), ("offset_2", C.c_float),
        ("use_leaves_generate", C.c_int), ("total_iter", C.c_int),
        ("beta", C.c_float), ("area", C.c_float), ("screen", C.c_float),
        ("knn_tri", C.c_int), ("knn_zero", C.c_int), ("as_thres", C.c_float), ("com_as", C.c_int),
    ]


_FIXTURE = os.path.join(os.path.dirname(_HERE), "tests", "golden", "mc_reference_loops.json")


def _reference_triangles():
    """The reference's triangles per case (src/TurboMC.cu:57-314) from the
    committed fixture (tests/golden/make_mc_fixture.py), as 256 x 16 int8."""
    import json

    with open(_FIXTURE) as f:
        cases = json.load(f)["cases"]
    tt = np.full((256, 16), -1, np.int8)
    for c in cases:
        flat = [e for t in c["tris"] for e in t]
        tt[c["case"], : len(flat)] = flat
    return tt.reshape(-1)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    L.dwgo_octree_build.restype = vp
    L.dwgo_octree_build.argtypes = [_f64p, C.c_int, C.c_int]
    L.dwgo_octree_free.argtypes = [vp]
    L.dwgo_octree_num_nodes.restype = C.c_int
    L.dwgo_octree_num_nodes.argtypes = [vp]
    L.dwgo_octree_export.argtypes = [vp, _i32p, _f64p, _f64p, _i32p, _i32p]
    L.dwgo_octree_lists.argtypes = [vp, _i64p, _i32p]
    L.dwgo_octree_dfs_order.argtypes = [vp, _i32p]
    L.dwgo_octree_dfs_starts.argtypes = [vp, _i32p]
    L.dwgo_moments.argtypes = [vp, _f32p, _f32p, _f32p, _f64p, _f64p, _f64p]
    L.dwgo_gwn_bh.argtypes = [vp, _f32p, _f32p, _f32p, _f32p, _f64p, _f64p, _f64p, _f32p,
                              C.c_longlong, C.c_float, C.c_float, C.c_int, C.c_int, C.c_float,
                              C.c_int, _f64p, _i64p]
    L.dwgo_gwn_bh_grad.argtypes = [vp, _f32p, _f32p, _f32p, _f32p, _f64p, _f64p, _f64p, _f32p,
                                   C.c_longlong, C.c_float, C.c_float, C.c_int, C.c_int, C.c_float,
                                   C.c_int, _f64p, _f64p]
    L.dwgo_gwn_exact.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, _f32p, C.c_longlong,
                                 C.c_float, C.c_int, C.c_int, C.c_float, C.c_int, _f64p]
    L.dwgo_voxel_grid.argtypes = [_f32p, C.c_int, C.c_float, C.c_int, _i32p, _f32p,
                                  C.POINTER(C.c_float)]
    L.dwgo_grid_points.argtypes = [_i32p, _f32p, C.c_float, _f32p]
    L.dwgo_mc_tables.argtypes = [_i32p, _i8p]
    L.dwgo_mc_polygons.argtypes = [_i32p, _i8p]
    L.dwgo_mc_set_triangles.argtypes = [_i8p]
    L.dwgo_mc_set_triangles(_reference_triangles())
    L.dwgo_marching_cubes.restype = C.c_longlong
    L.dwgo_marching_cubes.argtypes = [_f32p, _i32p, _f32p, C.c_float, C.c_float, vp, vp, vp,
                                      C.c_longlong, vp]
    L.dwgo_knn.argtypes = [_f32p, C.c_int, _f32p, C.c_longlong, C.c_int, C.c_int, _i32p]
    L.dwgo_diffuse_normals.restype = C.c_int
    L.dwgo_diffuse_normals.argtypes = [_i32p, _f32p, C.c_longlong, C.c_int, C.c_int, _f32p, _u8p]
    L.dwgo_zero_repair.argtypes = [_f32p, C.c_int, _f32p, _u8p, C.c_int, C.c_int]
    L.dwgo_gauss_map.argtypes = [_f32p, C.c_int, _f32p]
    L.dwgo_load_normals.argtypes = [_i32p, C.c_int, C.c_longlong, _f32p, _f32p]
    L.dwgo_radii.argtypes = [_f32p, C.c_int, _i32p, C.c_int, _f32p]
    L.dwgo_outlier_filter.argtypes = [_f32p, C.c_int, C.c_float]
    L.dwgo_expansion.argtypes = [vp, _f32p, _f32p, _f32p, _f64p, _f64p]
    L.dwgo_fwn.argtypes = [vp, _f32p, _f32p, _f32p, _f64p, _f64p, _f64p, _f64p, C.c_int, _f32p, C.c_longlong,
                           C.c_float, C.c_int, _f64p, _i64p]
    L.dwgo_pca_normals.argtypes = [_f32p, C.c_int, _i32p, C.c_int, _f32p, _f32p]
    L.dwgo_point_areas.argtypes = [_f32p, C.c_int, _i32p, C.c_int, _f32p, _f32p]
    L.dwgo_random_normals.argtypes = [C.c_int, _f32p]
    L.dwgo_reconstruct.restype = vp
    L.dwgo_reconstruct.argtypes = [_f32p, C.c_int, vp, C.POINTER(Params), C.c_int]
    L.dwgo_run_free.argtypes = [vp]
    L.dwgo_run_size.restype = C.c_longlong
    L.dwgo_run_size.argtypes = [vp, C.c_int]
    L.dwgo_run_get.restype = C.c_int
    L.dwgo_run_get.argtypes = [vp, C.c_char_p, vp]
    _lib = L
    return L


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


NTHREADS = max(1, min(os.cpu_count() or 1, 64))


class Octree:
    """igl::octreeDWG (deps/libigl/include/igl/octree.cpp:171-335)."""

    def __init__(self, P, max_depth):
        P64 = np.ascontiguousarray(P, dtype=np.float64)
        self.n = len(P64)
        self._h = lib().dwgo_octree_build(P64.reshape(-1), self.n, int(max_depth))
        M = lib().dwgo_octree_num_nodes(self._h)
        self.children = np.empty((M, 8), np.int32)
        self.centers = np.empty((M, 3), np.float64)
        self.widths = np.empty(M, np.float64)
        self.counts = np.empty(M, np.int32)
        self.depth = np.empty(M, np.int32)
        lib().dwgo_octree_export(self._h, self.children, self.centers, self.widths, self.counts,
                                 self.depth)

    @property
    def num_nodes(self):
        return len(self.counts)

    def lists(self):
        off = np.empty(self.num_nodes + 1, np.int64)
        tot = int(self.counts.astype(np.int64).sum())
        flat = np.empty(max(tot, 1), np.int32)
        lib().dwgo_octree_lists(self._h, off, flat)
        return off, flat[:tot]

    def dfs_order(self):
        perm = np.empty(max(self.n, 1), np.int32)
        lib().dwgo_octree_dfs_order(self._h, perm)
        return perm[: self.n]

    def dfs_starts(self):
        st = np.empty(self.num_nodes, np.int32)
        lib().dwgo_octree_dfs_starts(self._h, st)
        return st

    def moments(self, P, N, A):
        """fast_winding_number precompute, order 0 (fast_winding_number.cpp:9-120)."""
        M = self.num_nodes
        CM = np.empty((M, 3), np.float64)
        R = np.empty(M, np.float64)
        EC = np.empty((M, 3), np.float64)
        lib().dwgo_moments(self._h, _f32(P).reshape(-1), _f32(N).reshape(-1), _f32(A), CM, R, EC)
        return CM, R, EC

    def expansion(self, P, N, A, CM):
        """Expansion coefficients of orders 1 and 2 (fast_winding_number.cpp:87-105), (M, 36)."""
        HO = np.empty((self.num_nodes, 36), np.float64)
        lib().dwgo_expansion(self._h, _f32(P).reshape(-1), _f32(N).reshape(-1), _f32(A),
                             np.ascontiguousarray(CM, np.float64), HO)
        return HO

    def fwn(self, P, N, A, Q, order, beta=2.0, moments=None, nthreads=None):
        """Plain Barnes-Hut sum with far-field expansions of ``order`` (0-2),
        igl::fast_winding_number's expansion_eval; FP64.  ``moments`` =
        (CM, R, EC, HO) replaces the oracle's own.  Returns (w, terms)."""
        P = _f32(P).reshape(-1, 3)
        N = _f32(N).reshape(-1, 3)
        A = _f32(A)
        Q = _f32(Q).reshape(-1)
        nq = len(Q) // 3
        if moments is None:
            CM, R, EC = self.moments(P, N, A)
            HO = self.expansion(P, N, A, CM)
        else:
            CM, R, EC, HO = (np.ascontiguousarray(m, np.float64) for m in moments)
        out = np.empty(max(nq, 1), np.float64)
        terms = np.empty(max(nq, 1), np.int64)
        lib().dwgo_fwn(self._h, P.reshape(-1), N.reshape(-1), A, np.ascontiguousarray(CM), np.ascontiguousarray(R),
                       np.ascontiguousarray(EC), HO, int(order), Q, nq, float(beta), nthreads or NTHREADS, out, terms)
        return out[:nq], terms[:nq]

    def gwn(self, P, N, A, Q, beta=2.3, sigma=0.0, screened=True, radii=None, screen=0.0015,
            moments=None, nthreads=None):
        """Barnes-Hut GWN with the reference's per-query opening decisions
        (src/TurboLibiGWN.cu:328-836); FP64 sums.  Returns (w, terms)."""
        P = _f32(P).reshape(-1)
        N = _f32(N).reshape(-1)
        A = _f32(A)
        Q = _f32(Q).reshape(-1)
        nq = len(Q) // 3
        rad = _f32(radii) if radii is not None else np.zeros(1, np.float32)
        CM, R, EC = moments if moments is not None else self.moments(P.reshape(-1, 3), N.reshape(-1, 3), A)
        out = np.empty(max(nq, 1), np.float64)
        terms = np.empty(max(nq, 1), np.int64)
        lib().dwgo_gwn_bh(self._h, P, N, A, rad, np.ascontiguousarray(CM), np.ascontiguousarray(R),
                          np.ascontiguousarray(EC), Q, nq, beta, sigma, int(screened),
                          int(radii is not None), screen, nthreads or NTHREADS, out, terms)
        return out[:nq], terms[:nq]

    def gwn_grad(self, P, N, A, Q, beta=2.3, sigma=0.0, screened=True, radii=None, screen=0.0015,
                 moments=None, nthreads=None):
        """The sums of :meth:`gwn` and their analytic gradients with respect to
        the query (same decisions, FP64).  Returns (w, grad (nq x 3))."""
        P = _f32(P).reshape(-1)
        N = _f32(N).reshape(-1)
        A = _f32(A)
        Q = _f32(Q).reshape(-1)
        nq = len(Q) // 3
        rad = _f32(radii) if radii is not None else np.zeros(1, np.float32)
        CM, R, EC = moments if moments is not None else self.moments(P.reshape(-1, 3), N.reshape(-1, 3), A)
        out = np.empty(max(nq, 1), np.float64)
        g = np.empty(max(nq, 1) * 3, np.float64)
        lib().dwgo_gwn_bh_grad(self._h, P, N, A, rad, np.ascontiguousarray(CM), np.ascontiguousarray(R),
                               np.ascontiguousarray(EC), Q, nq, beta, sigma, int(screened),
                               int(radii is not None), screen, nthreads or NTHREADS, out, g)
        return out[:nq], g[: nq * 3].reshape(nq, 3)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.dwgo_octree_free(self._h)
            self._h = None


def gwn_exact(P, N, A, Q, sigma=0.0, screened=True, radii=None, screen=0.0015, nthreads=None):
    """Exact all-pairs sum of the same kernel (no far field)."""
    P = _f32(P).reshape(-1)
    Q = _f32(Q).reshape(-1)
    rad = _f32(radii) if radii is not None else np.zeros(1, np.float32)
    nq = len(Q) // 3
    out = np.empty(max(nq, 1), np.float64)
    lib().dwgo_gwn_exact(P, _f32(N).reshape(-1), _f32(A), rad, len(P) // 3, Q, nq, sigma,
                         int(screened), int(radii is not None), screen, nthreads or NTHREADS, out)
    return out[:nq]


def voxel_grid(P, offset, s):
    """igl::voxel_grid(V, offset, s, 1) in closed form: (res, origin, spacing)."""
    P = _f32(P).reshape(-1)
    res = np.empty(3, np.int32)
    org = np.empty(3, np.float32)
    h = C.c_float()
    lib().dwgo_voxel_grid(P, len(P) // 3, offset, int(s), res, org, C.byref(h))
    return res, org, np.float32(h.value)


def grid_points(res, origin, spacing):
    res = np.ascontiguousarray(res, np.int32)
    out = np.empty(int(np.prod(res.astype(np.int64))) * 3, np.float32)
    lib().dwgo_grid_points(res, _f32(origin), spacing, out)
    return out.reshape(-1, 3)


def mc_tables():
    """Edge masks and the reference's triangles per case (what the oracle's
    marching cubes uses)."""
    et = np.empty(256, np.int32)
    tt = np.empty(256 * 16, np.int8)
    lib().dwgo_mc_tables(et, tt)
    return et, tt.reshape(256, 16)


def mc_polygons():
    """Edge masks and the polygons the cube geometry implies, each fanned from
    its lowest edge (the oracle's own derivation, checked against the
    reference's triangles by the tests)."""
    et = np.empty(256, np.int32)
    tt = np.empty(256 * 16, np.int8)
    lib().dwgo_mc_polygons(et, tt)
    return et, tt.reshape(256, 16)


def marching_cubes(field, res, origin, spacing, iso, want=("tris", "centroids", "normals", "cases")):
    """src/TurboMC.cu:383-478 with deterministic (cell-major) triangle order."""
    field = _f32(field).reshape(-1)
    res = np.ascontiguousarray(res, np.int32)
    org = _f32(origin)
    T = lib().dwgo_marching_cubes(field, res, org, spacing, iso, None, None, None, 0, None)
    tris = np.empty((max(T, 1), 9), np.float32) if "tris" in want else None
    cen = np.empty((max(T, 1), 3), np.float32) if "centroids" in want else None
    nrm = np.empty((max(T, 1), 3), np.float32) if "normals" in want else None
    ncell = int(np.prod((res.astype(np.int64) - 1)))
    cases = np.empty(max(ncell, 1), np.uint8) if "cases" in want else None
    lib().dwgo_marching_cubes(field, res, org, spacing, iso, _ptr(tris), _ptr(cen), _ptr(nrm), T,
                              _ptr(cases))
    out = {"T": int(T)}
    if tris is not None:
        out["tris"] = tris[:T]
    if cen is not None:
        out["centroids"] = cen[:T]
    if nrm is not None:
        out["normals"] = nrm[:T]
    if cases is not None:
        out["cases"] = cases[:ncell]
    return out


def outlier_filter(A, thr):
    """OutlierFilter + AsFiltertoZero (src/TurboDWG.cu:991-1009, :442-454)."""
    A = np.ascontiguousarray(A, np.float32).copy()
    lib().dwgo_outlier_filter(A, len(A), C.c_float(thr))
    return A


def knn(P, Q, k, nthreads=None):
    """Brute-force k nearest, ordered by the cukd key (dist2 bits, id)."""
    P = _f32(P).reshape(-1)
    Q = _f32(Q).reshape(-1)
    nq = len(Q) // 3
    out = np.empty(max(nq * k, 1), np.int32)
    lib().dwgo_knn(P, len(P) // 3, Q, nq, int(k), nthreads or NTHREADS, out)
    return out[: nq * k].reshape(nq, k)


def diffuse_normals(knn_idx, tri_normals, normals):
    normals = _f32(normals).copy()
    L = len(normals)
    isz = np.zeros(max(L, 1), np.uint8)
    knn_idx = np.ascontiguousarray(knn_idx, np.int32)
    T, k = knn_idx.shape if knn_idx.size else (0, 15)
    zc = lib().dwgo_diffuse_normals(knn_idx.reshape(-1) if knn_idx.size else np.zeros(1, np.int32),
                                    _f32(tri_normals).reshape(-1) if T else np.zeros(3, np.float32),
                                    T, k, L, normals.reshape(-1), isz)
    return normals, isz[:L].astype(bool), zc


def zero_repair(Lpos, normals, is_zero, k=10, nthreads=None):
    normals = _f32(normals).copy()
    lib().dwgo_zero_repair(_f32(Lpos).reshape(-1), len(normals), normals.reshape(-1),
                           np.ascontiguousarray(is_zero, np.uint8), k, nthreads or NTHREADS)
    return normals


def gauss_map(P):
    P = _f32(P)
    out = np.empty_like(P)
    lib().dwgo_gauss_map(P.reshape(-1), len(P), out.reshape(-1))
    return out


def load_normals(knn_idx, leaf_normals):
    knn_idx = np.ascontiguousarray(knn_idx, np.int32)
    nq, k = knn_idx.shape
    out = np.empty((nq, 3), np.float32)
    lib().dwgo_load_normals(knn_idx.reshape(-1), k, nq, _f32(leaf_normals).reshape(-1),
                            out.reshape(-1))
    return out


def radii(P, knn_idx):
    P = _f32(P)
    knn_idx = np.ascontiguousarray(knn_idx, np.int32)
    out = np.empty(len(P), np.float32)
    lib().dwgo_radii(P.reshape(-1), len(P), knn_idx.reshape(-1), knn_idx.shape[1], out)
    return out


def pca_normals(P, knn_idx, view):
    """NormalEstimation (include/DWGProcess.h:152-200): smallest principal
    direction of each knn row, facing ``view``."""
    P = _f32(P)
    knn_idx = np.ascontiguousarray(knn_idx, np.int32)
    out = np.empty((len(P), 3), np.float32)
    lib().dwgo_pca_normals(P.reshape(-1), len(P), knn_idx.reshape(-1), knn_idx.shape[1],
                           _f32(view).reshape(3), out.reshape(-1))
    return out


def point_areas(P, knn_idx, normals):
    """igl::copyleft::cgal::point_areas (include/DWGProcess.h:345-378)."""
    P = _f32(P)
    knn_idx = np.ascontiguousarray(knn_idx, np.int32)
    out = np.empty(len(P), np.float32)
    lib().dwgo_point_areas(P.reshape(-1), len(P), knn_idx.reshape(-1), knn_idx.shape[1],
                           _f32(normals).reshape(-1), out)
    return out


def random_normals(n):
    """Seeded leaf normals of the --in_normal 2 --com_As 1 start."""
    out = np.empty((n, 3), np.float32)
    lib().dwgo_random_normals(int(n), out.reshape(-1))
    return out


DEFAULT_PARAMS = dict(in_normal=3, grid_reso=400, final_reso=500, kw=10, final_kw=10,
                      normal_kw=10, max_depth=10, lambda_=10.0, min_num=0, use_radii=0,
                      offset_1=0.05, offset_2=0.01, use_leaves_generate=0, total_iter=40,
                      beta=2.3, area=2e-6, screen=0.0015, knn_tri=15, knn_zero=10, as_thres=0.0,
                      com_as=0)


def reconstruct(P, normals=None, nthreads=None, **kw):
    """Full DWG reconstruction (include/DWGProcess.h:474-797, src/TurboDWG.cu:456-924)."""
    prm = dict(DEFAULT_PARAMS)
    prm.update(kw)
    p = Params(**prm)
    P = _f32(P)
    Nin = _f32(normals) if normals is not None else None
    h = lib().dwgo_reconstruct(P.reshape(-1), len(P), _ptr(Nin.reshape(-1)) if Nin is not None else None,
                               C.byref(p), nthreads or NTHREADS)
    L = lib()
    sz = [L.dwgo_run_size(h, i) for i in range(10)]
    Lc, Nn, T, it = sz[0], sz[1], sz[2], sz[3]
    fres = np.array(sz[4:7], np.int32)
    ires = np.array(sz[7:10], np.int32)
    out = {"L": Lc, "T": T, "final_res": fres, "iter_res": ires}

    def get(name, shape, dt):
        a = np.empty(max(int(np.prod(shape)), 1), dt)
        L.dwgo_run_get(h, name.encode(), a.ctypes.data_as(C.c_void_p))
        return a[: int(np.prod(shape))].reshape(shape)

    out["leaf_pos"] = get("leaf_pos", (Lc, 3), np.float32)
    out["leaf_nrm"] = get("leaf_nrm", (Lc, 3), np.float32)
    out["point_nrm"] = get("point_nrm", (Nn, 3), np.float32)
    out["tris"] = get("tris", (T, 9), np.float32)
    out["iso"] = get("iso", (it,), np.float32)
    out["tri_count"] = get("tri_count", (it,), np.int64)
    out["zero_count"] = get("zero_count", (it,), np.int32)
    out["final_field"] = get("final_field", (int(np.prod(fres.astype(np.int64))),), np.float32)
    out["final_iso"] = float(get("final_iso", (1,), np.float32)[0])
    L.dwgo_run_free(h)
    return out
