"""Python mirror of the reference's operator classes over the C ABI.

Class and method names follow the reference (DWGTech/DWG):

* ``TurboNormalInitialization.GaussMapInit``   -- include/TurboNormalInit.h:9-14
* ``TurboLibiGWN`` (PreLibiGWN, UpdateMassNormals, UpdateGWNInfo,
  TurboLibiGWNLaunch, TurboLibiScreenedGWNLaunch, EarseMemory)
                                                 -- include/Turbo_GWN_l.h:24-69
* ``TurboMC.TurboMarchingCubes``                 -- include/MarchingCubeCuda.h:35-44
* ``GenerateKDTreeForDWG`` / ``CudaKNNWithKDTreeforDWG``
                                                 -- include/TurboDWG.h:14-27
* ``TurboDWG`` (the iteration and meshing driver) -- include/TurboDWG.h:29-74

Eigen matrices and std::vector arguments of the reference become torch CUDA
tensors of shape (n, 3) / (n,), float32; the CPU octree inputs (O_PI, O_CH,
O_CM, O_R, O_EC) are replaced by a GPU octree built from the points.  Every
call runs the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi


def _req_cuda_f32(t, name, shape_last=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.float32:
        raise TypeError(f"{name} must be float32")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if shape_last is not None and (t.dim() != 2 or t.shape[1] != shape_last):
        raise ValueError(f"{name} must have shape (n, {shape_last})")
    return t


class TurboNormalInitialization:
    """Gauss-map normal initialisation (src/TurboNormalInit.cu:29-44)."""

    def GaussMapInit(self, point_pos, point_normal, bound_upper=None, bound_lower=None, point_num=None):
        _req_cuda_f32(point_pos, "point_pos", 3)
        _req_cuda_f32(point_normal, "point_normal", 3)
        n = point_pos.shape[0] if point_num is None else int(point_num)
        if bound_upper is not None or bound_lower is not None:
            # the reference passes the kd-tree bounds; they equal the bounding box
            pass
        capi.check(capi.load().dwg_gauss_map_init(capi.ptr(point_pos), n, capi.ptr(point_normal),
                                                  capi.stream_ptr()))
        return point_normal


class TurboLibiGWN:
    """Screened / plain generalised winding number with a GPU octree.

    ``TurboLibiGWN(points, max_depth, areas)`` replaces the reference's
    ``TurboLibiGWN(O_PI, O_CH, O_CM, O_R, O_EC)`` + ``PreLibiGWN``: the
    octree (octreeDWG topology) and its moments are built on the GPU."""

    def __init__(self, point_cloud=None, max_depth=10, areas=None):
        self._h = C.c_void_p()
        self.n = 0
        if point_cloud is not None:
            self.PreLibiGWN(point_cloud, max_depth, areas)

    def PreLibiGWN(self, point_cloud, max_depth=10, areas=None):
        _req_cuda_f32(point_cloud, "point_cloud", 3)
        self.EarseMemory()
        self.points = point_cloud
        self.n = point_cloud.shape[0]
        capi.check(capi.load().dwg_octree_build(capi.ptr(point_cloud), self.n, int(max_depth),
                                                capi.ptr(areas), capi.stream_ptr(), C.byref(self._h)))

    def num_nodes(self):
        v = C.c_int()
        capi.check(capi.load().dwg_octree_num_nodes(self._h, C.byref(v)))
        return v.value

    def UpdateMassNormals(self, i_Normals, i_As):
        capi.check(capi.load().dwg_octree_update_normals(self._h, capi.ptr(i_Normals), capi.ptr(i_As),
                                                         capi.stream_ptr()))

    def UpdateGWNInfo(self, i_Normals, point_cloud=None, i_As=None):
        capi.check(capi.load().dwg_octree_update_info(self._h, capi.ptr(i_Normals), capi.ptr(i_As),
                                                      capi.stream_ptr()))

    def _launch(self, query_points, i_Normals, i_As, radii, params, out_gwn, terms=None):
        _req_cuda_f32(query_points, "query_points", 3)
        nq = query_points.shape[0]
        if out_gwn is None:
            out_gwn = torch.empty(nq, dtype=torch.float32, device=query_points.device)
        capi.check(capi.load().dwg_gwn_points(
            self._h, capi.ptr(i_Normals), capi.ptr(i_As), capi.ptr(radii), capi.ptr(query_points), nq,
            C.byref(params), capi.ptr(out_gwn), capi.ptr(terms), capi.stream_ptr()))
        return out_gwn

    def TurboLibiGWNLaunch(self, query_points, point_cloud=None, query_size=None, i_Normals=None, i_As=None,
                           beta=2.3, out_gwn=None, precision=1, order=0):
        """Plain GWN, sum A (p-q).n / (4 pi r^3 + 1e-8) (src/TurboLibiGWN.cu:328-511,899-910);
        ``order`` 1 or 2 adds igl::fast_winding_number's far-field expansion
        terms (deps/libigl/include/igl/fast_winding_number.cpp:187-241)."""
        p = capi.gwn_params(beta=beta, sigma=0.0, screened=False, precision=precision, order=order)
        return self._launch(query_points, i_Normals, i_As, None, p, out_gwn)

    def TurboLibiScreenedGWNLaunch(self, query_points, point_cloud=None, query_size=None, i_Normals=None,
                                   i_As=None, i_radii=None, beta=2.3, sigma=10.0, out_gwn=None, use_radii=False,
                                   precision=1, screen=0.0015):
        """Screened GWN (src/TurboLibiGWN.cu:513-812,912-922)."""
        p = capi.gwn_params(beta=beta, sigma=sigma, screen=screen, screened=True, use_radii=use_radii,
                            precision=precision)
        return self._launch(query_points, i_Normals, i_As, i_radii if use_radii else None, p, out_gwn)

    def grid(self, res, origin, spacing, i_Normals=None, i_As=None, beta=2.3, sigma=10.0, screened=True,
             precision=1, out=None, terms=None, screen=0.0015, tile=0, order=0, lists=0, i_radii=None):
        """GWN at the closed-form grid origin + index * spacing (x fastest);
        ``tile`` picks the brick of samples a warp evaluates together;
        ``i_radii`` (per point) switches the screening radius to the points'
        radii (use_radii)."""
        res = np.ascontiguousarray(res, np.int32)
        org = np.ascontiguousarray(origin, np.float32)
        n = int(np.prod(res.astype(np.int64)))
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device="cuda")
        p = capi.gwn_params(beta=beta, sigma=sigma, screen=screen, screened=screened, precision=precision,
                            tile=tile, order=order, lists=lists, use_radii=i_radii is not None)
        capi.check(capi.load().dwg_gwn_grid(self._h, capi.ptr(i_Normals), capi.ptr(i_As), capi.ptr(i_radii),
                                            res.ctypes.data,
                                            org.ctypes.data, float(spacing), C.byref(p), capi.ptr(out),
                                            capi.ptr(terms), capi.stream_ptr()))
        return out

    def value_and_gradient(self, query_points=None, i_Normals=None, i_As=None, i_radii=None, beta=2.3, sigma=10.0,
                           screened=True, screen=0.0015, fp64=False, grid=None):
        """Sums and their gradients with respect to the query at points
        (``query_points``, (n, 3) float32 on the GPU) or at a grid
        (``grid`` = (res, origin, spacing)): (w, grad) tensors, float32 (FP32
        terms summed in FP64) or float64 (``fp64``: terms and sums in double).
        The reference has no gradient; see dwg_gwn_points_grad."""
        p = capi.gwn_params(beta=beta, sigma=sigma, screen=screen, screened=screened,
                            use_radii=i_radii is not None)
        dt = torch.float64 if fp64 else torch.float32
        L = capi.load()
        if grid is None:
            _req_cuda_f32(query_points, "query_points", 3)
            nq = query_points.shape[0]
        else:
            res = np.ascontiguousarray(grid[0], np.int32)
            org = np.ascontiguousarray(grid[1], np.float32)
            nq = int(np.prod(res.astype(np.int64)))
        w = torch.empty(nq, dtype=dt, device="cuda")
        g = torch.empty((nq, 3), dtype=dt, device="cuda")
        args = (self._h, capi.ptr(i_Normals), capi.ptr(i_As), capi.ptr(i_radii))
        if grid is None:
            fn = L.dwg_gwn_points_fp64 if fp64 else L.dwg_gwn_points_grad
            capi.check(fn(*args, capi.ptr(query_points), nq, C.byref(p), capi.ptr(w), capi.ptr(g), capi.stream_ptr()))
        else:
            fn = L.dwg_gwn_grid_fp64 if fp64 else L.dwg_gwn_grid_grad
            capi.check(fn(*args, res.ctypes.data, org.ctypes.data, float(grid[2]), C.byref(p), capi.ptr(w),
                          capi.ptr(g), capi.stream_ptr()))
        return w, g

    def values_fp64(self, query_points, i_Normals=None, i_As=None, i_radii=None, beta=2.3, sigma=10.0,
                    screened=True, screen=0.0015):
        """FP64 sums (terms and sums in double, the FP32 kernels' decisions)
        at points: a float64 tensor (dwg_gwn_points_fp64)."""
        _req_cuda_f32(query_points, "query_points", 3)
        p = capi.gwn_params(beta=beta, sigma=sigma, screen=screen, screened=screened, use_radii=i_radii is not None)
        w = torch.empty(query_points.shape[0], dtype=torch.float64, device=query_points.device)
        capi.check(capi.load().dwg_gwn_points_fp64(self._h, capi.ptr(i_Normals), capi.ptr(i_As), capi.ptr(i_radii),
                                                   capi.ptr(query_points), query_points.shape[0], C.byref(p),
                                                   capi.ptr(w), None, capi.stream_ptr()))
        return w

    def list_size(self):
        """(entries, weight slots) of the kept interaction list of grid()."""
        e = C.c_longlong()
        w = C.c_int()
        capi.check(capi.load().dwg_octree_list_size(self._h, C.byref(e), C.byref(w)))
        return e.value, w.value

    def status(self):
        """Sticky traversal error flags (0 = none); raises on a set flag."""
        f = C.c_uint()
        capi.check(capi.load().dwg_octree_status(self._h, C.byref(f)))
        return f.value

    def export(self):
        """Node table (host numpy): depth, pt_start, pt_count, skip, cm, radius, ec, perm."""
        M = self.num_nodes()
        out = dict(depth=np.empty(M, np.int32), pt_start=np.empty(M, np.int32), pt_count=np.empty(M, np.int32),
                   skip=np.empty(M, np.int32), cm=np.empty((M, 3), np.float64), radius=np.empty(M, np.float64),
                   ec=np.empty((M, 3), np.float64), perm=np.empty(max(self.n, 1), np.int32))
        capi.check(capi.load().dwg_octree_export(
            self._h, *[out[k].ctypes.data for k in ("depth", "pt_start", "pt_count", "skip", "cm", "radius",
                                                    "ec", "perm")]))
        out["perm"] = out["perm"][: self.n]
        return out

    def expansion(self):
        """FP64 far-field coefficients of orders 1 and 2, (M, 36): m1 (9), m2 (27)."""
        out = np.empty((self.num_nodes(), 36), np.float64)
        capi.check(capi.load().dwg_octree_expansion(self._h, out.ctypes.data, capi.stream_ptr()))
        return out

    def EarseMemory(self):
        if getattr(self, "_h", None) and self._h.value:
            capi.load().dwg_octree_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.EarseMemory()
        except Exception:
            pass


class TurboMC:
    """Marching cubes (src/TurboMC.cu:572-638)."""

    def TurboMarchingCubes(self, voxel_values, voxel_poses, res_x, res_y, res_z, threshold, iterations=0,
                           mesh_path="", mesh_full_path="", mid_points=None, mid_normals=None, test_iter=999999,
                           origin=None, spacing=None, tris=None, capacity=None):
        """Returns the triangle count; writes a binary STL when
        ``iterations == 123456`` (to mesh_full_path + '.stl') or when
        ``iterations % test_iter == 0`` with test_iter != 999999, as the
        reference does."""
        res = np.array([res_x, res_y, res_z], np.int32)
        ncell = (res_x - 1) * (res_y - 1) * (res_z - 1)
        if capacity is None:
            capacity = max(res_x * res_y * res_z // 2, 1000000)
        want_stl = (test_iter != 999999 and iterations % test_iter == 0) or iterations == 123456
        if want_stl and tris is None:
            tris = torch.empty((capacity, 9), dtype=torch.float32, device=voxel_values.device)
        org = np.ascontiguousarray(origin if origin is not None else [0, 0, 0], np.float32)
        T = C.c_longlong()
        cnt = torch.zeros(1, dtype=torch.int64, device=voxel_values.device)
        rc = capi.load().dwg_marching_cubes(
            capi.ptr(voxel_values), res.ctypes.data, capi.ptr(voxel_poses),
            org.ctypes.data if voxel_poses is None else None, float(spacing or 0.0), float(threshold),
            capi.ptr(tris), capi.ptr(mid_points), capi.ptr(mid_normals), int(capacity), capi.ptr(cnt),
            C.byref(T), capi.stream_ptr())
        capi.check(rc)
        del ncell
        if want_stl:
            path = (mesh_full_path + ".stl") if iterations == 123456 else f"{mesh_path}{iterations}iter.stl"
            host = tris[: T.value].cpu().numpy()
            capi.check(capi.load().dwg_write_stl(path.encode(), host.ctypes.data, T.value))
        return T.value


class KnnIndex:
    """GenerateKDTreeForDWG replacement (src/KNN_GWN.cu:183-212): a GPU index."""

    def __init__(self, points):
        _req_cuda_f32(points, "points", 3)
        self.points = points
        self._h = C.c_void_p()
        capi.check(capi.load().dwg_knn_build(capi.ptr(points), points.shape[0], capi.stream_ptr(),
                                             C.byref(self._h)))

    def query(self, queries, k, out=None):
        """CudaKNNWithKDTreeforDWG replacement (src/KNN_GWN.cu:490-715)."""
        _req_cuda_f32(queries, "queries", 3)
        if out is None:
            out = torch.empty((queries.shape[0], k), dtype=torch.int32, device=queries.device)
        capi.check(capi.load().dwg_knn_query(self._h, capi.ptr(queries), queries.shape[0], int(k), capi.ptr(out),
                                             capi.stream_ptr()))
        return out

    def __del__(self):
        try:
            if self._h.value:
                capi.load().dwg_knn_destroy(self._h)
        except Exception:
            pass


def GenerateKDTreeForDWG(d_points, d_normals=None, points_size=None, bound_upper=None, bound_lower=None):
    return KnnIndex(d_points)


def CudaKNNWithKDTreeforDWG(d_points, numPoints, d_queries, numQueries, bound_upper, bound_lower, d_results, k,
                            index=None):
    ix = index if index is not None else KnnIndex(d_points[:numPoints])
    ix.query(d_queries[:numQueries], k, out=d_results.view(numQueries, k))
    return d_results


def voxel_grid(points, offset, s):
    """igl::voxel_grid(V, offset, s, 1) in closed form -> (res[3], origin[3], spacing)."""
    _req_cuda_f32(points, "points", 3)
    res = np.empty(3, np.int32)
    org = np.empty(3, np.float32)
    h = C.c_float()
    capi.check(capi.load().dwg_voxel_grid(capi.ptr(points), points.shape[0], float(offset), int(s),
                                          capi.stream_ptr(), res.ctypes.data, org.ctypes.data, C.byref(h)))
    return res, org, np.float32(h.value)


def pca_normals(points, knn, view):
    """PCA normals of the --com_As 1 mode (pcl::NormalEstimation with
    setKSearch(10), include/DWGProcess.h:152-200): knn rows hold each point's
    nearest points, self included; normals face ``view`` (3 floats)."""
    _req_cuda_f32(points, "points", 3)
    knn = knn.contiguous()
    v = np.ascontiguousarray(np.asarray(view, np.float32).reshape(3))
    out = torch.empty_like(points)
    capi.check(capi.load().dwg_pca_normals(capi.ptr(points), points.shape[0], capi.ptr(knn), knn.shape[1],
                                           v.ctypes.data, capi.ptr(out), capi.stream_ptr()))
    return out


def point_areas(points, knn, normals):
    """igl::copyleft::cgal::point_areas (include/DWGProcess.h:345-378): the
    area of every point from its knn row (self first, <= 32 columns)."""
    _req_cuda_f32(points, "points", 3)
    _req_cuda_f32(normals, "normals", 3)
    knn = knn.contiguous()
    out = torch.empty(points.shape[0], dtype=torch.float32, device=points.device)
    capi.check(capi.load().dwg_point_areas(capi.ptr(points), points.shape[0], capi.ptr(knn), knn.shape[1],
                                           capi.ptr(normals), capi.ptr(out), capi.stream_ptr()))
    return out


class TurboDWG:
    """The DWG iteration + meshing driver (src/TurboDWG.cu:456-989), as one
    GPU pipeline: ``TurboDWG(points, normals=None, **flags)``, then
    ``TurboScreenedDWGLaunch(total_iters)`` and ``GenerateMesh()``."""

    def __init__(self, points, normals=None, init_model=None, **flags):
        _req_cuda_f32(points, "points", 3)
        if init_model is not None:
            flags["in_normal"] = 4
        self.params = capi.default_params(**flags)
        self.points = points
        self._h = C.c_void_p()
        if init_model is not None:
            capi.check(capi.load().dwg_pipeline_create_learned(capi.ptr(points), points.shape[0],
                                                               C.byref(self.params), init_model.handle,
                                                               capi.stream_ptr(), C.byref(self._h)))
        else:
            capi.check(capi.load().dwg_pipeline_create(capi.ptr(points), capi.ptr(normals), points.shape[0],
                                                       C.byref(self.params), capi.stream_ptr(),
                                                       C.byref(self._h)))

    def TurboScreenedDWGLaunch(self, total_iters=None):
        n = self.params.total_iter if total_iters is None else int(total_iters)
        capi.check(capi.load().dwg_pipeline_iterate(self._h, n))

    def GenerateMesh(self):
        capi.check(capi.load().dwg_pipeline_finalize(self._h))

    def size(self, what):
        v = C.c_longlong()
        capi.check(capi.load().dwg_pipeline_size(self._h, what.encode(), C.byref(v)))
        return v.value

    def get(self, what):
        sizes = {"leaf_pos": (self.size("leaves"), 3), "leaf_nrm": (self.size("leaves"), 3),
                 "point_nrm": (self.size("points"), 3), "iso": (self.size("iterations"),),
                 "field": (self.size("grid"),), "final_field": (self.size("final_grid"),),
                 "final_iso": (1,), "grid_res": (3,), "final_res": (3,), "grid_origin": (4,),
                 "final_origin": (4,)}
        dtypes = {"tri_count": np.int64, "zero_count": np.int32, "terms": np.uint64, "grid_res": np.int32,
                  "final_res": np.int32}
        if what == "tris":
            shape = (self.size("triangles"), 9)
        elif what in ("tri_count", "zero_count", "terms"):
            shape = (self.size("iterations"),)
        else:
            shape = sizes[what]
        a = np.empty(shape, dtypes.get(what, np.float32))
        if a.size:
            capi.check(capi.load().dwg_pipeline_get(self._h, what.encode(), a.ctypes.data))
        return a

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            capi.load().dwg_pipeline_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LearnedNormalInit:
    """The learned initialiser (replaces ``TurboNormalInitialization::
    GaussMapInit``, src/TurboNormalInit.cu:3-44, as the source of initial
    normals): ``LearnedNormalInit(path=None, seed=0)``; ``init_normals(points)``
    returns unit normals, ``features(points)`` the 12 network inputs,
    ``train_step(features, targets, lr)`` one Adam step."""

    FEATURES = 12

    def __init__(self, path=None, seed=0):
        self.handle = C.c_void_p()
        capi.check(capi.load().dwg_mlp_create(int(seed), capi.stream_ptr(), C.byref(self.handle)))
        if path is not None:
            self.load(path)

    @staticmethod
    def param_count():
        return int(capi.load().dwg_mlp_param_count())

    def load(self, path):
        capi.check(capi.load().dwg_mlp_load(self.handle, str(path).encode()))

    def save(self, path):
        capi.check(capi.load().dwg_mlp_save(self.handle, str(path).encode()))

    def get_params(self):
        out = np.empty(self.param_count(), np.float32)
        capi.check(capi.load().dwg_mlp_get_params(self.handle, out.ctypes.data, out.size))
        return out

    def set_params(self, flat):
        flat = np.ascontiguousarray(flat, np.float32)
        capi.check(capi.load().dwg_mlp_set_params(self.handle, flat.ctypes.data, flat.size))

    @staticmethod
    def features(points, out=None):
        import torch
        _req_cuda_f32(points, "points", 3)
        if out is None:
            out = torch.empty((points.shape[0], LearnedNormalInit.FEATURES), dtype=torch.float32,
                              device=points.device)
        capi.check(capi.load().dwg_mlp_features(capi.ptr(points), points.shape[0], capi.ptr(out),
                                                capi.stream_ptr()))
        return out

    def forward(self, features, out=None):
        import torch
        _req_cuda_f32(features, "features", self.FEATURES)
        if out is None:
            out = torch.empty((features.shape[0], 3), dtype=torch.float32, device=features.device)
        capi.check(capi.load().dwg_mlp_forward(self.handle, capi.ptr(features), features.shape[0], capi.ptr(out),
                                               capi.stream_ptr()))
        return out

    def init_normals(self, points, out=None):
        import torch
        _req_cuda_f32(points, "points", 3)
        if out is None:
            out = torch.empty_like(points)
        capi.check(capi.load().dwg_mlp_init_normals(self.handle, capi.ptr(points), points.shape[0], capi.ptr(out),
                                                    capi.stream_ptr()))
        return out

    def train_step(self, features, targets, lr):
        _req_cuda_f32(features, "features", self.FEATURES)
        _req_cuda_f32(targets, "targets", 3)
        loss = C.c_float()
        capi.check(capi.load().dwg_mlp_train_step(self.handle, capi.ptr(features), capi.ptr(targets),
                                                  features.shape[0], float(lr), C.byref(loss), capi.stream_ptr()))
        return loss.value

    def gradients(self, features, targets):
        loss = C.c_float()
        g = np.empty(self.param_count(), np.float32)
        capi.check(capi.load().dwg_mlp_gradients(self.handle, capi.ptr(features), capi.ptr(targets),
                                                 features.shape[0], C.byref(loss), g.ctypes.data, g.size,
                                                 capi.stream_ptr()))
        return loss.value, g

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            capi.load().dwg_mlp_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _DeviceInt64:
    """__cuda_array_interface__ of an int64 device buffer (a torch view, no copy)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<i8", "data": (int(ptr), False),
                                         "version": 2}


def exchange_tensor(t, group=None):
    """Element-wise sum of an int64 tensor over the ranks of ``group``, in
    place: NCCL sums device memory directly, other backends (gloo) a host copy."""
    import torch.distributed as dist
    if t.is_cuda and dist.get_backend(group) == "nccl":
        dist.all_reduce(t, group=group)
        torch.cuda.synchronize()
    elif t.is_cuda:
        h = t.cpu()
        dist.all_reduce(h, group=group)
        t.copy_(h)
        torch.cuda.synchronize()
    else:
        dist.all_reduce(t, group=group)
    return t


def torch_exchange(group=None):
    """The exchange function of a sharded pipeline over torch.distributed
    (keep the returned object alive while the pipeline runs)."""
    def fn(user, buf, count, stream):
        try:
            torch.cuda.synchronize()
            exchange_tensor(torch.as_tensor(_DeviceInt64(buf, count), device="cuda"), group)
            return 0
        except Exception as e:  # reported as a failed exchange by the library
            print(f"dwg_b200 exchange failed: {e}", flush=True)
            return 1
    return capi.EXCHANGE_FN(fn)


def slab_range(samples, rank, world):
    """z-samples (first, count) of rank ``rank``'s slab of a grid with ``samples`` z-samples."""
    z0, nz = C.c_int(), C.c_int()
    capi.check(capi.load().dwg_slab_range(int(samples), int(rank), int(world), C.byref(z0), C.byref(nz)))
    return z0.value, nz.value


def reconstruct_sharded(points, rank, world, exchange, normals=None, **flags):
    """Rank ``rank`` of a z-slab sharded reconstruction of one cloud (one
    process per GPU, ``exchange`` from :func:`torch_exchange`): leaf normals,
    iso values and triangle counts are those of the whole run, ``tris`` and
    ``final_field`` this rank's slab (``slab``: first z-sample and count of
    the iteration grid, then of the final grid)."""
    _req_cuda_f32(points, "points", 3)
    prm = capi.default_params(**flags)
    h = C.c_void_p()
    lib = capi.load()
    capi.check(lib.dwg_pipeline_create_sharded(capi.ptr(points), capi.ptr(normals), points.shape[0], C.byref(prm),
                                               int(rank), int(world), exchange, None, capi.stream_ptr(),
                                               C.byref(h)))
    try:
        capi.check(lib.dwg_pipeline_iterate(h, prm.total_iter))
        capi.check(lib.dwg_pipeline_finalize(h))
        out = {}

        def get(what, shape, dtype):
            a = np.empty(shape, dtype)
            if a.size:
                capi.check(lib.dwg_pipeline_get(h, what.encode(), a.ctypes.data))
            return a

        def size(what):
            v = C.c_longlong()
            capi.check(lib.dwg_pipeline_size(h, what.encode(), C.byref(v)))
            return v.value

        L, it = size("leaves"), size("iterations")
        out["leaf_pos"] = get("leaf_pos", (L, 3), np.float32)
        out["leaf_nrm"] = get("leaf_nrm", (L, 3), np.float32)
        out["iso"] = get("iso", (it,), np.float32)
        out["tri_count"] = get("tri_count", (it,), np.int64)
        out["zero_count"] = get("zero_count", (it,), np.int32)
        out["tris"] = get("tris", (size("triangles"), 9), np.float32)
        out["final_iso"] = get("final_iso", (1,), np.float32)
        out["final_res"] = get("final_res", (3,), np.int32)
        out["final_field"] = get("final_field", (size("final_grid"),), np.float32)
        out["slab"] = get("slab", (4,), np.int32)
        if not prm.use_leaves_generate:
            out["point_nrm"] = get("point_nrm", (size("points"), 3), np.float32)
        return out
    finally:
        lib.dwg_pipeline_destroy(h)


def reconstruct(points, normals=None, init_model=None, **flags):
    """Full reconstruction on the GPU; returns a dict of host arrays."""
    d = TurboDWG(points, normals, init_model=init_model, **flags)
    d.TurboScreenedDWGLaunch()
    d.GenerateMesh()
    out = {k: d.get(k) for k in ("leaf_pos", "leaf_nrm", "iso", "tri_count", "zero_count", "terms", "tris",
                                 "final_iso", "final_res")}
    if not d.params.use_leaves_generate:
        out["point_nrm"] = d.get("point_nrm")
    d.close()
    return out
