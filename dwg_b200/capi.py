"""ctypes binding of ``libdwg_b200.so`` (the C ABI declared in include/dwg_b200.h).

Arguments named ``*_dev`` take torch CUDA tensors (or raw device addresses);
the library never falls back to the CPU: if the shared library is missing or
fails to load, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdwg_b200.so")

DWG_OK = 0
DWG_ERR_INVALID = -1
DWG_ERR_CUDA = -2
DWG_ERR_OVERFLOW = -3
DWG_ERR_NOMEM = -4
DWG_ERR_DEVICE = -5


class DwgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dwg_b200 error {code}: {msg}")
        self.code = code


class GwnParams(C.Structure):
    _fields_ = [("beta", C.c_float), ("sigma", C.c_float), ("screen", C.c_float),
                ("screened", C.c_int), ("use_radii", C.c_int), ("precision", C.c_int), ("tile", C.c_int),
                ("order", C.c_int), ("lists", C.c_int)]


class Params(C.Structure):
    _fields_ = [
        ("in_normal", C.c_int), ("grid_reso", C.c_int), ("final_reso", C.c_int),
        ("kw", C.c_int), ("final_kw", C.c_int), ("normal_kw", C.c_int), ("max_depth", C.c_int),
        ("lambda_", C.c_float), ("min_num", C.c_int), ("use_radii", C.c_int),
        ("offset_1", C.c_float), ("offset_2", C.c_float), ("use_leaves_generate", C.c_int),
        ("total_iter", C.c_int), ("beta", C.c_float), ("area", C.c_float), ("screen", C.c_float),
        ("knn_tri", C.c_int), ("knn_zero", C.c_int), ("precision", C.c_int), ("use_graph", C.c_int),
        ("tile", C.c_int), ("as_thres", C.c_float), ("com_as", C.c_int), ("grid_lists", C.c_int),
    ]


class TuneResult(C.Structure):
    _fields_ = [("beta", C.c_float), ("tile", C.c_int), ("rms_err", C.c_float), ("max_err", C.c_float),
                ("grid_ms", C.c_float), ("ref_ms", C.c_float), ("ref_rms_err", C.c_float), ("field_rms", C.c_float)]


# name -> (restype, argtypes)
_vp = C.c_void_p
_i = C.c_int
_ll = C.c_longlong
_f = C.c_float
_SIGS = {
    "dwg_last_error": (C.c_char_p, []),
    "dwg_version": (C.c_char_p, []),
    "dwg_gauss_map_init": (_i, [_vp, _i, _vp, _vp]),
    "dwg_octree_build": (_i, [_vp, _i, _i, _vp, _vp, C.POINTER(_vp)]),
    "dwg_octree_destroy": (_i, [_vp]),
    "dwg_octree_num_nodes": (_i, [_vp, C.POINTER(_i)]),
    "dwg_octree_update_normals": (_i, [_vp, _vp, _vp, _vp]),
    "dwg_octree_update_info": (_i, [_vp, _vp, _vp, _vp]),
    "dwg_octree_status": (_i, [_vp, C.POINTER(C.c_uint)]),
    "dwg_octree_list_size": (_i, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
    "dwg_octree_export": (_i, [_vp] * 9),
    "dwg_octree_expansion": (_i, [_vp, _vp, _vp]),
    "dwg_gwn_points": (_i, [_vp, _vp, _vp, _vp, _vp, _ll, C.POINTER(GwnParams), _vp, _vp, _vp]),
    "dwg_gwn_points_counted": (_i, [_vp, _vp, _vp, _vp, _vp, _ll, C.POINTER(GwnParams), _vp, _vp, _vp]),
    "dwg_gwn_grid": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _f, C.POINTER(GwnParams), _vp, _vp, _vp]),
    "dwg_gwn_points_grad": (_i, [_vp, _vp, _vp, _vp, _vp, _ll, C.POINTER(GwnParams), _vp, _vp, _vp]),
    "dwg_gwn_grid_grad": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _f, C.POINTER(GwnParams), _vp, _vp, _vp]),
    "dwg_gwn_points_fp64": (_i, [_vp, _vp, _vp, _vp, _vp, _ll, C.POINTER(GwnParams), _vp, _vp, _vp]),
    "dwg_gwn_grid_fp64": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _f, C.POINTER(GwnParams), _vp, _vp, _vp]),
    "dwg_voxel_grid": (_i, [_vp, _i, _f, _i, _vp, _vp, _vp, _vp]),
    "dwg_marching_cubes": (_i, [_vp, _vp, _vp, _vp, _f, _f, _vp, _vp, _vp, _ll, _vp, _vp, _vp]),
    "dwg_mc_tables": (_i, [_vp, _vp]),
    "dwg_marching_cubes_noalloc": (_i, [_vp, _vp, _vp, _vp, _f, _f, _vp, _vp, _vp, _ll, _vp, _vp]),
    "dwg_knn_build": (_i, [_vp, _i, _vp, C.POINTER(_vp)]),
    "dwg_knn_destroy": (_i, [_vp]),
    "dwg_knn_query": (_i, [_vp, _vp, _ll, _i, _vp, _vp]),
    "dwg_knn": (_i, [_vp, _i, _vp, _ll, _i, _vp, _vp]),
    "dwg_diffuse_normals": (_i, [_vp, _vp, _ll, _i, _i, _vp, _vp, _vp, _vp]),
    "dwg_zero_repair": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp]),
    "dwg_load_normals": (_i, [_vp, _i, _ll, _vp, _vp, _vp]),
    "dwg_radii": (_i, [_vp, _i, _vp, _i, _vp, _vp]),
    "dwg_pca_normals": (_i, [_vp, _i, _vp, _i, _vp, _vp, _vp]),
    "dwg_point_areas": (_i, [_vp, _i, _vp, _i, _vp, _vp, _vp]),
    "dwg_params_default": (None, [C.POINTER(Params)]),
    "dwg_pipeline_create": (_i, [_vp, _vp, _i, C.POINTER(Params), _vp, C.POINTER(_vp)]),
    "dwg_pipeline_destroy": (_i, [_vp]),
    "dwg_pipeline_iterate": (_i, [_vp, _i]),
    "dwg_pipeline_finalize": (_i, [_vp]),
    "dwg_pipeline_size": (_i, [_vp, C.c_char_p, C.POINTER(_ll)]),
    "dwg_pipeline_get": (_i, [_vp, C.c_char_p, _vp]),
    "dwg_pipeline_device_ptr": (_i, [_vp, C.c_char_p, C.POINTER(_vp)]),
    "dwg_pipeline_create_sharded": (_i, [_vp, _vp, _i, C.POINTER(Params), _i, _i, _vp, _vp, _vp, C.POINTER(_vp)]),
    "dwg_slab_range": (_i, [_i, _i, _i, C.POINTER(_i), C.POINTER(_i)]),
    "dwg_autotune": (_i, [_vp, _i, C.POINTER(Params), _f, _i, _i, _vp, C.POINTER(TuneResult)]),
    "dwg_batch_create": (_i, [_vp, _vp, _i, _vp, _vp, C.POINTER(_vp)]),
    "dwg_batch_destroy": (_i, [_vp]),
    "dwg_batch_iterate": (_i, [_vp, _i]),
    "dwg_batch_finalize": (_i, [_vp]),
    "dwg_batch_cloud": (_i, [_vp, _i, C.POINTER(_vp)]),
    "dwg_mlp_param_count": (_ll, []),
    "dwg_mlp_create": (_i, [C.c_ulonglong, _vp, C.POINTER(_vp)]),
    "dwg_mlp_destroy": (_i, [_vp]),
    "dwg_mlp_set_params": (_i, [_vp, _vp, _ll]),
    "dwg_mlp_get_params": (_i, [_vp, _vp, _ll]),
    "dwg_mlp_load": (_i, [_vp, C.c_char_p]),
    "dwg_mlp_save": (_i, [_vp, C.c_char_p]),
    "dwg_mlp_features": (_i, [_vp, _i, _vp, _vp]),
    "dwg_mlp_forward": (_i, [_vp, _vp, _ll, _vp, _vp]),
    "dwg_mlp_gradients": (_i, [_vp, _vp, _vp, _ll, C.POINTER(_f), _vp, _ll, _vp]),
    "dwg_mlp_train_step": (_i, [_vp, _vp, _vp, _ll, _f, C.POINTER(_f), _vp]),
    "dwg_mlp_init_normals": (_i, [_vp, _vp, _i, _vp, _vp]),
    "dwg_pipeline_create_learned": (_i, [_vp, _i, C.POINTER(Params), _vp, _vp, C.POINTER(_vp)]),
    "dwg_reconstruct_host": (_i, [_vp, _vp, _i, C.POINTER(Params), _vp, _vp, _ll, C.POINTER(_ll), _vp]),
    "dwg_read_xyz": (_i, [C.c_char_p, _i, C.POINTER(C.POINTER(_f)), C.POINTER(C.POINTER(_f)), C.POINTER(_i)]),
    "dwg_free_host": (None, [_vp]),
    "dwg_write_stl": (_i, [C.c_char_p, _vp, _ll]),
    "dwg_write_stl_device": (_i, [C.c_char_p, _vp, _ll, _vp]),
    "dwg_write_xyz": (_i, [C.c_char_p, _vp, _vp, _i]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the shared library; raise if it is absent (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m dwg_b200.build` "
            "(dwg_b200 has no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return sorted(_SIGS)


def ptr(x):
    """Device (or host) address of a torch tensor / numpy array / int / None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(f"cannot take the address of {type(x)}")


def check(code):
    if code != DWG_OK:
        msg = load().dwg_last_error()
        raise DwgError(code, msg.decode() if msg else "")
    return code


def stream_ptr(stream=None):
    if stream is None:
        try:
            import torch
            return torch.cuda.current_stream().cuda_stream
        except Exception:  # pragma: no cover
            return None
    if hasattr(stream, "cuda_stream"):
        return stream.cuda_stream
    return stream


def default_params(**kw) -> Params:
    p = Params()
    load().dwg_params_default(C.byref(p))
    for k, v in kw.items():
        if k == "lambda":
            k = "lambda_"
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


# element-wise int64 sum over ranks: (user, buf_dev, count, stream) -> 0 on success
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p)


def gwn_params(beta=2.3, sigma=10.0, screen=0.0015, screened=True, use_radii=False, precision=1,
               tile=0, order=0, lists=0) -> GwnParams:
    return GwnParams(beta, sigma, screen, int(screened), int(use_radii), int(precision), int(tile), int(order),
                     int(lists))
