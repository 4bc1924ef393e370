"""Batched reconstruction (many clouds, one graph per iteration, one
persistent launch for all grid sums) against the same clouds reconstructed
one by one, and the grid brick shapes against each other."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import capi, datasets as D, turbo  # noqa: E402

pytestmark = pytest.mark.gpu


def clouds():
    out = []
    for kind, n, seed in (("sphere", 4000, 1), ("torus", 15000, 2), ("sq", 9000, 3)):
        if kind == "sphere":
            P, _ = D.sphere(n, noise=0.003, seed=seed)
        elif kind == "torus":
            P, _ = D.torus(n, seed=seed)
        else:
            P, _ = D.superquadric_union(n, k=3, outlier_frac=0.0, noise=0.002, seed=seed)
        Pn, _, _ = D.normalize(P)
        out.append(np.ascontiguousarray(Pn, np.float32))
    return out


def results(lib, h):
    def size(what):
        v = C.c_longlong()
        capi.check(lib.dwg_pipeline_size(h, what.encode(), C.byref(v)))
        return v.value

    def get(what, shape, dt):
        a = np.empty(shape, dt)
        capi.check(lib.dwg_pipeline_get(h, what.encode(), a.ctypes.data))
        return a

    L, it, T = size("leaves"), size("iterations"), size("triangles")
    return {"leaf_nrm": get("leaf_nrm", (L, 3), np.float32), "iso": get("iso", (it,), np.float32),
            "tri_count": get("tri_count", (it,), np.int64), "terms": get("terms", (it,), np.uint64),
            "field": get("field", (size("grid"),), np.float32), "tris": get("tris", (T, 9), np.float32)}


@pytest.mark.parametrize("tile,lists", [(0, 2), (3, 2), (0, 0), (3, 0)])
def test_batch_equals_single_clouds(dwg_lib, tile, lists):
    # the batch's persistent launch sums every cloud's grid; with lists 2 the
    # sums at the leaves replay each cloud's lists and kept weights
    lib = dwg_lib
    P = clouds()
    grids = [48, 64, 56]
    iters = 6
    dev = [torch.from_numpy(p).cuda() for p in P]
    prms = [capi.default_params(grid_reso=g, final_reso=g, total_iter=iters, tile=tile, grid_lists=lists)
            for g in grids]
    # one by one
    single = []
    for d, prm in zip(dev, prms):
        h = C.c_void_p()
        capi.check(lib.dwg_pipeline_create(capi.ptr(d), None, d.shape[0], C.byref(prm), None, C.byref(h)))
        try:
            capi.check(lib.dwg_pipeline_iterate(h, iters))
            capi.check(lib.dwg_pipeline_finalize(h))
            single.append(results(lib, h))
        finally:
            lib.dwg_pipeline_destroy(h)
    # batched
    ptrs = (C.c_void_p * len(dev))(*[capi.ptr(d) for d in dev])
    counts = (C.c_int * len(dev))(*[d.shape[0] for d in dev])
    parr = (capi.Params * len(prms))(*prms)
    b = C.c_void_p()
    capi.check(lib.dwg_batch_create(ptrs, counts, len(dev), parr, None, C.byref(b)))
    try:
        capi.check(lib.dwg_batch_iterate(b, 2))
        capi.check(lib.dwg_batch_iterate(b, iters - 2))  # graph replays continue the count
        capi.check(lib.dwg_batch_finalize(b))
        for i, ref in enumerate(single):
            h = C.c_void_p()
            capi.check(lib.dwg_batch_cloud(b, i, C.byref(h)))
            got = results(lib, h)
            for k in ref:
                assert np.array_equal(got[k], ref[k]), (i, k)
    finally:
        lib.dwg_batch_destroy(b)


def test_batch_rejects_mixed_tiles(dwg_lib):
    lib = dwg_lib
    P = clouds()[:2]
    dev = [torch.from_numpy(p).cuda() for p in P]
    prms = [capi.default_params(grid_reso=32, tile=0), capi.default_params(grid_reso=32, tile=1)]
    ptrs = (C.c_void_p * 2)(*[capi.ptr(d) for d in dev])
    counts = (C.c_int * 2)(*[d.shape[0] for d in dev])
    parr = (capi.Params * 2)(*prms)
    b = C.c_void_p()
    assert lib.dwg_batch_create(ptrs, counts, 2, parr, None, C.byref(b)) == capi.DWG_ERR_INVALID


def test_grid_tiles_are_bit_identical(dwg_lib):
    # a lane's terms come in the same order whatever brick it shares a warp with
    P = clouds()[1]
    Pd = torch.from_numpy(P).cuda()
    N = turbo.TurboNormalInitialization().GaussMapInit(Pd, torch.empty_like(Pd))
    A = torch.full((len(P),), 2e-6, device="cuda")
    tree = turbo.TurboLibiGWN(Pd, max_depth=10, areas=A)
    tree.UpdateMassNormals(N, A)
    res = np.array([45, 38, 21], np.int32)
    org = np.array([-0.55, -0.5, -0.2], np.float32)
    outs, terms = [], []
    for tile in range(4):
        out = torch.empty(int(np.prod(res)), device="cuda")
        t = torch.zeros(1, dtype=torch.int64, device="cuda")
        tree.grid(res, org, 0.025, sigma=10.0, precision=1, out=out, tile=tile, terms=t)
        outs.append(out.cpu().numpy())
        terms.append(int(t.item()))
    for k in range(1, 4):
        assert np.array_equal(outs[k], outs[0]), k
        assert terms[k] == terms[0]


def test_autotune_picks_a_setting_within_tolerance(dwg_lib):
    lib = dwg_lib
    P = clouds()[1]
    Pd = torch.from_numpy(P).cuda()
    prm = capi.default_params(grid_reso=64, final_reso=64)
    r = capi.TuneResult()
    # default criterion: no less accurate than the reference's beta 2.3
    capi.check(lib.dwg_autotune(capi.ptr(Pd), len(P), C.byref(prm), 0.0, 2048, 2, None, C.byref(r)))
    assert np.isclose([1.5, 1.8, 2.0, 2.3, 2.6, 3.0, 3.5, 4.5], r.beta, rtol=1e-6).any()
    assert 0 <= r.tile <= 3
    assert 0.0 <= r.rms_err <= r.ref_rms_err * 1.00001 and r.max_err >= r.rms_err
    assert r.grid_ms > 0 and r.ref_ms > 0 and r.field_rms > 0
    # an explicit absolute tolerance well above the reference's error admits beta 2.3
    capi.check(lib.dwg_autotune(capi.ptr(Pd), len(P), C.byref(prm), float(r.ref_rms_err) * 10, 2048, 2, None,
                                C.byref(r)))
    assert r.rms_err <= r.ref_rms_err * 10
    # a tolerance no opening ratio reaches is an error, not a silent choice
    assert lib.dwg_autotune(capi.ptr(Pd), len(P), C.byref(prm), 1e-12, 2048, 2, None,
                            C.byref(r)) == capi.DWG_ERR_INVALID
