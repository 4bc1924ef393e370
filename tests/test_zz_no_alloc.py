"""dwg_marching_cubes_noalloc: marching cubes for callers that cannot allocate
device memory while they mesh (graph capture in global mode, real-time loops,
hosts that own all device memory).  Its output must equal the allocating
entry point's, bit for bit, on consecutive calls that share its static
scratch array.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dwg_b200 import build, capi  # noqa: E402

pytestmark = pytest.mark.gpu


def blob_field(res, org, h, seed, n_blobs=6):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(res[2]), np.arange(res[1]), np.arange(res[0]), indexing="ij")
    G = np.stack([org[0] + x * h, org[1] + y * h, org[2] + z * h], -1).reshape(-1, 3).astype(np.float32)
    f = np.zeros(len(G))
    for _ in range(n_blobs):
        c = rng.uniform(-0.4, 0.4, 3)
        f += np.exp(-((G - c) ** 2).sum(1) / 0.03)
    return f.astype(np.float32)


def run(lib, fn, f_d, res, org, h, iso, cap):
    tris = torch.empty((cap, 9), dtype=torch.float32, device="cuda")
    cen = torch.empty((cap, 3), dtype=torch.float32, device="cuda")
    nrm = torch.empty((cap, 3), dtype=torch.float32, device="cuda")
    T = C.c_longlong(-1)
    if fn == "alloc":
        rc = lib.dwg_marching_cubes(capi.ptr(f_d), res.ctypes.data, None, org.ctypes.data, float(h), float(iso),
                                    capi.ptr(tris), capi.ptr(cen), capi.ptr(nrm), cap, None, C.byref(T), None)
    else:
        rc = lib.dwg_marching_cubes_noalloc(capi.ptr(f_d), res.ctypes.data, None, org.ctypes.data, float(h),
                                            float(iso), capi.ptr(tris), capi.ptr(cen), capi.ptr(nrm), cap,
                                            C.byref(T), None)
    capi.check(rc)
    torch.cuda.synchronize()
    t = T.value
    return t, tris[:t].cpu().numpy(), cen[:t].cpu().numpy(), nrm[:t].cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    build.build()
    lib = capi.load()
    cases = [(np.array([61, 53, 47], np.int32), np.float32(0.35), 11),
             (np.array([40, 72, 33], np.int32), np.float32(0.52), 12)]
    for res, iso, seed in cases:  # two calls in a row share the scratch array
        org = np.array([-0.6, -0.55, -0.5], np.float32)
        h = np.float32(0.019)
        f_d = torch.from_numpy(blob_field(res, org, h, seed)).cuda()
        cap = int(np.prod(res.astype(np.int64))) // 2
        a = run(lib, "alloc", f_d, res, org, h, iso, cap)
        b = run(lib, "noalloc", f_d, res, org, h, iso, cap)
        assert a[0] > 1000 and a[0] == b[0]
        for x, y in zip(a[1:], b[1:]):
            assert np.array_equal(x, y)


def test_noalloc_rejects_grids_beyond_its_limit():
    lib = capi.load()
    dummy = torch.zeros(4, dtype=torch.float32, device="cuda")
    res = np.array([1024, 1024, 256], np.int32)  # 267M cells > 134M
    org = np.zeros(3, np.float32)
    T = C.c_longlong(-1)
    rc = lib.dwg_marching_cubes_noalloc(capi.ptr(dummy), res.ctypes.data, None, org.ctypes.data, 0.01, 0.0, None,
                                        None, None, 0, C.byref(T), None)
    assert rc == capi.DWG_ERR_INVALID
    assert b"allocation-free limit" in lib.dwg_last_error()
