"""dwg_marching_cubes_noalloc: marching cubes for callers that cannot call
cudaMalloc while they mesh -- a real-time loop that must not allocate after
start-up (cudaMalloc and cudaFree can wait for the whole device), or an
application whose device memory is a fixed budget from its own pool.

Its output must equal the allocating entry point's, bit for bit, on calls in
a row that share its static scratch array; it must leave the device's free
memory unchanged; and it must keep the allocating path's behaviour on the
positions path and on overflow.  This file is collected last on purpose: a
run that stops at its first failure has run every other test by then."""
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
    return f.astype(np.float32), G


def outputs(cap):
    return (torch.empty((cap, 9), dtype=torch.float32, device="cuda"),
            torch.empty((cap, 3), dtype=torch.float32, device="cuda"),
            torch.empty((cap, 3), dtype=torch.float32, device="cuda"))


def call(lib, fn, f_d, res, org, h, iso, bufs, cap, pos_d=None):
    tris, cen, nrm = bufs
    T = C.c_longlong(-1)
    o = None if pos_d is not None else org.ctypes.data
    if fn == "alloc":
        rc = lib.dwg_marching_cubes(capi.ptr(f_d), res.ctypes.data, capi.ptr(pos_d), o, float(h), float(iso),
                                    capi.ptr(tris), capi.ptr(cen), capi.ptr(nrm), cap, None, C.byref(T), None)
    else:
        rc = lib.dwg_marching_cubes_noalloc(capi.ptr(f_d), res.ctypes.data, capi.ptr(pos_d), o, float(h),
                                            float(iso), capi.ptr(tris), capi.ptr(cen), capi.ptr(nrm), cap,
                                            C.byref(T), None)
    return rc, T.value


def host(bufs, t):
    return [b[:t].cpu().numpy() for b in bufs]


CASES = [(np.array([61, 53, 47], np.int32), np.float32(0.35), 11),
         (np.array([40, 72, 33], np.int32), np.float32(0.52), 12)]
ORG = np.array([-0.6, -0.55, -0.5], np.float32)
H = np.float32(0.019)


def test_noalloc_matches_allocating_entry_point_twice():
    build.build()
    lib = capi.load()
    for res, iso, seed in CASES:  # two calls in a row share the scratch array
        f, _ = blob_field(res, ORG, H, seed)
        f_d = torch.from_numpy(f).cuda()
        cap = int(np.prod(res.astype(np.int64))) // 2
        A, B = outputs(cap), outputs(cap)
        rc, ta = call(lib, "alloc", f_d, res, ORG, H, iso, A, cap)
        capi.check(rc)
        rc, tb = call(lib, "noalloc", f_d, res, ORG, H, iso, B, cap)
        capi.check(rc)
        torch.cuda.synchronize()
        assert ta > 1000 and ta == tb
        for x, y in zip(host(A, ta), host(B, tb)):
            assert np.array_equal(x, y)


def test_noalloc_allocates_no_device_memory():
    lib = capi.load()
    res, iso, seed = CASES[0]
    f, _ = blob_field(res, ORG, H, seed)
    f_d = torch.from_numpy(f).cuda()
    cap = int(np.prod(res.astype(np.int64))) // 2
    bufs = outputs(cap)
    capi.check(call(lib, "noalloc", f_d, res, ORG, H, iso, bufs, cap)[0])  # first call: address, tables
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        capi.check(call(lib, "noalloc", f_d, res, ORG, H, iso, bufs, cap)[0])
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_positions_path_matches_allocating_entry_point():
    lib = capi.load()
    res, iso, seed = CASES[1]
    f, G = blob_field(res, ORG, H, seed)
    f_d = torch.from_numpy(f).cuda()
    pos_d = torch.from_numpy(G).cuda()  # per-sample positions instead of origin + index * spacing
    cap = int(np.prod(res.astype(np.int64))) // 2
    A, B = outputs(cap), outputs(cap)
    rc, ta = call(lib, "alloc", f_d, res, ORG, H, iso, A, cap, pos_d)
    capi.check(rc)
    rc, tb = call(lib, "noalloc", f_d, res, ORG, H, iso, B, cap, pos_d)
    capi.check(rc)
    torch.cuda.synchronize()
    assert ta > 1000 and ta == tb
    for x, y in zip(host(A, ta), host(B, tb)):
        assert np.array_equal(x, y)


def test_noalloc_overflow_reports_the_count_and_keeps_the_first_triangles():
    lib = capi.load()
    res, iso, seed = CASES[0]
    f, _ = blob_field(res, ORG, H, seed)
    f_d = torch.from_numpy(f).cuda()
    full = int(np.prod(res.astype(np.int64))) // 2
    A = outputs(full)
    rc, T = call(lib, "alloc", f_d, res, ORG, H, iso, A, full)
    capi.check(rc)
    cap = T // 3
    B = outputs(cap)
    rc, tb = call(lib, "noalloc", f_d, res, ORG, H, iso, B, cap)
    torch.cuda.synchronize()
    assert rc == capi.DWG_ERR_OVERFLOW and tb == T
    assert b"exceed capacity" in lib.dwg_last_error()
    for x, y in zip(host(A, cap), host(B, cap)):
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
