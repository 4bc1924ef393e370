"""ctypes front end of ``oracle/_ref/libref_dwg.so``: the reference's own GPU
code (src/TurboDWG.cu, src/TurboLibiGWN.cu, src/TurboMC.cu,
src/TurboNormalInit.cu, src/KNN_GWN.cu of DWGTech/DWG), compiled unchanged by
``oracle/ref_dwg.mk``.

TEST INFRASTRUCTURE ONLY: the GPU tests compare the product with it.  The
reference's CPU preparation (include/DWGProcess.h: libigl's octree, the FP64
moment precompute, the voxel grid) needs Eigen, which is absent; it is
supplied here from the oracle's restatement of the same functions
(``oracle/dwg_oracle.c``), while everything the reference runs on the GPU --
the kd-tree order, the Gauss-map start, the DWG iterations and the final pass
-- is the reference's own code.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import struct
import tempfile

import numpy as np

from . import oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(_HERE, "_ref", "libref_dwg.so")
_lib = None


def available() -> bool:
    return os.path.exists(PATH)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    L = C.CDLL(PATH)
    vp = C.c_void_p
    L.refdwg_kd_sort.restype = C.c_int
    L.refdwg_kd_sort.argtypes = [vp, C.c_int, vp, vp, vp]
    L.refgwn_create.restype = vp
    L.refgwn_create.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]
    L.refgwn_free.argtypes = [vp]
    L.refgwn_eval.restype = C.c_int
    L.refgwn_eval.argtypes = [vp, vp, vp, vp, C.c_int, vp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, vp]
    L.refmc_run.restype = C.c_longlong
    L.refmc_run.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_float, vp, vp, C.c_longlong, C.c_char_p]
    L.refdwg_run.restype = C.c_int
    L.refdwg_run.argtypes = ([C.c_int, vp, vp, vp, vp, C.c_int, vp, vp, vp,
                              C.c_int, vp, vp, vp, vp, vp, vp,
                              C.c_float, C.c_int, C.c_int, C.c_float, C.c_int,
                              C.c_int, vp, vp, C.c_int, vp, vp, vp,
                              C.c_int, vp, vp, vp, vp, vp, vp,
                              C.c_int, C.c_int, C.c_char_p, C.c_char_p, vp, vp])
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def kd_sort(P):
    """GenerateKDTreeForGWN (src/KNN_GWN.cu:68-140): the points in the
    reference's kd-tree order, perm (sorted -> input index) and the bounds
    (lower xyz, upper xyz)."""
    P = _c(P, np.float32).reshape(-1, 3)
    out = np.empty_like(P)
    perm = np.empty(len(P), np.int32)
    bounds = np.empty(6, np.float32)
    rc = lib().refdwg_kd_sort(_p(P), len(P), _p(out), _p(perm), _p(bounds))
    if rc != 0:
        raise RuntimeError(f"refdwg_kd_sort failed ({rc})")
    return out, perm, bounds


class IglTree:
    """An igl::octreeDWG tree of ``P`` (the oracle's restatement) in the flat
    form the reference's TurboLibiGWN::PreLibiGWN takes, with FP64 order-0
    moments (fast_winding_number.cpp:9-120) for normals N and areas A."""

    def __init__(self, P, max_depth, N=None, A=None):
        self.P = _c(P, np.float32).reshape(-1, 3)
        self.t = O.Octree(self.P.astype(np.float64), max_depth)
        self.ch = _c(self.t.children, np.int32)
        off, flat = self.t.lists()
        self.off = _c(off, np.int64)
        self.flat = _c(flat if len(flat) else np.zeros(1, np.int32), np.int32)
        n = len(self.P)
        N = np.tile(np.float32([0, 0, 1]), (n, 1)) if N is None else N
        A = np.full(n, 2e-6, np.float32) if A is None else A
        CM, R, EC = self.t.moments(self.P, N, A)
        self.cm, self.r, self.ec = _c(CM, np.float64), _c(R, np.float64), _c(EC, np.float64)

    @property
    def M(self):
        return self.t.num_nodes

    def args(self):
        return [self.M, _p(self.ch), _p(self.off), _p(self.flat), _p(self.cm), _p(self.r), _p(self.ec)]


class RefGWN:
    """TurboLibiGWN (src/TurboLibiGWN.cu) on an igl octree of the points P."""

    def __init__(self, P, max_depth, A=None):
        self.tree = IglTree(P, max_depth, A=A)
        self.n = len(self.tree.P)
        self._h = lib().refgwn_create(_p(self.tree.P), self.n, *self.tree.args())

    def eval(self, N, A, Q, beta=2.3, sigma=0.0, screened=True, radii=None, info=False):
        """UpdateMassNormals (or UpdateGWNInfo) then the screened/plain sums at Q."""
        N = _c(N, np.float32).reshape(-1, 3)
        A = _c(A, np.float32)
        R = _c(radii if radii is not None else np.zeros(self.n), np.float32)
        Q = _c(Q, np.float32).reshape(-1, 3)
        out = np.empty(len(Q), np.float32)
        rc = lib().refgwn_eval(self._h, _p(N), _p(A), _p(R), int(info), _p(Q), len(Q), int(screened),
                               float(beta), float(sigma), int(radii is not None), _p(out))
        if rc != 0:
            raise RuntimeError(f"refgwn_eval failed ({rc})")
        return out

    def close(self):
        if self._h:
            lib().refgwn_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def marching_cubes(field, positions, res, iso):
    """TurboMC::TurboMarchingCubes (src/TurboMC.cu:572-638): (triangles T x 9,
    centroids, normals), all in the reference's atomicAdd order (the
    triangles from the binary STL the reference writes)."""
    res = [int(r) for r in res]
    G = res[0] * res[1] * res[2]
    cap = max(G // 2, 1000000)
    cen = np.empty((cap, 3), np.float32)
    nrm = np.empty((cap, 3), np.float32)
    wd = tempfile.mkdtemp(prefix="refmc_")
    base = os.path.join(wd, "mc")
    try:
        T = lib().refmc_run(_p(_c(field, np.float32)), _p(_c(positions, np.float32)), res[0], res[1], res[2],
                            float(iso), _p(cen), _p(nrm), cap, base.encode())
        if T < 0:
            raise RuntimeError("refmc_run failed")
        tris = read_stl(base + ".stl")
    finally:
        if os.path.exists(base + ".stl"):
            os.remove(base + ".stl")
        os.rmdir(wd)
    return tris, cen[:T].copy(), nrm[:T].copy()


def read_stl(path):
    with open(path, "rb") as f:
        f.read(80)
        (n,) = struct.unpack("<I", f.read(4))
        rec = np.frombuffer(f.read(50 * n), dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]))
    return rec["v"].reshape(n, 9).copy()


def bfs_leaves(tree, min_num=0):
    """GetOctreeLeaves (include/DWGProcess.h:383-428): the cell centres of the
    leaves holding more than min_num points, breadth-first."""
    ch, cnt, cen = tree.children, tree.counts, tree.centers
    out, queue, h = [], [0], 0
    while h < len(queue):
        i = queue[h]
        h += 1
        if ch[i, 0] == -1:
            if cnt[i] > min_num:
                out.append(i)
            continue
        queue.extend(int(c) for c in ch[i] if c != -1 and cnt[c] > 0)
    return cen[np.array(out, np.int64)].astype(np.float32)


def reconstruct(P, workdir=None, **kw):
    """The reference's DWG run on the normalised points P (N x 3 float32), with
    the CLI defaults of ``oracle.DEFAULT_PARAMS`` overridden by ``kw``
    (in_normal 3, use_leaves_generate 0, com_As 0 only).  Follows
    include/DWGProcess.h:99-227 (kd order of the points, octree on them) and
    :474-747 (leaves, kd order of the leaves, octree on them, radii, voxel
    grids, TurboDWG, final pass on the points).  Returns host arrays: the
    points in kd order and their input indices, leaves (kd order) and their
    normals after the iterations, the per-iteration mean winding number as
    printed (before halving), triangle and zero counts, the final point
    normals and triangles, and the device seconds of the two phases."""
    prm = dict(O.DEFAULT_PARAMS)
    prm.update(kw)
    assert prm["in_normal"] == 3 and prm["use_leaves_generate"] == 0 and prm["com_as"] == 0
    P = _c(P, np.float32).reshape(-1, 3)
    Pk, perm_p, pbounds = kd_sort(P)
    t1 = IglTree(Pk, prm["max_depth"])
    leaves = bfs_leaves(t1.t, prm["min_num"])
    Lk, _, lbounds = kd_sort(leaves)
    L = len(Lk)
    An = np.full(L, prm["area"], np.float32)
    t2 = IglTree(Lk, prm["max_depth"], A=An)
    # GetRadiiandAs (include/DWGProcess.h:283-381): the radii only enter the
    # sums with use_radii (the oracle's kNN is brute force, so skip it otherwise)
    kw_ = min(prm["kw"], L)
    if prm["use_radii"] and kw_ > 0:
        radii = O.radii(Lk, O.knn(Lk, Lk, kw_))
    else:
        radii = np.full(L, prm["screen"], np.float32)
    res1, org1, h1 = O.voxel_grid(Pk, prm["offset_1"], prm["grid_reso"])
    G1 = O.grid_points(res1, org1, h1)
    res2, org2, h2 = O.voxel_grid(Pk, prm["offset_2"], prm["final_reso"])
    G2 = O.grid_points(res2, org2, h2)
    PA = np.full(len(Pk), prm["area"], np.float32)
    t1 = IglTree(Pk, prm["max_depth"], A=PA)
    lnrm0 = np.tile(np.float32([0, 0, 1]), (L, 1))
    lnrm = np.empty_like(lnrm0)
    secs = np.zeros(2, np.float64)
    own = workdir is None
    wd = tempfile.mkdtemp(prefix="refdwg_") if own else workdir
    base = os.path.join(wd, "mesh")
    log = os.path.join(wd, "log.txt")
    r1 = _c(res1, np.int32)
    r2 = _c(res2, np.int32)
    rc = lib().refdwg_run(L, _p(Lk), _p(lnrm0), _p(An), _p(radii), len(G1), _p(G1), _p(r1), _p(lbounds),
                          *t2.args(),
                          float(prm["lambda_"]), int(prm["total_iter"]), int(prm["use_radii"]),
                          float(prm["as_thres"]), int(prm["in_normal"]),
                          len(Pk), _p(Pk), _p(PA), len(G2), _p(G2), _p(r2), _p(pbounds),
                          *t1.args(),
                          int(prm["final_kw"]), int(prm["normal_kw"]), base.encode(), log.encode(),
                          _p(lnrm), _p(secs))
    if rc != 0:
        raise RuntimeError(f"refdwg_run failed ({rc})")
    text = open(log).read()
    means = [float(x) for x in re.findall(r"W_mean = (\S+)", text)]
    tris_n = [int(x) for x in re.findall(r"Num triangles: (\d+)", text)]
    zeros, z_by_iter, it = [], {}, -1
    for line in text.splitlines():
        m = re.match(r"iter = (\d+)", line)
        if m:
            it = int(m.group(1))
        m = re.match(r"number of zero normals = (\d+)", line)
        if m:
            z_by_iter[it] = int(m.group(1))
    T_iter = prm["total_iter"]
    zeros = np.array([z_by_iter.get(t, 0) for t in range(T_iter)], np.int32)
    xyz = np.loadtxt(base + ".xyz", dtype=np.float64).reshape(-1, 6)
    tris = read_stl(base + ".stl")
    out = {
        "points": Pk, "perm": perm_p, "leaf_pos": Lk, "leaf_nrm": lnrm,
        "w_mean": np.array(means[:T_iter], np.float64),
        "tri_count": np.array(tris_n[:T_iter], np.int64), "zero_count": zeros,
        "point_pos": xyz[:, :3].astype(np.float32), "point_nrm": xyz[:, 3:].astype(np.float32),
        "tris": tris, "secs": secs.copy(), "iter_res": res1, "final_res": res2,
    }
    if own:
        for f in (base + ".xyz", base + ".stl", log):
            if os.path.exists(f):
                os.remove(f)
        os.rmdir(wd)
    return out


def reconstruct_isolated(P, timeout=1800, **kw):
    """:func:`reconstruct` in a child process.  The reference ends the process
    on a CUDA error (exit() in gpuErrchk, or an uncaught thrust exception);
    here that surfaces as a RuntimeError carrying the child's output."""
    import json
    import subprocess
    import sys

    wd = tempfile.mkdtemp(prefix="refdwg_child_")
    fin, fout = os.path.join(wd, "in.npz"), os.path.join(wd, "out.npz")
    np.savez(fin, P=_c(P, np.float32))
    root = os.path.dirname(_HERE)
    try:
        r = subprocess.run([sys.executable, "-m", "oracle.ref_dwg", fin, fout, json.dumps(kw)], cwd=root,
                           capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0 or not os.path.exists(fout):
            raise RuntimeError(f"reference run failed (rc {r.returncode}):\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}")
        with np.load(fout) as z:
            return {k: z[k] for k in z.files}
    finally:
        for f in (fin, fout):
            if os.path.exists(f):
                os.remove(f)
        os.rmdir(wd)


if __name__ == "__main__":
    import json
    import sys

    with np.load(sys.argv[1]) as z:
        P_in = z["P"]
    res_ = reconstruct(P_in, **json.loads(sys.argv[3]))
    np.savez(sys.argv[2], **res_)
