"""The profiling recipe of this repository: small, self-contained workloads
for profiler captures of the hot kernels, and a summariser of a profiler
launch list (the ncu summaries under profiles/ name the command that made
them).

    python profile_cases.py step     [--points N --grid R --iters T --reps K --shape torus|sq_union
                                      --grid-lists 0|1|2]
    python profile_cases.py gwn_grid [--points N --grid R --launches K --lists [1|2]]
    python profile_cases.py knn_tri  [--points N --grid R --launches K --shape torus|sq_union]
    python profile_cases.py mc       [--points N --grid R --launches K]
    python profile_cases.py summarize launches.csv

``step`` runs whole reconstructions (create, iterate, finalize) of the seeded
non-uniform torus (or the superquadric union) and prints per-phase host
timings; ``--grid-lists 0`` turns off the kept interaction lists and
screening weights (the same results bit for bit, a small fraction of the
device memory, for captures that save and restore it).  The single-kernel cases
first run one plain DWG iteration to obtain a realistic state (leaf normals,
iteration-0 field and triangles), then launch only the named kernel
``--launches`` times, so that a capture filtered by kernel name and launch
count sees warm, representative launches.  ``gwn_grid --lists 1`` records the
grid's interaction lists in its first call and replays them in the others;
``--lists 2`` also writes the screening weights in the first call and reads
them in the others.
``summarize`` turns a CSV launch
list (``gpu__time_duration.sum`` per launch) into per-kernel launches, total
time and share.
"""
from __future__ import annotations

import argparse
import collections
import csv
import ctypes as C
import re
import sys
import time

import os

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

_SHAPE = "torus"


def _cloud(n, seed=1000):
    from dwg_b200 import datasets as D
    if _SHAPE == "sq_union":  # 12 superquadrics + 1 % outliers
        P, _ = D.superquadric_union(int(round(n / 1.01)), seed=seed)
    else:
        P, _ = D.torus(n, seed=seed)
    Pn, _, _ = D.normalize(P)
    return Pn.astype(np.float32)


def case_step(a):
    import torch
    from dwg_b200 import capi
    lib = capi.load()
    P = _cloud(a.points)
    Pd = torch.from_numpy(P).cuda()
    prm = capi.default_params(grid_reso=a.grid, final_reso=a.grid, total_iter=a.iters, grid_lists=a.grid_lists)
    n = len(P)
    for rep in range(a.reps):
        h = C.c_void_p()
        torch.cuda.synchronize()
        t = [time.perf_counter()]
        capi.check(lib.dwg_pipeline_create(capi.ptr(Pd), None, n, C.byref(prm), None, C.byref(h)))
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        capi.check(lib.dwg_pipeline_iterate(h, a.iters))
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        capi.check(lib.dwg_pipeline_finalize(h))
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        lib.dwg_pipeline_destroy(h)
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        d = np.diff(t) * 1e3
        print(f"rep {rep}: create {d[0]:.1f} ms, {a.iters} iterations {d[1]:.1f} ms "
              f"({d[1] / max(1, a.iters):.2f}/it), finalize {d[2]:.1f} ms, destroy {d[3]:.1f} ms", flush=True)


def _iteration0_state(a):
    """Leaves, leaf normals, grid and the iteration-0 field / triangles."""
    import torch
    from dwg_b200 import turbo
    Pd = torch.from_numpy(_cloud(a.points)).cuda()
    d = turbo.TurboDWG(Pd, None, grid_reso=a.grid, final_reso=a.grid, total_iter=1, use_graph=0)
    st = {"leaf_pos": d.get("leaf_pos"), "leaf_nrm": d.get("leaf_nrm"), "res": d.get("grid_res"),
          "org": d.get("grid_origin")}
    d.TurboScreenedDWGLaunch(1)
    st["field"] = d.get("field")
    st["iso"] = float(d.get("iso")[0])
    d.close()
    torch.cuda.synchronize()
    return st


def case_gwn_grid(a):
    import torch
    from dwg_b200 import turbo
    st = _iteration0_state(a)
    L = len(st["leaf_pos"])
    lp = torch.from_numpy(st["leaf_pos"]).cuda()
    ln = torch.from_numpy(st["leaf_nrm"]).cuda()
    A = torch.full((L,), 2e-6, device="cuda")
    tree = turbo.TurboLibiGWN(lp, max_depth=10, areas=A)
    tree.UpdateMassNormals(ln, A)
    res, org = st["res"], st["org"]
    out = torch.empty(int(np.prod(res)), device="cuda")
    for _ in range(a.launches):
        tree.grid(res, org[:3], float(org[3]), sigma=20.0, precision=1, out=out, lists=a.lists)
    torch.cuda.synchronize()
    print("gwn_grid", res.tolist(), L, tree.status())


def _mc_buffers(res):
    import torch
    cap = max(int(np.prod(res)) // 2, 1000000)
    return (torch.empty((cap, 9), device="cuda"), torch.empty((cap, 3), device="cuda"),
            torch.empty((cap, 3), device="cuda"), cap)


def case_mc(a):
    import torch
    from dwg_b200 import turbo
    st = _iteration0_state(a)
    res, org = st["res"], st["org"]
    tris, cent, nrm, cap = _mc_buffers(res)
    mc = turbo.TurboMC()
    field = torch.from_numpy(st["field"]).cuda()
    for _ in range(a.launches):
        T = mc.TurboMarchingCubes(field, None, int(res[0]), int(res[1]), int(res[2]), st["iso"],
                                  mid_points=cent, mid_normals=nrm, origin=org[:3], spacing=float(org[3]),
                                  tris=tris, capacity=cap)
    torch.cuda.synchronize()
    print("mc", res.tolist(), T)


def case_knn_tri(a):
    import torch
    from dwg_b200 import turbo
    st = _iteration0_state(a)
    res, org = st["res"], st["org"]
    tris, cent, nrm, cap = _mc_buffers(res)
    mc = turbo.TurboMC()
    field = torch.from_numpy(st["field"]).cuda()
    T = mc.TurboMarchingCubes(field, None, int(res[0]), int(res[1]), int(res[2]), st["iso"],
                              mid_points=cent, mid_normals=nrm, origin=org[:3], spacing=float(org[3]),
                              tris=tris, capacity=cap)
    q = cent[:T].contiguous()
    idx = turbo.KnnIndex(torch.from_numpy(st["leaf_pos"]).cuda())
    out = torch.empty((T, 15), dtype=torch.int32, device="cuda")
    for _ in range(a.launches):
        idx.query(q, 15, out=out)
    torch.cuda.synchronize()
    print("knn_tri", T, len(st["leaf_pos"]))


def summarize(path, top=25):
    rows = list(csv.reader(open(path)))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    h = rows[hi]
    ki, mi, ui = h.index("Kernel Name"), h.index("Metric Value"), h.index("Metric Unit")
    scale = {"nsecond": 1e-6, "ns": 1e-6, "usecond": 1e-3, "us": 1e-3, "msecond": 1.0, "ms": 1.0,
             "second": 1e3, "s": 1e3}
    tot, cnt = collections.defaultdict(float), collections.Counter()
    for r in rows[hi + 1:]:
        if len(r) <= mi:
            continue
        v = float(r[mi].replace(",", "")) * scale[r[ui]]
        name = re.sub(r"\(.*", "", r[ki])[:90]
        tot[name] += v
        cnt[name] += 1
    T = sum(tot.values())
    lines = [f"total kernel time {T:.2f} ms over {sum(cnt.values())} launches",
             f"{'total ms':>10} {'share':>7} {'launches':>8}  kernel"]
    for k, v in sorted(tot.items(), key=lambda x: -x[1])[:top]:
        lines.append(f"{v:10.3f} {100 * v / T:6.2f}% {cnt[k]:8d}  {k}")
    return "\n".join(lines)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=["step", "gwn_grid", "knn_tri", "mc", "summarize"])
    ap.add_argument("path", nargs="?")
    ap.add_argument("--points", type=int, default=100000)
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--iters", type=int, default=30)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--launches", type=int, default=2)
    ap.add_argument("--shape", choices=["torus", "sq_union"], default="torus")
    ap.add_argument("--lists", type=int, nargs="?", const=1, default=0, choices=[0, 1, 2])
    ap.add_argument("--grid-lists", type=int, default=2, choices=[0, 1, 2])
    a = ap.parse_args(argv)
    global _SHAPE
    _SHAPE = a.shape
    if a.case == "summarize":
        print(summarize(a.path))
        return
    {"step": case_step, "gwn_grid": case_gwn_grid, "knn_tri": case_knn_tri, "mc": case_mc}[a.case](a)


if __name__ == "__main__":
    sys.exit(main())
