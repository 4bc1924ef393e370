#!/usr/bin/env python
"""Benchmark: DWG reconstruction throughput on B200 (one JSON line on rank 0).

Workload (default, --workload c3): the thin-feature union -- 1,000,000 points
on the surface of a union of 12 seeded superquadrics (exponents in [0.3, 3],
semi-axes in [0.05, 1], random rotations) plus 1 % uniform outliers in the
box, 1,010,000 points in all; reference-default DWG flags with grid_reso =
final_reso = 256 and 30 diffusion iterations.  One step = one full
reconstruction from device-resident points to the mesh in device memory (GPU
octrees, leaves, kNN index, 30 iterations of GWN / MC / kNN / diffusion,
final pass).  --workload c2 (nonuniform torus, 100k, 256^3) and c1 (noisy
sphere, 10k, 128^3) are the other single-GPU configurations.

value       Mpts/s = points / step time (sum over ranks for --gpus N; every
            rank reconstructs its own cloud, replicas -- the path has no
            cross-GPU exchange)
accuracy    the final field (the mesh's field) of the last timed step against
            the FP64 sums of the same state (FP64 terms and sums on the GPU
            with the same opening decisions, dwg_gwn_points_fp64, which the
            tests pin to the FP64 CPU restatement) on 2^20 seeded samples of
            the final grid: RMS and max error; "converged" = RMS <= 1e-4
e2e         the same through dwg_reconstruct_host: pinned host points in,
            mesh + point normals out, copies inside the timed region
roofline    the kernel with the largest device time in the kernel census of
            one step, timed alone with CUDA events on its stream; the other
            rooflines under "rooflines"
cpu_baseline  the reference's CPU winding-number path (igl::fast_winding_number:
            Barnes-Hut over the same sources and queries, order 0 with
            beta 2.3 as DWG, and libigl's default order 2 with beta 2), timed
            on a seeded sample of the queries of one reconstruction on all
            host cores and scaled to all of them (octree and moments timed)

--impl reference  the same CPU path as one JSON line with "impl": "reference"
            (each step a timed sample, the value scaled to a reconstruction),
            plus the reference's own GPU DWG run (its sources compiled
            unchanged, oracle/_ref) on the same cloud when that comparator is
            built: one full reconstruction, device seconds, measured.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpts/s to converged mesh at RMS GWN err≤1e-4; pair-evals/s; learned vs plain iters"
WORKLOADS = {
    "c3": dict(workload="thin-feature union: 1,000,000 points on 12 seeded superquadrics + 1% outliers "
                        "(1,010,000), 256^3 grid, 30 DWG iterations",
               dataset="c3_sq_union_1m", grid_reso=256, final_reso=256, total_iter=30, beta=2.3, max_depth=10),
    "c2": dict(workload="nonuniform torus 100k points, 256^3 grid, 30 DWG iterations",
               dataset="c2_torus_100k", grid_reso=256, final_reso=256, total_iter=30, beta=2.3, max_depth=10),
    "c1": dict(workload="noisy sphere 10k points, 128^3 grid, 30 DWG iterations",
               dataset="c1_sphere_10k", grid_reso=128, final_reso=128, total_iter=30, beta=2.3, max_depth=10),
}
PRECISION = {0: "fp32", 1: "fp32-terms-fp64-sum", 2: "fp32-accurate-terms-fp64-sum",
             3: "fp32-terms-compensated-fp32-sum"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", type=int, default=1, choices=sorted(PRECISION))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the precision, far-field, learned-start and batched-clouds reports")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip the run of the reference's own GPU code")
    a = ap.parse_args()
    a.cfg = WORKLOADS[a.workload]
    a.grid = a.cfg["grid_reso"]
    a.iters = a.cfg["total_iter"]
    return a


_CLOUDS = {}


def make_cloud(a, rank):
    """The workload's seeded cloud, normalised as the reference reads it."""
    key = (a.workload, rank)
    if key not in _CLOUDS:
        from dwg_b200 import datasets as D
        P, _ = D.make(a.cfg["dataset"], seed=1000 + rank)
        Pn, _, _ = D.normalize(P)
        _CLOUDS[key] = np.ascontiguousarray(Pn, np.float32)
    return _CLOUDS[key]


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# -------------------------------------------------------------- ours (GPU) --
def _timed_steps(one_step, lib, torch, stream, flush, steps, keep_last=False):
    """Device time of `steps` steps (CUDA events on the step's stream, L2
    flushed before each); returns (ms list, last pipeline or None)."""
    step_ms, last = [], None
    for i in range(steps):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h = one_step()
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        print(f"step: {step_ms[-1]:.1f} ms", file=sys.stderr)
        if keep_last and i == steps - 1:
            last = h
        else:
            lib.dwg_pipeline_destroy(h)
    return step_ms, last


def run_ours(a, rank, world, local_rank):
    import ctypes as C

    import torch

    from dwg_b200 import build, capi, turbo

    build.build()
    lib = capi.load()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    P = make_cloud(a, rank)
    npts = len(P)
    Pd = torch.from_numpy(P).to(dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    flush = torch.empty(int(256 * 2**20), dtype=torch.uint8, device=dev)  # > 126 MB L2

    def stepper(precision):
        prm = capi.default_params(grid_reso=a.grid, final_reso=a.grid, total_iter=a.iters, precision=precision,
                                  use_graph=1)

        def one_step():
            h = C.c_void_p()
            capi.check(lib.dwg_pipeline_create(capi.ptr(Pd), None, npts, C.byref(prm), sp, C.byref(h)))
            capi.check(lib.dwg_pipeline_iterate(h, a.iters))
            capi.check(lib.dwg_pipeline_finalize(h))
            return h
        return one_step, prm

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    one_step, prm = stepper(a.precision)
    # warm-up
    last = None
    for _ in range(max(a.warmup, 0)):
        h = one_step()
        torch.cuda.synchronize()
        if last is not None:
            lib.dwg_pipeline_destroy(last)
        last = h
    terms_per_iter = np.zeros(a.iters, np.uint64)
    tri_count = np.zeros(a.iters, np.int64)
    final_tris = 0
    if last is not None:
        v = C.c_longlong()
        capi.check(lib.dwg_pipeline_size(last, b"triangles", C.byref(v)))
        capi.check(lib.dwg_pipeline_get(last, b"terms", terms_per_iter.ctypes.data))
        capi.check(lib.dwg_pipeline_get(last, b"tri_count", tri_count.ctypes.data))
        final_tris = v.value
        lib.dwg_pipeline_destroy(last)
    census = kernel_census(one_step, lib, torch)

    # timed: device events per step, L2 flushed between steps
    clocks = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    step_ms, last = _timed_steps(one_step, lib, torch, stream, flush, a.steps, keep_last=True)
    barrier()
    torch.cuda.synchronize()
    ms = float(np.mean(step_ms))

    # end to end through the host entry point (pinned buffers, copies timed)
    Ph = torch.from_numpy(P).pin_memory()
    cap_tris = max(final_tris * 2, 1_000_000)
    tris_h = torch.empty((cap_tris, 9), dtype=torch.float32).pin_memory()
    nrm_h = torch.empty((npts, 3), dtype=torch.float32).pin_memory()
    e2e_ms, e2e_wall_ms = [], []
    ntri = C.c_longlong()
    for i in range(max(1, a.steps)):
        flush.fill_(2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        # synchronous: H2D of the points, reconstruction, D2H of mesh and normals
        capi.check(lib.dwg_reconstruct_host(capi.ptr(Ph), None, npts, C.byref(prm), capi.ptr(nrm_h),
                                            capi.ptr(tris_h), cap_tris, C.byref(ntri), sp))
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
        e2e_wall_ms.append((time.perf_counter() - t0) * 1e3)
        print(f"e2e call {i}: {e2e_ms[-1]:.1f} ms (device), {e2e_wall_ms[-1]:.1f} ms (host)", file=sys.stderr)
    clk = clocks.stop()

    # the converged criterion on the last timed step's final field
    acc = accuracy_gate(lib, capi, turbo, torch, dev, Pd, last, prm)
    lib.dwg_pipeline_destroy(last)

    # kernel-level rooflines
    peaks = load_peaks()
    roofs = {}
    for name, fn in (("gwn", gwn_roofline), ("knn", knn_roofline)):
        try:
            roofs[name] = fn(a, lib, capi, turbo, torch, dev, P, peaks)
        except Exception as e:  # a roofline must not take the headline line down
            roofs[name] = {"error": f"{type(e).__name__}: {e}"}
    dominant = _dominant_roofline(census, roofs)
    if census:
        census.pop("all", None)

    extras = {}
    if rank == 0 and not a.no_extras:
        for name, fn in (("precision_variants", precision_variants), ("precision", precision_report),
                         ("farfield", farfield_report), ("learned", learned_report), ("batched", batched_report)):
            try:
                extras[name] = fn(a, lib, capi, turbo, torch, dev, stepper, flush, stream, Pd)
            except Exception as e:  # a report must not take the headline line down
                extras[name] = {"error": f"{type(e).__name__}: {e}"}
            print(f"{name} report done", file=sys.stderr, flush=True)

    # max over ranks
    vals = torch.tensor([ms, float(np.mean(e2e_ms))], dtype=torch.float64, device=dev)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    ms, ems = float(vals[0]), float(vals[1])
    total_pts = npts * world
    out = {
        "metric": METRIC,
        "value": total_pts / (ms * 1e-3) / 1e6,
        "unit": "Mpts/s",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": ms,
        "step_ms": [round(x, 2) for x in step_ms],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded procedural clouds; no dataset)",
        "config": dict(a.cfg, points=npts, precision=PRECISION[a.precision], parallelism=f"replicas x{world}",
                       l2="flushed (256 MB write) between timed steps", triangles_final=int(final_tris)),
        "converged": acc.get("converged"),
        "accuracy": acc,
        "pair_evals_per_s": float(terms_per_iter.sum()) / (ms * 1e-3) * world,
        "terms_per_iteration": int(terms_per_iter.mean()) if len(terms_per_iter) else 0,
        "triangles_per_iteration": int(tri_count.mean()) if len(tri_count) else 0,
        "e2e": {"value": total_pts / (ems * 1e-3) / 1e6, "unit": "Mpts/s", "ms_per_step": ems,
                "host_wall_ms_per_step": float(np.mean(e2e_wall_ms)),
                "h2d_bytes_per_step": npts * 12, "d2h_bytes_per_step": int(ntri.value) * 36 + npts * 12},
        "gpu_launches": census["per_step"] * a.steps if census else None,
        "kernel_census": census,
        "roofline": roofs.get(dominant),
        "rooflines": roofs,
        "clocks": clk,
    }
    out.update(extras)
    return out


def _dominant_roofline(census, roofs):
    """The roofline of the kernel with the largest device time in one step
    (the GWN weight read or the cell-grouped kNN, whichever leads)."""
    if not census:
        return "gwn"
    rows = census.get("all", census.get("top", []))
    top = max(rows, key=lambda r: r["ms"]) if rows else None
    best = "knn" if top and ("k_knn" in top["kernel"] or "k_cq_" in top["kernel"]) else "gwn"
    return best if "error" not in roofs.get(best, {"error": 1}) else "gwn"


def kernel_census(one_step, lib, torch):
    """Kernels of one (untimed) step, counted from CUPTI activity records
    (graph replays included) by liblaunch_counter.so: per-step launch count
    of this library's kernels (dwg:: and its CUB instantiations) and the
    device-time share of the top ones."""
    import ctypes as C

    from dwg_b200 import build
    try:
        lc = C.CDLL(build.COUNTER)
    except OSError as e:
        print(f"kernel census unavailable: {e}", file=sys.stderr)
        return None
    lc.dwglc_report.argtypes = [C.c_char_p, C.c_int]
    torch.cuda.synchronize()
    if lc.dwglc_start() != 0:
        print("kernel census unavailable: CUPTI refused activity tracing", file=sys.stderr)
        return None
    h = one_step()
    torch.cuda.synchronize()
    lc.dwglc_stop()
    lib.dwg_pipeline_destroy(h)
    n = lc.dwglc_report(None, 0)
    buf = C.create_string_buffer(n)
    lc.dwglc_report(buf, n)
    rows = []
    for line in buf.value.decode().splitlines():
        name, cnt, ns = line.rsplit("\t", 2)
        if "dwg::" in name or "cub::" in name:
            rows.append((name, int(cnt), int(ns) / 1e6))
    total_ms = sum(r[2] for r in rows)
    rows.sort(key=lambda r: -r[2])
    fmt = [{"kernel": r[0][:80], "launches": r[1], "ms": round(r[2], 3),
            "share": round(r[2] / total_ms, 4) if total_ms else None} for r in rows]
    return {"per_step": sum(r[1] for r in rows), "kernel_ms_per_step": total_ms, "top": fmt[:8], "all": fmt}


def _pipeline_tensors(lib, capi, torch, dev, h, what, shape):
    import ctypes as C
    ptr = C.c_void_p()
    capi.check(lib.dwg_pipeline_device_ptr(h, what, C.byref(ptr)))
    t = torch.empty(shape, dtype=torch.float32, device=dev)
    nbytes = int(np.prod(shape)) * 4
    cudart_copy(torch, t, ptr.value, nbytes)
    # the copy runs on torch's stream; it must be done before the pipeline
    # is destroyed (dwg_pipeline_destroy waits for the pipeline's stream only)
    torch.cuda.current_stream(dev).synchronize()
    return t


def accuracy_gate(lib, capi, turbo, torch, dev, Pd, h, prm, samples=1 << 20):
    """The final field of pipeline h against the FP64 sums of the same state:
    an octree built the same way on the points (same depth and areas, hence
    the same nodes and opening decisions) with the final point normals,
    summed in FP64 on the GPU at seeded samples of the final grid."""
    import ctypes as C
    res = np.zeros(3, np.int32)
    org = np.zeros(4, np.float32)
    capi.check(lib.dwg_pipeline_get(h, b"final_res", res.ctypes.data))
    capi.check(lib.dwg_pipeline_get(h, b"final_origin", org.ctypes.data))
    n = int(Pd.shape[0])
    ng = int(np.prod(res.astype(np.int64)))
    field = _pipeline_tensors(lib, capi, torch, dev, h, b"final_field", (ng,))
    nrm = _pipeline_tensors(lib, capi, torch, dev, h, b"point_nrm", (n, 3))
    rng = np.random.default_rng(12345)
    sel = np.sort(rng.choice(ng, min(samples, ng), replace=False))
    x, y, z = sel % res[0], (sel // res[0]) % res[1], sel // (res[0] * res[1])
    h32 = np.float32(org[3])
    Q = np.stack([org[0] + x.astype(np.float32) * h32, org[1] + y.astype(np.float32) * h32,
                  org[2] + z.astype(np.float32) * h32], 1).astype(np.float32)
    area = torch.full((n,), float(prm.area), dtype=torch.float32, device=dev)
    tree = turbo.TurboLibiGWN(Pd, max_depth=int(prm.max_depth), areas=area)
    t0 = time.perf_counter()
    w64 = tree.values_fp64(torch.from_numpy(Q).to(dev), i_Normals=nrm, i_As=area, beta=float(prm.beta),
                           sigma=float(prm.lambda_), screened=True, screen=float(prm.screen))
    torch.cuda.synchronize()
    fp64_s = time.perf_counter() - t0
    tree.status()
    w32 = field[torch.from_numpy(sel).to(dev)].double()
    d = (w32 - w64).cpu().numpy()
    ref = w64.cpu().numpy()
    rms = float(np.sqrt(np.mean(d ** 2)))
    del C
    return {"field": "final field (the mesh's), last timed step", "samples": int(len(sel)),
            "rms_abs_err": rms, "max_abs_err": float(np.abs(d).max()),
            "field_rms": float(np.sqrt(np.mean(ref ** 2))), "field_max": float(np.abs(ref).max()),
            "threshold_rms": 1e-4, "converged": bool(rms <= 1e-4),
            "against": "FP64 terms and sums on the GPU, same octree and opening decisions (dwg_gwn_points_fp64)",
            "fp64_seconds": fp64_s}


def gwn_roofline(a, lib, capi, turbo, torch, dev, P, peaks):
    """The GWN grid kernel that reads kept screening weights (the iteration
    grid's sums in 28 of 30 iterations), timed alone on the iteration-0 state:
    HBM-bound, 272 algorithmic bytes per list entry + 4 per sample; the
    evaluating replay and the traversal beside it (20 FP32 flops per term)."""
    import ctypes as C
    prm = capi.default_params(grid_reso=a.grid, final_reso=a.grid, total_iter=0, precision=a.precision)
    h = C.c_void_p()
    Pd = torch.from_numpy(P).to(dev)
    sp = torch.cuda.current_stream(dev).cuda_stream
    capi.check(lib.dwg_pipeline_create(capi.ptr(Pd), None, len(P), C.byref(prm), sp, C.byref(h)))
    L = C.c_longlong()
    capi.check(lib.dwg_pipeline_size(h, b"leaves", C.byref(L)))
    n = L.value
    leaves = _pipeline_tensors(lib, capi, torch, dev, h, b"leaf_pos", (n, 3))
    nrm = _pipeline_tensors(lib, capi, torch, dev, h, b"leaf_nrm", (n, 3))
    res = np.zeros(3, np.int32)
    org = np.zeros(4, np.float32)
    capi.check(lib.dwg_pipeline_get(h, b"grid_res", res.ctypes.data))
    capi.check(lib.dwg_pipeline_get(h, b"grid_origin", org.ctypes.data))
    lib.dwg_pipeline_destroy(h)
    area = torch.full((n,), 2e-6, dtype=torch.float32, device=dev)
    tree = turbo.TurboLibiGWN(leaves, max_depth=a.cfg["max_depth"], areas=area)
    tree.UpdateMassNormals(nrm, area)
    out = torch.empty(int(np.prod(res.astype(np.int64))), dtype=torch.float32, device=dev)
    terms = torch.zeros(1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(lists):
        # the first call with lists records them (untimed); the reconstruction
        # replays them in every iteration after the first
        for _ in range(2):
            tree.grid(res, org[:3], float(org[3]), sigma=20.0, precision=a.precision, out=out, lists=lists)
        torch.cuda.synchronize()
        times = []
        for _ in range(5):
            terms.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            tree.grid(res, org[:3], float(org[3]), sigma=20.0, precision=a.precision, out=out, terms=terms,
                      lists=lists)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        tree.status()
        return float(np.median(times)) * 1e-3, float(terms.item())

    t_trav, n_trav = timed(0)
    t, nterm = timed(1)
    assert nterm == n_trav, (nterm, n_trav)
    t_w, n_w = timed(2)
    assert n_w == n_trav, (n_w, n_trav)
    entries, slots = tree.list_size()
    clk = float(peaks.get("sm_max_mhz", 1965.0))
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32_peak = sms * 128 * 2 * clk * 1e6 / 1e12
    mufu_peak = sms * 16 * clk * 1e6 / 1e12
    achieved = 20.0 * nterm / t / 1e12
    traffic = _traffic("gwn_wread", a.workload)
    nq = float(np.prod(res.astype(np.float64)))
    # kept weights read: 8 B per entry and lane (32 lanes), the 16-B entry, 8 B
    # offsets per group of 64 samples, 4 B per sample written; the node
    # records stay in L2 and are not counted
    wbytes = entries * (32 * 8 + 16) + nq / 64 * 8 + nq * 4
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    return {
        "kernel": f"k_gwn_wread (screened grid sums from kept weights; {res.tolist()} grid, iteration-0 state)",
        "bound": "hbm",
        "achieved": wbytes / t_w / 1e9,
        "peak": hbm,
        "unit": "GB/s",
        "frac": wbytes / t_w / 1e9 / hbm,
        "traffic": traffic,
        "peak_source": "of measured: hbm_gbs of MEASURED_PEAKS.json" if "hbm_gbs" in peaks else "of fallback 6650",
        "launch_ms": t_w * 1e3,
        "algorithmic_bytes": wbytes,
        "list_entries": entries,
        "weight_slots": slots,
        "pair_terms": nterm,
        "algorithmic": "272 B per list entry + 4 B per sample written (+8 B per 64 samples); terms counted in-kernel",
        "evaluating_launches": {
            "replay_ms": t * 1e3,
            "traversal_ms": t_trav * 1e3,
            "bound": "fp32 issue",
            "achieved_tflops": achieved,
            "peak_tflops": fp32_peak,
            "frac": achieved / fp32_peak,
            "peak_source": ("nominal FP32 SIMT = SMs x 128 lanes x 2 x sm_max_mhz of MEASURED_PEAKS.json "
                            "(the file measures HBM copy and bf16 GEMM only)"),
            "sfu_frac": 3.0 * nterm / t / 1e12 / mufu_peak,
            "algorithmic": "20 FP32 flops + 3 MUFU per pair term (screened)",
        },
    }


def knn_roofline(a, lib, capi, turbo, torch, dev, P, peaks):
    """The triangle kNN of an iteration (15 nearest leaves of every triangle
    centroid), timed alone on the iteration-0 mesh: 12 B per leaf + 12 B per
    query + 4 k B of indices written, against the HBM copy bandwidth (the
    kernel is bound by instruction issue; the fraction shows how far)."""
    import ctypes as C
    prm = capi.default_params(grid_reso=a.grid, final_reso=a.grid, total_iter=a.iters, precision=a.precision)
    h = C.c_void_p()
    Pd = torch.from_numpy(P).to(dev)
    capi.check(lib.dwg_pipeline_create(capi.ptr(Pd), None, len(P), C.byref(prm), None, C.byref(h)))
    capi.check(lib.dwg_pipeline_iterate(h, 1))
    L = C.c_longlong()
    capi.check(lib.dwg_pipeline_size(h, b"leaves", C.byref(L)))
    n = L.value
    leaves = _pipeline_tensors(lib, capi, torch, dev, h, b"leaf_pos", (n, 3))
    res = np.zeros(3, np.int32)
    org = np.zeros(4, np.float32)
    capi.check(lib.dwg_pipeline_get(h, b"grid_res", res.ctypes.data))
    capi.check(lib.dwg_pipeline_get(h, b"grid_origin", org.ctypes.data))
    ng = int(np.prod(res.astype(np.int64)))
    field = _pipeline_tensors(lib, capi, torch, dev, h, b"field", (ng,))
    iso = np.zeros(1, np.float32)
    capi.check(lib.dwg_pipeline_get(h, b"iso", iso.ctypes.data))
    lib.dwg_pipeline_destroy(h)
    cap = max(ng // 2, 1000000)
    cen = torch.empty((cap, 3), dtype=torch.float32, device=dev)
    T = turbo.TurboMC().TurboMarchingCubes(field, None, int(res[0]), int(res[1]), int(res[2]), float(iso[0]),
                                           mid_points=cen, origin=org[:3], spacing=float(org[3]))
    Qd = cen[:T].contiguous()
    ix = turbo.KnnIndex(leaves)
    k = 15
    out = torch.empty((T, k), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(2):
        ix.query(Qd, k, out=out)
    torch.cuda.synchronize()
    times = []
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ix.query(Qd, k, out=out)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    t = float(np.median(times)) * 1e-3
    nbytes = 12.0 * n + 12.0 * T + 4.0 * k * T
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    return {"kernel": "dwg_knn_query (k_cq_key/k_cq_scatter + k_knn_cells, k_knn_thread for overflow): "
                      f"15 nearest of {n} leaves for the {T} triangle centroids of iteration 0",
            "bound": "hbm", "achieved": nbytes / t / 1e9, "peak": hbm, "unit": "GB/s",
            "frac": nbytes / t / 1e9 / hbm, "traffic": _traffic("knn_cells", a.workload),
            "peak_source": "of measured: hbm_gbs of MEASURED_PEAKS.json" if "hbm_gbs" in peaks else "of fallback 6650",
            "launch_ms": t * 1e3, "algorithmic_bytes": nbytes, "queries": int(T), "points": int(n), "k": k,
            "algorithmic": "12 B per point + 12 B per query + 4 k B per query (ids written)",
            "queries_per_s": T / t}


def _traffic(kernel, workload):
    """DRAM bytes of one launch from the committed ncu figures (profiles/traffic.txt, JSON)."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "traffic.txt")))
        return d.get(f"{kernel}:{workload}")
    except Exception:
        return None


def precision_variants(a, lib, capi, turbo, torch, dev, stepper, flush, stream, Pd):
    """The same reconstruction with the other precision modes: device time of
    3 steps and the accuracy gate of each."""
    out = {}
    for prec in (0, 1, 3):
        one_step, prm = stepper(prec)
        h = one_step()
        torch.cuda.synchronize()
        lib.dwg_pipeline_destroy(h)
        ms, last = _timed_steps(one_step, lib, torch, stream, flush, 3, keep_last=True)
        acc = accuracy_gate(lib, capi, turbo, torch, dev, Pd, last, prm)
        lib.dwg_pipeline_destroy(last)
        out[PRECISION[prec]] = {"ms_per_step": float(np.mean(ms)), "Mpts_per_s": len(Pd) / np.mean(ms) / 1e3,
                                "final_field_rms_err_vs_fp64": acc["rms_abs_err"],
                                "final_field_max_err_vs_fp64": acc["max_abs_err"], "converged": acc["converged"]}
    return out


def _pipeline_state(lib, capi, torch, dev, P, flags, iters):
    """leaf positions / normals (host), grid res and origin after `iters` iterations"""
    import ctypes as C
    prm = capi.default_params(**flags)
    h = C.c_void_p()
    Pd = torch.from_numpy(np.ascontiguousarray(P, np.float32)).to(dev)
    capi.check(lib.dwg_pipeline_create(capi.ptr(Pd), None, len(P), C.byref(prm), None, C.byref(h)))
    try:
        if iters:
            capi.check(lib.dwg_pipeline_iterate(h, iters))
        L = C.c_longlong()
        capi.check(lib.dwg_pipeline_size(h, b"leaves", C.byref(L)))
        lp = np.empty((L.value, 3), np.float32)
        ln = np.empty((L.value, 3), np.float32)
        res = np.zeros(3, np.int32)
        org = np.zeros(4, np.float32)
        capi.check(lib.dwg_pipeline_get(h, b"leaf_pos", lp.ctypes.data))
        capi.check(lib.dwg_pipeline_get(h, b"leaf_nrm", ln.ctypes.data))
        capi.check(lib.dwg_pipeline_get(h, b"grid_res", res.ctypes.data))
        capi.check(lib.dwg_pipeline_get(h, b"grid_origin", org.ctypes.data))
    finally:
        lib.dwg_pipeline_destroy(h)
    return lp, ln, res, org


def precision_report(a, lib, capi, turbo, torch, dev, *_):
    """Error of the FP32 sums against FP64 sums with the same octree and
    opening decisions, per output (leaf field, grid field) and precision mode;
    the state is the bench cloud after 2 DWG iterations (sigma 20), the grid a
    seeded 20,000-sample subset.  FP64: dwg_gwn_points_fp64 on the GPU."""
    P = make_cloud(a, 0)
    lp, ln, res, org = _pipeline_state(lib, capi, torch, dev, P, dict(grid_reso=a.grid, final_reso=a.grid,
                                                                   total_iter=2), 2)
    n = len(lp)
    A = np.full(n, 2e-6, np.float32)
    rng = np.random.default_rng(7)
    ng = int(np.prod(res.astype(np.int64)))
    sel = rng.choice(ng, min(20000, ng), replace=False)
    idx = np.stack([sel % res[0], (sel // res[0]) % res[1], sel // (res[0] * res[1])], 1).astype(np.float32)
    Q = (org[None, :3].astype(np.float32) + idx * np.float32(org[3])).astype(np.float32)
    lpd, lnd = torch.from_numpy(lp).to(dev), torch.from_numpy(ln).to(dev)
    Ad, Qd = torch.from_numpy(A).to(dev), torch.from_numpy(Q).to(dev)
    tree = turbo.TurboLibiGWN(lpd, max_depth=a.cfg["max_depth"], areas=Ad)
    tree.UpdateMassNormals(lnd, Ad)
    ref_leaf = tree.values_fp64(lpd, beta=2.3, sigma=20.0).cpu().numpy()
    ref_grid = tree.values_fp64(Qd, beta=2.3, sigma=20.0).cpu().numpy()
    out = {"state": "bench cloud after 2 DWG iterations, sigma 20, beta 2.3; grid: 20,000 seeded samples",
           "against": "FP64 terms and sums on the GPU with the same decisions",
           "scale_rms": {"leaf": float(np.sqrt(np.mean(ref_leaf ** 2))), "grid": float(np.sqrt(np.mean(ref_grid ** 2)))}}
    for prec in (0, 1, 2, 3):
        wl = tree.TurboLibiScreenedGWNLaunch(lpd, i_Normals=None, i_As=None, beta=2.3, sigma=20.0,
                                             precision=prec).cpu().numpy().astype(np.float64)
        wg = tree.TurboLibiScreenedGWNLaunch(Qd, i_Normals=None, i_As=None, beta=2.3, sigma=20.0,
                                             precision=prec).cpu().numpy().astype(np.float64)
        el, eg = wl - ref_leaf, wg - ref_grid
        out[PRECISION[prec]] = {"leaf_field": {"max_abs": float(np.abs(el).max()), "rms": float(np.sqrt(np.mean(el ** 2)))},
                                "grid_field": {"max_abs": float(np.abs(eg).max()), "rms": float(np.sqrt(np.mean(eg ** 2)))}}
    # gradients: FP32 terms summed in FP64 against FP64
    _, g32 = tree.value_and_gradient(Qd, beta=2.3, sigma=20.0)
    _, g64 = tree.value_and_gradient(Qd, beta=2.3, sigma=20.0, fp64=True)
    eg = (g32.double() - g64).cpu().numpy()
    out["gradient_fp32_terms_fp64_sum"] = {"max_abs": float(np.abs(eg).max()), "rms": float(np.sqrt(np.mean(eg ** 2))),
                                           "scale_rms": float(torch.sqrt(torch.mean(g64 ** 2)))}
    return out


def farfield_report(a, lib, capi, turbo, torch, dev, *_):
    """Plain winding number with igl::fast_winding_number's far-field
    expansions of orders 0, 1, 2 (beta 2, libigl's default) on a torus of the
    bench's size class with its true normals: device time of the whole
    iteration grid, pair terms, and the error against the exact all-pairs sum
    (FP64 on the GPU, every node opened) on a seeded sample of grid points."""
    from dwg_b200 import datasets as D
    P0, N0 = D.torus(100_000, R=1.0, r=0.35, noise=0.003, seed=1000)
    P, _, sc = D.normalize(P0)
    P = np.ascontiguousarray(P, np.float32)
    N = np.ascontiguousarray(N0, np.float32)
    A = np.full(len(P), 4 * np.pi ** 2 * 1.0 * 0.35 / sc ** 2 / len(P), np.float32)  # torus area / n
    _, _, res, org = _pipeline_state(lib, capi, torch, dev, P, dict(grid_reso=256, final_reso=256, total_iter=0), 0)
    rng = np.random.default_rng(11)
    ng = int(np.prod(res.astype(np.int64)))
    sel = rng.choice(ng, min(20000, ng), replace=False)
    idx = np.stack([sel % res[0], (sel // res[0]) % res[1], sel // (res[0] * res[1])], 1).astype(np.float32)
    Q = (org[None, :3].astype(np.float32) + idx * np.float32(org[3])).astype(np.float32)
    Pd, Nd, Ad, Qd = (torch.from_numpy(x).to(dev) for x in (P, N, A, Q))
    tree = turbo.TurboLibiGWN(Pd, max_depth=10, areas=Ad)
    tree.UpdateMassNormals(Nd, Ad)
    exact = tree.values_fp64(Qd, beta=1e30, sigma=0.0, screened=False).cpu().numpy()
    out = {"state": f"torus {len(P)} points, true normals, uniform areas; grid {res.tolist()}; "
                    f"error sample: {len(Q)} seeded grid points against the exact all-pairs FP64 sum",
           "beta": 2.0, "field_rms": float(np.sqrt(np.mean(exact ** 2)))}
    grid_out = torch.empty(ng, dtype=torch.float32, device=dev)
    terms = torch.zeros(1, dtype=torch.int64, device=dev)
    for order in (0, 1, 2):
        w = tree.TurboLibiGWNLaunch(Qd, beta=2.0, order=order).cpu().numpy().astype(np.float64)
        for _ in range(2):
            tree.grid(res, org[:3], float(org[3]), beta=2.0, sigma=0.0, screened=False, order=order, out=grid_out)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        terms.zero_()
        e0.record()
        for _ in range(3):
            tree.grid(res, org[:3], float(org[3]), beta=2.0, sigma=0.0, screened=False, order=order, out=grid_out,
                      terms=terms)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        out[f"order{order}"] = {
            "grid_ms": ms, "pair_terms": int(terms.item()) // 3,
            "pair_terms_per_s": int(terms.item()) / 3 / (ms * 1e-3),
            "err_vs_exact": {"rms": float(np.sqrt(np.mean((w - exact) ** 2))), "max": float(np.abs(w - exact).max())}}
    return out


def learned_report(a, lib, capi, turbo, torch, dev, *_):
    """Plain (Gauss map) vs learned start on the bench cloud, with FP64 and
    compensated-FP32 sums, beside the true normals as the start (the best any
    initialiser can do): orientation agreement of the initial leaf normals
    with the true normals, warm create time, and the RMS distance of each
    iteration's grid field to the plain method's field after all iterations
    (sign-matched: the orientation flips every iteration); iterations to 1e-4
    (the north-star criterion) and to 2e-3."""
    from dwg_b200 import datasets as D
    from dwg_b200.train_init import DEFAULT_WEIGHTS
    Praw, Ntrue = D.make(a.cfg["dataset"], seed=1000)
    P, _, _ = D.normalize(Praw)
    Pd = torch.from_numpy(np.ascontiguousarray(P, np.float32)).to(dev)
    flags = dict(grid_reso=a.grid, final_reso=a.grid, total_iter=a.iters, use_graph=1, precision=1)
    model = turbo.LearnedNormalInit(DEFAULT_WEIGHTS)
    ref = turbo.TurboDWG(Pd, None, **flags)
    ref.TurboScreenedDWGLaunch(a.iters)
    w_ref = torch.from_numpy(ref.get("field")).to(dev)
    leaves = torch.from_numpy(ref.get("leaf_pos")).to(dev)
    ref.close()
    nb = turbo.KnnIndex(Pd).query(leaves, 1).cpu().numpy()[:, 0]
    truth = Ntrue[nb]
    out = {"weights": os.path.relpath(DEFAULT_WEIGHTS, ROOT),
           "reference_field": f"plain start (Gauss map, FP64 sums) after {a.iters} iterations"}
    Nd = torch.from_numpy(np.ascontiguousarray(Ntrue, np.float32)).to(dev)
    runs = (("plain", None, None, 1), ("learned", model, None, 1), ("learned_compensated", model, None, 3),
            ("true_normals", None, Nd, 1))
    for name, m, nrm, prec in runs:
        f = dict(flags, precision=prec)
        create = []
        for rep in range(2):  # the second create is the warm one
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d = turbo.TurboDWG(Pd, None, init_model=m, **f) if nrm is None else \
                turbo.TurboDWG(Pd, nrm, **dict(f, in_normal=1))
            torch.cuda.synchronize()
            create.append((time.perf_counter() - t0) * 1e3)
            if rep == 0:
                d.close()
        n0 = d.get("leaf_nrm")
        rms, it_ms = [], []
        for _ in range(a.iters):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d.TurboScreenedDWGLaunch(1)
            torch.cuda.synchronize()
            it_ms.append((time.perf_counter() - t0) * 1e3)
            w = torch.from_numpy(d.get("field")).to(dev)
            rms.append(float(min(torch.sqrt(torch.mean((w - w_ref) ** 2)), torch.sqrt(torch.mean((w + w_ref) ** 2)))))
        d.close()
        t4 = next((t + 1 for t, e in enumerate(rms) if e <= 1e-4), None)
        out[name] = {"init_orientation_agreement": float(((n0 * truth).sum(1) > 0).mean()),
                     "create_ms_cold": create[0], "create_ms_warm": create[1],
                     "rms_to_reference_every_5th": [round(x, 6) for x in rms[::5]],
                     "rms_floor_last_5": round(float(min(rms[-5:])), 6),
                     "iters_to_1e-4": t4, "iters_to_2e-3": next((t + 1 for t, e in enumerate(rms) if e <= 2e-3), None),
                     "ms_to_1e-4": (create[1] + sum(it_ms[:t4])) if t4 else None}
    return out


def batched_report(a, lib, capi, turbo, torch, dev, *_):
    """The batched-clouds configuration: 64 clouds of log-uniform size in
    [2,000, 200,000] (spheres, tori, 3-superquadric unions, noise 0.001-0.01),
    per-cloud grid clamp(round(128 (n/2000)^(1/3)), 128, 256), 30 iterations,
    in one batch (one graph per iteration, one persistent launch for all grid
    sums) against the same clouds one by one; device time with CUDA events."""
    import ctypes as C
    from dwg_b200 import datasets as D
    cl = D.batch(64, 2000, 200000, seed=0)
    dev_pts, prms = [], []
    for c in cl:
        Pn, _, _ = D.normalize(c["points"])
        dev_pts.append(torch.from_numpy(np.ascontiguousarray(Pn, np.float32)).to(dev))
        prms.append(capi.default_params(grid_reso=c["grid_reso"], final_reso=c["grid_reso"], total_iter=a.iters,
                                        precision=a.precision))
    npts = sum(int(d.shape[0]) for d in dev_pts)
    ptrs = (C.c_void_p * len(dev_pts))(*[capi.ptr(d) for d in dev_pts])
    counts = (C.c_int * len(dev_pts))(*[int(d.shape[0]) for d in dev_pts])
    parr = (capi.Params * len(prms))(*prms)
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def batch_run():
        b = C.c_void_p()
        capi.check(lib.dwg_batch_create(ptrs, counts, len(dev_pts), parr, None, C.byref(b)))
        capi.check(lib.dwg_batch_iterate(b, a.iters))
        capi.check(lib.dwg_batch_finalize(b))
        lib.dwg_batch_destroy(b)

    def one_by_one():
        for d, prm in zip(dev_pts, prms):
            h = C.c_void_p()
            capi.check(lib.dwg_pipeline_create(capi.ptr(d), None, int(d.shape[0]), C.byref(prm), None, C.byref(h)))
            capi.check(lib.dwg_pipeline_iterate(h, a.iters))
            capi.check(lib.dwg_pipeline_finalize(h))
            lib.dwg_pipeline_destroy(h)

    batch_run()  # warm-up
    ms_b = timed(batch_run)
    ms_s = timed(one_by_one)
    big = int(np.argmax([int(d.shape[0]) for d in dev_pts]))
    r = capi.TuneResult()
    # tolerance 0: no less accurate than the reference's beta = 2.3
    capi.check(lib.dwg_autotune(capi.ptr(dev_pts[big]), int(dev_pts[big].shape[0]), C.byref(prms[big]), 0.0, 4096,
                                2, None, C.byref(r)))
    return {"clouds": len(dev_pts), "points": npts, "iterations": a.iters,
            "batched": {"ms": ms_b, "Mpts_per_s": npts / ms_b / 1e3},
            "one_by_one": {"ms": ms_s, "Mpts_per_s": npts / ms_s / 1e3},
            "autotune_largest_cloud": {"points": int(dev_pts[big].shape[0]), "beta": r.beta, "tile": r.tile,
                                       "rms_err": r.rms_err, "max_err": r.max_err, "grid_ms": r.grid_ms,
                                       "reference_setting_grid_ms": r.ref_ms, "reference_rms_err": r.ref_rms_err,
                                       "field_rms": r.field_rms,
                                       "criterion": "RMS error vs exact sums no larger than at beta 2.3"}}


def cudart_copy(torch, dst, src_ptr, nbytes):
    """device-to-device copy from a raw library pointer into a torch tensor"""
    src = _raw_tensor(torch, src_ptr, nbytes, dst.device)
    dst.view(torch.uint8).view(-1)[:nbytes].copy_(src)


def _raw_tensor(torch, ptr, nbytes, device):
    class _Arr:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}
    return torch.as_tensor(_Arr(), device=device)


# ----------------------------------------------------------- CPU baselines --
class CpuWindingPath:
    """The reference's CPU winding-number path, igl::fast_winding_number
    (deps/libigl/include/igl/fast_winding_number.cpp:134-324: Barnes-Hut
    over an octree, parallel over queries), restated in FP64 by the oracle
    because Eigen is absent, on the sources and queries of one reconstruction
    of the workload: the octree leaves with Gauss-map normals and the default
    areas, queried at the leaves and at every iteration-grid sample in each
    of the iterations, then at the points and the final grid.  The octree and
    the moments are built and timed; query time is measured on a seeded
    sample and scaled to the reconstruction's query count."""

    def __init__(self, a, P):
        import oracle
        self.o = oracle
        self.a = a
        self.P = P
        t0 = time.perf_counter()
        t1 = oracle.Octree(P, a.cfg["max_depth"])
        leaf = (t1.children[:, 0] == -1) & (t1.counts > 0)
        self.L = t1.centers[leaf].astype(np.float32)
        self.build_points_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        self.t2 = oracle.Octree(self.L, a.cfg["max_depth"])
        self.build_leaves_s = time.perf_counter() - t0
        self.N = oracle.gauss_map(self.L)
        self.A = np.full(len(self.L), 2e-6, np.float32)
        t0 = time.perf_counter()
        self.mom = self.t2.moments(self.L, self.N, self.A)
        self.moments_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        self.ho = self.t2.expansion(self.L, self.N, self.A, self.mom[0])
        self.expansion_s = time.perf_counter() - t0
        self.res, self.org, self.h = oracle.voxel_grid(P, 0.05, a.grid)
        self.ng = int(np.prod(self.res.astype(np.int64)))
        self.queries = a.iters * (len(self.L) + self.ng) + (len(P) + self.ng)

    def sample(self, n, seed):
        rng = np.random.default_rng(seed)
        # grid and leaf queries in the proportion a reconstruction asks them
        frac_leaf = (self.a.iters * len(self.L) + len(self.P)) / self.queries
        nl = int(round(n * frac_leaf))
        ng = n - nl
        # distinct samples while the grid has enough of them (a small grid
        # timed for seconds needs more queries than it has samples)
        sel = rng.choice(self.ng, ng, replace=ng > self.ng)
        x, y, z = sel % self.res[0], (sel // self.res[0]) % self.res[1], sel // (self.res[0] * self.res[1])
        Qg = (self.org[None, :] + np.stack([x, y, z], 1).astype(np.float32) * self.h).astype(np.float32)
        Ql = self.L[rng.choice(len(self.L), nl, replace=True)]
        return np.concatenate([Qg, Ql]).astype(np.float32)

    def time_queries(self, order, beta, target_s, seed=0):
        """Queries timed until about target_s seconds have been spent."""
        n, spent, nq, terms = 2000, 0.0, 0, 0
        while True:
            Q = self.sample(n, seed + nq)
            t0 = time.perf_counter()
            _, tt = self.t2.fwn(self.L, self.N, self.A, Q, order, beta=beta, moments=(*self.mom, self.ho))
            dt = time.perf_counter() - t0
            spent += dt
            nq += len(Q)
            terms += int(tt.sum())
            if spent >= target_s:
                break
            n = int(min(4_000_000, max(2000, len(Q) * max(1.5, (target_s - spent) / max(dt, 1e-3)))))
        return {"queries_timed": nq, "seconds": spent, "per_query_s": spent / nq, "pair_evals_per_s": terms / spent}

    def estimate(self, order, beta, target_s):
        q = self.time_queries(order, beta, target_s)
        setup = self.build_points_s + self.build_leaves_s + self.a.iters * (
            self.moments_s + (self.expansion_s if order else 0.0))
        est = setup + q["per_query_s"] * self.queries
        return dict(q, order=order, beta=beta, setup_s=setup, queries_per_reconstruction=self.queries,
                    seconds_per_reconstruction_est=est, value=len(self.P) / est / 1e6)


def cpu_baseline(a, P=None, target_s=12.0):
    """The CPU winding-number path on the box's host cores (see CpuWindingPath):
    value from order 0 with beta 2.3 (DWG's setting); libigl's default order 2
    with beta 2 beside it."""
    import oracle
    if P is None:
        P = make_cloud(a, 0)
    path = CpuWindingPath(a, P)
    dwg_setting = path.estimate(0, 2.3, target_s)
    igl_default = path.estimate(2, 2.0, target_s / 2)
    return {
        "value": dwg_setting["value"], "unit": "Mpts/s", "cores": oracle.NTHREADS, "nproc": os.cpu_count(),
        "kind": "port",
        "sample": (f"igl::fast_winding_number restated (oracle, FP64, {oracle.NTHREADS} threads): "
                   f"{dwg_setting['queries_timed']} seeded queries (grid and leaves in a reconstruction's "
                   f"proportion) timed in {dwg_setting['seconds']:.1f} s, scaled to the "
                   f"{path.queries:,} queries of one reconstruction ({a.iters} iterations x ({len(path.L)} "
                   f"leaves + {path.ng} grid) + final pass) plus octree/moment builds; MC and kNN not counted"),
        "extrapolated": True,
        "order0_beta2.3": dwg_setting, "order2_beta2": igl_default,
    }


def reference_gpu_run(a, P):
    """The reference's own GPU DWG (src/TurboDWG.cu and the operators it calls,
    compiled unchanged into oracle/_ref/libref_dwg.so) on the same cloud and
    flags, in a child process; device seconds of the iterations and the final
    pass, measured once.  None when the comparator is not built."""
    from oracle import ref_dwg
    if not ref_dwg.available():
        return {"unavailable": "oracle/_ref/libref_dwg.so not built (needs the reference checkout at build time)"}
    kw = dict(grid_reso=a.grid, final_reso=a.cfg["final_reso"], total_iter=a.iters, as_thres=1e-7,
              max_depth=a.cfg["max_depth"])
    t0 = time.perf_counter()
    r = ref_dwg.reconstruct_isolated(P, timeout=900, **kw)
    wall = time.perf_counter() - t0
    secs = r["secs"]
    dev_s = float(secs[0] + secs[1])
    return {"value": len(P) / dev_s / 1e6, "unit": "Mpts/s", "device_seconds": dev_s,
            "iterations_seconds": float(secs[0]), "final_pass_seconds": float(secs[1]),
            "wall_seconds_incl_host_preparation": wall, "triangles_final": int(len(r["tris"])),
            "flags": dict(kw, note="as_thres 1e-7: the default 0 launches AsFiltertoZero with zero blocks and "
                                   "the pending launch error ends the reference's run under CUDA 12.9 thrust"),
            "what": "TurboDWG constructor -> TurboScreenedDWGLaunch -> GenerateMesh (output mode 3), CUDA events "
                    "around the calls; the host preparation (octrees, moments, voxel grids) from the oracle"}


def run_reference(a, rank, world):
    if rank != 0:
        return None
    P = make_cloud(a, 0)
    path = CpuWindingPath(a, P)
    steps, step_s = [], []
    last = None
    for i in range(max(a.warmup, 0) + max(a.steps, 1)):
        t0 = time.perf_counter()
        last = path.estimate(0, 2.3, 4.0)
        el = time.perf_counter() - t0
        if i >= a.warmup:
            steps.append(last["value"])
            step_s.append(el)
    v = float(np.mean(steps))
    import oracle
    cb = {"value": v, "unit": "Mpts/s", "cores": oracle.NTHREADS, "nproc": os.cpu_count(), "kind": "port",
          "sample": (f"per step: igl::fast_winding_number restated (oracle, FP64, {oracle.NTHREADS} threads), "
                     f"order 0, beta 2.3, {last['queries_timed']} seeded queries timed in {last['seconds']:.1f} s and "
                     f"scaled to the {path.queries:,} queries of one reconstruction plus octree/moment builds"),
          "extrapolated": True}
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "Mpts/s",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": float(np.mean(step_s)) * 1e3,
        "ms_per_step_is": "measured seconds of a step's timed sample (the value is scaled to a reconstruction)",
        "seconds_per_reconstruction_est": last["seconds_per_reconstruction_est"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded procedural clouds; no dataset)",
        "config": dict(a.cfg, points=len(P), parallelism="CPU, all host threads"),
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("the reference's DWG_CUDA executable needs Eigen 3.3.7, PCL 1.10 and CGAL 5.6.1 (absent); its "
                 "CPU winding-number path (igl::fast_winding_number) is timed as the oracle's restatement"),
    }
    if not a.no_reference_gpu:
        try:
            out["reference_gpu"] = reference_gpu_run(a, P)
        except Exception as e:
            out["reference_gpu"] = {"error": f"{type(e).__name__}: {str(e)[-400:]}"}
    return out


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        out = run_reference(a, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_ours(a, rank, world, local_rank)
    if rank == 0 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(a)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
