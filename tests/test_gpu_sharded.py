"""Z-slab sharded reconstruction: two ranks (processes) on the one GPU of
the test, exchanging through gloo on the host -- no kernel waits on another
rank.  Every rank must end with the leaf normals, iso values and triangle
counts of the one-GPU run, bit for bit, and the ranks' meshes concatenated in
rank order must be the one-GPU mesh."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

from dwg_b200 import datasets as D  # noqa: E402

pytestmark = pytest.mark.gpu

FLAGS = dict(grid_reso=48, final_reso=48, total_iter=4, max_depth=7)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cloud():
    P, _ = D.torus(6000, seed=31)
    Pn, _, _ = D.normalize(P)
    return np.ascontiguousarray(Pn, np.float32)


def _rank(rank, world, port, out_dir, flags):
    import datetime

    import torch.distributed as dist

    from dwg_b200 import turbo
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        ex = turbo.torch_exchange()
        r = turbo.reconstruct_sharded(torch.from_numpy(_cloud()).cuda(), rank, world, ex, **flags)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), **r)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_equals_one_gpu(tmp_path, world):
    from dwg_b200 import turbo
    one = turbo.reconstruct(torch.from_numpy(_cloud()).cuda(), **FLAGS)
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path), FLAGS)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    parts = [dict(np.load(tmp_path / f"rank{r}.npz")) for r in range(world)]
    for r in parts:
        assert np.array_equal(r["leaf_nrm"], one["leaf_nrm"])
        assert np.array_equal(r["iso"], one["iso"])
        assert np.array_equal(r["tri_count"], one["tri_count"])
        assert np.array_equal(r["zero_count"], one["zero_count"])
        assert np.array_equal(r["point_nrm"], one["point_nrm"])
        assert float(r["final_iso"][0]) == float(np.ravel(one["final_iso"])[0])
    # slabs tile the final grid; meshes concatenate to the one-GPU mesh
    fz = [tuple(r["slab"][2:]) for r in parts]
    assert fz[0][0] == 0 and fz[-1][0] + fz[-1][1] == int(one["final_res"][2])
    tris = np.concatenate([r["tris"] for r in parts])
    assert np.array_equal(tris, one["tris"])
