"""The host side of the z-slab sharded reconstruction, as two gloo ranks on
the CPU: the slab partition and the int64 sum that the ranks exchange."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))


def _slab_worker(rank, world, port):
    from dwg_b200 import turbo
    _init(rank, world, port)
    try:
        for samples in (3, 4, 17, 87, 256, 513):
            if samples - 1 < world:
                continue
            z0, nz = turbo.slab_range(samples, rank, world)
            got = [None] * world
            dist.all_gather_object(got, (z0, nz))
            # consecutive runs of cells that tile 0 .. samples-2, each with
            # its upper boundary sample; every run holds at least one cell
            assert got[0][0] == 0
            for r in range(world):
                assert got[r][1] >= 2
                if r + 1 < world:
                    assert got[r][0] + got[r][1] - 1 == got[r + 1][0]
            assert got[-1][0] + got[-1][1] == samples
    finally:
        dist.destroy_process_group()


def _sum_worker(rank, world, port):
    from dwg_b200 import turbo
    _init(rank, world, port)
    try:
        rng = np.random.default_rng(100 + rank)
        # fixed-point normal sums are large int64: the sum must be exact
        vals = rng.integers(-(1 << 60), 1 << 60, 1001, dtype=np.int64) // world
        t = torch.from_numpy(vals.copy())
        turbo.exchange_tensor(t)
        want = sum(np.random.default_rng(100 + r).integers(-(1 << 60), 1 << 60, 1001, dtype=np.int64) // world
                   for r in range(world))
        assert np.array_equal(t.numpy(), want)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_range_tiles_the_grid(world):
    mp.spawn(_slab_worker, args=(world, _free_port()), nprocs=world, join=True)


def test_exchange_sums_int64_exactly():
    mp.spawn(_sum_worker, args=(2, _free_port()), nprocs=2, join=True)


def test_slab_range_rejects_more_ranks_than_cells(dwg_lib):
    from dwg_b200 import capi, turbo
    with pytest.raises(capi.DwgError):
        turbo.slab_range(3, 0, 3)
