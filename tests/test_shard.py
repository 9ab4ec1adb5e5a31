"""Sharding over ranks on the CPU: the balanced partition; a world-size-2 gloo run in which
each rank steps its block of an uneven column batch with the oracle (no per-step collective,
one gather at the end) and must reproduce the single-process run exactly; and the same for
the bubble statistics of several level sets, each rank taking a block of the level sets."""
import os
import socket

import numpy as np
import pytest

from lica_boiling1d_b200 import shard


def test_partition_is_contiguous_balanced_and_complete():
    rng = np.random.default_rng(4)
    cells = rng.integers(128, 2049, 4096)
    for world in (1, 2, 3, 8):
        blocks = shard.partition(cells, world)
        assert blocks[0][0] == 0 and blocks[-1][1] == len(cells)
        assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
        sums = [int(cells[lo:hi].sum()) for lo, hi in blocks]
        assert max(sums) - min(sums) <= 2 * int(cells.max())
    assert shard.partition([5, 5], 4)[-1][1] == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _records(lo, hi, n, length, z0, props, steps):
    from oracle import oracle as O
    out = []
    for c in range(lo, hi):
        st = O.col_init(int(n[c]), float(length[c]), float(z0[c]), props[c])
        for _ in range(steps):
            assert O.col_step(st, int(n[c]), float(length[c]), props[c]) == 0
        out.append((c, st["scal"].tolist(), st["stats"].tolist(), float(st["t"].sum())))
    return out


def _worker(rank, world, port, case, steps, queue):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n, length, z0, props = case
    lo, hi = shard.partition(n, world)[rank]
    recs = shard.gather_histories(_records(lo, hi, n, length, z0, props, steps), world)
    if rank == 0:
        queue.put(recs)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_batch_matches_single_process():
    import torch.multiprocessing as mp
    from lica_boiling1d_b200.column import uneven_batch
    case = uneven_batch(5, seed=6, nmin=24, nmax=80)
    steps = 3
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, case, steps, queue)) for r in range(2)]
    for p in procs:
        p.start()
    got = queue.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n, length, z0, props = case
    ref = _records(0, len(n), n, length, z0, props, steps)
    assert got == ref


def _bubble_worker(rank, world, port, queue):
    import torch.distributed as dist
    from oracle import oracle as O
    from tests import bubble_cases as bc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    grid, psi, (u, v, w) = bc.three_bubbles(n1=24, n2=20, n3=28)
    lo, hi = shard.partition(np.ones(len(psi)), world)[rank]
    local = O.bubble_tracking(grid.as_dict(), psi[lo:hi], u, v, w, time=0.5, llvs0=1 + lo)
    recs = shard.gather_records(local, world)
    if rank == 0:
        queue.put(recs.tobytes())
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_bubble_statistics_match_single_process():
    import torch.multiprocessing as mp
    from oracle import oracle as O
    from tests import bubble_cases as bc
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bubble_worker, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    got = queue.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    grid, psi, (u, v, w) = bc.three_bubbles(n1=24, n2=20, n3=28)
    ref = O.bubble_tracking(grid.as_dict(), psi, u, v, w, time=0.5, llvs0=1)
    assert got == ref.tobytes()
