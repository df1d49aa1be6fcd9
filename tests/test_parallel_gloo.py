"""Multi-rank host logic on CPU: two gloo ranks shard one window's groups, advect
their slices (with the CPU oracle standing in for the GPU kernel, which runs per
group and so cannot tell a slice from the whole), and gather the FTLE field.  The
gathered field must equal the unsharded run bit for bit, and the timing reduction
must return the max over ranks."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pyftle_b200 import flows, parallel


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    shape = (40, 20)
    pts = flows.grid_points_2d(*shape)
    snaps = flows.double_gyre_snapshots(pts, np.arange(6) * 0.05)
    pos = flows.seeds_2d(flows.centroid_grid_2d(23, 11, (0.1, 1.9), (0.1, 0.9)), 1e-3)
    return shape, pts, snaps, pos


def _rank_main(rank, world, port, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from oracle import oracle as O

    info = parallel.init("gloo", timeout_s=60)
    try:
        shape, pts, snaps, pos = _case()
        N = pos.shape[0] // 4
        mine = parallel.shard_positions(torch.from_numpy(pos), 2, info.rank, info.world)
        g0, g1 = parallel.group_range(N, info.rank, info.world)
        assert mine.shape[0] == 4 * (g1 - g0)
        gmin, gdel = O.grid_axes(pts, shape)
        _, f = O.run_window(snaps, shape, gmin, gdel, mine.numpy(), integrator="rk4",
                            snap_dt=0.05)
        full = parallel.gather_field(torch.from_numpy(f), N)
        t = parallel.max_over_ranks(1.5 + info.rank)
        out_q.put((info.rank, full.numpy(), t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from oracle import oracle as O

    shape, pts, snaps, pos = _case()
    gmin, gdel = O.grid_axes(pts, shape)
    _, ref = O.run_window(snaps, shape, gmin, gdel, pos, integrator="rk4", snap_dt=0.05)
    for rank, field, t in res:
        np.testing.assert_array_equal(field, ref)
        assert t == 2.5


@pytest.mark.parametrize("n,world", [(10, 3), (7, 7), (3, 4), (1000, 8)])
def test_group_ranges_partition(n, world):
    spans = [parallel.group_range(n, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
    assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1


def test_shard_unshard_roundtrip():
    pos = torch.arange(6 * 11 * 3, dtype=torch.float64).reshape(66, 3)
    parts = [parallel.shard_positions(pos, 3, r, 4) for r in range(4)]
    assert torch.equal(parallel.unshard_positions(parts, 3), pos)
    assert parallel.windows_of_rank(10, 1, 4) == [1, 5, 9]
