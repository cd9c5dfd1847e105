"""Multi-rank host logic of bench.py on CPU: world size 2 over gloo. Each rank
runs its own replica domain; the job rate is N x steps / (max over ranks of
the device time), and every rank takes the same collective steps."""
import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        elapsed = [1.0 + rank, 0.5 + 2 * rank]       # rank 1 is the slow one
        got = bench.max_over_ranks(elapsed, world)
        out[rank] = (got, bench.job_rate(world, 10, got[0]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_world_size_2():
    world = 2
    port = 29500 + os.getpid() % 1000
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for rank in range(world):
        got, rate = out[rank]
        assert got == [2.0, 2.5]
        assert rate == pytest.approx(world * 10 / 2.0)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks([3.0, 4.0], 1) == [3.0, 4.0]
    assert bench.job_rate(1, 20, 2.0) == 10.0


def test_issue_roofline_of_the_dominant_kernel():
    """The instruction-issue roofline: warp instructions of one launch over 148
    SMs x 4 schedulers x the clock give the floor time; frac = floor / measured."""
    import bench
    cells = 256 ** 3
    r = bench.issue_roofline(2.0, cells, 2, 1965.0)
    rate = 148 * 4 * 1965.0e6
    assert r['bound'] == 'issue' and r['peak_warp_instructions_per_s'] == rate
    assert abs(r['floor_ms'] - bench.MEASURED_WARP_INSTRUCTIONS[(256, 2)] / rate * 1e3) < 1e-12
    assert abs(r['frac'] - r['floor_ms'] / 2.0) < 1e-12
    assert bench.issue_roofline(2.0, 64 ** 3, 2, 1965.0) is None      # no capture of that size
    assert bench.issue_roofline(2.0, cells, 2, None) is None           # no clock sampled


def _replica_digest(rank, size=20, steps=2):
    """Rank ``rank``'s replica of the bench scene (seeded as bench.py seeds it),
    advanced ``steps`` steps by the CPU oracle, reduced to a few numbers."""
    import numpy as np
    import bench
    from fluxfx_b200.physics.emission import pack_sources
    from oracle import smoke as S
    from oracle import solver as O
    grid, s, colliders, emitters, noise = bench.scene(size, 'FP32', bench.replica_seed(0, rank),
                                                      **bench.VARIANTS['plain'])
    g = S.Grid(grid.shape, grid.extent, np.float32)
    mask = S.raster_mask(g, [(c.shape, c.inverse_rows) for c in colliders])
    ref = O.OracleSmoke(grid.shape, grid.extent, s, np.float32, mask=mask)
    zeros = np.zeros(grid.cells, np.float32)
    ref.upload(density=zeros, temperature=zeros, velocity=noise)
    table = (pack_sources(emitters), len(emitters))
    for _ in range(steps):
        ref.step(0.02, sources=table)
    d = np.asarray(ref.density, np.float64)
    return (float(d.sum()), float(d.max()), int(ref.projector.last_cycles),
            tuple(float(np.abs(np.asarray(f)).max()) for f in ref.velocity))


def _replica_worker(rank, world, port, out):
    import time
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        dist.barrier()
        t0 = time.perf_counter()
        digest = _replica_digest(rank)
        elapsed = time.perf_counter() - t0
        gathered = [None] * world
        dist.all_gather_object(gathered, digest)
        slowest = bench.max_over_ranks([elapsed], world)[0]
        out[rank] = (gathered, slowest, elapsed)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_domains_are_independent_world_size_2():
    """Two ranks each advance their own seeded domain (the oracle standing in
    for the device solver, which needs a GPU): each rank's result equals the
    same domain advanced alone in one process, the two domains differ, every
    rank sees the same gathered results, and the timing is the slowest rank's."""
    world = 2
    port = 29500 + (os.getpid() + 7) % 1000
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_replica_worker, args=(world, port, out), nprocs=world, join=True)
    alone = [_replica_digest(rank) for rank in range(world)]
    assert alone[0] != alone[1]
    for rank in range(world):
        gathered, slowest, elapsed = out[rank]
        assert gathered == alone
        assert slowest == max(out[r][2] for r in range(world))
