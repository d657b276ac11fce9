"""Whole-instance sharding of the batching and serving forms (CPU).

Independent instances are owned by one rank each and stepped there with no
exchange; these tests check the ownership rule (disjoint, complete, balanced,
the same on every rank without communication) and the host-side report
gather, with two spawned ranks over gloo at 127.0.0.1.
"""
import os
import socket
import sys
import multiprocessing as mp
from pathlib import Path
import numpy as np
from afsi_gpu_b200.sharding import instance_cost, owned, shard_instances, shard_requests, gather_reports
from afsi_gpu_b200.serving import mix

ROOT = Path(__file__).resolve().parents[1]


def _batch_costs(count=64, seed=0):
    """Cell and point counts of the seeded batching workload (its grids and
    leaflet point counts, without building the batch)."""
    rng = np.random.default_rng(seed)
    shapes = ((128, 32), (256, 64), (384, 96), (512, 128))
    costs = []
    for _ in range(count):
        nx, ny = shapes[int(rng.integers(len(shapes)))]
        pts = int(rng.integers(5000, 40001))
        rng.standard_normal((pts, 2))   # the forces drawn between (keeps the seeded sequence)
        rng.standard_normal((nx, ny))   # the pressure right-hand side
        costs.append(instance_cost(nx * ny, pts))
    return costs


def test_instance_shards_are_disjoint_complete_and_balanced():
    costs = _batch_costs()
    for world in (1, 2, 4, 8):
        owner = shard_instances(costs, world)
        parts = [owned(owner, r) for r in range(world)]
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs)  # LPT bound
        assert shard_instances(costs, world) == owner        # deterministic


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group('gloo', timeout=timedelta(seconds=60))
    reqs = mix(200, rate=2000., seed=5)
    mine = shard_requests(reqs, world, rank)
    owner = shard_instances(_batch_costs(), world)
    report = dict(requests=len(mine), wall_s=1.0 + rank, rids=[r.rid for r in mine],
                  instances=owned(owner, rank))
    combined = gather_reports(report, dist)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, combined))


def test_ranks_agree_on_ownership_without_exchange_and_gather_reports():
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    results = dict(out.get(timeout=10) for _ in range(2))
    a, b = results[0], results[1]
    assert a['ranks'] == b['ranks'] == 2 and a['requests'] == b['requests'] == 200
    assert a['wall_s'] == b['wall_s'] == 2.0              # the slowest rank's time
    r0, r1 = (set(r['rids']) for r in a['per_rank'])
    assert not r0 & r1 and r0 | r1 == set(range(200))     # disjoint, complete sub-streams
    i0, i1 = (set(r['instances']) for r in a['per_rank'])
    assert not i0 & i1 and i0 | i1 == set(range(64))
    assert a['per_rank'] == b['per_rank']
