"""The multi-GPU path on the CPU: world size 2 over gloo.

The hot path does not shard (one grid per replica), so ``bench.py --gpus N``
runs N independent replicas: the ranks meet only at barriers and at the
max-over-ranks reduction of the timed region.  These tests run that host
logic in two spawned processes with the gloo backend: the rendezvous, the
reduction (the job's time is its slowest rank's, the same on every rank), the
whole-job rate, and the reference arm's rule that ranks other than 0 leave
without work.
"""
import argparse
import os
import socket
import sys
import multiprocessing as mp
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR='127.0.0.1',
                      MASTER_PORT=str(port))
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))


def _timing_worker(rank, world, port, out):
    _env(rank, world, port)
    import torch
    import bench
    args = argparse.Namespace(gpus=world, impl='reference', steps=4, warmup=3)
    dist, r, w = bench.dist_setup(args)
    elapsed = bench.max_over_ranks(1.0 + rank, dist, torch.device('cpu'))  # rank 1 is the slow one
    rate = bench.whole_job_rate(w, args.steps, elapsed)
    dist.barrier()
    dist.destroy_process_group()
    out.put((r, w, elapsed, rate))


def _reference_worker(rank, world, port, out):
    _env(rank, world, port)
    import bench
    args = argparse.Namespace(gpus=world, impl='reference', steps=1, warmup=0)
    if rank == 0:  # stands in for rank 0's reference run: join the group, leave
        dist, _, _ = bench.dist_setup(args)
        dist.destroy_process_group()
        out.put((rank, 'joined'))
    else:
        bench.run_reference(args)  # must return at once, with no work and no output
        out.put((rank, 'returned'))


def _run(target, world=2):
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0] * world, codes
    return sorted(out.get(timeout=10) for _ in range(world))


def test_replicas_time_is_the_slowest_rank_on_every_rank():
    results = _run(_timing_worker)
    assert [r[:2] for r in results] == [(0, 2), (1, 2)]
    for _, world, elapsed, rate in results:
        assert elapsed == 2.0  # max over ranks, seen by both
        assert rate == world * 4 / 2.0


def test_reference_arm_runs_on_rank_zero_only():
    results = _run(_reference_worker)
    assert results == [(0, 'joined'), (1, 'returned')]
