"""Whole-instance sharding of the batching and serving forms over GPUs.

Independent FSI instances (the batching form's channel instances, the
serving form's requests) need no exchange between GPUs: each rank owns a
subset and steps it alone, so there is no data-path collective.  The
reference has no multi-GPU code; this module only decides ownership.

* ``instance_cost`` estimates one instance's step work from its cell and
  point counts (the V-cycles scale with the cells, the transfers with the
  points);
* ``shard_instances`` splits instances over ``world`` ranks by greedy
  longest-processing-time assignment (largest first, to the least-loaded
  rank; ties to the lower rank), a deterministic function of the costs, so
  every rank computes the same partition with no communication;
* ``shard_requests`` routes a request stream the same way, rank by rank in
  arrival order, so every rank serves a disjoint sub-stream.

``gather_reports`` combines per-rank reports on the host (a host-side
metric gather through ``torch.distributed`` objects), never on the data path.
"""
import heapq


def instance_cost(cells, points, *, cell_weight=1.0, point_weight=0.35):
    """Relative step work of one instance: cells for the V-cycles, points for
    the transfers (the weight ratio of the batch step's measured phases)."""
    return cell_weight * float(cells) + point_weight * float(points)


def shard_instances(costs, world):
    """Rank of every instance: greedy longest-processing-time over `world`
    ranks.  Returns a list of rank ids, one per instance."""
    if world < 1:
        raise ValueError('world size must be at least 1')
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [(0.0, r) for r in range(world)]
    heapq.heapify(loads)
    owner = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(loads)
        owner[i] = r
        heapq.heappush(loads, (load + costs[i], r))
    return owner


def owned(owner, rank):
    """Indices owned by `rank`, in their original order."""
    return [i for i, r in enumerate(owner) if r == rank]


def request_cost(req):
    cells = req.n ** 3 if req.kind == '3d' else req.n * (req.n // 4)
    return instance_cost(cells, req.points)


def shard_requests(requests, world, rank):
    """The sub-stream of `requests` rank `rank` serves: requests in arrival
    order, each to the rank with the least assigned work so far (ties to the
    lower rank) — deterministic, so the ranks agree without communication."""
    if not 0 <= rank < world:
        raise ValueError('rank outside the world')
    loads = [0.0] * world
    mine = []
    for req in sorted(requests):
        r = min(range(world), key=lambda k: (loads[k], k))
        loads[r] += request_cost(req)
        if r == rank:
            mine.append(req)
    return mine


def gather_reports(report, dist=None):
    """Per-rank reports combined on every rank: total requests and steps/s,
    the slowest rank's wall time, and the per-rank list."""
    reports = [report]
    if dist is not None and dist.is_initialized():
        reports = [None] * dist.get_world_size()
        dist.all_gather_object(reports, report)
    wall = max(r['wall_s'] for r in reports)
    total = sum(r['requests'] for r in reports)
    return dict(ranks=len(reports), requests=total, wall_s=wall, steps_per_s=total / wall, per_rank=reports)
