"""Serving form: a request loop over device-resident FSI step states.

No counterpart in the reference (it steps one simulation in one process).
Step requests of different sizes arrive on a seeded Poisson schedule; each
names a kind (2D channel, or 3D closed box with a grid size), a point count
and a seed.  The server

* keeps one resident state per (kind, grid) and worker slot: the multigrid
  workspace with its captured graphs, the face-velocity field and the
  pressure right-hand side stay on the device between requests;
* admits a request when a worker slot is free and the HBM it needs (the
  point tables and outputs of the request, plus the resident state if that
  has to be built) fits in the budget, in arrival order;
* runs admitted requests on per-slot CUDA streams from worker threads, so the
  kernels of requests that arrived while others were running overlap on the
  device (continuous batching: a request enters as soon as a slot and the
  memory free up, not at batch boundaries);
* records per request the latency from arrival to completion, and reports
  p50/p99 latency beside throughput.

A step is prepare (binning and IB_4 weights) + spread of seeded N(0,1) point
forces + interpolation of the resident face velocity + a pressure multigrid
solve to 1e-10 (FP64).  Each result depends only on its request, not on what
else is running; ``tests/test_gpu_serving.py`` checks that a request's result
is the same alone and in the mix.
"""
import heapq
import threading
import time
from collections import defaultdict
from dataclasses import dataclass, field
import numpy as np
import torch
from . import cuda_ib, synthetic
from .grid import ChannelGrid, MACGrid
from .multigrid import ChannelMultigrid, GeometricMultigrid


@dataclass(order=True)
class Request:
    arrival: float                    # seconds from the start of the stream
    rid: int = field(compare=False)
    kind: str = field(compare=False)  # '2d' or '3d'
    n: int = field(compare=False)     # cells per axis (3D) or x cells (2D, ny = n/4)
    points: int = field(compare=False)
    seed: int = field(compare=False)


def shell_points(count, seed, *, center=(.5, .5, .5), semi=(.3, .2, .2), jitter=.01):
    """Points on a prolate spheroid shell (long axis x), seeded."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((count, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    r = 1 + jitter * rng.uniform(-1, 1, (count, 1))
    return np.asarray(center) + v * np.asarray(semi) * r


def mix(count, *, rate=2000., seed=0, scale=1.):
    """The serving mix: 50% 2D 256x64 with 20k points; 35% 3D 32^3-64^3 with
    50k-400k points; 15% 3D 96^3 with 800k points; Poisson arrivals at `rate`
    per second.  `scale` shrinks the point counts (tests)."""
    rng = np.random.default_rng(seed)
    t, out = 0., []
    for i in range(count):
        t += rng.exponential(1. / rate)
        u = rng.uniform()
        if u < .5:
            kind, n, pts = '2d', 256, 20000
        elif u < .85:
            kind, n, pts = '3d', int(rng.choice((32, 48, 64))), int(rng.integers(50000, 400001))
        else:
            kind, n, pts = '3d', 96, 800000
        out.append(Request(t, i, kind, n, max(1000, int(pts * scale)), int(rng.integers(1 << 30))))
    return out


class ResidentState:
    """Device-resident state of one (kind, grid) in one worker slot."""

    def __init__(self, kind, n, device):
        self.kind, self.n = kind, n
        if kind == '2d':
            self.grid = ChannelGrid((n, n // 4), (4., 1.))
            self.mg = ChannelMultigrid(self.grid, device=device, backend='b200-graph')
            vel = synthetic.fourier_velocity2d(self.grid, seed=n)
        else:
            self.grid = MACGrid((n, n, n), (1., 1., 1.))
            self.mg = GeometricMultigrid(self.grid, device=device, backend='b200-graph')
            vel = synthetic.fourier_velocity3d(self.grid, seed=n)
        self.velocity = tuple(v.to(device) for v in vel)
        self.bytes = self.mg.workspace.allocated_bytes + sum(v.numel() * 8 for v in self.velocity)

    def step(self, req, device):
        rng = np.random.default_rng(req.seed)
        if self.kind == '2d':
            hx, hy = self.grid.spacing
            pts = synthetic.ellipse_points(req.points, center=(2., .5), semi=(1.2, .3), spacing=hx,
                                           seed=req.seed)
            x = torch.as_tensor(pts, device=device)
            force = torch.as_tensor(rng.standard_normal((req.points, 2)), device=device)
            st = cuda_ib.prepare2d(self.grid, x)
            fields = cuda_ib.spread2d(self.grid, force, st)
            gathered = cuda_ib.gather2d(self.velocity, st)
        else:
            x = torch.as_tensor(shell_points(req.points, req.seed), device=device)
            force = torch.as_tensor(rng.standard_normal((req.points, 3)), device=device)
            st = cuda_ib.compact_prepare(self.grid, x)
            fields = cuda_ib.compact_spread(self.grid, force, st)
            gathered = cuda_ib.compact_gather(self.grid, self.velocity, st)
        r = rng.standard_normal(self.grid.shape)
        rhs = torch.as_tensor(r - r.mean(), device=device)
        p, info = self.mg.solve(rhs)
        return dict(fields=fields, velocity=gathered, pressure=p, cycles=info['cycles'])


def request_bytes(req):
    """HBM a request holds while it runs: its points, forces, stencil tables
    (FP64), gathered velocity and spread fields."""
    if req.kind == '2d':
        return req.points * (16 + 16 + 2 * 16 * 16 + 16) + 2 * (req.n + 1) * (req.n // 4 + 1) * 8
    return req.points * (24 + 24 + 3 * 3 * 8 + 3 * 12 * 8 + 24) + 3 * (req.n + 1) ** 3 * 8


class Server:
    """Continuous-batching request loop over `slots` worker threads."""

    def __init__(self, *, device='cuda', slots=4, budget_bytes=150 * 10 ** 9, keep_results=False):
        self.device = torch.device(device)
        if self.device.type != 'cuda':
            raise ValueError('the serving form requires a CUDA device; there is no CPU fallback')
        self.slots, self.budget = slots, budget_bytes
        self.keep_results = keep_results
        self.states = [dict() for _ in range(slots)]   # per slot: (kind, n) -> ResidentState
        self.resident = 0
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(slots)]

    def warm(self, requests):
        """Build the resident states the stream will need, in every slot,
        before serving (graph capture must not overlap running work)."""
        keys = sorted({(r.kind, r.n) for r in requests})
        for s in range(self.slots):
            for k in keys:
                if k not in self.states[s]:
                    st = ResidentState(*k, self.device)
                    if self.resident + st.bytes > self.budget:
                        raise MemoryError('resident states exceed the HBM budget')
                    self.states[s][k] = st
                    self.resident += st.bytes
        torch.cuda.synchronize(self.device)

    def run_one(self, req, slot):
        with torch.cuda.device(self.device), torch.cuda.stream(self.streams[slot]):
            out = self.states[slot][(req.kind, req.n)].step(req, self.device)
            self.streams[slot].synchronize()
        return out

    def serve(self, requests):
        """Serve `requests` (arrival times relative to now).  Returns
        (report, results by request id if keep_results)."""
        self.warm(requests)
        pending = list(requests)
        heapq.heapify(pending)
        lock = threading.Condition()
        free = list(range(self.slots))
        in_use = [0]
        peak = [0]
        done, results, errors = [], {}, []
        t0 = time.perf_counter()

        def worker(req, slot, need):
            try:
                out = self.run_one(req, slot)
                finish = time.perf_counter() - t0
                if self.keep_results:
                    results[req.rid] = {k: (tuple(t.clone() for t in v) if isinstance(v, tuple) else
                                            v.clone() if torch.is_tensor(v) else v) for k, v in out.items()}
                done.append((req, finish))
            except Exception as exc:  # reported after the loop
                errors.append((req.rid, repr(exc)))
            finally:
                with lock:
                    free.append(slot)
                    in_use[0] -= need
                    lock.notify_all()

        threads = []
        while pending:
            req = pending[0]
            now = time.perf_counter() - t0
            if req.arrival > now:
                time.sleep(min(req.arrival - now, .001))
                continue
            need = request_bytes(req)
            if need + self.resident > self.budget:
                heapq.heappop(pending)
                errors.append((req.rid, 'request larger than the HBM budget'))
                continue
            with lock:
                while not free or in_use[0] + need + self.resident > self.budget:
                    lock.wait()
                slot = free.pop()
                in_use[0] += need
                peak[0] = max(peak[0], in_use[0])
            heapq.heappop(pending)
            th = threading.Thread(target=worker, args=(req, slot, need), daemon=True)
            th.start()
            threads.append(th)
        for th in threads:
            th.join()
        wall = time.perf_counter() - t0
        if errors:
            raise RuntimeError(f'{len(errors)} requests failed, first: {errors[0]}')
        lat = np.array([finish - req.arrival for req, finish in done]) * 1e3
        by_kind = defaultdict(list)
        for req, finish in done:
            by_kind[f'{req.kind}-{req.n}'].append((finish - req.arrival) * 1e3)
        report = dict(requests=len(done), wall_s=wall, steps_per_s=len(done) / wall,
                      p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                      slots=self.slots, resident_bytes=self.resident, budget_bytes=self.budget,
                      peak_request_bytes=peak[0],
                      by_kind={k: dict(count=len(v), p50_ms=float(np.percentile(v, 50)),
                                       p99_ms=float(np.percentile(v, 99))) for k, v in sorted(by_kind.items())})
        return report, results

    def alone(self, req):
        """The request's result with nothing else running (slot 0)."""
        self.warm([req])
        return self.run_one(req, 0)
