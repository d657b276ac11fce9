"""Serving form: a continuous-batching request loop over device-resident FSI
step states.

No counterpart in the reference (it steps one simulation in one process).
Step requests of different sizes arrive on a seeded Poisson schedule; each
names a kind (2D channel, or 3D closed box with a grid size), a point count
and a seed, and carries its inputs (points, point forces, pressure right-hand
side) as pinned host buffers made before the stream starts.  A step copies
its inputs to the device, runs prepare (binning and IB_4 weights) + spread of
the point forces + interpolation of the resident face velocity + a pressure
solve to 1e-10, and copies its interpolated velocity and pressure back.

The server:

* keeps resident state on the device between requests: per lane the face
  velocity and the multigrid workspaces with their captured graphs; for 2D
  batches, one batch engine per batch size with its transfer tables, face
  arrays and solver workspaces;
* admits requests in arrival order when the HBM they need (their points,
  tables and outputs) fits the budget beside the resident state;
* batches: the 2D lane takes every admitted 2D request that is waiting when
  it becomes free (up to ``batch``) and steps them together, one launch per
  transfer operation for all of them (``BatchedChannels``) and, in the
  precision form, their pressure solves as batched FP32 V-cycles inside
  batched FP64 refinement (``BatchedRefinement``); requests that arrive while
  a batch runs form the next one (continuous batching, no batch boundaries
  to wait for);
* overlaps: 3D requests run on ``slots`` lanes, each a worker thread with its
  own CUDA stream, beside the 2D lane, so the kernels of requests in flight
  overlap on the device;
* records per request the latency from arrival to completion (results on
  the host) and reports p50/p99 beside throughput.

``precision='fp64'`` solves every pressure with FP64 V-cycles (per request);
``precision='fp32-refined'`` with FP32 V-cycles inside FP64 iterative
refinement (batched for 2D), both to the FP64 tolerance.  A request's result
does not depend on what else is running beyond the order of atomic additions
in its spread and, in the batched refinement, the refinement count (every
instance of a batch is refined until all meet their tolerance), so results
alone and in the mix agree to the solve tolerance
(``tests/test_gpu_serving.py``).
"""
import heapq
import queue
import threading
import time
from collections import defaultdict
from dataclasses import dataclass, field
import numpy as np
import torch
from . import cuda_ib, synthetic
from .grid import ChannelGrid, MACGrid
from .multigrid import ChannelMultigrid, GeometricMultigrid, RefinedMultigrid


@dataclass(order=True)
class Request:
    arrival: float                    # seconds from the start of the stream
    rid: int = field(compare=False)
    kind: str = field(compare=False)  # '2d' or '3d'
    n: int = field(compare=False)     # cells per axis (3D) or x cells (2D, ny = n/4)
    points: int = field(compare=False)
    seed: int = field(compare=False)
    inputs: dict = field(compare=False, default=None, repr=False)


def shell_points(count, seed, *, center=(.5, .5, .5), semi=(.3, .2, .2), jitter=.01):
    """Points on a prolate spheroid shell (long axis x), seeded."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((count, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    r = 1 + jitter * rng.uniform(-1, 1, (count, 1))
    return np.asarray(center) + v * np.asarray(semi) * r


def grid_of(kind, n):
    return ChannelGrid((n, n // 4), (4., 1.)) if kind == '2d' else MACGrid((n, n, n), (1., 1., 1.))


def make_inputs(req, *, pin=True):
    """The request's inputs as host tensors (pinned by default): points,
    N(0,1) point forces and a mean-free N(0,1) pressure right-hand side."""
    rng = np.random.default_rng(req.seed)
    g = grid_of(req.kind, req.n)
    if req.kind == '2d':
        pts = synthetic.ellipse_points(req.points, center=(2., .5), semi=(1.2, .3), spacing=g.spacing[0],
                                       seed=req.seed)
        force = rng.standard_normal((req.points, 2))
    else:
        pts = shell_points(req.points, req.seed)
        force = rng.standard_normal((req.points, 3))
    r = rng.standard_normal(g.shape)
    out = dict(points=torch.as_tensor(pts), force=torch.as_tensor(force), rhs=torch.as_tensor(r - r.mean()))
    return {k: v.pin_memory() for k, v in out.items()} if pin else out


def with_inputs(requests, *, pin=True):
    """The requests with their inputs made (outside any timed region)."""
    return [Request(r.arrival, r.rid, r.kind, r.n, r.points, r.seed, make_inputs(r, pin=pin)) for r in requests]


def mix(count, *, rate=2000., seed=0, scale=1.):
    """The serving mix: 50% 2D 256x64 with 20k points; 35% 3D 32^3-64^3 with
    50k-400k points; 15% 3D 96^3 with 800k points; Poisson arrivals at `rate`
    per second.  `scale` shrinks the point counts (tests).  Requests carry no
    inputs yet (``with_inputs``)."""
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


def request_bytes(req):
    """HBM a request holds while it runs: its points, forces, stencil tables
    (FP64), gathered velocity and spread fields."""
    if req.kind == '2d':
        return req.points * (16 + 16 + 2 * 16 * 16 + 16) + 2 * (req.n + 1) * (req.n // 4 + 1) * 8
    return req.points * (24 + 24 + 3 * 3 * 8 + 3 * 12 * 8 + 24) + 3 * (req.n + 1) ** 3 * 8


def _pinned_like(t):
    return torch.empty(t.shape, dtype=t.dtype, pin_memory=True)


class Lane3D:
    """Resident states of one 3D worker lane: per grid size the face velocity
    and the pressure solver (FP64, or FP32 V-cycles in FP64 refinement)."""

    def __init__(self, device, precision):
        self.device, self.precision = device, precision
        self.stream = torch.cuda.Stream(device=device)
        self.states = {}
        self.bytes = 0

    def state(self, n):
        if n not in self.states:
            g = grid_of('3d', n)
            mg = (GeometricMultigrid(g, device=self.device, backend='b200-graph') if self.precision == 'fp64' else
                  RefinedMultigrid(g, device=self.device))
            vel = tuple(v.to(self.device) for v in synthetic.fourier_velocity3d(g, seed=n))
            ws = mg.workspace if hasattr(mg, 'workspace') else mg.inner.workspace
            self.states[n] = (g, mg, vel)
            self.bytes += ws.allocated_bytes + sum(v.numel() * 8 for v in vel)
        return self.states[n]

    def step(self, req):
        g, mg, vel = self.state(req.n)
        inp = req.inputs
        x = inp['points'].to(self.device, non_blocking=True)
        force = inp['force'].to(self.device, non_blocking=True)
        rhs = inp['rhs'].to(self.device, non_blocking=True)
        st = cuda_ib.compact_prepare(g, x)
        fields = cuda_ib.compact_spread(g, force, st)
        gathered = cuda_ib.compact_gather(g, vel, st)
        p, info = mg.solve(rhs)
        out = dict(velocity=_pinned_like(gathered), pressure=_pinned_like(p))
        out['velocity'].copy_(gathered, non_blocking=True)
        out['pressure'].copy_(p, non_blocking=True)
        return dict(out, fields=fields, cycles=info['cycles'])


class Batch2D:
    """Batch engines for 2D requests of one (grid, point count): one
    ``BatchedChannels`` per batch size 1..capacity, built once with resident
    face velocities; a batch copies its requests' inputs into the engine's
    input arrays and replays its graphs."""

    def __init__(self, n, points, capacity, device, precision):
        from .batch import BatchedChannels, Schedule
        self.n, self.points, self.device, self.precision = n, points, device, precision
        g = grid_of('2d', n)
        self.grid = g
        warm = make_inputs(Request(0., -1, '2d', n, points, 1), pin=False)
        vel = tuple(v.numpy() for v in synthetic.fourier_velocity2d(g, seed=n))
        self.engines = {}
        self.bytes = 0
        for k in range(1, capacity + 1):
            b = BatchedChannels([g] * k, [warm['points'].numpy()] * k, [warm['force'].numpy()] * k, [vel] * k,
                                [warm['rhs'].numpy()] * k, device=device, transfer_dtype=torch.float64,
                                schedule=Schedule(streams=1, order='given', smoother='jacobi', cycles=5,
                                                  vcycles='batched', refined=True))
            if precision == 'fp64':
                # batched transfers, then one FP64 solve per request
                b.plain = [ChannelMultigrid(g, device=device, backend='b200-graph') for _ in range(k)]
                b.transfers(torch.cuda.current_stream(device))
            else:
                b.use(b.schedule)
                b.replay()
            self.engines[k] = b
            self.bytes += (b.x.numel() + b.force.numel() + b.u.numel() + b.v.numel() + b.u_in.numel() +
                           b.v_in.numel() + b.gathered.numel()) * 8 + b.ids.numel() * 16
        torch.cuda.synchronize(device)

    def run(self, reqs):
        b = self.engines[len(reqs)]
        P = self.points
        for i, r in enumerate(reqs):
            b.x[i * P:(i + 1) * P].copy_(r.inputs['points'], non_blocking=True)
            b.force[i * P:(i + 1) * P].copy_(r.inputs['force'], non_blocking=True)
            if self.precision != 'fp64':
                b.refinement().rhs(i).copy_(r.inputs['rhs'], non_blocking=True)
        if self.precision == 'fp64':
            b.transfers(torch.cuda.current_stream(self.device))
        else:
            b.replay()
        outs = []
        for i, r in enumerate(reqs):
            if self.precision == 'fp64':
                p, info = b.plain[i].solve(r.inputs['rhs'].to(self.device, non_blocking=True))
                cycles = info['cycles']
            else:
                p, cycles = b.pressure(i), None
            vel = b.velocities(i)
            out = dict(velocity=_pinned_like(vel), pressure=_pinned_like(p), cycles=cycles,
                       fields=tuple(f.clone() for f in b.fields(i)))
            out['velocity'].copy_(vel, non_blocking=True)
            out['pressure'].copy_(p, non_blocking=True)
            outs.append(out)
        return outs, b


class Server:
    """Continuous-batching request loop: one 2D batch lane and `slots` 3D
    lanes, each a worker thread with its own CUDA stream."""

    def __init__(self, *, device='cuda', slots=4, batch=8, budget_bytes=150 * 10 ** 9, keep_results=False,
                 precision='fp64'):
        self.device = torch.device(device)
        if self.device.type != 'cuda':
            raise ValueError('the serving form requires a CUDA device; there is no CPU fallback')
        if precision not in ('fp64', 'fp32-refined'):
            raise ValueError("precision must be 'fp64' or 'fp32-refined'")
        if slots < 1 or batch < 1:
            raise ValueError('at least one 3D lane and a batch of at least one')
        self.slots, self.batch, self.budget = slots, batch, budget_bytes
        self.keep_results, self.precision = keep_results, precision
        self.lanes = [Lane3D(self.device, precision) for _ in range(slots)]
        self.batches = {}   # (n, points) -> Batch2D
        self.stream2d = torch.cuda.Stream(device=self.device)

    @property
    def resident(self):
        return sum(l.bytes for l in self.lanes) + sum(b.bytes for b in self.batches.values())

    def warm(self, requests):
        """Build every resident state the stream will need before serving
        (graph capture must not overlap running work)."""
        for r in requests:
            if r.kind == '2d':
                key = (r.n, r.points)
                if key not in self.batches:
                    self.batches[key] = Batch2D(r.n, r.points, self.batch, self.device, self.precision)
            else:
                for lane in self.lanes:
                    lane.state(r.n)
        torch.cuda.synchronize(self.device)
        if self.resident > self.budget:
            raise MemoryError('resident states exceed the HBM budget')

    def _finish(self, stream, outs):
        stream.synchronize()
        return outs

    def serve(self, requests):
        """Serve `requests` (arrival times relative to now; inputs made here
        if missing, before the clock starts).  Returns (report, results by
        request id if keep_results)."""
        requests = [r if r.inputs is not None else with_inputs([r])[0] for r in requests]
        self.warm(requests)
        pending = list(requests)
        heapq.heapify(pending)
        cond = threading.Condition()
        in_use = [0]
        peak = [0]
        done, results, errors, batches = [], {}, [], []
        q2d, q3d = [], queue.Queue()
        finished = threading.Event()
        t0 = time.perf_counter()

        def release(reqs, outs):
            now = time.perf_counter() - t0
            with cond:
                for r, out in zip(reqs, outs):
                    done.append((r, now))
                    if self.keep_results:
                        results[r.rid] = out
                    in_use[0] -= request_bytes(r)
                cond.notify_all()

        def lane2d():
            while True:
                with cond:
                    while not q2d and not finished.is_set():
                        cond.wait()
                    if not q2d:
                        return
                    first = q2d[0]
                    take = [r for r in q2d if (r.n, r.points) == (first.n, first.points)][:self.batch]
                    for r in take:
                        q2d.remove(r)
                try:
                    with torch.cuda.device(self.device), torch.cuda.stream(self.stream2d):
                        outs, b = self.batches[(first.n, first.points)].run(take)
                        self.stream2d.synchronize()
                        b.check()
                    batches.append(len(take))
                    release(take, outs)
                except Exception as exc:  # reported after the loop
                    errors.append((first.rid, repr(exc)))
                    release(take, [None] * len(take))

        def lane3d(lane):
            while True:
                r = q3d.get()
                if r is None:
                    return
                try:
                    with torch.cuda.device(self.device), torch.cuda.stream(lane.stream):
                        out = lane.step(r)
                        lane.stream.synchronize()
                    release([r], [out])
                except Exception as exc:
                    errors.append((r.rid, repr(exc)))
                    release([r], [None])

        threads = [threading.Thread(target=lane2d, daemon=True)] + \
            [threading.Thread(target=lane3d, args=(lane,), daemon=True) for lane in self.lanes]
        for th in threads:
            th.start()
        resident = self.resident
        try:
            while pending:
                req = pending[0]
                now = time.perf_counter() - t0
                if req.arrival > now:
                    time.sleep(min(req.arrival - now, .001))
                    continue
                need = request_bytes(req)
                heapq.heappop(pending)
                if need + resident > self.budget:
                    errors.append((req.rid, 'request larger than the HBM budget'))
                    continue
                with cond:
                    while in_use[0] + need + resident > self.budget:
                        cond.wait()
                    in_use[0] += need
                    peak[0] = max(peak[0], in_use[0])
                    if req.kind == '2d':
                        q2d.append(req)
                        cond.notify_all()
                if req.kind != '2d':
                    q3d.put(req)
        finally:
            with cond:
                finished.set()
                cond.notify_all()
            for _ in self.lanes:
                q3d.put(None)
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
                      slots=self.slots, batch=self.batch, precision=self.precision, resident_bytes=resident,
                      budget_bytes=self.budget, peak_request_bytes=peak[0],
                      batches_2d=dict(count=len(batches), mean_size=float(np.mean(batches)) if batches else 0.,
                                      max_size=max(batches) if batches else 0),
                      h2d_bytes=int(sum(sum(v.numel() * v.element_size() for v in r.inputs.values())
                                        for r in requests)),
                      by_kind={k: dict(count=len(v), p50_ms=float(np.percentile(v, 50)),
                                       p99_ms=float(np.percentile(v, 99))) for k, v in sorted(by_kind.items())})
        return report, results

    def alone(self, req):
        """The request's result with nothing else running (a batch of one for 2D)."""
        req = req if req.inputs is not None else with_inputs([req])[0]
        self.warm([req])
        with torch.cuda.device(self.device):
            if req.kind == '2d':
                with torch.cuda.stream(self.stream2d):
                    outs, b = self.batches[(req.n, req.points)].run([req])
                    self.stream2d.synchronize()
                return outs[0]
            lane = self.lanes[0]
            with torch.cuda.stream(lane.stream):
                out = lane.step(req)
                lane.stream.synchronize()
            return out
