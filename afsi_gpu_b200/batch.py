"""Batching form: many independent 2D channel instances stepped together.

No counterpart in the reference, which builds one ``TriangleTransfer``
(``mac2d/transfer.py:19-127``) and one ``ChannelMultigrid``
(``mac2d/multigrid.py:16-134``) per instance and steps instances one at a
time.  Here a batch of instances with uneven grids and point counts is one
step:

* one launch each for the prepare, the spread and the gather of every
  instance (``afsi_b200_batch2d_*``): points of all instances back to back,
  face arrays back to back, batch-global stencil ids; positions and bases in
  FP64, weights and transfers in ``transfer_dtype`` (FP32 in the precision
  form);
* a fixed number of V-cycles per instance on its own FP32 workspace (FP64
  coarsest solve), either batched (``vcycles='batched'``, Jacobi: one launch
  per level operation for all instances and one launch for all their
  single-CTA coarse levels, ``afsi_b200_mg_batch_vcycles``), the same in one
  persistent cooperative launch (``vcycles='persistent'``,
  ``afsi_b200_mg_batch_persistent``), or per instance with the instances
  spread over ``streams`` capture streams so that their small level kernels
  overlap on the device;
* the whole step captured once as a CUDA graph and replayed;
* or, at the FP64 solve tolerance (``Schedule(refined=True)``): the pressure
  kept in FP64 per instance, and batched FP32 V-cycles inside batched FP64
  iterative refinement until every instance's FP64 residual meets
  max(atol, rtol ||b||) (``BatchedRefinement``); the refinement loop runs on the
  device as one graph with a WHILE node.

``autotune()`` chooses the schedule (batched or per-instance V-cycles, stream
count, instance order, smoother with the cycle count that reaches the
requested FP32 residual reduction on every instance) by measuring graph
replays, and keeps the fastest.
"""
import ctypes
from dataclasses import dataclass
import numpy as np
import torch
from . import _lib
from ._lib import call, ptr, dtype_code
from .grid import ChannelGrid
from .multigrid import ChannelMultigrid, MGOptions

# afsi_batch2d_instance (include/afsi_b200.h)
INSTANCE_DTYPE = np.dtype([('nx', '<i8'), ('ny', '<i8'), ('hx', '<f8'), ('hy', '<f8'), ('lx', '<f8'),
                           ('ly', '<f8'), ('point_offset', '<i8'), ('point_count', '<i8'), ('u_offset', '<i8'),
                           ('v_offset', '<i8')])


def leaflet_points(grid, count, seed, dtype=np.float64):
    """Two open leaflets, one hinged on each wall, as strips of points: a
    stand-in for the quadrature points of two P2 triangle strips."""
    rng = np.random.default_rng(seed)
    Lx, Ly = grid.lengths
    hx, hy = grid.spacing
    out = []
    for k, n in enumerate((count // 2, count - count // 2)):
        s = rng.uniform(0., 1., n)                # position along the leaflet
        t = rng.uniform(-.25, .25, n) * hx        # across the strip
        x0 = Lx * (.35 + .1 * k)
        y = (.02 + .4 * s) * Ly if k == 0 else (.98 - .4 * s) * Ly
        x = x0 + .08 * Lx * s * s + t
        out.append(np.stack((x, y), -1))
    return np.concatenate(out).astype(dtype)


@dataclass
class Schedule:
    streams: int = 4
    order: str = 'largest-first'
    smoother: str = 'jacobi'
    cycles: int = 6
    vcycles: str = 'streams'   # 'streams' (per instance over side streams), 'batched' or 'persistent' (Jacobi)
    refined: bool = False      # FP64 refinement to the solve tolerance; `cycles` V-cycles per refinement


class BatchedVCycles:
    """Jacobi V-cycles of many channel solvers advanced together
    (``afsi_b200_mg_batch_vcycles``): per cycle one launch per level operation
    and depth for all instances, one launch for all single-CTA coarse levels.
    Each solver's iterates are bitwise those of its own ``advance``.  `sources`
    (one right-hand side per solver, optional) are copied into the solvers'
    finest right-hand sides when a run starts."""

    def __init__(self, solvers, sources=None):
        if not solvers:
            raise ValueError('no solvers')
        lib = _lib.load()
        self.solvers = list(solvers)
        self.count = len(self.solvers)
        device = self.solvers[0].workspace.p[0].device
        if any(mg.workspace.p[0].device != device for mg in self.solvers):
            raise ValueError('batched V-cycles need every solver on one device')
        plans = [mg.workspace.plan for mg in self.solvers]
        self._plans = (ctypes.POINTER(_lib.MGPlan) * self.count)(*[ctypes.pointer(p) for p in plans])
        self._sources = None
        if sources is not None:
            if len(sources) != self.count:
                raise ValueError('one right-hand side per solver')
            for mg, r in zip(self.solvers, sources):
                w = mg.workspace.rhs[0]
                if r.shape != w.shape or r.dtype != w.dtype or r.device != w.device or not r.is_contiguous():
                    raise ValueError("each source must be a contiguous tensor like its solver's right-hand side")
            self._keep = list(sources)
            self._sources = (ctypes.c_void_p * self.count)(*[ptr(r) for r in sources])
        nbytes = lib.afsi_b200_mg_batch_table_bytes(self._plans, self.count)
        if nbytes < 0:
            raise ValueError(f'batched V-cycles: {lib.afsi_b200_last_error().decode(errors="replace")}')
        host = np.zeros(int(nbytes), np.uint8)
        call('afsi_b200_mg_batch_table', self._plans, self.count, self._sources, host.ctypes.data, int(nbytes))
        self.table = torch.as_tensor(host).to(device)
        self.sync = torch.zeros(int(lib.afsi_b200_mg_sync_bytes()), dtype=torch.uint8, device=device)

    def run(self, cycles, *, start=True, persistent=False):
        """`cycles` V-cycles of every solver on the current stream; with
        `start`, from a zero iterate, with the sources (if this batch has
        them) copied in as right-hand sides first.  persistent: all of it in
        one cooperative launch (``afsi_b200_mg_batch_persistent``) instead of
        one launch per level operation; the results are the same bit for bit."""
        s = torch.cuda.current_stream(self.table.device).cuda_stream
        if persistent:
            call('afsi_b200_mg_batch_persistent', self._plans, self.count, ptr(self.table), int(cycles), int(start),
                 ptr(self.sync), s)
        else:
            call('afsi_b200_mg_batch_vcycles', self._plans, self.count, ptr(self.table), int(cycles), int(start), s)

    def check(self):
        """Raise if a grid barrier of a persistent run timed out."""
        if int(self.sync[8:12].view(torch.int32).item()):
            raise RuntimeError('persistent batched V-cycles: a grid barrier timed out')


class BatchedRefinement:
    """FP64 iterative refinement of many channel pressure solves around
    batched FP32 V-cycles (``afsi_b200_batch_refine_*``).

    Each instance keeps an FP64 iterate and right-hand side (views into two
    batch arrays).  One refinement runs `cycles` batched Jacobi V-cycles of the
    FP32 solvers from zero on the float of the FP64 residual, adds the
    correction in FP64 and forms the new FP64 residual with the reference
    operator and its norm per instance.  Refinements repeat on the device
    until every instance meets its own tolerance max(atol, rtol ||b||), the
    tolerance of the FP64 solver (``mac2d/multigrid.py:94-99``), or
    `max_refinements` ran.  `run(cycles)` launches the whole loop (start plus
    a WHILE node) as one graph; `state()` reads the outcome with one host read.
    """

    def __init__(self, solvers, rhs, *, rtol=1e-10, atol=1e-12, max_refinements=12):
        self.solvers = list(solvers)
        self.count = len(self.solvers)
        if self.count != len(rhs) or not self.count:
            raise ValueError('one FP64 right-hand side per solver')
        lib = _lib.load()
        w0 = self.solvers[0].workspace
        device = w0.p[0].device
        for mg in self.solvers:
            w = mg.workspace
            if w.p[0].dtype != torch.float32 or mg.bc != 'channel' or mg.smoother != 'jacobi':
                raise ValueError('batched refinement takes FP32 Jacobi channel solvers')
        sizes = [mg.workspace.p[0].numel() for mg in self.solvers]
        self.offsets = np.concatenate(([0], np.cumsum(sizes))).astype(np.int64)
        self.b = torch.cat([torch.as_tensor(r, device=device, dtype=torch.float64).reshape(-1) for r in rhs])
        self.p = torch.zeros_like(self.b)
        inst = (_lib.RefineInstance * self.count)()
        for i, mg in enumerate(self.solvers):
            w, (nx, ny) = mg.workspace, mg.shapes[0]
            hx, hy = mg.spacings[0]
            inst[i].nx, inst[i].ny = nx, ny
            inst[i].h2[0], inst[i].h2[1] = hx * hx, hy * hy
            lo = int(self.offsets[i])
            inst[i].p = self.p.data_ptr() + lo * 8
            inst[i].b = self.b.data_ptr() + lo * 8
            inst[i].r32 = ptr(w.rhs[0])
            inst[i].e32 = ptr(w.p[0])
        self._inst = inst
        nbytes = lib.afsi_b200_batch_refine_bytes(inst, self.count)
        if nbytes < 0:
            raise ValueError(f'batched refinement: {lib.afsi_b200_last_error().decode(errors="replace")}')
        host = np.zeros(int(nbytes), np.uint8)
        call('afsi_b200_batch_refine_setup', inst, self.count, host.ctypes.data, int(nbytes))
        self.buffer = torch.as_tensor(host).to(device)
        self._state_off = int(lib.afsi_b200_batch_refine_state_offset(inst, self.count))
        self.vcycles = BatchedVCycles(self.solvers)   # table without sources: a start zeroes the iterates only
        with torch.cuda.device(device):
            self.vcycles.run(1, start=True)  # one eager run sets the kernels' attributes before any capture
        self.rtol, self.atol, self.max_refinements = float(rtol), float(atol), int(max_refinements)
        self._graphs = {}

    def rhs(self, i):
        return self.b[self.offsets[i]:self.offsets[i + 1]].view(self.solvers[i].shapes[0])

    def pressure(self, i):
        return self.p[self.offsets[i]:self.offsets[i + 1]].view(self.solvers[i].shapes[0])

    def _graph(self, cycles):
        if cycles not in self._graphs:
            handle = ctypes.c_void_p()
            before = _lib.launch_count()
            with torch.cuda.device(self.buffer.device):
                call('afsi_b200_batch_refine_graph_create', self._inst, self.count, ptr(self.buffer),
                     self.vcycles._plans, ptr(self.vcycles.table), int(cycles), self.rtol, self.atol,
                     self.max_refinements, ctypes.byref(handle))
            captured = _lib.launch_count() - before  # start + body, captured only
            _lib.forget_launches(captured)
            self._graphs[cycles] = (handle.value, captured - 1)
        return self._graphs[cycles]

    def run(self, cycles):
        """The refinement loop with `cycles` V-cycles per refinement on the current stream."""
        graph, _ = self._graph(cycles)
        call('afsi_b200_batch_refine_graph_launch', graph, torch.cuda.current_stream(self.buffer.device).cuda_stream)

    def run_launched(self, cycles):
        """The same loop driven from the host (one read per refinement), for checks."""
        s = torch.cuda.current_stream(self.buffer.device).cuda_stream
        args = (self._inst, self.count, ptr(self.buffer))
        call('afsi_b200_batch_refine_start', *args, self.rtol, self.atol, self.max_refinements, s)
        while True:
            st = self.state()
            if not st['unconverged'] or st['nonfinite'] or st['refinements'] >= self.max_refinements:
                return st
            self.vcycles.run(cycles, start=True)
            call('afsi_b200_batch_refine_step', *args, self.rtol, self.atol, self.max_refinements, s)

    def state(self):
        """Outcome of the last run: per-instance residual norms, tolerances and
        the refinement after which each first met its tolerance (-1: never)."""
        n = self.count
        words = self.buffer[self._state_off:self._state_off + (4 * n + 8) * 8].view(torch.float64).tolist()
        loop = words[4 * n:]
        return dict(norm=words[:n], tol=words[n:2 * n], rhs_norm=words[2 * n:3 * n],
                    done_at=[int(v) for v in words[3 * n:4 * n]], refinements=int(loop[0]),
                    unconverged=int(loop[1]), nonfinite=bool(loop[2]), worst_ratio=loop[3])

    def launches(self, cycles):
        """Native launches of one run: the start plus the body per refinement."""
        _, body = self._graph(cycles)
        return 1 + body * self.state()['refinements']

    def __del__(self):
        for graph, _ in getattr(self, '_graphs', {}).values():
            try:
                _lib.call('afsi_b200_batch_refine_graph_destroy', graph)
            except Exception:
                pass
        self._graphs = {}


class BatchedChannels:
    """A batch of independent 2D channel instances (grids, points, forces,
    face velocities, pressure right-hand sides), stepped together."""

    def __init__(self, grids, points, forces, velocities, pressures, *, device='cuda',
                 transfer_dtype=torch.float32, mg_dtype=torch.float32, schedule=None):
        if not (len(grids) == len(points) == len(forces) == len(velocities) == len(pressures)) or not grids:
            raise ValueError('one grid, point set, force set, velocity and pressure RHS per instance')
        if len(grids) > 1024:
            raise ValueError('at most 1024 instances per batch')
        device = torch.device(device)
        if device.type != 'cuda':
            raise ValueError('the batched form requires a CUDA device; there is no CPU fallback')
        _lib.load()
        self.device, self.grids = device, list(grids)
        self.transfer_dtype, self.mg_dtype = transfer_dtype, mg_dtype
        self.schedule = schedule or Schedule()
        counts = [int(len(p)) for p in points]
        self.point_offsets = np.concatenate(([0], np.cumsum(counts))).astype(np.int64)
        nu = [(g.shape[0] + 1) * g.shape[1] for g in grids]
        nv = [g.shape[0] * (g.shape[1] + 1) for g in grids]
        self.u_offsets = np.concatenate(([0], np.cumsum(nu))).astype(np.int64)
        self.v_offsets = np.concatenate(([0], np.cumsum(nv))).astype(np.int64)
        table = np.zeros(len(grids), INSTANCE_DTYPE)
        for i, g in enumerate(grids):
            table[i] = (g.shape[0], g.shape[1], g.spacing[0], g.spacing[1], g.lengths[0], g.lengths[1],
                        self.point_offsets[i], counts[i], self.u_offsets[i], self.v_offsets[i])
        self.table = torch.as_tensor(table.view(np.uint8), device=device)
        self.total = int(self.point_offsets[-1])
        self.nu, self.nv = int(self.u_offsets[-1]), int(self.v_offsets[-1])
        as_t = lambda a, dt: torch.as_tensor(np.asarray(a), device=device, dtype=dt)
        self.x = torch.cat([as_t(p, torch.float64) for p in points]).contiguous()
        self.force = torch.cat([as_t(f, transfer_dtype) for f in forces]).contiguous()
        self.u_in = torch.cat([as_t(v[0], transfer_dtype).reshape(-1) for v in velocities])
        self.v_in = torch.cat([as_t(v[1], transfer_dtype).reshape(-1) for v in velocities])
        self.rhs = [as_t(r, mg_dtype) for r in pressures]
        self.rhs64 = [as_t(r, torch.float64) for r in pressures]
        self.ids = torch.empty((2, self.total, 16), device=device, dtype=torch.int64)
        self.weights = torch.empty((2, self.total, 16), device=device, dtype=transfer_dtype)
        self.u = torch.zeros(self.nu, device=device, dtype=transfer_dtype)
        self.v = torch.zeros(self.nv, device=device, dtype=transfer_dtype)
        self.gathered = torch.empty((self.total, 2), device=device, dtype=transfer_dtype)
        self.status = torch.zeros(1, device=device, dtype=torch.int32)
        self._solvers = {}
        self._batched = None
        self._refinement = None
        self.graph = None

    # -- pieces of the step
    def solvers(self, smoother):
        """One FP32 workspace per instance and smoother (built once)."""
        if smoother not in self._solvers:
            opts = MGOptions(smooth=2 if smoother == 'red-black' else 4)
            self._solvers[smoother] = [ChannelMultigrid(g, device=self.device, dtype=self.mg_dtype,
                                                        coarse_dtype=torch.float64, backend='b200',
                                                        smoother=smoother, options=opts) for g in self.grids]
        return self._solvers[smoother]

    def transfers(self, stream):
        s = stream.cuda_stream
        code = dtype_code(self.transfer_dtype)
        n = len(self.grids)
        call('afsi_b200_batch2d_prepare', ptr(self.x), self.total, ptr(self.table), n, ptr(self.ids),
             ptr(self.weights), ptr(self.status), code, s)
        self.u.zero_()
        self.v.zero_()
        call('afsi_b200_batch2d_spread', ptr(self.force), ptr(self.ids), ptr(self.weights), self.total,
             ptr(self.table), n, ptr(self.u), ptr(self.v), self.nu, self.nv, ptr(self.status), code, s)
        call('afsi_b200_batch2d_gather', ptr(self.u_in), ptr(self.v_in), self.nu, self.nv, ptr(self.ids),
             ptr(self.weights), self.total, ptr(self.gathered), ptr(self.status), code, s)

    def cycles(self, index, schedule):
        mg = self.solvers(schedule.smoother)[index]
        w = mg.workspace
        w.rhs[0].copy_(self.rhs[index])
        w.p[0].zero_()
        w.vcycles(schedule.cycles)

    def batched(self):
        """The batched Jacobi V-cycles over the Jacobi workspaces (built once)."""
        if self._batched is None:
            self._batched = BatchedVCycles(self.solvers('jacobi'), self.rhs)
        return self._batched

    def refinement(self):
        """FP64 refinement around the batched FP32 Jacobi V-cycles (built once)."""
        if self._refinement is None:
            if self.mg_dtype != torch.float32:
                raise ValueError('the refined schedule runs FP32 V-cycles')
            self._refinement = BatchedRefinement(self.solvers('jacobi'), self.rhs64)
        return self._refinement

    def order(self, schedule):
        idx = list(range(len(self.grids)))
        if schedule.order == 'largest-first':
            idx.sort(key=lambda i: -(self.grids[i].shape[0] * self.grids[i].shape[1]))
        return idx

    def run(self, schedule=None):
        """The step on the current stream with a fork/join over `streams`
        side streams (eager, or inside a capture)."""
        schedule = schedule or self.schedule
        main = torch.cuda.current_stream(self.device)
        self.transfers(main)
        if schedule.refined:
            self.refinement().run(schedule.cycles)
            return
        if schedule.vcycles in ('batched', 'persistent'):
            if schedule.smoother != 'jacobi':
                raise ValueError('batched V-cycles use the Jacobi smoother')
            self.batched().run(schedule.cycles, persistent=schedule.vcycles == 'persistent')
            return
        if schedule.vcycles != 'streams':
            raise ValueError(f'unknown V-cycle schedule {schedule.vcycles!r}')
        side = [torch.cuda.Stream(device=self.device) for _ in range(schedule.streams)]
        for s in side:
            s.wait_stream(main)
        for k, i in enumerate(self.order(schedule)):
            with torch.cuda.stream(side[k % len(side)]):
                self.cycles(i, schedule)
        for s in side:
            main.wait_stream(s)

    def capture(self, schedule=None):
        """The step as a CUDA graph: everything, or with a refined schedule the
        transfers only (the refinement loop is its own graph, launched after)."""
        schedule = schedule or self.schedule
        self.solvers(schedule.smoother)
        if schedule.refined:
            self.refinement()._graph(schedule.cycles)
        elif schedule.vcycles in ('batched', 'persistent'):
            self.batched()
        step = (lambda: self.transfers(torch.cuda.current_stream(self.device))) if schedule.refined else \
            (lambda: self.run(schedule))
        with torch.cuda.device(self.device):
            warm = torch.cuda.Stream(device=self.device)
            warm.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(warm):
                self.run(schedule)
            torch.cuda.current_stream(self.device).wait_stream(warm)
            g = torch.cuda.CUDAGraph()
            before = _lib.launch_count()
            with torch.cuda.graph(g):
                step()
            launches = _lib.launch_count() - before
            _lib.forget_launches(launches)
        return g, launches

    def use(self, schedule):
        self.schedule = schedule
        self.graph, self.graph_launches = self.capture(schedule)

    def replay(self):
        if self.graph is None:
            self.use(self.schedule)
        self.graph.replay()
        _lib.count_replay(self.graph_launches)
        if self.schedule.refined:
            self.refinement().run(self.schedule.cycles)

    # -- results and checks
    def fields(self, i):
        g = self.grids[i]
        u = self.u[self.u_offsets[i]:self.u_offsets[i + 1]].view(g.face_shape(0))
        v = self.v[self.v_offsets[i]:self.v_offsets[i + 1]].view(g.face_shape(1))
        return u, v

    def velocities(self, i):
        return self.gathered[self.point_offsets[i]:self.point_offsets[i + 1]]

    def pressure(self, i, smoother=None):
        if self.schedule.refined and smoother is None:
            return self.refinement().pressure(i)
        return self.solvers(smoother or self.schedule.smoother)[i].workspace.p[0]

    def refined_report(self):
        """Cycles-to-tolerance per instance of the last refined run (one host read)."""
        st = self.refinement().state()
        c = self.schedule.cycles
        return dict(refinements=st['refinements'], unconverged=st['unconverged'], nonfinite=st['nonfinite'],
                    worst_relative_residual=st['worst_ratio'],
                    cycles_to_tolerance=[d * c if d >= 0 else None for d in st['done_at']],
                    max_norm_over_tol=max(n / t for n, t in zip(st['norm'], st['tol'])))

    def residual_reduction(self, smoother=None):
        """||rhs - A p|| / ||rhs|| per instance after the last step (FP32 workspaces)."""
        out = []
        for i, mg in enumerate(self.solvers(smoother or self.schedule.smoother)):
            out.append(mg.residual_norm().item() / max(self.rhs[i].double().norm().item(), 1e-300))
        return out

    def check(self):
        if self._batched is not None:
            self._batched.check()
        word = int(self.status.item())
        self.status.zero_()
        if word & _lib.FLAG_SUPPORT:
            raise ValueError('valve IB points leave the channel support region')
        if word & _lib.FLAG_INDEX:
            raise RuntimeError('batched stencil index outside its instance')

    # -- autotuner
    def autotune(self, *, target=1e-4, streams=(1, 4, 8, 16), orders=('given', 'largest-first'),
                 smoothers=('jacobi', 'red-black'), max_cycles=12, replays=5):
        """Fastest schedule whose V-cycles reduce every instance's FP32
        residual by `target`: for each smoother the smallest cycle count that
        meets the target (measured), then every (streams, order) and, for
        Jacobi, the batched V-cycles, measured by CUDA-event timing of graph
        replays.  Returns (schedule, table)."""
        table = []
        best = None
        for smoother in smoothers:
            cycles = None
            for c in range(1, max_cycles + 1):
                self.run(Schedule(streams=1, order='given', smoother=smoother, cycles=c))
                torch.cuda.synchronize(self.device)
                if max(self.residual_reduction(smoother)) <= target:
                    cycles = c
                    break
            if cycles is None:
                continue
            candidates = [Schedule(streams=s, order=order, smoother=smoother, cycles=cycles)
                          for s in streams for order in orders]
            if smoother == 'jacobi':
                candidates += [Schedule(streams=1, order='given', smoother=smoother, cycles=cycles, vcycles=v)
                               for v in ('batched', 'persistent')]
            for sch in candidates:
                g, launches = self.capture(sch)
                g.replay()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize(self.device)
                e0.record()
                for _ in range(replays):
                    g.replay()
                e1.record()
                torch.cuda.synchronize(self.device)
                ms = e0.elapsed_time(e1) / replays
                table.append(dict(streams=sch.streams, order=sch.order, smoother=smoother, cycles=cycles,
                                  vcycles=sch.vcycles, ms=ms, launches=launches))
                if best is None or ms < best[0]:
                    best = (ms, sch)
                del g
        if best is None:
            raise RuntimeError(f'no smoother reaches the residual reduction {target:g} in {max_cycles} cycles')
        self.use(best[1])
        return best[1], table


    def autotune_refined(self, *, cycles=(2, 3, 4, 5, 6, 8), replays=5):
        """Fastest refined schedule: for each count of V-cycles per refinement,
        one run to check that every instance meets its FP64 tolerance, then
        CUDA-event timing of `replays` whole steps (transfers graph plus the
        refinement loop); returns (schedule, table)."""
        table, best = [], None
        for c in cycles:
            sch = Schedule(streams=1, order='given', smoother='jacobi', cycles=int(c), vcycles='batched',
                           refined=True)
            self.use(sch)
            self.replay()
            rep = self.refined_report()
            row = dict(cycles_per_refinement=int(c), refinements=rep['refinements'],
                       converged=rep['unconverged'] == 0 and not rep['nonfinite'])
            if row['converged']:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize(self.device)
                e0.record()
                for _ in range(replays):
                    self.replay()
                e1.record()
                torch.cuda.synchronize(self.device)
                row['ms'] = e0.elapsed_time(e1) / replays
                if best is None or row['ms'] < best[0]:
                    best = (row['ms'], sch)
            table.append(row)
        if best is None:
            raise RuntimeError('no refined schedule met the FP64 tolerance on every instance')
        self.use(best[1])
        return best[1], table


def seeded_batch(count=64, *, seed=0, shapes=((128, 32), (256, 64), (384, 96), (512, 128)),
                 points=(5000, 40000), device='cuda', **kwargs):
    """The batching workload: `count` instances with seeded grid sizes,
    leaflet point counts in `points`, N(0,1) forces, seeded Fourier face
    velocities and mean-free N(0,1) pressure right-hand sides; lengths
    (4, 1) so that h is uniform per instance."""
    from . import synthetic
    rng = np.random.default_rng(seed)
    grids, pts, forces, vels, rhs = [], [], [], [], []
    for i in range(count):
        nx, ny = shapes[int(rng.integers(len(shapes)))]
        g = ChannelGrid((nx, ny), (4., 1.))
        n = int(rng.integers(points[0], points[1] + 1))
        grids.append(g)
        pts.append(leaflet_points(g, n, seed=seed * 1000 + i))
        forces.append(rng.standard_normal((n, 2)))
        vels.append(tuple(t.numpy() for t in synthetic.fourier_velocity2d(g, seed=seed * 1000 + i)))
        r = rng.standard_normal((nx, ny))
        rhs.append(r - r.mean())
    return BatchedChannels(grids, pts, forces, vels, rhs, device=device, **kwargs)
