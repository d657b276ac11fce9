"""Benchmark: IB transfer + MG V-cycle steps/s on the 3D P2 FP64 configuration.

Workload (one step, FP64, 64^3 MAC grid on the unit cube):
  P2 prepare (positions + shared Peskin tables) -> P2 spread of nodal forces
  -> P2 gather-assemble of a face velocity -> multigrid pressure solve of a
  mean-zero random right-hand side to 1e-10 relative residual (zero start).
Structure: truncated prolate-spheroid P2 shell (inner/outer semi-axes
0.25/0.32 by 0.15/0.22) of 38,400 elements, adaptive conical interaction
quadrature at point density 2 (order 4 everywhere: 2,457,600 points).
Inputs are seeded synthetic data; the 590 MB of stencil tables exceed the
126 MB L2, so every step streams from HBM (no explicit L2 flush needed).

``--impl b200`` (default) times the CUDA path; ``--impl reference`` times the
CPU restatement of the reference algorithm (the oracle) on this host.  With
``--gpus N`` under torchrun every rank runs an independent replica (the path
does not shard); the reported value is the whole-job steps/s from the slowest
rank.
"""
import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SHELL = dict(nr=3, ntheta=40, nphi=64)
GRID = dict(shape=(64, 64, 64), lengths=(1., 1., 1.))
METRIC = 'IB transfer+MG V-cycle steps/s (P2 prepare+spread+interpolate+pressure MG solve, FP64)'


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=50)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='b200', choices=('b200', 'reference'))
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--rows', default='all', choices=('all', 'step', 'p1'),
                    help="'step': the headline step line only, without the mass-solve, MG-form, batching and "
                         "serving rows (for profiler runs); 'p1': only the precision-form row on the 128^3 P1 "
                         "configuration, printed as its own JSON object (for profiler runs)")
    return ap.parse_args()


def workload():
    from afsi_gpu_b200 import synthetic
    from afsi_gpu_b200.grid import MACGrid
    grid = MACGrid(GRID['shape'], GRID['lengths'])
    X, cells = synthetic.p2_shell(**SHELL)
    rng = np.random.default_rng(12)
    coef = rng.standard_normal(X.shape)
    vel = [v.numpy() for v in synthetic.fourier_velocity3d(grid, seed=3)]
    rhs = synthetic.mean_free_normal(grid.shape, seed=4).numpy()
    return grid, X, cells, coef, vel, rhs


# ------------------------------------------------------------------- clocks

class Clocks:
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get('TMPDIR', '/tmp')) / f'afsi_clocks_{os.getpid()}.csv'

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.QUERY}',
                                          '--format=csv,noheader,nounits', '-lms', '50'],
                                         stdout=open(self.path, 'w'), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        self.skip = 0
        deadline = time.time() + 5  # the sampler's first row marks the start; rows before the region are idle
        while self.proc is not None and time.time() < deadline:
            rows = self._rows()
            if rows:
                self.skip = len(rows)
                break
            time.sleep(.02)
        return self

    def _rows(self):
        try:
            rows = [r.split(', ') for r in self.path.read_text().strip().splitlines() if r.strip()]
        except OSError:
            return []
        return [r for r in rows if len(r) >= 9]

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = self._rows()
        rows = rows[self.skip:] or rows[-1:]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip().lower() == 'active'})
        return dict(sm_mhz=float(np.median(sm)) if sm else None,
                    sm_max_mhz=float(rows[0][2]) if rows[0][2].replace('.', '').isdigit() else None,
                    reasons=reasons, samples=len(rows))


# ----------------------------------------------------------------- the step

class Step:
    """Device-resident inputs; one call = one hot-path step."""

    def __init__(self, grid, X, cells, coef, vel, rhs, device):
        from afsi_gpu_b200 import p2_cuda_transfer as p2t
        from afsi_gpu_b200.multigrid import GeometricMultigrid
        self.p2t = p2t
        self.grid = grid
        self.x = torch.as_tensor(X, device=device)
        self.cells = torch.as_tensor(cells, device=device)
        self.coef = torch.as_tensor(coef, device=device)
        self.vel = tuple(torch.as_tensor(v, device=device) for v in vel)
        self.rhs = torch.as_tensor(rhs, device=device)
        self.tr = p2t.P2Transfer(grid, self.x, self.cells)
        self.mg = GeometricMultigrid(grid, device=device, backend='b200-graph')
        self.events = None
        self.cycles = []

    def __call__(self, x=None, coef=None, vel=None, rhs=None, timing=None):
        """timing: nine CUDA events: before prepare and after each of the four
        phases, then the spread and gather-assemble kernels alone."""
        ev = timing
        if ev is not None:
            ev[0].record()
        # rule selection without a host read: the prepare runs with the cached
        # rule and is confirmed after the solve's own host read; a changed rule
        # (never on this workload) redoes the transfers
        deferred = self.tr.prepare_deferred(self.x if x is None else x)
        st = deferred.stencil
        if ev is not None:
            ev[1].record()
        coef = self.coef if coef is None else coef
        vel = self.vel if vel is None else vel
        fields = self.p2t.spread(self.tr, coef, st, events=None if ev is None else ev[5:7])
        if ev is not None:
            ev[2].record()
        nodal = self.p2t.assemble_velocity(self.tr, vel, st, events=None if ev is None else ev[7:9])
        if ev is not None:
            ev[3].record()
        p, info = self.mg.solve(self.rhs if rhs is None else rhs)
        if ev is not None:
            ev[4].record()
        confirmed = self.tr.confirm(deferred)
        if confirmed is not st:
            st = confirmed
            fields = self.p2t.spread(self.tr, coef, st)
            nodal = self.p2t.assemble_velocity(self.tr, vel, st)
        self.cycles.append(info['cycles'])
        return st, fields, nodal, p


def algorithmic_bytes(points, elements, nodes, faces, s=8):
    """Bytes a launch must move at minimum, per unit of work.

    Tables: base (2,P,3) int64 + phi (2,P,3,4) = 48 + 24*s per point.
    spread: tables + W (s/pt) + cells (80/elem) + nodal coef gathered per
    element (10*3*s) + face write (s/face).  gather: same reads with the face
    field read instead of written, plus the nodal rhs written (3*s/node)."""
    tables = points * (48 + 24 * s)
    common = tables + points * s + elements * (80 + 30 * s)
    return dict(prepare=tables + elements * 80 + nodes * 3 * s,
                spread=common + faces * s,
                gather=common + faces * s + nodes * 3 * s)


def mg_bytes_per_cycle(shapes, smooth=4, s=8):
    """Σ_l N_l·s·(6·smooth + 10.25): Jacobi read p,rhs / write p per sweep,
    gauge passes, residual-restrict and prolong-add, per V-cycle."""
    return sum(np.prod(sh) * s * (6 * smooth + 10.25) for sh in shapes[:-1])


def mass_pcg_row(X, cells, device, peak_gbs, solves=20):
    """Consistent-mass Jacobi-PCG (the solve inside every reference FE
    spread/interpolate, mac/transfer.py:105-140) on the P2 mass matrix of the
    bench mesh: its CSR pattern (every node pair of each element) does not
    depend on the quadrature rule, so the rule here is the degree-4 Keast
    rule.  The transfer's options (rtol 1e-12, atol 1e-13, check_every 4).

    Bytes per iteration: the SpMV reads the matrix (int32 column + value per
    entry, int64 row pointers), gathers d once and writes Ad; the update reads
    x, d, r, Ad and the per-row diagonal and writes x, r; the direction reads
    r, diagonal, d and writes d."""
    from afsi_gpu_b200.mass import MassSolver, SolverOptions
    from afsi_gpu_b200.quadrature import keast5, tabulate_p2, reference_determinants
    q, w = keast5()
    N = torch.as_tensor(tabulate_p2(q), device=device)
    W = reference_determinants(torch.as_tensor(X), torch.as_tensor(cells)).to(device)[:, None] * \
        torch.as_tensor(w, device=device)
    c = torch.as_tensor(cells, device=device)
    local = torch.einsum('eq,qa,qb->eab', W, N, N)
    rows = X.shape[0]
    ij = torch.stack((c[:, :, None].expand_as(local).reshape(-1), c[:, None, :].expand_as(local).reshape(-1)))
    M = torch.sparse_coo_tensor(ij, local.reshape(-1), (rows, rows)).coalesce().to_sparse_csr()
    diag = torch.zeros(rows, device=device, dtype=torch.float64).index_add(
        0, c.reshape(-1), local.diagonal(dim1=-2, dim2=-1).reshape(-1))
    solver = MassSolver(M, diag[:, None].expand(-1, 3),
                        SolverOptions(rtol=1e-12, atol=1e-13, max_iterations=500, check_every=4))
    g = torch.Generator(device=device).manual_seed(21)
    rhs = torch.randn((rows, 3), device=device, dtype=torch.float64, generator=g)
    for _ in range(3):
        x, info = solver.solve(rhs)
    stream = torch.cuda.current_stream(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    e0.record(stream)
    for _ in range(solves):
        x, info = solver.solve(rhs)
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1) / solves
    nnz = M.values().numel()
    vec = rows * 3 * 8
    per_it = nnz * 12 + (rows + 1) * 8 + 2 * vec + (7 * vec + rows * 8) + (4 * vec + rows * 8)
    us_it = ms * 1e3 / max(info.iterations, 1)
    gbs = per_it / (us_it * 1e-6) / 1e9
    return dict(rows=rows, nnz=int(nnz), iterations=info.iterations, ms_per_solve=ms, us_per_iteration=us_it,
                bytes_per_iteration=int(per_it), achieved_gbs=gbs, frac=gbs / peak_gbs,
                residual=info.residual_norm, tolerance=info.tolerance,
                note='one begin launch + one WHILE-loop graph launch per solve, one host read')


def mg_forms_row(grid, rhs, device, reps=10):
    """The 64^3 pressure solve of the step in its other forms, each to the
    same FP64 tolerance (rtol 1e-10): the reference's Jacobi smoother (the
    step's solver), the red-black Gauss-Seidel smoother (2 sweeps), and the
    precision form (FP32 V-cycles inside FP64 iterative refinement) with each
    smoother.  CUDA events around `reps` solves; `max_rel_diff` is the largest
    difference from the Jacobi FP64 solution over its largest value."""
    from afsi_gpu_b200.multigrid import GeometricMultigrid, MGOptions, RefinedMultigrid
    b = torch.as_tensor(rhs, device=device)
    solvers = dict(
        jacobi_fp64=GeometricMultigrid(grid, device=device, backend='b200-graph'),
        red_black_fp64=GeometricMultigrid(grid, device=device, backend='b200-graph', smoother='red-black',
                                          options=MGOptions(smooth=2)),
        jacobi_fp32_refined=RefinedMultigrid(grid, device=device),
        red_black_fp32_refined=RefinedMultigrid(grid, device=device, smoother='red-black',
                                                options=MGOptions(smooth=2)))
    stream = torch.cuda.current_stream(device)
    out, base = {}, None
    for name, mg in solvers.items():
        for _ in range(2):
            p, info = mg.solve(b)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        for _ in range(reps):
            p, info = mg.solve(b)
        e1.record(stream)
        torch.cuda.synchronize(device)
        if base is None:
            base = p
        out[name] = dict(ms_per_solve=e0.elapsed_time(e1) / reps, cycles=info['cycles'],
                         refinements=info.get('refinements'), residual=info['residual_norm'],
                         tolerance=info['tolerance'],
                         max_rel_diff=float((p - base).abs().max() / base.abs().max()))
    return out


def batch_form_row(device, count=64, replays=20):
    """Batching form: 64 seeded 2D channel instances (grids 128x32 .. 512x128,
    5k-40k leaflet points each, N(0,1) forces), FP32 transfers and V-cycles,
    one captured graph per step with the autotuned schedule (batched or
    per-instance V-cycles; fixed V-cycle count reaching a 1e-4 FP32 residual
    reduction on every instance).  The
    plain FP64 drop-in on the same GPU steps the same instances one at a time
    through the single-instance API (prepare2d with its support check,
    spread2d, gather2d, FP64 channel V-cycles, same cycle count).  Errors:
    largest difference of the FP32 batch from the FP64 plain step over the
    largest value, per output."""
    from afsi_gpu_b200 import cuda_ib
    from afsi_gpu_b200.batch import seeded_batch
    from afsi_gpu_b200.multigrid import ChannelMultigrid, MGOptions
    b = seeded_batch(count, seed=0, device=device)
    schedule, table = b.autotune(target=1e-4)
    stream = torch.cuda.current_stream(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b.replay()
    torch.cuda.synchronize(device)
    e0.record(stream)
    for _ in range(replays):
        b.replay()
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1) / replays
    b.check()
    # plain FP64 drop-in, one instance at a time
    opts = MGOptions(smooth=2 if schedule.smoother == 'red-black' else 4)
    plain = [ChannelMultigrid(g, device=device, backend='b200', smoother=schedule.smoother, options=opts)
             for g in b.grids]
    x = [b.x[b.point_offsets[i]:b.point_offsets[i + 1]] for i in range(count)]
    f = [b.force[b.point_offsets[i]:b.point_offsets[i + 1]].double() for i in range(count)]
    vel = [(b.u_in[b.u_offsets[i]:b.u_offsets[i + 1]].double().view(g.face_shape(0)),
            b.v_in[b.v_offsets[i]:b.v_offsets[i + 1]].double().view(g.face_shape(1)))
           for i, g in enumerate(b.grids)]
    rhs = [r.double() for r in b.rhs]

    def plain_step():
        out = []
        for i, g in enumerate(b.grids):
            st = cuda_ib.prepare2d(g, x[i])
            fields = cuda_ib.spread2d(g, f[i], st)
            gathered = cuda_ib.gather2d(vel[i], st)
            mg = plain[i]
            mg.initialize(torch.zeros_like(rhs[i]), rhs[i])
            out.append((fields, gathered, mg.advance(schedule.cycles)))
        return out

    plain_step()
    torch.cuda.synchronize(device)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    reps = 3
    for _ in range(reps):
        res = plain_step()
    p1.record(stream)
    torch.cuda.synchronize(device)
    plain_ms = p0.elapsed_time(p1) / reps

    def rel(a, ref):
        return float((a.double() - ref).abs().max() / ref.abs().max())

    err = dict(spread=max(max(rel(b.fields(i)[c], res[i][0][c]) for c in range(2)) for i in range(count)),
               interpolate=max(rel(b.velocities(i), res[i][1]) for i in range(count)),
               v_cycles=max(rel(b.pressure(i), res[i][2]) for i in range(count)))
    return dict(instances=count, points=b.total, faces=b.nu + b.nv,
                schedule=dict(streams=schedule.streams, order=schedule.order, smoother=schedule.smoother,
                              cycles=schedule.cycles, vcycles=schedule.vcycles),
                ms_per_batch_step=ms, instance_steps_per_s=count / (ms / 1e3),
                plain_fp64_ms_per_batch=plain_ms, plain_fp64_instance_steps_per_s=count / (plain_ms / 1e3),
                speedup_vs_plain_fp64=plain_ms / ms, error_vs_fp64=err,
                max_residual_reduction=max(b.residual_reduction()), graph_launches=b.graph_launches,
                autotune=table)


def serving_form_row(device, count=400):
    """Serving form: `count` requests of the serving mix (50% 2D 256x64 with
    20k points, 35% 3D 32^3-64^3 with 50k-400k points, 15% 3D 96^3 with 800k
    points; Poisson arrivals at 2000/s, seeded), each a full FP64 step
    (prepare, spread, interpolate, pressure solve to 1e-10) on resident
    states, admitted under a 150 GB budget.  8 worker slots (continuous
    batching) against 1 slot (requests one at a time, the plain drop-in)."""
    from afsi_gpu_b200.serving import Request, Server, mix
    reqs = mix(count, rate=2000., seed=0)
    out = {}
    for slots in (8, 1):
        server = Server(device=device, slots=slots)
        server.warm(reqs)
        server.serve(reqs[:16])  # warm-up
        report, _ = server.serve(reqs)
        out[f'slots_{slots}'] = report
    out['speedup_vs_one_slot'] = out['slots_8']['steps_per_s'] / out['slots_1']['steps_per_s']
    # 2000 req/s saturates the GPU (latency is queueing); the same mix at a
    # quarter of the saturated throughput shows the step latency itself, and
    # at half of it the knee where queueing starts
    server = Server(device=device, slots=8)
    below = mix(count // 2, rate=1., seed=1)
    server.serve([Request(0., r.rid, r.kind, r.n, r.points, r.seed) for r in below[:16]])  # warm-up
    for key, share in (('slots_8_below_saturation', .25), ('slots_8_half_saturation', .5)):
        rate = share * out['slots_8']['steps_per_s']
        report, _ = server.serve(mix(count // 2, rate=rate, seed=1))
        out[key] = dict(report, arrival_rate=rate)
    return out


def precision_form_row(grid, X, cells, coef, vel, rhs, device, steps=20):
    """Precision form of the step on the bench workload: FP64 positions and
    bases, FP32 weight tables and transfers, and the pressure solve as FP32
    V-cycles inside FP64 iterative refinement to the FP64 tolerance.  CUDA
    events around `steps` steps; errors are the largest differences from the
    FP64 step's outputs over their largest values."""
    from afsi_gpu_b200 import p2_cuda_transfer as p2t
    from afsi_gpu_b200.multigrid import GeometricMultigrid, RefinedMultigrid
    x = torch.as_tensor(X, device=device)
    c64 = torch.as_tensor(coef, device=device)
    v64 = tuple(torch.as_tensor(v, device=device) for v in vel)
    r64 = torch.as_tensor(rhs, device=device)
    tr64 = p2t.P2Transfer(grid, x, torch.as_tensor(cells, device=device))
    tr32 = p2t.P2Transfer(grid, x, torch.as_tensor(cells, device=device), transfer_dtype=torch.float32)
    mg64 = GeometricMultigrid(grid, device=device, backend='b200-graph')
    mg32 = RefinedMultigrid(grid, device=device)
    c32, v32 = c64.float(), tuple(v.float() for v in v64)

    def step(tr, mg, c, v):
        st = tr.prepare(x)
        return tr.spread(c, st), tr.assemble_velocity(v, st), mg.solve(r64)

    ref = step(tr64, mg64, c64, v64)
    stream = torch.cuda.current_stream(device)

    def timed(mg):
        for _ in range(3):
            out = step(tr32, mg, c32, v32)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        for _ in range(steps):
            out = step(tr32, mg, c32, v32)
        e1.record(stream)
        torch.cuda.synchronize(device)
        return out, e0.elapsed_time(e1) / steps

    def rel(a, b):
        return float((a.double() - b.double()).abs().max() / b.double().abs().max())

    rows = {}
    for name, mg in (('fp32_transfers_refined_mg', mg32), ('fp32_transfers_fp64_mg', mg64)):
        out, ms = timed(mg)
        info = out[2][1]
        rows[name] = dict(steps_per_s=1e3 / ms, ms_per_step=ms, transfer_dtype='f32', positions='f64',
                          mg=(f"FP32 V-cycles in FP64 refinement, {info['refinements']} refinements, "
                              f"{info['cycles']} FP32 cycles" if 'refinements' in info else
                              f"FP64 V-cycles, {info['cycles']} cycles"),
                          residual=info['residual_norm'], tolerance=info['tolerance'],
                          error_vs_fp64=dict(spread=max(rel(a, b) for a, b in zip(out[0], ref[0])),
                                             gather_assemble=rel(out[1], ref[1]),
                                             pressure=rel(out[2][0], ref[2][0])))
    return rows


P1_SHELL = dict(nr=2, ntheta=80, nphi=160, outer=(.224, .154, .154), inner=(.214, .144, .144))


def precision_p1_row(device, steps=5):
    """The precision form on its own configuration: 128^3 MAC grid, a thin P1
    tetrahedral prolate shell (128,000 elements, about 1.22 M adaptive
    interaction points at density 2), seeded uniform nodal forces in [-1, 1],
    a seeded Fourier face velocity and a mean-free N(0,1) pressure RHS.  A step
    is the P1 prepare and CSR assembly (positions, tables and contraction in
    FP64), the spread and the interpolate, and the pressure solve to the FP64
    tolerance.  Plain: FP64 operators and FP64 V-cycles.  Precision form: the
    assembled operator values rounded to FP32, FP32 spread / interpolate, and
    FP32 V-cycles inside FP64 iterative refinement.  CUDA events around each
    of `steps` steps after one untimed step, the median step reported (the
    assembly reads the host three times per step, so a busy host shows up as
    outliers); errors are the largest differences from the FP64 step's
    outputs over their largest values."""
    from afsi_gpu_b200 import synthetic
    from afsi_gpu_b200.grid import MACGrid
    from afsi_gpu_b200.multigrid import GeometricMultigrid, RefinedMultigrid
    from afsi_gpu_b200.p1_csr import P1CSRTransfer
    grid = MACGrid((128, 128, 128), (1., 1., 1.))
    X, cells = synthetic.prolate_shell(**P1_SHELL)
    rng = np.random.default_rng(21)
    x = torch.as_tensor(X, device=device)
    cells_t = torch.as_tensor(cells, device=device)
    c64 = torch.as_tensor(rng.uniform(-1., 1., (X.shape[0], 3)), device=device)
    v64 = tuple(v.to(device) for v in synthetic.fourier_velocity3d(grid, seed=21))
    r64 = synthetic.mean_free_normal(grid.shape, seed=21).to(device)
    budget = dict(max_entries=400_000_000)
    tr64 = P1CSRTransfer(grid, x, cells_t, **budget)
    tr32 = P1CSRTransfer(grid, x, cells_t, transfer_dtype=torch.float32, **budget)
    mg64 = GeometricMultigrid(grid, device=device, backend='b200-graph')
    mg32 = RefinedMultigrid(grid, device=device)
    c32, v32 = c64.float(), tuple(v.float() for v in v64)
    stream = torch.cuda.current_stream(device)

    def step(tr, mg, c, v):
        st = tr.prepare(x)
        return tr.spread(c, st), tr.interpolate_rhs(v, st), mg.solve(r64), st

    def timed(*args):
        out = step(*args)
        torch.cuda.synchronize(device)
        ms = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = step(*args)
            e1.record(stream)
            torch.cuda.synchronize(device)
            ms.append(e0.elapsed_time(e1))
        return out, float(np.median(ms))

    def rel(a, b):
        return float((a.double() - b.double()).abs().max() / b.double().abs().max())

    ref, ms64 = timed(tr64, mg64, c64, v64)
    out, ms32 = timed(tr32, mg32, c32, v32)
    info64, info32 = ref[2][1], out[2][1]
    return dict(workload=(f'128^3 MAC, P1 prolate shell {cells.shape[0]} elements / '
                          f'{ref[3].rule.point_count} points, uniform [-1,1] forces'),
                points=int(ref[3].rule.point_count), elements=int(cells.shape[0]),
                csr_nnz=int(ref[3].assembly['total_nnz']),
                plain_fp64=dict(steps_per_s=1e3 / ms64, ms_per_step=ms64, cycles=info64['cycles'],
                                residual=info64['residual_norm'], tolerance=info64['tolerance']),
                precision_form=dict(steps_per_s=1e3 / ms32, ms_per_step=ms32, transfer_dtype='f32',
                                    positions='f64',
                                    mg=(f"FP32 V-cycles in FP64 refinement, {info32['refinements']} refinements, "
                                        f"{info32['cycles']} FP32 cycles"),
                                    residual=info32['residual_norm'], tolerance=info32['tolerance']),
                speedup_vs_plain_fp64=ms64 / ms32,
                error_vs_fp64=dict(spread=max(rel(a, b) for a, b in zip(out[0], ref[0])),
                                   interpolate=rel(out[1], ref[1]), pressure=rel(out[2][0], ref[2][0])))


def deterministic_row(step, coef, device, reps=10):
    """The P2 spread of the step in its deterministic mode (tile-sorted,
    atomic-free, bitwise reproducible) beside the atomic spread: CUDA events
    around `reps` spreads each (the plan is built once per stencil, outside
    the timing), and the largest difference between the two."""
    from afsi_gpu_b200 import p2_cuda_transfer as p2t
    tr = step.tr
    st = tr.prepare(step.x)
    c = torch.as_tensor(coef, device=device)
    det = p2t.P2Transfer(step.grid, step.x, step.cells, deterministic=True)
    det.rules = tr.rules
    a = tr.spread(c, st)
    d = det.spread(c, st)
    again = det.spread(c, st)
    stream = torch.cuda.current_stream(device)
    out = {}
    for name, fn in (('atomic', lambda: tr.spread(c, st)), ('deterministic', lambda: det.spread(c, st))):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(device)
        out[f'{name}_ms'] = e0.elapsed_time(e1) / reps
    out['bitwise_reproducible'] = all(torch.equal(x, y) for x, y in zip(d, again))
    out['max_rel_diff_vs_atomic'] = max(float((x - y).abs().max() / y.abs().max()) for x, y in zip(d, a))
    return out


def load_traffic():
    path = ROOT / 'profiles' / 'traffic.json'
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def peaks():
    try:
        return json.loads((ROOT / 'MEASURED_PEAKS.json').read_text()), 'measured'
    except (OSError, ValueError):
        return dict(hbm_gbs=6650.0), 'fallback'


# ----------------------------------------------------------- cpu baselines

def cpu_step_time(grid, X, cells, coef, vel, rhs, fraction=0.05):
    """Oracle (NumPy port of the reference algorithm) on a bounded sample:
    the first `fraction` of the elements for the transfers (time scaled by the
    point ratio) and the full 64^3 multigrid solve."""
    from oracle import ib, mg
    from afsi_gpu_b200.quadrature import conical_rule, tabulate_p2, reference_determinants
    E = cells.shape[0]
    Es = max(1, int(E * fraction))
    sub = cells[:Es]
    q, w = conical_rule(4)
    N = tabulate_p2(q)
    W = reference_determinants(torch.as_tensor(X), torch.as_tensor(sub)).numpy()[:, None] * w
    t0 = time.perf_counter()
    base, phi, _ = ib.p2_prepare(X, [(sub, N)], grid.origin, grid.spacing, grid.shape)
    fields = ib.p2_spread(coef, [(sub, N, W)], base, phi, grid.shape, grid.volume)
    nodal = ib.p2_gather_assemble(vel, [(sub, N, W)], base, phi, grid.shape, X.shape[0])
    t1 = time.perf_counter()
    h = mg.Hierarchy(grid.shape, grid.spacing, 'neumann')
    p, info = mg.solve(h, rhs)
    t2 = time.perf_counter()
    transfer = (t1 - t0) * (E / Es)
    outputs = dict(sub=sub, N=N, W=W, fields=fields, nodal=nodal, p=p, cycles=info['cycles'])
    return transfer + (t2 - t1), dict(transfer_s=transfer, mg_s=t2 - t1, elements_sampled=Es, elements=E), outputs


def oracle_errors(step, X, coef, vel, outputs, p_device):
    """Relative errors (max |device - oracle| / max |oracle|) of the step's
    outputs against the FP64 oracle: spread and gather-assemble on the
    oracle's element sample (same cells, rule and weights), and the 64^3
    pressure solve of the timed steps."""
    from afsi_gpu_b200 import p2_cuda_transfer as p2t
    from afsi_gpu_b200.quadrature import InteractionRule, QuadratureGroup
    dev = step.x.device
    group = QuadratureGroup(torch.as_tensor(outputs['sub'], device=dev),
                            torch.as_tensor(outputs['N'], device=dev, dtype=torch.float64),
                            torch.as_tensor(outputs['W'], device=dev, dtype=torch.float64), 4)
    rule = InteractionRule((group,), None, group.weights.numel())
    base, phi = p2t.prepare(step.tr, step.x, rule)
    st = p2t.SharedAdaptiveStencil(base, phi, rule)
    fields = p2t.spread(step.tr, step.coef, st)
    nodal = p2t.assemble_velocity(step.tr, step.vel, st)

    def rel(a, b):
        b = np.asarray(b)
        return float(np.abs(np.asarray(a).reshape(b.shape) - b).max() / max(np.abs(b).max(), 1e-300))
    return dict(spread=max(rel(f.cpu().numpy(), o) for f, o in zip(fields, outputs['fields'])),
                gather_assemble=rel(nodal.cpu().numpy(), outputs['nodal']),
                mg_solve=rel(p_device, outputs['p']), mg_cycles_oracle=int(outputs['cycles']),
                sample='spread/gather on the CPU-baseline element sample; MG on the full 64^3 solve')


# --------------------------------------------------------------------- main

def _json(o):
    if isinstance(o, (np.integer,)):
        return int(o)
    if isinstance(o, (np.floating,)):
        return float(o)
    raise TypeError(type(o))


def max_over_ranks(value, dist, device):
    """The largest `value` over the ranks: a multi-GPU time is its slowest rank's."""
    if not dist:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def whole_job_rate(world, steps, elapsed):
    """Steps per second of the whole job: every replica ran `steps` steps."""
    return world * steps / elapsed


def dist_setup(args):
    if args.gpus > 1 or 'RANK' in os.environ:
        import torch.distributed as dist
        from datetime import timedelta
        backend = 'nccl' if args.impl == 'b200' else 'gloo'
        if args.impl == 'b200':
            torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
        return dist, dist.get_rank(), dist.get_world_size()
    return None, 0, 1


_ORACLE = {}


def _oracle_worker_init(X, coef, vel, shape, lengths, origin):
    """Reference-arm worker set-up: the step's static inputs, the rule tables
    and the oracle import, once per worker process."""
    from afsi_gpu_b200.quadrature import conical_rule, tabulate_p2
    torch.set_num_threads(1)  # one core per worker: the workers are the parallelism
    q, w = conical_rule(4)
    spacing = tuple(L / n for L, n in zip(lengths, shape))
    _ORACLE.update(X=X, coef=coef, vel=vel, shape=shape, origin=origin, spacing=spacing,
                   volume=float(np.prod(spacing)), N=tabulate_p2(q), w=w)


def _oracle_transfer_chunk(cells):
    """One worker's share of the reference arm: the oracle prepare, spread and
    gather-assemble of a chunk of elements (top level, so that a spawn pool
    can call it)."""
    from oracle import ib
    from afsi_gpu_b200.quadrature import reference_determinants
    o = _ORACLE
    W = reference_determinants(torch.as_tensor(o['X']), torch.as_tensor(cells)).numpy()[:, None] * o['w']
    base, phi, _ = ib.p2_prepare(o['X'], [(cells, o['N'])], o['origin'], o['spacing'], o['shape'])
    fields = ib.p2_spread(o['coef'], [(cells, o['N'], W)], base, phi, o['shape'], o['volume'])
    nodal = ib.p2_gather_assemble(o['vel'], [(cells, o['N'], W)], base, phi, o['shape'], o['X'].shape[0])
    return fields, nodal


def run_reference(args):
    dist, rank, world = dist_setup(args)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    grid, X, cells, coef, vel, rhs = workload()
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    from oracle import mg
    cores = max(1, len(os.sched_getaffinity(0)))
    E = cells.shape[0]
    times = []
    warm, timed = min(args.warmup, 1), min(args.steps, 10)
    init = (X, coef, vel, tuple(grid.shape), tuple(grid.lengths), tuple(grid.origin))
    for var in ('OMP_NUM_THREADS', 'OPENBLAS_NUM_THREADS', 'MKL_NUM_THREADS'):
        os.environ[var] = '1'  # inherited by the spawned workers
    with ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context('spawn'), initializer=_oracle_worker_init,
                             initargs=init) as pool:
        list(pool.map(_oracle_transfer_chunk, [cells[:8]] * cores))  # start every worker, import the oracle
        # use the worker count with the best element throughput on this host
        # (hosts whose cores share memory bandwidth stop scaling early)
        best = None
        k = 1
        while k <= cores:
            t0 = time.perf_counter()
            list(pool.map(_oracle_transfer_chunk, [cells[i * 512:(i + 1) * 512] for i in range(k)]))
            rate = k * 512 / (time.perf_counter() - t0)
            if best is None or rate > best[0]:
                best = (rate, k)
            k = k * 2 if k * 2 <= cores or k == cores else cores
        workers = best[1]
        Es = min(E, 512 * workers)  # element sample: 512 per worker, time scaled by E / Es
        tasks = [cells[c] for c in np.array_split(np.arange(Es), workers)]
        h = mg.Hierarchy(grid.shape, grid.spacing, 'neumann')
        for i in range(warm + timed):
            t0 = time.perf_counter()
            parts = list(pool.map(_oracle_transfer_chunk, tasks))
            fields = [sum(p[0][c] for p in parts) for c in range(3)]
            nodal = sum(p[1] for p in parts)
            t1 = time.perf_counter()
            p, info = mg.solve(h, rhs)
            t2 = time.perf_counter()
            if i >= warm:
                times.append((t1 - t0) * (E / Es) + (t2 - t1))
    step = float(np.mean(times))
    sample = (f'oracle (NumPy restatement of the reference CPU path): P2 prepare/spread/gather-assemble on '
              f'{Es} of {E} elements split over {workers} worker processes (the fastest count of 1..{cores} '
              f'host cores), time scaled by elements; full 64^3 MG solve in one process; {timed} steps after '
              f'{warm} warm-up')
    cores = workers
    value = 1.0 / step
    line = dict(metric=METRIC, value=value, unit='steps/s', impl='reference', n_gpus=args.gpus, steps=timed,
                warmup=warm, ms_per_step=step * 1e3, higher_is_better=True, scaling='weak',
                vs_baseline=None, dtype='f64', data='synthetic',
                config=dict(workload='3D P2 shell 38400 elements / 2457600 points, 64^3 MAC, FP64'),
                cpu_baseline=dict(value=value, unit='steps/s', cores=cores, kind='port', sample=sample),
                e2e=dict(value=value, unit='steps/s', h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line, default=_json))
    if dist:
        dist.destroy_process_group()


def run_b200(args):
    dist, rank, world = dist_setup(args)
    device = torch.device('cuda', torch.cuda.current_device())
    from afsi_gpu_b200 import _lib
    _lib.load()
    grid, X, cells, coef, vel, rhs = workload()
    step = Step(grid, X, cells, coef, vel, rhs, device)
    stream = torch.cuda.current_stream(device)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize(device)

    for _ in range(args.warmup):
        step()
    barrier()
    phases = []
    launches0 = _lib.launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(device.index) as clocks:
        barrier()
        start.record(stream)
        for _ in range(args.steps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(9)]
            step(timing=ev)
            phases.append(ev)
        stop.record(stream)
        barrier()
    launches = _lib.launch_count() - launches0
    elapsed = max_over_ranks(start.elapsed_time(stop) / 1e3, dist, device)
    names = ('prepare', 'spread', 'gather_assemble', 'mg_solve')
    phase_ms = {n: float(np.mean([ev[i].elapsed_time(ev[i + 1]) for ev in phases])) for i, n in enumerate(names)}
    spread_t = float(np.mean([ev[5].elapsed_time(ev[6]) for ev in phases])) / 1e3
    gather_t = float(np.mean([ev[7].elapsed_time(ev[8]) for ev in phases])) / 1e3

    # end to end through the public API with pinned host buffers: every step
    # copies its inputs in and its results out; the copies run on a copy
    # stream, double-buffered, so step k+1's inputs arrive and step k-1's
    # results leave while step k computes (a pipelined request loop)
    host = dict(x=torch.as_tensor(X).pin_memory(), coef=torch.as_tensor(coef).pin_memory(),
                vel=tuple(torch.as_tensor(v).pin_memory() for v in vel),
                rhs=torch.as_tensor(rhs).pin_memory())
    h2d = (host['x'].numel() + host['coef'].numel() + sum(v.numel() for v in host['vel'])
           + host['rhs'].numel()) * 8
    copy = torch.cuda.Stream(device=device)
    dev_in = [dict(x=torch.empty_like(host['x'], device=device), coef=torch.empty_like(host['coef'], device=device),
                   vel=tuple(torch.empty_like(v, device=device) for v in host['vel']),
                   rhs=torch.empty_like(host['rhs'], device=device)) for _ in range(2)]

    def copy_in(slot):
        """H2D of one step's inputs into buffer `slot` on the copy stream."""
        b = dev_in[slot]
        with torch.cuda.stream(copy):
            b['x'].copy_(host['x'], non_blocking=True)
            b['coef'].copy_(host['coef'], non_blocking=True)
            for d, h in zip(b['vel'], host['vel']):
                d.copy_(h, non_blocking=True)
            b['rhs'].copy_(host['rhs'], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(copy)
        return ev

    def e2e_run(count, outs=None):
        """`count` pipelined steps; returns the pinned result buffers."""
        ready = {0: copy_in(0)}
        done = None
        for k in range(count):
            if k + 1 < count:
                if done is not None:
                    copy.wait_event(done)  # step k-1 has finished reading that buffer
                ready[k + 1] = copy_in((k + 1) % 2)
            stream.wait_event(ready.pop(k))
            b = dev_in[k % 2]
            st, fields, nodal, p = step(b['x'], b['coef'], b['vel'], b['rhs'])
            results = list(fields) + [nodal, p]
            done = torch.cuda.Event()
            done.record(stream)
            if outs is None:  # pinned result buffers, allocated once outside the timed region
                outs = [[torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in results] for _ in range(2)]
            copy.wait_event(done)
            with torch.cuda.stream(copy):
                for o, t in zip(outs[k % 2], results):
                    t.record_stream(copy)
                    o.copy_(t, non_blocking=True)
        stream.wait_stream(copy)
        return outs

    outs = e2e_run(2)
    d2h = sum(o.numel() * o.element_size() for o in outs[0])
    torch.cuda.synchronize(device)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    copy.wait_stream(stream)
    e2e_steps = max(3, args.steps // 2)
    e2e_run(e2e_steps, outs)
    final = outs[(e2e_steps - 1) % 2]  # the last step's pinned results
    e1.record(stream)
    barrier()
    e2e_elapsed = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, device)

    if rank == 0:
        pk, pk_kind = peaks()
        P = step.tr.rule(step.x).point_count
        faces = sum(np.prod(grid.face_shape(c)) for c in range(3))
        ab = algorithmic_bytes(P, cells.shape[0], X.shape[0], faces)
        dominant, dt = ('p2_spread', spread_t) if spread_t >= gather_t else ('p2_gather_assemble', gather_t)
        byte_key = 'spread' if dominant == 'p2_spread' else 'gather'
        achieved = ab[byte_key] / dt / 1e9
        traffic = load_traffic().get(dominant)
        cpu = None
        errors = None
        if not args.no_cpu_baseline:
            cpu_t, info, outputs = cpu_step_time(grid, X, cells, coef, vel, rhs, fraction=0.05)
            cpu = dict(value=1 / cpu_t, unit='steps/s', cores=1, kind='port',
                       sample=(f'oracle (NumPy restatement) on {info["elements_sampled"]} of {info["elements"]} '
                               f'elements for the transfers (scaled by element count) + full 64^3 MG solve'))
            errors = oracle_errors(step, X, coef, vel, outputs, final[-1].numpy())
        extra = args.rows == 'all'
        mass = mass_pcg_row(X, cells, device, pk['hbm_gbs']) if extra else None
        forms = mg_forms_row(grid, rhs, device) if extra else None
        precision = precision_form_row(grid, X, cells, coef, vel, rhs, device) if extra else None
        if extra:
            precision['p1_128'] = precision_p1_row(device)
        deterministic = deterministic_row(step, coef, device) if extra else None
        batch = batch_form_row(device) if extra else None
        serving = serving_form_row(device) if extra else None
        step_ms = np.array([ev[0].elapsed_time(ev[4]) for ev in phases])
        line = dict(
            metric=METRIC, value=whole_job_rate(world, args.steps, elapsed), unit='steps/s', n_gpus=world, steps=args.steps,
            warmup=args.warmup, ms_per_step=elapsed / args.steps * 1e3, higher_is_better=True, scaling='weak',
            vs_baseline=None, dtype='f64', data='synthetic',
            config=dict(workload='3D P2 shell 38400 elements / 2457600 points, 64^3 MAC, FP64',
                        grid=list(GRID['shape']), elements=int(cells.shape[0]), points=int(P),
                        mg='Neumann V-cycles to 1e-10, Jacobi 2/3 x4, graph-replayed blocks of 2, cycles per solve '
                           f'{sorted(set(step.cycles))}',
                        l2='inputs larger than L2 (590 MB of stencil tables per step)',
                        parallelism=f'replicas x{world}'),
            roofline=dict(bound='hbm', kernel=dominant, achieved=achieved, peak=pk['hbm_gbs'], unit='GB/s',
                          frac=achieved / pk['hbm_gbs'], peak_kind=pk_kind,
                          traffic=(traffic * 1.0 if traffic else None),
                          algorithmic_bytes=ab[byte_key], launch_ms=dt * 1e3,
                          phases_ms=phase_ms),
            e2e=dict(value=whole_job_rate(world, e2e_steps, e2e_elapsed), unit='steps/s', h2d_bytes_per_step=int(h2d),
                     d2h_bytes_per_step=int(d2h)),
            gpu_launches=int(launches),
            clocks=clocks.summary(),
            latency_ms=dict(p50=float(np.percentile(step_ms, 50)), p99=float(np.percentile(step_ms, 99)),
                            mean=float(step_ms.mean())),
            oracle_error=errors,
            mass_pcg=mass,
            mg_forms=forms,
            precision_form=precision,
            deterministic_spread=deterministic,
            batch_form=batch,
            serving_form=serving,
            cpu_baseline=cpu)
        print(json.dumps(line, default=_json))
    if dist:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == 'reference':
        run_reference(args)
    elif args.rows == 'p1':
        print(json.dumps(precision_p1_row(torch.device('cuda', torch.cuda.current_device())), default=_json))
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
