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
WORKLOAD = '3D P2 shell 38400 elements / 2457600 points, 64^3 MAC, FP64'


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=50)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='b200', choices=('b200', 'reference'))
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--form', default='table-free', choices=('table-free', 'tables'),
                    help="transfer form of the headline step: 'table-free' (the transfer kernels form the stencil "
                         "rows) or 'tables' (the prepare writes the stencil tables; for profiler runs of the table "
                         "kernels)")
    ap.add_argument('--rows', default='all', choices=('all', 'step', 'p1', 'batch', 'p1free', 'stokes', 'det'),
                    help="'step': the headline step line only, without the mass-solve, MG-form, batching and "
                         "serving rows (for profiler runs); 'p1': only the precision-form row on the 128^3 P1 "
                         "configuration, printed as its own JSON object (for profiler runs); 'batch': only "
                         "`--steps` replays of the refined batch step after `--warmup`, summarised as JSON "
                         "(for profiler runs); 'p1free': `--steps` matrix-free P1 steps of the 128^3 "
                         "configuration (FP64 transfers, FP64 V-cycles); 'stokes': `--steps` FGMRES Stokes "
                         "solves of the 64^3 row (for profiler runs); 'det': the deterministic-transfer row of "
                         "the headline workload with `--steps` calls of each form (for profiler runs)")
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
    """Device-resident inputs; one call = one hot-path step.

    form: 'table-free' (the transfer kernels form each point's position, bases
    and weights themselves; the prepare selects and checks the rule) or
    'tables' (the prepare writes the (2,P,3) / (2,P,3,4) stencil tables that the
    spread and gather-assemble read back, the reference's P2 transfer)."""

    def __init__(self, grid, X, cells, coef, vel, rhs, device, form='table-free'):
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
        self.form = form
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
        x = self.x if x is None else x
        deferred = self.tr.prepare_table_free(x) if self.form == 'table-free' else self.tr.prepare_deferred(x)
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
        # the solve is queued without its host read (GeometricMultigrid.solve_deferred, as the
        # end-to-end loop runs it), so the step's end event marks the end of the device work
        pending = self.mg.solve_deferred(self.rhs if rhs is None else rhs)
        if ev is not None:
            ev[4].record()
        p, info = pending.result()
        confirmed = self.tr.confirm(deferred)
        if confirmed is not st:
            st = confirmed
            fields = self.p2t.spread(self.tr, coef, st)
            nodal = self.p2t.assemble_velocity(self.tr, vel, st)
        self.cycles.append(info['cycles'])
        return st, fields, nodal, p

    def launch(self, x, coef, vel, rhs):
        """The step's device work with no host read (the end-to-end loop):
        the prepare, the transfers and the pressure solve are queued, and
        ``finish`` makes the step's host reads later, after the next step has
        been queued."""
        deferred = self.tr.prepare_table_free(x) if self.form == 'table-free' else self.tr.prepare_deferred(x)
        st = deferred.stencil
        fields = self.p2t.spread(self.tr, coef, st)
        nodal = self.p2t.assemble_velocity(self.tr, vel, st)
        self.tr.note_transfers(deferred)
        pending = self.mg.solve_deferred(rhs)
        return dict(deferred=deferred, st=st, fields=fields, nodal=nodal, pending=pending)

    def finish(self, h):
        """The host half of a launched step: the solve's checks and cycle
        count, and the rule confirmation (a changed rule, never on this
        workload, would need the transfers again and is an error here)."""
        p, info = h['pending'].result()
        if self.tr.confirm(h['deferred']) is not h['st']:
            raise RuntimeError('the interaction rule changed inside the end-to-end loop')
        self.cycles.append(info['cycles'])
        return p


def algorithmic_bytes_table_free(points, elements, nodes, faces, s=8):
    """Bytes a table-free transfer launch must move at minimum: node
    positions and element connectivity (3*s per node, 80 per element), W
    (s per point), the rule tables (negligible), the nodal values (3*s per
    node) and the face field read and written (2*s per face; the gather reads
    it once and writes the nodal rhs, 3*s per node)."""
    common = nodes * 3 * s + elements * 80 + points * s + nodes * 3 * s
    return dict(spread=common + 2 * faces * s, gather=common + faces * s + nodes * 3 * s)


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


def _time_replays(b, replays, device):
    stream = torch.cuda.current_stream(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b.replay()
    torch.cuda.synchronize(device)
    e0.record(stream)
    for _ in range(replays):
        b.replay()
    e1.record(stream)
    torch.cuda.synchronize(device)
    return e0.elapsed_time(e1) / replays


def batch_form_row(device, count=64, replays=20, oracle_instances=6):
    """Batching form at the FP64 bar: 64 seeded 2D channel instances (grids
    128x32 .. 512x128, 5k-40k leaflet points each, N(0,1) forces).  One batch
    step: one prepare, spread and gather launch for all instances (FP64
    positions, weights and transfers; a captured graph), then the pressure of
    every instance to its own 1e-10 relative residual: batched FP32 Jacobi
    V-cycles inside batched FP64 iterative refinement, the loop on the device
    (one graph, WHILE node), cycles per refinement chosen by the autotuner.
    The plain FP64 drop-in on the same GPU steps the same instances one at a
    time through the single-instance API: prepare2d with its support check,
    spread2d, gather2d, and ChannelMultigrid.solve to 1e-10 (FP64 V-cycles,
    graph-replayed blocks).  Both sides report cycles to tolerance.  Errors:
    max |batch - plain| / max |plain| per output over all instances, and
    against the FP64 oracle (transfers and the channel solve to 1e-10) on
    `oracle_instances` instances.  The same step with FP32 weights and
    transfers is reported beside it with its (larger) errors."""
    from afsi_gpu_b200 import cuda_ib
    from afsi_gpu_b200.batch import seeded_batch
    from afsi_gpu_b200.multigrid import ChannelMultigrid
    from oracle import ib as oib, mg as omg
    b = seeded_batch(count, seed=0, device=device, transfer_dtype=torch.float64)
    schedule, table = b.autotune_refined()
    ms = _time_replays(b, replays, device)
    b.check()
    rep = b.refined_report()
    launches = b.graph_launches + b.refinement().launches(schedule.cycles)
    # plain FP64 drop-in, one instance at a time, each solved to its tolerance
    plain = [ChannelMultigrid(g, device=device, backend='b200-graph') for g in b.grids]
    x = [b.x[b.point_offsets[i]:b.point_offsets[i + 1]] for i in range(count)]
    f = [b.force[b.point_offsets[i]:b.point_offsets[i + 1]] for i in range(count)]
    vel = [(b.u_in[b.u_offsets[i]:b.u_offsets[i + 1]].view(g.face_shape(0)),
            b.v_in[b.v_offsets[i]:b.v_offsets[i + 1]].view(g.face_shape(1))) for i, g in enumerate(b.grids)]

    def plain_step():
        out = []
        for i, g in enumerate(b.grids):
            st = cuda_ib.prepare2d(g, x[i])
            fields = cuda_ib.spread2d(g, f[i], st)
            gathered = cuda_ib.gather2d(vel[i], st)
            p, info = plain[i].solve(b.rhs64[i])
            out.append((fields, gathered, p, info['cycles']))
        return out

    plain_step()
    stream = torch.cuda.current_stream(device)
    torch.cuda.synchronize(device)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    p0.record(stream)
    for _ in range(reps):
        res = plain_step()
    p1.record(stream)
    torch.cuda.synchronize(device)
    plain_ms = p0.elapsed_time(p1) / reps

    def vs_plain(bb):
        return dict(spread=max(max(rel_err(bb.fields(i)[c].cpu(), res[i][0][c].cpu()) for c in range(2))
                               for i in range(count)),
                    interpolate=max(rel_err(bb.velocities(i).cpu(), res[i][1].cpu()) for i in range(count)),
                    pressure=max(rel_err(bb.pressure(i).cpu(), res[i][2].cpu()) for i in range(count)))

    err_plain = vs_plain(b)
    # against the FP64 oracle on a few instances spread over the batch
    picks = sorted(set(int(k) for k in np.linspace(0, count - 1, oracle_instances)))
    eo = dict(spread=0., interpolate=0., pressure=0.)
    for i in picks:
        g = b.grids[i]
        ids, w = oib.prepare2d(x[i].cpu().numpy(), g.shape, g.spacing)
        ff, vv = f[i].cpu().numpy(), [v.cpu().numpy() for v in vel[i]]
        for c in range(2):
            eo['spread'] = max(eo['spread'], rel_err(b.fields(i)[c].reshape(-1).cpu(),
                                                     oib.indexed_spread(ff[:, c], ids[c], w[c], vel[i][c].numel(),
                                                                        g.volume)))
            eo['interpolate'] = max(eo['interpolate'], rel_err(b.velocities(i)[:, c].cpu(),
                                                               oib.indexed_gather(vv[c], ids[c], w[c])))
        pref, _ = omg.solve(omg.Hierarchy(g.shape, g.spacing, 'channel'), b.rhs64[i].cpu().numpy())
        eo['pressure'] = max(eo['pressure'], rel_err(b.pressure(i).cpu(), pref))
    eo['instances'] = picks
    # the FP32-transfer variant of the same step (does not meet 1e-8)
    b32 = seeded_batch(count, seed=0, device=device, transfer_dtype=torch.float32)
    s32, _ = b32.autotune_refined()
    ms32 = _time_replays(b32, replays, device)
    err32 = vs_plain(b32)
    meets = max(err_plain.values()) <= 1e-8 and max(v for k, v in eo.items() if k != 'instances') <= 1e-8
    return dict(instances=count, points=b.total, faces=b.nu + b.nv,
                form='FP64 transfers; batched FP32 V-cycles in batched FP64 refinement to 1e-10 per instance',
                schedule=dict(cycles_per_refinement=schedule.cycles, refinements=rep['refinements'],
                              vcycles=schedule.vcycles),
                ms_per_batch_step=ms, instance_steps_per_s=count / (ms / 1e3),
                cycles_to_tolerance=dict(batch=sorted(set(c for c in rep['cycles_to_tolerance'] if c is not None)),
                                         plain_fp64=sorted(set(r[3] for r in res))),
                unconverged=rep['unconverged'], worst_relative_residual=rep['worst_relative_residual'],
                plain_fp64_ms_per_batch=plain_ms, plain_fp64_instance_steps_per_s=count / (plain_ms / 1e3),
                speedup_vs_plain_fp64=plain_ms / ms, meets_1e_8=bool(meets),
                error_vs_plain_fp64=err_plain, error_vs_fp64_oracle=eo,
                launches_per_step=int(launches), autotune=table,
                fp32_transfers=dict(ms_per_batch_step=ms32, speedup_vs_plain_fp64=plain_ms / ms32,
                                    cycles_per_refinement=s32.cycles, error_vs_plain_fp64=err32,
                                    meets_1e_8=bool(max(err32.values()) <= 1e-8)))


STOKES = dict(dt=1e-3, rho=1., mu=.01)


def stokes_row(grid, device, solves=5):
    """Config 2's Stokes solve, timed as its own row: the CN saddle point
    H u + (dt/rho) G p = b, D u = 0 on the 64^3 grid (dt 1e-3, rho 1, mu 0.01:
    14 Helmholtz sweeps per solve), b a seeded divergence-free face field (the
    discrete curl of random edge potentials), solved by MG-preconditioned
    FGMRES to the reference's acceptance test (restart 20, preconditioner
    multigrid to 0.01).  FP64, and the precision form (FP32 preconditioner
    inside the FP64 FGMRES).  CUDA events around `solves` solves after one
    warm-up solve; CPU: the oracle's FGMRES (NumPy, one process), one solve;
    errors against the oracle's solution."""
    from afsi_gpu_b200 import synthetic
    from afsi_gpu_b200.stokes_fgmres import CNStokes
    from oracle import stokes as ostokes, mg as omg
    b = synthetic.divergence_free_faces(grid, seed=8)
    bd = tuple(t.to(device) for t in b)
    stream = torch.cuda.current_stream(device)
    P = ostokes.StokesProblem(grid.shape, grid.spacing, STOKES['dt'], STOKES['rho'], STOKES['mu'],
                              omg.Hierarchy(grid.shape, grid.spacing, 'neumann'))
    t0 = time.perf_counter()
    u_ref, p_ref, oinfo = ostokes.fgmres_solve(P, [t.numpy() for t in b])
    cpu_s = time.perf_counter() - t0
    out = dict(workload='64^3 MAC, CN saddle point, divergence-free seeded RHS, dt 1e-3 rho 1 mu 0.01',
               cpu_baseline=dict(ms_per_solve=cpu_s * 1e3, cores=1, kind='port',
                                 sample='one whole FGMRES solve of the oracle (NumPy restatement)',
                                 iterations=oinfo['iterations'], poisson_solves=oinfo['poisson_solves']))
    for precision in ('fp64', 'fp32-preconditioner'):
        flow = CNStokes(grid, device=device, precision=precision, **STOKES)
        res = flow.stokes(bd)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(solves):
            res = flow.stokes(bd)
        e1.record(stream)
        torch.cuda.synchronize(device)
        ms = e0.elapsed_time(e1) / solves
        st, pr = res.diagnostics['stokes'], res.diagnostics['pressure']
        err = dict(velocity=max(rel_err(res.velocity[c].cpu(), u_ref[c]) for c in range(3)),
                   pressure=rel_err(res.pressure.cpu(), p_ref))
        out[precision] = dict(ms_per_solve=ms, solves_per_s=1e3 / ms, iterations=st['iterations'],
                              operator_actions=st['operator_actions'], poisson_solves=pr['poisson_solves'],
                              v_cycles=pr['cycles'], helmholtz_sweeps_per_solve=st['helmholtz_iterations'],
                              momentum=[st['momentum_residual'], st['momentum_tolerance']],
                              divergence=[st['divergence_norm'], st['divergence_tolerance']],
                              error_vs_oracle=err, meets_1e_8=bool(max(err.values()) <= 1e-8),
                              speedup_vs_cpu_oracle=cpu_s * 1e3 / ms)
    out['fp32-preconditioner']['speedup_vs_fp64'] = out['fp64']['ms_per_solve'] / \
        out['fp32-preconditioner']['ms_per_solve']
    return out


def config1_row(device, steps=50, cpu_reps=5):
    """Config 1, the plain method: 2D 256x64 MAC on a 1.0 x 0.25 box (h =
    1/256), periodic in x with walls in y, FP64.  20,000 points on the
    centred ellipse with semi-axes 0.3 and 0.1 and radial jitter U(-0.2h,
    0.2h); N(0,1) point forces; a face velocity of 8 seeded Fourier modes; a
    mean-free N(0,1) pressure right-hand side.  One step: the prepare with its
    support screen, one IB_4 spread, one IB_4 interpolate and the multigrid
    solve to 1e-10 relative residual.  GPU: CUDA events around `steps` steps
    after 5 warm-up steps.  CPU: the oracle (NumPy, one process), median of
    `cpu_reps` steps.  Errors against the oracle's outputs."""
    from afsi_gpu_b200 import cuda_ib, synthetic
    from afsi_gpu_b200.grid import ChannelGrid
    from afsi_gpu_b200.multigrid import ChannelMultigrid
    from oracle import ib as oib, mg as omg
    grid = ChannelGrid((256, 64), (1., .25), periodic=True)
    pts = synthetic.ellipse_points(20000, spacing=1 / 256, seed=3)
    force = np.random.default_rng(5).standard_normal((20000, 2))
    vel = [v.numpy() for v in synthetic.fourier_velocity2d(grid, seed=2)]
    rhs = synthetic.mean_free_normal(grid.shape, seed=6).numpy()
    x, fd = torch.as_tensor(pts, device=device), torch.as_tensor(force, device=device)
    vd, rd = tuple(torch.as_tensor(v, device=device) for v in vel), torch.as_tensor(rhs, device=device)
    mg = ChannelMultigrid(grid, device=device, backend='b200-graph')

    def step():
        st = cuda_ib.prepare2d(grid, x)
        return cuda_ib.spread2d(grid, fd, st), cuda_ib.gather2d(vd, st), mg.solve(rd)

    for _ in range(5):
        out = step()
    stream = torch.cuda.current_stream(device)
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        out = step()
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1) / steps
    h = omg.Hierarchy(grid.shape, grid.spacing, 'periodic')
    times = []
    for _ in range(cpu_reps):
        t0 = time.perf_counter()
        ids, w = oib.prepare2d(pts, grid.shape, grid.spacing)
        sp = [oib.indexed_spread(force[:, c], ids[c], w[c], vel[c].size, grid.volume) for c in range(2)]
        ga = np.stack([oib.indexed_gather(vel[c], ids[c], w[c]) for c in range(2)], -1)
        pref, info = omg.solve(h, rhs)
        times.append(time.perf_counter() - t0)
    fields, gathered, (p, ginfo) = out
    return dict(workload='2D 256x64 MAC (1.0 x 0.25), periodic x / walls y, 20,000 ellipse points, FP64',
                steps_per_s=1e3 / ms, ms_per_step=ms, cycles=ginfo['cycles'], cycles_oracle=info['cycles'],
                residual=ginfo['residual_norm'], tolerance=ginfo['tolerance'],
                cpu_baseline=dict(steps_per_s=1 / float(np.median(times)), ms_per_step=float(np.median(times)) * 1e3,
                                  cores=1, kind='port', sample=f'whole step, median of {cpu_reps}'),
                error_vs_oracle=dict(spread=max(rel_err(fields[c].reshape(-1).cpu(), sp[c]) for c in range(2)),
                                     interpolate=rel_err(gathered.cpu(), ga), pressure=rel_err(p.cpu(), pref)))


def serving_form_row(device, count=400):
    """Serving form: `count` requests of the serving mix (50% 2D 256x64 with
    20k points, 35% 3D 32^3-64^3 with 50k-400k points, 15% 3D 96^3 with 800k
    points; Poisson arrivals at 2000/s, seeded), each a full step to the FP64
    tolerance on resident states: inputs (made before the clock starts, in
    pinned host memory) copied in, prepare, spread, interpolate and pressure
    solve, interpolated velocity and pressure copied back.  The server
    admits under a 150 GB budget, batches the 2D requests that are waiting
    when its 2D lane frees up (up to 8 per batch) and runs the 3D requests on
    4 lanes with their own streams.  Both precisions (FP64 V-cycles; FP32
    V-cycles inside FP64 refinement, batched for 2D), and the plain drop-in
    serving one request at a time for comparison; then the refined form
    below saturation (a quarter and a half of its saturated throughput)."""
    from afsi_gpu_b200.serving import Request, Server, mix, with_inputs
    reqs = with_inputs(mix(count, rate=2000., seed=0))
    out = {}
    for precision in ('fp64', 'fp32-refined'):
        server = Server(device=device, slots=4, batch=8, precision=precision)
        server.warm(reqs)
        server.serve(reqs[:16])  # warm-up
        report, _ = server.serve(reqs)
        out[precision] = report
    one = Server(device=device, slots=1, batch=1, precision='fp64')
    one.warm(reqs)
    t0 = time.perf_counter()
    for r in reqs:
        one.alone(r)
    wall = time.perf_counter() - t0
    out['one_at_a_time_fp64'] = dict(requests=len(reqs), wall_s=wall, steps_per_s=len(reqs) / wall,
                                     note='plain FP64 drop-in, each request alone, no batching or overlap')
    out['speedup_fp32_refined_vs_one_at_a_time'] = out['fp32-refined']['steps_per_s'] / (len(reqs) / wall)
    out['speedup_fp64_vs_one_at_a_time'] = out['fp64']['steps_per_s'] / (len(reqs) / wall)
    # 2000 req/s saturates the GPU (latency there is queueing); the same mix
    # at a quarter and a half of the refined form's saturated throughput shows
    # the step latency itself and the knee where queueing starts
    server = Server(device=device, slots=4, batch=8, precision='fp32-refined')
    below = mix(count // 2, rate=1., seed=1)
    made = with_inputs(below)
    server.warm(made)
    server.serve([Request(0., r.rid, r.kind, r.n, r.points, r.seed, r.inputs) for r in made[:16]])  # warm-up
    for key, share in (('fp32_refined_quarter_saturation', .25), ('fp32_refined_half_saturation', .5)):
        rate = share * out['fp32-refined']['steps_per_s']
        timed = mix(count // 2, rate=rate, seed=1)
        report, _ = server.serve([Request(t.arrival, r.rid, r.kind, r.n, r.points, r.seed, r.inputs)
                                  for t, r in zip(timed, made)])
        out[key] = dict(report, arrival_rate=rate)
    return out


def precision_form_row(grid, X, cells, coef, vel, rhs, device, oracle_out=None, steps=20):
    """Precision forms of the step on the bench workload, each timed with CUDA
    events around `steps` steps beside the plain FP64 step: FP64 positions and
    bases always; weight tables and transfers in FP64 or FP32; the pressure
    solve as FP64 V-cycles or as FP32 V-cycles inside FP64 iterative
    refinement, always to the FP64 tolerance.  Errors are max |form - oracle| /
    max |oracle| against the full-size FP64 oracle outputs (or, without them,
    against the GPU FP64 step), and meets_1e_8 says whether every output is
    within 1e-8."""
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
    stream = torch.cuda.current_stream(device)

    def step(tr, mg, c, v):
        st = tr.prepare(x)
        return tr.spread(c, st), tr.assemble_velocity(v, st), mg.solve(r64)

    def timed(*args):
        for _ in range(3):
            out = step(*args)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        for _ in range(steps):
            out = step(*args)
        e1.record(stream)
        torch.cuda.synchronize(device)
        return out, e0.elapsed_time(e1) / steps

    plain, plain_ms = timed(tr64, mg64, c64, v64)
    if oracle_out is not None:
        ref = ([np.asarray(f) for f in oracle_out['fields']], oracle_out['nodal'], oracle_out['p'])
        against = 'full-size FP64 oracle'
    else:
        ref = ([f.cpu() for f in plain[0]], plain[1].cpu(), plain[2][0].cpu())
        against = 'GPU FP64 step'

    def errors(out):
        return dict(spread=max(rel_err(a.cpu(), b) for a, b in zip(out[0], ref[0])),
                    gather_assemble=rel_err(out[1].cpu(), ref[1]), pressure=rel_err(out[2][0].cpu(), ref[2]))

    rows = dict(plain_fp64=dict(steps_per_s=1e3 / plain_ms, ms_per_step=plain_ms, error_vs_oracle=errors(plain)))
    for name, tr, mg, c, v in (('fp64_transfers_refined_mg', tr64, mg32, c64, v64),
                               ('fp32_transfers_refined_mg', tr32, mg32, c32, v32),
                               ('fp32_transfers_fp64_mg', tr32, mg64, c32, v32)):
        out, ms = timed(tr, mg, c, v)
        info = out[2][1]
        err = errors(out)
        rows[name] = dict(steps_per_s=1e3 / ms, ms_per_step=ms, speedup_vs_plain_fp64=plain_ms / ms,
                          transfer_dtype='f64' if tr is tr64 else 'f32', positions='f64',
                          mg=(f"FP32 V-cycles in FP64 refinement, {info['refinements']} refinements, "
                              f"{info['cycles']} FP32 cycles" if 'refinements' in info else
                              f"FP64 V-cycles, {info['cycles']} cycles"),
                          residual=info['residual_norm'], tolerance=info['tolerance'],
                          error_vs_oracle=err, meets_1e_8=bool(max(err.values()) <= 1e-8))
    rows['errors_against'] = against
    return rows


P1_SHELL = dict(nr=2, ntheta=80, nphi=160, outer=(.224, .154, .154), inner=(.214, .144, .144))


def precision_p1_row(device, steps=5):
    """Config 3 on its own configuration: 128^3 MAC grid, a thin P1
    tetrahedral prolate shell (128,000 elements, about 1.1 M adaptive
    interaction points at density 2), seeded uniform nodal forces in [-1, 1],
    a seeded Fourier face velocity and a mean-free N(0,1) pressure RHS.  A step
    is the P1 prepare, the spread, the interpolate and the pressure solve to
    the FP64 tolerance (1e-10).  Forms:
      csr_fp64:          the assembled-operator drop-in (CSR contraction and
                         SpMVs, FP64) with FP64 V-cycles;
      matrix_free_fp64:  the matrix-free element transfer (rows formed in the
                         kernels, no operator, FP64) with FP64 V-cycles;
      matrix_free_fp64_refined_mg: the same transfers, FP32 V-cycles inside FP64
                         refinement (meets the FP64 bar);
      precision_form:    matrix-free FP32 weights and transfers beside FP64
                         positions, FP32 V-cycles inside FP64 refinement.
    CUDA events around each of `steps` steps after one untimed step, the
    median reported; errors against the FP64 oracle (transfers on an element
    sample, the pressure on the full grid)."""
    from afsi_gpu_b200 import synthetic
    from afsi_gpu_b200.grid import MACGrid
    from afsi_gpu_b200.multigrid import GeometricMultigrid, RefinedMultigrid
    from afsi_gpu_b200.p1_csr import P1CSRTransfer
    from afsi_gpu_b200.p2_cuda_transfer import P1Transfer
    grid = MACGrid((128, 128, 128), (1., 1., 1.))
    X, cells = synthetic.prolate_shell(**P1_SHELL)
    rng = np.random.default_rng(21)
    x = torch.as_tensor(X, device=device)
    cells_t = torch.as_tensor(cells, device=device)
    c64 = torch.as_tensor(rng.uniform(-1., 1., (X.shape[0], 3)), device=device)
    v64 = tuple(v.to(device) for v in synthetic.fourier_velocity3d(grid, seed=21))
    r64 = synthetic.mean_free_normal(grid.shape, seed=21).to(device)
    c32, v32 = c64.float(), tuple(v.float() for v in v64)
    mg64 = GeometricMultigrid(grid, device=device, backend='b200-graph')
    mg32 = RefinedMultigrid(grid, device=device)
    stream = torch.cuda.current_stream(device)

    def csr_step(tr, mg, c, v):
        st = tr.prepare(x)
        return tr.spread(c, st), tr.interpolate_rhs(v, st), mg.solve(r64), st

    def free_step(tr, mg, c, v):
        # rule and support confirmed after the solve's own host read; a changed
        # rule (never on this workload) redoes the transfers
        deferred = tr.prepare_deferred(x)
        st = deferred.stencil
        f, r, p = tr.spread(c, st), tr.interpolate_rhs(v, st), mg.solve(r64)
        confirmed = tr.confirm(deferred)
        if confirmed is not st:
            st = confirmed
            f, r = tr.spread(c, st), tr.interpolate_rhs(v, st)
            tr.check(st)
        return f, r, p, st

    def timed(step, *args):
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

    budget = dict(max_entries=400_000_000)
    forms = {}
    csr, ms_csr = timed(csr_step, P1CSRTransfer(grid, x, cells_t, **budget), mg64, c64, v64)
    forms['csr_fp64'] = (csr, ms_csr, None)
    free64 = P1Transfer(grid, x, cells_t)
    free32 = P1Transfer(grid, x, cells_t, transfer_dtype=torch.float32)
    for name, tr, mg, c, v, dt in (('matrix_free_fp64', free64, mg64, c64, v64, None),
                                   ('matrix_free_fp64_refined_mg', free64, mg32, c64, v64, None),
                                   ('precision_form', free32, mg32, c32, v32, torch.float32)):
        out, ms = timed(free_step, tr, mg, c, v)
        forms[name] = (out, ms, dt)
    oracle = p1_oracle_errors(grid, X, cells, c64, v64, r64, device,
                              {name: (out[2][0], dt) for name, (out, _, dt) in forms.items()},
                              transfer={'csr_fp64': 'csr'})
    rows = {}
    for name, (out, ms, dt) in forms.items():
        info = out[2][1]
        rows[name] = dict(steps_per_s=1e3 / ms, ms_per_step=ms, speedup_vs_csr_fp64=ms_csr / ms,
                          transfer_dtype='f32' if dt is not None else 'f64',
                          mg=(f"FP32 V-cycles in FP64 refinement, {info['refinements']} refinements, "
                              f"{info['cycles']} FP32 cycles" if 'refinements' in info else
                              f"FP64 V-cycles, {info['cycles']} cycles"),
                          residual=info['residual_norm'], tolerance=info['tolerance'],
                          error_vs_oracle=oracle[name])
    rows['matrix_free_fp64']['speedup_vs_matrix_free_fp64'] = 1.
    base = forms['matrix_free_fp64'][1]
    for name in ('matrix_free_fp64_refined_mg', 'precision_form'):
        rows[name]['speedup_vs_matrix_free_fp64'] = base / forms[name][1]
    st = csr[3]
    return dict(workload=(f'128^3 MAC, P1 prolate shell {cells.shape[0]} elements / '
                          f'{st.rule.point_count} points, uniform [-1,1] forces'),
                points=int(st.rule.point_count), elements=int(cells.shape[0]),
                csr_nnz=int(st.assembly['total_nnz']), oracle_sample=oracle['sample'], **rows)


def p1_oracle_errors(grid, X, cells, coef, vel, rhs, device, forms, sample_elements=2000, transfer=None):
    """Errors of the P1 forms against the FP64 oracle.  Transfers on an
    element sample (every k-th element of the shell, so the sample spans it):
    the form's transfer built on the sampled cells alone, its spread and
    interpolate against the oracle's P1 quadrature transfer with the same rule
    (x_q = N x, F_q = (N coef) W, spread over the shared tables, U_q gathered
    and assembled with N W).  Pressure: the full 128^3 oracle solve to 1e-10.
    forms: name -> (pressure from the timed step, transfer dtype or None);
    transfer: name -> 'csr' for the assembled-operator forms (default: the
    matrix-free transfer)."""
    from afsi_gpu_b200.p1_csr import P1CSRTransfer
    from afsi_gpu_b200.p2_cuda_transfer import P1Transfer
    transfer = transfer or {}
    from oracle import ib as oib, mg as omg
    k = max(1, cells.shape[0] // sample_elements)
    sub = np.ascontiguousarray(cells[::k][:sample_elements])
    x = torch.as_tensor(X, device=device)
    pref, _ = omg.solve(omg.Hierarchy(grid.shape, grid.spacing, 'neumann'), rhs.cpu().numpy())
    coef_np = coef.cpu().numpy()
    vel_np = [v.cpu().numpy() for v in vel]
    out = dict(sample=f'transfers on {sub.shape[0]} of {cells.shape[0]} elements (every {k}th); '
                      f'pressure on the full grid')
    oracle_ref = None
    for name, (p, dtype) in forms.items():
        kw = {} if dtype is None else dict(transfer_dtype=dtype)
        cls = P1CSRTransfer if transfer.get(name) == 'csr' else P1Transfer
        tr = cls(grid, x, torch.as_tensor(sub, device=device), **kw)
        st = tr.prepare(x)
        cd = coef if dtype is None else coef.to(dtype)
        vd = vel if dtype is None else tuple(v.to(dtype) for v in vel)
        fields = tr.spread(cd, st)
        nodal = tr.interpolate_rhs(vd, st)
        if oracle_ref is None:
            groups = [(g.cells.cpu().numpy(), g.values.cpu().numpy(), g.weights.cpu().numpy())
                      for g in st.rule.groups]
            base, phi, _ = oib.p2_prepare(X, [(c, N) for c, N, _ in groups], grid.origin, grid.spacing,
                                          grid.shape)
            oracle_ref = (oib.p2_spread(coef_np, groups, base, phi, grid.shape, grid.volume),
                          oib.p2_gather_assemble(vel_np, groups, base, phi, grid.shape, X.shape[0]))
        out[name] = dict(spread=max(rel_err(f.cpu(), o) for f, o in zip(fields, oracle_ref[0])),
                         interpolate=rel_err(nodal.cpu(), oracle_ref[1]), pressure=rel_err(p.cpu(), pref))
        out[name]['meets_1e_8'] = bool(max(out[name].values()) <= 1e-8)
    return out


def table_form_row(grid, X, cells, coef, vel, rhs, device, steps, warmup, pk):
    """The headline step with the stencil tables (the reference's P2 transfer:
    the prepare writes the (2,P,3) / (2,P,3,4) tables, the spread and
    gather-assemble read them back), timed like the headline but without the
    flush (590 MB of tables per step exceed L2): steps/s, the phases, and the
    HBM roofline of its spread and gather-assemble kernels."""
    step = Step(grid, X, cells, coef, vel, rhs, device, form='tables')
    for _ in range(max(warmup, 3)):
        step()
    torch.cuda.synchronize(device)
    evs = []
    for _ in range(steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(9)]
        step(timing=ev)
        evs.append(ev)
    torch.cuda.synchronize(device)
    elapsed = sum(ev[0].elapsed_time(ev[4]) for ev in evs) / 1e3
    names = ('prepare', 'spread', 'gather_assemble', 'mg_solve')
    phase_ms = {n: float(np.mean([ev[i].elapsed_time(ev[i + 1]) for ev in evs])) for i, n in enumerate(names)}
    P = step.tr.rule(step.x).point_count
    faces = sum(np.prod(grid.face_shape(c)) for c in range(3))
    ab = algorithmic_bytes(P, cells.shape[0], X.shape[0], faces)
    traffic = load_traffic()
    out = dict(steps_per_s=steps / elapsed, ms_per_step=elapsed / steps * 1e3, phases_ms=phase_ms)
    for key, name, a, b in (('spread', 'p2_spread', 5, 6), ('gather', 'p2_gather_assemble', 7, 8)):
        dt = float(np.mean([ev[a].elapsed_time(ev[b]) for ev in evs])) / 1e3
        achieved = ab[key] / dt / 1e9
        out[f'roofline_{key}'] = dict(bound='hbm', kernel=name, achieved=achieved, peak=pk['hbm_gbs'], unit='GB/s',
                                      frac=achieved / pk['hbm_gbs'], traffic=traffic.get(name),
                                      algorithmic_bytes=ab[key], launch_ms=dt * 1e3)
    return out


def deterministic_row(step, coef, vel, device, reps=10):
    """The P2 transfers of the step in their deterministic modes (atomic-free,
    bitwise reproducible) beside the atomic ones, CUDA events around `reps`
    calls each.  Table form: the spread over the stencil tables, tile-sorted
    (the plan is built once per stencil, outside the timing).  Table-free
    form: the spread with element boxes in scratch slots reduced per face
    tile in element order, and the gather-assemble with element sums reduced
    per node.  Each deterministic output is computed twice (bitwise equal)
    and compared with the atomic one."""
    from afsi_gpu_b200 import p2_cuda_transfer as p2t
    tr = step.tr
    st = tr.prepare(step.x)
    free = tr.confirm(tr.prepare_table_free(step.x))
    c = torch.as_tensor(coef, device=device)
    v = tuple(torch.as_tensor(x, device=device) for x in vel)
    det = p2t.P2Transfer(step.grid, step.x, step.cells, deterministic=True)
    det.rules = tr.rules
    stream = torch.cuda.current_stream(device)
    out = {}
    runs = (('atomic', lambda: tr.spread(c, st)), ('deterministic', lambda: det.spread(c, st)),
            ('table_free_atomic', lambda: tr.spread(c, free)), ('table_free_deterministic', lambda: det.spread(c, free)),
            ('gather_table_free_atomic', lambda: tr.assemble_velocity(v, free)),
            ('gather_table_free_deterministic', lambda: det.assemble_velocity(v, free)))
    for name, fn in runs:
        ref, first, second = None, fn(), fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(device)
        out[f'{name}_ms'] = e0.elapsed_time(e1) / reps
        out.setdefault('_outputs', {})[name] = (first, second)
    tr.check(free)
    det.check(free)
    outs = out.pop('_outputs')
    as_list = lambda o: list(o) if isinstance(o, (tuple, list)) else [o]
    for name, ref in (('deterministic', 'atomic'), ('table_free_deterministic', 'table_free_atomic'),
                      ('gather_table_free_deterministic', 'gather_table_free_atomic')):
        d, again = (as_list(o) for o in outs[name])
        a = as_list(outs[ref][0])
        out[f'{name}_bitwise_reproducible'] = all(torch.equal(x, y) for x, y in zip(d, again))
        out[f'{name}_max_rel_diff_vs_atomic'] = max(float((x - y).abs().max() / y.abs().max()) for x, y in zip(d, a))
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

class OracleRun:
    """The oracle (NumPy restatement of the reference's CPU path) on the WHOLE
    bench workload per step: the P2 prepare, spread and gather-assemble of all
    elements, split over a spawn pool of single-threaded worker processes (one
    per host core), then the 64^3 multigrid solve in this process.  Used as the
    reference arm, as the GPU arm's CPU baseline, and as the full-size oracle
    the GPU outputs are checked against.  Nothing is sampled or scaled."""

    def __init__(self, grid, X, cells, coef, vel, rhs, workers=None):
        import multiprocessing as mp
        from oracle import mg
        self.workers = workers or max(1, len(os.sched_getaffinity(0)))
        for var in ('OMP_NUM_THREADS', 'OPENBLAS_NUM_THREADS', 'MKL_NUM_THREADS'):
            os.environ[var] = '1'  # inherited by the spawned workers
        from multiprocessing import shared_memory
        self.face_sizes = [int(np.prod(grid.face_shape(c))) for c in range(3)]
        self.nodes = int(X.shape[0])
        self.slot_floats = sum(self.face_sizes) + 3 * self.nodes
        # one output slot per worker task, summed here (no result pickling)
        self.shm = shared_memory.SharedMemory(create=True, size=self.workers * self.slot_floats * 8)
        init = (X, coef, vel, tuple(grid.shape), tuple(grid.lengths), tuple(grid.origin), self.shm.name,
                self.slot_floats)
        # every worker is started up front (a spawn pool: no fork after CUDA)
        self.pool = mp.get_context('spawn').Pool(self.workers, initializer=_oracle_worker_init, initargs=init)
        self.pool.map(_oracle_transfer_chunk, [(k, cells[:8]) for k in range(self.workers)], chunksize=1)
        self.tasks = [(k, cells[c]) for k, c in enumerate(np.array_split(np.arange(cells.shape[0]), self.workers))]
        self.grid = grid
        self.hierarchy = mg.Hierarchy(grid.shape, grid.spacing, 'neumann')
        self.rhs = rhs
        self.elements = int(cells.shape[0])

    def step(self):
        """One oracle step; returns (outputs, phase seconds, step seconds)."""
        from oracle import mg
        t0 = time.perf_counter()
        parts = self.pool.map(_oracle_transfer_chunk, self.tasks, chunksize=1)
        slots = np.ndarray((self.workers, self.slot_floats), dtype=np.float64, buffer=self.shm.buf)
        total = slots.sum(0)
        cut = np.cumsum([0] + self.face_sizes)
        fields = [total[cut[c]:cut[c + 1]].reshape(self.grid.face_shape(c)) for c in range(3)]
        nodal = total[cut[3]:].reshape(self.nodes, 3)
        del slots
        t1 = time.perf_counter()
        p, info = mg.solve(self.hierarchy, self.rhs)
        t2 = time.perf_counter()
        worst = np.max(parts, axis=0)  # slowest worker per phase
        phases = dict(prepare=float(worst[0]), spread=float(worst[1]), gather_assemble=float(worst[2]),
                      transfers_wall=t1 - t0, mg_solve=t2 - t1)
        return dict(fields=fields, nodal=nodal, p=p, cycles=info['cycles']), phases, t2 - t0

    def run(self, steps, warmup):
        times, phases, out = [], [], None
        for i in range(warmup + steps):
            out, ph, dt = self.step()
            if i >= warmup:
                times.append(dt)
                phases.append(ph)
        return out, times, phases

    def close(self):
        self.pool.close()
        self.pool.join()
        self.shm.close()
        self.shm.unlink()

    def sample(self, steps, warmup):
        return (f'oracle (NumPy restatement of the reference CPU path, FP64) on the whole workload every step: '
                f'P2 prepare/spread/gather-assemble of all {self.elements} elements split over {self.workers} '
                f'single-threaded worker processes, then the full 64^3 MG solve to 1e-10; {steps} steps after '
                f'{warmup} warm-up, nothing scaled')


def phase_stats(phases):
    """Median and p90 (ms) of each phase over the timed steps."""
    out = {}
    for k in phases[0]:
        v = np.array([ph[k] for ph in phases]) * 1e3
        out[k] = dict(median_ms=float(np.median(v)), p90_ms=float(np.percentile(v, 90)))
    return out


def rel_err(a, b):
    """max |a - b| / max |b| (FP64)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a.reshape(b.shape) - b).max() / max(np.abs(b).max(), 1e-300))


def oracle_errors(outputs, fields, nodal, p):
    """Errors of the GPU step's outputs against the full-size FP64 oracle."""
    return dict(spread=max(rel_err(f, o) for f, o in zip(fields, outputs['fields'])),
                gather_assemble=rel_err(nodal, outputs['nodal']), mg_solve=rel_err(p, outputs['p']),
                mg_cycles_oracle=int(outputs['cycles']),
                sample='all elements and points of the workload (no sample); max |gpu - oracle| / max |oracle|')


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


def _oracle_worker_init(X, coef, vel, shape, lengths, origin, shm_name, slot_floats):
    """Reference-arm worker set-up: the step's static inputs, the rule tables,
    the oracle import and the shared-memory output slots, once per worker."""
    from multiprocessing import shared_memory
    from afsi_gpu_b200.quadrature import conical_rule, tabulate_p2
    torch.set_num_threads(1)  # one core per worker: the workers are the parallelism
    q, w = conical_rule(4)
    spacing = tuple(L / n for L, n in zip(lengths, shape))
    shm = shared_memory.SharedMemory(name=shm_name)
    _ORACLE.update(X=X, coef=coef, vel=vel, shape=shape, origin=origin, spacing=spacing,
                   volume=float(np.prod(spacing)), N=tabulate_p2(q), w=w, shm=shm, slot_floats=slot_floats)


def _oracle_transfer_chunk(task):
    """One worker's share of an oracle step: the prepare, spread and
    gather-assemble of a chunk of elements, written into output slot `slot`
    of the shared block (top level, so that a spawn pool can call it)."""
    from oracle import ib
    from afsi_gpu_b200.quadrature import reference_determinants
    slot, cells = task
    o = _ORACLE
    t0 = time.perf_counter()
    W = reference_determinants(torch.as_tensor(o['X']), torch.as_tensor(cells)).numpy()[:, None] * o['w']
    base, phi, _ = ib.p2_prepare(o['X'], [(cells, o['N'])], o['origin'], o['spacing'], o['shape'])
    t1 = time.perf_counter()
    fields = ib.p2_spread(o['coef'], [(cells, o['N'], W)], base, phi, o['shape'], o['volume'])
    t2 = time.perf_counter()
    nodal = ib.p2_gather_assemble(o['vel'], [(cells, o['N'], W)], base, phi, o['shape'], o['X'].shape[0])
    t3 = time.perf_counter()
    out = np.ndarray((o['slot_floats'],), dtype=np.float64, buffer=o['shm'].buf, offset=slot * o['slot_floats'] * 8)
    np.concatenate([f.reshape(-1) for f in fields] + [nodal.reshape(-1)], out=out)
    return t1 - t0, t2 - t1, t3 - t2


def run_reference(args):
    dist, rank, world = dist_setup(args)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    grid, X, cells, coef, vel, rhs = workload()
    run = OracleRun(grid, X, cells, coef, vel, rhs)
    try:
        _, times, phases = run.run(args.steps, args.warmup)
    finally:
        run.close()
    step = float(np.mean(times))
    value = 1.0 / step
    sample = run.sample(args.steps, args.warmup)
    line = dict(metric=METRIC, value=value, unit='steps/s', impl='reference', n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=step * 1e3, higher_is_better=True, scaling='weak',
                vs_baseline=None, dtype='f64', data='synthetic', config=dict(workload=WORKLOAD),
                latency_ms=dict(p50=float(np.percentile(times, 50)) * 1e3, p90=float(np.percentile(times, 90)) * 1e3,
                                p99=float(np.percentile(times, 99)) * 1e3),
                phases=phase_stats(phases),
                cpu_baseline=dict(value=value, unit='steps/s', cores=run.workers, kind='port', sample=sample),
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
    step = Step(grid, X, cells, coef, vel, rhs, device, form=args.form)
    stream = torch.cuda.current_stream(device)
    # the table-free step's inputs and fields fit in L2 (126 MB): every timed
    # step starts from a flushed L2 (a 256 MB buffer written just before it,
    # outside the step's events)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=device)

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
            flush.zero_()
            step(timing=ev)
            phases.append(ev)
        stop.record(stream)
        barrier()
    launches = _lib.launch_count() - launches0
    # the K steps' device time, each from the start of its prepare to the end of its solve
    elapsed = max_over_ranks(sum(ev[0].elapsed_time(ev[4]) for ev in phases) / 1e3, dist, device)
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
        """`count` pipelined steps; returns the pinned result buffers.  Step k
        is queued before step k-1's host reads are made, so the device always
        has the next step in its queue."""
        ready = {0: copy_in(0)}
        done = None
        previous = None
        for k in range(count):
            if k + 1 < count:
                if done is not None:
                    copy.wait_event(done)  # step k-1 has finished reading that buffer
                ready[k + 1] = copy_in((k + 1) % 2)
            stream.wait_event(ready.pop(k))
            b = dev_in[k % 2]
            h = step.launch(b['x'], b['coef'], b['vel'], b['rhs'])
            results = list(h['fields']) + [h['nodal'], h['pending'].p]
            done = torch.cuda.Event()
            done.record(stream)
            if outs is None:  # pinned result buffers, allocated once outside the timed region
                outs = [[torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in results] for _ in range(2)]
            copy.wait_event(done)
            with torch.cuda.stream(copy):
                for o, t in zip(outs[k % 2], results):
                    t.record_stream(copy)
                    o.copy_(t, non_blocking=True)
            if previous is not None:
                step.finish(previous)
            previous = h
        step.finish(previous)
        stream.wait_stream(copy)
        return outs

    outs = e2e_run(2)
    d2h = sum(o.numel() * o.element_size() for o in outs[0])
    torch.cuda.synchronize(device)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    copy.wait_stream(stream)
    e2e_steps = max(3, args.steps)  # as many as the device-timed steps: one host stall weighs less
    e2e_run(e2e_steps, outs)
    final = outs[(e2e_steps - 1) % 2]  # the last step's pinned results
    e1.record(stream)
    barrier()
    e2e_elapsed = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, device)

    if rank == 0:
        pk, pk_kind = peaks()
        P = step.tr.rule(step.x).point_count
        faces = sum(np.prod(grid.face_shape(c)) for c in range(3))
        free = args.form == 'table-free'
        ab = (algorithmic_bytes_table_free if free else algorithmic_bytes)(P, cells.shape[0], X.shape[0], faces)
        names = ('p2_fused_spread', 'p2_fused_gather_assemble') if free else ('p2_spread', 'p2_gather_assemble')
        dominant, dt = (names[0], spread_t) if spread_t >= gather_t else (names[1], gather_t)
        byte_key = 'spread' if dominant == names[0] else 'gather'
        achieved = ab[byte_key] / dt / 1e9
        traffic = load_traffic().get(dominant)
        cpu = None
        errors = None
        oracle_out = None
        if not args.no_cpu_baseline:
            # the reference arm's measurement on a bounded number of steps; its
            # outputs are the full-size FP64 oracle for the error check
            run = OracleRun(grid, X, cells, coef, vel, rhs)
            try:
                oracle_out, cpu_times, cpu_phases = run.run(2, 1)
            finally:
                run.close()
            cpu = dict(value=1 / float(np.mean(cpu_times)), unit='steps/s', cores=run.workers, kind='port',
                       sample=run.sample(2, 1), phases=phase_stats(cpu_phases))
            errors = oracle_errors(oracle_out, [t.numpy() for t in final[:3]], final[3].numpy(), final[4].numpy())
        extra = args.rows == 'all'
        mass = mass_pcg_row(X, cells, device, pk['hbm_gbs']) if extra else None
        forms = mg_forms_row(grid, rhs, device) if extra else None
        precision = precision_form_row(grid, X, cells, coef, vel, rhs, device, oracle_out) if extra else None
        if extra:
            precision['p1_128'] = precision_p1_row(device)
        deterministic = deterministic_row(step, coef, vel, device) if extra else None
        tables = table_form_row(grid, X, cells, coef, vel, rhs, device, args.steps, args.warmup, pk) if extra else None
        batch = batch_form_row(device) if extra else None
        config1 = config1_row(device) if extra else None
        stokes = stokes_row(grid, device) if extra else None
        serving = serving_form_row(device) if extra else None
        step_ms = np.array([ev[0].elapsed_time(ev[4]) for ev in phases])
        line = dict(
            metric=METRIC, value=whole_job_rate(world, args.steps, elapsed), unit='steps/s', n_gpus=world, steps=args.steps,
            warmup=args.warmup, ms_per_step=elapsed / args.steps * 1e3, higher_is_better=True, scaling='weak',
            vs_baseline=None, dtype='f64', data='synthetic',
            config=dict(workload=WORKLOAD,
                        grid=list(GRID['shape']), elements=int(cells.shape[0]), points=int(P),
                        mg='Neumann V-cycles to 1e-10, Jacobi 2/3 x4, graph-replayed blocks of 2, cycles per solve '
                           f'{sorted(set(step.cycles))}',
                        transfers=('table-free: the spread and gather-assemble kernels form each point\'s position, '
                                   'bases and IB_4 weights from the nodal positions (no stencil tables); the prepare '
                                   'selects and checks the rule' if free else
                                   'tables: the prepare writes the (2,P,3) bases and (2,P,3,4) weights that the spread '
                                   'and gather-assemble read back'),
                        l2='L2 flushed before every timed step (256 MB written outside the step\'s events)',
                        parallelism=f'replicas x{world}'),
            roofline=dict(bound='hbm', kernel=dominant, achieved=achieved, peak=pk['hbm_gbs'], unit='GB/s',
                          frac=achieved / pk['hbm_gbs'], peak_kind=pk_kind,
                          traffic=(traffic * 1.0 if traffic else None),
                          algorithmic_bytes=ab[byte_key], launch_ms=dt * 1e3,
                          phases_ms=phase_ms,
                          note='the table-free kernels move about 40 MB per launch and are bound by FP64 issue and '
                               'latency, not HBM; the table form (the same step with stencil tables, '
                               'table_form_step) carries the HBM-bound roofline of its spread'),
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
            table_form_step=tables,
            batch_form=batch,
            config1=config1,
            stokes_fgmres=stokes,
            serving_form=serving,
            cpu_baseline=cpu)
        print(json.dumps(line, default=_json))
    if dist:
        dist.destroy_process_group()


def batch_only(args):
    """Replays of the refined batch step (64 instances, FP64 transfers, 5
    V-cycles per refinement) for profiler runs."""
    from afsi_gpu_b200.batch import Schedule, seeded_batch
    device = torch.device('cuda', torch.cuda.current_device())
    b = seeded_batch(64, seed=0, device=device, transfer_dtype=torch.float64)
    b.use(Schedule(streams=1, order='given', smoother='jacobi', cycles=5, vcycles='batched', refined=True))
    for _ in range(args.warmup):
        b.replay()
    ms = _time_replays(b, args.steps, device)
    rep = b.refined_report()
    # the same refinement kernels once more, launched one by one from the host
    # (profilers cannot look inside a graph that holds a conditional node)
    b.refinement().run_launched(5)
    torch.cuda.synchronize(device)
    print(json.dumps(dict(ms_per_batch_step=ms, refinements=rep['refinements'], unconverged=rep['unconverged'],
                          launches_per_step=b.graph_launches + b.refinement().launches(5))))


def p1free_only(args):
    """Matrix-free P1 steps of the 128^3 configuration for profiler runs."""
    from afsi_gpu_b200 import synthetic
    from afsi_gpu_b200.grid import MACGrid
    from afsi_gpu_b200.multigrid import GeometricMultigrid
    from afsi_gpu_b200.p2_cuda_transfer import P1Transfer
    device = torch.device('cuda', torch.cuda.current_device())
    grid = MACGrid((128, 128, 128), (1., 1., 1.))
    X, cells = synthetic.prolate_shell(**P1_SHELL)
    rng = np.random.default_rng(21)
    x = torch.as_tensor(X, device=device)
    tr = P1Transfer(grid, x, torch.as_tensor(cells, device=device))
    c = torch.as_tensor(rng.uniform(-1., 1., (X.shape[0], 3)), device=device)
    v = tuple(t.to(device) for t in synthetic.fourier_velocity3d(grid, seed=21))
    r = synthetic.mean_free_normal(grid.shape, seed=21).to(device)
    mg = GeometricMultigrid(grid, device=device, backend='b200-graph')
    st = tr.prepare(x)
    for k in range(args.warmup + args.steps):
        if k == args.warmup:
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
        tr.spread(c, st), tr.interpolate_rhs(v, st), mg.solve(r)
    torch.cuda.synchronize(device)
    tr.check(st)
    print(json.dumps(dict(points=st.rule.point_count, ms_per_step=(time.perf_counter() - t0) * 1e3 / max(args.steps, 1))))


def stokes_only(args):
    """FGMRES Stokes solves of the 64^3 row for profiler runs."""
    from afsi_gpu_b200 import synthetic
    from afsi_gpu_b200.grid import MACGrid
    from afsi_gpu_b200.stokes_fgmres import CNStokes
    device = torch.device('cuda', torch.cuda.current_device())
    grid = MACGrid(GRID['shape'], GRID['lengths'])
    b = tuple(t.to(device) for t in synthetic.divergence_free_faces(grid, seed=8))
    flow = CNStokes(grid, device=device, **STOKES)
    for k in range(args.warmup + args.steps):
        if k == args.warmup:
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
        res = flow.stokes(b)
    torch.cuda.synchronize(device)
    print(json.dumps(dict(iterations=res.diagnostics['stokes']['iterations'],
                          ms_per_solve=(time.perf_counter() - t0) * 1e3 / max(args.steps, 1))))


def det_only(args):
    """The deterministic-transfer row of the headline workload, alone."""
    device = torch.device('cuda', torch.cuda.current_device())
    grid, X, cells, coef, vel, rhs = workload()
    step = Step(grid, X, cells, coef, vel, rhs, device)
    print(json.dumps(deterministic_row(step, coef, vel, device, reps=max(args.steps, 1)), default=_json))


def main():
    args = parse()
    if args.impl == 'reference':
        run_reference(args)
    elif args.rows == 'batch':
        batch_only(args)
    elif args.rows == 'p1free':
        p1free_only(args)
    elif args.rows == 'stokes':
        stokes_only(args)
    elif args.rows == 'det':
        det_only(args)
    elif args.rows == 'p1':
        print(json.dumps(precision_p1_row(torch.device('cuda', torch.cuda.current_device())), default=_json))
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
