"""Generate the golden fixtures by running the reference afsi-torch 0.28.0 on CPU.

Run from the repository root in a container where the reference source tree is
available (it is not needed afterwards; the fixtures are committed):

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py REFERENCE_SRC

REFERENCE_SRC is the reference's ``src`` directory (the argument, or the
``AFSI_TORCH_SRC`` environment variable when no argument is given).  Every fixture is produced by
the reference's own public functions or the CPU expressions its classes use;
inputs are seeded.  Outputs are small ``.npz`` files next to this script.
"""
import os
import sys
from pathlib import Path
import numpy as np

SRC = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('AFSI_TORCH_SRC')
if not SRC:
    sys.exit('usage: make_golden.py REFERENCE_SRC  (or set AFSI_TORCH_SRC)')
sys.path.insert(0, SRC)
import torch  # noqa: E402
from afsi_torch import ib  # noqa: E402
from afsi_torch.ib import peskin4  # noqa: E402
from afsi_torch.mac.grid import MACGrid, negative_laplacian  # noqa: E402
from afsi_torch.mac.compact_transfer import _prepare, CompactFETransfer  # noqa: E402
from afsi_torch.mac.multigrid import GeometricMultigrid, MGOptions  # noqa: E402
from afsi_torch.mac.mg_workspace import TensorKernels  # noqa: E402
from afsi_torch.mac2d.grid import ChannelGrid  # noqa: E402
from afsi_torch.mac2d.transfer import TriangleTransfer  # noqa: E402
from afsi_torch.mac2d.multigrid import ChannelMultigrid  # noqa: E402
from afsi_torch.mac2d.mg_workspace import TensorKernels as ChannelKernels  # noqa: E402
from afsi_torch.mac.adaptive_transfer import (AdaptiveFETransfer, InteractionQuadratureOptions,  # noqa: E402
                                              gaussian_tetra_rule, _orders, _orders_p2)
from afsi_torch.tetrahedron import reference_nodes, tabulate, promote_p1  # noqa: E402
from afsi_torch.solid import prepare_p2  # noqa: E402
from afsi_torch.p1 import prepare_p1  # noqa: E402
from afsi_torch.mac.adaptive_transfer import AdaptiveP1Transfer  # noqa: E402
from afsi_torch.mac.assembled_transfer import AssembledP1Transfer  # noqa: E402
from afsi_torch.mac.hash_transfer_assembly import hash_slot  # noqa: E402
from afsi_torch.fluid.solvers import SolverOptions  # noqa: E402
from afsi_torch.mac.dirichlet_mg import DirichletMultigrid  # noqa: E402
from afsi_torch.mac.transfer import FETransfer  # noqa: E402
from afsi_torch.mac.mass_solver import MassSolver  # noqa: E402
from afsi_torch.mac.open_boundary import negative_laplacian as open_negative_laplacian  # noqa: E402

OUT = Path(__file__).resolve().parent
torch.set_default_dtype(torch.float64)


def save(name, **arrays):
    arrays = {k: (v.detach().cpu().numpy() if torch.is_tensor(v) else np.asarray(v)) for k, v in arrays.items()}
    np.savez_compressed(OUT / f'{name}.npz', **arrays)
    print(name, {k: v.shape for k, v in arrays.items()})


def peskin():
    d = torch.linspace(-2.5, 2.5, 1001)
    d = torch.cat((d, torch.tensor([0., .5, 1., 1.5, 2., -1., -2., 1 - 1e-15, 1 + 1e-15])))
    save('peskin', d=d, phi=peskin4(d))


def compact3d():
    g = torch.Generator().manual_seed(7)
    grid = MACGrid((12, 14, 16), (2., 3., 5.), (-.2, .1, -.4))
    h = torch.tensor(grid.spacing)
    lo = torch.tensor(grid.origin) + 2.05 * h
    hi = torch.tensor(grid.origin) + (torch.tensor(grid.shape) - 2.05) * h
    pts = lo + (hi - lo) * torch.rand((300, 3), generator=g)
    # a few points exactly on lattice knots / half knots
    pts[:4] = torch.tensor(grid.origin) + h * torch.tensor([[3., 4., 5.], [3.5, 4.5, 5.5], [5., 6.5, 7.], [9.5, 9., 12.5]])
    origins = torch.tensor([grid.face_origin(c) for c in range(3)])
    shared = torch.tensor([grid.origin, tuple(o + .5 * s for o, s in zip(grid.origin, grid.spacing))])
    offs = torch.arange(4)
    base, phi = _prepare(pts, origins, h, offs)
    sbase, sphi = _prepare(pts, shared, h, offs)
    t = object.__new__(CompactFETransfer)
    t.grid, t.axis_offsets, t.ib_backend = grid, offs, 'reference'
    from afsi_torch.mac.compact_transfer import CompactStencil
    st = CompactStencil(base.contiguous(), phi.contiguous())
    force = torch.randn((300, 3), generator=g)
    fields = t.spread_grid(force, st)
    vel = tuple(torch.randn(grid.face_shape(c), generator=g) for c in range(3))
    gathered = t.gather_grid(vel, st)
    save('compact3d', shape=grid.shape, lengths=grid.lengths, origin=grid.origin, spacing=grid.spacing,
         volume=grid.volume, points=pts, base=base, phi=phi, shared_base=sbase, shared_phi=sphi,
         force=force, u0=fields[0], u1=fields[1], u2=fields[2], v0=vel[0], v1=vel[1], v2=vel[2],
         gathered=gathered)


def transfer2d():
    g = torch.Generator().manual_seed(11)
    grid = ChannelGrid((32, 16), (2., 1.))
    hx, hy = grid.spacing
    P = 400
    x = 2 * hx + (grid.lengths[0] - 4 * hx) * torch.rand(P, generator=g)
    y = -hy + (grid.lengths[1] + 2 * hy) * torch.rand(P, generator=g)   # includes wall halo
    pts = torch.stack((x, y), -1)
    t = object.__new__(TriangleTransfer)
    t.grid = grid
    t.offsets = torch.cartesian_prod(torch.arange(4), torch.arange(4))
    ids, w = t._prepare(pts)
    force = torch.randn((P, 2), generator=g)
    spread = [torch.zeros(grid.face_shape(c)).reshape(-1).index_add(0, ids[c].reshape(-1),
              (force[:, c, None] * w[c] / grid.volume).reshape(-1)) for c in range(2)]
    vel = tuple(torch.randn(grid.face_shape(c), generator=g) for c in range(2))
    gathered = torch.stack([(u.reshape(-1)[i] * ww).sum(-1) for u, i, ww in zip(vel, ids, w)], -1)
    save('transfer2d', shape=grid.shape, lengths=grid.lengths, spacing=grid.spacing, volume=grid.volume,
         points=pts, ids0=ids[0], ids1=ids[1], w0=w[0], w1=w[1], force=force, s0=spread[0], s1=spread[1],
         v0=vel[0], v1=vel[1], gathered=gathered)


def p2():
    """Two P2 tetrahedra (promoted P1 pair), adaptive conical quadrature."""
    g = torch.Generator().manual_seed(5)
    X1 = torch.tensor([[0., 0., 0.], [1., 0., 0.], [0., 1., 0.], [0., 0., 1.], [2.2, 2.0, 2.1]]) * .4 + 1.7
    c1 = torch.tensor([[0, 1, 2, 3], [1, 2, 3, 4]])
    X, cells = promote_p1(X1, c1)
    geometry = prepare_p2(X, cells)
    grid = MACGrid((16, 12, 10), (5., 5.5, 6.), (-.2, .1, -.4))
    opt = InteractionQuadratureOptions(mode='adaptive', point_density=3., max_order=22,
                                       max_points=500000, rule_family='conical')
    tr = AdaptiveFETransfer(grid, geometry, fused=False, ib_backend='reference', quadrature_options=opt)
    x = X.clone()
    x[4, 1] += .017
    st = tr.prepare(x)
    coef = torch.sin(1.3 * X)
    force_q = torch.cat([tr._weighted_kernel(coef, gg.values, gg.cells, gg.weights) for gg in st.rule.groups])
    fields = tr.spread_grid(force_q, st)
    vel = tuple(torch.sin(grid.coordinates(c)[..., (c + 1) % 3]) for c in range(3))
    gathered = tr.gather_grid(vel, st)
    rhs = torch.zeros_like(tr.diagonal)
    off = 0
    for gg in st.rule.groups:
        n = gg.weights.numel()
        rhs += tr._assemble_kernel(gathered[off:off + n], gg.values, gg.cells, gg.weights, tr.diagonal)
        off += n
    groups = {}
    for k, gg in enumerate(st.rule.groups):
        groups[f'cells{k}'] = gg.cells
        groups[f'N{k}'] = gg.values
        groups[f'W{k}'] = gg.weights
        groups[f'order{k}'] = gg.order
    save('p2', shape=grid.shape, lengths=grid.lengths, origin=grid.origin, spacing=grid.spacing,
         volume=grid.volume, X=X, x=x, ngroups=len(st.rule.groups), base=st.base, phi=st.phi,
         coef=coef, force_q=force_q, u0=fields[0], u1=fields[1], u2=fields[2],
         v0=vel[0], v1=vel[1], v2=vel[2], gathered=gathered, rhs=rhs, **groups)


def mg3d():
    from math import pi
    grid = MACGrid((8, 12, 16), (2., 3., 4.))
    options = MGOptions(smooth=3)
    ref = GeometricMultigrid(grid, options=options)
    xyz = grid.coordinates()
    exact = torch.cos(pi * xyz[..., 0] / 2) * torch.cos(2 * pi * xyz[..., 1] / 3) * torch.cos(pi * xyz[..., 2] / 4)
    exact -= exact.mean()
    rhs = negative_laplacian(exact, grid.spacing)
    start = .1 * exact
    with torch.no_grad():
        cyc = ref._cycle(0, start, rhs)
    p, info = ref.solve(rhs, start)
    k = TensorKernels()
    g = torch.Generator().manual_seed(3)
    pp = torch.randn(grid.shape, generator=g)
    rr = torch.randn(grid.shape, generator=g)
    res = torch.empty_like(pp)
    k.residual(pp, rr, res, grid.spacing)
    sm = torch.empty_like(pp)
    k.smooth(pp, rr, ref.diagonals[0], sm, grid.spacing)
    coarse = torch.empty(tuple(n // 2 for n in grid.shape))
    k.restrict(pp, coarse)
    rres = torch.empty_like(coarse)
    k.residual_restrict(pp, rr, rres, grid.spacing)
    pro = pp.clone()
    k.prolong_add(coarse, pro)
    # 64^3-style five level solve on a random mean-zero RHS
    grid2 = MACGrid((16, 16, 32), (1., 1., 2.))
    mg2 = GeometricMultigrid(grid2)
    r2 = torch.randn(grid2.shape, generator=g)
    r2 -= r2.mean()
    p2, info2 = mg2.solve(r2)
    save('mg3d', shape=grid.shape, lengths=grid.lengths, spacing=grid.spacing, smooth=3,
         rhs=rhs, start=start, cycle=cyc, solution=p, cycles=info['cycles'], diag0=ref.diagonals[0],
         coarse_inverse=ref.coarse_inverse, pp=pp, rr=rr, residual=res, smoothed=sm, restricted=coarse,
         residual_restricted=rres, prolonged=pro,
         shape2=grid2.shape, lengths2=grid2.lengths, rhs2=r2, solution2=p2, cycles2=info2['cycles'],
         residual2=info2['residual_norm'])


def mg2d():
    g = torch.Generator().manual_seed(13)
    grid = ChannelGrid((32, 16), (2., 1.))
    mg = ChannelMultigrid(grid, fused=False)
    rhs = torch.randn(grid.shape, generator=g)
    start = .1 * torch.randn(grid.shape, generator=g)
    with torch.no_grad():
        cyc = mg._cycle(0, start, rhs)
    p, info = mg.solve(rhs)
    k = ChannelKernels()
    pp = torch.randn(grid.shape, generator=g)
    res = torch.empty_like(pp)
    k.residual(pp, rhs, res, grid.spacing)
    sm = torch.empty_like(pp)
    k.smooth(pp, rhs, mg.diagonals[0], sm, grid.spacing)
    rres = torch.empty(tuple(n // 2 for n in grid.shape))
    k.residual_restrict(pp, rhs, rres, grid.spacing)
    pro = pp.clone()
    k.prolong_add(rres, pro)
    big = ChannelGrid((256, 64), (8., 1.61))
    mgb = ChannelMultigrid(big, fused=False)
    rb = torch.randn(big.shape, generator=g)
    pb, infob = mgb.solve(rb)
    save('mg2d', shape=grid.shape, lengths=grid.lengths, spacing=grid.spacing, rhs=rhs, start=start,
         cycle=cyc, solution=p, cycles=info['cycles'], diag0=mg.diagonals[0], inverse=mg.inverse,
         pp=pp, residual=res, smoothed=sm, residual_restricted=rres, prolonged=pro,
         shape_b=big.shape, lengths_b=big.lengths, rhs_b=rb, solution_b=pb, cycles_b=infob['cycles'])


def orders():
    """Adaptive element orders (_orders_p2 / _orders) on seeded node clouds."""
    g = torch.Generator().manual_seed(6)
    x = torch.rand((300, 3), generator=g) * .3 + .2
    cells = torch.randint(0, 300, (500, 10), generator=g)
    edges = torch.tensor([[0, 1], [0, 2], [0, 3], [1, 2], [1, 3], [2, 3]])
    arrays = dict(x=x, cells=cells, dx=np.array([.011, .037]), density=np.array([2., 3.5]))
    for k, (dx, density) in enumerate(zip(arrays['dx'], arrays['density'])):
        arrays[f'p2_{k}'] = _orders_p2(x, cells, edges, float(dx), float(density))
        arrays[f'p1_{k}'] = _orders(x, cells[:, :4], edges, float(dx), float(density))
    save('orders', **arrays)


def kuhn_block(nx, ny, nz, h, origin, seed):
    """Cube block cut into six Kuhn tetrahedra per cube, nodes jittered."""
    g = torch.Generator().manual_seed(seed)
    idx = torch.arange((nx + 1) * (ny + 1) * (nz + 1)).reshape(nx + 1, ny + 1, nz + 1)
    grid = torch.stack(torch.meshgrid(*(torch.arange(n + 1.) for n in (nx, ny, nz)), indexing='ij'), -1)
    X = grid.reshape(-1, 3) * h + torch.tensor(origin) + (torch.rand((idx.numel(), 3), generator=g) - .5) * .2 * h
    cells = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                for perm in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
                    v, path = [i, j, k], [int(idx[i, j, k])]
                    for axis in perm:
                        v[axis] += 1
                        path.append(int(idx[v[0], v[1], v[2]]))
                    cells.append(path)
    return X, torch.tensor(cells)


def p1csr():
    """P1 CSR operators B_c (AssembledP1Transfer, coalesce backend) and the
    SplitMix64 bucket of the hash assembly, on two P1 meshes."""
    grid = MACGrid((12, 14, 16), (10., 12., 14.))
    cases = dict(
        pair=(torch.tensor([[4, 4, 4], [4.3, 4, 4], [4, 4.3, 4], [4, 4, 4.3], [4, 4, 2.6]]),
              torch.tensor([[0, 1, 2, 3], [0, 2, 1, 4]])),
        block=kuhn_block(4, 3, 3, .55, (3.2, 3.9, 4.6), seed=11))
    X, cells = cases['block']
    X[:, 0] = 3.2 + (X[:, 0] - 3.2) * (1 + .35 * (X[:, 0] - 3.2))  # stretched in x: several orders
    arrays = dict(shape=grid.shape, lengths=grid.lengths, origin=grid.origin)
    for name, (X, cells) in cases.items():
        geometry = prepare_p1(X, cells, degree=2)
        common = dict(quadrature_options=InteractionQuadratureOptions(mode='adaptive', stencil_backend='shared'),
                      fused=False, options=SolverOptions(rtol=1e-12, atol=1e-13))
        reference = AdaptiveP1Transfer(grid, geometry, **common)
        assembled = AssembledP1Transfer(grid, geometry, chunk_entries=512, **common)
        stencil = reference.prepare(X)
        B = assembled.assemble_stencil(stencil)
        arrays[f'{name}_X'] = X
        arrays[f'{name}_cells'] = cells
        if name == 'pair':
            arrays[f'{name}_base'] = stencil.base
            arrays[f'{name}_phi'] = stencil.phi
        arrays[f'{name}_ngroups'] = len(stencil.rule.groups)
        for k, gr in enumerate(stencil.rule.groups):
            arrays[f'{name}_cells{k}'] = gr.cells
            arrays[f'{name}_N{k}'] = gr.values
            arrays[f'{name}_W{k}'] = gr.weights
        for c, m in enumerate(B.gather):
            arrays[f'{name}_crow{c}'] = m.crow_indices()
            arrays[f'{name}_col{c}'] = m.col_indices()
            arrays[f'{name}_val{c}'] = m.values()
    keys = torch.cat((torch.arange(200), torch.arange(64) * 2147483649 + 4294967296,
                      torch.randint(0, 2 ** 62, (64,), generator=torch.Generator().manual_seed(12))))
    arrays['hash_keys'] = keys
    for cap in (128, 4096, 1 << 20):
        arrays[f'hash_slot_{cap}'] = torch.tensor([hash_slot(int(k), cap) for k in keys])
    save('p1csr', **arrays)


def dirichlet():
    """Open-box (zero face pressure) multigrid: operator, prolongation, one
    V-cycle and solves of the reference DirichletMultigrid (torch backend)."""
    g = torch.Generator().manual_seed(13)
    grid = MACGrid((8, 16, 8), (3., 5., 4.))
    solver = DirichletMultigrid(grid, backend='torch')
    xyz = grid.coordinates()
    exact = torch.sin(.7 * xyz[..., 0]) * torch.cos(.9 * xyz[..., 1]) + .4
    rhs = open_negative_laplacian(exact, grid.spacing)
    solution, info = solver.solve(rhs)
    p = torch.randn(grid.shape, generator=g)
    r = torch.randn(grid.shape, generator=g)
    coarse = torch.randn((4, 8, 4), generator=g)
    grid2 = MACGrid((16, 16, 32), (1., 1., 2.))
    solver2 = DirichletMultigrid(grid2, backend='torch')
    rhs2 = torch.randn(grid2.shape, generator=g)
    solution2, info2 = solver2.solve(rhs2)
    save('dirichlet', shape=grid.shape, lengths=grid.lengths, exact=exact, rhs=rhs, solution=solution,
         cycles=info['cycles'], p=p, r=r, apply=open_negative_laplacian(p, grid.spacing),
         cycle=solver.cycle(0, p, r), coarse=coarse, prolonged=solver.prolong(coarse, grid.shape),
         shape2=grid2.shape, lengths2=grid2.lengths, rhs2=rhs2, solution2=solution2, cycles2=info2['cycles'])


def mass():
    """Consistent FE mass matrix of a P2 block mesh (FETransfer) and Jacobi-PCG
    solves by the reference MassSolver: default schedule, warm start, and a
    schedule with frequent checks and restarts."""
    g = torch.Generator().manual_seed(14)
    X1, c1 = kuhn_block(3, 2, 2, 1., (2., 2., 2.), seed=14)
    X, cells = promote_p1(X1, c1)
    geometry = prepare_p2(X, cells)
    tr = FETransfer(MACGrid((12, 12, 12), (10., 10., 10.)), geometry)
    mass = tr.mass
    n = X.shape[0]
    rhs = torch.randn((n, 3), generator=g)
    initial = torch.randn((n, 3), generator=g) * .1
    default = SolverOptions(rtol=1e-12, atol=1e-13, max_iterations=500, check_every=4)
    busy = SolverOptions(rtol=1e-12, atol=1e-13, max_iterations=500, check_every=1, recompute_every=5)
    out = dict(crow=mass.crow_indices(), col=mass.col_indices(), values=mass.values(),
               diagonal=tr.diagonal[:, 0].contiguous(), rhs=rhs, initial=initial)
    for name, opts, init in (('default', default, None), ('warm', default, initial), ('busy', busy, None)):
        x, info = MassSolver(mass, tr.diagonal, opts).solve(rhs, init)
        out[f'{name}_x'] = x
        out[f'{name}_iterations'] = info.iterations
        out[f'{name}_residual'] = info.residual_norm
        out[f'{name}_tolerance'] = info.tolerance
    save('mass', **out)


def quadrature():
    arrays = {}
    like = torch.zeros(1)
    for n in range(2, 9):
        q, w = gaussian_tetra_rule(n, like, 'conical')
        N, _ = tabulate(q)
        arrays[f'q{n}'], arrays[f'w{n}'], arrays[f'N{n}'] = q, w, N
    save('quadrature', **arrays)


def stokes():
    """CN Helmholtz kernels (the reference's CPU kernel object) and the Stokes
    residual / pressure metrics by the reference grid operators, on a small
    anisotropic MAC grid with wall-free (zero normal wall) face fields."""
    from afsi_torch.mac.helmholtz import TorchHelmholtzKernels
    from afsi_torch.mac.grid import gradient, divergence, velocity_laplacian, zero_normal, slab
    g = torch.Generator().manual_seed(15)
    grid = MACGrid((10, 8, 6), (1.0, .9, .7))
    faces = lambda: zero_normal(tuple(torch.randn(grid.face_shape(c), generator=g, dtype=torch.float64)
                                      for c in range(3)))
    b, u = faces(), faces()
    p = torch.randn(grid.shape, generator=g, dtype=torch.float64)
    alpha, scale = .013, .7
    s2 = 2 * alpha * sum(1 / h ** 2 for h in grid.spacing)
    diagonal = []
    for c in range(3):
        d = torch.full(grid.face_shape(c), 1 + s2, dtype=torch.float64)
        for axis, h in enumerate(grid.spacing):
            if axis != c:
                d[slab(axis, 0, 1)] += alpha / h ** 2
                d[slab(axis, -1, None)] += alpha / h ** 2
        d[slab(c, 0, 1)] = 1.
        d[slab(c, -1, None)] = 1.
        diagonal.append(d)
    k = TorchHelmholtzKernels()
    params = torch.tensor([alpha, scale], dtype=torch.float64)
    out = dict(shape=grid.shape, lengths=grid.lengths, alpha=alpha, scale=scale, p=p)
    for c in range(3):
        out[f'b{c}'], out[f'u{c}'], out[f'd{c}'] = b[c], u[c], diagonal[c]
    for tag, pp in (('p', p), ('nop', None)):
        rhs = tuple(torch.empty_like(v) for v in b)
        first = tuple(torch.empty_like(v) for v in b)
        k.initialize(b, pp, diagonal, rhs, first, params, grid)
        second = tuple(torch.empty_like(v) for v in b)
        cur, nxt = first, second
        for c in range(3):
            out[f'{tag}_rhs{c}'], out[f'{tag}_init{c}'] = rhs[c].clone(), first[c].clone()
        for sweep in range(3):
            k.sweep(cur, rhs, diagonal, nxt, params, grid)
            cur, nxt = nxt, cur
        for c in range(3):
            out[f'{tag}_sweep3_{c}'] = cur[c]
    # Stokes residual (StokesWorkspace.measure, CPU branch) with dt/rho = scale
    gp = gradient(p, grid.spacing)
    momentum = tuple(v - alpha * velocity_laplacian(v, c, grid.spacing) + scale * gq - r
                     for c, (v, gq, r) in enumerate(zip(u, gp, b)))
    div = divergence(u, grid.spacing)
    out['norms'] = torch.stack((torch.sqrt(sum(v.square().sum() for v in momentum)), torch.linalg.vector_norm(div)))
    out['residual'] = -(1 / scale) * div
    out['start'] = torch.stack((torch.sqrt(sum(v.square().sum() for v in b)), p.mean(),
                                torch.isfinite(p).all().double()))
    rhs = torch.randn(grid.shape, generator=g, dtype=torch.float64)
    out['prhs'] = rhs
    out['pmetrics'] = torch.stack((rhs.sum(), rhs.abs().sum(), p.sum(), torch.linalg.vector_norm(rhs),
                                   torch.linalg.vector_norm(rhs - negative_laplacian(p, grid.spacing))))
    save('stokes', **out)


def cached():
    """Cached CSR pattern (mac/cached_transfer_assembly.py:97-175): a first
    build from a filled hash table, then an extension by a miss stream that
    holds new keys, keys already in the pattern and repeats."""
    from afsi_torch.mac.hash_transfer_assembly import HashWorkspace, cpu_accumulate
    from afsi_torch.mac.cached_transfer_assembly import CSRPatternCache, finish_cached_component
    g = torch.Generator().manual_seed(16)
    rows, shape = 40, (6, 5, 4)
    nf = 6 * 5 * 4
    ws = HashWorkspace()
    ws.reset(1024, torch.zeros(1, dtype=torch.float64))
    keys1 = torch.randint(0, rows * nf, (300,), generator=g)
    cpu_accumulate(keys1, torch.randn(300, generator=g, dtype=torch.float64), ws)
    cache = CSRPatternCache()
    out = dict(rows=rows, shape=shape, capacity=ws.capacity, table1_keys=ws.keys.clone(),
               table1_values=ws.values.clone())
    m1, t1 = finish_cached_component(ws, cache, rows, shape, 10 ** 6)
    out.update(slots1=cache.slots.to(torch.int64), order1=cache.transpose_order.to(torch.int64), crow1=cache.crow,
               cols1=cache.columns, tcrow1=cache.transpose_crow, tcols1=cache.transpose_columns,
               values1=m1.values(), reverse1=t1.values())
    fresh = torch.randint(0, rows * nf, (60,), generator=g)
    old = ws.keys[cache.slots.to(torch.int64)][torch.randint(0, cache.nnz, (30,), generator=g)]
    missing = torch.cat((fresh, old, fresh[:10]))
    vals = torch.randn(len(missing), generator=g, dtype=torch.float64)
    cpu_accumulate(missing, vals, ws)
    cache.scratch(len(missing), ws.values)
    cache.missing_keys[:len(missing)] = missing
    m2, t2 = finish_cached_component(ws, cache, rows, shape, 10 ** 6, missing=len(missing))
    out.update(missing=missing, table2_keys=ws.keys.clone(), table2_values=ws.values.clone(),
               slots2=cache.slots.to(torch.int64), order2=cache.transpose_order.to(torch.int64), crow2=cache.crow,
               cols2=cache.columns, tcrow2=cache.transpose_crow, tcols2=cache.transpose_columns,
               values2=m2.values(), reverse2=t2.values(), new_count=cache.last_sorted_keys)
    save('cached', **out)


def curl_rhs(grid, seed):
    """Seeded discrete curl of edge potentials that vanish on the boundary
    edges: face fields with zero wall-normal flux and zero discrete divergence."""
    g = torch.Generator().manual_seed(seed)
    nx, ny, nz = grid.shape
    hx, hy, hz = grid.spacing
    Ax = torch.randn((nx, ny + 1, nz + 1), generator=g, dtype=torch.float64)
    Ay = torch.randn((nx + 1, ny, nz + 1), generator=g, dtype=torch.float64)
    Az = torch.randn((nx + 1, ny + 1, nz), generator=g, dtype=torch.float64)
    for A, axes in ((Ax, (1, 2)), (Ay, (0, 2)), (Az, (0, 1))):
        for a in axes:
            A.index_fill_(a, torch.tensor([0, A.shape[a] - 1]), 0.)
    u = torch.diff(Az, dim=1) / hy - torch.diff(Ay, dim=2) / hz
    v = torch.diff(Ax, dim=2) / hz - torch.diff(Az, dim=0) / hx
    w = torch.diff(Ay, dim=0) / hx - torch.diff(Ax, dim=1) / hy
    return (u, v, w)


def fgmres():
    """The CN saddle-point solve by MG-preconditioned FGMRES
    (mac/stokes_fgmres.py:15-96 with nonlinear.py gmres), from a zero and from
    a random initial pressure, on a small anisotropic grid; plus one operator
    action and one preconditioner application on a random packed vector, built
    from the reference's own grid operators and flow methods exactly as the
    solve's closures build them."""
    from afsi_torch.mac.cnab import MACCNABFlow, CNABOptions
    from afsi_torch.mac.grid import zero_normal, gradient, divergence
    grid = MACGrid((16, 12, 10), (1.0, .9, .7))
    dt, rho, mu = 1e-3, 1., .01
    flow = MACCNABFlow(grid, dt=dt, rho=rho, mu=mu, cnab_options=CNABOptions(stokes_solver='fgmres',
                                                                              advection='centered'))
    g = torch.Generator().manual_seed(17)
    b = curl_rhs(grid, 7)
    b = tuple(v + 1e-3 * torch.randn(v.shape, generator=g, dtype=torch.float64) for v in b)
    out = dict(shape=grid.shape, lengths=grid.lengths, dt=dt, rho=rho, mu=mu, alpha=flow.alpha,
               helmholtz_iterations=flow.helmholtz_iterations)
    for c in range(3):
        out[f'b{c}'] = b[c]
    p0 = torch.randn(grid.shape, generator=g, dtype=torch.float64)
    out['p0'] = p0
    for tag, initial in (('zero', None), ('warm', p0)):
        res = flow.stokes(b, initial)
        st, pr = res.diagnostics['stokes'], res.diagnostics['pressure']
        for c in range(3):
            out[f'{tag}_u{c}'] = res.velocity[c]
        out[f'{tag}_p'] = res.pressure
        out[f'{tag}_info'] = np.array([st['iterations'], st['operator_actions'], pr['poisson_solves'], pr['cycles'],
                                       st['momentum_residual'], st['momentum_tolerance'], st['divergence_norm'],
                                       st['divergence_tolerance']])
    # one action and one preconditioner application (the solve's closures)
    h = min(grid.spacing)
    sizes = [grid.face_shape(c) for c in range(3)]
    v = [torch.randn(s, generator=g, dtype=torch.float64) for s in sizes]
    q = torch.randn(grid.shape, generator=g, dtype=torch.float64)
    gp = gradient(q, grid.spacing)
    hu = zero_normal(tuple(a - flow.alpha * l + h * gq for a, l, gq in zip(v, flow._lap(v), gp)))
    for c in range(3):
        out[f'v{c}'] = v[c]
        out[f'action_u{c}'] = hu[c]
    out['q'] = q
    out['action_q'] = -h * divergence(v, grid.spacing)
    tentative = flow._solve_helmholtz(tuple(v))
    rhs = -q / h - divergence(tentative, grid.spacing)
    rhs = rhs - rhs.mean()
    phi, info = flow.pressure_solver.solve(rhs, rtol=flow.cnab_options.stokes_preconditioner_rtol)
    grad = gradient(phi, grid.spacing)
    for c in range(3):
        out[f'pre_tentative{c}'] = tentative[c]
        out[f'pre_u{c}'] = tentative[c] - grad[c]
    qq = (phi + flow.alpha * rhs) / h
    out['pre_rhs'] = rhs
    out['pre_phi'] = phi
    out['pre_q'] = qq - qq.mean()
    out['pre_cycles'] = info['cycles']
    save('fgmres', **out)


if __name__ == '__main__':
    # make_golden.py REFERENCE_SRC [fixture ...]: all fixtures, or the named ones
    names = sys.argv[2:] or ['peskin', 'compact3d', 'transfer2d', 'p2', 'mg3d', 'mg2d', 'quadrature', 'orders',
                             'p1csr', 'dirichlet', 'mass', 'stokes', 'cached', 'fgmres']
    for name in names:
        globals()[name]()
