"""NumPy restatement of the IB consistent-mass Jacobi-PCG (oracle; test
infrastructure only).

``mac/mass_solver.py:12-103`` (afsi-torch 0.28.0): conjugate gradients on
M x = rhs for the (N,3) nodal block (one recurrence for the three columns,
all inner products over the whole block), Jacobi preconditioner z = r/diag,
breakdown guard on the curvature and rz, restart every ``recompute_every``
iterations, convergence checks every ``check_every`` iterations, and
acceptance only on the true residual ||rhs - M x||.
"""
from math import isfinite
import numpy as np


class PCGError(RuntimeError):
    pass


def csr_mm(crow, col, val, v):
    """M v for a CSR matrix (rows summed in column order, empty rows zero)."""
    rows = len(crow) - 1
    out = np.zeros((rows,) + v.shape[1:], dtype=np.result_type(val, v))
    if len(col) == 0:
        return out
    shape = (-1,) + (1,) * (v.ndim - 1)
    prod = np.asarray(val).reshape(shape) * v[col]
    filled = crow[1:] > crow[:-1]
    out[filled] = np.add.reduceat(prod, crow[:-1][filled], axis=0)
    return out


def solve(crow, col, val, diagonal, rhs, initial=None, *, rtol=1e-12, atol=1e-13, max_iterations=500,
          check_every=4, recompute_every=40):
    """Returns (x, iterations, true residual norm, tolerance)."""
    diag = np.asarray(diagonal, dtype=np.float64)[:, None] * np.ones((1, rhs.shape[1]))
    rhs = np.asarray(rhs, dtype=np.float64)
    x = np.zeros_like(rhs) if initial is None else np.array(initial, dtype=np.float64)
    rhs_norm = float(np.linalg.norm(rhs))
    tol = max(atol, rtol * rhs_norm)

    def true_residual():
        r = rhs - csr_mm(crow, col, val, x)
        return r, float(np.linalg.norm(r))

    r, true_norm = true_residual()
    if true_norm <= tol:
        return x, 0, true_norm, tol
    d = r / diag
    rz = float((r * d).sum())
    active, broken = True, False
    for iteration in range(1, max_iterations + 1):
        Ad = csr_mm(crow, col, val, d)
        curvature = float((d * Ad).sum())
        valid = isfinite(curvature) and curvature > 0 and isfinite(rz) and rz > 0
        broken = broken or (active and not valid)
        working = active and valid and not broken
        alpha = rz / curvature if working else 0.
        x = x + alpha * d
        r = r - alpha * Ad
        rn = float(np.linalg.norm(r))
        broken = broken or not isfinite(rn)
        active = working and rn > tol
        restart = iteration % recompute_every == 0
        check = restart or iteration % check_every == 0 or iteration == max_iterations
        converged = False
        if check:
            if broken:
                raise PCGError('PCG breakdown: operator/preconditioner must be positive definite and finite')
            converged = rn <= tol
        if restart or converged or iteration == max_iterations:
            r, true_norm = true_residual()
            if not isfinite(true_norm):
                raise PCGError('nonfinite true PCG residual')
            if true_norm <= tol:
                return x, iteration, true_norm, tol
            restart = True
            active = True
        z = r / diag
        next_rz = float((r * z).sum())
        if restart:
            d = z
        else:
            beta = next_rz / (rz if active else 1.)
            d = z + beta * d if active else np.zeros_like(d)
        rz = next_rz
    raise PCGError(f'PCG did not converge: {true_norm:g} > {tol:g}')
