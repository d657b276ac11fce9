"""The benchmark workloads' sizes, pinned with the oracle's order rule (no GPU).

The bench line and the docs quote these counts: the headline 3D P2 shell on
the 64^3 grid gives 2,457,600 interaction points (38,400 elements at order 4,
64 points each), and the precision form's thin P1 shell on the 128^3 grid
gives about 1.1 M points (128,000 elements at orders 2 and 3).  The counts
come from the adaptive rule of ``mac/adaptive_transfer.py:167-187`` as the
oracle restates it, with the rule's point counts (Keast's 15 points at
order 3 for P2, n^3 otherwise).
"""
import numpy as np
import bench
from afsi_gpu_b200 import synthetic
from afsi_gpu_b200.quadrature import conical_rule
from oracle import ib


def _points(orders):
    return sum(int(count) * len(conical_rule(n)[1]) for n, count in enumerate(np.bincount(orders)) if count)


def test_headline_p2_shell_has_the_quoted_point_count():
    X, cells = synthetic.p2_shell(**bench.SHELL)
    orders = ib.p2_orders(X, cells, 1 / bench.GRID['shape'][0], 2.)
    assert cells.shape[0] == 38400
    assert set(np.unique(orders)) == {4}
    assert _points(orders) == 2457600


def test_precision_p1_shell_has_about_1_1_million_points():
    X, cells = synthetic.prolate_shell(**bench.P1_SHELL)
    orders = ib.p1_orders(X, cells, 1 / 128, 2.)
    assert cells.shape[0] == 128000
    assert set(np.unique(orders)) <= {2, 3}
    assert _points(orders) == 1097920
