"""NumPy restatement of the P1 CSR contraction (oracle; test infrastructure only).

For component c of a P1 interaction rule, B_c[node, face] = Σ over the cells
holding the node, Σ over the cell's quadrature points of
W[e,q] · N[q,a] · φx·φy·φz, where the face lies in the point's 4x4x4 support.
The reference builds B_c by visiting every face ("site") of each cell's
support box and adding the cell's four nodal sums into a SplitMix64 hash
keyed ``node·nf + face`` (``mac/csrc/ib.cu:22-116``,
``mac/hash_transfer_assembly.py:1-165``), then sorts the unique keys into CSR
(``mac/assembled_transfer.py:78-96,151-216``).  The same steps are restated
here on the CPU.  Citations are afsi-torch 0.28.0 paths relative to
``src/afsi_torch``.
"""
import numpy as np

MASK64 = (1 << 64) - 1


def splitmix_bucket(key, capacity):
    """SplitMix64 finaliser of the signed key, masked to a power-of-two table
    (``mac/csrc/ib.cu:14-19``, ``mac/hash_transfer_assembly.py:17-23``)."""
    h = int(key) & MASK64
    h = ((h ^ (h >> 30)) * 0xbf58476d1ce4e5b9) & MASK64
    h = ((h ^ (h >> 27)) * 0x94d049bb133111eb) & MASK64
    return (h ^ (h >> 31)) & (capacity - 1)


class HashTable:
    """Open addressing with linear probing, at most 128 probes; a zero value
    is not inserted; a negative key or a failed probe sets the flag
    (``mac/csrc/ib.cu:21-47``, ``mac/hash_transfer_assembly.py:59-73``)."""

    def __init__(self, capacity, dtype=np.float64):
        if capacity < 1 or capacity & (capacity - 1):
            raise ValueError('power-of-two hash capacity required')
        self.capacity = capacity
        self.keys = np.full(capacity, -1, dtype=np.int64)
        self.values = np.zeros(capacity, dtype=dtype)
        self.flag = 0

    def insert(self, keys, values):
        for key, value in zip(np.asarray(keys).tolist(), np.asarray(values).tolist()):
            if value == 0:
                continue
            if key < 0:
                self.flag = 1
                continue
            slot = splitmix_bucket(key, self.capacity)
            for _ in range(128):
                previous = int(self.keys[slot])
                if previous in (-1, key):
                    self.keys[slot] = key
                    self.values[slot] += value
                    break
                slot = (slot + 1) & (self.capacity - 1)
            else:
                self.flag = 1

    def sorted_entries(self):
        """Occupied slots, sorted by key (``hash_transfer_assembly.py:76-81``)."""
        occupied = self.keys >= 0
        order = np.argsort(self.keys[occupied], kind='stable')
        return self.keys[occupied][order], self.values[occupied][order]


def component_tables(base, phi, c):
    """Per-point (P,3) bases and (P,3,4) weights of component c from the
    shared face/centre layout: axis a reads lattice (a != c)
    (``mac/assembled_transfer.py:30-43``)."""
    b = np.stack([base[int(a != c), :, a] for a in range(3)], -1)
    p = np.stack([phi[int(a != c), :, a, :] for a in range(3)], 1)
    return b, p


def component_plan(base_c, E, Q, offset):
    """Support box of each cell: low = min base, width = max - min + 4, and
    the prefix of box sizes (``mac/hash_transfer_assembly.py:122-138``)."""
    b = base_c[offset:offset + E * Q].reshape(E, Q, 3)
    low = b.min(1)
    width = b.max(1) - low + 4
    prefix = np.concatenate(([0], np.cumsum(width.prod(-1))))
    return low, width, prefix


def cell_entries(base_c, phi_c, cells, N, W, offset, low, width, shape):
    """Keys and values of every (cell, box site, node) in site order
    (``mac/assembled_transfer.py:46-66``)."""
    ny, nz = shape[1], shape[2]
    nf = shape[0] * ny * nz
    E, Q = W.shape
    keys, values = [], []
    for e in range(E):
        wx, wy, wz = width[e]
        xs, ys, zs = np.meshgrid(np.arange(wx), np.arange(wy), np.arange(wz), indexing='ij')
        site = np.stack((xs.ravel(), ys.ravel(), zs.ravel()), -1) + low[e]
        rows = offset + e * Q + np.arange(Q)
        d = site[:, None, :] - base_c[rows][None, :, :]            # (S,Q,3)
        inside = ((d >= 0) & (d < 4)).all(-1)
        k = np.ones(d.shape[:2], dtype=phi_c.dtype)
        for a in range(3):
            w = np.take_along_axis(phi_c[rows][None, :, a, :].repeat(len(site), 0),
                                   np.clip(d[..., a], 0, 3)[..., None], -1)[..., 0]
            k = k * w if a else w
        k = np.where(inside, k * W[e][None, :], 0)
        vals = k @ N                                               # (S,4)
        face = (site[:, 0] * ny + site[:, 1]) * nz + site[:, 2]
        keys.append(cells[e][None, :] * nf + face[:, None])
        values.append(vals)
    return np.concatenate(keys).reshape(-1), np.concatenate(values).reshape(-1)


def assemble(base, phi, groups, c, shape, node_count):
    """B_c as sorted unique (key, value) plus CSR (crow, col, val) over
    node_count rows and prod(shape) columns (``assembled_transfer.py:69-110``).
    groups: list of (cells (E,4), N (Q,4), W (E,Q))."""
    base_c, phi_c = component_tables(base, phi, c)
    nf = int(np.prod(shape))
    keys, values, offset = [], [], 0
    for cells, N, W in groups:
        E, Q = W.shape
        low, width, _ = component_plan(base_c, E, Q, offset)
        k, v = cell_entries(base_c, phi_c, cells, N, W, offset, low, width, shape)
        keys.append(k)
        values.append(v)
        offset += E * Q
    keys, values = np.concatenate(keys), np.concatenate(values)
    keep = values != 0
    unique, inverse = np.unique(keys[keep], return_inverse=True)
    summed = np.zeros(len(unique), dtype=values.dtype)
    np.add.at(summed, inverse, values[keep])
    rows, cols = unique // nf, unique % nf
    crow = np.zeros(node_count + 1, dtype=np.int64)
    np.add.at(crow, rows + 1, 1)
    return unique, summed, (np.cumsum(crow), cols, summed)


def csr_matvec(crow, col, val, x):
    """y = A x for CSR A."""
    y = np.zeros(len(crow) - 1, dtype=np.result_type(val, x))
    for r in range(len(crow) - 1):
        s, e = crow[r], crow[r + 1]
        y[r] = np.dot(val[s:e], x[col[s:e]])
    return y


def csr_transpose(crow, col, val, ncols):
    """CSR of Aᵀ with rows sorted by column index of A (stable in row order)."""
    rows = np.repeat(np.arange(len(crow) - 1), np.diff(crow))
    order = np.lexsort((rows, col))
    t_crow = np.zeros(ncols + 1, dtype=np.int64)
    np.add.at(t_crow, col + 1, 1)
    return np.cumsum(t_crow), rows[order], val[order]


def _pointers(idx, size):
    counts = np.bincount(idx, minlength=size)
    return np.concatenate(([0], np.cumsum(counts))).astype(np.int64)


def finish_cached(table_keys, table_values, rows, nf, old=None, missing=None):
    """``finish_cached_component`` (mac/cached_transfer_assembly.py:97-175):
    returns dict(slots, order, crow, cols, tcrow, tcols, values, reverse, new)
    for a first build (old None) or for the merge of `missing` keys into the
    pattern `old` (a dict of the same fields)."""
    table_keys = np.asarray(table_keys)
    if old is None:
        occupied = np.nonzero(table_keys >= 0)[0]
        order = np.argsort(table_keys[occupied], kind='stable')
        keys, slots = table_keys[occupied][order], occupied[order]
        rws, cols = keys // nf, keys % nf
        transpose = np.argsort(cols * rows + rws, kind='stable')
        crow, tcrow = _pointers(rws, rows), _pointers(cols, nf)
        new = len(keys)
    else:
        old_keys = table_keys[old['slots']]
        new_keys = np.unique(np.asarray(missing))
        at = np.searchsorted(old_keys, new_keys)
        exists = (at < len(old_keys)) & (old_keys[np.minimum(at, len(old_keys) - 1)] == new_keys)
        new_keys = new_keys[~exists]
        old_pos = np.arange(len(old_keys)) + np.searchsorted(new_keys, old_keys, side='right')
        new_pos = np.arange(len(new_keys)) + np.searchsorted(old_keys, new_keys)
        n = len(old_keys) + len(new_keys)
        keys = np.empty(n, np.int64)
        keys[old_pos], keys[new_pos] = old_keys, new_keys
        slots = np.empty(n, np.int64)
        slots[old_pos] = old['slots']
        slots[new_pos] = [int(np.nonzero(table_keys == k)[0][0]) for k in new_keys]
        rws, cols = keys // nf, keys % nf
        crow = old['crow'] + _pointers(new_keys // nf, rows)
        tcrow = old['tcrow'] + _pointers(new_keys % nf, nf)
        old_rev = old_keys[old['order']]
        old_rev = old_rev % nf * rows + old_rev // nf
        new_rev_keys = new_keys % nf * rows + new_keys // nf
        new_rev_order = np.argsort(new_rev_keys, kind='stable')
        new_rev = new_rev_keys[new_rev_order]
        old_rpos = np.arange(len(old_rev)) + np.searchsorted(new_rev, old_rev, side='right')
        new_rpos = np.arange(len(new_rev)) + np.searchsorted(old_rev, new_rev)
        transpose = np.empty(n, np.int64)
        transpose[old_rpos] = old_pos[old['order']]
        transpose[new_rpos] = new_pos[new_rev_order]
        new = len(new_keys)
    values = np.asarray(table_values)[slots]
    return dict(slots=slots, order=transpose, crow=crow, cols=cols, tcrow=tcrow, tcols=rws[transpose],
                values=values, reverse=values[transpose], new=new)
