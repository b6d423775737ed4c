"""CPU restatement of the reference's Barnes-Hut library, for accuracy
comparisons only (test infrastructure, like the rest of oracle/; nothing in
the library calls it).

The reference's tree gravity (misc/SPHgravtree_lib/grav_force_tree.cu over
libSequoia) cannot be built here: libSequoia's Makefile compiles its kernels
to sm_20 PTX, which nvcc 12.9 no longer targets.  This module restates its
algorithm so that its error on a given input and opening angle can be
measured and set beside this library's tree mode:

  * particles sorted along a Peano-Hilbert curve (support_kernels.cu:113-182;
    the index here is Skilling's construction, J. Skilling, AIP Conf. Proc.
    707, 381 (2004));
  * octree cells are the 3-bit prefixes of the key; a cell below level
    LEVEL_MIN = 3 always splits, deeper cells are leaves when they hold at
    most NLEAF = 64 particles (build_tree.cu:9, :456-459, :553-555,
    node_specs.h:21);
  * per cell: mass, centre of mass, the second moment per unit mass about it
    (compute_properties.cu:20-31, :270-288) and the tight bounding box; the
    opening radius is (l / theta)^2 with l twice the largest half size
    (compute_properties.cu:320-342);
  * groups of NCRIT = 64 consecutive particles (build_tree.cu:792-822,
    node_specs.h:23) with their tight bounding boxes;
  * a cell is opened when the gap between the group's and the cell's boxes
    is at most l / theta (dev_shared_traverse_functions.cu:305-337); opened
    leaves interact particle by particle with the softened kernel (body_body,
    dev_approximate_gravity.cu:60-140), accepted cells through monopole plus
    quadrupole (body_node, dev_approximate_gravity.cu:141-188).

Arithmetic is FP64 throughout, so the measured error is the algorithm's;
the particle pairs come from the oracle's row form (the CPU-path formulas,
which body_body follows for nkernel 0).
"""
from __future__ import annotations

import numpy as np

import oracle

NLEAF = 64
NCRIT = 64
LEVEL_MIN = 3
BITS = 21  # per axis: 63-bit keys


def hilbert_keys(pos: np.ndarray, bits: int = BITS) -> np.ndarray:
    """Peano-Hilbert index of each point (Skilling's axes-to-transpose, then
    the transposed bits interleaved most significant first)."""
    lo = pos.min(axis=0)
    span = max(float((pos.max(axis=0) - lo).max()), 1e-300)
    q = np.minimum(((pos - lo) / span * ((1 << bits) - 1)).astype(np.int64), (1 << bits) - 1)
    X = [q[:, 0].copy(), q[:, 1].copy(), q[:, 2].copy()]
    n = 3
    M = 1 << (bits - 1)
    Q = M
    while Q > 1:  # inverse undo
        P = Q - 1
        for i in range(n):
            hit = (X[i] & Q) != 0
            t = (X[0] ^ X[i]) & P
            X[0] = np.where(hit, X[0] ^ P, X[0] ^ t)
            if i:
                X[i] = np.where(hit, X[i], X[i] ^ t)
        Q >>= 1
    for i in range(1, n):  # Gray encode
        X[i] ^= X[i - 1]
    t = np.zeros_like(X[0])
    Q = M
    while Q > 1:
        t = np.where((X[n - 1] & Q) != 0, t ^ (Q - 1), t)
        Q >>= 1
    for i in range(n):
        X[i] ^= t
    key = np.zeros(pos.shape[0], dtype=np.uint64)
    for b in range(bits - 1, -1, -1):
        for i in range(n):
            key = (key << np.uint64(1)) | ((X[i] >> b) & 1).astype(np.uint64)
    return key


class Tree:
    """Cells of the sorted particles: ranges, children, leaf flags, multipoles, boxes."""

    def __init__(self, pos: np.ndarray, m: np.ndarray, keys: np.ndarray, theta: float):
        n = pos.shape[0]
        start, end, level, child0, nchild = [0], [n], [0], [-1], [0]
        frontier = [0]
        for lev in range(BITS):
            nxt = []
            sh = np.uint64(3 * (BITS - 1 - lev))
            for c in frontier:
                a, b = start[c], end[c]
                if lev >= LEVEL_MIN and b - a <= NLEAF:
                    continue  # leaf
                digits = (keys[a:b] >> sh) & np.uint64(7)
                cuts = np.flatnonzero(np.diff(digits)) + 1
                bounds = np.concatenate([[0], cuts, [b - a]]) + a
                child0[c] = len(start)
                nchild[c] = len(bounds) - 1
                for k in range(len(bounds) - 1):
                    start.append(int(bounds[k]))
                    end.append(int(bounds[k + 1]))
                    level.append(lev + 1)
                    child0.append(-1)
                    nchild.append(0)
                    nxt.append(len(start) - 1)
            frontier = nxt
            if not frontier:
                break
        self.start = np.array(start)
        self.end = np.array(end)
        self.child0 = np.array(child0)
        self.nchild = np.array(nchild)
        self.leaf = self.nchild == 0
        nn = len(start)
        self.mass = np.zeros(nn)
        self.com = np.zeros((nn, 3))
        self.q = np.zeros((nn, 3, 3))  # second moment per unit mass about the centre of mass
        self.centre = np.zeros((nn, 3))
        self.half = np.zeros((nn, 3))
        for c in range(nn):
            p, w = pos[start[c]:end[c]], m[start[c]:end[c]]
            M = w.sum()
            com = (w[:, None] * p).sum(axis=0) / M
            d = p - com
            self.mass[c] = M
            self.com[c] = com
            self.q[c] = (w[:, None, None] * d[:, :, None] * d[:, None, :]).sum(axis=0) / M
            lo, hi = p.min(axis=0), p.max(axis=0)
            self.centre[c] = 0.5 * (lo + hi)
            self.half[c] = 0.5 * (hi - lo)
        el = 2.0 * self.half.max(axis=1)
        self.op2 = (el / theta) ** 2 if theta > 0 else np.full(nn, np.inf)

    def walk(self, gc: np.ndarray, gh: np.ndarray):
        """Accepted cells and opened leaves of the group with box centre gc
        and half sizes gh (minimum-distance criterion)."""
        cells, leaves = [], []
        F = np.array([0])
        while F.size:
            # boxes compared with a 1e-12 relative margin: rounding must not
            # put a group's own particle (a one-particle leaf on the group
            # box's face) outside the group and make it act on itself
            slack = 1e-12 * (np.abs(gc) + gh + np.abs(self.centre[F]) + self.half[F])
            gap = np.maximum(np.abs(gc - self.centre[F]) - (gh + self.half[F]) - slack, 0.0)
            split = (gap ** 2).sum(axis=1) <= self.op2[F]
            cells.append(F[~split])
            leaves.append(F[split & self.leaf[F]])
            inner = F[split & ~self.leaf[F]]
            F = np.concatenate([np.arange(self.child0[c], self.child0[c] + self.nchild[c]) for c in inner]) \
                if inner.size else np.zeros(0, dtype=np.int64)
        return np.concatenate(cells), np.concatenate(leaves)


def body_node(p: np.ndarray, M: np.ndarray, com: np.ndarray, q: np.ndarray):
    """Monopole + quadrupole of cells (M, com, q per unit mass) at points p:
    returns (acc (k, 3), pot (k,)) summed over the cells."""
    dr = p[:, None, :] - com[None, :, :]                     # target - centre
    r2 = (dr ** 2).sum(axis=2)
    ids = 1.0 / np.sqrt(r2)
    D0, D1, D2, D3 = ids * M, -ids ** 3 * M, 3 * ids ** 5 * M, -15 * ids ** 7 * M
    qii = np.trace(q, axis1=1, axis2=2)[None, :]
    qd = np.einsum('cab,kcb->kca', q, dr)
    qrr = (qd * dr).sum(axis=2)
    c01 = D1 + 0.5 * D2 * qii + 0.5 * D3 * qrr
    acc = (c01[:, :, None] * dr + D2[:, :, None] * qd).sum(axis=1)
    pot = -(D0 + 0.5 * D1 * qii + 0.5 * D2 * qrr).sum(axis=1)
    return acc, pot


def forces(x, y, z, m, range2, theta: float, nkernel: int = 0, only=None):
    """The reference tree's (ax, ay, az, pot) for every particle, in input
    order.  With ``only`` (input indices), just the groups holding those
    particles are walked; the other rows come back as NaN."""
    pos = np.stack([x, y, z], axis=1).astype(np.float64)
    n = pos.shape[0]
    keys = hilbert_keys(pos)
    order = np.argsort(keys, kind='stable')
    ps, ms, r2s = pos[order], np.asarray(m, np.float64)[order], np.asarray(range2, np.float64)[order]
    tree = Tree(ps, ms, keys[order], theta)
    out = np.full((n, 4), np.nan)
    starts = range(0, n, NCRIT)
    if only is not None:
        inv = np.empty(n, dtype=np.int64)
        inv[order] = np.arange(n)
        starts = sorted(set(int(g) for g in (inv[np.asarray(only)] // NCRIT) * NCRIT))
    for g0 in starts:
        g1 = min(g0 + NCRIT, n)
        gp = ps[g0:g1]
        lo, hi = gp.min(axis=0), gp.max(axis=0)
        cells, leaves = tree.walk(0.5 * (lo + hi), 0.5 * (hi - lo))
        acc = np.zeros((g1 - g0, 3))
        pot = np.zeros(g1 - g0)
        if cells.size:
            a, p = body_node(gp, tree.mass[cells], tree.com[cells], tree.q[cells])
            acc += a
            pot += p
        # the group's own leaves are always opened (gap 0), so its particles
        # are among the sources; rows are their places in the sorted list
        src = np.sort(np.concatenate([np.arange(tree.start[c], tree.end[c]) for c in leaves]))
        rows = np.searchsorted(src, np.arange(g0, g1)).astype(np.int32)
        ax, ay, az, pp = oracle.rows(ps[src, 0], ps[src, 1], ps[src, 2], ms[src], r2s[src], nkernel,
                                     row_idx=rows, nthreads=1)
        acc += np.stack([ax, ay, az], axis=1)
        pot += pp
        out[g0:g1, :3] = acc
        out[g0:g1, 3] = pot
    res = np.empty((n, 4))
    res[order] = out
    return res[:, 0], res[:, 1], res[:, 2], res[:, 3]
