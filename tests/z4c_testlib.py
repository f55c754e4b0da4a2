"""Shared helpers of the test suite: golden-fixture loading, block-order
mapping between the reference (gid order) and the B200 context (grid order),
and the comparison metrics."""
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
NG = 4


class Case:
    """One golden fixture with its geometry."""

    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.rec = {k: z[k] for k in z.files}
        self.params = json.loads(str(self.rec["params"]))
        self.mesh = json.loads(str(self.rec["mesh"]))
        self.integrator = json.loads(str(self.rec["integrator"]))
        meta = self.rec["meta"]
        self.nx = [int(meta[0, 5]), int(meta[0, 6]), int(meta[0, 7])]
        self.nn = [n + 1 + 2 * NG for n in self.nx]
        self.nb = self.mesh["nb"]
        # reference gid -> grid index l0 + nb0*(l1 + nb1*l2)
        self.order = [int(m[2] + self.nb[0] * (m[3] + self.nb[1] * m[4])) for m in meta]

    def to_grid(self, a):
        out = np.empty_like(a)
        for g, o in enumerate(self.order):
            out[o] = a[g]
        return out

    def from_grid(self, a):
        return np.stack([a[o] for o in self.order])

    def blocks(self):
        """oracle Block geometry per block (gid order)."""
        import z4c_oracle as O
        out = []
        n0, n1 = self.nn[0], self.nn[1]
        for b in range(len(self.order)):
            xf, xv = self.rec["xf"][b], self.rec["xv"][b]
            out.append(O.Block(self.nx, self.rec["dx"][b],
                               [xf[:n0], xf[n0:n0 + n1], xf[n0 + n1:]],
                               [xv[:n0 - 1], xv[n0 - 1:n0 + n1 - 2], xv[n0 + n1 - 2:]]))
        return out

    def interior(self):
        nn = self.nn
        return (slice(None), slice(None), slice(NG, nn[2] - NG), slice(NG, nn[1] - NG),
                slice(NG, nn[0] - NG))


def rel_err(a, b):
    """Normwise relative difference over a register: max|a-b| / max|b|, over
    the finite entries of b; NaN/Inf positions must coincide."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    fin = np.isfinite(b)
    if not np.array_equal(fin, np.isfinite(a)):
        return np.inf
    d = np.abs(a[fin] - b[fin])
    m = np.abs(b[fin]).max() if fin.any() else 0.0
    if d.size == 0:
        return 0.0
    return float(d.max() / m) if m > 0 else float(d.max())


def var_rel_err(a, b, axis=1, floor=1e-10):
    """Worst per-variable normwise relative difference; a variable whose
    reference magnitude is below floor*max over all variables is measured
    against that floor (round-off noise around zero)."""
    a = np.asarray(a)
    b = np.asarray(b)
    big = np.nanmax(np.abs(np.where(np.isfinite(b), b, 0)))
    worst = 0.0
    for n in range(b.shape[axis]):
        an, bn = np.take(a, n, axis=axis), np.take(b, n, axis=axis)
        fin = np.isfinite(bn)
        if not np.array_equal(fin, np.isfinite(an)):
            return np.inf
        if not fin.any():
            continue
        d = np.abs(an[fin] - bn[fin]).max()
        m = max(np.abs(bn[fin]).max(), floor * big)
        worst = max(worst, d / m if m > 0 else d)
    return float(worst)


def bitwise(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.array_equal(np.nan_to_num(a, nan=7.0), np.nan_to_num(b, nan=7.0))
