"""Shared set-up of parity cases: one O-grid, the reference solver on it, and
the grid arrays in the reference layout that the oracle and the CUDA library
are fed with."""
from __future__ import annotations

import os
import tempfile

import numpy as np

from flowgpu import meshgen
from oracle import port
from oracle.ref import RefSolver


def make_case(nc, nr, curved, order, seed=3, mach=None, ramp=1111, tmp=None, **kw):
    g = meshgen.make_ogrid(nc, nr, seed=seed, curved=curved)
    fp = meshgen.FlowParams(order=order, mach=(mach if mach is not None else (0.5 if order == 1 else 0.8)),
                            ramp=ramp, **kw)
    d = tmp or tempfile.mkdtemp(prefix=f"case_{nc}x{nr}_")
    meshgen.write_case(d, g, fp)
    return d, g, fp


class ParityCase:
    """Reference after its first solve() (so that the lazily built edge
    weights, k=2 stencils and SVD factors exist), with the state before that
    step kept to start the other implementations from."""

    def __init__(self, nc, nr, curved, order, **kw):
        self.dir, self.grid, self.fp = make_case(nc, nr, curved, order, **kw)
        self.ref = RefSolver(self.dir)
        self.Q0 = self.ref.array("Q")
        self.xnb0 = self.ref.array("xn_bedges")
        self.dq1 = self.ref.solve(1)
        self.sizes, self.arrays = port.reference_arrays(self.ref, with_svd=(order == 3))
        self.arrays["xn_bedges"] = self.xnb0
        self.arrays["Q"] = self.Q0
        self.sizes["nelem"] = self.sizes["ntri"] + self.sizes["nquad"]
        self.ts = 1

    def ref_step(self):
        """Advance the reference one step (step 1 already ran at set-up)."""
        if self.ts > 1:
            self.ref.solve(self.ts)
        self.ts += 1


def bitwise(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b)


def ndiff(a, b):
    return int(np.count_nonzero(np.asarray(a) != np.asarray(b)))


def chunk_order(ia, ja, starts):
    """The row permutation of a mode 3 forward sweep, restated: chunks get
    the smallest colour no earlier adjacent chunk holds; colours ascending,
    chunks ascending, rows ascending."""
    nn = int(starts[-1]) - 1
    chunk_of = np.zeros(nn + 1, dtype=np.int64)
    for q in range(len(starts) - 1):
        chunk_of[starts[q]:starts[q + 1]] = q
    colour = []
    for q in range(len(starts) - 1):
        used = {colour[int(chunk_of[ja[k]])] for j in range(starts[q], starts[q + 1])
                for k in range(ia[j], ia[j + 1]) if chunk_of[ja[k]] < q}
        c = 0
        while c in used:
            c += 1
        colour.append(c)
    order = [j for c in range(max(colour) + 1) for q in range(len(colour)) if colour[q] == c
             for j in range(starts[q], starts[q + 1])]
    return np.asarray(order, dtype=np.int32), max(colour) + 1
