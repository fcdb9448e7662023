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

    def __init__(self, nc, nr, curved, order, quads=False, cylinder=False, **kw):
        if cylinder:  # triangles around the unit circle (curved wall bc 11)
            self.dir = tempfile.mkdtemp(prefix=f"cyl_{nc}x{nr}_")
            self.grid = None
            self.fp = make_cylinder_case(nc, nr, kw.get("seed", 4), self.dir, order=order)
        elif quads:  # quadrilaterals (quads="mixed": inner half quads, outer triangles)
            self.dir = tempfile.mkdtemp(prefix=f"qcase_{nc}x{nr}_")
            self.grid = None
            # M 0.5: at M 0.8 the blunt trailing edge of the straight-wall
            # grids drives the reference's k=2 ghost states non-physical
            self.fp = make_quad_case(nc, nr, kw.get("seed", 3), self.dir,
                                     mach=kw.get("mach") or 0.5, order=order,
                                     quad_rings=(nr - 1) // 2 if quads == "mixed" else None)
        else:
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


def make_quad_case(nc, nr, seed, d, mach=0.6, order=1, ramp=1111, quad_rings=None):
    """An O-grid of quadrilaterals (the generator's nodes, quads not split,
    straight walls), written as a case directory the reference reads;
    returns its params.  quad_rings: only the first that many rings of cells
    are quadrilaterals, the rest the generator's triangles (a mixed mesh)."""
    import os as _os
    g = meshgen.make_ogrid(nc, nr, seed=seed)
    x = g.x
    nid = lambda i, k: k * nc + (i % nc) + 1
    nq = nr - 1 if quad_rings is None else quad_rings
    tris = [t for t in g.tris.tolist() if min(t) > nq * nc] if nq < nr - 1 else []
    quads = []
    for k in range(nq):
        for i in range(nc):
            q = [nid(i, k), nid(i + 1, k), nid(i + 1, k + 1), nid(i, k + 1)]
            p = x[np.array(q) - 1]
            area = 0.5 * sum(p[j, 0] * p[(j + 1) % 4, 1] - p[(j + 1) % 4, 0] * p[j, 1]
                             for j in range(4))
            quads.append(q[::-1] if area < 0 else q)
    lines = ["#Number of grid points", str(len(x))] + ["%.17g %.17g" % (a, b) for a, b in x]
    lines += ["#Number of blocks", "1", "#Number of triangles", str(len(tris))]
    lines += ["%d %d %d" % tuple(t) for t in tris]
    lines += ["#Number of quads", str(len(quads))] + ["%d %d %d %d" % tuple(q) for q in quads]
    lines += ["#Number of boundaries", str(len(g.boundaries))]
    for b, (_, segs) in enumerate(g.boundaries):
        lines += ["#Number of edges on boundary %d" % (b + 1), str(len(segs))]
        lines += ["%d %d" % (s0, s1) for s0, s1 in segs]
    _os.makedirs(d, exist_ok=True)
    with open(_os.path.join(d, "grid.mesh"), "w") as f:
        f.write("\n".join(lines) + "\n")
    meshgen.write_bc(_os.path.join(d, "bc.dat"), g)
    fp = meshgen.FlowParams(order=order, mach=mach, ramp=ramp)
    meshgen.write_params(_os.path.join(d, "euler.params"), fp)
    return fp


def startup_parity_case(nc, nr, curved, order, foits, soits=0, **kw):
    """ParityCase for runs that start with `foits` first-order steps (and,
    for k=2, `soits` second-order ones).  The reference builds what a phase
    needs at that phase's first step (the LSQ edge weights at the first
    gradient, gradient.C:364-367; the grown k=2 stencils and their SVD
    factors at the first k=2 step, solve.C:57-114); these depend on the mesh
    alone, so they are taken from a second reference run advanced past
    them."""
    case = ParityCase(nc, nr, curved, order, foits=foits, soits=soits, **kw)
    if foits + soits > 0:
        geo = RefSolver(case.dir)
        for ts in range(1, foits + soits + 2):
            geo.solve(ts)
        _, a = port.reference_arrays(geo, with_svd=(order == 3))
        keys = []
        if order == 1 or soits > 0:
            keys.append("edge_weight")
        if order == 3:
            keys += ["gnsn", "gnnsn", "gnnsn1", "svd_m", "svd_off", "svd_U", "svd_VT", "svd_S"]
        for k in keys:
            case.arrays[k] = a[k]
        geo.close()
    return case


def make_cylinder_case(nc, nr, seed, d, mach=0.3, order=3, wall_bc=11, ramp=1111):
    """An O-grid of triangles around the unit circle (the reference's curved
    circular wall, bc 11) out to radius 20 (far field, bc 0), written as a
    case directory the reference reads; returns its params."""
    import os as _os
    rng = np.random.Generator(np.random.PCG64(seed))
    th = 2.0 * np.pi * np.arange(nc) / nc
    ratio = 20.0 ** (1.0 / (nr - 1))
    r = ratio ** np.arange(nr)
    r[-1] = 20.0
    x = np.stack([np.outer(r, np.cos(th)).ravel(), np.outer(r, np.sin(th)).ravel()], axis=1)
    nid = lambda i, k: k * nc + (i % nc) + 1
    diag = rng.integers(0, 2, size=(nr - 1, nc))
    tris = []
    for k in range(nr - 1):
        for i in range(nc):
            a, b, c, e = nid(i, k), nid(i + 1, k), nid(i + 1, k + 1), nid(i, k + 1)
            for t in ([a, b, c], [a, c, e]) if diag[k, i] else ([a, b, e], [b, c, e]):
                p = x[np.array(t) - 1]
                area = ((p[1, 0] - p[0, 0]) * (p[2, 1] - p[0, 1])
                        - (p[2, 0] - p[0, 0]) * (p[1, 1] - p[0, 1]))
                tris.append(t if area > 0 else [t[0], t[2], t[1]])
    far = [(nid(i, nr - 1), nid(i + 1, nr - 1)) for i in range(nc)]
    wall = [(nid(i + 1, 0), nid(i, 0)) for i in range(nc)]
    bnds = [(0, far), (wall_bc, wall)]
    lines = ["#Number of grid points", str(len(x))] + ["%.17g %.17g" % (a, b) for a, b in x]
    lines += ["#Number of blocks", "1", "#Number of triangles", str(len(tris))]
    lines += ["%d %d %d" % tuple(t) for t in tris]
    lines += ["#Number of quads", "0", "#Number of boundaries", str(len(bnds))]
    for b, (_, segs) in enumerate(bnds):
        lines += ["#Number of edges on boundary %d" % (b + 1), str(len(segs))]
        lines += ["%d %d" % (s0, s1) for s0, s1 in segs]
    _os.makedirs(d, exist_ok=True)
    with open(_os.path.join(d, "grid.mesh"), "w") as f:
        f.write("\n".join(lines) + "\n")
    with open(_os.path.join(d, "bc.dat"), "w") as f:
        f.write("".join("%d\n" % bc for bc, _ in bnds))
    fp = meshgen.FlowParams(order=order, mach=mach, ramp=ramp, alpha=0.0)
    meshgen.write_params(_os.path.join(d, "euler.params"), fp)
    return fp
