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


# ---- known-answer fields (the reference's DEBUG_GRAD / DEBUG_DERIVS checks) ----
# Linear fields q_v = c0 + cx x + cy y, one row per conserved variable, chosen
# so that density and pressure stay positive on meshes out to radius 20.5.
LINEAR_COEF = np.array([[10.0, 0.125, 0.25],
                        [0.0, 0.375, 0.5],
                        [0.0, 0.625, 0.75],
                        [500.0, 0.875, 1.0]])
# Quadratics q_v = c0 + cx x + cy y + cxx x^2/2 + cyy y^2/2 + cxy x y.
QUAD_COEF = np.array([[30.0, 0.1, 0.1, 0.002, 0.002, 0.001],
                      [0.0, 0.3, -0.2, 0.001, -0.001, 0.002],
                      [0.0, -0.1, 0.4, -0.002, 0.001, 0.001],
                      [600.0, 0.5, 0.5, 0.003, 0.003, -0.002]])


def linear_state(Q0, x, nn):
    """Q0 with the real nodes' rows set to LINEAR_COEF at their coordinates
    (the ghost rows keep Q0's values)."""
    Q = Q0.reshape(-1, 4).copy()
    X = x.reshape(-1, 2)[1:nn + 1]
    Q[1:nn + 1] = LINEAR_COEF[:, :1].T + X @ LINEAR_COEF[:, 1:].T
    return Q.ravel()


def quad_derivs(X):
    """(fx, fy, fxx, fyy, fxy) of every QUAD_COEF row at points X: (n, 4, 5)."""
    c = QUAD_COEF
    x, y = X[:, :1], X[:, 1:2]
    return np.stack([c[:, 1] + c[:, 3] * x + c[:, 5] * y, c[:, 2] + c[:, 4] * y + c[:, 5] * x,
                     np.broadcast_to(c[:, 3], (len(X), 4)), np.broadcast_to(c[:, 4], (len(X), 4)),
                     np.broadcast_to(c[:, 5], (len(X), 4))], axis=2)


def quad_values(X):
    """QUAD_COEF's four quadratics at points X: (n, 4)."""
    c = QUAD_COEF
    x, y = X[:, :1], X[:, 1:2]
    return c[:, 0] + c[:, 1] * x + c[:, 2] * y + c[:, 3] * x * x / 2 + c[:, 4] * y * y / 2 \
        + c[:, 5] * x * y


def quadratic_state(Q0, x, moments, nn):
    """Q0 with the real nodes' rows set to the control-volume averages of the
    QUAD_COEF quadratics.  A quadratic's Taylor series about the node is
    exact, so its average over the node's volume is the node value plus the
    derivatives times the volume's moments about the node (moments[0..4]:
    the averages of dx, dy, dx^2, dy^2 and dx dy)."""
    Q = Q0.reshape(-1, 4).copy()
    X = x.reshape(-1, 2)[1:nn + 1]
    mo = moments.reshape(-1, 9)[1:nn + 1, :5]
    D = quad_derivs(X)
    w = np.array([1.0, 1.0, 0.5, 0.5, 1.0])
    Q[1:nn + 1] = quad_values(X) + np.einsum("nvk,nk->nv", D, mo * w)
    return Q.ravel()


def interior_nodes(bedges, nbedges, nn):
    """Nodes with no boundary face (1-based)."""
    b = np.unique(np.asarray(bedges).reshape(-1, 5)[1:nbedges + 1, 0])
    return np.setdiff1d(np.arange(1, nn + 1), b)


def closure_leak(mesh):
    """Per node |sum of the outward face normals| / (sum of the face lengths)
    of its median-dual control volume (cv_calc.C:379-640, cv_calc_check_closure):
    interior faces from the subedges (+ for the edge's left node, - for its
    right), boundary pieces from each boundary node to the segment's midpoint
    (the subedge's face point, the curved midpoint on a curved wall), each
    the integral of the outward normal along it, which is the piece's chord
    turned clockwise."""
    A, S = mesh.arrays(), mesh.sizes
    nn, ns = S["nn"], S["nsubedges"]
    se = A["subedges"].reshape(-1, 2)[1:ns + 1]
    ed = A["edges"].reshape(-1, 2)
    xn = A["xn_subedges"].reshape(-1, 3)[1:ns + 1]
    xm = A["xm_subedges"].reshape(-1, 2)[1:ns + 1]
    x = A["x"].reshape(-1, 2)
    L, R = ed[se[:, 0], 0], ed[se[:, 0], 1]
    f = xn[:, :2] * xn[:, 2:3]
    v = np.zeros((nn + 1, 2))
    per = np.zeros(nn + 1)
    np.add.at(v, L, f)
    np.add.at(v, R, -f)
    np.add.at(per, L, xn[:, 2])
    np.add.at(per, R, xn[:, 2])
    lo, hi = np.minimum(L, R).astype(np.int64), np.maximum(L, R).astype(np.int64)
    keys = lo * (nn + 1) + hi
    order = np.argsort(keys, kind="stable")
    _, _, _, seg = mesh.segments()
    seg = seg.reshape(-1, 2).astype(np.int64)
    sk = np.minimum(seg[:, 0], seg[:, 1]) * (nn + 1) + np.maximum(seg[:, 0], seg[:, 1])
    pos = np.searchsorted(keys[order], sk)
    assert np.array_equal(keys[order][pos], sk), "a boundary segment without its subedge"
    M = xm[order[pos]]
    for a, b, node in ((x[seg[:, 0]], M, seg[:, 0]), (M, x[seg[:, 1]], seg[:, 1])):
        d = b - a
        np.add.at(v, node, np.stack([d[:, 1], -d[:, 0]], axis=1))
        np.add.at(per, node, np.hypot(d[:, 0], d[:, 1]))
    return np.hypot(v[1:, 0], v[1:, 1]) / per[1:]


KAT_KINDS = ["triangles", "curved", "quads", "mixed", "cylinder"]


def kat_mesh(kind, order):
    """A 64x16 O-grid (48x12 around the unit circle for 'cylinder') of one of
    KAT_KINDS, preprocessed by the library; returns (mesh, params)."""
    from flowgpu.prep import Mesh
    d = tempfile.mkdtemp(prefix=f"kat_{kind}_")
    if kind in ("triangles", "curved"):
        _, _, fp = make_case(64, 16, kind == "curved", order, tmp=d)
    elif kind == "quads":
        fp = make_quad_case(64, 16, 3, d, order=order)
    elif kind == "mixed":
        fp = make_quad_case(64, 16, 3, d, order=order, quad_rings=7)
    else:
        fp = make_cylinder_case(48, 12, 4, d, order=order)
    return Mesh.from_case(d, order=order), fp
