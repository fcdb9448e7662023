"""Seeded synthetic O-grids around a symmetric NACA 00xx airfoil.

Writes the reference's mesh format (the Karman ASCII format read by
mesh_io.C:31-277: node count, coordinates, one block, triangles, quads,
boundaries made of two-node segments), its ``bc.dat`` (mesh_io.C:282-297,
one boundary-condition id per boundary) and its ``euler.params``
(params.C:27-217, 24 ordered (comment, value) line pairs).

Mesh family (all sizes derive from the circumferential x radial node count):

* surface nodes are cosine-clustered in arc length on each airfoil surface;
* ring r sits at fraction xi_r = (g**r - 1)/(g**(Nr-1) - 1) of the way from
  the surface point to a far-field circle of radius 20 chords around
  (0.5, 0); g = 1.15 for 32 rings, and finer meshes keep the same total
  stretch g**31 (g = 1.15**(31/(Nr-1))) so that the family refines evenly;
* each quad is split along a diagonal drawn from the seed (Bernoulli 1/2);
* nodes off the two boundary rings are jittered by U(-0.1, 0.1) x the local
  tangential and radial spacing;
* triangles are counter-clockwise and every boundary segment n0 -> n1 has the
  domain on its left, as Build_Boundary_Edge_Data needs (geometry.C:732-744).

Airfoils: y = +-0.6 (0.2969 sqrt(x) - 0.1260 x - 0.3516 x^2 + 0.2843 x^3 + c4 x^4).
``curved=False`` uses c4 = -0.1015 (open trailing edge, closed by one
straight wall segment) with the whole surface as one inviscid wall (bc 1).
``curved=True`` uses c4 = -0.1036, the closed-trailing-edge airfoil that the
reference's curved-boundary code hard-codes (curved_boundaries.C:50,61-71),
with the upper surface tagged bc 17 and the lower bc 19.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

FARFIELD_RADIUS = 20.0
FARFIELD_CENTER = (0.5, 0.0)
C4_OPEN = -0.1015
C4_CLOSED = -0.1036


def naca_y(x, c4):
    x = np.asarray(x, dtype=np.float64)
    return 0.6 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x * x
                  + 0.2843 * x * x * x + c4 * x * x * x * x)


def _surface_points(n_seg: int, c4: float, upper: bool) -> np.ndarray:
    """n_seg+1 points from the trailing edge (x=1) to the leading edge (x=0),
    cosine-clustered in arc length."""
    beta = np.linspace(0.0, np.pi, 40001)
    xf = 0.5 * (1.0 + np.cos(beta))          # 1 -> 0
    yf = naca_y(xf, c4)
    s = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(xf), np.diff(yf)))])
    j = np.arange(n_seg + 1)
    st = s[-1] * 0.5 * (1.0 - np.cos(np.pi * j / n_seg))
    x = np.interp(st, s, xf)
    x[0], x[-1] = 1.0, 0.0
    y = naca_y(x, c4)
    if not upper:
        y = -y
    return np.stack([x, y], axis=1)


@dataclass
class OGrid:
    nc: int
    nr: int
    curved: bool
    x: np.ndarray                    # (N, 2)
    tris: np.ndarray                 # (T, 3) 1-based
    boundaries: list = field(default_factory=list)   # list of (bc, segs (S,2) 1-based)

    @property
    def nn(self):
        return self.x.shape[0]


def make_ogrid(nc: int, nr: int, seed: int = 0, curved: bool = False,
               jitter: float = 0.1) -> OGrid:
    if nc < 8 or nr < 3 or nc % 2:
        raise ValueError("need an even nc >= 8 and nr >= 3")
    rng = np.random.Generator(np.random.PCG64(seed))

    # ---- surface loop, counter-clockwise around the airfoil, i = 0 at TE ----
    if curved:
        nh = nc // 2
        up = _surface_points(nh, C4_CLOSED, True)        # TE .. LE
        lo = _surface_points(nh, C4_CLOSED, False)[::-1]  # LE .. TE
        surf = np.concatenate([up, lo[1:-1]])             # TE shared, LE shared
    else:
        nu = nc // 2
        nl = nc - 1 - nu
        up = _surface_points(nu, C4_OPEN, True)
        lo = _surface_points(nl, C4_OPEN, False)[::-1]
        surf = np.concatenate([up, lo[1:]])               # open TE: 2 TE nodes
    assert surf.shape[0] == nc

    # ---- far-field points at evenly spaced angles, TE at angle 0 ----
    theta = 2.0 * np.pi * np.arange(nc) / nc
    outer = np.stack([FARFIELD_CENTER[0] + FARFIELD_RADIUS * np.cos(theta),
                      FARFIELD_CENTER[1] + FARFIELD_RADIUS * np.sin(theta)], axis=1)

    g = 1.15 ** (31.0 / (nr - 1))
    r = np.arange(nr)
    xi = (g ** r - 1.0) / (g ** (nr - 1) - 1.0)
    pts = surf[None, :, :] + (outer - surf)[None, :, :] * xi[:, None, None]  # (nr, nc, 2)
    pts[0] = surf
    pts[-1] = outer

    # ---- jitter interior rings in the local (tangential, radial) frame ----
    if jitter > 0.0 and nr > 2:
        inner = pts[1:-1]
        tvec = np.roll(inner, -1, axis=1) - np.roll(inner, 1, axis=1)
        ht = 0.5 * np.linalg.norm(tvec, axis=2)
        that = tvec / (2.0 * ht[..., None])
        rvec = pts[2:] - pts[:-2]
        hr = 0.5 * np.linalg.norm(rvec, axis=2)
        rhat = rvec / (2.0 * hr[..., None])
        # the local spacing is the smaller of the two neighbour distances
        ht_loc = np.minimum(np.linalg.norm(inner - np.roll(inner, 1, axis=1), axis=2),
                            np.linalg.norm(np.roll(inner, -1, axis=1) - inner, axis=2))
        hr_loc = np.minimum(np.linalg.norm(inner - pts[:-2], axis=2),
                            np.linalg.norm(pts[2:] - inner, axis=2))
        u = rng.uniform(-jitter, jitter, size=(nr - 2, nc, 2))
        pts[1:-1] = inner + (u[..., 0] * ht_loc)[..., None] * that \
            + (u[..., 1] * hr_loc)[..., None] * rhat
        del ht, hr

    x = pts.reshape(-1, 2).copy()

    def nid(i, k):
        return k * nc + (i % nc) + 1

    # ---- triangles: two per quad, quads row by row; the seeded diagonal
    # picks (a,b,c)+(a,c,d) or (a,b,d)+(b,c,d) ----
    diag = rng.integers(0, 2, size=(nr - 1, nc))
    kk, ii = np.meshgrid(np.arange(nr - 1, dtype=np.int64), np.arange(nc, dtype=np.int64),
                         indexing="ij")
    a, b = nid(ii, kk), nid(ii + 1, kk)
    c, d = nid(ii + 1, kk + 1), nid(ii, kk + 1)
    on = (diag == 1)[..., None]
    t1 = np.where(on, np.stack([a, b, c], -1), np.stack([a, b, d], -1))
    t2 = np.where(on, np.stack([a, c, d], -1), np.stack([b, c, d], -1))
    tris = np.stack([t1, t2], axis=2).reshape(-1, 3).astype(np.int64)
    p = x[tris - 1]
    area2 = (p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) \
        - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1])
    flip = area2 < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    if np.any(area2 == 0):
        raise ValueError("degenerate triangle")

    # ---- boundaries: far field CCW (domain inside), airfoil CW (domain outside)
    ic = np.arange(nc, dtype=np.int64)
    far = np.stack([nid(ic, nr - 1), nid(ic + 1, nr - 1)], axis=1)
    wall = np.stack([nid(ic + 1, 0), nid(ic, 0)], axis=1)
    bnds = [(0, far)]
    if curved:
        nh = nc // 2
        bnds.append((17, wall[:nh]))     # upper: segments between TE(0) and LE(nh)
        bnds.append((19, wall[nh:]))     # lower
    else:
        bnds.append((1, wall))
    grid = OGrid(nc=nc, nr=nr, curved=curved, x=x, tris=tris, boundaries=bnds)
    _check_segments(grid)
    return grid


def _check_segments(g: OGrid):
    """Every boundary segment n0->n1 must be a CCW edge of one triangle."""
    t = np.asarray(g.tris, dtype=np.int64)
    base = np.int64(g.nn + 1)
    edges = np.sort(np.concatenate([t[:, 0] * base + t[:, 1], t[:, 1] * base + t[:, 2],
                                    t[:, 2] * base + t[:, 0]]))
    for _, segs in g.boundaries:
        sg = np.asarray(segs, dtype=np.int64).reshape(-1, 2)
        key = sg[:, 0] * base + sg[:, 1]
        at = np.minimum(np.searchsorted(edges, key), len(edges) - 1)
        bad = edges[at] != key
        if bad.any():
            n0, n1 = sg[np.argmax(bad)]
            raise ValueError(f"segment {n0}->{n1} has the domain on its right")


def write_mesh(path: str, g: OGrid):
    lines = ["#Number of grid points", str(g.nn)]
    lines += ["%.17g %.17g" % (a, b) for a, b in g.x]
    lines += ["#Number of blocks", "1", "#Number of triangles", str(len(g.tris))]
    lines += ["%d %d %d" % tuple(t) for t in g.tris]
    lines += ["#Number of quads", "0", "#Number of boundaries", str(len(g.boundaries))]
    for b, (_, segs) in enumerate(g.boundaries):
        lines += ["#Number of edges on boundary %d" % (b + 1), str(len(segs))]
        lines += ["%d %d" % (s0, s1) for s0, s1 in segs]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_bc(path: str, g: OGrid):
    with open(path, "w") as f:
        f.write("".join("%d\n" % bc for bc, _ in g.boundaries))


@dataclass
class FlowParams:
    """The fields of the reference's euler.params, in file order
    (params.C:44-217; PARAMS in include/params.h:19-76)."""
    nsteps: int = 100
    iter: int = 1
    jufreq: int = 1
    CFL: float = 1.0e4
    ramp: int = 100
    gamma: float = 1.4
    alpha: float = 1.25
    mach: float = 0.5
    subits: int = 2
    unsteady: int = 0
    tacc: int = 0
    mintime: float = 0.01
    method: int = 1
    order: int = 1
    foits: int = 0
    soits: int = 0
    toits: int = 0
    isrestart: int = 0
    limit: int = 2
    reorder: int = 1
    ic: int = 0
    p_or_cv: int = 0
    start_post_pro: int = 0
    post_pro_freq: int = 0

    FIELDS = ("nsteps", "iter", "jufreq", "CFL", "ramp", "gamma", "alpha", "mach", "subits",
              "unsteady", "tacc", "mintime", "method", "order", "foits", "soits", "toits",
              "isrestart", "limit", "reorder", "ic", "p_or_cv", "start_post_pro",
              "post_pro_freq")


def write_params(path: str, p: FlowParams):
    lines = []
    for name in FlowParams.FIELDS:
        v = getattr(p, name)
        lines.append("#" + name)
        lines.append(("%.17g" % v) if isinstance(v, float) else str(int(v)))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_case(dirpath: str, g: OGrid, p: FlowParams, mesh_name: str = "grid.mesh") -> str:
    os.makedirs(dirpath, exist_ok=True)
    write_mesh(os.path.join(dirpath, mesh_name), g)
    write_bc(os.path.join(dirpath, "bc.dat"), g)
    write_params(os.path.join(dirpath, "euler.params"), p)
    return os.path.join(dirpath, mesh_name)
