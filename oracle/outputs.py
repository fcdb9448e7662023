"""CPU restatement of the reference's solution writers (grid_io.C), the
checker of flow_surface_cp / flow_write_surface_cp / flow_write_tecplot.

Test infrastructure only: imported by tests/, never by the library.  Arrays
are in the reference's layout (1-based, array-of-structs): Q (nn+ng+1)*4,
x (nn+ng+1)*2, tri (ntri+1)*3 and quad (nquad+1)*4 with row 0 unused, and the
boundary segments as one list of (n0, n1) pairs per boundary (GRID::bs).
numpy evaluates each elementwise expression below in the written order with
IEEE double rounding and no contraction, as the reference's C does.
"""
from __future__ import annotations

import math

import numpy as np


def boundary_nodes(segments) -> list[int]:
    """Unique nodes of one boundary's segments in first-appearance order, n0
    before n1 of each segment (grid_io.C:1294-1349)."""
    seen, out = set(), []
    for n0, n1 in segments:
        for n in (n0, n1):
            if n not in seen:
                seen.add(n)
                out.append(int(n))
    return out


def surface_cp(Q: np.ndarray, nodes, gamma: float, mach: float) -> np.ndarray:
    """Pressure coefficient of the listed nodes from GRID::Q in conserved form
    (grid_io.C:1314-1320): P = (g-1)(e - r(u^2+v^2)/2), p_inf = 1/g (:879),
    Cp = (P/p_inf - 1) * 2/(g M^2)."""
    q = Q.reshape(-1, 4)[np.asarray(nodes, dtype=np.int64)]
    r = q[:, 0]
    u = q[:, 1] / r
    v = q[:, 2] / r
    e = q[:, 3]
    P = (gamma - 1.) * (e - 0.5 * r * (u * u + v * v))
    pinf = 1. / gamma
    return (P / pinf - 1.) * (2. / (gamma * mach * mach))


def _sort_g_key(line: str):
    """`sort -g` under the C locale (grid_io.C:1368): the leading number
    (lines without one first, NaN before every number), ties by the bytes of
    the whole line."""
    tok = line.split(None, 1)[0] if line.strip() else ""
    try:
        val = float(tok)
    except ValueError:
        return (0, 0.0, line.encode())
    if math.isnan(val):
        return (1, 0.0, line.encode())
    return (2, val, line.encode())


def surface_cp_files(Q, x, bbc, segments, gamma: float, mach: float) -> dict[int, bytes]:
    """write_surface_cp (grid_io.C:841-1375, the branch taken for order <= 6):
    per inviscid boundary b (bbc[b] != 0 and odd, :887) the bytes of
    surface_<b>_pressure.dat, lines "%f  %f" of (float) x and (float) Cp,
    sorted as the reference's shell sort leaves them.  bbc is 1-based;
    segments[b-1] lists boundary b's (n0, n1) pairs."""
    out = {}
    x = np.asarray(x, dtype=np.float64)
    for b in range(1, len(bbc)):
        bc = int(bbc[b])
        if bc == 0 or math.fmod(bc, 2) == 0:
            continue
        nodes = boundary_nodes(segments[b - 1])
        cp = surface_cp(Q, nodes, gamma, mach)
        lines = ["%f  %f\n" % (float(np.float32(x[2 * n])), float(np.float32(c)))
                 for n, c in zip(nodes, cp)]
        lines.sort(key=_sort_g_key)
        out[b] = "".join(lines).encode()
    return out


def tecplot_values(Q, nn: int, primitive: bool, tri_only: bool, gamma: float) -> np.ndarray:
    """The four values per real node a Tecplot file prints: Q (conserved,
    grid_io.C:138-141) or rho, u, v, P (grid_io.C:252-258 for a triangle-only
    mesh, grid_io.C:285-290 otherwise)."""
    q = Q.reshape(-1, 4)[1:nn + 1]
    if not primitive:
        return q.copy()
    rho = q[:, 0]
    u = q[:, 1] / rho
    v = q[:, 2] / rho
    E = q[:, 3]
    if tri_only:
        P = (gamma - 1.) * E - ((gamma - 1.) / 2.) * rho * (u * u + v * v)
    else:
        P = (gamma - 1.) * E - ((gamma - 1.) / (2. * rho)) * (u * u + v * v)
    return np.stack([rho, u, v, P], axis=1)


def tecplot_bytes(Q, x, nn: int, tri, quad, primitive: bool, gamma: float) -> bytes:
    """write_tecplot_solutionC (grid_io.C:102-199) / write_tecplot_solutionP
    (grid_io.C:216-331): header, one point-data zone of the nn real nodes and
    the element connectivity (triangles as degenerate quadrilaterals when the
    mesh has quadrilaterals)."""
    tri = np.asarray(tri).reshape(-1, 3)
    quad = np.asarray(quad).reshape(-1, 4)
    ntri, nquad = len(tri) - 1, len(quad) - 1
    vals = tecplot_values(Q, nn, primitive, nquad == 0, gamma)
    xy = np.asarray(x, dtype=np.float64).reshape(-1, 2)[1:nn + 1]
    parts = ['TITLE="data file"\n']
    if primitive:
        parts.append('VARIABLES="X", "Y", "Rho", "U", "V", "P"\n')
    else:
        parts.append('VARIABLES="X", "Y", "Rho", "Umom", "Vmom", "E"\n')
    if nquad == 0:
        parts.append("ZONE N=%d, E=%d, DATAPACKING=POINT, ZONETYPE=FETRIANGLE\n" % (nn, ntri))
    else:
        parts.append("ZONE N=%d, E=%d, DATAPACKING=POINT, ZONETYPE=FEQUADRILATERAL\n"
                     % (nn, ntri + nquad))
    fmt = "%.15e %.15e %.15e %.15e %.15e %.15e\n"
    parts.extend(fmt % (a, b, c, d, e, f) for (a, b), (c, d, e, f) in zip(xy.tolist(), vals.tolist()))
    parts.append("\n")
    if nquad == 0:
        parts.extend("%d %d %d\n" % tuple(t) for t in tri[1:].tolist())
    else:
        parts.extend("%d %d %d %d\n" % (t[0], t[1], t[2], t[2]) for t in tri[1:].tolist())
        parts.extend("%d %d %d %d\n" % tuple(t) for t in quad[1:].tolist())
    return "".join(parts).encode()
