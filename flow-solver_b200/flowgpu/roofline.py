"""Algorithmic (compulsory) DRAM bytes per launch of the main kernels.

Each figure counts every array element a launch must read or write once:
per-node records, per-face records, incidence lists, stencils, and the
outputs.  Neighbour gathers of node states are counted once per node (the
rest are cache hits by construction).  The achieved bandwidth of a launch is
these bytes over its measured duration; DRAM traffic measured by ncu well
above them would mean re-reads.
"""
from __future__ import annotations

import numpy as np


def _sizes(mesh) -> dict:
    v = mesh.view
    out = {"nn": v.nn, "ns": v.nsubedges, "ne": v.nedges, "nbe": v.nbedges, "stencil": 0}
    if mesh.order == 3:
        m = np.ctypeslib.as_array(v.svd_m, shape=(v.nn + 1,))
        out["stencil"] = int(m[1:].sum())
    nnz = int(np.ctypeslib.as_array(v.ia, shape=(v.nn + 2,))[v.nn + 1])
    out["nnz"] = nnz
    return out


def node_prepare_bytes(mesh) -> int:
    """k_node_prepare4: wave-speed sum and dt, the k=1 gradient or the k=2
    derivatives (x = V S^-1 U^T b over the node's stencil) and point value,
    and the Venkatakrishnan limiter over every face point.

    per node   read  nQ 32, x 16, cv_area 8, three incidence pointers 12
                     (k=2: moments 72, V^T 200, S 40, stencil pointer 4)
               write dt 8, phi 64 (k=1: grad 64; k=2: derivatives 160, point values 32)
    per subedge      two incidence entries 8, normal/length 32,
                     face point offsets 32 (k=1) or 3 Gauss points 48 (k=2)
    per edge         two neighbour entries 8 (k=1: two incidence entries 8, LSQ weights 32)
    per bedge        incidence entry 4, normal/length 24
    per stencil entry (k=2) index 4, weight 8, the row of U's first 5 columns 40
    """
    z = _sizes(mesh)
    k2 = mesh.order == 3
    per_node = 32 + 16 + 8 + 12 + 8 + 64 + ((72 + 200 + 40 + 4 + 160 + 32) if k2 else 64)
    per_sub = 8 + 32 + (48 if k2 else 32)
    per_edge = 8 + (0 if k2 else 8 + 32)
    per_bedge = 4 + 24
    return int(z["nn"] * per_node + z["ns"] * per_sub + z["ne"] * per_edge +
               z["nbe"] * per_bedge + z["stencil"] * 52)


def colour_sweep_bytes(mesh) -> int:
    """One whole multicolour FP32 sweep (all colour launches): per row the
    row record 16, right-hand side 32 (FP64), LU factors 64, the iterate
    written 16; per off-diagonal block its column 4, the block 64 (FP32) and
    the neighbour iterate 16."""
    z = _sizes(mesh)
    offd = z["nnz"] - z["nn"]
    return int(z["nn"] * (16 + 32 + 64 + 16) + offd * (4 + 64 + 16))


def ordered_sweep_bytes(mesh) -> int:
    """One FP64 ordered sweep (k_sweep_ordered): per block 128 B of LHS and
    4 B of column index, per row RHS, LU of the diagonal, dQ read and write
    (132 B per block + 96 B per row, the diagonal block counted as a block)."""
    z = _sizes(mesh)
    return int(132 * z["nnz"] + 96 * z["nn"])


def chunk_sweep_bytes(mesh) -> int:
    """One whole chunked FP32 sweep (precision mode 3, all colour launches):
    per row its 640-byte sweep record (header, right-hand side, LU factors,
    8 columns, 8 FP32 blocks) staged once, its iterate read through the
    chunk's window and written back (16 + 16)."""
    z = _sizes(mesh)
    return int(z["nn"] * (640 + 16 + 16))


def subedge_flux_bytes(mesh, jacobian: bool = True, approx: bool = False) -> int:
    """k_subedge_flux: per subedge its end nodes 8, normal/length 32 and the
    two node states 64 read (k=1 reconstruction: the two nodes' gradients
    128, limiters 16 and the face-point offsets 32), the flux 32 written and,
    with the Jacobian, dF/dqL and dF/dqR: 256 (FP64) or, for the approximate
    Jacobian of the precision form, 128 (FP32)."""
    z = _sizes(mesh)
    jac = (128 if approx else 256) if jacobian else 0
    per = 8 + 32 + 64 + (0 if mesh.order == 3 else 128 + 16 + 32) + 32 + jac
    return int(z["ns"] * per)


def assemble_bytes(mesh, precision: int = 3, approx: bool = False) -> int:
    """k_assemble4: per subedge incidence (two a subedge) its entry 4, the
    face's flux 32 and Jacobian block J read; per off-diagonal block its
    subedge pair 16 and the one or two face Jacobians (two a block on these
    meshes) 2J read; per node dt, cv_area 16 read, R and RHS 64 written and
    its row written: two 640-byte sweep records (mode 3), or FP64 blocks
    128 a block and LU factors 128 (mode 0).  J = 128 (FP64) or 64 (the
    approximate Jacobian's FP32 blocks)."""
    z = _sizes(mesh)
    offd = z["nnz"] - z["nn"]
    J = 64 if approx else 128
    row = 2 * 640 if precision == 3 else 128 * z["nnz"] / max(z["nn"], 1) + 128
    return int(2 * z["ns"] * (4 + 32 + J) + offd * (16 + 2 * J) + z["nn"] * (16 + 64 + row))


def faces_assemble_bytes(mesh) -> int:
    """k_faces_assemble (precision form, approximate Jacobian): per subedge
    incidence its entry and block slot 8, the face's end nodes 8,
    normal/length 32 and the other node's state 32 read (k=1: the two nodes'
    gradients and limiters 144 and the offsets 32); per node its own state
    32, dt and cv_area 16, R and RHS 64 and its two 640-byte sweep records;
    per boundary edge its flux and Jacobian 160 read."""
    z = _sizes(mesh)
    per_inc = 8 + 8 + 32 + 32 + (0 if mesh.order == 3 else 144 + 32)
    return int(2 * z["ns"] * per_inc + z["nn"] * (32 + 16 + 64 + 2 * 640) + z["nbe"] * 160)
