"""Benchmark and test workloads: seeded synthetic O-grids and flow conditions.

Each entry is a steady solve run to a 1e-10 drop of the density residual
norm ||R[:,0]||_2 (relative to the first pseudo-time step).  The reference's
CFL ramp is linear from 1 (init_memory.C:200-216); ramp = 1111 makes the
second step's CFL 10, so the ramp runs 1 -> 10 -> ... -> 1e4.

``steps_to_converge`` is the number of pseudo-time steps the solve takes.
It is a property of the workload alone: the CUDA drop-in reproduces the
reference's iterates bit for bit, so both take the same count.  It is used
to convert a timed sample of reference steps into reference solves/s.
"""
from __future__ import annotations

import os
import tempfile
from dataclasses import dataclass, replace

from . import meshgen


@dataclass(frozen=True)
class Workload:
    name: str
    nc: int
    nr: int
    curved: bool
    order: int
    mach: float
    alpha: float = 1.25
    ramp: int = 1111
    CFL: float = 1.0e4
    subits: int = 2
    limit: int = 2
    seed: int = 1
    drop: float = 1e-10
    max_steps: int = 20000
    steps_to_converge: int | None = None

    def params(self) -> meshgen.FlowParams:
        return meshgen.FlowParams(order=self.order, mach=self.mach, alpha=self.alpha,
                                  ramp=self.ramp, CFL=self.CFL, subits=self.subits,
                                  limit=self.limit, nsteps=self.max_steps)

    def grid(self) -> meshgen.OGrid:
        return meshgen.make_ogrid(self.nc, self.nr, seed=self.seed, curved=self.curved)

    def write(self, dirpath: str | None = None) -> str:
        """Write mesh, bc.dat and euler.params; returns the case directory."""
        d = dirpath or tempfile.mkdtemp(prefix=f"flow_{self.name}_")
        meshgen.write_case(d, self.grid(), self.params())
        return d


WORKLOADS = {
    # the headline workload: 512 x 128 O-grid, M 0.8, AoA 1.25, k=2, curved NACA 0012, FP64
    "ogrid512x128_k2_m080": Workload("ogrid512x128_k2_m080", 512, 128, True, 3, 0.8,
                                     steps_to_converge=4826),
    # a 16x smaller member of the same family, for quick runs
    "ogrid128x32_k2_m080": Workload("ogrid128x32_k2_m080", 128, 32, True, 3, 0.8,
                                    steps_to_converge=691),
    # the small k=1 case: 128 x 32 O-grid, M 0.5, straight walls (a parity case:
    # with the reference's limiter 2 it settles into a limit cycle)
    "ogrid128x32_k1_m050": Workload("ogrid128x32_k1_m050", 128, 32, False, 1, 0.5),
}

DEFAULT = "ogrid512x128_k2_m080"


def get(name: str) -> Workload:
    return WORKLOADS[name]


def with_steps(w: Workload, n: int) -> Workload:
    return replace(w, steps_to_converge=n)
