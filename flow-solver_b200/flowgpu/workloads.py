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
    # the precision form's mesh: 2048 x 512 O-grid (1.05M nodes), k=2, M 0.8
    "ogrid2048x512_k2_m080": Workload("ogrid2048x512_k2_m080", 2048, 512, True, 3, 0.8,
                                      max_steps=40000),
    # the largest mesh of the batch16 requests (request 3 of stream 0): the
    # roofline mesh of the batching bench
    "ogrid704x176_k2_m077": Workload("ogrid704x176_k2_m077", 704, 176, True, 3, 0.773228,
                                     alpha=-0.786252, seed=1003),
    # the largest mesh of the batch64 requests that the FP64 drop-in solves
    # (request 26 of stream 0, 181,476 nodes): the roofline mesh of the bench
    "ogrid852x213_k2_m076": Workload("ogrid852x213_k2_m076", 852, 213, True, 3, 0.762224,
                                     alpha=3.631312, seed=1026),
    # the small k=1 case: 128 x 32 O-grid, M 0.5, straight walls (a parity case:
    # with the reference's limiter 2 it settles into a limit cycle)
    "ogrid128x32_k1_m050": Workload("ogrid128x32_k1_m050", 128, 32, False, 1, 0.5),
}

DEFAULT = "ogrid512x128_k2_m080"   # the single-mesh drop-in workload
DEFAULT_BENCH = "batch64"           # bench.py's default: the batching form, 64 solves per GPU


def get(name: str) -> Workload:
    return WORKLOADS[name]


def with_steps(w: Workload, n: int) -> Workload:
    return replace(w, steps_to_converge=n)


@dataclass(frozen=True)
class BatchWorkload:
    """The batching form: ``n`` independent requests per GPU from the seeded
    request stream (flowgpu.serve.sample_request: node counts log-uniform in
    [2k, 200k] with a 4:1 circumferential:radial ratio, Mach U[0.3, 0.85],
    angle of attack U[-4, 6] degrees, k=1 or k=2), all admitted together to
    one server and each retired at a ``drop`` of ||R_rho|| or after
    ``max_steps`` pseudo-time steps.  ``precision``/``subits``: the served
    form (flow_set_precision mode and Gauss-Seidel sweeps per step).

    ``fp64_steps`` / ``fp64_status``: what the FP64 drop-in (bit-identical to
    the reference, so these are the reference's own counts) does on requests
    0..n-1 of the stream: steps taken and 0 converged, 256 stopped at
    max_steps, other values failed (a non-physical state).  Measured with
    ``bench.py --measure-fp64``.

    ``stall``, ``stall_drop``, ``stall_per_sqrt``: the server retires a solve
    whose best ||R_rho|| has not dropped by the factor ``stall_drop`` within
    max(``stall``, ``stall_per_sqrt`` * sqrt(nodes)) steps.  On batch64's
    requests served in precision mode 3 with 4 sweeps and the approximate
    face Jacobians, the longest run without a halving before convergence
    grows with the mesh (32 steps at 2k nodes, 128 at 41k, 320 at 181k: at
    most 0.75 sqrt(nodes)); the window max(160, 1.4 sqrt(nodes)) is at least
    1.9 times each converging solve's longest such run;
    ``autotune``: steps per kernel variant timed at admission."""
    name: str
    seed: int
    n: int
    max_steps: int
    drop: float
    precision: int
    subits: int
    chunk: int = 32
    fp64_steps: tuple | None = None
    fp64_status: tuple | None = None
    stall: int = 0
    stall_drop: float = 10.
    stall_per_sqrt: float = 0.
    autotune: int = 0
    fp64_forces: tuple | None = None  # raw lift/drag of the FP64 drop-in per request
    priority_policy: int = 0          # 1: larger meshes on higher-priority streams
    jacobian: int = 0                 # precision-form face Jacobians (flow_set_jacobian)
    fp64_steps4: tuple | None = None  # the FP64 drop-in's steps / status with 4 sweeps per step
    fp64_status4: tuple | None = None


BATCHES = {
    # the batching form as specified: 64 independent solves in one arena
    # (requests 0..63 of stream 0 on rank 0, the next 64 on rank 1, ...)
    "batch64": BatchWorkload("batch64", 0, 64, 8000, 1e-10, 3, 4, stall=160, stall_drop=2., stall_per_sqrt=1.4, autotune=4,
                             priority_policy=1, jacobian=2,
                             fp64_steps=(8000, 8000, 324, 8000, 4441, 8000, 921, 392, 8000, 64, 1249, 1148, 1065, 1395, 1487, 8000, 3827, 1262, 8000, 415, 3035, 64, 8000, 1475, 810, 8000, 7340, 3346, 64, 278, 536, 8000, 64, 1087, 2309, 415, 2513, 930, 8000, 8000, 8000, 64, 8000, 64, 3705, 8000, 6900, 1978, 5921, 8000, 4285, 1743, 1794, 8000, 3477, 8000, 2040, 64, 1585, 64, 64, 912, 8000, 2687),
                             fp64_status=(256, 256, 0, 256, 0, 256, 0, 0, 256, 44, 0, 0, 0, 0, 0, 256, 0, 0, 256, 0, 0, 44, 256, 0, 0, 256, 0, 0, 44, 0, 0, 256, 44, 0, 0, 0, 0, 0, 256, 256, 256, 44, 256, 44, 0, 256, 0, 0, 0, 256, 0, 0, 0, 256, 0, 256, 0, 44, 0, 44, 44, 0, 256, 0),
                             fp64_steps4=(8000, 8000, 172, 128, 2240, 8000, 474, 213, 64, 64, 640, 590, 556, 715, 760, 8000, 1907, 673, 8000, 230, 1536, 64, 8000, 746, 414, 8000, 3777, 1673, 64, 154, 286, 8000, 64, 563, 1160, 225, 1258, 479, 8000, 8000, 8000, 64, 8000, 64, 1847, 8000, 3444, 1003, 2978, 8000, 2215, 898, 911, 8000, 1744, 8000, 1023, 64, 833, 64, 64, 471, 8000, 1401),
                             fp64_status4=(256, 256, 0, 44, 0, 256, 0, 0, 44, 44, 0, 0, 0, 0, 0, 256, 0, 0, 256, 0, 0, 44, 256, 0, 0, 256, 0, 0, 44, 0, 0, 256, 44, 0, 0, 0, 0, 0, 256, 256, 256, 44, 256, 44, 0, 256, 0, 0, 0, 256, 0, 0, 0, 256, 0, 256, 0, 44, 0, 44, 44, 0, 256, 0),
                             fp64_forces=(None, None, (-0.025777386029756044, -0.0054055864833447076), None, (-0.0010171575037174392, -0.001240139392816858), None, (-0.027248649454864958, -0.003062564172084038), (-0.12773519262622307, -0.018852769853473013), None, None, (-0.018041588523432805, -0.002214218243070119), (0.002168299510290521, -0.0016691959198755204), (0.028612422320067932, -0.005656445411432563), (-0.0017219682626121772, -0.0013359229295129356), (-0.03246397561528733, -0.0029672357554528374), None, (-0.07621782393542069, -0.0048012799301380355), (-0.20986626352195453, -0.028688895204014832), None, (0.04666059516157848, -0.008005804230765284), (0.019087319252602365, -0.001482639953373573), None, None, (0.039936872659750385, -0.0038141957773608157), (0.0003257405055705526, -0.001822215172047123), None, (-0.19177442021253613, -0.01723684073456574), (0.0432973120624181, -0.00339450845774449), None, (0.03188269948663082, -0.007280141883886639), (0.018382161826746297, -0.0106550912117282), None, None, (-0.024456547136083084, -0.005018145472129145), (0.010818981126226179, -0.002387014107041504), (-0.04440898199151, -0.0075415065311262445), (0.0655803205867983, -0.004950069442132337), (-0.0023400526814139192, -0.001771997899719281), None, None, None, None, None, None, (-0.02007443256463631, -0.0037642781088572694), None, (-0.06933146954849441, -0.0035062312826888565), (-0.08868317689152848, -0.007610661826188901), (0.04559064820540709, -0.0026394350417630777), None, (-0.17617304809434906, -0.016650205797371188), (-0.026475309051357494, -0.008758498911407755), (0.004735135354381516, -0.0016012204784226426), None, (0.02617089666340069, -0.001790390307587515), None, (0.07619508554929875, -0.005998724380028264), None, (0.0537048432982277, -0.005541582009699136), None, None, (-0.0355744365642943, -0.005129144991253361), None, (0.19662866543828933, -0.02542728332062686))),
    # its first 16 requests: a quarter of the work, for quick runs
    "batch16": BatchWorkload(
        "batch16", 0, 16, 8000, 1e-10, 3, 4, stall=160, stall_drop=2., stall_per_sqrt=1.4, autotune=4, priority_policy=1,
        fp64_steps=(8000, 8000, 324, 8000, 4441, 8000, 921, 392, 8000, 64, 1249, 1148, 1065,
                    1395, 1487, 8000),
        fp64_status=(256, 256, 0, 256, 0, 256, 0, 0, 256, 44, 0, 0, 0, 0, 0, 256),
        fp64_forces=((0.04361406644387807, -0.0012359952118082152), (-0.1077942504305611, -0.0016940082793635751), (-0.025777386029756044, -0.0054055864833447076), (0.04696757004279522, -0.0057328563651535954), (-0.0010171575037174392, -0.001240139392816858), (-0.0023481805252991883, -0.0018965591568374796), (-0.027248649454864958, -0.003062564172084038), (-0.12773519262622307, -0.018852769853473013), (0.10544934901923901, -0.007440799548675984), None, (-0.018041588523432805, -0.002214218243070119), (0.002168299510290521, -0.0016691959198755204), (0.028612422320067932, -0.005656445411432563), (-0.0017219682626121772, -0.0013359229295129356), (-0.03246397561528733, -0.0029672357554528374), (-0.0480551902857968, -0.001438821319776097))),
}
