"""Synthetic solve problems with the shapes, materials and boundary conditions
of the measured workloads (there is no public dataset for this solver; the
reference ships only hand-run Abaqus decks).

Each builder returns a ``Problem``: mesh arrays, initial velocity, per-DOF BC
arrays, material and controls, plus the node sets needed to write the same
model as an ``.inp`` deck for the reference CPU stepper.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import mesh as M


@dataclasses.dataclass
class Problem:
    name: str
    mesh: M.Mesh
    v0: np.ndarray                     # (n_nodes, 3)
    bc_code: np.ndarray                # (3*n_nodes,) int8
    bc_value: np.ndarray               # (3*n_nodes,) float64
    material: M.Material
    controls: M.Controls
    cycles: int                        # cycles of the measured run
    end_time: Optional[float] = None   # run-to-time workloads
    fixed_sets: List[Tuple[str, str]] = dataclasses.field(default_factory=list)
    initial_velocity: List[Tuple[str, int, float]] = dataclasses.field(default_factory=list)
    per_node_velocity: bool = False

    def write_deck(self, dirpath: str, deck: str = "model.inp", period: Optional[float] = None) -> str:
        """Writes deck + project.txt for the reference stepper; returns the deck name."""
        import os
        per = period if period is not None else (self.end_time or self.controls.total_time)
        M.write_deck(os.path.join(dirpath, deck), self.mesh, self.material, period=per,
                     fixed_sets=self.fixed_sets, initial_velocity=self.initial_velocity,
                     node_velocities=self.v0 if self.per_node_velocity else None,
                     bulk_viscosity=(self.controls.cvisl, self.controls.cvisq), gravity=self.controls.gravity)
        M.write_project(dirpath, deck, self.controls)
        return deck


DEFAULT_CONTROLS = dict(c_dr=0.013, c_cr=0.1, factor=0.9, cvisl=0.06, cvisq=1.2)


def cantilever(nx: int = 20, ny: int = 4, nz: int = 4, lx: float = 2.0, ly: float = 0.4, lz: float = 0.4,
               vz: float = 5.0, cycles: int = 2000, E: float = 210e9, nu: float = 0.3, rho: float = 7850.0,
               yield_stress: float = 0.0, tangent: float = 0.0) -> Problem:
    """Cantilever block: x = 0 face fixed (PINNED), all other nodes start with
    vz; the 20x4x4 default is the reference-runnable parity case (320
    elements, 525 nodes, 2000 cycles, FP64)."""
    m = M.box_mesh(nx, ny, nz, lx, ly, lz)
    fix = M.face_nodes(m, 0, "min")
    free = np.setdiff1d(np.arange(m.n_nodes), fix)
    m.node_sets = {"Set-1": fix, "Set-2": free}
    v0 = np.zeros((m.n_nodes, 3))
    v0[free, 2] = vz
    code, val = M.bc_arrays(m.n_nodes, fixed=[(fix, 0, 2)])
    ctl = M.Controls(total_time=1.0, **DEFAULT_CONTROLS)
    return Problem("cantilever_%dx%dx%d" % (nx, ny, nz), m, v0, code, val,
                   M.Material(E, nu, rho, yield_stress, tangent), ctl, cycles,
                   fixed_sets=[("Set-1", "PINNED")], initial_velocity=[("Set-2", 3, vz)])


def smoothed_gaussian_velocity(dims: Tuple[int, int, int], std: float, seed: int, passes: int = 3) -> np.ndarray:
    """Per-node, per-component N(0, std) velocities on an (nx+1, ny+1, nz+1)
    node lattice, smoothed by ``passes`` Jacobi sweeps (each value replaced by
    the mean over itself and its existing face neighbours)."""
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    v = rng.normal(0.0, std, size=(nz + 1, ny + 1, nx + 1, 3))
    for _ in range(passes):
        s = v.copy()
        cnt = np.ones(v.shape[:3] + (1,))
        for ax in range(3):
            lo = [slice(None)] * 4
            hi = [slice(None)] * 4
            lo[ax] = slice(0, -1)
            hi[ax] = slice(1, None)
            s[tuple(lo)] += v[tuple(hi)]
            s[tuple(hi)] += v[tuple(lo)]
            cnt[tuple(lo)] += 1
            cnt[tuple(hi)] += 1
        v = s / cnt
    return v.reshape(-1, 3)


def block(nx: int = 256, ny: int = 128, nz: int = 64, lx: float = 1.0, ly: float = 0.5, lz: float = 0.25,
          cycles: int = 5000, seed: int = 20241203, plastic: bool = True) -> Problem:
    """Large elastic-plastic block (roofline workload): 256x128x64 hexahedra
    (2,097,152 elements, 2,154,945 nodes) over 1.0 x 0.5 x 0.25 m, J2 with
    E = 70 GPa, nu = 0.33, rho = 2700, yield 250 MPa and a 100 MPa tangent
    modulus; bottom face (z = 0) fixed; seeded Gaussian nodal velocities
    (std 2 m/s) smoothed by 3 Jacobi passes; 5000 cycles.

    Hourglass viscosity is the reference's default c_cr = 0.05
    (exDyna3D.cpp:701) with dt factor 0.9: the random field excites the
    hourglass modes strongly, and with c_cr = 0.1 the reference algorithm's
    stable-dt estimate (which ignores hourglass viscosity) lets the solution
    grow without bound within ~200 cycles, on the CPU as on the GPU."""
    m = M.box_mesh(nx, ny, nz, lx, ly, lz)
    fix = M.face_nodes(m, 2, "min")
    m.node_sets = {"Set-1": fix}
    v0 = smoothed_gaussian_velocity((nx, ny, nz), 2.0, seed)
    v0[fix] = 0.0
    code, val = M.bc_arrays(m.n_nodes, fixed=[(fix, 0, 2)])
    mat = M.Material(70e9, 0.33, 2700.0, 250e6 if plastic else 0.0, 100e6 if plastic else 0.0)
    ctl = M.Controls(total_time=1.0, **dict(DEFAULT_CONTROLS, c_cr=0.05))
    return Problem("block_%dx%dx%d" % (nx, ny, nz), m, v0, code, val, mat, ctl, cycles,
                   fixed_sets=[("Set-1", "ENCASTRE")], per_node_velocity=True)


def impact_bar(n_core: int = 24, n_ring: int = 11, n_layers: int = 120, radius: float = 3.2e-3,
               length: float = 32.4e-3, v_impact: float = -190.0, end_time: float = 80e-6,
               plastic: bool = True) -> Problem:
    """Taylor-type impact bar: butterfly-meshed copper cylinder (r = 3.2 mm,
    L = 32.4 mm; by default a 24x24 core block and four 24x11 ring blocks per
    layer, 120 layers: 195,840 elements) with J2 (E 117 GPa, nu 0.35, rho
    8930, yield 400 MPa, tangent 100 MPa), z = 0 face fixed in z only, all
    nodes at vz = -190 m/s, run to 80 us.  The deck writes the z constraint as ZSYMM: the reference
    reader takes a dof-range line "Set-1, 3, 3" without a fourth field as
    condition 3, which fixes nothing (dataIn.cpp:978-1003 with
    exDyna3D.cpp:477-481)."""
    m = M.butterfly_cylinder(radius, length, n_core, n_ring, n_layers)
    bot = M.face_nodes(m, 2, "min")
    allnodes = np.arange(m.n_nodes)
    m.node_sets = {"Set-1": bot, "Set-2": allnodes}
    v0 = np.zeros((m.n_nodes, 3))
    v0[:, 2] = v_impact
    code, val = M.bc_arrays(m.n_nodes, fixed=[(bot, 2, 2)])
    mat = M.Material(117e9, 0.35, 8930.0, 400e6 if plastic else 0.0, 100e6 if plastic else 0.0)
    ctl = M.Controls(total_time=end_time, **DEFAULT_CONTROLS)
    return Problem("impact_bar", m, v0, code, val, mat, ctl, cycles=0, end_time=end_time,
                   fixed_sets=[("Set-1", "ZSYMM")], initial_velocity=[("Set-2", 3, v_impact)])


# dt factor of the sweep and serving problems (stable over nu in [0.25, 0.4])
SWEEP_DT_FACTOR = 0.8


def _tip_ramp(m: M.Mesh, free: np.ndarray, v_tip: float, length: float) -> np.ndarray:
    """Initial vz growing linearly from 0 at the clamp (x = 0) to v_tip at x = length."""
    v0 = np.zeros((m.n_nodes, 3))
    v0[free, 2] = v_tip * m.x0[free, 0] / length
    return v0


def sweep_instance(index: int, seed: int = 7, ne_min: int = 2000, ne_max: int = 60000, cycles: int = 3000,
                   tangent: float = 100e6) -> Problem:
    """Member ``index`` of the batched parameter sweep: a cantilever (even
    index; aspect 5:1:1, nx = 5k, ny = nz = k) or a plate (odd index; 1 x 1 m,
    k x k x 4 cells) clamped at x = 0, with its element count drawn
    log-uniform in [ne_min, ne_max] and, per instance and seeded, E in
    [50, 250] GPa, nu in [0.25, 0.4], rho in [2000, 9000] kg/m^3, J2 yield in
    [150, 600] MPa (tangent modulus ``tangent``) and a tip velocity in [1, 50]
    m/s: vz ramps linearly from 0 at the clamp to the tip value.

    Elements are cubes (the plate's thickness is 4 of its k in-plane cells)
    and the dt factor is SWEEP_DT_FACTOR: the reference's stable-dt estimate
    (exDyna3D.cpp:663-686) ignores the hourglass stiffness and viscosity, and
    with dt = 0.9 CFL its own algorithm diverges within ~100 cycles for
    Poisson ratios above ~0.33 or flat elements, on the CPU as on the GPU."""
    rng = np.random.default_rng([seed, index])
    target = float(np.exp(rng.uniform(np.log(ne_min), np.log(ne_max))))
    E = rng.uniform(50e9, 250e9)
    nu = rng.uniform(0.25, 0.4)
    rho = rng.uniform(2000.0, 9000.0)
    ys = rng.uniform(150e6, 600e6)
    v_tip = rng.uniform(1.0, 50.0)
    if index % 2 == 0:
        k = max(2, int(round((target / 5.0) ** (1.0 / 3.0))))
        nx, ny, nz = 5 * k, k, k
        lx, ly, lz = 2.0, 0.4, 0.4
    else:
        k = max(2, int(round(np.sqrt(target / 4.0))))
        nx, ny, nz = k, k, 4
        lx, ly, lz = 1.0, 1.0, 4.0 / k
    m = M.box_mesh(nx, ny, nz, lx, ly, lz)
    fix = M.face_nodes(m, 0, "min")
    free = np.setdiff1d(np.arange(m.n_nodes), fix)
    m.node_sets = {"Set-1": fix}
    v0 = _tip_ramp(m, free, v_tip, lx)
    code, val = M.bc_arrays(m.n_nodes, fixed=[(fix, 0, 2)])
    ctl = M.Controls(total_time=1.0, **dict(DEFAULT_CONTROLS, factor=SWEEP_DT_FACTOR))
    return Problem("sweep_%d" % index, m, v0, code, val, M.Material(E, nu, rho, ys, tangent), ctl, cycles,
                   fixed_sets=[("Set-1", "ENCASTRE")], per_node_velocity=True)


@dataclasses.dataclass
class Request:
    """One solve request of the serving stream."""

    index: int
    arrival: float        # seconds after the stream starts
    problem: Problem


def serving_requests(n: int, rate: float = 50.0, seed: int = 11, ne_min: int = 1000, ne_max: int = 500000,
                     steps: Tuple[int, int] = (1000, 10000)) -> List[Request]:
    """The serving stream: ``n`` requests arriving as a Poisson process of
    ``rate`` per second, each a structured block (cantilever aspect 5:1:1 or
    a 1 x 1 m plate of k x k x 4 cubes, chosen by a seeded draw) with its element
    count log-uniform in [ne_min, ne_max], elastic or J2 (seeded, half each),
    material and tip velocity drawn as in the batched sweep, and a cycle
    count uniform in ``steps``; dt factor SWEEP_DT_FACTOR as in the sweep."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        target = float(np.exp(rng.uniform(np.log(ne_min), np.log(ne_max))))
        plate = bool(rng.integers(0, 2))
        plastic = bool(rng.integers(0, 2))
        E = rng.uniform(50e9, 250e9)
        nu = rng.uniform(0.25, 0.4)
        rho = rng.uniform(2000.0, 9000.0)
        ys = rng.uniform(150e6, 600e6)
        v_tip = rng.uniform(1.0, 50.0)
        cycles = int(rng.integers(steps[0], steps[1] + 1))
        if plate:
            k = max(2, int(round(np.sqrt(target / 4.0))))
            nx, ny, nz, lx, ly, lz = k, k, 4, 1.0, 1.0, 4.0 / k
        else:
            k = max(2, int(round((target / 5.0) ** (1.0 / 3.0))))
            nx, ny, nz, lx, ly, lz = 5 * k, k, k, 2.0, 0.4, 0.4
        m = M.box_mesh(nx, ny, nz, lx, ly, lz)
        fix = M.face_nodes(m, 0, "min")
        free = np.setdiff1d(np.arange(m.n_nodes), fix)
        m.node_sets = {"Set-1": fix}
        v0 = _tip_ramp(m, free, v_tip, lx)
        code, val = M.bc_arrays(m.n_nodes, fixed=[(fix, 0, 2)])
        mat = M.Material(E, nu, rho, ys if plastic else 0.0, 100e6 if plastic else 0.0)
        ctl = M.Controls(total_time=1.0, **dict(DEFAULT_CONTROLS, factor=SWEEP_DT_FACTOR))
        out.append(Request(i, t, Problem("request_%d" % i, m, v0, code, val, mat, ctl, cycles,
                                         fixed_sets=[("Set-1", "ENCASTRE")], per_node_velocity=True)))
    return out
