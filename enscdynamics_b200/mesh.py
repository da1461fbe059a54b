"""Structured hexahedral meshes and Abaqus-subset ``.inp`` decks.

The stepper consumes a mesh as plain arrays: reference coordinates ``x0``
(n_nodes x 3, float64), connectivity ``conn`` (n_elements x 8, uint32,
0-based) in the reference's local node order, initial velocities and per-DOF
boundary-condition codes.  This module builds those arrays for the workloads
the stepper is measured on (cantilever blocks, the butterfly-meshed impact
cylinder) and writes the same model as an ``.inp`` deck that the reference
reader (``DataIn::read_inp``, Explicit3D/source/dataIn.cpp:300-558) parses, so
the reference CPU stepper can run the identical problem.

Deck constraints that come from the reference reader and are honoured here:

* node and element ids are 1..N in order, because the reader discards the id
  column (dataIn.cpp:576, 660);
* node sets are written at assembly level with ``instance=``; part-level sets
  are never transferred to the solver (dataIn.cpp:1653-1684);
* set names contain ``SET-`` because boundary / initial-condition lines are
  recognised as set references only by that substring (dataIn.cpp:928,
  1052, 1144);
* set members are separated by ", " since the set parser splits on blanks
  (dataIn.cpp:684-696);
* coordinates are printed with ``repr`` so ``std::stod`` recovers the exact
  float64 values held in ``x0``.

Local node order follows the reference hexahedron (Element_HexN8.cpp:49-91):
0 (-1,-1,-1), 1 (+1,-1,-1), 2 (+1,+1,-1), 3 (-1,+1,-1), then 4..7 at +1.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

# BC code bits per DOF, as applied by apply_boundary_condition_vec / _a
# (exDyna3D.cpp:379-490, 2029-2145).
BC_FIXED = 1      # SPC: v := 0, a := 0, reaction recorded
BC_VELOCITY = 2   # prescribed velocity: v := value, a := 0


@dataclasses.dataclass
class Mesh:
    """A hexahedral mesh in the stepper's array form."""

    x0: np.ndarray                      # (n_nodes, 3) float64
    conn: np.ndarray                    # (n_elements, 8) uint32
    node_sets: Dict[str, np.ndarray] = dataclasses.field(default_factory=dict)  # 0-based ids
    dims: Optional[Tuple[int, int, int]] = None   # structured grid cells, if any

    @property
    def n_nodes(self) -> int:
        return int(self.x0.shape[0])

    @property
    def n_elements(self) -> int:
        return int(self.conn.shape[0])


@dataclasses.dataclass
class Material:
    """Material_elastic (Material_elastic.h:8-21) plus the J2 parameters."""

    E: float
    nu: float
    rho: float
    yield_stress: float = 0.0       # <= 0: elastic, as in the reference
    tangent_modulus: float = 0.0    # Et; hardening H = E*Et/(E-Et)

    @property
    def hardening(self) -> float:
        if self.yield_stress <= 0.0:
            return 0.0
        return self.E * self.tangent_modulus / (self.E - self.tangent_modulus)


@dataclasses.dataclass
class Controls:
    """Solver constants read from project.txt / the deck (exDyna3D.h:176-185)."""

    c_dr: float = 0.013
    c_cr: float = 0.05
    factor: float = 0.71
    cvisl: float = 0.06
    cvisq: float = 1.2
    total_time: float = 1.0
    gravity: Optional[Tuple[float, Tuple[float, float, float]]] = None  # (value, dir)
    # gravity amplitude: (time, value) points of the *Amplitude the *Dload names
    gravity_amplitude: Optional[Sequence[Tuple[float, float]]] = None


def box_mesh(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float,
             origin: Sequence[float] = (0.0, 0.0, 0.0)) -> Mesh:
    """Structured nx*ny*nz hexahedra over [origin, origin + (lx, ly, lz)].

    Nodes are numbered i-fastest (i along x), elements likewise, so a warp of
    consecutive elements touches consecutive nodes.
    """
    xs = origin[0] + lx * (np.arange(nx + 1, dtype=np.float64) / nx)
    ys = origin[1] + ly * (np.arange(ny + 1, dtype=np.float64) / ny)
    zs = origin[2] + lz * (np.arange(nz + 1, dtype=np.float64) / nz)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    x0 = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    sx, sy = nx + 1, (nx + 1) * (ny + 1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (i + sx * j + sy * k).ravel()
    conn = np.stack([n0, n0 + 1, n0 + 1 + sx, n0 + sx,
                     n0 + sy, n0 + 1 + sy, n0 + 1 + sx + sy, n0 + sx + sy], axis=1).astype(np.uint32)
    m = Mesh(x0=np.ascontiguousarray(x0), conn=np.ascontiguousarray(conn), dims=(nx, ny, nz))
    return m


def face_nodes(mesh: Mesh, axis: int, side: str = "min", tol: float = 1e-12) -> np.ndarray:
    """0-based ids of nodes on the min/max face of the bounding box along axis."""
    c = mesh.x0[:, axis]
    ref = c.min() if side == "min" else c.max()
    return np.nonzero(np.abs(c - ref) <= tol * max(1.0, abs(ref)))[0].astype(np.int64)


def butterfly_cylinder(radius: float, length: float, n_core: int, n_ring: int, n_layers: int) -> Mesh:
    """Butterfly ("O-grid") hexahedral mesh of a solid cylinder along z.

    The cross-section is a central square block of n_core x n_core cells
    (half-width radius/2 * 0.6 ... blended toward a circle) surrounded by four
    ring blocks of n_core x n_ring cells that map the square's edges onto the
    circle.  Layers are uniform in z from 0 to ``length``.  Elements per layer:
    n_core**2 + 4*n_core*n_ring.
    """
    # --- 2-D cross-section -------------------------------------------------
    a = 0.5 * radius                     # half-width of the core square
    t = np.linspace(-1.0, 1.0, n_core + 1)
    pts: Dict[Tuple, int] = {}
    coords: List[Tuple[float, float]] = []

    def pid(key, xy):
        if key not in pts:
            pts[key] = len(coords)
            coords.append(xy)
        return pts[key]

    # core lattice keyed by integer (ix, iy); slightly bulged toward the circle
    core_id = np.zeros((n_core + 1, n_core + 1), dtype=np.int64)
    for iy in range(n_core + 1):
        for ix in range(n_core + 1):
            u, v = t[ix], t[iy]
            sq = np.array([u, v]) * a
            # blend 25% toward the circle of radius a*sqrt(2) for better shape
            r = np.hypot(u, v)
            circ = np.array([u, v]) / max(r, 1e-300) * a * max(abs(u), abs(v)) * np.sqrt(2.0) if r > 0 else sq
            xy = 0.75 * sq + 0.25 * circ
            core_id[iy, ix] = pid(("c", ix, iy), (float(xy[0]), float(xy[1])))
    # boundary walk of the core square, counter-clockwise, 4*n_core points
    walk: List[Tuple[int, int]] = []
    for ix in range(n_core):
        walk.append((ix, 0))
    for iy in range(n_core):
        walk.append((n_core, iy))
    for ix in range(n_core, 0, -1):
        walk.append((ix, n_core))
    for iy in range(n_core, 0, -1):
        walk.append((0, iy))
    nb = len(walk)
    ring_id = np.zeros((n_ring + 1, nb), dtype=np.int64)
    for w, (ix, iy) in enumerate(walk):
        ring_id[0, w] = core_id[iy, ix]
        inner = np.array(coords[core_id[iy, ix]])
        ang = np.arctan2(inner[1], inner[0])
        outer = np.array([np.cos(ang), np.sin(ang)]) * radius
        for r in range(1, n_ring + 1):
            s = r / n_ring
            xy = (1.0 - s) * inner + s * outer
            ring_id[r, w] = pid(("r", r, w), (float(xy[0]), float(xy[1])))
    xy = np.array(coords, dtype=np.float64)
    quads: List[Tuple[int, int, int, int]] = []
    for iy in range(n_core):
        for ix in range(n_core):
            quads.append((core_id[iy, ix], core_id[iy, ix + 1], core_id[iy + 1, ix + 1], core_id[iy + 1, ix]))
    for r in range(n_ring):
        for w in range(nb):
            w1 = (w + 1) % nb
            # counter-clockwise: inner(w) -> outer(w) is radial, walk is CCW
            quads.append((ring_id[r, w], ring_id[r, w1], ring_id[r + 1, w1], ring_id[r + 1, w]))
    quads_a = np.array(quads, dtype=np.int64)
    # orient every quad counter-clockwise (positive signed area)
    p0, p1, p2, p3 = (xy[quads_a[:, q]] for q in range(4))
    area = 0.5 * ((p2[:, 0] - p0[:, 0]) * (p3[:, 1] - p1[:, 1]) - (p3[:, 0] - p1[:, 0]) * (p2[:, 1] - p0[:, 1]))
    flip = area < 0
    quads_a[flip] = quads_a[flip][:, ::-1]
    # --- extrude -----------------------------------------------------------
    n2 = xy.shape[0]
    zs = length * (np.arange(n_layers + 1, dtype=np.float64) / n_layers)
    x0 = np.empty(((n_layers + 1) * n2, 3), dtype=np.float64)
    for l in range(n_layers + 1):
        x0[l * n2:(l + 1) * n2, 0:2] = xy
        x0[l * n2:(l + 1) * n2, 2] = zs[l]
    lay = np.arange(n_layers, dtype=np.int64)[:, None, None] * n2
    bot = quads_a[None, :, :] + lay
    conn = np.concatenate([bot, bot + n2], axis=2).reshape(-1, 8).astype(np.uint32)
    return Mesh(x0=x0, conn=np.ascontiguousarray(conn))


# --------------------------------------------------------------------------
# boundary conditions and initial velocities in array form

def bc_arrays(n_nodes: int, fixed: Iterable[Tuple[np.ndarray, int, int]] = (),
              velocity: Iterable[Tuple[np.ndarray, int, int, float]] = ()) -> Tuple[np.ndarray, np.ndarray]:
    """Per-DOF BC code/value arrays (length 3*n_nodes).

    ``fixed``: (nodes, first_dof, last_dof) with 0-based dofs, inclusive.
    ``velocity``: (nodes, first_dof, last_dof, value).
    """
    code = np.zeros(3 * n_nodes, dtype=np.int8)
    value = np.zeros(3 * n_nodes, dtype=np.float64)
    for nodes, d0, d1, val in velocity:
        for d in range(d0, d1 + 1):
            code[3 * np.asarray(nodes) + d] |= BC_VELOCITY
            value[3 * np.asarray(nodes) + d] = val
    for nodes, d0, d1 in fixed:
        for d in range(d0, d1 + 1):
            code[3 * np.asarray(nodes) + d] |= BC_FIXED
    return code, value


def check_slot_clashes(conn: np.ndarray, n_nodes: int) -> int:
    """Number of nodes that occupy the same local slot in more than one element.

    The reference's assembly scatters each element's slot-k force into slot
    vector k (exDyna3D.cpp:584-634); with a clash the OpenMP loop races.  The
    node-centric gather here is deterministic either way; this count is
    reported for parity runs, where a clash-free mesh keeps the reference
    deterministic at any thread count.
    """
    clashes = 0
    for k in range(8):
        counts = np.bincount(conn[:, k].astype(np.int64), minlength=n_nodes)
        clashes += int(np.count_nonzero(counts > 1))
    return clashes


# --------------------------------------------------------------------------
# deck writer

def _fmt(v: float) -> str:
    return repr(float(v))


def _write_set(f, name: str, ids0: np.ndarray, instance: str = "Part-1-1") -> None:
    ids = np.asarray(ids0, dtype=np.int64) + 1
    f.write(f"*Nset, nset={name}, instance={instance}\n")
    for s in range(0, len(ids), 16):
        f.write(", ".join(str(int(v)) for v in ids[s:s + 16]) + "\n")


def write_deck(path: str, mesh: Mesh, material: Material, *, period: float,
               fixed_sets: Sequence[Tuple[str, str]] = (),
               initial_velocity: Sequence[Tuple[str, int, float]] = (),
               node_velocities: Optional[np.ndarray] = None,
               bulk_viscosity: Tuple[float, float] = (0.06, 1.2),
               gravity: Optional[Tuple[float, Tuple[float, float, float]]] = None,
               amplitude: Optional[Sequence[Tuple[float, float]]] = None) -> None:
    """Writes an ``.inp`` deck of the model for the reference reader.

    ``fixed_sets``: (set name, spec) with spec e.g. ``"PINNED"`` or ``"3, 3"``.
    ``initial_velocity``: (set name, 1-based dof, value).
    ``node_velocities``: optional (n_nodes, 3) array written as per-node
    initial-condition lines (node id, dof, value); zeros are skipped.
    Sets referenced must be present in ``mesh.node_sets`` (names contain
    ``Set-``).
    ``amplitude``: (time, value) points of the gravity load's amplitude,
    written on one line because DataIn::AMP keeps only the last data line of
    an *Amplitude block (dataIn.cpp:1249-1268).
    """
    with open(path, "w") as f:
        f.write("*Heading\n** generated by enscdynamics_b200.mesh\n")
        f.write("*Part, name=Part-1\n*Node\n")
        for i, (x, y, z) in enumerate(mesh.x0):
            f.write(f"{i + 1}, {_fmt(x)}, {_fmt(y)}, {_fmt(z)}\n")
        f.write("*Element, type=C3D8R\n")
        for e, c in enumerate(mesh.conn.astype(np.int64) + 1):
            f.write(f"{e + 1}, " + ", ".join(str(int(v)) for v in c) + "\n")
        f.write("*End Part\n*Assembly, name=Assembly\n*Instance, name=Part-1-1, part=Part-1\n*End Instance\n")
        for name, ids in mesh.node_sets.items():
            _write_set(f, name, ids)
        f.write("*End Assembly\n")
        f.write("*Material, name=Material-1\n*Density\n")
        f.write(f"{_fmt(material.rho)},\n*Elastic\n{_fmt(material.E)}, {_fmt(material.nu)}\n")
        for name, spec in fixed_sets:
            f.write(f"*Boundary\n{name}, {spec}\n")
        if initial_velocity or node_velocities is not None:
            f.write("*Initial Conditions, type=VELOCITY\n")
            for name, dof, val in initial_velocity:
                f.write(f"{name}, {dof}, {_fmt(val)}\n")
            if node_velocities is not None:
                for i in range(node_velocities.shape[0]):
                    for d in range(3):
                        val = node_velocities[i, d]
                        if val != 0.0:
                            f.write(f"{i + 1}, {d + 1}, {_fmt(val)}\n")
        if amplitude:
            f.write("*Amplitude, name=Amp-1\n")
            f.write(", ".join(f"{_fmt(t)}, {_fmt(a)}" for t, a in amplitude) + "\n")
        f.write("*Step, name=Step-1, nlgeom=YES\n*Dynamic, Explicit\n")
        f.write(f", {_fmt(period)}\n")
        f.write(f"*Bulk Viscosity\n{_fmt(bulk_viscosity[0])}, {_fmt(bulk_viscosity[1])}\n")
        if gravity is not None:
            g, d = gravity
            f.write("*Dload, amplitude=Amp-1\n" if amplitude else "*Dload\n")
            f.write(f", GRAV, {_fmt(g)}, {_fmt(d[0])}, {_fmt(d[1])}, {_fmt(d[2])}\n")
        f.write("*End Step\n")


def write_project(dirpath: str, deck_name: str, controls: Controls) -> str:
    """Writes the positional project.txt the reference reads
    (exDyna3D.cpp:698-772: c_dr on line 5, c_cr on line 8, factor on line 11,
    time_interval on line 14)."""
    p = os.path.join(dirpath, "project.txt")
    with open(p, "w") as f:
        f.write("#inp file name\n")
        f.write(deck_name + "\n")
        f.write("#\n# Stiffness Hourglass Control parameter\n")
        f.write(f"{_fmt(controls.c_dr)}\n")
        f.write("#\n# Viscosity Hourglass Control parameter\n")
        f.write(f"{_fmt(controls.c_cr)}\n")
        f.write("#\n# factor of time step\n")
        f.write(f"{_fmt(controls.factor)}\n")
        f.write("#\n# time interval of output\n")
        f.write("1.0\n")
    return p
