"""Shared helpers for the tests: golden fixtures and solver construction."""
import glob
import json
import os

import numpy as np

from enscdynamics_b200 import mesh as M
from enscdynamics_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# FP64 parity bar against the reference CPU stepper (relative to the field's
# max magnitude), as stated for the plain path.
REL_TOL_REFERENCE = 1e-9


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["meta"] = json.loads(str(d["meta"]))
    if "regenerate" in d["meta"]:
        d.update(regenerated_model(d["meta"]["regenerate"]))
    return d


def regenerated_model(spec):
    """Model arrays of a fixture that stores the parameters of its synthetic
    workload instead of the arrays: rebuilt and checked against the SHA-256
    the fixture recorded when the reference ran it."""
    import hashlib
    from enscdynamics_b200 import workloads as W
    assert spec["workload"] == "block", spec
    p = W.block(*spec["dims"], *spec["lengths"], seed=spec["seed"], plastic=False)
    arrays = dict(x0=p.mesh.x0, conn=p.mesh.conn, v0=p.v0, bc_code=p.bc_code, bc_value=p.bc_value)
    for k, a in arrays.items():
        h = hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
        assert h == spec["sha256"][k], f"rebuilt {k} differs from the array the reference ran"
    return arrays


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    b = np.asarray(b, dtype=np.float64).reshape(-1)
    scale = np.abs(b).max()
    if scale == 0.0:
        return float(np.abs(a).max())
    return float(np.abs(a - b).max() / scale)


def sampled(g, key, a):
    """The part of a computed field that fixture g holds: all of it, or (for
    a large reference deck) the rows at its sampled nodes / elements."""
    a = np.asarray(a)
    idx = "out_elements" if key in ("sigma", "qia") else "out_nodes"
    if idx not in g:
        return a.reshape(-1)
    rows = len(g["conn"]) if idx == "out_elements" else len(g["x0"])
    return a.reshape(rows, -1)[g[idx]].reshape(-1)


def material_controls(meta):
    mat = M.Material(meta["E"], meta["nu"], meta["rho"], meta.get("yield", 0.0), meta.get("tangent", 0.0))
    g = meta.get("gravity")
    ctl = M.Controls(c_dr=meta["c_dr"], c_cr=meta["c_cr"], factor=meta["factor"], cvisl=meta["cvisl"],
                     cvisq=meta["cvisq"], total_time=meta["total_time"],
                     gravity=None if g is None else (g[0], tuple(g[1])),
                     gravity_amplitude=meta.get("amplitude"))
    return mat, ctl


def oracle_for(g, setup_from_reference=False, **overrides):
    import pyoracle
    meta = dict(g["meta"])
    meta.update(overrides)
    setup = dict(bt=g["bt"], vol0=g["vol0"], inv_mass=g["inv_mass"]) if setup_from_reference else None
    return pyoracle.Oracle(g["x0"], g["conn"], g["v0"], g["bc_code"], g["bc_value"], E=meta["E"], nu=meta["nu"],
                           rho=meta["rho"], c_dr=meta["c_dr"], c_cr=meta["c_cr"], factor=meta["factor"],
                           cvisl=meta["cvisl"], cvisq=meta["cvisq"], total_time=meta["total_time"],
                           yield0=meta.get("yield", 0.0), hardening=meta.get("hardening", 0.0),
                           gravity=None if meta.get("gravity") is None else (meta["gravity"][0], meta["gravity"][1]),
                           amplitude=meta.get("amplitude"), setup=setup)


def run_len(g):
    meta = g["meta"]
    if meta["mode"] == "full":
        return 10 ** 6, meta["step_end"]
    return meta["cycles"], float("inf")


# the two-step deck of the drop-in tests: step periods
STEP1, STEP2 = 1.2e-3, 0.9e-3


def write_two_step_deck(d):
    p = W.cantilever(8, 2, 2, 0.8, 0.2, 0.2, vz=1.0)
    tip = M.face_nodes(p.mesh, 0, "max")
    p.mesh.node_sets["Set-3"] = tip
    deck = "model.inp"
    path = os.path.join(d, deck)
    M.write_deck(path, p.mesh, p.material, period=STEP1, fixed_sets=p.fixed_sets,
                 initial_velocity=p.initial_velocity, bulk_viscosity=(p.controls.cvisl, p.controls.cvisq),
                 gravity=(2.0e3, (0.0, 0.0, -1.0)), amplitude=[(0.0, 0.2), (6.0e-4, 1.0), (2.0e-3, 0.5)])
    with open(path, "a") as f:
        f.write("*Step, name=Step-2, nlgeom=YES\n*Dynamic, Explicit\n")
        f.write(f", {STEP2!r}\n")
        f.write("*Boundary, type=VELOCITY\nSet-3, 3, 3, -0.5\n")
        f.write("*End Step\n")
    M.write_project(d, deck, p.controls)
    return deck
