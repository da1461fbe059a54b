"""Generates the golden fixtures in this directory by running the reference
CPU stepper (compiled from the reference sources into oracle/_ref by
oracle/Makefile) on decks written by enscdynamics_b200.mesh.

Run in a container that has the reference checkout (REF, default: a
checkout named ``reference`` beside this repository):

    make -C oracle && python tests/golden/make_golden.py

Each fixture stores the model in array form (x0, conn, v0, BC arrays,
material, controls) and the reference's state after the run (u, v, x, sigma,
QIA, time, dt_i, dt_i_1, reactions).  Fixtures are small (<= a few thousand
elements) so the CPU restatement and the GPU stepper can be checked against
them anywhere, without the reference.

Two kinds of case:
  * decks written by enscdynamics_b200.mesh for the model in array form
    (``cases``);
  * the reference's own example decks (REF/inp, ``ref_deck_cases``): the
    model is taken from the reference's state after init() and the first
    step's setup, run for a bounded number of cycles inside that first step.
"""
from __future__ import annotations

import itertools
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from enscdynamics_b200 import mesh as M  # noqa: E402
from enscdynamics_b200 import workloads as W  # noqa: E402
import pyoracle  # noqa: E402


def cases():
    out = []
    # 1. the reference-runnable cantilever, 2000 cycles
    p = W.cantilever()
    out.append(("cantilever_20x4x4", p, "cycles", 2000))
    # 2. single element: bottom fixed, prescribed velocity on the top face
    m = M.box_mesh(1, 1, 1, 0.1, 0.1, 0.1)
    bot = M.face_nodes(m, 2, "min")
    top = M.face_nodes(m, 2, "max")
    m.node_sets = {"Set-1": bot, "Set-2": top}
    code, val = M.bc_arrays(m.n_nodes, fixed=[(bot, 0, 2)], velocity=[(top, 2, 2, -2.0)])
    p = W.Problem("single_element_velbc", m, np.zeros((m.n_nodes, 3)), code, val,
                  M.Material(200e9, 0.3, 7800.0), M.Controls(total_time=1.0, **W.DEFAULT_CONTROLS), 400,
                  fixed_sets=[("Set-1", "ENCASTRE")])
    p.velocity_sets = [("Set-2", 3, 3, -2.0)]
    out.append(("single_element_velbc", p, "cycles", 400))
    # 3. gravity-loaded cantilever with an initial velocity field
    p = W.cantilever(6, 2, 2, 0.6, 0.2, 0.2, vz=0.5)
    p.controls = M.Controls(total_time=1.0, gravity=(9.81, (0.0, 0.0, -1.0)), **W.DEFAULT_CONTROLS)
    out.append(("gravity_6x2x2", p, "cycles", 600))
    # 4. run to end time through exDyna3D::run() itself (last-step and
    #    total-time clamps fire in the final cycles)
    p = W.cantilever(4, 2, 2, 0.4, 0.2, 0.2, vz=3.0)
    p.controls = M.Controls(total_time=3.3e-4, **W.DEFAULT_CONTROLS)
    p.end_time = 3.3e-4
    out.append(("run_to_time_4x2x2", p, "full", None))
    # 5. slot clashes: elements with rotated local numbering so a node sits
    #    in the same local slot of two elements
    out.append(("slot_clash_2x2x1", clash_problem(), "cycles", 300))
    # 6. gravity under an amplitude: a ramp over the first segment, a cycle
    #    that crosses its end (the averaging branch of deal_amp) and factor 1
    #    after it, as deal_amp gives
    p = W.cantilever(6, 2, 2, 0.6, 0.2, 0.2, vz=0.5)
    p.controls = M.Controls(total_time=1.0, gravity=(9.81e3, (0.0, 0.0, -1.0)),
                            gravity_amplitude=[(0.0, 0.0), (3.0e-3, 1.0), (6.0e-3, 0.25), (1.0e-2, 0.8)],
                            **W.DEFAULT_CONTROLS)
    out.append(("gravity_amp_6x2x2", p, "cycles", 600))
    # 7. the impact bar's butterfly-meshed cylinder (nodes share local slots
    #    where the core meets the ring), elastic as the reference has no J2,
    #    z = 0 face fixed in z, all nodes at -190 m/s
    p = W.impact_bar(4, 2, 8, plastic=False)
    out.append(("impact_bar_4x2x8", p, "cycles", 300))
    return out


# the reference's example decks (REF/inp) and the cycles run in their first
# step (each stays inside it)
REF_DECKS = [("GenVirPa.inp", 200), ("Job-6.inp", 300), ("test_part1.inp", 300), ("test_single2.inp", 300),
             ("test_step.inp", 300), ("test_trans.inp", 300), ("test.inp", 100)]


# decks with more elements than this keep sampled results (SAMPLE_ROWS rows)
SAMPLE_ABOVE = 2000
SAMPLE_ROWS = 1000


def ref_deck_cases(ref):
    return [("refdeck_" + os.path.splitext(d)[0], os.path.join(ref, "inp", d), n) for d, n in REF_DECKS]


def _first_step(deck_path):
    """The first step's period and its gravity load (value, direction) or
    None, read from the deck text as the reference reader reads them
    (``*Dynamic, Explicit`` data line ``, period``; ``*Dload`` data line
    ``, GRAV, g, dx, dy, dz``)."""
    lines = open(deck_path).read().splitlines()
    period, grav, in_step, k = None, None, False, 0
    while k < len(lines):
        u = lines[k].strip().upper()
        if u.startswith("*STEP"):
            if in_step:
                break
            in_step = True
        elif in_step and u.startswith("*DYNAMIC"):
            period = float(lines[k + 1].split(",")[1])
        elif in_step and u.startswith("*DLOAD"):
            f = [t.strip() for t in lines[k + 1].split(",")]
            if len(f) >= 6 and f[1].upper() == "GRAV":
                grav = (float(f[2]), [float(f[3]), float(f[4]), float(f[5])])
        k += 1
    return period, grav


def make_ref_deck_fixture(name, deck_path, cycles):
    """Runs one of the reference's example decks through the harness and
    writes its fixture; returns the fixture's meta."""
    import shutil
    deck = os.path.basename(deck_path)
    period, grav = _first_step(deck_path)
    with tempfile.TemporaryDirectory() as d:
        shutil.copy(deck_path, d)
        M.write_project(d, deck, M.Controls(total_time=1.0, **W.DEFAULT_CONTROLS))
        pyoracle.run_reference(d, deck, "setup", dump=os.path.join(d, "s.bin"))
        s = pyoracle.read_dump(os.path.join(d, "s.bin"))
        info = pyoracle.run_reference(d, deck, "cycles", cycles, dump=os.path.join(d, "o.bin"))
        r = pyoracle.read_dump(os.path.join(d, "o.bin"))
    assert r["cycles"] == cycles and r["time"] <= period, (name, r["cycles"], r["time"], period)
    meta = dict(E=s["E"], nu=s["nu"], rho=s["rho"], c_dr=s["c_dr"], c_cr=s["c_cr"], factor=s["factor"],
                cvisl=s["cvisl"], cvisq=s["cvisq"], total_time=s["total_time"], gravity=grav, mode="cycles",
                cycles=int(r["cycles"]), amplitude=None, step_end=None, deck=deck)
    arrays = dict(x0=s["x"], conn=s["conn"], v0=s["u"], bc_code=s["bc_code"], bc_value=s["bc_value"],
                  clock=np.array([r["time"], r["dt_i"], r["dt_i_1"]]), meta=np.array(json.dumps(meta)))
    ne, nn = s["n_elements"], s["n_nodes"]
    if ne <= SAMPLE_ABOVE:
        arrays.update(bt=s["bt"], vol0=s["vol0"], inv_mass=s["inv_mass"], u=r["u"], v=r["v"], x=r["x"],
                      sigma=r["sigma"], qia=r["qia"], rf=r["rf"])
    else:
        # a large deck keeps the model whole but its results at seeded samples
        # of nodes and elements (out_nodes / out_elements), to stay small
        rng = np.random.default_rng(2026)
        on = np.sort(rng.choice(nn, SAMPLE_ROWS, replace=False))
        oe = np.sort(rng.choice(ne, SAMPLE_ROWS, replace=False))
        arrays.update(out_nodes=on, out_elements=oe, u=r["u"][on], v=r["v"][on], x=r["x"][on],
                      sigma=r["sigma"][oe])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print(name, info)
    return meta


def _rotations():
    """The 24 proper rotations of the reference hexahedron as node permutations."""
    xi = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                   [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]])
    perms = []
    for P in itertools.permutations(range(3)):
        for s in itertools.product((-1, 1), repeat=3):
            R = np.zeros((3, 3), dtype=int)
            for i in range(3):
                R[i, P[i]] = s[i]
            if round(np.linalg.det(R)) != 1:
                continue
            img = xi @ R.T
            perm = [int(np.nonzero((xi == img[k]).all(axis=1))[0][0]) for k in range(8)]
            perms.append(perm)
    return perms


def clash_problem():
    m = M.box_mesh(2, 2, 1, 0.2, 0.2, 0.1)
    rots = _rotations()
    rng = np.random.default_rng(7)
    base = m.conn.copy()
    for _ in range(1000):
        conn = np.stack([base[e][rots[rng.integers(len(rots))]] for e in range(base.shape[0])]).astype(np.uint32)
        if M.check_slot_clashes(conn, m.n_nodes) > 0:
            break
    m.conn = conn
    bot = M.face_nodes(m, 2, "min")
    free = np.setdiff1d(np.arange(m.n_nodes), bot)
    m.node_sets = {"Set-1": bot, "Set-2": free}
    v0 = np.zeros((m.n_nodes, 3))
    v0[free, 0] = 1.5
    code, val = M.bc_arrays(m.n_nodes, fixed=[(bot, 0, 2)])
    return W.Problem("slot_clash_2x2x1", m, v0, code, val, M.Material(70e9, 0.33, 2700.0),
                     M.Controls(total_time=1.0, **W.DEFAULT_CONTROLS), 300,
                     fixed_sets=[("Set-1", "PINNED")], initial_velocity=[("Set-2", 1, 1.5)])


# slab of the roofline block workload run through the reference: the block's
# element size (3.90625 mm cubes), material (elastic: the reference has no
# J2), controls and seeded smoothed-Gaussian velocity field, at 64x32x16
BLOCK_CASE = dict(name="block_64x32x16", dims=(64, 32, 16), lengths=(0.25, 0.125, 0.0625), seed=20241203,
                  cycles=200)


def _sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def block_problem(dims, lengths, seed):
    return W.block(*dims, *lengths, seed=seed, plastic=False)


def make_block_fixture():
    """The block workload's slab (BLOCK_CASE) through the reference stepper.
    The fixture keeps the reference's results at seeded samples of nodes and
    elements, and instead of the model arrays the parameters that rebuild
    them (workloads.block) with a SHA-256 of each rebuilt array, which the
    tests check before use."""
    c = BLOCK_CASE
    p = block_problem(c["dims"], c["lengths"], c["seed"])
    with tempfile.TemporaryDirectory() as d:
        deck = p.write_deck(d)
        pyoracle.run_reference(d, deck, "setup", dump=os.path.join(d, "s.bin"))
        s = pyoracle.read_dump(os.path.join(d, "s.bin"))
        assert np.array_equal(s["conn"], p.mesh.conn)
        assert np.array_equal(s["x"], p.mesh.x0)
        assert np.array_equal(s["bc_code"], p.bc_code)
        assert np.array_equal(s["bc_value"], p.bc_value)
        assert np.array_equal(s["u"].reshape(-1, 3), p.v0)  # the setup dump's u holds the initial velocities
        info = pyoracle.run_reference(d, deck, "cycles", c["cycles"], dump=os.path.join(d, "o.bin"))
        r = pyoracle.read_dump(os.path.join(d, "o.bin"))
    assert r["cycles"] == c["cycles"]
    ctl = p.controls
    meta = dict(E=p.material.E, nu=p.material.nu, rho=p.material.rho, c_dr=ctl.c_dr, c_cr=ctl.c_cr,
                factor=ctl.factor, cvisl=ctl.cvisl, cvisq=ctl.cvisq, total_time=ctl.total_time, gravity=None,
                mode="cycles", cycles=int(r["cycles"]), amplitude=None, step_end=None,
                regenerate=dict(workload="block", dims=list(c["dims"]), lengths=list(c["lengths"]),
                                seed=c["seed"],
                                sha256={k: _sha(a) for k, a in (("x0", p.mesh.x0), ("conn", p.mesh.conn),
                                                                 ("v0", p.v0), ("bc_code", p.bc_code),
                                                                 ("bc_value", p.bc_value))}))
    ne, nn = p.mesh.n_elements, p.mesh.n_nodes
    rng = np.random.default_rng(2026)
    on = np.sort(rng.choice(nn, SAMPLE_ROWS, replace=False))
    oe = np.sort(rng.choice(ne, SAMPLE_ROWS, replace=False))
    np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), out_nodes=on, out_elements=oe, u=r["u"][on],
                        v=r["v"][on], x=r["x"][on], sigma=r["sigma"][oe],
                        clock=np.array([r["time"], r["dt_i"], r["dt_i_1"]]), meta=np.array(json.dumps(meta)))
    print(c["name"], info)
    return meta


def write_case_deck(p, d):
    deck = "model.inp"
    per = p.end_time if p.end_time else p.controls.total_time
    M.write_deck(os.path.join(d, deck), p.mesh, p.material, period=per, fixed_sets=p.fixed_sets,
                 initial_velocity=p.initial_velocity, bulk_viscosity=(p.controls.cvisl, p.controls.cvisq),
                 gravity=p.controls.gravity, amplitude=p.controls.gravity_amplitude)
    vel = getattr(p, "velocity_sets", [])
    if vel:  # velocity conditions go inside the step: the reference does not
        # carry Initial-step velocity conditions into step 1 (exDyna3D.cpp:1859-1880)
        txt = open(os.path.join(d, deck)).read()
        block = "".join(f"*Boundary, type=VELOCITY\n{n}, {a}, {b}, {v!r}\n" for n, a, b, v in vel)
        txt = txt.replace("*End Step", block + "*End Step", 1)
        open(os.path.join(d, deck), "w").write(txt)
    M.write_project(d, deck, p.controls)
    return deck


def main(only=()):
    """Regenerates every fixture, or only the named ones (index.json keeps the others)."""
    assert pyoracle.harness_available(), "build the reference harness first: make -C oracle"
    index = {}
    ipath = os.path.join(HERE, "index.json")
    if only and os.path.exists(ipath):
        with open(ipath) as f:
            index = json.load(f)
    ref = os.environ.get("REF") or os.path.join(os.path.dirname(ROOT), "reference")
    for name, deck_path, cycles in ref_deck_cases(ref):
        if only and name not in only:
            continue
        index[name] = make_ref_deck_fixture(name, deck_path, cycles)
    if not only or BLOCK_CASE["name"] in only:
        index[BLOCK_CASE["name"]] = make_block_fixture()
    for name, p, mode, cycles in cases():
        if only and name not in only:
            continue
        with tempfile.TemporaryDirectory() as d:
            deck = write_case_deck(p, d)
            pyoracle.run_reference(d, deck, "setup", dump=os.path.join(d, "s.bin"))
            s = pyoracle.read_dump(os.path.join(d, "s.bin"))
            assert np.array_equal(s["conn"], p.mesh.conn), name
            assert np.array_equal(s["x"], p.mesh.x0), name
            assert np.array_equal(s["bc_code"], p.bc_code), name
            assert np.array_equal(s["bc_value"], p.bc_value), name
            info = pyoracle.run_reference(d, deck, mode, cycles, dump=os.path.join(d, "o.bin"))
            r = pyoracle.read_dump(os.path.join(d, "o.bin"))
        c = p.controls
        meta = dict(E=p.material.E, nu=p.material.nu, rho=p.material.rho, c_dr=c.c_dr, c_cr=c.c_cr,
                    factor=c.factor, cvisl=c.cvisl, cvisq=c.cvisq, total_time=c.total_time,
                    gravity=c.gravity, mode=mode, cycles=int(r["cycles"]),
                    amplitude=[list(t) for t in c.gravity_amplitude] if c.gravity_amplitude else None,
                    step_end=(p.end_time if mode == "full" else None))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), x0=p.mesh.x0, conn=p.mesh.conn, v0=p.v0,
                            bc_code=p.bc_code, bc_value=p.bc_value, bt=s["bt"], vol0=s["vol0"],
                            inv_mass=s["inv_mass"], u=r["u"], v=r["v"], x=r["x"], sigma=r["sigma"],
                            qia=r["qia"], rf=r["rf"],
                            clock=np.array([r["time"], r["dt_i"], r["dt_i_1"]]),
                            meta=np.array(json.dumps(meta)))
        index[name] = meta
        print(name, info)
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
