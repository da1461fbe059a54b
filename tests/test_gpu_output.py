"""Output snapshots (ensc_snapshot_begin / ensc_snapshot_wait) and stepping
that continues while the host handles them (ensc_step_until_async).

Bars:
  * the snapshot's x, u, v, sigma and reactions equal ensc_download's (and
    ensc_download_reactions') bit for bit;
  * its acceleration -- solution_a of the last cycle, which output_results
    writes (exDyna3D.cpp:231) -- equals the CPU restatement's assembled
    force, gravity, acceleration conditions and inverse mass of the same
    cycle bit for bit in FP64, and agrees within 2e-3 of the largest
    component in mixed precision (FP32 forces after 200 cycles);
  * a snapshot taken at an output pause, copied while the device already
    steps on to the next pause, holds the state of the pause (bit-identical
    to a run that stopped there), and the run that continued equals one that
    never paused.
"""
import math

import numpy as np
import pytest

from _common import load_golden, material_controls, oracle_for
from enscdynamics_b200 import capi
from enscdynamics_b200 import workloads as W

pytestmark = pytest.mark.gpu


def oracle_acceleration(o, g):
    """compute_a of the oracle's last cycle: force (+ gravity), the
    acceleration conditions, times the inverse mass, in the restatement's
    order."""
    a = o.force.copy()
    grav = g["meta"].get("gravity")
    if grav is not None:
        d = np.tile(np.asarray(grav[1], dtype=np.float64), len(a) // 3)
        a = a + 1.0 * grav[0] * d / o.inv_mass
    code = g["bc_code"]
    a[(code & 2) != 0] = 0.0
    a[((code & 1) != 0) & (a != 0.0)] = 0.0
    return a * o.inv_mass


@pytest.mark.parametrize("name", ["cantilever_20x4x4", "gravity_6x2x2", "slot_clash_2x2x1",
                                  "single_element_velbc"])
def test_snapshot_fields_and_acceleration_fp64(name):
    g = load_golden(name)
    mat, ctl = material_controls(g["meta"])
    n = min(300, g["meta"]["cycles"])
    o = oracle_for(g)
    o.run(n)
    with capi.Stepper(g["x0"], g["conn"], g["v0"], material=mat, controls=ctl) as s:
        s.set_bcs(g["bc_code"], g["bc_value"])
        rep = s.step(n)
        s.snapshot_begin()
        sn = s.snapshot_wait()
        st = s.download()
        rf = s.reactions()
    for k in ("x", "u", "v", "sigma"):
        assert np.array_equal(sn[k], st[k]), k
    assert np.array_equal(sn["rf"], rf)
    assert sn["time"] == rep["time"] and sn["total_cycles"] == rep["total_cycles"] and sn["status"] == 0
    assert np.array_equal(sn["a"].reshape(-1), oracle_acceleration(o, g))


@pytest.mark.parametrize("assembly", [capi.ASSEMBLY_SLOT, capi.ASSEMBLY_PATCH])
def test_snapshot_acceleration_mixed(assembly):
    g = load_golden("gravity_6x2x2")
    mat, ctl = material_controls(g["meta"])
    o = oracle_for(g)
    o.run(200)
    with capi.Stepper(g["x0"], g["conn"], g["v0"], material=mat, controls=ctl, precision=capi.MIXED,
                      assembly=assembly) as s:
        s.set_bcs(g["bc_code"], g["bc_value"])
        s.step(200)
        s.snapshot_begin()
        sn = s.snapshot_wait()
    # the mixed run's accelerations carry 200 cycles of FP32 force rounding
    # (measured: 3.5e-4 of the largest one)
    ref = oracle_acceleration(o, g)
    assert np.abs(sn["a"].reshape(-1) - ref).max() <= 2e-3 * np.abs(ref).max()


def test_snapshot_needs_a_force_pass_since_a_download():
    g = load_golden("cantilever_20x4x4")
    mat, ctl = material_controls(g["meta"])
    with capi.Stepper(g["x0"], g["conn"], g["v0"], material=mat, controls=ctl) as s:
        s.set_bcs(g["bc_code"], g["bc_value"])
        s.step(10)
        s.download()
        with pytest.raises(capi.EnscError, match="ENSC_ERR_ARG"):
            s.snapshot_begin()
        s.step(1)
        s.snapshot_begin()
        s.snapshot_wait()


def test_snapshot_overlaps_the_next_cycles():
    """The drop-in's output pattern: pause at an output time, begin the
    snapshot, enqueue the cycles to the next output time, then take the
    snapshot while they run."""
    p = W.block(32, 16, 8, 0.125, 0.0625, 0.03125)
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        r = s.step(200)
        t1 = r["time"] + 40 * r["dt_i"]
        t2 = t1 + 100 * r["dt_i"]
        r1 = s.step_until(10 ** 6, math.inf, t1)
        s.snapshot_begin()
        s.step_until_async(400, math.inf, t2)
        sn = s.snapshot_wait()
        r2 = s.sync()
        end = s.download()
    assert r2["time"] >= t2 and r2["cycles"] > 0
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        s.step(200)
        q1 = s.step_until(10 ** 6, math.inf, t1)
        at1 = s.download()
    assert q1["time"] == r1["time"] == sn["time"]
    for k in ("x", "u", "v", "sigma"):
        assert np.array_equal(sn[k], at1[k]), k
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        q = s.step(200 + r1["cycles"] + r2["cycles"])
        straight = s.download()
    assert q["time"] == r2["time"]
    for k in ("x", "u", "v", "sigma"):
        assert np.array_equal(end[k], straight[k]), k
