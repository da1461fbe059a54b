"""Parity of the sm_100a FP64 stepper (through the C ABI) with the oracle and
with the reference's golden outputs.

Bars:
  * against the CPU restatement (oracle): bit-for-bit (the FP64 kernels
    evaluate the same expressions in the same order without FMA);
  * against the reference CPU stepper's outputs: 1e-9 relative to each
    field's largest magnitude (REL_TOL_REFERENCE).
"""
import math

import numpy as np
import pytest

from _common import REL_TOL_REFERENCE, golden_names, load_golden, material_controls, oracle_for, rel, run_len, sampled
from enscdynamics_b200 import capi
from enscdynamics_b200 import mesh as M
from enscdynamics_b200 import workloads as W

pytestmark = pytest.mark.gpu


def stepper_for(g, setup_from_reference=False, **kw):
    mat, ctl = material_controls(g["meta"])
    extra = {}
    if setup_from_reference:
        extra = dict(bt=g["bt"], vol0=g["vol0"], inv_mass=g["inv_mass"])
    s = capi.Stepper(g["x0"], g["conn"], g["v0"], material=mat, controls=ctl, **extra, **kw)
    s.set_bcs(g["bc_code"], g["bc_value"])
    return s


@pytest.mark.parametrize("name", golden_names())
def test_fp64_matches_oracle_bitwise_and_reference(name):
    g = load_golden(name)
    n, end = run_len(g)
    o = oracle_for(g)
    o.run(n, end)
    with stepper_for(g) as s:
        rep = s.step(n, end)
        st = s.download()
        assert rep["cycles"] == g["meta"]["cycles"]
        assert rep["status"] == 0
        # bit-for-bit against the restatement
        assert np.array_equal(st["u"].reshape(-1), o.u)
        assert np.array_equal(st["v"].reshape(-1), o.v)
        assert np.array_equal(st["x"].reshape(-1), o.x)
        assert np.array_equal(st["sigma"].reshape(-1), o.sigma)
        assert np.array_equal(st["qia"].reshape(-1), o.qia)
        assert rep["time"] == o.time and rep["dt_i"] == o.dt[0] and rep["dt_i_1"] == o.dt[1]
        # against the reference's own outputs
        for k in ("u", "v", "x", "sigma"):
            err = rel(sampled(g, k, st[k]), g[k])
            assert err < REL_TOL_REFERENCE, (k, err)
        t, dti, _ = g["clock"]
        assert abs(rep["time"] - t) <= 1e-12 * t


@pytest.mark.parametrize("name", ["cantilever_20x4x4", "slot_clash_2x2x1"])
def test_fp64_with_reference_setup_constants(name):
    """Drop-in mode: the caller passes the reference's own B0^T, V0 and
    inverse mass (as exDyna3D_GPU does after init())."""
    g = load_golden(name)
    n, end = run_len(g)
    o = oracle_for(g, setup_from_reference=True)
    o.run(n, end)
    with stepper_for(g, setup_from_reference=True) as s:
        s.step(n, end)
        st = s.download()
    assert np.array_equal(st["u"].reshape(-1), o.u)
    assert np.array_equal(st["sigma"].reshape(-1), o.sigma)
    assert rel(st["u"], g["u"]) < REL_TOL_REFERENCE


def test_reactions_match_reference():
    g = load_golden("cantilever_20x4x4")
    n, end = run_len(g)
    with stepper_for(g) as s:
        s.step(n, end)
        rf = s.reactions()
    assert rel(rf, g["rf"]) < 1e-9


def test_j2_plastic_matches_oracle_bitwise():
    p = W.cantilever(8, 2, 2, 0.8, 0.2, 0.2, vz=40.0, yield_stress=150e6, tangent=2e9)
    mat, ctl = p.material, p.controls
    import pyoracle
    o = pyoracle.Oracle(p.mesh.x0, p.mesh.conn, p.v0, p.bc_code, p.bc_value, E=mat.E, nu=mat.nu, rho=mat.rho,
                        c_dr=ctl.c_dr, c_cr=ctl.c_cr, factor=ctl.factor, total_time=ctl.total_time,
                        yield0=mat.yield_stress, hardening=mat.hardening)
    o.run(800)
    assert o.eps_p.max() > 0.0  # the case does yield
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=mat, controls=ctl) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        s.step(800)
        st = s.download()
    assert np.array_equal(st["eps_p"], o.eps_p)
    assert np.array_equal(st["sigma"].reshape(-1), o.sigma)
    assert np.array_equal(st["u"].reshape(-1), o.u)


def test_impact_bar_j2_matches_oracle_bitwise():
    """The plastic impact bar on a reduced mesh (butterfly-meshed cylinder,
    6x6 core, 3 rings, 24 layers: 2592 elements, J2, -190 m/s onto a face
    fixed in z) run to its end time, 80 us (1618 cycles).  Its core and rings
    share local slots at nodes, so the forces go through the element-major
    rows and the node lists.  FP64 GPU equals the oracle bit for bit, and the
    bar yields (plastic strain above 1 at the impact face)."""
    import pyoracle
    p = W.impact_bar(6, 3, 24)
    assert M.check_slot_clashes(p.mesh.conn, p.mesh.n_nodes) > 0
    mat, ctl = p.material, p.controls
    o = pyoracle.Oracle(p.mesh.x0, p.mesh.conn, p.v0, p.bc_code, p.bc_value, E=mat.E, nu=mat.nu, rho=mat.rho,
                        c_dr=ctl.c_dr, c_cr=ctl.c_cr, factor=ctl.factor, cvisl=ctl.cvisl, cvisq=ctl.cvisq,
                        total_time=ctl.total_time, yield0=mat.yield_stress, hardening=mat.hardening)
    n = o.run(10 ** 6, p.end_time)
    assert o.time == p.end_time and o.eps_p.max() > 1.0
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=mat, controls=ctl) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        rep = s.step(10 ** 6, p.end_time)
        st = s.download()
    assert rep["cycles"] == n and rep["status"] == 0 and rep["time"] == o.time
    assert np.array_equal(st["eps_p"], o.eps_p)
    assert np.array_equal(st["sigma"].reshape(-1), o.sigma)
    assert np.array_equal(st["u"].reshape(-1), o.u)
    assert np.array_equal(st["v"].reshape(-1), o.v)


def test_energy_sums_match_oracle():
    g = load_golden("gravity_6x2x2")
    n, end = run_len(g)
    o = oracle_for(g)
    o.run(n, end)
    with stepper_for(g) as s:
        s.step(n, end)
        e = s.energy()
    oe = o.energy
    assert abs(e["kinetic0"] - o.kinetic0) <= 1e-12 * o.kinetic0
    for i, k in enumerate(("kinetic", "internal", "hourglass", "viscous", "external")):
        assert abs(e[k] - oe[i]) <= 1e-10 * max(abs(oe[i]), 1e-30), k


def test_chunked_steps_equal_one_run_and_restart():
    """Stepping in pieces, and restarting from a downloaded checkpoint into a
    fresh instance, reproduce a single uninterrupted run bit-for-bit."""
    g = load_golden("cantilever_20x4x4")
    with stepper_for(g) as a:
        a.step(700)
        ref = a.download()
        clock = a.step(0)
    with stepper_for(g) as b:
        b.step(250)
        mid = b.download()
        c1 = b.step(0)
        b.step(450)
        got = b.download()
    for k in ("u", "v", "x", "sigma", "qia"):
        assert np.array_equal(got[k], ref[k]), k
    with stepper_for(g) as c:
        c.upload_state(mid, c1["time"], c1["dt_i"], c1["dt_i_1"], c1["dt_stable_min"])
        c.step(450)
        got2 = c.download()
    for k in ("u", "v", "x", "sigma", "qia"):
        assert np.array_equal(got2[k], ref[k]), k


def test_determinism_repeat():
    p = W.block(24, 12, 8, 0.24, 0.12, 0.08, plastic=True)
    outs = []
    for _ in range(2):
        with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls) as s:
            s.set_bcs(p.bc_code, p.bc_value)
            s.step(300)
            outs.append(s.download())
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_block_matches_oracle_bitwise():
    p = W.block(24, 12, 8, 0.24, 0.12, 0.08, plastic=True)
    mat, ctl = p.material, p.controls
    import pyoracle
    o = pyoracle.Oracle(p.mesh.x0, p.mesh.conn, p.v0, p.bc_code, p.bc_value, E=mat.E, nu=mat.nu, rho=mat.rho,
                        c_dr=ctl.c_dr, c_cr=ctl.c_cr, factor=ctl.factor, total_time=ctl.total_time,
                        yield0=mat.yield_stress, hardening=mat.hardening)
    o.run(150)
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=mat, controls=ctl) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        s.step(150)
        st = s.download()
    assert np.array_equal(st["u"].reshape(-1), o.u)
    assert np.array_equal(st["sigma"].reshape(-1), o.sigma)


def test_errors_are_reported_not_fatal():
    m = M.box_mesh(2, 1, 1, 0.2, 0.1, 0.1)
    mat = M.Material(200e9, 0.3, 7800.0)
    ctl = M.Controls(total_time=1.0)
    with pytest.raises(capi.EnscError):
        capi.Stepper(m.x0, m.conn, None, material=mat, controls=ctl, device=99)
    with capi.Stepper(m.x0, m.conn, None, material=mat, controls=ctl) as s:
        with pytest.raises(capi.EnscError):
            s.step(-1)
        rep = s.step(10)
        assert rep["cycles"] == 10 and rep["status"] == 0


def test_pause_at_output_times_keeps_the_trajectory():
    """ensc_step_until stops after the cycle in which time reaches the pause
    time without shortening dt, so a run paused for output ends bit-identical
    to an uninterrupted one."""
    g = load_golden("cantilever_20x4x4")
    n = g["meta"]["cycles"]
    with stepper_for(g) as s:
        full = s.step(n)
        ref = s.download()
    t_end = full["time"]
    done = 0
    with stepper_for(g) as s:
        for frac in (0.1, 0.37, 0.8):
            pause = frac * t_end
            r = s.step_until(n - done, math.inf, pause)
            done += r["cycles"]
            assert r["time"] >= pause and r["time"] - r["dt_i_1"] < pause, (r, pause)
        r = s.step(n - done)
        assert done + r["cycles"] == n
        st = s.download()
    for k in ("x", "u", "v", "sigma", "qia"):
        assert np.array_equal(st[k], ref[k]), k
    assert r["time"] == full["time"]
