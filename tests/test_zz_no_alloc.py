"""ensc_step_noalloc: the stepper entry point for callers that may not call
cudaMalloc -- plug-ins inside a host application that owns and budgets all
device memory, solver loops whose device memory is fixed at start-up.  The
caller hands over device arrays it already owns; the stepper's scratch lives
in a fixed device array inside the library.

Each GPU case runs the same model through the regular entry points
(ensc_create / ensc_step, which allocate) and through ensc_step_noalloc on
caller-owned arrays, two calls in a row, and requires bit-identical state
after each call -- the tolerance the FP64 parity tests use against the CPU
restatement.  The cases cover the elastic cantilever, a J2 cantilever that
yields under gravity with an amplitude, a block at the element limit, a
caller-created stream, and a call with an unbounded cycle budget that must
return at its step end.  This file is collected last on purpose.
"""
import ctypes as C
import math

import numpy as np
import pytest

from enscdynamics_b200 import capi
from enscdynamics_b200 import mesh as M
from enscdynamics_b200 import workloads as W

CYCLES = 250
INT64_MAX = 2 ** 63 - 1


def _host_model(p):
    """SoA host arrays of the model in ensc_device_model's layout, with the
    element constants of the CPU restatement (also handed to the allocating
    path, so both start from the same bits)."""
    import pyoracle
    m, c = p.material, p.controls
    o = pyoracle.Oracle(p.mesh.x0, p.mesh.conn, p.v0, p.bc_code, p.bc_value, E=m.E, nu=m.nu, rho=m.rho,
                        c_dr=c.c_dr, c_cr=c.c_cr, factor=c.factor, cvisl=c.cvisl, cvisq=c.cvisq,
                        total_time=c.total_time, yield0=m.yield_stress, hardening=m.hardening)
    ne, nn = p.mesh.n_elements, p.mesh.n_nodes
    code = p.bc_code.reshape(nn, 3).astype(np.uint8)
    bc = (code[:, 0] | (code[:, 1] << 2) | (code[:, 2] << 4)).astype(np.uint8)
    v0 = p.v0.copy()  # raw initial velocity; the entry point applies the BCs after the init pass
    arrays = {
        "conn": np.ascontiguousarray(p.mesh.conn.T), "bt": np.ascontiguousarray(o.bt.reshape(ne, 24).T),
        "vol0": o.vol0.copy(), "cbrt_v0": o.cbrt_v0.copy(), "cbrt_v0sq": o.cbrt_v0sq.copy(),
        "inv_mass": o.inv_mass.reshape(nn, 3)[:, 0].copy(), "bc": bc,
        "bc_value": np.ascontiguousarray(p.bc_value.reshape(nn, 3).T),
        "node_elem": capi.noalloc_node_elem(p.mesh.conn, nn),
        "x": np.ascontiguousarray(p.mesh.x0.T), "u": np.zeros((3, nn)), "v": np.ascontiguousarray(v0.T),
        "sigma": np.zeros((6, ne)), "qia": np.zeros((12, ne)), "eps_p": np.zeros(ne), "rf": np.zeros((3, nn)),
    }
    amp = p.controls.gravity_amplitude
    if amp:
        arrays["gravity_amp"] = np.ascontiguousarray(amp, dtype=np.float64).reshape(-1)
    return o, arrays


def _params(p, stream=None):
    pr = capi.Params()
    c = p.controls
    pr.c_dr, pr.c_cr, pr.factor_timestep, pr.cvisl, pr.cvisq, pr.total_time = (
        c.c_dr, c.c_cr, c.factor, c.cvisl, c.cvisq, c.total_time)
    if c.gravity is not None:
        pr.gravity_on = 1
        pr.gravity_value = c.gravity[0]
        for i in range(3):
            pr.gravity_dir[i] = c.gravity[1][i]
    pr.precision = capi.FP64
    pr.device = 0
    pr.stream = stream
    return pr


def _material(p):
    m = p.material
    return capi.MaterialDesc(m.E, m.nu, m.rho, m.yield_stress, m.hardening)


def _cantilever():
    return W.cantilever()


def _j2_gravity_amplitude():
    """A cantilever that yields (40 m/s, 150 MPa) under gravity scaled by an
    amplitude whose segments the runs cross."""
    p = W.cantilever(8, 2, 2, 0.8, 0.2, 0.2, vz=40.0, yield_stress=150e6, tangent=2e9)
    p.controls = M.Controls(total_time=1.0, gravity=(9.81e3, (0.0, 0.3, -1.0)),
                            gravity_amplitude=[(0.0, 0.0), (1.0e-3, 1.0), (2.5e-3, 0.4), (1.0e-2, 0.9)],
                            **W.DEFAULT_CONTROLS)
    return p


def _block_at_limit():
    """The block workload's element size and velocity field at the element
    limit (32x32x32 = 32,768 elements), J2, with gravity."""
    p = W.block(32, 32, 32, 0.125, 0.125, 0.125)
    assert p.mesh.n_elements == capi.NOALLOC_MAX_ELEMENTS and p.mesh.n_nodes <= capi.NOALLOC_MAX_NODES
    p.controls = M.Controls(total_time=1.0, gravity=(9.81, (0.0, 0.0, -1.0)),
                            **dict(W.DEFAULT_CONTROLS, c_cr=0.05))
    return p


CASES = {"cantilever": _cantilever, "j2_gravity_amplitude": _j2_gravity_amplitude,
         "block_at_element_limit": _block_at_limit}


def _device_model(p, dev):
    ne, nn = p.mesh.n_elements, p.mesh.n_nodes
    model = capi.DeviceModel(nn, ne, *[dev[k].data_ptr() for k in (
        "conn", "bt", "vol0", "cbrt_v0", "cbrt_v0sq", "inv_mass", "bc", "bc_value", "node_elem",
        "x", "u", "v", "sigma", "qia", "eps_p", "rf")])
    if "gravity_amp" in dev:
        model.gravity_amp = dev["gravity_amp"].data_ptr()
        model.gravity_amp_n = dev["gravity_amp"].numel() // 2
    return model


def _reference_runs(p, o, calls, step_end=math.inf, cycles=CYCLES):
    """State after each call of the allocating path."""
    out = []
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls,
                      bt=o.bt, vol0=o.vol0, inv_mass=o.inv_mass) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        for _ in range(calls):
            rep = s.step(cycles, step_end)
            out.append((s.download(), rep))
    return out


def _state(dev):
    got = {k: dev[k].cpu().numpy().T for k in ("x", "u", "v", "sigma", "qia")}
    got["eps_p"] = dev["eps_p"].cpu().numpy()
    return got


def test_noalloc_rejects_oversized_mesh():
    lib = capi.load()
    p = W.cantilever()
    model = capi.DeviceModel()
    model.n_nodes = 10
    model.n_elements = capi.NOALLOC_MAX_ELEMENTS + 1
    clk = capi.NoallocClock()
    rc = lib.ensc_step_noalloc(C.byref(model), C.byref(_material(p)), C.byref(_params(p)), C.byref(clk), 1,
                               math.inf)
    assert rc == -1
    assert b"no-allocation limits" in lib.ensc_last_error(None)


def test_noalloc_node_table_rejects_slot_clashes():
    # the impact bar's butterfly mesh puts nodes in the same local slot of
    # two elements where its core meets the rings
    p = W.impact_bar(4, 2, 8)
    with pytest.raises(ValueError, match="local slot"):
        capi.noalloc_node_elem(p.mesh.conn, p.mesh.n_nodes)
    q = W.cantilever()
    t = capi.noalloc_node_elem(q.mesh.conn, q.mesh.n_nodes)
    for k in range(8):
        assert np.array_equal(t[k, q.mesh.conn[:, k]], np.arange(q.mesh.n_elements))


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_matches_allocating_entry_point_two_calls(case):
    import torch
    lib = capi.load()
    p = CASES[case]()
    o, host = _host_model(p)
    ref_states = _reference_runs(p, o, 2)
    dev = {k: torch.from_numpy(np.ascontiguousarray(a)).to("cuda") for k, a in host.items()}
    torch.cuda.synchronize()
    model = _device_model(p, dev)
    clk = capi.NoallocClock(0.0, 0.0, 0.0, 0.0, 1, 0)
    for call in range(2):
        rc = lib.ensc_step_noalloc(C.byref(model), C.byref(_material(p)), C.byref(_params(p)), C.byref(clk),
                                   CYCLES, math.inf)
        assert rc == 0, lib.ensc_last_error(None)
        assert clk.cycles == CYCLES
        ref, rep = ref_states[call]
        got = _state(dev)
        for k in got:
            assert np.array_equal(got[k], ref[k]), (case, call, k)
        assert clk.time == rep["time"] and clk.dt_i == rep["dt_i"] and clk.dt_i_1 == rep["dt_i_1"]
    if case == "j2_gravity_amplitude":
        assert got["eps_p"].max() > 0.0  # the case does yield


@pytest.mark.gpu
def test_noalloc_on_a_caller_stream_and_unbounded_budget_stops_at_step_end():
    """Two calls on a caller-created stream, each with max_cycles = INT64_MAX
    and a finite step end: each returns after the cycle that reaches its step
    end, with the allocating path's state and clock."""
    import torch
    lib = capi.load()
    p = _j2_gravity_amplitude()
    o, host = _host_model(p)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        dev = {k: torch.from_numpy(np.ascontiguousarray(a)).to("cuda") for k, a in host.items()}
    stream.synchronize()
    model = _device_model(p, dev)
    clk = capi.NoallocClock(0.0, 0.0, 0.0, 0.0, 1, 0)
    ends = (1.5e-3, 3.2e-3)
    refs = []
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls,
                      bt=o.bt, vol0=o.vol0, inv_mass=o.inv_mass) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        for t_end in ends:
            rep = s.step(10 ** 9, t_end)
            refs.append((s.download(), rep))
    for call, t_end in enumerate(ends):
        rc = lib.ensc_step_noalloc(C.byref(model), C.byref(_material(p)), C.byref(_params(p, stream.cuda_stream)),
                                   C.byref(clk), INT64_MAX, t_end)
        assert rc == 0, lib.ensc_last_error(None)
        ref, rep = refs[call]
        assert clk.time == t_end == rep["time"]
        assert clk.cycles == rep["cycles"] and 0 < clk.cycles < 10 ** 6
        got = _state(dev)
        for k in got:
            assert np.array_equal(got[k], ref[k]), (call, k)
