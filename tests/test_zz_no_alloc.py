"""ensc_step_noalloc: the stepper entry point for callers that cannot call
cudaMalloc (code running inside a stream capture it does not own, plug-ins
whose host application owns all device memory, loops with a budget fixed at
start-up).  The caller hands over device arrays it already owns; the
stepper's scratch lives in a fixed device array inside the library.

The GPU test runs the same model through the regular entry points
(ensc_create / ensc_step, which allocate) and through ensc_step_noalloc on
caller-owned arrays, two calls in a row, and requires bit-identical state
after each call -- the tolerance the FP64 parity tests use against the CPU
restatement.  This file is collected last on purpose.
"""
import ctypes as C
import math

import numpy as np
import pytest

from enscdynamics_b200 import capi
from enscdynamics_b200 import workloads as W

CYCLES = 250


def _host_model(p):
    """SoA host arrays of the model in ensc_device_model's layout."""
    import pyoracle
    m, c = p.material, p.controls
    o = pyoracle.Oracle(p.mesh.x0, p.mesh.conn, p.v0, p.bc_code, p.bc_value, E=m.E, nu=m.nu, rho=m.rho,
                        c_dr=c.c_dr, c_cr=c.c_cr, factor=c.factor, cvisl=c.cvisl, cvisq=c.cvisq,
                        total_time=c.total_time)
    ne, nn = p.mesh.n_elements, p.mesh.n_nodes
    node_elem = np.full((8, nn), 0xFFFFFFFF, dtype=np.uint32)
    for k in range(8):
        node_elem[k, p.mesh.conn[:, k]] = np.arange(ne, dtype=np.uint32)
    code = p.bc_code.reshape(nn, 3).astype(np.uint8)
    bc = (code[:, 0] | (code[:, 1] << 2) | (code[:, 2] << 4)).astype(np.uint8)
    v0 = p.v0.copy()  # raw initial velocity; the entry point applies the BCs after the init pass
    arrays = {
        "conn": np.ascontiguousarray(p.mesh.conn.T), "bt": np.ascontiguousarray(o.bt.reshape(ne, 24).T),
        "vol0": o.vol0.copy(), "cbrt_v0": o.cbrt_v0.copy(), "cbrt_v0sq": o.cbrt_v0sq.copy(),
        "inv_mass": o.inv_mass.reshape(nn, 3)[:, 0].copy(), "bc": bc,
        "bc_value": np.ascontiguousarray(p.bc_value.reshape(nn, 3).T), "node_elem": node_elem,
        "x": np.ascontiguousarray(p.mesh.x0.T), "u": np.zeros((3, nn)), "v": np.ascontiguousarray(v0.T),
        "sigma": np.zeros((6, ne)), "qia": np.zeros((12, ne)), "eps_p": np.zeros(ne), "rf": np.zeros((3, nn)),
    }
    return o, arrays


def _params(p):
    pr = capi.Params()
    c = p.controls
    pr.c_dr, pr.c_cr, pr.factor_timestep, pr.cvisl, pr.cvisq, pr.total_time = (
        c.c_dr, c.c_cr, c.factor, c.cvisl, c.cvisq, c.total_time)
    pr.precision = capi.FP64
    pr.device = 0
    pr.stream = None
    return pr


def _material(p):
    m = p.material
    return capi.MaterialDesc(m.E, m.nu, m.rho, m.yield_stress, m.hardening)


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


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_two_calls():
    import torch
    lib = capi.load()
    p = W.cantilever()
    o, host = _host_model(p)
    ne, nn = p.mesh.n_elements, p.mesh.n_nodes
    # regular path (allocates), fed the same element constants
    ref_states = []
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls,
                      bt=o.bt, vol0=o.vol0, inv_mass=o.inv_mass) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        for _ in range(2):
            rep = s.step(CYCLES)
            ref_states.append((s.download(), rep))
    # no-allocation path on caller-owned device arrays
    dev = {k: torch.from_numpy(np.ascontiguousarray(a)).to("cuda") for k, a in host.items()}
    torch.cuda.synchronize()
    model = capi.DeviceModel(nn, ne, *[dev[k].data_ptr() for k in (
        "conn", "bt", "vol0", "cbrt_v0", "cbrt_v0sq", "inv_mass", "bc", "bc_value", "node_elem",
        "x", "u", "v", "sigma", "qia", "eps_p", "rf")])
    clk = capi.NoallocClock(0.0, 0.0, 0.0, 0.0, 1, 0)
    for call in range(2):
        rc = lib.ensc_step_noalloc(C.byref(model), C.byref(_material(p)), C.byref(_params(p)), C.byref(clk),
                                   CYCLES, math.inf)
        assert rc == 0, lib.ensc_last_error(None)
        assert clk.cycles == CYCLES
        ref, rep = ref_states[call]
        got = {k: dev[k].cpu().numpy().T for k in ("x", "u", "v", "sigma", "qia")}
        for k in got:
            assert np.array_equal(got[k], ref[k]), (call, k)
        assert clk.time == rep["time"] and clk.dt_i == rep["dt_i"] and clk.dt_i_1 == rep["dt_i_1"]
