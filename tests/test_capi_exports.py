"""The C-ABI library loads on a machine without a GPU, exports every entry
point include/ensc_gpu.h declares, and rejects bad input on the host side
without touching a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from enscdynamics_b200 import capi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "ensc_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ensc_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(capi.LIB_PATH):
        build.build()
    return capi.load()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "ensc_create" in names and "ensc_step" in names and "ensc_destroy" in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    bound = {n for n, _, _ in capi.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_abi_version(lib):
    assert lib.ensc_abi_version() == 2


def _desc(nn, ne, conn, x0):
    return capi.MeshDesc(nn, ne, conn.ctypes.data_as(C.POINTER(C.c_uint32)),
                         x0.ctypes.data_as(C.POINTER(C.c_double)), None, None, None, None)


def test_create_rejects_empty_mesh(lib):
    conn = np.zeros((0, 8), dtype=np.uint32)
    x0 = np.zeros((0, 3))
    h = C.c_void_p()
    mat = capi.MaterialDesc(1e9, 0.3, 1000.0, 0.0, 0.0)
    p = capi.Params()
    p.factor_timestep = 0.9
    rc = lib.ensc_create(C.byref(_desc(0, 0, conn, x0)), C.byref(mat), C.byref(p), C.byref(h))
    assert rc == -1 and not h.value
    assert b"empty" in lib.ensc_last_error(None)


def test_create_rejects_out_of_range_connectivity(lib):
    conn = np.array([[0, 1, 2, 3, 4, 5, 6, 99]], dtype=np.uint32)
    x0 = np.zeros((8, 3))
    h = C.c_void_p()
    mat = capi.MaterialDesc(1e9, 0.3, 1000.0, 0.0, 0.0)
    p = capi.Params()
    p.factor_timestep = 0.9
    rc = lib.ensc_create(C.byref(_desc(8, 1, conn, x0)), C.byref(mat), C.byref(p), C.byref(h))
    assert rc == -1 and b"out of range" in lib.ensc_last_error(None)


def test_create_rejects_bad_material(lib):
    conn = np.arange(8, dtype=np.uint32).reshape(1, 8)
    x0 = np.zeros((8, 3))
    h = C.c_void_p()
    mat = capi.MaterialDesc(1e9, 0.5, 1000.0, 0.0, 0.0)
    p = capi.Params()
    p.factor_timestep = 0.9
    assert lib.ensc_create(C.byref(_desc(8, 1, conn, x0)), C.byref(mat), C.byref(p), C.byref(h)) == -1


def test_null_handle_calls_are_errors(lib):
    assert lib.ensc_step(None, 1, 1.0, None) == -1
    assert lib.ensc_set_bcs(None, None, None) == -1
    assert lib.ensc_device_bytes(None) == 0
    lib.ensc_destroy(None)


def test_stepper_fails_loudly_without_library(tmp_path):
    with pytest.raises(RuntimeError):
        capi.load.__wrapped__(str(tmp_path / "missing.so")) if hasattr(capi.load, "__wrapped__") else \
            _load_missing(str(tmp_path / "missing.so"))


def _load_missing(path):
    saved = capi._lib
    capi._lib = None
    try:
        capi.load(path)
    finally:
        capi._lib = saved


def test_batch_prepare_runs_on_the_host_only(lib):
    """ensc_batch_prepare makes no CUDA call: it works here, without a GPU,
    sizes the instance's device block and reports bad input through
    ensc_last_error(NULL)."""
    from enscdynamics_b200 import workloads as W
    p = W.block(6, 4, 3, 0.6, 0.4, 0.3)
    sizes = {}
    for prec in (capi.FP64, capi.MIXED):
        pr = capi.Prepared(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls, precision=prec)
        sizes[prec] = pr.device_bytes
        pr.close()
    assert sizes[capi.FP64] > sizes[capi.MIXED] > 0
    with pytest.raises(capi.EnscError, match="out of range"):
        bad = p.mesh.conn.copy()
        bad[0, 7] = p.mesh.n_nodes
        capi.Prepared(p.mesh.x0, bad, p.v0, material=p.material, controls=p.controls)
    with pytest.raises(capi.EnscError, match="precision"):
        capi.Prepared(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls, precision=5)
