"""ctypes binding of the C ABI in include/ensc_gpu.h (libensc_b200.so).

``Stepper`` owns one solver instance on one GPU.  There is no CPU fallback:
if the library or a GPU is missing, construction raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import Dict, Optional

import numpy as np

from . import mesh as _mesh

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "libensc_b200.so")

FP64 = 0
MIXED = 1
# force assembly (ensc_params.assembly)
ASSEMBLY_AUTO = 0
ASSEMBLY_SLOT = 1
ASSEMBLY_PATCH = 2

_ERR = {-1: "ENSC_ERR_ARG", -2: "ENSC_ERR_OOM", -3: "ENSC_ERR_CUDA", -4: "ENSC_ERR_NONFINITE",
        -5: "ENSC_ERR_INVERTED", -6: "ENSC_ERR_TIMEOUT", -7: "ENSC_ERR_NODEVICE"}

_P = C.POINTER(C.c_double)


class MeshDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("n_elements", C.c_int64), ("conn", C.POINTER(C.c_uint32)),
                ("x0", _P), ("v0", _P), ("bt", _P), ("vol0", _P), ("inv_mass", _P)]


class MaterialDesc(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("rho", C.c_double),
                ("yield_stress", C.c_double), ("hardening_modulus", C.c_double)]


class Params(C.Structure):
    _fields_ = [("c_dr", C.c_double), ("c_cr", C.c_double), ("factor_timestep", C.c_double),
                ("cvisl", C.c_double), ("cvisq", C.c_double), ("total_time", C.c_double),
                ("gravity_on", C.c_int32), ("gravity_value", C.c_double), ("gravity_dir", C.c_double * 3),
                ("precision", C.c_int32), ("device", C.c_int32), ("stream", C.c_void_p),
                ("graph_chunk", C.c_int32), ("assembly", C.c_int32)]


class PatchTables(C.Structure):
    _fields_ = [("n_elements", C.c_int64), ("n_nodes", C.c_int64), ("n_patches", C.c_int64),
                ("n_partials", C.c_int64), ("stored", C.POINTER(C.c_int32)),
                ("patch_first", C.POINTER(C.c_uint32)), ("inc_first", C.POINTER(C.c_uint32)),
                ("inc", C.POINTER(C.c_uint16)), ("node_first", C.POINTER(C.c_uint32)),
                ("node_partials", C.POINTER(C.c_uint32))]


class StepReport(C.Structure):
    _fields_ = [("time", C.c_double), ("dt_i", C.c_double), ("dt_i_1", C.c_double),
                ("cycles", C.c_int64), ("total_cycles", C.c_int64), ("status", C.c_int32), ("done", C.c_int32),
                ("dt_stable_min", C.c_double)]


class EnergyReport(C.Structure):
    _fields_ = [("kinetic", C.c_double), ("internal", C.c_double), ("hourglass", C.c_double),
                ("viscous", C.c_double), ("external", C.c_double), ("kinetic0", C.c_double)]


class Snapshot(C.Structure):
    """ensc_snapshot: host pointers into the library's pinned snapshot buffer."""
    _fields_ = [("x", _P), ("u", _P), ("v", _P), ("a", _P), ("rf", _P), ("sigma", _P),
                ("time", C.c_double), ("dt_i", C.c_double), ("dt_i_1", C.c_double),
                ("total_cycles", C.c_int64), ("status", C.c_int32)]


class DeviceModel(C.Structure):
    """ensc_device_model: caller-owned device arrays for ensc_step_noalloc."""
    _fields_ = [("n_nodes", C.c_int64), ("n_elements", C.c_int64), ("conn", C.c_void_p), ("bt", C.c_void_p),
                ("vol0", C.c_void_p), ("cbrt_v0", C.c_void_p), ("cbrt_v0sq", C.c_void_p),
                ("inv_mass", C.c_void_p), ("bc", C.c_void_p), ("bc_value", C.c_void_p), ("node_elem", C.c_void_p),
                ("x", C.c_void_p), ("u", C.c_void_p), ("v", C.c_void_p), ("sigma", C.c_void_p),
                ("qia", C.c_void_p), ("eps_p", C.c_void_p), ("rf", C.c_void_p),
                ("gravity_amp", C.c_void_p), ("gravity_amp_n", C.c_int32)]


class NoallocClock(C.Structure):
    _fields_ = [("time", C.c_double), ("dt_i", C.c_double), ("dt_i_1", C.c_double),
                ("dt_stable_min", C.c_double), ("init_pass", C.c_int32), ("cycles", C.c_int64)]


NOALLOC_MAX_ELEMENTS = 32768
NOALLOC_MAX_NODES = 262144


def noalloc_node_elem(conn: np.ndarray, n_nodes: int) -> np.ndarray:
    """The ``node_elem`` table of ensc_device_model ([8][n_nodes] uint32:
    the element holding node n in local slot k, or 0xFFFFFFFF) from the
    (n_elements, 8) connectivity.  ensc_step_noalloc keeps one element per
    slot, so a mesh where a node sits in the same local slot of two elements
    cannot run there: raises ValueError naming the first such node."""
    conn = np.asarray(conn, dtype=np.int64)
    ne = conn.shape[0]
    out = np.full((8, n_nodes), 0xFFFFFFFF, dtype=np.uint32)
    for k in range(8):
        col = conn[:, k]
        counts = np.bincount(col, minlength=n_nodes)
        if counts.max(initial=0) > 1:
            node = int(np.argmax(counts > 1))
            raise ValueError(f"node {node} sits in local slot {k} of {int(counts[node])} elements: "
                             "ensc_step_noalloc needs one element per node and slot")
        out[k, col] = np.arange(ne, dtype=np.uint32)
    return out


# every symbol include/ensc_gpu.h declares: (name, restype, argtypes)
SIGNATURES = [
    ("ensc_abi_version", C.c_int, []),
    ("ensc_create", C.c_int, [C.POINTER(MeshDesc), C.POINTER(MaterialDesc), C.POINTER(Params),
                              C.POINTER(C.c_void_p)]),
    ("ensc_set_bcs", C.c_int, [C.c_void_p, C.POINTER(C.c_int8), _P]),
    ("ensc_set_gravity", C.c_int, [C.c_void_p, C.c_int32, C.c_double, _P]),
    ("ensc_set_gravity_amplitude", C.c_int, [C.c_void_p, C.c_int32, _P]),
    ("ensc_step", C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.POINTER(StepReport)]),
    ("ensc_step_until", C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_double, C.POINTER(StepReport)]),
    ("ensc_step_async", C.c_int, [C.c_void_p, C.c_int64, C.c_double]),
    ("ensc_sync", C.c_int, [C.c_void_p, C.POINTER(StepReport)]),
    ("ensc_step_until_async", C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_double]),
    ("ensc_snapshot_begin", C.c_int, [C.c_void_p]),
    ("ensc_snapshot_wait", C.c_int, [C.c_void_p, C.POINTER(Snapshot)]),
    ("ensc_download", C.c_int, [C.c_void_p, _P, _P, _P, _P, _P, _P]),
    ("ensc_upload_state", C.c_int, [C.c_void_p, _P, _P, _P, _P, _P, _P, C.c_double, C.c_double, C.c_double,
                                    C.c_double]),
    ("ensc_energy", C.c_int, [C.c_void_p, C.POINTER(EnergyReport)]),
    ("ensc_download_reactions", C.c_int, [C.c_void_p, _P]),
    ("ensc_profile", C.c_int, [C.c_void_p, C.c_int64, C.c_double, _P, C.POINTER(C.c_int64)]),
    ("ensc_device_bytes", C.c_int64, [C.c_void_p]),
    ("ensc_kernels_per_cycle", C.c_int32, [C.c_void_p]),
    ("ensc_assembly", C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("ensc_destroy", None, [C.c_void_p]),
    ("ensc_step_noalloc", C.c_int, [C.POINTER(DeviceModel), C.POINTER(MaterialDesc), C.POINTER(Params),
                                    C.POINTER(NoallocClock), C.c_int64, C.c_double]),
    ("ensc_last_error", C.c_char_p, [C.c_void_p]),
    ("ensc_batch_create", C.c_int, [C.POINTER(Params), C.c_int32, C.c_int64, C.c_int64, C.c_int64,
                                    C.POINTER(C.c_void_p)]),
    ("ensc_batch_add", C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(MaterialDesc), C.POINTER(Params),
                                 C.POINTER(C.c_int32)]),
    ("ensc_batch_prepare", C.c_int, [C.POINTER(MeshDesc), C.POINTER(MaterialDesc), C.POINTER(Params),
                                     C.POINTER(C.c_void_p)]),
    ("ensc_prepared_assembly", C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                         C.POINTER(C.c_int64)]),
    ("ensc_prepared_patch_tables", C.c_int, [C.c_void_p, C.POINTER(PatchTables)]),
    ("ensc_batch_add_prepared", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Params), C.POINTER(C.c_int32)]),
    ("ensc_prepared_bytes", C.c_int64, [C.c_void_p]),
    ("ensc_prepared_destroy", None, [C.c_void_p]),
    ("ensc_batch_set_bcs", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int8), _P]),
    ("ensc_batch_set_gravity_amplitude", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, _P]),
    ("ensc_batch_arm", C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_double]),
    ("ensc_batch_run", C.c_int, [C.c_void_p, C.c_int64]),
    ("ensc_batch_sync", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("ensc_batch_report", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(StepReport)]),
    ("ensc_batch_energy", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(EnergyReport)]),
    ("ensc_batch_download", C.c_int, [C.c_void_p, C.c_int32, _P, _P, _P, _P, _P, _P]),
    ("ensc_batch_remove", C.c_int, [C.c_void_p, C.c_int32]),
    ("ensc_batch_device_bytes", C.c_int64, [C.c_void_p]),
    ("ensc_batch_instances", C.c_int32, [C.c_void_p]),
    ("ensc_batch_tuning", C.c_int, [C.c_void_p] + [C.POINTER(C.c_int32)] * 6),
    ("ensc_batch_destroy", None, [C.c_void_p]),
    ("ensc_batch_last_error", C.c_char_p, [C.c_void_p]),
]

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads the stepper library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m enscdynamics_b200.build`")
        lib = C.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class EnscError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERR.get(code, code)}: {msg}")
        self.code = code


def _dp(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_P)


def _descriptors(x0, conn, v0, material, controls, bt=None, vol0=None, inv_mass=None):
    """Mesh, material and control descriptors (plus the arrays they point into)."""
    keep = []

    def arr(a, dt):
        if a is None:
            return None
        b = np.ascontiguousarray(a, dtype=dt)
        keep.append(b)
        return b

    conn_a = arr(conn, np.uint32)
    x0_a = arr(x0, np.float64)
    v0_a = arr(v0, np.float64)
    m = MeshDesc(int(x0.shape[0]), int(conn.shape[0]), conn_a.ctypes.data_as(C.POINTER(C.c_uint32)), _dp(x0_a),
                 _dp(v0_a), _dp(arr(bt, np.float64)), _dp(arr(vol0, np.float64)), _dp(arr(inv_mass, np.float64)))
    mt = MaterialDesc(material.E, material.nu, material.rho, material.yield_stress, material.hardening)
    p = Params()
    p.c_dr, p.c_cr, p.factor_timestep = controls.c_dr, controls.c_cr, controls.factor
    p.cvisl, p.cvisq, p.total_time = controls.cvisl, controls.cvisq, controls.total_time
    if controls.gravity is not None:
        p.gravity_on = 1
        p.gravity_value = controls.gravity[0]
        for i in range(3):
            p.gravity_dir[i] = controls.gravity[1][i]
    return keep, m, mt, p


class Stepper:
    """One GPU solver instance behind the C ABI."""

    def __init__(self, x0: np.ndarray, conn: np.ndarray, v0: Optional[np.ndarray] = None, *,
                 material: _mesh.Material, controls: _mesh.Controls, precision: int = FP64,
                 bt: Optional[np.ndarray] = None, vol0: Optional[np.ndarray] = None,
                 inv_mass: Optional[np.ndarray] = None, device: int = 0, stream: Optional[int] = None,
                 graph_chunk: int = 0, assembly: int = ASSEMBLY_AUTO):
        lib = load()
        self._lib = lib
        self.h = C.c_void_p()
        self.n_nodes = int(x0.shape[0])
        self.n_elements = int(conn.shape[0])
        self._keep, m, mt, p = _descriptors(x0, conn, v0, material, controls, bt, vol0, inv_mass)
        p.precision = precision
        p.device = device
        p.stream = stream
        p.graph_chunk = graph_chunk
        p.assembly = assembly
        rc = lib.ensc_create(C.byref(m), C.byref(mt), C.byref(p), C.byref(self.h))
        if rc != 0:
            raise EnscError(rc, lib.ensc_last_error(None).decode())
        self.precision = precision
        if controls.gravity_amplitude:
            self.set_gravity_amplitude(controls.gravity_amplitude)

    # -- helpers -------------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != 0:
            raise EnscError(rc, self._lib.ensc_last_error(self.h).decode())

    def close(self) -> None:
        if self.h:
            self._lib.ensc_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- API -----------------------------------------------------------------
    def set_bcs(self, code: Optional[np.ndarray], value: Optional[np.ndarray] = None) -> None:
        c = None if code is None else np.ascontiguousarray(code, dtype=np.int8)
        v = None if value is None else np.ascontiguousarray(value, dtype=np.float64)
        self._check(self._lib.ensc_set_bcs(self.h, None if c is None else c.ctypes.data_as(C.POINTER(C.c_int8)),
                                           _dp(v)))

    def set_gravity(self, on: bool, value: float = 0.0, direction=(0.0, 0.0, 0.0)) -> None:
        d = np.ascontiguousarray(direction, dtype=np.float64)
        self._check(self._lib.ensc_set_gravity(self.h, int(on), float(value), _dp(d)))

    def set_gravity_amplitude(self, points) -> None:
        """(time, value) points of the gravity amplitude; empty removes it."""
        a = np.ascontiguousarray(points if points is not None else [], dtype=np.float64).reshape(-1)
        self._check(self._lib.ensc_set_gravity_amplitude(self.h, a.size // 2, _dp(a) if a.size else None))

    def step(self, max_cycles: int, step_end: float = math.inf) -> Dict[str, float]:
        r = StepReport()
        self._check(self._lib.ensc_step(self.h, int(max_cycles), float(step_end), C.byref(r)))
        return {k: getattr(r, k) for k, _ in StepReport._fields_}

    def step_until(self, max_cycles: int, step_end: float, pause: float) -> Dict[str, float]:
        r = StepReport()
        self._check(self._lib.ensc_step_until(self.h, int(max_cycles), float(step_end), float(pause), C.byref(r)))
        return {k: getattr(r, k) for k, _ in StepReport._fields_}

    def step_async(self, max_cycles: int, step_end: float = math.inf) -> None:
        self._check(self._lib.ensc_step_async(self.h, int(max_cycles), float(step_end)))

    def step_until_async(self, max_cycles: int, step_end: float, pause: float) -> None:
        self._check(self._lib.ensc_step_until_async(self.h, int(max_cycles), float(step_end), float(pause)))

    def snapshot_begin(self) -> None:
        """Captures the output fields now (in stream order) and starts their
        copy to host memory without waiting."""
        self._check(self._lib.ensc_snapshot_begin(self.h))

    def snapshot_wait(self) -> Dict[str, np.ndarray]:
        """Waits for the last snapshot and returns copies of its fields
        (x, u, v, a, rf: (n_nodes, 3); sigma: (n_elements, 6)) and clock."""
        sn = Snapshot()
        self._check(self._lib.ensc_snapshot_wait(self.h, C.byref(sn)))
        nn, ne = self.n_nodes, self.n_elements
        out = {k: np.ctypeslib.as_array(getattr(sn, k), shape=(nn * 3,)).reshape(nn, 3).copy()
               for k in ("x", "u", "v", "a", "rf")}
        out["sigma"] = np.ctypeslib.as_array(sn.sigma, shape=(ne * 6,)).reshape(ne, 6).copy()
        for k in ("time", "dt_i", "dt_i_1", "total_cycles", "status"):
            out[k] = getattr(sn, k)
        return out

    def sync(self) -> Dict[str, float]:
        r = StepReport()
        self._check(self._lib.ensc_sync(self.h, C.byref(r)))
        return {k: getattr(r, k) for k, _ in StepReport._fields_}

    def download(self, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        nn, ne = self.n_nodes, self.n_elements
        if out is None:
            out = {"x": np.empty((nn, 3)), "u": np.empty((nn, 3)), "v": np.empty((nn, 3)),
                   "sigma": np.empty((ne, 6)), "qia": np.empty((ne, 12)), "eps_p": np.empty(ne)}
        g = lambda k: _dp(out.get(k))  # noqa: E731
        self._check(self._lib.ensc_download(self.h, g("x"), g("u"), g("v"), g("sigma"), g("qia"), g("eps_p")))
        return out

    def upload_state(self, state: Dict[str, np.ndarray], time: float, dt_i: float, dt_i_1: float,
                     dt_stable_min: float = 0.0) -> None:
        arrays = {k: (None if state.get(k) is None else np.ascontiguousarray(state[k], dtype=np.float64))
                  for k in ("x", "u", "v", "sigma", "qia", "eps_p")}
        self._check(self._lib.ensc_upload_state(self.h, *[_dp(arrays[k]) for k in ("x", "u", "v", "sigma", "qia",
                                                                                     "eps_p")],
                                                float(time), float(dt_i), float(dt_i_1), float(dt_stable_min)))

    def energy(self) -> Dict[str, float]:
        r = EnergyReport()
        self._check(self._lib.ensc_energy(self.h, C.byref(r)))
        return {k: getattr(r, k) for k, _ in EnergyReport._fields_}

    def reactions(self) -> np.ndarray:
        rf = np.empty((self.n_nodes, 3))
        self._check(self._lib.ensc_download_reactions(self.h, _dp(rf)))
        return rf

    KERNELS = ("cycle_begin", "edge_prepass", "begin_exact", "element", "node")

    def profile(self, max_cycles: int, step_end: float = math.inf) -> Dict[str, Dict[str, float]]:
        """Per-kernel CUDA-event durations (ms summed, launches) over max_cycles."""
        ms = (C.c_double * 5)()
        n = (C.c_int64 * 5)()
        self._check(self._lib.ensc_profile(self.h, int(max_cycles), float(step_end), ms, n))
        return {k: {"ms": ms[i], "launches": int(n[i])} for i, k in enumerate(self.KERNELS)}

    @property
    def device_bytes(self) -> int:
        return int(self._lib.ensc_device_bytes(self.h))

    @property
    def kernels_per_cycle(self) -> int:
        return int(self._lib.ensc_kernels_per_cycle(self.h))

    @property
    def assembly(self) -> Dict[str, int]:
        """The force assembly in use (ensc_assembly), its patches and partials."""
        a, np_, nq = C.c_int32(), C.c_int64(), C.c_int64()
        self._check(self._lib.ensc_assembly(self.h, C.byref(a), C.byref(np_), C.byref(nq)))
        return {"assembly": int(a.value), "patches": int(np_.value), "partials": int(nq.value)}


class Prepared:
    """An instance prepared on the host for Batch.add_prepared
    (ensc_batch_prepare): element constants, lumped mass, node tables and
    the device rows, all held by the library (the mesh arrays are not read
    again).  The work runs in the C library without the interpreter lock, so
    several requests can be prepared on threads while a batch steps."""

    def __init__(self, x0: np.ndarray, conn: np.ndarray, v0: Optional[np.ndarray] = None, *,
                 material: _mesh.Material, controls: _mesh.Controls, precision: int = MIXED,
                 assembly: int = ASSEMBLY_AUTO):
        lib = load()
        self._lib = lib
        self.h = C.c_void_p()
        keep, m, mt, p = _descriptors(x0, conn, v0, material, controls)
        p.precision = int(precision)
        p.assembly = int(assembly)
        rc = lib.ensc_batch_prepare(C.byref(m), C.byref(mt), C.byref(p), C.byref(self.h))
        if rc != 0:
            raise EnscError(rc, lib.ensc_last_error(None).decode())
        del keep
        self.controls = controls
        self._params = p
        self.precision = precision
        self.sizes = (int(x0.shape[0]), int(conn.shape[0]))

    @property
    def device_bytes(self) -> int:
        return int(self._lib.ensc_prepared_bytes(self.h))

    @property
    def assembly(self) -> Dict[str, int]:
        """The force assembly the instance uses, its patches and partials."""
        a, np_, nq = C.c_int32(), C.c_int64(), C.c_int64()
        rc = self._lib.ensc_prepared_assembly(self.h, C.byref(a), C.byref(np_), C.byref(nq))
        if rc != 0:
            raise EnscError(rc, self._lib.ensc_last_error(None).decode())
        return {"assembly": int(a.value), "patches": int(np_.value), "partials": int(nq.value)}

    def patch_tables(self) -> Dict[str, np.ndarray]:
        """Copies of the patch tables (ensc_prepared_patch_tables)."""
        t = PatchTables()
        rc = self._lib.ensc_prepared_patch_tables(self.h, C.byref(t))
        if rc != 0:
            raise EnscError(rc, self._lib.ensc_last_error(None).decode())
        ne, nn, npch, nq = int(t.n_elements), int(t.n_nodes), int(t.n_patches), int(t.n_partials)

        def arr(ptr, n):
            return np.ctypeslib.as_array(ptr, shape=(n,)).copy()
        return {"stored": arr(t.stored, ne), "patch_first": arr(t.patch_first, npch + 1),
                "inc_first": arr(t.inc_first, nq + 1), "inc": arr(t.inc, 8 * ne),
                "node_first": arr(t.node_first, nn + 1), "node_partials": arr(t.node_partials, nq)}

    def close(self) -> None:
        if self.h:
            self._lib.ensc_prepared_destroy(self.h)
            self.h = C.c_void_p()
            self._keep = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent solver instances stepped together (ensc_batch_* ABI).

    Each instance is what a Stepper over the same arguments would be; the
    batch runs one launch per cycle phase for all of them."""

    def __init__(self, *, max_instances: int, max_elements: int, max_nodes: int, budget_bytes: int,
                 precision: int = MIXED, device: int = 0, stream: Optional[int] = None, graph_chunk: int = 0,
                 assembly: int = ASSEMBLY_AUTO):
        lib = load()
        self._lib = lib
        self.h = C.c_void_p()
        p = Params()
        p.precision = precision
        p.device = device
        p.stream = stream
        p.graph_chunk = graph_chunk
        p.assembly = assembly
        p.factor_timestep = 1.0
        rc = lib.ensc_batch_create(C.byref(p), int(max_instances), int(max_elements), int(max_nodes),
                                   int(budget_bytes), C.byref(self.h))
        if rc != 0:
            raise EnscError(rc, lib.ensc_last_error(None).decode())
        self.precision = precision
        self.assembly = assembly
        self.sizes: Dict[int, tuple] = {}

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise EnscError(rc, self._lib.ensc_batch_last_error(self.h).decode())

    def close(self) -> None:
        if self.h:
            self._lib.ensc_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add(self, x0: np.ndarray, conn: np.ndarray, v0: Optional[np.ndarray] = None, *,
            material: _mesh.Material, controls: _mesh.Controls, bt: Optional[np.ndarray] = None,
            vol0: Optional[np.ndarray] = None, inv_mass: Optional[np.ndarray] = None) -> int:
        keep, m, mt, p = _descriptors(x0, conn, v0, material, controls, bt, vol0, inv_mass)
        slot = C.c_int32(-1)
        self._check(self._lib.ensc_batch_add(self.h, C.byref(m), C.byref(mt), C.byref(p), C.byref(slot)))
        del keep
        self.sizes[slot.value] = (int(x0.shape[0]), int(conn.shape[0]))
        if controls.gravity_amplitude:
            self.set_gravity_amplitude(slot.value, controls.gravity_amplitude)
        return slot.value

    def add_prepared(self, prep: Prepared) -> int:
        """Adds an instance prepared by Prepared (ensc_batch_add_prepared);
        the Prepared object may be closed afterwards."""
        slot = C.c_int32(-1)
        self._check(self._lib.ensc_batch_add_prepared(self.h, prep.h, C.byref(prep._params), C.byref(slot)))
        self.sizes[slot.value] = prep.sizes
        if prep.controls.gravity_amplitude:
            self.set_gravity_amplitude(slot.value, prep.controls.gravity_amplitude)
        return slot.value

    def set_gravity_amplitude(self, slot: int, points) -> None:
        a = np.ascontiguousarray(points if points is not None else [], dtype=np.float64).reshape(-1)
        self._check(self._lib.ensc_batch_set_gravity_amplitude(self.h, int(slot), a.size // 2,
                                                               _dp(a) if a.size else None))

    def set_bcs(self, slot: int, code: Optional[np.ndarray], value: Optional[np.ndarray] = None) -> None:
        c = None if code is None else np.ascontiguousarray(code, dtype=np.int8)
        v = None if value is None else np.ascontiguousarray(value, dtype=np.float64)
        self._check(self._lib.ensc_batch_set_bcs(
            self.h, int(slot), None if c is None else c.ctypes.data_as(C.POINTER(C.c_int8)), _dp(v)))

    def arm(self, slot: int, max_cycles: int, step_end: float = math.inf) -> None:
        self._check(self._lib.ensc_batch_arm(self.h, int(slot), int(max_cycles), float(step_end)))

    def run(self, cycles: int) -> None:
        self._check(self._lib.ensc_batch_run(self.h, int(cycles)))

    def sync(self) -> int:
        n = C.c_int32(0)
        self._check(self._lib.ensc_batch_sync(self.h, C.byref(n)))
        return n.value

    def report(self, slot: int) -> Dict[str, float]:
        r = StepReport()
        self._check(self._lib.ensc_batch_report(self.h, int(slot), C.byref(r)))
        return {k: getattr(r, k) for k, _ in StepReport._fields_}

    def energy(self, slot: int) -> Dict[str, float]:
        r = EnergyReport()
        self._check(self._lib.ensc_batch_energy(self.h, int(slot), C.byref(r)))
        return {k: getattr(r, k) for k, _ in EnergyReport._fields_}

    def download(self, slot: int, fields=("x", "u", "v", "sigma", "qia", "eps_p")) -> Dict[str, np.ndarray]:
        nn, ne = self.sizes[slot]
        shapes = {"x": (nn, 3), "u": (nn, 3), "v": (nn, 3), "sigma": (ne, 6), "qia": (ne, 12), "eps_p": (ne,)}
        out = {k: np.empty(shapes[k]) for k in fields}
        g = lambda k: _dp(out.get(k))  # noqa: E731
        self._check(self._lib.ensc_batch_download(self.h, int(slot), g("x"), g("u"), g("v"), g("sigma"), g("qia"),
                                                  g("eps_p")))
        return out

    def remove(self, slot: int) -> None:
        self._check(self._lib.ensc_batch_remove(self.h, int(slot)))
        self.sizes.pop(slot, None)

    @property
    def device_bytes(self) -> int:
        return int(self._lib.ensc_batch_device_bytes(self.h))

    @property
    def instances(self) -> int:
        return int(self._lib.ensc_batch_instances(self.h))

    @property
    def tuning(self) -> Dict[str, int]:
        """The autotuner's launch choices (0 until its first tuning completes)
        and the batch's force assembly."""
        v = [C.c_int32() for _ in range(6)]
        self._check(self._lib.ensc_batch_tuning(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("mult_element", "mult_node", "graph_cycles", "node_threads", "elements_per_thread",
                         "assembly"), (x.value for x in v)))
