"""Test infrastructure -- NOT part of the product.

Python access to the two checkers:

* ``Oracle``: ctypes wrapper of the plain-C restatement (ensc_oracle.c), built
  into oracle/_build/libensc_oracle.so by oracle/Makefile;
* ``run_reference`` / ``read_dump``: the reference CPU stepper compiled from
  its own sources into oracle/_ref/ensc_ref_harness (oracle/ref_harness.cpp),
  run on an ``.inp`` deck in a scratch directory, and its binary state dump.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libensc_oracle.so")
HARNESS = os.path.join(HERE, "_ref", "ensc_ref_harness")


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class _Params(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("rho", C.c_double),
                ("G", C.c_double), ("K", C.c_double), ("lam", C.c_double), ("wos", C.c_double),
                ("yield0", C.c_double), ("hardening", C.c_double),
                ("c_dr", C.c_double), ("c_cr", C.c_double), ("factor", C.c_double),
                ("cvisl", C.c_double), ("cvisq", C.c_double), ("total_time", C.c_double),
                ("gravity_on", C.c_int32), ("gravity_value", C.c_double), ("gravity_dir", C.c_double * 3),
                ("amp_n", C.c_int32), ("amp", C.POINTER(C.c_double))]


_P = C.POINTER(C.c_double)


class _State(C.Structure):
    _fields_ = [("nn", C.c_int64), ("ne", C.c_int64), ("conn", C.POINTER(C.c_uint32)),
                ("x", _P), ("u", _P), ("v", _P), ("inv_mass", _P), ("rf", _P),
                ("sigma", _P), ("qia", _P), ("eps_p", _P), ("bt", _P), ("vol0", _P),
                ("cbrt_v0", _P), ("cbrt_v0sq", _P), ("len", _P), ("dtstable", _P),
                ("force", _P), ("slots", _P),
                ("bc_code", C.POINTER(C.c_int8)), ("bc_value", _P),
                ("time", C.c_double), ("dt_i", C.c_double), ("dt_i_1", C.c_double),
                ("cycles", C.c_int64), ("energy", C.c_double * 5)]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        lib.ensc_oracle_material_update.argtypes = [C.POINTER(_Params)]
        lib.ensc_oracle_setup.argtypes = [C.c_int64, C.c_int64, C.POINTER(C.c_uint32), _P, C.c_double,
                                          _P, _P, _P, _P, _P]
        lib.ensc_oracle_cbrt_pair.argtypes = [C.c_int64, _P, _P, _P]
        lib.ensc_oracle_init_pass.argtypes = [C.POINTER(_Params), C.POINTER(_State)]
        lib.ensc_oracle_apply_bc_v.argtypes = [C.POINTER(_State)]
        lib.ensc_oracle_kinetic.argtypes = [C.POINTER(_State)]
        lib.ensc_oracle_kinetic.restype = C.c_double
        lib.ensc_oracle_cycles.argtypes = [C.POINTER(_Params), C.POINTER(_State), C.c_int64, C.c_double]
        lib.ensc_oracle_cycles.restype = C.c_int64
        _lib = lib
    return _lib


def _ptr(a: np.ndarray, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


class Oracle:
    """CPU restatement of one solver instance (FP64)."""

    def __init__(self, x0, conn, v0, bc_code, bc_value, *, E, nu, rho, c_dr=0.013, c_cr=0.05,
                 factor=0.71, cvisl=0.06, cvisq=1.2, total_time=1.0, yield0=0.0, hardening=0.0,
                 gravity=None, amplitude=None, setup: Optional[Dict[str, np.ndarray]] = None):
        lib = _load()
        self.nn = int(x0.shape[0])
        self.ne = int(conn.shape[0])
        nn, ne = self.nn, self.ne
        self.conn = np.ascontiguousarray(conn, dtype=np.uint32)
        self.x = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1).copy()
        self.u = np.zeros(3 * nn)
        self.v = np.ascontiguousarray(v0, dtype=np.float64).reshape(-1).copy()
        self.rf = np.zeros(3 * nn)
        self.sigma = np.zeros(6 * ne)
        self.qia = np.zeros(12 * ne)
        self.eps_p = np.zeros(ne)
        self.len = np.zeros(ne)
        self.dtstable = np.zeros(ne)
        self.force = np.zeros(3 * nn)
        self.slots = np.zeros(8 * 3 * nn)
        self.bc_code = np.ascontiguousarray(bc_code, dtype=np.int8).copy()
        self.bc_value = np.ascontiguousarray(bc_value, dtype=np.float64).copy()
        self.p = _Params(E=E, nu=nu, rho=rho, yield0=yield0, hardening=hardening, c_dr=c_dr, c_cr=c_cr,
                         factor=factor, cvisl=cvisl, cvisq=cvisq, total_time=total_time)
        if gravity is not None:
            self.p.gravity_on = 1
            self.p.gravity_value = gravity[0]
            for i in range(3):
                self.p.gravity_dir[i] = gravity[1][i]
        if amplitude is not None and len(amplitude) > 0:
            self.amp = np.ascontiguousarray(amplitude, dtype=np.float64).reshape(-1).copy()
            self.p.amp_n = self.amp.size // 2
            self.p.amp = _ptr(self.amp)
        lib.ensc_oracle_material_update(C.byref(self.p))
        self.bt = np.zeros(24 * ne)
        self.vol0 = np.zeros(ne)
        self.cbrt_v0 = np.zeros(ne)
        self.cbrt_v0sq = np.zeros(ne)
        self.inv_mass = np.zeros(3 * nn)
        lib.ensc_oracle_setup(nn, ne, _ptr(self.conn, C.c_uint32), _ptr(self.x), rho, _ptr(self.bt),
                              _ptr(self.vol0), _ptr(self.cbrt_v0), _ptr(self.cbrt_v0sq), _ptr(self.inv_mass))
        if setup is not None:  # adopt externally computed constants (e.g. the reference's)
            self.bt[:] = setup["bt"].reshape(-1)
            self.vol0[:] = setup["vol0"]
            self.inv_mass[:] = setup["inv_mass"].reshape(-1)
            # the C library's cbrt, as the reference (NumPy's cbrt can differ in the last bit)
            lib.ensc_oracle_cbrt_pair(ne, _ptr(self.vol0), _ptr(self.cbrt_v0), _ptr(self.cbrt_v0sq))
        s = _State()
        s.nn, s.ne = nn, ne
        s.conn = _ptr(self.conn, C.c_uint32)
        for name in ("x", "u", "v", "inv_mass", "rf", "sigma", "qia", "eps_p", "bt", "vol0", "cbrt_v0",
                     "cbrt_v0sq", "len", "dtstable", "force", "slots", "bc_value"):
            setattr(s, name, _ptr(getattr(self, name)))
        s.bc_code = _ptr(self.bc_code, C.c_int8)
        self.s = s
        lib.ensc_oracle_init_pass(C.byref(self.p), C.byref(self.s))
        lib.ensc_oracle_apply_bc_v(C.byref(self.s))
        self.s.energy[0] = lib.ensc_oracle_kinetic(C.byref(self.s))
        self.kinetic0 = self.s.energy[0]

    def set_bcs(self, code, value) -> None:
        self.bc_code[:] = code
        self.bc_value[:] = value
        _load().ensc_oracle_apply_bc_v(C.byref(self.s))

    def run(self, cycles: int, step_end: float = float("inf")) -> int:
        return int(_load().ensc_oracle_cycles(C.byref(self.p), C.byref(self.s), int(cycles), float(step_end)))

    @property
    def time(self) -> float:
        return self.s.time

    @property
    def dt(self):
        return self.s.dt_i, self.s.dt_i_1

    @property
    def energy(self) -> np.ndarray:
        return np.array(list(self.s.energy))

    @property
    def wos(self) -> float:
        return self.p.wos


# --------------------------------------------------------------------------
# reference harness

_SCAL = ["time", "dt_i", "dt_i_1", "total_time", "E", "nu", "rho", "G", "K", "lambda", "wos",
         "c_dr", "c_cr", "factor", "cvisl", "cvisq"]


def read_dump(path: str) -> Dict[str, np.ndarray]:
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:8] == b"ENSCDMP1", "not a harness dump"
    nn, ne, cyc = np.frombuffer(raw, dtype=np.int64, count=3, offset=8)
    nn, ne = int(nn), int(ne)
    off = 32
    scal = np.frombuffer(raw, dtype=np.float64, count=16, offset=off)
    off += 128
    out: Dict[str, np.ndarray] = {"n_nodes": nn, "n_elements": ne, "cycles": int(cyc)}
    for k, v in zip(_SCAL, scal):
        out[k] = float(v)

    def take(name, count, dtype, shape):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off).reshape(shape)
        off += count * np.dtype(dtype).itemsize
        out[name] = a.copy()

    for name in ("x", "u", "v", "inv_mass", "rf"):
        take(name, 3 * nn, np.float64, (nn, 3))
    take("sigma", 6 * ne, np.float64, (ne, 6))
    take("qia", 12 * ne, np.float64, (ne, 12))
    take("bt", 24 * ne, np.float64, (ne, 8, 3))
    take("vol0", ne, np.float64, (ne,))
    take("dtstable", ne, np.float64, (ne,))
    take("length", ne, np.float64, (ne,))
    take("conn", 8 * ne, np.uint32, (ne, 8))
    take("bc_code", 3 * nn, np.int8, (3 * nn,))
    take("bc_value", 3 * nn, np.float64, (3 * nn,))
    assert off == len(raw), "dump size mismatch"
    return out


def harness_available() -> bool:
    return os.path.exists(HARNESS) and os.access(HARNESS, os.X_OK)


def run_reference(workdir: str, deck: str, mode: str, cycles: Optional[int] = None, dump: Optional[str] = None,
                  threads: int = 1, timeout: Optional[float] = None) -> dict:
    """Runs the reference harness in ``workdir`` (which holds project.txt)."""
    args = [HARNESS, deck, mode]
    if mode in ("cycles", "time"):
        args.append(str(int(cycles)))
    if mode in ("cycles", "full", "setup"):
        args.append(dump)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run(args, cwd=workdir, env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference harness failed ({r.returncode}): {r.stderr[-2000:]}")
    line = [l for l in r.stdout.splitlines() if l.startswith("{")]
    return json.loads(line[-1]) if line else {}
