"""The C++ drop-in (ensc_dropin: the reference program with exDyna3D_GPU in
place of exDyna3D) against the reference's own exDyna3D::run() on the same
multi-step deck.

The deck exercises what the drop-in keeps from the reference: the deck
reader, init(), step switches with their boundary-condition and gravity
inheritance (step 2 adds a velocity condition on the tip, keeps the clamped
face through SPC inheritance and inherits step 1's gravity with its
amplitude), the last-step clamp at each step end, and output times.

Bars: FP64 nodal x, u, v and element sigma, QIA within REL_TOL_REFERENCE of
the reference (relative to each field's largest magnitude), the same cycle
count and final clock; mixed precision within 1e-5 of the reference's
displacements.  Both programs are built where the reference sources are
present (the harness by oracle/Makefile, the drop-in by
enscdynamics_b200/dropin/Makefile) and travel with the repository.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from _common import REL_TOL_REFERENCE, STEP1, STEP2, rel, write_two_step_deck

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle  # noqa: E402

DROPIN = os.path.join(ROOT, "enscdynamics_b200", "_lib", "ensc_dropin")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(DROPIN) and pyoracle.harness_available()),
                                 reason="drop-in or reference harness not built (needs the reference sources)")]

def run_dropin(d, deck, *args):
    out = subprocess.run([DROPIN, *args, "--dump", os.path.join(d, "gpu.bin"), deck], cwd=d,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return pyoracle.read_dump(os.path.join(d, "gpu.bin"))


@pytest.fixture(scope="module")
def reference_run(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("dropin"))
    deck = write_two_step_deck(d)
    pyoracle.run_reference(d, deck, "full", dump=os.path.join(d, "ref.bin"))
    return d, deck, pyoracle.read_dump(os.path.join(d, "ref.bin"))


def test_dropin_fp64_matches_reference_run(reference_run):
    d, deck, ref = reference_run
    gpu = run_dropin(d, deck, "--no-output")
    assert gpu["cycles"] == ref["cycles"] and gpu["cycles"] > 100
    assert abs(gpu["time"] - (STEP1 + STEP2)) <= 1e-15 and gpu["time"] == ref["time"]
    assert abs(gpu["dt_i"] - ref["dt_i"]) <= 1e-12 * ref["dt_i"]
    for k in ("x", "u", "v", "sigma", "qia"):
        assert rel(gpu[k], ref[k]) < REL_TOL_REFERENCE, (k, rel(gpu[k], ref[k]))
    # step 2's condition is in force at the end: tip nodes move at -0.5 in z
    tip = np.nonzero(ref["bc_code"].reshape(-1, 3)[:, 2] & 2)[0]
    assert tip.size > 0
    assert np.all(gpu["v"].reshape(-1, 3)[tip, 2] == -0.5)


def test_dropin_mixed_within_tolerance(reference_run):
    d, deck, ref = reference_run
    gpu = run_dropin(d, deck, "--no-output", "--precision", "mixed")
    assert gpu["cycles"] == ref["cycles"]
    assert rel(gpu["u"], ref["u"]) <= 1e-5, rel(gpu["u"], ref["u"])


def test_dropin_writes_results_at_output_times(reference_run):
    d, deck, ref = reference_run
    for f in os.listdir(d):
        if f.endswith(".vtu"):
            os.unlink(os.path.join(d, f))
    gpu = run_dropin(d, deck)
    files = sorted(f for f in os.listdir(d) if f.startswith("solution_") and f.endswith(".vtu"))
    assert len(files) >= 2
    # the state is the same whether or not the run pauses for output
    for k in ("u", "v", "sigma"):
        assert rel(gpu[k], ref[k]) < REL_TOL_REFERENCE, k
    import xml.etree.ElementTree as ET
    root = ET.parse(os.path.join(d, files[-1])).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    nn, ne = ref["x"].size // 3, ref["conn"].size // 8
    assert int(piece.get("NumberOfPoints")) == nn
    assert int(piece.get("NumberOfCells")) == ne
    arrays = {a.get("Name"): a for a in piece.iter("DataArray")}
    assert {"a", "force", "u", "v", "Stress", "connectivity", "offsets", "types"} <= set(arrays)
    # the acceleration written is the output cycle's (zero on constrained
    # DOFs); its bit-exactness is tested through the C ABI (test_gpu_output)
    assert np.all(np.isfinite(vtu_array(arrays["u"], np.float64)))
    assert np.array_equal(vtu_array(arrays["connectivity"], np.int64), gpu["conn"].astype(np.int64).reshape(-1))
    a = vtu_array(arrays["a"], np.float64).reshape(nn, 3)
    code = gpu["bc_code"].reshape(nn, 3)
    assert np.all(np.isfinite(a)) and np.all(a[code != 0] == 0.0)
    assert np.abs(a[code == 0]).max() > 0.0
    assert not np.any(vtu_array(arrays["force"], np.float64))  # the reference never fills solution_f


def vtu_array(el, dtype):
    """Values of an inline base64 DataArray (UInt64 byte-count header)."""
    import base64
    raw = base64.b64decode("".join(el.text.split()))
    n = int(np.frombuffer(raw[:8], dtype=np.uint64)[0])
    return np.frombuffer(raw[8:8 + n], dtype=dtype)
