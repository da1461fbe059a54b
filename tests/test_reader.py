"""The fast deck reader (DataInFast, enscdynamics_b200/dropin/deck_reader.cpp)
against the reference's own reader (DataIn, Explicit3D/source/dataIn.cpp:
300-558) on the same decks: ensc_reader_bench reads each deck with both and
compares every member they fill in the solver -- nodes, hexahedra, sets,
surfaces, steps with their conditions and loads, initial velocities,
amplitudes, material, bulk viscosity, total time, output interval -- byte for
byte.

Decks: the reference's own examples (from a reference checkout, where one is
present) and decks written by enscdynamics_b200.mesh for the measured
workloads: per-node initial velocities, a multi-step deck with velocity
conditions, gravity and an amplitude, the butterfly-meshed impact bar with a
ZSYMM condition.  Both programs are built where the reference sources are
(enscdynamics_b200/dropin/Makefile)."""
import glob
import json
import os
import subprocess

import pytest

from _common import write_two_step_deck
from enscdynamics_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "enscdynamics_b200", "_lib", "ensc_reader_bench")
REF = os.environ.get("REF") or os.path.join(os.path.dirname(ROOT), "reference")

pytestmark = pytest.mark.skipif(not os.path.exists(BENCH), reason="ensc_reader_bench not built (needs the "
                                                                  "reference sources)")


def check(deck, cwd):
    r = subprocess.run([BENCH, deck, "1"], cwd=cwd, capture_output=True, text=True, timeout=300)
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert r.returncode == 0 and out["identical"], (deck, out, r.stderr[-500:])
    return out


@pytest.mark.parametrize("deck", sorted(glob.glob(os.path.join(REF, "inp", "*.inp"))) or ["none"])
def test_reference_example_decks(deck, tmp_path):
    if deck == "none":
        pytest.skip("no reference checkout")
    out = check(deck, str(tmp_path))
    assert out["elements"] > 0


@pytest.mark.parametrize("name", ["cantilever", "block_per_node_velocity", "two_step", "impact_bar"])
def test_generated_decks(name, tmp_path):
    d = str(tmp_path)
    if name == "cantilever":
        deck = W.cantilever().write_deck(d)
    elif name == "block_per_node_velocity":
        deck = W.block(24, 12, 8, 0.24, 0.12, 0.08).write_deck(d)
    elif name == "two_step":
        deck = write_two_step_deck(d)
    else:
        deck = W.impact_bar(4, 2, 8).write_deck(d)
    out = check(os.path.join(d, deck), d)
    assert out["elements"] > 0 and out["record_bytes"] > 0
