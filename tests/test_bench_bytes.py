"""The algorithmic byte counts the roofline fractions divide by: per element
and per node of each pass, as the bench's docstrings state them."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def per_unit(f, *args, **kw):
    """(bytes per element, bytes per node) of a linear byte count."""
    b00 = f(0, 0, *args, **kw)
    return f(1, 0, *args, **kw) - b00, f(0, 1, *args, **kw) - b00


def test_fp64_bytes_per_element_and_node():
    assert per_unit(bench.element_pass_bytes, True) == (712 + 16, 72)
    assert per_unit(bench.element_pass_bytes, False) == (712, 72)
    assert per_unit(bench.node_pass_bytes) == (192, 153)
    assert per_unit(bench.cycle_bytes, False) == (904, 225)
    assert per_unit(bench.cycle_bytes, True) == (904 + 16, 225)


def test_mixed_bytes_per_element_and_node():
    # slot assembly; the node pass reads and writes x alone (the u rows hold
    # x minus the reference position)
    assert per_unit(bench.element_pass_bytes, True, True) == (364, 36)
    assert per_unit(bench.node_pass_bytes, True) == (96, 93)
    assert per_unit(bench.cycle_bytes, False, True) == (452, 129)
    assert per_unit(bench.cycle_bytes, True, True) == (452 + 8, 129)


def test_block_cycle_bytes_are_far_above_l2():
    ne, nn = 256 * 128 * 64, 257 * 129 * 65
    l2 = 126e6
    assert bench.cycle_bytes(ne, nn, True, True) > 9 * l2
    assert bench.cycle_bytes(ne, nn, True, False) > 19 * l2
