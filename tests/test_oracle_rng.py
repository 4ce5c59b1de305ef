"""Pins the oracle's random-number restatements: WELL19937a against the reference's own generator (golden
vectors produced by the reference C file, tests/golden/make_golden.py), Philox4x32-10 against the published
known-answer vectors of Salmon et al. (SC'11)."""
import glob
import os

import numpy as np
import pytest

import pyoracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "well19937a_*.txt"))))
def test_well_matches_reference_golden(path):
    seed = int(os.path.basename(path)[len("well19937a_"):-4])
    ref = [float.fromhex(l) for l in open(path).read().split("\n")[1:] if l]
    got = pyoracle.well_stream(seed, len(ref))
    assert len(ref) == 2000
    assert np.array_equal(got, np.array(ref)), "oracle WELL19937a differs from the reference generator"


@pytest.mark.skipif(not os.path.exists(pyoracle.REF_WELL), reason="reference generator not built here")
def test_well_matches_compiled_reference_long_stream():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mg", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    ref = mg.reference_stream(987654321, 20000)
    assert np.array_equal(pyoracle.well_stream(987654321, 20000), np.array(ref))


def test_well_range():
    v = pyoracle.well_stream(42, 50000)
    assert v.min() >= 0.0 and v.max() < 1.0
    assert abs(v.mean() - 0.5) < 0.01


@pytest.mark.parametrize("ctr,key,expect", [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(ctr, key, expect):
    assert pyoracle.philox(ctr, key) == expect


@pytest.mark.parametrize("ctr,key,expect", [
    ((0, 0), 0, (0xff1dae59, 0x6cd10df2)),
    ((0xffffffff, 0xffffffff), 0xffffffff, (0x2c3f628b, 0xab4fd7ad)),
    ((0x243f6a88, 0x85a308d3), 0x13198a2e, (0xdd7ce038, 0xf62a4c12)),
])
def test_philox2x32_known_answers(ctr, key, expect):
    assert pyoracle.philox2x32(ctr, key) == expect
