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


# SplitMix64's published reference outputs (the sequential generator of Steele, Lea and Flood as distributed with the
# xoshiro generators): seed 0 and seed 1234567
@pytest.mark.parametrize("seed,expect", [
    (0, [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]),
    (1234567, [6457827717110365317, 3203168211198807973, 9817491932198370423, 4593380528125082431,
               16408922859458223821]),
])
def test_splitmix64_known_answers(seed, expect):
    assert pyoracle.splitmix64_stream(seed, len(expect)) == expect
    # the direct evaluation at a position, as the decision draws use it, is the same sequence
    assert [pyoracle.splitmix64_at(seed, n + 1) for n in range(len(expect))] == expect


def test_decision_draw_positions():
    """A decision draw is output (step << 32 | id) of the stream seeded with mix64(seed ^ tag): stepping that stream
    one state at a time reaches the same words, and distinct (id, step) give distinct draws."""
    seed, tag = 0x0123456789ABCDEF, 0x4D430000
    s0 = pyoracle.lib().oracle_mix64(seed ^ tag)
    seq = pyoracle.splitmix64_stream(s0, 40)
    for pid in range(1, 41):
        z = seq[pid - 1]
        assert pyoracle.decision_draw(seed, tag, 0, pid) == (z >> 32, z & 0xFFFFFFFF)
    draws = {pyoracle.decision_draw(seed, tag, st, pid) for st in range(50) for pid in range(200)}
    assert len(draws) == 50 * 200
    # word 0 is uniform enough for a Bernoulli(P_max) selection at P_max = 1/64: counts over 2^16 draws
    hits = sum(pyoracle.decision_draw(seed, tag, st, pid)[0] < (1 << 26) for st in range(64) for pid in range(1024))
    assert abs(hits - 1024) < 5 * 32
