"""UPDATE_WALL_POTENTIALS with its waveform and amplitude-profile parts (pic2d_WallPotentials.f90:1-206;
PREPARE_WAVEFORMS and PREPARE_OSCILLATIONS_AMPLITUDE_PROFILE, pic2d_Setup.f90:150-412): the product's deck reader and
its host-side potential series (edp_deck_potential_series) against the oracle's restatement, which reads the same
files itself, bit for bit over several periods; fresh runs and runs continued at a later step. Runs without a GPU."""
import os

import numpy as np
import pytest

import pyoracle
from edipic_b200 import decks, read_deck

REFERENCE = os.environ.get("EDIPIC_REFERENCE", "")


def _compare(d, objects, steps, t0=0):
    dk = read_deck(d)
    prof = pyoracle.wall_profiles(d)
    for obj in objects:
        got = dk.potential_series(obj, t0, steps)
        w = prof[obj]
        w.adjust_phase(t0)
        want = np.array([w.value(t) for t in range(t0, t0 + steps)])
        assert np.array_equal(got, want), (obj, np.abs(got - want).max())
    return dk, prof


def test_pulsed_waveform_on_a_wall(tmp_path):
    """The top wall (object 2) carries a harmonic oscillation, a custom waveform of 1 GHz and an amplitude profile
    that switches the oscillating part off for most of each 19.5 ns pulse period: the phase is re-anchored at every
    profile period, the waveform's times snap to whole waveform periods at the pulse edges."""
    d = decks.write_deck(str(tmp_path), "cfg0", ncx=64, ncy=32, wall_potentials={2: 12.0},
                         oscillations={2: (30.0, 731.0, 15.0)},
                         waveforms={2: (50.0, 1.0e9, [(0.0, -1.0), (0.49, -0.5), (0.51, 1.0), (1.0, 0.5)])},
                         amplitude_profiles={2: [(0.0, 1.0), (5.0, 1.0), (5.0, 0.0), (19.5, 0.0)]})
    dk, prof = _compare(d, [0, 1], 12000)
    harm, wf, ap = dk.potential_profile(1)
    assert wf is not None and ap is not None
    assert list(wf[0]) == prof[1].wf_t and list(ap[0]) == prof[1].ap_t
    s = dk.potential_series(1, 0, 12000)
    per = ap[0][-1]
    assert np.all(s[ap[0][2]:per] == s[ap[0][2]])            # amplitude 0: the constant potential only
    assert np.abs(s[:ap[0][1]] - harm[0]).max() > 0          # oscillating within the pulse
    _compare(d, [1], 3000, t0=per * 2 + 17)                   # a run continued in the middle of a period


def test_oscillating_inner_object(tmp_path):
    """A metal inner object (object 5) oscillating harmonically, and a waveform without an amplitude profile on a
    wall of a walled domain."""
    d = decks.write_deck(str(tmp_path), "cfg2", ncx=64, ncy=64, inner=(20, 24, 36, 32, -40.0),
                         oscillations={5: (25.0, 1000.0, 45.0)},
                         waveforms={3: (10.0, 2.0e9, [(0.0, 0.0), (0.25, 1.0), (0.75, -1.0), (1.0, 0.0)])})
    dk, _ = _compare(d, [0, 1, 2, 3, 4], 2000)
    assert 4 in dk.potential_profiles and 3 in dk.potential_profiles
    assert dk.params.inner_phi[0] == dk.potential_series(4, 0, 1)[0]   # UPDATE_WALL_POTENTIALS(0) at set-up


def test_inconsistent_files_turn_the_profile_off(tmp_path):
    """A waveform with too many points for its period, a zero amplitude, or one point is off, as the reference only
    warns and goes on without it."""
    for k, wf in enumerate([(50.0, 1.0e11, [(0.0, 1.0), (0.3, 2.0), (0.6, 3.0), (1.0, 1.0)]),
                            (0.0, 1.0e9, [(0.0, 1.0), (1.0, 1.0)]),
                            (50.0, 1.0e9, [(0.0, 1.0)])]):
        d = decks.write_deck(str(tmp_path / str(k)), "cfg0", ncx=64, ncy=32, waveforms={2: wf})
        dk = read_deck(d)
        assert dk.potential_profile(1)[1] is None
        _compare(d, [1], 50)


@pytest.mark.skipif(not REFERENCE or not os.path.isdir(REFERENCE), reason="EDIPIC_REFERENCE unset or not a directory")
def test_reference_waveform_decks():
    """The reference's own example decks with a waveform and an amplitude profile, read as text by both sides."""
    seen = 0
    for name in ("input_data_waveform_amplitude_profiling", "input_data_files_waveform"):
        d = os.path.join(REFERENCE, name)
        if not os.path.isdir(d):
            continue
        try:
            dk = read_deck(d)
        except Exception:
            continue    # outside the supported deck subset (the external-circuit deck)
        objs = sorted(dk.potential_profiles)
        assert objs, name
        _compare(d, objs, 20000)
        seen += 1
    assert seen >= 1
