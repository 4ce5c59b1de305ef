"""The product's deck reader (edp_deck_read, C++) against the oracle's independent reading of the same files:
normalisation, geometry and the e-n collision probability table (bit for bit), RCX constants and the Maxwell
table. Runs without a GPU."""
import ctypes as C
import math
import os

import numpy as np
import pytest

import pyoracle
from edipic_b200 import decks, read_deck

# the reference source tree (its example decks), named by the environment; the tests that read it skip without it
REFERENCE = os.environ.get("EDIPIC_REFERENCE", "")


@pytest.fixture(scope="module", params=["cfg0", "cfg1", "cfg2", "cfg4"])
def deck(request, tmp_path_factory):
    d = decks.write_deck(str(tmp_path_factory.mktemp(request.param)), request.param)
    return request.param, d, read_deck(d)


def test_normalisation(deck):
    name, _d, dk = deck
    p = dk.params
    assert math.isclose(p.delta_x_m, 1e-4, rel_tol=1e-6)
    assert math.isclose(p.delta_t_s, decks.CONFIGS[name]["dt"], rel_tol=1e-4)
    assert p.ncx == decks.CONFIGS[name]["ncx"] and p.ncy == decks.CONFIGS[name]["ncy"]
    assert p.periodic_x == (1 if decks.CONFIGS[name]["periodic"] else 0)
    # E_scale = m_e V_scale/(e dt), B_scale = m_e/(e dt), F_scale = e N dx^2/eps0 (pic2d_CurProblemValues.f90:893-900)
    assert math.isclose(p.b_scale_t, 9.109534e-31 / (1.602189e-19 * p.delta_t_s), rel_tol=1e-12)
    assert math.isclose(p.e_scale_vm, p.b_scale_t * p.v_scale_ms, rel_tol=1e-12)


def test_mcc_table_matches_oracle_bitwise(deck):
    _name, d, dk = deck
    t, p = dk.tables, dk.params
    neu = pyoracle.read_neutral_deck(d)
    ot = pyoracle.MccTables(neu, p.n_subcycles, p.delta_t_s)
    assert t.en_on == 1 and t.n_act == ot.t.n_act == 3
    assert t.n_values == ot.t.n_values
    assert t.max_colliding_fraction == ot.t.max_colliding_fraction
    nv = t.n_values
    e = np.ctypeslib.as_array(t.energy_eV, shape=(nv + 1,))
    pr = np.ctypeslib.as_array(t.prob, shape=((nv + 1) * t.n_act,))
    assert np.array_equal(e, ot.energy)
    assert np.array_equal(pr, ot.prob)
    assert [t.seg_index[i] for i in range(t.n_seg + 1)] == [ot.t.seg_index[i] for i in range(t.n_seg + 1)]
    assert [t.threshold_eV[i] for i in range(3)] == [0.0, 11.55, 15.76]
    # cumulative, normalised, non-decreasing (:300-322)
    P = pr.reshape(nv + 1, 3)
    assert np.all(np.diff(P, axis=1) >= 0) and P.max() == 1.0 and P.min() >= 0.0


def test_rcx_and_maxwell_match_oracle(deck):
    _name, d, dk = deck
    t, p = dk.tables, dk.params
    neu = pyoracle.read_neutral_deck(d)
    pt = pyoracle.lib().oracle_rcx_probab_thermal(5.0e-19, 0.0, neu["t_k"], neu["n_m3"], p.ion_mass_me[0],
                                                  p.delta_t_s, p.n_subcycles)
    assert t.rcx_on[0] == 1
    assert math.isclose(t.rcx_probab_thermal[0], pt, rel_tol=1e-13)
    v, _vi = pyoracle.maxwell_tables()
    mv = np.ctypeslib.as_array(t.maxwell_v, shape=(t.maxwell_rmax + 1,))
    assert np.array_equal(mv, v)


def test_missing_deck_is_an_io_error(tmp_path):
    from edipic_b200 import EdpError
    with pytest.raises(EdpError) as e:
        read_deck(str(tmp_path))
    assert e.value.code == -8


@pytest.mark.skipif(not REFERENCE or not os.path.isdir(REFERENCE), reason="EDIPIC_REFERENCE unset or not a directory")
def test_reference_example_decks_parse_or_are_rejected_cleanly():
    """The reference's own example decks: the supported subset (metal/periodic walls, metal inner objects) parses;
    decks with dielectric walls or vacuum gaps are rejected with EDP_ERR_IO rather than misread."""
    from edipic_b200 import EdpError
    seen = 0
    for name in sorted(os.listdir(REFERENCE)):
        d = os.path.join(REFERENCE, name)
        if not (name.startswith("input_data") and os.path.isdir(d)):
            continue
        seen += 1
        try:
            dk = read_deck(d)
        except EdpError as e:
            assert e.code == -8
            continue
        p = dk.params
        assert p.ncx > 0 and p.ncy > 0 and p.delta_t_s > 0
        if dk.tables.en_on:
            neu = pyoracle.read_neutral_deck(d)
            ot = pyoracle.MccTables(neu, p.n_subcycles, p.delta_t_s)
            nv = dk.tables.n_values
            pr = np.ctypeslib.as_array(dk.tables.prob, shape=((nv + 1) * dk.tables.n_act,))
            assert np.array_equal(pr, ot.prob), name
    assert seen == 11


def test_wall_material_ion_emission(tmp_path):
    """init_material_<NAME>.dat of the walls: ion-material model 2 gives the ion-induced emission parameters per
    wall and ion species (pic2d_Materials.f90:150-188); model 0 gives none."""
    d = read_deck(decks.write_deck(str(tmp_path / "a"), "cfg4", ncx=64, ncy=32, ppc=4))
    assert d.ion_emission == {(0, 1): (0.1, 0.0, 10000.0, 2.0), (1, 1): (0.1, 0.0, 10000.0, 2.0)}
    d = read_deck(decks.write_deck(str(tmp_path / "b"), "cfg2", ncx=64, ncy=32, ppc=4,
                                   ion_emission=(1.25, 5.0, 500.0, 1.5)))
    # the four walls and the inner object (object 4) share the material METAL1
    assert d.ion_emission == {(w, 1): (1.25, 5.0, 500.0, 1.5) for w in range(5)}
    d = read_deck(decks.write_deck(str(tmp_path / "c"), "cfg0", ncx=64, ncy=32, ppc=4))
    assert d.ion_emission == {}


@pytest.mark.skipif(not REFERENCE or not os.path.isdir(REFERENCE), reason="EDIPIC_REFERENCE unset or not a directory")
def test_reference_ion_emission_deck():
    """The reference's periodic ion-induced emission example: both walls' material file read as text here must give
    the reader's values."""
    d = os.path.join(REFERENCE, "input_data_dc_periodic_ion_induced_EE")
    lines = open(os.path.join(d, "init_material_METAL2.dat")).read().splitlines()
    k = next(i for i, L in enumerate(lines) if "ION-MATERIAL INTERACTION MODEL" in L)
    assert int(lines[k + 1][7:8]) == 2
    want = (float(lines[k + 4][7:12]), float(lines[k + 6][2:12]), float(lines[k + 8][2:12]),
            float(lines[k + 10][2:12]))
    got = read_deck(d).ion_emission
    assert got == {(0, 1): want, (1, 1): want}
    assert want == (0.2, 100.0, 10000.0, 2.0)


def test_wall_material_ion_reflection(tmp_path):
    d = read_deck(decks.write_deck(str(tmp_path / "r"), "cfg2", ncx=64, ncy=32, ppc=4, ion_reflection=True))
    assert d.ion_wall_model == [1, 1, 1, 1, 1]   # the walls, then the inner object
    assert d.ion_emission == {}
    d = read_deck(decks.write_deck(str(tmp_path / "e"), "cfg4", ncx=64, ncy=32, ppc=4))
    assert d.ion_wall_model == [2, 2, 0, 0]


def test_oracle_reads_the_deck_independently(deck):
    """The oracle's own reading of the decks (pyoracle.read_deck: the reference's READ edit descriptors and its
    normalisation formulas, pic2d_CurProblemValues.f90:157-1255, pic2d_ExternalFields.f90:36-145,
    pic2d_inCollisionsGeneralProc.f90:3-90) gives every constant the device cycle uses, bit for bit equal to the
    product's edp_deck_read. The whole-cycle parity tests build the oracle's cycle from this reading only."""
    _name, d, dk = deck
    p, t = dk.params, dk.tables
    o = pyoracle.read_deck(d)
    assert (o["ncx"], o["ncy"], int(o["periodic"])) == (p.ncx, p.ncy, p.periodic_x)
    assert o["N_of_particles_cell"] == p.n_of_particles_cell and o["N_subcycles"] == p.n_subcycles
    assert o["seed"] == p.seed
    for a, b in (("delta_t_s", "delta_t_s"), ("delta_x_m", "delta_x_m"), ("V_scale_ms", "v_scale_ms"),
                 ("E_scale_Vm", "e_scale_vm"), ("B_scale_T", "b_scale_t"), ("F_scale_V", "f_scale_v"),
                 ("Bx_ext", "bx"), ("By_ext", "by"), ("Bz_ext", "bz"), ("Ez_ext", "ez")):
        assert o[a] == getattr(p, b), a
    assert int(o["ions_sense_magnetic_field"]) == p.ions_sense_b and int(o["ions_sense_Ez"]) == p.ions_sense_ez
    assert o["energy_factor_eV"] == t.energy_factor_eV
    ion = o["ions"][0]
    assert ion["Ms"] == p.ion_mass_me[0] and ion["Qs"] == p.ion_charge[0]
    for side, w in o["walls"].items():
        assert (w["phi_const"], w["phi_var"], w["omega"], w["phase"]) == (
            p.wall_phi_const[side], p.wall_phi_var[side], p.wall_omega[side], p.wall_phase[side]), side
    assert len(o["inner"]) == p.n_inner
    for k, (il, jb, ir, jt) in enumerate(o["inner"]):
        assert (il, jb, ir, jt) == (p.inner_ileft[k], p.inner_jbottom[k], p.inner_iright[k], p.inner_jtop[k])
        b = o["inner_objects"][k]
        assert b["phi_const"] + b["phi_var"] * math.sin(b["phase"]) == p.inner_phi[k]
    assert o["ion_velocity_factor"] == [t.ion_velocity_factor[q] for q in range(t.n_act)]
    r = o["rcx"]
    assert t.rcx_on[0] == 1 and r["species"] == 1
    assert (r["prob_factor"], r["sigma_1eV"], r["alpha"], r["probab_thermal"], r["vfactor"]) == (
        t.rcx_prob_factor, t.rcx_sigma_1eV, t.rcx_alpha, t.rcx_probab_thermal[0], t.rcx_vfactor[0])
    # E from phi (CALCULATE_ELECTRIC_FIELD_FFTX_LINSYSY, pic2d_ElectricFieldCalc_FFT_X.f90:1350-1351)
    assert o["factor2_E"] == p.f_scale_v / (p.e_scale_vm * 2.0 * p.delta_x_m)
    assert o["factor_rho"] == 1.0 / p.n_of_particles_cell
