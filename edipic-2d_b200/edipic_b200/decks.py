"""Synthetic input decks for the benchmark configurations, written in the reference's fixed-column format.

Each file follows the edit descriptors with which EDIPIC-2D reads it (init_configuration.dat:
pic2d_CurProblemValues.f90:157-330; init_simcontrol.dat :830-845; init_particles.dat :1005-1031;
init_extfields.dat pic2d_ExternalFields.f90:36-72; init_bo_NN.dat pic2d_Setup.f90:76-99; neutral decks
pic2d_enCollisionsGeneralProc.f90:63-190; RCX pic2d_inCollisionsGeneralProc.f90:56-60), so the same directory
can be read by the reference and by edp_deck_read. Cross sections are analytic synthetic shapes (not
measured data) tabulated on 200 log-spaced energies.

Normalisation: dx = 0.1 mm and dt = dx / (N_max_vel v_Te) are reached with N_of_cells_debye = 1 and a scale
temperature/density chosen for them (T_scale = 1.9741945 eV, N_scale = 2.1820009e16 m^-3); the per-cell count of
the scale density, N_of_particles_cell, is the integer nearest to N_scale * ppc / n_init.
"""
import math
import os

import numpy as np

T_SCALE_EV = 1.9741945
N_SCALE_M3 = 2.1820009e16
E_EXC_EV = 11.55
E_ION_EV = 15.76

CONFIGS = {
    # name: (ncx, ncy, periodic, ppc, n_init, dt_s, steps, B_gauss (Bx, By), inner object, top RF (V, MHz))
    "cfg0": dict(ncx=128, ncy=128, periodic=True, ppc=64, n_init=1.0e16, dt=5e-12, steps=1000, bx=0.0, by=0.0),
    "cfg1": dict(ncx=1024, ncy=1024, periodic=True, ppc=200, n_init=1.0e16, dt=5e-12, steps=200, sort_every=20,
                 bx=100.0 * math.cos(math.radians(30.0)), by=100.0 * math.sin(math.radians(30.0))),
    "cfg2": dict(ncx=512, ncy=512, periodic=False, ppc=100, n_init=1.0e16, dt=5e-12, steps=2000, bx=0.0, by=0.0,
                 inner=(224, 112, 288, 144, -100.0)),
    "cfg4": dict(ncx=2048, ncy=512, periodic=True, ppc=100, n_init=5.0e15, dt=1e-11, steps=100000, bx=0.0, by=0.0,
                 top_rf=(200.0, 13.56), ion_emission=(0.1, 0.0, 10000.0, 2.0)),
}


# electron-induced emission of the wall material, all three models off (fields of edp_see_params)
SEE_OFF = dict(elastic_model=0, elastic_type=0, inelastic_model=0, true_model=0, elastic_yield=0.0,
               elastic_emin_ev=0.0, elastic_emax_ev=0.0, elastic_e0_ev=0.0, elastic_emax_coef_ev=0.0, elastic_max=0.0,
               elastic_de_ev=0.0, elastic_frac_classic=0.0, inelastic_yield=0.0, inelastic_emin_ev=0.0,
               inelastic_emax_ev=0.0, inelastic_frac_classic=0.0, true_t_ev=0.0, true_yield=0.0, true_emin_ev=0.0,
               true_emax_ev=0.0, classic_e0_ev=0.0, classic_emax_ev=0.0, classic_max=0.0, classic_k_smooth=0.0)


def sigma_elastic(e):
    return 1.0e-19 / (1.0 + e / 15.0) + 5.0e-21


def sigma_lotz(e, eth, c):
    x = np.maximum(e / eth, 1.0)
    return c * np.log(x) / x


def _blocks(n_total):
    """Split n_total cells into (blocks, cells per block) with at most 999 cells per block (the i3 field)."""
    for nb in range(1, n_total + 1):
        if n_total % nb == 0 and n_total // nb <= 999:
            return nb, n_total // nb
    raise ValueError(n_total)


def _segments():
    # energy grid of the collision probability table: (upper boundary, resolution) [eV]
    return 0.0, [(0.1, 0.01), (1.0, 0.02), (10.0, 0.05), (30.0, 0.05), (100.0, 0.5), (1000.0, 5.0)]


def write_deck(directory, name="cfg0", ncx=None, ncy=None, ppc=None, steps=None, seed=0, n_subcycles=1,
               collisions=True, rcx=True, bx=None, by=None, inner=None, wall_potentials=None, n_gas=3.2e21,
               ion_emission=None, ion_reflection=False, electron_emission=None, wall_injection=None, ez=0.0,
               ions_sense_b=False, ions_sense_ez=False, oscillations=None, waveforms=None, amplitude_profiles=None,
               en_collisions=True):
    """ion_emission: (yield, E_min [eV], E_max [eV], T_emit [eV]) of ion-induced electron emission at every wall
    (the wall material METAL1), False for none, None for the configuration's default. ion_reflection: the walls
    reflect all ions specularly instead (ion-material model 1). electron_emission: fields of edp_see_params (models
    and parameters of electron-induced emission, energies in eV) for the walls' material; all models off by default.
    wall_injection: {wall (0 below, 1 above, 2 left, 3 right; 4 + n metal inner object n): (electrons per step, model,
    T_normal, T_parallel, beam energy [eV])}, the constant electron emission of init_bo_NN.dat. ez: uniform Z electric field [V/cm];
    ions_sense_b / ions_sense_ez: the ions feel the magnetic / Z electric field (init_extfields.dat flags).
    Time dependence of metal objects, keyed by the reference's object number (1-based: the four boundary objects,
    then the inner objects): oscillations {n: (amplitude [V], frequency [MHz], phase [deg])} in init_bo_NN.dat;
    waveforms {n: (amplitude [V], frequency [Hz], [(fraction of the period, value), ...])} written as
    init_bo_NN_waveform.dat; amplitude_profiles {n: [(time [ns], factor), ...]} as init_bo_NN_amplitude_profile.dat.
    en_collisions=False keeps the neutral gas (for charge exchange) with its electron-neutral processes deactivated."""
    cfg = dict(CONFIGS[name])
    ncx = ncx or cfg["ncx"]
    ncy = ncy or cfg["ncy"]
    ppc = ppc or cfg["ppc"]
    steps = steps or cfg["steps"]
    bx = cfg["bx"] if bx is None else bx
    by = cfg["by"] if by is None else by
    inner = cfg.get("inner") if inner is None else (inner or None)
    periodic = cfg["periodic"]
    dt = cfg["dt"]
    os.makedirs(directory, exist_ok=True)
    dx = 1.0e-4
    v_te = math.sqrt(2.0 * T_SCALE_EV * 1.602189e-19 / 9.109534e-31)
    n_max_vel = int(round(dx / dt / v_te))
    n_ppc = int(round(N_SCALE_M3 * ppc / cfg["n_init"]))
    nx_total = ncx if periodic else ncx - 1
    ny_total = ncy - 1
    nbx, ngx = _blocks(nx_total)
    nby, ngy = _blocks(ny_total)
    gmi, gmj = nx_total + 1, ny_total + 1
    w = lambda fn, lines: open(os.path.join(directory, fn), "w").write("\n".join(lines) + "\n")

    objs = []   # (type, [segments])
    if periodic:
        objs = [(2, [(0, 0, 0, gmj)]), (1, [(0, gmj, gmi, gmj)]), (2, [(gmi, 0, gmi, gmj)]), (1, [(0, 0, gmi, 0)])]
    else:
        objs = [(1, [(0, 0, 0, gmj)]), (1, [(0, gmj, gmi, gmj)]), (1, [(gmi, 0, gmi, gmj)]), (1, [(0, 0, gmi, 0)])]
    # inner objects: (ileft, jbottom, iright, jtop, phi) for a metal one, (..., phi, eps) for a dielectric one
    inner_list = ([inner] if isinstance(inner, tuple) else list(inner)) if inner else []
    cf = [
        "---dddd.ddddddd----- scale electron temperature [eV]", f"   {T_SCALE_EV:12.7f}",
        "---+d.dddddddE+dd--- scale electron density [m^-3]", f"   {N_SCALE_M3:14.7E}",
        "---ddd---------- cells per scale Debye length", f"   {1:3d}",
        "---ddd---------- maximal expected velocity [scale thermal velocities]", f"   {n_max_vel:3d}",
        "---ddd---------- blocks along X", f"   {nbx:3d}",
        "---ddd---------- blocks along Y", f"   {nby:3d}",
        "---ddd---------- cells along X in a block", f"   {ngx:3d}",
        "---ddd---------- cells along Y in a block", f"   {ngy:3d}",
        "--dddd---------- macroparticles per cell for the scale density", f"  {n_ppc:4d}",
        "-----d---------- blocks in a cluster along X", f"     {min(nbx, 9):1d}",
        "-----d---------- blocks in a cluster along Y", f"     {min(nby, 9):1d}",
        "---ddd---ddd---- boundary objects // inner objects", f"   {len(objs):3d}   {len(inner_list):3d}",
    ]
    for k, (ty, segs) in enumerate(objs):
        cf += [f"===dd===dd=== object type, number of segments // #{k + 1}", f"   {ty:2d}   {len(segs):2d}",
               "---dddddd---dddddd---dddddd---dddddd--- segment start X/Y end X/Y"]
        cf += [f"   {a:6d}   {b:6d}   {c:6d}   {d:6d}" for (a, b, c, d) in segs]
    for obj in inner_list:
        il, jb, ir, jt = obj[:4]
        cf += ["===dd=== object type", f"   {4 if len(obj) > 5 else 1:2d}",
               "---dddddd---dddddd---dddddd---dddddd--- left bottom X/Y, right top X/Y",
               f"   {il:6d}   {jb:6d}   {ir:6d}   {jt:6d}"]
    w("init_configuration.dat", cf)

    w("init_simcontrol.dat", [
        "---ddddddd.ddd----- simulation time [ns]", f"   {steps * dt * 1e9:11.3f}",
        "--------dd--------- electron sub-cycles per ion cycle (odd)", f"        {n_subcycles:2d}",
        "------dddd--------- ion cycles between cluster load balancing", f"      {10:4d}",
        "------dddd--------- cluster balancing events between global balancing", f"      {10:4d}",
        "---ddddddd--------- ion cycles between checkpoints", f"   {0:7d}",
        "---------d--------- use checkpoint", f"         {0:1d}",
        "--dddddddd--------- time step of the checkpoint", f"  {0:8d}",
    ])
    w("init_particles.dat", [
        "---dddd.ddd----- initial electron temperature [eV]", f"   {2.0:8.3f}",
        "---+d.dddE+dd--- initial electron density [m^-3]", f"   {cfg['n_init']:10.3E}",
        "------d--------- number of ion species", f"      {1:1d}",
        "---ddd.d---+d---dddd.ddd---ddd.dd-- ion mass / charge / temperature / concentration",
        f"   {40.0:5.1f}   {1:2d}   {0.03:8.3f}   {100.0:6.2f}",
        "---ddddddddd---- seed", f"   {seed:9d}",
    ])
    w("init_extfields.dat", [
        "---ddddd.ddd--- X-magnetic field [Gauss]", f"   {bx:9.3f}",
        "---ddddd.ddd--- Y-magnetic field [Gauss]", f"   {by:9.3f}",
        "--------------- Z-magnetic field profile",
        "---ddddd.ddd--- y_Bmax [cm]", f"   {0.0:9.3f}",
        "---ddddd.ddd--- BZ at y=0 [Gauss]", f"   {0.0:9.3f}",
        "---ddddd.ddd--- BZ at y_Bmax [Gauss]", f"   {0.0:9.3f}",
        "---ddddd.ddd--- BZ at y=Lsys [Gauss]", f"   {0.0:9.3f}",
        "---ddddd.ddd--- decay length below y_Bmax [cm]", f"   {1.0:9.3f}",
        "---ddddd.ddd--- decay length above y_Bmax [cm]", f"   {1.0:9.3f}",
        "---ddddd.ddd--- Z-electric field [V/cm]", f"   {ez:9.3f}",
        "-------d------- ions sense magnetic field", f"       {int(bool(ions_sense_b)):1d}",
        "-------d------- ions sense Z-electric field", f"       {int(bool(ions_sense_ez)):1d}",
    ])

    osc = oscillations or {}

    def bo(n, phi, amp=0.0, mhz=0.0, inj=(0.0, 0, 0.0, 0.0, 0.0), material="METAL1"):
        phase = 0.0
        if n in osc:
            amp, mhz, phase = osc[n]
        w(f"init_bo_{n:02d}.dat", [
            "------AAAAAA--- material", f"      {material}",
            "---ddddd.ddd--- constant potential [V]", f"   {phi:9.3f}",
            "---ddddd.ddd--- amplitude of oscillations [V]", f"   {amp:9.3f}",
            "---ddddd.ddd--- frequency [MHz]", f"   {mhz:9.3f}",
            "---ddddd.ddd--- phase [deg]", f"   {phase:9.3f}",
            "---ddddd.ddd--- electrons injected per step", f"   {inj[0]:9.3f}",
            "-------d------- emission model", f"       {int(inj[1]):1d}",
            "----dddd.ddd--- emitted temperature normal [eV]", f"    {inj[2]:8.3f}",
            "----dddd.ddd--- emitted temperature parallel [eV]", f"    {inj[3]:8.3f}",
            "----dddd.ddd--- beam energy [eV]", f"    {inj[4]:8.3f}",
            "-------d------- save collided ions", f"       {0:1d}",
            "-------d------- save collided electrons", f"       {0:1d}",
        ])
    iee = cfg.get("ion_emission") if ion_emission is None else (ion_emission or None)
    # init_material_METAL1.dat in the layout PREPARE_WALL_MATERIALS reads (pic2d_Materials.f90:79-188): electron
    # reflection and secondary emission off, ion-material model 2 (ion-induced emission) or 0 (absorption)
    see = dict(SEE_OFF, **(electron_emission or {}))
    i1, f5, f6, f10 = (lambda v: f"       {int(v):1d}"), (lambda v: f"       {v:5.3f}"), (lambda v: f"      {v:6.3f}"), \
        (lambda v: f"  {v:10.3f}")
    mat = [
        "------dd.ddd- dielectric constant", f6(1.0),
        "=======d===== elastic electron reflection model", i1(see["elastic_model"]),
        "-------d----- elastic electron reflection type", i1(see["elastic_type"]),
        "------------- elastic reflection, model 1",
        "-------d.ddd- coefficient", f5(see["elastic_yield"]),
        "--dddddd.ddd- E_min [eV]", f10(see["elastic_emin_ev"]),
        "--dddddd.ddd- E_max [eV]", f10(see["elastic_emax_ev"]),
        "------------- elastic reflection, model 2",
        "--dddddd.ddd- threshold [eV]", f10(see["elastic_e0_ev"]),
        "--dddddd.ddd- energy of the maximum [eV]", f10(see["elastic_emax_coef_ev"]),
        "-------d.ddd- maximum", f5(see["elastic_max"]),
        "--dddddd.ddd- decay scale [eV]", f10(see["elastic_de_ev"]),
        "-------d.ddd- high-energy fraction", f5(see["elastic_frac_classic"]),
        "=======d===== inelastic electron reflection model", i1(see["inelastic_model"]),
        "------------- inelastic reflection, model 1",
        "-------d.ddd- coefficient", f5(see["inelastic_yield"]),
        "--dddddd.ddd- E_min [eV]", f10(see["inelastic_emin_ev"]),
        "--dddddd.ddd- E_max [eV]", f10(see["inelastic_emax_ev"]),
        "------------- inelastic reflection, model 2",
        "-------d.ddd- fraction", f5(see["inelastic_frac_classic"]),
        "=======d===== true secondary emission model", i1(see["true_model"]),
        "--dddddd.ddd- temperature [eV]", f10(see["true_t_ev"]),
        "------------- true secondary emission, model 1",
        "-------d.ddd- coefficient", f5(see["true_yield"]),
        "--dddddd.ddd- E_min [eV]", f10(see["true_emin_ev"]),
        "--dddddd.ddd- E_max [eV]", f10(see["true_emax_ev"]),
        "------------- true secondary emission, model 2",
        "--dddddd.ddd- threshold [eV]", f10(see["classic_e0_ev"]),
        "--dddddd.ddd- energy of the maximum [eV]", f10(see["classic_emax_ev"]),
        "------dd.ddd- maximum", f6(see["classic_max"]),
        "-------d.ddd- smoothness", f5(see["classic_k_smooth"]),
        "=======d===== ION-MATERIAL INTERACTION MODEL (0 absorb, 1 reflect, 2 ion-induced electron emission)",
        f"       {1 if ion_reflection else (2 if iee else 0):1d}",
    ]
    if ion_reflection:
        iee = None
    if iee:
        yld, e0, e1, t = iee
        for s in range(1):   # one ion species (Ar+)
            mat += [
                f"------------- ION-INDUCED ELECTRON EMISSION, ION SPECIES {s + 1}",
                "-------d.ddd- coefficient", f"       {yld:5.3f}",
                "--dddddd.ddd- E_min [eV]", f"  {e0:10.3f}",
                "--dddddd.ddd- E_max [eV]", f"  {e1:10.3f}",
                "--dddddd.ddd- temperature of emitted electrons [eV]", f"  {t:10.3f}",
            ]
    w("init_material_METAL1.dat", mat)
    mat_rest = mat[2:]
    wp = wall_potentials or {}
    for k, (ty, _s) in enumerate(objs):
        if ty == 1:
            amp, mhz = (0.0, 0.0)
            if k == 1 and cfg.get("top_rf"):
                amp, mhz = cfg["top_rf"]
            wall = (2, 1, 3, 0)[k]   # objects: left, above, right, below
            bo(k + 1, wp.get(k + 1, 0.0), amp, mhz, (wall_injection or {}).get(wall, (0.0, 0, 0.0, 0.0, 0.0)))
    for q, obj in enumerate(inner_list):
        if len(obj) > 5:   # dielectric: its own material, whose first value is the permittivity
            mname = f"DIEL{q:02d}"
            w(f"init_material_{mname}.dat", ["------dd.ddd- dielectric constant", f"      {obj[5]:6.3f}"] + mat_rest)
            bo(len(objs) + q + 1, obj[4], material=mname)
        else:
            bo(len(objs) + q + 1, obj[4], inj=(wall_injection or {}).get(4 + q, (0.0, 0, 0.0, 0.0, 0.0)))
    for n, (amp_v, nu_hz, pts) in (waveforms or {}).items():
        w(f"init_bo_{n:02d}_waveform.dat", [f"  {amp_v}  potential amplitude [V]", f"  {nu_hz:.6e}   frequency [Hz]",
                                             "# time as a fraction of the period, value",
                                             "# (values are multiplied by the amplitude)"]
          + [f"  {a}   {b}" for a, b in pts])
    for n, pts in (amplitude_profiles or {}).items():
        w(f"init_bo_{n:02d}_amplitude_profile.dat", ["time [ns], amplitude factor"] + [f"  {a}   {b}" for a, b in pts])

    if not collisions:
        w("init_neutrals.dat", ["----------dd--- number of neutral species", f"          {0:2d}"])
        return directory
    t_gas_k = 0.03 * 1.602189e-19 / 1.38064852e-23
    w("init_neutrals.dat", [
        "----------dd--- number of neutral species", f"          {1:2d}",
        "------AAAAAA--- neutral gas code", "      Argon0",
        "--#d.dddE#dd--- density [m^-3]", f"  {n_gas:10.3E}",
        "-----ddddd.d--- temperature [K]", f"     {t_gas_k:7.1f}",
    ])
    e0, segs = _segments()
    nl = ["---ddd.ddd--- mass [amu]", f"   {39.948:7.3f}", "--------dd--- number of collisional processes",
          f"        {3:2d}"]
    for k, ty in enumerate((10, 20, 30)):
        nl += [f"---dd--d--dd--d- collision #{k + 1} :: type / activated / ion species / save",
               f"   {ty:2d}  {int(bool(en_collisions)):1d}  {(1 if ty == 30 else 0):2d}  {0:1d}"]
    nl += ["--------dd--- number of energy segments", f"        {len(segs):2d}",
           "--ddddd.ddd------------- minimal energy [eV]", f"  {e0:9.3f}"]
    for k, (up, st) in enumerate(segs):
        nl += [f"--ddddd.ddd---ddd.ddd--- segment {k + 1} :: upper boundary / resolution [eV]", f"  {up:9.3f}   {st:7.3f}"]
    w("init_neutral_Argon0.dat", nl)
    tables = {
        (1, 10): (np.logspace(-2, 3, 200), sigma_elastic),
        (2, 20): (np.logspace(math.log10(E_EXC_EV), 3, 200), lambda e: sigma_lotz(e, E_EXC_EV, 5.0e-20)),
        (3, 30): (np.logspace(math.log10(E_ION_EV), 3, 200), lambda e: sigma_lotz(e, E_ION_EV, 8.0e-20)),
    }
    for (pid, ty), (en, fn) in tables.items():
        rows = [f"  {len(en):4d}"] + [f"    {e:9.3f}  {float(fn(e)):10.3E}" for e in en]
        w(f"init_neutral_Argon0_crsect_coll_id_{pid:02d}_type_{ty:02d}.dat", rows)
    if rcx:
        w("init_neutral_Argon0_rcx_param.dat", ["ion species / sigma at 1 eV [m^2] / alpha", "1  5.0e-19  0.0"])
    return directory
