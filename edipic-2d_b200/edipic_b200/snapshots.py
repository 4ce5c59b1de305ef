"""CREATE_SNAPSHOT (pic2d_Snapshots.f90:303-1202) for a device Simulation, one cluster over the domain: the potential,
field, density, current, velocity, energy, temperature and heat-flux files `_NNNN_<name>_2D.bin` in the reference's
gnuplot binary layout (SAVE_GLOBAL_2D_ARRAY, :1207-1355), and the velocity distributions `_NNNN_vdf1d.bin` /
`_NNNN_vdf2d.bin` (SAVE_ALL_VDF1D/2D, :1359-1705). Moments and histograms come from the device (edp_collect_moments,
edp_calculate_vdf): no particle leaves the GPU. The unit conversions are the reference's, in REAL arithmetic.
"""
import ctypes as C
import os

import numpy as np

from . import library

E_CL = 1.602189e-19
M_E_KG = 9.109534e-31
AMU_KG = 1.660565e-27

# save_data(k) of init_snapshots.dat -> file name; "{s}" is the ion species digit
NAMES = {
    1: "F_V", 2: "EX_Vm", 3: "EY_Vm", 4: "JXsum_Am2", 5: "JYsum_Am2", 6: "JZsum_Am2",
    7: "Ne_m3", 8: "JXe_Am2", 9: "JYe_Am2", 10: "JZe_Am2", 11: "VXe_ms", 12: "VYe_ms", 13: "VZe_ms",
    14: "WXe_eV", 15: "WYe_eV", 16: "WZe_eV", 17: "TXe_eV", 18: "TYe_eV", 19: "TZe_eV",
    20: "QXe_Wm2", 21: "QYe_Wm2", 22: "QZe_Wm2",
    23: "Ni_{s}_m3", 24: "JXi_{s}_Am2", 25: "JYi_{s}_Am2", 26: "JZi_{s}_Am2", 27: "VXi_{s}_ms", 28: "VYi_{s}_ms",
    29: "VZi_{s}_ms", 30: "WXi_{s}_eV", 31: "WYi_{s}_eV", 32: "WZi_{s}_eV", 33: "TXi_{s}_eV", 34: "TYi_{s}_eV",
    35: "TZi_{s}_eV", 36: "QXi_{s}_Wm2", 37: "QYi_{s}_Wm2", 38: "QZi_{s}_Wm2",
}
N, VX, VY, VZ, WX, WY, WZ, VXVY, VXVZ, VYVZ, QX, QY, QZ = range(13)


def _f32(x):
    return np.float32(x)


def write_2d(path, arr, delta_x_m):
    """SAVE_GLOBAL_2D_ARRAY of one [ny, nx] node array."""
    a = np.ascontiguousarray(arr, dtype=np.float32)
    rc = library().edp_write_snapshot_2d(str(path).encode(), a.ctypes.data_as(C.POINTER(C.c_float)), a.shape[1],
                                           a.shape[0], delta_x_m)
    if rc != 0:
        raise OSError(f"edp_write_snapshot_2d({path}) = {rc}")


def read_2d(path):
    """The inverse of write_2d: (x [m], y [m], arr [ny, nx])."""
    raw = np.fromfile(path, dtype=np.float32)
    nx = int(raw[0])
    m = raw.reshape(-1, nx + 1)
    return m[0, 1:], m[1:, 0], m[1:, 1:]


def scales(sim):
    """The conversion factors of pic2d_CurProblemValues.f90:893-903."""
    p, d = sim.params, sim.deck
    n_scale = d.n_plasma_m3 / p.n_of_particles_cell
    v = p.v_scale_ms
    return dict(
        N_scale_part_m3=n_scale,
        current_factor_Am2=E_CL * v * n_scale,
        energy_factor_eV=0.5 * M_E_KG * v ** 2 / E_CL,
        temperature_factor_eV=M_E_KG * v ** 2 / E_CL,
        heat_flow_factor_Wm2=0.5 * M_E_KG * v ** 2 * n_scale,
    )


def _temperature(m, w, v, factor):
    out = np.maximum(_f32(0.0), m[w] - m[v] ** 2) * _f32(factor)
    out[m[N] <= 0] = 0.0   # nodes without particles, pic2d_Snapshots.f90:688-689
    return out


def create_snapshot(sim, current_snap, directory=".", save=tuple(range(1, 39)), vdf=None):
    """Writes the files of the save_data flags in `save` for snapshot number current_snap into directory and returns
    their paths. vdf = dict(nbox=(nx, ny), n_max_vel_e=.., n_vbins_e=.., n_max_vel_i=.., n_vbins_i=.., two_d=bool)
    also writes the velocity distributions."""
    from . import ELECTRONS, FIELD_EX, FIELD_EY, FIELD_PHI

    p = sim.params
    sc = scales(sim)
    dx = p.delta_x_m
    save = set(save)
    written = []

    def put(name, arr):
        path = os.path.join(directory, f"_{current_snap:04d}_{name}_2D.bin")
        write_2d(path, arr, dx)
        written.append(path)

    if 1 in save:
        put(NAMES[1], (sim.field(FIELD_PHI) * p.f_scale_v).astype(np.float32))
    if 2 in save:
        put(NAMES[2], (sim.field(FIELD_EX) * p.e_scale_vm).astype(np.float32))
    if 3 in save:
        put(NAMES[3], (sim.field(FIELD_EY) * p.e_scale_vm).astype(np.float32))
    jsum = {}
    if save & set(range(4, 23)):
        m = sim.collect_moments(ELECTRONS)
        # the electron part of the total current; the reference's z sum takes VY here (:571-577), kept as written
        for k, v in ((4, VX), (5, VY), (6, VY)):
            if k in save:
                jsum[k] = -m[N] * m[v]
        for k, v in ((7, None), (8, VX), (9, VY), (10, VZ)):
            if k in save:
                put(NAMES[k], m[N] * _f32(sc["N_scale_part_m3"]) if v is None
                    else -m[N] * m[v] * _f32(sc["current_factor_Am2"]))
        for k, v in ((11, VX), (12, VY), (13, VZ)):
            if k in save:
                put(NAMES[k], m[v] * _f32(p.v_scale_ms))
        for k, w in ((14, WX), (15, WY), (16, WZ)):
            if k in save:
                put(NAMES[k], m[w] * _f32(sc["energy_factor_eV"]))
        for k, w, v in ((17, WX, VX), (18, WY, VY), (19, WZ, VZ)):
            if k in save:
                put(NAMES[k], _temperature(m, w, v, sc["temperature_factor_eV"]))
        for k, q in ((20, QX), (21, QY), (22, QZ)):
            if k in save:
                put(NAMES[k], m[N] * m[q] * _f32(sc["heat_flow_factor_Wm2"]))
    for s in range(1, p.n_ion_species + 1):
        if not (save & ({4, 5, 6} | set(range(23, 39)))):
            break
        m = sim.collect_moments(s)
        qs, ms = p.ion_charge[s - 1], p.ion_mass_me[s - 1]
        for k, v in ((4, VX), (5, VY), (6, VZ)):
            if k in save:
                jsum[k] = jsum[k] + _f32(qs) * m[N] * m[v]
        name = lambda k: NAMES[k].format(s=s)
        if 23 in save:
            put(name(23), m[N] * _f32(sc["N_scale_part_m3"]))
        for k, v in ((24, VX), (25, VY), (26, VZ)):
            if k in save:
                put(name(k), m[N] * m[v] * _f32(qs * sc["current_factor_Am2"]))
        for k, v in ((27, VX), (28, VY), (29, VZ)):
            if k in save:
                put(name(k), m[v] * _f32(p.v_scale_ms))
        for k, w in ((30, WX), (31, WY), (32, WZ)):
            if k in save:
                put(name(k), m[w] * _f32(ms * sc["energy_factor_eV"]))
        for k, w, v in ((33, WX, VX), (34, WY, VY), (35, WZ, VZ)):
            if k in save:
                put(name(k), _temperature(m, w, v, ms * sc["temperature_factor_eV"]))
        for k, q in ((36, QX), (37, QY), (38, QZ)):
            if k in save:
                put(name(k), m[N] * m[q] * _f32(ms * sc["heat_flow_factor_Wm2"]))
    for k in (4, 5, 6):
        if k in jsum:
            put(NAMES[k], jsum[k] * _f32(sc["current_factor_Am2"]))
    if vdf:
        written += write_vdf(sim, current_snap, directory, **vdf)
    return written


def write_vdf(sim, current_snap, directory, nbox=(1, 1), n_max_vel_e=4, n_vbins_e=10, n_max_vel_i=4, n_vbins_i=10,
              two_d=False):
    """CALCULATE_ELECTRON_VDF / CALCULATE_ION_VDF on the device and SAVE_ALL_VDF1D (and SAVE_ALL_VDF2D)."""
    from . import ELECTRONS

    p, lib = sim.params, library()
    xarea = float(p.ncx + 1 if sim.periodic else p.ncx)
    e1, e2, _ = sim.calculate_vdf(ELECTRONS, nbox, n_max_vel_e, n_vbins_e, two_d)
    ions = [sim.calculate_vdf(s, nbox, n_max_vel_i, n_vbins_i)[0] for s in range(1, p.n_ion_species + 1)]
    i1 = np.ascontiguousarray(np.stack(ions) if ions else np.zeros((0,), np.int32), dtype=np.int32)
    amu = np.array([p.ion_mass_me[s] * M_E_KG / AMU_KG for s in range(p.n_ion_species)] or [0.0])
    i32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    out = [os.path.join(directory, f"_{current_snap:04d}_vdf1d.bin")]
    rc = lib.edp_write_vdf1d(out[0].encode(), nbox[0], nbox[1], xarea, float(p.ncy), p.delta_x_m, n_max_vel_e,
                             n_vbins_e, n_max_vel_i, n_vbins_i, p.n_ion_species, sim.deck.t_e_ev,
                             amu.ctypes.data_as(C.POINTER(C.c_double)), i32(np.ascontiguousarray(e1)), i32(i1))
    if rc != 0:
        raise OSError(f"edp_write_vdf1d = {rc}")
    if two_d:
        out.append(os.path.join(directory, f"_{current_snap:04d}_vdf2d.bin"))
        rc = lib.edp_write_vdf2d(out[1].encode(), nbox[0], nbox[1], xarea, float(p.ncy), p.delta_x_m, n_max_vel_e,
                                 n_vbins_e, sim.deck.t_e_ev, i32(np.ascontiguousarray(e2)))
        if rc != 0:
            raise OSError(f"edp_write_vdf2d = {rc}")
    return out
