"""ORACLE (test infrastructure only): ctypes front end of liboracle.so, the CPU FP64 restatement of
EDIPIC-2D's particle cycle (oracle.cpp, oracle_rng.c), plus a reader of the neutral-gas decks that follows
INITIATE_ELECTRON_NEUTRAL_COLLISIONS (pic2d_enCollisionsGeneralProc.f90:63-200) independently of the product's
deck reader. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module.
"""
import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_WELL = os.path.join(HERE, "_ref", "libwell_ref.so")

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_U32 = C.POINTER(C.c_uint32)
_I64 = C.POINTER(C.c_int64)


class Well(C.Structure):
    _fields_ = [("v", C.c_uint32 * 624), ("i", C.c_int)]


class Geom(C.Structure):
    _fields_ = [("ncx", C.c_int32), ("ncy", C.c_int32), ("periodic", C.c_int32), ("n_inner", C.c_int32),
                ("ileft", C.c_int32 * 4), ("jbottom", C.c_int32 * 4), ("iright", C.c_int32 * 4),
                ("jtop", C.c_int32 * 4)]


class Species(C.Structure):
    _fields_ = [("bx", C.c_double), ("by", C.c_double), ("bz", C.c_double), ("ez", C.c_double),
                ("is_ion", C.c_int32), ("qm2", C.c_double), ("nsub", C.c_int32), ("ions_sense_b", C.c_int32),
                ("ions_sense_ez", C.c_int32)]


class Parts(C.Structure):
    _fields_ = [("n", C.c_int64), ("x", _D), ("y", _D), ("vx", _D), ("vy", _D), ("vz", _D), ("tag", _I32),
                ("id", _U32)]


class Crsect(C.Structure):
    _fields_ = [("n_points", C.c_int32), ("energy_eV", _D), ("crsect_m2", _D), ("type", C.c_int32)]


class MccTable(C.Structure):
    _fields_ = [("n_act", C.c_int32), ("n_seg", C.c_int32), ("n_values", C.c_int32),
                ("seg_value", C.c_double * 33), ("seg_step", C.c_double * 32), ("seg_index", C.c_int32 * 33),
                ("energy_eV", _D), ("prob", _D), ("max_colliding_fraction", C.c_double), ("type", C.c_int32 * 8),
                ("threshold_eV", C.c_double * 8)]


class MccCtx(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("step", C.c_uint32), ("energy_factor_eV", C.c_double),
                ("neutral_mass_amu", C.c_double), ("ion_velocity_factor", C.c_double), ("maxwell_v", _D)]


class Rcx(C.Structure):
    _fields_ = [("prob_factor", C.c_double), ("v_scale_ms", C.c_double), ("factor_eV", C.c_double),
                ("sigma_1eV", C.c_double), ("alpha", C.c_double), ("probab_thermal", C.c_double),
                ("vfactor", C.c_double)]


class Cycle(C.Structure):
    _fields_ = [("geom", Geom), ("e_sp", Species), ("i_sp", Species), ("factor_rho", C.c_double),
                ("ion_charge", C.c_double), ("factor2_E", C.c_double), ("factor1_E", C.c_double),
                ("phi_bottom", C.c_double), ("phi_top", C.c_double), ("mcc", C.POINTER(MccTable)),
                ("mcc_ctx", MccCtx), ("rcx", Rcx), ("rcx_on", C.c_int32), ("nthreads", C.c_int32),
                ("born_e", Parts), ("born_i", Parts), ("cap_born", C.c_int64),
                ("next_id_e", C.c_uint32), ("next_id_i", C.c_uint32), ("n_sub_phase", C.c_int32)]


_lib = None


class Emit(C.Structure):
    _fields_ = [("on", C.c_int32 * 8), ("yld", C.c_double * 8), ("emin", C.c_double * 8),
                ("emax", C.c_double * 8), ("fconv", C.c_double * 8), ("ms", C.c_double), ("species", C.c_uint32),
                ("maxwell_v", _D), ("maxwell_inj", _D)]


class See(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("m_el", "m_in", "m_tr", "refl_random")] + \
        [(n, C.c_double) for n in ("el_yield", "el_emin", "el_emax", "el_e0", "el_emaxc", "el_max", "el_de", "el_frac",
                                   "in_yield", "in_emin", "in_emax", "in_frac", "tr_yield", "tr_emin", "tr_emax",
                                   "cl_e0", "cl_emax", "cl_max", "cl_k", "lowest", "fconv")] + \
        [("maxwell_v", _D), ("maxwell_inj", _D)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise OSError(f"{LIB} missing: run make -C oracle")
        L = C.CDLL(LIB)
        sig = {
            "oracle_well_seed": ([C.POINTER(Well), C.c_int32], None),
            "oracle_well_next": ([C.POINTER(Well)], C.c_double),
            "oracle_philox4x32_10": ([_U32, _U32, _U32], None),
            "oracle_mix64": ([C.c_uint64], C.c_uint64),
            "oracle_splitmix64_at": ([C.c_uint64, C.c_uint64], C.c_uint64),
            "oracle_splitmix64_stream": ([C.c_uint64, C.c_int64, C.POINTER(C.c_uint64)], None),
            "oracle_nx_nodes": ([C.POINTER(Geom)], C.c_int32),
            "oracle_push": ([C.POINTER(Geom), C.POINTER(Species), _D, _D, C.POINTER(Parts), _I64], None),
            "oracle_push_hits": ([C.POINTER(Geom), C.POINTER(Species), _D, _D, C.POINTER(Parts), _I64, _D,
                                  C.c_int64, _I64], None),
            "oracle_ion_emission": ([C.POINTER(Emit), C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_uint32, C.c_uint64, C.c_uint32, C.c_double, C.c_double, _D,
                                     C.c_int32], C.c_int32),
            "oracle_vdf": ([C.POINTER(Parts), C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32,
                            _I32, _I32], C.c_int64),
            "oracle_see": ([C.POINTER(See), C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                            C.c_uint32, C.c_uint64, C.c_uint32, C.c_double, C.c_double, _D, C.c_int32], C.c_int32),
            "oracle_wall_injection": ([C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32,
                                       C.c_uint32, C.c_uint64, C.c_double, C.c_double, _D, _D, _D, C.c_int32],
                                      C.c_int32),
            "oracle_inner_injection": ([C.POINTER(Geom), C.c_int32, C.c_double, C.c_int32, C.c_double, C.c_double,
                                        C.c_double, C.c_uint32, C.c_uint64, _D, _D, _D, C.c_int32, _I32], C.c_int32),
            "oracle_cg_solve_eps": ([C.POINTER(Geom), _D, _D, _D, _D, C.c_double, C.c_int32, _D, _D], C.c_int32),
            "oracle_inner_hit": ([C.POINTER(Geom), _D, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                  C.c_double, _D], C.c_int32),
            "oracle_ion_reflect": ([C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, _D], None),
            "oracle_ion_emission_face": ([C.POINTER(Emit), C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_double, C.c_uint32, C.c_uint64, C.c_uint32, _D,
                                          C.c_int32], C.c_int32),
            "oracle_see_face": ([C.POINTER(See), C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_uint32, C.c_uint64, C.c_uint32, _D, C.c_int32], C.c_int32),
            "oracle_inner_cross": ([C.POINTER(Geom), C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                    _I32, _D, _D], C.c_int32),
            "oracle_inner_charge": ([C.POINTER(Geom), C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, _D],
                                    None),
            "oracle_deposit": ([C.POINTER(Geom), C.POINTER(Parts), C.c_double, _D], None),
            "oracle_fold_and_wall_scale": ([C.POINTER(Geom), _D], None),
            "oracle_collect_moments": ([C.POINTER(Geom), C.POINTER(Species), _D, _D, C.POINTER(Parts), _D], None),
            "oracle_maxwell_tables": ([_D, _D], None),
            "oracle_maxwell_sample": ([_D, C.c_double], C.c_double),
            "oracle_en_frequency": ([C.POINTER(Crsect), C.c_double, C.c_double, C.c_int32, C.c_double], C.c_double),
            "oracle_mcc_n_values": ([C.c_int32, _D, _D], C.c_int32),
            "oracle_mcc_build": ([C.POINTER(MccTable), C.c_int32, C.POINTER(Crsect), C.c_double, C.c_int32,
                                  C.c_double], None),
            "oracle_mcc_choose": ([C.POINTER(MccTable), C.c_double, C.c_double], C.c_int32),
            "oracle_mcc_philox": ([C.POINTER(MccTable), C.POINTER(MccCtx), C.POINTER(Parts), C.POINTER(Parts),
                                   C.POINTER(Parts), C.c_int64, _I64], None),
            "oracle_rcx_probab_thermal": ([C.c_double] * 6 + [C.c_int32], C.c_double),
            "oracle_rcx_philox": ([C.POINTER(Rcx), C.POINTER(MccCtx), C.c_uint32, C.POINTER(Parts)], C.c_int64),
            "oracle_fftx_solve": ([C.POINTER(Geom), _D, C.c_double, C.c_double, _D], None),
            "oracle_efield": ([C.POINTER(Geom), _D, C.c_double, C.c_double, _D, _D, _D, _D], None),
            "oracle_cg_solve": ([C.POINTER(Geom), _D, _D, _D, C.c_double, C.c_int32, _D, _D], C.c_int32),
            "oracle_cycle_step": ([C.POINTER(Cycle), C.POINTER(Parts), C.POINTER(Parts), C.c_int64, C.c_int64, _D,
                                   _I64], C.c_int64),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def dp(a):
    return a.ctypes.data_as(_D)


# ------------------------------------------------------------------------------------------ RNG
def well_stream(seed, n):
    s = Well()
    lib().oracle_well_seed(C.byref(s), seed)
    return np.array([lib().oracle_well_next(C.byref(s)) for _ in range(n)])


def philox(ctr, key):
    out = (C.c_uint32 * 4)()
    lib().oracle_philox4x32_10((C.c_uint32 * 4)(*ctr), (C.c_uint32 * 2)(*key), out)
    return tuple(out)


def splitmix64_stream(seed, count):
    """The first `count` outputs of SplitMix64 seeded with `seed`, stepped one state at a time."""
    out = (C.c_uint64 * count)()
    lib().oracle_splitmix64_stream(seed, count, out)
    return list(out)


def splitmix64_at(seed, n):
    """Output n (n >= 1) of SplitMix64 seeded with `seed`, evaluated directly at its position."""
    return lib().oracle_splitmix64_at(seed, n)


def decision_draw(seed, tag, step, pid):
    """The collision decision draw (word 0, word 1) of particle `pid` at `step` in stream `tag`."""
    z = splitmix64_at(lib().oracle_mix64(seed ^ tag), (step << 32) | pid)
    return (z >> 32, z & 0xFFFFFFFF)


def maxwell_tables():
    v = np.zeros(9001)
    vi = np.zeros(4501)
    lib().oracle_maxwell_tables(dp(v), dp(vi))
    return v, vi


# ------------------------------------------------------------------------------------- particles
class ParticleSet:
    """SoA FP64 particle columns with spare capacity, wrapped in the oracle's Parts struct."""

    def __init__(self, x, y, vx, vy, vz, ids=None, cap=None):
        n = len(x)
        cap = cap or n
        self.cols = {k: np.zeros(cap) for k in ("x", "y", "vx", "vy", "vz")}
        for k, v in zip(("x", "y", "vx", "vy", "vz"), (x, y, vx, vy, vz)):
            self.cols[k][:n] = v
        self.tag = np.zeros(cap, dtype=np.int32)
        self.id = np.zeros(cap, dtype=np.uint32)
        self.id[:n] = np.arange(n, dtype=np.uint32) if ids is None else ids
        self.s = Parts(n, *[dp(self.cols[k]) for k in ("x", "y", "vx", "vy", "vz")],
                       self.tag.ctypes.data_as(_I32), self.id.ctypes.data_as(_U32))

    @property
    def n(self):
        return self.s.n

    def arrays(self):
        n = self.s.n
        d = {k: v[:n].copy() for k, v in self.cols.items()}
        d["id"] = self.id[:n].copy()
        return d


def geom(ncx, ncy, periodic, inner=()):
    g = Geom(ncx, ncy, 1 if periodic else 0, len(inner))
    for k, (il, jb, ir, jt) in enumerate(inner):
        g.ileft[k], g.jbottom[k], g.iright[k], g.jtop[k] = il, jb, ir, jt
    return g


def nodes_shape(g):
    return (g.ncy + 1, lib().oracle_nx_nodes(C.byref(g)))


def push(g, sp, ex, ey, parts):
    hits = np.zeros(8, dtype=np.int64)
    lib().oracle_push(C.byref(g), C.byref(sp), dp(np.ascontiguousarray(ex)), dp(np.ascontiguousarray(ey)),
                      C.byref(parts.s), hits.ctypes.data_as(_I64))
    return hits


def push_hits(g, sp, ex, ey, parts, cap=1 << 20):
    """oracle_push plus the wall-hit rows {wall, X, Y, vx, vy, vz, id} of every domain-wall absorption."""
    hits = np.zeros(8, dtype=np.int64)
    rows = np.zeros((cap, 7))
    n = C.c_int64(0)
    lib().oracle_push_hits(C.byref(g), C.byref(sp), dp(np.ascontiguousarray(ex)), dp(np.ascontiguousarray(ey)),
                           C.byref(parts.s), hits.ctypes.data_as(_I64), dp(rows), cap, C.byref(n))
    assert n.value <= cap
    return hits, rows[:n.value].copy()


class IonEmission:
    """Ion-induced electron emission of one ion species at the four walls (oracle_ion_emission). Energies in eV are
    converted with energy_factor_ev (0.5 m_e V_scale^2 / e); t_emit in eV the same way."""

    def __init__(self, walls, ms, energy_factor_ev, species=0):
        self.v, self.vi = maxwell_tables()
        self.s = Emit()
        for w, (yld, e0, e1, t) in walls.items():
            self.s.on[w] = 1 if yld > 0 else 0
            self.s.yld[w] = yld
            self.s.emin[w] = e0 / energy_factor_ev
            self.s.emax[w] = e1 / energy_factor_ev
            self.s.fconv[w] = np.sqrt(t / energy_factor_ev)
        self.s.ms = ms
        self.s.species = species
        self.s.maxwell_v = dp(self.v)
        self.s.maxwell_inj = dp(self.vi)

    def emit(self, wall, x, y, vx, vy, vz, ident, seed, step, xmax, ymax, cap=64):
        out = np.zeros((cap, 5))
        n = lib().oracle_ion_emission(C.byref(self.s), int(wall), x, y, vx, vy, vz, int(ident), seed, step, xmax,
                                      ymax, dp(out), cap)
        assert n <= cap
        return out[:n]

    def emit_face(self, obj, dirflag, at, x, y, vx, vy, vz, ident, seed, step, cap=64):
        out = np.zeros((cap, 5))
        n = lib().oracle_ion_emission_face(C.byref(self.s), int(obj), int(dirflag), at, x, y, vx, vy, vz, int(ident),
                                           seed, step, dp(out), cap)
        assert n <= cap
        return out[:n]


# the sides of an inner object (segments 1 left, 2 top, 3 right, 4 bottom) as INJECT_* dirflags and their coordinate
def inner_face(g, n, m):
    return {1: (3, g.ileft[n]), 2: (4, g.jtop[n]), 3: (1, g.iright[n]), 4: (2, g.jbottom[n])}[m]


def inner_cross(g, x, y, vx, vy, xmul):
    """(object or -1, segment, x, y) of the trajectory's first crossing of an inner object's outline"""
    m, xc, yc = C.c_int32(), C.c_double(), C.c_double()
    n = lib().oracle_inner_cross(C.byref(g), x, y, vx, vy, xmul, C.byref(m), C.byref(xc), C.byref(yc))
    return n, m.value, xc.value, yc.value


def inner_charge(g, n, m, xc, yc, q, surf):
    lib().oracle_inner_charge(C.byref(g), int(n), int(m), xc, yc, q, dp(surf))


def inner_electron_impact(g, see, dielectric, row, seed, step, surf):
    """DO_ELECTRON_COLL_WITH_INNER_OBJECT (pic2d_ElectronWallCollisions.f90:561-645) for one absorbed electron (a
    push_hits row of object 4 + n): the electrons the object's material emits from the side crossed first
    (ElectronEmission by object in `see`), with a dielectric's outline taking -1 and +1 per emitted electron."""
    _obj, x, y, vx, vy, vz, ident = row
    n, m, xc, yc = inner_cross(g, x, y, vx, vy, 1.0)
    if n < 0:
        return np.zeros((0, 5))
    if dielectric.get(n):
        inner_charge(g, n, m, xc, yc, -1.0, surf)
    if 4 + n not in see:
        return np.zeros((0, 5))
    dirflag, at = inner_face(g, n, m)
    out, k = see[4 + n].emit_face(dirflag, at, xc, yc, vx, vy, vz, int(ident), seed, step)
    if dielectric.get(n) and k > 0:
        inner_charge(g, n, m, xc, yc, float(k), surf)
    return out


def inner_ion_impact(g, em, reflect, dielectric, q, row, seed, step, xmul, surf):
    """DO_ION_COLL_WITH_INNER_OBJECT (pic2d_IonWallCollisions.f90:484-575) for one absorbed ion (a push_hits row of
    object 4 + n): (emitted electrons, reflected ion row or None). A reflecting object returns the ion 1e-6 outside
    the side crossed first, its normal velocity reversed (INJECT_REFLECTED_ION, pic2d_IonEmissions.f90:374-492); a
    dielectric takes the charge q, and +1 per emitted electron, at the crossing (surf updated)."""
    _obj, x, y, vx, vy, vz, ident = row
    n, m, xc, yc = inner_cross(g, x, y, vx, vy, xmul)
    if n < 0:
        return np.zeros((0, 5)), None
    dirflag, at = inner_face(g, n, m)
    if reflect.get(4 + n):
        nx, ny, v = xc, yc, [vx, vy, vz]
        if dirflag == 1:
            nx, v[0] = at + 1e-6, -vx
        elif dirflag == 3:
            nx, v[0] = at - 1e-6, -vx
        elif dirflag == 4:
            ny, v[1] = at + 1e-6, -vy
        else:
            ny, v[1] = at - 1e-6, -vy
        return np.zeros((0, 5)), np.array([nx, ny] + v)
    if dielectric.get(n):
        inner_charge(g, n, m, xc, yc, q, surf)
    out = em.emit_face(4 + n, dirflag, at, xc, yc, vx, vy, vz, int(ident), seed, step)
    if dielectric.get(n) and len(out):
        inner_charge(g, n, m, xc, yc, float(len(out)), surf)
    return out, None


def vdf(parts, nbox, xmax, ymax, fvc, n_max_vel_s, n_vbins, two_d=False):
    """oracle_vdf: (h1 [3, nbox, reclen], h2 [nbox, reclen, reclen] or None, skipped)."""
    nb = nbox[0] * nbox[1]
    vmin = -n_max_vel_s * n_vbins
    rl = -2 * vmin
    h1 = np.zeros((3, nb, rl), dtype=np.int32)
    h2 = np.zeros((nb, rl, rl), dtype=np.int32) if two_d else None
    i32 = lambda a: a.ctypes.data_as(_I32) if a is not None else None
    sk = lib().oracle_vdf(C.byref(parts.s), nbox[0], nbox[1], xmax, ymax, fvc, vmin, i32(h1), i32(h2))
    return h1, h2, sk


class ElectronEmission:
    """Electron-induced emission of one wall (oracle_see) from a dict of the material-file parameters in eV (the
    fields of edp_see_params), converted to code units as PREPARE_WALL_MATERIALS does (pic2d_Materials.f90:195-244)
    with energy_factor_ev."""

    def __init__(self, prm, energy_factor_ev):
        ef = energy_factor_ev
        self.v, self.vi = maxwell_tables()
        s = See()
        s.m_el, s.m_in, s.m_tr = prm["elastic_model"], prm["inelastic_model"], prm["true_model"]
        s.refl_random = 1 if prm["elastic_type"] else 0
        s.el_yield, s.el_emin, s.el_emax = prm["elastic_yield"], prm["elastic_emin_ev"] / ef, prm["elastic_emax_ev"] / ef
        s.el_e0, s.el_emaxc = prm["elastic_e0_ev"] / ef, prm["elastic_emax_coef_ev"] / ef
        s.el_max, s.el_de, s.el_frac = prm["elastic_max"], prm["elastic_de_ev"] / ef, prm["elastic_frac_classic"]
        s.in_yield, s.in_emin = prm["inelastic_yield"], prm["inelastic_emin_ev"] / ef
        s.in_emax, s.in_frac = prm["inelastic_emax_ev"] / ef, prm["inelastic_frac_classic"]
        s.tr_yield, s.tr_emin, s.tr_emax = prm["true_yield"], prm["true_emin_ev"] / ef, prm["true_emax_ev"] / ef
        s.cl_e0, s.cl_emax = prm["classic_e0_ev"] / ef, prm["classic_emax_ev"] / ef
        s.cl_max, s.cl_k = prm["classic_max"], prm["classic_k_smooth"]
        s.fconv = np.sqrt(prm["true_t_ev"] / ef)
        lo = 1.0e6 / ef
        lo = min(lo, {1: s.el_emin, 2: s.el_e0}.get(s.m_el, lo))
        lo = min(lo, {1: s.in_emin, 2: s.cl_e0}.get(s.m_in, lo))
        lo = min(lo, {1: s.tr_emin, 2: s.cl_e0}.get(s.m_tr, lo))
        s.lowest = lo
        s.maxwell_v, s.maxwell_inj = dp(self.v), dp(self.vi)
        self.s = s

    def emit(self, wall, x, y, vx, vy, vz, ident, seed, step, xmax, ymax, cap=64):
        out = np.zeros((cap, 5))
        n = lib().oracle_see(C.byref(self.s), int(wall), x, y, vx, vy, vz, int(ident), seed, step, xmax, ymax,
                             dp(out), cap)
        assert n <= cap
        return out[:max(n, 0)], n

    def emit_face(self, dirflag, at, x, y, vx, vy, vz, ident, seed, step, cap=64):
        out = np.zeros((cap, 5))
        n = lib().oracle_see_face(C.byref(self.s), int(dirflag), at, x, y, vx, vy, vz, int(ident), seed, step,
                                  dp(out), cap)
        assert n <= cap
        return out[:max(n, 0)], n


def wall_injection(wall, n, model, t_normal_ev, t_parallel_ev, beam_ev, energy_factor_ev, step, seed, xmax, ymax):
    """oracle_wall_injection with the temperatures converted as PREPARE_SETUP_VALUES does (pic2d_Setup.f90:103-126):
    rows {x, y, vx, vy, vz}."""
    ef = energy_factor_ev
    fp = np.sqrt(t_parallel_ev / ef)
    if model == 0:
        fn, vb = np.sqrt(t_normal_ev / ef), 0.0
    else:
        fn, vb = np.sqrt(0.25 * t_normal_ev ** 2 / (beam_ev * ef)), np.sqrt(beam_ev / ef)
    v, vi = maxwell_tables()
    cap = int(n) + 2
    out = np.zeros((cap, 5))
    m = lib().oracle_wall_injection(n, model, fn, fp, vb, wall, step, seed, xmax, ymax, dp(v), dp(vi), dp(out), cap)
    return out[:m]


def inner_injection(g, n, n_per_step, model, t_normal_ev, t_parallel_ev, beam_ev, energy_factor_ev, step, seed):
    """oracle_inner_injection for metal inner object n with the temperatures converted as for the walls: (rows
    {x, y, vx, vy, vz}, counts of sides 1 left, 2 top, 3 right, 4 bottom)."""
    ef = energy_factor_ev
    fp = np.sqrt(t_parallel_ev / ef)
    if model == 0:
        fn, vb = np.sqrt(t_normal_ev / ef), 0.0
    else:
        fn, vb = np.sqrt(0.25 * t_normal_ev ** 2 / (beam_ev * ef)), np.sqrt(beam_ev / ef)
    v, vi = maxwell_tables()
    cap = 4 * int(n_per_step) + 8
    out = np.zeros((cap, 5))
    per = np.zeros(4, dtype=np.int32)
    m = lib().oracle_inner_injection(C.byref(g), n, n_per_step, model, fn, fp, vb, step, seed, dp(v), dp(vi),
                                     dp(out), cap, per.ctypes.data_as(_I32))
    assert m <= cap
    return out[:m], per


def ion_reflect(wall, x, y, vx, vy, vz, xmax, ymax):
    out = np.zeros(5)
    lib().oracle_ion_reflect(int(wall), x, y, vx, vy, vz, xmax, ymax, dp(out))
    return out


def deposit(g, parts, weight=1.0, fold=True):
    rho = np.zeros(nodes_shape(g))
    lib().oracle_deposit(C.byref(g), C.byref(parts.s), weight, dp(rho))
    if fold:
        lib().oracle_fold_and_wall_scale(C.byref(g), dp(rho))
    return rho


def collect_moments(g, sp, ex, ey, parts):
    """COLLECT_ELECTRON_MOMENTS / COLLECT_ION_MOMENTS: [13, ny, nx] (N, VX, VY, VZ, WX, WY, WZ, VXVY, VXVZ, VYVZ,
    QX, QY, QZ)."""
    ny, nx = nodes_shape(g)
    out = np.zeros((13, ny, nx))
    ex = np.ascontiguousarray(ex if ex is not None else np.zeros((ny, nx)))
    ey = np.ascontiguousarray(ey if ey is not None else np.zeros((ny, nx)))
    lib().oracle_collect_moments(C.byref(g), C.byref(sp), dp(ex), dp(ey), C.byref(parts.s), dp(out))
    return out


def fftx_solve(g, rho_total, phi_bottom=0.0, phi_top=0.0):
    phi = np.zeros(nodes_shape(g))
    lib().oracle_fftx_solve(C.byref(g), dp(np.ascontiguousarray(rho_total)), phi_bottom, phi_top, dp(phi))
    return phi


def efield(g, phi, f2, f1):
    ex = np.zeros(nodes_shape(g))
    ey = np.zeros(nodes_shape(g))
    lib().oracle_efield(C.byref(g), dp(np.ascontiguousarray(phi)), f2, f1, dp(ex), dp(ey), None, None)
    return ex, ey


def cg_solve(g, rho_total, wall_phi, inner_phi, rtol=1e-12, max_it=100000, phi0=None):
    phi = np.zeros(nodes_shape(g)) if phi0 is None else np.array(phi0, dtype=np.float64)
    rel = C.c_double()
    it = lib().oracle_cg_solve(C.byref(g), dp(np.ascontiguousarray(rho_total)),
                               dp(np.asarray(wall_phi, dtype=np.float64)),
                               dp(np.asarray(list(inner_phi) + [0.0] * 4, dtype=np.float64)), rtol, max_it, dp(phi),
                               C.byref(rel))
    return phi, it, rel.value


def cg_solve_eps(g, rho_total, wall_phi, inner_phi, inner_eps, rtol=1e-12, max_it=100000, phi0=None):
    """oracle_cg_solve_eps: the CG solve with dielectric inner objects (inner_eps[n] > 0)."""
    phi = np.zeros(nodes_shape(g)) if phi0 is None else np.array(phi0, dtype=np.float64)
    rel = C.c_double()
    pad = lambda v: dp(np.asarray(list(v) + [0.0] * (4 - len(v)), dtype=np.float64))
    it = lib().oracle_cg_solve_eps(C.byref(g), dp(np.ascontiguousarray(rho_total)),
                                   dp(np.asarray(wall_phi, dtype=np.float64)), pad(inner_phi), pad(inner_eps), rtol,
                                   max_it, dp(phi), C.byref(rel))
    return phi, it, rel.value


def inner_hit(g, inner_eps, x, y, vx, vy, xmul, q, surf):
    """oracle_inner_hit: adds the outline charge of one absorbed particle to surf (node grid); returns the object."""
    e = np.asarray(list(inner_eps) + [0.0] * (4 - len(inner_eps)), dtype=np.float64)
    return lib().oracle_inner_hit(C.byref(g), dp(e), x, y, vx, vy, xmul, q, dp(surf))


# ------------------------------------------------------------------------------ collision tables
def _field(line, skip, width):
    return line[skip:skip + width].strip()


def read_neutral_deck(directory):
    """init_neutrals.dat, init_neutral_<NAME>.dat and the cross-section files, as the reference reads them."""
    rd = lambda fn: open(os.path.join(directory, fn)).read().splitlines()
    nl = rd("init_neutrals.dat")
    name = nl[3][6:12]
    n_m3 = float(_field(nl[5], 2, 10))
    t_k = float(_field(nl[7], 5, 7))
    dl = rd(f"init_neutral_{name}.dat")
    mass = float(_field(dl[1], 3, 7))
    ncp = int(_field(dl[3], 8, 2))
    procs = []
    pos = 4
    for q in range(ncp):
        ln = dl[pos + 1]
        procs.append(dict(type=int(_field(ln, 3, 2)), act=int(_field(ln, 7, 1) or 0), isp=int(_field(ln, 10, 2) or 0)))
        pos += 2
    nseg = int(_field(dl[pos + 1], 8, 2))
    pos += 2
    seg_value = [float(_field(dl[pos + 1], 2, 9))]
    pos += 2
    seg_step = []
    for _ in range(nseg):
        ln = dl[pos + 1]
        seg_value.append(float(_field(ln, 2, 9)))
        seg_step.append(float(_field(ln, 14, 7)))
        pos += 2
    cs = []
    for q, pr in enumerate(procs):
        if not pr["act"]:
            continue
        xl = rd(f"init_neutral_{name}_crsect_coll_id_{q + 1:02d}_type_{pr['type']:02d}.dat")
        npt = int(_field(xl[0], 2, 4))
        e = np.array([float(_field(xl[1 + k], 4, 9)) for k in range(npt)])
        s = np.array([float(_field(xl[1 + k], 15, 10)) for k in range(npt)])
        cs.append(dict(type=pr["type"], e=e, s=s, isp=pr["isp"]))
    return dict(name=name, n_m3=n_m3, t_k=t_k, mass=mass, seg_value=seg_value, seg_step=seg_step, cs=cs)


class MccTables:
    """INITIATE_ELECTRON_NEUTRAL_COLLISIONS table built by the oracle; keeps its arrays alive."""

    def __init__(self, neutral, nsub, dt_s):
        self.keep = []
        crs = (Crsect * len(neutral["cs"]))()
        for k, c in enumerate(neutral["cs"]):
            e = np.ascontiguousarray(c["e"])
            s = np.ascontiguousarray(c["s"])
            self.keep += [e, s]
            crs[k] = Crsect(len(e), dp(e), dp(s), c["type"])
        self.crs = crs
        t = MccTable()
        t.n_seg = len(neutral["seg_step"])
        for i, v in enumerate(neutral["seg_value"]):
            t.seg_value[i] = v
        for i, v in enumerate(neutral["seg_step"]):
            t.seg_step[i] = v
        nv = lib().oracle_mcc_n_values(t.n_seg, t.seg_value, t.seg_step)
        self.energy = np.zeros(nv + 1)
        self.prob = np.zeros((nv + 1) * len(neutral["cs"]))
        t.energy_eV = dp(self.energy)
        t.prob = dp(self.prob)
        lib().oracle_mcc_build(C.byref(t), len(neutral["cs"]), crs, neutral["n_m3"], nsub, dt_s)
        self.t = t

    def choose(self, energy_ev, r):
        return np.array([lib().oracle_mcc_choose(C.byref(self.t), float(e), float(q)) for e, q in zip(energy_ev, r)],
                        dtype=np.int32)


# ------------------------------------------------------------------------------------ deck reading
# The oracle reads the init_*.dat decks itself, with the edit descriptors of the reference's READ statements, and
# derives the normalisation and collision constants with the reference's formulas; nothing here comes from the
# product's deck reader. Physical constants of pic2d_Modules.f90:161-168.
E_CL, M_E_KG, EPS0_FM, AMU_KG, KB_JK, PI = 1.602189e-19, 9.109534e-31, 8.854188e-12, 1.660565e-27, 1.38064852e-23, \
    3.141592653589793


def fortran_field(line, skip, width, kind, decimals=0):
    """One fixed-width field of a formatted Fortran READ: columns [skip, skip+width); blanks are ignored, an empty
    field reads as zero, and a real field written without a decimal point carries `decimals` implied digits."""
    f = line[skip:skip + width].replace(" ", "").replace("\t", "")
    if kind == "i":
        return int(f) if f else 0
    if not f:
        return 0.0
    f = f.replace("d", "e").replace("D", "e")
    mant = f.split("e")[0].split("E")[0]
    v = float(f)
    if "." not in mant and decimals:
        v /= 10.0 ** decimals
    return v


class _Lines:
    def __init__(self, path):
        self.v = [ln.rstrip("\r") for ln in open(path).read().splitlines()]
        self.k = 0

    def next(self):
        self.k += 1
        return self.v[self.k - 1]

    def value(self, skip, width, kind, decimals=0):
        """a header line, then the value line (the deck layout of READ (9,'(A1)') buf; READ (9, fmt) value)"""
        self.next()
        return fortran_field(self.next(), skip, width, kind, decimals)


def read_deck(directory):
    """INITIATE_PARAMETERS (pic2d_CurProblemValues.f90), PREPARE_EXTERNAL_FIELDS (pic2d_ExternalFields.f90:36-145),
    the boundary-object files of PREPARE_SETUP_VALUES (pic2d_Setup.f90:60-100), SET_ION_SPECIES (:1505-1507) and
    the ion-neutral set-up (pic2d_inCollisionsGeneralProc.f90:3-90, pic2d_inCollisionsSpecificProc.f90:4-44) for
    the deck subset the oracle's cycle covers: one cluster, metal or periodic boundary objects, rectangular inner
    objects, uniform external fields, one neutral species. Returns a dict of module values."""
    path = lambda fn: os.path.join(directory, fn)
    d = {}
    # SET_PHYSICAL_CONSTANTS (:3-55): eps_0 from init_physconstants.dat when it holds a positive value
    eps0 = EPS0_FM
    if os.path.exists(path("init_physconstants.dat")):
        try:
            v = float(open(path("init_physconstants.dat")).read().splitlines()[1].split()[0].replace("d", "e"))
            if v > 0.0:
                eps0 = v
        except (IndexError, ValueError):
            pass
    d["eps_0_Fm"] = eps0
    # init_configuration.dat (:157-330)
    cf = _Lines(path("init_configuration.dat"))
    T_e_eV = cf.value(3, 12, "f", 7)
    N_plasma_m3 = cf.value(3, 14, "e", 7)
    N_of_cells_debye = cf.value(3, 3, "i")
    N_max_vel = cf.value(3, 3, "i")
    N_blocks_x = cf.value(3, 3, "i")
    N_blocks_y = cf.value(3, 3, "i")
    N_grid_block_x = cf.value(3, 3, "i")
    N_grid_block_y = cf.value(3, 3, "i")
    N_of_particles_cell = cf.value(2, 4, "i")
    cf.value(5, 1, "i")
    cf.value(5, 1, "i")
    cf.next()
    ln = cf.next()
    n_bo, n_io = fortran_field(ln, 3, 3, "i"), fortran_field(ln, 9, 3, "i")
    gmi = N_blocks_x * N_grid_block_x + 1   # global_maximal_i/j (:913-914)
    gmj = N_blocks_y * N_grid_block_y + 1
    objs = []
    for _n in range(n_bo):
        cf.next()
        ln = cf.next()
        ty, ns = fortran_field(ln, 3, 2, "i"), fortran_field(ln, 8, 2, "i")
        cf.next()
        segs = []
        for _m in range(ns):
            ln = cf.next()
            segs.append(tuple(fortran_field(ln, c, 6, "i") for c in (3, 12, 21, 30)))
        objs.append((ty, segs))
    inner = []
    for _n in range(n_io):
        cf.next()
        ty = fortran_field(cf.next(), 3, 2, "i")
        cf.next()
        ln = cf.next()
        inner.append((ty,) + tuple(fortran_field(ln, c, 6, "i") for c in (3, 12, 21, 30)))
    periodic = any(abs(ty) == 2 for ty, _s in objs)   # PERIODIC_PIPELINE_X (:399-415)
    side = {}   # 0 below, 1 above, 2 left, 3 right -> boundary object number (1-based)
    for n, (ty, segs) in enumerate(objs):
        for (i0, j0, i1, j1) in segs:
            if j0 == j1 == 0:
                s_ = 0
            elif j0 == j1 == gmj:
                s_ = 1
            elif i0 == i1 == 0:
                s_ = 2
            elif i0 == i1 == gmi:
                s_ = 3
            else:
                continue
            if ty == 1:
                side[s_] = n + 1
    d.update(ncx=gmi - 1 if periodic else gmi, ncy=gmj, periodic=periodic, N_of_particles_cell=N_of_particles_cell,
             N_max_vel=N_max_vel, T_e_eV=T_e_eV, N_plasma_m3=N_plasma_m3,
             inner=[(il, jb, ir, jt) for (_t, il, jb, ir, jt) in inner], inner_type=[t for (t, *_r) in inner])
    # scales (:719-723, :893-900)
    v_Te_ms = math.sqrt(2.0 * T_e_eV * E_CL / M_E_KG)
    W_plasma_s1 = math.sqrt(N_plasma_m3 * (E_CL * E_CL) / (eps0 * M_E_KG))
    L_debye_m = v_Te_ms / W_plasma_s1
    delta_x_m = L_debye_m / N_of_cells_debye
    delta_t_s = delta_x_m / (N_max_vel * v_Te_ms)
    V_scale_ms = N_max_vel * v_Te_ms
    E_scale_Vm = M_E_KG * V_scale_ms / (E_CL * delta_t_s)
    B_scale_T = M_E_KG / (E_CL * delta_t_s)
    F_scale_V = E_CL * N_plasma_m3 * (delta_x_m * delta_x_m) / eps0
    energy_factor_eV = 0.5 * M_E_KG * (V_scale_ms * V_scale_ms) / E_CL
    d.update(delta_x_m=delta_x_m, delta_t_s=delta_t_s, V_scale_ms=V_scale_ms, E_scale_Vm=E_scale_Vm,
             B_scale_T=B_scale_T, F_scale_V=F_scale_V, energy_factor_eV=energy_factor_eV,
             factor_rho=1.0 / N_of_particles_cell,
             factor2_E=F_scale_V / (E_scale_Vm * 2.0 * delta_x_m), factor1_E=F_scale_V / (E_scale_Vm * delta_x_m))
    # init_simcontrol.dat (:830-845)
    sc = _Lines(path("init_simcontrol.dat"))
    t_sim_ns = sc.value(3, 11, "f", 3)
    d["N_subcycles"] = sc.value(8, 2, "i")
    d["Max_T_cntr"] = int(t_sim_ns / (1.0e9 * delta_t_s))
    # init_particles.dat (:1005-1031); SET_ION_SPECIES (:1505-1507)
    pf = _Lines(path("init_particles.dat"))
    d["init_Te_eV"] = pf.value(3, 8, "f", 3)
    d["init_Ne_m3"] = pf.value(3, 10, "e", 3)
    n_spec = pf.value(6, 1, "i")
    pf.next()
    ions = []
    for _s in range(n_spec):
        ln = pf.next()
        m_amu, q = fortran_field(ln, 3, 5, "f", 1), fortran_field(ln, 11, 2, "i")
        ti = fortran_field(ln, 16, 8, "f", 3)
        Ms = (AMU_KG * m_amu) / M_E_KG
        ions.append(dict(M_i_amu=m_amu, Qs=q, init_Ti_eV=ti, Ms=Ms, QM2s=0.5 * q / Ms,
                         QM2sNsub=d["N_subcycles"] * (0.5 * q / Ms)))
    d["ions"] = ions
    d["seed"] = pf.value(3, 9, "i")
    # init_extfields.dat (pic2d_ExternalFields.f90:36-145)
    bx = by = bz = ez = 0.0
    sense_b = sense_ez = False
    if os.path.exists(path("init_extfields.dat")):
        ef = _Lines(path("init_extfields.dat"))
        bx = ef.value(3, 9, "f", 3)
        by = ef.value(3, 9, "f", 3)
        ef.next()
        ef.value(3, 9, "f", 3)          # y_Bmax
        ef.value(3, 9, "f", 3)          # Bz_0
        bz_max = ef.value(3, 9, "f", 3)
        ef.value(3, 9, "f", 3)          # Bz_Lsys
        ef.value(3, 9, "f", 3)
        ef.value(3, 9, "f", 3)
        ez = ef.value(3, 9, "f", 3)
        sense_b = ef.value(7, 1, "i") == 1
        sense_ez = ef.value(7, 1, "i") == 1
        bx, by, bz = bx * 1.0e-4 / B_scale_T, by * 1.0e-4 / B_scale_T, bz_max * 1.0e-4 / B_scale_T   # Bz_ext = Bz_max
        ez = ez * 100.0 / E_scale_Vm
    d.update(Bx_ext=bx, By_ext=by, Bz_ext=bz, Ez_ext=ez, ions_sense_magnetic_field=sense_b, ions_sense_Ez=sense_ez)

    # init_bo_NN.dat (pic2d_Setup.f90:60-100), normalised as pic2d_CurProblemValues.f90:1218-1221
    def bo(n):
        fn = path(f"init_bo_{n:02d}.dat")
        if not os.path.exists(fn):
            return dict(material="", phi_const=0.0, phi_var=0.0, omega=0.0, phase=0.0, number=n)
        b = _Lines(fn)
        b.next()
        mat = b.next()[6:12]
        c0, var, om, ph = (b.value(3, 9, "f", 3) for _ in range(4))
        return dict(material=mat, phi_const=c0 / F_scale_V, phi_var=var / F_scale_V, omega=om * 2.0e6 * PI * delta_t_s,
                    phase=ph * PI / 180.0, number=n)
    d["walls"] = {s_: bo(n) for s_, n in side.items()}
    d["inner_objects"] = [bo(n_bo + k + 1) for k in range(n_io)]
    # neutrals and collisions
    if os.path.exists(path("init_neutrals.dat")):
        nl = open(path("init_neutrals.dat")).read().splitlines()
        n_neutral = fortran_field(nl[1], 10, 2, "i")
    else:
        n_neutral = 0
    d["neutral"] = None
    d["rcx"] = None
    if n_neutral >= 1:
        neu = read_neutral_deck(directory)
        d["neutral"] = neu
        # ion_velocity_factor of the ions an ionisation produces (pic2d_enCollisionsGeneralProc.f90:224)
        d["ion_velocity_factor"] = [
            math.sqrt(neu["t_k"] * KB_JK / (T_e_eV * E_CL)) / (N_max_vel * math.sqrt(ions[c["isp"] - 1]["Ms"]))
            if 1 <= c["isp"] <= n_spec else 0.0 for c in neu["cs"]]
        rf = path(f"init_neutral_{neu['name']}_rcx_param.dat")
        if os.path.exists(rf):
            toks = open(rf).read().splitlines()[1].replace(",", " ").split()
            s_, sig, alpha = int(toks[0]), float(toks[1].replace("d", "e")), float(toks[2].replace("d", "e"))
            if 1 <= s_ <= n_spec:
                Ms = ions[s_ - 1]["Ms"]
                tg_ev = neu["t_k"] * KB_JK / E_CL
                lf = 1.0 - alpha * math.log(max(1.5 * tg_ev, 0.001))
                sig_th = sig * (lf * lf)                                                 # sigma_rcx_m2 (:35-44)
                vmean = math.sqrt(2.54647908947033 * tg_ev * E_CL / (Ms * M_E_KG))
                d["rcx"] = dict(
                    species=s_, sigma_1eV=sig, alpha=alpha,
                    vfactor=math.sqrt(neu["t_k"] * KB_JK / (T_e_eV * E_CL * Ms)) / N_max_vel,        # :83
                    probab_thermal=neu["n_m3"] * sig_th * vmean * delta_t_s * d["N_subcycles"],     # :4-31
                    prob_factor=neu["n_m3"] * delta_t_s * d["N_subcycles"],                         # :103
                    factor_eV=Ms * energy_factor_eV)                                                # :102
    return d


# --------------------------------------------------------------------------------- whole cycle
class OracleCycle:
    """The oracle's cycle (oracle_cycle_step: MainProg order, N_subcycles from the deck) set up from the deck by the
    oracle's own reader (read_deck above) and its own tables. Particles are given as FP64 columns; capacity for
    appended particles. Wall potentials follow UPDATE_WALL_POTENTIALS each step (WallProfile)."""

    def __init__(self, deck_dir, electrons, ions, seed, nthreads=1, cap_factor=1.3):
        dk = self.deck = read_deck(deck_dir)
        n_e, n_i = len(electrons[0]), len(ions[0])
        self.pe = ParticleSet(*electrons[:5], ids=electrons[5] if len(electrons) > 5 else None,
                              cap=int(n_e * cap_factor) + 1024)
        self.pi = ParticleSet(*ions[:5], ids=ions[5] if len(ions) > 5 else None, cap=int(n_i * cap_factor) + 1024)
        nb = max(n_e // 4, 4096)
        mk = lambda: ParticleSet(*(np.zeros(0),) * 5, cap=nb)
        self.be, self.bi = mk(), mk()
        nsub = dk["N_subcycles"]
        self.mv, _ = maxwell_tables()
        g = geom(dk["ncx"], dk["ncy"], dk["periodic"], dk["inner"])
        ion = dk["ions"][0]
        c = Cycle()
        c.geom = g
        c.e_sp = Species(dk["Bx_ext"], dk["By_ext"], dk["Bz_ext"], dk["Ez_ext"], 0, 0.0, nsub, 0, 0)
        c.i_sp = Species(dk["Bx_ext"], dk["By_ext"], dk["Bz_ext"], dk["Ez_ext"], 1, ion["QM2s"], nsub,
                         int(dk["ions_sense_magnetic_field"]), int(dk["ions_sense_Ez"]))
        c.factor_rho = dk["factor_rho"]
        c.ion_charge = float(ion["Qs"])
        c.factor2_E, c.factor1_E = dk["factor2_E"], dk["factor1_E"]
        self.mcc = None
        neu = dk["neutral"]
        if neu is not None and neu["cs"]:
            self.mcc = MccTables(neu, nsub, dk["delta_t_s"])
            c.mcc = C.pointer(self.mcc.t)
            ivf = max(dk["ion_velocity_factor"])
            c.mcc_ctx = MccCtx(seed, 0, dk["energy_factor_eV"], neu["mass"], ivf, dp(self.mv))
        else:
            c.mcc_ctx = MccCtx(seed, 0, dk["energy_factor_eV"], 0.0, 0.0, dp(self.mv))
        r = dk["rcx"]
        if r is not None:
            c.rcx = Rcx(r["prob_factor"], dk["V_scale_ms"], r["factor_eV"], r["sigma_1eV"], r["alpha"],
                        r["probab_thermal"], r["vfactor"])
            c.rcx_on = 1
        c.nthreads = nthreads
        c.born_e, c.born_i, c.cap_born = self.be.s, self.bi.s, nb
        c.next_id_e = int(self.pe.id[:n_e].max()) + 1 if n_e else 0
        c.next_id_i = int(self.pi.id[:n_i].max()) + 1 if n_i else 0
        c.n_sub_phase = 0
        self.c = c
        self.t_cntr = 0
        self.walls = wall_profiles(deck_dir, dk)
        ny, nx = nodes_shape(g)
        self.work = np.zeros(9 * nx * ny)
        self.counters = np.zeros(16, dtype=np.int64)

    def step(self, n=1):
        processed = 0
        for _ in range(n):
            w = self.walls
            self.c.phi_bottom = w[0].value(self.t_cntr) if 0 in w else 0.0
            self.c.phi_top = w[1].value(self.t_cntr) if 1 in w else 0.0
            processed += lib().oracle_cycle_step(C.byref(self.c), C.byref(self.pe.s), C.byref(self.pi.s),
                                                 len(self.pe.cols["x"]), len(self.pi.cols["x"]), dp(self.work),
                                                 self.counters.ctypes.data_as(_I64))
            self.t_cntr += 1
        return processed


class WallProfile:
    """UPDATE_WALL_POTENTIALS for one metal object (pic2d_WallPotentials.f90:1-165): Harmonic_Oscillation (with the
    phase re-anchored at each amplitude-profile period), Custom_Waveform and Amplitude_Profile, with the waveform
    values, amplitude factors and interpolation weight in single precision as the reference's REAL variables; the two
    optional files read as PREPARE_WAVEFORMS and PREPARE_OSCILLATIONS_AMPLITUDE_PROFILE read them
    (pic2d_Setup.f90:150-412)."""

    def __init__(self, obj, directory=None, number=None, delta_t_s=None, f_scale_v=None):
        self.phi_const, self.phi_var = obj["phi_const"], obj["phi_var"]
        self.omega, self.phase = obj["omega"], obj["phase"]
        self.phase_adjusted = self.phase
        self.wf_t, self.wf_phi, self.ap_t, self.ap_factor = [], [], [], []
        if directory is not None:
            self._read_waveform(os.path.join(directory, f"init_bo_{number:02d}_waveform.dat"), delta_t_s, f_scale_v)
            self._read_amplitude(os.path.join(directory, f"init_bo_{number:02d}_amplitude_profile.dat"), delta_t_s)

    @staticmethod
    def _pairs(lines):
        out = []
        for ln in lines:
            tok = ln.replace(",", " ").split()
            if not tok:
                continue
            if len(tok) < 2:
                break
            try:
                a, b = float(tok[0].replace("d", "e")), float(tok[1].replace("d", "e"))
            except ValueError:
                break
            out.append((tok[0].replace("d", "e"), tok[1].replace("d", "e")))
        return out

    def _read_waveform(self, path, dt, fsc):
        if not os.path.exists(path):
            return
        L = open(path).read().splitlines()
        pts = self._pairs(L[4:])
        n = len(pts)
        if n <= 1:
            return
        phi_v, nu = float(L[0].split()[0].replace("d", "e")), float(L[1].split()[0].replace("d", "e"))
        if phi_v == 0.0:
            return
        period = int(1.0 / (nu * dt))
        if period < n - 1:
            return
        t = [int(np.float32(a) * np.float32(period)) for a, _b in pts]          # REAL * INTEGER
        v = [np.float32((phi_v / fsc) * float(np.float32(b))) for _a, b in pts]
        t[0], t[-1] = 0, period
        for i in range(1, n - 1):
            t[i] = max(t[i], t[i - 1] + 1)
        if t[-1] > t[-2]:
            self.wf_t, self.wf_phi = t, v

    def _read_amplitude(self, path, dt):
        if not os.path.exists(path):
            return
        pts = self._pairs(open(path).read().splitlines()[1:])
        n = len(pts)
        if n <= 1:
            return
        t = [int(float(np.float32(a)) * 1.0e-9 / dt) for a, _b in pts]
        f = [np.float32(b) for _a, b in pts]
        t[0] = 0
        for i in range(1, n - 1):
            t[i] = max(t[i], t[i - 1] + 1)
        if self.wf_t:
            wp = self.wf_t[-1]
            for i in range(n - 1):
                if f[i] == 0.0 and f[i + 1] != 0.0:
                    d = t[i + 1] - t[i]
                    t[i] = wp * (t[i] // wp)
                    t[i + 1] = t[i] + d
            for i in range(1, n):
                if f[i - 1] != 0.0 and f[i] == 0.0:
                    d = t[i] - t[i - 1]
                    t[i] = wp * (t[i] // wp)
                    t[i - 1] = t[i] - d
            t[-1] = wp * (t[-1] // wp)
        if all(t[i + 1] > t[i] for i in range(n - 1)):
            self.ap_t, self.ap_factor = t, f

    @staticmethod
    def _interp(tt, vv, t):
        per = tt[-1]
        my = t - (t // per) * per
        for i in range(len(tt) - 1):
            if tt[i] <= my <= tt[i + 1]:
                ai = np.float32((tt[i + 1] - my) / (tt[i + 1] - tt[i]))
                return float(np.float32(vv[i] * ai)) + float(vv[i + 1]) * (1.0 - float(ai))
        return None

    def adjust_phase(self, start_t):
        """ADJUST_HARMONIC_OSCILLATIONS_PHASE (pic2d_WallPotentials.f90:180-206) for a run continued at start_t"""
        if start_t == 0 or not self.ap_t:
            return
        per = self.ap_t[-1]
        my = (start_t // per) * per
        n_periods = int((self.omega * my) / (2.0 * PI))
        self.phase_adjusted = n_periods * 2.0 * PI + self.phase - self.omega * my

    def value(self, t):
        if self.ap_t:
            per = self.ap_t[-1]
            if t == (t // per) * per:
                n_periods = int((self.omega * t) / (2.0 * PI))
                self.phase_adjusted = n_periods * 2.0 * PI + self.phase - self.omega * t
            harm = self.phi_var * math.sin(self.omega * t + self.phase_adjusted)
        else:
            harm = self.phi_var * math.sin(self.omega * t + self.phase)
        wf = 0.0
        if self.wf_t:
            r = self._interp(self.wf_t, self.wf_phi, t)
            wf = 0.0 if r is None else r
        amp = 1.0
        if self.ap_t:
            r = self._interp(self.ap_t, self.ap_factor, t)
            amp = 1.0 if r is None else r
        return self.phi_const + (harm + wf) * amp


def wall_profiles(deck_dir, dk=None):
    """{object (0..3 walls by side, 4 + n inner objects): WallProfile} of the deck's metal objects."""
    dk = dk or read_deck(deck_dir)
    out = {}
    for side, w in dk["walls"].items():
        out[side] = WallProfile(w, deck_dir, w["number"], dk["delta_t_s"], dk["F_scale_V"])
    for k, w in enumerate(dk["inner_objects"]):
        if dk["inner_type"][k] == 1:
            out[4 + k] = WallProfile(w, deck_dir, w["number"], dk["delta_t_s"], dk["F_scale_V"])
    return out
