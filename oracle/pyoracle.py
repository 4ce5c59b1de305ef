"""ORACLE (test infrastructure only): ctypes front end of liboracle.so, the CPU FP64 restatement of
EDIPIC-2D's particle cycle (oracle.cpp, oracle_rng.c), plus a reader of the neutral-gas decks that follows
INITIATE_ELECTRON_NEUTRAL_COLLISIONS (pic2d_enCollisionsGeneralProc.f90:63-200) independently of the product's
deck reader. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module.
"""
import ctypes as C
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
                ("next_id_e", C.c_uint32), ("next_id_i", C.c_uint32)]


_lib = None


class Emit(C.Structure):
    _fields_ = [("on", C.c_int32 * 4), ("yld", C.c_double * 4), ("emin", C.c_double * 4),
                ("emax", C.c_double * 4), ("fconv", C.c_double * 4), ("ms", C.c_double), ("species", C.c_uint32),
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
            "oracle_philox2x32_10": ([_U32, C.c_uint32, _U32], None),
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
            "oracle_cg_solve_eps": ([C.POINTER(Geom), _D, _D, _D, _D, C.c_double, C.c_int32, _D, _D], C.c_int32),
            "oracle_inner_hit": ([C.POINTER(Geom), _D, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                  C.c_double, _D], C.c_int32),
            "oracle_ion_reflect": ([C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, _D], None),
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


def philox2x32(ctr, key):
    out = (C.c_uint32 * 2)()
    lib().oracle_philox2x32_10((C.c_uint32 * 2)(*ctr), key, out)
    return tuple(out)


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


# --------------------------------------------------------------------------------- whole cycle
class OracleCycle:
    """The oracle's cycle (oracle_cycle_step: MainProg order with N_subcycles = 1) set up from a deck and the
    product-independent tables above. Particles are given as FP64 columns; capacity for appended particles."""

    def __init__(self, deck_dir, params, tables, electrons, ions, seed, nthreads=1, cap_factor=1.3):
        p, t = params, tables
        n_e, n_i = len(electrons[0]), len(ions[0])
        self.pe = ParticleSet(*electrons[:5], ids=electrons[5] if len(electrons) > 5 else None,
                              cap=int(n_e * cap_factor) + 1024)
        self.pi = ParticleSet(*ions[:5], ids=ions[5] if len(ions) > 5 else None, cap=int(n_i * cap_factor) + 1024)
        nb = max(n_e // 4, 4096)
        mk = lambda: ParticleSet(*(np.zeros(0),) * 5, cap=nb)
        self.be, self.bi = mk(), mk()
        self.neu = read_neutral_deck(deck_dir)
        self.mcc = MccTables(self.neu, p.n_subcycles, p.delta_t_s)
        self.mv, _ = maxwell_tables()
        inner = [(p.inner_ileft[k], p.inner_jbottom[k], p.inner_iright[k], p.inner_jtop[k]) for k in range(p.n_inner)]
        g = geom(p.ncx, p.ncy, p.periodic_x, inner)
        c = Cycle()
        c.geom = g
        c.e_sp = Species(p.bx, p.by, p.bz, p.ez, 0, 0.0, p.n_subcycles, 0, 0)
        c.i_sp = Species(p.bx, p.by, p.bz, p.ez, 1, 0.5 * p.ion_charge[0] / p.ion_mass_me[0], p.n_subcycles,
                         p.ions_sense_b, p.ions_sense_ez)
        c.factor_rho = 1.0 / p.n_of_particles_cell
        c.ion_charge = float(p.ion_charge[0])
        c.factor2_E = p.f_scale_v / (p.e_scale_vm * 2.0 * p.delta_x_m)
        c.factor1_E = p.f_scale_v / (p.e_scale_vm * p.delta_x_m)
        c.phi_bottom, c.phi_top = p.wall_phi_const[0], p.wall_phi_const[1]
        c.mcc = C.pointer(self.mcc.t)
        c.mcc_ctx = MccCtx(seed, 0, t.energy_factor_eV, self.neu["mass"], t.ion_velocity_factor[2], dp(self.mv))
        c.rcx = Rcx(t.rcx_prob_factor, p.v_scale_ms, p.ion_mass_me[0] * t.energy_factor_eV, t.rcx_sigma_1eV,
                    t.rcx_alpha, t.rcx_probab_thermal[0], t.rcx_vfactor[0])
        c.rcx_on = int(t.rcx_on[0])
        c.nthreads = nthreads
        c.born_e, c.born_i, c.cap_born = self.be.s, self.bi.s, nb
        c.next_id_e = int(self.pe.id[:n_e].max()) + 1 if n_e else 0
        c.next_id_i = int(self.pi.id[:n_i].max()) + 1 if n_i else 0
        self.c = c
        ny, nx = nodes_shape(g)
        self.work = np.zeros(7 * nx * ny)
        self.counters = np.zeros(16, dtype=np.int64)

    def step(self, n=1):
        processed = 0
        for _ in range(n):
            processed += lib().oracle_cycle_step(C.byref(self.c), C.byref(self.pe.s), C.byref(self.pi.s),
                                                 len(self.pe.cols["x"]), len(self.pi.cols["x"]), dp(self.work),
                                                 self.counters.ctypes.data_as(_I64))
        return processed
