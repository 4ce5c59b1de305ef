"""Host-side mirror of EDIPIC-2D's per-step particle-cycle interface on one B200.

The reference drives its hot path through argument-less Fortran subroutines called in a fixed order from
MainProg (src/pic2d_MainProgram.f90:151-309). `Simulation` exposes the same steps under the same names, each
a thin call into the C ABI of libedipic_b200.so (include/edipic_gpu.h); there is no CPU implementation behind
them, and a missing library or GPU raises instead of falling back.
"""
import ctypes as C

import numpy as np

from . import _abi
from ._abi import SeeParams  # noqa: F401
from ._abi import (ELECTRONS, FIELD_ACC_EX, FIELD_ACC_EY, FIELD_EX, FIELD_EY, FIELD_PHI, FIELD_RHO_TOTAL,
                   FIELD_SURFACE_CHARGE, IONS,
                   PREC_FP64, PREC_MIXED, PRECOND_MG, PRECOND_NONE, SOLVER_CG, SOLVER_FFTX, WARM_LEARNED, WARM_PREVIOUS,
                   WARM_USER, WARM_ZERO, Counters,
                   Params, Tables)

__all__ = ["Simulation", "EdpError", "read_deck", "library", "Params", "Tables", "Counters", "ELECTRONS", "IONS",
           "PREC_MIXED", "PREC_FP64", "SOLVER_FFTX", "SOLVER_CG", "FIELD_EX", "FIELD_EY", "FIELD_ACC_EX",
           "FIELD_ACC_EY", "FIELD_PHI", "FIELD_RHO_TOTAL", "FIELD_SURFACE_CHARGE", "WARM_ZERO", "WARM_PREVIOUS", "WARM_USER", "WARM_LEARNED",
           "PRECOND_NONE", "PRECOND_MG"]

_lib = None


def library():
    """The loaded libedipic_b200.so (loaded once)."""
    global _lib
    if _lib is None:
        _lib = _abi.load()
    return _lib


class EdpError(RuntimeError):
    def __init__(self, code, where, message=""):
        self.code = code
        super().__init__(f"{where}: {_abi.ERROR_NAMES.get(code, code)} {message}".strip())


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


class Deck:
    """A parsed input-deck directory (init_*.dat files), as INITIATE_PARAMETERS and the collision set-up read it.
    Keeps the C-side table arrays alive while params/tables are in use."""

    def __init__(self, directory):
        self.lib = library()
        self.handle = C.c_void_p()
        self.params = Params()
        self.tables = Tables()
        rc = self.lib.edp_deck_read(str(directory).encode(), C.byref(self.handle), C.byref(self.params),
                                    C.byref(self.tables))
        if rc != 0:
            raise EdpError(rc, "edp_deck_read", str(directory))
        te, ne, tev, npl = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        ti = (C.c_double * _abi.MAX_ION)()
        nmv = C.c_int32()
        maxt = C.c_int64()
        self.lib.edp_deck_initial_plasma(self.handle, C.byref(te), C.byref(ne), ti, C.byref(tev), C.byref(nmv),
                                         C.byref(npl), C.byref(maxt))
        self.init_te_ev, self.init_ne_m3, self.t_e_ev = te.value, ne.value, tev.value
        self.init_ti_ev = [ti[s] for s in range(_abi.MAX_ION)]
        self.n_max_vel, self.n_plasma_m3, self.max_t_cntr = nmv.value, npl.value, maxt.value
        # ion-induced electron emission of the walls' materials: {(wall, ion species): (yield, E_min, E_max, T)}
        self.ion_emission = {}
        self.ion_wall_model = [0, 0, 0, 0]   # 0 absorb, 1 reflect, 2 ion-induced emission; walls, then inner objects
        self.electron_emission = {}           # {wall: SeeParams} of the walls whose material emits electrons
        self.wall_injection = {}              # {object: (N per step, model, T_normal, T_parallel, W_beam)}
        buf = (C.c_double * 4)()
        model = C.c_int32()
        for wall in range(4):
            if self.lib.edp_deck_ion_wall_model(self.handle, wall, C.byref(model)) == 0:
                self.ion_wall_model[wall] = model.value
            see, on = _abi.SeeParams(), C.c_int32()
            if self.lib.edp_deck_electron_emission(self.handle, wall, C.byref(see), C.byref(on)) == 0 and on.value:
                self.electron_emission[wall] = see
            inj = (C.c_double * 5)()
            if self.lib.edp_deck_wall_injection(self.handle, wall, inj) == 0 and inj[0] > 0.0:
                self.wall_injection[wall] = (inj[0], int(inj[1]), inj[2], inj[3], inj[4])
            for s in range(1, self.params.n_ion_species + 1):
                if self.lib.edp_deck_ion_emission(self.handle, wall, s, buf) == 0 and buf[0] > 0.0:
                    self.ion_emission[(wall, s)] = tuple(buf)
        # the inner objects' materials (objects 4 + n): ion reflection and ion-induced emission
        for obj in range(4, 4 + self.params.n_inner):
            if self.lib.edp_deck_ion_wall_model(self.handle, obj, C.byref(model)) == 0 and model.value:
                self.ion_wall_model.append(model.value)
            else:
                self.ion_wall_model.append(0)
            see, on = _abi.SeeParams(), C.c_int32()
            if self.lib.edp_deck_electron_emission(self.handle, obj, C.byref(see), C.byref(on)) == 0 and on.value:
                self.electron_emission[obj] = see
            # constant electron emission: metal inner objects only (PERFORM_ELECTRON_EMISSION_SETUP_INNER_OBJECTS)
            inj = (C.c_double * 5)()
            if (self.params.inner_eps[obj - 4] == 0.0 and self.lib.edp_deck_wall_injection(self.handle, obj, inj) == 0
                    and inj[0] > 0.0):
                self.wall_injection[obj] = (inj[0], int(inj[1]), inj[2], inj[3], inj[4])
            for s in range(1, self.params.n_ion_species + 1):
                if self.lib.edp_deck_ion_emission(self.handle, obj, s, buf) == 0 and buf[0] > 0.0:
                    self.ion_emission[(obj, s)] = tuple(buf)
        # time dependence of the metal objects' potentials (walls 0..3, inner objects 4 + n): those with a waveform,
        # an amplitude profile, or an oscillating inner object (walls' harmonic fields are in params already)
        self.potential_profiles = {}
        for obj in range(4 + _abi.MAX_INNER):
            prof = self.potential_profile(obj)
            if prof[1] is not None or prof[2] is not None or (obj >= 4 and prof[0][1] != 0.0):
                self.potential_profiles[obj] = prof

    def potential_profile(self, obj):
        """(harmonic {phi_const, phi_var, omega, phase}, (wf_T_cntr, wf_phi) or None, (ap_T_cntr, ap_factor) or None)
        of metal object obj as the deck sets it up (edp_deck_potential_profile)."""
        harm = np.zeros(4)
        nw, na = C.c_int32(), C.c_int32()
        self.lib.edp_deck_potential_profile(self.handle, obj, _dp(harm), C.byref(nw), None, None, C.byref(na), None,
                                            None)
        wt, wv = np.zeros(nw.value, dtype=np.int32), np.zeros(nw.value, dtype=np.float32)
        at, av = np.zeros(na.value, dtype=np.int32), np.zeros(na.value, dtype=np.float32)
        i32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        f32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        self.lib.edp_deck_potential_profile(self.handle, obj, _dp(harm), C.byref(nw), i32(wt), f32(wv), C.byref(na),
                                            i32(at), f32(av))
        return harm, ((wt, wv) if nw.value else None), ((at, av) if na.value else None)

    def potential_series(self, obj, t0, n):
        """UPDATE_WALL_POTENTIALS of metal object obj for steps t0 .. t0 + n - 1 (no device needed)."""
        out = np.zeros(int(n))
        rc = self.lib.edp_deck_potential_series(self.handle, obj, int(t0), int(n), _dp(out))
        if rc != 0:
            raise EdpError(rc, "edp_deck_potential_series")
        return out

    def close(self):
        if self.handle:
            self.lib.edp_deck_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_deck(directory):
    return Deck(directory)


class Simulation:
    """One device context. Method names follow the reference subroutines they replace."""

    def __init__(self, deck, precision=PREC_MIXED, sort_every=None, fuse_collisions=True, capacity=None, seed=None,
                 strip=None):
        """strip = (own columns, ghost columns on the left, on the right, global column of local column 0): one x
        strip of the deck's domain (edp_set_strip), a walled-x context of own + ghost columns whose field comes
        from a context of the whole grid. Its inner objects are the deck's, in its columns."""
        self.lib = library()
        self.deck = deck if isinstance(deck, Deck) else Deck(deck)
        p = Params.from_buffer_copy(self.deck.params)
        p.precision = precision
        strip_frame = None
        if strip is not None:
            own, gl, gr, x_first = (int(v) for v in strip)
            strip_frame = (gl, gr, x_first, p.ncx, p.periodic_x)
            p.ncx = own + gl + gr
            p.periodic_x = 0
            p.solver = SOLVER_CG
            for n in range(p.n_inner):   # strip columns; an object past the strip is clipped one column beyond it
                p.inner_ileft[n] = min(max(p.inner_ileft[n] - x_first, -1), p.ncx + 1)
                p.inner_iright[n] = min(max(p.inner_iright[n] - x_first, -1), p.ncx + 1)
        if sort_every is not None:
            p.sort_every = sort_every
        p.fuse_collisions = 1 if fuse_collisions else 0
        if capacity is not None:
            for s, v in enumerate(capacity):
                p.capacity[s] = int(v)
        if seed is not None:
            p.seed = int(seed)
        self.params = p
        self.ctx = C.c_void_p()
        rc = self.lib.edp_init(C.byref(p), C.byref(self.deck.tables), C.byref(self.ctx))
        if rc != 0:
            raise EdpError(rc, "edp_init")
        if strip_frame is not None:
            self._check(self.lib.edp_set_strip(self.ctx, *strip_frame), "edp_set_strip")
        self.periodic = bool(p.periodic_x)
        self.nx_ref = p.ncx + 2 if self.periodic else p.ncx + 1
        self.ny_ref = p.ncy + 1
        for (wall, s), (yld, e0, e1, t) in self.deck.ion_emission.items():
            self.set_ion_emission(wall, s, yld, e0, e1, t)
        for wall, model in enumerate(self.deck.ion_wall_model):
            if model == 1:
                self.set_ion_reflection(wall, True)
        for wall, see in self.deck.electron_emission.items():
            self.set_electron_emission(wall, see)
        for wall, (n, model, tn, tp, wb) in self.deck.wall_injection.items():
            self.set_wall_injection(wall, n, model, tn, tp, wb)
        for obj, (harm, wf, ap) in self.deck.potential_profiles.items():
            if obj < 4 or obj - 4 < p.n_inner:
                self.set_potential_profile(obj, harm, wf, ap)

    # ------------------------------------------------------------------------------------ plumbing
    def _check(self, rc, where):
        if rc != 0:
            buf = C.create_string_buffer(512)
            self.lib.edp_last_error(self.ctx, buf, 512)
            raise EdpError(rc, where, buf.value.decode(errors="replace"))

    def close(self):
        if self.ctx:
            self.lib.edp_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream(self):
        """The cudaStream_t (as an integer) on which the context runs its work."""
        ptr = C.c_void_p()
        self._check(self.lib.edp_get_stream(self.ctx, C.byref(ptr)), "edp_get_stream")
        return ptr.value or 0

    def set_id_base(self, base, end=None):
        """First id of the particles the context creates from now on, and one past its last (disjoint ranges for
        ranks of a cluster; born particles past the end are refused, edp_set_id_range)."""
        if end is None:
            self._check(self.lib.edp_set_id_base(self.ctx, int(base)), "edp_set_id_base")
        else:
            self._check(self.lib.edp_set_id_range(self.ctx, int(base), int(end)), "edp_set_id_range")

    def reduce_list(self):
        """[(device pointer, count, is_int64)] of the densities deposited since the last call (edp_reduce_list)."""
        ptrs, counts, ints, n = (C.c_void_p * 8)(), (C.c_int64 * 8)(), (C.c_int32 * 8)(), C.c_int32()
        self._check(self.lib.edp_reduce_list(self.ctx, 8, ptrs, counts, ints, C.byref(n)), "edp_reduce_list")
        return [(ptrs[k], counts[k], bool(ints[k])) for k in range(n.value)]

    def device_buffer(self, which, species=0):
        """(device pointer, element count) of the fixed-point density of `species` (which 0), the field (1) or the
        accumulated field (2), internal node layout (edp_device_buffer)."""
        ptr, n = C.c_void_p(), C.c_int64()
        self._check(self.lib.edp_device_buffer(self.ctx, int(which), int(species), C.byref(ptr), C.byref(n)),
                    "edp_device_buffer")
        return ptr.value, n.value

    def synchronize(self):
        self._check(self.lib.edp_synchronize(self.ctx), "edp_synchronize")

    # ------------------------------------------------------------------------------------ particles
    def distribute_particles(self, per_cell, init_te_ev=None, init_ti_ev=None):
        """DISTRIBUTE_PARTICLES (pic2d_CurProblemValues.f90:3127-3325) on the device: per_cell electrons and
        ions per cell, ions at the electron positions, Maxwellian velocities of the deck's initial temperatures."""
        d = self.deck
        te = d.init_te_ev if init_te_ev is None else init_te_ev
        fconv_e = np.sqrt(te / d.t_e_ev) / d.n_max_vel
        self._check(self.lib.edp_distribute_particles(self.ctx, ELECTRONS, int(per_cell), fconv_e, 0, 0),
                    "edp_distribute_particles")
        for s in range(self.params.n_ion_species):
            ti = d.init_ti_ev[s] if init_ti_ev is None else init_ti_ev
            fconv_i = np.sqrt(ti / d.t_e_ev) / (d.n_max_vel * np.sqrt(self.params.ion_mass_me[s]))
            self._check(self.lib.edp_distribute_particles(self.ctx, IONS + s, int(per_cell), fconv_i, 1, 1),
                        "edp_distribute_particles")

    def upload_particles(self, species, x, y, vx, vy, vz, tag=None, ids=None):
        cols = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, vx, vy, vz)]
        n = len(cols[0])
        t = None if tag is None else np.ascontiguousarray(tag, dtype=np.int32)
        i = None if ids is None else np.ascontiguousarray(ids, dtype=np.uint32)
        self._check(self.lib.edp_upload_particles(
            self.ctx, species, n, *[_dp(a) for a in cols],
            t.ctypes.data_as(C.POINTER(C.c_int32)) if t is not None else None,
            i.ctypes.data_as(C.POINTER(C.c_uint32)) if i is not None else None), "edp_upload_particles")

    def download_particles(self, species, cap=None):
        if cap is None:
            cap = self.counters().n_particles[species] + 16
        out = {k: np.zeros(cap) for k in ("x", "y", "vx", "vy", "vz")}
        out["tag"] = np.zeros(cap, dtype=np.int32)
        out["id"] = np.zeros(cap, dtype=np.uint32)
        n = C.c_int64()
        self._check(self.lib.edp_download_particles(
            self.ctx, species, cap, C.byref(n), *[_dp(out[k]) for k in ("x", "y", "vx", "vy", "vz")],
            out["tag"].ctypes.data_as(C.POINTER(C.c_int32)), out["id"].ctypes.data_as(C.POINTER(C.c_uint32))),
            "edp_download_particles")
        return {k: v[:n.value] for k, v in out.items()}

    # ------------------------------------------------------------------------------------ per-step cycle
    def _node_array(self):
        return np.zeros((self.ny_ref, self.nx_ref))

    def gather_electron_charge_density(self):
        """GATHER_ELECTRON_CHARGE_DENSITY: c_rho on the reference node grid (after fold and wall factors)."""
        out = self._node_array()
        self._check(self.lib.edp_gather_charge_density(self.ctx, ELECTRONS, _dp(out)), "edp_gather_charge_density")
        return out

    def gather_ion_charge_density(self, species=0):
        """GATHER_ION_CHARGE_DENSITY: Qs-weighted c_rho_i of one ion species."""
        out = self._node_array()
        self._check(self.lib.edp_gather_charge_density(self.ctx, IONS + species, _dp(out)),
                    "edp_gather_charge_density")
        return out

    def update_wall_potentials(self, t_cntr):
        self._check(self.lib.edp_update_wall_potentials(self.ctx, int(t_cntr)), "edp_update_wall_potentials")

    def set_potential_profile(self, obj, harmonic, waveform=None, amplitude=None):
        """Time dependence of metal object obj's potential (edp_set_potential_profile): harmonic {phi_const, phi_var,
        omega, phase}; waveform / amplitude: (T_cntr array, value array) or None."""
        h = np.ascontiguousarray(harmonic, dtype=np.float64)
        wt, wv = (np.ascontiguousarray(waveform[0], dtype=np.int32), np.ascontiguousarray(waveform[1], dtype=np.float32)) \
            if waveform is not None else (np.zeros(0, np.int32), np.zeros(0, np.float32))
        at, av = (np.ascontiguousarray(amplitude[0], dtype=np.int32), np.ascontiguousarray(amplitude[1], dtype=np.float32)) \
            if amplitude is not None else (np.zeros(0, np.int32), np.zeros(0, np.float32))
        i32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        f32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        self._check(self.lib.edp_set_potential_profile(self.ctx, int(obj), _dp(h), wt.size, i32(wt), f32(wv), at.size,
                                                       i32(at), f32(av)), "edp_set_potential_profile")

    def solve_poisson_fftx_linsysy(self, want_phi=False):
        """SOLVE_POISSON_FFTX_LINSYSY + CALCULATE_ELECTRIC_FIELD_FFTX_LINSYSY."""
        out = self._node_array() if want_phi else None
        self._check(self.lib.edp_field_fftx(self.ctx, _dp(out)), "edp_field_fftx")
        return out

    def solve_potential_with_cg(self, rtol=1e-8, max_it=20000, warm_start=WARM_PREVIOUS):
        """SOLVE_POTENTIAL_WITH_PETSC + CALCULATE_ELECTRIC_FIELD, with the device CG; returns iterations."""
        it = C.c_int32()
        self._check(self.lib.edp_field_cg(self.ctx, rtol, max_it, warm_start, C.byref(it)), "edp_field_cg")
        return it.value

    def load_warm_start(self, theta):
        """Loads the learned warm start's FP32 parameter vector (edipic_b200.warmstart.param_layout order)."""
        a = np.ascontiguousarray(theta, dtype=np.float32)
        self._check(self.lib.edp_warmstart_load(self.ctx, a.ctypes.data_as(C.POINTER(C.c_float)), a.size),
                    "edp_warmstart_load")

    def predict_warm_start(self):
        """The network's guess for the current density (node layout) and the residual norms of the previous
        potential and of the guess."""
        g = self._node_array()
        res = np.zeros(2)
        self._check(self.lib.edp_warmstart_predict(self.ctx, _dp(g), _dp(res)), "edp_warmstart_predict")
        return g, res

    def set_cg_preconditioner(self, kind):
        """PRECOND_MG (default): a multigrid V-cycle per CG iteration; PRECOND_NONE: plain CG."""
        self._check(self.lib.edp_set_cg_preconditioner(self.ctx, kind), "edp_set_cg_preconditioner")

    def set_ion_emission(self, wall, ion_species, yield_, emin_ev, emax_ev, t_emit_ev):
        """Ion-induced electron emission of a domain wall (0 below, 1 above, 2 left, 3 right) for an ion species
        (1-based): PROCESS_ION_INDUCED_ELECTRON_EMISSION (pic2d_IonEmissions.f90:1-348). yield_ 0 turns it off."""
        self._check(self.lib.edp_set_ion_emission(self.ctx, wall, ion_species, yield_, emin_ev, emax_ev, t_emit_ev),
                    "edp_set_ion_emission")

    def set_step(self, t_cntr):
        """Start_T_cntr of a continued run: the next step is t_cntr (at ion sub-cycle 0)."""
        self._check(self.lib.edp_set_step(self.ctx, int(t_cntr)), "edp_set_step")

    def set_ion_reflection(self, wall, on=True):
        """Ion-material model 1: the wall reflects every ion specularly (INJECT_REFLECTED_ION,
        pic2d_IonEmissions.f90:374-492)."""
        self._check(self.lib.edp_set_ion_reflection(self.ctx, wall, 1 if on else 0), "edp_set_ion_reflection")

    def set_electron_emission(self, wall, params=None, **kw):
        """Electron-induced electron emission of a wall (PROCESS_ELECTRON_INDUCED_ELECTRON_EMISSION,
        pic2d_SEEmission.f90:4-151): params is a SeeParams, or its fields as keywords; None (and no keywords)
        switches the wall off."""
        if params is None and kw:
            params = _abi.SeeParams(**kw)
        self._check(self.lib.edp_set_electron_emission(self.ctx, wall, C.byref(params) if params is not None else None),
                    "edp_set_electron_emission")

    def set_wall_injection(self, wall, n_per_step, model=0, t_normal_ev=0.0, t_parallel_ev=0.0, beam_energy_ev=0.0):
        """Constant electron emission from a wall every step (PERFORM_ELECTRON_EMISSION_SETUP, pic2d_Setup.f90:599):
        model 0 thermal, 1 beam."""
        self._check(self.lib.edp_set_wall_injection(self.ctx, wall, float(n_per_step), int(model), float(t_normal_ev),
                                                    float(t_parallel_ev), float(beam_energy_ev)),
                    "edp_set_wall_injection")

    def emission_counts(self):
        """Electrons emitted by each object (walls 0-3, then inner objects; ion and electron impacts), cumulative:
        electron_emit_count."""
        out = np.zeros(4 + _abi.MAX_INNER, np.int64)
        self._check(self.lib.edp_query_emission(self.ctx, out.ctypes.data_as(C.POINTER(C.c_int64))),
                    "edp_query_emission")
        return out

    def advance_electrons(self):
        self._check(self.lib.edp_advance_electrons(self.ctx), "edp_advance_electrons")

    def advance_ions(self):
        self._check(self.lib.edp_advance_ions(self.ctx), "edp_advance_ions")

    def perform_electron_neutral_collisions(self):
        cnt = (C.c_int64 * _abi.MAX_COLPROC)()
        self._check(self.lib.edp_collide_en(self.ctx, cnt), "edp_collide_en")
        return np.array(cnt[:], dtype=np.int64)

    def perform_resonant_charge_exchange(self):
        n = C.c_int64()
        self._check(self.lib.edp_collide_rcx(self.ctx, C.byref(n)), "edp_collide_rcx")
        return n.value

    def end_ion_cycle(self):
        """PROCESS_ADDED_IONS + CLEAR_ACCUMULATED_FIELDS; advances T_cntr."""
        self._check(self.lib.edp_end_ion_cycle(self.ctx), "edp_end_ion_cycle")

    def step(self, n=1):
        self._check(self.lib.edp_step(self.ctx, int(n)), "edp_step")

    # ------------------------------------------------------------------------------------ diagnostics
    def counters(self):
        c = Counters()
        self._check(self.lib.edp_query_counters(self.ctx, C.byref(c)), "edp_query_counters")
        return c

    def field(self, which):
        out = self._node_array()
        self._check(self.lib.edp_get_field(self.ctx, which, _dp(out)), "edp_get_field")
        return out

    def set_field(self, which, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.ny_ref, self.nx_ref)
        self._check(self.lib.edp_set_field(self.ctx, which, _dp(a)), "edp_set_field")

    def energy_histogram(self, species, edges_ev):
        """Counts of the species' particles by kinetic energy in eV between the given edges (edp_energy_histogram)."""
        e = np.ascontiguousarray(edges_ev, dtype=np.float64)
        out = np.zeros(e.size - 1, dtype=np.int64)
        self._check(self.lib.edp_energy_histogram(self.ctx, species, out.size, _dp(e),
                                                  out.ctypes.data_as(C.POINTER(C.c_int64))), "edp_energy_histogram")
        return out

    def moments(self, species):
        out = np.zeros(7)
        self._check(self.lib.edp_moments(self.ctx, species, _dp(out)), "edp_moments")
        return out

    def collect_moments(self, species):
        """COLLECT_ELECTRON_MOMENTS / COLLECT_ION_MOMENTS: [13, ny, nx] FP32 in the reference node layout (N, VX,
        VY, VZ, WX, WY, WZ, VXVY, VXVZ, VYVZ, QX, QY, QZ)."""
        out = np.zeros((13, self.ny_ref, self.nx_ref), dtype=np.float32)
        self._check(self.lib.edp_collect_moments(self.ctx, species, out.ctypes.data_as(C.POINTER(C.c_float))),
                    "edp_collect_moments")
        return out

    def calculate_vdf(self, species, nbox=(1, 1), n_max_vel_s=4, n_vbins=10, two_d=False, n_max_vel=None):
        """CALCULATE_ELECTRON_VDF / CALCULATE_ION_VDF (pic2d_VelocityDistributions.f90:3-393): returns
        (vdf1d [3, nbox, 2 n_max_vel_s n_vbins] for vx, vy, vz; vdf2d [nbox, vy bin, vx bin] or None; skipped).
        Box k = ibox + jbox * nbox[0]; bin b covers [b, b + 1) / n_vbins thermal velocities, b from
        -n_max_vel_s n_vbins. n_max_vel defaults to the deck's velocity scale N_max_vel."""
        nmv = self.deck.n_max_vel if n_max_vel is None else n_max_vel
        nb = nbox[0] * nbox[1]
        rl = 2 * n_max_vel_s * n_vbins
        v1 = np.zeros((3, nb, rl), dtype=np.int32)
        v2 = np.zeros((nb, rl, rl), dtype=np.int32) if two_d else None
        sk = C.c_int64(0)
        i32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32)) if a is not None else None
        self._check(self.lib.edp_calculate_vdf(self.ctx, species, nmv, nbox[0], nbox[1], n_max_vel_s, n_vbins, i32(v1),
                                               i32(v2), C.byref(sk)), "edp_calculate_vdf")
        return v1, v2, sk.value

    def mcc_choose(self, energy_ev, r):
        e = np.ascontiguousarray(energy_ev, dtype=np.float64)
        rr = np.ascontiguousarray(r, dtype=np.float64)
        out = np.zeros(len(e), dtype=np.int32)
        self._check(self.lib.edp_mcc_choose(self.ctx, len(e), _dp(e), _dp(rr), out.ctypes.data_as(C.POINTER(C.c_int32))),
                    "edp_mcc_choose")
        return out
