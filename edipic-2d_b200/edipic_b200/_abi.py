"""ctypes mirror of include/edipic_gpu.h (the C ABI of libedipic_b200.so).

The structures below must stay field-for-field identical to the C header; tests/test_abi.py checks the
symbol list and the structure sizes against the compiled library.
"""
import ctypes as C
import os

MAX_ION = 4
MAX_INNER = 4
MAX_COLPROC = 8
MAX_SEG = 32
MAX_SPECIES = 1 + MAX_ION
N_HIT = 4 + MAX_INNER
ABI_VERSION = 2

OK, ERR_ARG, ERR_CUDA, ERR_CAPACITY, ERR_BOUNDS, ERR_NOT_CONVERGED, ERR_TIMEOUT, ERR_STATE, ERR_IO = \
    0, -1, -2, -3, -4, -5, -6, -7, -8
PREC_MIXED, PREC_FP64 = 0, 1
SOLVER_FFTX, SOLVER_CG = 0, 1
ELECTRONS, IONS = 0, 1
FIELD_EX, FIELD_EY, FIELD_ACC_EX, FIELD_ACC_EY, FIELD_PHI, FIELD_RHO_TOTAL, FIELD_SURFACE_CHARGE = range(7)
WARM_ZERO, WARM_PREVIOUS, WARM_USER = 0, 1, 2
PRECOND_NONE, PRECOND_MG = 0, 1
WARM_LEARNED = 3

ERROR_NAMES = {
    ERR_ARG: "EDP_ERR_ARG", ERR_CUDA: "EDP_ERR_CUDA", ERR_CAPACITY: "EDP_ERR_CAPACITY",
    ERR_BOUNDS: "EDP_ERR_BOUNDS", ERR_NOT_CONVERGED: "EDP_ERR_NOT_CONVERGED", ERR_TIMEOUT: "EDP_ERR_TIMEOUT",
    ERR_STATE: "EDP_ERR_STATE", ERR_IO: "EDP_ERR_IO",
}


class Params(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("ncx", C.c_int32), ("ncy", C.c_int32), ("periodic_x", C.c_int32),
        ("n_subcycles", C.c_int32), ("n_of_particles_cell", C.c_int32),
        ("delta_t_s", C.c_double), ("delta_x_m", C.c_double),
        ("v_scale_ms", C.c_double), ("e_scale_vm", C.c_double), ("b_scale_t", C.c_double), ("f_scale_v", C.c_double),
        ("bx", C.c_double), ("by", C.c_double), ("bz", C.c_double), ("ez", C.c_double),
        ("ions_sense_b", C.c_int32), ("ions_sense_ez", C.c_int32), ("n_ion_species", C.c_int32),
        ("ion_charge", C.c_int32 * MAX_ION), ("ion_mass_me", C.c_double * MAX_ION),
        ("wall_phi_const", C.c_double * 4), ("wall_phi_var", C.c_double * 4), ("wall_omega", C.c_double * 4),
        ("wall_phase", C.c_double * 4),
        ("n_inner", C.c_int32), ("inner_ileft", C.c_int32 * MAX_INNER), ("inner_jbottom", C.c_int32 * MAX_INNER),
        ("inner_iright", C.c_int32 * MAX_INNER), ("inner_jtop", C.c_int32 * MAX_INNER),
        ("inner_phi", C.c_double * MAX_INNER),
        ("seed", C.c_uint64), ("precision", C.c_int32), ("solver", C.c_int32), ("sort_every", C.c_int32),
        ("fuse_collisions", C.c_int32), ("capacity", C.c_int64 * MAX_SPECIES),
        ("inner_eps", C.c_double * MAX_INNER),
    ]


class Tables(C.Structure):
    _fields_ = [
        ("en_on", C.c_int32), ("n_act", C.c_int32), ("n_seg", C.c_int32), ("n_values", C.c_int32),
        ("seg_value", C.c_double * (MAX_SEG + 1)), ("seg_step", C.c_double * MAX_SEG),
        ("seg_index", C.c_int32 * (MAX_SEG + 1)),
        ("energy_eV", C.POINTER(C.c_double)), ("prob", C.POINTER(C.c_double)),
        ("max_colliding_fraction", C.c_double),
        ("colproc_type", C.c_int32 * MAX_COLPROC), ("threshold_eV", C.c_double * MAX_COLPROC),
        ("ion_species_produced", C.c_int32 * MAX_COLPROC), ("ion_velocity_factor", C.c_double * MAX_COLPROC),
        ("neutral_mass_amu", C.c_double), ("energy_factor_eV", C.c_double),
        ("rcx_on", C.c_int32 * MAX_ION), ("rcx_prob_factor", C.c_double), ("rcx_sigma_1eV", C.c_double),
        ("rcx_alpha", C.c_double), ("rcx_probab_thermal", C.c_double * MAX_ION),
        ("rcx_vfactor", C.c_double * MAX_ION),
        ("maxwell_rmax", C.c_int32), ("maxwell_v", C.POINTER(C.c_double)),
    ]


class SeeParams(C.Structure):
    """edp_see_params: electron-induced emission of one wall material, energies in eV."""
    _fields_ = [("elastic_model", C.c_int32), ("elastic_type", C.c_int32), ("inelastic_model", C.c_int32),
                ("true_model", C.c_int32)] + [(n, C.c_double) for n in (
                    "elastic_yield", "elastic_emin_ev", "elastic_emax_ev", "elastic_e0_ev", "elastic_emax_coef_ev",
                    "elastic_max", "elastic_de_ev", "elastic_frac_classic", "inelastic_yield", "inelastic_emin_ev",
                    "inelastic_emax_ev", "inelastic_frac_classic", "true_t_ev", "true_yield", "true_emin_ev",
                    "true_emax_ev", "classic_e0_ev", "classic_emax_ev", "classic_max", "classic_k_smooth")]


class Counters(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int64 * MAX_SPECIES), ("electron_hits", C.c_int64 * N_HIT),
        ("ion_hits", C.c_int64 * N_HIT), ("en_collisions", C.c_int64 * MAX_COLPROC),
        ("rcx_collisions", C.c_int64 * MAX_ION), ("step", C.c_int64), ("cg_iterations", C.c_int32),
        ("cg_relres", C.c_double), ("error_flags", C.c_int32), ("kernel_launches", C.c_int64),
    ]


P = C.POINTER
_D = P(C.c_double)
_I32 = P(C.c_int32)
_U32 = P(C.c_uint32)
_I64 = P(C.c_int64)
_CTX = C.c_void_p

SIGNATURES = {
    "edp_init": [P(Params), P(Tables), P(C.c_void_p)],
    "edp_destroy": [_CTX],
    "edp_last_error": [_CTX, C.c_char_p, C.c_size_t],
    "edp_set_sync": [_CTX, C.c_int],
    "edp_synchronize": [_CTX],
    "edp_get_stream": [_CTX, P(C.c_void_p)],
    "edp_sort_particles": [_CTX],
    "edp_warmstart_timing": [_CTX, _D],
    "edp_energy_histogram": [_CTX, C.c_int, C.c_int32, _D, P(C.c_int64)],
    "edp_set_push_kernel": [_CTX, C.c_int32],
    "edp_set_sort_in_push": [_CTX, C.c_int32],
    "edp_upload_particles": [_CTX, C.c_int, C.c_int64, _D, _D, _D, _D, _D, _I32, _U32],
    "edp_download_particles": [_CTX, C.c_int, C.c_int64, _I64, _D, _D, _D, _D, _D, _I32, _U32],
    "edp_distribute_particles": [_CTX, C.c_int, C.c_int32, C.c_double, C.c_int32, C.c_int32],
    "edp_gather_charge_density": [_CTX, C.c_int, _D],
    "edp_update_wall_potentials": [_CTX, C.c_int64],
    "edp_set_potential_profile": [_CTX, C.c_int32, _D, C.c_int32, P(C.c_int32), P(C.c_float), C.c_int32,
                                  P(C.c_int32), P(C.c_float)],
    "edp_field_fftx": [_CTX, _D],
    "edp_field_cg": [_CTX, C.c_double, C.c_int32, C.c_int32, _I32],
    "edp_set_cg_preconditioner": [_CTX, C.c_int32],
    "edp_set_ion_emission": [_CTX, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double],
    "edp_query_emission": [_CTX, _I64],
    "edp_set_ion_reflection": [_CTX, C.c_int32, C.c_int32],
    "edp_set_electron_emission": [_CTX, C.c_int32, P(SeeParams)],
    "edp_set_wall_injection": [_CTX, C.c_int32, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double],
    "edp_advance_electrons": [_CTX],
    "edp_advance_ions": [_CTX],
    "edp_collide_en": [_CTX, _I64],
    "edp_collide_rcx": [_CTX, _I64],
    "edp_end_ion_cycle": [_CTX],
    "edp_step": [_CTX, C.c_int32],
    "edp_set_step": [_CTX, C.c_int64],
    "edp_set_id_base": [_CTX, C.c_uint64],
    "edp_set_id_range": [_CTX, C.c_uint64, C.c_uint64],
    "edp_reduce_list": [_CTX, C.c_int32, P(C.c_void_p), _I64, _I32, _I32],
    "edp_set_strip": [_CTX, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32],
    "edp_strip_take": [_CTX, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, _I64, _I64],
    "edp_strip_put": [_CTX, C.c_int32, C.c_void_p, C.c_int64, C.c_double],
    "edp_strip_add_density": [_CTX, C.c_int32, C.c_void_p, C.c_int32, C.c_int32],
    "edp_strip_set_field": [_CTX, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32],
    "edp_device_buffer": [_CTX, C.c_int32, C.c_int32, P(C.c_void_p), _I64],
    "edp_query_counters": [_CTX, P(Counters)],
    "edp_get_field": [_CTX, C.c_int, _D],
    "edp_set_field": [_CTX, C.c_int, _D],
    "edp_moments": [_CTX, C.c_int, _D],
    "edp_mcc_choose": [_CTX, C.c_int64, _D, _D, _I32],
    "edp_collect_moments": [_CTX, C.c_int, P(C.c_float)],
    "edp_calculate_vdf": [_CTX, C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _I32, _I32, _I64],
    "edp_poisson_fftx_noalloc": [C.c_int32, C.c_int32, C.c_void_p, C.c_double, C.c_double, C.c_void_p,
                                 C.c_void_p],
    "edp_warmstart_load": [_CTX, P(C.c_float), C.c_int64],
    "edp_warmstart_predict": [_CTX, _D, _D],
    "edp_nn_conv3x3_fwd": [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                           C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p],
    "edp_nn_flip_transpose": [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p],
    "edp_nn_error": [_I32],
    "edp_nn_conv_select": [C.c_int32],
    "edp_nn_wgrad_select": [C.c_int32],
    "edp_nn_conv3x3_wgrad": [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                             C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p],
    "edp_nn_pool": [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p],
    "edp_nn_pool_bwd": [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                        C.c_void_p],
    "edp_nn_upsample": [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p],
    "edp_nn_upsample_bwd": [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                            C.c_void_p, C.c_void_p],
    "edp_nn_relu_bwd": [C.c_int64, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                        C.c_void_p],
    "edp_nn_head_fwd": [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                        C.c_void_p],
    "edp_nn_head_bwd": [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                        C.c_void_p, C.c_void_p, C.c_void_p],
    "edp_nn_adam": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float, C.c_float,
                    C.c_float, C.c_int32, C.c_void_p, C.c_void_p],
    "edp_deck_read": [C.c_char_p, P(C.c_void_p), P(Params), P(Tables)],
    "edp_deck_initial_plasma": [C.c_void_p, _D, _D, _D, _D, _I32, _D, _I64],
    "edp_deck_ion_emission": [C.c_void_p, C.c_int32, C.c_int32, _D],
    "edp_deck_ion_wall_model": [C.c_void_p, C.c_int32, _I32],
    "edp_deck_electron_emission": [C.c_void_p, C.c_int32, P(SeeParams), _I32],
    "edp_deck_wall_injection": [C.c_void_p, C.c_int32, _D],
    "edp_deck_potential_profile": [C.c_void_p, C.c_int32, _D, P(C.c_int32), P(C.c_int32), P(C.c_float),
                                   P(C.c_int32), P(C.c_int32), P(C.c_float)],
    "edp_deck_potential_series": [C.c_void_p, C.c_int32, C.c_int64, C.c_int64, _D],
    "edp_deck_free": [C.c_void_p],
    "edp_write_snapshot_2d": [C.c_char_p, P(C.c_float), C.c_int32, C.c_int32, C.c_double],
    "edp_write_vdf1d": [C.c_char_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                        C.c_int32, C.c_int32, C.c_int32, C.c_double, _D, _I32, _I32],
    "edp_write_vdf2d": [C.c_char_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                        C.c_double, _I32],
}

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libedipic_b200.so")


def load(path=LIB_PATH):
    """Load the C-ABI library and declare every entry point. Raises OSError when it is missing."""
    if not os.path.exists(path):
        raise OSError(f"libedipic_b200.so not built at {path}: run __graft_entry__.build() or make -C edipic-2d_b200")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    return lib
