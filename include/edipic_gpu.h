/*
 * edipic_gpu.h -- C ABI of the B200 particle cycle of EDIPIC-2D (sm_100a).
 *
 * The reference's hot path is a set of argument-less Fortran subroutines acting on module globals and
 * called from MainProg in a fixed order (src/pic2d_MainProgram.f90:151-309). Each entry point below
 * replaces one of them; the reference routine is cited beside it. A Fortran host binds these functions
 * through ISO_C_BINDING (edipic-2d_b200/fortran/edipic_gpu_mod.f90); every argument is a plain pointer,
 * integer or double.
 *
 * Conventions
 *  - Every function returns EDP_OK (0) or a negative EDP_ERR_* code and never aborts the process.
 *    edp_last_error() returns the message of the last failure on a context.
 *  - Device work is ordered on the context's CUDA stream. Entry points that return host data synchronise;
 *    the others return as soon as their work is queued unless edp_set_sync(ctx, 1) was called.
 *  - Node arrays exchanged with the host use the reference's cluster layout, x fastest:
 *      periodic-x domain : (ncx+2) x (ncy+1) nodes, columns ncx and ncx+1 repeat columns 0 and 1
 *                          (the overlap cell of a self-connected periodic cluster);
 *      walled domain     : (ncx+1) x (ncy+1) nodes.
 *  - Positions are in cells, velocities in cells per time step, fields in E_scale, potentials in F_scale
 *    (pic2d_CurProblemValues.f90:719-723, 893-900).
 *  - One context per GPU and host thread; a context is not thread safe.
 */
#ifndef EDIPIC_GPU_H
#define EDIPIC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EDP_ABI_VERSION 2

enum edp_status {
    EDP_OK = 0,
    EDP_ERR_ARG = -1,            /* invalid argument or configuration */
    EDP_ERR_CUDA = -2,           /* CUDA runtime error (allocation, launch) */
    EDP_ERR_CAPACITY = -3,       /* particle or add-list capacity exceeded on the device */
    EDP_ERR_BOUNDS = -4,         /* a particle was found outside the domain (ADVANCE_* Error-1/-2 checks) */
    EDP_ERR_NOT_CONVERGED = -5,  /* CG did not reach the tolerance within max_it */
    EDP_ERR_TIMEOUT = -6,        /* a bounded device-side wait gave up */
    EDP_ERR_STATE = -7,          /* call out of order (e.g. solve before upload) */
    EDP_ERR_IO = -8              /* deck file missing or malformed */
};

enum edp_precision { EDP_PREC_MIXED = 0, EDP_PREC_FP64 = 1 };
enum edp_solver { EDP_SOLVER_FFTX = 0, EDP_SOLVER_CG = 1 };
enum edp_species { EDP_ELECTRONS = 0, EDP_IONS = 1 /* ion species s is EDP_IONS + s */ };
enum edp_field {
    EDP_FIELD_EX = 0, EDP_FIELD_EY = 1, EDP_FIELD_ACC_EX = 2, EDP_FIELD_ACC_EY = 3,
    EDP_FIELD_PHI = 4, EDP_FIELD_RHO_TOTAL = 5,
    EDP_FIELD_SURFACE_CHARGE = 6   /* charge on the outlines of the dielectric inner objects per node, in macroparticle
                                      charges (whole_object%surface_charge); zero without dielectrics */
};
/* initial guess of edp_field_cg. LEARNED: the previous potential plus the update the loaded network
 * (edp_warmstart_load) predicts from its residual against the new density; the previous potential is kept
 * whenever the prediction's residual is not smaller. The network is also judged by wall time: after the first
 * three LEARNED calls (the network, the network timed, the previous potential timed), the network runs while the
 * solves it started are faster on average than those from the previous potential, else only on every 64th call (to
 * re-measure), and the previous potential starts the others. */
enum edp_warm_start { EDP_WARM_ZERO = 0, EDP_WARM_PREVIOUS = 1, EDP_WARM_USER = 2, EDP_WARM_LEARNED = 3 };
/* preconditioner of edp_field_cg: NONE is Jacobi, which is plain CG here because the operator's diagonal is
 * constant; MG (the default) is one symmetric geometric-multigrid V-cycle per iteration */
enum edp_precond { EDP_PRECOND_NONE = 0, EDP_PRECOND_MG = 1 };

#define EDP_MAX_ION_SPECIES 4
#define EDP_MAX_INNER 4
#define EDP_MAX_COLPROC 8
#define EDP_MAX_SEGMENTS 32

/* Boundary objects: sides 0 below, 1 above, 2 left, 3 right; inner metal rectangles 4.. . */
#define EDP_N_HIT_COUNTERS (4 + EDP_MAX_INNER)

/* Problem description. Values are those of the reference's module data after INITIATE_PARAMETERS
 * (pic2d_CurProblemValues.f90:59-1255); the deck reader below fills it from init_*.dat files. */
typedef struct edp_params {
    int32_t abi_version;            /* EDP_ABI_VERSION */
    int32_t ncx, ncy;               /* cells: period N along x (periodic) or global_maximal_i; global_maximal_j */
    int32_t periodic_x;             /* 1: self-connected periodic cluster with metal walls below/above */
    int32_t n_subcycles;            /* N_subcycles (odd) */
    int32_t n_of_particles_cell;    /* N_of_particles_cell, density normalisation */
    double delta_t_s, delta_x_m;
    double v_scale_ms, e_scale_vm, b_scale_t, f_scale_v;
    double bx, by, bz, ez;          /* uniform external fields, normalised (Bx_ext/B_scale ...) */
    int32_t ions_sense_b, ions_sense_ez;
    int32_t n_ion_species;
    int32_t ion_charge[EDP_MAX_ION_SPECIES];        /* Qs */
    double ion_mass_me[EDP_MAX_ION_SPECIES];        /* Ms = M_i / m_e */
    /* metal boundary potentials (normalised), phi = phi_const + phi_var*sin(omega*T + phase)
       (UPDATE_WALL_POTENTIALS, pic2d_WallPotentials.f90:1-93; omega in rad per step) */
    double wall_phi_const[4], wall_phi_var[4], wall_omega[4], wall_phase[4];
    int32_t n_inner;
    int32_t inner_ileft[EDP_MAX_INNER], inner_jbottom[EDP_MAX_INNER];
    int32_t inner_iright[EDP_MAX_INNER], inner_jtop[EDP_MAX_INNER];
    double inner_phi[EDP_MAX_INNER];
    uint64_t seed;                  /* seed of all device random streams (SplitMix64 decisions, Philox variates) */
    int32_t precision;              /* edp_precision */
    int32_t solver;                 /* edp_solver */
    int32_t sort_every;             /* cell sort period in steps (mixed precision), 0 = never */
    int32_t fuse_collisions;        /* 1: MCC/RCX run in the push epilogue (same variates as the separate pass) */
    int64_t capacity[1 + EDP_MAX_ION_SPECIES];      /* particle slots per species (0 = automatic) */
    /* inner object k: 0 = METAL_WALL (potential inner_phi[k]); > 0 = DIELECTRIC with that permittivity (eps_diel of
       its material): its nodes are unknowns of the CG solve with the face permittivities of SET_EPS_ISHIFTED /
       SET_EPS_JSHIFTED (pic2d_PETSc_Solver.F90:1724-2045) and the particles it absorbs charge its outline
       (DO_ELECTRON_COLL_WITH_INNER_OBJECT, pic2d_ElectronWallCollisions.f90:561-645). CG solver only. */
    double inner_eps[EDP_MAX_INNER];
} edp_params;

/* Collision and sampling tables, as built on the host by INITIATE_ELECTRON_NEUTRAL_COLLISIONS
 * (pic2d_enCollisionsGeneralProc.f90:5-325), INITIATE_ION_NEUTRAL_COLLISIONS
 * (pic2d_inCollisionsGeneralProc.f90:3-90) and PrepareMaxwellDistribIntegral
 * (pic2d_ElectronWallCollisions.f90:835-929). One neutral species. */
typedef struct edp_tables {
    int32_t en_on;                       /* electron-neutral collisions active */
    int32_t n_act;                       /* N_of_activated_colproc */
    int32_t n_seg, n_values;             /* N_of_energy_segments, N_of_energy_values */
    double seg_value[EDP_MAX_SEGMENTS + 1];
    double seg_step[EDP_MAX_SEGMENTS];
    int32_t seg_index[EDP_MAX_SEGMENTS + 1];
    const double* energy_eV;             /* [n_values+1] */
    const double* prob;                  /* prob_colproc_energy, [(n_values+1)*n_act], prob[i*n_act + p-1] */
    double max_colliding_fraction;
    int32_t colproc_type[EDP_MAX_COLPROC];          /* 10, 11, 20, 30 */
    double threshold_eV[EDP_MAX_COLPROC];
    int32_t ion_species_produced[EDP_MAX_COLPROC];  /* 1-based, ionisation only */
    double ion_velocity_factor[EDP_MAX_COLPROC];
    double neutral_mass_amu;
    double energy_factor_eV;             /* 0.5 m_e V_scale^2 / e */
    /* resonant charge exchange per ion species */
    int32_t rcx_on[EDP_MAX_ION_SPECIES];
    double rcx_prob_factor;              /* n_gas * dt * N_subcycles */
    double rcx_sigma_1eV, rcx_alpha;
    double rcx_probab_thermal[EDP_MAX_ION_SPECIES];
    double rcx_vfactor[EDP_MAX_ION_SPECIES];
    /* Maxwellian inverse CDF v(0:R_max) */
    int32_t maxwell_rmax;
    const double* maxwell_v;
} edp_tables;

/* Electron-induced electron emission of one wall material (init_material_<NAME>.dat lines 3-56, read by
 * PREPARE_WALL_MATERIALS, pic2d_Materials.f90:84-149); energies and temperature in eV as in the file. Models:
 * 0 off, 1 constant coefficient between E_min and E_max, 2 the energy- and angle-dependent forms of Coeff_SEE_*
 * (pic2d_SEEmission.f90:1054-1208). */
typedef struct edp_see_params {
    int32_t elastic_model, elastic_type;        /* Emitted_model(1); Elast_refl_type 0 specular, 1 random */
    int32_t inelastic_model, true_model;        /* Emitted_model(2), Emitted_model(3) */
    double elastic_yield, elastic_emin_ev, elastic_emax_ev;                         /* elastic, model 1 */
    double elastic_e0_ev, elastic_emax_coef_ev, elastic_max, elastic_de_ev;        /* elastic, model 2 */
    double elastic_frac_classic;                /* Frac_elast_highenergy */
    double inelastic_yield, inelastic_emin_ev, inelastic_emax_ev;                   /* inelastic, model 1 */
    double inelastic_frac_classic;              /* Frac_inelastic (model 2) */
    double true_t_ev;                           /* T_see_true_eV */
    double true_yield, true_emin_ev, true_emax_ev;                                  /* true secondaries, model 1 */
    double classic_e0_ev, classic_emax_ev, classic_max, classic_k_smooth;          /* model 2 and the classic form */
} edp_see_params;

/* Counters of one step (COLLECT_PARTICLE_BOUNDARY_HITS, collision counters, particle totals). */
typedef struct edp_counters {
    int64_t n_particles[1 + EDP_MAX_ION_SPECIES];           /* live particles */
    int64_t electron_hits[EDP_N_HIT_COUNTERS];              /* whole_object(n)%electron_hit_count, cumulative */
    int64_t ion_hits[EDP_N_HIT_COUNTERS];
    int64_t en_collisions[EDP_MAX_COLPROC];                 /* collision_e_neutral(1)%counter(p), cumulative */
    int64_t rcx_collisions[EDP_MAX_ION_SPECIES];
    int64_t step;                                           /* T_cntr */
    int32_t cg_iterations;                                  /* last CG solve */
    double cg_relres;
    int32_t error_flags;                                    /* device error word (bit set per EDP_ERR_*) */
    int64_t kernel_launches;                                /* kernels this context launched so far */
} edp_counters;

typedef struct edp_ctx edp_ctx;

/* ---- set-up / tear-down ------------------------------------------------------------------------- */
/* after INITIATE_*_COLLISIONS (pic2d_MainProgram.f90:36-60): copies params and tables to the device */
int edp_init(const edp_params* p, const edp_tables* t, edp_ctx** out);
/* end of MainProg (pic2d_MainProgram.f90:414-419) */
int edp_destroy(edp_ctx* ctx);
int edp_last_error(const edp_ctx* ctx, char* buf, size_t len);
int edp_set_sync(edp_ctx* ctx, int sync);
int edp_synchronize(edp_ctx* ctx);
/* the context's CUDA stream (a cudaStream_t), e.g. to record timing events on it */
int edp_get_stream(edp_ctx* ctx, void** stream_out);
/* No counterpart in the reference (it keeps particles in arrival order). Re-sorts every species' particles by tile
 * now (mixed precision; a no-op for FP64) and restarts the sort period counted by the cycle (sort_every). Results
 * do not depend on when sorts happen; this only moves the cost. Synchronises. */
int edp_sort_particles(edp_ctx* ctx);
/* No counterpart in the reference. Kernel of the mixed-precision push over the sorted particles: 0 one CTA per
 * sorted chunk, the threads load their particles; 1 persistent CTAs whose particle columns are streamed into shared
 * memory by bulk copies, 4 particles per thread, 2 stages in flight; 2 the same with 2 particles per thread and 3
 * stages; 3 as 0 with 2 particles per thread (more resident warps); 4 (default) as 0 with each thread's next 4
 * particles copied into shared memory by cp.async while it pushes the current ones. All give the same results;
 * only the speed differs. */
int edp_set_push_kernel(edp_ctx* ctx, int32_t kind);
/* No counterpart in the reference. on = 1 (default): a periodic sort (every sort_every steps) is done by each
 * species' next push, which writes the pushed particles straight to their sorted slots (keys of their cells before
 * the push); on = 0: a separate pass at the end of the step. Same results. */
int edp_set_sort_in_push(edp_ctx* ctx, int32_t on);

/* ---- particles ----------------------------------------------------------------------------------- */
/* after DISTRIBUTE_PARTICLES (pic2d_CurProblemValues.f90:3127-3325) or a checkpoint read: the host's
 * AoS TYPE particle arrays, split into columns. ids may be NULL (then 0..n-1 are assigned). */
int edp_upload_particles(edp_ctx* ctx, int species, int64_t n, const double* x, const double* y,
                         const double* vx, const double* vy, const double* vz, const int32_t* tag,
                         const uint32_t* id);
/* for checkpoints/snapshots: copies live particles back (compacted), n_out receives the count */
int edp_download_particles(edp_ctx* ctx, int species, int64_t cap, int64_t* n_out, double* x, double* y,
                           double* vx, double* vy, double* vz, int32_t* tag, uint32_t* id);
/* DISTRIBUTE_PARTICLES on the device: per_cell particles in every cell, uniform positions, Maxwellian
 * velocities of width factor_convert (sqrt(T_init/T_scale)/N_max_vel [/sqrt(Ms)]), vz zeroed when
 * zero_vz (ions, :3298). Ion species s takes the positions of the electrons when copy_positions. */
int edp_distribute_particles(edp_ctx* ctx, int species, int32_t per_cell, double factor_convert,
                             int32_t zero_vz, int32_t copy_positions_from_electrons);

/* ---- per-step cycle ------------------------------------------------------------------------------ */
/* GATHER_ELECTRON_CHARGE_DENSITY (pic2d_ElectronDynamics.f90:1535-1975) / GATHER_ION_CHARGE_DENSITY
 * (pic2d_IonDynamics.f90:1540-2003). The deposit itself is fused into the pushes; this call only
 * converts the accumulated fixed-point density to FP64 with the periodic fold and wall factors and,
 * when rho_out != NULL, copies it to the host (species EDP_ELECTRONS: c_rho; EDP_IONS: c_rho_i, Qs-weighted). */
int edp_gather_charge_density(edp_ctx* ctx, int species, double* rho_out);
/* UPDATE_WALL_POTENTIALS (pic2d_WallPotentials.f90:1-165) for step T_cntr: every metal wall and metal inner object
 * takes phi_const + (Harmonic_Oscillation + Custom_Waveform) * Amplitude_Profile. Call it for consecutive steps:
 * with an amplitude profile the oscillation's phase is re-anchored at each profile period start. */
int edp_update_wall_potentials(edp_ctx* ctx, int64_t t_cntr);
/* The time dependence of one metal object's potential, as PREPARE_WAVEFORMS and
 * PREPARE_OSCILLATIONS_AMPLITUDE_PROFILE leave it in whole_object (pic2d_Setup.f90:150-412): object 0..3 are the
 * walls (below, above, left, right), 4 + n inner object n. harmonic = {phi_const, phi_var, omega [rad/step],
 * phase [rad]}, normalised; the waveform's n_wf points (wf_T_cntr, wf_phi normalised, REAL) and the amplitude
 * profile's n_ap points (ap_T_cntr, ap_factor, REAL), each 0 for none, times rising from 0 (the last is the
 * period). Without this call walls follow edp_params' harmonic fields and inner objects keep inner_phi. */
int edp_set_potential_profile(edp_ctx* ctx, int32_t object, const double* harmonic, int32_t n_wf,
                              const int32_t* wf_t_cntr, const float* wf_phi, int32_t n_ap, const int32_t* ap_t_cntr,
                              const float* ap_factor);
/* SOLVE_POISSON_FFTX_LINSYSY + CALCULATE_ELECTRIC_FIELD_FFTX_LINSYSY
 * (pic2d_ElectricFieldCalc_FFT_X.f90:3-1547): phi_out may be NULL */
int edp_field_fftx(edp_ctx* ctx, double* phi_out);
/* SOLVE_POTENTIAL_WITH_PETSC + CALCULATE_ELECTRIC_FIELD (pic2d_ElectricFieldCalc_PETSc.F90:7-805,
 * pic2d_PETSc_Solver.F90:31-40): preconditioned CG on the same operator, FP64 dots, until the relative residual
 * |b - A phi| / |b| <= rtol. iters_out receives the first iteration that met rtol (the potential may carry up to
 * one more convergence-check block of iterations). */
int edp_field_cg(edp_ctx* ctx, double rtol, int32_t max_it, int32_t warm_start, int32_t* iters_out);
/* selects the preconditioner of edp_field_cg (edp_precond) */
int edp_set_cg_preconditioner(edp_ctx* ctx, int32_t kind);
/* Ion-induced electron emission of a domain wall (ion-material interaction model 2, pic2d_Materials.f90:150-188;
 * PROCESS_ION_INDUCED_ELECTRON_EMISSION, pic2d_IonEmissions.f90:1-348): ions of ion_species (1-based) absorbed by
 * wall (0 below, 1 above, 2 left, 3 right) with energy in (emin_ev, emax_ev) emit on average `yield` electrons with
 * temperature t_emit_ev, within the ion's energy. The emitted electrons join the electron arrays at the end of the
 * step (edp_end_ion_cycle) and are counted per wall (edp_query_emission). yield 0 switches the wall off. wall 4 + n
 * is inner object n (DO_ION_COLL_WITH_INNER_OBJECT, pic2d_IonWallCollisions.f90:484-575): the electrons leave the
 * side the ion's trajectory crossed first, 1e-6 outside it at the crossing point, and a dielectric object takes +1
 * per emitted electron there besides the ion's charge. */
int edp_set_ion_emission(edp_ctx* ctx, int32_t wall, int32_t ion_species, double yield, double emin_ev,
                         double emax_ev, double t_emit_ev);
/* Ion-material model 1 (pic2d_Materials.f90:159-161): wall (0 below, 1 above, 2 left, 3 right) reflects every ion
 * specularly (INJECT_REFLECTED_ION, pic2d_IonEmissions.f90:374-492). The hit is counted, and the ion returns 1e-6
 * inside the wall with the normal velocity reversed, through the ion add list at the end of the step. Reflection
 * takes precedence over emission on the same wall. on = 0 restores absorption. wall 4 + n is inner object n: the
 * ion returns 1e-6 outside the side it crossed first. */
int edp_set_ion_reflection(edp_ctx* ctx, int32_t wall, int32_t on);
/* Electron-induced electron emission of a domain wall (0 below, 1 above, 2 left, 3 right):
 * PROCESS_ELECTRON_INDUCED_ELECTRON_EMISSION (pic2d_SEEmission.f90:4-151) for every electron the wall absorbs
 * (PROCESS_ELECTRON_COLL_WITH_BOUNDARY_*, pic2d_ElectronWallCollisions.f90:3-287): elastic reflection, inelastic
 * backscattering or true secondaries. The emitted electrons join at the end of the step and are counted with
 * edp_query_emission. wall 4 + n is inner object n (DO_ELECTRON_COLL_WITH_INNER_OBJECT,
 * pic2d_ElectronWallCollisions.f90:561-645): the electrons leave the side crossed first, 1e-6 outside it at the
 * crossing, and a dielectric object takes +1 per electron leaving it besides the absorbed electron's -1.
 * params = NULL, or all three models 0, switches the wall off. Returns EDP_ERR_ARG when a
 * model number is outside 0-2. A wall whose elastic and inelastic coefficients add up to more than 1 at some
 * impact sets the model error (EDP_ERR_STATE from edp_query_counters), where the reference stops. */
int edp_set_electron_emission(edp_ctx* ctx, int32_t wall, const edp_see_params* params);
/* Constant electron emission from a domain wall, PERFORM_ELECTRON_EMISSION_SETUP (pic2d_Setup.f90:599-1001), run by
 * edp_end_ion_cycle every step (pic2d_MainProgram.f90:353): n_per_step macroparticles (the fraction as a
 * probability) uniformly along the wall, 1e-6 inside it; model 0 thermal (normal speed from the flux-weighted
 * half-Maxwellian of temperature t_normal_ev), model 1 a beam of energy beam_energy_ev with energy spread t_normal_ev
 * (beam_energy_ev > 1.5 t_normal_ev, else EDP_ERR_ARG, pic2d_Setup.f90:107-121); tangential components Maxwellian of
 * t_parallel_ev. n_per_step = 0 switches the wall off. wall = 4 + n: metal inner object n
 * (PERFORM_ELECTRON_EMISSION_SETUP_INNER_OBJECTS, pic2d_Setup.f90:1005-1591): each side strictly inside the domain
 * emits REAL(n_per_step) * REAL(open) / REAL(L) per step from its open cells (not covered by a wall or another inner
 * object; L = the open cells of all four sides), 1e-6 outside the side, the normal velocity pointing out; a
 * dielectric object is refused. */
int edp_set_wall_injection(edp_ctx* ctx, int32_t wall, double n_per_step, int32_t model, double t_normal_ev,
                           double t_parallel_ev, double beam_energy_ev);
/* ADVANCE_ELECTRONS (pic2d_ElectronDynamics.f90:3-513), fused with the next step's electron deposit and,
 * when fuse_collisions and this is an ion step, with PERFORM_ELECTRON_NEUTRAL_COLLISIONS */
int edp_advance_electrons(edp_ctx* ctx);
/* ADVANCE_IONS (pic2d_IonDynamics.f90:3-524), fused with the ion deposit and, when fused, with RCX */
int edp_advance_ions(edp_ctx* ctx);
/* PERFORM_ELECTRON_NEUTRAL_COLLISIONS (pic2d_enCollisionsGeneralProc.f90:332-654): a separate pass unless
 * the push already did it; counters_out[p] receives this step's count of process p (may be NULL) */
int edp_collide_en(edp_ctx* ctx, int64_t* counters_out);
/* PERFORM_RESONANT_CHARGE_EXCHANGE (pic2d_inCollisionsSpecificProc.f90:48-126) */
int edp_collide_rcx(edp_ctx* ctx, int64_t* count_out);
/* End of a time step, called every step. On ion steps: PROCESS_ADDED_IONS (pic2d_MainProgram.f90:300,
 * pic2d_IonDynamics.f90:1468-1537), CLEAR_ACCUMULATED_FIELDS (:306, pic2d_ElectricFieldCalc_PETSc.F90:809-829) and
 * PROCESS_ADDED_ELECTRONS (:363, pic2d_ElectronDynamics.f90:1429-1531): the ions and electrons born by this step's
 * ionisations join their arrays and the next step's density. Every step: advances T_cntr and runs the periodic sort. */
int edp_end_ion_cycle(edp_ctx* ctx);
/* Start_T_cntr of a run continued from a checkpoint (READ_CHECKPOINT_POSIX, pic2d_Checkpoints.f90:1002; the loop
 * of pic2d_MainProgram.f90:98 resumes at the saved T_cntr): the next step is t_cntr, at ion sub-cycle n_sub = 0,
 * where checkpoints are taken (:103-108). The step counter keys the device's random streams and the wall
 * potentials. */
int edp_set_step(edp_ctx* ctx, int64_t t_cntr);
/* Several ranks (one GPU each) sharing one cluster's particles, as the reference's processes of a cluster do: each
 * context holds the whole grid and its own share of the particles. After each step (after edp_end_ion_cycle) and
 * after the initial distribution or upload, the caller sums, in place and over the ranks, the accumulators this
 * call lists (the cluster reduce of c_rho, GATHER_ELECTRON_CHARGE_DENSITY pic2d_ElectronDynamics.f90:1641 and
 * GATHER_ION_CHARGE_DENSITY): the densities deposited since the previous call, device buffers of count[k] int64
 * (mixed precision, fixed point, so the sum is exact and order-independent) or FP64 values. The sum must be ordered
 * on the context's stream (edp_get_stream). Every rank then solves the same field. Not with dielectric objects. */
int edp_reduce_list(edp_ctx* ctx, int32_t max, void** ptr, int64_t* count, int32_t* is_int64, int32_t* n_out);
/* ids of the particles the context creates from now on (distribution, upload without ids) start at base
 * (< 2^32); ranks sharing a cluster take disjoint ranges so that their random streams differ. After an upload
 * with ids, particles born later continue after the largest uploaded id, and never below base. */
int edp_set_id_base(edp_ctx* ctx, uint64_t base);
/* The same with the end of the range: ids stay in [base, end), end <= 2^32 (edp_set_id_base takes end = 2^32).
 * Distribution and uploads without ids that need more ids than the range holds return EDP_ERR_CAPACITY. A particle
 * born after the range is used up is not appended (its id would belong to another rank and repeat that particle's
 * random streams); the next edp_query_counters returns EDP_ERR_CAPACITY. */
int edp_set_id_range(edp_ctx* ctx, uint64_t base, uint64_t end);
/* ---- x strips of a domain (the reference's clusters along x, pic2d_ParticleExchange.f90:3-1762; density sums
 * of the shared nodes GATHER_ELECTRON_CHARGE_DENSITY pic2d_ElectronDynamics.f90:1645-1800) ----------------------
 * A strip context covers its own columns plus ghost columns on each side that faces another strip (none on a side
 * that is the domain's wall; in a periodic domain every side faces a strip). It is set up walled in x (CG solver,
 * never used) with ncx = own + ghost_left + ghost_right, mixed precision, metal inner objects only (in its own
 * columns: shifted by -x_first) and no wall emission, then marked with edp_set_strip before any particle is
 * uploaded. Its local column c is global column x_first + c (modulo ncx_global when periodic). Particles that leave
 * the strip and its ghost columns through a side that is not the domain's wall in one step are an error
 * (EDP_ERR_BOUNDS at the next check); walls count their hits as the whole domain does. Per step, for each species:
 * zero the density of a context holding the whole grid (edp_device_buffer), edp_strip_add_density from every strip
 * (sum over ranks), the field solve on the whole grid (edp_field_fftx or edp_field_cg), edp_strip_set_field into
 * every strip, the strip's own advance / collide / end_ion_cycle calls, then edp_strip_take and edp_strip_put to
 * move the particles that ended the step in ghost columns to the neighbour owning them. Their charge was deposited
 * by the sender. */
int edp_set_strip(edp_ctx* ctx, int32_t ghost_left, int32_t ghost_right, int32_t x_first, int32_t ncx_global,
                  int32_t periodic);
/* Takes the particles of species `species` in the left (local columns < ghost_left) and right
 * (>= ncx - ghost_right) ghost columns out of the strip into caller device buffers of records of 8 doubles (x, y in local cells, vx,
 * vy, vz, id, tag, 0): left[cap_left * 8], right[cap_right * 8]; n_left / n_right receive the counts.
 * When a side holds more particles than its buffer, the call returns EDP_ERR_CAPACITY: the first cap records of
 * that side are written and those particles leave the strip, the others stay in their ghost columns, and n_left /
 * n_right receive the whole counts found. The context stays usable; a caller moves the records it got and calls
 * again with buffers of at least the remaining count. Synchronises. */
int edp_strip_take(edp_ctx* ctx, int32_t species, double* left, int64_t cap_left, double* right, int64_t cap_right,
                   int64_t* n_left, int64_t* n_right);
/* Appends n records (device buffer, edp_strip_take's layout) with x shifted by x_shift cells, keeping their ids
 * and tags and depositing nothing. */
int edp_strip_put(edp_ctx* ctx, int32_t species, const double* records, int64_t n, double x_shift);
/* Adds the strip's fixed-point density of one species into global_dev[(ncy + 1) * nx_global] (the internal node
 * layout of the whole-grid context: nx_global = ncx periodic, ncx + 1 walled; column c at (x_first + c) mod
 * nx_global), on the strip's stream. */
int edp_strip_add_density(edp_ctx* ctx, int32_t species, uint64_t* global_dev, int32_t nx_global, int32_t x_first);
/* Copies the strip's columns of a whole-grid field (float2 (Ex, Ey) per node, layout as above) and of its
 * accumulated field for the ions into the strip. */
int edp_strip_set_field(edp_ctx* ctx, const void* e_global_dev, const void* acc_global_dev, int32_t nx_global,
                        int32_t x_first);
/* Device pointer and element count of a context's arrays: which = 0 the fixed-point density of `species`
 * (uint64 per node), 1 the field (float2 per node), 2 the accumulated field of the ions (float2); mixed
 * precision, internal node layout (periodic: ncx columns). */
int edp_device_buffer(edp_ctx* ctx, int32_t which, int32_t species, void** ptr, int64_t* count);

/* One or more whole steps of pic2d_MainProgram.f90:151-309 in order (convenience for drivers). */
int edp_step(edp_ctx* ctx, int32_t nsteps);

/* ---- diagnostics / test access -------------------------------------------------------------------- */
int edp_query_counters(edp_ctx* ctx, edp_counters* out);
/* electrons emitted by ion impacts on each object since the start (out[EDP_N_HIT_COUNTERS], walls first) */
int edp_query_emission(edp_ctx* ctx, int64_t* out);
/* node arrays in the reference layout (see Conventions) */
int edp_get_field(edp_ctx* ctx, int which, double* out);
int edp_set_field(edp_ctx* ctx, int which, const double* in);
/* FP64 sums of report_total_number_of_particles (pic2d_Diagnostics.f90:321-460): N, sum vx, vy, vz,
 * sum vx^2, vy^2, vz^2 for one species */
int edp_moments(edp_ctx* ctx, int species, double out[7]);
/* COLLECT_ELECTRON_MOMENTS (pic2d_ElectronMoments.f90:3-425; what ADVANCE_ELECTRONS_PLUS deposits on a snapshot
 * step, before the push) / COLLECT_ION_MOMENTS (pic2d_IonMoments.f90:3-348) with the current field: 13 node grids
 * in the reference layout, out[m][j][i], m = N, VX, VY, VZ, WX, WY, WZ, VXVY, VXVZ, VYVZ, QX, QY, QZ (cs_N ...
 * cs_QZ after normalisation and ADJUST_DENSITY_AT_WALL_BOUNDARIES). */
int edp_collect_moments(edp_ctx* ctx, int species, float* out);
/* CALCULATE_ELECTRON_VDF / CALCULATE_ION_VDF (pic2d_VelocityDistributions.f90:3-393) for one species (0 electrons,
 * s ions), one cluster over the domain: nbox_x x nbox_y boxes (N_vdfbox_x/y of init_snapshots.dat) splitting
 * [0, c_X_area_max] x [0, ncy], c_X_area_max = ncx (walled) or ncx + 1 (periodic: the overlap node), bins of
 * 1/n_vbins thermal velocities up to +-n_max_vel_s of them (N_vbins_e/i, N_max_vel_e/i); n_max_vel is the deck's
 * velocity scale N_max_vel. vdf1d[3][nbox][2 n_max_vel_s n_vbins] = evxdf, evydf, evzdf (isvxdf.. for ions),
 * box = ibox + jbox nbox_x; vdf2d[nbox][vy bin][vx bin] = evxvydf, or NULL to skip it. skipped receives the
 * number of particles outside the bins (may be NULL). */
int edp_calculate_vdf(edp_ctx* ctx, int species, int32_t n_max_vel, int32_t nbox_x, int32_t nbox_y,
                      int32_t n_max_vel_s, int32_t n_vbins, int32_t* vdf1d, int32_t* vdf2d, int64_t* skipped);
/* No counterpart in the reference (its EEDF comes from the snapshot VDFs of downloaded particles). Counts of the
 * species' particles by kinetic energy in eV, E = |v|^2 energy_factor_eV (times Ms for ions), in the bins
 * [edges_ev[k], edges_ev[k+1]), k < n_bins <= 256; energies outside the edges are not counted. Synchronises. */
int edp_energy_histogram(edp_ctx* ctx, int species, int32_t n_bins, const double* edges_ev, int64_t* counts);
/* kind selection of PERFORM_ELECTRON_NEUTRAL_COLLISIONS (:447-485) evaluated on the device for given
 * (energy, r) pairs: kind_out[k] = indx_coll (n_act+1 = null collision) */
int edp_mcc_choose(edp_ctx* ctx, int64_t n, const double* energy_eV, const double* r, int32_t* kind_out);

/* ---- allocation-free FFT_X solve ------------------------------------------------------------------ */
/* No counterpart in the reference. For callers that cannot allocate device memory (a host whose GPU memory is
 * owned by another runtime or pool, or that must not allocate once running): solves the FFT_X Poisson problem
 * of SOLVE_POISSON_FFTX_LINSYSY for metal walls without any allocation. rho_dev (input) and phi_dev (output)
 * are device buffers of the caller in the periodic reference layout, (ncx+2) x (ncy+1) FP64 nodes x fastest,
 * rho_dev holding factor_rho*(rho_i - rho_e); phi_bottom/phi_top are the normalised wall potentials; stream is
 * a cudaStream_t (NULL = default stream). The workspace is a file-scope device array of
 * EDP_NOALLOC_SCRATCH_BYTES (16 MiB) that every GPU loading this library keeps until exit; (ncy+1)*(ncx/2+1)*24 +
 * ncx*8 bytes plus up to 512 bytes of section alignment must fit in it, else EDP_ERR_CAPACITY. The largest grids
 * that fit: 512 x 2718, 1024 x 1360 (so the 1024 x 1024 grid fits, and 1024 x 1361 does not), 2048 x 680,
 * 4096 x 339 cells. The first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current and keeps it; make that call before any stream capture, and do not call this entry point
 * on a device after cudaDeviceReset (the kept address would be stale). All calls share the array, so calls that
 * overlap on the GPU race: order them on one stream. If a CUDA error from earlier work is pending on the calling
 * thread, the call returns EDP_ERR_CUDA before it queues anything and leaves that error pending. Work is queued on
 * the stream and the call returns without synchronising. */
#define EDP_NOALLOC_SCRATCH_BYTES (16u << 20)
int edp_poisson_fftx_noalloc(int32_t ncx, int32_t ncy, const double* rho_dev, double phi_bottom, double phi_top,
                             double* phi_dev, void* stream);

/* ---- learned warm start of the CG solve ----------------------------------------------------------- */
/* No counterpart in the reference (its PETSc solve always starts from zero). A 4-level convolutional
 * encoder-decoder (channels 32-64-128-256, 3x3 kernels, 4x4 average pooling, nearest upsampling, skip
 * concatenation, ReLU; BF16 weights and activations, FP32 accumulation) maps the residual r0 = b - A phi_prev of
 * the previous potential, divided by its RMS s, and the Dirichlet mask to the update (phi - phi_prev) / s =
 * K o0 + o1 of its two FP32 heads, K = L^2 / (2 pi^2) with L the larger cell count. Each level pools 4 x 4, so the
 * 9 x 9 bottleneck of a 513-node grid (padded to 576) sees the whole domain. blob holds FP32 parameters in
 * the order EDP_WARMSTART_LAYERS lists: per convolution the weights [c_out][3][3][c_in] then the biases [c_out];
 * last the two heads, each weights [3][3][32] and bias. */
#define EDP_WARMSTART_N_CONV 14
#define EDP_WARMSTART_LAYERS {{32, 32}, {32, 32}, {32, 64}, {64, 64}, {64, 128}, {128, 128}, {128, 256}, \
                              {256, 256}, {384, 128}, {128, 128}, {192, 64}, {64, 64}, {96, 32}, {32, 32}}
int edp_warmstart_load(edp_ctx* ctx, const float* blob, int64_t n_floats);
/* the network's forward pass on the current residual: fills guess_out (reference node layout) with
 * phi_prev + predicted update; the residual norms of phi_prev and of the guess go to res_out[0..1] */
int edp_warmstart_predict(edp_ctx* ctx, double* guess_out, double* res_out);
/* the wall-time judge of EDP_WARM_LEARNED: out[4] = {average seconds of the solves the network started (negative:
 * none yet), of those the previous potential started, LEARNED calls, calls on which the network ran} */
int edp_warmstart_timing(edp_ctx* ctx, double* out);

/* Kernels of the network, on caller-owned device memory and a caller stream (cudaStream_t), for training.
 * Activations are NHWC BF16, c1, c2 and c_out multiples of 32 (c2 may be 0: one input tensor). */
int edp_nn_conv3x3_fwd(int32_t nimg, int32_t h, int32_t w, const void* x1, int32_t c1, const void* x2, int32_t c2,
                       const void* wt, const float* bias, int32_t cout, int32_t relu, void* y, void* stream);
int edp_nn_flip_transpose(const void* wt, int32_t cout, int32_t cin, void* out, void* stream);
/* nonzero in *out when a bounded wait of the tensor-core convolution gave up since the last call (then cleared) */
int edp_nn_error(int32_t* out);
/* the forward kernel edp_nn_conv3x3_fwd uses (process-wide): 0 automatic (the persistent halo kernel for layers of at
 * least 296 patches of 8 x 16 pixels with c_out 32 or 64, or 128 when the weights fit in shared memory,
 * 9 c_in c_out 2 <= 112 KiB, else the tile kernel), 1 the tile kernel, 2 the halo kernel (EDP_ERR_ARG where it does
 * not apply). No counterpart in the reference. */
int edp_nn_conv_select(int32_t mode);
int edp_nn_conv3x3_wgrad(int32_t nimg, int32_t h, int32_t w, const void* x1, int32_t c1, const void* x2, int32_t c2,
                         const void* dz, int32_t cout, float* dw, float* db, void* stream);
/* the weight-gradient kernel edp_nn_conv3x3_wgrad uses (process-wide): 0 (default) tcgen05 with the taps stacked in
 * M, 2 tcgen05 with the taps' accumulators side by side in N, 1 mma.sync. No counterpart in the reference. */
int edp_nn_wgrad_select(int32_t mode);
/* f x f average pooling (h, w: input size) and nearest f x upsampling (h, w: output size), f = 2 or 4 */
int edp_nn_pool(int32_t nimg, int32_t h, int32_t w, int32_t c, int32_t f, const void* x, void* y, void* stream);
int edp_nn_pool_bwd(int32_t nimg, int32_t h, int32_t w, int32_t c, int32_t f, const void* dy, void* dx,
                    int32_t accumulate, void* stream);
int edp_nn_upsample(int32_t nimg, int32_t h, int32_t w, int32_t c, int32_t f, const void* x, void* y, void* stream);
int edp_nn_upsample_bwd(int32_t nimg, int32_t h, int32_t w, int32_t c, int32_t cs, int32_t f, const void* dy, void* dx,
                        void* stream);
int edp_nn_relu_bwd(int64_t npix, int32_t c, const void* dy, int32_t cs, int32_t co, const void* dy2, const void* y,
                    void* dz, void* stream);
/* head: the 3x3 convolution to one FP32 output channel; bh points to its bias on the device */
int edp_nn_head_fwd(int32_t nimg, int32_t h, int32_t w, int32_t c, const void* x, const float* wh, const float* bh,
                    float* out, void* stream);
int edp_nn_head_bwd(int32_t nimg, int32_t h, int32_t w, int32_t c, const void* x, const float* wh, const float* dout,
                    void* dx, float* dwh, float* dbh, void* stream);
int edp_nn_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2, float eps,
                int32_t step, void* p_bf16, void* stream);

/* ---- deck reader (host side of INITIATE_PARAMETERS and the collision set-up) --------------------- */
/* Reads init_configuration.dat, init_simcontrol.dat, init_particles.dat, init_extfields.dat,
 * init_bo_NN.dat, init_neutrals.dat, init_neutral_<NAME>.dat, its cross-section files and
 * init_neutral_<NAME>_rcx_param.dat from directory dir (pic2d_CurProblemValues.f90:157-1031,
 * pic2d_ExternalFields.f90:3-195, pic2d_Setup.f90:60-100, pic2d_enCollisionsGeneralProc.f90:5-325,
 * pic2d_inCollisionsGeneralProc.f90:3-90). The deck owns the table arrays that t points into. */
typedef struct edp_deck edp_deck;
int edp_deck_read(const char* dir, edp_deck** out, edp_params* p, edp_tables* t);
/* initial plasma of init_particles.dat: init_Te_eV, init_Ne_m3, init_Ti_eV(s), T_e_eV, N_max_vel ... */
int edp_deck_initial_plasma(const edp_deck* d, double* init_te_ev, double* init_ne_m3, double* init_ti_ev,
                            double* t_e_ev, int32_t* n_max_vel, double* n_plasma_m3, int64_t* max_t_cntr);
/* ion-induced electron emission of wall (0 below, 1 above, 2 left, 3 right; 4 + n inner object n) for ion_species
 * (1-based), from the object's init_material_<NAME>.dat: out = {yield, E_min [eV], E_max [eV], T_emit [eV]}, all 0
 * when the material has no emission (pic2d_Materials.f90:150-188) */
int edp_deck_ion_emission(const edp_deck* d, int32_t wall, int32_t ion_species, double* out);
/* ion-material interaction model of the object's material (0 absorption, 1 specular reflection, 2 ion-induced
 * emission); objects as above */
int edp_deck_ion_wall_model(const edp_deck* d, int32_t wall, int32_t* model);
/* constant electron emission of a wall (0-3) or inner object (4 + n) (init_bo_NN.dat, pic2d_Setup.f90:86-95):
 * out = {N_electron_constant_emit (a REAL: rounded to single precision), model_constant_emit, T_normal [eV],
 * T_parallel [eV], beam energy [eV]} */
int edp_deck_wall_injection(const edp_deck* d, int32_t wall, double* out);
/* electron-induced emission parameters of the object's material (walls 0-3, inner objects 4 + n); *enabled = 1 when any
 * of the three models is on */
int edp_deck_electron_emission(const edp_deck* d, int32_t wall, edp_see_params* out, int32_t* enabled);
/* the time dependence of metal object `object` (0..3 walls, 4 + n inner objects) as the deck sets it up,
 * in edp_set_potential_profile's layout: counts always, arrays when not NULL (call once for the counts) */
int edp_deck_potential_profile(const edp_deck* d, int32_t object, double* harmonic, int32_t* n_wf, int32_t* wf_t_cntr,
                               float* wf_phi, int32_t* n_ap, int32_t* ap_t_cntr, float* ap_factor);
/* UPDATE_WALL_POTENTIALS of that object for steps t0 .. t0 + n - 1 of a run started (or continued, with
 * ADJUST_HARMONIC_OSCILLATIONS_PHASE) at t0, without a device: out[n] */
int edp_deck_potential_series(const edp_deck* d, int32_t object, int64_t t0, int64_t n, double* out);
int edp_deck_free(edp_deck* d);

/* ---- snapshot files (host side of CREATE_SNAPSHOT, pic2d_Snapshots.f90:303-1202), one cluster ---------------- */
/* SAVE_GLOBAL_2D_ARRAY (:1207-1355): gnuplot binary matrix of REAL values; row 0 = {nx_nodes, x_i = i delta_x_m},
 * row 1 + j = {j delta_x_m, arr[j][0 .. nx_nodes - 1]}; arr[ny_nodes][nx_nodes] in the reference node layout */
int edp_write_snapshot_2d(const char* path, const float* arr, int32_t nx_nodes, int32_t ny_nodes, double delta_x_m);
/* SAVE_ALL_VDF1D (:1359-1544) of edp_calculate_vdf's electron and ion histograms (i1d = [n_spec][3][nbox][bins]);
 * x_area_max, y_area_max = the cluster's c_X_area_max, c_Y_area_max in cells */
int edp_write_vdf1d(const char* path, int32_t nbox_x, int32_t nbox_y, double x_area_max, double y_area_max,
                    double delta_x_m, int32_t n_max_vel_e, int32_t n_vbins_e, int32_t n_max_vel_i, int32_t n_vbins_i,
                    int32_t n_spec, double t_e_ev, const double* m_i_amu, const int32_t* e1d, const int32_t* i1d);
/* SAVE_ALL_VDF2D (:1548-1705) of the electron vx-vy histograms */
int edp_write_vdf2d(const char* path, int32_t nbox_x, int32_t nbox_y, double x_area_max, double y_area_max,
                    double delta_x_m, int32_t n_max_vel_e, int32_t n_vbins_e, double t_e_ev, const int32_t* e2d);

#ifdef __cplusplus
}
#endif
#endif /* EDIPIC_GPU_H */
