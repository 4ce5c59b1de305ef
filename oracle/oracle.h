/*
 * ORACLE (test infrastructure only): CPU FP64 restatement of EDIPIC-2D's per-step particle cycle.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load liboracle.so.
 * The product library never links or calls it.
 *
 * Every function cites the reference routine it restates (paths relative to the EDIPIC-2D tree).
 */
#ifndef EDIPIC_ORACLE_H
#define EDIPIC_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- random numbers (oracle_rng.c) */
typedef struct { uint32_t v[624]; int i; } oracle_well_t;
void   oracle_well_set_state(oracle_well_t* s, const uint32_t* words, int index);
void   oracle_well_seed(oracle_well_t* s, int32_t seed);
double oracle_well_next(oracle_well_t* s);
void   oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
uint64_t oracle_mix64(uint64_t z);
uint64_t oracle_splitmix64_at(uint64_t s0, uint64_t n);
void   oracle_splitmix64_stream(uint64_t s0, int64_t count, uint64_t* out);

/* ---------------------------------------------------------------- geometry
 * Node (i,j) of the reference's cluster arrays, one cluster covering the whole domain.
 *  periodic != 0 : self-connected periodic-x cluster, nodes i = 0..ncx+1 (node ncx+1 overlaps node 1,
 *                  node 0 overlaps node ncx), metal walls at j = 0 (object 0) and j = ncy (object 1).
 *  periodic == 0 : walls on four sides, nodes i = 0..ncx; objects 0 below, 1 above, 2 left, 3 right.
 *  inner objects k = 0..n_inner-1 are metal rectangles [ileft,iright]x[jbottom,jtop] (object 4+k).
 */
typedef struct {
    int32_t ncx, ncy, periodic, n_inner;
    int32_t ileft[4], jbottom[4], iright[4], jtop[4];
} oracle_geom_t;

int32_t oracle_nx_nodes(const oracle_geom_t* g);   /* ncx+2 (periodic) or ncx+1 */

/* external fields and species constants (normalised as in pic2d_ExternalFields.f90:75-110) */
typedef struct {
    double bx, by, bz, ez;      /* B in units of B_scale, Ez in E_scale */
    int32_t is_ion;             /* 0 electrons, 1 ions */
    double qm2;                 /* ions: QM2s = 0.5*Qs/Ms */
    int32_t nsub;               /* N_subcycles */
    int32_t ions_sense_b, ions_sense_ez;
} oracle_species_t;

/* particle array in SoA FP64 form, the reference's TYPE particle split into columns */
typedef struct {
    int64_t n;
    double *x, *y, *vx, *vy, *vz;
    int32_t* tag;
    uint32_t* id;
} oracle_parts_t;

/* ADVANCE_ELECTRONS (pic2d_ElectronDynamics.f90:3-513) / ADVANCE_IONS (pic2d_IonDynamics.f90:3-524):
 * one push of every particle with the field (EX,EY) on the node grid, wall/inner-object absorption with
 * swap-with-last removal (REMOVE_ELECTRON :517-555) and hit counting per object. */
void oracle_push(const oracle_geom_t* g, const oracle_species_t* sp, const double* EX, const double* EY,
                 oracle_parts_t* p, int64_t* hits);

/* oracle_push that also records each domain-wall absorption (objects 0-3) as 7 doubles
 * {wall, X, Y, vx, vy, vz, id}: the position after the move (X wrapped on the periodic cluster) and the pushed
 * velocity, in push order; at most cap rows, *n_hit receives the number of absorptions. */
void oracle_push_hits(const oracle_geom_t* g, const oracle_species_t* sp, const double* EX, const double* EY,
                      oracle_parts_t* p, int64_t* hits, double* hit_rows, int64_t cap, int64_t* n_hit);

/* CIC deposit of GATHER_ELECTRON_CHARGE_DENSITY (pic2d_ElectronDynamics.f90:1597-1639) into rho
 * (zeroed here), scaled by weight (ions: Qs). No fold, no wall factors. */
void oracle_deposit(const oracle_geom_t* g, const oracle_parts_t* p, double weight, double* rho);
/* periodic fold (:1661-1667) and wall factors (:1802-1880) */
void oracle_fold_and_wall_scale(const oracle_geom_t* g, double* rho);
/* COLLECT_ELECTRON_MOMENTS (pic2d_ElectronMoments.f90:3-425) / COLLECT_ION_MOMENTS (pic2d_IonMoments.f90:3-348)
 * with the overlap fold, normalisation and ADJUST_DENSITY_AT_WALL_BOUNDARIES: out[13 * nodes] (N, VX, VY, VZ,
 * WX, WY, WZ, VXVY, VXVZ, VYVZ, QX, QY, QZ); EX/EY are used for electrons only. */
void oracle_collect_moments(const oracle_geom_t* g, const oracle_species_t* sp, const double* EX, const double* EY,
                            const oracle_parts_t* p, double* out);

/* CALCULATE_ELECTRON_VDF / CALCULATE_ION_VDF (pic2d_VelocityDistributions.f90:3-393) for one cluster over
 * [0, xmax] x [0, ymax]: nbx x nby boxes, bins INT(v fvc) (minus one for v < 0) in [vmin, -vmin - 1];
 * h1[3][nbox][reclen] counts vx, vy, vz, h2[nbox][vy][vx] (may be NULL), reclen = -2 vmin. Returns the number of
 * skipped particles. h1/h2 are zeroed here. */
int64_t oracle_vdf(const oracle_parts_t* p, int32_t nbx, int32_t nby, double xmax, double ymax, double fvc,
                   int32_t vmin, int32_t* h1, int32_t* h2);

/* ---------------------------------------------------------------- Maxwell sampler */
/* PrepareMaxwellDistribIntegral (pic2d_ElectronWallCollisions.f90:835-929); v[0..9000], v_inj[0..4500] */
void   oracle_maxwell_tables(double* v, double* v_inj);
/* GetMaxwellVelocity (:961-985) driven by one uniform variate */
double oracle_maxwell_sample(const double* v, double u);

/* ---------------------------------------------------------------- ion-induced electron emission */
/* one ion species at the four domain walls (0 below, 1 above, 2 left, 3 right), in code units
 * (pic2d_Materials.f90:165-188): yield between emin and emax (energies Ms v^2), fconv = sqrt(T_emit/T_e)/N_max_vel */
typedef struct {
    int32_t on[8];   /* the walls 0 below, 1 above, 2 left, 3 right, then inner object n at 4 + n */
    double yield[8], emin[8], emax[8], fconv[8];
    double ms;
    uint32_t species;            /* 0-based ion species */
    const double* maxwell_v;     /* v[0..9000] */
    const double* maxwell_inj;   /* v_inj[0..4500] */
} oracle_emit_t;
/* PROCESS_ION_INDUCED_ELECTRON_EMISSION and INJECT_ION_IMPACT_EXTRACTED_ELECTRON (pic2d_IonEmissions.f90:1-348)
 * for an ion absorbed by `wall` at (x, y) (PROCESS_ION_COLL_WITH_BOUNDARY_*, pic2d_IonWallCollisions.f90:63-303,
 * clamps the coordinate along the wall into [0, xmax] x [0, ymax] first; done here) with velocity v. Writes the
 * emitted electrons as rows {x, y, vx, vy, vz} (room for cap rows) and returns their number. Variates:
 * Philox4x32-10, key {id, seed_lo}, counter {step, 0x45450000 + species, block, seed_hi}; block 0 word 0 draws
 * the fractional part of the yield, block 1 + e words 0, 1, 2 the normal speed of electron e (GetInjMaxwellVelocity)
 * and its two tangential components (GetMaxwellVelocity) in x, y, z order. */
int32_t oracle_ion_emission(const oracle_emit_t* em, int32_t wall, double x, double y, double vx, double vy,
                            double vz, uint32_t id, uint64_t seed, uint32_t step, double xmax, double ymax,
                            double* out, int32_t cap);
/* the same for object `obj` (0..7) emitting from a surface given by INJECT_ION_IMPACT_EXTRACTED_ELECTRON's dirflag
 * (1 normal +x, 2 -y, 3 -x, 4 +y) at coordinate `at`, from the point (x, y) on it (no clamping) */
int32_t oracle_ion_emission_face(const oracle_emit_t* em, int32_t obj, int32_t dirflag, double at, double x, double y,
                                 double vx, double vy, double vz, uint32_t id, uint64_t seed, uint32_t step,
                                 double* out, int32_t cap);

/* electron-induced emission of one domain wall, in code units (PREPARE_WALL_MATERIALS, pic2d_Materials.f90:84-244) */
typedef struct {
    int32_t m_el, m_in, m_tr, refl_random;
    double el_yield, el_emin, el_emax, el_e0, el_emaxc, el_max, el_de, el_frac;
    double in_yield, in_emin, in_emax, in_frac;
    double tr_yield, tr_emin, tr_emax;
    double cl_e0, cl_emax, cl_max, cl_k;
    double lowest, fconv;
    const double* maxwell_v;     /* v[0..9000] */
    const double* maxwell_inj;   /* v_inj[0..4500] */
} oracle_see_t;
/* PROCESS_ELECTRON_INDUCED_ELECTRON_EMISSION (pic2d_SEEmission.f90:4-151) with INJECT_ELASTIC_REFLECTED_ELECTRON,
 * INJECT_INELASTIC_BACKSCATTERED_ELECTRON, INJECT_TRUE_SECONDARY_ELECTRON and the Coeff_SEE_* functions for an
 * electron absorbed by `wall` at (x, y) (clamped along the wall here) with velocity v: rows {x, y, vx, vy, vz} of the
 * emitted electrons (room for cap), returns their number or -1 when elastic + inelastic coefficients exceed 1.
 * Variates: Philox4x32-10, key {id, seed_lo}, counter {step, 0x53450000, block, seed_hi}: block 0 words 0-3 = the
 * process choice R, the two angle variates, the backscattered speed variate or the fractional true yield; block
 * 1 + e = true secondary e (normal speed, two tangential components). */
int32_t oracle_see(const oracle_see_t* w, int32_t wall, double x, double y, double vx, double vy, double vz,
                   uint32_t id, uint64_t seed, uint32_t step, double xmax, double ymax, double* out, int32_t cap);
/* the same from the surface given by dirflag (1 normal +x, 2 -y, 3 -x, 4 +y) at coordinate `at` (no clamping) */
int32_t oracle_see_face(const oracle_see_t* w, int32_t dirflag, double at, double x, double y, double vx, double vy,
                        double vz, uint32_t id, uint64_t seed, uint32_t step, double* out, int32_t cap);

/* PERFORM_ELECTRON_EMISSION_SETUP (pic2d_Setup.f90:599-1001) of one domain wall for one cluster over
 * [0, xmax] x [0, ymax]: INT(n) electrons plus one with probability n - INT(n), uniform along the wall, 1e-6 inside;
 * model 0 normal speed GetInjMaxwellVelocity * fn, model 1 MAX(0, vb + GetMaxwellVelocity * fn); tangential
 * GetMaxwellVelocity * fp. Variates: Philox4x32-10, key {0xE1000000 + wall, seed_lo}, counter {step, 0x43450000,
 * block, seed_hi}; block 0 word 0 the fraction; block 1 + e words 0-3: place, normal, tangential (in-plane), z.
 * Rows {x, y, vx, vy, vz}; returns the count. */
int32_t oracle_wall_injection(double n, int32_t model, double fn, double fp, double vb, int32_t wall, uint32_t step,
                              uint64_t seed, double xmax, double ymax, const double* maxwell_v,
                              const double* maxwell_inj, double* out, int32_t cap);

/* PERFORM_ELECTRON_EMISSION_SETUP_INNER_OBJECTS (pic2d_Setup.f90:1005-1591) of metal inner object n for one cluster
 * over the domain: each side strictly inside the cluster emits REAL(N) * REAL(open) / REAL(L) per step (integer
 * part, then one more with that probability), open = its cells not covered by a wall or another inner object inside
 * [cross_min, cross_max), L = the open cells of the four sides; places by the walk over the open cells, 1e-6
 * outside the side, normal velocity out. Variates as oracle_wall_injection with key 0xE1000000 + 4 + 4 n + (m - 1)
 * for side m (1 left, 2 top, 3 right, 4 bottom). Rows {x, y, vx, vy, vz} (at most cap); per_side[4] the counts;
 * returns the total. */
int32_t oracle_inner_injection(const oracle_geom_t* g, int32_t n, double n_emit, int32_t model, double fn, double fp,
                               double vb, uint32_t step, uint64_t seed, const double* maxwell_v,
                               const double* maxwell_inj, double* out, int32_t cap, int32_t* per_side);

/* INJECT_REFLECTED_ION (pic2d_IonEmissions.f90:374-492) for a domain wall: the ion returns 1e-6 inside the wall
 * (coordinate along the wall clamped into the domain) with its normal velocity reversed; out = {x, y, vx, vy, vz} */
void oracle_ion_reflect(int32_t wall, double x, double y, double vx, double vy, double vz, double xmax, double ymax,
                        double* out);

/* ---------------------------------------------------------------- electron-neutral collisions */
typedef struct {
    int32_t n_points;
    const double* energy_eV;
    const double* crsect_m2;
    int32_t type;               /* 10, 11, 20, 30 */
} oracle_crsect_t;

typedef struct {
    int32_t n_act, n_seg, n_values;
    double seg_value[33];       /* energy_segment_boundary_value(0:n_seg) */
    double seg_step[32];        /* energy_segment_step(1:n_seg) -> [0..n_seg-1] */
    int32_t seg_index[33];      /* energy_segment_boundary_index(0:n_seg) */
    double* energy_eV;          /* [n_values+1], caller-owned */
    double* prob;               /* [(n_values+1) * n_act], prob[i*n_act + (p-1)], caller-owned */
    double max_colliding_fraction;
    int32_t type[8];
    double threshold_eV[8];
} oracle_mcc_table_t;

/* frequency_of_en_collision (pic2d_enCollisionsSpecificProc.f90:4-57) */
double oracle_en_frequency(const oracle_crsect_t* cs, double energy_eV, double n_m3, int32_t nsub, double dt_s);
/* INITIATE_ELECTRON_NEUTRAL_COLLISIONS table part (pic2d_enCollisionsGeneralProc.f90:236-322).
 * tab->seg_* must be set; tab->energy_eV / tab->prob must point to arrays of the right size
 * (query the size with oracle_mcc_n_values first). */
int32_t oracle_mcc_n_values(int32_t n_seg, const double* seg_value, const double* seg_step);
void oracle_mcc_build(oracle_mcc_table_t* tab, int32_t n_act, const oracle_crsect_t* cs,
                      double n_m3, int32_t nsub, double dt_s);
/* collision kind selection of PERFORM_ELECTRON_NEUTRAL_COLLISIONS (:447-485): returns indx_coll in 1..n_act,
 * or n_act+1 for the null collision */
int32_t oracle_mcc_choose(const oracle_mcc_table_t* tab, double energy_eV, double r);

/* scattering of en_Collision_* (pic2d_enCollisionsSpecificProc.f90:61-639) given its uniform variates.
 * kind 10/11/20: u[0] angle, u[1] azimuth. kind 30: u[0] ejected energy, u[1..2] scattered electron angles,
 * u[3..4] ejected electron angles, u[5..7] ion Maxwellian. Returns 1 when a new electron+ion were produced
 * (their velocities in new_e[3], new_i[3]), 0 otherwise. v[3] is updated in place. */
int32_t oracle_en_scatter(int32_t kind, double energy_eV, double threshold_eV, double neutral_mass_amu,
                          double ion_velocity_factor, const double* maxwell_v, const double* u,
                          double* v, double* new_e, double* new_i);

/* Per-particle null-collision MCC with the variate layout shared with the GPU kernels:
 *   decision draws: SplitMix64 seeded with mix64(seed ^ 0x4D430000) at position (step << 32) | id: {select = high
 *   half, kind r = low half};
 *   scattering variates: Philox4x32-10, key = {id, seed_lo}, counter = {step, 0, block 1/2, seed_hi};
 *   u = (x + 0.5) * 2^-32.
 * Ionisation products are appended to *born_e / *born_i (capacity checked). counters[k] counts kind k+1. */
typedef struct {
    uint64_t seed;
    uint32_t step;
    double energy_factor_eV;   /* m_e V_scale^2 / (2 e) */
    double neutral_mass_amu;
    double ion_velocity_factor;
    const double* maxwell_v;
} oracle_mcc_ctx_t;
void oracle_mcc_philox(const oracle_mcc_table_t* tab, const oracle_mcc_ctx_t* c, oracle_parts_t* e,
                       oracle_parts_t* born_e, oracle_parts_t* born_i, int64_t cap_born, int64_t* counters);

/* PERFORM_RESONANT_CHARGE_EXCHANGE (pic2d_inCollisionsSpecificProc.f90:48-126): hit variate = high half of the
 * SplitMix64 decision draw of stream 0x52430000 | species (seeded with mix64(seed ^ tag), position (step << 32) | id),
 * Maxwellian from Philox4x32-10 block 1 of stream 1 + (species << 8). Returns the number of exchanges. */
typedef struct {
    double prob_factor;        /* ngas * dt * N_subcycles */
    double v_scale_ms;
    double factor_eV;          /* Ms * energy_factor_eV */
    double sigma_1eV, alpha;
    double probab_thermal;     /* calculate_thermal_cx_probab :4-31 */
    double vfactor;
} oracle_rcx_t;
double oracle_rcx_probab_thermal(double sigma_1eV, double alpha, double T_K, double n_m3, double Ms,
                                 double dt_s, int32_t nsub);
int64_t oracle_rcx_philox(const oracle_rcx_t* r, const oracle_mcc_ctx_t* c, uint32_t species, oracle_parts_t* ions);

/* ---------------------------------------------------------------- field solvers */
/* SOLVE_POISSON_FFTX_LINSYSY (pic2d_ElectricFieldCalc_FFT_X.f90:3-1320) for the periodic geometry:
 * rho_total = factor_rho*(rho_i - rho_e) on the reference node grid (after fold/wall factors);
 * phi_bottom/phi_top the metal wall potentials (normalised). Output phi on the node grid
 * (columns ncx, ncx+1 filled with the periodic copies). */
void oracle_fftx_solve(const oracle_geom_t* g, const double* rho_total, double phi_bottom, double phi_top, double* phi);

/* CALCULATE_ELECTRIC_FIELD_FFTX_LINSYSY (:1324-1547) and CALCULATE_ELECTRIC_FIELD (ElectricFieldCalc_PETSc.F90:360-805):
 * E = -grad(phi) * factor, central inside, one-sided on walls; acc += E when acc_ex != NULL. */
void oracle_efield(const oracle_geom_t* g, const double* phi, double factor2, double factor1,
                   double* ex, double* ey, double* acc_ex, double* acc_ey);

/* The PETSc operator of SolverInitialization (pic2d_PETSc_Solver.F90:42-1350) for eps = 1 with metal walls and
 * metal inner objects (Dirichlet identity rows) and the RHS of SOLVE_POTENTIAL_WITH_PETSC
 * (ElectricFieldCalc_PETSc.F90:38-186), solved in FP64 by CG on the Dirichlet-eliminated SPD system.
 * phi holds the initial guess on entry (node grid); returns iterations, or -1 if not converged. */
int32_t oracle_cg_solve(const oracle_geom_t* g, const double* rho_total, const double* wall_phi /*4*/,
                        const double* inner_phi, double rtol, int32_t max_it, double* phi, double* relres_out);

/* the CG solve with dielectric inner objects: inner_eps[n] > 0 makes object n a dielectric of that permittivity
 * (its nodes unknowns, the faces weighted as SET_EPS_ISHIFTED/JSHIFTED, pic2d_PETSc_Solver.F90:1724-2045) */
int32_t oracle_cg_solve_eps(const oracle_geom_t* g, const double* rho_total, const double* wall_phi,
                            const double* inner_phi, const double* inner_eps, double rtol, int32_t max_it, double* phi,
                            double* relres_out);
/* TRY_ELECTRON_COLL_WITH_INNER_OBJECT / TRY_ION_COLL_WITH_INNER_OBJECT and DO_*_COLL_WITH_INNER_OBJECT
 * (pic2d_ElectronWallCollisions.f90:470-742, pic2d_IonWallCollisions.f90:391-560): the first crossing of the
 * trajectory (x - vx*xmul, y - vy*xmul) -> (x, y) with an inner object's outline, and the charge q (-1 electrons,
 * Qs ions) split over the two outline nodes next to it when that object is a dielectric (inner_eps > 0), added to
 * surf on the node grid. Returns the object, -1 when the trajectory crosses none. */
int32_t oracle_inner_hit(const oracle_geom_t* g, const double* inner_eps, double x, double y, double vx, double vy,
                         double xmul, double q, double* surf);
/* its two parts: the crossing (object returned; segment m 1 left, 2 top, 3 right, 4 bottom; crossing point) and the
 * charge q on the outline nodes next to a crossing */
int32_t oracle_inner_cross(const oracle_geom_t* g, double x, double y, double vx, double vy, double xmul,
                           int32_t* m_out, double* xc_out, double* yc_out);
void oracle_inner_charge(const oracle_geom_t* g, int32_t n_do, int32_t mcross, double xcross, double ycross, double q,
                         double* surf);

/* ---------------------------------------------------------------- whole cycle (CPU baseline) */
typedef struct {
    oracle_geom_t geom;
    oracle_species_t e_sp, i_sp;
    double factor_rho;          /* 1/N_of_particles_cell */
    double ion_charge;          /* Qs */
    double factor2_E, factor1_E;
    double phi_bottom, phi_top;
    const oracle_mcc_table_t* mcc;
    oracle_mcc_ctx_t mcc_ctx;
    oracle_rcx_t rcx;
    int32_t rcx_on;
    int32_t nthreads;
    /* add lists of this step's ionisations; both join their arrays at the end of the step
       (PROCESS_ADDED_IONS, pic2d_MainProgram.f90:300; PROCESS_ADDED_ELECTRONS, :363) */
    oracle_parts_t born_e, born_i;
    int64_t cap_born;
    uint32_t next_id_e, next_id_i;  /* id of the next particle that joins (max id + 1 at the start) */
    int32_t n_sub_phase;            /* n_sub of MainProg: electron steps since the last ion step (0 at the start) */
} oracle_cycle_t;

/* one electron step in the order of pic2d_MainProgram.f90:151-363. The ion density is gathered only when
 * n_sub == 0 (:151), the electron density every step; FFT_X solve; E, with acc_E += E (CALCULATE_ELECTRIC_FIELD_*);
 * electron push. On the ion step (n_sub + 1 == N_subcycles, :196) the ions are pushed on acc_E with QM2sNsub and
 * X += V N_subcycles (ADVANCE_IONS, pic2d_IonDynamics.f90:86-155), then MCC, RCX, the born ions and electrons
 * join, acc_E is cleared (CLEAR_ACCUMULATED_FIELDS) and n_sub returns to 0. Particle arrays must have room for the
 * appended particles (cap). work[9 * node grid] keeps rho_i and acc_E between calls. Returns particles pushed. */
int64_t oracle_cycle_step(oracle_cycle_t* c, oracle_parts_t* e, oracle_parts_t* i, int64_t cap_e, int64_t cap_i,
                          double* work /* 9 * node grid */, int64_t* counters /* [16] */);

#ifdef __cplusplus
}
#endif
#endif
