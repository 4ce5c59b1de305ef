// Internal definitions of the EDIPIC-2D B200 particle cycle: device context, random streams and the
// collision arithmetic shared by the fused and the separate collision passes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/edipic_gpu.h"
#include "../host/potentials.h"

#define EDP_MAX_SPECIES (1 + EDP_MAX_ION_SPECIES)

// tile geometry of the mixed-precision push: particles are sorted tile by tile; a CTA stages the
// field and accumulates the density of its tile plus a halo of HALO cells in shared memory.
#define EDP_TILE 16
#define EDP_HALO 2
#define EDP_WIN_CELLS (EDP_TILE + 2 * EDP_HALO)
#define EDP_WIN_NODES (EDP_WIN_CELLS + 1)
#define EDP_CHUNK 8192          // particles per CTA work item inside one tile
// CG runs in blocks of iterations (the host reads the residual norms back once per block); a block keeps its
// scalars (r.z, p.Ap, r.r after each iteration) in one of two areas, the previous block's in the other
#define EDP_CG_CHECK_MG 2
#define EDP_CG_CHECK_PLAIN 8
#define EDP_CG_AREA (4 * EDP_CG_CHECK_PLAIN + 4)
#define EDP_CG_SCALARS (2 + 2 * EDP_CG_AREA)
#define EDP_PUSH_THREADS 256
#define EDP_ITEMS 4             // particles per thread per iteration (128-bit loads)

// fixed-point density scale: one macroparticle = 2^32 units
#define EDP_FIX_ONE 4294967296.0
#define EDP_FIX_INV 2.3283064365386962890625e-10

// device error word bits
#define EDP_EFLAG_CAPACITY 1
#define EDP_EFLAG_BOUNDS 2
#define EDP_EFLAG_PENDING 4
#define EDP_EFLAG_TIMEOUT 8   // a bounded device-side wait gave up
#define EDP_EFLAG_SEE_MODEL 16   // elastic + inelastic emission coefficients above 1 at some electron impact
#define EDP_EFLAG_IDS 32         // a born particle found the context's id range used up (not appended)

struct edp_chunk {      // one CTA work item of the sorted push
    int64_t start, end; // slot range
    int32_t wx0, wy0;   // window origin (cells), tile origin minus halo
};

// device-resident per-step scalars and counters (one allocation, read back by edp_query_counters)
struct edp_dev_counters {
    unsigned long long n_slots[EDP_MAX_SPECIES];   // high-water slot count (append cursor)
    unsigned long long n_live[EDP_MAX_SPECIES];
    unsigned long long e_hits[EDP_N_HIT_COUNTERS];
    unsigned long long e_emit[EDP_N_HIT_COUNTERS];   // electrons emitted by each object (ion impacts)
    unsigned long long i_hits[EDP_N_HIT_COUNTERS];
    unsigned long long en_coll[EDP_MAX_COLPROC];
    unsigned long long en_coll_step[EDP_MAX_COLPROC];
    unsigned long long rcx[EDP_MAX_ION_SPECIES];
    unsigned long long rcx_step[EDP_MAX_ION_SPECIES];
    unsigned long long born_e_count;               // electrons born by ionisation this step
    unsigned long long hit_count;                  // records in the wall-hit list
    unsigned long long born_i_count[EDP_MAX_ION_SPECIES];
    unsigned long long next_id[EDP_MAX_SPECIES];
    unsigned int error_flags;
    unsigned int pad;
    double cg_scalars[8];                           // rr, pAp, rr_new, bnorm2, ...
};

struct edp_species_mixed {
    int32_t* cell = nullptr;   // cell (j << 16) | i, -1 dead
    float *ox = nullptr, *oy = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;
    uint32_t* id = nullptr;
    int32_t* tag = nullptr;
};

// sort key of a mixed-precision particle in slot k: its 16 x 16-cell tile, then (k / 32) mod 256, so that runs of 32
// source slots stay together and runs interleave inside a tile (see sort.cu)
__device__ __forceinline__ uint32_t edp_tile_key(int cell, int64_t k, int ntx)
{
    int i = cell & 0xFFFF, j = cell >> 16;
    return ((uint32_t)((j >> 4) * ntx + (i >> 4)) << 8) | (uint32_t)((k >> 5) & 255);
}

// Programmatic dependent launch for chains of short dependent kernels (the CG and multigrid kernels of a solve, the
// convolutions of a network pass): a kernel launched by edp_launch_dependent may become resident while the kernel
// before it in the stream is still running. Its first statement is edp_dependent_start(): it waits until that kernel
// has completed and its writes are visible (griddepcontrol.wait, which returns at once for a kernel launched without
// the attribute), then lets the kernel after it be launched (griddepcontrol.launch_dependents; that launch happens
// once every CTA of this grid has said so or exited, so a waiting dependent never holds resources that a CTA of this
// grid still needs).
__device__ __forceinline__ void edp_dependent_start()
{
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
template <typename... KArgs, typename... Args>
inline cudaError_t edp_launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                        Args&&... args)
{
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args&&>(args)...);
}

// the lanes of the (full) warp holding the same key as this lane; a run of 32 sorted slots mostly shares one key,
// which a shuffle and a vote settle without the slower match
__device__ __forceinline__ unsigned edp_warp_peers(uint32_t key)
{
    const uint32_t k0 = __shfl_sync(0xFFFFFFFFu, key, 0);
    return __all_sync(0xFFFFFFFFu, key == k0) ? 0xFFFFFFFFu : __match_any_sync(0xFFFFFFFFu, key);
}

struct edp_species_fp64 {
    double *x = nullptr, *y = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;  // x < -1e29: dead
    uint32_t* id = nullptr;
    int32_t* tag = nullptr;
};

// born particles waiting to join a main array (FP64 in both precisions; small)
struct edp_born {
    double *x = nullptr, *y = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;
    int64_t cap = 0;
};

// wall hits of the species being pushed while its walls emit or reflect: position, velocity, id, wall | species << 8
// (the electron push fills it for electron-induced emission, the ion push for the ion-wall interactions; each push
// is followed by the kernel that consumes and clears it)
struct edp_hits {
    double *x = nullptr, *y = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;
    uint32_t* id = nullptr;
    int32_t* ws = nullptr;
    int64_t cap = 0;
};

struct edp_mcc_dev;
struct edp_warmstart;   // learned warm start of the CG solve (warmstart.cu)
struct edp_emit_dev;    // ion-induced electron emission parameters (below)
struct edp_see_dev;     // electron-induced electron emission parameters (below)

// constant electron emission of the four domain walls (PERFORM_ELECTRON_EMISSION_SETUP), code units
// sides of the inner objects that emit: side 4 n + (m - 1) of inner object n, m = 1 left, 2 top, 3 right, 4 bottom
// (the segment numbers of PERFORM_ELECTRON_EMISSION_SETUP_INNER_OBJECTS)
#define EDP_INJECT_SIDES (4 * EDP_MAX_INNER)
#define EDP_INJECT_MAX_CELLS 65536   // open cells over all sides
struct edp_inject_dev {
    double n[EDP_N_HIT_COUNTERS];       // walls: N_electron_constant_emit, macroparticles per step
    int model[EDP_N_HIT_COUNTERS];      // 0 thermal, 1 beam (walls, then inner objects)
    double fn[EDP_N_HIT_COUNTERS], fp[EDP_N_HIT_COUNTERS];   // factor_convert_vinj_normal/parallel_constant_emit
    double vb[EDP_N_HIT_COUNTERS];      // v_ebeam_constant_emit
    double side_n[EDP_INJECT_SIDES];    // inner objects: macroparticles per step from the side (0: none)
    double side_at[EDP_INJECT_SIDES];   // X (sides 1, 3) or Y (2, 4) of the emitted electrons, 1e-6 outside
    int side_open[EDP_INJECT_SIDES];    // open (not covered) cells of the side in [cmin, cmax)
    int side_off[EDP_INJECT_SIDES];     // their first entry in open_cells
    int side_cmin[EDP_INJECT_SIDES], side_cmax[EDP_INJECT_SIDES];   // cross_j/i_min, cross_j/i_max
    const int* open_cells;              // cell index along the side (j for sides 1, 3; i for 2, 4), by side
    const double* maxwell_v;
    const double* maxwell_inj;
    int rmax, rmax_inj;
};

// one level of the multigrid preconditioner: (nx+1) x (ny+1) nodes, x fastest, spacing 2^level
#define EDP_MG_MAX_LEVELS 16
struct edp_mg_level {
    int32_t nx = 0, ny = 0;
    double* u = nullptr;      // correction (level 0: the preconditioned residual z)
    double* f = nullptr;      // right-hand side (level 0: the CG residual r)
    int8_t* mask = nullptr;   // 1: Dirichlet node, correction fixed at 0
};

// add lists as seen by the kernels
struct edp_born_dev {
    edp_born born_e;
    edp_born born_i[EDP_MAX_ION_SPECIES];
};

// constant parameters handed to kernels by value
struct edp_kparams {
    int32_t ncx, ncy, periodic, nxg, nyg;     // nxg = node columns stored (ncx periodic, ncx+1 walled)
    int32_t n_inner;
    int32_t ileft[EDP_MAX_INNER], jbottom[EDP_MAX_INNER], iright[EDP_MAX_INNER], jtop[EDP_MAX_INNER];
    int32_t nsub;
    uint32_t seed_lo, seed_hi;
    int32_t diel_mask;                        // bit n: inner object n is a dielectric
    int32_t ion_inner_mask;                   // bit n: inner object n emits electrons under ion impact or reflects ions
    int32_t see_inner_mask;                   // bit n: inner object n emits electrons under electron impact
    int32_t strip;                            // 1: one x strip of a domain (edp_set_strip)
    int32_t strip_gl, strip_gr;               // ghost columns on its left / right; 0: that side is the domain's wall
    int32_t strip_x0, strip_ncx;              // global column of local column 0, columns of the whole domain
    int32_t strip_periodic;                   // the whole domain is periodic in x
};

struct edp_ctx {
    edp_params p;
    edp_kparams kp;
    std::string last_error;
    cudaStream_t stream = nullptr;
    int device = 0;
    int sync = 0;
    int64_t t_cntr = 0;           // T_cntr
    int32_t n_sub_phase = 0;      // n_sub of MainProg
    int32_t nspec = 1;            // electrons + ion species
    int64_t cap[EDP_MAX_SPECIES] = {0};
    int64_t host_slots[EDP_MAX_SPECIES] = {0};   // host-side upper bound of n_slots
    int64_t sorted_end[EDP_MAX_SPECIES] = {0};   // slots [0, sorted_end) are tile-sorted
    int64_t steps_since_sort = 0;
    int sort_due[EDP_MAX_SPECIES] = {0};   // the next push of the species sorts it (fused_sort)
    int32_t fused_sort = 1;                // periodic sorts inside the push (1) or as a separate pass (0)
    uint64_t id_base = 0;             // first id of the particles this context creates (distribution, upload)
    uint64_t id_end = 1ull << 32;     // one past the last id of the context's range (edp_set_id_range)
    uint32_t dirty = 0;               // bit s: species s's density was deposited since the last edp_reduce_list
    int uploaded[EDP_MAX_SPECIES] = {0};

    // particles
    edp_species_mixed pm[EDP_MAX_SPECIES], pm_alt[EDP_MAX_SPECIES];
    edp_species_fp64 pd[EDP_MAX_SPECIES];
    edp_born born_e;              // ionisation electrons of this step (joined at the end of the step)
    edp_born born_i[EDP_MAX_ION_SPECIES];
    int64_t born_cap = 0;

    // sort
    edp_chunk* chunks[EDP_MAX_SPECIES] = {nullptr};
    int64_t n_chunks[EDP_MAX_SPECIES] = {0};
    int64_t chunk_cap[EDP_MAX_SPECIES] = {0};
    uint32_t* sort_count = nullptr;   // per-cell counters (ncells + 1)
    unsigned long long* sort_offset = nullptr;
    unsigned long long* scan_tmp = nullptr;
    int32_t ntx = 0, nty = 0;         // tiles

    // grids
    float2* E2 = nullptr;             // mixed: (EX, EY) per node, FP32
    float2* acc2 = nullptr;           // mixed: accumulated field for ions
    double *Ex = nullptr, *Ey = nullptr, *accx = nullptr, *accy = nullptr;   // FP64 field
    unsigned long long* rho_fix[EDP_MAX_SPECIES] = {nullptr};   // mixed: fixed-point density per species
    double* rho_d[EDP_MAX_SPECIES] = {nullptr};                  // FP64 path density per species
    double* rho_total = nullptr;      // factor_rho*(rho_i - rho_e) with wall factors
    double* phi = nullptr;
    double* phi_prev = nullptr;
    double2* spec = nullptr;          // FFT_X spectrum [nyg][nm]
    double* aeq = nullptr;            // a_eq [nm][nyg]
    double2* twiddle = nullptr;       // exp(+2 pi i k / N), k < N/2
    int32_t nm = 0;
    // CG workspace
    double *cg_b = nullptr, *cg_r = nullptr, *cg_p = nullptr, *cg_Ap = nullptr, *cg_z = nullptr;
    int8_t* cg_kind = nullptr;        // 0 unknown, 1 Dirichlet
    double* cg_sc = nullptr;          // CG scalars: |b|^2, r.r before iteration 0, two areas of block scalars
    cudaGraphExec_t cg_exec[2][3] = {};   // [multigrid][first block, odd block, even block]: captured iterations
    int64_t cg_exec_launches[2][3] = {};  // kernels in each captured block
    unsigned long long* strip_cnt = nullptr;   // left / right record counts of edp_strip_take
    int32_t precond = 1;              // edp_precond
    int32_t mg_nlev = 0, mg_lc = 0;   // multigrid levels; levels >= mg_lc run inside one CTA
    edp_mg_level mg[EDP_MG_MAX_LEVELS];
    size_t mg_smem = 0;               // shared memory of the coarse-level kernel
    double* mg_cinv = nullptr;        // inverse of the coarsest level's operator (mg_cn x mg_cn), or null
    int32_t* mg_cidx = nullptr;       // node index of each coarsest-level unknown
    int32_t mg_cn = 0;
    edp_warmstart* ws = nullptr;      // network of the learned warm start, once loaded
    edp_emit_dev* emit_dev = nullptr; // ion-induced electron emission (device copy of emit_h)
    edp_emit_dev* emit_h = nullptr;   // host copy
    edp_hits hits;                    // wall hits of the current push
    int emit_on = 0;                  // ion wall hits are recorded: some wall emits or reflects ions
    edp_see_dev* see_dev = nullptr;   // electron-induced electron emission (device copy of see_h)
    edp_see_dev* see_h = nullptr;
    int see_on = 0;                   // electron wall hits are recorded
    double *epsx = nullptr, *epsy = nullptr;   // face permittivities (dielectric inner objects), node-indexed
    unsigned long long* surf = nullptr;        // surface charge of the dielectric outlines per node, 2^32 units
    edp_inject_dev inject{};          // constant electron emission (by value into the kernel)
    int inject_on = 0;
    double* maxwell_inj = nullptr;    // GetInjMaxwellVelocity table on the device
    int* inject_cells = nullptr;      // open cells of the emitting sides of inner objects (edp_inject_dev)
    int32_t last_ws_used = 0;         // the last CG solve started from the network's guess
    // wall time of learned-start solves (the network ran) and of previous-start ones, running averages in seconds
    // (negative: none yet), and the learned-start calls so far: the network runs while it pays, and is re-tried on
    // every 64th call once it does not
    double ws_t_net = -1.0, ws_t_prev = -1.0;
    int64_t ws_calls = 0, ws_runs = 0;
    int32_t last_cg_iters = 0;
    double last_cg_relres = 0.0;
    double last_cg_relres0 = 0.0;     // relative residual of the initial guess

    // tables
    double* mcc_prob = nullptr;
    double* mcc_energy = nullptr;
    double* maxwell_v = nullptr;
    edp_mcc_dev* mcc_dev = nullptr;  // device copy of the collision table descriptor
    edp_born_dev* born_dev = nullptr; // device copy of the add-list descriptors
    uint32_t* sel_list = nullptr;     // electron slots selected for a collision in the fused push
    unsigned long long* sel_count = nullptr;
    int64_t sel_cap = 0;
    edp_tables tab;                   // scalar part (pointers are host pointers; device copies above)
    int32_t host_n_act = 0;

    edp_dev_counters* dc = nullptr;   // device counters
    edp_dev_counters* hc = nullptr;   // pinned host mirror

    // constant Boris rotation matrices (uniform B): [0] electrons, [1+s] ion species
    double K[EDP_MAX_SPECIES][9];
    void* dev_small = nullptr;        // 4 KB device block for kernel pointer tables
    double phi_wall[4];               // current wall potentials (normalised)
    double phi_inner[EDP_MAX_INNER];  // current potentials of the metal inner objects (normalised)
    EdpPotentialProfile pot[4 + EDP_MAX_INNER];   // their time dependence (walls by side, then inner objects)
    int64_t launches = 0;             // kernels launched (reported by edp_query_counters)
    // mixed push over the sorted chunks: 0 one CTA per chunk with the threads' own loads; 1 persistent CTAs with
    // bulk-copy staging, 4 particles per thread, 2 stages; 2 the same with 2 particles per thread, 3 stages; 3 as 0
    // with 2 particles per thread; 4 (default, measured 1.5 % faster than 0 at cfg1) as 0 with each thread's next
    // particles copied ahead by cp.async
    int32_t push_kernel = 4;
};

// ------------------------------------------------------------------------------------------ Philox
__host__ __device__ inline void edp_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                           uint32_t k1, uint32_t out[4])
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

// The per-particle collision decision draws: SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014), the generator whose state after n steps is s0 + n * gamma and whose output is the
// mix64 finaliser of that state, evaluated at position n = (step << 32) | id of the stream seeded by
// s0 = mix64(seed ^ tag). One draw per particle and step, keyed by (id, step) and independent of the slot order, like
// the Philox variates; with the stream's position of id 0 computed once per launch (edp_draw_base) a draw costs one
// 32 x 64-bit and two 64-bit multiplies where Philox2x32-10 takes ten dependent 32-bit rounds, and the push makes one
// for every particle. Word 0 of a draw is its high half, word 1 its low half.
#define EDP_SPLITMIX_GAMMA 0x9E3779B97F4A7C15ull
__host__ __device__ inline uint64_t edp_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// the state of the decision stream `tag` at position (step << 32) with id 0 (one per launch)
__host__ __device__ inline uint64_t edp_draw_base(uint32_t seed_lo, uint32_t seed_hi, uint32_t tag, uint32_t step)
{
    const uint64_t s0 = edp_mix64((((uint64_t)seed_hi << 32) | seed_lo) ^ tag);
    return s0 + ((uint64_t)step << 32) * EDP_SPLITMIX_GAMMA;
}
// the draw of particle `id` at the position that `base` names
__host__ __device__ inline uint64_t edp_draw(uint64_t base, uint32_t id)
{
    return edp_mix64(base + (uint64_t)id * EDP_SPLITMIX_GAMMA);
}

// stream tags of the decision draws
#define EDP_SEL_MCC 0x4D430000u
#define EDP_SEL_RCX(s) (0x52430000u | (uint32_t)(s))

// uniform in (0,1), exactly representable: (x + 1/2) 2^-32
__host__ __device__ inline double edp_u01(uint32_t x) { return ((double)x + 0.5) * 2.3283064365386962890625e-10; }

// random streams (counter word 1)
#define EDP_STREAM_MCC 0u
#define EDP_STREAM_RCX(s) (1u + ((uint32_t)(s) << 8))
#define EDP_STREAM_INIT(sp) (2u + ((uint32_t)(sp) << 8))
#define EDP_STREAM_EMIT(s) (0x45450000u + (uint32_t)(s))   // ion-induced electron emission, ion species s
#define EDP_STREAM_SEE 0x53450000u                          // electron-induced electron emission
#define EDP_STREAM_INJECT 0x43450000u                       // constant electron emission of the walls
#define EDP_INJECT_KEY 0xE1000000u                          // Philox key word 0 of wall w's injection: KEY + w

// --------------------------------------------------------------------------- collision tables (device)
struct edp_mcc_dev {
    const double* prob;       // [(n_values+1) * n_act]
    const double* energy;     // [n_values+1]
    const double* maxwell_v;  // [rmax+1]
    int32_t n_act, n_seg, n_values, rmax;
    double seg_value[EDP_MAX_SEGMENTS + 1];
    double seg_step[EDP_MAX_SEGMENTS];
    int32_t seg_index[EDP_MAX_SEGMENTS + 1];
    double pmax;
    unsigned long long pmax_x;              // (x + 1/2) 2^-32 < pmax  <=>  x < pmax_x, for 32-bit Philox words x
    int32_t type[EDP_MAX_COLPROC];
    double thr[EDP_MAX_COLPROC];
    int32_t ion_species[EDP_MAX_COLPROC];   // 0-based, -1 none
    double ion_vfactor[EDP_MAX_COLPROC];
    double mass_amu, energy_factor;
    int32_t on;
};

struct edp_rcx_dev {
    const double* maxwell_v;
    int32_t on, rmax;
    double prob_factor, v_scale, factor_eV, sigma_1eV, alpha, pth2, vfactor;
    double k2;   // (n_gas dt N_sub sigma V_scale)^2, the energy-independent factor when alpha == 0
};

// GetMaxwellVelocity (pic2d_ElectronWallCollisions.f90:961-985)
__device__ inline double edp_maxwell(const double* v, int rmax, double u)
{
    double R = rmax * u;
    int indx = (int)R;
    if (indx < rmax) return __ldg(&v[indx]) + (R - indx) * (__ldg(&v[indx + 1]) - __ldg(&v[indx]));
    return __ldg(&v[rmax]);
}

// kind selection of PERFORM_ELECTRON_NEUTRAL_COLLISIONS (pic2d_enCollisionsGeneralProc.f90:451-485) with the
// arithmetic spelled out in round-to-nearest intrinsics, so it matches the oracle bit for bit.
__device__ inline int edp_mcc_choose_dev(const edp_mcc_dev& m, double E, double r)
{
    int indx;
    double a0, a1;
    if (E >= m.seg_value[m.n_seg]) {
        indx = m.n_values - 1;
        a1 = 1.0;
        a0 = 0.0;
    } else if (E < m.seg_value[0]) {
        indx = 0;
        a1 = 0.0;
        a0 = 1.0;
    } else {
        int seg = 1;
        for (int i = m.n_seg - 1; i >= 0; --i)
            if (E >= m.seg_value[i]) {
                seg = i + 1;
                break;
            }
        double step = m.seg_step[seg - 1];
        double fi = __dadd_rn((double)m.seg_index[seg - 1], __ddiv_rn(__dsub_rn(E, m.seg_value[seg - 1]), step));
        indx = (int)fi;
        indx = max(0, min(indx, m.n_values - 1));
        a1 = __ddiv_rn(__dsub_rn(E, __ldg(&m.energy[indx])), step);
        a0 = __dsub_rn(1.0, a1);
    }
    const int na = m.n_act;
    int k;
    for (k = na; k >= 1; --k) {
        double thr = __fma_rn(a1, __ldg(&m.prob[(int64_t)(indx + 1) * na + k - 1]),
                              __dmul_rn(a0, __ldg(&m.prob[(int64_t)indx * na + k - 1])));
        if (r > thr) break;
    }
    return k + 1;
}

__device__ inline void edp_rotate(double cosk, double sink, double cosf, double sinf, double Vx, double Vy,
                                  double Vz, double& ox, double& oy, double& oz)
{
    double V = sqrt(Vx * Vx + Vy * Vy + Vz * Vz);
    double Vxy = sqrt(Vx * Vx + Vy * Vy);
    if (Vxy > 1.0e-20) {
        double a = Vx / Vxy, b = Vy / Vxy;
        ox = Vx * cosk + (sinf * V * b + cosf * Vz * a) * sink;
        oy = Vy * cosk - (sinf * V * a - cosf * Vz * b) * sink;
        oz = Vz * cosk - Vxy * cosf * sink;
    } else {
        ox = fabs(Vz) * sink * cosf;
        oy = fabs(Vz) * sink * sinf;
        oz = Vz * cosk;
    }
}

__device__ inline double edp_okh(double e, double R)
{
    double c = 1.0 - 2.0 * R / (1.0 + 8.0 * (e / 27.21) * (1.0 - R));
    return fmax(fmin(0.999999999999, c), -0.999999999999);
}

// result of one electron's MCC test
struct edp_mcc_out {
    int kind_index;   // 0 none, else 1..n_act (counted)
    int born;         // ionisation produced an electron + ion
    double ne[3], ni[3];
    int ion_species;
};

// Selection of PERFORM_ELECTRON_NEUTRAL_COLLISIONS as a per-electron Bernoulli(P_max) test. The decision draw of the
// electron (stream EDP_SEL_MCC): word 0 is the selection variate, word 1 the kind variate r. Returns r when selected.
__device__ __forceinline__ bool edp_mcc_select(const edp_mcc_dev* m, uint32_t id, uint32_t step, uint32_t seed_lo,
                                               uint32_t seed_hi, double& r)
{
    const uint64_t z = edp_draw(edp_draw_base(seed_lo, seed_hi, EDP_SEL_MCC, step), id);
    if ((unsigned long long)(uint32_t)(z >> 32) >= m->pmax_x) return false;
    r = edp_u01((uint32_t)z);
    return true;
}

// Kind choice and scattering of one selected electron (en_Collision_*, pic2d_enCollisionsSpecificProc.f90:61-639),
// blocks 1-2 of Philox stream 0 hold the scattering variates. Out of line: it runs for P_max of the electrons.
static __device__ __noinline__ void edp_mcc_collide(const edp_mcc_dev* mp, uint32_t id, uint32_t step,
                                                    uint32_t seed_lo, uint32_t seed_hi, double r, double* v,
                                                    edp_mcc_out* out)
{
    const edp_mcc_dev& m = *mp;
    edp_mcc_out& o = *out;
    o.kind_index = 0;
    o.born = 0;
    double vx = v[0], vy = v[1], vz = v[2];
    double v2 = __fma_rn(vz, vz, __fma_rn(vy, vy, __dmul_rn(vx, vx)));
    double E = __dmul_rn(v2, m.energy_factor);
    int ki = edp_mcc_choose_dev(m, E, r);
    if (ki > m.n_act) return;
    int kind = m.type[ki - 1];
    double thr = m.thr[ki - 1];
    if ((kind == 20 || kind == 30) && E <= thr) return;
    uint32_t b1[4], b2[4];
    edp_philox(step, EDP_STREAM_MCC, 1u, seed_hi, id, seed_lo, b1);
    double u0 = edp_u01(b1[0]), u1 = edp_u01(b1[1]), u2 = edp_u01(b1[2]), u3 = edp_u01(b1[3]);
    double ox, oy, oz;
    o.kind_index = ki;
    if (kind == 10 || kind == 11) {
        double c = (kind == 10) ? edp_okh(E, u0) : fmax(fmin(0.999999999999, 1.0 - 2.0 * u0), -0.999999999999);
        double ks = acos(c), s = sin(ks), fi = u1 * 6.28318530718;
        edp_rotate(c, s, cos(fi), sin(fi), vx, vy, vz, ox, oy, oz);
        double alpha = sqrt(1.0 - (0.001097161 / m.mass_amu) * (1.0 - c));
        v[0] = ox * alpha;
        v[1] = oy * alpha;
        v[2] = oz * alpha;
        return;
    }
    if (kind == 20) {
        double esc = fmax(0.0, E - thr);
        double c = edp_okh(esc, u0);
        double ks = acos(c), s = sin(ks), fi = u1 * 6.28318530718;
        edp_rotate(c, s, cos(fi), sin(fi), vx, vy, vz, ox, oy, oz);
        double alpha = sqrt(esc / E);
        v[0] = ox * alpha;
        v[1] = oy * alpha;
        v[2] = oz * alpha;
        return;
    }
    // ionisation, B = 10 eV (pic2d_enCollisionsSpecificProc.f90:451-629)
    edp_philox(step, EDP_STREAM_MCC, 2u, seed_hi, id, seed_lo, b2);
    double u4 = edp_u01(b2[0]), u5 = edp_u01(b2[1]), u6 = edp_u01(b2[2]), u7 = edp_u01(b2[3]);
    const double B = 10.0;
    double eej = B * tan(u0 * atan(0.5 * (E - thr) / B));
    eej = fmax(0.0, fmin(eej, 0.5 * (E - thr)));
    double esc = fmax(0.0, E - thr - eej);
    double csc = edp_okh(esc, u1), ksc = acos(csc), ssc = sin(ksc), fsc = u2 * 6.28318530718;
    double cej = edp_okh(eej, u3), kej = acos(cej), sej = sin(kej), fej = u4 * 6.28318530718;
    edp_rotate(csc, ssc, cos(fsc), sin(fsc), vx, vy, vz, ox, oy, oz);
    double asc = sqrt(esc / E);
    v[0] = ox * asc;
    v[1] = oy * asc;
    v[2] = oz * asc;
    edp_rotate(cej, sej, cos(fej), sin(fej), vx, vy, vz, ox, oy, oz);
    double aej = sqrt(eej / E);
    o.ne[0] = ox * aej;
    o.ne[1] = oy * aej;
    o.ne[2] = oz * aej;
    double f = m.ion_vfactor[ki - 1];
    o.ni[0] = edp_maxwell(m.maxwell_v, m.rmax, u5) * f;
    o.ni[1] = edp_maxwell(m.maxwell_v, m.rmax, u6) * f;
    o.ni[2] = edp_maxwell(m.maxwell_v, m.rmax, u7) * f;
    o.ion_species = m.ion_species[ki - 1];
    o.born = (o.ion_species >= 0) ? 1 : 0;
}

// PERFORM_ELECTRON_NEUTRAL_COLLISIONS + en_Collision_* for one electron (the separate passes)
__device__ inline edp_mcc_out edp_mcc_electron(const edp_mcc_dev* m, uint32_t id, uint32_t step, uint32_t seed_lo,
                                               uint32_t seed_hi, double& vx, double& vy, double& vz)
{
    edp_mcc_out o;
    o.kind_index = 0;
    o.born = 0;
    double r;
    if (!edp_mcc_select(m, id, step, seed_lo, seed_hi, r)) return o;
    double v[3] = {vx, vy, vz};
    edp_mcc_collide(m, id, step, seed_lo, seed_hi, r, v, &o);
    vx = v[0];
    vy = v[1];
    vz = v[2];
    return o;
}

// PERFORM_RESONANT_CHARGE_EXCHANGE (pic2d_inCollisionsSpecificProc.f90:90-121) for one ion; true on exchange.
// The test r <= sqrt(P^2 + P_th^2), P = n dt N_sub |v| V_scale sigma(E), is evaluated as r^2 <= P^2 + P_th^2.
// the same with the decision word w0 (word 0 of the ion's decision draw in stream EDP_SEL_RCX(species)) drawn by the
// caller
__device__ __forceinline__ bool edp_rcx_ion_drawn(const edp_rcx_dev& r, uint32_t w0, uint32_t id, uint32_t step,
                                                  uint32_t species, uint32_t seed_lo, uint32_t seed_hi, double& vx,
                                                  double& vy, double& vz);
__device__ __forceinline__ bool edp_rcx_ion(const edp_rcx_dev& r, uint32_t id, uint32_t step, uint32_t species,
                                            uint32_t seed_lo, uint32_t seed_hi, double& vx, double& vy, double& vz)
{
    const uint64_t z = edp_draw(edp_draw_base(seed_lo, seed_hi, EDP_SEL_RCX(species), step), id);
    return edp_rcx_ion_drawn(r, (uint32_t)(z >> 32), id, step, species, seed_lo, seed_hi, vx, vy, vz);
}
__device__ __forceinline__ bool edp_rcx_ion_drawn(const edp_rcx_dev& r, uint32_t w0, uint32_t id, uint32_t step,
                                                  uint32_t species, uint32_t seed_lo, uint32_t seed_hi, double& vx,
                                                  double& vy, double& vz)
{
    double vsq = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
    double k2 = r.k2;
    if (r.alpha != 0.0) {
        double l = __dsub_rn(1.0, __dmul_rn(r.alpha, log(fmax(__dmul_rn(vsq, r.factor_eV), 0.001))));
        double k = __dmul_rn(__dmul_rn(r.prob_factor, __dmul_rn(__dmul_rn(r.sigma_1eV, l), l)), r.v_scale);
        k2 = __dmul_rn(k, k);
    }
    double p2 = __dadd_rn(__dmul_rn(k2, vsq), r.pth2);
    double u = edp_u01(w0);
    if (!(__dmul_rn(u, u) <= p2)) return false;
    uint32_t b[4];
    edp_philox(step, EDP_STREAM_RCX(species), 1u, seed_hi, id, seed_lo, b);
    vx = edp_maxwell(r.maxwell_v, r.rmax, edp_u01(b[0])) * r.vfactor;
    vy = edp_maxwell(r.maxwell_v, r.rmax, edp_u01(b[1])) * r.vfactor;
    vz = edp_maxwell(r.maxwell_v, r.rmax, edp_u01(b[2])) * r.vfactor;
    return true;
}

// --------------------------------------------------------------------------------- host helpers
int edp_fail(edp_ctx* c, int code, const std::string& msg);
// Raises a kernel's dynamic shared memory limit to at least `bytes`. The limit belongs to the kernel for the whole
// process, so a context that needs less never lowers what another context set.
int edp_raise_smem_limit(edp_ctx* c, const void* kernel, size_t bytes);
int edp_cuda_check(edp_ctx* c, cudaError_t e, const char* what);
#define EDP_CUDA(ctx, call)                                            \
    do {                                                               \
        cudaError_t _e = (call);                                       \
        if (_e != cudaSuccess) return edp_cuda_check((ctx), _e, #call); \
    } while (0)
#define TRY(x)                       \
    do {                             \
        int _r = (x);                \
        if (_r != EDP_OK) return _r; \
    } while (0)

edp_mcc_dev edp_make_mcc_dev(const edp_ctx* c);
edp_rcx_dev edp_make_rcx_dev(const edp_ctx* c, int s);

// kernels launched from edp_api.cu, defined in the other translation units
int edp_launch_push(edp_ctx* c, int species, bool ion_step, bool fuse);
int edp_launch_ion_emission(edp_ctx* c);
int edp_launch_electron_emission(edp_ctx* c);
int edp_launch_wall_injection(edp_ctx* c);
int edp_launch_collide_en(edp_ctx* c);
int edp_launch_collide_rcx(edp_ctx* c);
int edp_launch_append_born(edp_ctx* c);
int edp_launch_sort(edp_ctx* c, int species);
// the sort done by the next push of a species (edp_end_ion_cycle marks it due): the histogram and scans of the
// pre-push keys (edp_sort_prepare), the push writing every particle to its sorted slot in the other arrays, then
// edp_sort_finish (slot count, swap, chunk list)
int edp_sort_prepare(edp_ctx* c, int species, unsigned long long** cursor);
int edp_sort_finish(edp_ctx* c, int species);
int edp_launch_density(edp_ctx* c);
int edp_launch_fftx(edp_ctx* c);
int edp_launch_efield(edp_ctx* c);
int edp_launch_cg(edp_ctx* c, double rtol, int max_it, int warm, int* iters);
int edp_mg_setup(edp_ctx* c);                                  // level hierarchy and masks (CG contexts)
int edp_mg_apply(edp_ctx* c, const double* r, double* z);     // z = M^-1 r, one symmetric V-cycle
void edp_mg_free(edp_ctx* c);
void edp_warmstart_free(edp_ctx* c);
int edp_warmstart_forward(edp_ctx* c, const double* rr0);   // guess from the residual in cg_r
int edp_warmstart_residual(edp_ctx* c);                     // residual of the guess
const double* edp_warmstart_rr(edp_ctx* c);                 // device |r|^2 of the guess
cudaError_t edp_warmstart_accept(edp_ctx* c, double* rr_dst);
const double* edp_warmstart_guess(edp_ctx* c);
int edp_launch_distribute(edp_ctx* c, int species, int per_cell, double factor_convert, int zero_vz, int copy_pos);
int edp_launch_upload(edp_ctx* c, int species, int64_t n, const double* dx, const double* dy, const double* dvx,
                      const double* dvy, const double* dvz, const int32_t* dtag, const uint32_t* did);
int edp_launch_download(edp_ctx* c, int species, int64_t cap, int64_t* n_out, double* x, double* y, double* vx,
                        double* vy, double* vz, int32_t* tag, uint32_t* id);
int edp_launch_moments(edp_ctx* c, int species, double out[7]);
int edp_launch_mcc_choose(edp_ctx* c, int64_t n, const double* E, const double* r, int32_t* out);
int edp_fields_prepare(edp_ctx* c);   // one-time FFT/CG tables
int edp_dielectrics_setup(edp_ctx* c); // face permittivities and the surface-charge grid (dielectric inner objects)
int edp_launch_deposit(edp_ctx* c, int species);   // CIC deposit of the whole array without a push

// ------------------------------------------------------------------------------ ion-induced electron emission
// Parameters of PROCESS_ION_INDUCED_ELECTRON_EMISSION (pic2d_IonEmissions.f90:1-56) for the four domain walls
// (0 below, 1 above, 2 left, 3 right) and each ion species, as read from init_material_*.dat
// (pic2d_Materials.f90:165-188): a constant yield for impact energies in (emin, emax), energies in the code's units
// (an ion's energy is Ms v^2, an electron's v^2), and the velocity factor sqrt(T_emit / energy_factor_eV) of the
// emitted electrons (= sqrt(T_emit / T_e) / N_max_vel, :188).
struct edp_emit_dev {
    // per object: the four domain walls (0 below, 1 above, 2 left, 3 right), then inner object n at 4 + n
    int reflect[EDP_N_HIT_COUNTERS];   // ion-material model 1: the object reflects every ion specularly
    int on[EDP_N_HIT_COUNTERS][EDP_MAX_ION_SPECIES];
    double yield[EDP_N_HIT_COUNTERS][EDP_MAX_ION_SPECIES];
    double emin[EDP_N_HIT_COUNTERS][EDP_MAX_ION_SPECIES], emax[EDP_N_HIT_COUNTERS][EDP_MAX_ION_SPECIES];
    double fconv[EDP_N_HIT_COUNTERS][EDP_MAX_ION_SPECIES];
    double ms[EDP_MAX_ION_SPECIES];
    const double* maxwell_v;   // GetMaxwellVelocity table, rmax + 1 values
    const double* maxwell_inj; // GetInjMaxwellVelocity table, rmax_inj + 1 values
    int rmax, rmax_inj;
};

// GetInjMaxwellVelocity (pic2d_ElectronWallCollisions.f90:933-957) driven by one uniform variate
__device__ inline double edp_maxwell_inj(const double* v, int rmax, double u)
{
    double R = rmax * u;
    int indx = (int)R;
    if (indx < rmax) return __ldg(&v[indx]) + (R - indx) * (__ldg(&v[indx + 1]) - __ldg(&v[indx]));
    return __ldg(&v[rmax]);
}

// One electron emitted with a thermal velocity into the domain from wall `wall` at (x, y) (INJECT_ION_IMPACT_
// EXTRACTED_ELECTRON, pic2d_IonEmissions.f90:91-348, and INJECT_TRUE_SECONDARY_ELECTRON, pic2d_SEEmission.f90:794-1050,
// for the domain walls): 1e-6 inside the wall, normal speed from the injection table (variate w0), tangential
// components from the Maxwell table (w1, w2) in x, y, z order, all times f, then scaled down to the energy left
// (`energy`, which the electron's energy reduces). Returns false, emitting nothing, when no energy is left.
// The emitting surface: its outward normal (0 +y, 1 -y, 2 +x, 3 -x: the domain wall below, above, left, right, or an
// inner object's top, bottom, right, left side) and its coordinate along that normal
struct edp_face {
    int dir;
    double at;
};
__device__ __forceinline__ edp_face edp_wall_face(int wall, double xmax, double ymax)
{
    edp_face f;
    f.dir = wall;
    f.at = wall == 0 ? 0.0 : wall == 1 ? ymax : wall == 2 ? 0.0 : xmax;
    return f;
}

__device__ inline bool edp_emit_thermal(const double* maxwell_v, int rmax, const double* maxwell_inj, int rmax_inj,
                                        edp_face face, double x, double y, double f, double& energy,
                                        const uint32_t w[4], double& nx, double& ny, double v[3])
{
    if (energy <= 0.0) return false;
    const double un = edp_maxwell_inj(maxwell_inj, rmax_inj, edp_u01(w[0]));
    const double t1 = edp_maxwell(maxwell_v, rmax, edp_u01(w[1]));
    const double t2 = edp_maxwell(maxwell_v, rmax, edp_u01(w[2]));
    switch (face.dir) {
    case 0: nx = x; ny = face.at + 1.0e-6; v[0] = t1; v[1] = un; v[2] = t2; break;    // normal +y (dirflag 4)
    case 1: nx = x; ny = face.at - 1.0e-6; v[0] = t1; v[1] = -un; v[2] = t2; break;   // normal -y (dirflag 2)
    case 2: nx = face.at + 1.0e-6; ny = y; v[0] = un; v[1] = t1; v[2] = t2; break;    // normal +x (dirflag 1)
    default: nx = face.at - 1.0e-6; ny = y; v[0] = -un; v[1] = t1; v[2] = t2; break;  // normal -x (dirflag 3)
    }
    v[0] *= f;
    v[1] *= f;
    v[2] *= f;
    const double en = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (en > energy) {   // the electron takes what is left of the primary's energy
        const double alpha = sqrt(energy / en);
        v[0] *= alpha;
        v[1] *= alpha;
        v[2] *= alpha;
        energy = 0.0;
    } else {
        energy -= en;
    }
    return true;
}

// PROCESS_ION_INDUCED_ELECTRON_EMISSION + INJECT_ION_IMPACT_EXTRACTED_ELECTRON (pic2d_IonEmissions.f90:1-342) for an
// ion of species s absorbed by wall `wall` at (x, y) (the tangential coordinate already inside the domain) with
// velocity v. Variates: Philox4x32-10, key {id, seed_lo}, counter {step, EDP_STREAM_EMIT(s), block, seed_hi};
// block 0 word 0 decides the fractional part of the yield, block 1 + e words 0, 1, 2 give electron e's normal
// (injection) component and its two tangential components in x, y, z order. Emitted electrons start 1e-6 inside the
// wall and go to `out` (the electron add list). Returns the number emitted.
template <class Out>
__device__ __noinline__ int edp_emit_electrons(const edp_emit_dev* em, int s, int wall, double x, double y,
                                               double vx, double vy, double vz, uint32_t id, uint32_t step,
                                               uint32_t seed_lo, uint32_t seed_hi, edp_face face, Out out)
{
    if (!em->on[wall][s]) return 0;
    double energy = em->ms[s] * (vx * vx + vy * vy + vz * vz);
    if (energy <= em->emin[wall][s] || energy >= em->emax[wall][s]) return 0;
    double coef = em->yield[wall][s];
    if (coef == 0.0) return 0;
    energy = fmax(0.0, energy - em->emin[wall][s]);
    const double f = em->fconv[wall][s];
    int n = 0, e = 0;
    auto inject = [&]() {
        uint32_t w[4];
        if (energy <= 0.0) return;
        edp_philox(step, EDP_STREAM_EMIT(s), 1u + (uint32_t)e, seed_hi, id, seed_lo, w);
        double nx, ny, v[3];
        if (!edp_emit_thermal(em->maxwell_v, em->rmax, em->maxwell_inj, em->rmax_inj, face, x, y, f, energy, w, nx,
                              ny, v))
            return;
        ++e;
        out(nx, ny, v);
        ++n;
    };
    while (coef >= 1.0) {
        inject();
        coef -= 1.0;
    }
    if (coef == 0.0) return n;
    uint32_t w0[4];
    edp_philox(step, EDP_STREAM_EMIT(s), 0u, seed_hi, id, seed_lo, w0);
    if (edp_u01(w0[0]) < coef) inject();
    return n;
}

// Electron-induced electron emission of the four domain walls in code units (energies of an electron are v^2):
// the parameters of edp_see_params converted as PREPARE_WALL_MATERIALS does (pic2d_Materials.f90:195-244).
struct edp_see_wall {
    int on, m_el, m_in, m_tr, refl_random;
    double el_yield, el_emin, el_emax, el_e0, el_emaxc, el_max, el_de, el_frac;
    double in_yield, in_emin, in_emax, in_frac;
    double tr_yield, tr_emin, tr_emax;
    double cl_e0, cl_emax, cl_max, cl_k;
    double lowest;   // lowest_energy_for_see
    double fconv;    // factor_convert_seetrue_vinj = sqrt(T_see / T_e) / N_max_vel
};
struct edp_see_dev {
    edp_see_wall w[EDP_N_HIT_COUNTERS];   // the domain walls, then inner object n at 4 + n
    const double* maxwell_v;
    const double* maxwell_inj;
    int rmax, rmax_inj;
};

// Coeff_SEE_Classic (pic2d_SEEmission.f90:1171-1208); its exponent k is a REAL (single precision) variable
__device__ inline double edp_see_classic(const edp_see_wall& w, double e, double theta)
{
    if (!(e > w.cl_e0)) return 0.0;
    const double emax_t = w.cl_emax * (1.0 + 0.318309886 * w.cl_k * theta * theta);
    const double v = (e - w.cl_e0) / (emax_t - w.cl_e0);
    const double cmax = w.cl_max * (1.0 + 0.159154943 * w.cl_k * theta * theta);
    const double k = v < 1.0 ? (double)0.62f : (double)0.25f;
    return cmax * pow(v * exp(1.0 - v), k);
}

// Coeff_SEE_Elastic / _Inelastic / _True (:1054-1167); a model-1 coefficient outside its window is 0
__device__ inline double edp_see_elastic(const edp_see_wall& w, double e, double theta)
{
    if (w.m_el == 1) return (e > w.el_emin && e <= w.el_emax) ? w.el_yield : 0.0;
    if (w.m_el != 2) return 0.0;
    if (e >= w.el_emaxc)
        return w.el_max * exp(-(e - w.el_emaxc) / w.el_de) * (e - w.el_emaxc + w.el_de) / w.el_de +
               w.el_frac * edp_see_classic(w, e, theta);
    if (e > w.el_e0)
        return w.el_max * exp(-(e - w.el_emaxc) / (w.el_emaxc - w.el_e0)) * (e - w.el_e0) / (w.el_emaxc - w.el_e0) +
               w.el_frac * edp_see_classic(w, e, theta);
    return 0.0;
}
__device__ inline double edp_see_inelastic(const edp_see_wall& w, double e, double theta)
{
    if (w.m_in == 1) return (e > w.in_emin && e <= w.in_emax) ? w.in_yield : 0.0;
    if (w.m_in == 2) return w.in_frac * edp_see_classic(w, e, theta);
    return 0.0;
}
__device__ inline double edp_see_true(const edp_see_wall& w, double e, double theta)
{
    if (w.m_tr == 1) return (e > w.tr_emin && e <= w.tr_emax) ? w.tr_yield : 0.0;
    if (w.m_tr != 2) return 0.0;
    return fmax(0.0, edp_see_classic(w, e, theta) * (1.0 - w.el_frac - w.in_frac));
}

// A reflected or backscattered electron of speed `speed` leaving the surface `face` at angle theta from the normal
// and azimuth fi (INJECT_ELASTIC_REFLECTED_ELECTRON / INJECT_INELASTIC_BACKSCATTERED_ELECTRON; a domain wall, or an
// inner object's side with m = -1, 1e-6 outside it)
__device__ inline void edp_see_scatter(edp_face face, double x, double y, double speed, double theta, double fi,
                                       double& nx, double& ny, double v[3])
{
    const double c = speed * cos(theta), s1 = speed * sin(theta) * sin(fi), s2 = speed * sin(theta) * cos(fi);
    switch (face.dir) {
    case 0: nx = x; ny = face.at + 1.0e-6; v[0] = s1; v[1] = c; v[2] = s2; break;
    case 1: nx = x; ny = face.at - 1.0e-6; v[0] = s1; v[1] = -c; v[2] = s2; break;
    case 2: nx = face.at + 1.0e-6; ny = y; v[0] = c; v[1] = s1; v[2] = s2; break;
    default: nx = face.at - 1.0e-6; ny = y; v[0] = -c; v[1] = s1; v[2] = s2; break;
    }
}

// PROCESS_ELECTRON_INDUCED_ELECTRON_EMISSION (pic2d_SEEmission.f90:4-151) for an electron absorbed by `wall` at
// (x, y) (coordinate along the wall already clamped) with velocity v. Variates: Philox4x32-10, key {id, seed_lo},
// counter {step, EDP_STREAM_SEE, block, seed_hi}. Block 0: word 0 chooses the process, words 1 and 2 the angles
// (ASIN(R), 2 pi R), word 3 the backscattered speed (sqrt(R)) or the fractional true yield; block 1 + e: true
// secondary e (as edp_emit_thermal). Emitted electrons go to `out`; returns their number, or -1 when the elastic
// and inelastic coefficients add up to more than 1 (the reference stops there).
template <class Out>
__device__ __noinline__ int edp_see_electrons(const edp_see_dev* sd, int wall, double x, double y, double vx,
                                              double vy, double vz, uint32_t id, uint32_t step, uint32_t seed_lo,
                                              uint32_t seed_hi, edp_face face, Out out)
{
    const edp_see_wall& w = sd->w[wall];
    if (!w.on) return 0;
    double e = vx * vx + vy * vy + vz * vz;
    if (e <= w.lowest) return 0;
    const double v = sqrt(e);
    double theta = 0.0;
    if (v != 0.0) theta = acos(fmin(1.0, fabs(face.dir >= 2 ? vx : vy) / v));
    const double ce = edp_see_elastic(w, e, theta), ci = edp_see_inelastic(w, e, theta);
    if (ce + ci > 1.0) return -1;
    double ct = edp_see_true(w, e, theta);
    const double ctot = ce + ci + ct;
    if (ctot == 0.0) return 0;
    uint32_t b0[4];
    edp_philox(step, EDP_STREAM_SEE, 0u, seed_hi, id, seed_lo, b0);
    const double R = edp_u01(b0[0]);
    double nx, ny, nv[3];
    if (R <= ce) {   // INJECT_ELASTIC_REFLECTED_ELECTRON :155-557
        if (!w.refl_random) {
            nx = x;
            ny = y;
            nv[0] = vx;
            nv[1] = vy;
            nv[2] = vz;
            switch (face.dir) {
            case 0: ny = face.at + 1.0e-6; nv[1] = -vy; break;
            case 1: ny = face.at - 1.0e-6; nv[1] = -vy; break;
            case 2: nx = face.at + 1.0e-6; nv[0] = -vx; break;
            default: nx = face.at - 1.0e-6; nv[0] = -vx; break;
            }
        } else {
            edp_see_scatter(face, x, y, v, asin(fmin(edp_u01(b0[1]), 1.0)), 6.283185307179 * edp_u01(b0[2]), nx, ny,
                            nv);
        }
        out(nx, ny, nv);
        return 1;
    }
    if (R > ce && R <= ce + ci) {   // INJECT_INELASTIC_BACKSCATTERED_ELECTRON :561-790
        const double th = asin(fmin(edp_u01(b0[1]), 1.0)), fi = 6.283185307179 * edp_u01(b0[2]);
        edp_see_scatter(face, x, y, v * sqrt(edp_u01(b0[3])), th, fi, nx, ny, nv);
        out(nx, ny, nv);
        return 1;
    }
    if (ct <= 0.0) return 0;
    double energy = e;
    if (w.m_tr == 1) energy = fmax(0.0, e - w.tr_emin);
    else if (w.m_tr == 2) energy = fmax(0.0, e - w.cl_e0);
    int n = 0, k = 0;
    auto inject = [&]() {   // INJECT_TRUE_SECONDARY_ELECTRON :794-1050
        uint32_t wb[4];
        if (energy <= 0.0) return;
        edp_philox(step, EDP_STREAM_SEE, 1u + (uint32_t)k, seed_hi, id, seed_lo, wb);
        if (!edp_emit_thermal(sd->maxwell_v, sd->rmax, sd->maxwell_inj, sd->rmax_inj, face, x, y, w.fconv, energy, wb,
                              nx, ny, nv))
            return;
        ++k;
        out(nx, ny, nv);
        ++n;
    };
    if (ctot <= 1.0) {
        if (R > ce + ci && R <= ctot) inject();
        return n;
    }
    ct = ct / (1.0 - (ce + ci));
    while (ct >= 1.0) {
        inject();
        ct -= 1.0;
    }
    if (edp_u01(b0[3]) < ct) inject();
    return n;
}

// ------------------------------------------------------------------------------------- dielectric inner objects
// CHECK_INTERSECTION_WITH_VERTICAL_SEGMENT (pic2d_ElectronWallCollisions.f90:746-779) of the trajectory (xo, yo) ->
// (x, y) with the segment x = xs, ys0 <= y <= ys1: true and the crossing's y when they cross
__device__ inline bool edp_cross_vertical(double xo, double yo, double x, double y, double xs, double ys0, double ys1,
                                          double& yc)
{
    if (fmax(xo, x) < xs || fmin(xo, x) > xs || fmax(yo, y) < ys0 || fmin(yo, y) > ys1 || xo == x) return false;
    yc = yo + (y - yo) * (xs - xo) / (x - xo);
    if (!isfinite(yc) || yc < ys0 || yc > ys1 || yc < fmin(y, yo) || yc > fmax(y, yo)) return false;
    return true;
}

// The trajectory's first crossing of an inner object's outline (FIND_CLOSEST_INTERSECTION_WITH_OBJECT, :649-742,
// over all inner objects as TRY_ELECTRON_COLL_WITH_INNER_OBJECT :470-557 / TRY_ION_COLL_WITH_INNER_OBJECT,
// pic2d_IonWallCollisions.f90:391-480; segments 1 left, 2 top, 3 right, 4 bottom; ties keep the earlier one). Returns
// the object index and the segment m and crossing (bx, by), or -1 when no crossing is found.
__device__ inline int edp_inner_cross(const edp_kparams& kp, double X, double Y, double vx, double vy, double xmul,
                                      int& bm, double& bx, double& by)
{
    const double xo = X - vx * xmul, yo = Y - vy * xmul;
    int best = -1;
    double bd = 0.0;
    bm = 0;
    bx = by = 0.0;
    for (int n = 0; n < kp.n_inner; ++n) {
        const double il = kp.ileft[n], ir = kp.iright[n], jb = kp.jbottom[n], jt = kp.jtop[n];
        for (int m = 1; m <= 4; ++m) {
            double xc, yc;
            bool ok;
            if (m == 1 || m == 3) {
                xc = m == 1 ? il : ir;
                ok = edp_cross_vertical(xo, yo, X, Y, xc, jb, jt, yc);
            } else {   // a horizontal segment is the vertical case with x and y exchanged
                yc = m == 2 ? jt : jb;
                ok = edp_cross_vertical(yo, xo, Y, X, yc, il, ir, xc);
            }
            if (!ok) continue;
            const double d = (xc - xo) * (xc - xo) + (yc - yo) * (yc - yo);
            if (best >= 0 && d >= bd) continue;
            best = n;
            bm = m;
            bx = xc;
            by = yc;
            bd = d;
        }
    }
    return best;
}

// The charge q given to the two outline nodes of dielectric object `obj` next to the crossing (bx, by) on segment m
// (DO_ELECTRON_COLL_WITH_INNER_OBJECT :561-645 / DO_ION_COLL_WITH_INNER_OBJECT; an electron emitted there gives
// +1 with the same split, INJECT_ION_IMPACT_EXTRACTED_ELECTRON pic2d_IonEmissions.f90:232-330): the node fractions
// are the fractional part of the crossing coordinate, as there. surf holds the charge per node in units of 2^-32.
__device__ inline void edp_inner_charge(const edp_kparams& kp, unsigned long long* surf, int obj, int bm, double bx,
                                        double by, double q)
{
    const int il = kp.ileft[obj], ir = kp.iright[obj], jb = kp.jbottom[obj], jt = kp.jtop[obj];
    const int64_t w = kp.nxg;
    int64_t na, nb;   // the outline nodes i and i+1 of the reference's numbering
    double fa;        // fraction of the charge at node i
    switch (bm) {
    case 1: {   // left side, coll_direction_flag 3
        const int k = min((int)(by - jb), jt - jb - 1);
        na = (int64_t)(jb + k) * w + il;
        nb = na + w;
        fa = 1.0 - (by - (double)(int)by);
        break;
    }
    case 2: {   // top side, flag 4
        const int k = min((int)(bx - il), ir - il - 1);
        na = (int64_t)jt * w + il + k;
        nb = na + 1;
        fa = 1.0 - (bx - (double)(int)bx);
        break;
    }
    case 3: {   // right side from the top, flag 1
        const int k = min((int)(jt - by), jt - jb - 1);
        na = (int64_t)(jt - k) * w + ir;
        nb = na - w;
        fa = by - (double)(int)by;
        break;
    }
    default: {   // bottom side from the right, flag 2; past the last node the outline closes at (ileft, jbottom)
        const int k = min((int)(ir - bx), ir - il - 1);
        na = (int64_t)jb * w + ir - k;
        nb = na - 1;
        fa = bx - (double)(int)bx;
        break;
    }
    }
    const long long qa = __double2ll_rn(fa * EDP_FIX_ONE);
    const long long qb = 4294967296LL - qa;
    atomicAdd(&surf[na], (unsigned long long)__double2ll_rn(q * (double)qa));
    atomicAdd(&surf[nb], (unsigned long long)__double2ll_rn(q * (double)qb));
}

// The emitting face of inner object `obj` at segment m: outward normal and the side's coordinate
__device__ __forceinline__ edp_face edp_inner_face(const edp_kparams& kp, int obj, int bm)
{
    edp_face f;
    switch (bm) {
    case 1: f.dir = 3; f.at = (double)kp.ileft[obj]; break;     // left side: normal -x (dirflag 3)
    case 2: f.dir = 0; f.at = (double)kp.jtop[obj]; break;      // top side: normal +y (dirflag 4)
    case 3: f.dir = 2; f.at = (double)kp.iright[obj]; break;    // right side: normal +x (dirflag 1)
    default: f.dir = 1; f.at = (double)kp.jbottom[obj]; break;  // bottom side: normal -y (dirflag 2)
    }
    return f;
}

// crossing plus the charge of a dielectric object; returns the object or -1
__device__ inline int edp_inner_hit(const edp_kparams& kp, unsigned long long* surf, double X, double Y, double vx,
                                    double vy, double xmul, double q)
{
    int bm;
    double bx, by;
    const int best = edp_inner_cross(kp, X, Y, vx, vy, xmul, bm, bx, by);
    if (best >= 0 && ((kp.diel_mask >> best) & 1)) edp_inner_charge(kp, surf, best, bm, bx, by, q);
    return best;
}
