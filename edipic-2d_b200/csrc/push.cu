// Fused push + charge deposit (+ collisions) of EDIPIC-2D's particle cycle on sm_100a.
//
//  ADVANCE_ELECTRONS  pic2d_ElectronDynamics.f90:3-513     bilinear E gather, Boris rotation, move, walls
//  ADVANCE_IONS       pic2d_IonDynamics.f90:3-524          same on acc_E with QM2s and N_subcycles
//  GATHER_*_CHARGE_DENSITY  pic2d_ElectronDynamics.f90:1597-1639 / pic2d_IonDynamics.f90:1540-2003 (CIC)
//  PERFORM_ELECTRON_NEUTRAL_COLLISIONS / PERFORM_RESONANT_CHARGE_EXCHANGE in the epilogue when fused.
//
// Mixed precision: int32 packed cell (j<<16 | i) + FP32 in-cell offsets and FP32 velocities, 128-bit loads
// (4 particles per thread). Particles are tile-sorted; one CTA handles a chunk of one tile, stages the
// field of the tile + halo in shared memory and accumulates the deposit there in 64-bit fixed point
// (2^32 units per macroparticle) before one flush of global atomics. Particles that left the window
// (and the unsorted tail of newly appended particles) use global memory directly.
#include "edp_internal.cuh"

namespace {

struct PushArgs {
    edp_kparams kp;
    edp_species_mixed P;
    const edp_chunk* chunks;
    int64_t n_chunks;
    int64_t tail_start;
    const unsigned long long* n_slots;
    int64_t tail_ctas;
    const float2* E;
    unsigned long long* rho;
    float K[9];
    float qh, ez_term, xmul;
    int use_rot, species, do_coll;
    uint32_t step;
    uint64_t draw_base;            // edp_draw_base of this species' decision stream at this step
    const edp_mcc_dev* mcc;
    edp_rcx_dev rcx;
    edp_dev_counters* dc;
    uint32_t* sel_list;
    unsigned long long* sel_count;
    int64_t sel_cap;
    edp_hits hits;                 // wall-hit list of ion-induced electron emission
    int emit_on;
    int need_id;                   // the ids are read: collisions, or hits recorded for emission
    // sort inside the push: every particle goes to slot cursor[key of its pre-push cell and source slot]++ of D
    edp_species_mixed D;
    unsigned long long* cursor;
    int ntx;
    int64_t cap;
};

__device__ __forceinline__ int wrapx(int lx, const edp_kparams& kp)
{
    if (kp.periodic) {
        if (lx >= kp.ncx) lx -= kp.ncx;
        else if (lx < 0) lx += kp.ncx;
    }
    return lx;
}

// wall classification of the walled domain (SURROUNDED_BY_WALL corners), :212-518
__device__ __forceinline__ int wall_object(double X, double Y, double xmax, double ymax)
{
    if (X < 0.0) {
        if (Y >= 1.0 && Y <= ymax - 1.0) return 2;
        if (Y < 1.0) return ((0.0 - X) < (0.0 - Y)) ? 0 : 2;
        return ((0.0 - X) < (Y - ymax)) ? 1 : 2;
    }
    if (X > xmax) {
        if (Y >= 1.0 && Y <= ymax - 1.0) return 3;
        if (Y < 1.0) return ((X - xmax) < (0.0 - Y)) ? 0 : 3;
        return ((X - xmax) < (Y - ymax)) ? 1 : 3;
    }
    return (Y > ymax) ? 1 : 0;
}

__device__ __forceinline__ void record_born(const edp_born& b, unsigned long long* count, unsigned int* eflag,
                                            double x, double y, const double* v)
{
    unsigned long long k = atomicAdd(count, 1ull);
    if ((int64_t)k >= b.cap) {
        atomicOr(eflag, EDP_EFLAG_PENDING);
        return;
    }
    b.x[k] = x;
    b.y[k] = y;
    b.vx[k] = v[0];
    b.vy[k] = v[1];
    b.vz[k] = v[2];
}

// An ion absorbed by a domain wall while ion-induced electron emission is on: its record goes to the wall-hit list
// (the emission itself runs in ion_emission_kernel after the push, so that the push keeps no call frame).
__device__ __forceinline__ void record_hit(const edp_hits& h, edp_dev_counters* dc, int wall, int s, double x,
                                           double y, double vx, double vy, double vz, uint32_t id)
{
    unsigned long long k = atomicAdd(&dc->hit_count, 1ull);
    if ((int64_t)k >= h.cap) {
        atomicOr(&dc->error_flags, EDP_EFLAG_PENDING);
        return;
    }
    h.x[k] = x;
    h.y[k] = y;
    h.vx[k] = vx;
    h.vy[k] = vy;
    h.vz[k] = vz;
    h.id[k] = id;
    h.ws[k] = wall | (s << 8);
}

// Shared state of one CTA of the mixed push: field window, density window and per-CTA counters.
// The fixed-point density (2^32 units per macroparticle) is kept as two 32-bit accumulators per node,
// hi = sum(q >> 16) and lo = sum(q & 0xFFFF), so that every shared update is a native 32-bit atomic;
// a CTA handles at most EDP_CHUNK particles, which bounds both sums below 2^30.
#define EDP_SEL_SMEM 1024
struct Smem {
    float2 E[EDP_WIN_NODES * EDP_WIN_NODES];
    int hi[EDP_WIN_NODES * EDP_WIN_NODES];
    unsigned lo[EDP_WIN_NODES * EDP_WIN_NODES];
    unsigned long long cnt[32];   // [0..7] hits, [8..15] en kinds, [16] rcx, [17] removed
    uint32_t sel[EDP_SEL_SMEM];   // slots selected for an electron-neutral collision
    unsigned nsel;
};

// deposit of consecutive particles of one thread that land in the same cell, merged in registers
struct DepAcc {
    int b;   // window index of the (i, j) node, -1 when empty
    long long q00, q10, q01, q11;
};

__device__ __forceinline__ void smem_add(Smem& s, int n, long long q)
{
    atomicAdd(&s.hi[n], (int)(q >> 16));
    atomicAdd(&s.lo[n], (unsigned)(q & 0xFFFF));
}

__device__ __forceinline__ void dep_flush(Smem& s, DepAcc& d)
{
    if (d.b < 0) return;
    smem_add(s, d.b, d.q00);
    smem_add(s, d.b + 1, d.q10);
    smem_add(s, d.b + EDP_WIN_NODES, d.q01);
    smem_add(s, d.b + EDP_WIN_NODES + 1, d.q11);
    d.b = -1;
}

// Electrons selected for a collision in the push epilogue: slot indices gathered per CTA in shared memory and
// appended to a global list that collide_selected_kernel scatters (the same Philox variates as the separate pass).
__device__ __forceinline__ void select_slot(const PushArgs& a, Smem& s, uint32_t slot)
{
    unsigned q = atomicAdd(&s.nsel, 1u);
    if (q < EDP_SEL_SMEM) {
        s.sel[q] = slot;
        return;
    }
    unsigned long long g = atomicAdd(a.sel_count, 1ull);
    if ((int64_t)g < a.sel_cap) a.sel_list[g] = slot;
    else atomicOr(&a.dc->error_flags, EDP_EFLAG_PENDING);
}

// column offset inside a window; periodic domains have a power-of-two period (the FFT_X length)
template <bool PER>
__device__ __forceinline__ int win_dx(int d, const edp_kparams& kp)
{
    return PER ? (d & (kp.ncx - 1)) : d;
}

// round-to-nearest-even of 0 <= x <= 2^51 to an integer with one FP64 add: x + 1.5 * 2^52 has a unit in the last
// place of 1, so the sum is rounded to an integer and its low mantissa bits hold it (the classic magic-number
// conversion); equal to __double2ll_rn(x) on that range, on the FP64 pipe instead of the conversion unit
__device__ __forceinline__ long long fix_round(double x)
{
    const double magic = 6755399441055744.0;   // 1.5 * 2^52
    return __double_as_longlong(__dadd_rn(x, magic)) - __double_as_longlong(magic);
}

// One particle. Returns false when it was absorbed (the caller stores cell = -1).
// ION: ion species (acc_E, RCX) instead of electrons (E, MCC selection); PER: periodic x; ROT: Boris rotation.
// The collision decision word of one particle: word 0 of its decision draw keyed by (id, step), in the stream of MCC
// selection (electrons) or charge exchange (ions) whose base the host computed for this launch.
__device__ __forceinline__ uint32_t push_draw(const PushArgs& a, uint32_t id)
{
    return (uint32_t)(edp_draw(a.draw_base, id) >> 32);
}

template <bool ION, bool PER, bool ROT>
__device__ __forceinline__ bool push_one(const PushArgs& a, Smem& s, bool windowed, int wx0, int wy0, DepAcc& acc,
                                         int& cell, float& ox, float& oy, float& vx, float& vy, float& vz, uint32_t id,
                                         bool& selected)
{
    const edp_kparams& kp = a.kp;
    int i = cell & 0xFFFF, j = cell >> 16;
    // ---- gather (bilinear, :82-86)
    int lx = win_dx<PER>(i - wx0, kp), ly = j - wy0;
    float2 e00, e10, e01, e11;
    if (windowed && (unsigned)lx < EDP_WIN_CELLS && (unsigned)ly < EDP_WIN_CELLS) {
        int b = ly * EDP_WIN_NODES + lx;
        e00 = s.E[b];
        e10 = s.E[b + 1];
        e01 = s.E[b + EDP_WIN_NODES];
        e11 = s.E[b + EDP_WIN_NODES + 1];
    } else {
        int i1 = i + 1;
        if (PER && i1 == kp.ncx) i1 = 0;
        int64_t r0 = (int64_t)j * kp.nxg, r1 = r0 + kp.nxg;
        e00 = __ldg(&a.E[r0 + i]);
        e10 = __ldg(&a.E[r0 + i1]);
        e01 = __ldg(&a.E[r1 + i]);
        e11 = __ldg(&a.E[r1 + i1]);
    }
    float axp = ox, axm = 1.0f - ox, ayp = oy, aym = 1.0f - oy;
    float w00 = axm * aym, w10 = axp * aym, w01 = axm * ayp, w11 = axp * ayp;
    float EX = e00.x * w00 + e10.x * w10 + e01.x * w01 + e11.x * w11;
    float EY = e00.y * w00 + e10.y * w10 + e01.y * w01 + e11.y * w11;
    // ---- Boris (:95-130 / ions :99-149)
    const float q = a.qh;
    if (ROT) {
        float mx = vx + q * EX, my = vy + q * EY, mz = vz + a.ez_term;
        float px = a.K[0] * mx + a.K[1] * my + a.K[2] * mz;
        float py = a.K[3] * mx + a.K[4] * my + a.K[5] * mz;
        float pz = a.K[6] * mx + a.K[7] * my + a.K[8] * mz;
        vx = px + q * EX;
        vy = py + q * EY;
        vz = pz + a.ez_term;
    } else if (ION) {
        vx = vx + (q + q) * EX;
        vy = vy + (q + q) * EY;
        vz = vz + (a.ez_term + a.ez_term);
    } else {
        vx = (vx + q * EX) + q * EX;
        vy = (vy + q * EY) + q * EY;
        vz = (vz + a.ez_term) + a.ez_term;
    }
    // ---- move (:148-149 / :154-155)
    float nx = ox + vx * a.xmul, ny = oy + vy * a.xmul;
    float fx = floorf(nx), fy = floorf(ny);
    int ni = i + (int)fx, nj = j + (int)fy;
    nx -= fx;
    ny -= fy;
    if (nx >= 1.0f) { nx -= 1.0f; ++ni; }
    if (ny >= 1.0f) { ny -= 1.0f; ++nj; }
    // ---- inner objects (:160-172): strictly inside
    for (int n = 0; n < kp.n_inner; ++n) {
        bool in = (ni > kp.ileft[n] || (ni == kp.ileft[n] && nx > 0.0f)) && ni < kp.iright[n] &&
                  (nj > kp.jbottom[n] || (nj == kp.jbottom[n] && ny > 0.0f)) && nj < kp.jtop[n];
        if (in) {
            atomicAdd(&s.cnt[4 + n], 1ull);
            // the crossing is found after the push: a dielectric's outline takes the charge, an ion-emitting or
            // ion-reflecting object answers the ion
            if (((kp.diel_mask | (ION ? kp.ion_inner_mask : kp.see_inner_mask)) >> n) & 1)
                record_hit(a.hits, a.dc, 4 + n, ION ? a.species - 1 : 0, (double)ni + (double)nx,
                           (double)nj + (double)ny, vx, vy, vz, id);
            return false;
        }
    }
    // ---- domain boundaries (:174-511)
    if (PER) {
        if (ni < 0) ni += kp.ncx;
        else if (ni >= kp.ncx) ni -= kp.ncx;
        if (nj < 0 || nj > kp.ncy || (nj == kp.ncy && ny > 0.0f)) {
            const int wall = nj < 0 ? 0 : 1;
            atomicAdd(&s.cnt[wall], 1ull);
            if (a.emit_on)
                record_hit(a.hits, a.dc, wall, ION ? a.species - 1 : 0, (double)ni + (double)nx,
                           (double)nj + (double)ny, vx, vy, vz, id);
            return false;
        }
    } else {
        bool outx = ni < 0 || ni > kp.ncx || (ni == kp.ncx && nx > 0.0f);
        bool outy = nj < 0 || nj > kp.ncy || (nj == kp.ncy && ny > 0.0f);
        if (outx || outy) {
            int obj;
            if (kp.strip) {
                // the walls of the whole domain, in its coordinates; leaving the strip and its ghost columns through a
                // side that is not a wall of the domain is an error
                const bool wall_x = outx && ((ni < 0 && kp.strip_gl == 0) || (ni >= 0 && kp.strip_gr == 0));
                if (!outy && !wall_x) {
                    atomicOr(&a.dc->error_flags, EDP_EFLAG_BOUNDS);
                    return false;
                }
                if (kp.strip_periodic) obj = nj < 0 ? 0 : 1;
                else obj = wall_object((double)(ni + kp.strip_x0) + (double)nx, (double)nj + (double)ny,
                                       (double)kp.strip_ncx, (double)kp.ncy);
            } else {
                obj = wall_object((double)ni + (double)nx, (double)nj + (double)ny, (double)kp.ncx, (double)kp.ncy);
            }
            atomicAdd(&s.cnt[obj], 1ull);
            if (a.emit_on)
                record_hit(a.hits, a.dc, obj, ION ? a.species - 1 : 0, (double)ni + (double)nx,
                           (double)nj + (double)ny, vx, vy, vz, id);
            return false;
        }
        if (ni == kp.ncx) { ni = kp.ncx - 1; nx = 1.0f; }   // X == c_X_area_max (:68)
    }
    if (nj == kp.ncy) { nj = kp.ncy - 1; ny = 1.0f; }       // Y == c_Y_area_max (:69)
    cell = (nj << 16) | ni;
    ox = nx;
    oy = ny;
    // ---- deposit (:1597-1639): exact FP64 weights of the FP32 offsets, rounded to 2^-32; the fourth weight
    // takes the remainder so that every particle deposits exactly 2^32 units
    // (the 2^32 scaling is exact, so folding it into one factor rounds the same way)
    const double dx = (double)nx, dy = (double)ny, mxd = __dsub_rn(1.0, dx);
    const double A = __dmul_rn(__dsub_rn(1.0, dy), EDP_FIX_ONE), B = __dmul_rn(dy, EDP_FIX_ONE);
    // both roundings give the same integers on this range; which one keeps the kernel out of spills at 64 registers
    // differs by species (measured: the magic add for electrons, the conversion for ions)
    const long long q00 = ION ? __double2ll_rn(__dmul_rn(mxd, A)) : fix_round(__dmul_rn(mxd, A));
    const long long q10 = ION ? __double2ll_rn(__dmul_rn(dx, A)) : fix_round(__dmul_rn(dx, A));
    const long long q01 = ION ? __double2ll_rn(__dmul_rn(mxd, B)) : fix_round(__dmul_rn(mxd, B));
    const long long q11 = 4294967296LL - q00 - q10 - q01;
    const int dlx = win_dx<PER>(ni - wx0, kp), dly = nj - wy0;
    if (windowed && (unsigned)dlx < EDP_WIN_CELLS && (unsigned)dly < EDP_WIN_CELLS) {
        const int b = dly * EDP_WIN_NODES + dlx;
        if (b != acc.b) {
            dep_flush(s, acc);
            acc.b = b;
            acc.q00 = q00;
            acc.q10 = q10;
            acc.q01 = q01;
            acc.q11 = q11;
        } else {
            acc.q00 += q00;
            acc.q10 += q10;
            acc.q01 += q01;
            acc.q11 += q11;
        }
    } else {
        int i1 = ni + 1;
        if (PER && i1 == kp.ncx) i1 = 0;
        int64_t r0 = (int64_t)nj * kp.nxg, r1 = r0 + kp.nxg;
        atomicAdd(&a.rho[r0 + ni], (unsigned long long)q00);
        atomicAdd(&a.rho[r0 + i1], (unsigned long long)q10);
        atomicAdd(&a.rho[r1 + ni], (unsigned long long)q01);
        atomicAdd(&a.rho[r1 + i1], (unsigned long long)q11);
    }
    // ---- collisions in the epilogue, with the variates of the separate passes
    // the decision draw after the push, for the particles still present (as edp_mcc_select / edp_rcx_ion)
    if (!ION && a.do_coll) selected = (unsigned long long)push_draw(a, id) < a.mcc->pmax_x;
    if (ION && a.do_coll) {
        double dvx = vx, dvy = vy, dvz = vz;
        if (edp_rcx_ion_drawn(a.rcx, push_draw(a, id), id, a.step, (uint32_t)(a.species - 1), kp.seed_lo,
                              kp.seed_hi, dvx, dvy, dvz)) {
            vx = (float)dvx;
            vy = (float)dvy;
            vz = (float)dvz;
            atomicAdd(&s.cnt[16], 1ull);
        }
    }
    return true;
}

// vector access to IPT consecutive 32-bit values (IPT = 4: 128-bit, 2: 64-bit), streaming (not kept in L1/L2)
template <int IPT>
__device__ __forceinline__ void vload(const void* p, int64_t g, uint32_t* v)
{
    if constexpr (IPT == 4) {
        const uint4 x = __ldcs(reinterpret_cast<const uint4*>(p) + g);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else {
        const uint2 x = __ldcs(reinterpret_cast<const uint2*>(p) + g);
        v[0] = x.x; v[1] = x.y;
    }
}
template <int IPT>
__device__ __forceinline__ void vstore(void* p, int64_t g, const uint32_t* v)
{
    if constexpr (IPT == 4) __stcs(reinterpret_cast<uint4*>(p) + g, make_uint4(v[0], v[1], v[2], v[3]));
    else __stcs(reinterpret_cast<uint2*>(p) + g, make_uint2(v[0], v[1]));
}

// The push, deposit and stores of IPT consecutive slots [IPT g, IPT g + IPT) whose columns are in registers; `full`:
// the whole group lies in [lo, hi) (vector stores), else only the slots inside are stored.
template <bool ION, bool PER, bool ROT, bool WIN, int IPT>
__device__ __forceinline__ void push_group_body(const PushArgs& a, Smem& s, int wx0, int wy0, int64_t g, int64_t lo,
                                                int64_t hi, bool full, int* c, float* ox, float* oy, float* vx,
                                                float* vy, float* vz, const uint32_t* id)
{
    const int64_t base = g * IPT;
    bool sel[IPT];
    DepAcc acc;
    acc.b = -1;
#pragma unroll
    for (int e = 0; e < IPT; ++e) {
        sel[e] = false;
        if (c[e] < 0) continue;
        if (!push_one<ION, PER, ROT>(a, s, WIN, wx0, wy0, acc, c[e], ox[e], oy[e], vx[e], vy[e], vz[e], id[e],
                                     sel[e])) {
            c[e] = -1;
            sel[e] = false;
            atomicAdd(&s.cnt[17], 1ull);
        }
    }
    dep_flush(s, acc);
#pragma unroll
    for (int e = 0; e < IPT; ++e)
        if (sel[e]) select_slot(a, s, (uint32_t)(base + e));
    if (full) {
        vstore<IPT>(a.P.cell, g, reinterpret_cast<const uint32_t*>(c));
        vstore<IPT>(a.P.ox, g, reinterpret_cast<const uint32_t*>(ox));
        vstore<IPT>(a.P.oy, g, reinterpret_cast<const uint32_t*>(oy));
        vstore<IPT>(a.P.vx, g, reinterpret_cast<const uint32_t*>(vx));
        vstore<IPT>(a.P.vy, g, reinterpret_cast<const uint32_t*>(vy));
        vstore<IPT>(a.P.vz, g, reinterpret_cast<const uint32_t*>(vz));
    } else {
#pragma unroll
        for (int e = 0; e < IPT; ++e) {
            int64_t k = base + e;
            if (k < lo || k >= hi) continue;
            a.P.cell[k] = c[e];
            if (c[e] < 0) continue;
            a.P.ox[k] = ox[e];
            a.P.oy[k] = oy[e];
            a.P.vx[k] = vx[e];
            a.P.vy[k] = vy[e];
            a.P.vz[k] = vz[e];
        }
    }
}

// IPT consecutive slots [IPT g, IPT g + IPT). WIN: a sorted chunk, always whole groups (tiles are padded to
// multiples of EDP_ITEMS), gathered and deposited through the shared window. Otherwise the unsorted tail, restricted
// to [lo, hi).
template <bool ION, bool PER, bool ROT, bool WIN, int IPT>
__device__ __forceinline__ void push_group(const PushArgs& a, Smem& s, int wx0, int wy0, int64_t g, int64_t lo,
                                           int64_t hi)
{
    const int64_t base = g * IPT;
    const bool full = WIN || (base >= lo && base + IPT <= hi);
    int c[IPT];
    float ox[IPT], oy[IPT], vx[IPT], vy[IPT], vz[IPT];
    uint32_t id[IPT];
    if (full) {
        vload<IPT>(a.P.cell, g, reinterpret_cast<uint32_t*>(c));
        vload<IPT>(a.P.ox, g, reinterpret_cast<uint32_t*>(ox));
        vload<IPT>(a.P.oy, g, reinterpret_cast<uint32_t*>(oy));
        vload<IPT>(a.P.vx, g, reinterpret_cast<uint32_t*>(vx));
        vload<IPT>(a.P.vy, g, reinterpret_cast<uint32_t*>(vy));
        vload<IPT>(a.P.vz, g, reinterpret_cast<uint32_t*>(vz));
        if (a.need_id) {
            vload<IPT>(a.P.id, g, id);
        } else {
#pragma unroll
            for (int e = 0; e < IPT; ++e) id[e] = 0u;
        }
    } else {
#pragma unroll
        for (int e = 0; e < IPT; ++e) {
            int64_t k = base + e;
            bool ok = k >= lo && k < hi;
            c[e] = ok ? a.P.cell[k] : -1;
            ox[e] = ok ? a.P.ox[k] : 0.f;
            oy[e] = ok ? a.P.oy[k] : 0.f;
            vx[e] = ok ? a.P.vx[k] : 0.f;
            vy[e] = ok ? a.P.vy[k] : 0.f;
            vz[e] = ok ? a.P.vz[k] : 0.f;
            id[e] = ok ? a.P.id[k] : 0u;
        }
    }
    push_group_body<ION, PER, ROT, WIN, IPT>(a, s, wx0, wy0, g, lo, hi, full, c, ox, oy, vx, vy, vz, id);
}

// 16-byte copy global -> shared that bypasses L1 (cp.async.cg)
__device__ __forceinline__ void pf_copy16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}

// The sorted chunk of one CTA with 4 particles per thread, each thread's next group copied ahead into shared memory
// by cp.async while it pushes the current one, so that every warp has its next loads in flight during its
// arithmetic. A thread reads back only the 16-byte pieces it copied itself: no barrier, only its own wait.
template <bool ION, bool PER, bool ROT>
__device__ __forceinline__ void push_chunk_prefetch(const PushArgs& a, Smem& s, int wx0, int wy0, int64_t lo,
                                                    int64_t hi)
{
    __shared__ __align__(16) uint4 pf[7][EDP_PUSH_THREADS];
    const int ncol = a.need_id ? 7 : 6;
    const uint32_t d0 = (uint32_t)__cvta_generic_to_shared(&pf[0][threadIdx.x]);
    const void* col[7] = {a.P.cell, a.P.ox, a.P.oy, a.P.vx, a.P.vy, a.P.vz, a.P.id};
    auto issue = [&](int64_t g) {
#pragma unroll
        for (int k = 0; k < 7; ++k)
            if (k < ncol) pf_copy16(d0 + (uint32_t)(k * EDP_PUSH_THREADS * 16), reinterpret_cast<const uint4*>(col[k]) + g);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    int64_t g = lo / 4 + threadIdx.x;
    if (g * 4 < hi) issue(g);
    for (; g * 4 < hi; g += blockDim.x) {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        int c[4];
        float ox[4], oy[4], vx[4], vy[4], vz[4];
        uint32_t id[4] = {0u, 0u, 0u, 0u};
        const uint4 v0 = pf[0][threadIdx.x], v1 = pf[1][threadIdx.x], v2 = pf[2][threadIdx.x];
        const uint4 v3 = pf[3][threadIdx.x], v4 = pf[4][threadIdx.x], v5 = pf[5][threadIdx.x];
        if (ncol == 7) {
            const uint4 v6 = pf[6][threadIdx.x];
            id[0] = v6.x; id[1] = v6.y; id[2] = v6.z; id[3] = v6.w;
        }
        c[0] = (int)v0.x; c[1] = (int)v0.y; c[2] = (int)v0.z; c[3] = (int)v0.w;
        ox[0] = __uint_as_float(v1.x); ox[1] = __uint_as_float(v1.y); ox[2] = __uint_as_float(v1.z); ox[3] = __uint_as_float(v1.w);
        oy[0] = __uint_as_float(v2.x); oy[1] = __uint_as_float(v2.y); oy[2] = __uint_as_float(v2.z); oy[3] = __uint_as_float(v2.w);
        vx[0] = __uint_as_float(v3.x); vx[1] = __uint_as_float(v3.y); vx[2] = __uint_as_float(v3.z); vx[3] = __uint_as_float(v3.w);
        vy[0] = __uint_as_float(v4.x); vy[1] = __uint_as_float(v4.y); vy[2] = __uint_as_float(v4.z); vy[3] = __uint_as_float(v4.w);
        vz[0] = __uint_as_float(v5.x); vz[1] = __uint_as_float(v5.y); vz[2] = __uint_as_float(v5.z); vz[3] = __uint_as_float(v5.w);
        const int64_t gn = g + blockDim.x;
        if (gn * 4 < hi) issue(gn);   // the pieces just read are in registers; the copies may overwrite them
        push_group_body<ION, PER, ROT, true, 4>(a, s, wx0, wy0, g, lo, hi, true, c, ox, oy, vx, vy, vz, id);
    }
}

// The push of a sort step over a block of 128 slots [b, b + 128) taken by one warp, lane l holding slots
// b + 32 e + l (e < 4): the loads are coalesced per element, and the 32 lanes of an element are 32 consecutive source
// slots, which share their sort key run, so each particle's write to its sorted slot in a.D (the cursor of the key of
// its cell before the push and its source slot) is a coalesced 128-byte run per column. A particle absorbed now
// leaves a dead slot, compacted by the next sort. Called warp-uniformly (every lane, every block).
template <bool ION, bool PER, bool ROT, bool WIN>
__device__ __forceinline__ void scatter_body(const PushArgs& a, Smem& s, int wx0, int wy0, int64_t b, int* c,
                                             float* ox, float* oy, float* vx, float* vy, float* vz,
                                             const uint32_t* id, const int* tag)
{
    const int lane = threadIdx.x & 31;
    int cpre[4];
    bool sel[4];
    DepAcc acc;
    acc.b = -1;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        cpre[e] = c[e];
        sel[e] = false;
        if (c[e] < 0) continue;
        if (!push_one<ION, PER, ROT>(a, s, WIN, wx0, wy0, acc, c[e], ox[e], oy[e], vx[e], vy[e], vz[e], id[e],
                                     sel[e])) {
            c[e] = -1;
            sel[e] = false;
            atomicAdd(&s.cnt[17], 1ull);
        }
    }
    dep_flush(s, acc);
    __syncwarp();
    // the four cursor atomics are issued before any of their results is used, so their round trips overlap
    uint32_t key[4];
    unsigned peers[4];
    unsigned long long b0[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        key[e] = cpre[e] >= 0 ? edp_tile_key(cpre[e], b + 32 * e + lane, a.ntx) : 0xFFFFFFFFu;
        peers[e] = edp_warp_peers(key[e]);
        b0[e] = 0;
        if (key[e] != 0xFFFFFFFFu && lane == __ffs(peers[e]) - 1)
            b0[e] = atomicAdd(&a.cursor[key[e]], (unsigned long long)__popc(peers[e]));
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const unsigned long long base = __shfl_sync(0xFFFFFFFFu, b0[e], __ffs(peers[e]) - 1);
        if (key[e] == 0xFFFFFFFFu) continue;
        const unsigned long long pos = base + __popc(peers[e] & ((1u << lane) - 1u));
        if ((int64_t)pos >= a.cap) {
            atomicOr(&a.dc->error_flags, EDP_EFLAG_CAPACITY);
            continue;
        }
        __stcs(a.D.cell + pos, c[e]);
        if (c[e] < 0) continue;
        __stcs(a.D.ox + pos, ox[e]);
        __stcs(a.D.oy + pos, oy[e]);
        __stcs(a.D.vx + pos, vx[e]);
        __stcs(a.D.vy + pos, vy[e]);
        __stcs(a.D.vz + pos, vz[e]);
        __stcs(a.D.id + pos, id[e]);
        __stcs(a.D.tag + pos, tag[e]);
        if (sel[e]) select_slot(a, s, (uint32_t)pos);
    }
}

template <bool ION, bool PER, bool ROT, bool WIN>
__device__ __forceinline__ void push_block_scatter(const PushArgs& a, Smem& s, int wx0, int wy0, int64_t b,
                                                   int64_t lo, int64_t hi)
{
    const int lane = threadIdx.x & 31;
    int c[4], tag[4];
    float ox[4], oy[4], vx[4], vy[4], vz[4];
    uint32_t id[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int64_t k = b + 32 * e + lane;
        const bool ok = k >= lo && k < hi;
        c[e] = ok ? __ldcs(a.P.cell + k) : -1;
        ox[e] = ok ? __ldcs(a.P.ox + k) : 0.f;
        oy[e] = ok ? __ldcs(a.P.oy + k) : 0.f;
        vx[e] = ok ? __ldcs(a.P.vx + k) : 0.f;
        vy[e] = ok ? __ldcs(a.P.vy + k) : 0.f;
        vz[e] = ok ? __ldcs(a.P.vz + k) : 0.f;
        id[e] = ok ? __ldcs(a.P.id + k) : 0u;
        tag[e] = ok ? __ldcs(a.P.tag + k) : 0;
    }
    scatter_body<ION, PER, ROT, WIN>(a, s, wx0, wy0, b, c, ox, oy, vx, vy, vz, id, tag);
}

// IPT particles per thread: 4 (128-bit accesses, 4 CTAs of 256 per SM) or 2 (64-bit, 5 CTAs per SM). SCAT: the
// push of a sort step, writing every particle to its sorted slot of a.D
template <bool ION, bool PER, bool ROT, int IPT, bool SCAT, bool PF>
__global__ void __launch_bounds__(EDP_PUSH_THREADS, IPT == 4 ? 4 : 5) push_mixed_kernel(PushArgs a)
{
    __shared__ Smem s;
    const edp_kparams& kp = a.kp;
    if (threadIdx.x < 32) s.cnt[threadIdx.x] = 0ull;
    if (threadIdx.x == 0) s.nsel = 0u;
    const bool windowed = blockIdx.x < a.n_chunks;
    int64_t lo, hi;
    int wx0 = 0, wy0 = 0;
    if (windowed) {
        edp_chunk ch = a.chunks[blockIdx.x];
        lo = ch.start;
        hi = ch.end;
        wx0 = ch.wx0;
        wy0 = ch.wy0;
        for (int t = threadIdx.x; t < EDP_WIN_NODES * EDP_WIN_NODES; t += blockDim.x) {
            int lx = t % EDP_WIN_NODES, ly = t / EDP_WIN_NODES;
            int gx = wrapx(wx0 + lx, kp), gy = wy0 + ly;
            bool ok = gx >= 0 && gx < kp.nxg && gy >= 0 && gy < kp.nyg;
            s.E[t] = ok ? __ldg(&a.E[(int64_t)gy * kp.nxg + gx]) : make_float2(0.f, 0.f);
            s.hi[t] = 0;
            s.lo[t] = 0u;
        }
    } else {
        lo = a.tail_start;
        hi = (int64_t)*a.n_slots;
    }
    __syncthreads();
    if constexpr (SCAT) {
        const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        const int64_t b0 = lo & ~(int64_t)127;   // blocks aligned to 128 slots: a lane's key run is its 32-slot group
        if (windowed) {
            for (int64_t b = b0 + 128 * warp; b < hi; b += 128 * nw)
                push_block_scatter<ION, PER, ROT, true>(a, s, wx0, wy0, b, lo, hi);
        } else {
            const int64_t t = blockIdx.x - a.n_chunks;
            for (int64_t b = b0 + 128 * (t * nw + warp); b < hi; b += 128 * nw * a.tail_ctas)
                push_block_scatter<ION, PER, ROT, false>(a, s, 0, 0, b, lo, hi);
        }
    } else if (windowed) {
        if constexpr (PF) {
            push_chunk_prefetch<ION, PER, ROT>(a, s, wx0, wy0, lo, hi);
        } else {
            for (int64_t g = lo / IPT + threadIdx.x; g * IPT < hi; g += blockDim.x)
                push_group<ION, PER, ROT, true, IPT>(a, s, wx0, wy0, g, lo, hi);
        }
    } else {
        int64_t t = blockIdx.x - a.n_chunks;
        int64_t g0 = lo / IPT;
        for (int64_t g = g0 + t * blockDim.x + threadIdx.x; g * IPT < hi; g += a.tail_ctas * blockDim.x)
            push_group<ION, PER, ROT, false, IPT>(a, s, 0, 0, g, lo, hi);
    }
    __syncthreads();
    if (windowed) {
        for (int t = threadIdx.x; t < EDP_WIN_NODES * EDP_WIN_NODES; t += blockDim.x) {
            long long v = (long long)s.hi[t] * 65536LL + (long long)s.lo[t];
            if (v == 0) continue;
            int lx = t % EDP_WIN_NODES, ly = t / EDP_WIN_NODES;
            int gx = wrapx(wx0 + lx, kp), gy = wy0 + ly;
            if (gx >= 0 && gx < kp.nxg && gy >= 0 && gy < kp.nyg)
                atomicAdd(&a.rho[(int64_t)gy * kp.nxg + gx], (unsigned long long)v);
            else atomicOr(&a.dc->error_flags, EDP_EFLAG_BOUNDS);
        }
    }
    if (!ION) {
        __shared__ unsigned long long sel_base;
        const unsigned nsel = min(s.nsel, (unsigned)EDP_SEL_SMEM);
        if (threadIdx.x == 0 && nsel) sel_base = atomicAdd(a.sel_count, (unsigned long long)nsel);
        __syncthreads();
        for (unsigned q = threadIdx.x; q < nsel; q += blockDim.x) {
            unsigned long long g = sel_base + q;
            if ((int64_t)g < a.sel_cap) a.sel_list[g] = s.sel[q];
            else atomicOr(&a.dc->error_flags, EDP_EFLAG_PENDING);
        }
    }
    if (threadIdx.x < 32) {
        unsigned long long v = s.cnt[threadIdx.x];
        if (v) {
            int k = threadIdx.x;
            if (k < 8) atomicAdd(ION ? &a.dc->i_hits[k] : &a.dc->e_hits[k], v);
            else if (k < 16) {
                atomicAdd(&a.dc->en_coll[k - 8], v);
                atomicAdd(&a.dc->en_coll_step[k - 8], v);
            } else if (k == 16) {
                atomicAdd(&a.dc->rcx[a.species - 1], v);
                atomicAdd(&a.dc->rcx_step[a.species - 1], v);
            } else if (k == 17) {
                atomicAdd(&a.dc->n_live[a.species], (unsigned long long)(-(long long)v));
            }
        }
    }
}

// ------------------------------------------------------------------------ streaming push (bulk-copy staging)
// The same push over the sorted chunks, with the particle columns brought into shared memory by the bulk-copy
// engine instead of by the threads' own loads. A persistent CTA walks its chunks (blockIdx.x, + gridDim.x, ...) in
// sub-chunks of SUB particles; thread 0 keeps NST sub-chunks in flight (one cp.async.bulk per column, completion
// counted on the stage's mbarrier), so HBM streams the next sub-chunks, across chunk boundaries and through the
// window flushes, while the warps compute. The threads read their IPT particles from shared memory and write the
// results straight to global memory. Every wait is bounded: a wait that gives up raises EDP_EFLAG_TIMEOUT, and the
// CTA waits (bounded) for its copies in flight before it returns.
__device__ __forceinline__ uint32_t push_smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool push_mbar_wait(uint32_t bar, uint32_t parity)
{
    for (long long it = 0; it < (1LL << 22); ++it) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P;\n\t}\n"
                     : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

struct StreamCursor {
    int64_t chunk, off, end;   // chunk index; first slot of the sub-chunk; end of the chunk
};

template <int SUB>
__device__ __forceinline__ void cursor_first(const PushArgs& a, StreamCursor& c)
{
    c.chunk = blockIdx.x;
    if (c.chunk < a.n_chunks) {
        const edp_chunk ch = a.chunks[c.chunk];
        c.off = ch.start;
        c.end = ch.end;
    }
}

template <int SUB>
__device__ __forceinline__ void cursor_next(const PushArgs& a, StreamCursor& c)
{
    c.off += SUB;
    if (c.off < c.end) return;
    c.chunk += gridDim.x;
    if (c.chunk < a.n_chunks) {
        const edp_chunk ch = a.chunks[c.chunk];
        c.off = ch.start;
        c.end = ch.end;
    }
}

// columns of a stage: cell, ox, oy, vx, vy, vz, id
#define EDP_STREAM_COLS 7

template <int SUB>
__device__ __forceinline__ void stream_issue(const PushArgs& a, const StreamCursor& c, uint32_t stage_base,
                                             uint32_t bar, int ncols)
{
    const int64_t n = min((int64_t)SUB, c.end - c.off);   // a multiple of EDP_ITEMS: 16-byte sizes and addresses
    const uint32_t bytes = (uint32_t)(n * 4);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes * ncols)
                 : "memory");
    const void* src[EDP_STREAM_COLS] = {a.P.cell + c.off, a.P.ox + c.off, a.P.oy + c.off, a.P.vx + c.off,
                                        a.P.vy + c.off, a.P.vz + c.off, a.P.id + c.off};
    for (int k = 0; k < ncols; ++k)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                     ::"r"(stage_base + (uint32_t)(k * SUB * 4)), "l"(src[k]), "r"(bytes), "r"(bar)
                     : "memory");
}

template <bool PER>
__device__ __forceinline__ void window_load(const PushArgs& a, Smem& s, int wx0, int wy0)
{
    const edp_kparams& kp = a.kp;
    for (int t = threadIdx.x; t < EDP_WIN_NODES * EDP_WIN_NODES; t += blockDim.x) {
        int lx = t % EDP_WIN_NODES, ly = t / EDP_WIN_NODES;
        int gx = wrapx(wx0 + lx, kp), gy = wy0 + ly;
        bool ok = gx >= 0 && gx < kp.nxg && gy >= 0 && gy < kp.nyg;
        s.E[t] = ok ? __ldg(&a.E[(int64_t)gy * kp.nxg + gx]) : make_float2(0.f, 0.f);
        s.hi[t] = 0;
        s.lo[t] = 0u;
    }
}

__device__ __forceinline__ void window_flush(const PushArgs& a, Smem& s, int wx0, int wy0)
{
    const edp_kparams& kp = a.kp;
    for (int t = threadIdx.x; t < EDP_WIN_NODES * EDP_WIN_NODES; t += blockDim.x) {
        long long v = (long long)s.hi[t] * 65536LL + (long long)s.lo[t];
        if (v == 0) continue;
        int lx = t % EDP_WIN_NODES, ly = t / EDP_WIN_NODES;
        int gx = wrapx(wx0 + lx, kp), gy = wy0 + ly;
        if (gx >= 0 && gx < kp.nxg && gy >= 0 && gy < kp.nyg)
            atomicAdd(&a.rho[(int64_t)gy * kp.nxg + gx], (unsigned long long)v);
        else atomicOr(&a.dc->error_flags, EDP_EFLAG_BOUNDS);
    }
}

template <bool ION, bool PER, bool ROT, int IPT, int NST>
__global__ void __launch_bounds__(EDP_PUSH_THREADS, IPT == 4 ? 3 : 4) push_stream_kernel(PushArgs a)
{
    constexpr int SUB = EDP_PUSH_THREADS * IPT;
    constexpr int STAGE_BYTES = EDP_STREAM_COLS * SUB * 4;
    extern __shared__ __align__(128) unsigned char stage_mem[];
    __shared__ Smem s;
    __shared__ __align__(8) uint64_t full[NST];
    int fail = 0;
    const int tid = threadIdx.x;
    const int ncols = a.need_id ? EDP_STREAM_COLS : EDP_STREAM_COLS - 1;
    const uint32_t stage0 = push_smem_u32(stage_mem);
    if (tid < 32) s.cnt[tid] = 0ull;
    if (tid == 0) {
        s.nsel = 0u;
        for (int k = 0; k < NST; ++k) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(push_smem_u32(&full[k])));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    // producer: thread 0 fills every stage first
    StreamCursor prod;
    int64_t issued = 0;
    if (tid == 0) {
        cursor_first<SUB>(a, prod);
        for (int k = 0; k < NST && prod.chunk < a.n_chunks; ++k) {
            stream_issue<SUB>(a, prod, stage0 + (uint32_t)(k * STAGE_BYTES), push_smem_u32(&full[k]), ncols);
            ++issued;
            cursor_next<SUB>(a, prod);
        }
    }
    StreamCursor cur;
    cursor_first<SUB>(a, cur);
    int64_t win = -1, consumed = 0;
    int wx0 = 0, wy0 = 0;
    int st = 0;
    uint32_t ph = 0;
    for (; cur.chunk < a.n_chunks; cursor_next<SUB>(a, cur)) {
        if (cur.chunk != win) {   // a new chunk: flush the previous window, stage the new field window
            if (win >= 0) {
                __syncthreads();
                window_flush(a, s, wx0, wy0);
                __syncthreads();
            }
            const edp_chunk ch = a.chunks[cur.chunk];
            wx0 = ch.wx0;
            wy0 = ch.wy0;
            window_load<PER>(a, s, wx0, wy0);
            win = cur.chunk;
        }
        const bool landed = push_mbar_wait(push_smem_u32(&full[st]), ph);
        // the stage has landed; every thread is done with the previous stage and the window; the same verdict
        // reaches every thread
        if (__syncthreads_or(landed ? 0 : 1)) {
            fail = 1;
            break;
        }
        // refill the stage the previous sub-chunk used
        if (tid == 0 && consumed > 0 && prod.chunk < a.n_chunks) {
            const int ps = (st + NST - 1) % NST;
            stream_issue<SUB>(a, prod, stage0 + (uint32_t)(ps * STAGE_BYTES), push_smem_u32(&full[ps]), ncols);
            ++issued;
            cursor_next<SUB>(a, prod);
        }
        const int64_t base = cur.off + (int64_t)tid * IPT;
        if (base < cur.end) {
            const unsigned char* sb = stage_mem + st * STAGE_BYTES;
            int c[IPT];
            float ox[IPT], oy[IPT], vx[IPT], vy[IPT], vz[IPT];
            uint32_t id[IPT];
            const bool with_id = ncols == EDP_STREAM_COLS;
            if constexpr (IPT == 4) {
                const int4 c4 = reinterpret_cast<const int4*>(sb)[tid];
                const float4 ox4 = reinterpret_cast<const float4*>(sb + 1 * SUB * 4)[tid];
                const float4 oy4 = reinterpret_cast<const float4*>(sb + 2 * SUB * 4)[tid];
                const float4 vx4 = reinterpret_cast<const float4*>(sb + 3 * SUB * 4)[tid];
                const float4 vy4 = reinterpret_cast<const float4*>(sb + 4 * SUB * 4)[tid];
                const float4 vz4 = reinterpret_cast<const float4*>(sb + 5 * SUB * 4)[tid];
                const uint4 id4 = with_id ? reinterpret_cast<const uint4*>(sb + 6 * SUB * 4)[tid] : make_uint4(0, 0, 0, 0);
                c[0] = c4.x; c[1] = c4.y; c[2] = c4.z; c[3] = c4.w;
                ox[0] = ox4.x; ox[1] = ox4.y; ox[2] = ox4.z; ox[3] = ox4.w;
                oy[0] = oy4.x; oy[1] = oy4.y; oy[2] = oy4.z; oy[3] = oy4.w;
                vx[0] = vx4.x; vx[1] = vx4.y; vx[2] = vx4.z; vx[3] = vx4.w;
                vy[0] = vy4.x; vy[1] = vy4.y; vy[2] = vy4.z; vy[3] = vy4.w;
                vz[0] = vz4.x; vz[1] = vz4.y; vz[2] = vz4.z; vz[3] = vz4.w;
                id[0] = id4.x; id[1] = id4.y; id[2] = id4.z; id[3] = id4.w;
            } else {
                const int2 c2 = reinterpret_cast<const int2*>(sb)[tid];
                const float2 ox2 = reinterpret_cast<const float2*>(sb + 1 * SUB * 4)[tid];
                const float2 oy2 = reinterpret_cast<const float2*>(sb + 2 * SUB * 4)[tid];
                const float2 vx2 = reinterpret_cast<const float2*>(sb + 3 * SUB * 4)[tid];
                const float2 vy2 = reinterpret_cast<const float2*>(sb + 4 * SUB * 4)[tid];
                const float2 vz2 = reinterpret_cast<const float2*>(sb + 5 * SUB * 4)[tid];
                const uint2 id2 = with_id ? reinterpret_cast<const uint2*>(sb + 6 * SUB * 4)[tid] : make_uint2(0, 0);
                c[0] = c2.x; c[1] = c2.y;
                ox[0] = ox2.x; ox[1] = ox2.y;
                oy[0] = oy2.x; oy[1] = oy2.y;
                vx[0] = vx2.x; vx[1] = vx2.y;
                vy[0] = vy2.x; vy[1] = vy2.y;
                vz[0] = vz2.x; vz[1] = vz2.y;
                id[0] = id2.x; id[1] = id2.y;
            }
            DepAcc acc;
            acc.b = -1;
#pragma unroll
            for (int e = 0; e < IPT; ++e) {
                if (c[e] < 0) continue;
                bool sel = false;
                if (!push_one<ION, PER, ROT>(a, s, true, wx0, wy0, acc, c[e], ox[e], oy[e], vx[e], vy[e], vz[e], id[e],
                                             sel)) {
                    c[e] = -1;
                    atomicAdd(&s.cnt[17], 1ull);
                } else if (sel) {
                    select_slot(a, s, (uint32_t)(base + e));
                }
            }
            dep_flush(s, acc);
            if constexpr (IPT == 4) {
                const int64_t g = base / 4;
                __stcs(reinterpret_cast<int4*>(a.P.cell) + g, make_int4(c[0], c[1], c[2], c[3]));
                __stcs(reinterpret_cast<float4*>(a.P.ox) + g, make_float4(ox[0], ox[1], ox[2], ox[3]));
                __stcs(reinterpret_cast<float4*>(a.P.oy) + g, make_float4(oy[0], oy[1], oy[2], oy[3]));
                __stcs(reinterpret_cast<float4*>(a.P.vx) + g, make_float4(vx[0], vx[1], vx[2], vx[3]));
                __stcs(reinterpret_cast<float4*>(a.P.vy) + g, make_float4(vy[0], vy[1], vy[2], vy[3]));
                __stcs(reinterpret_cast<float4*>(a.P.vz) + g, make_float4(vz[0], vz[1], vz[2], vz[3]));
            } else {
                const int64_t g = base / 2;
                __stcs(reinterpret_cast<int2*>(a.P.cell) + g, make_int2(c[0], c[1]));
                __stcs(reinterpret_cast<float2*>(a.P.ox) + g, make_float2(ox[0], ox[1]));
                __stcs(reinterpret_cast<float2*>(a.P.oy) + g, make_float2(oy[0], oy[1]));
                __stcs(reinterpret_cast<float2*>(a.P.vx) + g, make_float2(vx[0], vx[1]));
                __stcs(reinterpret_cast<float2*>(a.P.vy) + g, make_float2(vy[0], vy[1]));
                __stcs(reinterpret_cast<float2*>(a.P.vz) + g, make_float2(vz[0], vz[1]));
            }
        }
        ++consumed;
        if (++st == NST) {
            st = 0;
            ph ^= 1u;
        }
    }
    __syncthreads();
    if (fail) {
        // a wait gave up: wait (bounded) for the copies still in flight into this CTA's stages, then leave
        if (tid == 0) {
            atomicOr(&a.dc->error_flags, EDP_EFLAG_TIMEOUT);
            for (int64_t k = consumed; k < issued; ++k)
                push_mbar_wait(push_smem_u32(&full[k % NST]), (uint32_t)((k / NST) & 1));
        }
        return;
    }
    if (win >= 0) window_flush(a, s, wx0, wy0);
    if (!ION) {
        __shared__ unsigned long long sel_base;
        const unsigned nsel = min(s.nsel, (unsigned)EDP_SEL_SMEM);
        if (tid == 0 && nsel) sel_base = atomicAdd(a.sel_count, (unsigned long long)nsel);
        __syncthreads();
        for (unsigned q = tid; q < nsel; q += blockDim.x) {
            unsigned long long g = sel_base + q;
            if ((int64_t)g < a.sel_cap) a.sel_list[g] = s.sel[q];
            else atomicOr(&a.dc->error_flags, EDP_EFLAG_PENDING);
        }
    }
    if (tid < 32) {
        unsigned long long v = s.cnt[tid];
        if (v) {
            int k = tid;
            if (k < 8) atomicAdd(ION ? &a.dc->i_hits[k] : &a.dc->e_hits[k], v);
            else if (k < 16) {
                atomicAdd(&a.dc->en_coll[k - 8], v);
                atomicAdd(&a.dc->en_coll_step[k - 8], v);
            } else if (k == 16) {
                atomicAdd(&a.dc->rcx[a.species - 1], v);
                atomicAdd(&a.dc->rcx_step[a.species - 1], v);
            } else if (k == 17) {
                atomicAdd(&a.dc->n_live[a.species], (unsigned long long)(-(long long)v));
            }
        }
    }
}

struct SelArgs {
    edp_kparams kp;
    edp_species_mixed P;
    const uint32_t* sel_list;
    const unsigned long long* sel_count;
    int64_t sel_cap;
    uint32_t step;
    const edp_mcc_dev* mcc;
    const edp_born_dev* born;
    edp_dev_counters* dc;
};

// kind choice and scattering of the electrons the push selected (PERFORM_ELECTRON_NEUTRAL_COLLISIONS :447-485 and
// en_Collision_*), on the post-push velocities, with the selection's kind variate recomputed from Philox block 0
__global__ void __launch_bounds__(256) collide_selected_kernel(SelArgs a)
{
    __shared__ unsigned long long cnt[EDP_MAX_COLPROC];
    if (threadIdx.x < EDP_MAX_COLPROC) cnt[threadIdx.x] = 0ull;
    __syncthreads();
    unsigned long long n = *a.sel_count;
    if ((int64_t)n > a.sel_cap) n = (unsigned long long)a.sel_cap;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < (int64_t)n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t slot = a.sel_list[k];
        const uint32_t id = a.P.id[slot];
        double r;
        if (!edp_mcc_select(a.mcc, id, a.step, a.kp.seed_lo, a.kp.seed_hi, r)) continue;
        double v[3] = {(double)a.P.vx[slot], (double)a.P.vy[slot], (double)a.P.vz[slot]};
        edp_mcc_out o;
        edp_mcc_collide(a.mcc, id, a.step, a.kp.seed_lo, a.kp.seed_hi, r, v, &o);
        if (!o.kind_index) continue;
        a.P.vx[slot] = (float)v[0];
        a.P.vy[slot] = (float)v[1];
        a.P.vz[slot] = (float)v[2];
        atomicAdd(&cnt[o.kind_index - 1], 1ull);
        if (o.born) {
            const int c = a.P.cell[slot];
            const double X = (double)(c & 0xFFFF) + (double)a.P.ox[slot];
            const double Y = (double)(c >> 16) + (double)a.P.oy[slot];
            record_born(a.born->born_e, &a.dc->born_e_count, &a.dc->error_flags, X, Y, o.ne);
            record_born(a.born->born_i[o.ion_species], &a.dc->born_i_count[o.ion_species], &a.dc->error_flags, X, Y,
                        o.ni);
        }
    }
    __syncthreads();
    if (threadIdx.x < EDP_MAX_COLPROC && cnt[threadIdx.x]) {
        atomicAdd(&a.dc->en_coll[threadIdx.x], cnt[threadIdx.x]);
        atomicAdd(&a.dc->en_coll_step[threadIdx.x], cnt[threadIdx.x]);
    }
}

// ---------------------------------------------------------------------------------------- FP64 path
struct PushArgs64 {
    edp_kparams kp;
    edp_species_fp64 P;
    const unsigned long long* n_slots;
    const double *Ex, *Ey;
    double* rho;
    double K[9];
    double qh, ez_term;
    int xmul, use_rot, is_ion, species, do_mcc, do_rcx;
    uint32_t step;
    const edp_mcc_dev* mcc;
    edp_rcx_dev rcx;
    edp_dev_counters* dc;
    edp_born born_e;
    edp_born born_i[EDP_MAX_ION_SPECIES];
    edp_hits hits;              // wall-hit list of ion-induced electron emission
    int emit_on;
};

// The plain FP64 cycle: one particle per thread, the reference's arithmetic in FP64, global atomics.
__global__ void __launch_bounds__(256) push_fp64_kernel(PushArgs64 a)
{
    __shared__ unsigned long long cnt[32];
    const edp_kparams& kp = a.kp;
    if (threadIdx.x < 32) cnt[threadIdx.x] = 0ull;
    __syncthreads();
    const int64_t n = (int64_t)*a.n_slots;
    const double xmax = kp.periodic ? (double)kp.ncx : (double)kp.ncx, ymax = (double)kp.ncy;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double X = a.P.x[k];
        if (X < -1.0e29) continue;
        double Y = a.P.y[k];
        int i = (int)X, j = (int)Y;
        if (!kp.periodic && X == xmax) i = kp.ncx - 1;
        if (Y == ymax) j = kp.ncy - 1;
        int i1 = i + 1;
        if (kp.periodic && i1 == kp.ncx) i1 = 0;
        int64_t r0 = (int64_t)j * kp.nxg, r1 = r0 + kp.nxg;
        double axp = X - (double)i, axm = 1.0 - axp, ayp = Y - (double)j, aym = 1.0 - ayp;
        double EX = a.Ex[r0 + i] * axm * aym + a.Ex[r0 + i1] * axp * aym + a.Ex[r1 + i] * axm * ayp +
                    a.Ex[r1 + i1] * axp * ayp;
        double EY = a.Ey[r0 + i] * axm * aym + a.Ey[r0 + i1] * axp * aym + a.Ey[r1 + i] * axm * ayp +
                    a.Ey[r1 + i1] * axp * ayp;
        double vx = a.P.vx[k], vy = a.P.vy[k], vz = a.P.vz[k];
        double q = a.qh;
        if (a.use_rot) {
            double mx = vx + q * EX, my = vy + q * EY, mz = vz + a.ez_term;
            double px = a.K[0] * mx + a.K[1] * my + a.K[2] * mz;
            double py = a.K[3] * mx + a.K[4] * my + a.K[5] * mz;
            double pz = a.K[6] * mx + a.K[7] * my + a.K[8] * mz;
            vx = px + q * EX;
            vy = py + q * EY;
            vz = pz + a.ez_term;
        } else if (a.is_ion) {
            vx = vx + (q + q) * EX;
            vy = vy + (q + q) * EY;
            vz = vz + (a.ez_term + a.ez_term);
        } else {
            vx = (vx + q * EX) + q * EX;
            vy = (vy + q * EY) + q * EY;
            vz = (vz + a.ez_term) + a.ez_term;
        }
        X = X + vx * a.xmul;
        Y = Y + vy * a.xmul;
        int obj = -1;
        for (int n2 = 0; n2 < kp.n_inner; ++n2) {
            if (X <= (double)kp.ileft[n2] || X >= (double)kp.iright[n2]) continue;
            if (Y <= (double)kp.jbottom[n2] || Y >= (double)kp.jtop[n2]) continue;
            obj = 4 + n2;
            break;
        }
        if (obj < 0) {
            if (kp.periodic) {
                if (X < 0.0) X += (double)kp.ncx;
                else if (X >= (double)kp.ncx) X -= (double)kp.ncx;
                if (Y < 0.0) obj = 0;
                else if (Y > ymax) obj = 1;
            } else if (X < 0.0 || X > xmax || Y < 0.0 || Y > ymax) {
                obj = wall_object(X, Y, xmax, ymax);
            }
        }
        if (obj >= 0) {
            a.P.x[k] = -1.0e30;
            atomicAdd(&cnt[obj], 1ull);
            atomicAdd(&cnt[17], 1ull);
            if ((a.emit_on && obj < 4) ||
                (obj >= 4 &&
                 (((kp.diel_mask | (a.is_ion ? kp.ion_inner_mask : kp.see_inner_mask)) >> (obj - 4)) & 1)))
                record_hit(a.hits, a.dc, obj, a.is_ion ? a.species - 1 : 0, X, Y, vx, vy, vz, a.P.id[k]);
            continue;
        }
        // deposit
        i = (int)X;
        j = (int)Y;
        if (!kp.periodic && X == xmax) i = kp.ncx - 1;
        if (Y == ymax) j = kp.ncy - 1;
        i1 = i + 1;
        if (kp.periodic && i1 == kp.ncx) i1 = 0;
        r0 = (int64_t)j * kp.nxg;
        r1 = r0 + kp.nxg;
        double dx = X - (double)i, dy = Y - (double)j;
        double vij = (1.0 - dx) * (1.0 - dy), vip1j = dx * (1.0 - dy), vijp1 = (1.0 - dx) * dy;
        atomicAdd(&a.rho[r0 + i], vij);
        atomicAdd(&a.rho[r0 + i1], vip1j);
        atomicAdd(&a.rho[r1 + i], vijp1);
        atomicAdd(&a.rho[r1 + i1], 1.0 - vij - vip1j - vijp1);
        if (a.do_mcc) {
            edp_mcc_out o = edp_mcc_electron(a.mcc, a.P.id[k], a.step, kp.seed_lo, kp.seed_hi, vx, vy, vz);
            if (o.kind_index) {
                atomicAdd(&cnt[8 + o.kind_index - 1], 1ull);
                if (o.born) {
                    record_born(a.born_e, &a.dc->born_e_count, &a.dc->error_flags, X, Y, o.ne);
                    record_born(a.born_i[o.ion_species], &a.dc->born_i_count[o.ion_species], &a.dc->error_flags,
                                X, Y, o.ni);
                }
            }
        }
        if (a.do_rcx) {
            if (edp_rcx_ion(a.rcx, a.P.id[k], a.step, (uint32_t)(a.species - 1), kp.seed_lo, kp.seed_hi, vx, vy, vz))
                atomicAdd(&cnt[16], 1ull);
        }
        a.P.x[k] = X;
        a.P.y[k] = Y;
        a.P.vx[k] = vx;
        a.P.vy[k] = vy;
        a.P.vz[k] = vz;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long v = cnt[threadIdx.x];
        if (v) {
            int k = threadIdx.x;
            if (k < 8) atomicAdd(a.is_ion ? &a.dc->i_hits[k] : &a.dc->e_hits[k], v);
            else if (k < 16) {
                atomicAdd(&a.dc->en_coll[k - 8], v);
                atomicAdd(&a.dc->en_coll_step[k - 8], v);
            } else if (k == 16) {
                atomicAdd(&a.dc->rcx[a.species - 1], v);
                atomicAdd(&a.dc->rcx_step[a.species - 1], v);
            } else if (k == 17) {
                atomicAdd(&a.dc->n_live[a.species], (unsigned long long)(-(long long)v));
            }
        }
    }
}

// --------------------------------------------------------------------------- separate collision passes
struct CollArgs {
    edp_kparams kp;
    int precision, species;
    edp_species_mixed Pm;
    edp_species_fp64 Pd;
    const unsigned long long* n_slots;
    uint32_t step;
    const edp_mcc_dev* mcc;
    edp_rcx_dev rcx;
    edp_dev_counters* dc;
    edp_born born_e;
    edp_born born_i[EDP_MAX_ION_SPECIES];
};

// PERFORM_ELECTRON_NEUTRAL_COLLISIONS as its own pass over the electron array
__global__ void collide_en_kernel(CollArgs a)
{
    __shared__ unsigned long long cnt[EDP_MAX_COLPROC];
    if (threadIdx.x < EDP_MAX_COLPROC) cnt[threadIdx.x] = 0ull;
    __syncthreads();
    const int64_t n = (int64_t)*a.n_slots;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double vx, vy, vz, X, Y;
        uint32_t id;
        if (a.precision == EDP_PREC_MIXED) {
            int c = a.Pm.cell[k];
            if (c < 0) continue;
            vx = a.Pm.vx[k];
            vy = a.Pm.vy[k];
            vz = a.Pm.vz[k];
            X = (double)(c & 0xFFFF) + (double)a.Pm.ox[k];
            Y = (double)(c >> 16) + (double)a.Pm.oy[k];
            id = a.Pm.id[k];
        } else {
            X = a.Pd.x[k];
            if (X < -1.0e29) continue;
            Y = a.Pd.y[k];
            vx = a.Pd.vx[k];
            vy = a.Pd.vy[k];
            vz = a.Pd.vz[k];
            id = a.Pd.id[k];
        }
        edp_mcc_out o = edp_mcc_electron(a.mcc, id, a.step, a.kp.seed_lo, a.kp.seed_hi, vx, vy, vz);
        if (!o.kind_index) continue;
        atomicAdd(&cnt[o.kind_index - 1], 1ull);
        if (a.precision == EDP_PREC_MIXED) {
            a.Pm.vx[k] = (float)vx;
            a.Pm.vy[k] = (float)vy;
            a.Pm.vz[k] = (float)vz;
        } else {
            a.Pd.vx[k] = vx;
            a.Pd.vy[k] = vy;
            a.Pd.vz[k] = vz;
        }
        if (o.born) {
            record_born(a.born_e, &a.dc->born_e_count, &a.dc->error_flags, X, Y, o.ne);
            record_born(a.born_i[o.ion_species], &a.dc->born_i_count[o.ion_species], &a.dc->error_flags, X, Y, o.ni);
        }
    }
    __syncthreads();
    if (threadIdx.x < EDP_MAX_COLPROC && cnt[threadIdx.x]) {
        atomicAdd(&a.dc->en_coll[threadIdx.x], cnt[threadIdx.x]);
        atomicAdd(&a.dc->en_coll_step[threadIdx.x], cnt[threadIdx.x]);
    }
}

// PERFORM_RESONANT_CHARGE_EXCHANGE as its own pass over one ion species
__global__ void collide_rcx_kernel(CollArgs a)
{
    __shared__ unsigned long long cnt;
    if (threadIdx.x == 0) cnt = 0ull;
    __syncthreads();
    const int64_t n = (int64_t)*a.n_slots;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double vx, vy, vz;
        uint32_t id;
        if (a.precision == EDP_PREC_MIXED) {
            if (a.Pm.cell[k] < 0) continue;
            vx = a.Pm.vx[k];
            vy = a.Pm.vy[k];
            vz = a.Pm.vz[k];
            id = a.Pm.id[k];
        } else {
            if (a.Pd.x[k] < -1.0e29) continue;
            vx = a.Pd.vx[k];
            vy = a.Pd.vy[k];
            vz = a.Pd.vz[k];
            id = a.Pd.id[k];
        }
        if (!edp_rcx_ion(a.rcx, id, a.step, (uint32_t)(a.species - 1), a.kp.seed_lo, a.kp.seed_hi, vx, vy, vz)) continue;
        atomicAdd(&cnt, 1ull);
        if (a.precision == EDP_PREC_MIXED) {
            a.Pm.vx[k] = (float)vx;
            a.Pm.vy[k] = (float)vy;
            a.Pm.vz[k] = (float)vz;
        } else {
            a.Pd.vx[k] = vx;
            a.Pd.vy[k] = vy;
            a.Pd.vz[k] = vz;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && cnt) {
        atomicAdd(&a.dc->rcx[a.species - 1], cnt);
        atomicAdd(&a.dc->rcx_step[a.species - 1], cnt);
    }
}

// ------------------------------------------------------------------------------------- appending
struct AppendArgs {
    edp_kparams kp;
    int precision, species;
    edp_species_mixed Pm;
    edp_species_fp64 Pd;
    int64_t cap;
    edp_born src;
    const unsigned long long* src_count;
    unsigned long long* n_slots;
    unsigned long long* n_live;
    unsigned long long* next_id;
    unsigned long long id_end;   // one past the context's last id
    unsigned long long* rho_fix;
    double* rho_d;
    edp_dev_counters* dc;
};

// PROCESS_ADDED_ELECTRONS / PROCESS_ADDED_IONS (pic2d_ElectronDynamics.f90:1429-1531,
// pic2d_IonDynamics.f90:1468-1537), called at the end of the step (pic2d_MainProgram.f90:300, :363): the add list
// joins the main array and is deposited at its birth positions into the density the next step's field solve uses
// (the density GATHER_*_CHARGE_DENSITY takes at the start of the next step).
__global__ void append_kernel(AppendArgs a)
{
    const edp_kparams& kp = a.kp;
    const int64_t n = (int64_t)*a.src_count;
    const int64_t nread = n < a.src.cap ? n : a.src.cap;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nread; k += (int64_t)gridDim.x * blockDim.x) {
        double X = a.src.x[k], Y = a.src.y[k];
        double vx = a.src.vx[k], vy = a.src.vy[k], vz = a.src.vz[k];
        const unsigned long long id_l = atomicAdd(a.next_id, 1ull);
        if (id_l >= a.id_end) {   // the range is used up: an id of another rank's range would repeat its streams
            atomicOr(&a.dc->error_flags, EDP_EFLAG_IDS);
            continue;
        }
        const uint32_t id = (uint32_t)id_l;
        unsigned long long slot = atomicAdd(a.n_slots, 1ull);
        if ((int64_t)slot >= a.cap) {
            atomicOr(&a.dc->error_flags, EDP_EFLAG_CAPACITY);
            continue;
        }
        atomicAdd(a.n_live, 1ull);
        int i = (int)X, j = (int)Y;
        if (!kp.periodic && i == kp.ncx) i = kp.ncx - 1;
        if (j == kp.ncy) j = kp.ncy - 1;
        if (kp.periodic && i >= kp.ncx) i -= kp.ncx;
        double dx = X - (double)((int)X), dy = Y - (double)j;
        if (!kp.periodic && (int)X == kp.ncx) dx = 1.0;
        int i1 = i + 1;
        if (kp.periodic && i1 == kp.ncx) i1 = 0;
    int64_t r0 = (int64_t)j * kp.nxg, r1 = r0 + kp.nxg;
        if (a.precision == EDP_PREC_MIXED) {
            float fx = (float)dx, fy = (float)dy;
            a.Pm.cell[slot] = (j << 16) | i;
            a.Pm.ox[slot] = fx;
            a.Pm.oy[slot] = fy;
            a.Pm.vx[slot] = (float)vx;
            a.Pm.vy[slot] = (float)vy;
            a.Pm.vz[slot] = (float)vz;
            a.Pm.id[slot] = id;
            a.Pm.tag[slot] = 0;
            double ddx = fx, ddy = fy;
            double vij = (1.0 - ddx) * (1.0 - ddy), vip1j = ddx * (1.0 - ddy), vijp1 = (1.0 - ddx) * ddy;
            long long q00 = __double2ll_rn(vij * EDP_FIX_ONE), q10 = __double2ll_rn(vip1j * EDP_FIX_ONE);
            long long q01 = __double2ll_rn(vijp1 * EDP_FIX_ONE), q11 = 4294967296LL - q00 - q10 - q01;
            atomicAdd(&a.rho_fix[r0 + i], (unsigned long long)q00);
            atomicAdd(&a.rho_fix[r0 + i1], (unsigned long long)q10);
            atomicAdd(&a.rho_fix[r1 + i], (unsigned long long)q01);
            atomicAdd(&a.rho_fix[r1 + i1], (unsigned long long)q11);
        } else {
            a.Pd.x[slot] = (double)i + dx;
            a.Pd.y[slot] = Y;
            a.Pd.vx[slot] = vx;
            a.Pd.vy[slot] = vy;
            a.Pd.vz[slot] = vz;
            a.Pd.id[slot] = id;
            a.Pd.tag[slot] = 0;
            double vij = (1.0 - dx) * (1.0 - dy), vip1j = dx * (1.0 - dy), vijp1 = (1.0 - dx) * dy;
            atomicAdd(&a.rho_d[r0 + i], vij);
            atomicAdd(&a.rho_d[r0 + i1], vip1j);
            atomicAdd(&a.rho_d[r1 + i], vijp1);
            atomicAdd(&a.rho_d[r1 + i1], 1.0 - vij - vip1j - vijp1);
        }
    }
}

void fill_rot(const edp_ctx* c, int species, float* Kf, double* Kd)
{
    for (int q = 0; q < 9; ++q) {
        if (Kf) Kf[q] = (float)c->K[species][q];
        if (Kd) Kd[q] = c->K[species][q];
    }
}

}  // namespace

// ------------------------------------------------------------------------------------------- launch
template <bool ION, bool PER, bool ROT, int IPT, int NST>
static int launch_stream_variant(edp_ctx* c, const PushArgs& a)
{
    auto k = push_stream_kernel<ION, PER, ROT, IPT, NST>;
    const size_t smem = (size_t)NST * EDP_STREAM_COLS * EDP_PUSH_THREADS * IPT * 4;
    TRY(edp_raise_smem_limit(c, (const void*)k, smem));
    static int per_sm[2][2][2] = {};   // resident CTAs per SM of this instantiation, found once per process
    static int n_sm = 0;
    int& r = per_sm[ION][PER][ROT];
    if (!r) {
        EDP_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k, EDP_PUSH_THREADS, smem));
        if (r < 1) r = 1;
    }
    if (!n_sm) EDP_CUDA(c, cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, c->device));
    const int64_t grid = std::min<int64_t>(a.n_chunks, (int64_t)n_sm * r);
    k<<<(unsigned)grid, EDP_PUSH_THREADS, smem, c->stream>>>(a);
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

template <int IPT, int NST>
static int launch_stream_kind(edp_ctx* c, int variant, const PushArgs& a)
{
    switch (variant) {
    case 0: return launch_stream_variant<false, false, false, IPT, NST>(c, a);
    case 1: return launch_stream_variant<false, false, true, IPT, NST>(c, a);
    case 2: return launch_stream_variant<false, true, false, IPT, NST>(c, a);
    case 3: return launch_stream_variant<false, true, true, IPT, NST>(c, a);
    case 4: return launch_stream_variant<true, false, false, IPT, NST>(c, a);
    case 5: return launch_stream_variant<true, false, true, IPT, NST>(c, a);
    case 6: return launch_stream_variant<true, true, false, IPT, NST>(c, a);
    default: return launch_stream_variant<true, true, true, IPT, NST>(c, a);
    }
}

static int launch_stream_push(edp_ctx* c, int variant, int kind, const PushArgs& a)
{
    return kind == 2 ? launch_stream_kind<2, 3>(c, variant, a) : launch_stream_kind<4, 2>(c, variant, a);
}

template <int IPT, bool SCAT, bool PF>
static int launch_classic_push(edp_ctx* c, int variant, unsigned gr, const PushArgs& a)
{
    switch (variant) {
    case 0: push_mixed_kernel<false, false, false, IPT, SCAT, PF><<<gr, EDP_PUSH_THREADS, 0, c->stream>>>(a); break;
    case 1: push_mixed_kernel<false, false, true, IPT, SCAT, PF><<<gr, EDP_PUSH_THREADS, 0, c->stream>>>(a); break;
    case 2: push_mixed_kernel<false, true, false, IPT, SCAT, PF><<<gr, EDP_PUSH_THREADS, 0, c->stream>>>(a); break;
    case 3: push_mixed_kernel<false, true, true, IPT, SCAT, PF><<<gr, EDP_PUSH_THREADS, 0, c->stream>>>(a); break;
    case 4: push_mixed_kernel<true, false, false, IPT, SCAT, PF><<<gr, EDP_PUSH_THREADS, 0, c->stream>>>(a); break;
    case 5: push_mixed_kernel<true, false, true, IPT, SCAT, PF><<<gr, EDP_PUSH_THREADS, 0, c->stream>>>(a); break;
    case 6: push_mixed_kernel<true, true, false, IPT, SCAT, PF><<<gr, EDP_PUSH_THREADS, 0, c->stream>>>(a); break;
    default: push_mixed_kernel<true, true, true, IPT, SCAT, PF><<<gr, EDP_PUSH_THREADS, 0, c->stream>>>(a); break;
    }
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

int edp_set_push_kernel(edp_ctx* c, int32_t kind)
{
    if (!c || kind < 0 || kind > 4) return edp_fail(c, EDP_ERR_ARG, "edp_set_push_kernel");
    c->push_kernel = kind;
    return EDP_OK;
}

int edp_launch_push(edp_ctx* c, int sp, bool ion_step, bool fuse)
{
    const edp_params& p = c->p;
    const bool is_ion = sp > 0;
    const int s = sp - 1;
    const double qh = is_ion ? 0.5 * p.ion_charge[s] / p.ion_mass_me[s] : -0.5;
    double ez_term;
    int use_rot;
    if (!is_ion) {
        ez_term = -0.5 * p.ez;
        use_rot = (p.bx != 0.0 || p.by != 0.0 || p.bz != 0.0);
    } else {
        ez_term = p.ions_sense_ez ? qh * p.ez * p.n_subcycles : 0.0;
        use_rot = p.ions_sense_b && (p.bx != 0.0 || p.by != 0.0 || p.bz != 0.0);
    }
    const bool do_mcc = fuse && !is_ion && ion_step && c->tab.en_on;
    const bool do_rcx = fuse && is_ion && ion_step && c->tab.rcx_on[s];
    if (p.precision == EDP_PREC_MIXED) {
        PushArgs a;
        memset(&a, 0, sizeof(a));
        a.kp = c->kp;
        a.P = c->pm[sp];
        a.chunks = c->chunks[sp];
        a.n_chunks = c->n_chunks[sp];
        a.tail_start = c->sorted_end[sp];
        a.n_slots = &c->dc->n_slots[sp];
        a.E = is_ion ? c->acc2 : c->E2;
        a.rho = c->rho_fix[sp];
        fill_rot(c, sp, a.K, nullptr);
        a.qh = (float)qh;
        a.ez_term = (float)ez_term;
        a.xmul = is_ion ? (float)p.n_subcycles : 1.0f;
        a.use_rot = use_rot;
        a.species = sp;
        a.do_coll = do_mcc || do_rcx;
        a.step = (uint32_t)c->t_cntr;
        a.draw_base = edp_draw_base(c->kp.seed_lo, c->kp.seed_hi, is_ion ? EDP_SEL_RCX((uint32_t)s) : EDP_SEL_MCC,
                                    a.step);
        a.mcc = c->mcc_dev;
        if (do_rcx) a.rcx = edp_make_rcx_dev(c, s);
        a.dc = c->dc;
        a.sel_list = c->sel_list;
        a.sel_count = c->sel_count;
        a.sel_cap = c->sel_cap;
        a.hits = c->hits;
        a.emit_on = is_ion ? c->emit_on : c->see_on;
        a.need_id = a.do_coll || a.emit_on || (is_ion ? c->kp.ion_inner_mask : c->kp.see_inner_mask) != 0;
        if (do_mcc) EDP_CUDA(c, cudaMemsetAsync(c->sel_count, 0, sizeof(unsigned long long), c->stream));
        int64_t tail = c->host_slots[sp] - c->sorted_end[sp];
        if (tail < 0) tail = 0;
        int64_t per_cta = (int64_t)EDP_PUSH_THREADS * EDP_ITEMS * 8;
        a.tail_ctas = (tail + per_cta - 1) / per_cta;
        if (a.tail_ctas < 1) a.tail_ctas = 1;
        // a sort due for this species happens in this push: the particles go to their sorted slots in the other
        // arrays (the keys are those of the cells before the push, so a particle ends within a cell of its tile)
        const bool fused = c->sort_due[sp] != 0;
        if (fused) {
            unsigned long long* cur = nullptr;
            TRY(edp_sort_prepare(c, sp, &cur));
            a.D = c->pm_alt[sp];
            a.cursor = cur;
            a.ntx = c->ntx;
            a.cap = c->cap[sp];
        }
        ++c->launches;
        const int variant = (is_ion ? 4 : 0) | (c->kp.periodic ? 2 : 0) | (use_rot ? 1 : 0);
        bool classic = true;
        if ((c->push_kernel == 1 || c->push_kernel == 2) && a.n_chunks > 0 && !fused) {
            // the sorted chunks by the streaming kernel, the unsorted tail (if any) by the per-chunk kernel
            TRY(launch_stream_push(c, variant, c->push_kernel, a));
            a.n_chunks = 0;
            classic = tail > 0;
            if (classic) ++c->launches;
        }
        const unsigned gr = (unsigned)(a.n_chunks + a.tail_ctas);
        if (classic) {
            if (fused) TRY((launch_classic_push<4, true, false>(c, variant, gr, a)));
            else if (c->push_kernel == 3) TRY((launch_classic_push<2, false, false>(c, variant, gr, a)));
            else if (c->push_kernel == 4) TRY((launch_classic_push<4, false, true>(c, variant, gr, a)));
            else TRY((launch_classic_push<4, false, false>(c, variant, gr, a)));
        }
        if (fused) TRY(edp_sort_finish(c, sp));   // the sorted arrays are the species' arrays from here on
        if (do_mcc) {
            SelArgs b;
            memset(&b, 0, sizeof(b));
            b.kp = c->kp;
            b.P = c->pm[sp];
            b.sel_list = c->sel_list;
            b.sel_count = c->sel_count;
            b.sel_cap = c->sel_cap;
            b.step = (uint32_t)c->t_cntr;
            b.mcc = c->mcc_dev;
            b.born = c->born_dev;
            b.dc = c->dc;
            // one resident wave: the selected list is strided over exactly the CTAs that fit at once, so no CTA
            // waits for a second wave on a few SMs
            static int coll_sm = 0, coll_per_sm = 0;
            if (!coll_sm) {
                EDP_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&coll_per_sm, collide_selected_kernel,
                                                                          256, 0));
                EDP_CUDA(c, cudaDeviceGetAttribute(&coll_sm, cudaDevAttrMultiProcessorCount, c->device));
                coll_per_sm = std::max(coll_per_sm, 1);
            }
            ++c->launches;
            collide_selected_kernel<<<(unsigned)(coll_sm * coll_per_sm), 256, 0, c->stream>>>(b);
        }
    } else {
        PushArgs64 a;
        memset(&a, 0, sizeof(a));
        a.kp = c->kp;
        a.P = c->pd[sp];
        a.n_slots = &c->dc->n_slots[sp];
        a.Ex = is_ion ? c->accx : c->Ex;
        a.Ey = is_ion ? c->accy : c->Ey;
        a.rho = c->rho_d[sp];
        fill_rot(c, sp, nullptr, a.K);
        a.qh = qh;
        a.ez_term = ez_term;
        a.xmul = is_ion ? p.n_subcycles : 1;
        a.use_rot = use_rot;
        a.is_ion = is_ion;
        a.species = sp;
        a.do_mcc = do_mcc;
        a.do_rcx = do_rcx;
        a.step = (uint32_t)c->t_cntr;
        a.mcc = c->mcc_dev;
        if (do_rcx) a.rcx = edp_make_rcx_dev(c, s);
        a.dc = c->dc;
        a.born_e = c->born_e;
        for (int q = 0; q < EDP_MAX_ION_SPECIES; ++q) a.born_i[q] = c->born_i[q];
        a.hits = c->hits;
        a.emit_on = is_ion ? c->emit_on : c->see_on;
        int64_t n = c->host_slots[sp];
        int64_t grid = (n + 255) / 256;
        if (grid > 148 * 64) grid = 148 * 64;
        if (grid < 1) grid = 1;
        ++c->launches;
        push_fp64_kernel<<<(unsigned)grid, 256, 0, c->stream>>>(a);
    }
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

// The wall interaction of every recorded ion hit of this ion step (PROCESS_ION_COLL_WITH_BOUNDARY_*,
// pic2d_IonWallCollisions.f90:3-303, which first clamps the coordinate along the wall into the domain): a reflecting
// wall returns the ion specularly, 1e-6 inside the wall, through the ion add list (INJECT_REFLECTED_ION,
// pic2d_IonEmissions.f90:374-492); otherwise PROCESS_ION_INDUCED_ELECTRON_EMISSION.
struct IonCharges {
    double qs[EDP_MAX_ION_SPECIES];
};

__global__ void __launch_bounds__(256) ion_emission_kernel(edp_hits h, const edp_emit_dev* em, edp_born_dev* born,
                                                           edp_dev_counters* dc, edp_kparams kp, uint32_t step,
                                                           unsigned long long* surf, IonCharges qs)
{
    const int64_t n = min((int64_t)dc->hit_count, h.cap);
    const double xmax = (double)kp.ncx, ymax = (double)kp.ncy;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int ws = h.ws[k], wall = ws & 255, s = ws >> 8;
        if (wall >= 4) {
            // an inner object (DO_ION_COLL_WITH_INNER_OBJECT, pic2d_IonWallCollisions.f90:484-575): the side the
            // trajectory crossed first (ions move V N_subcycles per step); a reflecting object returns the ion; a
            // dielectric takes the charge Qs; an emitting one emits from the crossing point, and a dielectric takes
            // +1 per emitted electron there
            int bm;
            double bx, by;
            const int obj = edp_inner_cross(kp, h.x[k], h.y[k], h.vx[k], h.vy[k], (double)kp.nsub, bm, bx, by);
            if (obj < 0) continue;
            const int o = 4 + obj;
            const edp_face face = edp_inner_face(kp, obj, bm);
            const bool diel = (kp.diel_mask >> obj) & 1;
            if (em && em->reflect[o]) {   // INJECT_REFLECTED_ION, pic2d_IonEmissions.f90:374-492 (m = -1)
                double v[3] = {h.vx[k], h.vy[k], h.vz[k]};
                double nx = bx, ny = by;
                switch (face.dir) {
                case 0: ny = face.at + 1.0e-6; v[1] = -v[1]; break;
                case 1: ny = face.at - 1.0e-6; v[1] = -v[1]; break;
                case 2: nx = face.at + 1.0e-6; v[0] = -v[0]; break;
                default: nx = face.at - 1.0e-6; v[0] = -v[0]; break;
                }
                record_born(born->born_i[s], &dc->born_i_count[s], &dc->error_flags, nx, ny, v);
                continue;
            }
            if (diel) edp_inner_charge(kp, surf, obj, bm, bx, by, qs.qs[s]);
            if (!em) continue;
            const edp_born born_e = born->born_e;
            const int m = edp_emit_electrons(em, s, o, bx, by, h.vx[k], h.vy[k], h.vz[k], h.id[k], step, kp.seed_lo,
                                             kp.seed_hi, face, [&](double nx, double ny, const double* v) {
                                                 record_born(born_e, &dc->born_e_count, &dc->error_flags, nx, ny, v);
                                             });
            if (m) {
                atomicAdd(&dc->e_emit[o], (unsigned long long)m);
                if (diel) edp_inner_charge(kp, surf, obj, bm, bx, by, (double)m);
            }
            continue;
        }
        if (!em) continue;
        const double x = fmin(fmax(h.x[k], 0.0), xmax), y = fmin(fmax(h.y[k], 0.0), ymax);
        if (em->reflect[wall]) {
            double v[3] = {h.vx[k], h.vy[k], h.vz[k]};
            double nx = x, ny = y;
            switch (wall) {
            case 0: ny = 1.0e-6; v[1] = -v[1]; break;
            case 1: ny = ymax - 1.0e-6; v[1] = -v[1]; break;
            case 2: nx = 1.0e-6; v[0] = -v[0]; break;
            default: nx = xmax - 1.0e-6; v[0] = -v[0]; break;
            }
            record_born(born->born_i[s], &dc->born_i_count[s], &dc->error_flags, nx, ny, v);
            continue;
        }
        const edp_born born_e = born->born_e;
        const int m = edp_emit_electrons(em, s, wall, x, y, h.vx[k], h.vy[k], h.vz[k], h.id[k], step, kp.seed_lo,
                                         kp.seed_hi, edp_wall_face(wall, xmax, ymax),
                                         [&](double nx, double ny, const double* v) {
                                             record_born(born_e, &dc->born_e_count, &dc->error_flags, nx, ny, v);
                                         });
        if (m) atomicAdd(&dc->e_emit[wall], (unsigned long long)m);
    }
}

// PROCESS_ELECTRON_INDUCED_ELECTRON_EMISSION for every electron wall hit of this step (the coordinate along the wall
// clamped into the domain first, pic2d_ElectronWallCollisions.f90:21, :93, :165, :237)
__global__ void __launch_bounds__(256) electron_emission_kernel(edp_hits h, const edp_see_dev* sd, edp_born born_e,
                                                                edp_dev_counters* dc, edp_kparams kp, uint32_t step,
                                                                unsigned long long* surf)
{
    const int64_t n = min((int64_t)dc->hit_count, h.cap);
    const double xmax = (double)kp.ncx, ymax = (double)kp.ncy;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int wall = h.ws[k] & 255;
        if (wall >= 4) {
            // an inner object (DO_ELECTRON_COLL_WITH_INNER_OBJECT, pic2d_ElectronWallCollisions.f90:561-645): the side
            // the trajectory crossed first; a dielectric's outline takes the electron's charge there, an emitting
            // object emits from the crossing (PROCESS_ELECTRON_INDUCED_ELECTRON_EMISSION with m = -1), and a dielectric
            // takes +1 per electron leaving it
            int bm;
            double bx, by;
            const int obj = edp_inner_cross(kp, h.x[k], h.y[k], h.vx[k], h.vy[k], 1.0, bm, bx, by);
            if (obj < 0) continue;
            const bool diel = (kp.diel_mask >> obj) & 1;
            if (diel) edp_inner_charge(kp, surf, obj, bm, bx, by, -1.0);
            if (!sd) continue;
            const int o = 4 + obj;
            const int m = edp_see_electrons(sd, o, bx, by, h.vx[k], h.vy[k], h.vz[k], h.id[k], step, kp.seed_lo,
                                            kp.seed_hi, edp_inner_face(kp, obj, bm),
                                            [&](double nx, double ny, const double* v) {
                                                record_born(born_e, &dc->born_e_count, &dc->error_flags, nx, ny, v);
                                            });
            if (m < 0) {
                atomicOr(&dc->error_flags, EDP_EFLAG_SEE_MODEL);
            } else if (m) {
                atomicAdd(&dc->e_emit[o], (unsigned long long)m);
                if (diel) edp_inner_charge(kp, surf, obj, bm, bx, by, (double)m);
            }
            continue;
        }
        if (!sd) continue;
        const double x = fmin(fmax(h.x[k], 0.0), xmax), y = fmin(fmax(h.y[k], 0.0), ymax);
        const int m = edp_see_electrons(sd, wall, x, y, h.vx[k], h.vy[k], h.vz[k], h.id[k], step, kp.seed_lo,
                                        kp.seed_hi, edp_wall_face(wall, xmax, ymax),
                                        [&](double nx, double ny, const double* v) {
                                            record_born(born_e, &dc->born_e_count, &dc->error_flags, nx, ny, v);
                                        });
        if (m < 0) atomicOr(&dc->error_flags, EDP_EFLAG_SEE_MODEL);
        else if (m) atomicAdd(&dc->e_emit[wall], (unsigned long long)m);
    }
}

int edp_launch_electron_emission(edp_ctx* c)
{
    ++c->launches;
    const bool any_see = c->see_on || c->kp.see_inner_mask;
    electron_emission_kernel<<<148 * 2, 256, 0, c->stream>>>(c->hits, any_see ? c->see_dev : nullptr, c->born_e,
                                                           c->dc, c->kp, (uint32_t)c->t_cntr, c->surf);
    EDP_CUDA(c, cudaGetLastError());
    EDP_CUDA(c, cudaMemsetAsync(&c->dc->hit_count, 0, sizeof(unsigned long long), c->stream));
    return EDP_OK;
}

// PERFORM_ELECTRON_EMISSION_SETUP (pic2d_Setup.f90:599-1001) for one cluster over the domain: wall blockIdx.y < 4
// emits INT(n) electrons and one more with probability n - INT(n) (:627-690); PERFORM_ELECTRON_EMISSION_SETUP_INNER_
// OBJECTS (:1005-1591): blockIdx.y = 4 + s for side s of an inner object, which emits INT(n_s) + Bernoulli electrons
// spread uniformly over its open cells, 1e-6 outside the side, with the normal velocity pointing out. Variates:
// Philox4x32-10, key {EDP_INJECT_KEY + blockIdx.y, seed_lo}, counter {step, EDP_STREAM_INJECT, block, seed_hi}; block
// 0 word 0 for the fraction, block 1 + e for electron e: word 0 its place along the wall or side, word 1 the normal
// speed, words 2 and 3 the tangential components (the one in the domain's plane, then z).
__global__ void __launch_bounds__(256) wall_injection_kernel(edp_inject_dev in, edp_born born_e,
                                                             edp_dev_counters* dc, edp_kparams kp, uint32_t step)
{
    const int y = blockIdx.y;
    const int side = y - 4, obj = y < 4 ? y : 4 + side / 4, seg = side % 4 + 1;
    const double n = y < 4 ? in.n[y] : in.side_n[side];
    if (!(n > 0.0)) return;
    const uint32_t key = EDP_INJECT_KEY + (uint32_t)y;
    int count = (int)n;
    uint32_t w0[4];
    edp_philox(step, EDP_STREAM_INJECT, 0u, kp.seed_hi, key, kp.seed_lo, w0);
    if (edp_u01(w0[0]) < n - (double)count) ++count;
    const double xmax = (double)kp.ncx, ymax = (double)kp.ncy;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        uint32_t w[4];
        edp_philox(step, EDP_STREAM_INJECT, 1u + (uint32_t)e, kp.seed_hi, key, kp.seed_lo, w);
        double vn;
        if (in.model[obj] == 0) {
            vn = edp_maxwell_inj(in.maxwell_inj, in.rmax_inj, edp_u01(w[1])) * in.fn[obj];
        } else {
            vn = fmax(0.0, in.vb[obj] + edp_maxwell(in.maxwell_v, in.rmax, edp_u01(w[1])) * in.fn[obj]);
        }
        const double t1 = edp_maxwell(in.maxwell_v, in.rmax, edp_u01(w[2])) * in.fp[obj];
        const double t2 = edp_maxwell(in.maxwell_v, in.rmax, edp_u01(w[3])) * in.fp[obj];
        const double r = edp_u01(w[0]);
        double x, yy, v[3];
        if (y < 4) {
            switch (y) {
            case 0: x = fmin(fmax(r * xmax, 0.0), xmax); yy = 1.0e-6; v[0] = t1; v[1] = vn; v[2] = t2; break;
            case 1: x = fmin(fmax(r * xmax, 0.0), xmax); yy = ymax - 1.0e-6; v[0] = t1; v[1] = -vn; v[2] = t2; break;
            case 2: x = 1.0e-6; yy = fmin(fmax(r * ymax, 0.0), ymax); v[0] = vn; v[1] = t1; v[2] = t2; break;
            default: x = xmax - 1.0e-6; yy = fmin(fmax(r * ymax, 0.0), ymax); v[0] = -vn; v[1] = t1; v[2] = t2; break;
            }
        } else {
            // the place along the side: d = r (open - 1e-6) walks the open cells, a whole cell at a time
            // (:1064-1078); d - k is exact, as the reference's k subtractions of 1 are
            const int open = in.side_open[side];
            double d = r * ((double)open - 1.0e-6);
            int k = (int)d;
            if (k > open - 1) k = open - 1;
            d -= (double)k;
            const double c0 = (double)in.open_cells[in.side_off[side] + k];
            double t = fmax(c0, fmin(c0 + d, c0 + 1.0));
            t = fmin(fmax(t, (double)in.side_cmin[side]), (double)in.side_cmax[side] - 1.0e-6);
            const double at = in.side_at[side];
            switch (seg) {
            case 1: x = at; yy = t; v[0] = -vn; v[1] = t1; v[2] = t2; break;   // left: out along -x
            case 3: x = at; yy = t; v[0] = vn; v[1] = t1; v[2] = t2; break;    // right
            case 2: x = t; yy = at; v[0] = t1; v[1] = vn; v[2] = t2; break;    // top
            default: x = t; yy = at; v[0] = t1; v[1] = -vn; v[2] = t2; break;  // bottom
            }
        }
        record_born(born_e, &dc->born_e_count, &dc->error_flags, x, yy, v);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&dc->e_emit[obj], (unsigned long long)count);
}

int edp_launch_wall_injection(edp_ctx* c)
{
    double nmax = 0.0;
    for (int w = 0; w < 4; ++w) nmax = std::max(nmax, c->inject.n[w]);
    for (int s = 0; s < EDP_INJECT_SIDES; ++s) nmax = std::max(nmax, c->inject.side_n[s]);
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>(((int64_t)nmax + 256) / 256, 148));
    ++c->launches;
    wall_injection_kernel<<<dim3((unsigned)blocks, 4 + EDP_INJECT_SIDES), 256, 0, c->stream>>>(
        c->inject, c->born_e, c->dc, c->kp, (uint32_t)c->t_cntr);
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

int edp_launch_ion_emission(edp_ctx* c)
{
    ++c->launches;
    IonCharges qs;
    for (int s = 0; s < EDP_MAX_ION_SPECIES; ++s) qs.qs[s] = (double)c->p.ion_charge[s];
    ion_emission_kernel<<<148 * 2, 256, 0, c->stream>>>(c->hits, c->emit_on ? c->emit_dev : nullptr, c->born_dev,
                                                      c->dc, c->kp, (uint32_t)c->t_cntr, c->surf, qs);
    EDP_CUDA(c, cudaGetLastError());
    EDP_CUDA(c, cudaMemsetAsync(&c->dc->hit_count, 0, sizeof(unsigned long long), c->stream));
    return EDP_OK;
}

static CollArgs coll_args(edp_ctx* c, int sp)
{
    CollArgs a;
    memset(&a, 0, sizeof(a));
    a.kp = c->kp;
    a.precision = c->p.precision;
    a.species = sp;
    a.Pm = c->pm[sp];
    a.Pd = c->pd[sp];
    a.n_slots = &c->dc->n_slots[sp];
    a.step = (uint32_t)c->t_cntr;
    a.dc = c->dc;
    a.born_e = c->born_e;
    for (int q = 0; q < EDP_MAX_ION_SPECIES; ++q) a.born_i[q] = c->born_i[q];
    return a;
}

static unsigned grid_for(int64_t n)
{
    int64_t g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    if (g < 1) g = 1;
    return (unsigned)g;
}

int edp_launch_collide_en(edp_ctx* c)
{
    if (!c->tab.en_on) return EDP_OK;
    CollArgs a = coll_args(c, 0);
    a.mcc = c->mcc_dev;
    ++c->launches;
    collide_en_kernel<<<grid_for(c->host_slots[0]), 256, 0, c->stream>>>(a);
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

int edp_launch_collide_rcx(edp_ctx* c)
{
    for (int s = 0; s < c->p.n_ion_species; ++s) {
        if (!c->tab.rcx_on[s]) continue;
        CollArgs a = coll_args(c, 1 + s);
        a.rcx = edp_make_rcx_dev(c, s);
        ++c->launches;
        collide_rcx_kernel<<<grid_for(c->host_slots[1 + s]), 256, 0, c->stream>>>(a);
        EDP_CUDA(c, cudaGetLastError());
    }
    return EDP_OK;
}

static AppendArgs append_args(edp_ctx* c, int sp)
{
    AppendArgs a;
    memset(&a, 0, sizeof(a));
    a.kp = c->kp;
    a.precision = c->p.precision;
    a.species = sp;
    a.Pm = c->pm[sp];
    a.Pd = c->pd[sp];
    a.cap = c->cap[sp];
    a.n_slots = &c->dc->n_slots[sp];
    a.n_live = &c->dc->n_live[sp];
    a.next_id = &c->dc->next_id[sp];
    a.id_end = (unsigned long long)c->id_end;
    a.rho_fix = c->rho_fix[sp];
    a.rho_d = c->rho_d[sp];
    a.dc = c->dc;
    return a;
}

// the add lists of this step's ionisations join their arrays: ions (PROCESS_ADDED_IONS, pic2d_MainProgram.f90:300),
// then electrons (PROCESS_ADDED_ELECTRONS, :363)
int edp_launch_append_born(edp_ctx* c)
{
    for (int s = 0; s < c->p.n_ion_species; ++s) {
        if (!c->uploaded[1 + s]) continue;
        AppendArgs a = append_args(c, 1 + s);
        a.src = c->born_i[s];
        a.src_count = &c->dc->born_i_count[s];
        ++c->launches;
        append_kernel<<<148 * 2, 256, 0, c->stream>>>(a);
        EDP_CUDA(c, cudaGetLastError());
        c->host_slots[1 + s] += c->born_cap;
    }
    AppendArgs a = append_args(c, 0);
    a.src = c->born_e;
    a.src_count = &c->dc->born_e_count;
    ++c->launches;
    append_kernel<<<148 * 2, 256, 0, c->stream>>>(a);
    EDP_CUDA(c, cudaGetLastError());
    c->host_slots[0] += c->born_cap;
    return EDP_OK;
}
