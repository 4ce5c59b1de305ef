// C ABI of the EDIPIC-2D B200 particle cycle: context lifecycle, particle I/O, step orchestration.
// The call order of one step follows MainProg (pic2d_MainProgram.f90:151-309).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <map>
#include <mutex>

#include "edp_internal.cuh"

int edp_fail(edp_ctx* c, int code, const std::string& msg)
{
    if (c) c->last_error = msg;
    return code;
}

int edp_cuda_check(edp_ctx* c, cudaError_t e, const char* what)
{
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
    return edp_fail(c, EDP_ERR_CUDA, buf);
}

edp_mcc_dev edp_make_mcc_dev(const edp_ctx* c)
{
    edp_mcc_dev m;
    memset(&m, 0, sizeof(m));
    const edp_tables& t = c->tab;
    m.prob = c->mcc_prob;
    m.energy = c->mcc_energy;
    m.maxwell_v = c->maxwell_v;
    m.n_act = t.n_act;
    m.n_seg = t.n_seg;
    m.n_values = t.n_values;
    m.rmax = t.maxwell_rmax;
    for (int i = 0; i <= t.n_seg; ++i) {
        m.seg_value[i] = t.seg_value[i];
        m.seg_index[i] = t.seg_index[i];
    }
    for (int i = 0; i < t.n_seg; ++i) m.seg_step[i] = t.seg_step[i];
    m.pmax = t.max_colliding_fraction;
    m.pmax_x = (unsigned long long)std::ceil(std::ldexp(t.max_colliding_fraction, 32) - 0.5);
    for (int p = 0; p < EDP_MAX_COLPROC; ++p) {
        m.type[p] = t.colproc_type[p];
        m.thr[p] = t.threshold_eV[p];
        m.ion_species[p] = t.ion_species_produced[p] - 1;
        m.ion_vfactor[p] = t.ion_velocity_factor[p];
    }
    m.mass_amu = t.neutral_mass_amu;
    m.energy_factor = t.energy_factor_eV;
    m.on = t.en_on;
    return m;
}

edp_rcx_dev edp_make_rcx_dev(const edp_ctx* c, int s)
{
    edp_rcx_dev r;
    memset(&r, 0, sizeof(r));
    const edp_tables& t = c->tab;
    r.maxwell_v = c->maxwell_v;
    r.rmax = t.maxwell_rmax;
    r.on = t.rcx_on[s];
    r.prob_factor = t.rcx_prob_factor;
    r.v_scale = c->p.v_scale_ms;
    r.factor_eV = c->p.ion_mass_me[s] * t.energy_factor_eV;
    r.sigma_1eV = t.rcx_sigma_1eV;
    r.alpha = t.rcx_alpha;
    r.pth2 = t.rcx_probab_thermal[s] * t.rcx_probab_thermal[s];
    r.vfactor = t.rcx_vfactor[s];
    double k = (r.prob_factor * ((r.sigma_1eV * 1.0) * 1.0)) * r.v_scale;
    r.k2 = k * k;
    return r;
}

namespace {

template <class T>
int dalloc(edp_ctx* c, T** p, size_t n)
{
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return edp_cuda_check(c, e, "cudaMalloc");
    return EDP_OK;
}

// Boris rotation matrix K11..K33 (pic2d_ElectronDynamics.f90:91-113) for uniform B
void rotation(double ax, double ay, double az, double* K)
{
    double ax2 = ax * ax, ay2 = ay * ay, az2 = az * az, th = ax2 + ay2 + az2, inv = 1.0 / (1.0 + th);
    K[0] = (1.0 - th + 2.0 * ax2) * inv;
    K[1] = 2.0 * (ax * ay + az) * inv;
    K[2] = 2.0 * (ax * az - ay) * inv;
    K[3] = 2.0 * (ax * ay - az) * inv;
    K[4] = (1.0 - th + 2.0 * ay2) * inv;
    K[5] = 2.0 * (ay * az + ax) * inv;
    K[6] = 2.0 * (ax * az + ay) * inv;
    K[7] = 2.0 * (ay * az - ax) * inv;
    K[8] = (1.0 - th + 2.0 * az2) * inv;
}

// the wall-hit list with room for cap records (any previous list is released: it holds nothing between pushes)
static int alloc_hits(edp_ctx* c, int64_t cap)
{
    edp_hits& h = c->hits;
    for (void* q : {(void*)h.x, (void*)h.y, (void*)h.vx, (void*)h.vy, (void*)h.vz, (void*)h.id, (void*)h.ws})
        if (q) cudaFree(q);
    h = edp_hits();
    h.cap = cap;
    TRY(dalloc(c, &h.x, cap));
    TRY(dalloc(c, &h.y, cap));
    TRY(dalloc(c, &h.vx, cap));
    TRY(dalloc(c, &h.vy, cap));
    TRY(dalloc(c, &h.vz, cap));
    TRY(dalloc(c, &h.id, cap));
    TRY(dalloc(c, &h.ws, cap));
    return EDP_OK;
}

int alloc_species(edp_ctx* c, int sp, int64_t n)
{
    if (c->cap[sp] > 0) {
        if (n <= c->cap[sp]) return EDP_OK;
        return edp_fail(c, EDP_ERR_CAPACITY, "particle count exceeds the capacity allocated for this species");
    }
    int64_t cap = c->p.capacity[sp] > 0 ? c->p.capacity[sp] : (n + n / 4 + 65536);
    cap = (cap + 3) & ~(int64_t)3;
    if (n > cap) return edp_fail(c, EDP_ERR_CAPACITY, "particle count exceeds params.capacity");
    c->cap[sp] = cap;
    if (c->p.precision == EDP_PREC_MIXED) {
        for (int b = 0; b < 2; ++b) {
            edp_species_mixed& m = b ? c->pm_alt[sp] : c->pm[sp];
            if (b && c->p.sort_every <= 0) break;
            TRY(dalloc(c, &m.cell, cap));
            TRY(dalloc(c, &m.ox, cap));
            TRY(dalloc(c, &m.oy, cap));
            TRY(dalloc(c, &m.vx, cap));
            TRY(dalloc(c, &m.vy, cap));
            TRY(dalloc(c, &m.vz, cap));
            TRY(dalloc(c, &m.id, cap));
            TRY(dalloc(c, &m.tag, cap));
        }
    } else {
        edp_species_fp64& d = c->pd[sp];
        TRY(dalloc(c, &d.x, cap));
        TRY(dalloc(c, &d.y, cap));
        TRY(dalloc(c, &d.vx, cap));
        TRY(dalloc(c, &d.vy, cap));
        TRY(dalloc(c, &d.vz, cap));
        TRY(dalloc(c, &d.id, cap));
        TRY(dalloc(c, &d.tag, cap));
    }
    if (sp == 0) {
        // add lists for ionisation products: a small fraction of the electron capacity
        int64_t bc = std::max<int64_t>(65536, cap / 64);
        c->born_cap = bc;
        if (c->hits.x && c->hits.cap < bc) TRY(alloc_hits(c, bc));   // as large as the electron add list
        {
            edp_born& e = c->born_e;
            e.cap = bc;
            TRY(dalloc(c, &e.x, bc));
            TRY(dalloc(c, &e.y, bc));
            TRY(dalloc(c, &e.vx, bc));
            TRY(dalloc(c, &e.vy, bc));
            TRY(dalloc(c, &e.vz, bc));
        }
        for (int s = 0; s < c->p.n_ion_species; ++s) {
            edp_born& e = c->born_i[s];
            e.cap = bc;
            TRY(dalloc(c, &e.x, bc));
            TRY(dalloc(c, &e.y, bc));
            TRY(dalloc(c, &e.vx, bc));
            TRY(dalloc(c, &e.vy, bc));
            TRY(dalloc(c, &e.vz, bc));
        }
        edp_born_dev h;
        h.born_e = c->born_e;
        for (int s = 0; s < EDP_MAX_ION_SPECIES; ++s) h.born_i[s] = c->born_i[s];
        TRY(dalloc(c, &c->born_dev, 1));
        EDP_CUDA(c, cudaMemcpy(c->born_dev, &h, sizeof(h), cudaMemcpyHostToDevice));
        // selection list of the fused collision test: P_max of the electrons on average, with headroom
        double pm = c->tab.en_on ? c->tab.max_colliding_fraction : 0.0;
        c->sel_cap = std::max<int64_t>(65536, (int64_t)((double)cap * std::min(1.0, 2.0 * pm + 0.01)));
        TRY(dalloc(c, &c->sel_list, c->sel_cap));
        TRY(dalloc(c, &c->sel_count, 1));
    }
    return EDP_OK;
}

int finish_sync(edp_ctx* c)
{
    if (!c->sync) return EDP_OK;
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    return EDP_OK;
}

// -------------------------------------------------------------------------------- utility kernels
__global__ void upload_kernel(edp_kparams kp, int precision, int64_t n, int64_t base, const double* x, const double* y,
                              const double* vx, const double* vy, const double* vz, const int32_t* tag,
                              const uint32_t* id, edp_species_mixed m, edp_species_fp64 d, unsigned int* eflag,
                              uint64_t id_base)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double X = x[k], Y = y[k];
        bool bad = !(Y >= 0.0 && Y <= (double)kp.ncy);
        if (kp.periodic) {
            if (X >= (double)kp.ncx) X -= (double)kp.ncx;   // overlap cell of the reference layout
            bad = bad || !(X >= 0.0 && X < (double)kp.ncx);
        } else {
            bad = bad || !(X >= 0.0 && X <= (double)kp.ncx);
        }
        if (bad) atomicOr(eflag, EDP_EFLAG_BOUNDS);
        int64_t slot = base + k;
        uint32_t pid = id ? id[k] : (uint32_t)(id_base + (uint64_t)k);
        int32_t t = tag ? tag[k] : 0;
        if (precision == EDP_PREC_MIXED) {
            int i = (int)X, j = (int)Y;
            float ox, oy;
            if (!kp.periodic && i == kp.ncx) {
                i = kp.ncx - 1;
                ox = 1.0f;
            } else {
                ox = (float)(X - (double)i);
                if (ox >= 1.0f) {
                    ox -= 1.0f;
                    ++i;
                    if (kp.periodic && i == kp.ncx) i = 0;
                }
            }
            if (j == kp.ncy) {
                j = kp.ncy - 1;
                oy = 1.0f;
            } else {
                oy = (float)(Y - (double)j);
                if (oy >= 1.0f) {
                    if (j + 1 < kp.ncy) {
                        oy -= 1.0f;
                        ++j;
                    } else {
                        oy = 1.0f;
                    }
                }
            }
            m.cell[slot] = bad ? -1 : ((j << 16) | i);
            m.ox[slot] = ox;
            m.oy[slot] = oy;
            m.vx[slot] = (float)vx[k];
            m.vy[slot] = (float)vy[k];
            m.vz[slot] = (float)vz[k];
            m.id[slot] = pid;
            m.tag[slot] = t;
        } else {
            d.x[slot] = bad ? -1.0e30 : X;
            d.y[slot] = Y;
            d.vx[slot] = vx[k];
            d.vy[slot] = vy[k];
            d.vz[slot] = vz[k];
            d.id[slot] = pid;
            d.tag[slot] = t;
        }
    }
}

__global__ void deposit_mixed_kernel(edp_kparams kp, edp_species_mixed m, const unsigned long long* n_slots,
                                     unsigned long long* rho)
{
    const int64_t n = (int64_t)*n_slots;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int c = m.cell[k];
        if (c < 0) continue;
        int i = c & 0xFFFF, j = c >> 16;
        double dx = (double)m.ox[k], dy = (double)m.oy[k];
        double vij = (1.0 - dx) * (1.0 - dy), vip1j = dx * (1.0 - dy), vijp1 = (1.0 - dx) * dy;
        long long q00 = __double2ll_rn(vij * EDP_FIX_ONE), q10 = __double2ll_rn(vip1j * EDP_FIX_ONE);
        long long q01 = __double2ll_rn(vijp1 * EDP_FIX_ONE), q11 = 4294967296LL - q00 - q10 - q01;
        int i1 = i + 1;
        if (kp.periodic && i1 == kp.ncx) i1 = 0;
        int64_t r0 = (int64_t)j * kp.nxg, r1 = r0 + kp.nxg;
        atomicAdd(&rho[r0 + i], (unsigned long long)q00);
        atomicAdd(&rho[r0 + i1], (unsigned long long)q10);
        atomicAdd(&rho[r1 + i], (unsigned long long)q01);
        atomicAdd(&rho[r1 + i1], (unsigned long long)q11);
    }
}

__global__ void deposit_fp64_kernel(edp_kparams kp, edp_species_fp64 d, const unsigned long long* n_slots, double* rho)
{
    const int64_t n = (int64_t)*n_slots;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double X = d.x[k];
        if (X < -1.0e29) continue;
        double Y = d.y[k];
        int i = (int)X, j = (int)Y;
        if (!kp.periodic && X == (double)kp.ncx) i = kp.ncx - 1;
        if (Y == (double)kp.ncy) j = kp.ncy - 1;
        int i1 = i + 1;
        if (kp.periodic && i1 == kp.ncx) i1 = 0;
        double dx = X - (double)i, dy = Y - (double)j;
        double vij = (1.0 - dx) * (1.0 - dy), vip1j = dx * (1.0 - dy), vijp1 = (1.0 - dx) * dy;
        int64_t r0 = (int64_t)j * kp.nxg, r1 = r0 + kp.nxg;
        atomicAdd(&rho[r0 + i], vij);
        atomicAdd(&rho[r0 + i1], vip1j);
        atomicAdd(&rho[r1 + i], vijp1);
        atomicAdd(&rho[r1 + i1], 1.0 - vij - vip1j - vijp1);
    }
}

// DISTRIBUTE_PARTICLES (pic2d_CurProblemValues.f90:3127-3325): per_cell particles in each cell, uniform offsets,
// Maxwellian components from the inverse-CDF table, Philox stream EDP_STREAM_INIT keyed by the particle id.
__global__ void distribute_kernel(edp_kparams kp, int precision, int sp, int per_cell, double fconv, int zero_vz,
                                  int copy_pos, const double* maxwell_v, int rmax, int64_t base_id,
                                  edp_species_mixed m, edp_species_fp64 d, edp_species_mixed me, edp_species_fp64 de,
                                  int64_t n)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        uint32_t id = (uint32_t)(base_id + k);
        uint32_t b0[4], b1[4];
        edp_philox(0u, EDP_STREAM_INIT(sp), 0u, kp.seed_hi, id, kp.seed_lo, b0);
        edp_philox(0u, EDP_STREAM_INIT(sp), 1u, kp.seed_hi, id, kp.seed_lo, b1);
        int64_t cellno = k / per_cell;
        int i = (int)(cellno % kp.ncx), j = (int)(cellno / kp.ncx);
        double X, Y;
        if (copy_pos) {
            if (precision == EDP_PREC_MIXED) {
                int c = me.cell[k];
                X = (double)(c & 0xFFFF) + (double)me.ox[k];
                Y = (double)(c >> 16) + (double)me.oy[k];
                if (c < 0) X = -1.0e30;
            } else {
                X = de.x[k];
                Y = de.y[k];
            }
        } else {
            float fx = (float)edp_u01(b0[0]), fy = (float)edp_u01(b0[1]);
            if (fx >= 1.0f) fx = 0.99999994f;
            if (fy >= 1.0f) fy = 0.99999994f;
            X = (double)i + (double)fx;
            Y = (double)j + (double)fy;
        }
        double vx = edp_maxwell(maxwell_v, rmax, edp_u01(b0[2])) * fconv;
        double vy = edp_maxwell(maxwell_v, rmax, edp_u01(b0[3])) * fconv;
        double vz = zero_vz ? 0.0 : edp_maxwell(maxwell_v, rmax, edp_u01(b1[0])) * fconv;
        bool dead = X < -1.0e29;
        for (int q = 0; q < kp.n_inner && !dead; ++q)
            if (X > (double)kp.ileft[q] && X < (double)kp.iright[q] && Y > (double)kp.jbottom[q] && Y < (double)kp.jtop[q])
                dead = true;
        if (precision == EDP_PREC_MIXED) {
            int ii = (int)X, jj = (int)Y;
            m.cell[k] = dead ? -1 : ((jj << 16) | ii);
            m.ox[k] = dead ? 0.f : (float)(X - ii);
            m.oy[k] = dead ? 0.f : (float)(Y - jj);
            m.vx[k] = (float)vx;
            m.vy[k] = (float)vy;
            m.vz[k] = (float)vz;
            m.id[k] = id;
            m.tag[k] = 0;
        } else {
            d.x[k] = dead ? -1.0e30 : X;
            d.y[k] = Y;
            d.vx[k] = vx;
            d.vy[k] = vy;
            d.vz[k] = vz;
            d.id[k] = id;
            d.tag[k] = 0;
        }
    }
}

__global__ void count_live_kernel(edp_kparams kp, int precision, edp_species_mixed m, edp_species_fp64 d, int64_t n,
                                  unsigned long long* live)
{
    unsigned long long acc = 0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        acc += (precision == EDP_PREC_MIXED) ? (m.cell[k] >= 0) : (d.x[k] > -1.0e29);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(live, acc);
}

__global__ void moments_kernel(int precision, edp_species_mixed m, edp_species_fp64 d, const unsigned long long* n_slots,
                               double* out)
{
    const int64_t n = (int64_t)*n_slots;
    double a[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double vx, vy, vz;
        if (precision == EDP_PREC_MIXED) {
            if (m.cell[k] < 0) continue;
            vx = m.vx[k];
            vy = m.vy[k];
            vz = m.vz[k];
        } else {
            if (d.x[k] < -1.0e29) continue;
            vx = d.vx[k];
            vy = d.vy[k];
            vz = d.vz[k];
        }
        a[0] += 1.0;
        a[1] += vx;
        a[2] += vy;
        a[3] += vz;
        a[4] += vx * vx;
        a[5] += vy * vy;
        a[6] += vz * vz;
    }
    for (int q = 0; q < 7; ++q) {
        double v = a[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&out[q], v);
    }
}

__global__ void mcc_choose_kernel(edp_mcc_dev m, int64_t n, const double* E, const double* r, int32_t* out)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        out[k] = edp_mcc_choose_dev(m, E[k], r[k]);
}

__global__ void reset_born_kernel(edp_dev_counters* dc)
{
    dc->born_e_count = 0ull;
    for (int s = 0; s < EDP_MAX_ION_SPECIES; ++s) dc->born_i_count[s] = 0ull;
}

__global__ void reset_step_counters_kernel(edp_dev_counters* dc)
{
    for (int p = 0; p < EDP_MAX_COLPROC; ++p) dc->en_coll_step[p] = 0ull;
    for (int s = 0; s < EDP_MAX_ION_SPECIES; ++s) dc->rcx_step[s] = 0ull;
}

// node array: device canonical layout -> reference layout on the host side buffer (periodic: 2 overlap columns)
__global__ void expand_kernel(edp_kparams kp, int mode, const double* src, const float2* src2, int comp, double* dst,
                              int wout)
{
    int64_t n = (int64_t)wout * kp.nyg;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(q % wout), j = (int)(q / wout);
        int ic = kp.periodic ? (i % kp.ncx) : i;
        int64_t s = (int64_t)j * kp.nxg + ic;
        dst[q] = (mode == 0) ? src[s] : (comp == 0 ? (double)src2[s].x : (double)src2[s].y);
    }
}

__global__ void contract_kernel(edp_kparams kp, int mode, const double* src, int wout, double* dst, float2* dst2, int comp)
{
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(q % kp.nxg), j = (int)(q / kp.nxg);
        double v = src[(int64_t)j * wout + i];
        if (mode == 0) dst[q] = v;
        else if (comp == 0) dst2[q].x = (float)v;
        else dst2[q].y = (float)v;
    }
}

// one species' density with the wall factors, FP64 on the canonical grid
__global__ void species_density_kernel(edp_kparams kp, int precision, const unsigned long long* fix, const double* dd,
                                       double w, double* out)
{
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(q % kp.nxg), j = (int)(q / kp.nxg);
        double r = (precision == EDP_PREC_MIXED) ? (double)(long long)fix[q] * EDP_FIX_INV : dd[q];
        double f = 1.0;
        if (kp.periodic) {
            if (j == 0 || j == kp.ncy) f = 2.0;
        } else {
            bool ex = (i == 0 || i == kp.ncx), ey = (j == 0 || j == kp.ncy);
            f = (ex && ey) ? 4.0 : ((ex || ey) ? 2.0 : 1.0);
        }
        out[q] = w * r * f;
    }
}

unsigned grid_of(int64_t n, int64_t cap_blocks = 148 * 16)
{
    int64_t g = (n + 255) / 256;
    g = std::min(g, cap_blocks);
    return (unsigned)std::max<int64_t>(g, 1);
}

int ref_width(const edp_ctx* c) { return c->kp.periodic ? c->p.ncx + 2 : c->p.ncx + 1; }

int zero_density(edp_ctx* c, int sp)
{
    const int64_t nn = (int64_t)c->kp.nxg * c->kp.nyg;
    c->dirty |= 1u << sp;
    if (c->p.precision == EDP_PREC_MIXED)
        EDP_CUDA(c, cudaMemsetAsync(c->rho_fix[sp], 0, nn * sizeof(unsigned long long), c->stream));
    else
        EDP_CUDA(c, cudaMemsetAsync(c->rho_d[sp], 0, nn * sizeof(double), c->stream));
    return EDP_OK;
}

int after_particles_changed(edp_ctx* c, int sp)
{
    // live count, then the initial sort and the deposit the first field solve needs
    c->hc->n_live[sp] = 0;
    EDP_CUDA(c, cudaMemsetAsync(&c->dc->n_live[sp], 0, sizeof(unsigned long long), c->stream));
    ++c->launches;
    count_live_kernel<<<grid_of(c->host_slots[sp]), 256, 0, c->stream>>>(c->kp, c->p.precision, c->pm[sp], c->pd[sp],
                                                                          c->host_slots[sp], &c->dc->n_live[sp]);
    EDP_CUDA(c, cudaGetLastError());
    c->sorted_end[sp] = 0;
    c->n_chunks[sp] = 0;
    if (c->p.precision == EDP_PREC_MIXED && c->p.sort_every > 0) TRY(edp_launch_sort(c, sp));
    TRY(zero_density(c, sp));
    TRY(edp_launch_deposit(c, sp));
    c->uploaded[sp] = 1;
    return EDP_OK;
}

}  // namespace

int edp_raise_smem_limit(edp_ctx* c, const void* kernel, size_t bytes)
{
    static std::mutex mu;
    static std::map<const void*, size_t> limit;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = limit[kernel];
    if (bytes <= cur) return EDP_OK;
    EDP_CUDA(c, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
    return EDP_OK;
}


int edp_launch_deposit(edp_ctx* c, int sp)
{
    ++c->launches;
    if (c->p.precision == EDP_PREC_MIXED)
        deposit_mixed_kernel<<<grid_of(c->host_slots[sp]), 256, 0, c->stream>>>(c->kp, c->pm[sp], &c->dc->n_slots[sp],
                                                                                 c->rho_fix[sp]);
    else
        deposit_fp64_kernel<<<grid_of(c->host_slots[sp]), 256, 0, c->stream>>>(c->kp, c->pd[sp], &c->dc->n_slots[sp],
                                                                                c->rho_d[sp]);
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

// ======================================================================================= public ABI
extern "C" {

int edp_init(const edp_params* p, const edp_tables* t, edp_ctx** out)
{
    if (!p || !t || !out) return EDP_ERR_ARG;
    *out = nullptr;
    if (p->abi_version != EDP_ABI_VERSION) return EDP_ERR_ARG;
    if (p->ncx < 2 || p->ncy < 2 || p->ncx > 32768 || p->ncy > 32767) return EDP_ERR_ARG;
    if (p->n_ion_species < 1 || p->n_ion_species > EDP_MAX_ION_SPECIES) return EDP_ERR_ARG;
    if (p->n_subcycles < 1 || (p->n_subcycles % 2) == 0) return EDP_ERR_ARG;
    if (p->n_of_particles_cell < 1 || p->n_inner < 0 || p->n_inner > EDP_MAX_INNER) return EDP_ERR_ARG;
    for (int n = 0; n < p->n_inner; ++n) {
        if (!(p->inner_eps[n] >= 0.0) || !std::isfinite(p->inner_eps[n])) return EDP_ERR_ARG;
        if (p->inner_eps[n] > 0.0 && p->solver != EDP_SOLVER_CG) return EDP_ERR_ARG;   // dielectrics: CG only
    }
    if (p->solver == EDP_SOLVER_FFTX) {
        if (!p->periodic_x || (p->ncx & (p->ncx - 1)) != 0 || p->ncx > 4096) return EDP_ERR_ARG;
    } else if (p->solver == EDP_SOLVER_CG) {
        if (p->periodic_x) return EDP_ERR_ARG;
    } else {
        return EDP_ERR_ARG;
    }
    if (p->precision != EDP_PREC_MIXED && p->precision != EDP_PREC_FP64) return EDP_ERR_ARG;
    if (t->en_on && (t->n_act < 1 || t->n_act > EDP_MAX_COLPROC || t->n_seg < 1 || t->n_seg > EDP_MAX_SEGMENTS ||
                     !t->prob || !t->energy_eV))
        return EDP_ERR_ARG;
    if (!t->maxwell_v || t->maxwell_rmax < 1) return EDP_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return EDP_ERR_CUDA;

    edp_ctx* c = new edp_ctx();
    c->p = *p;
    c->tab = *t;
    cudaGetDevice(&c->device);
    c->nspec = 1 + p->n_ion_species;
    edp_kparams& kp = c->kp;
    memset(&kp, 0, sizeof(kp));
    kp.ncx = p->ncx;
    kp.ncy = p->ncy;
    kp.periodic = p->periodic_x;
    kp.nxg = p->periodic_x ? p->ncx : p->ncx + 1;
    kp.nyg = p->ncy + 1;
    kp.n_inner = p->n_inner;
    for (int n = 0; n < p->n_inner; ++n) {
        kp.ileft[n] = p->inner_ileft[n];
        kp.jbottom[n] = p->inner_jbottom[n];
        kp.iright[n] = p->inner_iright[n];
        kp.jtop[n] = p->inner_jtop[n];
        if (p->inner_eps[n] > 0.0) kp.diel_mask |= 1 << n;
    }
    kp.nsub = p->n_subcycles;
    kp.seed_lo = (uint32_t)p->seed;
    kp.seed_hi = (uint32_t)(p->seed >> 32);
    rotation(-0.5 * p->bx, -0.5 * p->by, -0.5 * p->bz, c->K[0]);
    for (int s = 0; s < p->n_ion_species; ++s) {
        double qn = p->n_subcycles * 0.5 * p->ion_charge[s] / p->ion_mass_me[s];
        rotation(qn * p->bx, qn * p->by, qn * p->bz, c->K[1 + s]);
    }
    int r = EDP_OK;
    auto fail = [&](int code) {
        edp_destroy(c);
        return code;
    };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(EDP_ERR_CUDA);
    if (cudaMalloc(&c->dc, sizeof(edp_dev_counters)) != cudaSuccess) return fail(EDP_ERR_CUDA);
    if (cudaMallocHost(&c->hc, sizeof(edp_dev_counters)) != cudaSuccess) return fail(EDP_ERR_CUDA);
    memset(c->hc, 0, sizeof(edp_dev_counters));
    cudaMemset(c->dc, 0, sizeof(edp_dev_counters));
    if (cudaMalloc(&c->dev_small, 4096) != cudaSuccess) return fail(EDP_ERR_CUDA);
    const int64_t nn = (int64_t)kp.nxg * kp.nyg;
    if (p->precision == EDP_PREC_MIXED) {
        if ((r = dalloc(c, &c->E2, nn)) || (r = dalloc(c, &c->acc2, nn))) return fail(r);
        for (int s = 0; s < c->nspec; ++s)
            if ((r = dalloc(c, &c->rho_fix[s], nn))) return fail(r);
        cudaMemset(c->E2, 0, nn * sizeof(float2));
        cudaMemset(c->acc2, 0, nn * sizeof(float2));
    } else {
        if ((r = dalloc(c, &c->Ex, nn)) || (r = dalloc(c, &c->Ey, nn)) || (r = dalloc(c, &c->accx, nn)) ||
            (r = dalloc(c, &c->accy, nn)))
            return fail(r);
        for (int s = 0; s < c->nspec; ++s)
            if ((r = dalloc(c, &c->rho_d[s], nn))) return fail(r);
        cudaMemset(c->Ex, 0, nn * sizeof(double));
        cudaMemset(c->Ey, 0, nn * sizeof(double));
        cudaMemset(c->accx, 0, nn * sizeof(double));
        cudaMemset(c->accy, 0, nn * sizeof(double));
    }
    if ((r = dalloc(c, &c->rho_total, nn)) || (r = dalloc(c, &c->phi, nn)) || (r = dalloc(c, &c->phi_prev, nn)))
        return fail(r);
    cudaMemset(c->phi, 0, nn * sizeof(double));
    cudaMemset(c->rho_total, 0, nn * sizeof(double));
    if (p->solver == EDP_SOLVER_CG) {
        if ((r = dalloc(c, &c->cg_b, nn)) || (r = dalloc(c, &c->cg_r, nn)) || (r = dalloc(c, &c->cg_p, nn)) ||
            (r = dalloc(c, &c->cg_Ap, nn)) || (r = dalloc(c, &c->cg_z, nn)) || (r = dalloc(c, &c->cg_kind, nn)) ||
            (r = dalloc(c, &c->cg_sc, EDP_CG_SCALARS)))
            return fail(r);
    }
    // sort workspace
    c->ntx = (p->ncx + EDP_TILE - 1) / EDP_TILE;
    c->nty = (p->ncy + EDP_TILE - 1) / EDP_TILE;
    if (p->precision == EDP_PREC_MIXED) {
        int64_t ntiles = (int64_t)c->ntx * c->nty, nkeys = ntiles * 256;
        if ((r = dalloc(c, &c->sort_count, nkeys + 1)) || (r = dalloc(c, &c->sort_offset, nkeys + 1)) ||
            (r = dalloc(c, &c->scan_tmp, 2 * ntiles + nkeys + 4)))
            return fail(r);
    }
    // tables
    if (t->en_on) {
        int64_t np = (int64_t)(t->n_values + 1) * t->n_act;
        if ((r = dalloc(c, &c->mcc_prob, np)) || (r = dalloc(c, &c->mcc_energy, t->n_values + 1))) return fail(r);
        cudaMemcpy(c->mcc_prob, t->prob, np * sizeof(double), cudaMemcpyHostToDevice);
        cudaMemcpy(c->mcc_energy, t->energy_eV, (t->n_values + 1) * sizeof(double), cudaMemcpyHostToDevice);
    }
    if ((r = dalloc(c, &c->maxwell_v, t->maxwell_rmax + 1))) return fail(r);
    cudaMemcpy(c->maxwell_v, t->maxwell_v, (t->maxwell_rmax + 1) * sizeof(double), cudaMemcpyHostToDevice);
    c->tab.prob = nullptr;
    c->tab.energy_eV = nullptr;
    c->tab.maxwell_v = nullptr;
    {
        edp_mcc_dev m = edp_make_mcc_dev(c);
        if ((r = dalloc(c, &c->mcc_dev, 1))) return fail(r);
        cudaMemcpy(c->mcc_dev, &m, sizeof(m), cudaMemcpyHostToDevice);
    }
    if ((r = edp_fields_prepare(c))) return fail(r);
    if (p->solver == EDP_SOLVER_CG && (r = edp_mg_setup(c))) return fail(r);
    if (kp.diel_mask) {
        if ((r = edp_dielectrics_setup(c))) return fail(r);
        if ((r = alloc_hits(c, 65536))) return fail(r);   // grows with the electron add list
    }
    for (int s = 0; s < 4; ++s) {
        EdpPotentialProfile& q = c->pot[s];
        q.phi_const = p->wall_phi_const[s];
        q.phi_var = p->wall_phi_var[s];
        q.omega = p->wall_omega[s];
        q.phase = q.phase_adjusted = p->wall_phase[s];
        c->phi_wall[s] = q.value(0);
    }
    for (int n = 0; n < EDP_MAX_INNER; ++n) {   // constant until edp_set_potential_profile gives a time dependence
        c->pot[4 + n].phi_const = p->inner_phi[n];
        c->phi_inner[n] = p->inner_phi[n];
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(EDP_ERR_CUDA);
    *out = c;
    return EDP_OK;
}

int edp_destroy(edp_ctx* c)
{
    if (!c) return EDP_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    auto F = [](void* q) {
        if (q) cudaFree(q);
    };
    for (int s = 0; s < EDP_MAX_SPECIES; ++s) {
        for (edp_species_mixed* m : {&c->pm[s], &c->pm_alt[s]}) {
            F(m->cell); F(m->ox); F(m->oy); F(m->vx); F(m->vy); F(m->vz); F(m->id); F(m->tag);
        }
        edp_species_fp64& d = c->pd[s];
        F(d.x); F(d.y); F(d.vx); F(d.vy); F(d.vz); F(d.id); F(d.tag);
        F(c->chunks[s]);
        F(c->rho_fix[s]);
        F(c->rho_d[s]);
    }
    {
        edp_born& e = c->born_e;
        F(e.x); F(e.y); F(e.vx); F(e.vy); F(e.vz);
    }
    for (int s = 0; s < EDP_MAX_ION_SPECIES; ++s) {
        edp_born& e = c->born_i[s];
        F(e.x); F(e.y); F(e.vx); F(e.vy); F(e.vz);
    }
    F(c->sort_count); F(c->sort_offset); F(c->scan_tmp);
    F(c->E2); F(c->acc2); F(c->Ex); F(c->Ey); F(c->accx); F(c->accy);
    F(c->rho_total); F(c->phi); F(c->phi_prev); F(c->spec); F(c->aeq); F(c->twiddle);
    F(c->cg_b); F(c->cg_r); F(c->cg_p); F(c->cg_Ap); F(c->cg_z); F(c->cg_kind); F(c->cg_sc); F(c->strip_cnt);
    for (auto& row : c->cg_exec)
        for (auto& g : row)
            if (g) cudaGraphExecDestroy(g);
    edp_mg_free(c);
    edp_warmstart_free(c);
    F(c->mcc_prob); F(c->mcc_energy); F(c->maxwell_v); F(c->maxwell_inj); F(c->emit_dev); F(c->inject_cells);
    delete c->emit_h;
    delete c->see_h;
    F(c->see_dev);
    F(c->epsx); F(c->epsy); F(c->surf);
    F(c->hits.x); F(c->hits.y); F(c->hits.vx); F(c->hits.vy); F(c->hits.vz); F(c->hits.id); F(c->hits.ws);
    F(c->dc); F(c->dev_small); F(c->mcc_dev); F(c->born_dev); F(c->sel_list); F(c->sel_count);
    if (c->hc) cudaFreeHost(c->hc);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return EDP_OK;
}

int edp_last_error(const edp_ctx* c, char* buf, size_t len)
{
    if (!c || !buf || len == 0) return EDP_ERR_ARG;
    snprintf(buf, len, "%s", c->last_error.c_str());
    return EDP_OK;
}

int edp_set_sync(edp_ctx* c, int sync)
{
    if (!c) return EDP_ERR_ARG;
    c->sync = sync;
    return EDP_OK;
}

int edp_get_stream(edp_ctx* c, void** out)
{
    if (!c || !out) return EDP_ERR_ARG;
    *out = (void*)c->stream;
    return EDP_OK;
}

int edp_sort_particles(edp_ctx* c)
{
    if (!c) return EDP_ERR_ARG;
    for (int s = 0; s < c->nspec; ++s)
        if (c->uploaded[s]) TRY(edp_launch_sort(c, s));
    c->steps_since_sort = 0;
    return finish_sync(c);
}

int edp_synchronize(edp_ctx* c)
{
    if (!c) return EDP_ERR_ARG;
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    return EDP_OK;
}

int edp_upload_particles(edp_ctx* c, int sp, int64_t n, const double* x, const double* y, const double* vx,
                         const double* vy, const double* vz, const int32_t* tag, const uint32_t* id)
{
    if (!c || sp < 0 || sp >= c->nspec || n < 0 || (n > 0 && (!x || !y || !vx || !vy || !vz)))
        return edp_fail(c, EDP_ERR_ARG, "edp_upload_particles: bad arguments");
    if (!id && c->id_base + (uint64_t)n > c->id_end)
        return edp_fail(c, EDP_ERR_CAPACITY, "edp_upload_particles: more particles than ids left in the context's range");
    TRY(alloc_species(c, sp, n));
    // staging copies of the host columns
    double* dbuf = nullptr;
    int32_t* tbuf = nullptr;
    uint32_t* ibuf = nullptr;
    const int64_t nn = std::max<int64_t>(n, 1);
    EDP_CUDA(c, cudaMalloc(&dbuf, nn * 5 * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&tbuf, nn * sizeof(int32_t)));
    EDP_CUDA(c, cudaMalloc(&ibuf, nn * sizeof(uint32_t)));
    const double* cols[5] = {x, y, vx, vy, vz};
    for (int q = 0; q < 5; ++q)
        if (n) EDP_CUDA(c, cudaMemcpyAsync(dbuf + q * nn, cols[q], n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (tag && n) EDP_CUDA(c, cudaMemcpyAsync(tbuf, tag, n * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    if (id && n) EDP_CUDA(c, cudaMemcpyAsync(ibuf, id, n * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
        ++c->launches;
    if (n)
        upload_kernel<<<grid_of(n), 256, 0, c->stream>>>(c->kp, c->p.precision, n, 0, dbuf, dbuf + nn, dbuf + 2 * nn,
                                                         dbuf + 3 * nn, dbuf + 4 * nn, tag ? tbuf : nullptr,
                                                         id ? ibuf : nullptr, c->pm[sp], c->pd[sp], &c->dc->error_flags,
                                                         c->id_base);
    EDP_CUDA(c, cudaGetLastError());
    unsigned long long ns = (unsigned long long)n, nid = (unsigned long long)(c->id_base + n);
    if (id && n) {   // new particles continue after the uploaded ids, inside this context's range (edp_set_id_base)
        std::vector<uint32_t> h(id, id + n);
        nid = std::max<unsigned long long>((unsigned long long)*std::max_element(h.begin(), h.end()) + 1ull,
                                           (unsigned long long)c->id_base);
    }
    EDP_CUDA(c, cudaMemcpyAsync(&c->dc->n_slots[sp], &ns, sizeof(ns), cudaMemcpyHostToDevice, c->stream));
    EDP_CUDA(c, cudaMemcpyAsync(&c->dc->next_id[sp], &nid, sizeof(nid), cudaMemcpyHostToDevice, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(dbuf);
    cudaFree(tbuf);
    cudaFree(ibuf);
    c->host_slots[sp] = n;
    TRY(after_particles_changed(c, sp));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    unsigned int flags = 0;
    EDP_CUDA(c, cudaMemcpy(&flags, &c->dc->error_flags, sizeof(flags), cudaMemcpyDeviceToHost));
    if (flags & EDP_EFLAG_BOUNDS) return edp_fail(c, EDP_ERR_BOUNDS, "edp_upload_particles: particle outside the domain");
    return EDP_OK;
}

int edp_distribute_particles(edp_ctx* c, int sp, int32_t per_cell, double fconv, int32_t zero_vz, int32_t copy_pos)
{
    if (!c || sp < 0 || sp >= c->nspec || per_cell < 1) return edp_fail(c, EDP_ERR_ARG, "edp_distribute_particles");
    if (copy_pos && (sp == 0 || !c->uploaded[0])) return edp_fail(c, EDP_ERR_STATE, "electrons must be distributed first");
    const int64_t n = (int64_t)per_cell * c->p.ncx * c->p.ncy;
    if (c->id_base + (uint64_t)n > c->id_end)
        return edp_fail(c, EDP_ERR_CAPACITY, "edp_distribute_particles: more particles than ids left in the context's range");
    if (copy_pos && (n != c->host_slots[0] || c->sorted_end[0] != 0))
        return edp_fail(c, EDP_ERR_STATE, "ions copy electron positions: same per_cell, before the electron sort");
    TRY(alloc_species(c, sp, n));
    const int64_t base_id = (int64_t)c->id_base;
    ++c->launches;
    distribute_kernel<<<grid_of(n, 148 * 64), 256, 0, c->stream>>>(
        c->kp, c->p.precision, sp, per_cell, fconv, zero_vz, copy_pos, c->maxwell_v, c->tab.maxwell_rmax, base_id,
        c->pm[sp], c->pd[sp], c->pm[0], c->pd[0], n);
    EDP_CUDA(c, cudaGetLastError());
    unsigned long long ns = (unsigned long long)n;
    EDP_CUDA(c, cudaMemcpyAsync(&c->dc->n_slots[sp], &ns, sizeof(ns), cudaMemcpyHostToDevice, c->stream));
    const unsigned long long nid = (unsigned long long)(base_id + n);
    EDP_CUDA(c, cudaMemcpyAsync(&c->dc->next_id[sp], &nid, sizeof(nid), cudaMemcpyHostToDevice, c->stream));
    c->host_slots[sp] = n;
    // the electron array is sorted only after the ions copied its positions
    if (sp == 0 && copy_pos == 0) {
        c->hc->n_live[sp] = 0;
        EDP_CUDA(c, cudaMemsetAsync(&c->dc->n_live[sp], 0, sizeof(unsigned long long), c->stream));
        ++c->launches;
        count_live_kernel<<<grid_of(n), 256, 0, c->stream>>>(c->kp, c->p.precision, c->pm[sp], c->pd[sp], n,
                                                             &c->dc->n_live[sp]);
        TRY(zero_density(c, sp));
        TRY(edp_launch_deposit(c, sp));
        c->uploaded[sp] = 1;
        c->sorted_end[sp] = 0;
        c->n_chunks[sp] = 0;
        EDP_CUDA(c, cudaStreamSynchronize(c->stream));
        return EDP_OK;
    }
    TRY(after_particles_changed(c, sp));
    if (copy_pos && c->p.precision == EDP_PREC_MIXED && c->p.sort_every > 0 && c->sorted_end[0] == 0)
        TRY(edp_launch_sort(c, 0));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    return EDP_OK;
}

int edp_download_particles(edp_ctx* c, int sp, int64_t cap, int64_t* n_out, double* x, double* y, double* vx,
                           double* vy, double* vz, int32_t* tag, uint32_t* id)
{
    if (!c || sp < 0 || sp >= c->nspec || !n_out) return edp_fail(c, EDP_ERR_ARG, "edp_download_particles");
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    unsigned long long ns = 0;
    EDP_CUDA(c, cudaMemcpy(&ns, &c->dc->n_slots[sp], sizeof(ns), cudaMemcpyDeviceToHost));
    const int64_t n = (int64_t)ns;
    int64_t w = 0;
    if (c->p.precision == EDP_PREC_MIXED) {
        std::vector<int32_t> cell(n), tg(n);
        std::vector<float> ox(n), oy(n), fvx(n), fvy(n), fvz(n);
        std::vector<uint32_t> ids(n);
        const edp_species_mixed& m = c->pm[sp];
        if (n) {
            EDP_CUDA(c, cudaMemcpy(cell.data(), m.cell, n * 4, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(ox.data(), m.ox, n * 4, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(oy.data(), m.oy, n * 4, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(fvx.data(), m.vx, n * 4, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(fvy.data(), m.vy, n * 4, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(fvz.data(), m.vz, n * 4, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(ids.data(), m.id, n * 4, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(tg.data(), m.tag, n * 4, cudaMemcpyDeviceToHost));
        }
        for (int64_t k = 0; k < n; ++k) {
            if (cell[k] < 0) continue;
            if (w < cap) {
                if (x) x[w] = (double)(cell[k] & 0xFFFF) + (double)ox[k];
                if (y) y[w] = (double)(cell[k] >> 16) + (double)oy[k];
                if (vx) vx[w] = fvx[k];
                if (vy) vy[w] = fvy[k];
                if (vz) vz[w] = fvz[k];
                if (tag) tag[w] = tg[k];
                if (id) id[w] = ids[k];
            }
            ++w;
        }
    } else {
        std::vector<double> hx(n), hy(n), hvx(n), hvy(n), hvz(n);
        std::vector<int32_t> tg(n);
        std::vector<uint32_t> ids(n);
        const edp_species_fp64& d = c->pd[sp];
        if (n) {
            EDP_CUDA(c, cudaMemcpy(hx.data(), d.x, n * 8, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(hy.data(), d.y, n * 8, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(hvx.data(), d.vx, n * 8, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(hvy.data(), d.vy, n * 8, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(hvz.data(), d.vz, n * 8, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(ids.data(), d.id, n * 4, cudaMemcpyDeviceToHost));
            EDP_CUDA(c, cudaMemcpy(tg.data(), d.tag, n * 4, cudaMemcpyDeviceToHost));
        }
        for (int64_t k = 0; k < n; ++k) {
            if (hx[k] < -1.0e29) continue;
            if (w < cap) {
                if (x) x[w] = hx[k];
                if (y) y[w] = hy[k];
                if (vx) vx[w] = hvx[k];
                if (vy) vy[w] = hvy[k];
                if (vz) vz[w] = hvz[k];
                if (tag) tag[w] = tg[k];
                if (id) id[w] = ids[k];
            }
            ++w;
        }
    }
    *n_out = w;
    if (w > cap) return edp_fail(c, EDP_ERR_CAPACITY, "edp_download_particles: host buffer too small");
    return EDP_OK;
}

int edp_gather_charge_density(edp_ctx* c, int sp, double* rho_out)
{
    if (!c || sp < 0 || sp >= c->nspec) return edp_fail(c, EDP_ERR_ARG, "edp_gather_charge_density");
    if (!rho_out) return EDP_OK;
    const int w = ref_width(c);
    const int64_t nref = (int64_t)w * c->kp.nyg;
    double *tmp = nullptr, *ref = nullptr;
    EDP_CUDA(c, cudaMalloc(&tmp, (int64_t)c->kp.nxg * c->kp.nyg * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&ref, nref * sizeof(double)));
    double wgt = sp == 0 ? 1.0 : (double)c->p.ion_charge[sp - 1];
    ++c->launches;
    species_density_kernel<<<grid_of(nref), 256, 0, c->stream>>>(c->kp, c->p.precision, c->rho_fix[sp], c->rho_d[sp],
                                                                  wgt, tmp);
    ++c->launches;
    expand_kernel<<<grid_of(nref), 256, 0, c->stream>>>(c->kp, 0, tmp, nullptr, 0, ref, w);
    EDP_CUDA(c, cudaGetLastError());
    EDP_CUDA(c, cudaMemcpyAsync(rho_out, ref, nref * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(tmp);
    cudaFree(ref);
    return EDP_OK;
}

int edp_update_wall_potentials(edp_ctx* c, int64_t t)
{
    if (!c || t < 0 || t > INT32_MAX) return EDP_ERR_ARG;
    for (int s = 0; s < 4; ++s) c->phi_wall[s] = c->pot[s].value((int32_t)t);
    for (int n = 0; n < c->p.n_inner; ++n)
        if (c->p.inner_eps[n] == 0.0) c->phi_inner[n] = c->pot[4 + n].value((int32_t)t);   // metal objects only
    return EDP_OK;
}

int edp_set_potential_profile(edp_ctx* c, int32_t object, const double* harmonic, int32_t n_wf, const int32_t* wf_t,
                              const float* wf_phi, int32_t n_ap, const int32_t* ap_t, const float* ap_factor)
{
    if (!c || object < 0 || object >= 4 + EDP_MAX_INNER || !harmonic || n_wf < 0 || n_ap < 0 || n_wf == 1 ||
        n_ap == 1 || (n_wf && (!wf_t || !wf_phi)) || (n_ap && (!ap_t || !ap_factor)))
        return edp_fail(c, EDP_ERR_ARG, "edp_set_potential_profile");
    for (int32_t k = 0; k + 1 < n_wf; ++k)
        if (!(wf_t[k + 1] > wf_t[k]) || wf_t[0] != 0) return edp_fail(c, EDP_ERR_ARG, "waveform times must rise from 0");
    for (int32_t k = 0; k + 1 < n_ap; ++k)
        if (!(ap_t[k + 1] > ap_t[k]) || ap_t[0] != 0)
            return edp_fail(c, EDP_ERR_ARG, "amplitude-profile times must rise from 0");
    EdpPotentialProfile& q = c->pot[object];
    q.phi_const = harmonic[0];
    q.phi_var = harmonic[1];
    q.omega = harmonic[2];
    q.phase = harmonic[3];
    q.wf_t.assign(wf_t, wf_t + n_wf);
    q.wf_phi.assign(wf_phi, wf_phi + n_wf);
    q.ap_t.assign(ap_t, ap_t + n_ap);
    q.ap_factor.assign(ap_factor, ap_factor + n_ap);
    q.adjust_phase((int32_t)c->t_cntr);
    // the potential of the current step, as UPDATE_WALL_POTENTIALS at set-up
    EdpPotentialProfile q0 = q;
    const double v = q0.value((int32_t)c->t_cntr);
    if (object < 4) c->phi_wall[object] = v;
    else c->phi_inner[object - 4] = v;
    return EDP_OK;
}

int edp_field_fftx(edp_ctx* c, double* phi_out)
{
    if (!c) return EDP_ERR_ARG;
    if (c->p.solver != EDP_SOLVER_FFTX) return edp_fail(c, EDP_ERR_STATE, "context was not set up for FFT_X");
    TRY(edp_launch_density(c));
    TRY(edp_launch_fftx(c));
    TRY(edp_launch_efield(c));
    if (phi_out) TRY(edp_get_field(c, EDP_FIELD_PHI, phi_out));
    return finish_sync(c);
}

int edp_set_cg_preconditioner(edp_ctx* c, int32_t kind)
{
    if (!c || (kind != EDP_PRECOND_NONE && kind != EDP_PRECOND_MG)) return edp_fail(c, EDP_ERR_ARG, "preconditioner");
    if (kind == EDP_PRECOND_MG && c->mg_nlev == 0) return edp_fail(c, EDP_ERR_STATE, "context was not set up for CG");
    c->precond = kind;
    return EDP_OK;
}

// GetInjMaxwellVelocity's table v_inj(0:R_max_inj) for the flux-weighted half-Maxwellian t exp(-t^2), t >= 0
// (PrepareMaxwellDistribIntegral, pic2d_ElectronWallCollisions.f90:889-915): the inverse of its running integral at
// R_max_inj equal steps.
static std::vector<double> injection_maxwell_table(int rmax)
{
    const int n = 90000;
    const double vmin = 0.0, dv = 3.0 / n;
    std::vector<double> F(n + 4, 0.0), v(rmax + 1, 0.0);
    for (int i = 1; i <= n + 3; ++i) {
        const double t = vmin + ((double)(float)i - 0.5) * dv;
        F[i] = F[i - 1] + std::exp(-(t * t)) * t;
    }
    const double tot = F[n];
    v[0] = vmin;
    int count = 0;
    for (int i = 1; i <= n + 3 && count < rmax; ++i)
        if ((int)(F[i] * rmax / tot) - count == 1) v[++count] = vmin + i * dv;
    return v;
}

// device state of the ion-wall interactions, made on first use: the wall-hit list, the injection table and the
// parameter block
static int wall_state(edp_ctx* c)
{
    if (!c->emit_h) {
        const int rmax_inj = 4500;
        std::vector<double> v = injection_maxwell_table(rmax_inj);
        TRY(dalloc(c, &c->maxwell_inj, rmax_inj + 1));
        EDP_CUDA(c, cudaMemcpy(c->maxwell_inj, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
        TRY(dalloc(c, &c->emit_dev, 1));
        if (!c->hits.x) TRY(alloc_hits(c, std::max<int64_t>(65536, c->born_cap)));   // the electron add list's size
        c->emit_h = new edp_emit_dev();
        memset(c->emit_h, 0, sizeof(edp_emit_dev));
        c->emit_h->maxwell_v = c->maxwell_v;
        c->emit_h->rmax = c->tab.maxwell_rmax;
        c->emit_h->maxwell_inj = c->maxwell_inj;
        c->emit_h->rmax_inj = rmax_inj;
    }
    return EDP_OK;
}

static int upload_wall_state(edp_ctx* c)
{
    const edp_emit_dev& h = *c->emit_h;
    c->emit_on = 0;
    c->kp.ion_inner_mask = 0;
    for (int w = 0; w < EDP_N_HIT_COUNTERS; ++w) {
        int any = h.reflect[w];
        for (int q = 0; q < EDP_MAX_ION_SPECIES; ++q) any |= h.on[w][q];
        c->emit_on |= any;
        if (w >= 4 && any) c->kp.ion_inner_mask |= 1 << (w - 4);
    }
    EDP_CUDA(c, cudaMemcpyAsync(c->emit_dev, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    return EDP_OK;
}

int edp_set_ion_emission(edp_ctx* c, int32_t wall, int32_t ion_species, double yield, double emin_ev, double emax_ev,
                         double t_emit_ev)
{
    if (c && c->kp.strip) return edp_fail(c, EDP_ERR_STATE, "no wall emission on a strip");
    if (!c || wall < 0 || wall >= 4 + c->p.n_inner || ion_species < 1 || ion_species >= c->nspec || !(yield >= 0.0) ||
        !(emax_ev > emin_ev) || !(t_emit_ev >= 0.0))
        return edp_fail(c, EDP_ERR_ARG, "edp_set_ion_emission");
    TRY(wall_state(c));
    edp_emit_dev& h = *c->emit_h;
    const int s = ion_species - 1;
    const double ef = c->tab.energy_factor_eV;
    h.on[wall][s] = yield > 0.0;
    h.yield[wall][s] = yield;
    h.emin[wall][s] = emin_ev / ef;
    h.emax[wall][s] = emax_ev / ef;
    h.fconv[wall][s] = std::sqrt(t_emit_ev / ef);
    h.ms[s] = c->p.ion_mass_me[s];
    return upload_wall_state(c);
}

int edp_set_electron_emission(edp_ctx* c, int32_t wall, const edp_see_params* sp)
{
    if (c && c->kp.strip) return edp_fail(c, EDP_ERR_STATE, "no wall emission on a strip");
    if (!c || wall < 0 || wall >= 4 + c->p.n_inner) return edp_fail(c, EDP_ERR_ARG, "edp_set_electron_emission");
    if (sp && (sp->elastic_model < 0 || sp->elastic_model > 2 || sp->inelastic_model < 0 || sp->inelastic_model > 2 ||
               sp->true_model < 0 || sp->true_model > 2))
        return edp_fail(c, EDP_ERR_ARG, "edp_set_electron_emission: model outside 0-2");
    TRY(wall_state(c));
    if (!c->see_h) {
        TRY(dalloc(c, &c->see_dev, 1));
        c->see_h = new edp_see_dev();
        memset(c->see_h, 0, sizeof(edp_see_dev));
        c->see_h->maxwell_v = c->maxwell_v;
        c->see_h->rmax = c->tab.maxwell_rmax;
        c->see_h->maxwell_inj = c->maxwell_inj;
        c->see_h->rmax_inj = c->emit_h->rmax_inj;
    }
    edp_see_wall& w = c->see_h->w[wall];
    memset(&w, 0, sizeof(w));
    if (sp && sp->elastic_model + sp->inelastic_model + sp->true_model > 0) {
        // PREPARE_WALL_MATERIALS, pic2d_Materials.f90:195-244: energies to code units, the emission temperature to
        // a velocity factor, and the lowest energy at which any model emits
        const double ef = c->tab.energy_factor_eV;
        w.on = 1;
        w.m_el = sp->elastic_model;
        w.m_in = sp->inelastic_model;
        w.m_tr = sp->true_model;
        w.refl_random = sp->elastic_type != 0;
        w.el_yield = sp->elastic_yield;
        w.el_emin = sp->elastic_emin_ev / ef;
        w.el_emax = sp->elastic_emax_ev / ef;
        w.el_e0 = sp->elastic_e0_ev / ef;
        w.el_emaxc = sp->elastic_emax_coef_ev / ef;
        w.el_max = sp->elastic_max;
        w.el_de = sp->elastic_de_ev / ef;
        w.el_frac = sp->elastic_frac_classic;
        w.in_yield = sp->inelastic_yield;
        w.in_emin = sp->inelastic_emin_ev / ef;
        w.in_emax = sp->inelastic_emax_ev / ef;
        w.in_frac = sp->inelastic_frac_classic;
        w.tr_yield = sp->true_yield;
        w.tr_emin = sp->true_emin_ev / ef;
        w.tr_emax = sp->true_emax_ev / ef;
        w.cl_e0 = sp->classic_e0_ev / ef;
        w.cl_emax = sp->classic_emax_ev / ef;
        w.cl_max = sp->classic_max;
        w.cl_k = sp->classic_k_smooth;
        w.fconv = std::sqrt(sp->true_t_ev / ef);
        double lo = 1.0e6 / ef;
        if (w.m_el == 1) lo = std::min(lo, w.el_emin);
        if (w.m_el == 2) lo = std::min(lo, w.el_e0);
        if (w.m_in == 1) lo = std::min(lo, w.in_emin);
        if (w.m_in == 2) lo = std::min(lo, w.cl_e0);
        if (w.m_tr == 1) lo = std::min(lo, w.tr_emin);
        if (w.m_tr == 2) lo = std::min(lo, w.cl_e0);
        w.lowest = lo;
    }
    c->see_on = 0;   // the domain walls; inner objects by bit
    for (int q = 0; q < 4; ++q) c->see_on |= c->see_h->w[q].on;
    c->kp.see_inner_mask = 0;
    for (int n = 0; n < EDP_MAX_INNER; ++n)
        if (c->see_h->w[4 + n].on) c->kp.see_inner_mask |= 1 << n;
    EDP_CUDA(c, cudaMemcpyAsync(c->see_dev, c->see_h, sizeof(edp_see_dev), cudaMemcpyHostToDevice, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    return EDP_OK;
}

// Covered cells of the sides of inner object n (pic2d_CurProblemValues.f90:603-683): a cell of a side is covered when
// a domain wall's segment lies on it or another inner object touches or overlaps it. Side m = 1 left, 2 top, 3 right,
// 4 bottom; cells along the side from its start (jbottom or ileft). The domain walls are the segments j = 0 and
// j = ncy for all i, and, on a walled domain, i = 0 and i = ncx for all j.
static std::vector<char> inner_side_covered(const edp_ctx* c, int n, int m)
{
    const edp_kparams& k = c->kp;
    const bool vertical = m == 1 || m == 3;
    const int at = m == 1 ? k.ileft[n] : m == 3 ? k.iright[n] : m == 2 ? k.jtop[n] : k.jbottom[n];
    const int a0 = vertical ? k.jbottom[n] : k.ileft[n], a1 = vertical ? k.jtop[n] : k.iright[n];
    std::vector<char> cov(std::max(0, a1 - a0), 0);
    for (int q = a0; q < a1; ++q) {
        bool c1 = false;
        if (vertical) c1 = !c->p.periodic_x && (at == 0 || at == k.ncx) && q >= 0 && q < k.ncy;
        else c1 = (at == 0 || at == k.ncy);
        for (int o = 0; o < k.n_inner && !c1; ++o) {
            if (o == n) continue;
            if (vertical) c1 = at >= k.ileft[o] && at <= k.iright[o] && q >= k.jbottom[o] && q < k.jtop[o];
            else c1 = at >= k.jbottom[o] && at <= k.jtop[o] && q >= k.ileft[o] && q < k.iright[o];
        }
        cov[q - a0] = c1;
    }
    return cov;
}

// The emitting sides of inner object n for N macroparticles per step (PERFORM_ELECTRON_EMISSION_SETUP_INNER_OBJECTS,
// pic2d_Setup.f90:1005-1591, one cluster over the domain): a side inside the domain emits
// REAL(N) * REAL(open) / REAL(L) per step, `open` its cells not covered inside [cross_min, cross_max), L the open
// cells of all four sides; the open cells are listed for the placement.
static int inner_injection_sides(edp_ctx* c, int n, double n_emit, std::vector<int>* cells)
{
    const edp_kparams& k = c->kp;
    edp_inject_dev& in = c->inject;
    const int xmax_idx = c->p.periodic_x ? k.ncx + 1 : k.ncx;   // c_indx_x_max of the one cluster
    const int ymax_idx = k.ncy;
    std::vector<char> cov[4];
    int L = 0;
    for (int m = 1; m <= 4; ++m) {
        cov[m - 1] = inner_side_covered(c, n, m);
        for (char v : cov[m - 1]) L += !v;
    }
    for (int m = 1; m <= 4; ++m) {
        const int s = 4 * n + (m - 1);
        in.side_n[s] = 0.0;
        in.side_open[s] = 0;
        const bool vertical = m == 1 || m == 3;
        const int at = m == 1 ? k.ileft[n] : m == 3 ? k.iright[n] : m == 2 ? k.jtop[n] : k.jbottom[n];
        const int a0 = vertical ? k.jbottom[n] : k.ileft[n], a1 = vertical ? k.jtop[n] : k.iright[n];
        const int lim = vertical ? xmax_idx : ymax_idx;       // the side must lie strictly inside the cluster
        const int alim = vertical ? ymax_idx : xmax_idx;
        if (!(n_emit > 0.0) || L == 0 || !(at > 0 && at < lim) || !(a0 < alim && a1 > 0)) continue;
        const int cmin = std::max(a0, 0), cmax = std::min(a1, alim - 1);
        in.side_off[s] = (int)cells->size();
        for (int q = cmin; q < cmax; ++q)
            if (!cov[m - 1][q - a0]) cells->push_back(q);
        const int open = (int)cells->size() - in.side_off[s];
        if (open == 0) continue;
        in.side_open[s] = open;
        in.side_cmin[s] = cmin;
        in.side_cmax[s] = cmax;
        in.side_at[s] = (m == 1 || m == 4) ? (double)at - 1.0e-6 : (double)at + 1.0e-6;
        in.side_n[s] = (double)((float)n_emit * (float)open / (float)L);   // single precision, as the reference
    }
    return EDP_OK;
}

int edp_set_wall_injection(edp_ctx* c, int32_t wall, double n_per_step, int32_t model, double t_normal_ev,
                           double t_parallel_ev, double beam_energy_ev)
{
    if (c && c->kp.strip) return edp_fail(c, EDP_ERR_STATE, "no wall emission on a strip");
    if (!c || wall < 0 || wall >= 4 + c->p.n_inner || !(n_per_step >= 0.0) || n_per_step > 1.0e9 || model < 0 ||
        model > 1 || !(t_normal_ev >= 0.0) || !(t_parallel_ev >= 0.0))
        return edp_fail(c, EDP_ERR_ARG, "edp_set_wall_injection");
    if (c->p.periodic_x && (wall == 2 || wall == 3) && n_per_step > 0.0)
        return edp_fail(c, EDP_ERR_ARG, "edp_set_wall_injection: a periodic domain has walls below and above only");
    if (wall >= 4 && c->p.inner_eps[wall - 4] > 0.0 && n_per_step > 0.0)
        return edp_fail(c, EDP_ERR_ARG, "edp_set_wall_injection: only metal inner objects emit");
    if (model == 1 && n_per_step > 0.0 && !(beam_energy_ev > 1.5 * t_normal_ev))
        return edp_fail(c, EDP_ERR_ARG, "edp_set_wall_injection: beam energy spread above the beam energy / 1.5");
    TRY(wall_state(c));
    // PREPARE_SETUP_VALUES, pic2d_Setup.f90:103-126: sqrt(T / T_e) / N_max_vel = sqrt(T / energy_factor_eV)
    const double ef = c->tab.energy_factor_eV;
    edp_inject_dev& in = c->inject;
    in.maxwell_v = c->maxwell_v;
    in.rmax = c->tab.maxwell_rmax;
    in.maxwell_inj = c->maxwell_inj;
    in.rmax_inj = c->emit_h->rmax_inj;
    in.n[wall] = n_per_step;
    in.model[wall] = model;
    in.fp[wall] = std::sqrt(t_parallel_ev / ef);
    if (model == 0) {
        in.fn[wall] = std::sqrt(t_normal_ev / ef);
        in.vb[wall] = 0.0;
    } else {
        in.fn[wall] = n_per_step > 0.0 ? std::sqrt(0.25 * t_normal_ev * t_normal_ev / (beam_energy_ev * ef)) : 0.0;
        in.vb[wall] = std::sqrt(std::max(beam_energy_ev, 0.0) / ef);
    }
    // the sides of all emitting inner objects, listed again
    std::vector<int> cells;
    for (int n = 0; n < c->p.n_inner; ++n) TRY(inner_injection_sides(c, n, in.n[4 + n], &cells));
    if (cells.size() > EDP_INJECT_MAX_CELLS) return edp_fail(c, EDP_ERR_CAPACITY, "edp_set_wall_injection: sides");
    if (!cells.empty()) {
        if (!c->inject_cells) TRY(dalloc(c, &c->inject_cells, EDP_INJECT_MAX_CELLS));
        EDP_CUDA(c, cudaMemcpy(c->inject_cells, cells.data(), cells.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    in.open_cells = c->inject_cells;
    c->inject_on = 0;
    for (int w = 0; w < 4; ++w) c->inject_on |= in.n[w] > 0.0;
    for (int s = 0; s < EDP_INJECT_SIDES; ++s) c->inject_on |= in.side_n[s] > 0.0;
    return EDP_OK;
}

int edp_set_ion_reflection(edp_ctx* c, int32_t wall, int32_t on)
{
    if (c && c->kp.strip) return edp_fail(c, EDP_ERR_STATE, "no wall emission on a strip");
    if (!c || wall < 0 || wall >= 4 + c->p.n_inner) return edp_fail(c, EDP_ERR_ARG, "edp_set_ion_reflection");
    TRY(wall_state(c));
    c->emit_h->reflect[wall] = on ? 1 : 0;
    return upload_wall_state(c);
}

int edp_field_cg(edp_ctx* c, double rtol, int32_t max_it, int32_t warm, int32_t* iters_out)
{
    if (!c || max_it < 1 || !(rtol > 0.0) || warm < EDP_WARM_ZERO || warm > EDP_WARM_LEARNED)
        return edp_fail(c, EDP_ERR_ARG, "edp_field_cg");
    if (c->p.solver != EDP_SOLVER_CG) return edp_fail(c, EDP_ERR_STATE, "context was not set up for CG");
    TRY(edp_launch_density(c));
    int it = 0;
    int r = edp_launch_cg(c, rtol, max_it, warm, &it);
    if (iters_out) *iters_out = it;
    TRY(edp_launch_efield(c));
    if (r != EDP_OK) return r;
    return finish_sync(c);
}

int edp_advance_electrons(edp_ctx* c)
{
    if (!c) return EDP_ERR_ARG;
    if (!c->uploaded[0]) return edp_fail(c, EDP_ERR_STATE, "electrons not uploaded");
    const bool ion_step = (c->n_sub_phase + 1) == c->p.n_subcycles;
    const bool fuse = c->p.fuse_collisions != 0;
    ++c->launches;
    reset_step_counters_kernel<<<1, 1, 0, c->stream>>>(c->dc);
    TRY(zero_density(c, 0));
    TRY(edp_launch_push(c, 0, ion_step, fuse));
    if (c->see_on || c->kp.diel_mask || c->kp.see_inner_mask) TRY(edp_launch_electron_emission(c));
    return finish_sync(c);
}

int edp_advance_ions(edp_ctx* c)
{
    if (!c) return EDP_ERR_ARG;
    const bool ion_step = (c->n_sub_phase + 1) == c->p.n_subcycles;
    if (!ion_step) return EDP_OK;
    const bool fuse = c->p.fuse_collisions != 0;
    for (int s = 0; s < c->p.n_ion_species; ++s) {
        if (!c->uploaded[1 + s]) continue;
        TRY(zero_density(c, 1 + s));
        TRY(edp_launch_push(c, 1 + s, true, fuse));
    }
    if (c->emit_on || c->kp.diel_mask) TRY(edp_launch_ion_emission(c));
    return finish_sync(c);
}

int edp_collide_en(edp_ctx* c, int64_t* counters_out)
{
    if (!c) return EDP_ERR_ARG;
    const bool ion_step = (c->n_sub_phase + 1) == c->p.n_subcycles;
    if (ion_step && !c->p.fuse_collisions) TRY(edp_launch_collide_en(c));
    if (counters_out) {
        EDP_CUDA(c, cudaStreamSynchronize(c->stream));
        unsigned long long h[EDP_MAX_COLPROC];
        EDP_CUDA(c, cudaMemcpy(h, c->dc->en_coll_step, sizeof(h), cudaMemcpyDeviceToHost));
        for (int p = 0; p < EDP_MAX_COLPROC; ++p) counters_out[p] = (int64_t)h[p];
    }
    return finish_sync(c);
}

int edp_collide_rcx(edp_ctx* c, int64_t* count_out)
{
    if (!c) return EDP_ERR_ARG;
    const bool ion_step = (c->n_sub_phase + 1) == c->p.n_subcycles;
    if (ion_step && !c->p.fuse_collisions) TRY(edp_launch_collide_rcx(c));
    if (count_out) {
        EDP_CUDA(c, cudaStreamSynchronize(c->stream));
        unsigned long long h[EDP_MAX_ION_SPECIES];
        EDP_CUDA(c, cudaMemcpy(h, c->dc->rcx_step, sizeof(h), cudaMemcpyDeviceToHost));
        int64_t s = 0;
        for (int q = 0; q < EDP_MAX_ION_SPECIES; ++q) s += (int64_t)h[q];
        *count_out = s;
    }
    return finish_sync(c);
}

int edp_end_ion_cycle(edp_ctx* c)
{
    if (!c) return EDP_ERR_ARG;
    const bool ion_step = (c->n_sub_phase + 1) == c->p.n_subcycles;
    const int64_t nn = (int64_t)c->kp.nxg * c->kp.nyg;
    // PERFORM_ELECTRON_EMISSION_SETUP (pic2d_MainProgram.f90:353)
    if (c->inject_on) TRY(edp_launch_wall_injection(c));
    if (ion_step || c->see_on || c->inject_on) {
        // collisions run only on ion steps, so only then, or when walls emit electrons, can the add lists hold
        // anything (PROCESS_ADDED_ELECTRONS runs every step, pic2d_MainProgram.f90:363)
        TRY(edp_launch_append_born(c));
        ++c->launches;
        reset_born_kernel<<<1, 1, 0, c->stream>>>(c->dc);
    }
    if (ion_step) {
        if (c->p.precision == EDP_PREC_MIXED) {
            EDP_CUDA(c, cudaMemsetAsync(c->acc2, 0, nn * sizeof(float2), c->stream));
        } else {
            EDP_CUDA(c, cudaMemsetAsync(c->accx, 0, nn * sizeof(double), c->stream));
            EDP_CUDA(c, cudaMemsetAsync(c->accy, 0, nn * sizeof(double), c->stream));
        }
        c->n_sub_phase = 0;
    } else {
        c->n_sub_phase++;
    }
    EDP_CUDA(c, cudaGetLastError());
    c->t_cntr++;
    c->steps_since_sort++;
    if (c->p.precision == EDP_PREC_MIXED && c->p.sort_every > 0 && c->steps_since_sort >= c->p.sort_every &&
        c->n_sub_phase == 0) {
        for (int s = 0; s < c->nspec; ++s) {
            if (!c->uploaded[s]) continue;
            if (c->fused_sort) c->sort_due[s] = 1;   // done by the species' next push
            else TRY(edp_launch_sort(c, s));
        }
        c->steps_since_sort = 0;
    }
    return finish_sync(c);
}

int edp_set_sort_in_push(edp_ctx* c, int32_t on)
{
    if (!c) return EDP_ERR_ARG;
    c->fused_sort = on ? 1 : 0;
    if (!on)
        for (int s = 0; s < c->nspec; ++s)
            if (c->sort_due[s]) TRY(edp_launch_sort(c, s));
    return EDP_OK;
}

int edp_set_id_range(edp_ctx* c, uint64_t base, uint64_t end)
{
    if (!c || base >= end || end > (1ull << 32)) return edp_fail(c, EDP_ERR_ARG, "edp_set_id_range");
    c->id_base = base;
    c->id_end = end;
    return EDP_OK;
}

int edp_set_id_base(edp_ctx* c, uint64_t base)
{
    if (!c || base >= (1ull << 32)) return edp_fail(c, EDP_ERR_ARG, "edp_set_id_base");
    return edp_set_id_range(c, base, 1ull << 32);
}

int edp_reduce_list(edp_ctx* c, int32_t max, void** ptr, int64_t* count, int32_t* is_int64, int32_t* n_out)
{
    if (!c || !ptr || !count || !is_int64 || !n_out || max < 0) return edp_fail(c, EDP_ERR_ARG, "edp_reduce_list");
    if (c->kp.diel_mask) return edp_fail(c, EDP_ERR_STATE, "edp_reduce_list: dielectric objects on one rank only");
    const int64_t nn = (int64_t)c->kp.nxg * c->kp.nyg;
    const bool mixed = c->p.precision == EDP_PREC_MIXED;
    int32_t n = 0;
    for (int s = 0; s < c->nspec; ++s) {
        if (!((c->dirty >> s) & 1) || !c->uploaded[s]) continue;
        if (n == max) return edp_fail(c, EDP_ERR_ARG, "edp_reduce_list: max too small");
        ptr[n] = mixed ? (void*)c->rho_fix[s] : (void*)c->rho_d[s];
        count[n] = nn;
        is_int64[n] = mixed ? 1 : 0;
        ++n;
    }
    c->dirty = 0;
    *n_out = n;
    return EDP_OK;
}

int edp_set_step(edp_ctx* c, int64_t t_cntr)
{
    if (!c || t_cntr < 0 || t_cntr > INT32_MAX) return edp_fail(c, EDP_ERR_ARG, "edp_set_step");
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->t_cntr = t_cntr;
    c->n_sub_phase = 0;
    for (auto& q : c->pot) q.adjust_phase((int32_t)t_cntr);   // ADJUST_HARMONIC_OSCILLATIONS_PHASE (MainProgram:94)
    return EDP_OK;
}

int edp_step(edp_ctx* c, int32_t nsteps)
{
    if (!c || nsteps < 0) return EDP_ERR_ARG;
    for (int32_t k = 0; k < nsteps; ++k) {
        TRY(edp_update_wall_potentials(c, c->t_cntr));
        if (c->p.solver == EDP_SOLVER_FFTX) {
            TRY(edp_launch_density(c));
            TRY(edp_launch_fftx(c));
            TRY(edp_launch_efield(c));
        } else {
            TRY(edp_launch_density(c));
            int it = 0;
            TRY(edp_launch_cg(c, 1e-8, 100000, EDP_WARM_PREVIOUS, &it));
            TRY(edp_launch_efield(c));
        }
        TRY(edp_advance_electrons(c));
        TRY(edp_advance_ions(c));
        TRY(edp_collide_en(c, nullptr));
        TRY(edp_collide_rcx(c, nullptr));
        TRY(edp_end_ion_cycle(c));
    }
    return EDP_OK;
}

int edp_query_counters(edp_ctx* c, edp_counters* out)
{
    if (!c || !out) return EDP_ERR_ARG;
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    EDP_CUDA(c, cudaMemcpy(c->hc, c->dc, sizeof(edp_dev_counters), cudaMemcpyDeviceToHost));
    memset(out, 0, sizeof(*out));
    for (int s = 0; s < c->nspec; ++s) out->n_particles[s] = (int64_t)c->hc->n_live[s];
    for (int k = 0; k < EDP_N_HIT_COUNTERS; ++k) {
        out->electron_hits[k] = (int64_t)c->hc->e_hits[k];
        out->ion_hits[k] = (int64_t)c->hc->i_hits[k];
    }
    for (int p = 0; p < EDP_MAX_COLPROC; ++p) out->en_collisions[p] = (int64_t)c->hc->en_coll[p];
    for (int s = 0; s < EDP_MAX_ION_SPECIES; ++s) out->rcx_collisions[s] = (int64_t)c->hc->rcx[s];
    out->step = c->t_cntr;
    out->cg_iterations = c->last_cg_iters;
    out->cg_relres = c->last_cg_relres;
    out->error_flags = (int32_t)c->hc->error_flags;
    out->kernel_launches = c->launches;
    for (int s = 0; s < c->nspec; ++s) c->host_slots[s] = std::max<int64_t>((int64_t)c->hc->n_slots[s], 0);
    if (c->hc->error_flags & EDP_EFLAG_CAPACITY) return edp_fail(c, EDP_ERR_CAPACITY, "particle capacity exceeded");
    if (c->hc->error_flags & EDP_EFLAG_PENDING) return edp_fail(c, EDP_ERR_CAPACITY, "add-list capacity exceeded");
    if (c->hc->error_flags & EDP_EFLAG_BOUNDS) return edp_fail(c, EDP_ERR_BOUNDS, "particle outside the domain");
    if (c->hc->error_flags & EDP_EFLAG_TIMEOUT) return edp_fail(c, EDP_ERR_TIMEOUT, "a bounded device wait gave up");
    if (c->hc->error_flags & EDP_EFLAG_IDS)
        return edp_fail(c, EDP_ERR_CAPACITY, "particle id range used up: born particles were not appended");
    if (c->hc->error_flags & EDP_EFLAG_SEE_MODEL)
        return edp_fail(c, EDP_ERR_STATE, "elastic + inelastic emission coefficients above 1 (secondary emission model)");
    return EDP_OK;
}

int edp_query_emission(edp_ctx* c, int64_t* out)
{
    if (!c || !out) return EDP_ERR_ARG;
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    EDP_CUDA(c, cudaMemcpy(c->hc, c->dc, sizeof(edp_dev_counters), cudaMemcpyDeviceToHost));
    for (int k = 0; k < EDP_N_HIT_COUNTERS; ++k) out[k] = (int64_t)c->hc->e_emit[k];
    return EDP_OK;
}

// the outline surface charge between its fixed-point accumulators (2^32 units per charge) and FP64 node values
__global__ void surf_to_double_kernel(const unsigned long long* s, double* d, int64_t n)
{
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        d[q] = (double)(long long)s[q] * EDP_FIX_INV;
}
__global__ void double_to_surf_kernel(const double* d, unsigned long long* s, int64_t n)
{
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        s[q] = (unsigned long long)__double2ll_rn(d[q] * EDP_FIX_ONE);
}

int edp_get_field(edp_ctx* c, int which, double* out)
{
    if (!c || !out) return EDP_ERR_ARG;
    const int w = ref_width(c);
    const int64_t nref = (int64_t)w * c->kp.nyg;
    double* ref = nullptr;
    EDP_CUDA(c, cudaMalloc(&ref, nref * sizeof(double)));
    const bool mixed = c->p.precision == EDP_PREC_MIXED;
    ++c->launches;
    switch (which) {
    case EDP_FIELD_EX: expand_kernel<<<grid_of(nref), 256, 0, c->stream>>>(c->kp, mixed, c->Ex, c->E2, 0, ref, w); break;
    case EDP_FIELD_EY: expand_kernel<<<grid_of(nref), 256, 0, c->stream>>>(c->kp, mixed, c->Ey, c->E2, 1, ref, w); break;
    case EDP_FIELD_ACC_EX: expand_kernel<<<grid_of(nref), 256, 0, c->stream>>>(c->kp, mixed, c->accx, c->acc2, 0, ref, w); break;
    case EDP_FIELD_ACC_EY: expand_kernel<<<grid_of(nref), 256, 0, c->stream>>>(c->kp, mixed, c->accy, c->acc2, 1, ref, w); break;
    case EDP_FIELD_PHI: expand_kernel<<<grid_of(nref), 256, 0, c->stream>>>(c->kp, 0, c->phi, nullptr, 0, ref, w); break;
    case EDP_FIELD_RHO_TOTAL: expand_kernel<<<grid_of(nref), 256, 0, c->stream>>>(c->kp, 0, c->rho_total, nullptr, 0, ref, w); break;
    case EDP_FIELD_SURFACE_CHARGE:   // dielectrics exist on walled domains only, where the two layouts agree
        if (c->surf) surf_to_double_kernel<<<grid_of(nref), 256, 0, c->stream>>>(c->surf, ref, nref);
        else cudaMemsetAsync(ref, 0, nref * sizeof(double), c->stream);
        break;
    default: cudaFree(ref); return edp_fail(c, EDP_ERR_ARG, "edp_get_field: unknown field");
    }
    EDP_CUDA(c, cudaGetLastError());
    EDP_CUDA(c, cudaMemcpyAsync(out, ref, nref * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(ref);
    return EDP_OK;
}

int edp_set_field(edp_ctx* c, int which, const double* in)
{
    if (!c || !in) return EDP_ERR_ARG;
    const int w = ref_width(c);
    const int64_t nref = (int64_t)w * c->kp.nyg;
    double* ref = nullptr;
    EDP_CUDA(c, cudaMalloc(&ref, nref * sizeof(double)));
    EDP_CUDA(c, cudaMemcpyAsync(ref, in, nref * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const bool mixed = c->p.precision == EDP_PREC_MIXED;
    const int64_t nn = (int64_t)c->kp.nxg * c->kp.nyg;
    ++c->launches;
    switch (which) {
    case EDP_FIELD_EX: contract_kernel<<<grid_of(nn), 256, 0, c->stream>>>(c->kp, mixed, ref, w, c->Ex, c->E2, 0); break;
    case EDP_FIELD_EY: contract_kernel<<<grid_of(nn), 256, 0, c->stream>>>(c->kp, mixed, ref, w, c->Ey, c->E2, 1); break;
    case EDP_FIELD_ACC_EX: contract_kernel<<<grid_of(nn), 256, 0, c->stream>>>(c->kp, mixed, ref, w, c->accx, c->acc2, 0); break;
    case EDP_FIELD_ACC_EY: contract_kernel<<<grid_of(nn), 256, 0, c->stream>>>(c->kp, mixed, ref, w, c->accy, c->acc2, 1); break;
    case EDP_FIELD_PHI: contract_kernel<<<grid_of(nn), 256, 0, c->stream>>>(c->kp, 0, ref, w, c->phi, nullptr, 0); break;
    case EDP_FIELD_RHO_TOTAL: contract_kernel<<<grid_of(nn), 256, 0, c->stream>>>(c->kp, 0, ref, w, c->rho_total, nullptr, 0); break;
    case EDP_FIELD_SURFACE_CHARGE:
        if (!c->surf) {
            cudaFree(ref);
            return edp_fail(c, EDP_ERR_STATE, "edp_set_field: no dielectric inner objects");
        }
        double_to_surf_kernel<<<grid_of(nn), 256, 0, c->stream>>>(ref, c->surf, nn);
        break;
    default: cudaFree(ref); return edp_fail(c, EDP_ERR_ARG, "edp_set_field: unknown field");
    }
    EDP_CUDA(c, cudaGetLastError());
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(ref);
    return EDP_OK;
}

int edp_moments(edp_ctx* c, int sp, double out[7])
{
    if (!c || !out || sp < 0 || sp >= c->nspec) return EDP_ERR_ARG;
    double* d = nullptr;
    EDP_CUDA(c, cudaMalloc(&d, 7 * sizeof(double)));
    EDP_CUDA(c, cudaMemsetAsync(d, 0, 7 * sizeof(double), c->stream));
    ++c->launches;
    moments_kernel<<<grid_of(c->host_slots[sp]), 256, 0, c->stream>>>(c->p.precision, c->pm[sp], c->pd[sp],
                                                                       &c->dc->n_slots[sp], d);
    EDP_CUDA(c, cudaGetLastError());
    EDP_CUDA(c, cudaMemcpyAsync(out, d, 7 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(d);
    return EDP_OK;
}

int edp_mcc_choose(edp_ctx* c, int64_t n, const double* E, const double* r, int32_t* out)
{
    if (!c || n < 0 || (n && (!E || !r || !out))) return EDP_ERR_ARG;
    if (!c->tab.en_on) return edp_fail(c, EDP_ERR_STATE, "no electron-neutral collisions configured");
    if (n == 0) return EDP_OK;
    double *dE = nullptr, *dr = nullptr;
    int32_t* dout = nullptr;
    EDP_CUDA(c, cudaMalloc(&dE, n * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&dr, n * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&dout, n * sizeof(int32_t)));
    EDP_CUDA(c, cudaMemcpyAsync(dE, E, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    EDP_CUDA(c, cudaMemcpyAsync(dr, r, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ++c->launches;
    mcc_choose_kernel<<<grid_of(n), 256, 0, c->stream>>>(edp_make_mcc_dev(c), n, dE, dr, dout);
    EDP_CUDA(c, cudaGetLastError());
    EDP_CUDA(c, cudaMemcpyAsync(out, dout, n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(dE);
    cudaFree(dr);
    cudaFree(dout);
    return EDP_OK;
}

}  // extern "C"
