// Field part of the cycle:
//  density   the deposit (fixed point or FP64) -> rho = (sum_s Qs rho_s - rho_e)/N_ppc with the wall factors
//            of GATHER_ELECTRON_CHARGE_DENSITY (pic2d_ElectronDynamics.f90:1802-1880) and the combination of
//            SOLVE_POISSON_FFTX_LINSYSY (pic2d_ElectricFieldCalc_FFT_X.f90:72-85)
//  FFT_X     SOLVE_POISSON_FFTX_LINSYSY (:3-1320): real FFT of every row along x, per-mode tridiagonal solve
//            along y with the spectral diagonal -2 - 4 pi^2 n^2/N^2 and a_eq of PREPARE_SYS_Y
//            (pic2d_Prepare_FFTX_SYSY.f90:826-899), inverse FFT. The row transforms are radix-2 in shared
//            memory, one CTA per row; the Thomas sweeps run one thread per mode with coalesced rows.
//  E         CALCULATE_ELECTRIC_FIELD_FFTX_LINSYSY (:1324-1547) / CALCULATE_ELECTRIC_FIELD
//            (pic2d_ElectricFieldCalc_PETSc.F90:360-805), acc_E += E
//  CG        replacement of SOLVE_POTENTIAL_WITH_PETSC (pic2d_ElectricFieldCalc_PETSc.F90:7-355) on the operator of
//            SolverInitialization (pic2d_PETSc_Solver.F90:42-1350) with Dirichlet nodes eliminated, FP64 dots.
#include <cmath>
#include <vector>

#include <chrono>

#include "edp_internal.cuh"

namespace {

__global__ void density_kernel(edp_kparams kp, int precision, int nion, const unsigned long long* const* rho_fix,
                               const double* const* rho_d, const double* qs, double factor_rho,
                               const unsigned long long* surf, double* out)
{
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(q % kp.nxg), j = (int)(q / kp.nxg);
        double re, ri = 0.0;
        if (precision == EDP_PREC_MIXED) {
            re = (double)(long long)rho_fix[0][q] * EDP_FIX_INV;
            for (int s = 0; s < nion; ++s) ri += qs[s] * ((double)(long long)rho_fix[1 + s][q] * EDP_FIX_INV);
        } else {
            re = rho_d[0][q];
            for (int s = 0; s < nion; ++s) ri += qs[s] * rho_d[1 + s][q];
        }
        double f = 1.0;
        if (kp.periodic) {
            if (j == 0 || j == kp.ncy) f = 2.0;
        } else {
            bool ex = (i == 0 || i == kp.ncx), ey = (j == 0 || j == kp.ncy);
            f = (ex && ey) ? 4.0 : ((ex || ey) ? 2.0 : 1.0);
        }
        double v = (ri * f) - (re * f);
        // the surface charge of the dielectric outlines, subtracted from rho_e (pic2d_ElectronDynamics.f90:1903-1909)
        if (surf) v += (double)(long long)surf[q] * EDP_FIX_INV;
        out[q] = factor_rho * v;
    }
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// in-place radix-2 DIT FFT of N complex values already stored in bit-reversed order; sign +1 uses tw, -1 conj(tw)
__device__ void smem_fft(double2* x, int N, const double2* __restrict__ tw, int sign)
{
    for (int len = 2; len <= N; len <<= 1) {
        const int half = len >> 1, stride = N / len;
        for (int b = threadIdx.x; b < N / 2; b += blockDim.x) {
            int grp = b / half, k = b - grp * half;
            int a = grp * len + k, c = a + half;
            double2 w = __ldg(&tw[k * stride]);
            if (sign < 0) w.y = -w.y;
            double2 t = cmul(w, x[c]);
            double2 u = x[a];
            x[a] = make_double2(u.x + t.x, u.y + t.y);
            x[c] = make_double2(u.x - t.x, u.y - t.y);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int bitrev(int v, int logn) { return (int)(__brev((unsigned)v) >> (32 - logn)); }

__global__ void fftx_forward(edp_kparams kp, const double* __restrict__ rho, double phi_bottom, double phi_top,
                             const double2* __restrict__ tw, int logn, int nm, double2* __restrict__ spec)
{
    extern __shared__ double2 x[];
    const int N = kp.ncx, j = blockIdx.x;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double v = rho[(int64_t)j * kp.nxg + i];
        if (j == 0) v = phi_bottom;
        if (j == kp.ncy) v = phi_top;
        x[bitrev(i, logn)] = make_double2(v, 0.0);
    }
    __syncthreads();
    smem_fft(x, N, tw, +1);
    for (int m = threadIdx.x; m < nm; m += blockDim.x) {
        double2 v = x[m];
        if (m == 0 || m == N / 2) v.y = 0.0;
        spec[(int64_t)j * nm + m] = v;
    }
}

// SOLVE_POISSON_FFTX_LINSYSY :690-756 for metal walls (a_eq(0) = a_eq(J) = 0). The forward sweep
//   rr(j) = (-y(j) - rr(j-1)) a(j),  j = 1..J-1,  rr(0) = y(0)
// and the back substitution phi(j) = rr(j) - a(j) phi(j+1), phi(J) = y(J), are first-order affine recurrences.
// The interior rows of a mode are cut into kTmSegs segments. A thread composes the maps of its segment, the
// compositions are scanned over the segments (shuffles inside a warp, shared memory across the warps), and the
// thread re-sweeps its rows from its incoming value. Same recurrence, reassociated. A warp holds 8 consecutive
// modes x 4 segments (lane = 8 segment + mode), so every row is read and written as 128 contiguous bytes.
struct Aff {   // x -> c + b x, complex c, real b
    double cx, cy, b;
};

__device__ __forceinline__ Aff aff_after(const Aff& late, const Aff& early)   // late o early
{
    return Aff{late.cx + late.b * early.cx, late.cy + late.b * early.cy, late.b * early.b};
}

__device__ __forceinline__ Aff shfl_aff(const Aff& a, bool up, int off)
{
    Aff r;
    r.cx = up ? __shfl_up_sync(0xFFFFFFFFu, a.cx, off) : __shfl_down_sync(0xFFFFFFFFu, a.cx, off);
    r.cy = up ? __shfl_up_sync(0xFFFFFFFFu, a.cy, off) : __shfl_down_sync(0xFFFFFFFFu, a.cy, off);
    r.b = up ? __shfl_up_sync(0xFFFFFFFFu, a.b, off) : __shfl_down_sync(0xFFFFFFFFu, a.b, off);
    return r;
}

constexpr int kTmModes = 8, kTmWarps = 16, kTmSegs = 4 * kTmWarps;

__global__ void __launch_bounds__(32 * kTmWarps) fftx_thomas(int J, int nm, const double* __restrict__ aeq,
                                                             double2* __restrict__ spec)
{
    __shared__ Aff part[kTmWarps][kTmModes];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ml = lane & 7, sw = lane >> 3;
    const int m = blockIdx.x * kTmModes + ml;
    const bool active = m < nm;
    const int mm = active ? m : nm - 1;   // lanes past the last mode shadow it without storing
    const int seg = 4 * w + sw;
    const int per = (J - 1 + kTmSegs - 1) / kTmSegs;
    const int j0 = 1 + seg * per, j1 = min(j0 + per, J);   // interior rows [j0, j1) of this segment
    // ---- forward sweep
    Aff f{0.0, 0.0, 1.0};
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
        const double a = aeq[(int64_t)j * nm + mm];
        const double2 y = spec[(int64_t)j * nm + mm];
        f = aff_after(Aff{-a * y.x, -a * y.y, -a}, f);
    }
    for (int off = 8; off < 32; off <<= 1) {   // inclusive over the warp's segments, earliest first
        Aff p = shfl_aff(f, true, off);
        if (lane >= off) f = aff_after(f, p);
    }
    if (sw == 3) part[w][ml] = f;
    __syncthreads();
    Aff inc{0.0, 0.0, 1.0};
    for (int q = 0; q < w; ++q) inc = aff_after(part[q][ml], inc);
    Aff ex = shfl_aff(f, true, 8);
    if (sw > 0) inc = aff_after(ex, inc);
    const double2 rr0 = spec[mm];   // transformed wall row
    double2 prev = make_double2(inc.cx + inc.b * rr0.x, inc.cy + inc.b * rr0.y);
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
        const double a = aeq[(int64_t)j * nm + mm];
        const double2 y = spec[(int64_t)j * nm + mm];
        prev = make_double2((-y.x - prev.x) * a, (-y.y - prev.y) * a);
        if (active) spec[(int64_t)j * nm + mm] = prev;
    }
    // ---- back substitution, segments composed from the top
    Aff g{0.0, 0.0, 1.0};
#pragma unroll 4
    for (int j = j1 - 1; j >= j0; --j) {
        const double a = aeq[(int64_t)j * nm + mm];
        const double2 r = spec[(int64_t)j * nm + mm];
        g = aff_after(Aff{r.x, r.y, -a}, g);
    }
    for (int off = 8; off < 32; off <<= 1) {   // inclusive over the warp's segments, latest first
        Aff p = shfl_aff(g, false, off);
        if (lane + off < 32) g = aff_after(g, p);
    }
    __syncthreads();   // every thread has read the forward totals
    if (sw == 0) part[w][ml] = g;
    __syncthreads();
    Aff inb{0.0, 0.0, 1.0};
    for (int q = kTmWarps - 1; q > w; --q) inb = aff_after(part[q][ml], inb);
    Aff ey = shfl_aff(g, false, 8);
    if (sw < 3) inb = aff_after(ey, inb);
    const double2 phiJ = spec[(int64_t)J * nm + mm];
    double2 next = make_double2(inb.cx + inb.b * phiJ.x, inb.cy + inb.b * phiJ.y);
#pragma unroll 4
    for (int j = j1 - 1; j >= j0; --j) {
        const double a = aeq[(int64_t)j * nm + mm];
        const double2 r = spec[(int64_t)j * nm + mm];
        next = make_double2(r.x - a * next.x, r.y - a * next.y);
        if (active) spec[(int64_t)j * nm + mm] = next;
    }
    // row 0 keeps rr(0) = phi(0) since a_eq(0) = 0
}

__global__ void fftx_inverse(edp_kparams kp, const double2* __restrict__ spec, const double2* __restrict__ tw, int logn,
                             int nm, double* __restrict__ phi)
{
    extern __shared__ double2 x[];
    const int N = kp.ncx, j = blockIdx.x;
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        double2 v;
        if (m < nm) v = spec[(int64_t)j * nm + m];
        else {
            v = spec[(int64_t)j * nm + (N - m)];
            v.y = -v.y;
        }
        x[bitrev(m, logn)] = v;
    }
    __syncthreads();
    smem_fft(x, N, tw, -1);
    const double inv = 1.0 / N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) phi[(int64_t)j * kp.nxg + i] = x[i].x * inv;
}

__global__ void efield_kernel(edp_kparams kp, const double* __restrict__ phi, double f2, double f1, int precision,
                              float2* E2, float2* acc2, double* Ex, double* Ey, double* accx, double* accy)
{
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    const int J = kp.ncy;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(q % kp.nxg), j = (int)(q / kp.nxg);
        auto P = [&](int ii, int jj) { return phi[(int64_t)jj * kp.nxg + ii]; };
        double ex, ey;
        if (kp.periodic) {
            int im = i == 0 ? kp.ncx - 1 : i - 1, ip = i == kp.ncx - 1 ? 0 : i + 1;
            ex = f2 * (P(im, j) - P(ip, j));
        } else {
            if (i == 0) ex = f1 * (P(0, j) - P(1, j));
            else if (i == kp.ncx) ex = f1 * (P(kp.ncx - 1, j) - P(kp.ncx, j));
            else ex = f2 * (P(i - 1, j) - P(i + 1, j));
        }
        if (j == 0) ey = f1 * (P(i, 0) - P(i, 1));
        else if (j == J) ey = f1 * (P(i, J - 1) - P(i, J));
        else ey = f2 * (P(i, j - 1) - P(i, j + 1));
        if (precision == EDP_PREC_MIXED) {
            E2[q] = make_float2((float)ex, (float)ey);
            float2 a = acc2[q];
            acc2[q] = make_float2(a.x + (float)ex, a.y + (float)ey);
        } else {
            Ex[q] = ex;
            Ey[q] = ey;
            accx[q] += ex;
            accy[q] += ey;
        }
    }
}

// ------------------------------------------------------------------------------------------ CG
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    return v;
}

struct CgGeom {
    edp_kparams kp;
    double wall[4];
    double inner[EDP_MAX_INNER];
    const double *epsx, *epsy;   // face permittivities, or null (vacuum everywhere)
};

// 1 for a Dirichlet node (walls and metal inner objects, value in *val); the nodes of dielectric objects are unknowns
__device__ __forceinline__ int cg_node_kind(const CgGeom& g, int i, int j, double* val)
{
    const edp_kparams& kp = g.kp;
    for (int n = 0; n < kp.n_inner; ++n)
        if (!((kp.diel_mask >> n) & 1) && i >= kp.ileft[n] && i <= kp.iright[n] && j >= kp.jbottom[n] &&
            j <= kp.jtop[n]) {
            *val = g.inner[n];
            return 1;
        }
    if (j == 0) { *val = g.wall[0]; return 1; }
    if (j == kp.ncy) { *val = g.wall[1]; return 1; }
    if (i == 0) { *val = g.wall[2]; return 1; }
    if (i == kp.ncx) { *val = g.wall[3]; return 1; }
    return 0;
}

// Dirichlet values, RHS with eliminated neighbours, initial guess; accumulates |b|^2
__global__ void cg_setup(CgGeom g, const double* __restrict__ rho, int warm, const double* __restrict__ x0,
                         int8_t* kind, double* phi, double* b, double* scal)
{
    const edp_kparams& kp = g.kp;
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    double acc = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(q % kp.nxg), j = (int)(q / kp.nxg);
        double v;
        int k = cg_node_kind(g, i, j, &v);
        kind[q] = (int8_t)k;
        if (k) {
            phi[q] = v;
            b[q] = 0.0;
            continue;
        }
        double s = rho[q], d;
        const int64_t w = kp.nxg;
        const bool e = g.epsx != nullptr;
        if (cg_node_kind(g, i - 1, j, &d)) s += (e ? g.epsx[q] : 1.0) * d;
        if (cg_node_kind(g, i + 1, j, &d)) s += (e ? g.epsx[q + 1] : 1.0) * d;
        if (cg_node_kind(g, i, j - 1, &d)) s += (e ? g.epsy[q] : 1.0) * d;
        if (cg_node_kind(g, i, j + 1, &d)) s += (e ? g.epsy[q + w] : 1.0) * d;
        b[q] = s;
        phi[q] = (warm == EDP_WARM_ZERO) ? 0.0 : x0[q];
        acc += s * s;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(&scal[0], acc);
}

// the operator of SolverInitialization (pic2d_PETSc_Solver.F90:311-..., sign reversed): sum over the four faces of
// eps_face (v_q - v_neighbour), Dirichlet neighbours moved to the right-hand side; eps = 1 without dielectrics
__device__ __forceinline__ double apply_A(const edp_kparams& kp, const int8_t* kind, const double* v, int64_t q,
                                          const double* ex, const double* ey)
{
    const int64_t w = kp.nxg;
    if (ex) {
        const double cw = ex[q], ce = ex[q + 1], cs = ey[q], cn = ey[q + w];
        double s = (cw + ce + cs + cn) * v[q];
        if (!kind[q - 1]) s -= cw * v[q - 1];
        if (!kind[q + 1]) s -= ce * v[q + 1];
        if (!kind[q - w]) s -= cs * v[q - w];
        if (!kind[q + w]) s -= cn * v[q + w];
        return s;
    }
    double s = 4.0 * v[q];
    if (!kind[q - 1]) s -= v[q - 1];
    if (!kind[q + 1]) s -= v[q + 1];
    if (!kind[q - w]) s -= v[q - w];
    if (!kind[q + w]) s -= v[q + w];
    return s;
}

// r = b - A x, p = r, rr accumulated
__global__ void cg_residual(edp_kparams kp, const int8_t* kind, const double* x, const double* b, double* r, double* p,
                            double* rr, const double* ex, const double* ey)
{
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    double acc = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        if (kind[q]) {
            r[q] = 0.0;
            p[q] = 0.0;
            continue;
        }
        double v = b[q] - apply_A(kp, kind, x, q, ex, ey);
        r[q] = v;
        p[q] = v;
        acc += v * v;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(rr, acc);
}

__global__ void cg_spmv(edp_kparams kp, const int8_t* kind, const double* p, double* Ap, double* pAp, const double* ex,
                        const double* ey)
{
    edp_dependent_start();
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    double acc = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        if (kind[q]) {
            Ap[q] = 0.0;
            continue;
        }
        double v = apply_A(kp, kind, p, q, ex, ey);
        Ap[q] = v;
        acc += p[q] * v;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(pAp, acc);
}

__global__ void cg_update(edp_kparams kp, const int8_t* kind, const double* rr, const double* pAp, const double* p,
                          const double* Ap, double* x, double* r, double* rr_new)
{
    edp_dependent_start();
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    const double alpha = *rr / *pAp;
    double acc = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        if (kind[q]) continue;
        x[q] += alpha * p[q];
        double v = r[q] - alpha * Ap[q];
        r[q] = v;
        acc += v * v;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(rr_new, acc);
}

// sum of a.b over the unknown nodes
__global__ void pcg_dot(edp_kparams kp, const int8_t* kind, const double* a, const double* b, double* out)
{
    edp_dependent_start();
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    double acc = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        if (!kind[q]) acc += a[q] * b[q];
    acc = block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(out, acc);
}

// p = z + (rz / rz_old) p; rz_old == nullptr starts a new direction sequence (p = z)
__global__ void pcg_direction(edp_kparams kp, const int8_t* kind, const double* rz, const double* rz_old,
                              const double* z, double* p)
{
    edp_dependent_start();
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    const double beta = rz_old ? *rz / *rz_old : 0.0;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        p[q] = kind[q] ? 0.0 : z[q] + beta * p[q];
}

unsigned grid_nodes(const edp_kparams& kp)
{
    int64_t n = (int64_t)kp.nxg * kp.nyg;
    int64_t g = (n + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace

int edp_fields_prepare(edp_ctx* c)
{
    if (c->p.solver != EDP_SOLVER_FFTX) return EDP_OK;
    const int N = c->p.ncx, J = c->p.ncy;
    c->nm = N / 2 + 1;
    std::vector<double2> tw(N / 2);
    const double PI = 3.141592653589793;
    for (int k = 0; k < N / 2; ++k) tw[k] = make_double2(std::cos(2.0 * PI * k / N), std::sin(2.0 * PI * k / N));
    // a_eq of PREPARE_SYS_Y (pic2d_Prepare_FFTX_SYSY.f90:834-899) for metal walls, layout [j][n]
    std::vector<double> a((size_t)(J + 1) * c->nm);
    for (int m = 0; m < c->nm; ++m) {
        double d = -2.0 - 4.0 * PI * PI * (double)m * (double)m / ((double)N * (double)N);
        a[m] = 0.0;
        for (int j = 1; j <= J - 1; ++j) a[(size_t)j * c->nm + m] = 1.0 / (d - a[(size_t)(j - 1) * c->nm + m]);
        a[(size_t)J * c->nm + m] = 0.0;
    }
    EDP_CUDA(c, cudaMalloc(&c->twiddle, tw.size() * sizeof(double2)));
    EDP_CUDA(c, cudaMalloc(&c->aeq, a.size() * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&c->spec, (size_t)(J + 1) * c->nm * sizeof(double2)));
    EDP_CUDA(c, cudaMemcpy(c->twiddle, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice));
    EDP_CUDA(c, cudaMemcpy(c->aeq, a.data(), a.size() * sizeof(double), cudaMemcpyHostToDevice));
    size_t smem = (size_t)N * sizeof(double2);
    if (smem > 48 * 1024) {
        TRY(edp_raise_smem_limit(c, (const void*)fftx_forward, smem));
        TRY(edp_raise_smem_limit(c, (const void*)fftx_inverse, smem));
    }
    return EDP_OK;
}

// SET_EPS_ISHIFTED / SET_EPS_JSHIFTED (pic2d_PETSc_Solver.F90:1724-2045): the permittivity of the face between nodes
// (i-1, j) and (i, j) (xface) or (i, j-1) and (i, j). A face inside a dielectric takes its eps; a face on the outline
// of one or two dielectrics averages them with vacuum, or with each other; a face inside a metal object, or on the
// outline of two, is 0; a face on one metal outline takes the dielectric average or 1.
static double face_eps(const edp_params& p, int i, int j, bool xface)
{
    auto covers = [&](int n) {
        if (xface)
            return i - 1 >= p.inner_ileft[n] && i - 1 <= p.inner_iright[n] && j >= p.inner_jbottom[n] &&
                   j <= p.inner_jtop[n] && i <= p.inner_iright[n];
        return i >= p.inner_ileft[n] && i <= p.inner_iright[n] && j - 1 >= p.inner_jbottom[n] &&
               j - 1 <= p.inner_jtop[n] && j <= p.inner_jtop[n];
    };
    auto on_outline = [&](int n) {
        return xface ? (j == p.inner_jtop[n] || j == p.inner_jbottom[n])
                     : (i == p.inner_ileft[n] || i == p.inner_iright[n]);
    };
    double eps = 0.0;
    int count = 0;
    bool inside = false;
    for (int n = 0; n < p.n_inner; ++n) {
        if (!(p.inner_eps[n] > 0.0) || !covers(n)) continue;
        if (on_outline(n)) {
            ++count;
            eps += p.inner_eps[n];
        } else {
            inside = true;
            eps = p.inner_eps[n];
            count = 1;
            break;
        }
    }
    bool on_metal = false;
    for (int n = 0; n < p.n_inner; ++n) {
        if (p.inner_eps[n] > 0.0 || !covers(n)) continue;
        if (!on_outline(n) || on_metal) return 0.0;
        on_metal = true;
    }
    if (on_metal) return count == 0 ? 1.0 : eps / count;
    if (count == 0) return 1.0;
    if (count == 1) return inside ? eps : (1.0 + eps) / 2.0;
    return eps / (double)count;   // two outlines meet (three cannot on non-overlapping rectangles)
}

int edp_dielectrics_setup(edp_ctx* c)
{
    const edp_kparams& kp = c->kp;
    const int64_t nn = (int64_t)kp.nxg * kp.nyg;
    std::vector<double> ex(nn, 1.0), ey(nn, 1.0);
    for (int j = 0; j <= c->p.ncy; ++j)
        for (int i = 0; i < kp.nxg; ++i) {
            if (i >= 1) ex[(int64_t)j * kp.nxg + i] = face_eps(c->p, i, j, true);
            if (j >= 1) ey[(int64_t)j * kp.nxg + i] = face_eps(c->p, i, j, false);
        }
    EDP_CUDA(c, cudaMalloc(&c->epsx, nn * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&c->epsy, nn * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&c->surf, nn * sizeof(unsigned long long)));
    EDP_CUDA(c, cudaMemcpy(c->epsx, ex.data(), nn * sizeof(double), cudaMemcpyHostToDevice));
    EDP_CUDA(c, cudaMemcpy(c->epsy, ey.data(), nn * sizeof(double), cudaMemcpyHostToDevice));
    EDP_CUDA(c, cudaMemset(c->surf, 0, nn * sizeof(unsigned long long)));
    return EDP_OK;
}

int edp_launch_density(edp_ctx* c)
{
    struct Ptrs {
        const unsigned long long* f[EDP_MAX_SPECIES];
        const double* d[EDP_MAX_SPECIES];
        double qs[EDP_MAX_ION_SPECIES];
    } h;
    for (int s = 0; s < EDP_MAX_SPECIES; ++s) {
        h.f[s] = c->rho_fix[s];
        h.d[s] = c->rho_d[s];
    }
    for (int s = 0; s < EDP_MAX_ION_SPECIES; ++s) h.qs[s] = (double)c->p.ion_charge[s];
    static_assert(sizeof(Ptrs) <= 4096, "pointer table");
    Ptrs* d = reinterpret_cast<Ptrs*>(c->dev_small);
    EDP_CUDA(c, cudaMemcpyAsync(d, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
    ++c->launches;
    density_kernel<<<grid_nodes(c->kp), 256, 0, c->stream>>>(c->kp, c->p.precision, c->p.n_ion_species, d->f, d->d,
                                                             d->qs, 1.0 / c->p.n_of_particles_cell, c->surf,
                                                             c->rho_total);
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

int edp_launch_fftx(edp_ctx* c)
{
    const int N = c->p.ncx;
    int logn = 0;
    while ((1 << logn) < N) ++logn;
    size_t smem = (size_t)N * sizeof(double2);
    int thr = std::min(128, std::max(32, N / 2));   // 8 rows of 1024 in flight per SM: one wave at 1025 rows
    ++c->launches;
    fftx_forward<<<c->kp.nyg, thr, smem, c->stream>>>(c->kp, c->rho_total, c->phi_wall[0], c->phi_wall[1], c->twiddle,
                                                     logn, c->nm, c->spec);
    ++c->launches;
    fftx_thomas<<<(c->nm + kTmModes - 1) / kTmModes, 32 * kTmWarps, 0, c->stream>>>(c->p.ncy, c->nm, c->aeq, c->spec);
    ++c->launches;
    fftx_inverse<<<c->kp.nyg, thr, smem, c->stream>>>(c->kp, c->spec, c->twiddle, logn, c->nm, c->phi);
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

int edp_launch_efield(edp_ctx* c)
{
    const double f2 = c->p.f_scale_v / (c->p.e_scale_vm * 2.0 * c->p.delta_x_m);
    const double f1 = c->p.f_scale_v / (c->p.e_scale_vm * c->p.delta_x_m);
    ++c->launches;
    efield_kernel<<<grid_nodes(c->kp), 256, 0, c->stream>>>(c->kp, c->phi, f2, f1, c->p.precision, c->E2, c->acc2,
                                                            c->Ex, c->Ey, c->accx, c->accy);
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

// Iterations k0 .. k0+n-1 of (preconditioned) CG, launched on the context's stream with no host synchronisation,
// so that a whole block can be captured as a graph. Block b = k0 / check accumulates its scalars in area b & 1 (zeroed
// first): r.z of iteration j of the block at 4j, p.Ap at 4j+1, r.r after it at 4j+2. Values of the previous block
// are read from the other area, which this block does not touch; r.r before iteration 0 is scalar [1].
static int cg_block(edp_ctx* c, const CgGeom& g, bool mg, int k0, int n, int check)
{
    const edp_kparams& kp = g.kp;
    const unsigned gr = grid_nodes(kp);
    double* S = c->cg_sc;
    double* A = S + 2 + ((k0 / check) & 1) * EDP_CG_AREA;
    double* P = S + 2 + (((k0 / check) + 1) & 1) * EDP_CG_AREA;
    EDP_CUDA(c, cudaMemsetAsync(A, 0, 4 * check * sizeof(double), c->stream));
    // r.r after iteration m (m >= 0) of the solve, for m in this block or the previous one
    auto rr_after = [&](int m) { return m >= k0 ? A + 4 * (m - k0) + 2 : P + 4 * (m - (k0 - check)) + 2; };
    auto rr_before = [&](int k) { return k == 0 ? S + 1 : rr_after(k - 1); };
    for (int j = 0; j < n; ++j) {
        const int k = k0 + j;
        double* rz = A + 4 * j;
        double* pAp = A + 4 * j + 1;
        if (mg) {
            TRY(edp_mg_apply(c, c->cg_r, c->cg_z));
            ++c->launches;
            EDP_CUDA(c, edp_launch_dependent(pcg_dot, dim3(gr), dim3(256), 0, c->stream, kp, (const int8_t*)c->cg_kind,
                                              (const double*)c->cg_r, (const double*)c->cg_z, rz));
            const double* rz_prev = k == 0 ? nullptr : (j ? A + 4 * (j - 1) : P + 4 * (check - 1));
            ++c->launches;
            EDP_CUDA(c, edp_launch_dependent(pcg_direction, dim3(gr), dim3(256), 0, c->stream, kp, (const int8_t*)c->cg_kind,
                                              (const double*)rz, rz_prev, (const double*)c->cg_z, c->cg_p));
        } else {
            rz = rr_before(k);
            if (k) {
                ++c->launches;
                EDP_CUDA(c, edp_launch_dependent(pcg_direction, dim3(gr), dim3(256), 0, c->stream, kp,
                                                  (const int8_t*)c->cg_kind, (const double*)rz,
                                                  (const double*)rr_before(k - 1), (const double*)c->cg_r, c->cg_p));
            }
        }
        ++c->launches;
        EDP_CUDA(c, edp_launch_dependent(cg_spmv, dim3(gr), dim3(256), 0, c->stream, kp, (const int8_t*)c->cg_kind,
                                          (const double*)c->cg_p, c->cg_Ap, pAp, g.epsx, g.epsy));
        ++c->launches;
        EDP_CUDA(c, edp_launch_dependent(cg_update, dim3(gr), dim3(256), 0, c->stream, kp, (const int8_t*)c->cg_kind,
                                          (const double*)rz, (const double*)pAp, (const double*)c->cg_p,
                                          (const double*)c->cg_Ap, c->phi, c->cg_r, A + 4 * j + 2));
    }
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

int edp_launch_cg(edp_ctx* c, double rtol, int max_it, int warm, int* iters)
{
    const edp_kparams& kp = c->kp;
    const bool mg = c->precond == EDP_PRECOND_MG && c->mg_nlev > 0;
    CgGeom g;
    g.kp = kp;
    for (int s = 0; s < 4; ++s) g.wall[s] = c->phi_wall[s];
    for (int n = 0; n < EDP_MAX_INNER; ++n) g.inner[n] = c->phi_inner[n];
    g.epsx = c->epsx;
    g.epsy = c->epsy;
    // scalars: [0] |b|^2, [1] r.r before iteration 0, then the two block areas (cg_block)
    double* scal = c->cg_sc;
    EDP_CUDA(c, cudaMemsetAsync(scal, 0, 2 * sizeof(double), c->stream));
    const unsigned gr = grid_nodes(kp);
    // the network was trained on the vacuum operator: with dielectric objects the previous potential starts the solve
    if (warm == EDP_WARM_LEARNED && kp.diel_mask) warm = EDP_WARM_PREVIOUS;
    const bool asked = warm == EDP_WARM_LEARNED;
    if (asked && !c->ws) return edp_fail(c, EDP_ERR_STATE, "no warm-start network loaded");
    // the network runs unless the solves it started were slower on average than those from the previous potential
    // (then only every 64th call re-tries it); the first call (which may also capture the CG graphs) is not timed,
    // the second times the network's start and the third the previous potential's
    bool learned = false;
    int64_t k_call = -1;
    if (asked) {
        k_call = c->ws_calls++;
        if (k_call < 2) learned = true;
        else if (k_call == 2) learned = false;
        else learned = c->ws_t_net < c->ws_t_prev || k_call % 64 == 0;
        if (learned) ++c->ws_runs;
    }
    const auto t_start = std::chrono::steady_clock::now();
    ++c->launches;
    cg_setup<<<gr, 256, 0, c->stream>>>(g, c->rho_total, warm, c->phi, c->cg_kind, c->phi, c->cg_b, scal);
    ++c->launches;
    cg_residual<<<gr, 256, 0, c->stream>>>(kp, c->cg_kind, c->phi, c->cg_b, c->cg_r, c->cg_p, &scal[1],
                                           c->epsx, c->epsy);
    if (learned) {
        TRY(edp_warmstart_forward(c, &scal[1]));
        TRY(edp_warmstart_residual(c));
    }
    double h[3] = {0.0, 0.0, 0.0};
    EDP_CUDA(c, cudaMemcpyAsync(h, scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (learned) EDP_CUDA(c, cudaMemcpyAsync(h + 2, edp_warmstart_rr(c), sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    double bn = std::sqrt(h[0]);
    if (bn == 0.0) bn = 1.0;
    double rel = std::sqrt(h[1]) / bn;
    c->last_ws_used = 0;
    if (learned && h[2] < h[1]) {   // the network's guess has the smaller residual: start from it
        EDP_CUDA(c, edp_warmstart_accept(c, &scal[1]));
        rel = std::sqrt(h[2]) / bn;
        c->last_ws_used = 1;
    }
    c->last_cg_relres0 = rel;
    int it = 0, done_at = rel <= rtol ? 0 : -1;
    const int check = mg ? EDP_CG_CHECK_MG : EDP_CG_CHECK_PLAIN;
    std::vector<double> blk(4 * check);
    while (done_at < 0 && it < max_it) {
        const int n = std::min(max_it - it, check);
        double* area = scal + 2 + ((it / check) & 1) * EDP_CG_AREA;
        if (n == check) {   // a whole block: replayed from its captured graph
            const int which = it == 0 ? 0 : 1 + ((it / check) & 1);
            cudaGraphExec_t& ex = c->cg_exec[mg][which];
            if (!ex) {
                const int64_t l0 = c->launches;
                EDP_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                const int e = cg_block(c, g, mg, it, check, check);
                cudaGraph_t graph = nullptr;
                const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
                if (e != EDP_OK) {
                    if (graph) cudaGraphDestroy(graph);
                    return e;
                }
                EDP_CUDA(c, ce);
                const cudaError_t ie = cudaGraphInstantiate(&ex, graph, 0);
                cudaGraphDestroy(graph);
                EDP_CUDA(c, ie);
                c->cg_exec_launches[mg][which] = c->launches - l0;
                c->launches = l0;
            }
            EDP_CUDA(c, cudaGraphLaunch(ex, c->stream));
            c->launches += c->cg_exec_launches[mg][which];
        } else {
            TRY(cg_block(c, g, mg, it, n, check));
        }
        // residual norms after iterations it+1 .. it+n; the iteration count is the first that met rtol
        EDP_CUDA(c, cudaMemcpyAsync(blk.data(), area, 4 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        EDP_CUDA(c, cudaStreamSynchronize(c->stream));
        for (int j = 0; j < n && done_at < 0; ++j)
            if (std::sqrt(blk[4 * j + 2]) / bn <= rtol) done_at = it + j + 1;
        rel = std::sqrt(blk[4 * (n - 1) + 2]) / bn;   // the solution carries the whole block
        it += n;
    }
    EDP_CUDA(c, cudaGetLastError());
    const int reported = done_at >= 0 ? done_at : it;
    c->last_cg_iters = reported;
    c->last_cg_relres = rel;
    if (iters) *iters = reported;
    if (asked && k_call > 0) {   // the solve's wall time (it ends synchronised) into the running average of its start
        const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        double& avg = learned ? c->ws_t_net : c->ws_t_prev;
        avg = avg < 0.0 ? t : 0.75 * avg + 0.25 * t;
    }
    return done_at >= 0 ? EDP_OK : edp_fail(c, EDP_ERR_NOT_CONVERGED, "CG did not converge within max_it");
}

extern "C" int edp_warmstart_timing(edp_ctx* c, double* out)
{
    if (!c || !out) return EDP_ERR_ARG;
    out[0] = c->ws_t_net;
    out[1] = c->ws_t_prev;
    out[2] = (double)c->ws_calls;
    out[3] = (double)c->ws_runs;
    return EDP_OK;
}

// The network's guess for the current density without solving: guess_out (node layout) and the residual norms of
// the previous potential and of the guess. The potential itself is left unchanged.
extern "C" int edp_warmstart_predict(edp_ctx* c, double* guess_out, double* res_out)
{
    if (!c || !guess_out || !res_out) return EDP_ERR_ARG;
    if (c->p.solver != EDP_SOLVER_CG) return edp_fail(c, EDP_ERR_STATE, "context was not set up for CG");
    if (!c->ws) return edp_fail(c, EDP_ERR_STATE, "no warm-start network loaded");
    TRY(edp_launch_density(c));
    const edp_kparams& kp = c->kp;
    CgGeom g;
    g.kp = kp;
    for (int s = 0; s < 4; ++s) g.wall[s] = c->phi_wall[s];
    for (int n = 0; n < EDP_MAX_INNER; ++n) g.inner[n] = c->phi_inner[n];
    g.epsx = c->epsx;
    g.epsy = c->epsy;
    double* scal = nullptr;
    EDP_CUDA(c, cudaMallocAsync(&scal, 2 * sizeof(double), c->stream));
    EDP_CUDA(c, cudaMemsetAsync(scal, 0, 2 * sizeof(double), c->stream));
    const unsigned gr = grid_nodes(kp);
    c->launches += 2;
    cg_setup<<<gr, 256, 0, c->stream>>>(g, c->rho_total, EDP_WARM_PREVIOUS, c->phi, c->cg_kind, c->phi, c->cg_b, scal);
    cg_residual<<<gr, 256, 0, c->stream>>>(kp, c->cg_kind, c->phi, c->cg_b, c->cg_r, c->cg_p, &scal[1],
                                           c->epsx, c->epsy);
    TRY(edp_warmstart_forward(c, &scal[1]));
    TRY(edp_warmstart_residual(c));
    double h[2];
    EDP_CUDA(c, cudaMemcpyAsync(&h[0], &scal[1], sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaMemcpyAsync(&h[1], edp_warmstart_rr(c), sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    const size_t nb = (size_t)kp.nxg * kp.nyg * sizeof(double);
    EDP_CUDA(c, cudaMemcpyAsync(guess_out, edp_warmstart_guess(c), nb, cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaFreeAsync(scal, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    res_out[0] = std::sqrt(h[0]);
    res_out[1] = std::sqrt(h[1]);
    return EDP_OK;
}
