// Geometric multigrid V-cycle used as the preconditioner of the CG solve that replaces the PETSc path
// (pic2d_ElectricFieldCalc_PETSc.F90:7-355; pic2d_PETSc_Solver.F90:42-1350 builds the same 5-point operator with
// Dirichlet rows for the walls and the metal inner objects and solves it with GMRES + BoomerAMG).
//
// Operator on level l (spacing h = 2^l finest cells): (4 u_ij - sum of the 4 neighbours) / h^2 on unknown nodes,
// Dirichlet nodes (walls, inner objects) carry a zero correction. A coarse node (I, J) is the fine node (2I, 2J) and
// is Dirichlet when that node is. Restriction is full weighting (1/16 [1 2 1; 2 4 2; 1 2 1]) of the masked residual,
// prolongation is bilinear into unknown nodes, so R = P^T / 4. Smoothing is red-black Gauss-Seidel: nu sweeps red
// then black on the way down and nu sweeps black then red on the way up, the adjoint order, and the coarsest level
// gets a palindromic sequence of sweeps. With a zero initial guess on every level the V-cycle is therefore a
// symmetric positive definite operator, as preconditioned CG requires.
//
// Levels whose node count is small run inside one CTA from shared memory (one launch for the whole bottom of
// the cycle); the finer levels are one launch per half sweep, restriction and prolongation.
#include "edp_internal.cuh"

#include <vector>

namespace {

constexpr int kNu = 2;                 // RB sweeps before and after the coarse correction
constexpr int kCoarsestSweeps = 24;    // RB sweep pairs on the coarsest level
constexpr int kCtaNodes = 4225;        // levels with at most this many nodes (65 x 65) run in the coarse CTA
constexpr int kCoarseThreads = 1024;
constexpr int kDirectMax = 256;        // the coarsest level is solved exactly (dense inverse) up to this many unknowns

struct Lev {
    double* u;
    const double* f;
    const int8_t* mask;
    int nx, ny;
    double h2;
};

// one half sweep of red-black Gauss-Seidel over the nodes with (i + j) % 2 == color. With first, the level starts
// from a zero correction: nodes of the colour take h^2 f / 4 and every other node is set to zero.
__device__ __forceinline__ void half_sweep(const Lev& L, int color, bool first, int64_t t0, int64_t stride)
{
    const int w = L.nx + 1;
    if (first) {
        const int64_t n = (int64_t)w * (L.ny + 1);
        for (int64_t q = t0; q < n; q += stride) {
            const int i = (int)(q % w), j = (int)(q / w);
            double v = 0.0;
            if (!L.mask[q] && ((i + j) & 1) == color) v = 0.25 * L.h2 * L.f[q];
            L.u[q] = v;
        }
        return;
    }
    const int hw = (w + 1) >> 1;
    const int64_t n = (int64_t)hw * (L.ny + 1);
    for (int64_t k = t0; k < n; k += stride) {
        const int j = (int)(k / hw);
        const int i = 2 * (int)(k % hw) + ((j + color) & 1);
        if (i > L.nx) continue;
        const int64_t q = (int64_t)j * w + i;
        if (L.mask[q]) continue;   // walls are Dirichlet, so every unknown node has four in-range neighbours
        L.u[q] = 0.25 * (L.h2 * L.f[q] + L.u[q - 1] + L.u[q + 1] + L.u[q - w] + L.u[q + w]);
    }
}

__device__ __forceinline__ double residual_at(const Lev& L, int64_t q)
{
    if (L.mask[q]) return 0.0;
    const int w = L.nx + 1;
    return L.f[q] - (4.0 * L.u[q] - L.u[q - 1] - L.u[q + 1] - L.u[q - w] - L.u[q + w]) / L.h2;
}

// coarse right-hand side = full weighting of the fine residual
__device__ __forceinline__ void restrict_to(const Lev& F, double* fc, const int8_t* maskc, int nxc, int nyc,
                                            int64_t t0, int64_t stride)
{
    const int wc = nxc + 1, w = F.nx + 1;
    const int64_t n = (int64_t)wc * (nyc + 1);
    for (int64_t Q = t0; Q < n; Q += stride) {
        if (maskc[Q]) {
            fc[Q] = 0.0;
            continue;
        }
        const int I = (int)(Q % wc), J = (int)(Q / wc);
        const int64_t q = (int64_t)(2 * J) * w + 2 * I;
        double s = 4.0 * residual_at(F, q);
        s += 2.0 * (residual_at(F, q - 1) + residual_at(F, q + 1) + residual_at(F, q - w) + residual_at(F, q + w));
        s += residual_at(F, q - w - 1) + residual_at(F, q - w + 1) + residual_at(F, q + w - 1) + residual_at(F, q + w + 1);
        fc[Q] = s * 0.0625;
    }
}

// fine correction += bilinear interpolation of the coarse correction (unknown fine nodes only)
__device__ __forceinline__ void prolong_add(const Lev& F, const double* uc, int nxc, int64_t t0, int64_t stride)
{
    const int w = F.nx + 1, wc = nxc + 1;
    const int64_t n = (int64_t)w * (F.ny + 1);
    for (int64_t q = t0; q < n; q += stride) {
        if (F.mask[q]) continue;
        const int i = (int)(q % w), j = (int)(q / w);
        const int I = i >> 1, J = j >> 1;
        const int64_t Q = (int64_t)J * wc + I;
        double e;
        if (!(i & 1) && !(j & 1)) e = uc[Q];
        else if (!(j & 1)) e = 0.5 * (uc[Q] + uc[Q + 1]);
        else if (!(i & 1)) e = 0.5 * (uc[Q] + uc[Q + wc]);
        else e = 0.25 * (uc[Q] + uc[Q + 1] + uc[Q + wc] + uc[Q + wc + 1]);
        F.u[q] += e;
    }
}

// The 2 kNu half-sweeps of one smoothing pass of a level in one launch (temporal blocking): a CTA stages a tile of
// kTx x kTy nodes with a halo of kHalo = 2 kNu nodes, runs the half-sweeps on a region that loses one node on every
// side per half-sweep, and writes back the tile. Every update reads the values the sequence of whole-grid
// half-sweeps would, in the same order, so the result is the same to the bit. zero_start: the pass starts from a
// zero correction (pre-smoothing). uc: the coarse correction, prolonged and added while the tile is staged
// (post-smoothing, prolong_add's interpolation).
constexpr int kTx = 32, kTy = 16, kHalo = 2 * kNu;
constexpr int kSw = kTx + 2 * kHalo, kSh = kTy + 2 * kHalo;

__global__ void __launch_bounds__(256) mg_smooth_kernel(Lev L, int first_color, int zero_start, const double* uc,
                                                        int nxc)
{
    edp_dependent_start();
    __shared__ double su[kSh][kSw];
    __shared__ double sf[kSh][kSw];
    __shared__ int8_t sm[kSh][kSw];
    const int w = L.nx + 1, wc = nxc + 1;
    const int x0 = blockIdx.x * kTx - kHalo, y0 = blockIdx.y * kTy - kHalo;
    for (int k = threadIdx.x; k < kSw * kSh; k += blockDim.x) {
        const int lx = k % kSw, ly = k / kSw, i = x0 + lx, j = y0 + ly;
        double u = 0.0, f = 0.0;
        int8_t m = 1;   // outside the grid: never updated, never read by an unknown node (walls are Dirichlet)
        if (i >= 0 && i <= L.nx && j >= 0 && j <= L.ny) {
            const int64_t q = (int64_t)j * w + i;
            m = L.mask[q];
            f = L.f[q];
            if (!zero_start) u = L.u[q];
            if (uc && !m) {
                const int I = i >> 1, J = j >> 1;
                const int64_t Q = (int64_t)J * wc + I;
                double e;
                if (!(i & 1) && !(j & 1)) e = uc[Q];
                else if (!(j & 1)) e = 0.5 * (uc[Q] + uc[Q + 1]);
                else if (!(i & 1)) e = 0.5 * (uc[Q] + uc[Q + wc]);
                else e = 0.25 * (uc[Q] + uc[Q + 1] + uc[Q + wc] + uc[Q + wc + 1]);
                u += e;
            }
        }
        su[ly][lx] = u;
        sf[ly][lx] = f;
        sm[ly][lx] = m;
    }
    __syncthreads();
    for (int h = 0; h < kHalo; ++h) {
        const int color = first_color ^ (h & 1);
        const int lo = h + 1, nxr = kSw - 2 * lo, nyr = kSh - 2 * lo;
        for (int k = threadIdx.x; k < nxr * nyr; k += blockDim.x) {
            const int lx = lo + k % nxr, ly = lo + k / nxr;
            if (sm[ly][lx] || (((x0 + lx) + (y0 + ly)) & 1) != color) continue;
            su[ly][lx] = 0.25 * (L.h2 * sf[ly][lx] + su[ly][lx - 1] + su[ly][lx + 1] + su[ly - 1][lx] + su[ly + 1][lx]);
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < kTx * kTy; k += blockDim.x) {
        const int lx = kHalo + k % kTx, ly = kHalo + k / kTx, i = x0 + lx, j = y0 + ly;
        if (i <= L.nx && j <= L.ny) L.u[(int64_t)j * w + i] = su[ly][lx];
    }
}

__global__ void mg_restrict_kernel(Lev F, double* fc, const int8_t* maskc, int nxc, int nyc)
{
    edp_dependent_start();
    restrict_to(F, fc, maskc, nxc, nyc, (int64_t)blockIdx.x * blockDim.x + threadIdx.x,
                (int64_t)gridDim.x * blockDim.x);
}

struct CoarseArgs {
    int nlev;                             // levels handled here: lc .. lc + nlev - 1
    int nx[EDP_MG_MAX_LEVELS], ny[EDP_MG_MAX_LEVELS];
    double h2[EDP_MG_MAX_LEVELS];
    const int8_t* mask[EDP_MG_MAX_LEVELS];
    const double* f_in;                   // right-hand side of the top level here
    double* u_out;                        // its correction
    const double* cinv;                   // inverse of the coarsest level's operator on its cn unknowns, or null
    const int32_t* cidx;                  // node of each unknown
    int cn;
};

// The bottom of the V-cycle in one CTA: every level lives in shared memory, phases are separated by barriers.
__global__ void __launch_bounds__(kCoarseThreads, 1) mg_coarse_kernel(CoarseArgs a)
{
    edp_dependent_start();
    extern __shared__ __align__(16) unsigned char sm[];
    Lev L[EDP_MG_MAX_LEVELS];
    size_t off = 0;
    for (int l = 0; l < a.nlev; ++l) {
        const int64_t n = (int64_t)(a.nx[l] + 1) * (a.ny[l] + 1);
        L[l].u = reinterpret_cast<double*>(sm + off);
        off += n * sizeof(double);
        L[l].f = reinterpret_cast<const double*>(sm + off);
        off += n * sizeof(double);
        L[l].mask = reinterpret_cast<const int8_t*>(sm + off);
        off += (n + 15) & ~(int64_t)15;
        L[l].nx = a.nx[l];
        L[l].ny = a.ny[l];
        L[l].h2 = a.h2[l];
    }
    const int t = threadIdx.x, T = blockDim.x;
    for (int l = 0; l < a.nlev; ++l) {
        const int64_t n = (int64_t)(a.nx[l] + 1) * (a.ny[l] + 1);
        int8_t* m = const_cast<int8_t*>(L[l].mask);
        for (int64_t q = t; q < n; q += T) m[q] = a.mask[l][q];
    }
    {
        const int64_t n = (int64_t)(a.nx[0] + 1) * (a.ny[0] + 1);
        double* f0 = const_cast<double*>(L[0].f);
        for (int64_t q = t; q < n; q += T) f0[q] = a.f_in[q];
    }
    __syncthreads();
    const int last = a.nlev - 1;
    for (int l = 0; l < last; ++l) {
        for (int s = 0; s < kNu; ++s) {
            half_sweep(L[l], 0, s == 0, t, T);
            __syncthreads();
            half_sweep(L[l], 1, false, t, T);
            __syncthreads();
        }
        restrict_to(L[l], const_cast<double*>(L[l + 1].f), L[l + 1].mask, a.nx[l + 1], a.ny[l + 1], t, T);
        __syncthreads();
    }
    if (a.cinv) {   // exact: u = A^-1 f on the unknowns, one warp per row
        const int64_t n = (int64_t)(a.nx[last] + 1) * (a.ny[last] + 1);
        for (int64_t q = t; q < n; q += T) L[last].u[q] = 0.0;
        __syncthreads();
        const int lane = t & 31;
        for (int r = t >> 5; r < a.cn; r += T >> 5) {
            const double* row = a.cinv + (int64_t)r * a.cn;
            double acc = 0.0;
            for (int k = lane; k < a.cn; k += 32) acc += row[k] * L[last].f[a.cidx[k]];
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
            if (lane == 0) L[last].u[a.cidx[r]] = acc;
        }
        __syncthreads();
    } else {
        for (int s = 0; s < kCoarsestSweeps; ++s) {
            half_sweep(L[last], 0, s == 0, t, T);
            __syncthreads();
            half_sweep(L[last], 1, false, t, T);
            __syncthreads();
        }
        for (int s = 0; s < kCoarsestSweeps; ++s) {
            half_sweep(L[last], 1, false, t, T);
            __syncthreads();
            half_sweep(L[last], 0, false, t, T);
            __syncthreads();
        }
    }
    for (int l = last - 1; l >= 0; --l) {
        prolong_add(L[l], L[l + 1].u, a.nx[l + 1], t, T);
        __syncthreads();
        for (int s = 0; s < kNu; ++s) {
            half_sweep(L[l], 1, false, t, T);
            __syncthreads();
            half_sweep(L[l], 0, false, t, T);
            __syncthreads();
        }
    }
    const int64_t n = (int64_t)(a.nx[0] + 1) * (a.ny[0] + 1);
    for (int64_t q = t; q < n; q += T) a.u_out[q] = L[0].u[q];
}

unsigned grid_of_nodes(int nx, int ny)
{
    int64_t n = (int64_t)(nx + 1) * (ny + 1);
    int64_t g = (n + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    return (unsigned)(g < 1 ? 1 : g);
}

Lev lev_of(const edp_ctx* c, int l, double* u, const double* f)
{
    Lev L;
    L.u = u;
    L.f = f;
    L.mask = c->mg[l].mask;
    L.nx = c->mg[l].nx;
    L.ny = c->mg[l].ny;
    L.h2 = (double)(1 << l) * (double)(1 << l);
    return L;
}

}  // namespace

// The coarsest level's operator (4 u - neighbours) / h^2 on its unknown nodes, inverted once on the host (Gauss-Jordan
// with partial pivoting, FP64): the V-cycle then solves that level exactly, which keeps it symmetric.
static int coarsest_inverse(edp_ctx* c, const std::vector<int8_t>& mask, int nx, int ny, double h2)
{
    const int w = nx + 1;
    std::vector<int32_t> idx, pos(mask.size(), -1);
    for (size_t q = 0; q < mask.size(); ++q)
        if (!mask[q]) {
            pos[q] = (int32_t)idx.size();
            idx.push_back((int32_t)q);
        }
    const int n = (int)idx.size();
    if (n == 0 || n > kDirectMax) return EDP_OK;
    std::vector<double> a((size_t)n * n, 0.0), inv((size_t)n * n, 0.0);
    for (int r = 0; r < n; ++r) {
        const int q = idx[r], i = q % w, j = q / w;
        a[(size_t)r * n + r] = 4.0 / h2;
        const int nb[4][2] = {{i - 1, j}, {i + 1, j}, {i, j - 1}, {i, j + 1}};
        for (const auto& e : nb) {
            if (e[0] < 0 || e[0] > nx || e[1] < 0 || e[1] > ny) continue;
            const int k = pos[(size_t)e[1] * w + e[0]];
            if (k >= 0) a[(size_t)r * n + k] = -1.0 / h2;
        }
        inv[(size_t)r * n + r] = 1.0;
    }
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int r = col + 1; r < n; ++r)
            if (std::fabs(a[(size_t)r * n + col]) > std::fabs(a[(size_t)piv * n + col])) piv = r;
        if (a[(size_t)piv * n + col] == 0.0) return EDP_OK;   // singular: keep the sweeps
        if (piv != col)
            for (int k = 0; k < n; ++k) {
                std::swap(a[(size_t)piv * n + k], a[(size_t)col * n + k]);
                std::swap(inv[(size_t)piv * n + k], inv[(size_t)col * n + k]);
            }
        const double d = 1.0 / a[(size_t)col * n + col];
        for (int k = 0; k < n; ++k) {
            a[(size_t)col * n + k] *= d;
            inv[(size_t)col * n + k] *= d;
        }
        for (int r = 0; r < n; ++r) {
            if (r == col) continue;
            const double f = a[(size_t)r * n + col];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                a[(size_t)r * n + k] -= f * a[(size_t)col * n + k];
                inv[(size_t)r * n + k] -= f * inv[(size_t)col * n + k];
            }
        }
    }
    EDP_CUDA(c, cudaMalloc(&c->mg_cinv, (size_t)n * n * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&c->mg_cidx, (size_t)n * sizeof(int32_t)));
    EDP_CUDA(c, cudaMemcpy(c->mg_cinv, inv.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice));
    EDP_CUDA(c, cudaMemcpy(c->mg_cidx, idx.data(), (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice));
    c->mg_cn = n;
    return EDP_OK;
}

int edp_mg_setup(edp_ctx* c)
{
    const edp_params& p = c->p;
    // levels: halve while both cell counts stay even and the coarse grid keeps at least 2 x 2 cells
    int nl = 1;
    c->mg[0].nx = p.ncx;
    c->mg[0].ny = p.ncy;
    while (nl < EDP_MG_MAX_LEVELS) {
        const int nx = c->mg[nl - 1].nx, ny = c->mg[nl - 1].ny;
        if ((nx & 1) || (ny & 1) || nx < 4 || ny < 4) break;
        c->mg[nl].nx = nx / 2;
        c->mg[nl].ny = ny / 2;
        ++nl;
    }
    c->mg_nlev = nl;
    int lc = 0;
    while (lc < nl && (int64_t)(c->mg[lc].nx + 1) * (c->mg[lc].ny + 1) > kCtaNodes) ++lc;
    if (lc == nl) lc = nl - 1;   // the coarsest level is large (odd sizes): it still runs in the CTA
    c->mg_lc = lc;
    size_t smem = 0;
    for (int l = lc; l < nl; ++l) {
        const size_t n = (size_t)(c->mg[l].nx + 1) * (c->mg[l].ny + 1);
        smem += 2 * n * sizeof(double) + ((n + 15) & ~(size_t)15);
    }
    if (smem > 220 * 1024) {   // cell counts without enough factors of 2: plain CG only
        c->mg_nlev = 0;
        c->precond = EDP_PRECOND_NONE;
        return EDP_OK;
    }
    c->mg_smem = smem;
    TRY(edp_raise_smem_limit(c, (const void*)mg_coarse_kernel, smem));
    // Dirichlet masks: walls, and the metal inner objects, of the finest node at (2^l I, 2^l J)
    for (int l = 0; l < nl; ++l) {
        edp_mg_level& m = c->mg[l];
        const int w = m.nx + 1;
        const size_t n = (size_t)w * (m.ny + 1);
        std::vector<int8_t> h(n);
        for (int J = 0; J <= m.ny; ++J)
            for (int I = 0; I <= m.nx; ++I) {
                const int i = I << l, j = J << l;
                int8_t k = (i == 0 || j == 0 || i == p.ncx || j == p.ncy) ? 1 : 0;
                for (int o = 0; o < p.n_inner; ++o)
                    if (!(p.inner_eps[o] > 0.0) && i >= p.inner_ileft[o] && i <= p.inner_iright[o] && j >= p.inner_jbottom[o] && j <= p.inner_jtop[o])
                        k = 1;
                h[(size_t)J * w + I] = k;
            }
        EDP_CUDA(c, cudaMalloc(&m.mask, n));
        EDP_CUDA(c, cudaMemcpy(m.mask, h.data(), n, cudaMemcpyHostToDevice));
        if (l > 0) {
            EDP_CUDA(c, cudaMalloc(&m.u, n * sizeof(double)));
            EDP_CUDA(c, cudaMalloc(&m.f, n * sizeof(double)));
        }
        if (l == nl - 1) TRY(coarsest_inverse(c, h, m.nx, m.ny, (double)(1 << l) * (double)(1 << l)));
    }
    return EDP_OK;
}

void edp_mg_free(edp_ctx* c)
{
    for (int l = 0; l < c->mg_nlev; ++l) {
        cudaFree(c->mg[l].mask);
        if (l > 0) {
            cudaFree(c->mg[l].u);
            cudaFree(c->mg[l].f);
        }
        c->mg[l] = edp_mg_level();
    }
    c->mg_nlev = 0;
    cudaFree(c->mg_cinv);
    cudaFree(c->mg_cidx);
    c->mg_cinv = nullptr;
    c->mg_cidx = nullptr;
    c->mg_cn = 0;
}

int edp_mg_apply(edp_ctx* c, const double* r, double* z)
{
    const int nl = c->mg_nlev, lc = c->mg_lc;
    auto u_of = [&](int l) { return l == 0 ? z : c->mg[l].u; };
    auto f_of = [&](int l) { return l == 0 ? r : (const double*)c->mg[l].f; };
    auto tiles = [](const Lev& L) { return dim3((unsigned)((L.nx + kTx) / kTx), (unsigned)((L.ny + kTy) / kTy)); };
    for (int l = 0; l < lc; ++l) {
        Lev L = lev_of(c, l, u_of(l), f_of(l));
        ++c->launches;   // pre-smoothing from a zero correction: red, black, red, black
        EDP_CUDA(c, edp_launch_dependent(mg_smooth_kernel, tiles(L), dim3(256), 0, c->stream, L, 0, 1,
                                          (const double*)nullptr, 0));
        ++c->launches;
        EDP_CUDA(c, edp_launch_dependent(mg_restrict_kernel, dim3(grid_of_nodes(c->mg[l + 1].nx, c->mg[l + 1].ny)),
                                          dim3(256), 0, c->stream, L, c->mg[l + 1].f,
                                          (const int8_t*)c->mg[l + 1].mask, c->mg[l + 1].nx, c->mg[l + 1].ny));
    }
    CoarseArgs a;
    memset(&a, 0, sizeof(a));
    a.nlev = nl - lc;
    for (int l = lc; l < nl; ++l) {
        a.nx[l - lc] = c->mg[l].nx;
        a.ny[l - lc] = c->mg[l].ny;
        a.h2[l - lc] = (double)(1 << l) * (double)(1 << l);
        a.mask[l - lc] = c->mg[l].mask;
    }
    a.f_in = f_of(lc);
    a.u_out = u_of(lc);
    a.cinv = c->mg_cinv;
    a.cidx = c->mg_cidx;
    a.cn = c->mg_cn;
    ++c->launches;
    EDP_CUDA(c, edp_launch_dependent(mg_coarse_kernel, dim3(1), dim3(kCoarseThreads), c->mg_smem, c->stream, a));
    for (int l = lc - 1; l >= 0; --l) {
        Lev L = lev_of(c, l, u_of(l), f_of(l));
        ++c->launches;   // prolongation, then post-smoothing: black, red, black, red
        EDP_CUDA(c, edp_launch_dependent(mg_smooth_kernel, tiles(L), dim3(256), 0, c->stream, L, 1, 0,
                                          (const double*)c->mg[l + 1].u, c->mg[l + 1].nx));
    }
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}
