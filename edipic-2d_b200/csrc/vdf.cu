// Velocity distribution functions: CALCULATE_ELECTRON_VDF / CALCULATE_ION_VDF (pic2d_VelocityDistributions.f90:3-393)
// on the particles in HBM, for one cluster over the whole domain.
//
// The cluster area [0, c_X_area_max] x [0, c_Y_area_max] is split into nbx x nby boxes at X = i * c_X_area_max / nbx,
// Y = j * c_Y_area_max / nby (xsplit/ysplit, :63-75). c_X_area_max = c_indx_x_max is ncx on a walled domain and
// ncx + 1 on the self-connected periodic cluster (its overlap node, pic2d_CurProblemValues.f90:1310, :1331);
// positions here are the periodic images in [0, ncx). Each velocity component is binned as INT(v * fvc), one less
// for v < 0 (:99-117), with fvc = N_max_vel * N_vbins (* sqrt(Ms) for ions, :74 of the ion routine), bins
// vmin = -N_max_vel_s * N_vbins .. vmax = -vmin - 1. A particle with any component outside that range is skipped
// and counted (:101-118). Counts: 1D histograms of vx, vy, vz per box and, when asked, the 2D vx-vy histogram per
// box (:122-136).
//
// One CTA keeps private copies of the histograms in shared memory when they fit (the 1D ones always do at the
// reference's sizes) and adds them to the global counts once; otherwise it adds each count to global memory.
#include <algorithm>
#include <vector>

#include "edp_internal.cuh"

namespace {

constexpr int kMaxBoxes = 16;   // per direction (the deck's i1 fields allow 9)

struct VdfArgs {
    int precision;
    edp_species_mixed m;
    edp_species_fp64 d;
    const unsigned long long* n_slots;
    int nbx, nby, nbox;
    double xsplit[kMaxBoxes], ysplit[kMaxBoxes];
    double fvc;
    int vmin, vmax, reclen;
    unsigned* h1;            // [3][nbox][reclen], global
    unsigned* h2;            // [nbox][reclen (vy)][reclen (vx)], global, or null
    int h1_shared, h2_shared;
    unsigned long long* skipped;
};

// the bin of one velocity component, or INT_MIN when out of range (the reference's INT of a value beyond the
// integer range is not defined; such values are far outside every bin range and count as skipped)
__device__ __forceinline__ int vbin(double v, double fvc, int vmin, int vmax)
{
    const double t = v * fvc;
    if (!(fabs(t) < 1073741824.0)) return INT_MIN;
    int b = (int)t;
    if (v < 0.0) b -= 1;
    return (b < vmin || b > vmax) ? INT_MIN : b;
}

__global__ void __launch_bounds__(256) vdf_kernel(VdfArgs a)
{
    extern __shared__ unsigned sh[];
    const int n1 = 3 * a.nbox * a.reclen;
    const int64_t n2 = (int64_t)a.nbox * a.reclen * a.reclen;
    unsigned* s1 = sh;
    unsigned* s2 = sh + (a.h1_shared ? n1 : 0);
    if (a.h1_shared)
        for (int q = threadIdx.x; q < n1; q += blockDim.x) s1[q] = 0u;
    if (a.h2 && a.h2_shared)
        for (int64_t q = threadIdx.x; q < n2; q += blockDim.x) s2[q] = 0u;
    __shared__ unsigned long long skip_cta;
    if (threadIdx.x == 0) skip_cta = 0ull;
    __syncthreads();
    unsigned* h1 = a.h1_shared ? s1 : a.h1;
    unsigned* h2 = a.h2 ? (a.h2_shared ? s2 : a.h2) : nullptr;
    unsigned long long skip = 0ull;
    const int64_t n = (int64_t)*a.n_slots;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double X, Y, vx, vy, vz;
        if (a.precision == EDP_PREC_MIXED) {
            const int cell = a.m.cell[k];
            if (cell < 0) continue;
            X = (double)(cell & 0xFFFF) + (double)a.m.ox[k];
            Y = (double)(cell >> 16) + (double)a.m.oy[k];
            vx = a.m.vx[k];
            vy = a.m.vy[k];
            vz = a.m.vz[k];
        } else {
            X = a.d.x[k];
            if (X < -1.0e29) continue;
            Y = a.d.y[k];
            vx = a.d.vx[k];
            vy = a.d.vy[k];
            vz = a.d.vz[k];
        }
        int ib = a.nbx - 1;
        for (int i = 0; i < a.nbx - 1; ++i)
            if (X < a.xsplit[i]) { ib = i; break; }
        int jb = a.nby - 1;
        for (int j = 0; j < a.nby - 1; ++j)
            if (Y < a.ysplit[j]) { jb = j; break; }
        const int box = ib + jb * a.nbx;
        const int bx = vbin(vx, a.fvc, a.vmin, a.vmax);
        const int by = bx == INT_MIN ? INT_MIN : vbin(vy, a.fvc, a.vmin, a.vmax);
        const int bz = by == INT_MIN ? INT_MIN : vbin(vz, a.fvc, a.vmin, a.vmax);
        if (bz == INT_MIN) {
            ++skip;
            continue;
        }
        const int base = box * a.reclen - a.vmin;
        atomicAdd(&h1[base + bx], 1u);
        atomicAdd(&h1[a.nbox * a.reclen + base + by], 1u);
        atomicAdd(&h1[2 * a.nbox * a.reclen + base + bz], 1u);
        if (h2) atomicAdd(&h2[((int64_t)box * a.reclen + (by - a.vmin)) * a.reclen + (bx - a.vmin)], 1u);
    }
    if (skip) atomicAdd(&skip_cta, skip);
    __syncthreads();
    if (threadIdx.x == 0 && skip_cta) atomicAdd(a.skipped, skip_cta);
    if (a.h1_shared)
        for (int q = threadIdx.x; q < n1; q += blockDim.x)
            if (s1[q]) atomicAdd(&a.h1[q], s1[q]);
    if (a.h2 && a.h2_shared)
        for (int64_t q = threadIdx.x; q < n2; q += blockDim.x)
            if (s2[q]) atomicAdd(&a.h2[q], s2[q]);
}

}  // namespace

extern "C" int edp_calculate_vdf(edp_ctx* c, int species, int32_t n_max_vel, int32_t nbox_x, int32_t nbox_y,
                                 int32_t n_max_vel_s, int32_t n_vbins, int32_t* vdf1d, int32_t* vdf2d,
                                 int64_t* skipped)
{
    if (!c || !vdf1d || species < 0 || species >= c->nspec || n_max_vel < 1 || nbox_x < 1 || nbox_y < 1 ||
        nbox_x > kMaxBoxes || nbox_y > kMaxBoxes || n_max_vel_s < 1 || n_vbins < 1 ||
        (int64_t)n_max_vel_s * n_vbins > (1 << 20))
        return edp_fail(c, EDP_ERR_ARG, "edp_calculate_vdf");
    if (!c->uploaded[species]) return edp_fail(c, EDP_ERR_STATE, "species not uploaded");
    VdfArgs a;
    memset(&a, 0, sizeof(a));
    a.precision = c->p.precision;
    a.m = c->pm[species];
    a.d = c->pd[species];
    a.n_slots = &c->dc->n_slots[species];
    a.nbx = nbox_x;
    a.nby = nbox_y;
    a.nbox = nbox_x * nbox_y;
    // xsplit(i) = c_X_area_min + DBLE(i) * (c_X_area_max - c_X_area_min) / N_vdfbox_x (:65-67), one cluster
    const double xarea = (double)(c->p.periodic_x ? c->p.ncx + 1 : c->p.ncx);
    for (int i = 1; i < nbox_x; ++i) a.xsplit[i - 1] = 0.0 + (double)i * xarea / nbox_x;
    for (int j = 1; j < nbox_y; ++j) a.ysplit[j - 1] = 0.0 + (double)j * (double)c->p.ncy / nbox_y;
    a.fvc = (double)(n_max_vel * n_vbins);
    if (species > 0) a.fvc *= std::sqrt(c->p.ion_mass_me[species - 1]);
    a.vmin = -n_max_vel_s * n_vbins;
    a.vmax = n_max_vel_s * n_vbins - 1;
    a.reclen = 2 * n_max_vel_s * n_vbins;
    const int64_t n1 = 3LL * a.nbox * a.reclen;
    const int64_t n2 = vdf2d ? (int64_t)a.nbox * a.reclen * a.reclen : 0;
    if (n2 > ((int64_t)1 << 31)) return edp_fail(c, EDP_ERR_ARG, "edp_calculate_vdf: 2D histogram too large");
    const int64_t kSmem = 160 * 1024 / 4;   // private copies up to 160 KB per CTA
    a.h1_shared = n1 <= kSmem;
    a.h2_shared = vdf2d && a.h1_shared && n1 + n2 <= kSmem;
    const size_t smem = 4 * (size_t)((a.h1_shared ? n1 : 0) + (a.h2_shared ? n2 : 0));
    unsigned* buf = nullptr;
    const size_t bytes = (size_t)(n1 + n2) * 4 + 16;
    EDP_CUDA(c, cudaMallocAsync(&buf, bytes, c->stream));
    EDP_CUDA(c, cudaMemsetAsync(buf, 0, bytes, c->stream));
    a.h1 = buf;
    a.h2 = vdf2d ? buf + n1 : nullptr;
    a.skipped = reinterpret_cast<unsigned long long*>(buf + n1 + n2 + ((n1 + n2) & 1));
    if (smem > 48 * 1024)
        TRY(edp_raise_smem_limit(c, (const void*)vdf_kernel, smem));
    // about 64 particles per thread, so that the private copies are flushed rarely
    const int64_t slots = c->host_slots[species];
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((slots + 256 * 64 - 1) / (256 * 64), 148 * 4));
    ++c->launches;
    vdf_kernel<<<(unsigned)grid, 256, smem, c->stream>>>(a);
    EDP_CUDA(c, cudaGetLastError());
    EDP_CUDA(c, cudaMemcpyAsync(vdf1d, a.h1, n1 * 4, cudaMemcpyDeviceToHost, c->stream));
    if (vdf2d) EDP_CUDA(c, cudaMemcpyAsync(vdf2d, a.h2, n2 * 4, cudaMemcpyDeviceToHost, c->stream));
    unsigned long long sk = 0;
    EDP_CUDA(c, cudaMemcpyAsync(&sk, a.skipped, 8, cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaFreeAsync(buf, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    if (skipped) *skipped = (int64_t)sk;
    return EDP_OK;
}

// ------------------------------------------------------------------------------------------ energy distribution
// Counts of the particles of one species by kinetic energy in eV (the electron energy distribution of the long-run
// comparison, the EEDF, without downloading the particles): E = (vx^2 + vy^2 + vz^2) * energy_factor_eV (* Ms for
// ions, PERFORM_RESONANT_CHARGE_EXCHANGE's factor_eV), in the bins [edges[k], edges[k+1]); energies outside
// [edges[0], edges[n_bins]) are not counted. Private shared-memory histograms per CTA, one global add per bin.
namespace {

constexpr int kMaxEnergyBins = 256;

__global__ void __launch_bounds__(256) energy_hist_kernel(int precision, edp_species_mixed m, edp_species_fp64 d,
                                                          const unsigned long long* n_slots, double factor,
                                                          const double* edges, int n_bins,
                                                          unsigned long long* counts)
{
    __shared__ double e[kMaxEnergyBins + 1];
    __shared__ unsigned h[kMaxEnergyBins];
    for (int k = threadIdx.x; k <= n_bins; k += blockDim.x) e[k] = edges[k];
    for (int k = threadIdx.x; k < n_bins; k += blockDim.x) h[k] = 0u;
    __syncthreads();
    const int64_t n = (int64_t)*n_slots;
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
        const double en = (vx * vx + vy * vy + vz * vz) * factor;
        if (!(en >= e[0] && en < e[n_bins])) continue;
        int lo = 0, hi = n_bins;   // e[lo] <= en < e[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (en >= e[mid]) lo = mid;
            else hi = mid;
        }
        atomicAdd(&h[lo], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n_bins; k += blockDim.x)
        if (h[k]) atomicAdd(&counts[k], (unsigned long long)h[k]);
}

}  // namespace

extern "C" int edp_energy_histogram(edp_ctx* c, int species, int32_t n_bins, const double* edges_ev, int64_t* counts)
{
    if (!c || species < 0 || species >= c->nspec || n_bins < 1 || n_bins > kMaxEnergyBins || !edges_ev || !counts)
        return edp_fail(c, EDP_ERR_ARG, "edp_energy_histogram");
    for (int k = 0; k < n_bins; ++k)
        if (!(edges_ev[k + 1] > edges_ev[k])) return edp_fail(c, EDP_ERR_ARG, "edp_energy_histogram: edges must rise");
    if (!c->uploaded[species]) return edp_fail(c, EDP_ERR_STATE, "species not uploaded");
    double factor = c->tab.energy_factor_eV;
    if (species > 0) factor *= c->p.ion_mass_me[species - 1];
    double* dev_edges = nullptr;
    unsigned long long* dev_counts = nullptr;
    EDP_CUDA(c, cudaMallocAsync(&dev_edges, (n_bins + 1) * sizeof(double), c->stream));
    EDP_CUDA(c, cudaMallocAsync(&dev_counts, n_bins * sizeof(unsigned long long), c->stream));
    EDP_CUDA(c, cudaMemcpyAsync(dev_edges, edges_ev, (n_bins + 1) * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    EDP_CUDA(c, cudaMemsetAsync(dev_counts, 0, n_bins * sizeof(unsigned long long), c->stream));
    ++c->launches;
    energy_hist_kernel<<<148 * 8, 256, 0, c->stream>>>(c->p.precision, c->pm[species], c->pd[species],
                                                      &c->dc->n_slots[species], factor, dev_edges, n_bins, dev_counts);
    EDP_CUDA(c, cudaGetLastError());
    std::vector<unsigned long long> h(n_bins);
    EDP_CUDA(c, cudaMemcpyAsync(h.data(), dev_counts, n_bins * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                c->stream));
    EDP_CUDA(c, cudaFreeAsync(dev_edges, c->stream));
    EDP_CUDA(c, cudaFreeAsync(dev_counts, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < n_bins; ++k) counts[k] = (int64_t)h[k];
    return EDP_OK;
}
