// Velocity moments on the node grid: COLLECT_ELECTRON_MOMENTS (pic2d_ElectronMoments.f90:3-425), which is also what
// ADVANCE_ELECTRONS_AND_CALCULATE_MOMENTS_2D (pic2d_ElectronDynamicsWithVDFMoments.f90:156-) deposits during the push
// of a snapshot step, and COLLECT_ION_MOMENTS (pic2d_IonMoments.f90:3-348).
//
// Per particle, at its current position with CIC weights in FP32 (:148-157): 1, v, v_x^2.., v_x v_y.., |v|^2 v for
// v = the stored velocity (ions) or, for electrons, the mean of the stored velocity and its Boris update in the
// current field (:159-243). Sums go to FP32 shared-memory windows of the sorted tiles (particles outside the window
// and the unsorted tail go straight to FP64 global sums), then to FP64 node sums; the finish kernel normalises per
// node (:356-419) and scales the density at the walls (ADJUST_DENSITY_AT_WALL_BOUNDARIES :1829-1934).
#include "edp_internal.cuh"

namespace {

constexpr int kNM = 13;
constexpr int kWin = EDP_WIN_NODES * EDP_WIN_NODES;

struct MomArgs {
    edp_kparams kp;
    int precision;
    edp_species_mixed m;
    edp_species_fp64 d;
    const unsigned long long* n_slots;
    const edp_chunk* chunks;
    int64_t n_chunks;
    int64_t tail_start;
    int64_t tail_ctas;
    int electron;                  // average with the Boris update
    const float2* E2;              // mixed-precision field
    const double *Ex, *Ey;         // FP64 field
    double K[9];                   // Boris rotation of the electrons
    double ez;                     // Ez (normalised)
    double* sum;                   // [13][nodes], FP64
};

__device__ __forceinline__ int wrap_x(int x, const edp_kparams& kp)
{
    if (!kp.periodic) return x;
    x %= kp.ncx;
    return x < 0 ? x + kp.ncx : x;
}

// moments of one particle at cell (i, j), offsets (fx, fy) in [0, 1]
__device__ __forceinline__ void particle_moments(const MomArgs& a, int i, int j, double fx, double fy, double vx,
                                                 double vy, double vz, float w[4], float mo[kNM])
{
    const edp_kparams& kp = a.kp;
    const float ax1 = (float)fx, ax0 = 1.0f - ax1, ay1 = (float)fy, ay0 = 1.0f - ay1;
    w[0] = ax0 * ay0;
    w[1] = ax1 * ay0;
    w[2] = ax0 * ay1;
    w[3] = 1.0f - w[0] - w[1] - w[2];
    if (a.electron) {
        const int i1 = (kp.periodic && i + 1 == kp.ncx) ? 0 : i + 1;
        const int64_t r0 = (int64_t)j * kp.nxg, r1 = r0 + kp.nxg;
        const double dx1 = fx, dx0 = 1.0 - fx, dy1 = fy, dy0 = 1.0 - fy;
        double ex, ey;
        if (a.precision == EDP_PREC_MIXED) {
            const float2 e00 = a.E2[r0 + i], e10 = a.E2[r0 + i1], e01 = a.E2[r1 + i], e11 = a.E2[r1 + i1];
            ex = e00.x * dx0 * dy0 + e10.x * dx1 * dy0 + e01.x * dx0 * dy1 + e11.x * dx1 * dy1;
            ey = e00.y * dx0 * dy0 + e10.y * dx1 * dy0 + e01.y * dx0 * dy1 + e11.y * dx1 * dy1;
        } else {
            ex = a.Ex[r0 + i] * dx0 * dy0 + a.Ex[r0 + i1] * dx1 * dy0 + a.Ex[r1 + i] * dx0 * dy1 +
                 a.Ex[r1 + i1] * dx1 * dy1;
            ey = a.Ey[r0 + i] * dx0 * dy0 + a.Ey[r0 + i1] * dx1 * dy0 + a.Ey[r1 + i] * dx0 * dy1 +
                 a.Ey[r1 + i1] * dx1 * dy1;
        }
        const double um = vx - 0.5 * ex, vm = vy - 0.5 * ey, wm = vz - 0.5 * a.ez;
        const double nx = a.K[0] * um + a.K[1] * vm + a.K[2] * wm - 0.5 * ex;
        const double ny = a.K[3] * um + a.K[4] * vm + a.K[5] * wm - 0.5 * ey;
        const double nz = a.K[6] * um + a.K[7] * vm + a.K[8] * wm - 0.5 * a.ez;
        vx = 0.5 * (vx + nx);
        vy = 0.5 * (vy + ny);
        vz = 0.5 * (vz + nz);
    }
    const float rx = (float)vx, ry = (float)vy, rz = (float)vz;
    const float x2 = rx * rx, y2 = ry * ry, z2 = rz * rz, v2 = x2 + y2 + z2;
    mo[0] = 1.0f;
    mo[1] = rx;
    mo[2] = ry;
    mo[3] = rz;
    mo[4] = x2;
    mo[5] = y2;
    mo[6] = z2;
    mo[7] = rx * ry;
    mo[8] = rx * rz;
    mo[9] = ry * rz;
    mo[10] = v2 * rx;
    mo[11] = v2 * ry;
    mo[12] = v2 * rz;
}

__device__ __forceinline__ void add_global(const MomArgs& a, int i, int j, const float w[4], const float mo[kNM])
{
    const edp_kparams& kp = a.kp;
    const int64_t nn = (int64_t)kp.nxg * kp.nyg;
    const int i1 = (kp.periodic && i + 1 == kp.ncx) ? 0 : i + 1;
    const int64_t q[4] = {(int64_t)j * kp.nxg + i, (int64_t)j * kp.nxg + i1, (int64_t)(j + 1) * kp.nxg + i,
                          (int64_t)(j + 1) * kp.nxg + i1};
    for (int m = 0; m < kNM; ++m)
        for (int c = 0; c < 4; ++c) atomicAdd(&a.sum[m * nn + q[c]], (double)(mo[m] * w[c]));
}

__global__ void __launch_bounds__(256) moments_mixed_kernel(MomArgs a)
{
    __shared__ float acc[kNM][kWin];
    const edp_kparams& kp = a.kp;
    const bool windowed = blockIdx.x < a.n_chunks;
    int64_t lo, hi, stride, first;
    int wx0 = 0, wy0 = 0;
    if (windowed) {
        const edp_chunk ch = a.chunks[blockIdx.x];
        lo = ch.start;
        hi = ch.end;
        wx0 = ch.wx0;
        wy0 = ch.wy0;
        for (int t = threadIdx.x; t < kNM * kWin; t += blockDim.x) (&acc[0][0])[t] = 0.0f;
        first = lo + threadIdx.x;
        stride = blockDim.x;
    } else {
        lo = a.tail_start;
        hi = (int64_t)*a.n_slots;
        first = lo + (blockIdx.x - a.n_chunks) * blockDim.x + threadIdx.x;
        stride = a.tail_ctas * blockDim.x;
    }
    __syncthreads();
    for (int64_t k = first; k < hi; k += stride) {
        const int cell = a.m.cell[k];
        if (cell < 0) continue;
        const int i = cell & 0xFFFF, j = cell >> 16;
        float w[4], mo[kNM];
        particle_moments(a, i, j, a.m.ox[k], a.m.oy[k], a.m.vx[k], a.m.vy[k], a.m.vz[k], w, mo);
        const int lx = i - wx0, ly = j - wy0;   // the window keeps the unwrapped i + 1 column
        if (windowed && lx >= 0 && lx + 1 < EDP_WIN_NODES && ly >= 0 && ly + 1 < EDP_WIN_NODES) {
            const int b = ly * EDP_WIN_NODES + lx;
            for (int m = 0; m < kNM; ++m) {
                atomicAdd(&acc[m][b], mo[m] * w[0]);
                atomicAdd(&acc[m][b + 1], mo[m] * w[1]);
                atomicAdd(&acc[m][b + EDP_WIN_NODES], mo[m] * w[2]);
                atomicAdd(&acc[m][b + EDP_WIN_NODES + 1], mo[m] * w[3]);
            }
        } else {
            add_global(a, i, j, w, mo);
        }
    }
    if (!windowed) return;
    __syncthreads();
    const int64_t nn = (int64_t)kp.nxg * kp.nyg;
    for (int t = threadIdx.x; t < kWin; t += blockDim.x) {
        const int gx = wrap_x(wx0 + t % EDP_WIN_NODES, kp), gy = wy0 + t / EDP_WIN_NODES;
        if (gx < 0 || gx >= kp.nxg || gy < 0 || gy >= kp.nyg) continue;   // such nodes received nothing
        const int64_t q = (int64_t)gy * kp.nxg + gx;
        for (int m = 0; m < kNM; ++m)
            if (acc[m][t] != 0.0f) atomicAdd(&a.sum[m * nn + q], (double)acc[m][t]);
    }
}

__global__ void moments_fp64_kernel(MomArgs a)
{
    const edp_kparams& kp = a.kp;
    const int64_t n = (int64_t)*a.n_slots;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double X = a.d.x[k];
        if (X < -1.0e29) continue;
        const double Y = a.d.y[k];
        int i = (int)X, j = (int)Y;
        if (!kp.periodic && i == kp.ncx) i = kp.ncx - 1;
        if (kp.periodic && i >= kp.ncx) i -= kp.ncx;
        if (j == kp.ncy) j = kp.ncy - 1;
        double fx = X - (double)((int)X), fy = Y - (double)j;
        if (!kp.periodic && (int)X == kp.ncx) fx = 1.0;
        float w[4], mo[kNM];
        particle_moments(a, i, j, fx, fy, a.d.vx[k], a.d.vy[k], a.d.vz[k], w, mo);
        add_global(a, i, j, w, mo);
    }
}

// normalisation per node and the wall factors of the density, then the reference node layout (float)
__global__ void moments_finish_kernel(edp_kparams kp, const double* __restrict__ sum, int wout, float* __restrict__ out)
{
    const int64_t nn = (int64_t)kp.nxg * kp.nyg, nref = (int64_t)wout * kp.nyg;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nref; r += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(r % wout), j = (int)(r / wout);
        const int ic = kp.periodic ? i % kp.ncx : i;
        const int64_t q = (int64_t)j * kp.nxg + ic;
        double c[kNM];
        for (int m = 0; m < kNM; ++m) c[m] = sum[m * nn + q];
        if (c[0] > 1.0e-9) {
            const double inv = 1.0 / c[0];
            for (int m = 1; m <= 6; ++m) c[m] *= inv;
            for (int m = 7; m <= 9; ++m) c[m] = 2.0 * c[m] * inv;
            double t = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
            t = t + t - c[4] - c[5] - c[6];
            const double qx = c[10] * inv + (t - c[4] - c[4]) * c[1] - c[7] * c[2] - c[8] * c[3];
            const double qy = c[11] * inv - c[7] * c[1] + (t - c[5] - c[5]) * c[2] - c[9] * c[3];
            const double qz = c[12] * inv - c[8] * c[1] - c[9] * c[2] + (t - c[6] - c[6]) * c[3];
            c[10] = qx;
            c[11] = qy;
            c[12] = qz;
        } else {
            for (int m = 0; m < kNM; ++m) c[m] = 0.0;
        }
        const bool edge_y = j == 0 || j == kp.ncy;
        const bool edge_x = !kp.periodic && (i == 0 || i == kp.ncx);
        if (edge_y && edge_x) c[0] *= 4.0;
        else if (edge_y || edge_x) c[0] *= 2.0;
        for (int m = 0; m < kNM; ++m) out[m * nref + r] = (float)c[m];
    }
}

}  // namespace

extern "C" int edp_collect_moments(edp_ctx* c, int species, float* out)
{
    if (!c || !out || species < 0 || species >= c->nspec) return EDP_ERR_ARG;
    if (!c->uploaded[species]) return edp_fail(c, EDP_ERR_STATE, "species not uploaded");
    const edp_kparams& kp = c->kp;
    const int64_t nn = (int64_t)kp.nxg * kp.nyg;
    const int wout = kp.periodic ? c->p.ncx + 2 : c->p.ncx + 1;
    const int64_t nref = (int64_t)wout * kp.nyg;
    double* sum = nullptr;
    float* dout = nullptr;
    EDP_CUDA(c, cudaMallocAsync(&sum, kNM * nn * sizeof(double), c->stream));
    EDP_CUDA(c, cudaMallocAsync(&dout, kNM * nref * sizeof(float), c->stream));
    EDP_CUDA(c, cudaMemsetAsync(sum, 0, kNM * nn * sizeof(double), c->stream));
    MomArgs a;
    memset(&a, 0, sizeof(a));
    a.kp = kp;
    a.precision = c->p.precision;
    a.m = c->pm[species];
    a.d = c->pd[species];
    a.n_slots = &c->dc->n_slots[species];
    a.electron = species == 0;
    a.E2 = c->E2;
    a.Ex = c->Ex;
    a.Ey = c->Ey;
    for (int q = 0; q < 9; ++q) a.K[q] = c->K[0][q];
    a.ez = c->p.ez;
    a.sum = sum;
    ++c->launches;
    if (c->p.precision == EDP_PREC_MIXED) {
        a.chunks = c->chunks[species];
        a.n_chunks = c->n_chunks[species];
        a.tail_start = c->sorted_end[species];
        int64_t tail = c->host_slots[species] - c->sorted_end[species];
        a.tail_ctas = std::max<int64_t>(1, std::min<int64_t>((tail + 1023) / 1024, 148 * 8));
        moments_mixed_kernel<<<(unsigned)(a.n_chunks + a.tail_ctas), 256, 0, c->stream>>>(a);
    } else {
        int64_t g = std::max<int64_t>(1, std::min<int64_t>((c->host_slots[species] + 255) / 256, 148 * 32));
        moments_fp64_kernel<<<(unsigned)g, 256, 0, c->stream>>>(a);
    }
    ++c->launches;
    moments_finish_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((nref + 255) / 256, 148 * 8)), 256, 0,
                            c->stream>>>(kp, sum, wout, dout);
    EDP_CUDA(c, cudaGetLastError());
    EDP_CUDA(c, cudaMemcpyAsync(out, dout, kNM * nref * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaFreeAsync(sum, c->stream));
    EDP_CUDA(c, cudaFreeAsync(dout, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    return EDP_OK;
}
