// FFT_X Poisson solve that allocates no memory, for callers that cannot allocate device memory themselves.
//
// A Fortran host embedded in a larger code often does not own the GPU allocator: the device memory belongs to
// another runtime (a coupled solver, a memory pool, a framework that forbids allocation after start-up), or the
// call has to be made where an allocation would stall or fail. edp_poisson_fftx_noalloc serves those callers: it
// takes the charge density and returns the potential in buffers the caller already owns, and keeps its own
// workspace (spectrum, elimination coefficients, twiddles) in one file-scope device array of fixed size,
// EDP_NOALLOC_SCRATCH_BYTES, which every GPU that loads this library holds until the process exits.
//
// Because every call shares that array, calls that overlap on the GPU (different streams, or different host
// threads on the same device) race on it: order them on one stream. Each call rewrites all the workspace it
// reads, so nothing is carried over from the previous call.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "edp_internal.cuh"

#define EDP_NOALLOC_MAX_DEVICES 64

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[EDP_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[EDP_NOALLOC_MAX_DEVICES] = {nullptr};

// host-side set-up, once per device with that device current: the array's name is only a host-side stand-in,
// the kernels need the device address. The address is kept for the life of the process; cudaDeviceReset would
// make it stale, which the header tells callers.
int scratch_address(void** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= EDP_NOALLOC_MAX_DEVICES) return EDP_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return EDP_ERR_CUDA;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return EDP_OK;
}

__device__ __forceinline__ double2 cmul2(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ int brev(int v, int logn) { return (int)(__brev((unsigned)v) >> (32 - logn)); }

// twiddles exp(+2 pi i k / N), k < N/2
__global__ void na_twiddles(int N, double2* tw)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < N / 2) {
        double s, c;
        sincospi(2.0 * (double)k / (double)N, &s, &c);
        tw[k] = make_double2(c, s);
    }
}

__device__ void na_fft(double2* x, int N, const double2* tw, int sign)
{
    for (int len = 2; len <= N; len <<= 1) {
        const int half = len >> 1, stride = N / len;
        for (int b = threadIdx.x; b < N / 2; b += blockDim.x) {
            int grp = b / half, k = b - grp * half;
            int a = grp * len + k, c = a + half;
            double2 w = tw[k * stride];
            if (sign < 0) w.y = -w.y;
            double2 t = cmul2(w, x[c]);
            double2 u = x[a];
            x[a] = make_double2(u.x + t.x, u.y + t.y);
            x[c] = make_double2(u.x - t.x, u.y - t.y);
        }
        __syncthreads();
    }
}

// row j of the reference-layout density (ncx+2 columns): xband(0) = c_rho(N), xband(1:N-1) = c_rho(1:N-1);
// metal wall rows carry their potential (SOLVE_POISSON_FFTX_LINSYSY, pic2d_ElectricFieldCalc_FFT_X.f90:101-262)
__global__ void na_forward(int N, int J, int logn, int nm, const double* rho, double phi_bottom, double phi_top,
                           const double2* tw, double2* spec)
{
    extern __shared__ double2 x[];
    const int j = blockIdx.x, w = N + 2;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double v = rho[(int64_t)j * w + (i == 0 ? N : i)];
        if (j == 0) v = phi_bottom;
        if (j == J) v = phi_top;
        x[brev(i, logn)] = make_double2(v, 0.0);
    }
    __syncthreads();
    na_fft(x, N, tw, +1);
    for (int m = threadIdx.x; m < nm; m += blockDim.x) {
        double2 v = x[m];
        if (m == 0 || m == N / 2) v.y = 0.0;
        spec[(int64_t)j * nm + m] = v;
    }
}

// per-mode tridiagonal solve with the spectral diagonal -2 - 4 pi^2 m^2/N^2 and the elimination coefficients
// a_eq of PREPARE_SYS_Y (pic2d_Prepare_FFTX_SYSY.f90:834-899) formed during the forward sweep, metal walls
__global__ void na_thomas(int N, int J, int nm, double* aeq, double2* spec)
{
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nm) return;
    const double PI = 3.141592653589793;
    const double d = -2.0 - 4.0 * PI * PI * (double)m * (double)m / ((double)N * (double)N);
    double a = 0.0;
    aeq[m] = 0.0;
    double2 prev = spec[m];
    for (int j = 1; j <= J - 1; ++j) {
        a = 1.0 / (d - a);
        aeq[(int64_t)j * nm + m] = a;
        double2 y = spec[(int64_t)j * nm + m];
        prev = make_double2((-y.x - prev.x) * a, (-y.y - prev.y) * a);
        spec[(int64_t)j * nm + m] = prev;
    }
    double2 next = spec[(int64_t)J * nm + m];
    for (int j = J - 1; j >= 0; --j) {
        double aj = (j == 0) ? 0.0 : aeq[(int64_t)j * nm + m];
        double2 r = spec[(int64_t)j * nm + m];
        next = make_double2(r.x - aj * next.x, r.y - aj * next.y);
        spec[(int64_t)j * nm + m] = next;
    }
}

__global__ void na_inverse(int N, int logn, int nm, const double2* spec, const double2* tw, double* phi)
{
    extern __shared__ double2 x[];
    const int j = blockIdx.x, w = N + 2;
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        double2 v;
        if (m < nm) v = spec[(int64_t)j * nm + m];
        else {
            v = spec[(int64_t)j * nm + (N - m)];
            v.y = -v.y;
        }
        x[brev(m, logn)] = v;
    }
    __syncthreads();
    na_fft(x, N, tw, -1);
    const double inv = 1.0 / N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) phi[(int64_t)j * w + i] = x[i].x * inv;
    __syncthreads();
    if (threadIdx.x == 0) {
        phi[(int64_t)j * w + N] = x[0].x * inv;       // periodic copies of the overlap columns
        phi[(int64_t)j * w + N + 1] = x[1].x * inv;
    }
}

}  // namespace

extern "C" int edp_poisson_fftx_noalloc(int32_t ncx, int32_t ncy, const double* rho_dev, double phi_bottom,
                                        double phi_top, double* phi_dev, void* stream)
{
    if (ncx < 4 || ncy < 2 || (ncx & (ncx - 1)) != 0 || ncx > 4096 || !rho_dev || !phi_dev) return EDP_ERR_ARG;
    // an error left pending by the caller's earlier work is reported here, before anything is queued, and stays
    // pending; the status returned at the end then belongs to this call's own launches
    if (cudaPeekAtLastError() != cudaSuccess) return EDP_ERR_CUDA;
    const int nm = ncx / 2 + 1;
    // workspace sections, each starting on a 256-byte boundary (double2 accesses need 16-byte alignment)
    auto align256 = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t spec_bytes = (size_t)(ncy + 1) * nm * sizeof(double2);
    const size_t aeq_bytes = (size_t)(ncy + 1) * nm * sizeof(double);
    const size_t tw_bytes = (size_t)(ncx / 2) * sizeof(double2);
    const size_t aeq_off = align256(spec_bytes);
    const size_t tw_off = align256(aeq_off + aeq_bytes);
    const size_t need = tw_off + tw_bytes;
    if (need > (size_t)EDP_NOALLOC_SCRATCH_BYTES) return EDP_ERR_CAPACITY;
    void* base = nullptr;
    int r = scratch_address(&base);
    if (r != EDP_OK) return r;
    double2* spec = reinterpret_cast<double2*>(base);
    double* aeq = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + aeq_off);
    double2* tw = reinterpret_cast<double2*>(static_cast<unsigned char*>(base) + tw_off);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int logn = 0;
    while ((1 << logn) < ncx) ++logn;
    const size_t smem = (size_t)ncx * sizeof(double2);
    if (smem > 48 * 1024) {
        if (cudaFuncSetAttribute(na_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaFuncSetAttribute(na_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return EDP_ERR_CUDA;
    }
    const int thr = ncx / 2 < 32 ? 32 : (ncx / 2 > 512 ? 512 : ncx / 2);
    na_twiddles<<<(ncx / 2 + 255) / 256, 256, 0, s>>>(ncx, tw);
    na_forward<<<ncy + 1, thr, smem, s>>>(ncx, ncy, logn, nm, rho_dev, phi_bottom, phi_top, tw, spec);
    na_thomas<<<(nm + 127) / 128, 128, 0, s>>>(ncx, ncy, nm, aeq, spec);
    na_inverse<<<ncy + 1, thr, smem, s>>>(ncx, logn, nm, spec, tw, phi_dev);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}
