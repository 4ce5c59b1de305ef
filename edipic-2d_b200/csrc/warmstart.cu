// Learned warm start of the CG solve (no counterpart in the reference, whose PETSc solve starts from zero):
// the encoder-decoder of nn.cu run on the residual of the previous potential. The network sees the node grid as
// an image padded to multiples of 64 (three 4x4 poolings): channel 0 = r0 / s at unknown nodes, channel 1 = 1 at
// Dirichlet nodes and padding, channels 2..31 = 0; its two FP32 heads o0, o1 give the guess phi_prev + s (K o0 + o1)
// at unknown nodes (s = RMS of r0 over the unknowns, K = L^2 / (2 pi^2)). The guess is used only when its residual is
// smaller than the previous potential's; CG then iterates to the same tolerance either way.
#include "edp_internal.cuh"

#include <cuda_bf16.h>

#include <cmath>
#include <vector>

typedef __nv_bfloat16 bf16;

struct edp_warmstart {
    int H = 0, W = 0;
    double K = 1.0;
    int64_t n_unknown = 0;
    bf16* w[EDP_WARMSTART_N_CONV] = {nullptr};
    float* b[EDP_WARMSTART_N_CONV] = {nullptr};
    float* wh = nullptr;       // two heads, each [9][32] then the bias
    // activations (NHWC BF16)
    bf16 *in = nullptr, *e0 = nullptr, *s0 = nullptr, *p0 = nullptr, *e1 = nullptr, *s1 = nullptr, *p1 = nullptr;
    bf16 *e2 = nullptr, *s2 = nullptr, *p2 = nullptr, *ba = nullptr, *bb = nullptr, *u2 = nullptr, *d2a = nullptr;
    bf16 *d2b = nullptr, *u1 = nullptr, *d1a = nullptr, *d1b = nullptr, *u0 = nullptr, *d0a = nullptr, *d0b = nullptr;
    float* out = nullptr;      // head 0 (smooth, scaled by K)
    float* out1 = nullptr;     // head 1 (grid scale)
    double* guess = nullptr;   // node grid
    double* r1 = nullptr;
    double* p1n = nullptr;
    double* scal = nullptr;    // [0] |r0|^2, [1] |r1|^2
};

namespace {

const int kLayers[EDP_WARMSTART_N_CONV][2] = EDP_WARMSTART_LAYERS;

__global__ void ws_input_kernel(edp_kparams kp, const int8_t* __restrict__ kind, const double* __restrict__ r0,
                                const double* __restrict__ rr0, double n_unknown, int H, int W, bf16* __restrict__ in)
{
    const double s = (*rr0 > 0.0) ? sqrt(*rr0 / n_unknown) : 1.0;
    const float inv = (float)(1.0 / s);
    const int64_t npix = (int64_t)H * W;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % W), y = (int)(p / W);
        float v0 = 0.0f, v1 = 1.0f;
        if (x < kp.nxg && y < kp.nyg) {
            const int64_t q = (int64_t)y * kp.nxg + x;
            if (!kind[q]) {
                v0 = (float)r0[q] * inv;
                v1 = 0.0f;
            }
        }
        uint4* dst = reinterpret_cast<uint4*>(in + p * 32);
        __nv_bfloat162 h01 = __floats2bfloat162_rn(v0, v1);
        uint4 first = make_uint4(*reinterpret_cast<uint32_t*>(&h01), 0u, 0u, 0u);
        dst[0] = first;
        dst[1] = make_uint4(0u, 0u, 0u, 0u);
        dst[2] = make_uint4(0u, 0u, 0u, 0u);
        dst[3] = make_uint4(0u, 0u, 0u, 0u);
    }
}

__global__ void ws_guess_kernel(edp_kparams kp, const int8_t* __restrict__ kind, const double* __restrict__ phi,
                                const float* __restrict__ out, const float* __restrict__ out1,
                                const double* __restrict__ rr0, double n_unknown, double K, int W,
                                double* __restrict__ guess)
{
    const double s = (*rr0 > 0.0) ? sqrt(*rr0 / n_unknown) : 1.0;
    const int64_t n = (int64_t)kp.nxg * kp.nyg;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % kp.nxg), j = (int)(q / kp.nxg);
        const int64_t pix = (int64_t)j * W + i;
        guess[q] = kind[q] ? phi[q] : phi[q] + s * (K * (double)out[pix] + (double)out1[pix]);
    }
}

__device__ __forceinline__ double block_sum_d(double v)
{
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    return v;
}

// r = b - A x over the unknowns (A = 4 - neighbours, Dirichlet neighbours eliminated into b), p = r, |r|^2
__global__ void ws_residual_kernel(edp_kparams kp, const int8_t* __restrict__ kind, const double* __restrict__ x,
                                   const double* __restrict__ b, double* __restrict__ r, double* __restrict__ p,
                                   double* rr)
{
    const int64_t n = (int64_t)kp.nxg * kp.nyg;
    const int64_t w = kp.nxg;
    double acc = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        if (kind[q]) {
            r[q] = 0.0;
            p[q] = 0.0;
            continue;
        }
        double s = 4.0 * x[q];
        if (!kind[q - 1]) s -= x[q - 1];
        if (!kind[q + 1]) s -= x[q + 1];
        if (!kind[q - w]) s -= x[q - w];
        if (!kind[q + w]) s -= x[q + w];
        const double v = b[q] - s;
        r[q] = v;
        p[q] = v;
        acc += v * v;
    }
    acc = block_sum_d(acc);
    if (threadIdx.x == 0) atomicAdd(rr, acc);
}

unsigned grid_n(int64_t n)
{
    int64_t g = (n + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    return (unsigned)(g < 1 ? 1 : g);
}

int conv(edp_ctx* c, int layer, int h, int w, const bf16* x1, int c1, const bf16* x2, int c2, bf16* y)
{
    edp_warmstart* ws = c->ws;
    ++c->launches;
    const int r = edp_nn_conv3x3_fwd(1, h, w, x1, c1, x2, c2, ws->w[layer], ws->b[layer], kLayers[layer][1], 1, y,
                                     c->stream);
    return r == EDP_OK ? EDP_OK : edp_fail(c, r, "warm-start convolution");
}

}  // namespace

void edp_warmstart_free(edp_ctx* c)
{
    edp_warmstart* ws = c->ws;
    if (!ws) return;
    for (int l = 0; l < EDP_WARMSTART_N_CONV; ++l) {
        cudaFree(ws->w[l]);
        cudaFree(ws->b[l]);
    }
    void* bufs[] = {ws->wh, ws->in, ws->e0, ws->s0, ws->p0, ws->e1, ws->s1, ws->p1, ws->e2, ws->s2, ws->p2, ws->ba,
                    ws->bb, ws->u2, ws->d2a, ws->d2b, ws->u1, ws->d1a, ws->d1b, ws->u0, ws->d0a, ws->d0b, ws->out,
                    ws->out1, ws->guess, ws->r1, ws->p1n, ws->scal};
    for (void* q : bufs) cudaFree(q);
    delete ws;
    c->ws = nullptr;
}

// forward pass on the residual in c->cg_r (|r0|^2 at rr0): fills ws->guess
int edp_warmstart_forward(edp_ctx* c, const double* rr0)
{
    edp_warmstart* ws = c->ws;
    const int H = ws->H, W = ws->W;
    const edp_kparams& kp = c->kp;
    ++c->launches;
    ws_input_kernel<<<grid_n((int64_t)H * W), 256, 0, c->stream>>>(kp, c->cg_kind, c->cg_r, rr0, (double)ws->n_unknown,
                                                                   H, W, ws->in);
    TRY(conv(c, 0, H, W, ws->in, 32, nullptr, 0, ws->e0));
    TRY(conv(c, 1, H, W, ws->e0, 32, nullptr, 0, ws->s0));
    c->launches += 1;
    TRY(edp_nn_pool(1, H, W, 32, 4, ws->s0, ws->p0, c->stream));
    TRY(conv(c, 2, H / 4, W / 4, ws->p0, 32, nullptr, 0, ws->e1));
    TRY(conv(c, 3, H / 4, W / 4, ws->e1, 64, nullptr, 0, ws->s1));
    c->launches += 1;
    TRY(edp_nn_pool(1, H / 4, W / 4, 64, 4, ws->s1, ws->p1, c->stream));
    TRY(conv(c, 4, H / 16, W / 16, ws->p1, 64, nullptr, 0, ws->e2));
    TRY(conv(c, 5, H / 16, W / 16, ws->e2, 128, nullptr, 0, ws->s2));
    c->launches += 1;
    TRY(edp_nn_pool(1, H / 16, W / 16, 128, 4, ws->s2, ws->p2, c->stream));
    TRY(conv(c, 6, H / 64, W / 64, ws->p2, 128, nullptr, 0, ws->ba));
    TRY(conv(c, 7, H / 64, W / 64, ws->ba, 256, nullptr, 0, ws->bb));
    c->launches += 1;
    TRY(edp_nn_upsample(1, H / 16, W / 16, 256, 4, ws->bb, ws->u2, c->stream));
    TRY(conv(c, 8, H / 16, W / 16, ws->u2, 256, ws->s2, 128, ws->d2a));
    TRY(conv(c, 9, H / 16, W / 16, ws->d2a, 128, nullptr, 0, ws->d2b));
    c->launches += 1;
    TRY(edp_nn_upsample(1, H / 4, W / 4, 128, 4, ws->d2b, ws->u1, c->stream));
    TRY(conv(c, 10, H / 4, W / 4, ws->u1, 128, ws->s1, 64, ws->d1a));
    TRY(conv(c, 11, H / 4, W / 4, ws->d1a, 64, nullptr, 0, ws->d1b));
    c->launches += 1;
    TRY(edp_nn_upsample(1, H, W, 64, 4, ws->d1b, ws->u0, c->stream));
    TRY(conv(c, 12, H, W, ws->u0, 64, ws->s0, 32, ws->d0a));
    TRY(conv(c, 13, H, W, ws->d0a, 32, nullptr, 0, ws->d0b));
    c->launches += 1;
    TRY(edp_nn_head_fwd(1, H, W, 32, ws->d0b, ws->wh, ws->wh + 9 * 32, ws->out, c->stream));
    c->launches += 1;
    TRY(edp_nn_head_fwd(1, H, W, 32, ws->d0b, ws->wh + 9 * 32 + 1, ws->wh + 2 * 9 * 32 + 1, ws->out1, c->stream));
    ++c->launches;
    ws_guess_kernel<<<grid_n((int64_t)kp.nxg * kp.nyg), 256, 0, c->stream>>>(
        kp, c->cg_kind, c->phi, ws->out, ws->out1, rr0, (double)ws->n_unknown, ws->K, W, ws->guess);
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

// residual of ws->guess into ws->r1 / ws->p1n with |r1|^2 at ws->scal[1]
int edp_warmstart_residual(edp_ctx* c)
{
    edp_warmstart* ws = c->ws;
    EDP_CUDA(c, cudaMemsetAsync(ws->scal + 1, 0, sizeof(double), c->stream));
    ++c->launches;
    ws_residual_kernel<<<grid_n((int64_t)c->kp.nxg * c->kp.nyg), 256, 0, c->stream>>>(c->kp, c->cg_kind, ws->guess,
                                                                                     c->cg_b, ws->r1, ws->p1n,
                                                                                     ws->scal + 1);
    EDP_CUDA(c, cudaGetLastError());
    return EDP_OK;
}

const double* edp_warmstart_rr(edp_ctx* c) { return c->ws->scal + 1; }

// the guess becomes the CG start: potential, residual, first direction and |r|^2
cudaError_t edp_warmstart_accept(edp_ctx* c, double* rr_dst)
{
    edp_warmstart* ws = c->ws;
    const size_t nb = (size_t)c->kp.nxg * c->kp.nyg * sizeof(double);
    cudaError_t e = cudaMemcpyAsync(c->phi, ws->guess, nb, cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->cg_r, ws->r1, nb, cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->cg_p, ws->p1n, nb, cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rr_dst, ws->scal + 1, sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    return e;
}

const double* edp_warmstart_guess(edp_ctx* c) { return c->ws->guess; }

extern "C" int edp_warmstart_load(edp_ctx* c, const float* blob, int64_t n)
{
    if (!c || !blob) return EDP_ERR_ARG;
    if (c->p.solver != EDP_SOLVER_CG) return edp_fail(c, EDP_ERR_STATE, "the learned warm start is for CG contexts");
    int64_t need = 2 * (9 * 32 + 1);
    for (int l = 0; l < EDP_WARMSTART_N_CONV; ++l) need += (int64_t)9 * kLayers[l][0] * kLayers[l][1] + kLayers[l][1];
    if (n != need) return edp_fail(c, EDP_ERR_ARG, "warm-start parameter count does not match the network");
    edp_warmstart_free(c);
    edp_warmstart* ws = new edp_warmstart();
    c->ws = ws;
    const edp_kparams& kp = c->kp;
    ws->H = (kp.nyg + 63) / 64 * 64;
    ws->W = (kp.nxg + 63) / 64 * 64;
    const double L = (double)std::max(c->p.ncx, c->p.ncy);
    ws->K = L * L / (2.0 * 3.141592653589793 * 3.141592653589793);
    // unknown nodes: not on a wall, not in an inner object
    int64_t nu = 0;
    for (int j = 1; j < c->p.ncy; ++j)
        for (int i = 1; i < c->p.ncx; ++i) {
            bool in = false;
            for (int o = 0; o < c->p.n_inner; ++o)
                if (i >= c->p.inner_ileft[o] && i <= c->p.inner_iright[o] && j >= c->p.inner_jbottom[o] &&
                    j <= c->p.inner_jtop[o])
                    in = true;
            nu += in ? 0 : 1;
        }
    ws->n_unknown = nu > 0 ? nu : 1;
    const float* q = blob;
    for (int l = 0; l < EDP_WARMSTART_N_CONV; ++l) {
        const int64_t nw = (int64_t)9 * kLayers[l][0] * kLayers[l][1];
        std::vector<bf16> hw(nw);
        for (int64_t k = 0; k < nw; ++k) hw[k] = __float2bfloat16(q[k]);
        q += nw;
        EDP_CUDA(c, cudaMalloc(&ws->w[l], nw * sizeof(bf16)));
        EDP_CUDA(c, cudaMemcpy(ws->w[l], hw.data(), nw * sizeof(bf16), cudaMemcpyHostToDevice));
        EDP_CUDA(c, cudaMalloc(&ws->b[l], kLayers[l][1] * sizeof(float)));
        EDP_CUDA(c, cudaMemcpy(ws->b[l], q, kLayers[l][1] * sizeof(float), cudaMemcpyHostToDevice));
        q += kLayers[l][1];
    }
    EDP_CUDA(c, cudaMalloc(&ws->wh, 2 * (9 * 32 + 1) * sizeof(float)));
    EDP_CUDA(c, cudaMemcpy(ws->wh, q, 2 * (9 * 32 + 1) * sizeof(float), cudaMemcpyHostToDevice));
    const int64_t p0 = (int64_t)ws->H * ws->W, p1 = p0 / 16, p2 = p0 / 256, p3 = p0 / 4096;
    auto act = [&](bf16** ptr, int64_t pix, int ch) -> int {
        EDP_CUDA(c, cudaMalloc(ptr, pix * ch * sizeof(bf16)));
        return EDP_OK;
    };
    TRY(act(&ws->in, p0, 32));
    TRY(act(&ws->e0, p0, 32));
    TRY(act(&ws->s0, p0, 32));
    TRY(act(&ws->p0, p1, 32));
    TRY(act(&ws->e1, p1, 64));
    TRY(act(&ws->s1, p1, 64));
    TRY(act(&ws->p1, p2, 64));
    TRY(act(&ws->e2, p2, 128));
    TRY(act(&ws->s2, p2, 128));
    TRY(act(&ws->p2, p3, 128));
    TRY(act(&ws->ba, p3, 256));
    TRY(act(&ws->bb, p3, 256));
    TRY(act(&ws->u2, p2, 256));
    TRY(act(&ws->d2a, p2, 128));
    TRY(act(&ws->d2b, p2, 128));
    TRY(act(&ws->u1, p1, 128));
    TRY(act(&ws->d1a, p1, 64));
    TRY(act(&ws->d1b, p1, 64));
    TRY(act(&ws->u0, p0, 64));
    TRY(act(&ws->d0a, p0, 32));
    TRY(act(&ws->d0b, p0, 32));
    const int64_t nn = (int64_t)kp.nxg * kp.nyg;
    EDP_CUDA(c, cudaMalloc(&ws->out, p0 * sizeof(float)));
    EDP_CUDA(c, cudaMalloc(&ws->out1, p0 * sizeof(float)));
    EDP_CUDA(c, cudaMalloc(&ws->guess, nn * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&ws->r1, nn * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&ws->p1n, nn * sizeof(double)));
    EDP_CUDA(c, cudaMalloc(&ws->scal, 2 * sizeof(double)));
    return EDP_OK;
}
