// Kernels of the learned warm start of the CG solve: a 4-level convolutional encoder-decoder that maps the
// residual of the previous potential against the new charge density to a potential update.
//
// Tensors are NHWC: activations BF16 [images][h][w][channels], 3x3 convolution weights BF16 [c_out][3][3][c_in]
// (tap = 3 ky + kx, offsets ky - 1, kx - 1), biases and all gradients of weights FP32. Convolutions are implicit
// GEMMs on the BF16 tensor cores with FP32 accumulation; the forward (and through it the data gradient) runs on
// tcgen05 with TMA-loaded operands and tensor-memory accumulators, the weight gradient on mma.sync:
//   forward  y[p][n]      = act(sum_{tap, c} x[p + off(tap)][c] w[n][tap][c] + b[n])       M = pixels, N = c_out
//   dgrad    dx[p][c]     = sum_{tap', n} dz[p + off(tap')][n] w[n][8 - tap'][c]          (the forward kernel on
//                           the flipped, transposed weight copy)
//   wgrad    dw[n][tap][c] += sum_p dz[p][n] x[p + off(tap)][c]                            M = c_out, K = pixels
// Pixels outside the image read zero (padding 1). The input of a forward convolution may be the channel
// concatenation of two tensors (the decoder's upsampled path and the encoder's skip), read in place.
#include "edp_internal.cuh"

#include <cuda.h>
#include <cuda_bf16.h>

#include <mutex>
#include <vector>

namespace {

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid)
{
    const int sz = valid ? 16 : 0;   // 0: zero-fill the 16 bytes
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(addr));
}

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// byte offset of 16-byte chunk c of row r in a tile whose rows hold `cpr` chunks (4: 64 B rows, 8: 128 B rows);
// the XOR spreads the 8 rows an ldmatrix reads over all 32 banks
__device__ __forceinline__ int swz(int r, int c, int cpr)
{
    const int x = cpr == 8 ? (r & 7) : ((r >> 1) & 3);
    return r * cpr * 16 + ((c ^ x) << 4);
}

// ------------------------------------------------------------------------------------------ forward / dgrad
struct ConvArgs {
    int nimg, h, w;
    const bf16* x1;   // [P][c1]
    int c1;
    const bf16* x2;   // [P][c2] or null
    int c2;
    const bf16* wt;   // [cout][9][c1 + c2]
    const float* bias;
    int cout;
    int relu;
    bf16* y;          // [P][cout]
};

constexpr int kStages = 3;   // cp.async pipeline depth of the weight-gradient kernel

// ------------------------------------------------------------------------------------------ tcgen05 helpers
constexpr int kTcThreads = 256;
constexpr long long kSpinLimit = 1LL << 22;   // try_wait polls; a healthy wait ends far sooner

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (long long it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P;\n\t}\n"
                     : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// ------------------------------------------------------------------------------------------ forward on TMA + tcgen05
// The same implicit GEMM with both operands brought in by the tensor memory access unit. A CTA owns a 16 x 8-pixel
// patch of one image (128 rows of A) and BN output channels. K runs in chunks of CW channels of one tap
// (CW = 64, or 32 when c_in or the concatenation split is not a multiple of 64): A is the 4-D box
// (CW channels, 16 x, 8 y, 1 image) at (c, x0 + dx, y0 + dy, n) of the NHWC activations, zero-filled where the
// patch leaves the image, B the 2-D box (CW, BN) at (k, n0) of the [c_out][9 c_in] weights; both arrive in the
// K-major swizzled layout the MMA descriptors name (128-byte swizzle for CW = 64, 64-byte for CW = 32). Thread 0
// issues the copies (expect-tx on the stage's full barrier) and the MMAs (committed to the stage's empty barrier);
// the other warps join for the epilogue. Every wait is bounded.
struct TmaArgs {
    int nimg, h, w, c1, c2, cout, relu, tiles_x, tiles_y;
    const float* bias;
    bf16* y;
    int* err;
    float* ws;   // split K (gridDim.z slices): FP32 partial sums [slice][P][cout], summed by conv_finish_kernel
};

template <int BN, int CW>
__global__ void __launch_bounds__(kTcThreads, 1)
    conv3x3_fwd_tma_kernel(const __grid_constant__ CUtensorMap mx1, const __grid_constant__ CUtensorMap mx2,
                           const __grid_constant__ CUtensorMap mw, TmaArgs ta)
{
    edp_dependent_start();
    constexpr int STAGES = 4;
    constexpr int A_BYTES = 128 * CW * 2, B_BYTES = BN * CW * 2, STAGE = A_BYTES + B_BYTES;
    constexpr uint32_t TMEM_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((128u >> 4) << 24);
    // K-major descriptor: 8-row atoms of 8 x (CW * 2) bytes, layout 2 = 128-byte swizzle, 4 = 64-byte swizzle
    constexpr uint64_t DESC_HI = ((uint64_t)((8 * CW * 2) >> 4) << 32) | ((uint64_t)1 << 46) |
                                 ((uint64_t)(CW == 64 ? 2 : 4) << 61) | ((uint64_t)1 << 16);
    extern __shared__ unsigned char dsm[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
    __shared__ uint32_t tmem_base_sh;
    __shared__ int fail_sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (smem_u32(dsm) + 1023u) & ~1023u;
    const int tile = blockIdx.x;
    const int tx = tile % ta.tiles_x, ty = (tile / ta.tiles_x) % ta.tiles_y, img = tile / (ta.tiles_x * ta.tiles_y);
    const int x0 = tx * 16, y0 = ty * 8;
    const int n0 = blockIdx.y * BN;
    const int cin = ta.c1 + ta.c2;
    // K slice of this CTA (the whole K range unless the layer is split over gridDim.z slices)
    const int KT_all = 9 * cin / CW;
    const int kbeg = (int)(((int64_t)blockIdx.z * KT_all) / gridDim.z);
    const int KT = (int)(((int64_t)(blockIdx.z + 1) * KT_all) / gridDim.z) - kbeg;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        fail_sh = 0;
        for (int s = 0; s < STAGES; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[s])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    if (tid == 0) {
        auto issue = [&](int kt) {
            const int s = kt % STAGES;
            const uint32_t As = base + s * STAGE, Bs = As + A_BYTES, fb = smem_u32(&full[s]);
            const int k0 = (kbeg + kt) * CW, tap = k0 / cin, ci = k0 - tap * cin;
            const int xx = x0 + tap % 3 - 1, yy = y0 + tap / 3 - 1;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"(STAGE) : "memory");
            const CUtensorMap* ma = ci < ta.c1 ? &mx1 : &mx2;
            const int ca = ci < ta.c1 ? ci : ci - ta.c1;
            asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
                         ::"r"(As), "l"(ma), "r"(ca), "r"(xx), "r"(yy), "r"(img), "r"(fb) : "memory");
            asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                         ::"r"(Bs), "l"(&mw), "r"(k0), "r"(n0), "r"(fb) : "memory");
        };
        int issued = 0;
        for (; issued < STAGES - 1 && issued < KT; ++issued) issue(issued);
        int kt = 0;
        for (; kt < KT; ++kt) {
            const int s = kt % STAGES;
            if (!mbar_wait(smem_u32(&full[s]), (uint32_t)((kt / STAGES) & 1))) {
                fail_sh = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t As = base + s * STAGE, Bs = As + A_BYTES;
            for (int ks = 0; ks < CW / 16; ++ks) {
                const uint64_t da = DESC_HI | (uint64_t)(((As + 32 * ks) >> 4) & 0x3FFFu);
                const uint64_t db = DESC_HI | (uint64_t)(((Bs + 32 * ks) >> 4) & 0x3FFFu);
                const uint32_t acc = (kt > 0 || ks > 0) ? 1u : 0u;
                asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                             ::"r"(tmem), "l"(da), "l"(db), "r"(IDESC), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         ::"r"(smem_u32(&empty[s])) : "memory");
            if (issued < KT) {   // chunk `issued` reuses the stage of chunk issued - STAGES = kt - 1
                const int old = issued - STAGES;
                if (old >= 0 && !mbar_wait(smem_u32(&empty[old % STAGES]), (uint32_t)((old / STAGES) & 1))) {
                    fail_sh = 1;
                    ++kt;
                    break;
                }
                issue(issued++);
            }
        }
        // copies in flight and the last MMAs finish before the epilogue reads or the CTA leaves
        for (int q = kt; q < issued; ++q) mbar_wait(smem_u32(&full[q % STAGES]), (uint32_t)((q / STAGES) & 1));
        if (kt > 0 && !mbar_wait(smem_u32(&empty[(kt - 1) % STAGES]), (uint32_t)(((kt - 1) / STAGES) & 1)))
            fail_sh = 2;
        if (fail_sh) atomicExch(ta.err, 1);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (fail_sh == 0) {
        // epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (patch rows), column half w / 4
        const int wl = warp & 3, wh = warp >> 2;
        const int cols = BN / 2;
        const int r = wl * 32 + lane;
        const int px = x0 + (r & 15), py = y0 + (r >> 4);
        const bool inside = px < ta.w && py < ta.h;
        const int64_t p = ((int64_t)img * ta.h + py) * ta.w + px;
        for (int c0 = wh * cols; c0 < (wh + 1) * cols; c0 += 16) {
            uint32_t v[16];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15},"
                         " [%16];\n"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                           "=r"(v[14]), "=r"(v[15])
                         : "r"(tmem + ((uint32_t)(wl * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (inside && ta.ws) {
                const int64_t P = (int64_t)ta.nimg * ta.h * ta.w;
                float4* d = reinterpret_cast<float4*>(ta.ws + ((int64_t)blockIdx.z * P + p) * ta.cout + n0 + c0);
                for (int q = 0; q < 4; ++q)
                    d[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                                       __uint_as_float(v[4 * q + 2]), __uint_as_float(v[4 * q + 3]));
            } else if (inside) {
                uint32_t pk[8];
                for (int q = 0; q < 8; ++q) {
                    const int n = n0 + c0 + 2 * q;
                    float v0 = __uint_as_float(v[2 * q]) + (ta.bias ? ta.bias[n] : 0.0f);
                    float v1 = __uint_as_float(v[2 * q + 1]) + (ta.bias ? ta.bias[n + 1] : 0.0f);
                    if (ta.relu) {
                        v0 = fmaxf(v0, 0.0f);
                        v1 = fmaxf(v1, 0.0f);
                    }
                    __nv_bfloat162 h2 = __floats2bfloat162_rn(v0, v1);
                    pk[q] = *reinterpret_cast<uint32_t*>(&h2);
                }
                uint4* dst = reinterpret_cast<uint4*>(ta.y + p * ta.cout + n0 + c0);
                dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// ------------------------------------------------------------------------------------------ persistent halo forward
// The same convolution as a persistent, warp-specialised kernel for the layers with many pixels and few channels.
// A tile is an 8 x 16-pixel patch (M = 128 rows of the implicit GEMM, row r = pixel (r % 8, r / 8)). Its input is
// brought in ONCE as a 10 x 18-pixel halo and serves all nine taps: the halo of a 32-channel chunk lies in shared
// memory as four planes of 8 channels, plane s holding pixel q at byte 16 q (the canonical K-major layout without
// swizzle: core matrices of 8 pixels x 16 bytes), so the A operand of tap (dx, dy) is the same planes read from
// pixel 10 dy + dx on: stride between 8-row groups (SBO) = one halo row = 160 bytes, between the two 8-channel
// halves of a K step (LBO) = one plane (planes 128-byte aligned for the TMA copies; in the weight gradient, whose
// halo is copied by cp.async, padded instead so that the 16-byte writes of eight lanes, two pixels x four planes,
// hit all 32 banks). The weights of the whole layer stay in shared memory (loaded once by TMA, 64-byte
// swizzle, one (32, c_out) box per tap and chunk).
// Roles: warp 0, lane 0, copies each halo by TMA, one (8 channels, 10, 18) box per plane, zero-filled off the image,
// into a ring of stages (expect-tx on the stage's full barrier); warp 1, lane 0, loads the weights and issues the
// MMAs (tcgen05.mma, accumulators in one of two tensor-memory buffers, committed to the stage's empty barrier and,
// after the tile's last chunk, to the buffer's full barrier); warps 2-5 (one per quarter of the tensor-memory lanes)
// read the accumulators back (tcgen05.ld), add them and the bias, apply ReLU and store BF16, then release the buffer.
// Tiles are taken round-robin by the persistent CTAs, so the next tile's copies and MMAs overlap this tile's
// epilogue. Every wait is bounded; a wait that gives up sets the error word and stops every role.
constexpr int kHaloThreads = 224;     // weight gradient: 2 copy warps, 1 MMA warp, 4 epilogue warps
constexpr int kHaloMmaWarp = 1;       // forward halo kernel: the TMA warp, the MMA warp, 4 epilogue warps
constexpr int kHaloFwdThreads = 192;
constexpr int kHaloStages = 4;
constexpr int kHaloBoxBytes = 180 * 16;               // one plane of the halo: 10 x 18 pixels x 8 channels
constexpr int kHaloPlane = 2944;                      // plane stride: 184 pixel slots, 128-byte aligned (TMA)
constexpr int kHaloStage = 4 * kHaloPlane;            // one 32-channel chunk
constexpr int kHaloStagePad = 12288;                  // the halo rounded up to 1 KiB: streamed weights follow it
constexpr int kWgPlane = 2912;                        // weight gradient (cp.async): 182 slots, bank-spread writes
constexpr int kWgHaloStage = 4 * kWgPlane;
constexpr int kHaloMaxWeights = 112 * 1024;           // largest resident weight set (9 x c_in x c_out x 2 bytes)
template <int BN>
constexpr int kHaloAcc = BN == 128 ? 1 : 2;   // partial accumulators per tile
template <int BN>
constexpr int kHaloTmemCols = 2 * kHaloAcc<BN> * BN <= 128 ? 128 : 256;   // two tiles' accumulators

struct HaloArgs {
    const bf16* x1;
    const bf16* x2;
    int c1, c2, nimg, h, w, cout, relu, tiles_x, tiles_y;
    int64_t n_tiles;
    const float* bias;
    bf16* y;
    int* err;
};

__device__ __forceinline__ bool mbar_wait_or_fail(uint32_t bar, uint32_t parity, volatile int* fail)
{
    for (long long it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P;\n\t}\n"
                     : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
        if ((it & 1023) == 1023 && *fail) return false;
    }
    *fail = 1;
    return false;
}

template <int BN, bool STREAM>
__global__ void __launch_bounds__(kHaloFwdThreads, 1)
    conv3x3_fwd_halo_kernel(const __grid_constant__ CUtensorMap mw, const __grid_constant__ CUtensorMap mx1,
                            const __grid_constant__ CUtensorMap mx2, HaloArgs a)
{
    edp_dependent_start();
    // NACC partial accumulators per tile (tap % NACC), summed in the epilogue: consecutive MMAs of the short (small N)
    // chains go to independent accumulators; two tiles' sets of them (double buffering)
    constexpr int NACC = kHaloAcc<BN>;
    constexpr uint32_t TMEM_COLS = kHaloTmemCols<BN>;
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((128u >> 4) << 24);
    // A: no swizzle, LBO = one plane (K direction), SBO = one halo row of 10 pixels (M direction)
    constexpr uint64_t DESC_A = ((uint64_t)(160 >> 4) << 32) | ((uint64_t)(kHaloPlane >> 4) << 16) | ((uint64_t)1 << 46);
    // B: 64-byte swizzle, 8-row atoms of 64 bytes (SBO = 512 bytes), LBO unused
    constexpr uint64_t DESC_B = ((uint64_t)(512 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)4 << 61) |
                                ((uint64_t)1 << 16);
    constexpr int B_CHUNK = BN * 64;   // bytes of one (tap, chunk) weight box
    // STREAM: the weights do not stay; each stage holds a chunk's halo and the chunk's nine (32, c_out) weight boxes
    constexpr int SST = STREAM ? kHaloStagePad + 9 * B_CHUNK : kHaloStage;
    extern __shared__ unsigned char dsm[];
    __shared__ __align__(8) uint64_t full[kHaloStages], empty[kHaloStages], acc_full[2], acc_empty[2], wbar, done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int fail_sh;
    __shared__ float bias_sh[BN];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cin = a.c1 + a.c2, n_chunks = cin / 32;
    const uint32_t wbase = (smem_u32(dsm) + 1023u) & ~1023u;
    const uint32_t hbase = STREAM ? wbase : wbase + (uint32_t)(9 * n_chunks * B_CHUNK);

    for (int i = tid; i < BN; i += blockDim.x) bias_sh[i] = a.bias ? a.bias[i] : 0.0f;
    if (warp == kHaloMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        fail_sh = 0;
        for (int s = 0; s < kHaloStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[s])));
        }
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&acc_full[b])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;\n" ::"r"(smem_u32(&acc_empty[b])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&wbar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&done_bar)));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base_sh;
    const int64_t stride = gridDim.x;

    if (warp == 0) {
        // ---------------- halo producer (lane 0): four TMA boxes of (8 channels, 10 x, 18 y) per 32-channel chunk,
        // one per plane, zero-filled where the halo leaves the image
        if (lane == 0) {
            int64_t it = 0;
            for (int64_t t = blockIdx.x; t < a.n_tiles && !fail_sh; t += stride) {
                const int tx = (int)(t % a.tiles_x), ty = (int)((t / a.tiles_x) % a.tiles_y);
                const int img = (int)(t / ((int64_t)a.tiles_x * a.tiles_y));
                const int gx0 = tx * 8 - 1, gy0 = ty * 16 - 1;
                bool ok = true;
                for (int cc = 0; cc < n_chunks; ++cc, ++it) {
                    const int s = (int)(it % kHaloStages);
                    if (it >= kHaloStages &&
                        !mbar_wait_or_fail(smem_u32(&empty[s]), (uint32_t)(((it / kHaloStages) - 1) & 1), &fail_sh)) {
                        ok = false;
                        break;
                    }
                    const int c0 = cc * 32;
                    const CUtensorMap* m = c0 < a.c1 ? &mx1 : &mx2;
                    const int co = c0 < a.c1 ? c0 : c0 - a.c1;
                    const uint32_t st = hbase + (uint32_t)(s * SST), fb = smem_u32(&full[s]);
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb),
                                 "r"(4 * kHaloBoxBytes + (STREAM ? 9 * B_CHUNK : 0)) : "memory");
                    if constexpr (STREAM)
                        for (int tap = 0; tap < 9; ++tap)
                            asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                                         ::"r"(st + (uint32_t)(kHaloStagePad + tap * B_CHUNK)), "l"(&mw),
                                           "r"(tap * cin + c0), "r"(0), "r"(fb) : "memory");
                    for (int pl = 0; pl < 4; ++pl)
                        asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
                                     ::"r"(st + (uint32_t)(pl * kHaloPlane)), "l"(m), "r"(co + 8 * pl), "r"(gx0), "r"(gy0),
                                       "r"(img), "r"(fb) : "memory");
                }
                if (!ok) break;
            }
            // copies still in flight (their stages not consumed after a failure) land before the CTA leaves
            for (int64_t q = it > kHaloStages ? it - kHaloStages : 0; q < it; ++q)
                mbar_wait(smem_u32(&full[q % kHaloStages]), (uint32_t)((q / kHaloStages) & 1));
        }
        __syncwarp();
    } else if (warp == kHaloMmaWarp) {
        // ---------------- weights once, then the MMAs (lane 0)
        if (lane == 0) {
            bool ok = true;
            if constexpr (!STREAM) {
                const uint32_t wb = smem_u32(&wbar);
                const uint32_t bytes = (uint32_t)(9 * n_chunks * B_CHUNK);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(wb), "r"(bytes) : "memory");
                for (int k = 0; k < 9 * n_chunks; ++k)
                    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                                 ::"r"(wbase + (uint32_t)(k * B_CHUNK)), "l"(&mw), "r"(k * 32), "r"(0), "r"(wb) : "memory");
                ok = mbar_wait_or_fail(wb, 0u, &fail_sh);
            }
            int64_t it = 0, tl = 0;
            for (int64_t t = blockIdx.x; ok && t < a.n_tiles && !fail_sh; t += stride, ++tl) {
                const int buf = (int)(tl & 1);
                if (tl >= 2 && !mbar_wait_or_fail(smem_u32(&acc_empty[buf]), (uint32_t)(((tl >> 1) - 1) & 1), &fail_sh))
                    break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(buf * NACC * BN);
                for (int cc = 0; cc < n_chunks; ++cc, ++it) {
                    const int s = (int)(it % kHaloStages);
                    if (!mbar_wait_or_fail(smem_u32(&full[s]), (uint32_t)((it / kHaloStages) & 1), &fail_sh)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    const uint32_t As = hbase + (uint32_t)(s * SST);
                    for (int ks = 0; ks < 2; ++ks) {
                        for (int tap = 0; tap < 9; ++tap) {
                            const uint32_t a0 = As + (uint32_t)(((tap / 3) * 10 + tap % 3) * 16);
                            const uint32_t b0 = STREAM ? As + (uint32_t)(kHaloStagePad + tap * B_CHUNK)
                                                       : wbase + (uint32_t)((tap * n_chunks + cc) * B_CHUNK);
                            const uint64_t da = DESC_A | (uint64_t)(((a0 + (uint32_t)(2 * ks * kHaloPlane)) >> 4) & 0x3FFFu);
                            const uint64_t db = DESC_B | (uint64_t)(((b0 + 32u * ks) >> 4) & 0x3FFFu);
                            const uint32_t accum = (cc > 0 || ks > 0 || tap >= NACC) ? 1u : 0u;
                            asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                         "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                                         ::"r"(acc + (uint32_t)((tap % NACC) * BN)), "l"(da), "l"(db), "r"(IDESC),
                                           "r"(accum));
                        }
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                                 ::"r"(smem_u32(&empty[s])) : "memory");
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                             ::"r"(smem_u32(&acc_full[buf])) : "memory");
            }
            // every MMA issued has finished before the accumulators are released
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         ::"r"(smem_u32(&done_bar)) : "memory");
            mbar_wait_or_fail(smem_u32(&done_bar), 0u, &fail_sh);
        }
        __syncwarp();
    }
    if (warp > kHaloMmaWarp) {
        // ---------------- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31; lane 0 waits for the
        // warp, so that the whole warp takes the same path through the .sync.aligned loads
        const int q = warp & 3;
        const int r = q * 32 + lane;
        int64_t tl = 0;
        for (int64_t t = blockIdx.x; t < a.n_tiles; t += stride, ++tl) {
            const int buf = (int)(tl & 1);
            int go = 0;
            if (lane == 0) go = !fail_sh && mbar_wait_or_fail(smem_u32(&acc_full[buf]), (uint32_t)((tl >> 1) & 1), &fail_sh);
            if (!__shfl_sync(0xFFFFFFFFu, go, 0)) break;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const int tx = (int)(t % a.tiles_x), ty = (int)((t / a.tiles_x) % a.tiles_y);
            const int img = (int)(t / ((int64_t)a.tiles_x * a.tiles_y));
            const int px = tx * 8 + (r & 7), py = ty * 16 + (r >> 3);
            const bool inside = px < a.w && py < a.h;
            const int64_t p = ((int64_t)img * a.h + py) * a.w + px;
#pragma unroll
            for (int c0 = 0; c0 < BN; c0 += 16) {
                float f[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) f[k] = 0.0f;
#pragma unroll
                for (int j = 0; j < NACC; ++j) {
                    uint32_t v[16];
                    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15},"
                                 " [%16];\n"
                                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                                   "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                                   "=r"(v[14]), "=r"(v[15])
                                 : "r"(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((buf * NACC + j) * BN + c0)));
                    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                    for (int k = 0; k < 16; ++k) f[k] += __uint_as_float(v[k]);
                }
                if (inside) {
                    uint32_t pk[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        float v0 = f[2 * k] + bias_sh[c0 + 2 * k];
                        float v1 = f[2 * k + 1] + bias_sh[c0 + 2 * k + 1];
                        if (a.relu) {
                            v0 = fmaxf(v0, 0.0f);
                            v1 = fmaxf(v1, 0.0f);
                        }
                        __nv_bfloat162 h2 = __floats2bfloat162_rn(v0, v1);
                        pk[k] = *reinterpret_cast<uint32_t*>(&h2);
                    }
                    uint4* dst = reinterpret_cast<uint4*>(a.y + p * a.cout + c0);
                    dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                    dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&acc_empty[buf])) : "memory");
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (fail_sh && tid == 0) atomicExch(a.err, 1);
    if (warp == kHaloMmaWarp) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// y = act(sum of the ks partial sums + bias) in BF16 for the split-K path, the slices summed in order; 4 channels per
// thread
__global__ void conv_finish_kernel(const float* __restrict__ ws, int ks, int64_t n4, int cout,
                                   const float* __restrict__ bias, int relu, bf16* __restrict__ y)
{
    edp_dependent_start();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        float4 v = reinterpret_cast<const float4*>(ws)[i];
        for (int z = 1; z < ks; ++z) {
            const float4 u = reinterpret_cast<const float4*>(ws)[z * n4 + i];
            v.x += u.x;
            v.y += u.y;
            v.z += u.z;
            v.w += u.w;
        }
        const int n = (int)((4 * i) % cout);
        if (bias) {
            v.x += bias[n];
            v.y += bias[n + 1];
            v.z += bias[n + 2];
            v.w += bias[n + 3];
        }
        if (relu) {
            v.x = fmaxf(v.x, 0.f);
            v.y = fmaxf(v.y, 0.f);
            v.z = fmaxf(v.z, 0.f);
            v.w = fmaxf(v.w, 0.f);
        }
        __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
        reinterpret_cast<uint2*>(y)[i] = make_uint2(*reinterpret_cast<uint32_t*>(&a), *reinterpret_cast<uint32_t*>(&b));
    }
}

// FP32 workspace of the split-K path, one per (device, stream). Grown on demand: the old buffer is freed after the
// stream has finished with it.
float* splitk_workspace(cudaStream_t s, size_t bytes)
{
    struct Ws {
        int dev;
        cudaStream_t stream;
        float* p;
        size_t bytes;
    };
    static std::mutex mu;
    static std::vector<Ws> all;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    Ws* w = nullptr;
    for (auto& x : all)
        if (x.dev == dev && x.stream == s) w = &x;
    if (!w) {
        all.push_back({dev, s, nullptr, 0});
        w = &all.back();
    }
    if (w->bytes < bytes) {
        if (w->p) {
            if (cudaStreamSynchronize(s) != cudaSuccess) return nullptr;
            cudaFree(w->p);
            w->p = nullptr;
            w->bytes = 0;
        }
        if (cudaMalloc(&w->p, bytes) != cudaSuccess) return nullptr;
        w->bytes = bytes;
    }
    return w->p;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// Tensor maps already encoded, by what they encode (kind, address, sizes): a layer called again with the same
// buffers, as every solve's inference and every training step does, copies its maps instead of encoding them. A map
// holds no reference to the memory, so a buffer freed and another placed at the same address with the same sizes
// needs exactly the same map.
struct MapKey {
    int kind;
    const void* p;
    int a, b, c, d, e;
    bool operator==(const MapKey& o) const
    {
        return kind == o.kind && p == o.p && a == o.a && b == o.b && c == o.c && d == o.d && e == o.e;
    }
};

bool map_cached(const MapKey& k, CUtensorMap* m, bool (*make)(const MapKey&, CUtensorMap*))
{
    constexpr int kEntries = 256;
    static std::mutex mu;
    static MapKey keys[kEntries];
    static CUtensorMap maps[kEntries];
    static int used = 0, next = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    MapKey key = k;
    key.e = key.e * 64 + dev;   // maps are per device
    {
        std::lock_guard<std::mutex> lock(mu);
        for (int i = 0; i < used; ++i)
            if (keys[i] == key) {
                *m = maps[i];
                return true;
            }
    }
    if (!make(k, m)) return false;
    std::lock_guard<std::mutex> lock(mu);
    keys[next] = key;
    maps[next] = *m;
    next = (next + 1) % kEntries;
    if (used < kEntries) ++used;
    return true;
}

// NHWC activations with c channels: dims (c, w, h, n), box (cw, 16, 8, 1)
bool make_act(const MapKey& k, CUtensorMap* m)
{
    const void* x = k.p;
    const int nimg = k.a, h = k.b, w = k.c, c = k.d, cw = k.e;
    EncodeTiledFn f = encode_fn();
    if (!f) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)nimg};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * 2 * w, (cuuint64_t)c * 2 * w * h};
    const cuuint32_t box[4] = {(cuuint32_t)cw, 16, 8, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, cw == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool map_act(CUtensorMap* m, const void* x, int nimg, int h, int w, int c, int cw)
{
    return map_cached(MapKey{0, x, nimg, h, w, c, cw}, m, make_act);
}

// NHWC activations with c channels for the halo kernel: dims (c, w, h, n), box (8 channels, 10, 18, 1) without
// swizzle, which lands in shared memory as one plane (pixel q of the 10 x 18 halo at byte 16 q)
bool make_halo(const MapKey& k, CUtensorMap* m)
{
    const void* x = k.p;
    const int nimg = k.a, h = k.b, w = k.c, c = k.d;
    EncodeTiledFn f = encode_fn();
    if (!f) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)nimg};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * 2 * w, (cuuint64_t)c * 2 * w * h};
    const cuuint32_t box[4] = {8, 10, 18, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool map_halo(CUtensorMap* m, const void* x, int nimg, int h, int w, int c)
{
    return map_cached(MapKey{1, x, nimg, h, w, c, 0}, m, make_halo);
}

// NHWC tensor with c channels for the weight gradient's patches: box (cb channels, 8 x, 16 y, 1), an 8 x 16 patch
// as 128 pixel rows of cb channels (pixel q = 8 y + x), in the 64-byte (cb = 32) or 128-byte (cb = 64) swizzle
bool make_patch(const MapKey& k, CUtensorMap* m)
{
    const void* x = k.p;
    const int nimg = k.a, h = k.b, w = k.c, c = k.d, cb = k.e;
    EncodeTiledFn f = encode_fn();
    if (!f) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)nimg};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * 2 * w, (cuuint64_t)c * 2 * w * h};
    const cuuint32_t box[4] = {(cuuint32_t)cb, 8, 16, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, cb == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool map_patch(CUtensorMap* m, const void* x, int nimg, int h, int w, int c, int cb)
{
    return map_cached(MapKey{3, x, nimg, h, w, c, cb}, m, make_patch);
}

// weights [cout][k]: dims (k, cout), box (cw, bn)
bool make_wt(const MapKey& key, CUtensorMap* m)
{
    const void* wt = key.p;
    const int k = key.a, cout = key.b, cw = key.c, bn = key.d;
    EncodeTiledFn f = encode_fn();
    if (!f) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)cout};
    const cuuint64_t strides[1] = {(cuuint64_t)k * 2};
    const cuuint32_t box[2] = {(cuuint32_t)cw, (cuuint32_t)bn};
    const cuuint32_t estr[2] = {1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(wt), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, cw == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool map_wt(CUtensorMap* m, const void* wt, int k, int cout, int cw, int bn)
{
    return map_cached(MapKey{2, wt, k, cout, cw, bn, 0}, m, make_wt);
}

template <int BN, int CW>
int launch_tma(const ConvArgs& c, int* err, cudaStream_t s)
{
    constexpr int SMEM = 4 * (128 * CW * 2 + BN * CW * 2) + 1024;
    static bool configured[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return EDP_ERR_CUDA;
    if (!configured[dev]) {
        if (cudaFuncSetAttribute(conv3x3_fwd_tma_kernel<BN, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) !=
            cudaSuccess)
            return EDP_ERR_CUDA;
        configured[dev] = true;
    }
    CUtensorMap m1, m2, mw;
    if (!map_act(&m1, c.x1, c.nimg, c.h, c.w, c.c1, CW)) return EDP_ERR_CUDA;
    if (c.c2 > 0) {
        if (!map_act(&m2, c.x2, c.nimg, c.h, c.w, c.c2, CW)) return EDP_ERR_CUDA;
    } else {
        m2 = m1;
    }
    if (!map_wt(&mw, c.wt, 9 * (c.c1 + c.c2), c.cout, CW, BN)) return EDP_ERR_CUDA;
    TmaArgs ta;
    ta.nimg = c.nimg;
    ta.h = c.h;
    ta.w = c.w;
    ta.c1 = c.c1;
    ta.c2 = c.c2;
    ta.cout = c.cout;
    ta.relu = c.relu;
    ta.tiles_x = (c.w + 15) / 16;
    ta.tiles_y = (c.h + 7) / 8;
    ta.bias = c.bias;
    ta.y = c.y;
    ta.err = err;
    ta.ws = nullptr;
    const int64_t ctas = (int64_t)ta.tiles_x * ta.tiles_y * c.nimg * (c.cout / BN);
    // a layer with fewer CTAs than SMs splits its K range (taps x channel chunks, at least two chunks per slice) over
    // about one CTA per SM; the slices' FP32 partial sums go to a workspace and are added in order by the finish
    const int kt_all = 9 * (c.c1 + c.c2) / CW;
    int ks = 1;
    if (ctas < 148) {
        ks = (int)((148 + ctas - 1) / ctas);
        if (ks > kt_all / 2) ks = kt_all / 2;
        if (ks < 1) ks = 1;
    }
    const int64_t P = (int64_t)c.nimg * c.h * c.w;
    if (ks > 1) {
        ta.ws = splitk_workspace(s, (size_t)ks * P * c.cout * sizeof(float));
        if (!ta.ws) return EDP_ERR_CUDA;
    }
    dim3 grid((unsigned)(ta.tiles_x * ta.tiles_y * c.nimg), c.cout / BN, (unsigned)ks);
    if (edp_launch_dependent(conv3x3_fwd_tma_kernel<BN, CW>, grid, dim3(kTcThreads), SMEM, s, m1, m2, mw, ta) != cudaSuccess)
        return EDP_ERR_CUDA;
    if (ks > 1) {
        const int64_t n4 = P * c.cout / 4;
        int64_t g = (n4 + 255) / 256;
        if (g > 148 * 8) g = 148 * 8;
        if (edp_launch_dependent(conv_finish_kernel, dim3((unsigned)g), dim3(256), 0, s, (const float*)ta.ws, ks, n4, c.cout,
                             c.bias, c.relu, c.y) != cudaSuccess)
            return EDP_ERR_CUDA;
    }
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

template <int CW>
int launch_tma_cout(const ConvArgs& a, int* err, cudaStream_t s)
{
    switch (a.cout) {   // one CTA covers all output channels (two halves above 256)
    case 32: return launch_tma<32, CW>(a, err, s);
    case 64: return launch_tma<64, CW>(a, err, s);
    case 96: return launch_tma<96, CW>(a, err, s);
    case 128: return launch_tma<128, CW>(a, err, s);
    case 192: return launch_tma<192, CW>(a, err, s);
    case 256: return launch_tma<256, CW>(a, err, s);
    case 384: return launch_tma<192, CW>(a, err, s);
    default: return EDP_ERR_ARG;
    }
}

// the persistent halo kernel for c_out = BN: all 9 x c_in x BN weights resident, as many CTAs per SM as shared memory
// and the two accumulators per CTA in tensor memory (512 columns per SM) allow, one per SM at least. STREAM: the
// weights come with each chunk's halo instead of staying.
template <int BN, bool STREAM>
int launch_halo(const ConvArgs& c, int* err, cudaStream_t s)
{
    const int n_chunks = (c.c1 + c.c2) / 32;
    const int smem = STREAM ? 1024 + kHaloStages * (kHaloStagePad + 9 * BN * 64)
                            : 1024 + 9 * n_chunks * BN * 64 + kHaloStages * kHaloStage;
    static int configured[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return EDP_ERR_CUDA;
    if (configured[dev] < smem) {
        if (cudaFuncSetAttribute(conv3x3_fwd_halo_kernel<BN, STREAM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem) != cudaSuccess ||
            cudaFuncSetAttribute(conv3x3_fwd_halo_kernel<BN, STREAM>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 100) != cudaSuccess)
            return EDP_ERR_CUDA;
        configured[dev] = smem;
    }
    CUtensorMap mw, mx1, mx2;
    if (!map_wt(&mw, c.wt, 9 * (c.c1 + c.c2), c.cout, 32, BN)) return EDP_ERR_CUDA;
    if (!map_halo(&mx1, c.x1, c.nimg, c.h, c.w, c.c1)) return EDP_ERR_CUDA;
    if (c.c2 > 0) {
        if (!map_halo(&mx2, c.x2, c.nimg, c.h, c.w, c.c2)) return EDP_ERR_CUDA;
    } else {
        mx2 = mx1;
    }
    HaloArgs a;
    a.x1 = c.x1;
    a.x2 = c.x2;
    a.c1 = c.c1;
    a.c2 = c.c2;
    a.nimg = c.nimg;
    a.h = c.h;
    a.w = c.w;
    a.cout = c.cout;
    a.relu = c.relu;
    a.tiles_x = (c.w + 7) / 8;
    a.tiles_y = (c.h + 15) / 16;
    a.n_tiles = (int64_t)a.tiles_x * a.tiles_y * c.nimg;
    a.bias = c.bias;
    a.y = c.y;
    a.err = err;
    int sms = 0, smem_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
        return EDP_ERR_CUDA;
    // CTAs per SM: shared memory (1 KiB per CTA reserved by the driver) and the 512 tensor-memory columns of an SM
    int per_sm = smem_sm / (smem + 1024);
    if (per_sm > 512 / kHaloTmemCols<BN>) per_sm = 512 / kHaloTmemCols<BN>;
    if (per_sm < 1) per_sm = 1;
    const int64_t grid = a.n_tiles < (int64_t)sms * per_sm ? a.n_tiles : (int64_t)sms * per_sm;
    if (edp_launch_dependent(conv3x3_fwd_halo_kernel<BN, STREAM>, dim3((unsigned)grid), dim3(kHaloFwdThreads), smem, s, mw,
                         mx1, mx2, a) != cudaSuccess)
        return EDP_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

// 0: the halo kernel where it applies (c_out 32, 64 or 128 with the weights resident in shared memory, or 32 and 64
// with them streamed, at least two tiles per SM), else the tile kernel; 1: always the tile kernel; 2: always the halo
// kernel (refused where it does not apply)
int g_conv_mode = 0;

bool halo_resident(const ConvArgs& c) { return 9LL * (c.c1 + c.c2) * c.cout * 2 <= kHaloMaxWeights; }

bool halo_possible(const ConvArgs& c)
{
    return c.cout == 32 || c.cout == 64 || (c.cout == 128 && halo_resident(c));
}

bool halo_applies(const ConvArgs& c)
{
    const int64_t tiles = (int64_t)((c.w + 7) / 8) * ((c.h + 15) / 16) * c.nimg;
    return halo_possible(c) && tiles >= 2 * 148;
}

// wt_t[c][8 - tap][n] = wt[n][tap][c]: the weights of the data gradient
__global__ void flip_transpose_kernel(const bf16* __restrict__ wt, int cout, int cin, bf16* __restrict__ out)
{
    const int64_t total = (int64_t)cout * 9 * cin;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(q % cin);
        const int tap = (int)((q / cin) % 9);
        const int n = (int)(q / ((int64_t)cin * 9));
        out[((int64_t)c * 9 + (8 - tap)) * cout + n] = wt[q];
    }
}

// ------------------------------------------------------------------------------------------ weight gradient
struct WgradArgs {
    int nimg, h, w;
    const bf16* x;    // [P][cin] (a concatenated input is passed as x1 | x2 split at c1)
    int c1;
    const bf16* x2;
    int c2;
    const bf16* dz;   // [P][cout]
    int cout;
    float* dw;        // [cout][9][cin], accumulated
    int64_t pix_per_cta;
};

constexpr int kWK = 32;   // pixels per K step

template <int BM, int BN>
__global__ void __launch_bounds__((BM / 32) * (BN / 16) * 32) conv3x3_wgrad_kernel(WgradArgs a)
{
    constexpr int WARPS_M = BM / 32, WARPS_N = BN / 16, NT = WARPS_M * WARPS_N * 32;
    constexpr int A_CPR = BM / 8, B_CPR = BN / 8;               // 16-byte chunks per smem row (4 or 8)
    constexpr int A_BYTES = kWK * BM * 2, B_BYTES = kWK * BN * 2;
    __shared__ __align__(128) unsigned char sm[kStages * (A_BYTES + B_BYTES)];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp % WARPS_M, wn = warp / WARPS_M;
    const int cin = a.c1 + a.c2;
    const int ntile_c = cin / BN, ntile_o = a.cout / BM;
    int tile = blockIdx.y;
    const int co0 = (tile % ntile_o) * BM;
    tile /= ntile_o;
    const int ci0 = (tile % ntile_c) * BN;
    const int tap = tile / ntile_c;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    const int64_t P = (int64_t)a.nimg * a.h * a.w;
    const int64_t p_begin = (int64_t)blockIdx.x * a.pix_per_cta;
    int64_t p_end = p_begin + a.pix_per_cta;
    if (p_end > P) p_end = P;
    if (p_begin >= p_end) return;
    const int KT = (int)((p_end - p_begin + kWK - 1) / kWK);
    const bf16* xs;
    int xcs, xco;
    if (ci0 < a.c1) { xs = a.x; xcs = a.c1; xco = ci0; }
    else { xs = a.x2; xcs = a.c2; xco = ci0 - a.c1; }

    auto load_stage = [&](int s, int kt) {
        unsigned char* As = sm + s * (A_BYTES + B_BYTES);
        unsigned char* Bs = As + A_BYTES;
        const int64_t pk = p_begin + (int64_t)kt * kWK;
        for (int idx = tid; idx < kWK * A_CPR; idx += NT) {
            const int r = idx / A_CPR, c = idx % A_CPR;
            const int64_t p = pk + r;
            const bool ok = p < p_end;
            const bf16* g = ok ? a.dz + p * a.cout + co0 + c * 8 : a.dz;
            cp_async16(smem_u32(As + swz(r, c, A_CPR)), g, ok);
        }
        for (int idx = tid; idx < kWK * B_CPR; idx += NT) {
            const int r = idx / B_CPR, c = idx % B_CPR;
            const int64_t p = pk + r;
            bool ok = p < p_end;
            const bf16* g = xs;
            if (ok) {
                const int x = (int)(p % a.w), y = (int)((p / a.w) % a.h);
                const int64_t b = p / ((int64_t)a.w * a.h);
                const int yy = y + dy, xx = x + dx;
                ok = yy >= 0 && yy < a.h && xx >= 0 && xx < a.w;
                if (ok) g = xs + ((b * a.h + yy) * a.w + xx) * xcs + xco + c * 8;
            }
            cp_async16(smem_u32(Bs + swz(r, c, B_CPR)), g, ok);
        }
    };

    float acc[2][2][4];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0f;

    for (int s = 0; s < kStages - 1; ++s) {
        if (s < KT) load_stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<kStages - 2>();
        __syncthreads();
        if (kt + kStages - 1 < KT) load_stage((kt + kStages - 1) % kStages, kt + kStages - 1);
        cp_async_commit();
        const unsigned char* As = sm + (kt % kStages) * (A_BYTES + B_BYTES);
        const unsigned char* Bs = As + A_BYTES;
        for (int ks = 0; ks < 2; ++ks) {
            const int kb = ks * 16;
            uint32_t af[2][4], bfr[2][2];
            for (int i = 0; i < 2; ++i) {   // A (m = c_out, k = pixel) stored [k][m]: transposed loads
                const int r = kb + (lane & 7) + ((lane >> 4) << 3);
                const int m = wm * 32 + i * 16 + (((lane >> 3) & 1) << 3);
                ldsm_x4_t(smem_u32(As + swz(r, m >> 3, A_CPR)), af[i][0], af[i][1], af[i][2], af[i][3]);
            }
            {   // B (k = pixel, n = c_in) stored [k][n]: transposed loads, two n8 tiles
                const int r = kb + (lane & 7) + (((lane >> 3) & 1) << 3);
                const int n = wn * 16 + ((lane >> 4) << 3);
                ldsm_x4_t(smem_u32(Bs + swz(r, n >> 3, B_CPR)), bfr[0][0], bfr[0][1], bfr[1][0], bfr[1][1]);
            }
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
        }
    }
    cp_async_wait<0>();

    const int g = lane >> 2, t = lane & 3;
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int q = 0; q < 4; ++q) {
                const int co = co0 + wm * 32 + i * 16 + g + 8 * (q >> 1);
                const int ci = ci0 + wn * 16 + j * 8 + 2 * t + (q & 1);
                atomicAdd(&a.dw[((int64_t)co * 9 + tap) * cin + ci], acc[i][j][q]);
            }
}

// ------------------------------------------------------------------------------------------ weight gradient on tcgen05
// dw[n][tap][c] += sum_p dz[p][n] x[p + off(tap)][c] as one GEMM per tap with M = output channels (a chunk of M = 64
// or 128 of them), N = a 32-channel chunk of the input, K = pixels. The pixels come in 8 x 16 patches as in the
// halo forward kernel: the patch of dz lies in shared memory as planes of 8 output channels (pixel q at byte 16 q),
// which is the canonical MN-major layout without swizzle for A (8-channel groups one plane apart = SBO, 8-pixel groups
// 128 bytes apart = LBO); the 10 x 18 halo of x lies as four planes of 8 input channels, and the B operand of tap
// (dx, dy) is the same planes read from pixel 10 dy + dx on (MN-major: channel groups one plane apart = SBO, 8-pixel
// groups = patch rows one halo row apart = LBO of 160 bytes). One patch and one halo serve all nine taps, whose
// accumulators (9 x 32 FP32 columns) stay in tensor memory for the CTA's whole pixel range. Pixels are split over
// the CTAs (patches taken round-robin); at the end each CTA adds its partial sums to dw with vector FP32 reductions.
// Roles as in the halo forward kernel: warps 0-1 copy (cp.async, zero-filled off the image), warp 2 lane 0 issues
// the MMAs, warps 3-6 read the accumulators back. With M = 64 the accumulator rows 16 q .. 16 q + 15 sit in lanes
// 32 q .. 32 q + 15 of tensor memory; output channels past c_out read zero planes.
constexpr int kWgStages = 3;
constexpr int kDzPlane = 2064;   // 129 pixel slots of 16 bytes (128 used)

struct WgradTcArgs {
    const bf16* x1;
    const bf16* x2;
    int c1, c2;
    const bf16* dz;
    int cout, nimg, h, w, tiles_x, tiles_y;
    int64_t n_tiles;
    float* dw;
    int* err;
};

template <int M>
__global__ void __launch_bounds__(kHaloThreads, 1) conv3x3_wgrad_tc_kernel(WgradTcArgs a)
{
    constexpr int NP = M / 8;                                   // dz planes
    constexpr int STAGE = NP * kDzPlane + kWgHaloStage;
    constexpr uint32_t TMEM_COLS = 512;                         // 9 taps x 32 columns
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((32u >> 3) << 17) |
                               ((uint32_t)(M >> 4) << 24);
    constexpr uint64_t DESC_A = ((uint64_t)(kDzPlane >> 4) << 32) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)1 << 46);
    constexpr uint64_t DESC_B = ((uint64_t)(kWgPlane >> 4) << 32) | ((uint64_t)(160 >> 4) << 16) | ((uint64_t)1 << 46);
    extern __shared__ unsigned char dsm[];
    __shared__ __align__(8) uint64_t full[kWgStages], empty[kWgStages], done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int fail_sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c0 = blockIdx.y * 32;                              // input channels of this CTA
    const int m0 = blockIdx.z * M;                               // output channels of this CTA
    const int mvalid = a.cout - m0 < M ? a.cout - m0 : M;
    const uint32_t base = (smem_u32(dsm) + 127u) & ~127u;
    unsigned char* gbase = dsm + (base - smem_u32(dsm));

    // planes past c_out stay zero in every stage
    for (int st = 0; st < kWgStages; ++st)
        for (int b = (mvalid / 8) * kDzPlane + tid * 16; b < NP * kDzPlane; b += kHaloThreads * 16)
            *reinterpret_cast<uint4*>(gbase + st * STAGE + b) = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        fail_sh = 0;
        for (int st = 0; st < kWgStages; ++st) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&full[st])), "r"(64));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[st])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&done_bar)));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base_sh;
    const int64_t stride = gridDim.x;
    bool any = false;   // this CTA has at least one patch (every role sees the same)
    if (blockIdx.x < a.n_tiles) any = true;

    if (warp < 2) {
        // ---------------- producer: dz patch planes and the x halo of each patch
        const int pt = tid;
        const bf16* xs = c0 < a.c1 ? a.x1 : a.x2;
        const int xcs = c0 < a.c1 ? a.c1 : a.c2, xco = c0 < a.c1 ? c0 : c0 - a.c1;
        const int nzp = mvalid / 8;
        int64_t it = 0;
        for (int64_t t = blockIdx.x; t < a.n_tiles && !fail_sh; t += stride, ++it) {
            const int s = (int)(it % kWgStages);
            if (it >= kWgStages &&
                !mbar_wait_or_fail(smem_u32(&empty[s]), (uint32_t)(((it / kWgStages) - 1) & 1), &fail_sh))
                break;
            const int tx = (int)(t % a.tiles_x), ty = (int)((t / a.tiles_x) % a.tiles_y);
            const int img = (int)(t / ((int64_t)a.tiles_x * a.tiles_y));
            const uint32_t st = base + (uint32_t)(s * STAGE);
            for (int q = pt; q < 128 * nzp; q += 64) {
                const int px = q / nzp, pl = q - px * nzp;
                const int gx = tx * 8 + (px & 7), gy = ty * 16 + (px >> 3);
                const bool ok = gx < a.w && gy < a.h;
                const bf16* g = ok ? a.dz + (((int64_t)img * a.h + gy) * a.w + gx) * a.cout + m0 + 8 * pl : a.dz;
                cp_async16(st + (uint32_t)(pl * kDzPlane + px * 16), g, ok);
            }
            const uint32_t hs = st + (uint32_t)(NP * kDzPlane);
            for (int q = pt; q < 180 * 4; q += 64) {
                const int px = q >> 2, pl = q & 3;
                const int gx = tx * 8 - 1 + px % 10, gy = ty * 16 - 1 + px / 10;
                const bool ok = gx >= 0 && gx < a.w && gy >= 0 && gy < a.h;
                const bf16* g = ok ? xs + (((int64_t)img * a.h + gy) * a.w + gx) * xcs + xco + 8 * pl : xs;
                cp_async16(hs + (uint32_t)(pl * kWgPlane + px * 16), g, ok);
            }
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(&full[s])) : "memory");
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
    } else if (warp == 2) {
        if (lane == 0) {
            int64_t it = 0;
            for (int64_t t = blockIdx.x; t < a.n_tiles && !fail_sh; t += stride, ++it) {
                const int s = (int)(it % kWgStages);
                if (!mbar_wait_or_fail(smem_u32(&full[s]), (uint32_t)((it / kWgStages) & 1), &fail_sh)) break;
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t As = base + (uint32_t)(s * STAGE), Hs = As + (uint32_t)(NP * kDzPlane);
                // K steps outside, taps inside: consecutive MMAs go to the nine independent accumulators, so that
                // none waits for the one before it
                for (int ks = 0; ks < 8; ++ks) {
                    const uint64_t da = DESC_A | (uint64_t)(((As + (uint32_t)(256 * ks)) >> 4) & 0x3FFFu);
                    for (int tap = 0; tap < 9; ++tap) {
                        const uint32_t b0 = Hs + (uint32_t)(((tap / 3) * 10 + tap % 3) * 16);
                        const uint64_t db = DESC_B | (uint64_t)(((b0 + (uint32_t)(320 * ks)) >> 4) & 0x3FFFu);
                        const uint32_t accum = (it > 0 || ks > 0) ? 1u : 0u;
                        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                                     ::"r"(tmem + (uint32_t)(tap * 32)), "l"(da), "l"(db), "r"(IDESC), "r"(accum));
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                             ::"r"(smem_u32(&empty[s])) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         ::"r"(smem_u32(&done_bar)) : "memory");
            mbar_wait_or_fail(smem_u32(&done_bar), 0u, &fail_sh);
        }
        __syncwarp();
    }
    __syncthreads();   // the producer and the MMAs are done (or gave up)
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp >= 3 && any && !fail_sh) {
        const int q = warp & 3;
        const int r = M == 128 ? q * 32 + lane : q * 16 + lane;   // accumulator row of this lane
        const bool valid = (M == 128 || lane < 16) && r < mvalid;
        for (int tap = 0; tap < 9; ++tap) {
            for (int h = 0; h < 2; ++h) {
                uint32_t v[16];
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15},"
                             " [%16];\n"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                               "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                               "=r"(v[14]), "=r"(v[15])
                             : "r"(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(tap * 32 + 16 * h)));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                if (valid) {
                    float* d = a.dw + ((int64_t)(m0 + r) * 9 + tap) * (a.c1 + a.c2) + c0 + 16 * h;
#pragma unroll
                    for (int k = 0; k < 16; k += 4)
                        asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n"
                                     ::"l"(d + k), "f"(__uint_as_float(v[k])), "f"(__uint_as_float(v[k + 1])),
                                       "f"(__uint_as_float(v[k + 2])), "f"(__uint_as_float(v[k + 3]))
                                     : "memory");
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (fail_sh && tid == 0) atomicExch(a.err, 1);
    if (warp == 2) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// ------------------------------------------------------------------------------------------ weight gradient, taps in M
// The weight gradient with the taps stacked along M: dw[n][tap][c] = sum_q dz[q - off(tap)][n] x[q][c] is, per
// group of 4 taps, one GEMM with M = (tap, c) rows (4 taps x a 32-channel chunk of x = 128), N = n (a chunk of NB
// output channels), K = the pixels q of an 8 x 16 patch. Its A operand is four copies of the x patch shifted by the
// four taps' offsets, B the dz patch, both MN-major: each copy is one TMA box of (32 channels, 8 x, 16 y) of the NHWC
// tensor, zero-filled off the image, landing as 128 pixel rows of 64 bytes in the 64-byte swizzle (one swizzle atom
// of 32 channels across, 8-pixel groups 512 bytes apart = SBO, the taps one copy apart = LBO); dz comes the same way,
// or as 64-channel boxes in the 128-byte swizzle. Taps 0-3 and 4-7 are two M = 128 MMAs per K step, tap 8 an
// M = 64 MMA (its copy followed by a zero copy), so a patch takes 24 MMAs where the taps in N would take 72 of
// M = 64 with half of each padding when c_out = 32. The three accumulators (3 x NB columns) stay
// in tensor memory for the CTA's whole pixel range; at the end each lane adds its row (one tap and x channel) to dw
// for every n (red.global.add.f32, 32 consecutive channels per warp and n). Roles: warp 0 lane 0 copies (TMA),
// warp 1 lane 0 issues the MMAs, warps 2-5 read the accumulators back. Every wait is bounded.
constexpr int kTapThreads = 192;
constexpr int kTapStages = 2;
constexpr int kTapCopy = 128 * 64;                     // one shifted copy: 128 pixels x 32 channels (64-byte swizzle)
constexpr int kTapXBytes = 10 * kTapCopy;              // 9 taps, then a zero copy after tap 8

template <int NB>
__global__ void __launch_bounds__(kTapThreads, 1) conv3x3_wgrad_tap_kernel(const __grid_constant__ CUtensorMap mx1,
                                                                        const __grid_constant__ CUtensorMap mx2,
                                                                        const __grid_constant__ CUtensorMap mdz,
                                                                        WgradTcArgs a)
{
    constexpr int STAGE = kTapXBytes + NB * 256;   // + the dz patch: 128 pixels x NB channels
    constexpr uint32_t TMEM_COLS = 3 * NB <= 128 ? 128 : 3 * NB <= 256 ? 256 : 512;
    // A and B both MN-major (bits 15, 16), M = 128 or 64, N = NB
    constexpr uint32_t IDESC128 = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                                  ((uint32_t)(NB >> 3) << 17) | ((128u >> 4) << 24);
    constexpr uint32_t IDESC64 = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                                 ((uint32_t)(NB >> 3) << 17) | ((64u >> 4) << 24);
    // MN-major, swizzled: the 32 channels of a tap copy are one 64-byte swizzle atom per pixel row, 8-pixel groups
    // 512 bytes apart (SBO), the taps one copy apart (LBO); dz: 32 channels in the same 64-byte layout, or 64-channel
    // groups of 128-byte rows (8-pixel groups 1024 bytes apart, groups 128 pixels x 128 bytes apart)
    constexpr uint64_t DESC_A = ((uint64_t)(512 >> 4) << 32) | ((uint64_t)(kTapCopy >> 4) << 16) | ((uint64_t)1 << 46) |
                                ((uint64_t)4 << 61);
    constexpr int B_ROW = NB == 32 ? 64 : 128;      // bytes per pixel row of the dz patch
    constexpr uint64_t DESC_B = ((uint64_t)((8 * B_ROW) >> 4) << 32) | ((uint64_t)((128 * B_ROW) >> 4) << 16) |
                                ((uint64_t)1 << 46) | ((uint64_t)(NB == 32 ? 4 : 2) << 61);
    extern __shared__ unsigned char dsm[];
    __shared__ __align__(8) uint64_t full[kTapStages], empty[kTapStages], done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int fail_sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cin = a.c1 + a.c2;
    const int c0 = blockIdx.y * 32;    // x channels of this CTA
    const int n0 = blockIdx.z * NB;    // output channels of this CTA
    const uint32_t base = (smem_u32(dsm) + 1023u) & ~1023u;
    unsigned char* gbase = dsm + (base - smem_u32(dsm));

    // the copy after tap 8's stays zero: the M = 64 MMA of tap 8 reads it as its padding rows
    for (int st = 0; st < kTapStages; ++st)
        for (int b = 9 * kTapCopy + tid * 16; b < 10 * kTapCopy; b += kTapThreads * 16)
            *reinterpret_cast<uint4*>(gbase + st * STAGE + b) = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        fail_sh = 0;
        for (int st = 0; st < kTapStages; ++st) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[st])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[st])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&done_bar)));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // the zero planes, for the MMAs' async reads
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base_sh;
    const int64_t stride = gridDim.x;

    if (warp == 0) {
        // ---------------- copies (lane 0): per patch the 36 planes of the nine shifted x copies and the dz planes
        if (lane == 0) {
            const CUtensorMap* mx = c0 < a.c1 ? &mx1 : &mx2;
            const int xco = c0 < a.c1 ? c0 : c0 - a.c1;
            constexpr uint32_t BYTES = 9 * kTapCopy + NB * 256;
            int64_t it = 0;
            for (int64_t t = blockIdx.x; t < a.n_tiles && !fail_sh; t += stride, ++it) {
                const int s = (int)(it % kTapStages);
                if (it >= kTapStages &&
                    !mbar_wait_or_fail(smem_u32(&empty[s]), (uint32_t)(((it / kTapStages) - 1) & 1), &fail_sh))
                    break;
                const int tx = (int)(t % a.tiles_x), ty = (int)((t / a.tiles_x) % a.tiles_y);
                const int img = (int)(t / ((int64_t)a.tiles_x * a.tiles_y));
                const int px0 = tx * 8, py0 = ty * 16;
                const uint32_t st = base + (uint32_t)(s * STAGE), fb = smem_u32(&full[s]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"(BYTES) : "memory");
                for (int tap = 0; tap < 9; ++tap)
                    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
                                 ::"r"(st + (uint32_t)(tap * kTapCopy)), "l"(mx), "r"(xco), "r"(px0 + tap % 3 - 1),
                                   "r"(py0 + tap / 3 - 1), "r"(img), "r"(fb) : "memory");
                for (int j = 0; j < NB * 2 / B_ROW; ++j)
                    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
                                 ::"r"(st + (uint32_t)(kTapXBytes + j * 128 * B_ROW)), "l"(&mdz),
                                   "r"(n0 + j * (B_ROW / 2)), "r"(px0), "r"(py0), "r"(img), "r"(fb) : "memory");
            }
            // copies still in flight after a failure land before the CTA leaves
            for (int64_t q = it > kTapStages ? it - kTapStages : 0; q < it; ++q)
                mbar_wait(smem_u32(&full[q % kTapStages]), (uint32_t)((q / kTapStages) & 1));
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMAs (lane 0): per K step of 16 pixels, taps 0-3, taps 4-7 (M = 128), tap 8 (M = 64)
        if (lane == 0) {
            int64_t it = 0;
            for (int64_t t = blockIdx.x; t < a.n_tiles && !fail_sh; t += stride, ++it) {
                const int s = (int)(it % kTapStages);
                if (!mbar_wait_or_fail(smem_u32(&full[s]), (uint32_t)((it / kTapStages) & 1), &fail_sh)) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t xs = base + (uint32_t)(s * STAGE), zs = xs + (uint32_t)kTapXBytes;
                for (int ks = 0; ks < 8; ++ks) {
                    // a K step is 16 pixel rows: two 8-row groups
                    const uint64_t db = DESC_B | (uint64_t)(((zs + (uint32_t)(16 * B_ROW * ks)) >> 4) & 0x3FFFu);
                    const uint32_t accum = (it > 0 || ks > 0) ? 1u : 0u;
                    for (int g = 0; g < 3; ++g) {
                        const uint64_t da =
                            DESC_A | (uint64_t)(((xs + (uint32_t)(g * 4 * kTapCopy + 1024 * ks)) >> 4) & 0x3FFFu);
                        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                                     ::"r"(tmem + (uint32_t)(g * NB)), "l"(da), "l"(db),
                                       "r"(g < 2 ? IDESC128 : IDESC64), "r"(accum));
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                             ::"r"(smem_u32(&empty[s])) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         ::"r"(smem_u32(&done_bar)) : "memory");
            mbar_wait_or_fail(smem_u32(&done_bar), 0u, &fail_sh);
        }
        __syncwarp();
    }
    __syncthreads();   // the copies and the MMAs are done (or gave up)
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp >= 2 && blockIdx.x < a.n_tiles && !fail_sh) {
        // ---------------- the accumulators into dw: warp quarter q = warp % 4 reads lanes 32 q .. 32 q + 31
        const int q = warp & 3;
        for (int g = 0; g < 3; ++g) {
            // M = 128 groups: row 32 q + lane = tap 4 g + q, x channel lane; the M = 64 group (tap 8): rows 0-15 in
            // lanes 0-15, rows 16-31 in lanes 32-47, x channel 16 q + lane
            if (g == 2 && q > 1) break;
            const int tap = g < 2 ? 4 * g + q : 8;
            const int c = g < 2 ? lane : 16 * q + lane;
            const bool valid = g < 2 || lane < 16;
            float* d = a.dw + ((int64_t)n0 * 9 + tap) * cin + c0 + c;
            for (int h = 0; h < NB / 16; ++h) {
                uint32_t v[16];
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15},"
                             " [%16];\n"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                               "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                               "=r"(v[14]), "=r"(v[15])
                             : "r"(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(g * NB + 16 * h)));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                if (valid)
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        atomicAdd(d + (int64_t)(16 * h + j) * 9 * cin, __uint_as_float(v[j]));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (fail_sh && tid == 0) atomicExch(a.err, 1);
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// one CTA per SM (two stages of the nine shifted x copies and the dz patch take most of its shared memory), the
// patches split over the CTAs of each (x chunk, output chunk) pair
template <int NB>
int launch_wgrad_tap(const WgradArgs& w, int* err, cudaStream_t s)
{
    constexpr int SMEM = 1024 + kTapStages * (kTapXBytes + NB * 256);
    static bool configured[64] = {false};
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return EDP_ERR_CUDA;
    if (!configured[dev]) {
        if (cudaFuncSetAttribute(conv3x3_wgrad_tap_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) !=
            cudaSuccess)
            return EDP_ERR_CUDA;
        configured[dev] = true;
    }
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return EDP_ERR_CUDA;
    CUtensorMap mx1, mx2, mdz;
    if (!map_patch(&mx1, w.x, w.nimg, w.h, w.w, w.c1, 32)) return EDP_ERR_CUDA;
    if (w.c2 > 0) {
        if (!map_patch(&mx2, w.x2, w.nimg, w.h, w.w, w.c2, 32)) return EDP_ERR_CUDA;
    } else {
        mx2 = mx1;
    }
    if (!map_patch(&mdz, w.dz, w.nimg, w.h, w.w, w.cout, NB == 32 ? 32 : 64)) return EDP_ERR_CUDA;
    WgradTcArgs a;
    a.x1 = w.x;
    a.x2 = w.x2;
    a.c1 = w.c1;
    a.c2 = w.c2;
    a.dz = w.dz;
    a.cout = w.cout;
    a.nimg = w.nimg;
    a.h = w.h;
    a.w = w.w;
    a.tiles_x = (w.w + 7) / 8;
    a.tiles_y = (w.h + 15) / 16;
    a.n_tiles = (int64_t)a.tiles_x * a.tiles_y * w.nimg;
    a.dw = w.dw;
    a.err = err;
    const int n_c = (w.c1 + w.c2) / 32, n_n = w.cout / NB;
    int64_t split = (sms + (int64_t)n_c * n_n - 1) / ((int64_t)n_c * n_n);
    if (split > a.n_tiles) split = a.n_tiles;
    if (split < 1) split = 1;
    conv3x3_wgrad_tap_kernel<NB><<<dim3((unsigned)split, (unsigned)n_c, (unsigned)n_n), kTapThreads, SMEM, s>>>(
        mx1, mx2, mdz, a);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

// 0 (default): the weight gradient on tcgen05 with the taps in M; 2: on tcgen05 with the taps in N; 1: mma.sync
int g_wgrad_mode = 0;

// one CTA per SM (its 9 x 32 accumulator columns take 512 of tensor memory), the patches split over the CTAs of each
// (input chunk, output chunk) pair
template <int M>
int launch_wgrad_tc(const WgradArgs& w, int* err, cudaStream_t s)
{
    constexpr int SMEM = 128 + kWgStages * ((M / 8) * kDzPlane + kWgHaloStage);
    static bool configured[64] = {false};
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return EDP_ERR_CUDA;
    if (!configured[dev]) {
        if (cudaFuncSetAttribute(conv3x3_wgrad_tc_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) !=
            cudaSuccess)
            return EDP_ERR_CUDA;
        configured[dev] = true;
    }
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return EDP_ERR_CUDA;
    WgradTcArgs a;
    a.x1 = w.x;
    a.x2 = w.x2;
    a.c1 = w.c1;
    a.c2 = w.c2;
    a.dz = w.dz;
    a.cout = w.cout;
    a.nimg = w.nimg;
    a.h = w.h;
    a.w = w.w;
    a.tiles_x = (w.w + 7) / 8;
    a.tiles_y = (w.h + 15) / 16;
    a.n_tiles = (int64_t)a.tiles_x * a.tiles_y * w.nimg;
    a.dw = w.dw;
    a.err = err;
    const int n_c = (w.c1 + w.c2) / 32, n_m = (w.cout + M - 1) / M;
    int64_t split = (sms + (int64_t)n_c * n_m - 1) / ((int64_t)n_c * n_m);
    if (split > a.n_tiles) split = a.n_tiles;
    if (split < 1) split = 1;
    conv3x3_wgrad_tc_kernel<M><<<dim3((unsigned)split, (unsigned)n_c, (unsigned)n_m), kHaloThreads, SMEM, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

// db[n] += sum_p dz[p][n]
__global__ void bias_grad_kernel(const bf16* __restrict__ dz, int64_t P, int cout, float* db)
{
    extern __shared__ float red[];
    const int c = threadIdx.x % cout, lanes = blockDim.x / cout, l = threadIdx.x / cout;
    float s = 0.0f;
    if (threadIdx.x < lanes * cout)
        for (int64_t p = (int64_t)blockIdx.x * lanes + l; p < P; p += (int64_t)gridDim.x * lanes)
            s += __bfloat162float(dz[p * cout + c]);
    red[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x < cout) {
        float t = 0.0f;
        for (int k = 0; k < lanes; ++k) t += red[k * cout + threadIdx.x];
        atomicAdd(&db[threadIdx.x], t);
    }
}

// ------------------------------------------------------------------------------------------ glue
// f x f average pooling, NHWC, h and w multiples of f (f = 2 or 4)
__global__ void pool_fwd_kernel(const bf16* __restrict__ x, int nimg, int h, int w, int c, int f,
                                bf16* __restrict__ y)
{
    const int ho = h / f, wo = w / f;
    const float inv = 1.0f / (float)(f * f);
    const int64_t total = (int64_t)nimg * ho * wo * c;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int ch = (int)(q % c);
        int64_t r = q / c;
        const int X = (int)(r % wo);
        r /= wo;
        const int Y = (int)(r % ho);
        const int64_t b = r / ho;
        float v = 0.0f;
        for (int dy = 0; dy < f; ++dy)
            for (int dx = 0; dx < f; ++dx) v += __bfloat162float(x[((b * h + f * Y + dy) * w + f * X + dx) * c + ch]);
        y[q] = __float2bfloat16(inv * v);
    }
}

// dx (+)= pool backward of dy: every input pixel gets 1 / f^2 of its output's gradient
__global__ void pool_bwd_kernel(const bf16* __restrict__ dy, int nimg, int h, int w, int c, int f,
                                bf16* __restrict__ dx, int accumulate)
{
    const float inv = 1.0f / (float)(f * f);
    const int64_t total = (int64_t)nimg * h * w * c;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int ch = (int)(q % c);
        int64_t r = q / c;
        const int x = (int)(r % w);
        r /= w;
        const int y = (int)(r % h);
        const int64_t b = r / h;
        float v = inv * __bfloat162float(dy[((b * (h / f) + y / f) * (w / f) + x / f) * c + ch]);
        if (accumulate) v += __bfloat162float(dx[q]);
        dx[q] = __float2bfloat16(v);
    }
}

// nearest f x upsampling, NHWC (h, w: output size)
__global__ void up_fwd_kernel(const bf16* __restrict__ x, int nimg, int h, int w, int c, int f, bf16* __restrict__ y)
{
    const int64_t total = (int64_t)nimg * h * w * c;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int ch = (int)(q % c);
        int64_t r = q / c;
        const int xx = (int)(r % w);
        r /= w;
        const int yy = (int)(r % h);
        const int64_t b = r / h;
        y[q] = x[((b * (h / f) + yy / f) * (w / f) + xx / f) * c + ch];
    }
}

// dx = sum of the f^2 output gradients of each input pixel; dy has cs channels of which the first c are read
__global__ void up_bwd_kernel(const bf16* __restrict__ dy, int nimg, int h, int w, int c, int cs, int f,
                              bf16* __restrict__ dx)
{
    const int ho = h / f, wo = w / f;
    const int64_t total = (int64_t)nimg * ho * wo * c;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int ch = (int)(q % c);
        int64_t r = q / c;
        const int X = (int)(r % wo);
        r /= wo;
        const int Y = (int)(r % ho);
        const int64_t b = r / ho;
        float v = 0.0f;
        for (int dyy = 0; dyy < f; ++dyy)
            for (int dxx = 0; dxx < f; ++dxx)
                v += __bfloat162float(dy[((b * h + f * Y + dyy) * w + f * X + dxx) * cs + ch]);
        dx[q] = __float2bfloat16(v);
    }
}

// dz = dy * (y > 0) (ReLU backward through the layer's own output); dy may have cs >= c channels (first c read,
// starting at channel offset co), with an optional second term dy2 [P][c] added first
__global__ void relu_bwd_kernel(const bf16* __restrict__ dy, int cs, int co, const bf16* __restrict__ dy2,
                                const bf16* __restrict__ y, int64_t P, int c, bf16* __restrict__ dz)
{
    const int64_t total = P * c;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int ch = (int)(q % c);
        const int64_t p = q / c;
        float v = __bfloat162float(dy[p * cs + co + ch]);
        if (dy2) v += __bfloat162float(dy2[q]);
        dz[q] = __float2bfloat16(__bfloat162float(y[q]) > 0.0f ? v : 0.0f);
    }
}

// head: out[p] = sum_{tap, c} x[p + off(tap)][c] wh[tap][c] + bh   (c_out = 1, FP32)
__global__ void head_fwd_kernel(const bf16* __restrict__ x, int nimg, int h, int w, int c, const float* __restrict__ wh,
                                const float* __restrict__ bhp, float* __restrict__ out)
{
    const int64_t P = (int64_t)nimg * h * w;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
        const int xx = (int)(p % w), yy = (int)((p / w) % h);
        const int64_t b = p / ((int64_t)w * h);
        float s = *bhp;
        for (int tap = 0; tap < 9; ++tap) {
            const int y2 = yy + tap / 3 - 1, x2 = xx + tap % 3 - 1;
            if (y2 < 0 || y2 >= h || x2 < 0 || x2 >= w) continue;
            const bf16* xp = x + ((b * h + y2) * w + x2) * c;
            const float* wp = wh + tap * c;
            for (int k = 0; k < c; k += 2) {
                const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(xp + k));
                s += v.x * wp[k] + v.y * wp[k + 1];
            }
        }
        out[p] = s;
    }
}

// head backward: dx[p][c] = sum_tap dout[p - off(tap)] wh[tap][c]; dwh[tap][c] += sum_p dout[p] x[p + off(tap)][c];
// dbh += sum_p dout[p]. A thread owns one channel pair (the grid stride is a multiple of c / 2) and keeps its
// weight-gradient partial sums in registers.
__global__ void head_bwd_kernel(const bf16* __restrict__ x, int nimg, int h, int w, int c, const float* __restrict__ wh,
                                const float* __restrict__ dout, bf16* __restrict__ dx, float* dwh, float* dbh)
{
    extern __shared__ float part[];   // [9 * c + 1]
    for (int k = threadIdx.x; k < 9 * c + 1; k += blockDim.x) part[k] = 0.0f;
    __syncthreads();
    const int64_t P = (int64_t)nimg * h * w;
    const int cp = c / 2;
    const int64_t total = P * cp;
    float gw[9][2], gb = 0.0f;
    for (int tap = 0; tap < 9; ++tap) gw[tap][0] = gw[tap][1] = 0.0f;
    const int k = 2 * (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) % cp);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = q / cp;
        const int xx = (int)(p % w), yy = (int)((p / w) % h);
        const int64_t b = p / ((int64_t)w * h);
        float g0 = 0.0f, g1 = 0.0f;
        const float d = dout[p];
        for (int tap = 0; tap < 9; ++tap) {
            const int oy = tap / 3 - 1, ox = tap % 3 - 1;
            // data gradient: the output pixel p - off(tap) read this pixel through tap
            const int ys = yy - oy, xs = xx - ox;
            if (ys >= 0 && ys < h && xs >= 0 && xs < w) {
                const float dd = dout[(b * h + ys) * w + xs];
                g0 += dd * wh[tap * c + k];
                g1 += dd * wh[tap * c + k + 1];
            }
            // weight gradient: this output pixel reads p + off(tap)
            const int y2 = yy + oy, x2 = xx + ox;
            if (y2 >= 0 && y2 < h && x2 >= 0 && x2 < w) {
                const float2 v =
                    __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(x + ((b * h + y2) * w + x2) * c + k));
                gw[tap][0] += d * v.x;
                gw[tap][1] += d * v.y;
            }
        }
        if (dx) *reinterpret_cast<__nv_bfloat162*>(dx + p * c + k) = __floats2bfloat162_rn(g0, g1);
        if (k == 0) gb += d;
    }
    for (int tap = 0; tap < 9; ++tap) {
        atomicAdd(&part[tap * c + k], gw[tap][0]);
        atomicAdd(&part[tap * c + k + 1], gw[tap][1]);
    }
    if (k == 0) atomicAdd(&part[9 * c], gb);
    __syncthreads();
    for (int j = threadIdx.x; j < 9 * c; j += blockDim.x) atomicAdd(&dwh[j], part[j]);
    if (threadIdx.x == 0) atomicAdd(dbh, part[9 * c]);
}

// Adam step on FP32 master parameters; the BF16 copies of the convolution weights are rewritten
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2, bf16* __restrict__ p_bf16)
{
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const float gq = g[q];
        const float mq = b1 * m[q] + (1.0f - b1) * gq;
        const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        const float pq = p[q] - lr * (mq / c1) / (sqrtf(vq / c2) + eps);
        p[q] = pq;
        if (p_bf16) p_bf16[q] = __float2bfloat16(pq);
    }
}

// one device word per GPU for the bounded waits of the tcgen05 kernels
int* tc_error_word()
{
    static int* words[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (!words[dev]) {
        if (cudaMalloc(&words[dev], sizeof(int)) != cudaSuccess) return nullptr;
        if (cudaMemset(words[dev], 0, sizeof(int)) != cudaSuccess) return nullptr;
    }
    return words[dev];
}

unsigned grid_for(int64_t n, int per = 256)
{
    int64_t g = (n + per - 1) / per;
    if (g > 148 * 16) g = 148 * 16;
    return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace

// ------------------------------------------------------------------------------------------ C ABI
extern "C" {

int edp_nn_conv3x3_fwd(int32_t nimg, int32_t h, int32_t w, const void* x1, int32_t c1, const void* x2, int32_t c2,
                       const void* wt, const float* bias, int32_t cout, int32_t relu, void* y, void* stream)
{
    if (nimg < 1 || h < 1 || w < 1 || !x1 || !wt || !y || c1 < 32 || c1 % 32 || c2 < 0 || c2 % 32 || (c2 && !x2) ||
        cout < 32 || cout % 32 || c1 + c2 > 1024)
        return EDP_ERR_ARG;
    ConvArgs a;
    a.nimg = nimg;
    a.h = h;
    a.w = w;
    a.x1 = (const bf16*)x1;
    a.c1 = c1;
    a.x2 = (const bf16*)x2;
    a.c2 = c2;
    a.wt = (const bf16*)wt;
    a.bias = bias;
    a.cout = cout;
    a.relu = relu;
    a.y = (bf16*)y;
    cudaStream_t s = (cudaStream_t)stream;
    int* err = tc_error_word();
    if (!err) return EDP_ERR_CUDA;
    const bool halo = g_conv_mode == 2 || (g_conv_mode == 0 && halo_applies(a));
    if (halo) {
        if (!halo_possible(a)) return EDP_ERR_ARG;
        const bool res = halo_resident(a);
        switch (cout) {
        case 32: return res ? launch_halo<32, false>(a, err, s) : launch_halo<32, true>(a, err, s);
        case 64: return res ? launch_halo<64, false>(a, err, s) : launch_halo<64, true>(a, err, s);
        case 128: return launch_halo<128, false>(a, err, s);
        default: return EDP_ERR_ARG;
        }
    }
    // 64-channel chunks when neither c_in nor the concatenation split breaks them, else 32
    if (c1 % 64 == 0 && c2 % 64 == 0) return launch_tma_cout<64>(a, err, s);
    return launch_tma_cout<32>(a, err, s);
}

/* which weight-gradient kernel edp_nn_conv3x3_wgrad uses: 0 (default) tcgen05 with the taps in M, 2 tcgen05 with
 * the taps in N, 1 mma.sync */
int edp_nn_wgrad_select(int32_t mode)
{
    if (mode < 0 || mode > 2) return EDP_ERR_ARG;
    g_wgrad_mode = mode;
    return EDP_OK;
}

/* which forward kernel edp_nn_conv3x3_fwd uses: 0 automatic, 1 the tile kernel, 2 the persistent halo kernel */
int edp_nn_conv_select(int32_t mode)
{
    if (mode < 0 || mode > 2) return EDP_ERR_ARG;
    g_conv_mode = mode;
    return EDP_OK;
}

/* bounded-wait error word of the tcgen05 kernels: nonzero once a wait gave up; reading clears it */
int edp_nn_error(int32_t* out)
{
    int* err = tc_error_word();
    if (!err || !out) return EDP_ERR_ARG;
    int h = 0;
    if (cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return EDP_ERR_CUDA;
    if (h && cudaMemset(err, 0, sizeof(int)) != cudaSuccess) return EDP_ERR_CUDA;
    *out = h;
    return EDP_OK;
}

int edp_nn_flip_transpose(const void* wt, int32_t cout, int32_t cin, void* out, void* stream)
{
    if (!wt || !out || cout < 1 || cin < 1) return EDP_ERR_ARG;
    flip_transpose_kernel<<<grid_for((int64_t)cout * 9 * cin), 256, 0, (cudaStream_t)stream>>>(
        (const bf16*)wt, cout, cin, (bf16*)out);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

int edp_nn_conv3x3_wgrad(int32_t nimg, int32_t h, int32_t w, const void* x1, int32_t c1, const void* x2, int32_t c2,
                         const void* dz, int32_t cout, float* dw, float* db, void* stream)
{
    if (nimg < 1 || h < 1 || w < 1 || !x1 || !dz || !dw || c1 < 32 || c1 % 32 || c2 < 0 || c2 % 32 ||
        (c2 && !x2) || cout < 32 || cout % 32)
        return EDP_ERR_ARG;
    WgradArgs a;
    a.nimg = nimg;
    a.h = h;
    a.w = w;
    a.x = (const bf16*)x1;
    a.c1 = c1;
    a.x2 = (const bf16*)x2;
    a.c2 = c2;
    a.dz = (const bf16*)dz;
    a.cout = cout;
    a.dw = dw;
    const int64_t P = (int64_t)nimg * h * w;
    const int cin = c1 + c2;
    cudaStream_t s = (cudaStream_t)stream;
    if (g_wgrad_mode != 1) {
        int* err = tc_error_word();
        if (!err) return EDP_ERR_CUDA;
        int rc;
        if (g_wgrad_mode == 2) {
            rc = cout % 128 == 0 ? launch_wgrad_tc<128>(a, err, s) : launch_wgrad_tc<64>(a, err, s);
        } else {
            // output channels per CTA: the largest of 128, 64, 32 that divides c_out
            const int nb = cout % 128 == 0 ? 128 : cout % 64 == 0 ? 64 : 32;
            rc = nb == 128 ? launch_wgrad_tap<128>(a, err, s)
                 : nb == 64 ? launch_wgrad_tap<64>(a, err, s)
                            : launch_wgrad_tap<32>(a, err, s);
        }
        if (rc != EDP_OK) return rc;
        if (db) {
            const int lanes = 1024 / cout;
            bias_grad_kernel<<<grid_for(P, 1024), lanes * cout, lanes * cout * sizeof(float), s>>>((const bf16*)dz, P,
                                                                                                cout, db);
        }
        return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
    }
    const int bm = cout % 64 == 0 ? 64 : 32;
    // the input-channel tile must not straddle the two concatenated tensors
    const int bn = (cin % 64 == 0 && c1 % 64 == 0) ? 64 : 32;
    const int64_t tiles = (int64_t)(cout / bm) * 9 * (cin / bn);
    // K split: about 4 CTAs per SM overall, at least 1024 pixels per CTA
    int64_t per = (P * tiles + 148 * 4 - 1) / (148 * 4);
    if (per < 1024) per = 1024;
    per = (per + kWK - 1) / kWK * kWK;
    a.pix_per_cta = per;
    dim3 grid((unsigned)((P + per - 1) / per), (unsigned)tiles);
    if (bm == 64 && bn == 64) conv3x3_wgrad_kernel<64, 64><<<grid, 256, 0, s>>>(a);
    else if (bm == 64) conv3x3_wgrad_kernel<64, 32><<<grid, 128, 0, s>>>(a);
    else if (bn == 64) conv3x3_wgrad_kernel<32, 64><<<grid, 128, 0, s>>>(a);
    else conv3x3_wgrad_kernel<32, 32><<<grid, 64, 0, s>>>(a);
    if (db) {
        const int lanes = 1024 / cout;
        bias_grad_kernel<<<grid_for(P, 1024), lanes * cout, lanes * cout * sizeof(float), s>>>((const bf16*)dz, P,
                                                                                            cout, db);
    }
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

int edp_nn_pool(int32_t nimg, int32_t h, int32_t w, int32_t c, int32_t f, const void* x, void* y, void* stream)
{
    if ((f != 2 && f != 4) || h % f || w % f || !x || !y) return EDP_ERR_ARG;
    pool_fwd_kernel<<<grid_for((int64_t)nimg * h * w * c / (f * f)), 256, 0, (cudaStream_t)stream>>>(
        (const bf16*)x, nimg, h, w, c, f, (bf16*)y);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

int edp_nn_pool_bwd(int32_t nimg, int32_t h, int32_t w, int32_t c, int32_t f, const void* dy, void* dx,
                    int32_t accumulate, void* stream)
{
    if ((f != 2 && f != 4) || h % f || w % f || !dy || !dx) return EDP_ERR_ARG;
    pool_bwd_kernel<<<grid_for((int64_t)nimg * h * w * c), 256, 0, (cudaStream_t)stream>>>(
        (const bf16*)dy, nimg, h, w, c, f, (bf16*)dx, accumulate);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

int edp_nn_upsample(int32_t nimg, int32_t h, int32_t w, int32_t c, int32_t f, const void* x, void* y, void* stream)
{
    if ((f != 2 && f != 4) || h % f || w % f || !x || !y) return EDP_ERR_ARG;
    up_fwd_kernel<<<grid_for((int64_t)nimg * h * w * c), 256, 0, (cudaStream_t)stream>>>((const bf16*)x, nimg, h, w, c,
                                                                                      f, (bf16*)y);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

int edp_nn_upsample_bwd(int32_t nimg, int32_t h, int32_t w, int32_t c, int32_t cs, int32_t f, const void* dy, void* dx,
                        void* stream)
{
    if ((f != 2 && f != 4) || h % f || w % f || !dy || !dx || cs < c) return EDP_ERR_ARG;
    up_bwd_kernel<<<grid_for((int64_t)nimg * h * w * c / (f * f)), 256, 0, (cudaStream_t)stream>>>(
        (const bf16*)dy, nimg, h, w, c, cs, f, (bf16*)dx);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

int edp_nn_relu_bwd(int64_t P, int32_t c, const void* dy, int32_t cs, int32_t co, const void* dy2, const void* y,
                    void* dz, void* stream)
{
    if (!dy || !y || !dz || cs < co + c) return EDP_ERR_ARG;
    relu_bwd_kernel<<<grid_for(P * c), 256, 0, (cudaStream_t)stream>>>((const bf16*)dy, cs, co, (const bf16*)dy2,
                                                                       (const bf16*)y, P, c, (bf16*)dz);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

int edp_nn_head_fwd(int32_t nimg, int32_t h, int32_t w, int32_t c, const void* x, const float* wh, const float* bh,
                    float* out, void* stream)
{
    if (!x || !wh || !bh || !out || c % 2) return EDP_ERR_ARG;
    head_fwd_kernel<<<grid_for((int64_t)nimg * h * w), 256, 0, (cudaStream_t)stream>>>((const bf16*)x, nimg, h, w, c,
                                                                                    wh, bh, out);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

int edp_nn_head_bwd(int32_t nimg, int32_t h, int32_t w, int32_t c, const void* x, const float* wh, const float* dout,
                    void* dx, float* dwh, float* dbh, void* stream)
{
    if (!x || !wh || !dout || !dwh || !dbh || c % 2 || 256 % (c / 2)) return EDP_ERR_ARG;
    head_bwd_kernel<<<grid_for((int64_t)nimg * h * w * c / 2), 256, (9 * c + 1) * sizeof(float),
                      (cudaStream_t)stream>>>((const bf16*)x, nimg, h, w, c, wh, dout, (bf16*)dx, dwh, dbh);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

int edp_nn_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2, float eps,
                int32_t step, void* p_bf16, void* stream)
{
    if (!p || !g || !m || !v || n < 1 || step < 1) return EDP_ERR_ARG;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, beta1, beta2, eps, c1, c2,
                                                               (bf16*)p_bf16);
    return cudaGetLastError() == cudaSuccess ? EDP_OK : EDP_ERR_CUDA;
}

}  // extern "C"
