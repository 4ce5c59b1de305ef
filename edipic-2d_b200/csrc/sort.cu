// Cell sort of the mixed-precision particle arrays (no reference analogue: EDIPIC-2D keeps particles in
// arrival order). Counting sort on a tile-major cell key, so that every EDP_TILE x EDP_TILE tile is one
// contiguous slot range and, inside it, particles of one cell are adjacent. Dead slots are dropped, which
// is also the compaction of particles removed at walls since the last sort.
#include <algorithm>
#include <vector>

#include "edp_internal.cuh"

namespace {

__device__ __forceinline__ uint32_t tile_key(int cell, int ntx)
{
    int i = cell & 0xFFFF, j = cell >> 16;
    return ((uint32_t)((j >> 4) * ntx + (i >> 4)) << 8) | (uint32_t)(((j & 15) << 4) | (i & 15));
}

__global__ void hist_kernel(const int32_t* __restrict__ cell, const unsigned long long* n_slots, int ntx,
                            uint32_t* __restrict__ count)
{
    const int64_t n = (int64_t)*n_slots;
    const int lane = threadIdx.x & 31;
    for (int64_t k0 = (int64_t)blockIdx.x * blockDim.x; k0 < n; k0 += (int64_t)gridDim.x * blockDim.x) {
        int64_t k = k0 + threadIdx.x;
        int c = k < n ? cell[k] : -1;
        uint32_t key = c >= 0 ? tile_key(c, ntx) : 0xFFFFFFFFu;
        unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
        if (key != 0xFFFFFFFFu && lane == __ffs(peers) - 1) atomicAdd(&count[key], (uint32_t)__popc(peers));
    }
}

// exclusive scan, three phases: per-block scan (2048 keys), scan of block sums, add
#define SCAN_BLOCK 2048
__global__ void scan_local(const uint32_t* __restrict__ in, unsigned long long* __restrict__ out,
                           unsigned long long* __restrict__ bsum, int64_t n)
{
    __shared__ unsigned long long s[SCAN_BLOCK];
    const int64_t base = (int64_t)blockIdx.x * SCAN_BLOCK;
    for (int t = threadIdx.x; t < SCAN_BLOCK; t += blockDim.x) s[t] = (base + t < n) ? in[base + t] : 0ull;
    __syncthreads();
    for (int off = 1; off < SCAN_BLOCK; off <<= 1) {
        unsigned long long v[SCAN_BLOCK / 256];
        int q = 0;
        for (int t = threadIdx.x; t < SCAN_BLOCK; t += blockDim.x, ++q) v[q] = (t >= off) ? s[t - off] : 0ull;
        __syncthreads();
        q = 0;
        for (int t = threadIdx.x; t < SCAN_BLOCK; t += blockDim.x, ++q) s[t] += v[q];
        __syncthreads();
    }
    for (int t = threadIdx.x; t < SCAN_BLOCK; t += blockDim.x)
        if (base + t < n) out[base + t] = (t == 0) ? 0ull : s[t - 1];
    if (threadIdx.x == 0) bsum[blockIdx.x] = s[SCAN_BLOCK - 1];
}

__global__ void scan_sums(unsigned long long* bsum, int64_t nb, unsigned long long* total)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long acc = 0;
    for (int64_t b = 0; b < nb; ++b) {
        unsigned long long v = bsum[b];
        bsum[b] = acc;
        acc += v;
    }
    *total = acc;
}

__global__ void scan_add(unsigned long long* out, const unsigned long long* bsum, int64_t n)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] += bsum[k / SCAN_BLOCK];
}

__global__ void copy_u64(unsigned long long* dst, const unsigned long long* src, int64_t n)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = src[k];
}

__global__ void scatter_kernel(edp_species_mixed src, edp_species_mixed dst, const unsigned long long* n_slots,
                               int ntx, unsigned long long* __restrict__ cursor)
{
    const int64_t n = (int64_t)*n_slots;
    const int lane = threadIdx.x & 31;
    for (int64_t k0 = (int64_t)blockIdx.x * blockDim.x; k0 < n; k0 += (int64_t)gridDim.x * blockDim.x) {
        int64_t k = k0 + threadIdx.x;
        int c = k < n ? src.cell[k] : -1;
        uint32_t key = c >= 0 ? tile_key(c, ntx) : 0xFFFFFFFFu;
        unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
        int leader = __ffs(peers) - 1;
        unsigned long long base = 0;
        if (key != 0xFFFFFFFFu && lane == leader) base = atomicAdd(&cursor[key], (unsigned long long)__popc(peers));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        if (key == 0xFFFFFFFFu) continue;
        unsigned long long pos = base + __popc(peers & ((1u << lane) - 1u));
        dst.cell[pos] = c;
        dst.ox[pos] = src.ox[k];
        dst.oy[pos] = src.oy[k];
        dst.vx[pos] = src.vx[k];
        dst.vy[pos] = src.vy[k];
        dst.vz[pos] = src.vz[k];
        dst.id[pos] = src.id[k];
        dst.tag[pos] = src.tag[k];
    }
}

__global__ void tile_starts(const unsigned long long* offset, int64_t ntiles, const unsigned long long* total,
                            unsigned long long* out)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntiles) out[t] = offset[t << 8];
    if (t == ntiles) out[t] = *total;
}

__global__ void set_slots(unsigned long long* n_slots, unsigned long long* n_live, const unsigned long long* total)
{
    *n_slots = *total;
    *n_live = *total;
}

}  // namespace

int edp_launch_sort(edp_ctx* c, int sp)
{
    if (c->p.precision != EDP_PREC_MIXED) return EDP_OK;
    const int64_t ntiles = (int64_t)c->ntx * c->nty;
    const int64_t nkeys = ntiles * 256;
    const int64_t nslots = std::max<int64_t>(c->host_slots[sp], 1);
    unsigned grid = (unsigned)std::min<int64_t>((nslots + 255) / 256, 148 * 16);
    EDP_CUDA(c, cudaMemsetAsync(c->sort_count, 0, nkeys * sizeof(uint32_t), c->stream));
    ++c->launches;
    hist_kernel<<<grid, 256, 0, c->stream>>>(c->pm[sp].cell, &c->dc->n_slots[sp], c->ntx, c->sort_count);
    const int64_t nb = (nkeys + SCAN_BLOCK - 1) / SCAN_BLOCK;
    unsigned long long* bsum = c->scan_tmp;
    unsigned long long* total = c->scan_tmp + nb;
    unsigned long long* cursor = c->scan_tmp + nb + 1;
    unsigned long long* starts = cursor + nkeys;
    ++c->launches;
    scan_local<<<(unsigned)nb, 256, 0, c->stream>>>(c->sort_count, c->sort_offset, bsum, nkeys);
    ++c->launches;
    scan_sums<<<1, 32, 0, c->stream>>>(bsum, nb, total);
    ++c->launches;
    scan_add<<<(unsigned)((nkeys + 255) / 256), 256, 0, c->stream>>>(c->sort_offset, bsum, nkeys);
    ++c->launches;
    copy_u64<<<(unsigned)((nkeys + 255) / 256), 256, 0, c->stream>>>(cursor, c->sort_offset, nkeys);
    ++c->launches;
    scatter_kernel<<<grid, 256, 0, c->stream>>>(c->pm[sp], c->pm_alt[sp], &c->dc->n_slots[sp], c->ntx, cursor);
    ++c->launches;
    tile_starts<<<(unsigned)((ntiles + 1 + 255) / 256), 256, 0, c->stream>>>(c->sort_offset, ntiles, total, starts);
    ++c->launches;
    set_slots<<<1, 1, 0, c->stream>>>(&c->dc->n_slots[sp], &c->dc->n_live[sp], total);
    EDP_CUDA(c, cudaGetLastError());
    std::swap(c->pm[sp], c->pm_alt[sp]);
    std::vector<unsigned long long> h(ntiles + 1);
    EDP_CUDA(c, cudaMemcpyAsync(h.data(), starts, (ntiles + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    std::vector<edp_chunk> ch;
    ch.reserve(ntiles * 2);
    for (int64_t t = 0; t < ntiles; ++t) {
        int64_t s0 = (int64_t)h[t], s1 = (int64_t)h[t + 1];
        int tx = (int)(t % c->ntx), ty = (int)(t / c->ntx);
        for (int64_t a = s0; a < s1; a += EDP_CHUNK) {
            edp_chunk e;
            e.start = a;
            e.end = std::min<int64_t>(a + EDP_CHUNK, s1);
            e.wx0 = tx * EDP_TILE - EDP_HALO;
            e.wy0 = ty * EDP_TILE - EDP_HALO;
            ch.push_back(e);
        }
    }
    if ((int64_t)ch.size() > c->chunk_cap[sp]) {
        if (c->chunks[sp]) cudaFree(c->chunks[sp]);
        c->chunk_cap[sp] = (int64_t)ch.size() + 1024;
        EDP_CUDA(c, cudaMalloc(&c->chunks[sp], c->chunk_cap[sp] * sizeof(edp_chunk)));
    }
    if (!ch.empty())
        EDP_CUDA(c, cudaMemcpyAsync(c->chunks[sp], ch.data(), ch.size() * sizeof(edp_chunk), cudaMemcpyHostToDevice,
                                    c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->n_chunks[sp] = (int64_t)ch.size();
    c->sorted_end[sp] = (int64_t)h[ntiles];
    c->host_slots[sp] = (int64_t)h[ntiles];
    return EDP_OK;
}
