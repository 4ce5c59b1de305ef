// Tile sort of the mixed-precision particle arrays (no reference analogue: EDIPIC-2D keeps particles in
// arrival order). Counting sort on a key of (tile, (source slot / 32) mod 256), so that every EDP_TILE x EDP_TILE
// tile is one contiguous slot range. Inside a tile the 256 sub-buckets interleave runs of 32 source slots: a run
// (one scatter warp) stays contiguous, so its stores and its counter atomic stay coalesced, while the 128
// consecutive particles of one push warp come from four runs 8192 source slots apart. Long runs of one cell (the
// initial distribution fills the slots cell by cell) are thereby spread over the tile, and the lanes of a push
// warp do not pile their shared-memory deposits onto one node; a plain cell order made the push 9 % slower on
// 1024^2 cells at 200 particles per cell. Dead slots are dropped, which is also the compaction of particles
// removed at walls since the last sort. Each tile's range is padded with dead slots to a multiple of EDP_ITEMS, so
// the push reads and writes every tile in whole 128-bit groups.
#include <algorithm>
#include <vector>

#include "edp_internal.cuh"

namespace {

__device__ __forceinline__ uint32_t tile_key(int cell, int64_t k, int ntx) { return edp_tile_key(cell, k, ntx); }

__global__ void hist_kernel(const int32_t* __restrict__ cell, const unsigned long long* n_slots, int ntx,
                            uint32_t* __restrict__ count)
{
    const int64_t n = (int64_t)*n_slots;
    const int lane = threadIdx.x & 31;
    // four blocks of slots per round, their loads issued together
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k0 = (int64_t)blockIdx.x * blockDim.x; k0 < n; k0 += 4 * step) {
        int c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t k = k0 + u * step + threadIdx.x;
            c[u] = k < n ? __ldcs(cell + k) : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t k = k0 + u * step + threadIdx.x;
            const uint32_t key = c[u] >= 0 ? tile_key(c[u], k, ntx) : 0xFFFFFFFFu;
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
            if (key != 0xFFFFFFFFu && lane == __ffs(peers) - 1) atomicAdd(&count[key], (uint32_t)__popc(peers));
        }
    }
}

// exclusive scan of the 256 sub-bucket counts of one tile (one CTA per tile); tile_total[t] = live particles in it
__global__ void tile_scan_kernel(const uint32_t* __restrict__ count, unsigned long long* __restrict__ local,
                                 unsigned long long* __restrict__ tile_total)
{
    __shared__ unsigned warp_sum[8];
    const int t = blockIdx.x, k = threadIdx.x, lane = k & 31, w = k >> 5;
    const unsigned v = count[(int64_t)t * 256 + k];
    unsigned x = v;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    unsigned base = 0;
    for (int q = 0; q < w; ++q) base += warp_sum[q];
    local[(int64_t)t * 256 + k] = (unsigned long long)(base + x - v);
    if (k == 255) tile_total[t] = (unsigned long long)(base + x);
}

// exclusive scan over the tiles of the padded tile sizes (one CTA); tile_base[ntiles] = padded total,
// live = number of live particles
__global__ void tiles_scan_kernel(const unsigned long long* __restrict__ tile_total, int64_t ntiles,
                                  unsigned long long* __restrict__ tile_base, unsigned long long* live)
{
    __shared__ unsigned long long part[1024];
    const int64_t per = (ntiles + blockDim.x - 1) / blockDim.x;
    const int64_t t0 = threadIdx.x * per, t1 = min(t0 + per, ntiles);
    unsigned long long s = 0, l = 0;
    for (int64_t t = t0; t < t1; ++t) {
        unsigned long long v = tile_total[t];
        s += (v + (EDP_ITEMS - 1)) & ~(unsigned long long)(EDP_ITEMS - 1);
        l += v;
    }
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long acc = 0;
        for (int q = 0; q < (int)blockDim.x; ++q) {
            unsigned long long v = part[q];
            part[q] = acc;
            acc += v;
        }
        tile_base[ntiles] = acc;
    }
    __syncthreads();
    unsigned long long acc = part[threadIdx.x];
    for (int64_t t = t0; t < t1; ++t) {
        tile_base[t] = acc;
        acc += (tile_total[t] + (EDP_ITEMS - 1)) & ~(unsigned long long)(EDP_ITEMS - 1);
    }
    // live total
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xFFFFFFFFu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(live, l);
}

// scatter cursors = tile base + offset inside the tile; padding slots at each tile's end marked dead
__global__ void cursor_kernel(const unsigned long long* __restrict__ local, const unsigned long long* __restrict__ tile_base,
                              const unsigned long long* __restrict__ tile_total, int64_t ntiles,
                              unsigned long long* __restrict__ cursor, int32_t* __restrict__ dst_cell, int64_t cap,
                              unsigned int* eflag)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < ntiles * 256) cursor[k] = tile_base[k >> 8] + local[k];
    if (k < ntiles) {
        const unsigned long long e = tile_base[k] + tile_total[k];
        for (unsigned long long q = e; q < tile_base[k + 1]; ++q) {
            if ((int64_t)q < cap) dst_cell[q] = -1;
            else atomicOr(eflag, EDP_EFLAG_CAPACITY);
        }
    }
}

__global__ void scatter_kernel(edp_species_mixed src, edp_species_mixed dst, const unsigned long long* n_slots,
                               int ntx, unsigned long long* __restrict__ cursor, int64_t cap, unsigned int* eflag)
{
    const int64_t n = (int64_t)*n_slots;
    const int lane = threadIdx.x & 31;
    for (int64_t k0 = (int64_t)blockIdx.x * blockDim.x; k0 < n; k0 += (int64_t)gridDim.x * blockDim.x) {
        int64_t k = k0 + threadIdx.x;
        int c = k < n ? src.cell[k] : -1;
        uint32_t key = c >= 0 ? tile_key(c, k, ntx) : 0xFFFFFFFFu;
        unsigned peers = edp_warp_peers(key);
        int leader = __ffs(peers) - 1;
        unsigned long long base = 0;
        if (key != 0xFFFFFFFFu && lane == leader) base = atomicAdd(&cursor[key], (unsigned long long)__popc(peers));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        if (key == 0xFFFFFFFFu) continue;
        unsigned long long pos = base + __popc(peers & ((1u << lane) - 1u));
        if ((int64_t)pos >= cap) {   // the padded total exceeds the capacity: reported, nothing written
            atomicOr(eflag, EDP_EFLAG_CAPACITY);
            continue;
        }
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

__global__ void set_slots(unsigned long long* n_slots, unsigned long long* n_live, const unsigned long long* total,
                          const unsigned long long* live)
{
    *n_slots = *total;
    if (n_live) *n_live = *live;
}

}  // namespace

// histogram of the keys of the current particles, the scans, the cursors of the other arrays and their padding
// slots (marked dead); the scratch layout is tile_total[ntiles] | tile_base[ntiles+1] | cursor[nkeys] | live[1]
int edp_sort_prepare(edp_ctx* c, int sp, unsigned long long** cursor_out)
{
    const int64_t ntiles = (int64_t)c->ntx * c->nty;
    const int64_t nkeys = ntiles * 256;
    const int64_t nslots = std::max<int64_t>(c->host_slots[sp], 1);
    unsigned grid = (unsigned)std::min<int64_t>((nslots + 255) / 256, 148 * 16);
    unsigned long long* tile_total = c->scan_tmp;
    unsigned long long* tile_base = tile_total + ntiles;
    unsigned long long* cursor = tile_base + ntiles + 1;
    unsigned long long* live = cursor + nkeys;
    EDP_CUDA(c, cudaMemsetAsync(c->sort_count, 0, nkeys * sizeof(uint32_t), c->stream));
    EDP_CUDA(c, cudaMemsetAsync(live, 0, sizeof(unsigned long long), c->stream));
    ++c->launches;
    hist_kernel<<<grid, 256, 0, c->stream>>>(c->pm[sp].cell, &c->dc->n_slots[sp], c->ntx, c->sort_count);
    ++c->launches;
    tile_scan_kernel<<<(unsigned)ntiles, 256, 0, c->stream>>>(c->sort_count, c->sort_offset, tile_total);
    ++c->launches;
    tiles_scan_kernel<<<1, 1024, 0, c->stream>>>(tile_total, ntiles, tile_base, live);
    ++c->launches;
    cursor_kernel<<<(unsigned)((nkeys + 255) / 256), 256, 0, c->stream>>>(c->sort_offset, tile_base, tile_total,
                                                                           ntiles, cursor, c->pm_alt[sp].cell,
                                                                           c->cap[sp], &c->dc->error_flags);
    EDP_CUDA(c, cudaGetLastError());
    *cursor_out = cursor;
    return EDP_OK;
}

// after the particles were written to their sorted slots in pm_alt: slot count (and, for the separate pass, the live
// count), swap, and the chunk list of the new order (one synchronisation)
static int sort_finish(edp_ctx* c, int sp, bool set_live)
{
    const int64_t ntiles = (int64_t)c->ntx * c->nty;
    const int64_t nkeys = ntiles * 256;
    unsigned long long* tile_total = c->scan_tmp;
    unsigned long long* tile_base = tile_total + ntiles;
    unsigned long long* live = tile_base + ntiles + 1 + nkeys;
    ++c->launches;
    set_slots<<<1, 1, 0, c->stream>>>(&c->dc->n_slots[sp], set_live ? &c->dc->n_live[sp] : nullptr,
                                      tile_base + ntiles, live);
    EDP_CUDA(c, cudaGetLastError());
    std::swap(c->pm[sp], c->pm_alt[sp]);
    std::vector<unsigned long long> h(ntiles + 1);
    EDP_CUDA(c, cudaMemcpyAsync(h.data(), tile_base, (ntiles + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    if ((int64_t)h[ntiles] > c->cap[sp])
        return edp_fail(c, EDP_ERR_CAPACITY, "sorted particles with tile padding exceed the capacity");
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
    c->sort_due[sp] = 0;
    return EDP_OK;
}

int edp_sort_finish(edp_ctx* c, int sp) { return sort_finish(c, sp, false); }

int edp_launch_sort(edp_ctx* c, int sp)
{
    if (c->p.precision != EDP_PREC_MIXED) return EDP_OK;
    const int64_t nslots = std::max<int64_t>(c->host_slots[sp], 1);
    unsigned grid = (unsigned)std::min<int64_t>((nslots + 255) / 256, 148 * 16);
    unsigned long long* cursor = nullptr;
    TRY(edp_sort_prepare(c, sp, &cursor));
    ++c->launches;
    scatter_kernel<<<grid, 256, 0, c->stream>>>(c->pm[sp], c->pm_alt[sp], &c->dc->n_slots[sp], c->ntx, cursor,
                                                c->cap[sp], &c->dc->error_flags);
    EDP_CUDA(c, cudaGetLastError());
    return sort_finish(c, sp, true);
}
