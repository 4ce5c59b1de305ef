// x strips of a periodic domain over several contexts (the reference's clusters along x:
// pic2d_ParticleExchange.f90:3-1762 moves the particles between neighbouring clusters, and GATHER_*_CHARGE_DENSITY
// pic2d_ElectronDynamics.f90:1645-1800 sums the densities of the nodes the clusters share).
//
// A strip context holds its own columns plus ghost columns on the sides that face another strip (a side on the
// domain's wall has none). Its particles are pushed against the field copied from a context that solves the whole
// grid, and deposit into the strip's nodes, ghost nodes included; the strips' densities are summed into the whole
// grid before the next solve. After a step, particles in
// the ghost columns belong to a neighbour: edp_strip_take lifts them out as records, the caller moves the records,
// and edp_strip_put appends them to the neighbour without depositing (the sender already did). Positions keep
// their FP32 in-cell offsets and ids, so a run over strips does the arithmetic of the one-context run.
#include "edp_internal.cuh"

namespace {

constexpr int kRec = 8;   // doubles per record: x, y, vx, vy, vz, id, tag, 0

__device__ __forceinline__ int pos_mod(int a, int n)
{
    int r = a % n;
    return r < 0 ? r + n : r;
}

// A particle leaves the strip only when its record was written: one past a full buffer stays in its ghost column,
// is still counted in cnt, and a later call with a larger buffer takes it.
__global__ void strip_take_kernel(edp_kparams kp, edp_species_mixed P, const unsigned long long* n_slots,
                                  double* left, int64_t cap_l, double* right, int64_t cap_r, unsigned long long* cnt,
                                  unsigned long long* n_live)
{
    const int64_t n = (int64_t)*n_slots;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int c = P.cell[k];
        if (c < 0) continue;
        const int i = c & 0xFFFF;
        const int side = i < kp.strip_gl ? 0 : (i >= kp.ncx - kp.strip_gr ? 1 : -1);
        if (side < 0) continue;
        const unsigned long long pos = atomicAdd(&cnt[side], 1ull);
        if ((int64_t)pos < (side ? cap_r : cap_l)) {
            double* r = (side ? right : left) + (int64_t)pos * kRec;
            r[0] = (double)i + (double)P.ox[k];
            r[1] = (double)(c >> 16) + (double)P.oy[k];
            r[2] = (double)P.vx[k];
            r[3] = (double)P.vy[k];
            r[4] = (double)P.vz[k];
            r[5] = (double)P.id[k];
            r[6] = (double)P.tag[k];
            r[7] = 0.0;
            P.cell[k] = -1;
            atomicAdd(n_live, (unsigned long long)(-1LL));
        }
    }
}

__global__ void strip_put_kernel(edp_kparams kp, edp_species_mixed P, const double* rec, int64_t n, double shift,
                                 unsigned long long* n_slots, unsigned long long* n_live, int64_t cap,
                                 unsigned int* eflag)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double* r = rec + k * kRec;
        const double X = r[0] + shift, Y = r[1];
        if (!(X >= 0.0 && X <= (double)kp.ncx && Y >= 0.0 && Y <= (double)kp.ncy)) {
            atomicOr(eflag, EDP_EFLAG_BOUNDS);
            continue;
        }
        const unsigned long long slot = atomicAdd(n_slots, 1ull);
        if ((int64_t)slot >= cap) {
            atomicOr(eflag, EDP_EFLAG_CAPACITY);
            continue;
        }
        int i = (int)X, j = (int)Y;
        float ox, oy;
        if (i == kp.ncx) {   // X == c_X_area_max, as the upload stores it
            i = kp.ncx - 1;
            ox = 1.0f;
        } else {
            ox = (float)(X - (double)i);   // exact: an integer shift of an FP32 offset
        }
        if (j == kp.ncy) {
            j = kp.ncy - 1;
            oy = 1.0f;
        } else {
            oy = (float)(Y - (double)j);
        }
        P.cell[slot] = (j << 16) | i;
        P.ox[slot] = ox;
        P.oy[slot] = oy;
        P.vx[slot] = (float)r[2];
        P.vy[slot] = (float)r[3];
        P.vz[slot] = (float)r[4];
        P.id[slot] = (uint32_t)r[5];
        P.tag[slot] = (int32_t)r[6];
        atomicAdd(n_live, 1ull);
    }
}

__global__ void strip_add_density_kernel(const unsigned long long* __restrict__ local, int nxl, int nyl,
                                         unsigned long long* __restrict__ global, int nxg, int x_first)
{
    const int64_t n = (int64_t)nxl * nyl;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long v = local[q];
        if (!v) continue;
        const int il = (int)(q % nxl), j = (int)(q / nxl);
        atomicAdd(&global[(int64_t)j * nxg + pos_mod(x_first + il, nxg)], v);
    }
}

__global__ void strip_field_kernel(const float2* __restrict__ e, const float2* __restrict__ acc, int nxg, int x_first,
                                   float2* __restrict__ el, float2* __restrict__ accl, int nxl, int nyl)
{
    const int64_t n = (int64_t)nxl * nyl;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int il = (int)(q % nxl), j = (int)(q / nxl);
        const int64_t src = (int64_t)j * nxg + pos_mod(x_first + il, nxg);
        el[q] = e[src];
        if (acc) accl[q] = acc[src];
    }
}

unsigned grid_for_n(int64_t n)
{
    int64_t g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    return (unsigned)(g < 1 ? 1 : g);
}

int sync_if_asked(edp_ctx* c)   // calls are synchronous at the ABI edge unless the context runs asynchronously
{
    if (c->sync) EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    return EDP_OK;
}

int check_flags(edp_ctx* c)
{
    unsigned int flags = 0;
    EDP_CUDA(c, cudaMemcpy(&flags, &c->dc->error_flags, sizeof(flags), cudaMemcpyDeviceToHost));
    if (flags & EDP_EFLAG_BOUNDS)
        return edp_fail(c, EDP_ERR_BOUNDS, "a particle left the strip and its ghost columns in one step");
    if (flags & EDP_EFLAG_CAPACITY) return edp_fail(c, EDP_ERR_CAPACITY, "strip record buffer or particle capacity");
    return EDP_OK;
}

}  // namespace

int edp_set_strip(edp_ctx* c, int32_t ghost_left, int32_t ghost_right, int32_t x_first, int32_t ncx_global,
                  int32_t periodic)
{
    if (!c || ghost_left < 0 || ghost_right < 0 || ncx_global < 2 || (periodic && (!ghost_left || !ghost_right)) ||
        (!periodic && (x_first < 0 || x_first + c->p.ncx > ncx_global)))
        return edp_fail(c, EDP_ERR_ARG, "edp_set_strip: ghost columns, position in the domain");
    if (c->kp.periodic || c->p.precision != EDP_PREC_MIXED || c->kp.diel_mask || c->p.ncx <= ghost_left + ghost_right)
        return edp_fail(c, EDP_ERR_STATE, "a strip is a walled-x, mixed-precision context without dielectric objects, "
                                          "wider than its ghost margins");
    if (c->emit_on || c->see_on || c->inject_on) return edp_fail(c, EDP_ERR_STATE, "no wall emission on a strip");
    for (int s = 0; s < c->nspec; ++s)
        if (c->uploaded[s]) return edp_fail(c, EDP_ERR_STATE, "edp_set_strip before the particles are uploaded");
    if (!c->strip_cnt) EDP_CUDA(c, cudaMalloc(&c->strip_cnt, 2 * sizeof(unsigned long long)));
    c->kp.strip = 1;
    c->kp.strip_gl = ghost_left;
    c->kp.strip_gr = ghost_right;
    c->kp.strip_x0 = x_first;
    c->kp.strip_ncx = ncx_global;
    c->kp.strip_periodic = periodic ? 1 : 0;
    return EDP_OK;
}

int edp_strip_take(edp_ctx* c, int32_t sp, double* left, int64_t cap_left, double* right, int64_t cap_right,
                   int64_t* n_left, int64_t* n_right)
{
    if (!c || !n_left || !n_right || sp < 0 || sp >= c->nspec || cap_left < 0 || cap_right < 0 ||
        (cap_left && !left) || (cap_right && !right))
        return edp_fail(c, EDP_ERR_ARG, "edp_strip_take");
    if (!c->kp.strip) return edp_fail(c, EDP_ERR_STATE, "not a strip context");
    *n_left = *n_right = 0;
    if (!c->uploaded[sp]) return EDP_OK;
    EDP_CUDA(c, cudaMemsetAsync(c->strip_cnt, 0, 2 * sizeof(unsigned long long), c->stream));
    ++c->launches;
    strip_take_kernel<<<grid_for_n(c->host_slots[sp]), 256, 0, c->stream>>>(
        c->kp, c->pm[sp], &c->dc->n_slots[sp], left, cap_left, right, cap_right, c->strip_cnt, &c->dc->n_live[sp]);
    EDP_CUDA(c, cudaGetLastError());
    unsigned long long h[2];
    EDP_CUDA(c, cudaMemcpyAsync(h, c->strip_cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    EDP_CUDA(c, cudaStreamSynchronize(c->stream));
    *n_left = (int64_t)h[0];
    *n_right = (int64_t)h[1];
    int r = check_flags(c);
    if (r != EDP_OK) return r;
    // not a device error flag: the context stays usable, and the particles past the buffers are still in the strip
    if ((int64_t)h[0] > cap_left || (int64_t)h[1] > cap_right)
        return edp_fail(c, EDP_ERR_CAPACITY, "edp_strip_take: record buffer smaller than the ghost-column count");
    return EDP_OK;
}

int edp_strip_put(edp_ctx* c, int32_t sp, const double* rec, int64_t n, double x_shift)
{
    if (!c || sp < 0 || sp >= c->nspec || n < 0 || (n && !rec)) return edp_fail(c, EDP_ERR_ARG, "edp_strip_put");
    if (!c->kp.strip) return edp_fail(c, EDP_ERR_STATE, "not a strip context");
    if (!c->uploaded[sp]) return edp_fail(c, EDP_ERR_STATE, "edp_strip_put before the species was uploaded");
    if (n == 0) return EDP_OK;
    if (c->host_slots[sp] + n > c->cap[sp]) return edp_fail(c, EDP_ERR_CAPACITY, "edp_strip_put: particle capacity");
    ++c->launches;
    strip_put_kernel<<<grid_for_n(n), 256, 0, c->stream>>>(c->kp, c->pm[sp], rec, n, x_shift, &c->dc->n_slots[sp],
                                                          &c->dc->n_live[sp], c->cap[sp], &c->dc->error_flags);
    EDP_CUDA(c, cudaGetLastError());
    c->host_slots[sp] += n;
    return sync_if_asked(c);
}

int edp_strip_add_density(edp_ctx* c, int32_t sp, uint64_t* global_dev, int32_t nx_global, int32_t x_first)
{
    if (!c || sp < 0 || sp >= c->nspec || !global_dev || nx_global < 1) return edp_fail(c, EDP_ERR_ARG, "edp_strip_add_density");
    if (!c->kp.strip) return edp_fail(c, EDP_ERR_STATE, "not a strip context");
    ++c->launches;
    strip_add_density_kernel<<<grid_for_n((int64_t)c->kp.nxg * c->kp.nyg), 256, 0, c->stream>>>(
        c->rho_fix[sp], c->kp.nxg, c->kp.nyg, reinterpret_cast<unsigned long long*>(global_dev), nx_global, x_first);
    EDP_CUDA(c, cudaGetLastError());
    return sync_if_asked(c);
}

int edp_strip_set_field(edp_ctx* c, const void* e_global, const void* acc_global, int32_t nx_global, int32_t x_first)
{
    if (!c || !e_global || nx_global < 1) return edp_fail(c, EDP_ERR_ARG, "edp_strip_set_field");
    if (!c->kp.strip) return edp_fail(c, EDP_ERR_STATE, "not a strip context");
    ++c->launches;
    strip_field_kernel<<<grid_for_n((int64_t)c->kp.nxg * c->kp.nyg), 256, 0, c->stream>>>(
        static_cast<const float2*>(e_global), static_cast<const float2*>(acc_global), nx_global, x_first, c->E2,
        c->acc2, c->kp.nxg, c->kp.nyg);
    EDP_CUDA(c, cudaGetLastError());
    return sync_if_asked(c);
}

int edp_device_buffer(edp_ctx* c, int32_t which, int32_t sp, void** ptr, int64_t* count)
{
    if (!c || !ptr || !count) return EDP_ERR_ARG;
    if (c->p.precision != EDP_PREC_MIXED) return edp_fail(c, EDP_ERR_STATE, "edp_device_buffer: mixed precision");
    *count = (int64_t)c->kp.nxg * c->kp.nyg;
    if (which == 0) {
        if (sp < 0 || sp >= c->nspec) return edp_fail(c, EDP_ERR_ARG, "edp_device_buffer: species");
        *ptr = c->rho_fix[sp];
    } else if (which == 1) {
        *ptr = c->E2;
    } else if (which == 2) {
        *ptr = c->acc2;
    } else {
        return edp_fail(c, EDP_ERR_ARG, "edp_device_buffer: which");
    }
    return EDP_OK;
}
