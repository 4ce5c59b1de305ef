// Snapshot files in the reference's binary layouts, for one cluster over the whole domain. Host code: the arrays come
// from edp_collect_moments / edp_get_field / edp_calculate_vdf. All values are written in the machine's byte order as
// 4-byte REAL / INTEGER, as MPI_FILE_WRITE writes them with the native representation.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../include/edipic_gpu.h"

namespace {

struct File {
    FILE* f;
    explicit File(const char* path) : f(std::fopen(path, "wb")) {}
    ~File()
    {
        if (f) std::fclose(f);
    }
    bool put(const void* p, size_t bytes) { return f && std::fwrite(p, 1, bytes, f) == bytes; }
};

// box edges in metres: REAL(area_min * dx), REAL((area_min + DBLE(i) * (area_max - area_min) / N) * dx), REAL(area_max
// * dx) (pic2d_Snapshots.f90:1412-1426 of SAVE_ALL_VDF1D, the same in SAVE_ALL_VDF2D)
std::vector<float> box_edges(int32_t n, double area_max, double dx)
{
    std::vector<float> e(n + 1);
    e[0] = (float)(0.0 * dx);
    for (int i = 1; i < n; ++i) e[i] = (float)((0.0 + (double)i * (area_max - 0.0) / n) * dx);
    e[n] = (float)(area_max * dx);
    return e;
}

}  // namespace

extern "C" {

// SAVE_GLOBAL_2D_ARRAY (pic2d_Snapshots.f90:1207-1355) with one cluster: a gnuplot binary matrix. Row 0 is
// {REAL(global_maximal_i + 1), x_0 .. x_gmi} with x_i = REAL(i * delta_x_m); row 1 + j is {REAL(j * delta_x_m),
// arr(0:gmi, j)} for j = 0 .. gmj. arr is [ny_nodes][nx_nodes], nx_nodes = global_maximal_i + 1.
int edp_write_snapshot_2d(const char* path, const float* arr, int32_t nx_nodes, int32_t ny_nodes, double delta_x_m)
{
    if (!path || !arr || nx_nodes < 1 || ny_nodes < 1) return EDP_ERR_ARG;
    File f(path);
    if (!f.f) return EDP_ERR_IO;
    std::vector<float> row(nx_nodes + 1);
    row[0] = (float)nx_nodes;
    for (int i = 0; i < nx_nodes; ++i) row[1 + i] = (float)(i * delta_x_m);
    if (!f.put(row.data(), row.size() * 4)) return EDP_ERR_IO;
    for (int j = 0; j < ny_nodes; ++j) {
        row[0] = (float)(j * delta_x_m);
        for (int i = 0; i < nx_nodes; ++i) row[1 + i] = arr[(int64_t)j * nx_nodes + i];
        if (!f.put(row.data(), row.size() * 4)) return EDP_ERR_IO;
    }
    return EDP_OK;
}

// SAVE_ALL_VDF1D (pic2d_Snapshots.f90:1359-1544) with one cluster: header {nbx, nby, vmin_e, vmax_e, vmin_i, vmax_i,
// N_vbins_e, N_vbins_i, N_spec} (INTEGER), {T_e_eV, M_i_amu(1:N_spec)} (REAL); then per box (i fastest) its edges
// {x0, x1, y0, y1} (REAL) and evxdf, evydf, evzdf, then isvxdf, isvydf, isvzdf of each ion species (INTEGER).
// e1d = [3][nbox][2 n_max_vel_e n_vbins_e] and i1d = [n_spec][3][nbox][2 n_max_vel_i n_vbins_i] as edp_calculate_vdf
// returns them; x_area_max, y_area_max = c_X_area_max, c_Y_area_max of the cluster.
int edp_write_vdf1d(const char* path, int32_t nbx, int32_t nby, double x_area_max, double y_area_max,
                    double delta_x_m, int32_t n_max_vel_e, int32_t n_vbins_e, int32_t n_max_vel_i, int32_t n_vbins_i,
                    int32_t n_spec, double t_e_ev, const double* m_i_amu, const int32_t* e1d, const int32_t* i1d)
{
    if (!path || nbx < 1 || nby < 1 || n_spec < 0 || n_spec > EDP_MAX_ION_SPECIES || !e1d || (n_spec && !i1d) ||
        (n_spec && !m_i_amu))
        return EDP_ERR_ARG;
    File f(path);
    if (!f.f) return EDP_ERR_IO;
    const int32_t rle = 2 * n_max_vel_e * n_vbins_e, rli = 2 * n_max_vel_i * n_vbins_i, nbox = nbx * nby;
    const int32_t head[9] = {nbx, nby, -rle / 2, rle / 2 - 1, -rli / 2, rli / 2 - 1, n_vbins_e, n_vbins_i, n_spec};
    if (!f.put(head, sizeof(head))) return EDP_ERR_IO;
    std::vector<float> r(1 + n_spec);
    r[0] = (float)t_e_ev;
    for (int s = 0; s < n_spec; ++s) r[1 + s] = (float)m_i_amu[s];
    if (!f.put(r.data(), r.size() * 4)) return EDP_ERR_IO;
    const std::vector<float> xs = box_edges(nbx, x_area_max, delta_x_m), ys = box_edges(nby, y_area_max, delta_x_m);
    for (int j = 0; j < nby; ++j)
        for (int i = 0; i < nbx; ++i) {
            const int n = i + j * nbx;
            const float edges[4] = {xs[i], xs[i + 1], ys[j], ys[j + 1]};
            if (!f.put(edges, sizeof(edges))) return EDP_ERR_IO;
            for (int c = 0; c < 3; ++c)
                if (!f.put(e1d + ((int64_t)c * nbox + n) * rle, (size_t)rle * 4)) return EDP_ERR_IO;
            for (int s = 0; s < n_spec; ++s)
                for (int c = 0; c < 3; ++c)
                    if (!f.put(i1d + (((int64_t)s * 3 + c) * nbox + n) * rli, (size_t)rli * 4)) return EDP_ERR_IO;
        }
    return EDP_OK;
}

// SAVE_ALL_VDF2D (pic2d_Snapshots.f90:1548-1705) with one cluster: header {nbx, nby, vmin_e, vmax_e, N_vbins_e}
// (INTEGER), {T_e_eV} (REAL); then per box its edges {x0, x1, y0, y1} (REAL) and evxvydf(vx, vy) with vx fastest
// (INTEGER). e2d = [nbox][vy][vx] as edp_calculate_vdf returns it.
int edp_write_vdf2d(const char* path, int32_t nbx, int32_t nby, double x_area_max, double y_area_max,
                    double delta_x_m, int32_t n_max_vel_e, int32_t n_vbins_e, double t_e_ev, const int32_t* e2d)
{
    if (!path || nbx < 1 || nby < 1 || !e2d) return EDP_ERR_ARG;
    File f(path);
    if (!f.f) return EDP_ERR_IO;
    const int32_t rl = 2 * n_max_vel_e * n_vbins_e;
    const int32_t head[5] = {nbx, nby, -rl / 2, rl / 2 - 1, n_vbins_e};
    if (!f.put(head, sizeof(head))) return EDP_ERR_IO;
    const float te = (float)t_e_ev;
    if (!f.put(&te, 4)) return EDP_ERR_IO;
    const std::vector<float> xs = box_edges(nbx, x_area_max, delta_x_m), ys = box_edges(nby, y_area_max, delta_x_m);
    for (int j = 0; j < nby; ++j)
        for (int i = 0; i < nbx; ++i) {
            const int n = i + j * nbx;
            const float edges[4] = {xs[i], xs[i + 1], ys[j], ys[j + 1]};
            if (!f.put(edges, sizeof(edges))) return EDP_ERR_IO;
            if (!f.put(e2d + (int64_t)n * rl * rl, (size_t)rl * rl * 4)) return EDP_ERR_IO;
        }
    return EDP_OK;
}

}  // extern "C"
