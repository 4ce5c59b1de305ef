// ORACLE (test infrastructure only): CPU FP64 restatement of EDIPIC-2D's per-step particle cycle.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load liboracle.so; the
// product library never links or calls it. Each function names the reference routine it restates.
// Built with -ffp-contract=off so the multiply/add order written here is the order executed.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// physical constants of pic2d_Modules.f90:161-168
const double E_CL = 1.602189e-19;
const double M_E_KG = 9.109534e-31;
const double PI = 3.141592653589793;

inline int64_t node(const oracle_geom_t* g, int i, int j) { return (int64_t)j * oracle_nx_nodes(g) + i; }

struct Area {
    double xmin, xmax, ymin, ymax;
    int ixmax, jymax;  // c_indx_x_max, c_indx_y_max
};

Area area_of(const oracle_geom_t* g)
{
    Area a;
    a.xmin = 0.0;
    a.ymin = 0.0;
    a.ixmax = g->periodic ? g->ncx + 1 : g->ncx;
    a.jymax = g->ncy;
    a.xmax = (double)a.ixmax;
    a.ymax = (double)a.jymax;
    return a;
}

inline void remove_particle(oracle_parts_t* p, int64_t k)
{
    // REMOVE_ELECTRON (pic2d_ElectronDynamics.f90:517-555): the last particle takes slot k
    int64_t last = p->n - 1;
    if (k < last) {
        p->x[k] = p->x[last];
        p->y[k] = p->y[last];
        p->vx[k] = p->vx[last];
        p->vy[k] = p->vy[last];
        p->vz[k] = p->vz[last];
        p->tag[k] = p->tag[last];
        p->id[k] = p->id[last];
    }
    p->n = last;
}

inline double uniform(uint32_t x) { return ((double)x + 0.5) * 0x1p-32; }

// the collision decision draw of particle `id` at `step` in stream `tag`: SplitMix64 seeded with mix64(seed ^ tag) at
// position (step << 32) | id; word 0 is the high half
void decision_draw(uint32_t id, uint64_t seed, uint32_t step, uint32_t tag, uint32_t out[2])
{
    const uint64_t z = oracle_splitmix64_at(oracle_mix64(seed ^ tag), ((uint64_t)step << 32) | id);
    out[0] = (uint32_t)(z >> 32);
    out[1] = (uint32_t)z;
}

void philox_block(uint32_t id, uint64_t seed, uint32_t step, uint32_t stream, uint32_t block, uint32_t out[4])
{
    uint32_t ctr[4] = {step, stream, block, (uint32_t)(seed >> 32)};
    uint32_t key[2] = {id, (uint32_t)seed};
    oracle_philox4x32_10(ctr, key, out);
}

}  // namespace

extern "C" {

int32_t oracle_nx_nodes(const oracle_geom_t* g) { return g->periodic ? g->ncx + 2 : g->ncx + 1; }

// ------------------------------------------------------------------------------------------- push
// ADVANCE_ELECTRONS pic2d_ElectronDynamics.f90:3-513 and ADVANCE_IONS pic2d_IonDynamics.f90:3-524 for a
// single cluster covering the domain. Object numbering for hits: 0 below, 1 above, 2 left, 3 right, 4+k inner.
void oracle_push(const oracle_geom_t* g, const oracle_species_t* sp, const double* EX, const double* EY,
                 oracle_parts_t* p, int64_t* hits)
{
    int64_t n_hit = 0;
    oracle_push_hits(g, sp, EX, EY, p, hits, nullptr, 0, &n_hit);
}

void oracle_push_hits(const oracle_geom_t* g, const oracle_species_t* sp, const double* EX, const double* EY,
                      oracle_parts_t* p, int64_t* hits, double* hit_rows, int64_t cap, int64_t* n_hit)
{
    auto record = [&](int obj, double X, double Y, int64_t k) {
        if (hit_rows && *n_hit < cap) {
            double* r = hit_rows + 7 * *n_hit;
            r[0] = obj; r[1] = X; r[2] = Y; r[3] = p->vx[k]; r[4] = p->vy[k]; r[5] = p->vz[k]; r[6] = p->id[k];
        }
        ++*n_hit;
    };
    const Area a = area_of(g);
    const double L = (double)g->ncx;  // L_period_X
    int64_t k = 0;
    while (k < p->n) {
        double X = p->x[k], Y = p->y[k];
        int i = (int)X, j = (int)Y;
        if (X == a.xmax) i = a.ixmax - 1;
        if (Y == a.ymax) j = a.jymax - 1;
        double ax_ip1 = X - (double)i, ax_i = 1.0 - ax_ip1;
        double ay_jp1 = Y - (double)j, ay_j = 1.0 - ay_jp1;
        const double* fx = EX;
        const double* fy = EY;
        double E_X = fx[node(g, i, j)] * ax_i * ay_j + fx[node(g, i + 1, j)] * ax_ip1 * ay_j +
                     fx[node(g, i, j + 1)] * ax_i * ay_jp1 + fx[node(g, i + 1, j + 1)] * ax_ip1 * ay_jp1;
        double E_Y = fy[node(g, i, j)] * ax_i * ay_j + fy[node(g, i + 1, j)] * ax_ip1 * ay_j +
                     fy[node(g, i, j + 1)] * ax_i * ay_jp1 + fy[node(g, i + 1, j + 1)] * ax_ip1 * ay_jp1;
        double vx = p->vx[k], vy = p->vy[k], vz = p->vz[k];
        if (!sp->is_ion) {
            double E_Z = sp->ez;
            double alfa_x = -0.5 * sp->bx, alfa_y = -0.5 * sp->by, alfa_z = -0.5 * sp->bz;
            double ax2 = alfa_x * alfa_x, ay2 = alfa_y * alfa_y, az2 = alfa_z * alfa_z;
            double theta2 = ax2 + ay2 + az2;
            double inv = 1.0 / (1.0 + theta2);
            double K11 = (1.0 - theta2 + 2.0 * ax2) * inv, K12 = 2.0 * (alfa_x * alfa_y + alfa_z) * inv,
                   K13 = 2.0 * (alfa_x * alfa_z - alfa_y) * inv;
            double K21 = 2.0 * (alfa_x * alfa_y - alfa_z) * inv, K22 = (1.0 - theta2 + 2.0 * ay2) * inv,
                   K23 = 2.0 * (alfa_y * alfa_z + alfa_x) * inv;
            double K31 = 2.0 * (alfa_x * alfa_z + alfa_y) * inv, K32 = 2.0 * (alfa_y * alfa_z - alfa_x) * inv,
                   K33 = (1.0 - theta2 + 2.0 * az2) * inv;
            double VXm = vx - 0.5 * E_X, VYm = vy - 0.5 * E_Y, VZm = vz - 0.5 * E_Z;
            double VXp = K11 * VXm + K12 * VYm + K13 * VZm;
            double VYp = K21 * VXm + K22 * VYm + K23 * VZm;
            double VZp = K31 * VXm + K32 * VYm + K33 * VZm;
            vx = VXp - 0.5 * E_X;
            vy = VYp - 0.5 * E_Y;
            vz = VZp - 0.5 * E_Z;
            X = X + vx;
            Y = Y + vy;
        } else {
            double E_Z = sp->ions_sense_ez ? sp->ez * sp->nsub : 0.0;
            double q = sp->qm2;
            if (sp->ions_sense_b) {
                double qn = q * sp->nsub;
                double alfa_x = qn * sp->bx, alfa_y = qn * sp->by, alfa_z = qn * sp->bz;
                double ax2 = alfa_x * alfa_x, ay2 = alfa_y * alfa_y, az2 = alfa_z * alfa_z;
                double theta2 = ax2 + ay2 + az2;
                double inv = 1.0 / (1.0 + theta2);
                double K11 = (1.0 - theta2 + 2.0 * ax2) * inv, K12 = 2.0 * (alfa_x * alfa_y + alfa_z) * inv,
                       K13 = 2.0 * (alfa_x * alfa_z - alfa_y) * inv;
                double K21 = 2.0 * (alfa_x * alfa_y - alfa_z) * inv, K22 = (1.0 - theta2 + 2.0 * ay2) * inv,
                       K23 = 2.0 * (alfa_y * alfa_z + alfa_x) * inv;
                double K31 = 2.0 * (alfa_x * alfa_z + alfa_y) * inv, K32 = 2.0 * (alfa_y * alfa_z - alfa_x) * inv,
                       K33 = (1.0 - theta2 + 2.0 * az2) * inv;
                double VXm = vx + q * E_X, VYm = vy + q * E_Y, VZm = vz + q * E_Z;
                double VXp = K11 * VXm + K12 * VYm + K13 * VZm;
                double VYp = K21 * VXm + K22 * VYm + K23 * VZm;
                double VZp = K31 * VXm + K32 * VYm + K33 * VZm;
                vx = VXp + q * E_X;
                vy = VYp + q * E_Y;
                vz = VZp + q * E_Z;
            } else {
                vx = vx + (q + q) * E_X;
                vy = vy + (q + q) * E_Y;
                vz = vz + (q + q) * E_Z;
            }
            X = X + vx * sp->nsub;
            Y = Y + vy * sp->nsub;
        }
        p->vx[k] = vx;
        p->vy[k] = vy;
        p->vz[k] = vz;

        // inner objects (:160-172): strictly inside the rectangle
        bool hit_inner = false;
        for (int n = 0; n < g->n_inner; ++n) {
            if (X <= (double)g->ileft[n] || X >= (double)g->iright[n]) continue;
            if (Y <= (double)g->jbottom[n] || Y >= (double)g->jtop[n]) continue;
            hits[4 + n]++;
            record(4 + n, X, Y, k);
            hit_inner = true;
            break;
        }
        if (hit_inner) {
            remove_particle(p, k);
            continue;
        }
        if (X >= a.xmin && X <= a.xmax && Y >= a.ymin && Y <= a.ymax) {
            p->x[k] = X;
            p->y[k] = Y;
            ++k;
            continue;
        }
        if (g->periodic) {
            // self-connected periodic cluster (:185-210, :304-330, :430-443, :476-488)
            if (X < a.xmin) X += L;
            else if (X > a.xmax) X -= L;
            if (Y < a.ymin) {
                hits[0]++;
                record(0, X, Y, k);
                remove_particle(p, k);
            } else if (Y > a.ymax) {
                hits[1]++;
                record(1, X, Y, k);
                remove_particle(p, k);
            } else {
                p->x[k] = X;
                p->y[k] = Y;
                ++k;
            }
            continue;
        }
        // walls on four sides, corners of type SURROUNDED_BY_WALL (:212-300, :332-420, :445-474, :490-518)
        int obj;
        if (X < a.xmin) {
            if (Y >= a.ymin + 1.0 && Y <= a.ymax - 1.0) obj = 2;
            else if (Y < a.ymin + 1.0) obj = ((a.xmin - X) < (a.ymin - Y)) ? 0 : 2;
            else obj = ((a.xmin - X) < (Y - a.ymax)) ? 1 : 2;
        } else if (X > a.xmax) {
            if (Y >= a.ymin + 1.0 && Y <= a.ymax - 1.0) obj = 3;
            else if (Y < a.ymin + 1.0) obj = ((X - a.xmax) < (a.ymin - Y)) ? 0 : 3;
            else obj = ((X - a.xmax) < (Y - a.ymax)) ? 1 : 3;
        } else if (Y > a.ymax) {
            obj = 1;
        } else {
            obj = 0;
        }
        hits[obj]++;
        record(obj, X, Y, k);
        remove_particle(p, k);
    }
}

// GATHER_ELECTRON_CHARGE_DENSITY pic2d_ElectronDynamics.f90:1597-1639 (the CIC loop; weight = Qs for ions)
void oracle_deposit(const oracle_geom_t* g, const oracle_parts_t* p, double weight, double* rho)
{
    const Area a = area_of(g);
    const int64_t nn = (int64_t)oracle_nx_nodes(g) * (g->ncy + 1);
    std::fill(rho, rho + nn, 0.0);
    for (int64_t k = 0; k < p->n; ++k) {
        double X = p->x[k], Y = p->y[k];
        int i = (int)X, j = (int)Y;
        if (X == a.xmax) i = a.ixmax - 1;
        if (Y == a.ymax) j = a.jymax - 1;
        double ax_ip1 = X - (double)i, ax_i = 1.0 - ax_ip1;
        double ay_jp1 = Y - (double)j, ay_j = 1.0 - ay_jp1;
        double vij = ax_i * ay_j, vip1j = ax_ip1 * ay_j, vijp1 = ax_i * ay_jp1;
        rho[node(g, i, j)] += weight * vij;
        rho[node(g, i + 1, j)] += weight * vip1j;
        rho[node(g, i, j + 1)] += weight * vijp1;
        rho[node(g, i + 1, j + 1)] += weight * (1.0 - vij - vip1j - vijp1);
    }
}

// periodic fold :1661-1667 and wall factors :1802-1880
// COLLECT_ELECTRON_MOMENTS (pic2d_ElectronMoments.f90:3-425) and COLLECT_ION_MOMENTS (pic2d_IonMoments.f90:3-348):
// 13 CIC-weighted node sums at the particles' current positions (weights in REAL arithmetic :148-157), of the
// velocity v = (VX, VY, VZ) for ions (pic2d_IonMoments.f90:154-166) and, for electrons, of the mean of the stored
// velocity and its Boris update with the current field (:159-243); overlap columns folded
// (SYNCHRONIZE_MOMENTS_IN_OVERLAP_NODES, :353 and :428-), normalised per node (:356-419) and the density scaled at
// the walls (ADJUST_DENSITY_AT_WALL_BOUNDARIES :422 and :1829-1934, one cluster: flat walls x2, corners x4). out[m * nodes + node], m = N, VX, VY, VZ, WX, WY, WZ,
// VXVY, VXVZ, VYVZ, QX, QY, QZ. Sums are kept in FP64 (the reference keeps REAL).
void oracle_collect_moments(const oracle_geom_t* g, const oracle_species_t* sp, const double* EX, const double* EY,
                            const oracle_parts_t* p, double* out)
{
    const Area a = area_of(g);
    const int nx = oracle_nx_nodes(g);
    const int64_t nn = (int64_t)nx * (g->ncy + 1);
    for (int64_t q = 0; q < 13 * nn; ++q) out[q] = 0.0;
    for (int64_t k = 0; k < p->n; ++k) {
        const double X = p->x[k], Y = p->y[k];
        int i = (int)X, j = (int)Y;
        if (X == a.xmax) i = a.ixmax - 1;
        if (Y == a.ymax) j = a.jymax - 1;
        const float ax_ip1 = (float)(X - (double)i), ax_i = 1.0f - ax_ip1;
        const float ay_jp1 = (float)(Y - (double)j), ay_j = 1.0f - ay_jp1;
        const float vij = ax_i * ay_j, vip1j = ax_ip1 * ay_j, vijp1 = ax_i * ay_jp1;
        const float vip1jp1 = 1.0f - vij - vip1j - vijp1;
        double ux = p->vx[k], uy = p->vy[k], uz = p->vz[k];
        if (!sp->is_ion) {
            const double dx1 = X - (double)i, dx0 = 1.0 - dx1, dy1 = Y - (double)j, dy0 = 1.0 - dy1;
            const double E_X = EX[node(g, i, j)] * dx0 * dy0 + EX[node(g, i + 1, j)] * dx1 * dy0 +
                               EX[node(g, i, j + 1)] * dx0 * dy1 + EX[node(g, i + 1, j + 1)] * dx1 * dy1;
            const double E_Y = EY[node(g, i, j)] * dx0 * dy0 + EY[node(g, i + 1, j)] * dx1 * dy0 +
                               EY[node(g, i, j + 1)] * dx0 * dy1 + EY[node(g, i + 1, j + 1)] * dx1 * dy1;
            const double E_Z = sp->ez;
            const double alfa_x = -0.5 * sp->bx, alfa_y = -0.5 * sp->by, alfa_z = -0.5 * sp->bz;
            const double ax2 = alfa_x * alfa_x, ay2 = alfa_y * alfa_y, az2 = alfa_z * alfa_z;
            const double theta2 = ax2 + ay2 + az2, inv = 1.0 / (1.0 + theta2);
            const double K11 = (1.0 - theta2 + 2.0 * ax2) * inv, K12 = 2.0 * (alfa_x * alfa_y + alfa_z) * inv,
                         K13 = 2.0 * (alfa_x * alfa_z - alfa_y) * inv;
            const double K21 = 2.0 * (alfa_x * alfa_y - alfa_z) * inv, K22 = (1.0 - theta2 + 2.0 * ay2) * inv,
                         K23 = 2.0 * (alfa_y * alfa_z + alfa_x) * inv;
            const double K31 = 2.0 * (alfa_x * alfa_z + alfa_y) * inv, K32 = 2.0 * (alfa_y * alfa_z - alfa_x) * inv,
                         K33 = (1.0 - theta2 + 2.0 * az2) * inv;
            const double VXm = ux - 0.5 * E_X, VYm = uy - 0.5 * E_Y, VZm = uz - 0.5 * E_Z;
            const double nvx = K11 * VXm + K12 * VYm + K13 * VZm - 0.5 * E_X;
            const double nvy = K21 * VXm + K22 * VYm + K23 * VZm - 0.5 * E_Y;
            const double nvz = K31 * VXm + K32 * VYm + K33 * VZm - 0.5 * E_Z;
            ux = 0.5 * (ux + nvx);
            uy = 0.5 * (uy + nvy);
            uz = 0.5 * (uz + nvz);
        }
        const float rvx = (float)ux, rvy = (float)uy, rvz = (float)uz;
        const float rvx2 = rvx * rvx, rvy2 = rvy * rvy, rvz2 = rvz * rvz;
        const float v2 = rvx2 + rvy2 + rvz2;
        const float m[13] = {1.0f, rvx, rvy, rvz, rvx2, rvy2, rvz2, rvx * rvy, rvx * rvz, rvy * rvz,
                             v2 * rvx, v2 * rvy, v2 * rvz};
        const int64_t n00 = node(g, i, j), n10 = node(g, i + 1, j), n01 = node(g, i, j + 1), n11 = node(g, i + 1, j + 1);
        for (int q = 0; q < 13; ++q) {
            double* o = out + q * nn;
            o[n00] += (double)(m[q] * vij);
            o[n10] += (double)(m[q] * vip1j);
            o[n01] += (double)(m[q] * vijp1);
            o[n11] += (double)(m[q] * vip1jp1);
        }
    }
    if (g->periodic) {   // overlap columns, as the density fold
        const int imax = nx - 1;
        for (int q = 0; q < 13; ++q) {
            double* o = out + q * nn;
            for (int j = 0; j <= g->ncy; ++j) {
                o[node(g, 1, j)] += o[node(g, imax, j)];
                o[node(g, imax - 1, j)] += o[node(g, 0, j)];
                o[node(g, 0, j)] = o[node(g, imax - 1, j)];
                o[node(g, imax, j)] = o[node(g, 1, j)];
            }
        }
    }
    for (int64_t nd = 0; nd < nn; ++nd) {
        double* c[13];
        for (int q = 0; q < 13; ++q) c[q] = out + q * nn + nd;
        if (*c[0] > 1.0e-9) {
            const double inv_N = 1.0 / *c[0];
            for (int q = 1; q <= 6; ++q) *c[q] *= inv_N;
            for (int q = 7; q <= 9; ++q) *c[q] = 2.0 * *c[q] * inv_N;
            const double vx = *c[1], vy = *c[2], vz = *c[3], wx = *c[4], wy = *c[5], wz = *c[6];
            double t = vx * vx + vy * vy + vz * vz;
            t = t + t - wx - wy - wz;
            *c[10] = *c[10] * inv_N + (t - wx - wx) * vx - *c[7] * vy - *c[8] * vz;
            *c[11] = *c[11] * inv_N - *c[7] * vx + (t - wy - wy) * vy - *c[9] * vz;
            *c[12] = *c[12] * inv_N - *c[8] * vx - *c[9] * vy + (t - wz - wz) * vz;
        } else {
            for (int q = 0; q < 13; ++q) *c[q] = 0.0;
        }
    }
    double* N = out;
    const int imax = nx - 1, jmax = g->ncy;
    if (g->periodic) {
        for (int i = 0; i <= imax; ++i) {
            N[node(g, i, jmax)] *= 2.0;
            N[node(g, i, 0)] *= 2.0;
        }
        return;
    }
    for (int j = 1; j <= jmax - 1; ++j) {
        N[node(g, 0, j)] *= 2.0;
        N[node(g, imax, j)] *= 2.0;
    }
    for (int i = 1; i <= imax - 1; ++i) {
        N[node(g, i, jmax)] *= 2.0;
        N[node(g, i, 0)] *= 2.0;
    }
    N[node(g, 0, 0)] *= 4.0;
    N[node(g, 0, jmax)] *= 4.0;
    N[node(g, imax, 0)] *= 4.0;
    N[node(g, imax, jmax)] *= 4.0;
}

void oracle_fold_and_wall_scale(const oracle_geom_t* g, double* rho)
{
    const int nx = oracle_nx_nodes(g);
    const int imax = nx - 1, jmax = g->ncy;
    if (g->periodic) {
        for (int j = 0; j <= jmax; ++j) {
            rho[node(g, 1, j)] += rho[node(g, imax, j)];
            rho[node(g, imax - 1, j)] += rho[node(g, 0, j)];
            rho[node(g, 0, j)] = rho[node(g, imax - 1, j)];
            rho[node(g, imax, j)] = rho[node(g, 1, j)];
        }
        for (int i = 0; i <= imax; ++i) {
            rho[node(g, i, jmax)] *= 2.0;
            rho[node(g, i, 0)] *= 2.0;
        }
        return;
    }
    for (int j = 1; j <= jmax - 1; ++j) {
        rho[node(g, 0, j)] *= 2.0;
        rho[node(g, imax, j)] *= 2.0;
    }
    for (int i = 1; i <= imax - 1; ++i) {
        rho[node(g, i, jmax)] *= 2.0;
        rho[node(g, i, 0)] *= 2.0;
    }
    rho[node(g, 0, 0)] *= 4.0;
    rho[node(g, 0, jmax)] *= 4.0;
    rho[node(g, imax, 0)] *= 4.0;
    rho[node(g, imax, jmax)] *= 4.0;
}

// ---------------------------------------------------------------------------------- Maxwell sampler
// PrepareMaxwellDistribIntegral pic2d_ElectronWallCollisions.f90:835-929 (U_max = 3, R_max = 9000,
// R_max_inj = 4500 from pic2d_Modules.f90:949-951)
void oracle_maxwell_tables(double* v, double* v_inj)
{
    const double U_max = 3.0;
    const int R_max = 9000, R_max_inj = 4500;
    std::vector<double> F(180004, 0.0);
    {
        const int N = 180000;
        const double Vmin = -U_max, Vmax = U_max, dV = (Vmax - Vmin) / N;
        F[0] = 0.0;
        for (int i = 1; i <= N + 3; ++i) {
            double u = Vmin + ((double)i - 0.5) * dV;
            F[i] = F[i - 1] + std::exp(-(u * u));
        }
        double t = F[N];
        for (int i = 0; i <= N + 3; ++i) F[i] = F[i] * R_max / t;
        v[0] = Vmin;
        int count = 0;
        for (int i = 1; i <= N + 3; ++i) {
            if ((int)F[i] - count == 1) {
                ++count;
                v[count] = Vmin + i * dV;
                if (count == R_max) break;
            }
        }
    }
    {
        const int N = 90000;
        const double Vmin = 0.0, Vmax = U_max, dV = (Vmax - Vmin) / N;
        std::fill(F.begin(), F.end(), 0.0);
        for (int i = 1; i <= N + 3; ++i) {
            double t = Vmin + ((double)(float)i - 0.5) * dV;
            F[i] = F[i - 1] + std::exp(-(t * t)) * t;
        }
        double t = F[N];
        for (int i = 1; i <= N + 3; ++i) F[i] = F[i] * R_max_inj / t;
        v_inj[0] = Vmin;
        int count = 0;
        for (int i = 1; i <= N + 3; ++i) {
            if ((int)F[i] - count == 1) {
                ++count;
                v_inj[count] = Vmin + i * dV;
                if (count == R_max_inj) break;
            }
        }
    }
}

// GetMaxwellVelocity :961-985
double oracle_maxwell_sample(const double* v, double u)
{
    const int R_max = 9000;
    double R = R_max * u;
    int indx = (int)R;
    if (indx < R_max) return v[indx] + (R - indx) * (v[indx + 1] - v[indx]);
    return v[R_max];
}

// CALCULATE_ELECTRON_VDF pic2d_VelocityDistributions.f90:3-206 (and CALCULATE_ION_VDF :211-393, which differs only in
// fvc and the per-species layout), the loop over particles of one cluster
int64_t oracle_vdf(const oracle_parts_t* p, int32_t nbx, int32_t nby, double xmax, double ymax, double fvc,
                   int32_t vmin, int32_t* h1, int32_t* h2)
{
    const int32_t vmax = -vmin - 1, reclen = -2 * vmin, nbox = nbx * nby;
    std::fill(h1, h1 + 3 * (int64_t)nbox * reclen, 0);
    if (h2) std::fill(h2, h2 + (int64_t)nbox * reclen * reclen, 0);
    std::vector<double> xsplit(nbx), ysplit(nby);
    for (int i = 1; i < nbx; ++i) xsplit[i] = 0.0 + (double)i * (xmax - 0.0) / nbx;
    for (int j = 1; j < nby; ++j) ysplit[j] = 0.0 + (double)j * (ymax - 0.0) / nby;
    // INT(v * fvc), one less for negative v; values beyond the integer range count as out of range
    auto bin = [&](double v, bool* ok) {
        double t = v * fvc;
        if (!(std::fabs(t) < 1073741824.0)) { *ok = false; return 0; }
        int b = (int)t;
        if (v < 0.0) b -= 1;
        *ok = b >= vmin && b <= vmax;
        return b;
    };
    int64_t skip = 0;
    for (int64_t k = 0; k < p->n; ++k) {
        int ibox = nbx;
        for (int i = 1; i <= nbx - 1; ++i)
            if (p->x[k] < xsplit[i]) { ibox = i; break; }
        int jbox = nby;
        for (int j = 1; j <= nby - 1; ++j)
            if (p->y[k] < ysplit[j]) { jbox = j; break; }
        const int n = (ibox - 1) + (jbox - 1) * nbx;
        bool ok;
        int bx = bin(p->vx[k], &ok);
        if (!ok) { ++skip; continue; }
        int by = bin(p->vy[k], &ok);
        if (!ok) { ++skip; continue; }
        int bz = bin(p->vz[k], &ok);
        if (!ok) { ++skip; continue; }
        const int64_t pos1 = (int64_t)n * reclen - vmin;
        h1[pos1 + bx]++;
        h1[(int64_t)nbox * reclen + pos1 + by]++;
        h1[2 * (int64_t)nbox * reclen + pos1 + bz]++;
        if (h2) h2[((int64_t)n * reclen + (by - vmin)) * reclen + (bx - vmin)]++;
    }
    return skip;
}

// GetInjMaxwellVelocity pic2d_ElectronWallCollisions.f90:933-957
static double maxwell_inj_sample(const double* v, double u)
{
    const int R_max_inj = 4500;
    double R = R_max_inj * u;
    int indx = (int)R;
    if (indx < R_max_inj) return v[indx] + (R - indx) * (v[indx + 1] - v[indx]);
    return v[R_max_inj];
}

// PROCESS_ION_INDUCED_ELECTRON_EMISSION pic2d_IonEmissions.f90:1-89 (Coeff_ii_EE_True :350-372 is the constant
// yield inside (minE, maxE); the angle of incidence is computed there but not used) and
// INJECT_ION_IMPACT_EXTRACTED_ELECTRON :91-348 for the domain walls (m > 0): position 1e-6 inside the wall,
// normal component from the injection distribution, tangential ones Maxwellian, all times the conversion factor,
// scaled down to the ion's remaining energy when above it.
// INJECT_ION_IMPACT_EXTRACTED_ELECTRON's placement by the struck surface: dirflag 1 (normal +x), 2 (-y), 3 (-x),
// 4 (+y) at coordinate `at` (the domain wall's, or the inner object's side: xmax + 1e-6, ymin - 1e-6, xmin - 1e-6,
// ymax + 1e-6 for m = -1, pic2d_IonEmissions.f90:232-330)
int32_t oracle_ion_emission_face(const oracle_emit_t* em, int32_t obj, int32_t dirflag, double at, double x, double y,
                                 double vx, double vy, double vz, uint32_t id, uint64_t seed, uint32_t step,
                                 double* out, int32_t cap)
{
    if (!em->on[obj]) return 0;
    const int wall = obj;
    double energy_inc = em->ms * (vx * vx + vy * vy + vz * vz);
    if (energy_inc <= em->emin[wall]) return 0;
    if (energy_inc >= em->emax[wall]) return 0;
    double coef_total = em->yield[wall];
    if (coef_total == 0.0) return 0;
    energy_inc = std::max(0.0, energy_inc - em->emin[wall]);
    const uint32_t stream = 0x45450000u + em->species;
    int32_t n = 0;
    uint32_t block = 1;
    auto inject = [&]() {
        if (energy_inc <= 0.0) return;
        uint32_t w[4];
        philox_block(id, seed, step, stream, block++, w);
        double un = maxwell_inj_sample(em->maxwell_inj, uniform(w[0]));
        double t1 = oracle_maxwell_sample(em->maxwell_v, uniform(w[1]));
        double t2 = oracle_maxwell_sample(em->maxwell_v, uniform(w[2]));
        double xn, yn, v[3];
        if (dirflag == 1) {
            xn = at + 1.0e-6; yn = y; v[0] = un; v[1] = t1; v[2] = t2;
        } else if (dirflag == 3) {
            xn = at - 1.0e-6; yn = y; v[0] = -un; v[1] = t1; v[2] = t2;
        } else if (dirflag == 4) {
            xn = x; yn = at + 1.0e-6; v[0] = t1; v[1] = un; v[2] = t2;
        } else {
            xn = x; yn = at - 1.0e-6; v[0] = t1; v[1] = -un; v[2] = t2;
        }
        const double f = em->fconv[wall];
        for (double& c : v) c *= f;
        double energy_new = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (energy_new > energy_inc) {
            double alpha = std::sqrt(energy_inc / energy_new);
            for (double& c : v) c *= alpha;
            energy_inc = 0.0;
        } else {
            energy_inc -= energy_new;
        }
        if (n < cap) {
            double* r = out + 5 * n;
            r[0] = xn; r[1] = yn; r[2] = v[0]; r[3] = v[1]; r[4] = v[2];
        }
        ++n;
    };
    while (coef_total >= 1.0) {
        inject();
        coef_total -= 1.0;
    }
    if (coef_total == 0.0) return n;
    uint32_t w0[4];
    philox_block(id, seed, step, stream, 0u, w0);
    if (uniform(w0[0]) < coef_total) inject();
    return n;
}

int32_t oracle_ion_emission(const oracle_emit_t* em, int32_t wall, double x, double y, double vx, double vy,
                            double vz, uint32_t id, uint64_t seed, uint32_t step, double xmax, double ymax,
                            double* out, int32_t cap)
{
    if (!em->on[wall]) return 0;
    x = std::min(std::max(x, 0.0), xmax);
    y = std::min(std::max(y, 0.0), ymax);
    // domain walls: left dirflag 1 at 0, right 3 at xmax, below 4 at 0, above 2 at ymax
    const int32_t dirflag = wall == 2 ? 1 : wall == 3 ? 3 : wall == 0 ? 4 : 2;
    const double at = wall == 3 ? xmax : wall == 1 ? ymax : 0.0;
    return oracle_ion_emission_face(em, wall, dirflag, at, x, y, vx, vy, vz, id, seed, step, out, cap);
}

// Coeff_SEE_Classic pic2d_SEEmission.f90:1171-1208 (k is a REAL variable: 0.62 in single precision)
static double see_classic(const oracle_see_t* w, double energy, double theta)
{
    if (!(energy > w->cl_e0)) return 0.0;
    double energy_max_theta = w->cl_emax * (1.0 + 0.318309886 * w->cl_k * theta * theta);
    double v = (energy - w->cl_e0) / (energy_max_theta - w->cl_e0);
    double coeff_max_theta = w->cl_max * (1.0 + 0.159154943 * w->cl_k * theta * theta);
    float k = v < 1.0 ? 0.62f : 0.25f;
    return coeff_max_theta * std::pow(v * std::exp(1.0 - v), (double)k);
}

// Coeff_SEE_Elastic :1054-1099, Coeff_SEE_Inelastic :1103-1134, Coeff_SEE_True :1139-1167
static double see_elastic(const oracle_see_t* w, double e, double th)
{
    switch (w->m_el) {
    case 1: return (e > w->el_emin && e <= w->el_emax) ? w->el_yield : 0.0;
    case 2:
        if (e >= w->el_emaxc)
            return w->el_max * std::exp(-(e - w->el_emaxc) / w->el_de) * (e - w->el_emaxc + w->el_de) / w->el_de +
                   w->el_frac * see_classic(w, e, th);
        if (e > w->el_e0)
            return w->el_max * std::exp(-(e - w->el_emaxc) / (w->el_emaxc - w->el_e0)) * (e - w->el_e0) /
                       (w->el_emaxc - w->el_e0) +
                   w->el_frac * see_classic(w, e, th);
        return 0.0;
    default: return 0.0;
    }
}
static double see_inelastic(const oracle_see_t* w, double e, double th)
{
    if (w->m_in == 1) return (e > w->in_emin && e <= w->in_emax) ? w->in_yield : 0.0;
    if (w->m_in == 2) return w->in_frac * see_classic(w, e, th);
    return 0.0;
}
static double see_true(const oracle_see_t* w, double e, double th)
{
    if (w->m_tr == 1) return (e > w->tr_emin && e <= w->tr_emax) ? w->tr_yield : 0.0;
    if (w->m_tr != 2) return 0.0;
    double c = see_classic(w, e, th) * (1.0 - w->el_frac - w->in_frac);
    return c < 0.0 ? 0.0 : c;
}

// the electron leaves the surface given by dirflag (1 normal +x, 2 -y, 3 -x, 4 +y) at coordinate `at`, 1e-6 outside
// it: a domain wall (m > 0) or an inner object's side (m = -1, pic2d_SEEmission.f90:388-544)
int32_t oracle_see_face(const oracle_see_t* w, int32_t dirflag, double at, double x, double y, double vx, double vy,
                        double vz, uint32_t id, uint64_t seed, uint32_t step, double* out, int32_t cap)
{
    const uint32_t stream = 0x53450000u;
    const bool xnormal = dirflag == 1 || dirflag == 3;
    double energy_inc = vx * vx + vy * vy + vz * vz;
    if (energy_inc <= w->lowest) return 0;
    double v = std::sqrt(energy_inc), theta_inc = 0.0;
    if (v != 0.0) theta_inc = std::acos(std::min(1.0, std::fabs(xnormal ? vx : vy) / v));
    double ce = see_elastic(w, energy_inc, theta_inc), ci = see_inelastic(w, energy_inc, theta_inc);
    if (ce + ci > 1.0) return -1;
    double ct = see_true(w, energy_inc, theta_inc), ctot = ce + ci + ct;
    if (ctot == 0.0) return 0;
    uint32_t b0[4];
    philox_block(id, seed, step, stream, 0u, b0);
    double R = uniform(b0[0]);
    int32_t n = 0;
    auto put = [&](double nx, double ny, double a, double b, double c) {
        if (n < cap) {
            double* r = out + 5 * n;
            r[0] = nx; r[1] = ny; r[2] = a; r[3] = b; r[4] = c;
        }
        ++n;
    };
    // the position and the direction of a scattered electron leaving the wall (the domain-wall branches)
    auto scatter = [&](double speed, double theta, double fi) {
        double c = speed * std::cos(theta), s1 = speed * std::sin(theta) * std::sin(fi),
               s2 = speed * std::sin(theta) * std::cos(fi);
        if (dirflag == 1) put(at + 1.0e-6, y, c, s1, s2);
        else if (dirflag == 2) put(x, at - 1.0e-6, s1, -c, s2);
        else if (dirflag == 3) put(at - 1.0e-6, y, -c, s1, s2);
        else put(x, at + 1.0e-6, s1, c, s2);
    };
    if (R <= ce) {   // INJECT_ELASTIC_REFLECTED_ELECTRON :155-557
        if (!w->refl_random) {
            if (dirflag == 1) put(at + 1.0e-6, y, -vx, vy, vz);
            else if (dirflag == 2) put(x, at - 1.0e-6, vx, -vy, vz);
            else if (dirflag == 3) put(at - 1.0e-6, y, -vx, vy, vz);
            else put(x, at + 1.0e-6, vx, -vy, vz);
        } else {
            scatter(v, std::asin(std::min(uniform(b0[1]), 1.0)), 6.283185307179 * uniform(b0[2]));
        }
        return n;
    }
    if (R > ce && R <= ce + ci) {   // INJECT_INELASTIC_BACKSCATTERED_ELECTRON :561-790
        double th = std::asin(std::min(uniform(b0[1]), 1.0)), fi = 6.283185307179 * uniform(b0[2]);
        scatter(v * std::sqrt(uniform(b0[3])), th, fi);
        return n;
    }
    if (ct <= 0.0) return 0;
    if (w->m_tr == 1) energy_inc = std::max(0.0, energy_inc - w->tr_emin);
    else if (w->m_tr == 2) energy_inc = std::max(0.0, energy_inc - w->cl_e0);
    uint32_t block = 1;
    auto inject = [&]() {   // INJECT_TRUE_SECONDARY_ELECTRON :794-1050
        if (energy_inc <= 0.0) return;
        uint32_t wb[4];
        philox_block(id, seed, step, stream, block++, wb);
        double un = maxwell_inj_sample(w->maxwell_inj, uniform(wb[0]));
        double t1 = oracle_maxwell_sample(w->maxwell_v, uniform(wb[1]));
        double t2 = oracle_maxwell_sample(w->maxwell_v, uniform(wb[2]));
        double xn, yn, nv[3];
        if (dirflag == 1) { xn = at + 1.0e-6; yn = y; nv[0] = un; nv[1] = t1; nv[2] = t2; }
        else if (dirflag == 2) { xn = x; yn = at - 1.0e-6; nv[0] = t1; nv[1] = -un; nv[2] = t2; }
        else if (dirflag == 3) { xn = at - 1.0e-6; yn = y; nv[0] = -un; nv[1] = t1; nv[2] = t2; }
        else { xn = x; yn = at + 1.0e-6; nv[0] = t1; nv[1] = un; nv[2] = t2; }
        for (double& c : nv) c *= w->fconv;
        double energy_new = nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2];
        if (energy_new > energy_inc) {
            double alpha = std::sqrt(energy_inc / energy_new);
            for (double& c : nv) c *= alpha;
            energy_inc = 0.0;
        } else {
            energy_inc -= energy_new;
        }
        put(xn, yn, nv[0], nv[1], nv[2]);
    };
    if (ctot <= 1.0) {
        if (R > ce + ci && R <= ctot) inject();
        return n;
    }
    ct = ct / (1.0 - (ce + ci));
    while (ct >= 1.0) {
        inject();
        ct -= 1.0;
    }
    if (uniform(b0[3]) < ct) inject();
    return n;
}

int32_t oracle_see(const oracle_see_t* w, int32_t wall, double x, double y, double vx, double vy, double vz,
                   uint32_t id, uint64_t seed, uint32_t step, double xmax, double ymax, double* out, int32_t cap)
{
    x = std::min(std::max(x, 0.0), xmax);
    y = std::min(std::max(y, 0.0), ymax);
    const int32_t dirflag = wall == 2 ? 1 : wall == 3 ? 3 : wall == 0 ? 4 : 2;
    const double at = wall == 3 ? xmax : wall == 1 ? ymax : 0.0;
    return oracle_see_face(w, dirflag, at, x, y, vx, vy, vz, id, seed, step, out, cap);
}

// PERFORM_ELECTRON_EMISSION_SETUP pic2d_Setup.f90:618-1001: one local part per wall covering the whole wall
// (corners of a single cluster), so the count is N_electron_constant_emit and the place spans the wall
int32_t oracle_wall_injection(double n, int32_t model, double fn, double fp, double vb, int32_t wall, uint32_t step,
                              uint64_t seed, double xmax, double ymax, const double* maxwell_v,
                              const double* maxwell_inj, double* out, int32_t cap)
{
    const uint32_t key = 0xE1000000u + (uint32_t)wall, stream = 0x43450000u;
    if (n <= 0.0) return 0;
    int32_t count = (int32_t)n;
    uint32_t w0[4];
    philox_block(key, seed, step, stream, 0u, w0);
    if (uniform(w0[0]) < n - (double)count) ++count;
    for (int32_t e = 0; e < count && e < cap; ++e) {
        uint32_t w[4];
        philox_block(key, seed, step, stream, 1u + (uint32_t)e, w);
        double vn = model == 0 ? maxwell_inj_sample(maxwell_inj, uniform(w[1])) * fn
                               : std::max(0.0, vb + oracle_maxwell_sample(maxwell_v, uniform(w[1])) * fn);
        double t1 = oracle_maxwell_sample(maxwell_v, uniform(w[2])) * fp;
        double t2 = oracle_maxwell_sample(maxwell_v, uniform(w[3])) * fp;
        double r = uniform(w[0]);
        double* o = out + 5 * e;
        if (wall == 0) { o[0] = std::min(std::max(r * xmax, 0.0), xmax); o[1] = 1.0e-6; o[2] = t1; o[3] = vn; }
        else if (wall == 1) { o[0] = std::min(std::max(r * xmax, 0.0), xmax); o[1] = ymax - 1.0e-6; o[2] = t1; o[3] = -vn; }
        else if (wall == 2) { o[0] = 1.0e-6; o[1] = std::min(std::max(r * ymax, 0.0), ymax); o[2] = vn; o[3] = t1; }
        else { o[0] = xmax - 1.0e-6; o[1] = std::min(std::max(r * ymax, 0.0), ymax); o[2] = -vn; o[3] = t1; }
        o[4] = t2;
    }
    return count;
}

// Covered cells of segment m of inner object n (pic2d_CurProblemValues.f90:603-683): the walls of the domain are the
// boundary objects (horizontal segments j = 0 and j = ncy over all i; on a walled domain also the vertical segments
// i = 0 and i = ncx over j in [0, ncy)), the other inner objects come second. Index: cell - segment start.
static std::vector<bool> inner_segment_covered(const oracle_geom_t* g, int n, int m)
{
    const int il = g->ileft[n], ir = g->iright[n], jb = g->jbottom[n], jt = g->jtop[n];
    std::vector<bool> cov;
    if (m == 1 || m == 3) {
        const int istart = m == 1 ? il : ir;
        for (int j = jb; j < jt; ++j) {
            bool c = false;
            // boundary objects: vertical wall segments with the same i
            if (!g->periodic && (istart == 0 || istart == g->ncx) && j >= 0 && j < g->ncy) c = true;
            for (int o = 0; o < g->n_inner && !c; ++o) {
                if (o == n) continue;
                if (istart < g->ileft[o] || istart > g->iright[o]) continue;
                if (j >= g->jbottom[o] && j < g->jtop[o]) c = true;
            }
            cov.push_back(c);
        }
    } else {
        const int jstart = m == 2 ? jt : jb;
        for (int i = il; i < ir; ++i) {
            bool c = jstart == 0 || jstart == g->ncy;
            for (int o = 0; o < g->n_inner && !c; ++o) {
                if (o == n) continue;
                if (jstart < g->jbottom[o] || jstart > g->jtop[o]) continue;
                if (i >= g->ileft[o] && i < g->iright[o]) c = true;
            }
            cov.push_back(c);
        }
    }
    return cov;
}

int32_t oracle_inner_injection(const oracle_geom_t* g, int32_t n, double n_emit, int32_t model, double fn, double fp,
                               double vb, uint32_t step, uint64_t seed, const double* maxwell_v,
                               const double* maxwell_inj, double* out, int32_t cap, int32_t* per_side)
{
    const uint32_t stream = 0x43450000u;
    std::vector<bool> cov[5];
    int32_t L = 0;
    for (int m = 1; m <= 4; ++m) {
        cov[m] = inner_segment_covered(g, n, m);
        for (bool c : cov[m]) L += c ? 0 : 1;
    }
    // c_indx_x/y_min and _max of the one cluster: 0 and the last node's index
    const int cxmin = 0, cxmax = g->periodic ? g->ncx + 1 : g->ncx, cymin = 0, cymax = g->ncy;
    int32_t total = 0;
    for (int m = 1; m <= 4; ++m) {
        per_side[m - 1] = 0;
        const bool vert = m == 1 || m == 3;
        const int at = m == 1 ? g->ileft[n] : m == 3 ? g->iright[n] : m == 2 ? g->jtop[n] : g->jbottom[n];
        const int a0 = vert ? g->jbottom[n] : g->ileft[n], a1 = vert ? g->jtop[n] : g->iright[n];
        if (n_emit <= 0.0 || L == 0) continue;
        if (vert) {
            if (!(at > cxmin && at < cxmax)) continue;
            if (!(a0 < cymax && a1 > cymin)) continue;
        } else {
            if (!(at > cymin && at < cymax)) continue;
            if (!(a0 < cxmax && a1 > cxmin)) continue;
        }
        const int cmin = std::max(a0, vert ? cymin : cxmin), cmax = std::min(a1, (vert ? cymax : cxmax) - 1);
        int count_open = 0;
        for (int q = cmin; q < cmax; ++q)
            if (!cov[m][q - a0]) ++count_open;
        // REAL arithmetic: N_electron_constant_emit * REAL(count_open) / REAL(L)
        const double add = (double)((float)n_emit * (float)count_open / (float)L);
        if (count_open == 0) continue;
        const uint32_t key = 0xE1000000u + 4u + 4u * (uint32_t)n + (uint32_t)(m - 1);
        int32_t count = (int32_t)add;
        uint32_t w0[4];
        philox_block(key, seed, step, stream, 0u, w0);
        if (uniform(w0[0]) < add - (double)count) ++count;
        for (int32_t e = 0; e < count; ++e) {
            uint32_t w[4];
            philox_block(key, seed, step, stream, 1u + (uint32_t)e, w);
            // the walk over the open cells, one subtraction of 1 per open cell (:1064-1078)
            double d = uniform(w[0]) * ((double)count_open - 1.0e-6);
            double t = 0.0;
            for (int q = cmin; q < cmax; ++q) {
                if (cov[m][q - a0]) continue;
                if (d < 1.0) {
                    t = std::max((double)q, std::min((double)q + d, (double)(q + 1)));
                    break;
                }
                d -= 1.0;
            }
            t = std::min(std::max(t, (double)cmin), (double)cmax - 1.0e-6);
            double vn = model == 0 ? maxwell_inj_sample(maxwell_inj, uniform(w[1])) * fn
                                   : std::max(0.0, vb + oracle_maxwell_sample(maxwell_v, uniform(w[1])) * fn);
            double t1 = oracle_maxwell_sample(maxwell_v, uniform(w[2])) * fp;
            double t2 = oracle_maxwell_sample(maxwell_v, uniform(w[3])) * fp;
            if (total < cap) {
                double* o = out + 5 * total;
                if (m == 1) { o[0] = (double)at - 1.0e-6; o[1] = t; o[2] = -vn; o[3] = t1; }
                else if (m == 3) { o[0] = (double)at + 1.0e-6; o[1] = t; o[2] = vn; o[3] = t1; }
                else if (m == 2) { o[0] = t; o[1] = (double)at + 1.0e-6; o[2] = t1; o[3] = vn; }
                else { o[0] = t; o[1] = (double)at - 1.0e-6; o[2] = t1; o[3] = -vn; }
                o[4] = t2;
            }
            ++total;
        }
        per_side[m - 1] = count;
    }
    return total;
}

// CHECK_INTERSECTION_WITH_VERTICAL_SEGMENT / _HORIZONTAL_SEGMENT pic2d_ElectronWallCollisions.f90:746-812
static bool cross_vertical(double xorg, double yorg, double x, double y, double xseg, double ymin, double ymax,
                           double* ycross)
{
    if (std::max(xorg, x) < xseg || std::min(xorg, x) > xseg) return false;
    if (std::max(yorg, y) < ymin || std::min(yorg, y) > ymax) return false;
    if (xorg == x) return false;
    double yc = yorg + (y - yorg) * (xseg - xorg) / (x - xorg);
    if (!std::isfinite(yc) || yc < ymin || yc > ymax || yc < std::min(y, yorg) || yc > std::max(y, yorg)) return false;
    *ycross = yc;
    return true;
}
static bool cross_horizontal(double xorg, double yorg, double x, double y, double yseg, double xmin, double xmax,
                             double* xcross)
{
    if (std::max(yorg, y) < yseg || std::min(yorg, y) > yseg) return false;
    if (std::max(xorg, x) < xmin || std::min(xorg, x) > xmax) return false;
    if (yorg == y) return false;
    double xc = xorg + (x - xorg) * (yseg - yorg) / (y - yorg);
    if (!std::isfinite(xc) || xc < xmin || xc > xmax || xc < std::min(x, xorg) || xc > std::max(x, xorg)) return false;
    *xcross = xc;
    return true;
}

int32_t oracle_inner_cross(const oracle_geom_t* g, double x, double y, double vx, double vy, double xmul,
                           int32_t* m_out, double* xc_out, double* yc_out)
{
    const double xorg = x - vx * xmul, yorg = y - vy * xmul;
    int n_do = -1, mcross = -1;
    double xcross = 0.0, ycross = 0.0, distorg = 0.0;
    for (int n = 0; n < g->n_inner; ++n)
        for (int m = 1; m <= 4; ++m) {   // FIND_CLOSEST_INTERSECTION_WITH_OBJECT :649-742, segments as :277-300
            double xc = 0.0, yc = 0.0;
            bool ok;
            if (m == 1 || m == 3) {
                xc = m == 1 ? g->ileft[n] : g->iright[n];
                ok = cross_vertical(xorg, yorg, x, y, xc, g->jbottom[n], g->jtop[n], &yc);
            } else {
                yc = m == 2 ? g->jtop[n] : g->jbottom[n];
                ok = cross_horizontal(xorg, yorg, x, y, yc, g->ileft[n], g->iright[n], &xc);
            }
            if (!ok) continue;
            double d = (xc - xorg) * (xc - xorg) + (yc - yorg) * (yc - yorg);
            if (mcross != -1 && d >= distorg) continue;
            n_do = n;
            mcross = m;
            xcross = xc;
            ycross = yc;
            distorg = d;
        }
    *m_out = mcross;
    *xc_out = xcross;
    *yc_out = ycross;
    return n_do;
}

void oracle_inner_charge(const oracle_geom_t* g, int32_t n_do, int32_t mcross, double xcross, double ycross, double q,
                         double* surf)
{
    // the outline numbering of DO_ELECTRON_COLL_WITH_INNER_OBJECT :582-640: position 1 = (ileft, jbottom), up the
    // left side, along the top, down the right side, back along the bottom
    const int il = g->ileft[n_do], ir = g->iright[n_do], jb = g->jbottom[n_do], jt = g->jtop[n_do];
    const int i_left_top = jt - jb + 1, i_right_top = i_left_top + ir - il, i_right_bottom = i_right_top + jt - jb;
    const int i_left_bottom_bis = i_right_bottom + ir - il - 1;
    auto pos_node = [&](int pos) -> int64_t {
        if (pos <= i_left_top) return node(g, il, jb + pos - 1);
        if (pos <= i_right_top) return node(g, il + pos - i_left_top, jt);
        if (pos <= i_right_bottom) return node(g, ir, jt - (pos - i_right_top));
        return node(g, ir - (pos - i_right_bottom), jb);
    };
    int i = 0, ip1 = 0;
    double dqi = 0.0, dqip1 = 0.0;
    switch (mcross) {
    case 1:   // coll_direction_flag 3
        i = std::min((int)(ycross - jb) + 1, i_left_top - 1);
        dqip1 = ycross - (int)ycross;
        dqi = 1.0 - dqip1;
        ip1 = i + 1;
        break;
    case 2:   // flag 4
        i = std::min((int)(xcross - il) + i_left_top, i_right_top - 1);
        dqip1 = xcross - (int)xcross;
        dqi = 1.0 - dqip1;
        ip1 = i + 1;
        break;
    case 3:   // flag 1
        i = std::min((int)(jt - ycross) + i_right_top, i_right_bottom - 1);
        dqi = ycross - (int)ycross;
        dqip1 = 1.0 - dqi;
        ip1 = i + 1;
        break;
    default:  // flag 2
        i = std::min((int)(ir - xcross) + i_right_bottom, i_left_bottom_bis);
        dqi = xcross - (int)xcross;
        dqip1 = 1.0 - dqi;
        ip1 = (i == i_left_bottom_bis) ? 1 : i + 1;
        break;
    }
    surf[pos_node(i)] += q * dqi;
    surf[pos_node(ip1)] += q * dqip1;
}

int32_t oracle_inner_hit(const oracle_geom_t* g, const double* inner_eps, double x, double y, double vx, double vy,
                         double xmul, double q, double* surf)
{
    int32_t m = -1;
    double xc = 0.0, yc = 0.0;
    const int32_t n = oracle_inner_cross(g, x, y, vx, vy, xmul, &m, &xc, &yc);
    if (n >= 0 && inner_eps[n] > 0.0) oracle_inner_charge(g, n, m, xc, yc, q, surf);
    return n;
}

// INJECT_REFLECTED_ION pic2d_IonEmissions.f90:374-430 (m > 0, the domain walls)
void oracle_ion_reflect(int32_t wall, double x, double y, double vx, double vy, double vz, double xmax, double ymax,
                        double* out)
{
    x = std::min(std::max(x, 0.0), xmax);
    y = std::min(std::max(y, 0.0), ymax);
    out[0] = x; out[1] = y; out[2] = vx; out[3] = vy; out[4] = vz;
    if (wall == 2) { out[0] = 1.0e-6; out[2] = -vx; }
    else if (wall == 3) { out[0] = xmax - 1.0e-6; out[2] = -vx; }
    else if (wall == 0) { out[1] = 1.0e-6; out[3] = -vy; }
    else { out[1] = ymax - 1.0e-6; out[3] = -vy; }
}

// --------------------------------------------------------------------------- e-n collision table
// frequency_of_en_collision pic2d_enCollisionsSpecificProc.f90:4-57
double oracle_en_frequency(const oracle_crsect_t* cs, double energy_eV, double n_m3, int32_t nsub, double dt_s)
{
    const int N = cs->n_points;
    const double* e = cs->energy_eV;
    const double* s = cs->crsect_m2;
    double f;
    if (energy_eV >= e[N - 1]) {
        f = s[N - 1] * std::sqrt(2.0 * energy_eV * E_CL / M_E_KG);
    } else if (energy_eV < e[0]) {
        f = (cs->type < 20) ? s[0] * std::sqrt(2.0 * energy_eV * E_CL / M_E_KG) : 0.0;
    } else {
        int j;  // 1-based in the reference, 0-based here
        for (j = 0; j < N - 1; ++j)
            if (energy_eV >= e[j] && energy_eV < e[j + 1]) break;
        j = std::min(j, N - 2);
        double ej = e[j], ejp1 = e[j + 1];
        double fj = s[j] * std::sqrt(2.0 * ej * E_CL / M_E_KG);
        double fjp1 = s[j + 1] * std::sqrt(2.0 * ejp1 * E_CL / M_E_KG);
        f = fj + (fjp1 - fj) * (energy_eV - ej) / (ejp1 - ej);
    }
    return f * n_m3 * nsub * dt_s;
}

// energy grid of INITIATE_ELECTRON_NEUTRAL_COLLISIONS pic2d_enCollisionsGeneralProc.f90:236-279
int32_t oracle_mcc_n_values(int32_t n_seg, const double* seg_value, const double* seg_step)
{
    int32_t n = 0;
    for (int i = 1; i <= n_seg; ++i) n += (int32_t)((seg_value[i] - seg_value[i - 1]) / seg_step[i - 1] + 0.001);
    return n;
}

// probability table :281-322
void oracle_mcc_build(oracle_mcc_table_t* t, int32_t n_act, const oracle_crsect_t* cs, double n_m3, int32_t nsub,
                      double dt_s)
{
    t->n_act = n_act;
    t->n_values = oracle_mcc_n_values(t->n_seg, t->seg_value, t->seg_step);
    t->seg_index[0] = 0;
    for (int i = 1; i <= t->n_seg; ++i)
        t->seg_index[i] =
            t->seg_index[i - 1] + (int32_t)((t->seg_value[i] - t->seg_value[i - 1]) / t->seg_step[i - 1] + 0.001);
    t->energy_eV[0] = t->seg_value[0];
    for (int i = 1; i <= t->n_seg; ++i) {
        for (int j = t->seg_index[i - 1] + 1; j <= t->seg_index[i] - 1; ++j)
            t->energy_eV[j] = t->seg_value[i - 1] + (j - t->seg_index[i - 1]) * t->seg_step[i - 1];
        t->energy_eV[t->seg_index[i]] = t->seg_value[i];
    }
    const int NV = t->n_values;
    double* P = t->prob;
    for (int ie = 0; ie <= NV; ++ie) {
        double en = t->energy_eV[ie];
        P[(int64_t)ie * n_act + 0] = oracle_en_frequency(&cs[0], en, n_m3, nsub, dt_s);
        for (int p = 1; p < n_act; ++p)
            P[(int64_t)ie * n_act + p] = P[(int64_t)ie * n_act + p - 1] + oracle_en_frequency(&cs[p], en, n_m3, nsub, dt_s);
    }
    int imax = 0;
    for (int ie = 1; ie <= NV; ++ie)
        if (P[(int64_t)ie * n_act + n_act - 1] > P[(int64_t)imax * n_act + n_act - 1]) imax = ie;
    double pmax = P[(int64_t)imax * n_act + n_act - 1];
    t->max_colliding_fraction = 1.0 - std::exp(-pmax);
    for (int ie = 0; ie <= NV; ++ie)
        for (int p = 0; p < n_act; ++p) {
            double v = P[(int64_t)ie * n_act + p] / pmax;
            P[(int64_t)ie * n_act + p] = std::max(0.0, std::min(1.0, v));
        }
    P[(int64_t)imax * n_act + n_act - 1] = 1.0;
    for (int ie = 0; ie <= NV; ++ie)
        for (int p = 0; p < n_act - 1; ++p)
            P[(int64_t)ie * n_act + p + 1] = std::max(P[(int64_t)ie * n_act + p], P[(int64_t)ie * n_act + p + 1]);
    for (int p = 0; p < n_act; ++p) {
        t->type[p] = cs[p].type;
        t->threshold_eV[p] = (cs[p].type >= 20) ? cs[p].energy_eV[0] : 0.0;
    }
}

// kind selection of PERFORM_ELECTRON_NEUTRAL_COLLISIONS :451-485. The weighted threshold is formed with
// explicit fused multiply-adds (fma(a1, P1, a0*P0)) so that the GPU kernels can reproduce it bit for bit.
int32_t oracle_mcc_choose(const oracle_mcc_table_t* t, double energy_eV, double r)
{
    const int na = t->n_act;
    int indx;
    double a0, a1;
    if (energy_eV >= t->seg_value[t->n_seg]) {
        indx = t->n_values - 1;
        a1 = 1.0;
        a0 = 0.0;
    } else if (energy_eV < t->seg_value[0]) {
        indx = 0;
        a1 = 0.0;
        a0 = 1.0;
    } else {
        int seg = 1;
        for (int i = t->n_seg - 1; i >= 0; --i)
            if (energy_eV >= t->seg_value[i]) {
                seg = i + 1;
                break;
            }
        double step = t->seg_step[seg - 1];
        double fi = (double)t->seg_index[seg - 1] + (energy_eV - t->seg_value[seg - 1]) / step;
        indx = (int)fi;
        indx = std::max(0, std::min(indx, t->n_values - 1));
        a1 = (energy_eV - t->energy_eV[indx]) / step;
        a0 = 1.0 - a1;
    }
    int k;
    for (k = na; k >= 1; --k) {
        double thr = std::fma(a1, t->prob[(int64_t)(indx + 1) * na + k - 1], a0 * t->prob[(int64_t)indx * na + k - 1]);
        if (r > thr) break;
    }
    return k + 1;
}

// velocity rotation common to en_Collision_* (e.g. pic2d_enCollisionsSpecificProc.f90:117-144)
static void rotate(double cosk, double sink, double cosf, double sinf, const double* v, double* out)
{
    double Vx = v[0], Vy = v[1], Vz = v[2];
    double V = std::sqrt(Vx * Vx + Vy * Vy + Vz * Vz);
    double Vxy = std::sqrt(Vx * Vx + Vy * Vy);
    if (Vxy > 1.0e-20) {
        double a = Vx / Vxy, b = Vy / Vxy;
        out[0] = Vx * cosk + (sinf * V * b + cosf * Vz * a) * sink;
        out[1] = Vy * cosk - (sinf * V * a - cosf * Vz * b) * sink;
        out[2] = Vz * cosk - Vxy * cosf * sink;
    } else {
        out[0] = std::fabs(Vz) * sink * cosf;
        out[1] = std::fabs(Vz) * sink * sinf;
        out[2] = Vz * cosk;
    }
}

static double clampc(double c) { return std::max(std::min(0.999999999999, c), -0.999999999999); }
static double okhrimovskyy(double e, double R) { return 1.0 - 2.0 * R / (1.0 + 8.0 * (e / 27.21) * (1.0 - R)); }

// en_Collision_Elastic_10 :61-183, _Elastic_11 :187-269, _Inelastic_20 :273-394, _Ionization_30 :398-639
int32_t oracle_en_scatter(int32_t kind, double energy_eV, double threshold_eV, double neutral_mass_amu,
                          double ion_velocity_factor, const double* maxwell_v, const double* u, double* v,
                          double* new_e, double* new_i)
{
    double out[3];
    if (kind == 10 || kind == 11) {
        double c = (kind == 10) ? okhrimovskyy(energy_eV, u[0]) : 1.0 - 2.0 * u[0];
        c = clampc(c);
        double ksi = std::acos(c), s = std::sin(ksi);
        double fi = u[1] * 6.28318530718;
        rotate(c, s, std::cos(fi), std::sin(fi), v, out);
        double alpha = std::sqrt(1.0 - (0.001097161 / neutral_mass_amu) * (1.0 - c));
        v[0] = out[0] * alpha;
        v[1] = out[1] * alpha;
        v[2] = out[2] * alpha;
        return 0;
    }
    if (kind == 20) {
        if (energy_eV <= threshold_eV) return 0;
        double esc = std::max(0.0, energy_eV - threshold_eV);
        double c = clampc(okhrimovskyy(esc, u[0]));
        double ksi = std::acos(c), s = std::sin(ksi);
        double fi = u[1] * 6.28318530718;
        rotate(c, s, std::cos(fi), std::sin(fi), v, out);
        double alpha = std::sqrt(esc / energy_eV);
        v[0] = out[0] * alpha;
        v[1] = out[1] * alpha;
        v[2] = out[2] * alpha;
        return 0;
    }
    // kind 30, ionisation with B = 10 eV (:451)
    if (energy_eV <= threshold_eV) return 0;
    const double B = 10.0;
    double eej = B * std::tan(u[0] * std::atan(0.5 * (energy_eV - threshold_eV) / B));
    eej = std::max(0.0, std::min(eej, 0.5 * (energy_eV - threshold_eV)));
    double esc = std::max(0.0, energy_eV - threshold_eV - eej);
    double csc = clampc(okhrimovskyy(esc, u[1]));
    double ksc = std::acos(csc), ssc = std::sin(ksc);
    double fsc = u[2] * 6.28318530718;
    double cej = clampc(okhrimovskyy(eej, u[3]));
    double kej = std::acos(cej), sej = std::sin(kej);
    double fej = u[4] * 6.28318530718;
    double vin[3] = {v[0], v[1], v[2]};
    double osc[3], oej[3];
    rotate(csc, ssc, std::cos(fsc), std::sin(fsc), vin, osc);
    double asc = std::sqrt(esc / energy_eV);
    v[0] = osc[0] * asc;
    v[1] = osc[1] * asc;
    v[2] = osc[2] * asc;
    rotate(cej, sej, std::cos(fej), std::sin(fej), vin, oej);
    double aej = std::sqrt(eej / energy_eV);
    new_e[0] = oej[0] * aej;
    new_e[1] = oej[1] * aej;
    new_e[2] = oej[2] * aej;
    new_i[0] = oracle_maxwell_sample(maxwell_v, u[5]) * ion_velocity_factor;
    new_i[1] = oracle_maxwell_sample(maxwell_v, u[6]) * ion_velocity_factor;
    new_i[2] = oracle_maxwell_sample(maxwell_v, u[7]) * ion_velocity_factor;
    return 1;
}

static void append(oracle_parts_t* p, int64_t cap, double x, double y, const double* v, uint32_t id)
{
    if (p->n >= cap) return;
    int64_t k = p->n++;
    p->x[k] = x;
    p->y[k] = y;
    p->vx[k] = v[0];
    p->vy[k] = v[1];
    p->vz[k] = v[2];
    p->tag[k] = 0;
    p->id[k] = id;
}

// PERFORM_ELECTRON_NEUTRAL_COLLISIONS :332-485 with a per-particle Bernoulli(P_max) selection in place of the
// binary-tree draw of floor(P_max N) distinct particles; kind choice and scattering as in the reference.
static void mcc_range(const oracle_mcc_table_t* tab, const oracle_mcc_ctx_t* c, oracle_parts_t* e, int64_t lo,
                      int64_t hi, std::vector<double>* out, int64_t* counters)
{
    const double pmax = tab->max_colliding_fraction;
    for (int64_t k = lo; k < hi; ++k) {
        uint32_t w[2];
        decision_draw(e->id[k], c->seed, c->step, 0x4D430000u, w);
        if (!(uniform(w[0]) < pmax)) continue;
        double r = uniform(w[1]);
        double vx = e->vx[k], vy = e->vy[k], vz = e->vz[k];
        double v2 = std::fma(vz, vz, std::fma(vy, vy, vx * vx));
        double en = v2 * c->energy_factor_eV;
        int kind_index = oracle_mcc_choose(tab, en, r);
        if (kind_index > tab->n_act) continue;
        uint32_t b1[4], b2[4];
        philox_block(e->id[k], c->seed, c->step, 0u, 1u, b1);
        philox_block(e->id[k], c->seed, c->step, 0u, 2u, b2);
        double u[8] = {uniform(b1[0]), uniform(b1[1]), uniform(b1[2]), uniform(b1[3]),
                       uniform(b2[0]), uniform(b2[1]), uniform(b2[2]), uniform(b2[3])};
        double v[3] = {vx, vy, vz}, ne[3], ni[3];
        int kind = tab->type[kind_index - 1];
        int born = oracle_en_scatter(kind, en, tab->threshold_eV[kind_index - 1], c->neutral_mass_amu,
                                     c->ion_velocity_factor, c->maxwell_v, u, v, ne, ni);
        // en_Collision_Inelastic_20 / _Ionization_30 return before counting when below threshold
        if ((kind == 20 || kind == 30) && en <= tab->threshold_eV[kind_index - 1]) continue;
        e->vx[k] = v[0];
        e->vy[k] = v[1];
        e->vz[k] = v[2];
        counters[kind_index - 1]++;
        if (born) {
            double rec[8] = {e->x[k], e->y[k], ne[0], ne[1], ne[2], ni[0], ni[1], ni[2]};
            out->insert(out->end(), rec, rec + 8);
        }
    }
}

// Per-particle null-collision MCC; thread slices keep their ionisation products in order, so the add lists are
// the same as in a serial pass.
void oracle_mcc_philox(const oracle_mcc_table_t* tab, const oracle_mcc_ctx_t* c, oracle_parts_t* e,
                       oracle_parts_t* born_e, oracle_parts_t* born_i, int64_t cap_born, int64_t* counters)
{
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    std::vector<std::vector<double>> born(nt);
    std::vector<std::vector<int64_t>> cnt(nt, std::vector<int64_t>(8, 0));
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        int64_t lo = e->n * t / nt, hi = e->n * (t + 1) / nt;
        mcc_range(tab, c, e, lo, hi, &born[t], cnt[t].data());
    }
    for (int t = 0; t < nt; ++t) {
        for (int q = 0; q < 8; ++q) counters[q] += cnt[t][q];
        for (size_t r = 0; r < born[t].size(); r += 8) {
            const double* b = &born[t][r];
            // born particles carry no id of the parent run (marked 0xFFFFFFFF); the device numbers them itself
            append(born_e, cap_born, b[0], b[1], b + 2, 0xFFFFFFFFu);
            append(born_i, cap_born, b[0], b[1], b + 5, 0xFFFFFFFFu);
        }
    }
}

// ------------------------------------------------------------------------------------------ RCX
// calculate_thermal_cx_probab pic2d_inCollisionsSpecificProc.f90:4-31 with sigma_rcx_m2 :35-44
double oracle_rcx_probab_thermal(double sigma_1eV, double alpha, double T_K, double n_m3, double Ms, double dt_s,
                                 int32_t nsub)
{
    const double KB = 1.38064852e-23;
    double Tgas_eV = T_K * KB / E_CL;
    double e = std::max(1.5 * Tgas_eV, 0.001);
    double l = 1.0 - alpha * std::log(e);
    double sig = sigma_1eV * l * l;
    double vmean = std::sqrt(2.54647908947033 * Tgas_eV * E_CL / (Ms * M_E_KG));
    return n_m3 * sig * vmean * dt_s * nsub;
}

// PERFORM_RESONANT_CHARGE_EXCHANGE :48-126
int64_t oracle_rcx_philox(const oracle_rcx_t* r, const oracle_mcc_ctx_t* c, uint32_t species, oracle_parts_t* ions)
{
    int64_t count = 0;
    double pt2 = r->probab_thermal * r->probab_thermal;
#pragma omp parallel for reduction(+ : count) schedule(static)
    for (int64_t k = 0; k < ions->n; ++k) {
        double vx = ions->vx[k], vy = ions->vy[k], vz = ions->vz[k];
        // probab_rcx = n dt N_sub |v| V_scale sigma(E); hit when r <= sqrt(probab_rcx^2 + P_th^2), written here as
        // r^2 <= (n dt N_sub sigma(E) V_scale)^2 |v|^2 + P_th^2 (the same test without the two square roots)
        double vsq = vx * vx + vy * vy + vz * vz;
        double l = 1.0;
        if (r->alpha != 0.0) l = 1.0 - r->alpha * std::log(std::max(vsq * r->factor_eV, 0.001));
        double kf = (r->prob_factor * ((r->sigma_1eV * l) * l)) * r->v_scale_ms;
        double p2 = (kf * kf) * vsq + pt2;
        uint32_t w[2];
        decision_draw(ions->id[k], c->seed, c->step, 0x52430000u | species, w);
        double u = uniform(w[0]);
        if (u * u <= p2) {
            uint32_t b[4];
            philox_block(ions->id[k], c->seed, c->step, 1u + (species << 8), 1u, b);
            ions->vx[k] = oracle_maxwell_sample(c->maxwell_v, uniform(b[0])) * r->vfactor;
            ions->vy[k] = oracle_maxwell_sample(c->maxwell_v, uniform(b[1])) * r->vfactor;
            ions->vz[k] = oracle_maxwell_sample(c->maxwell_v, uniform(b[2])) * r->vfactor;
            ++count;
        }
    }
    return count;
}

// ------------------------------------------------------------------------------------- FFT_X solve
// Radix-2 complex FFT (Danielson-Lanczos, iterative, bit reversal), sign = +1 forward kernel exp(+2 pi i jk/N)
// as in FOUR1_8 (pic2d_ElectricFieldCalc_FFT_X.f90:1648-1710); twiddles are evaluated directly.
static void fft_complex(std::vector<double>& re, std::vector<double>& im, int sign)
{
    const int n = (int)re.size();
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            std::swap(re[i], re[j]);
            std::swap(im[i], im[j]);
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1;
        for (int k = 0; k < half; ++k) {
            double ang = sign * 2.0 * PI * k / len;
            double wr = std::cos(ang), wi = std::sin(ang);
            for (int s = 0; s < n; s += len) {
                int a = s + k, b = a + half;
                double tr = wr * re[b] - wi * im[b];
                double ti = wr * im[b] + wi * re[b];
                re[b] = re[a] - tr;
                im[b] = im[a] - ti;
                re[a] += tr;
                im[a] += ti;
            }
        }
    }
}

// SOLVE_POISSON_FFTX_LINSYSY :66-1320 (single cluster, metal walls): row FFT, per-mode Thomas with the spectral
// diagonal -2 - 4 pi^2 n^2/N^2 and a_eq of PREPARE_SYS_Y (pic2d_Prepare_FFTX_SYSY.f90:834-899), inverse FFT.
void oracle_fftx_solve(const oracle_geom_t* g, const double* rho, double phi_bottom, double phi_top, double* phi)
{
    const int N = g->ncx, J = g->ncy, nx = oracle_nx_nodes(g);
    const int nm = N / 2 + 1;
    std::vector<double> Fre((size_t)(J + 1) * nm), Fim((size_t)(J + 1) * nm);
    std::vector<double> re(N), im(N);
    for (int j = 0; j <= J; ++j) {
        for (int i = 0; i < N; ++i) {
            // xband(1:N-1) = c_rho(1:N-1), xband(0) = c_rho(N) (:155-262)
            double v = (i == 0) ? rho[node(g, N, j)] : rho[node(g, i, j)];
            if (j == 0) v = phi_bottom;
            if (j == J) v = phi_top;
            re[i] = v;
            im[i] = 0.0;
        }
        fft_complex(re, im, +1);
        for (int m = 0; m < nm; ++m) {
            Fre[(size_t)j * nm + m] = re[m];
            Fim[(size_t)j * nm + m] = (m == 0 || m == N / 2) ? 0.0 : im[m];
        }
    }
    std::vector<double> aeq(J + 1), rr(J + 1), ri(J + 1);
    for (int m = 0; m < nm; ++m) {
        double d = -2.0 - 4.0 * PI * PI * (double)m * (double)m / ((double)N * (double)N);
        aeq[0] = 0.0;
        for (int j = 1; j <= J - 1; ++j) aeq[j] = 1.0 / (d - aeq[j - 1]);
        aeq[J] = 0.0;
        rr[0] = Fre[m];
        ri[0] = Fim[m];
        for (int j = 1; j <= J - 1; ++j) {
            rr[j] = (-Fre[(size_t)j * nm + m] - rr[j - 1]) * aeq[j];
            ri[j] = (-Fim[(size_t)j * nm + m] - ri[j - 1]) * aeq[j];
        }
        rr[J] = Fre[(size_t)J * nm + m];
        ri[J] = Fim[(size_t)J * nm + m];
        Fre[(size_t)J * nm + m] = rr[J];
        Fim[(size_t)J * nm + m] = ri[J];
        for (int j = J - 1; j >= 0; --j) {
            Fre[(size_t)j * nm + m] = rr[j] - aeq[j] * Fre[(size_t)(j + 1) * nm + m];
            Fim[(size_t)j * nm + m] = ri[j] - aeq[j] * Fim[(size_t)(j + 1) * nm + m];
        }
    }
    for (int j = 0; j <= J; ++j) {
        for (int m = 0; m < nm; ++m) {
            re[m] = Fre[(size_t)j * nm + m];
            im[m] = Fim[(size_t)j * nm + m];
        }
        for (int m = nm; m < N; ++m) {  // Hermitian completion of the real signal's spectrum
            re[m] = re[N - m];
            im[m] = -im[N - m];
        }
        fft_complex(re, im, -1);
        for (int i = 0; i < N; ++i) phi[node(g, i, j)] = re[i] / N;
        phi[node(g, N, j)] = phi[node(g, 0, j)];
        phi[node(g, N + 1, j)] = phi[node(g, 1, j)];
        (void)nx;
    }
}

// CALCULATE_ELECTRIC_FIELD_FFTX_LINSYSY :1341-1545 (periodic) and CALCULATE_ELECTRIC_FIELD
// (pic2d_ElectricFieldCalc_PETSc.F90:385-452, walls everywhere)
void oracle_efield(const oracle_geom_t* g, const double* phi, double f2, double f1, double* ex, double* ey,
                   double* acc_ex, double* acc_ey)
{
    const int nx = oracle_nx_nodes(g), imax = nx - 1, J = g->ncy;
    auto P = [&](int i, int j) { return phi[node(g, i, j)]; };
    for (int j = 0; j <= J; ++j)
        for (int i = 0; i <= imax; ++i) {
            double EXv = 0.0, EYv = 0.0;
            if (g->periodic) {
                int ii = i;
                if (i == 0) ii = imax - 1;          // E(0) = E(N)  (left neighbour copy)
                if (i == imax) ii = 1;              // E(N+1) = E(1)
                EXv = f2 * (P(ii - 1, j) - P(ii + 1, j));
                if (j == 0) EYv = f1 * (P(ii, 0) - P(ii, 1));
                else if (j == J) EYv = f1 * (P(ii, J - 1) - P(ii, J));
                else EYv = f2 * (P(ii, j - 1) - P(ii, j + 1));
            } else {
                if (i == 0) EXv = f1 * (P(0, j) - P(1, j));
                else if (i == imax) EXv = f1 * (P(imax - 1, j) - P(imax, j));
                else EXv = f2 * (P(i - 1, j) - P(i + 1, j));
                if (j == 0) EYv = f1 * (P(i, 0) - P(i, 1));
                else if (j == J) EYv = f1 * (P(i, J - 1) - P(i, J));
                else EYv = f2 * (P(i, j - 1) - P(i, j + 1));
            }
            ex[node(g, i, j)] = EXv;
            ey[node(g, i, j)] = EYv;
            if (acc_ex) {
                acc_ex[node(g, i, j)] += EXv;
                acc_ey[node(g, i, j)] += EYv;
            }
        }
}

// ------------------------------------------------------------------------------------------- CG
static int node_kind(const oracle_geom_t* g, int i, int j, int* inner)
{
    // 0 unknown, 1 wall (0 below, 1 above, 2 left, 3 right via *inner = -1-side), 2 inner metal (index in *inner)
    const int imax = g->ncx, J = g->ncy;
    for (int n = 0; n < g->n_inner; ++n)
        if (i >= g->ileft[n] && i <= g->iright[n] && j >= g->jbottom[n] && j <= g->jtop[n]) {
            *inner = n;
            return 2;
        }
    if (j == 0) { *inner = -1; return 1; }
    if (j == J) { *inner = -2; return 1; }
    if (i == 0) { *inner = -3; return 1; }
    if (i == imax) { *inner = -4; return 1; }
    return 0;
}

// SET_EPS_ISHIFTED (x face between nodes (i-1, j) and (i, j)) / SET_EPS_JSHIFTED (y face between (i, j-1) and
// (i, j)), pic2d_PETSc_Solver.F90:1724-2045, for the inner objects of g (eps[n] > 0 dielectric, 0 metal)
static double set_eps_face(const oracle_geom_t* g, const double* eps_of, int i, int j, bool xface)
{
    double eps = 0.0;
    int count = 0;
    bool inside_dielectric = false, on_metal_surface = false;
    for (int pass = 0; pass < 2; ++pass)   // pass 0: dielectric objects, pass 1: metal objects
        for (int n = 0; n < g->n_inner; ++n) {
            const bool metal = !(eps_of[n] > 0.0);
            if (metal != (pass == 1)) continue;
            const int il = g->ileft[n], ir = g->iright[n], jb = g->jbottom[n], jt = g->jtop[n];
            bool covered, outline;
            if (xface) {
                covered = !(i - 1 < il || i - 1 > ir || j < jb || j > jt || i > ir);
                outline = j == jt || j == jb;
            } else {
                covered = !(i < il || i > ir || j - 1 < jb || j - 1 > jt || j > jt);
                outline = i == il || i == ir;
            }
            if (!covered) continue;
            if (pass == 0) {
                if (outline) {
                    ++count;
                    eps += eps_of[n];
                } else {
                    inside_dielectric = true;
                    eps = eps_of[n];
                    count = 1;
                    break;
                }
            } else {
                if (!outline || on_metal_surface) return 0.0;
                on_metal_surface = true;
            }
        }
    if (on_metal_surface) return count == 0 ? 1.0 : eps / count;
    if (count == 0) return 1.0;
    if (count == 1) return inside_dielectric ? eps : (1.0 + eps) / 2.0;
    return eps / (double)count;
}

static int32_t cg_general(const oracle_geom_t* g, const double* rho, const double* wall_phi, const double* inner_phi,
                          const double* inner_eps, double rtol, int32_t max_it, double* phi, double* relres_out);

int32_t oracle_cg_solve(const oracle_geom_t* g, const double* rho, const double* wall_phi, const double* inner_phi,
                        double rtol, int32_t max_it, double* phi, double* relres_out)
{
    return cg_general(g, rho, wall_phi, inner_phi, nullptr, rtol, max_it, phi, relres_out);
}

int32_t oracle_cg_solve_eps(const oracle_geom_t* g, const double* rho, const double* wall_phi, const double* inner_phi,
                            const double* inner_eps, double rtol, int32_t max_it, double* phi, double* relres_out)
{
    return cg_general(g, rho, wall_phi, inner_phi, inner_eps, rtol, max_it, phi, relres_out);
}

static int32_t cg_general(const oracle_geom_t* g, const double* rho, const double* wall_phi, const double* inner_phi,
                          const double* inner_eps, double rtol, int32_t max_it, double* phi, double* relres_out)
{
    const int nx = oracle_nx_nodes(g), J = g->ncy;
    const int64_t nn = (int64_t)nx * (J + 1);
    std::vector<int8_t> kind(nn);
    // face permittivities of the operator: ex at node (i, j) = face to (i-1, j); ey = face to (i, j-1)
    std::vector<double> ex(nn, 1.0), ey(nn, 1.0);
    if (inner_eps)
        for (int j = 0; j <= J; ++j)
            for (int i = 0; i < nx; ++i) {
                if (i >= 1) ex[node(g, i, j)] = set_eps_face(g, inner_eps, i, j, true);
                if (j >= 1) ey[node(g, i, j)] = set_eps_face(g, inner_eps, i, j, false);
            }
    for (int j = 0; j <= J; ++j)
        for (int i = 0; i < nx; ++i) {
            int w = 0;
            int k = node_kind(g, i, j, &w);
            if (k == 2 && inner_eps && inner_eps[w] > 0.0) k = 0;   // dielectric nodes are unknowns
            kind[node(g, i, j)] = (int8_t)k;
            if (k == 1) phi[node(g, i, j)] = wall_phi[-1 - w];
            if (k == 2) phi[node(g, i, j)] = inner_phi[w];
        }
    // A = -(5-point Laplacian) on unknown nodes, b = rho + Dirichlet neighbours
    std::vector<double> b(nn, 0.0), x(nn, 0.0), r(nn, 0.0), p(nn, 0.0), Ap(nn, 0.0);
    const int di[4] = {-1, 1, 0, 0}, dj[4] = {0, 0, -1, 1};
    // the face towards neighbour d of node q
    auto face = [&](int64_t q, int d) {
        switch (d) {
        case 0: return ex[q];
        case 1: return ex[q + 1];
        case 2: return ey[q];
        default: return ey[q + nx];
        }
    };
    for (int j = 1; j < J; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            int64_t q = node(g, i, j);
            if (kind[q]) continue;
            double s = rho[q];
            for (int d = 0; d < 4; ++d) {
                int64_t q2 = node(g, i + di[d], j + dj[d]);
                if (kind[q2]) s += face(q, d) * phi[q2];
            }
            b[q] = s;
            x[q] = phi[q];
        }
    auto apply = [&](const std::vector<double>& in, std::vector<double>& out) {
        for (int j = 1; j < J; ++j)
            for (int i = 1; i < nx - 1; ++i) {
                int64_t q = node(g, i, j);
                if (kind[q]) continue;
                double s = 0.0;
                for (int d = 0; d < 4; ++d) {
                    int64_t q2 = node(g, i + di[d], j + dj[d]);
                    s += face(q, d) * in[q];
                    if (!kind[q2]) s -= face(q, d) * in[q2];
                }
                out[q] = s;
            }
    };
    apply(x, Ap);
    double bn = 0.0, rr = 0.0;
    for (int64_t q = 0; q < nn; ++q)
        if (!kind[q]) {
            r[q] = b[q] - Ap[q];
            p[q] = r[q];
            bn += b[q] * b[q];
            rr += r[q] * r[q];
        }
    bn = std::sqrt(bn);
    if (bn == 0.0) bn = 1.0;
    int it = 0;
    double rel = std::sqrt(rr) / bn;
    while (rel > rtol && it < max_it) {
        apply(p, Ap);
        double pAp = 0.0;
        for (int64_t q = 0; q < nn; ++q)
            if (!kind[q]) pAp += p[q] * Ap[q];
        double alpha = rr / pAp;
        double rr2 = 0.0;
        for (int64_t q = 0; q < nn; ++q)
            if (!kind[q]) {
                x[q] += alpha * p[q];
                r[q] -= alpha * Ap[q];
                rr2 += r[q] * r[q];
            }
        double beta = rr2 / rr;
        rr = rr2;
        for (int64_t q = 0; q < nn; ++q)
            if (!kind[q]) p[q] = r[q] + beta * p[q];
        ++it;
        rel = std::sqrt(rr) / bn;
    }
    for (int64_t q = 0; q < nn; ++q)
        if (!kind[q]) phi[q] = x[q];
    if (relres_out) *relres_out = rel;
    return rel <= rtol ? it : -1;
}

// ----------------------------------------------------------------------------------- whole cycle
static void deposit_threads(const oracle_geom_t* g, const oracle_parts_t* p, double w, double* rho, int nthreads)
{
    const int64_t nn = (int64_t)oracle_nx_nodes(g) * (g->ncy + 1);
#ifdef _OPENMP
    if (nthreads > 1) {
        std::vector<std::vector<double>> part(nthreads, std::vector<double>(nn, 0.0));
#pragma omp parallel num_threads(nthreads)
        {
            int t = omp_get_thread_num();
            int64_t lo = p->n * t / nthreads, hi = p->n * (t + 1) / nthreads;
            oracle_parts_t sub = *p;
            sub.x += lo; sub.y += lo; sub.vx += lo; sub.vy += lo; sub.vz += lo; sub.tag += lo; sub.id += lo;
            sub.n = hi - lo;
            oracle_deposit(g, &sub, w, part[t].data());
        }
        std::fill(rho, rho + nn, 0.0);
        for (int t = 0; t < nthreads; ++t)
            for (int64_t q = 0; q < nn; ++q) rho[q] += part[t][q];
        return;
    }
#endif
    (void)nthreads;
    oracle_deposit(g, p, w, rho);
}

// push in thread-sized slices; each slice compacts itself, slices are then concatenated in order
static void push_threads(const oracle_geom_t* g, const oracle_species_t* sp, const double* EX, const double* EY,
                         oracle_parts_t* p, int64_t* hits, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 1) {
        std::vector<int64_t> lo(nthreads), cnt(nthreads);
        std::vector<std::vector<int64_t>> h(nthreads, std::vector<int64_t>(8, 0));
#pragma omp parallel num_threads(nthreads)
        {
            int t = omp_get_thread_num();
            int64_t a = p->n * t / nthreads, b = p->n * (t + 1) / nthreads;
            oracle_parts_t sub = *p;
            sub.x += a; sub.y += a; sub.vx += a; sub.vy += a; sub.vz += a; sub.tag += a; sub.id += a;
            sub.n = b - a;
            oracle_push(g, sp, EX, EY, &sub, h[t].data());
            lo[t] = a;
            cnt[t] = sub.n;
        }
        int64_t w = cnt[0];
        for (int t = 1; t < nthreads; ++t) {
            std::memmove(p->x + w, p->x + lo[t], cnt[t] * sizeof(double));
            std::memmove(p->y + w, p->y + lo[t], cnt[t] * sizeof(double));
            std::memmove(p->vx + w, p->vx + lo[t], cnt[t] * sizeof(double));
            std::memmove(p->vy + w, p->vy + lo[t], cnt[t] * sizeof(double));
            std::memmove(p->vz + w, p->vz + lo[t], cnt[t] * sizeof(double));
            std::memmove(p->tag + w, p->tag + lo[t], cnt[t] * sizeof(int32_t));
            std::memmove(p->id + w, p->id + lo[t], cnt[t] * sizeof(uint32_t));
            w += cnt[t];
        }
        p->n = w;
        for (int t = 0; t < nthreads; ++t)
            for (int o = 0; o < 8; ++o) hits[o] += h[t][o];
        return;
    }
#endif
    (void)nthreads;
    oracle_push(g, sp, EX, EY, p, hits);
}

int64_t oracle_cycle_step(oracle_cycle_t* c, oracle_parts_t* e, oracle_parts_t* ion, int64_t cap_e, int64_t cap_i,
                          double* work, int64_t* counters)
{
    const oracle_geom_t* g = &c->geom;
    const int64_t nn = (int64_t)oracle_nx_nodes(g) * (g->ncy + 1);
#ifdef _OPENMP
    omp_set_num_threads(c->nthreads > 0 ? c->nthreads : 1);
#endif
    double* rho_e = work;
    double* rho_i = work + nn;
    double* rho = work + 2 * nn;
    double* phi = work + 3 * nn;
    double* ex = work + 4 * nn;
    double* ey = work + 5 * nn;
    double* acc_ex = work + 7 * nn;
    double* acc_ey = work + 8 * nn;
    const int32_t nsub = c->i_sp.nsub > 0 ? c->i_sp.nsub : 1;
    const bool ion_step = c->n_sub_phase + 1 == nsub;
    int64_t processed = e->n + (ion_step ? ion->n : 0);
    // GATHER_ION_CHARGE_DENSITY when n_sub == 0 / GATHER_ELECTRON_CHARGE_DENSITY (MainProgram:151-157)
    if (c->n_sub_phase == 0) {
        deposit_threads(g, ion, c->ion_charge, rho_i, c->nthreads);
        oracle_fold_and_wall_scale(g, rho_i);
        std::fill(acc_ex, acc_ex + nn, 0.0);   // acc_E starts the ion cycle at zero
        std::fill(acc_ey, acc_ey + nn, 0.0);
    }
    deposit_threads(g, e, 1.0, rho_e, c->nthreads);
    oracle_fold_and_wall_scale(g, rho_e);
    for (int64_t q = 0; q < nn; ++q) rho[q] = c->factor_rho * (rho_i[q] - rho_e[q]);
    // SOLVE_POISSON_FFTX_LINSYSY + CALCULATE_ELECTRIC_FIELD_FFTX_LINSYSY (:182-191), acc_E += E
    oracle_fftx_solve(g, rho, c->phi_bottom, c->phi_top, phi);
    oracle_efield(g, phi, c->factor2_E, c->factor1_E, ex, ey, acc_ex, acc_ey);
    // ADVANCE_ELECTRONS_PLUS (:210)
    push_threads(g, &c->e_sp, ex, ey, e, counters + 8, c->nthreads);
    if (!ion_step) {
        c->n_sub_phase++;
        c->mcc_ctx.step++;
        return processed;
    }
    // ADVANCE_IONS_PLUS on the accumulated field (:231)
    push_threads(g, &c->i_sp, acc_ex, acc_ey, ion, counters + 8, c->nthreads);
    // PERFORM_ELECTRON_NEUTRAL_COLLISIONS (:275), PERFORM_RESONANT_CHARGE_EXCHANGE (:287)
    c->born_e.n = 0;
    c->born_i.n = 0;
    if (c->mcc) oracle_mcc_philox(c->mcc, &c->mcc_ctx, e, &c->born_e, &c->born_i, c->cap_born, counters);
    if (c->rcx_on) counters[4] += oracle_rcx_philox(&c->rcx, &c->mcc_ctx, 0u, ion);
    // PROCESS_ADDED_IONS (:300), then PROCESS_ADDED_ELECTRONS (:363)
    for (int64_t k = 0; k < c->born_i.n; ++k) {
        double v[3] = {c->born_i.vx[k], c->born_i.vy[k], c->born_i.vz[k]};
        append(ion, cap_i, c->born_i.x[k], c->born_i.y[k], v, c->next_id_i++);
    }
    for (int64_t k = 0; k < c->born_e.n; ++k) {
        double v[3] = {c->born_e.vx[k], c->born_e.vy[k], c->born_e.vz[k]};
        append(e, cap_e, c->born_e.x[k], c->born_e.y[k], v, c->next_id_e++);
    }
    // CLEAR_ACCUMULATED_FIELDS (:303); n_sub = 0
    std::fill(acc_ex, acc_ex + nn, 0.0);
    std::fill(acc_ey, acc_ey + nn, 0.0);
    c->n_sub_phase = 0;
    c->mcc_ctx.step++;
    return processed;
}

}  // extern "C"
