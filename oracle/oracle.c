/*
 * FP64 CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle.h). Restates the reference
 * kernels operation for operation; compiled with -ffp-contract=off, OpenMP over the
 * independent outer loops.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979 /* co_info_structs.h:7 */

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

#define AT(x, y, z) ((int64_t)(x) + (int64_t)(y) * (NX) + (int64_t)(z) * (NX) * (NX))

static inline double clampd(double v, double lo, double hi) {
    /* rrgsim::common::clamp (co_device_utils.cuh:44-48) */
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}
static inline int clampi(int v, int lo, int hi) {
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}

/* ---------------------------------------------------------------------------------------- */
/* nbody.cu:19-65 */
void orc_direct_acc(int64_t n, const double* pos, const double* mass, const double* soft2,
                    double* acc) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
        const double si = soft2[i];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double dx = pos[3 * j] - px;
            const double dy = pos[3 * j + 1] - py;
            const double dz = pos[3 * j + 2] - pz;
            const double den = 1. / sqrt(dx * dx + dy * dy + dz * dz + 0.5 * (si + soft2[j]));
            const double k = mass[j] * (den * den * den);
            fx += dx * k;
            fy += dy * k;
            fz += dz * k;
        }
        acc[3 * i] = fx;
        acc[3 * i + 1] = fy;
        acc[3 * i + 2] = fz;
    }
}

/* nbody.cu:67-114 */
void orc_direct_grav(int64_t n, const double* pos, const double* mass, const double* soft2,
                     double* grav) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
        const double si = soft2[i];
        double s = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double dx = pos[3 * j] - px;
            const double dy = pos[3 * j + 1] - py;
            const double dz = pos[3 * j + 2] - pz;
            s += mass[j] / sqrt(dx * dx + dy * dy + dz * dz + 0.5 * (si + soft2[j]));
        }
        grav[i] = -s;
    }
}

/* nbody.cu:122-152 */
void orc_predict(int64_t n, const double* acc, const double* vel, double* pos, double* vstar,
                 double dt) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) {
            const double v = vel[3 * i + k];
            vstar[3 * i + k] = v + dt * acc[3 * i + k];
            pos[3 * i + k] = pos[3 * i + k] + dt * 0.5 * (v + vstar[3 * i + k]);
        }
    }
}

/* nbody.cu:159-181 */
void orc_correct(int64_t n, const double* acc, double* vel, const double* vstar, double dt) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k)
            vel[3 * i + k] = 0.5 * (vel[3 * i + k] + vstar[3 * i + k] + dt * acc[3 * i + k]);
    }
}

/* rrgsim_integration_nbody.cuh:50-56 */
void orc_nbody_steps(int64_t n, double* pos, double* vel, double* acc, const double* mass,
                     const double* soft2, double dt, int nsteps) {
    double* vstar = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    for (int s = 0; s < nsteps; ++s) {
        orc_predict(n, acc, vel, pos, vstar, dt);
        orc_direct_acc(n, pos, mass, soft2, acc);
        orc_correct(n, acc, vel, vstar, dt);
    }
    free(vstar);
}

/* ---------------------------------------------------------------------------------------- */
/* CIC weights, rm_p2mesh.cu:184-216 */
static void cic_axis(double x, const orc_grid* g, double inv_dx, int* i0, int* i1, double* w0,
                     double* w1) {
    const int NXm1 = g->nx - 1;
    double u = (x - g->domain_min) * inv_dx - 0.5;
    if (!(u >= 0.0)) u = 0.0; /* NaN -> 0 (the reference would index out of bounds) */
    u = clampd(u, 0, (double)NXm1 - 1E-6);
    *i0 = (int)floor(u);
    *i1 = *i0 + 1 < NXm1 ? *i0 + 1 : NXm1;
    const double f = u - *i0;
    *w0 = 1.0 - f;
    *w1 = f;
}

static void cic_particle(const double* p, const orc_grid* g, double inv_dx, int64_t* idx,
                         double* w) {
    const int NX = g->nx;
    int i0, i1, j0, j1, k0, k1;
    double wx0, wx1, wy0, wy1, wz0, wz1;
    cic_axis(p[0], g, inv_dx, &i0, &i1, &wx0, &wx1);
    cic_axis(p[1], g, inv_dx, &j0, &j1, &wy0, &wy1);
    cic_axis(p[2], g, inv_dx, &k0, &k1, &wz0, &wz1);
    /* rm_p2mesh.cu:219-235 */
    w[0] = wx0 * wy0 * wz0; idx[0] = AT(i0, j0, k0);
    w[1] = wx1 * wy0 * wz0; idx[1] = AT(i1, j0, k0);
    w[2] = wx0 * wy1 * wz0; idx[2] = AT(i0, j1, k0);
    w[3] = wx1 * wy1 * wz0; idx[3] = AT(i1, j1, k0);
    w[4] = wx0 * wy0 * wz1; idx[4] = AT(i0, j0, k1);
    w[5] = wx1 * wy0 * wz1; idx[5] = AT(i1, j0, k1);
    w[6] = wx0 * wy1 * wz1; idx[6] = AT(i0, j1, k1);
    w[7] = wx1 * wy1 * wz1; idx[7] = AT(i1, j1, k1);
}

void orc_cic_fp64(int64_t n, const double* pos, const double* mass, const orc_grid* g,
                  double* grid) {
    const int64_t nc = (int64_t)g->nx * g->nx * g->nx;
    memset(grid, 0, sizeof(double) * (size_t)nc);
    const double inv_dx = 1. / g->dx;
    for (int64_t p = 0; p < n; ++p) {
        int64_t idx[8];
        double w[8];
        cic_particle(pos + 3 * p, g, inv_dx, idx, w);
        for (int c = 0; c < 8; ++c) grid[idx[c]] += mass[p] * w[c];
    }
}

void orc_cic_fixed(int64_t n, const double* pos, const double* mass, const orc_grid* g,
                   int shift, uint64_t* grid) {
    const int64_t nc = (int64_t)g->nx * g->nx * g->nx;
    memset(grid, 0, sizeof(uint64_t) * (size_t)nc);
    const double inv_dx = 1. / g->dx;
    const double scale = ldexp(1.0, shift);
    for (int64_t p = 0; p < n; ++p) {
        int64_t idx[8];
        double w[8];
        cic_particle(pos + 3 * p, g, inv_dx, idx, w);
        const double ms = mass[p] * scale;
        for (int c = 0; c < 8; ++c) grid[idx[c]] += (uint64_t)llrint(ms * w[c]);
    }
}

/* ---------------------------------------------------------------------------------------- */
/* wave.cu:18-104 */
static double coord(const orc_grid* g, int i) { return g->domain_min + i * g->dx; }

static int wrap(int i, int n) { return (i < 0) ? i + n : ((i >= n) ? i - n : i); }

static double layer_diss(const orc_grid* g, double x) {
    const double x_in = 0.5 * g->sim_l;
    const double d = fabs(x) - x_in;
    return (d > 0) ? g->diss_extra * d * d : 0.0;
}

static double monopole_phi(const orc_grid* g, double x, double y, double z) {
    const double rx = x - g->com[0], ry = y - g->com[1], rz = z - g->com[2];
    const double dist = sqrt(rx * rx + ry * ry + rz * rz);
    const double r = fmax(dist, g->r_min);
    return -1. * g->bc_mass / r;
}

static double psi_at(const orc_grid* g, const double* phi, int i, int j, int k) {
    const int NX = g->nx;
    return phi[AT(i, j, k)] - monopole_phi(g, coord(g, i), coord(g, j), coord(g, k));
}

static double upwind_axis(const orc_grid* g, const double* phi, double psi0, double n_comp,
                          int ix, int iy, int iz, int axis) {
    const int NX = g->nx;
    const int i0 = (axis == 0) ? ix : (axis == 1) ? iy : iz;
    int in = (n_comp > 0) ? i0 - 1 : i0 + 1;
    if (in < 0 || in >= NX) in = 2 * i0 - in;
    int jx = ix, jy = iy, jz = iz;
    if (axis == 0) jx = in;
    else if (axis == 1) jy = in;
    else jz = in;
    const double d = (psi0 - psi_at(g, phi, jx, jy, jz)) / ((i0 - in) * g->dx);
    return n_comp * d;
}

static double radiative_boundary(const orc_grid* g, const double* phi, int ix, int iy, int iz) {
    const double C = g->wave_speed, DT = g->dt;
    const double x = coord(g, ix), y = coord(g, iy), z = coord(g, iz);
    const double rx = x - g->com[0], ry = y - g->com[1], rz = z - g->com[2];
    const double r = fmax(sqrt(rx * rx + ry * ry + rz * rz), g->r_min);
    const double nx = rx / r, ny = ry / r, nz = rz / r;
    const double psi0 = psi_at(g, phi, ix, iy, iz);
    const double dpsi_dr = upwind_axis(g, phi, psi0, nx, ix, iy, iz, 0) +
                           upwind_axis(g, phi, psi0, ny, ix, iy, iz, 1) +
                           upwind_axis(g, phi, psi0, nz, ix, iy, iz, 2);
    const double psi_new = psi0 - C * DT * (dpsi_dr + psi0 / r);
    return psi_new + monopole_phi(g, x, y, z);
}

/* wave.cu:106-193 */
void orc_wave_iteration(const orc_grid* g, const double* phi, const double* phi_old,
                        const double* mass, double* phi_new) {
    const int NX = g->nx;
    const double DX = g->dx, C = g->wave_speed, DT = g->dt, DISS_BASE = g->diss_base;
    const int periodic = (g->bc_type == 1);
#pragma omp parallel for collapse(2) schedule(static)
    for (int iz = 0; iz < NX; ++iz)
        for (int iy = 0; iy < NX; ++iy)
            for (int ix = 0; ix < NX; ++ix) {
                const int on_edge = ix == 0 || ix == NX - 1 || iy == 0 || iy == NX - 1 ||
                                    iz == 0 || iz == NX - 1;
                if (!periodic && on_edge) {
                    double v;
                    switch (g->bc_type) {
                        case 2: v = monopole_phi(g, coord(g, ix), coord(g, iy), coord(g, iz)); break;
                        case 3: v = radiative_boundary(g, phi, ix, iy, iz); break;
                        default: v = 0.; break;
                    }
                    phi_new[AT(ix, iy, iz)] = v;
                    continue;
                }
                const double G = 1.;
                double rho = mass[AT(ix, iy, iz)] / (DX * DX * DX);
                if (periodic) rho -= g->rho_mean;
                const double f = 4 * ORC_PI * G * rho;
                double diss = DISS_BASE;
                if (!periodic || g->keep_layer) {
                    diss += layer_diss(g, coord(g, ix));
                    diss += layer_diss(g, coord(g, iy));
                    diss += layer_diss(g, coord(g, iz));
                }
                const int DIM = 3;
                const double Q = diss * C * DT * 0.5;
                const double W = 1 + Q;
                const double K = C * C * DT * DT / (DX * DX);
                const double K_MAIN = K / W;
                const double K_F = -C * C * DT * DT / W;
                const double K_ACTUAL = 2 * (1 - DIM * K) / W;
                const double K_OLD = (Q - 1) / W;
                int xm = ix - 1, xp = ix + 1, ym = iy - 1, yp = iy + 1, zm = iz - 1, zp = iz + 1;
                if (periodic) {
                    xm = wrap(xm, NX); xp = wrap(xp, NX);
                    ym = wrap(ym, NX); yp = wrap(yp, NX);
                    zm = wrap(zm, NX); zp = wrap(zp, NX);
                }
                const double lap_sum = phi[AT(xm, iy, iz)] + phi[AT(xp, iy, iz)] +
                                       phi[AT(ix, ym, iz)] + phi[AT(ix, yp, iz)] +
                                       phi[AT(ix, iy, zm)] + phi[AT(ix, iy, zp)];
                phi_new[AT(ix, iy, iz)] = lap_sum * K_MAIN + phi[AT(ix, iy, iz)] * K_ACTUAL +
                                          phi_old[AT(ix, iy, iz)] * K_OLD + f * K_F;
            }
}

/* wave_steady_checker.cu:30-84, 95-127 */
double orc_steady_rel_diff(int64_t ncells, const double* u_new, const double* u_old) {
    double diff = 0.0, absu = 0.0;
    for (int64_t i = 0; i < ncells; ++i) {
        diff = fmax(diff, fabs(u_new[i] - u_old[i]));
        absu = fmax(absu, fabs(u_new[i]));
    }
    return diff / (absu + 1.E-30);
}

/* wave.cu:230-297 */
int orc_solve_wave(const orc_grid* g, double** prev, double** curr, double** next,
                   const double* mass, int max_iterations, double* last_rel) {
    const int64_t nc = (int64_t)g->nx * g->nx * g->nx;
    int hold = 0, it = 0;
    double rel = -1.0;
    for (int iter = 0; iter < max_iterations; ++iter) {
        orc_wave_iteration(g, *curr, *prev, mass, *next);
        double* t = *prev; *prev = *curr; *curr = t;   /* swap(prev, curr) */
        t = *curr; *curr = *next; *next = t;           /* swap(curr, next) */
        it = iter + 1;
        if (iter && iter % g->steady_check_step == 0) {
            rel = orc_steady_rel_diff(nc, *curr, *prev);
            if (rel < g->tolerance) ++hold;
            else hold = 0;
            if (hold >= g->steady_hold_steps) break;
        }
    }
    if (last_rel) *last_rel = rel;
    return it;
}

/* rm_p2mesh.cu:238-290 */
void orc_gradient(const orc_grid* g, const double* phi, double* acc3) {
    const int NX = g->nx;
    const double coef = -1. / g->dx;
#pragma omp parallel for collapse(2) schedule(static)
    for (int iz = 0; iz < NX; ++iz)
        for (int iy = 0; iy < NX; ++iy)
            for (int ix = 0; ix < NX; ++ix) {
                const int64_t xyz = AT(ix, iy, iz);
                double dx, dy, dz;
                if (ix == 0) dx = phi[AT(ix + 1, iy, iz)] - phi[xyz];
                else if (ix == NX - 1) dx = phi[xyz] - phi[AT(ix - 1, iy, iz)];
                else dx = 0.5 * (phi[AT(ix + 1, iy, iz)] - phi[AT(ix - 1, iy, iz)]);
                if (iy == 0) dy = phi[AT(ix, iy + 1, iz)] - phi[xyz];
                else if (iy == NX - 1) dy = phi[xyz] - phi[AT(ix, iy - 1, iz)];
                else dy = 0.5 * (phi[AT(ix, iy + 1, iz)] - phi[AT(ix, iy - 1, iz)]);
                if (iz == 0) dz = phi[AT(ix, iy, iz + 1)] - phi[xyz];
                else if (iz == NX - 1) dz = phi[xyz] - phi[AT(ix, iy, iz - 1)];
                else dz = 0.5 * (phi[AT(ix, iy, iz + 1)] - phi[AT(ix, iy, iz - 1)]);
                acc3[3 * xyz] = dx * coef;
                acc3[3 * xyz + 1] = dy * coef;
                acc3[3 * xyz + 2] = dz * coef;
            }
}

/* rm_mesh2p.cu:48-114 */
void orc_interp(int64_t n, const double* pos, const orc_grid* g, const double* acc3,
                double* acc) {
    const int nx = g->nx;
    const double dx = g->dx, dmin = g->domain_min;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
        const double fx = (pos[3 * p] - dmin) / dx - 0.5;
        const double fy = (pos[3 * p + 1] - dmin) / dx - 0.5;
        const double fz = (pos[3 * p + 2] - dmin) / dx - 0.5;
        /* the reference passes its double to floorf: the float-rounded value is floored */
        int i0 = (int)floorf((float)fx), j0 = (int)floorf((float)fy), k0 = (int)floorf((float)fz);
        int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
        const double wx = fx - i0, wy = fy - j0, wz = fz - k0;
        i0 = clampi(i0, 0, nx - 1); i1 = clampi(i1, 0, nx - 1);
        j0 = clampi(j0, 0, nx - 1); j1 = clampi(j1, 0, nx - 1);
        k0 = clampi(k0, 0, nx - 1); k1 = clampi(k1, 0, nx - 1);
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int k = 0; k <= 1; k++) {
            const int kk = (k == 0) ? k0 : k1;
            const double wk = (k == 0) ? (1.0 - wz) : wz;
            for (int j = 0; j <= 1; j++) {
                const int jj = (j == 0) ? j0 : j1;
                const double wj = (j == 0) ? (1.0 - wy) : wy;
                for (int i = 0; i <= 1; i++) {
                    const int ii = (i == 0) ? i0 : i1;
                    const double wi = (i == 0) ? (1.0 - wx) : wx;
                    const double weight = wi * wj * wk;
                    const int64_t idx = (int64_t)kk * nx * nx + (int64_t)jj * nx + ii;
                    ax += weight * acc3[3 * idx];
                    ay += weight * acc3[3 * idx + 1];
                    az += weight * acc3[3 * idx + 2];
                }
            }
        }
        acc[3 * p] = ax;
        acc[3 * p + 1] = ay;
        acc[3 * p + 2] = az;
    }
}

/* rm_p2mesh.cu:37-53 */
void orc_ngp_cell(int64_t n, const double* pos, const orc_grid* g, int64_t* cell) {
    const int NX = g->nx;
    for (int64_t p = 0; p < n; ++p) {
        int ix = 0, iy = 0, iz = 0;
        const double fx = (pos[3 * p] - g->domain_min) / g->dx;
        const double fy = (pos[3 * p + 1] - g->domain_min) / g->dx;
        const double fz = (pos[3 * p + 2] - g->domain_min) / g->dx;
        ix = clampi(fx == fx ? (int)fx : 0, 0, NX - 1);
        iy = clampi(fy == fy ? (int)fy : 0, 0, NX - 1);
        iz = clampi(fz == fz ? (int)fz : 0, 0, NX - 1);
        cell[p] = AT(ix, iy, iz);
    }
}

/* rm_mesh2p.cu:29-38 */
void orc_ngp_phi(int64_t n, const double* pos, const orc_grid* g, const double* phi,
                 double* grav) {
    int64_t* cell = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    orc_ngp_cell(n, pos, g, cell);
    for (int64_t p = 0; p < n; ++p) grav[p] = phi[cell[p]];
    free(cell);
}

/* rrgsim_integration_rect.cuh:99-112 */
void orc_pm_steps(int64_t n, double* pos, double* vel, double* acc, const double* mass,
                  const orc_grid* g, int iterations, double dt, double** prev, double** curr,
                  double** next, double* mgrid, double* acc3, int nsteps) {
    double* vstar = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    for (int s = 0; s < nsteps; ++s) {
        orc_predict(n, acc, vel, pos, vstar, dt);
        orc_cic_fp64(n, pos, mass, g, mgrid);
        orc_solve_wave(g, prev, curr, next, mgrid, iterations, NULL);
        orc_gradient(g, *curr, acc3);
        orc_interp(n, pos, g, acc3, acc);
        orc_correct(n, acc, vel, vstar, dt);
    }
    free(vstar);
}

/* nbody.cu:246-291 */
void orc_conservation(int64_t n, const double* pos, const double* vel, const double* mass,
                      const double* grav, double* out) {
    double Ek = 0, Ep = 0, P[3] = {0, 0, 0}, L[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i) {
        const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        const double m = mass[i];
        const double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
        P[0] += m * vx;
        P[1] += m * vy;
        P[2] += m * vz;
        L[0] += m * (vz * y - vy * z);
        L[1] += m * (vx * z - vz * x);
        L[2] += m * (vy * x - vx * y);
        Ek += m * (vx * vx + vy * vy + vz * vz);
        Ep += m * grav[i];
    }
    out[0] = Ek * 0.5;
    out[1] = Ep * 0.5;
    out[2] = P[0]; out[3] = P[1]; out[4] = P[2];
    out[5] = L[0]; out[6] = L[1]; out[7] = L[2];
}

/* nbody.cu:293-439 (sum of m x over sum of m) */
void orc_mass_center(int64_t n, const double* pos, const double* mass, double* out) {
    double s[3] = {0, 0, 0}, M = 0;
    for (int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) s[k] += pos[3 * i + k] * mass[i];
        M += mass[i];
    }
    for (int k = 0; k < 3; ++k) out[k] = M > 0.0 ? s[k] / M : 0.0;
    out[3] = M;
}

/* ---------------------------------------------------------------------------------------- */
/* synthetic exponential disk (the generator of rrg_generate_exp_disk, restated) */
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
typedef struct { uint64_t s[4]; } orc_rng;

static void rng_seed(orc_rng* g, uint64_t seed) {
    uint64_t z = seed;
    for (int k = 0; k < 4; ++k) {
        z += 0x9e3779b97f4a7c15ULL;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
        x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
        g->s[k] = x ^ (x >> 31);
    }
}

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t rng_next(orc_rng* g) {
    uint64_t* s = g->s;
    const uint64_t r = rotl64(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return r;
}

static double rng_uniform(orc_rng* g) { return (double)(rng_next(g) >> 11) * 0x1.0p-53; }
static double rng_uniform_open(orc_rng* g) {
    return ((double)(rng_next(g) >> 11) + 0.5) * 0x1.0p-53;
}
static double rng_normal(orc_rng* g) {
    const double u1 = rng_uniform_open(g), u2 = rng_uniform(g);
    return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

void orc_exp_disk(uint64_t seed, int64_t n, double disk_mass, double scale_length, double z0,
                  double r_max, double z_max, double disp_frac, double* pos, double* vel) {
    orc_rng g;
    rng_seed(&g, seed);
    const double Rd = scale_length;
    const double fmx = 1.0 - (1.0 + r_max / Rd) * exp(-r_max / Rd);
    for (int64_t i = 0; i < n; ++i) {
        const double u = rng_uniform(&g) * fmx;
        double lo = 0.0, hi = r_max / Rd;
        for (int it = 0; it < 80; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (1.0 - (1.0 + mid) * exp(-mid) < u) lo = mid;
            else hi = mid;
        }
        const double R = 0.5 * (lo + hi) * Rd;
        const double ph = 2.0 * M_PI * rng_uniform(&g);
        double z;
        do {
            const double w = rng_uniform_open(&g);
            z = z0 * atanh(2.0 * w - 1.0);
        } while (!(fabs(z) < z_max));
        const double c = cos(ph), s = sin(ph);
        pos[3 * i] = R * c;
        pos[3 * i + 1] = R * s;
        pos[3 * i + 2] = z;
        const double x = R / Rd;
        const double menc = disk_mass * (1.0 - (1.0 + x) * exp(-x));
        const double vc = R > 0 ? sqrt(1.0 * menc / R) : 0.0;
        const double sig = disp_frac * vc;
        vel[3 * i] = -vc * s + sig * rng_normal(&g);
        vel[3 * i + 1] = vc * c + sig * rng_normal(&g);
        vel[3 * i + 2] = sig * rng_normal(&g);
    }
}
