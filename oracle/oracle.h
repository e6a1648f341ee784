/*
 * FP64 CPU oracle of the RRGalaxSim galaxy-dynamics hot path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C (OpenMP) restatement of the reference kernels, used by the tests as the checker and
 * by the benchmark as the CPU baseline. The product library (librrg.so) never links or calls it.
 * Each function cites the reference file:line (relative to the reference project root) it
 * follows. Compiled with -ffp-contract=off so every operation is rounded on its own.
 *
 * Arrays are AoS doubles like the reference's real3 (x, y, z per particle); grids are
 * x-fastest AT(x, y, z) = x + y nx + z nx^2 (solver/lib/rrgsim_common/include/co_device_utils.cuh:61).
 */
#ifndef RRG_ORACLE_H
#define RRG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Grid + wave + boundary parameters in one struct (GridInfo, WaveParams, BoundaryParams of
 * solver/lib/rrgsim_common/include/co_info_structs.h:16-69 and co_boundary.cuh:11-26). */
typedef struct {
    int32_t nx;
    double dx;
    double domain_min;
    double sim_l;
    double wave_speed;
    double dt;
    double diss_base;
    double diss_extra;
    int32_t bc_type; /* 0 zero Dirichlet, 1 periodic, 2 monopole Dirichlet, 3 monopole radiative */
    double bc_mass;
    double com[3];
    double r_min;
    double rho_mean;
    int32_t keep_layer;
    double tolerance;
    int32_t steady_check_step;
    int32_t steady_hold_steps;
} orc_grid;

int orc_num_threads(void);
void orc_set_threads(int n);

/* acceleration_kernel_blocked_: solver/lib/rrgsim_nbody/src/nbody.cu:19-65 */
void orc_direct_acc(int64_t n, const double* pos, const double* mass, const double* soft2,
                    double* acc);
/* grav_kernel_blocked_: nbody.cu:67-114 (self term kept, sign at :113) */
void orc_direct_grav(int64_t n, const double* pos, const double* mass, const double* soft2,
                     double* grav);
/* predict_step_: nbody.cu:122-152 */
void orc_predict(int64_t n, const double* acc, const double* vel, double* pos, double* vstar,
                 double dt);
/* correct_step_: nbody.cu:159-181 */
void orc_correct(int64_t n, const double* acc, double* vel, const double* vstar, double dt);
/* NBodyIntegrationSolver::calc_step (solver/app/include/rrgsim_integration_nbody.cuh:50-56),
 * nsteps times; acc must hold a(x) on entry and holds a(x_new) on exit. */
void orc_nbody_steps(int64_t n, double* pos, double* vel, double* acc, const double* mass,
                     const double* soft2, double dt, int nsteps);

/* deposit_cell_mass_CIC_: solver/lib/rrgsim_rect_mesh/src/rm_p2mesh.cu:176-236, summed in
 * particle order (the reference's FP64 atomics sum in an unspecified order). grid is zeroed. */
void orc_cic_fp64(int64_t n, const double* pos, const double* mass, const orc_grid* g,
                  double* grid);
/* The same weights, each corner value m w rounded to int64 fixed point round(m w 2^shift)
 * and summed exactly (order-independent). grid is zeroed. */
void orc_cic_fixed(int64_t n, const double* pos, const double* mass, const orc_grid* g,
                   int shift, uint64_t* grid);

/* wave_diss_iteration: solver/lib/rrgsim_wave/src/wave.cu:106-193 (all boundary types) */
void orc_wave_iteration(const orc_grid* g, const double* phi, const double* phi_old,
                        const double* mass, double* phi_new);
/* reduce_step_error + SteadyStateChecker::calc_max_diff:
 * solver/lib/rrgsim_wave/src/wave_steady_checker.cu:30-84, 95-127 */
double orc_steady_rel_diff(int64_t ncells, const double* u_new, const double* u_old);
/* solve_wave_equation: wave.cu:230-297. prev/curr/next rotate exactly like the reference
 * (pointers swapped in place: on return *curr holds the latest level). Returns iterations run. */
int orc_solve_wave(const orc_grid* g, double** prev, double** curr, double** next,
                   const double* mass, int max_iterations, double* last_rel);

/* calc_acceleration_field_: rm_p2mesh.cu:238-290 (acc3 is nx^3 x 3) */
void orc_gradient(const orc_grid* g, const double* phi, double* acc3);
/* interpolate_acceleration_to_particles_kernel: solver/lib/rrgsim_rect_mesh/src/rm_mesh2p.cu:
 * 48-114 (floorf of the double fraction kept, :68-70) */
void orc_interp(int64_t n, const double* pos, const orc_grid* g, const double* acc3,
                double* acc);
/* assign_particles_to_cells_ cell (rm_p2mesh.cu:37-53) + projectCellPhiOnParticles
 * (rm_mesh2p.cu:29-38) */
void orc_ngp_cell(int64_t n, const double* pos, const orc_grid* g, int64_t* cell);
void orc_ngp_phi(int64_t n, const double* pos, const orc_grid* g, const double* phi,
                 double* grav);

/* RectWaveIntegrationSolver::calc_step (solver/app/include/rrgsim_integration_rect.cuh:
 * 99-112), nsteps times. State: pos, vel, acc (a on particles), wave levels prev/curr/next
 * (rotated in place), mass grid scratch (nx^3), acc3 grid scratch (nx^3 x 3). */
void orc_pm_steps(int64_t n, double* pos, double* vel, double* acc, const double* mass,
                  const orc_grid* g, int iterations, double dt, double** prev, double** curr,
                  double** next, double* mgrid, double* acc3, int nsteps);

/* calc_conservation: nbody.cu:246-291. out = {Ek, Ep, Px, Py, Pz, Lx, Ly, Lz} */
void orc_conservation(int64_t n, const double* pos, const double* vel, const double* mass,
                      const double* grav, double* out);
/* calc_mass_center: nbody.cu:293-439. out = {cx, cy, cz, M} */
void orc_mass_center(int64_t n, const double* pos, const double* mass, double* out);

/* The benchmark's synthetic exponential disk (no bulge), restated here so that the timed CPU
 * arm needs nothing of the product library: xoshiro256** seeded through SplitMix64; R from the
 * truncated enclosed-mass CDF 1 - (1 + x) e^-x by 80 bisection steps; z = z0 atanh(2w - 1)
 * below z_max; circular speed sqrt(M(<R) / R) plus Gaussian dispersion (Box-Muller). Draw for
 * draw and operation for operation the generator of rrg_generate_exp_disk, so the same seed
 * gives the same bits. pos, vel: n x 3. */
void orc_exp_disk(uint64_t seed, int64_t n, double disk_mass, double scale_length, double z0,
                  double r_max, double z_max, double disp_frac, double* pos, double* vel);

#ifdef __cplusplus
}
#endif

#endif
