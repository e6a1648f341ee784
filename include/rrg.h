/*
 * rrg.h — C ABI of the B200 galaxy-dynamics library (librrg.so).
 *
 * Plain C types only: pointers, sizes, POD structs, int status codes. No C++ or torch types
 * cross this boundary and no exception leaves it. Every entry point returns an rrg_status;
 * the message of the last failure is read with rrg_last_error().
 *
 * The library replaces the solver libraries of RRGalaxSim (solver/lib/rrgsim_{nbody,rect_mesh,
 * wave,io,common}). Each declaration names the reference interface it stands in for as
 * file:line, relative to the reference project root.
 *
 * Ownership and threading
 *   - A context (rrg_ctx) owns its device buffers. It is not thread-safe; distinct contexts
 *     are independent (the reference keeps its parameters in process-global __constant__
 *     symbols, solver/lib/rrgsim_common/src/co_device_structs.cu:7-13, so it can hold only
 *     one simulation per process; this library has no such globals).
 *   - Operator calls are asynchronous on the context stream unless stated otherwise. Calls
 *     that return host data (rrg_get_*, rrg_calc_conservation, rrg_solve_wave_equation when it
 *     checks convergence) synchronise that stream.
 *   - rrg_dev_* entry points borrow caller-owned device memory and run on the caller's
 *     cudaStream_t (passed as void*).
 */
#ifndef RRG_H
#define RRG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define RRG_API __attribute__((visibility("default")))
#else
#define RRG_API
#endif

/* ------------------------------------------------------------------------------------------ */
/* Status codes                                                                                */
/* ------------------------------------------------------------------------------------------ */
typedef enum {
    RRG_OK = 0,
    RRG_ERR_INVALID = 1,     /* bad argument, bad size, NaN in input, missing section       */
    RRG_ERR_CUDA = 2,        /* a CUDA runtime error (message holds cudaGetErrorString)      */
    RRG_ERR_NOMEM = 3,       /* device or host allocation failed                             */
    RRG_ERR_IO = 4,          /* file missing, unreadable, malformed or unwritable            */
    RRG_ERR_STATE = 5,       /* call out of order (e.g. wave solve before a grid exists)     */
    RRG_ERR_UNSUPPORTED = 6  /* valid request this build does not implement                  */
} rrg_status;

/* Arithmetic of the particle path.
 *   RRG_PREC_FP32  : FP32 state and pair arithmetic (rsqrt on the SFU), FP32 accumulation.
 *   RRG_PREC_MIXED : FP32 pairs with compensated (Kahan) accumulation over j-tiles, positions
 *                    kept as double-float (hi, lo) pairs so pair differences and the drift
 *                    keep ~48 bits.
 *   RRG_PREC_FP64  : FP64 throughout (the reference's default `real`,
 *                    solver/lib/rrgsim_common/include/co_types.h:4-18); a checking path. */
typedef enum { RRG_PREC_FP32 = 0, RRG_PREC_MIXED = 1, RRG_PREC_FP64 = 2 } rrg_precision;

/* Boundary types of the wave solver: solver/lib/rrgsim_common/include/co_boundary.cuh:4-9 */
typedef enum {
    RRG_BC_ZERO_DIRICHLET = 0,
    RRG_BC_PERIODIC = 1,
    RRG_BC_MONOPOLE_DIRICHLET = 2,
    RRG_BC_MONOPOLE_RADIATIVE = 3
} rrg_boundary_type;

/* ------------------------------------------------------------------------------------------ */
/* Parameter structs (field meaning identical to the reference structs cited)                  */
/* ------------------------------------------------------------------------------------------ */

/* SimParams: solver/lib/rrgsim_common/include/co_sim_params.h:12-20 */
typedef struct {
    double time_max;
    double dt_save;
    double dt_dynamics;
    uint64_t saves_without_dump; /* UINT64_MAX when absent from params.json */
    int32_t use_wave_model;      /* set when grid_params and wave_params are both present */
} rrg_sim_params;

/* GridInfo: solver/lib/rrgsim_common/include/co_info_structs.h:16-33 */
typedef struct {
    int32_t nx;
    double dx;
    double domain_l;   /* nx * dx */
    double domain_min; /* -domain_l / 2 */
    double domain_max; /* +domain_l / 2 */
    double bc_l;       /* bc_frac / 2 * domain_l */
    double sim_l;      /* (1 - bc_frac) * domain_l */
} rrg_grid_info;

/* WaveParams: solver/lib/rrgsim_common/include/co_info_structs.h:36-69 */
typedef struct {
    double diss_base;
    double diss_extra;
    double wave_speed;
    double dt; /* 0.5 dx / (c sqrt 3), filled by the parser (io_json.cpp:170-179) */
    int32_t setup_iterations;
    int32_t iterations;
    double tolerance;
    int32_t print_step;
    int32_t steady_check_step;
    int32_t steady_hold_steps;
} rrg_wave_params;

/* ConservationInfo: solver/lib/rrgsim_nbody/include/nbody.cuh:13-23 (E = Ek + Ep) */
typedef struct {
    double time;
    double Ek;
    double Ep;
    double momentum[3];
    double angular[3];
} rrg_conservation;

/* IniGalaxyData: solver/lib/rrgsim_io/include/io_ini_galaxy_data.h:11-18.
 * Empty path string = component absent (JSON null or missing key). */
typedef struct {
    double mass_star;
    double mass_dark;
    double soft_star;
    double soft_dark;
    char ini_file_star[1024];
    char ini_file_dark[1024];
} rrg_ini_params;

/* ParsedParams: solver/lib/rrgsim_io/include/io_json.h:20-25 */
typedef struct {
    rrg_ini_params ini;
    rrg_sim_params sim;
    int32_t has_grid;
    rrg_grid_info grid;
    int32_t has_wave;
    rrg_wave_params wave;
} rrg_parsed_params;

typedef struct rrg_ctx rrg_ctx;

/* ------------------------------------------------------------------------------------------ */
/* Library / errors                                                                            */
/* ------------------------------------------------------------------------------------------ */

/* Version string of this library. */
RRG_API const char* rrg_version(void);

/* Message of the last failed call on ctx; ctx == NULL gives the calling thread's last
 * message from a call that had no context (or failed to create one). Never NULL. */
RRG_API const char* rrg_last_error(const rrg_ctx* ctx);

/* Number of kernels this library has launched in this process (all contexts and rrg_dev_*
 * calls; graph replays count each kernel node). Used to report launch counts. */
RRG_API uint64_t rrg_kernel_launch_count(void);

/* ------------------------------------------------------------------------------------------ */
/* Context lifecycle — replaces initialize_particles_context_ / initialize_grid_context_       */
/* (solver/lib/rrgsim_common/src/co_particles_context.cu:22-46, co_grid_context.cu:20-42)     */
/* ------------------------------------------------------------------------------------------ */

/* Creates a context on CUDA device `device` computing in `precision` (rrg_precision). */
RRG_API rrg_status rrg_create(int device, int precision, rrg_ctx** out);
RRG_API rrg_status rrg_destroy(rrg_ctx* ctx);

/* Makes the context launch on `stream` (a cudaStream_t; NULL = the context's own stream).
 * Once the context has a grid, the stream it launches on carries a persisting L2
 * access-policy window over the context's deposit grids and wave levels (48 MB at 128^3), and
 * the process's persisting L2 set-aside is sized to it: every PM step reads and rewrites those
 * grids, and keeping them in L2 shortens the step by ~3%. The window moves with the context to
 * a new stream, and rrg_destroy takes it off a caller's stream. Environment RRG_L2_PERSIST=0
 * leaves L2 alone. */
RRG_API rrg_status rrg_set_stream(rrg_ctx* ctx, void* stream);
RRG_API rrg_status rrg_synchronize(rrg_ctx* ctx);

/* Uploads particles: pos/vel are n x 3 doubles (AoS, as real3 in the reference), mass and
 * soft2 are n doubles (ParticlesData, solver/lib/rrgsim_common/include/co_particles.h:7-14).
 * The reference needs n % 256 == 0 (io_particles_csv.cpp:122-125); this library takes any
 * n >= 1. NaN/Inf in any input, or a negative mass or soft2, is RRG_ERR_INVALID.
 * Acceleration and potential start at zero, time at 0. */
RRG_API rrg_status rrg_load_particles(rrg_ctx* ctx, int64_t n, const double* pos,
                                      const double* vel, const double* mass,
                                      const double* soft2);
RRG_API int64_t rrg_num_particles(const rrg_ctx* ctx);

/* Downloads the particle state in the original particle order (ParticlesContext::
 * fill_device_data, co_particles_context.cu:7-18). Any pointer may be NULL. pos/vel/acc are
 * n x 3, grav is n. Synchronises the context stream. */
RRG_API rrg_status rrg_get_particles(rrg_ctx* ctx, double* pos, double* vel, double* acc,
                                     double* grav);

/* Simulation time and iteration counters kept with the context (ParticlesContext_::time,
 * ::iter). rrg_solver_calc_steps advances them. */
RRG_API rrg_status rrg_get_time(const rrg_ctx* ctx, double* time, uint64_t* iter);

/* Allocates the grid (5 x nx^3 arrays in the reference). grid->domain_* must be filled
 * (rrg_grid_info_from_json_values fills them the way io_json.cpp:28-40 does). */
RRG_API rrg_status rrg_init_grid(rrg_ctx* ctx, const rrg_grid_info* grid);

/* Wave parameters (copied to __constant__ wave_params_ by the reference,
 * rrgsim_integration_rect.cuh:23-31). */
RRG_API rrg_status rrg_set_wave_params(rrg_ctx* ctx, const rrg_wave_params* wave);

/* Downloads the grid: mass (cell mass, nx^3), grav (potential, nx^3), acc (nx^3 x 3),
 * x-fastest AT(x,y,z) = x + y nx + z nx^2 (co_device_utils.cuh:61). Any pointer may be NULL.
 * GridContext::fill_device_data, solver/lib/rrgsim_common/src/co_grid_context.cu:8-18. */
RRG_API rrg_status rrg_get_grid(rrg_ctx* ctx, double* mass, double* grav, double* acc);

/* Uploads a potential into the wave state (both time levels), for tests and restarts. */
RRG_API rrg_status rrg_set_grid_potential(rrg_ctx* ctx, const double* grav);

/* Fixed-point scale of the deposit: the grid holds round(m w 2^S) in int64 per cell. */
RRG_API rrg_status rrg_get_deposit_scale(const rrg_ctx* ctx, int32_t* shift_s);

/* ------------------------------------------------------------------------------------------ */
/* Operators — one per reference free function                                                 */
/* ------------------------------------------------------------------------------------------ */

/* predict_step: solver/lib/rrgsim_nbody/src/nbody.cu:122-152, 183-198 */
RRG_API rrg_status rrg_predict_step(rrg_ctx* ctx, double dt);
/* nbody_acceleration: nbody.cu:19-65, 200-213 */
RRG_API rrg_status rrg_nbody_acceleration(rrg_ctx* ctx);
/* nbody_grav: nbody.cu:67-114, 215-228 (self term kept, as the reference does) */
RRG_API rrg_status rrg_nbody_grav(rrg_ctx* ctx);
/* correct_step: nbody.cu:159-181, 230-244 */
RRG_API rrg_status rrg_correct_step(rrg_ctx* ctx, double dt);

/* convert_particles_to_grid: solver/lib/rrgsim_rect_mesh/src/rm_p2mesh.cu:398-451 (CIC of
 * particle mass, :176-236). Deposits into int64 fixed point: bit-exact, order-independent. */
RRG_API rrg_status rrg_convert_particles_to_grid(rrg_ctx* ctx);

/* set_boundary_periodic: solver/lib/rrgsim_wave/src/wave.cu:214-228 */
RRG_API rrg_status rrg_set_boundary_periodic(rrg_ctx* ctx, double total_mass, int keep_layer);
/* set_boundary_monopole: wave.cu:196-211 (r_min = dx / 2) */
RRG_API rrg_status rrg_set_boundary_monopole(rrg_ctx* ctx, double total_mass,
                                             const double center_of_mass[3], int radiative);
/* Zero-Dirichlet boundary (BoundaryType::ZeroDirichlet, the reference's default value). */
RRG_API rrg_status rrg_set_boundary_zero(rrg_ctx* ctx);

/* solve_wave_equation: wave.cu:230-297 with SteadyStateChecker
 * (wave_steady_checker.cu:88-152). Runs up to max_iterations substeps; every
 * steady_check_step substeps it compares max|dphi| / (max|phi| + 1e-30) with the tolerance
 * and stops after steady_hold_steps consecutive passes. iterations_run and last_rel_diff may
 * be NULL. Synchronises when a check falls inside the run. */
RRG_API rrg_status rrg_solve_wave_equation(rrg_ctx* ctx, int max_iterations,
                                           int* iterations_run, double* last_rel_diff);

/* calc_acceleration_field: rm_p2mesh.cu:238-290, 337-354 */
RRG_API rrg_status rrg_calc_acceleration_field(rrg_ctx* ctx);
/* No reference counterpart: rrg_solve_wave_equation for exactly `iterations` substeps without
 * steady-state checks, then rrg_calc_acceleration_field, as one call. Periodic FP32 / MIXED
 * grids of 32, 64 or 128 cells without an absorbing layer run it as one persistent kernel
 * (source, substeps and gradient in one launch, the per-step wave solve of the fused stepping
 * path); everything else launches the separate kernels. The results are the same bits either
 * way. iterations >= 1. */
RRG_API rrg_status rrg_solve_wave_and_field(rrg_ctx* ctx, int iterations);
/* No reference counterpart. The device memory through which the persistent wave solve's thread
 * blocks synchronise, for diagnostics: per block an epoch counter (uint32, 128 bytes apart,
 * block = z-chunk x blocks-along-y + y-block), the error word (the uint32 at byte 65532,
 * non-zero after a wait between blocks ran out), then the face buffers. Zeroed by
 * rrg_init_grid; writing it makes the next solve report an error (or compute garbage).
 * Synchronising calls (rrg_synchronize, rrg_get_particles, rrg_calc_conservation) turn a set
 * error word into RRG_ERR_CUDA and zero the memory again. */
RRG_API rrg_status rrg_wave_solve_sync(rrg_ctx* ctx, void** dev_ptr, size_t* bytes);
/* project_grid_acceleration_on_particles: solver/lib/rrgsim_rect_mesh/src/rm_mesh2p.cu:
 * 48-114, 129-152 (trilinear) */
RRG_API rrg_status rrg_project_grid_acceleration_on_particles(rrg_ctx* ctx);
/* project_grid_grav_on_particles: rm_mesh2p.cu:29-38, 154-168 (NGP cell of the particle) */
RRG_API rrg_status rrg_project_grid_grav_on_particles(rrg_ctx* ctx);

/* calc_conservation: nbody.cu:246-291, as FP64 device reductions. Synchronises. */
RRG_API rrg_status rrg_calc_conservation(rrg_ctx* ctx, rrg_conservation* out);
/* calc_mass_center: nbody.cu:293-439, FP64. Synchronises. */
/* The same reductions, asynchronous: enqueues them on the context stream with a copy of the
 * raw sums (sum m v^2, sum m phi, P[3], L[3], then four zeros) into `sums` (12 doubles of host
 * memory) and returns without waiting. Pinned memory that the device can address (cudaHostAlloc,
 * or cudaHostRegister with mapping) receives them from the reduction kernel itself; other host
 * memory through a copy, asynchronous only when pinned. Read
 * them after the stream has passed that point; rrg_conservation_from_sums converts. No
 * reference counterpart: it lets a host loop overlap the read of one step's diagnostics with
 * the next step. */
RRG_API rrg_status rrg_calc_conservation_async(rrg_ctx* ctx, double* sums);
RRG_API rrg_status rrg_conservation_from_sums(const double* sums, double time,
                                              rrg_conservation* out);
RRG_API rrg_status rrg_calc_mass_center(rrg_ctx* ctx, double center_of_mass[3],
                                        double* total_mass);

/* ------------------------------------------------------------------------------------------ */
/* Integration strategies — IntegrationSolver (solver/app/include/rrgsim_integration.cuh:     */
/* 22-42) with NBodyIntegrationSolver (rrgsim_integration_nbody.cuh) and                      */
/* RectWaveIntegrationSolver (rrgsim_integration_rect.cuh)                                     */
/* ------------------------------------------------------------------------------------------ */

/* init: picks the wave strategy when sim->use_wave_model is set (then the grid and wave
 * parameters must already be set), the direct N-body strategy otherwise. */
RRG_API rrg_status rrg_solver_init(rrg_ctx* ctx, const rrg_sim_params* sim);
/* precalc: N-body: potential + acceleration; wave: deposit, periodic boundary with total
 * mass 1 (rrgsim_integration_rect.cuh:65-69), setup_iterations relaxation, gradient. */
RRG_API rrg_status rrg_solver_precalc(rrg_ctx* ctx);
/* calc_step, nsteps times. Fused kernels, replayed as CUDA graphs; advances time and iter. */
RRG_API rrg_status rrg_solver_calc_steps(rrg_ctx* ctx, int nsteps);
/* Records and instantiates every CUDA graph that the next rrg_solver_calc_steps(ctx, nsteps)
 * replays, so that call launches without recording. Runs nothing on the device and leaves
 * the state as it was. No counterpart in the reference (it has no graphs). */
RRG_API rrg_status rrg_solver_prepare(rrg_ctx* ctx, int nsteps);
/* sync_particles_and_grid: potential (and, in wave mode, acceleration) on particles. */
RRG_API rrg_status rrg_solver_sync(rrg_ctx* ctx);
/* Precalc for a restored state (resume from a dump, wiring read_particles_dump,
 * io_particles_bin.cu:39-77, which the reference never calls): N-body as precalc; wave mode
 * deposits and takes the gradient of the potential set by rrg_set_wave_state, without the
 * setup relaxation. */
RRG_API rrg_status rrg_solver_resume(rrg_ctx* ctx);
/* The two wave levels (current and previous, nx^3 FP64 each, x fastest) out of / into the
 * context, for saving and restoring the wave state with a dump. */
RRG_API rrg_status rrg_get_wave_state(rrg_ctx* ctx, double* phi_cur, double* phi_prev);
RRG_API rrg_status rrg_set_wave_state(rrg_ctx* ctx, const double* phi_cur,
                                      const double* phi_prev);

/* Sorts particles by grid cell (counting sort) so deposits from one warp hit few cells.
 * Host-visible order is unchanged (rrg_get_particles undoes the permutation). The wave
 * strategy re-sorts on its own every `interval` steps (default 64); 0 disables it. Results do
 * not depend on the interval. */
RRG_API rrg_status rrg_set_sort_interval(rrg_ctx* ctx, int interval);

/* enable != 0: in wave mode the last particle pass of every rrg_solver_calc_steps call also
 * forms the conservation sums of the state it leaves (8 double-doubles per 256 particles), so
 * that rrg_calc_conservation / rrg_calc_conservation_async right after the call only combine
 * them (one small kernel) instead of reading every particle again. Any other call that may
 * change the state in between makes them recompute from the particles. The sums are the same
 * double-double reductions either way. Off by default: it costs the pass a little when no
 * diagnostics follow. No reference counterpart (calc_conservation, nbody.cu:246-291, always
 * reads the particles). */
RRG_API rrg_status rrg_set_step_sums(rrg_ctx* ctx, int enable);

/* ------------------------------------------------------------------------------------------ */
/* Host I/O — the rrgsim executable's boundary (no GPU needed)                                 */
/* ------------------------------------------------------------------------------------------ */

/* parse_params_json: solver/lib/rrgsim_io/src/io_json.cpp:188-242 (+ from_json :13-131,
 * validate_dependent_fields :170-186). Defaults as the reference. */
RRG_API rrg_status rrg_parse_params_json(const char* path, rrg_parsed_params* out);

/* read_simple_particles_data: solver/lib/rrgsim_io/src/io_particles_csv.cpp:89-134, for one
 * component (read_particles_data_component, :11-87). Reads "N t" then N rows of
 * "x y z vx vy vz". Appends to the arrays after `n_before` particles; the mass of each new
 * particle is component_mass / (n_before + N), as the reference divides by the cumulative
 * count (:37,46). capacity is the room of the output arrays in particles. */
RRG_API rrg_status rrg_read_ic_component(const char* path, double component_mass,
                                         double component_soft, int64_t n_before,
                                         int64_t capacity, double* pos, double* vel,
                                         double* mass, double* soft2, int64_t* n_read);
/* Number of particles an IC file's header announces (first token). */
RRG_API rrg_status rrg_ic_header_count(const char* path, int64_t* n);
/* Writes an IC text file in the reference format (header "N t", rows "x y z vx vy vz"). */
RRG_API rrg_status rrg_write_ic_text(const char* path, int64_t n, double t, const double* pos,
                                     const double* vel);

/* write_particles_dump: solver/lib/rrgsim_io/src/io_particles_bin.cu:9-37. Writes
 * <dir>/S_{iter:>5d}.bin = uint64 N, float64 t, float64 pos[N][3], float64 vel[N][3]. */
RRG_API rrg_status rrg_write_dump(const char* dump_dir, uint64_t iter, double time, int64_t n,
                                  const double* pos, const double* vel);
/* read_particles_dump: io_particles_bin.cu:39-77 (header only when pos/vel are NULL). */
RRG_API rrg_status rrg_read_dump(const char* path, int64_t capacity, int64_t* n, double* time,
                                 double* pos, double* vel);

/* The wave state beside a snapshot: <dir>/W_{iter:>5d}.bin = uint64 nx, float64 t,
 * float64 phi_cur[nx^3], float64 phi_prev[nx^3]. No counterpart in the reference (its dump holds
 * particles only); with it a wave-mode run resumes exactly. */
RRG_API rrg_status rrg_write_wave_state(const char* dump_dir, uint64_t iter, double time,
                                        int32_t nx, const double* phi_cur,
                                        const double* phi_prev);
RRG_API rrg_status rrg_read_wave_state(const char* path, int32_t nx, double* time,
                                       double* phi_cur, double* phi_prev);

/* The whole `rrgsim <work_dir>` run (solver/app/src/rrgsim.cu:12-62 and integrate(),
 * solver/app/src/rrgsim_integration.cu:19-146): parses params.json, reads the ICs (paths
 * relative to work_dir, '\' accepted), integrates on `device`, writes dump/ and data/.
 * Returns RRG_OK, or an error (the reference logs and exits 0). */
RRG_API rrg_status rrg_run(const char* work_dir, int device, int precision);
/* The same run continued from <work_dir>/dump/S_{iter:>5d}.bin (and W_{iter:>5d}.bin in wave
 * mode) of an earlier run with the same params.json: masses and softening from the ICs,
 * positions, velocities and time from the dump, the save cadence and dump count replayed up
 * to that time, data/ tables appended to. `rrgsim <work_dir> --resume <iter>`. */
RRG_API rrg_status rrg_run_resume(const char* work_dir, uint64_t iteration, int device,
                                  int precision);

/* ------------------------------------------------------------------------------------------ */
/* Synthetic initial conditions (no counterpart in the reference, which ships no generator)   */
/* ------------------------------------------------------------------------------------------ */

/* Plummer sphere, G = 1: Aarseth, Henon & Wielen (1974) radii truncated at r_max, isotropic
 * velocities from the distribution function by rejection. Deterministic in seed. */
RRG_API rrg_status rrg_generate_plummer(uint64_t seed, int64_t n, double total_mass,
                                        double scale_radius, double r_max, double* pos,
                                        double* vel);
/* Exponential disk: surface density ~ exp(-R/Rd) truncated at r_max, sech^2(z/z0) vertical
 * profile truncated at |z| < z_max, circular speed from the enclosed disk mass (spherical
 * approximation) plus extra_mass_inside(R) (pass bulge_mass/bulge_a for a Plummer bulge,
 * 0 for none), plus Gaussian dispersion sigma = disp_frac * v_c per component. */
RRG_API rrg_status rrg_generate_exp_disk(uint64_t seed, int64_t n, double disk_mass,
                                         double scale_length, double z0, double r_max,
                                         double z_max, double disp_frac, double bulge_mass,
                                         double bulge_a, double* pos, double* vel);

/* ------------------------------------------------------------------------------------------ */
/* Batched ensemble of independent galaxies (no counterpart in the reference, which runs one  */
/* simulation per process). Each galaxy follows the N-body strategy                           */
/* (solver/app/include/rrgsim_integration_nbody.cuh:50-56) in FP32, all galaxies in one      */
/* persistent force launch over a device work-list, steps replayed as CUDA graphs.            */
/* ------------------------------------------------------------------------------------------ */
typedef struct rrg_ensemble rrg_ensemble;

/* counts[g] particles per galaxy; pos/vel (total x 3), mass (total) concatenated galaxy after
 * galaxy; soft2_per_galaxy[g] is each galaxy's softening squared. autotune_tiles != 0 times
 * the tile variants and j-chunk sizes on this work-list and keeps the fastest. Computes the
 * initial accelerations. */
RRG_API rrg_status rrg_ensemble_create(int device, int ngal, const int64_t* counts,
                                       const double* pos, const double* vel,
                                       const double* mass, const double* soft2_per_galaxy,
                                       double dt, int autotune_tiles, rrg_ensemble** out);
RRG_API rrg_status rrg_ensemble_destroy(rrg_ensemble* e);
RRG_API rrg_status rrg_ensemble_set_stream(rrg_ensemble* e, void* stream);
/* nsteps leapfrog steps of every galaxy (batched, graph-replayed). */
RRG_API rrg_status rrg_ensemble_step(rrg_ensemble* e, int nsteps);
/* The same steps with one unbatched force launch per galaxy (comparison baseline). plain != 0
 * launches in the reference's shape (acceleration_kernel_blocked_, nbody.cu:19-65 and
 * :200-213: one i-particle per thread, 256-thread blocks, no j-split); plain == 0 uses the
 * library's single-galaxy kernel without a j-split. */
RRG_API rrg_status rrg_ensemble_step_sequential(rrg_ensemble* e, int nsteps, int plain);
RRG_API rrg_status rrg_ensemble_synchronize(rrg_ensemble* e);
/* Downloads the state (any pointer may be NULL), in the order given at creation. */
RRG_API rrg_status rrg_ensemble_get(rrg_ensemble* e, double* pos, double* vel, double* acc);
/* The tile variant (1: 2 i-particles per thread, 2: 4), j-chunk, work items and the timed
 * force evaluation the autotuner settled on. */
RRG_API rrg_status rrg_ensemble_tuning(const rrg_ensemble* e, int* variant, int* jchunk,
                                       int* num_items, double* force_ms);

/* ------------------------------------------------------------------------------------------ */
/* Differentiable direct N-body (no counterpart in the reference). Hand-written adjoint of    */
/* the leapfrog of nbody.cu:122-181 with the direct-sum force of nbody.cu:19-65: one         */
/* vector-Jacobian product of the force per step, states recomputed from checkpoints.        */
/* ------------------------------------------------------------------------------------------ */
typedef struct rrg_adjoint rrg_adjoint;

/* precision RRG_PREC_FP32 or RRG_PREC_FP64; soft2 has n entries; checkpoint_every K > 0
 * keeps (x, v) every K steps and recomputes the steps between (K <= 0: keep only the start). */
RRG_API rrg_status rrg_adjoint_create(int device, int precision, int64_t n, double dt,
                                      int nsteps, int checkpoint_every, const double* soft2,
                                      rrg_adjoint** out);
RRG_API rrg_status rrg_adjoint_destroy(rrg_adjoint* a);
/* Device memory in the object's precision: x0[i] = (x, y, z, m), v0[i] = (vx, vy, vz, 0), both
 * n x 4. Runs nsteps leapfrog steps; x_out / v_out (may be NULL) receive the final state.
 * Checks on the device whether all masses are equal (equal masses take faster kernels in
 * FP32), which waits for the stream once per call. */
RRG_API rrg_status rrg_adjoint_forward(rrg_adjoint* a, const void* x0, const void* v0,
                                       void* x_out, void* v_out, void* stream);
/* Cotangents of the final (x, v) (n x 4, w ignored; NULL = zero) in; out gx[i] = (dL/dx,
 * dL/dy, dL/dz, dL/dm) and gv[i] = (dL/dvx, dL/dvy, dL/dvz, 0) of the initial state. */
RRG_API rrg_status rrg_adjoint_backward(rrg_adjoint* a, const void* gx_final,
                                        const void* gv_final, void* gx_out, void* gv_out,
                                        void* stream);
/* enabled = 0: backward skips dL/dm (the w slot of gx_out is then 0), which saves about a sixth
 * of the FP32 pair work. Default 1. */
RRG_API rrg_status rrg_adjoint_set_mass_gradient(rrg_adjoint* a, int enabled);
/* Differentiable particle-mesh steps (periodic wave potential): hand-written adjoint of the
 * RectWave step (solver/app/include/rrgsim_integration_rect.cuh:99-112) — trilinear-gather
 * adjoint of the CIC deposit, CIC-scatter adjoint of the interpolation, transposed gradient,
 * time-reversed wave stencil. The initial potential is a fixed input. */
typedef struct rrg_pm_adjoint rrg_pm_adjoint;
/* m_max: the largest particle mass (sets the deposit's fixed-point scale); total_mass_for_rho:
 * the mass whose mean density the periodic source subtracts (1 in the reference's precalc);
 * wave->iterations substeps per step with wave->dt, wave_speed and diss_base. */
RRG_API rrg_status rrg_pm_adjoint_create(int device, int precision, int64_t n, double m_max,
                                         const rrg_grid_info* grid, const rrg_wave_params* wave,
                                         double total_mass_for_rho, double dt, int nsteps,
                                         int checkpoint_every, rrg_pm_adjoint** out);
RRG_API rrg_status rrg_pm_adjoint_destroy(rrg_pm_adjoint* a);
/* x0 (x, y, z, m), v0: n x 4 device memory of the precision; phi_prev0 / phi_cur0: the two
 * wave levels (nx^3) the steps start from. */
RRG_API rrg_status rrg_pm_adjoint_forward(rrg_pm_adjoint* a, const void* x0, const void* v0,
                                          const void* phi_prev0, const void* phi_cur0,
                                          void* x_out, void* v_out, void* phi_out, void* stream);
RRG_API rrg_status rrg_pm_adjoint_backward(rrg_pm_adjoint* a, const void* gx_final,
                                           const void* gv_final, void* gx_out, void* gv_out,
                                           void* stream);

/* Vector-Jacobian product of the direct-sum acceleration in FP32 or FP64 on caller memory:
 * posm/lam/out n x 4 of that precision (out[i] = (dx, dy, dz, dm)); hsoft NULL = uniform. */
RRG_API rrg_status rrg_dev_direct_vjp(const void* posm, const void* hsoft, double uniform_hsoft,
                                      int64_t n, const void* lam, void* out, int precision,
                                      void* stream);

/* ------------------------------------------------------------------------------------------ */
/* Raw device kernels on caller memory (used by the Python/torch binding)                     */
/* ------------------------------------------------------------------------------------------ */

/* Direct-sum forces, FP32: posm is n x float4 (x, y, z, m); hsoft is n floats holding
 * soft2/2 (NULL = every particle uses uniform_hsoft); out is n x float4 (ax, ay, az, phi)
 * with phi = -sum m_j / sqrt(r^2 + (s_i + s_j)/2) (self term kept). precision is
 * RRG_PREC_FP32 or RRG_PREC_MIXED (MIXED also reads poslo, n x float4 low parts; may be NULL
 * otherwise). Same arithmetic as rrg_nbody_acceleration. */
RRG_API rrg_status rrg_dev_direct_forces_f32(const void* posm, const void* poslo,
                                             const void* hsoft, float uniform_hsoft, int64_t n,
                                             void* out, int precision, void* stream);

/* Vector-Jacobian product of the direct-sum acceleration a(x, m), FP32: lam is n x float4
 * (cotangent of ax, ay, az; w ignored); out is n x float4 (d<lam,a>/dx, dy, dz, dm). */
RRG_API rrg_status rrg_dev_direct_vjp_f32(const void* posm, const void* hsoft,
                                          float uniform_hsoft, int64_t n, const void* lam,
                                          void* out, void* stream);

/* Same result as rrg_dev_direct_forces_f32 in RRG_PREC_FP32, for callers that cannot let a
 * library allocate device memory (a host that reserves its whole memory budget up front, a
 * plugin inside another framework's allocator, a loop that must not risk an allocation). It
 * allocates nothing: its scratch is one fixed 4 MiB device array per GPU, held until the
 * process exits. n must be in [1, 1048576]; larger n is RRG_ERR_INVALID. The first call on a
 * device looks up that array's device address (make it before any stream capture); the
 * address is kept for the life of the process, so it does not survive a reset of the device
 * (cudaDeviceReset, or a primary-context reset by the host framework). All calls share the
 * array: calls that overlap on the GPU race. No counterpart in the reference. */
RRG_API rrg_status rrg_dev_direct_forces_f32_noalloc(const void* posm, const void* hsoft,
                                                     float uniform_hsoft, int64_t n, void* out,
                                                     void* stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* RRG_H */
