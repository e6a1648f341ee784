// Launchers of the sm_100a kernels (implemented in direct.cu, pm.cu, wave_solve.cu,
// integrate.cu).
#pragma once

#include "common.cuh"

namespace rrg {

// ---------------------------------------------------------------------------------------------
// Direct-sum gravity (nbody.cu:19-114): a_i = sum_j m_j d_ij (|d_ij|^2 + h_i + h_j)^-3/2,
// phi_i = -sum_j m_j (|d_ij|^2 + h_i + h_j)^-1/2, h = soft2 / 2, self pair included.
// ---------------------------------------------------------------------------------------------
enum DirectEpiMode {
    EPI_STORE = 0,            // acc[i] = a (and pot[i] = phi when requested)
    EPI_CORRECT = 1,          // v = (u + dt a) / 2 -> vel; acc[i] = a
    EPI_CORRECT_PREDICT = 2,  // v as above, then u' = v + (v + dt a), x' = x + dt/2 u' -> pos_out
                              // (v and a stored as well where vel / acc are non-null)
};

struct DirectEpi {
    int mode = EPI_STORE;
    double dt = 0.0;
    void* acc = nullptr;      // V4<R> (ax, ay, az, 0)
    void* pot = nullptr;      // R[n]
    void* vel = nullptr;      // V4<R>
    void* u = nullptr;        // V4<R> holding v + v* (the reference's vel + vel_predicted_)
    void* pos_out = nullptr;  // V4<R> (x, y, z, m) after the drift
    void* lo_out = nullptr;   // V4<float> low parts after the drift (MIXED)
};

struct DirectLaunch {
    int prec = RRG_PREC_FP32;
    const void* posm = nullptr;   // V4<R> (x, y, z, m); for MIXED the hi parts
    const void* poslo = nullptr;  // V4<float> (MIXED only)
    const void* hsoft = nullptr;  // R[n] soft2/2, or nullptr -> uniform_hsoft
    double uniform_hsoft = 0.0;
    double uniform_mass = -1.0;   // >= 0: every particle has this mass (FP32 paired kernels)
    int64_t n = 0;
    bool want_pot = false;
    DirectEpi epi;
    int splits = 0;               // j-splits; 0 = choose
    int variant = 0;              // FP32 kernel variant (direct.cu); 0 = choose
    void* scratch = nullptr;      // partial sums when splits > 1
    size_t scratch_bytes = 0;
    cudaStream_t stream = nullptr;
};

int direct_choose_splits(int prec, int64_t n, int sms);
size_t direct_scratch_bytes(int prec, int64_t n, int splits);
void launch_direct(const DirectLaunch& L);

// VJP of a(x, m) (FP32): out_i = (d<lam,a>/dx_i, d<lam,a>/dm_i).
void launch_direct_vjp_f32(const void* posm, const void* hsoft, float uniform_hsoft, int64_t n,
                           const void* lam, void* out, cudaStream_t stream);

// ---------------------------------------------------------------------------------------------
// Leapfrog pieces (nbody.cu:122-181) on the context state.
// ---------------------------------------------------------------------------------------------
// v* = v + dt a; u = v + v*; x += dt/2 u   (MIXED: x kept as hi + lo)
void launch_predict(int prec, int64_t n, void* posm, void* poslo, const void* vel,
                    const void* acc, void* u, double dt, cudaStream_t s);
// v = (u + dt a) / 2
void launch_correct(int prec, int64_t n, void* vel, const void* acc, const void* u, double dt,
                    cudaStream_t s);

// FP64 reductions of the state (calc_conservation, nbody.cu:246-291; centre of mass,
// nbody.cu:293-439). out[0..11] = Ek2 (sum m v^2), Ep2 (sum m phi), P[3], L[3], and with com
// also M, Mx[3] (else 0), summed in double-double, so independent of the particles' memory order.
// partial holds nblocks x 12 x 2 doubles.
void launch_conservation(int prec, int64_t n, const void* posm, const void* poslo,
                         const void* vel, const void* pot, double* partial, int nblocks,
                         double* out, cudaStream_t s, bool com);
int conservation_blocks(int64_t n);
// The second stage alone, over value-major records (the fused particle pass's PM_SUMS: value k
// of block b at partial[(k nblocks + b) 2], nvals values): out[0..11], values from nvals on 0.
void launch_conservation_finish_value_major(const double* partial, int nblocks, int nvals,
                                            double* out, cudaStream_t s);

// Checks of an upload of particles (rrg_load_particles) on the device. Offending indices are
// stored as 0xffffffff - i under an atomic maximum, so 0 means none and the lowest i wins.
struct LoadCheck {
    unsigned int bad_pv, bad_mass, bad_soft;  // non-finite position / velocity; mass or soft2
                                              // negative or not finite
    unsigned int mass_varies, soft_varies;    // some mass (soft2) differs from the first
    unsigned int pad;
    unsigned long long mass_max_bits;         // bit pattern of the largest valid mass (>= 0)
};
// chk must be zeroed before the launch.
void launch_check_state(int64_t n, const double* pos3, const double* vel3, const double* mass,
                        const double* soft2, LoadCheck* chk, int sms, cudaStream_t s);

// Conversions between the host FP64 AoS layout and the device state.
void launch_pack_state(int prec, int64_t n, const double* pos3, const double* vel3,
                       const double* mass, const double* soft2, void* posm, void* poslo,
                       void* vel, void* hsoft, cudaStream_t s);
// Gathers back into the original order through id (sorted slot -> original index).
void launch_unpack_state(int prec, int64_t n, const int32_t* id, const void* posm,
                         const void* poslo, const void* vel, const void* acc, const void* pot,
                         double* pos3, double* vel3, double* acc3, double* grav,
                         cudaStream_t s);

// ---------------------------------------------------------------------------------------------
// Particle-mesh (rm_p2mesh.cu, rm_mesh2p.cu, wave.cu)
// ---------------------------------------------------------------------------------------------
struct WaveCoef {
    // per-cell coefficients are uniform unless the dissipation layer is on
    double K_MAIN, K_ACTUAL, K_OLD, K_F;
    // for the non-uniform case (layer dissipation or non-periodic boundaries)
    double C, DT, DX, diss_base, diss_extra, sim_l, domain_min;
    int bc_type;
    int keep_layer;
    double rho_mean;
    double bc_mass, com[3], r_min;
};

// CIC deposit into int64 fixed point (rm_p2mesh.cu:176-236): cell += round(m w 2^S).
void launch_cic_deposit(int prec, int64_t n, const void* posm, const void* poslo,
                        const GridDev& g, int shift_s, unsigned long long* grid,
                        cudaStream_t s);
// Wave source from the fixed-point mass: src = 4 pi G (m 2^-S / dx^3 - rho_mean) [* K_F when
// uniform], stored in R; optionally zeroes the fixed-point grid.
void launch_wave_source(int prec, int nx, const unsigned long long* mgrid, int shift_s,
                        double dx, double rho_mean, double scale, void* src, bool zero_grid,
                        cudaStream_t s);
// One damped-wave substep (wave.cu:106-193): phi_old_inout <- phi_new.
// If maxbits != nullptr also folds max|phi_new - phi| and max|phi_new| into maxbits[0..1].
void launch_wave_step(int prec, int nx, const void* phi, void* phi_old_inout, const void* src,
                      const WaveCoef& c, unsigned long long* maxbits, cudaStream_t s);
// One adjoint substep of the PM adjoint on a periodic FP32 grid with the float4 stencil:
// P <- km L6(C) + ka C + beta P, F += kf C. False (nothing launched) where the rows do not tile.
bool launch_wave_adjoint_step(int nx, const float* C, float* P, float* F, double km, double ka,
                              double beta, double kf, cudaStream_t s);
// a = -grad phi on the grid (rm_p2mesh.cu:238-290): acc4[c] = (ax, ay, az, phi[c]).
void launch_gradient(int prec, int nx, double dx, const void* phi, void* acc4, cudaStream_t s);
// One damped-wave update of four x-cells (wave_diss_iteration, wave.cu:106-193, periodic box,
// uniform coefficients): new = K_MAIN (sum of the six neighbours) + K_ACTUAL phi + K_OLD phi_old
// + K_F src. Every rounding is written out, so every FP32 kernel that uses it (one launch per
// substep, the persistent solves, whichever block computes a cell) gives the same bits.
// (The float4 form with two cells per paired FP32 instruction gives the same bits and measured
// 90.8 against 91.1 us per persistent solve: the substeps are not bound by the stencil's issue.)
__device__ __forceinline__ float wave_cell(float a, float b, float ym, float yp, float zm,
                                           float zp, float c, float po, float s, float km,
                                           float ka, float ko, float kf) {
    const float nb = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(a, b), ym), yp), zm), zp);
    return __fmaf_rn(s, kf, __fmaf_rn(po, ko, __fmaf_rn(c, ka, __fmul_rn(nb, km))));
}
// c: four cells of a row; lft / rgt: the cells left of c.x and right of c.w
__device__ __forceinline__ float4 wave_cell4(const float4 c, float lft, float rgt,
                                             const float4 ym, const float4 yp, const float4 zm,
                                             const float4 zp, const float4 po, const float4 s,
                                             float km, float ka, float ko, float kf) {
    float4 o;
    o.x = wave_cell(lft, c.y, ym.x, yp.x, zm.x, zp.x, c.x, po.x, s.x, km, ka, ko, kf);
    o.y = wave_cell(c.x, c.z, ym.y, yp.y, zm.y, zp.y, c.y, po.y, s.y, km, ka, ko, kf);
    o.z = wave_cell(c.y, c.w, ym.z, yp.z, zm.z, zp.z, c.z, po.z, s.z, km, ka, ko, kf);
    o.w = wave_cell(c.z, rgt, ym.w, yp.w, zm.w, zp.w, c.w, po.w, s.w, km, ka, ko, kf);
    return o;
}

// The wave source of one cell from its fixed-point deposit q (mass = q 2^-S): 4 pi G (rho -
// rho_sub) with G = 1 and the reference's PI (co_info_structs.h:7), before any rounding to FP32.
// Every FP32 source in the library is this value rounded.
__device__ __forceinline__ double wave_source_value(unsigned long long q, double inv_scale,
                                                    double inv_dx3, double rho_sub) {
    const double mass = __dmul_rn(static_cast<double>(q), inv_scale);
    const double rho = __dsub_rn(__dmul_rn(mass, inv_dx3), rho_sub);
    return __dmul_rn(4.0 * 3.14159265358979, rho);
}

// Incremental form of one solve (the fused steps' FP32 / MIXED solves on periodic grids). With
// the levels written phi = phi0 + d, phi0 the current level at the start of the solve, every
// substep becomes
//   d_new = K_MAIN L6(d) + K_ACTUAL d + K_OLD d_old + g,
//   g     = K_F src + K_MAIN L6(phi0) + (K_ACTUAL + K_OLD - 1) phi0,
// (L6: the sum of the six neighbours), starting from d = 0 and d_old = phi_prev - phi0. g is
// evaluated once per solve in FP64 and rounded once; the increments are small next to phi, so
// the FP32 rounding of 20 substeps lands on them instead of on phi, and phi0 + d is rounded once
// at the end. kao = K_ACTUAL + K_OLD - 1. Arguments: src the FP64 source, l / r the x
// neighbours, ym .. zp the y and z neighbours, c the cell, all of phi0.
__device__ __forceinline__ float wave_inc_source(double src, float l, float r, float ym,
                                                 float yp, float zm, float zp, float c,
                                                 double kf, double km, double kao) {
    double l6 = __dadd_rn(static_cast<double>(l), static_cast<double>(r));
    l6 = __dadd_rn(l6, static_cast<double>(ym));
    l6 = __dadd_rn(l6, static_cast<double>(yp));
    l6 = __dadd_rn(l6, static_cast<double>(zm));
    l6 = __dadd_rn(l6, static_cast<double>(zp));
    return __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(kf, src), __dmul_rn(km, l6)),
                                       __dmul_rn(kao, static_cast<double>(c))));
}
// four x-cells of a row (as wave_cell4); s: their FP64 sources
__device__ __forceinline__ float4 wave_inc_source4(const double s[4], const float4 c, float lft,
                                                   float rgt, const float4 ym, const float4 yp,
                                                   const float4 zm, const float4 zp, double kf,
                                                   double km, double kao) {
    float4 o;
    o.x = wave_inc_source(s[0], lft, c.y, ym.x, yp.x, zm.x, zp.x, c.x, kf, km, kao);
    o.y = wave_inc_source(s[1], c.x, c.z, ym.y, yp.y, zm.y, zp.y, c.y, kf, km, kao);
    o.z = wave_inc_source(s[2], c.y, c.w, ym.z, yp.z, zm.z, zp.z, c.z, kf, km, kao);
    o.w = wave_inc_source(s[3], c.z, rgt, ym.w, yp.w, zm.w, zp.w, c.w, kf, km, kao);
    return o;
}
__device__ __forceinline__ float4 f4_sub(const float4 a, const float4 b) {
    return make_float4(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z),
                       __fsub_rn(a.w, b.w));
}
__device__ __forceinline__ float4 f4_add(const float4 a, const float4 b) {
    return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z),
                       __fadd_rn(a.w, b.w));
}

// The incremental solve's preparation, one streaming launch over the grid: g and
// d_old = phi_prev - phi0 per cell, d = 0 (unless null), the plain FP32 source into src (unless
// null), the next deposit target mg_zero cleared (unless null). One launch per substep (where
// the persistent kernels do not apply, and RRG_WAVE_PERSIST=0) then runs launch_wave_step on
// (d, d_old, g) with K_F = 1, and finish writes phi0 + d_final and
// phi0 + d_before into fin and prv (either may be phi0 itself). FP32 grids, periodic, uniform.
void launch_wave_inc_prep(int nx, const unsigned long long* mg, unsigned long long* mg_zero,
                          int shift_s, double dx, double rho_sub, const float* phi0,
                          const float* phi_prev, const WaveCoef& w, float* g, float* d,
                          float* d_old, float* src, cudaStream_t s);
void launch_wave_inc_finish(int nx, const float* phi0, const float* d_fin, const float* d_prv,
                            float* fin, float* prv, cudaStream_t s);

// One PM step's whole FP32 wave solve in one persistent cooperative kernel (wave_solve.cu):
// source from the deposit mg (mg_zero cleared), `iterations` substeps over the levels phi0 /
// phi1 (cur: which holds the current level; the result lands in phi[cur ^ (iterations & 1)],
// the level before it in the other), then the gradient into acc4 (skipped when acc4 is null);
// the source is also stored to src unless src is null. The substeps run in the incremental form
// (wave_inc_source): the same bits as launch_wave_inc_prep + launch_wave_step x iterations +
// launch_wave_inc_finish + launch_gradient.
// Periodic box without an absorbing layer only. sync: wave_solve_sync_bytes(nx) of device memory, zeroed
// before the first use and kept between calls; its word at byte 65532 becomes non-zero when a
// wait between blocks ran out (the step is then invalid and the memory must be zeroed again).
// Returns false, launching nothing, where it does not apply (nx, residency,
// RRG_WAVE_PERSIST=0).
bool wave_solve_applicable(int nx);
size_t wave_solve_sync_bytes(int nx);
constexpr size_t kWaveSyncErrOffset = 65532;
bool launch_wave_solve(int nx, int iterations, float* phi0, float* phi1, int cur,
                       const unsigned long long* mg, unsigned long long* mg_zero, int shift_s,
                       double dx, double rho_sub, const WaveCoef& w, float* src, float4* acc4,
                       unsigned int* sync, size_t sync_bytes, cudaStream_t s);
// Trilinear gather of acc4 to particles (rm_mesh2p.cu:48-114).
void launch_interp(int prec, int64_t n, const void* posm, const void* poslo, const GridDev& g,
                   const void* acc4, void* acc, cudaStream_t s);
// NGP potential lookup (rm_mesh2p.cu:29-38 with the cell of rm_p2mesh.cu:25-49).
void launch_ngp_phi(int prec, int64_t n, const void* posm, const void* poslo, const GridDev& g,
                    const void* phi, void* pot, cudaStream_t s);

// NGP averages of particle potential / acceleration per cell (rm_p2mesh.cu:142-174):
// count[] (nx^3 ints, zeroed by the caller) receives the cell counts; phi_grid (R, nx^3) and
// acc4_grid (V4<R>, nx^3) must be zeroed by the caller; either may be nullptr.
void launch_ngp_project(int prec, int64_t n, const void* posm, const void* poslo,
                        const GridDev& g, int* count, const void* pot, const void* acc,
                        void* phi_grid, void* acc4_grid, cudaStream_t s);

// Fused particle pass of the wave strategy: optional [trilinear interp + correct] then
// optional [predict + CIC deposit]. PM_SUMS (with PM_INTERP_CORRECT | PM_WRITE_SYNC) also
// writes each block's double-double sums of the 8 conservation terms of the synced state into
// `partial` (value-major: [8][blocks of 256 particles][2]), for
// launch_conservation_finish_value_major.
enum PmMode { PM_INTERP_CORRECT = 1, PM_PREDICT_DEPOSIT = 2, PM_WRITE_SYNC = 4, PM_SUMS = 8 };
struct PmParticleArgs {
    int prec;
    int64_t n;
    void* posm;
    void* poslo;
    void* vel;    // V4<R> synced velocity (read when !INTERP_CORRECT, written when WRITE_SYNC)
    void* acc;    // V4<R> synced acceleration (same rules)
    void* u;      // V4<R>
    const void* acc4;  // grid field
    GridDev g;
    int shift_s;
    unsigned long long* mgrid;
    double dt;
    void* pos_out = nullptr;  // predicted positions (and MIXED low parts) go here when set,
    void* lo_out = nullptr;   // else they overwrite posm / poslo in place
    const void* pot = nullptr;  // R[n] particle potential, read by PM_SUMS
    double* partial = nullptr;  // PM_SUMS block records
};
constexpr int kPmThreads = 256;
constexpr int kPmSumValues = 8;  // values per PM_SUMS block record
void launch_pm_particles(const PmParticleArgs& a, int mode, cudaStream_t s);

// Counting sort by CIC base cell (sort.cu): keys + histogram, exclusive scan, destinations,
// then one scatter per particle array.
size_t sort_scan_temp_bytes(int64_t ncells);
void launch_cell_keys(int prec, int64_t n, const void* posm, const void* poslo,
                      const GridDev& g, uint32_t* keys, uint32_t* counts, cudaStream_t s);
void launch_scan_counts(const uint32_t* counts, uint32_t* offsets, int64_t ncells, void* temp,
                        size_t temp_bytes, cudaStream_t s);
void launch_sort_dest(int64_t n, const uint32_t* keys, const uint32_t* offsets,
                      uint32_t* cursor, uint32_t* dest, cudaStream_t s);
void launch_permute(int64_t n, size_t elem_bytes, const uint32_t* dest, const void* in,
                    void* out, cudaStream_t s);
void launch_iota(int64_t n, int32_t* id, cudaStream_t s);

}  // namespace rrg
