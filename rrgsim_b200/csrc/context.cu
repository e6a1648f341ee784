// C-ABI implementation: contexts, operators, integration strategies, CUDA graphs.
//
// Device state of a context (R = float for FP32/MIXED, double for FP64):
//   posm[2]  V4<R>  (x, y, z, m)        two buffers: the fused direct step reads one, writes
//                                         the other
//   poslo[2] V4<float> low parts of x, y, z (MIXED)
//   vel, acc V4<R>  synced velocity / acceleration (x_n, v_n, a_n)
//   u        V4<R>  v + v* of the last predict (the reference's vel + vel_predicted_)
//   pot      R      potential per particle
//   hsoft    R      soft2 / 2 per particle (absent when all particles share one softening)
// Grid (nx^3 cells, AT(x,y,z) = x + y nx + z nx^2):
//   mg[2]    uint64 fixed-point cell mass (the last deposit is mg[mg_cur]; the other is zero
//                   outside a calc_steps call)
//   src      R      4 pi G (rho - rho_mean)
//   phi[2]   R      potential at the current and the previous wave level
//   acc4     V4<R>  (ax, ay, az, phi) after calc_acceleration_field
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "host_io.h"
#include "kernels.cuh"

namespace rrg {

static std::atomic<uint64_t> g_launches{0};
static thread_local bool t_capturing = false;
static thread_local std::string t_error;

void set_thread_error(const std::string& msg) { t_error = msg; }

void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
bool capturing_now() { return t_capturing; }
void set_capturing(bool on) { t_capturing = on; }

int num_sms(int device) {
    int v = 0;
    RRG_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    return v;
}

// Minimal RAII device buffer.
struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() { release(); }
    bool owned = true;  // false: a view into another buffer (not freed here)
    void release() {
        if (p && owned) cudaFree(p);
        p = nullptr;
        bytes = 0;
        owned = true;
    }
    void view(void* q, size_t b) {
        release();
        p = q;
        bytes = b;
        owned = false;
    }
    void alloc(size_t b) {
        if (b == bytes && p) return;
        release();
        if (b == 0) return;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            p = nullptr;
            (void)cudaGetLastError();
            throw Error(RRG_ERR_NOMEM, "cudaMalloc(" + std::to_string(b) + " B) failed: " +
                                           cudaGetErrorString(e));
        }
        bytes = b;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

struct GraphExec {
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
    // the context's grid flags after the recorded steps, set again at every replay
    bool src_dirty = false, src_valid = true, wave_solve_used = false;
};

}  // namespace rrg

using namespace rrg;

struct rrg_ctx {
    int device = 0;
    int prec = RRG_PREC_FP32;
    size_t rsz = 4;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    int sms = 148;

    // particles
    int64_t n = 0;
    Buf posm[2], poslo[2], vel, acc, u, pot, hsoft, id;
    int cur = 0;
    bool soft_uniform = true;
    double uniform_hsoft = 0.0;
    double mass_max = 0.0;
    double uniform_mass = -1.0;  // >= 0 when every particle has this mass
    bool sorted = false;
    int splits = 1;
    Buf scratch;

    // grid
    bool has_grid = false;
    rrg_grid_info grid{};
    GridDev gdev{};
    Buf arena;                       // holds mg[0], mg[1], phi[0], phi[1] (views)
    cudaStream_t l2_stream = nullptr;  // the stream that carries the arena's L2 window
    Buf mg[2], src, phi[2], acc4;
    int mg_cur = 0;
    int phi_cur = 0;
    bool src_dirty = true;
    bool src_valid = true;           // false: the fused steps left the source grid unwritten
    int shift_s = 0;
    bool has_wave = false;
    rrg_wave_params wave{};
    int bc_type = RRG_BC_ZERO_DIRICHLET;
    double bc_mass = 0.0, com[3] = {0, 0, 0}, r_min = 0.0, rho_mean = 0.0;
    int keep_layer = 0;
    Buf maxbits;
    Buf wsync;                       // the persistent solve's progress counters and error word
    bool wave_solve_used = false;

    // reductions / transfers
    Buf red_partial, red_out, dl, chk;
    double* host_red = nullptr;
    // rrg_set_step_sums: the last particle pass of each fused chunk also writes the conservation
    // sums' block records (step_partial); sums_ready says they describe the current state (every
    // entry point clears it unless it leaves the state as it found it)
    bool step_sums = false;
    mutable bool sums_ready = false;
    Buf step_partial;

    // solver
    bool solver_ready = false;
    bool wave_mode = false;
    rrg_sim_params sim{};
    double time = 0.0;
    uint64_t iter = 0;
    int sort_interval = -1;          // -1: the strategy's default (64 steps in wave mode)
    // Wave mode, between calc_steps calls: the last particle pass also predicted the next step,
    // so posm[1 - cur] (and poslo[1 - cur]) hold x_{n+1}, u its v + v*, and mg[1 - mg_cur] its
    // deposit. The synced state (x_n, v_n, a_n, deposit of x_n) is untouched; the next
    // calc_steps adopts the prediction instead of predicting again.
    bool pending = false;
    int64_t steps_since_sort = INT64_MAX / 2;
    Buf sort_keys, sort_dest, sort_counts, sort_offsets, sort_cursor, sort_temp, sort_stage;
    size_t sort_temp_bytes = 0;
    std::map<std::tuple<int, int, int, int, bool, bool>, GraphExec> graphs;

    ~rrg_ctx() {
        for (auto& kv : graphs)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (host_red) cudaFreeHost(host_red);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    void* P() const { return posm[cur].p; }
    void* L() const { return prec == RRG_PREC_MIXED ? poslo[cur].p : nullptr; }
    const void* H() const { return soft_uniform ? nullptr : hsoft.p; }
};

namespace {

#define RRG_ENTRY(ctx, ...)                                                                   \
    try {                                                                                     \
        RRG_REQUIRE((ctx) != nullptr, RRG_ERR_INVALID, "null context");                       \
        RRG_CUDA(cudaSetDevice((ctx)->device));                                               \
        const bool entry_sums_ready = (ctx)->sums_ready;                                      \
        (ctx)->sums_ready = false;                                                            \
        (void)entry_sums_ready;                                                               \
        __VA_ARGS__;                                                                          \
        return RRG_OK;                                                                        \
    } catch (const Error& e) {                                                                \
        if (ctx) (ctx)->err = e.what();                                                       \
        t_error = e.what();                                                                   \
        return e.code;                                                                        \
    } catch (const std::exception& e) {                                                       \
        if (ctx) (ctx)->err = e.what();                                                       \
        t_error = e.what();                                                                   \
        return RRG_ERR_INVALID;                                                               \
    }

void require_particles(rrg_ctx* c) {
    RRG_REQUIRE(c->n > 0, RRG_ERR_STATE, "no particles loaded");
}
void require_grid(rrg_ctx* c) {
    RRG_REQUIRE(c->has_grid, RRG_ERR_STATE, "no grid: call rrg_init_grid first");
}

size_t v4b(const rrg_ctx* c) { return 4 * c->rsz; }

void ensure_download(rrg_ctx* c, size_t bytes) {
    if (c->dl.bytes < bytes) c->dl.alloc(bytes);
}

WaveCoef wave_coef(const rrg_ctx* c) {
    WaveCoef w{};
    const double C = c->wave.wave_speed, DT = c->wave.dt, DX = c->grid.dx;
    const double diss = c->wave.diss_base;
    const double Q = diss * C * DT * 0.5;
    const double W = 1 + Q;
    const double K = C * C * DT * DT / (DX * DX);
    w.K_MAIN = K / W;
    w.K_F = -C * C * DT * DT / W;
    w.K_ACTUAL = 2 * (1 - 3 * K) / W;
    w.K_OLD = (Q - 1) / W;
    w.C = C;
    w.DT = DT;
    w.DX = DX;
    w.diss_base = c->wave.diss_base;
    w.diss_extra = c->wave.diss_extra;
    w.sim_l = c->grid.sim_l;
    w.domain_min = c->grid.domain_min;
    w.bc_type = c->bc_type;
    w.keep_layer = c->keep_layer;
    w.rho_mean = c->rho_mean;
    w.bc_mass = c->bc_mass;
    w.com[0] = c->com[0];
    w.com[1] = c->com[1];
    w.com[2] = c->com[2];
    w.r_min = c->r_min;
    return w;
}

// ---------------------------------------------------------------------------------------------
// building blocks shared by the operator calls and the fused solver steps
// ---------------------------------------------------------------------------------------------
void direct(rrg_ctx* c, bool want_pot, const DirectEpi& epi) {
    DirectLaunch L;
    L.prec = c->prec;
    L.posm = c->P();
    L.poslo = c->L();
    L.hsoft = c->H();
    L.uniform_hsoft = c->uniform_hsoft;
    L.uniform_mass = c->uniform_mass;
    L.n = c->n;
    L.want_pot = want_pot;
    L.epi = epi;
    L.splits = c->splits;
    L.scratch = c->scratch.p;
    L.scratch_bytes = c->scratch.bytes;
    L.stream = c->stream;
    launch_direct(L);
}

void wave_source(rrg_ctx* c, bool zero_other) {
    // reads mg[mg_cur]; clears mg[1 - mg_cur] when asked (the next deposit target)
    const double rho_sub = (c->bc_type == RRG_BC_PERIODIC) ? c->rho_mean : 0.0;
    launch_wave_source(c->prec, c->grid.nx, c->mg[c->mg_cur].as<unsigned long long>(),
                       c->shift_s, c->grid.dx, rho_sub, 1.0, c->src.p, false, c->stream);
    if (zero_other) {
        // cleared with a memset node: the source kernel must not touch the deposit it reads
        RRG_CUDA(cudaMemsetAsync(c->mg[1 - c->mg_cur].p, 0, c->mg[1 - c->mg_cur].bytes,
                                 c->stream));
    }
    c->src_dirty = false;
    c->src_valid = true;
}

void wave_substep(rrg_ctx* c, const WaveCoef& w, unsigned long long* maxbits) {
    launch_wave_step(c->prec, c->grid.nx, c->phi[c->phi_cur].p, c->phi[1 - c->phi_cur].p,
                     c->src.p, w, maxbits, c->stream);
    c->phi_cur = 1 - c->phi_cur;
}

void gradient(rrg_ctx* c) {
    launch_gradient(c->prec, c->grid.nx, c->grid.dx, c->phi[c->phi_cur].p, c->acc4.p, c->stream);
}

// the gradient of level phi[k] into acc4
void gradient_after(rrg_ctx* c, int k) {
    launch_gradient(c->prec, c->grid.nx, c->grid.dx, c->phi[k].p, c->acc4.p, c->stream);
}

// One solve of the fused steps (source, `iterations` substeps, gradient) on FP32 / MIXED
// periodic grids without an absorbing layer, in the incremental form (wave_inc_source): each
// solve advances increments over its first level, so the FP32 roundings of the substeps land on
// the increments, and the level is rounded once at the end. It runs as the persistent kernel
// where that applies (32, 64, 128 cells, all blocks resident at once, RRG_WAVE_PERSIST not 0),
// else one launch per substep with the same bits: a preparation (the increments' source and
// first increment, the plain source when store_src, the next deposit target cleared), the
// substeps, the finish (the levels in full) and the gradient; the increments and their source
// live in the field buffer (acc4: 4 floats per cell), which the gradient rewrites at the end.
// False (nothing launched) on other grids and precisions: the caller launches the reference's
// full-level form (wave_source + wave_substep x iterations + gradient).
bool solve_step_fused(rrg_ctx* c, const WaveCoef& w, int iterations, bool store_src) {
    if (c->prec == RRG_PREC_FP64 || c->bc_type != RRG_BC_PERIODIC || c->keep_layer) return false;
    const int nx = c->grid.nx;
    if (launch_wave_solve(nx, iterations, c->phi[0].as<float>(), c->phi[1].as<float>(),
                          c->phi_cur, c->mg[c->mg_cur].as<unsigned long long>(),
                          c->mg[1 - c->mg_cur].as<unsigned long long>(), c->shift_s, c->grid.dx,
                          c->rho_mean, w, store_src ? c->src.as<float>() : nullptr,
                          c->acc4.as<float4>(), c->wsync.as<unsigned int>(), c->wsync.bytes,
                          c->stream)) {
        c->wave_solve_used = true;
    } else {
        const size_t nc = static_cast<size_t>(nx) * nx * nx;
        float* a4 = c->acc4.as<float>();
        float* d[2] = {a4, a4 + nc};
        float* g = a4 + 2 * nc;
        float* phi0 = c->phi[c->phi_cur].as<float>();
        launch_wave_inc_prep(nx, c->mg[c->mg_cur].as<unsigned long long>(),
                             c->mg[1 - c->mg_cur].as<unsigned long long>(), c->shift_s,
                             c->grid.dx, c->rho_mean, phi0, c->phi[1 - c->phi_cur].as<float>(),
                             w, g, d[0], d[1], store_src ? c->src.as<float>() : nullptr,
                             c->stream);
        WaveCoef wi = w;
        wi.K_F = 1.0;
        int cur = 0;
        for (int k = 0; k < iterations; ++k) {
            launch_wave_step(c->prec, nx, d[cur], d[1 - cur], g, wi, nullptr, c->stream);
            cur = 1 - cur;
        }
        // final level into phi[phi_cur ^ (iterations & 1)], the one before into the other
        const int fin = c->phi_cur ^ (iterations & 1);
        launch_wave_inc_finish(nx, phi0, d[cur], d[1 - cur], c->phi[fin].as<float>(),
                               c->phi[1 - fin].as<float>(), c->stream);
        gradient_after(c, fin);
    }
    if (iterations % 2 == 1) c->phi_cur = 1 - c->phi_cur;
    c->src_dirty = false;
    c->src_valid = store_src;
    return true;
}

// The deposit grids and the wave levels (the arena, 48 MB at 128^3) stay resident in L2 across
// a step's kernels: a persisting access-policy window over the arena on the context stream, with
// the process's persisting L2 set-aside sized to it (at most what the device allows; 79 MB of
// the 126 MB on B200). Every step reads and rewrites all four grids, and the particle data and
// the field would otherwise push them out between the particle pass and the solve: 121.8
// against 125.4 us per PM step on 128^3 (the field in the window too: 123.8). Best effort: a
// device or configuration without persisting L2 runs without it. RRG_L2_PERSIST=0 turns it off.
bool l2_persist_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("RRG_L2_PERSIST");
        return !(e && std::atoi(e) == 0);
    }();
    return on;
}

void set_l2_window(cudaStream_t s, const void* base, size_t bytes, float hit) {
    cudaStreamAttrValue v{};
    v.accessPolicyWindow.base_ptr = const_cast<void*>(base);
    v.accessPolicyWindow.num_bytes = bytes;
    v.accessPolicyWindow.hitRatio = hit;
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    if (cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &v) != cudaSuccess)
        (void)cudaGetLastError();
}

void apply_l2_window(rrg_ctx* c) {
    if (!l2_persist_enabled() || !c->arena.p) return;
    int maxp = 0, maxw = 0;
    if (cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, c->device) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, c->device) !=
            cudaSuccess) {
        (void)cudaGetLastError();
        return;
    }
    if (maxp <= 0 || maxw <= 0) return;
    const size_t want = std::min(c->arena.bytes, static_cast<size_t>(maxp));
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
        (void)cudaGetLastError();
        return;
    }
    const size_t win = std::min(c->arena.bytes, static_cast<size_t>(maxw));
    set_l2_window(c->stream, c->arena.p, win,
                  std::min(1.0f, static_cast<float>(want) / static_cast<float>(win)));
    c->l2_stream = c->stream;
}

// the window off again on a stream that the context leaves (a caller's stream keeps no trace)
void clear_l2_window(rrg_ctx* c) {
    if (c->l2_stream == nullptr) return;
    set_l2_window(c->l2_stream, nullptr, 0, 0.f);
    c->l2_stream = nullptr;
}

// After a synchronisation: the persistent solve's error word is set when a wait between its
// thread blocks ran out, which leaves the steps since the last check invalid.
void check_wave_solve(rrg_ctx* c) {
    if (!c->wave_solve_used || !c->wsync.p) return;
    unsigned int e = 0;
    RRG_CUDA(cudaMemcpyAsync(&e, c->wsync.as<char>() + kWaveSyncErrOffset, 4,
                             cudaMemcpyDeviceToHost, c->stream));
    RRG_CUDA(cudaStreamSynchronize(c->stream));
    if (e != 0) {
        RRG_CUDA(cudaMemsetAsync(c->wsync.p, 0, c->wsync.bytes, c->stream));
        RRG_CUDA(cudaStreamSynchronize(c->stream));
        throw Error(RRG_ERR_CUDA,
                    "wave solve: a wait between thread blocks timed out; the state is invalid");
    }
}

PmParticleArgs pm_args(rrg_ctx* c, int deposit_target) {
    PmParticleArgs a;
    a.prec = c->prec;
    a.n = c->n;
    a.posm = c->P();
    a.poslo = c->L();
    a.vel = c->vel.p;
    a.acc = c->acc.p;
    a.u = c->u.p;
    a.acc4 = c->acc4.p;
    a.g = c->gdev;
    a.shift_s = c->shift_s;
    a.mgrid = deposit_target >= 0 ? c->mg[deposit_target].as<unsigned long long>() : nullptr;
    a.dt = c->sim.dt_dynamics;
    a.pot = c->pot.p;
    a.partial = c->step_partial.as<double>();
    return a;
}

// Block records of the particle pass's conservation sums (PM_SUMS): 8 double-doubles per
// block of kPmThreads particles.
int step_sum_blocks(const rrg_ctx* c) { return div_up(c->n, kPmThreads); }
void alloc_step_partial(rrg_ctx* c) {
    if (c->step_sums && c->n > 0)
        c->step_partial.alloc(static_cast<size_t>(step_sum_blocks(c)) * kPmSumValues * 2 *
                              sizeof(double));
}

// Steady-state controlled relaxation (solve_wave_equation, wave.cu:230-297). Host-synchronous
// only on check iterations.
int solve_wave(rrg_ctx* c, int max_iterations, double* last_rel) {
    require_grid(c);
    RRG_REQUIRE(c->has_wave, RRG_ERR_STATE, "no wave parameters");
    RRG_REQUIRE(max_iterations >= 0, RRG_ERR_INVALID, "max_iterations must be >= 0");
    RRG_REQUIRE(c->wave.steady_check_step > 0, RRG_ERR_INVALID,
                "steady_check_step must be positive (used as a modulus, wave.cu:275)");
    if (c->src_dirty || !c->src_valid) wave_source(c, false);
    const WaveCoef w = wave_coef(c);
    int hold = 0;
    double rel = -1.0;
    int it = 0;
    for (int iter = 0; iter < max_iterations; ++iter) {
        const bool check = iter && (iter % c->wave.steady_check_step == 0);
        if (check) RRG_CUDA(cudaMemsetAsync(c->maxbits.p, 0, 16, c->stream));
        wave_substep(c, w, check ? c->maxbits.as<unsigned long long>() : nullptr);
        it = iter + 1;
        if (check) {
            unsigned long long bits[2];
            RRG_CUDA(cudaMemcpyAsync(bits, c->maxbits.p, 16, cudaMemcpyDeviceToHost, c->stream));
            RRG_CUDA(cudaStreamSynchronize(c->stream));
            double d, a;
            std::memcpy(&d, &bits[0], 8);
            std::memcpy(&a, &bits[1], 8);
            rel = d / (a + 1e-30);
            if (rel < c->wave.tolerance) ++hold;
            else hold = 0;
            if (hold >= c->wave.steady_hold_steps) break;
        }
    }
    if (last_rel) *last_rel = rel;
    return it;
}

void drop_graphs(rrg_ctx* c) {
    for (auto& kv : c->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    c->graphs.clear();
}

void set_periodic(rrg_ctx* c, double total_mass, int keep_layer) {
    drop_graphs(c);
    const double L = c->grid.nx * c->grid.dx;
    c->bc_type = RRG_BC_PERIODIC;
    c->bc_mass = total_mass;
    c->rho_mean = total_mass / (L * L * L);
    c->keep_layer = keep_layer ? 1 : 0;
    c->src_dirty = true;
}

void deposit_operator(rrg_ctx* c) {
    RRG_CUDA(cudaMemsetAsync(c->mg[c->mg_cur].p, 0, c->mg[c->mg_cur].bytes, c->stream));
    launch_cic_deposit(c->prec, c->n, c->P(), c->L(), c->gdev, c->shift_s,
                       c->mg[c->mg_cur].as<unsigned long long>(), c->stream);
    c->src_dirty = true;
}

// Discards a pending prediction (any call that changes the state); clears its deposit so that
// mg[1 - mg_cur] is zero again.
void drop_pending(rrg_ctx* c) {
    if (!c->pending) return;
    RRG_CUDA(cudaMemsetAsync(c->mg[1 - c->mg_cur].p, 0, c->mg[1 - c->mg_cur].bytes, c->stream));
    c->pending = false;
}

// Counting sort of the synced particle state by CIC base cell. Every array is scattered into a
// staging buffer and copied back in place, so buffer addresses (and recorded graphs) stay.
void sort_particles(rrg_ctx* c) {
    require_particles(c);
    require_grid(c);
    const int64_t n = c->n;
    const int64_t nc = static_cast<int64_t>(c->grid.nx) * c->grid.nx * c->grid.nx;
    if (c->sort_keys.bytes < 4 * static_cast<size_t>(n)) {
        c->sort_keys.alloc(4 * n);
        c->sort_dest.alloc(4 * n);
        c->sort_stage.alloc(v4b(c) * n);
    }
    if (c->sort_counts.bytes < 4 * static_cast<size_t>(nc + 1)) {
        c->sort_counts.alloc(4 * (nc + 1));
        c->sort_offsets.alloc(4 * (nc + 1));
        c->sort_cursor.alloc(4 * (nc + 1));
        c->sort_temp_bytes = sort_scan_temp_bytes(nc);
        c->sort_temp.alloc(std::max<size_t>(c->sort_temp_bytes, 256));
    }
    if (!c->sorted) {
        c->id.alloc(4 * n);
        launch_iota(n, c->id.as<int32_t>(), c->stream);
    }
    // with a pending prediction the predicted positions give the keys (they are deposited
    // next) and the prediction is permuted; its deposit grid is a sum over particles and does
    // not depend on their order
    const bool keep = c->pending;
    const int other = 1 - c->cur;
    const bool mixed = c->prec == RRG_PREC_MIXED;
    RRG_CUDA(cudaMemsetAsync(c->sort_counts.p, 0, c->sort_counts.bytes, c->stream));
    RRG_CUDA(cudaMemsetAsync(c->sort_cursor.p, 0, c->sort_cursor.bytes, c->stream));
    launch_cell_keys(c->prec, n, keep ? c->posm[other].p : c->P(),
                     mixed ? (keep ? c->poslo[other].p : c->L()) : nullptr, c->gdev,
                     c->sort_keys.as<uint32_t>(), c->sort_counts.as<uint32_t>(), c->stream);
    launch_scan_counts(c->sort_counts.as<uint32_t>(), c->sort_offsets.as<uint32_t>(), nc,
                       c->sort_temp.p, c->sort_temp_bytes, c->stream);
    launch_sort_dest(n, c->sort_keys.as<uint32_t>(), c->sort_offsets.as<uint32_t>(),
                     c->sort_cursor.as<uint32_t>(), c->sort_dest.as<uint32_t>(), c->stream);
    auto permute = [&](void* arr, size_t elem) {
        if (!arr) return;
        launch_permute(n, elem, c->sort_dest.as<uint32_t>(), arr, c->sort_stage.p, c->stream);
        RRG_CUDA(cudaMemcpyAsync(arr, c->sort_stage.p, elem * n, cudaMemcpyDeviceToDevice,
                                 c->stream));
    };
    if (keep) {
        // the prediction and its u; the synced positions, velocities and accelerations are
        // not read again: the sort is always followed by a chunk that adopts the prediction,
        // and its last pass rewrites all three before the call returns
        permute(c->posm[other].p, v4b(c));
        if (mixed) permute(c->poslo[other].p, sizeof(V4<float>));
        permute(c->u.p, v4b(c));
    } else {
        permute(c->P(), v4b(c));
        if (mixed) permute(c->L(), sizeof(V4<float>));
        permute(c->vel.p, v4b(c));
        permute(c->acc.p, v4b(c));
    }
    permute(c->pot.p, c->rsz);
    if (!c->soft_uniform) permute(c->hsoft.p, c->rsz);
    permute(c->id.p, 4);
    c->sorted = true;
    c->steps_since_sort = 0;
}

// ---------------------------------------------------------------------------------------------
// Fused solver steps
// ---------------------------------------------------------------------------------------------
// N-body: [predict] then nsteps direct-sum launches whose epilogue is correct (+ next predict).
void record_nbody_steps(rrg_ctx* c, int nsteps) {
    launch_predict(c->prec, c->n, c->P(), c->L(), c->vel.p, c->acc.p, c->u.p,
                   c->sim.dt_dynamics, c->stream);
    for (int s = 0; s < nsteps; ++s) {
        DirectEpi e;
        e.dt = c->sim.dt_dynamics;
        e.u = c->u.p;
        if (s + 1 < nsteps) {
            e.mode = EPI_CORRECT_PREDICT;
            e.pos_out = c->posm[1 - c->cur].p;
            e.lo_out = c->prec == RRG_PREC_MIXED ? c->poslo[1 - c->cur].p : nullptr;
            direct(c, false, e);
            c->cur = 1 - c->cur;
        } else {
            e.mode = EPI_CORRECT;
            e.vel = c->vel.p;
            e.acc = c->acc.p;
            direct(c, false, e);
        }
    }
}

// Wave: [predict + deposit] then per step: source, `iterations` substeps, gradient, fused
// particle pass (interp + correct [+ next predict + deposit]).
// prologue = false: the chunk starts from an adopted prediction (see rrg_ctx::pending). The
// last pass corrects and syncs step n and already predicts step n + 1 into the other position
// buffer and the zeroed deposit grid, leaving the synced state in place.
void record_wave_steps(rrg_ctx* c, int nsteps, bool prologue) {
    const WaveCoef w = wave_coef(c);
    if (prologue) {
        const int t = 1 - c->mg_cur;  // known zero
        PmParticleArgs a = pm_args(c, t);
        launch_pm_particles(a, PM_PREDICT_DEPOSIT, c->stream);
        c->mg_cur = t;
    }
    for (int s = 0; s < nsteps; ++s) {
        if (!solve_step_fused(c, w, c->wave.iterations, false)) {
            wave_source(c, true);
            for (int k = 0; k < c->wave.iterations; ++k) wave_substep(c, w, nullptr);
            gradient(c);
        }
        if (s + 1 < nsteps) {
            const int t = 1 - c->mg_cur;
            PmParticleArgs a = pm_args(c, t);
            launch_pm_particles(a, PM_INTERP_CORRECT | PM_PREDICT_DEPOSIT, c->stream);
            c->mg_cur = t;
        } else {
            PmParticleArgs a = pm_args(c, 1 - c->mg_cur);  // zeroed by this step's source pass
            a.pos_out = c->posm[1 - c->cur].p;
            a.lo_out = c->prec == RRG_PREC_MIXED ? c->poslo[1 - c->cur].p : nullptr;
            launch_pm_particles(a, PM_INTERP_CORRECT | PM_WRITE_SYNC | PM_PREDICT_DEPOSIT |
                                       (c->step_sums ? PM_SUMS : 0),
                                c->stream);
        }
    }
}

// Wave strategy step by step with steady checks inside each solve (used when a check falls
// inside the per-step iterations, so control flow depends on device data).
void wave_steps_unfused(rrg_ctx* c, int nsteps) {
    for (int s = 0; s < nsteps; ++s) {
        launch_predict(c->prec, c->n, c->P(), c->L(), c->vel.p, c->acc.p, c->u.p,
                       c->sim.dt_dynamics, c->stream);
        deposit_operator(c);
        solve_wave(c, c->wave.iterations, nullptr);
        gradient(c);
        launch_interp(c->prec, c->n, c->P(), c->L(), c->gdev, c->acc4.p, c->acc.p, c->stream);
        launch_correct(c->prec, c->n, c->vel.p, c->acc.p, c->u.p, c->sim.dt_dynamics, c->stream);
    }
}

// The executable graph of the next `nsteps`-step chunk, recorded and instantiated on first use
// (recording launches nothing); advances the buffer roles and flags as running the chunk does.
GraphExec& chunk_graph(rrg_ctx* c, int nsteps) {
    bool prologue = true;
    if (c->wave_mode && c->pending) {
        // adopt the prediction the previous chunk left
        c->cur = 1 - c->cur;
        c->mg_cur = 1 - c->mg_cur;
        c->pending = false;
        prologue = false;
    }
    const bool sums = c->wave_mode && c->step_sums;
    const auto key = std::make_tuple(nsteps, c->cur, c->mg_cur, c->phi_cur, prologue, sums);
    auto it = c->graphs.find(key);
    const int cur0 = c->cur, mg0 = c->mg_cur, phi0 = c->phi_cur;
    if (it == c->graphs.end()) {
        cudaGraph_t g = nullptr;
        RRG_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        set_capturing(true);
        try {
            if (c->wave_mode) record_wave_steps(c, nsteps, prologue);
            else record_nbody_steps(c, nsteps);
        } catch (...) {
            set_capturing(false);
            cudaStreamEndCapture(c->stream, &g);
            if (g) cudaGraphDestroy(g);
            c->cur = cur0;
            c->mg_cur = mg0;
            c->phi_cur = phi0;
            throw;
        }
        set_capturing(false);
        RRG_CUDA(cudaStreamEndCapture(c->stream, &g));
        GraphExec ge;
        size_t nn = 0;
        RRG_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
        std::vector<cudaGraphNode_t> nodes(nn);
        if (nn) RRG_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
        for (auto& nd : nodes) {
            cudaGraphNodeType t;
            RRG_CUDA(cudaGraphNodeGetType(nd, &t));
            if (t == cudaGraphNodeTypeKernel) ++ge.kernels;
        }
        cudaError_t e = cudaGraphInstantiate(&ge.exec, g, 0);
        cudaGraphDestroy(g);
        RRG_CUDA(e);
        ge.src_dirty = c->src_dirty;
        ge.src_valid = c->src_valid;
        ge.wave_solve_used = c->wave_solve_used;
        it = c->graphs.emplace(key, ge).first;
    } else {
        // replaying: advance the buffer roles exactly as recording did
        if (c->wave_mode) {
            const int flips = prologue ? nsteps : nsteps - 1;
            c->mg_cur = (flips % 2 == 1) ? 1 - mg0 : mg0;
            if (c->wave.iterations % 2 == 1) c->phi_cur = (nsteps % 2 == 1) ? 1 - phi0 : phi0;
            c->src_dirty = it->second.src_dirty;
            c->src_valid = it->second.src_valid;
            c->wave_solve_used = c->wave_solve_used || it->second.wave_solve_used;
        } else {
            c->cur = ((nsteps - 1) % 2 == 1) ? 1 - cur0 : cur0;
        }
    }
    if (c->wave_mode) c->pending = true;
    return it->second;
}

void run_graph(rrg_ctx* c, int nsteps) {
    GraphExec& ge = chunk_graph(c, nsteps);
    RRG_CUDA(cudaGraphLaunch(ge.exec, c->stream));
    count_launches(ge.kernels);
}

// The chunks a calc_steps(nsteps) call runs, in order: at most 64 steps each, and in wave mode
// cut at every re-sort of the particles by cell (every `interval` steps). `each(chunk, sort)`
// is called per chunk; `sort` is true when the particles are re-sorted before it.
template <typename F>
void for_each_chunk(rrg_ctx* c, int nsteps, int64_t& steps_since_sort, F each) {
    // long runs are recorded once per chunk length and replayed; in wave mode the particles are
    // re-sorted by cell between chunks every sort_interval steps (64: the deposit sorts a
    // disordered warp by cell itself, so only the gathers' locality degrades between sorts;
    // 16, 32 and 64 steps measured 125.7, 124.0 and 123.2 us per step on the 2^20-particle
    // disk)
    const int interval = c->wave_mode ? (c->sort_interval < 0 ? 64 : c->sort_interval) : 0;
    int left = nsteps;
    while (left > 0) {
        int chunk = std::min(left, 64);
        bool sort = false;
        if (interval > 0) {
            if (steps_since_sort >= interval) {
                sort = true;
                steps_since_sort = 0;
            }
            chunk = static_cast<int>(std::min<int64_t>(chunk, interval - steps_since_sort));
        }
        each(chunk, sort);
        steps_since_sort += chunk;
        left -= chunk;
    }
}

bool checks_inside_steps(const rrg_ctx* c) {
    return c->wave_mode && c->wave.steady_check_step > 0 &&
           c->wave.iterations > c->wave.steady_check_step;
}

}  // namespace

// ================================================================================================
// C ABI
// ================================================================================================
extern "C" {

RRG_API const char* rrg_version(void) { return "rrgsim-b200 0.1 (sm_100a)"; }

RRG_API const char* rrg_last_error(const rrg_ctx* ctx) {
    if (ctx) return ctx->err.c_str();
    return t_error.c_str();
}

RRG_API uint64_t rrg_kernel_launch_count(void) { return g_launches.load(); }

RRG_API rrg_status rrg_create(int device, int precision, rrg_ctx** out) {
    try {
        RRG_REQUIRE(out != nullptr, RRG_ERR_INVALID, "rrg_create: out is NULL");
        RRG_REQUIRE(precision >= RRG_PREC_FP32 && precision <= RRG_PREC_FP64, RRG_ERR_INVALID,
                    "rrg_create: unknown precision");
        int count = 0;
        RRG_CUDA(cudaGetDeviceCount(&count));
        RRG_REQUIRE(device >= 0 && device < count, RRG_ERR_INVALID,
                    "rrg_create: no CUDA device " + std::to_string(device));
        RRG_CUDA(cudaSetDevice(device));
        auto* c = new rrg_ctx();
        c->device = device;
        c->prec = precision;
        c->rsz = precision == RRG_PREC_FP64 ? 8 : 4;
        c->sms = num_sms(device);
        cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete c;
            RRG_CUDA(e);
        }
        c->stream = c->own_stream;
        e = cudaMallocHost(&c->host_red, 16 * sizeof(double));
        if (e != cudaSuccess) {
            delete c;
            RRG_CUDA(e);
        }
        *out = c;
        return RRG_OK;
    } catch (const Error& e) {
        t_error = e.what();
        return e.code;
    }
}

RRG_API rrg_status rrg_destroy(rrg_ctx* ctx) {
    if (!ctx) return RRG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->l2_stream != ctx->own_stream) clear_l2_window(ctx);
    delete ctx;
    return RRG_OK;
}

RRG_API rrg_status rrg_set_stream(rrg_ctx* ctx, void* stream) {
    RRG_ENTRY(ctx, {
        clear_l2_window(ctx);
        ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
        apply_l2_window(ctx);
    })
}

RRG_API rrg_status rrg_synchronize(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
        check_wave_solve(ctx);
        ctx->sums_ready = entry_sums_ready;
    })
}

RRG_API rrg_status rrg_load_particles(rrg_ctx* ctx, int64_t n, const double* pos,
                                      const double* vel, const double* mass,
                                      const double* soft2) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        RRG_REQUIRE(n >= 1, RRG_ERR_INVALID, "rrg_load_particles: n must be >= 1");
        RRG_REQUIRE(n < (int64_t(1) << 31), RRG_ERR_INVALID,
                    "rrg_load_particles: n must be < 2^31");
        RRG_REQUIRE(pos && vel && mass && soft2, RRG_ERR_INVALID,
                    "rrg_load_particles: NULL array");

        // stage the FP64 host arrays on the device and check them there: the lowest index of
        // a non-finite position or velocity, of a mass or softening that is negative or not
        // finite; the largest mass; whether masses and softenings are uniform. Nothing of the
        // context changes before the checks pass.
        const size_t stage = static_cast<size_t>(n) * 8 * sizeof(double);
        ensure_download(ctx, stage);
        double* d = ctx->dl.as<double>();
        RRG_CUDA(cudaMemcpyAsync(d, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice,
                                 ctx->stream));
        RRG_CUDA(cudaMemcpyAsync(d + 3 * n, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice,
                                 ctx->stream));
        RRG_CUDA(cudaMemcpyAsync(d + 6 * n, mass, n * sizeof(double), cudaMemcpyHostToDevice,
                                 ctx->stream));
        RRG_CUDA(cudaMemcpyAsync(d + 7 * n, soft2, n * sizeof(double), cudaMemcpyHostToDevice,
                                 ctx->stream));
        if (!ctx->chk.p) ctx->chk.alloc(sizeof(LoadCheck));
        RRG_CUDA(cudaMemsetAsync(ctx->chk.p, 0, sizeof(LoadCheck), ctx->stream));
        launch_check_state(n, d, d + 3 * n, d + 6 * n, d + 7 * n, ctx->chk.as<LoadCheck>(),
                           ctx->sms, ctx->stream);
        LoadCheck ck;
        RRG_CUDA(cudaMemcpyAsync(ctx->host_red, ctx->chk.p, sizeof(LoadCheck),
                                 cudaMemcpyDeviceToHost, ctx->stream));
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
        std::memcpy(&ck, ctx->host_red, sizeof(LoadCheck));
        {
            // the lowest offending particle; at one particle positions and velocities are
            // reported first, then the mass, then the softening
            const int64_t none = INT64_MAX;
            const auto at = [&](unsigned int v) {
                return v ? static_cast<int64_t>(0xffffffffu - v) : none;
            };
            const int64_t ipv = at(ck.bad_pv), im = at(ck.bad_mass), is = at(ck.bad_soft);
            const int64_t first = std::min(ipv, std::min(im, is));
            RRG_REQUIRE(first == none || first != ipv, RRG_ERR_INVALID,
                        "rrg_load_particles: non-finite position/velocity at particle " +
                            std::to_string(first));
            RRG_REQUIRE(first == none || first != im, RRG_ERR_INVALID,
                        "rrg_load_particles: bad mass at particle " + std::to_string(first));
            RRG_REQUIRE(first == none, RRG_ERR_INVALID,
                        "rrg_load_particles: bad soft2 at particle " + std::to_string(first));
        }
        double mmax = 0.0;
        std::memcpy(&mmax, &ck.mass_max_bits, sizeof(double));
        const bool uniform = ck.soft_varies == 0;
        const bool umass = ck.mass_varies == 0;
        ctx->uniform_mass = umass ? mass[0] : -1.0;

        // recorded graphs stay valid when the new particles reuse every buffer and launch value
        const auto layout = [&]() {
            return std::vector<const void*>{ctx->posm[0].p, ctx->posm[1].p, ctx->poslo[0].p,
                                            ctx->poslo[1].p, ctx->vel.p, ctx->acc.p, ctx->u.p,
                                            ctx->pot.p, ctx->hsoft.p, ctx->scratch.p,
                                            ctx->step_partial.p};
        };
        const auto before = layout();
        const int64_t n_before = ctx->n;
        const int shift_before = ctx->shift_s;
        const double hsoft_before = ctx->uniform_hsoft;
        const bool uniform_before = ctx->soft_uniform;

        ctx->n = n;
        ctx->cur = 0;
        ctx->soft_uniform = uniform;
        ctx->uniform_hsoft = 0.5 * soft2[0];
        ctx->mass_max = mmax;
        ctx->sorted = false;
        ctx->time = 0.0;
        ctx->iter = 0;
        {
            int e = 0;
            std::frexp(mmax > 0 ? mmax : 1.0, &e);
            ctx->shift_s = 26 - e;  // m_max 2^S <= 2^26: one contribution fits 27 bits
        }
        const size_t vb = v4b(ctx) * n;
        ctx->posm[0].alloc(vb);
        ctx->posm[1].alloc(vb);
        if (ctx->prec == RRG_PREC_MIXED) {
            ctx->poslo[0].alloc(sizeof(V4<float>) * n);
            ctx->poslo[1].alloc(sizeof(V4<float>) * n);
        } else {
            ctx->poslo[0].release();
            ctx->poslo[1].release();
        }
        ctx->vel.alloc(vb);
        ctx->acc.alloc(vb);
        ctx->u.alloc(vb);
        ctx->pot.alloc(ctx->rsz * n);
        if (!uniform) ctx->hsoft.alloc(ctx->rsz * n);
        else ctx->hsoft.release();
        // the id buffer stays allocated (its contents are rewritten by the first sort); freeing
        // and allocating it again on every reload cost the host two synchronous driver calls
        ctx->steps_since_sort = INT64_MAX / 2;
        ctx->splits = direct_choose_splits(ctx->prec, n, ctx->sms);
        const size_t sb = direct_scratch_bytes(ctx->prec, n, ctx->splits);
        if (sb) ctx->scratch.alloc(sb);
        const int rb = conservation_blocks(n);
        ctx->red_partial.alloc(static_cast<size_t>(rb) * 12 * 2 * sizeof(double));  // (hi, lo)
        ctx->red_out.alloc(16 * sizeof(double));
        alloc_step_partial(ctx);
        if (layout() != before || n != n_before || ctx->shift_s != shift_before ||
            ctx->uniform_hsoft != hsoft_before || ctx->soft_uniform != uniform_before)
            drop_graphs(ctx);

        // pack the staged arrays into the device state
        launch_pack_state(ctx->prec, n, d, d + 3 * n, d + 6 * n, d + 7 * n, ctx->posm[0].p,
                          ctx->poslo[0].p, ctx->vel.p, uniform ? nullptr : ctx->hsoft.p,
                          ctx->stream);
        RRG_CUDA(cudaMemsetAsync(ctx->acc.p, 0, vb, ctx->stream));
        RRG_CUDA(cudaMemsetAsync(ctx->u.p, 0, vb, ctx->stream));
        RRG_CUDA(cudaMemsetAsync(ctx->pot.p, 0, ctx->rsz * n, ctx->stream));
        // no wait: the host arrays were copied before the checks, and the packing kernels run
        // ahead of whatever the caller enqueues next on the context stream
    })
}

RRG_API int64_t rrg_num_particles(const rrg_ctx* ctx) { return ctx ? ctx->n : 0; }

RRG_API rrg_status rrg_get_particles(rrg_ctx* ctx, double* pos, double* vel, double* acc,
                                     double* grav) {
    RRG_ENTRY(ctx, {
        require_particles(ctx);
        const int64_t n = ctx->n;
        ensure_download(ctx, static_cast<size_t>(n) * 10 * sizeof(double));
        double* d = ctx->dl.as<double>();
        launch_unpack_state(ctx->prec, n, ctx->sorted ? ctx->id.as<int32_t>() : nullptr,
                            ctx->P(), ctx->L(), ctx->vel.p, ctx->acc.p, ctx->pot.p,
                            pos ? d : nullptr, vel ? d + 3 * n : nullptr,
                            acc ? d + 6 * n : nullptr, grav ? d + 9 * n : nullptr, ctx->stream);
        if (pos) RRG_CUDA(cudaMemcpyAsync(pos, d, 3 * n * 8, cudaMemcpyDeviceToHost, ctx->stream));
        if (vel)
            RRG_CUDA(cudaMemcpyAsync(vel, d + 3 * n, 3 * n * 8, cudaMemcpyDeviceToHost, ctx->stream));
        if (acc)
            RRG_CUDA(cudaMemcpyAsync(acc, d + 6 * n, 3 * n * 8, cudaMemcpyDeviceToHost, ctx->stream));
        if (grav)
            RRG_CUDA(cudaMemcpyAsync(grav, d + 9 * n, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
        check_wave_solve(ctx);
        ctx->sums_ready = entry_sums_ready;
    })
}

RRG_API rrg_status rrg_get_time(const rrg_ctx* ctx, double* time, uint64_t* iter) {
    if (!ctx) return RRG_ERR_INVALID;
    if (time) *time = ctx->time;
    if (iter) *iter = ctx->iter;
    return RRG_OK;
}

RRG_API rrg_status rrg_init_grid(rrg_ctx* ctx, const rrg_grid_info* grid) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        RRG_REQUIRE(grid != nullptr, RRG_ERR_INVALID, "rrg_init_grid: NULL grid");
        RRG_REQUIRE(grid->nx >= 2 && grid->nx <= 1024, RRG_ERR_INVALID,
                    "rrg_init_grid: nx must be in [2, 1024]");
        RRG_REQUIRE(grid->dx > 0 && std::isfinite(grid->dx), RRG_ERR_INVALID,
                    "rrg_init_grid: dx must be positive");
        ctx->grid = *grid;
        ctx->gdev.nx = grid->nx;
        ctx->gdev.dx = grid->dx;
        ctx->gdev.domain_min = grid->domain_min;
        ctx->gdev.inv_dx = 1.0 / grid->dx;
        ctx->gdev.sim_l = grid->sim_l;
        const size_t nc = static_cast<size_t>(grid->nx) * grid->nx * grid->nx;
        {
            // the two deposit grids and the two wave levels in one allocation, so that one L2
            // access-policy window covers them
            const auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
            const size_t bm = up(nc * 8), bp = up(nc * ctx->rsz);
            ctx->arena.alloc(2 * bm + 2 * bp);
            char* base = ctx->arena.as<char>();
            ctx->mg[0].view(base, nc * 8);
            ctx->mg[1].view(base + bm, nc * 8);
            ctx->phi[0].view(base + 2 * bm, nc * ctx->rsz);
            ctx->phi[1].view(base + 2 * bm + bp, nc * ctx->rsz);
        }
        ctx->acc4.alloc(nc * v4b(ctx));
        ctx->src.alloc(nc * ctx->rsz);
        apply_l2_window(ctx);
        ctx->maxbits.alloc(16);
        ctx->wsync.alloc(wave_solve_sync_bytes(grid->nx));
        for (Buf* b : {&ctx->mg[0], &ctx->mg[1], &ctx->src, &ctx->phi[0], &ctx->phi[1],
                       &ctx->acc4, &ctx->maxbits, &ctx->wsync})
            RRG_CUDA(cudaMemsetAsync(b->p, 0, b->bytes, ctx->stream));
        ctx->mg_cur = 0;
        ctx->phi_cur = 0;
        ctx->src_dirty = true;
        ctx->has_grid = true;
        ctx->bc_type = RRG_BC_ZERO_DIRICHLET;
        for (auto& kv : ctx->graphs)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        ctx->graphs.clear();
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
    })
}

RRG_API rrg_status rrg_set_wave_params(rrg_ctx* ctx, const rrg_wave_params* wave) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        RRG_REQUIRE(wave != nullptr, RRG_ERR_INVALID, "rrg_set_wave_params: NULL");
        RRG_REQUIRE(std::isfinite(wave->dt) && wave->dt > 0, RRG_ERR_INVALID,
                    "rrg_set_wave_params: dt must be positive (0.5 dx / (c sqrt 3))");
        RRG_REQUIRE(wave->iterations >= 0 && wave->setup_iterations >= 0, RRG_ERR_INVALID,
                    "rrg_set_wave_params: negative iteration count");
        ctx->wave = *wave;
        ctx->has_wave = true;
        for (auto& kv : ctx->graphs)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        ctx->graphs.clear();
    })
}

RRG_API rrg_status rrg_get_grid(rrg_ctx* ctx, double* mass, double* grav, double* acc) {
    RRG_ENTRY(ctx, {
        require_grid(ctx);
        const size_t nc = static_cast<size_t>(ctx->grid.nx) * ctx->grid.nx * ctx->grid.nx;
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
        if (mass) {
            std::vector<unsigned long long> q(nc);
            RRG_CUDA(cudaMemcpy(q.data(), ctx->mg[ctx->mg_cur].p, nc * 8, cudaMemcpyDeviceToHost));
            const double inv = std::ldexp(1.0, -ctx->shift_s);
            for (size_t i = 0; i < nc; ++i) mass[i] = static_cast<double>(q[i]) * inv;
        }
        if (grav) {
            if (ctx->rsz == 8) {
                RRG_CUDA(cudaMemcpy(grav, ctx->phi[ctx->phi_cur].p, nc * 8, cudaMemcpyDeviceToHost));
            } else {
                std::vector<float> f(nc);
                RRG_CUDA(cudaMemcpy(f.data(), ctx->phi[ctx->phi_cur].p, nc * 4, cudaMemcpyDeviceToHost));
                for (size_t i = 0; i < nc; ++i) grav[i] = f[i];
            }
        }
        if (acc) {
            if (ctx->rsz == 8) {
                std::vector<V4<double>> f(nc);
                RRG_CUDA(cudaMemcpy(f.data(), ctx->acc4.p, nc * 32, cudaMemcpyDeviceToHost));
                for (size_t i = 0; i < nc; ++i) {
                    acc[3 * i] = f[i].x;
                    acc[3 * i + 1] = f[i].y;
                    acc[3 * i + 2] = f[i].z;
                }
            } else {
                std::vector<V4<float>> f(nc);
                RRG_CUDA(cudaMemcpy(f.data(), ctx->acc4.p, nc * 16, cudaMemcpyDeviceToHost));
                for (size_t i = 0; i < nc; ++i) {
                    acc[3 * i] = f[i].x;
                    acc[3 * i + 1] = f[i].y;
                    acc[3 * i + 2] = f[i].z;
                }
            }
        }
        ctx->sums_ready = entry_sums_ready;
    })
}

RRG_API rrg_status rrg_set_grid_potential(rrg_ctx* ctx, const double* grav) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_grid(ctx);
        RRG_REQUIRE(grav != nullptr, RRG_ERR_INVALID, "rrg_set_grid_potential: NULL");
        const size_t nc = static_cast<size_t>(ctx->grid.nx) * ctx->grid.nx * ctx->grid.nx;
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int k = 0; k < 2; ++k) {
            if (ctx->rsz == 8) {
                RRG_CUDA(cudaMemcpy(ctx->phi[k].p, grav, nc * 8, cudaMemcpyHostToDevice));
            } else {
                std::vector<float> f(grav, grav + nc);
                RRG_CUDA(cudaMemcpy(ctx->phi[k].p, f.data(), nc * 4, cudaMemcpyHostToDevice));
            }
        }
    })
}

RRG_API rrg_status rrg_get_deposit_scale(const rrg_ctx* ctx, int32_t* shift_s) {
    if (!ctx || !shift_s) return RRG_ERR_INVALID;
    *shift_s = ctx->shift_s;
    return RRG_OK;
}

// ---------------------------------------------------------------------------------------------
RRG_API rrg_status rrg_predict_step(rrg_ctx* ctx, double dt) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_particles(ctx);
        launch_predict(ctx->prec, ctx->n, ctx->P(), ctx->L(), ctx->vel.p, ctx->acc.p, ctx->u.p,
                       dt, ctx->stream);
    })
}

RRG_API rrg_status rrg_nbody_acceleration(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_particles(ctx);
        DirectEpi e;
        e.mode = EPI_STORE;
        e.acc = ctx->acc.p;
        direct(ctx, false, e);
    })
}

RRG_API rrg_status rrg_nbody_grav(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        require_particles(ctx);
        // potential only: accelerations go to the scratch download buffer and are dropped
        ensure_download(ctx, v4b(ctx) * ctx->n);
        DirectEpi e;
        e.mode = EPI_STORE;
        e.acc = ctx->dl.p;
        e.pot = ctx->pot.p;
        direct(ctx, true, e);
    })
}

RRG_API rrg_status rrg_correct_step(rrg_ctx* ctx, double dt) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_particles(ctx);
        launch_correct(ctx->prec, ctx->n, ctx->vel.p, ctx->acc.p, ctx->u.p, dt, ctx->stream);
    })
}

RRG_API rrg_status rrg_convert_particles_to_grid(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_particles(ctx);
        require_grid(ctx);
        deposit_operator(ctx);
    })
}

RRG_API rrg_status rrg_set_boundary_periodic(rrg_ctx* ctx, double total_mass, int keep_layer) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_grid(ctx);
        set_periodic(ctx, total_mass, keep_layer);
    })
}

RRG_API rrg_status rrg_set_boundary_monopole(rrg_ctx* ctx, double total_mass,
                                             const double center_of_mass[3], int radiative) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_grid(ctx);
        RRG_REQUIRE(center_of_mass != nullptr, RRG_ERR_INVALID, "NULL centre of mass");
        drop_graphs(ctx);
        ctx->bc_type = radiative ? RRG_BC_MONOPOLE_RADIATIVE : RRG_BC_MONOPOLE_DIRICHLET;
        ctx->bc_mass = total_mass;
        for (int k = 0; k < 3; ++k) ctx->com[k] = center_of_mass[k];
        ctx->r_min = 0.5 * ctx->grid.dx;
        ctx->rho_mean = 0.0;
        ctx->keep_layer = 0;
        ctx->src_dirty = true;
    })
}

RRG_API rrg_status rrg_set_boundary_zero(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_grid(ctx);
        drop_graphs(ctx);
        ctx->bc_type = RRG_BC_ZERO_DIRICHLET;
        ctx->rho_mean = 0.0;
        ctx->src_dirty = true;
    })
}

RRG_API rrg_status rrg_solve_wave_equation(rrg_ctx* ctx, int max_iterations,
                                           int* iterations_run, double* last_rel_diff) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        const int it = solve_wave(ctx, max_iterations, last_rel_diff);
        if (iterations_run) *iterations_run = it;
    })
}

RRG_API rrg_status rrg_solve_wave_and_field(rrg_ctx* ctx, int iterations) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_grid(ctx);
        RRG_REQUIRE(ctx->has_wave, RRG_ERR_STATE, "no wave parameters");
        RRG_REQUIRE(iterations >= 1, RRG_ERR_INVALID, "iterations must be >= 1");
        const WaveCoef w = wave_coef(ctx);
        if (!solve_step_fused(ctx, w, iterations, true)) {
            if (ctx->src_dirty || !ctx->src_valid) wave_source(ctx, false);
            for (int k = 0; k < iterations; ++k) wave_substep(ctx, w, nullptr);
            gradient(ctx);
        }
    })
}

RRG_API rrg_status rrg_wave_solve_sync(rrg_ctx* ctx, void** dev_ptr, size_t* bytes) {
    RRG_ENTRY(ctx, {
        require_grid(ctx);
        RRG_REQUIRE(dev_ptr && bytes, RRG_ERR_INVALID, "rrg_wave_solve_sync: NULL");
        *dev_ptr = ctx->wsync.p;
        *bytes = ctx->wsync.bytes;
    })
}

RRG_API rrg_status rrg_calc_acceleration_field(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_grid(ctx);
        gradient(ctx);
    })
}

RRG_API rrg_status rrg_project_grid_acceleration_on_particles(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_particles(ctx);
        require_grid(ctx);
        launch_interp(ctx->prec, ctx->n, ctx->P(), ctx->L(), ctx->gdev, ctx->acc4.p, ctx->acc.p,
                      ctx->stream);
    })
}

RRG_API rrg_status rrg_project_grid_grav_on_particles(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        require_particles(ctx);
        require_grid(ctx);
        launch_ngp_phi(ctx->prec, ctx->n, ctx->P(), ctx->L(), ctx->gdev,
                       ctx->phi[ctx->phi_cur].p, ctx->pot.p, ctx->stream);
    })
}

// The 12 sums of the current state into `out` (device-addressable): from the block records the
// last fused particle pass left when they still describe the state (`ready`), else by a pass
// over the particles.
static void conservation_sums(rrg_ctx* ctx, bool com, bool ready, double* out) {
    if (ready && !com) {
        launch_conservation_finish_value_major(ctx->step_partial.as<double>(),
                                               step_sum_blocks(ctx), kPmSumValues, out,
                                               ctx->stream);
    } else {
        launch_conservation(ctx->prec, ctx->n, ctx->P(), ctx->L(), ctx->vel.p, ctx->pot.p,
                            ctx->red_partial.as<double>(), conservation_blocks(ctx->n), out,
                            ctx->stream, com);
    }
}

static void reduce_state(rrg_ctx* ctx, bool com, bool ready) {
    conservation_sums(ctx, com, ready, ctx->red_out.as<double>());
    RRG_CUDA(cudaMemcpyAsync(ctx->host_red, ctx->red_out.p, 12 * sizeof(double),
                             cudaMemcpyDeviceToHost, ctx->stream));
    RRG_CUDA(cudaStreamSynchronize(ctx->stream));
    check_wave_solve(ctx);
}

RRG_API rrg_status rrg_calc_conservation(rrg_ctx* ctx, rrg_conservation* out) {
    RRG_ENTRY(ctx, {
        require_particles(ctx);
        RRG_REQUIRE(out != nullptr, RRG_ERR_INVALID, "NULL output");
        reduce_state(ctx, false, entry_sums_ready);
        ctx->sums_ready = entry_sums_ready;
        const double* r = ctx->host_red;
        out->time = ctx->time;
        out->Ek = 0.5 * r[0];
        out->Ep = 0.5 * r[1];
        for (int k = 0; k < 3; ++k) {
            out->momentum[k] = r[2 + k];
            out->angular[k] = r[5 + k];
        }
    })
}

RRG_API rrg_status rrg_calc_conservation_async(rrg_ctx* ctx, double* sums) {
    RRG_ENTRY(ctx, {
        require_particles(ctx);
        RRG_REQUIRE(sums != nullptr, RRG_ERR_INVALID, "NULL output");
        // pinned host memory that this device can address takes the sums straight from the
        // finishing kernel: no copy-engine hop between the step's kernels
        double* out = ctx->red_out.as<double>();
        bool direct = false;
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, sums) == cudaSuccess && at.type == cudaMemoryTypeHost &&
            at.devicePointer != nullptr) {
            out = static_cast<double*>(at.devicePointer);
            direct = true;
        } else {
            (void)cudaGetLastError();
        }
        conservation_sums(ctx, false, entry_sums_ready, out);
        if (!direct)
            RRG_CUDA(cudaMemcpyAsync(sums, ctx->red_out.p, 12 * sizeof(double),
                                     cudaMemcpyDeviceToHost, ctx->stream));
        ctx->sums_ready = entry_sums_ready;
    })
}

RRG_API rrg_status rrg_conservation_from_sums(const double* sums, double time,
                                              rrg_conservation* out) {
    if (!sums || !out) return RRG_ERR_INVALID;
    out->time = time;
    out->Ek = 0.5 * sums[0];
    out->Ep = 0.5 * sums[1];
    for (int k = 0; k < 3; ++k) {
        out->momentum[k] = sums[2 + k];
        out->angular[k] = sums[5 + k];
    }
    return RRG_OK;
}

RRG_API rrg_status rrg_calc_mass_center(rrg_ctx* ctx, double center_of_mass[3],
                                        double* total_mass) {
    RRG_ENTRY(ctx, {
        require_particles(ctx);
        reduce_state(ctx, true, false);
        ctx->sums_ready = entry_sums_ready;
        const double* r = ctx->host_red;
        const double M = r[8];
        for (int k = 0; k < 3; ++k)
            if (center_of_mass) center_of_mass[k] = M > 0 ? r[9 + k] / M : 0.0;
        if (total_mass) *total_mass = M;
    })
}

// ---------------------------------------------------------------------------------------------
RRG_API rrg_status rrg_solver_init(rrg_ctx* ctx, const rrg_sim_params* sim) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_particles(ctx);
        RRG_REQUIRE(sim != nullptr, RRG_ERR_INVALID, "NULL sim params");
        RRG_REQUIRE(std::isfinite(sim->dt_dynamics) && sim->dt_dynamics > 0, RRG_ERR_INVALID,
                    "dt_dynamics must be positive");
        ctx->sim = *sim;
        ctx->wave_mode = sim->use_wave_model != 0;
        if (ctx->wave_mode) {
            RRG_REQUIRE(ctx->has_grid, RRG_ERR_STATE,
                        "No grid info for rect wave integration solver");
            RRG_REQUIRE(ctx->has_wave, RRG_ERR_STATE,
                        "No wave params for rect wave integration solver");
        }
        for (auto& kv : ctx->graphs)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        ctx->graphs.clear();
        ctx->solver_ready = true;
    })
}

RRG_API rrg_status rrg_solver_precalc(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        RRG_REQUIRE(ctx->solver_ready, RRG_ERR_STATE, "rrg_solver_init first");
        if (ctx->wave_mode) {
            deposit_operator(ctx);
            set_periodic(ctx, 1.0, 0);  // total mass fixed to 1: rrgsim_integration_rect.cuh:65
            solve_wave(ctx, ctx->wave.setup_iterations, nullptr);
            gradient(ctx);
        } else {
            DirectEpi e;
            e.mode = EPI_STORE;
            e.acc = ctx->acc.p;
            e.pot = ctx->pot.p;
            direct(ctx, true, e);
        }
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
    })
}

// Precalc for a state restored from a snapshot (and, in wave mode, from its wave state): the
// forces come from the restored positions and potential without the setup relaxation, so the
// next step starts where the saved run stood.
RRG_API rrg_status rrg_solver_resume(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        RRG_REQUIRE(ctx->solver_ready, RRG_ERR_STATE, "rrg_solver_init first");
        if (ctx->wave_mode) {
            deposit_operator(ctx);
            set_periodic(ctx, 1.0, 0);  // as precalc: rrgsim_integration_rect.cuh:65
            gradient(ctx);
        } else {
            DirectEpi e;
            e.mode = EPI_STORE;
            e.acc = ctx->acc.p;
            e.pot = ctx->pot.p;
            direct(ctx, true, e);
        }
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
    })
}

namespace {
void copy_level(rrg_ctx* ctx, void* dev, double* host_out, const double* host_in) {
    const size_t nc = static_cast<size_t>(ctx->grid.nx) * ctx->grid.nx * ctx->grid.nx;
    if (ctx->rsz == 8) {
        if (host_out) RRG_CUDA(cudaMemcpy(host_out, dev, nc * 8, cudaMemcpyDeviceToHost));
        else RRG_CUDA(cudaMemcpy(dev, host_in, nc * 8, cudaMemcpyHostToDevice));
    } else {
        std::vector<float> f(nc);
        if (host_out) {
            RRG_CUDA(cudaMemcpy(f.data(), dev, nc * 4, cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < nc; ++i) host_out[i] = f[i];
        } else {
            for (size_t i = 0; i < nc; ++i) f[i] = static_cast<float>(host_in[i]);
            RRG_CUDA(cudaMemcpy(dev, f.data(), nc * 4, cudaMemcpyHostToDevice));
        }
    }
}
}  // namespace

RRG_API rrg_status rrg_get_wave_state(rrg_ctx* ctx, double* phi_cur, double* phi_prev) {
    RRG_ENTRY(ctx, {
        require_grid(ctx);
        RRG_REQUIRE(phi_cur && phi_prev, RRG_ERR_INVALID, "rrg_get_wave_state: NULL");
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
        copy_level(ctx, ctx->phi[ctx->phi_cur].p, phi_cur, nullptr);
        copy_level(ctx, ctx->phi[1 - ctx->phi_cur].p, phi_prev, nullptr);
        ctx->sums_ready = entry_sums_ready;
    })
}

RRG_API rrg_status rrg_set_wave_state(rrg_ctx* ctx, const double* phi_cur,
                                      const double* phi_prev) {
    RRG_ENTRY(ctx, {
        drop_pending(ctx);
        require_grid(ctx);
        RRG_REQUIRE(phi_cur && phi_prev, RRG_ERR_INVALID, "rrg_set_wave_state: NULL");
        RRG_CUDA(cudaStreamSynchronize(ctx->stream));
        copy_level(ctx, ctx->phi[ctx->phi_cur].p, nullptr, phi_cur);
        copy_level(ctx, ctx->phi[1 - ctx->phi_cur].p, nullptr, phi_prev);
    })
}

RRG_API rrg_status rrg_solver_calc_steps(rrg_ctx* ctx, int nsteps) {
    RRG_ENTRY(ctx, {
        RRG_REQUIRE(ctx->solver_ready, RRG_ERR_STATE, "rrg_solver_init first");
        RRG_REQUIRE(nsteps >= 0, RRG_ERR_INVALID, "nsteps must be >= 0");
        if (nsteps > 0) {
            if (checks_inside_steps(ctx)) {
                drop_pending(ctx);
                wave_steps_unfused(ctx, nsteps);
            } else {
                if (ctx->wave_mode && ctx->src_dirty && !ctx->pending) {
                    // keep the invariant "mg[1 - mg_cur] is zero" before the fused steps
                    RRG_CUDA(cudaMemsetAsync(ctx->mg[1 - ctx->mg_cur].p, 0,
                                             ctx->mg[1 - ctx->mg_cur].bytes, ctx->stream));
                }
                for_each_chunk(ctx, nsteps, ctx->steps_since_sort, [&](int chunk, bool sort) {
                    if (sort) sort_particles(ctx);  // (a pending prediction is permuted along)
                    run_graph(ctx, chunk);
                });
                // the last chunk's last particle pass left the synced state's sums
                ctx->sums_ready = ctx->wave_mode && ctx->step_sums;
            }
            for (int s = 0; s < nsteps; ++s) {
                ctx->iter += 1;
                ctx->time += ctx->sim.dt_dynamics;
            }
        }
    })
}

RRG_API rrg_status rrg_solver_prepare(rrg_ctx* ctx, int nsteps) {
    RRG_ENTRY(ctx, {
        RRG_REQUIRE(ctx->solver_ready, RRG_ERR_STATE, "rrg_solver_init first");
        RRG_REQUIRE(nsteps >= 0, RRG_ERR_INVALID, "nsteps must be >= 0");
        if (nsteps > 0 && !checks_inside_steps(ctx)) {
            // walk the chunks of that call, recording what is missing, then put the roles back
            const int cur = ctx->cur, mg_cur = ctx->mg_cur, phi_cur = ctx->phi_cur;
            const bool pending = ctx->pending, src_dirty = ctx->src_dirty,
                       src_valid = ctx->src_valid, used = ctx->wave_solve_used;
            int64_t since = ctx->steps_since_sort;
            try {
                for_each_chunk(ctx, nsteps, since, [&](int chunk, bool) {
                    chunk_graph(ctx, chunk);
                });
            } catch (...) {
                ctx->cur = cur, ctx->mg_cur = mg_cur, ctx->phi_cur = phi_cur;
                ctx->pending = pending, ctx->src_dirty = src_dirty, ctx->src_valid = src_valid;
                ctx->wave_solve_used = used;
                throw;
            }
            ctx->cur = cur, ctx->mg_cur = mg_cur, ctx->phi_cur = phi_cur;
            ctx->pending = pending, ctx->src_dirty = src_dirty, ctx->src_valid = src_valid;
            ctx->wave_solve_used = used;
        }
    })
}

RRG_API rrg_status rrg_solver_sync(rrg_ctx* ctx) {
    RRG_ENTRY(ctx, {
        RRG_REQUIRE(ctx->solver_ready, RRG_ERR_STATE, "rrg_solver_init first");
        if (ctx->wave_mode) {
            launch_ngp_phi(ctx->prec, ctx->n, ctx->P(), ctx->L(), ctx->gdev,
                           ctx->phi[ctx->phi_cur].p, ctx->pot.p, ctx->stream);
            launch_interp(ctx->prec, ctx->n, ctx->P(), ctx->L(), ctx->gdev, ctx->acc4.p,
                          ctx->acc.p, ctx->stream);
        } else {
            ensure_download(ctx, v4b(ctx) * ctx->n);
            DirectEpi e;
            e.mode = EPI_STORE;
            e.acc = ctx->dl.p;
            e.pot = ctx->pot.p;
            direct(ctx, true, e);
            if (ctx->has_grid) {
                // rrgsim_integration_nbody.cuh:32-48: CIC mass, then NGP cell averages of the
                // particle potential and acceleration; the cell counts live in the (unused in
                // this strategy) source buffer
                deposit_operator(ctx);
                RRG_CUDA(cudaMemsetAsync(ctx->src.p, 0, ctx->src.bytes, ctx->stream));
                RRG_CUDA(cudaMemsetAsync(ctx->phi[ctx->phi_cur].p, 0,
                                         ctx->phi[ctx->phi_cur].bytes, ctx->stream));
                RRG_CUDA(cudaMemsetAsync(ctx->acc4.p, 0, ctx->acc4.bytes, ctx->stream));
                launch_ngp_project(ctx->prec, ctx->n, ctx->P(), ctx->L(), ctx->gdev,
                                   ctx->src.as<int>(), ctx->pot.p, ctx->acc.p,
                                   ctx->phi[ctx->phi_cur].p, ctx->acc4.p, ctx->stream);
            }
        }
    })
}

RRG_API rrg_status rrg_set_sort_interval(rrg_ctx* ctx, int interval) {
    RRG_ENTRY(ctx, {
        RRG_REQUIRE(interval >= 0, RRG_ERR_INVALID, "interval must be >= 0");
        ctx->sort_interval = interval;
        ctx->sums_ready = entry_sums_ready;
    })
}

RRG_API rrg_status rrg_set_step_sums(rrg_ctx* ctx, int enable) {
    RRG_ENTRY(ctx, {
        ctx->step_sums = enable != 0;
        alloc_step_partial(ctx);
    })
}

// ---------------------------------------------------------------------------------------------
RRG_API rrg_status rrg_dev_direct_forces_f32(const void* posm, const void* poslo,
                                             const void* hsoft, float uniform_hsoft, int64_t n,
                                             void* out, int precision, void* stream) {
    try {
        RRG_REQUIRE(posm && out && n > 0, RRG_ERR_INVALID, "rrg_dev_direct_forces_f32: bad args");
        RRG_REQUIRE(precision == RRG_PREC_FP32 || precision == RRG_PREC_MIXED, RRG_ERR_INVALID,
                    "rrg_dev_direct_forces_f32: precision must be FP32 or MIXED");
        int dev = 0;
        RRG_CUDA(cudaGetDevice(&dev));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        DirectLaunch L;
        L.prec = precision;
        L.posm = posm;
        L.poslo = poslo;
        L.hsoft = hsoft;
        L.uniform_hsoft = uniform_hsoft;
        L.n = n;
        L.want_pot = true;
        // write (ax, ay, az, phi) into out: acc slot gets a, the potential goes to w through a
        // strided view is not possible, so compute into out then patch w with the potential
        L.epi.mode = EPI_STORE;
        L.epi.acc = out;
        L.splits = direct_choose_splits(precision, n, num_sms(dev));
        L.scratch_bytes = direct_scratch_bytes(precision, n, L.splits);
        // the split partials are float4 records: they start on a 256-byte boundary behind the
        // potential whatever n is
        const size_t pot_bytes = (sizeof(float) * static_cast<size_t>(n) + 255) & ~size_t(255);
        void* pot = nullptr;
        RRG_CUDA(cudaMallocAsync(&pot, pot_bytes + L.scratch_bytes, s));
        L.epi.pot = pot;
        L.scratch = L.scratch_bytes ? static_cast<char*>(pot) + pot_bytes : nullptr;
        L.stream = s;
        try {
            launch_direct(L);
        } catch (...) {
            cudaFreeAsync(pot, s);
            throw;
        }
        // out[i].w = pot[i]
        RRG_CUDA(cudaMemcpy2DAsync(static_cast<char*>(out) + 12, 16, pot, 4, 4, n,
                                   cudaMemcpyDeviceToDevice, s));
        RRG_CUDA(cudaFreeAsync(pot, s));
        return RRG_OK;
    } catch (const Error& e) {
        t_error = e.what();
        return e.code;
    }
}

RRG_API rrg_status rrg_dev_direct_vjp_f32(const void* posm, const void* hsoft,
                                          float uniform_hsoft, int64_t n, const void* lam,
                                          void* out, void* stream) {
    try {
        RRG_REQUIRE(posm && lam && out && n > 0, RRG_ERR_INVALID,
                    "rrg_dev_direct_vjp_f32: bad args");
        launch_direct_vjp_f32(posm, hsoft, uniform_hsoft, n, lam, out,
                              static_cast<cudaStream_t>(stream));
        return RRG_OK;
    } catch (const Error& e) {
        t_error = e.what();
        return e.code;
    }
}

}  // extern "C"
