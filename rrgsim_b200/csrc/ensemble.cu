// Batched ensemble of independent galaxies on sm_100a: one persistent direct-sum launch over a
// device work-list, graph-captured leapfrog steps, autotuned tiles.
//
// Every galaxy runs the reference's N-body step (predict, direct-sum acceleration, correct;
// solver/app/include/rrgsim_integration_nbody.cuh:50-56, kernels nbody.cu:19-65, 122-181) in
// FP32. Instead of one launch per galaxy, all galaxies' particles sit in one array and the
// force work is cut into items (galaxy, i-tile, j-chunk) of near-equal cost, handed out to
// resident CTAs through an atomic counter. Small galaxies then no longer leave most of the GPU
// idle, and the whole ensemble step is two launches. Each item writes its partial sums; a
// finish pass adds them in a fixed order (deterministic) and applies the leapfrog epilogue.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "host_io.h"
#include "kernels.cuh"

namespace rrg {
namespace {

constexpr int kBS = 256;
constexpr float kPad = 1e18f;

struct EnsGalaxy {
    int64_t off;       // first particle
    int64_t part_off;  // first partial
    int32_t n;
    int32_t splits;
    float h2;          // soft2 of the galaxy (h_i + h_j)
    float m;           // particle mass when every particle of the ensemble galaxy has one
};

struct EnsItem {
    int32_t g, i0, j0, j1, s;
};

struct EnsForceParams {
    const V4<float>* posm;
    const EnsGalaxy* gal;
    const EnsItem* items;
    int num_items;
    unsigned int* counter;
    V4<float>* part;
};

// Persistent force kernel: 2 G i-particles per thread, paired FP32 ops as in
// direct_f32jp_kernel: each f32x2 instruction takes one i against two consecutive j, so one
// pair of shared-memory loads feeds 2 G x 2 pairs. Shared layout per j-pair q:
// (x_2q, x_2q+1, y_2q, y_2q+1), (z_2q, z_2q+1, m_2q, m_2q+1); the two lanes add at the end.
// UMASS: all particles of each galaxy share its mass gg.m (multiplied in once per sum).
template <int G, bool UMASS>
__global__ void __launch_bounds__(kBS, 2) ens_forces_kernel(const EnsForceParams p) {
    constexpr int IPT = 2 * G;
    __shared__ float4 s_xy[kBS / 2];
    __shared__ float4 s_zm[kBS / 2];
    __shared__ int s_item;
    const int tid = threadIdx.x;
    float* const fxy = reinterpret_cast<float*>(s_xy);
    float* const fzm = reinterpret_cast<float*>(s_zm);
    const int q0 = tid >> 1, e0 = tid & 1;
    for (;;) {
        __syncthreads();  // previous item fully done with s_item and the tiles
        if (tid == 0) s_item = static_cast<int>(atomicAdd(p.counter, 1u));
        __syncthreads();
        const int it = s_item;
        if (it >= p.num_items) break;
        const EnsItem w = p.items[it];
        const EnsGalaxy gg = p.gal[w.g];
        const float2 hs = make_float2(gg.h2, gg.h2);
        float2 nx[IPT], ny[IPT], nz[IPT];
#pragma unroll
        for (int q = 0; q < IPT; ++q) {
            const int li = w.i0 + q * kBS + tid;
            V4<float> pi = v4<float>(0.f, 0.f, 0.f, 0.f);
            if (li < gg.n) pi = p.posm[gg.off + li];
            nx[q] = make_float2(-pi.x, -pi.x);
            ny[q] = make_float2(-pi.y, -pi.y);
            nz[q] = make_float2(-pi.z, -pi.z);
        }
        float2 ax[IPT], ay[IPT], az[IPT];
#pragma unroll
        for (int q = 0; q < IPT; ++q) ax[q] = ay[q] = az[q] = make_float2(0.f, 0.f);
        const int je = min(w.j1, gg.n);
        V4<float> nxt = v4<float>(kPad, kPad, kPad, 0.f);
        if (w.j0 + tid < je) nxt = p.posm[gg.off + w.j0 + tid];
        for (int j0 = w.j0; j0 < je; j0 += kBS) {
            __syncthreads();
            fxy[4 * q0 + e0] = nxt.x;
            fxy[4 * q0 + 2 + e0] = nxt.y;
            fzm[4 * q0 + e0] = nxt.z;
            fzm[4 * q0 + 2 + e0] = nxt.w;
            __syncthreads();
            nxt = v4<float>(kPad, kPad, kPad, 0.f);
            if (j0 + kBS + tid < je) nxt = p.posm[gg.off + j0 + kBS + tid];
            float2 tx[IPT], ty[IPT], tz[IPT];
#pragma unroll
            for (int q = 0; q < IPT; ++q) tx[q] = ty[q] = tz[q] = make_float2(0.f, 0.f);
#pragma unroll 8
            for (int k = 0; k < kBS / 2; ++k) {
                const float4 xy = s_xy[k];
                const float4 zm = s_zm[k];
                const float2 px = make_float2(xy.x, xy.y), py = make_float2(xy.z, xy.w);
                const float2 pz = make_float2(zm.x, zm.y), pm = make_float2(zm.z, zm.w);
#pragma unroll
                for (int q = 0; q < IPT; ++q) {
                    const float2 dx = __fadd2_rn(px, nx[q]);
                    const float2 dy = __fadd2_rn(py, ny[q]);
                    const float2 dz = __fadd2_rn(pz, nz[q]);
                    const float2 r2 =
                        __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, hs)));
                    const float2 inv = make_float2(rsqrt_sfu(r2.x), rsqrt_sfu(r2.y));
                    const float2 minv = UMASS ? inv : __fmul2_rn(pm, inv);
                    const float2 kk = __fmul2_rn(minv, __fmul2_rn(inv, inv));
                    tx[q] = __ffma2_rn(dx, kk, tx[q]);
                    ty[q] = __ffma2_rn(dy, kk, ty[q]);
                    tz[q] = __ffma2_rn(dz, kk, tz[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < IPT; ++q) {
                ax[q] = __fadd2_rn(ax[q], tx[q]);
                ay[q] = __fadd2_rn(ay[q], ty[q]);
                az[q] = __fadd2_rn(az[q], tz[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < IPT; ++q) {
            const int li = w.i0 + q * kBS + tid;
            if (li >= gg.n) continue;
            const float sc = UMASS ? gg.m : 1.f;
            p.part[gg.part_off + static_cast<int64_t>(w.s) * gg.n + li] =
                v4<float>(sc * (ax[q].x + ax[q].y), sc * (ay[q].x + ay[q].y),
                          sc * (az[q].x + az[q].y), 0.f);
        }
    }
}

struct EnsFinishParams {
    int64_t ntot;
    const int32_t* gid;
    const EnsGalaxy* gal;
    const V4<float>* part;
    const V4<float>* posm;
    V4<float>* pos_out;
    V4<float>* vel;
    V4<float>* acc;
    V4<float>* u;
    float dt;
    int mode;  // EPI_STORE, EPI_CORRECT, EPI_CORRECT_PREDICT
};

// Fixed-order FP64 sum of a particle's partials + the leapfrog epilogue (as apply_epi).
__global__ void __launch_bounds__(256) ens_finish_kernel(const EnsFinishParams p) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= p.ntot) return;
    const EnsGalaxy gg = p.gal[p.gid[i]];
    const int64_t li = i - gg.off;
    double sx = 0, sy = 0, sz = 0;
    for (int s = 0; s < gg.splits; ++s) {
        const V4<float> v = p.part[gg.part_off + static_cast<int64_t>(s) * gg.n + li];
        sx += v.x;
        sy += v.y;
        sz += v.z;
    }
    const float ax = static_cast<float>(sx), ay = static_cast<float>(sy),
                az = static_cast<float>(sz);
    if (p.mode == EPI_STORE) {
        p.acc[i] = v4<float>(ax, ay, az, 0.f);
        return;
    }
    const float dt = p.dt;
    const V4<float> uu = p.u[i];
    const float vx = 0.5f * (uu.x + dt * ax), vy = 0.5f * (uu.y + dt * ay),
                vz = 0.5f * (uu.z + dt * az);
    if (p.mode == EPI_CORRECT) {
        p.vel[i] = v4<float>(vx, vy, vz, 0.f);
        p.acc[i] = v4<float>(ax, ay, az, 0.f);
        return;
    }
    const float ux = vx + (vx + dt * ax), uy = vy + (vy + dt * ay), uz = vz + (vz + dt * az);
    p.u[i] = v4<float>(ux, uy, uz, 0.f);
    const float hdt = dt * 0.5f;
    const V4<float> q = p.posm[i];
    p.pos_out[i] = v4<float>(q.x + hdt * ux, q.y + hdt * uy, q.z + hdt * uz, q.w);
}

__global__ void __launch_bounds__(256) ens_predict_kernel(int64_t n, V4<float>* __restrict__ posm,
                                                          const V4<float>* __restrict__ vel,
                                                          const V4<float>* __restrict__ acc,
                                                          V4<float>* __restrict__ u, float dt) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V4<float> v = vel[i], a = acc[i];
    const float ux = v.x + (v.x + dt * a.x), uy = v.y + (v.y + dt * a.y),
                uz = v.z + (v.z + dt * a.z);
    u[i] = v4<float>(ux, uy, uz, 0.f);
    const float hdt = dt * 0.5f;
    V4<float> q = posm[i];
    q.x = q.x + hdt * ux;
    q.y = q.y + hdt * uy;
    q.z = q.z + hdt * uz;
    posm[i] = q;
}

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    void alloc(size_t b) {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (!b) return;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            p = nullptr;
            (void)cudaGetLastError();
            throw Error(RRG_ERR_NOMEM, std::string("ensemble: cudaMalloc failed: ") +
                                           cudaGetErrorString(e));
        }
        bytes = b;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

}  // namespace
}  // namespace rrg

using namespace rrg;

struct rrg_ensemble {
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    std::string err;
    int ngal = 0;
    int64_t ntot = 0;
    double dt = 0.0;
    std::vector<int64_t> counts, offs;
    std::vector<float> h2;
    std::vector<float> gmass;  // per-galaxy particle mass (all equal within every galaxy)
    bool umass = false;
    DevBuf posm[2], vel, acc, u, gid, gal, items, part, counter;
    int cur = 0;
    int variant = 1;      // 1: G = 1 (2 i per thread), 2: G = 2 (4 i per thread)
    int jchunk = 4096;
    int num_items = 0;
    int grid = 0;
    std::vector<std::pair<int, cudaGraphExec_t>> graphs;  // (nsteps, cur parity) -> exec
    std::vector<std::pair<int, uint64_t>> graph_kernels;
    double tuned_ms = 0.0;
    ~rrg_ensemble() {
        for (auto& g : graphs)
            if (g.second) cudaGraphExecDestroy(g.second);
        if (own) cudaStreamDestroy(own);
    }
};

namespace {

void drop_ens_graphs(rrg_ensemble* e) {
    for (auto& g : e->graphs)
        if (g.second) cudaGraphExecDestroy(g.second);
    e->graphs.clear();
    e->graph_kernels.clear();
}

// Work-list for a tile variant and j-chunk: items of (i-tile x j-chunk), largest first.
void build_worklist(rrg_ensemble* e, int variant, int jchunk) {
    const int ipt = variant == 2 ? 4 : 2;
    const int itile = kBS * ipt;
    std::vector<EnsGalaxy> gal(e->ngal);
    std::vector<EnsItem> items;
    int64_t part_off = 0;
    for (int g = 0; g < e->ngal; ++g) {
        const int n = static_cast<int>(e->counts[g]);
        const int splits = (n + jchunk - 1) / jchunk;
        gal[g] = EnsGalaxy{e->offs[g], part_off, n, splits, e->h2[g], e->gmass[g]};
        part_off += static_cast<int64_t>(splits) * n;
        for (int i0 = 0; i0 < n; i0 += itile)
            for (int s = 0; s < splits; ++s)
                items.push_back(EnsItem{g, i0, s * jchunk, std::min(n, (s + 1) * jchunk), s});
    }
    std::stable_sort(items.begin(), items.end(), [&](const EnsItem& a, const EnsItem& b) {
        const int64_t ca = static_cast<int64_t>(std::min(itile, gal[a.g].n - a.i0)) * (a.j1 - a.j0);
        const int64_t cb = static_cast<int64_t>(std::min(itile, gal[b.g].n - b.i0)) * (b.j1 - b.j0);
        return ca > cb;
    });
    e->gal.alloc(sizeof(EnsGalaxy) * gal.size());
    e->items.alloc(sizeof(EnsItem) * std::max<size_t>(items.size(), 1));
    e->part.alloc(sizeof(V4<float>) * static_cast<size_t>(std::max<int64_t>(part_off, 1)));
    RRG_CUDA(cudaMemcpy(e->gal.p, gal.data(), sizeof(EnsGalaxy) * gal.size(),
                        cudaMemcpyHostToDevice));
    RRG_CUDA(cudaMemcpy(e->items.p, items.data(), sizeof(EnsItem) * items.size(),
                        cudaMemcpyHostToDevice));
    e->num_items = static_cast<int>(items.size());
    e->variant = variant;
    e->jchunk = jchunk;
    int nb = 0;
    if (variant == 2)
        RRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ens_forces_kernel<2, false>, kBS, 0));
    else
        RRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ens_forces_kernel<1, false>, kBS, 0));
    e->grid = std::min(num_sms(e->device) * std::max(nb, 1), std::max(e->num_items, 1));
    drop_ens_graphs(e);
}

void launch_forces(rrg_ensemble* e, const void* posm) {
    RRG_CUDA(cudaMemsetAsync(e->counter.p, 0, sizeof(unsigned int), e->stream));
    EnsForceParams p;
    p.posm = static_cast<const V4<float>*>(posm);
    p.gal = e->gal.as<EnsGalaxy>();
    p.items = e->items.as<EnsItem>();
    p.num_items = e->num_items;
    p.counter = e->counter.as<unsigned int>();
    p.part = e->part.as<V4<float>>();
    if (e->umass) {
        if (e->variant == 2) ens_forces_kernel<2, true><<<e->grid, kBS, 0, e->stream>>>(p);
        else ens_forces_kernel<1, true><<<e->grid, kBS, 0, e->stream>>>(p);
    } else {
        if (e->variant == 2) ens_forces_kernel<2, false><<<e->grid, kBS, 0, e->stream>>>(p);
        else ens_forces_kernel<1, false><<<e->grid, kBS, 0, e->stream>>>(p);
    }
    RRG_LAUNCHED();
}

void launch_finish(rrg_ensemble* e, int mode, const void* posm, void* pos_out) {
    EnsFinishParams f;
    f.ntot = e->ntot;
    f.gid = e->gid.as<int32_t>();
    f.gal = e->gal.as<EnsGalaxy>();
    f.part = e->part.as<V4<float>>();
    f.posm = static_cast<const V4<float>*>(posm);
    f.pos_out = static_cast<V4<float>*>(pos_out);
    f.vel = e->vel.as<V4<float>>();
    f.acc = e->acc.as<V4<float>>();
    f.u = e->u.as<V4<float>>();
    f.dt = static_cast<float>(e->dt);
    f.mode = mode;
    ens_finish_kernel<<<div_up(e->ntot, 256), 256, 0, e->stream>>>(f);
    RRG_LAUNCHED();
}

void record_steps(rrg_ensemble* e, int nsteps) {
    ens_predict_kernel<<<div_up(e->ntot, 256), 256, 0, e->stream>>>(
        e->ntot, e->posm[e->cur].as<V4<float>>(), e->vel.as<V4<float>>(), e->acc.as<V4<float>>(),
        e->u.as<V4<float>>(), static_cast<float>(e->dt));
    RRG_LAUNCHED();
    for (int s = 0; s < nsteps; ++s) {
        launch_forces(e, e->posm[e->cur].p);
        if (s + 1 < nsteps) {
            launch_finish(e, EPI_CORRECT_PREDICT, e->posm[e->cur].p, e->posm[1 - e->cur].p);
            e->cur = 1 - e->cur;
        } else {
            launch_finish(e, EPI_CORRECT, e->posm[e->cur].p, nullptr);
        }
    }
}

void run_steps(rrg_ensemble* e, int nsteps) {
    const int key = nsteps * 2 + e->cur;
    for (size_t k = 0; k < e->graphs.size(); ++k) {
        if (e->graphs[k].first == key) {
            RRG_CUDA(cudaGraphLaunch(e->graphs[k].second, e->stream));
            count_launches(e->graph_kernels[k].second);
            if ((nsteps - 1) % 2 == 1) e->cur = 1 - e->cur;
            return;
        }
    }
    const int cur0 = e->cur;
    cudaGraph_t g = nullptr;
    RRG_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    set_capturing(true);
    try {
        record_steps(e, nsteps);
    } catch (...) {
        set_capturing(false);
        cudaStreamEndCapture(e->stream, &g);
        if (g) cudaGraphDestroy(g);
        e->cur = cur0;
        throw;
    }
    set_capturing(false);
    RRG_CUDA(cudaStreamEndCapture(e->stream, &g));
    cudaGraphExec_t ex = nullptr;
    cudaError_t err = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    RRG_CUDA(err);
    e->graphs.emplace_back(key, ex);
    e->graph_kernels.emplace_back(key, static_cast<uint64_t>(1 + 2 * nsteps));
    RRG_CUDA(cudaGraphLaunch(ex, e->stream));
    count_launches(1 + 2 * nsteps);
}

// Times one force evaluation per (variant, j-chunk) candidate and keeps the fastest.
void autotune(rrg_ensemble* e) {
    cudaEvent_t a, b;
    RRG_CUDA(cudaEventCreate(&a));
    RRG_CUDA(cudaEventCreate(&b));
    float best = 1e30f;
    int bv = 1, bj = 4096;
    for (int v : {1, 2}) {
        for (int j : {1024, 2048, 4096, 8192, 16384}) {
            build_worklist(e, v, j);
            launch_forces(e, e->posm[e->cur].p);  // warm
            RRG_CUDA(cudaEventRecord(a, e->stream));
            for (int r = 0; r < 2; ++r) launch_forces(e, e->posm[e->cur].p);
            RRG_CUDA(cudaEventRecord(b, e->stream));
            RRG_CUDA(cudaEventSynchronize(b));
            float ms = 0.f;
            RRG_CUDA(cudaEventElapsedTime(&ms, a, b));
            if (ms < best) {
                best = ms;
                bv = v;
                bj = j;
            }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    build_worklist(e, bv, bj);
    e->tuned_ms = best / 2;
}

#define ENS_ENTRY(e, ...)                                                                    \
    try {                                                                                    \
        RRG_REQUIRE((e) != nullptr, RRG_ERR_INVALID, "null ensemble");                       \
        RRG_CUDA(cudaSetDevice((e)->device));                                                \
        __VA_ARGS__;                                                                         \
        return RRG_OK;                                                                       \
    } catch (const Error& x) {                                                               \
        if (e) (e)->err = x.what();                                                          \
        set_thread_error(x.what());                                                          \
        return x.code;                                                                       \
    }

}  // namespace

extern "C" {

RRG_API rrg_status rrg_ensemble_create(int device, int ngal, const int64_t* counts,
                                       const double* pos, const double* vel,
                                       const double* mass, const double* soft2_per_galaxy,
                                       double dt, int autotune_tiles, rrg_ensemble** out) {
    rrg_ensemble* e = nullptr;
    try {
        RRG_REQUIRE(out && counts && pos && vel && mass && soft2_per_galaxy, RRG_ERR_INVALID,
                    "rrg_ensemble_create: NULL argument");
        RRG_REQUIRE(ngal >= 1, RRG_ERR_INVALID, "rrg_ensemble_create: ngal must be >= 1");
        RRG_REQUIRE(std::isfinite(dt) && dt > 0, RRG_ERR_INVALID,
                    "rrg_ensemble_create: dt must be positive");
        RRG_CUDA(cudaSetDevice(device));
        e = new rrg_ensemble();
        e->device = device;
        e->ngal = ngal;
        e->dt = dt;
        int64_t tot = 0;
        for (int g = 0; g < ngal; ++g) {
            RRG_REQUIRE(counts[g] >= 1 && counts[g] < (int64_t(1) << 30), RRG_ERR_INVALID,
                        "rrg_ensemble_create: galaxy sizes must be in [1, 2^30)");
            RRG_REQUIRE(std::isfinite(soft2_per_galaxy[g]) && soft2_per_galaxy[g] >= 0,
                        RRG_ERR_INVALID, "rrg_ensemble_create: bad softening");
            e->counts.push_back(counts[g]);
            e->offs.push_back(tot);
            e->h2.push_back(static_cast<float>(soft2_per_galaxy[g]));
            e->gmass.push_back(static_cast<float>(mass[tot]));
            tot += counts[g];
        }
        RRG_REQUIRE(tot < (int64_t(1) << 31), RRG_ERR_INVALID,
                    "rrg_ensemble_create: more than 2^31 particles");
        for (int64_t i = 0; i < 3 * tot; ++i)
            RRG_REQUIRE(std::isfinite(pos[i]) && std::isfinite(vel[i]), RRG_ERR_INVALID,
                        "rrg_ensemble_create: non-finite position or velocity");
        e->ntot = tot;
        // equal masses within every galaxy: the paired kernel folds the mass out of the pair
        e->umass = true;
        for (int g = 0; g < ngal && e->umass; ++g)
            for (int64_t k = 1; k < counts[g] && e->umass; ++k)
                e->umass = mass[e->offs[g] + k] == mass[e->offs[g]];
        RRG_CUDA(cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking));
        e->stream = e->own;
        const size_t vb = sizeof(V4<float>) * tot;
        e->posm[0].alloc(vb);
        e->posm[1].alloc(vb);
        e->vel.alloc(vb);
        e->acc.alloc(vb);
        e->u.alloc(vb);
        e->gid.alloc(sizeof(int32_t) * tot);
        e->counter.alloc(sizeof(unsigned int));
        std::vector<V4<float>> hp(tot), hv(tot);
        std::vector<int32_t> hg(tot);
        for (int g = 0; g < ngal; ++g)
            for (int64_t k = 0; k < counts[g]; ++k) {
                const int64_t i = e->offs[g] + k;
                hp[i] = v4<float>(static_cast<float>(pos[3 * i]), static_cast<float>(pos[3 * i + 1]),
                                  static_cast<float>(pos[3 * i + 2]), static_cast<float>(mass[i]));
                hv[i] = v4<float>(static_cast<float>(vel[3 * i]), static_cast<float>(vel[3 * i + 1]),
                                  static_cast<float>(vel[3 * i + 2]), 0.f);
                hg[i] = g;
            }
        RRG_CUDA(cudaMemcpy(e->posm[0].p, hp.data(), vb, cudaMemcpyHostToDevice));
        RRG_CUDA(cudaMemcpy(e->vel.p, hv.data(), vb, cudaMemcpyHostToDevice));
        RRG_CUDA(cudaMemcpy(e->gid.p, hg.data(), sizeof(int32_t) * tot, cudaMemcpyHostToDevice));
        if (autotune_tiles) autotune(e);
        else build_worklist(e, 1, 4096);
        // initial accelerations (the strategy's precalc)
        launch_forces(e, e->posm[0].p);
        launch_finish(e, EPI_STORE, e->posm[0].p, nullptr);
        RRG_CUDA(cudaStreamSynchronize(e->stream));
        *out = e;
        return RRG_OK;
    } catch (const Error& x) {
        set_thread_error(x.what());
        delete e;
        return x.code;
    }
}

RRG_API rrg_status rrg_ensemble_destroy(rrg_ensemble* e) {
    if (!e) return RRG_OK;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    delete e;
    return RRG_OK;
}

RRG_API rrg_status rrg_ensemble_set_stream(rrg_ensemble* e, void* stream) {
    ENS_ENTRY(e, {
        e->stream = stream ? static_cast<cudaStream_t>(stream) : e->own;
        drop_ens_graphs(e);
    })
}

RRG_API rrg_status rrg_ensemble_step(rrg_ensemble* e, int nsteps) {
    ENS_ENTRY(e, {
        RRG_REQUIRE(nsteps >= 0, RRG_ERR_INVALID, "nsteps must be >= 0");
        int left = nsteps;
        while (left > 0) {
            const int chunk = std::min(left, 32);
            run_steps(e, chunk);
            left -= chunk;
        }
    })
}

// One force launch per galaxy (no batching): the comparison baseline. plain != 0 uses the
// reference's launch shape (one i-particle per thread, 256-thread blocks, no j-split, scalar
// FP32 pairs); plain == 0 the library's own single-galaxy kernel without a j-split.
RRG_API rrg_status rrg_ensemble_step_sequential(rrg_ensemble* e, int nsteps, int plain) {
    ENS_ENTRY(e, {
        RRG_REQUIRE(nsteps >= 0, RRG_ERR_INVALID, "nsteps must be >= 0");
        for (int s = 0; s < nsteps; ++s) {
            ens_predict_kernel<<<div_up(e->ntot, 256), 256, 0, e->stream>>>(
                e->ntot, e->posm[e->cur].as<V4<float>>(), e->vel.as<V4<float>>(),
                e->acc.as<V4<float>>(), e->u.as<V4<float>>(), static_cast<float>(e->dt));
            RRG_LAUNCHED();
            for (int g = 0; g < e->ngal; ++g) {
                DirectLaunch L;
                L.prec = RRG_PREC_FP32;
                L.posm = e->posm[e->cur].as<V4<float>>() + e->offs[g];
                L.uniform_hsoft = 0.5 * e->h2[g];
                L.n = e->counts[g];
                L.epi.mode = EPI_CORRECT;
                L.epi.dt = e->dt;
                L.epi.vel = e->vel.as<V4<float>>() + e->offs[g];
                L.epi.acc = e->acc.as<V4<float>>() + e->offs[g];
                L.epi.u = e->u.as<V4<float>>() + e->offs[g];
                L.splits = 1;  // one launch per galaxy
                L.variant = plain ? 1 : 0;
                L.stream = e->stream;
                launch_direct(L);
            }
        }
    })
}

RRG_API rrg_status rrg_ensemble_get(rrg_ensemble* e, double* pos, double* vel, double* acc) {
    ENS_ENTRY(e, {
        std::vector<V4<float>> hp(e->ntot), hv(e->ntot), ha(e->ntot);
        const size_t vb = sizeof(V4<float>) * e->ntot;
        RRG_CUDA(cudaStreamSynchronize(e->stream));
        RRG_CUDA(cudaMemcpy(hp.data(), e->posm[e->cur].p, vb, cudaMemcpyDeviceToHost));
        RRG_CUDA(cudaMemcpy(hv.data(), e->vel.p, vb, cudaMemcpyDeviceToHost));
        RRG_CUDA(cudaMemcpy(ha.data(), e->acc.p, vb, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < e->ntot; ++i) {
            if (pos) { pos[3 * i] = hp[i].x; pos[3 * i + 1] = hp[i].y; pos[3 * i + 2] = hp[i].z; }
            if (vel) { vel[3 * i] = hv[i].x; vel[3 * i + 1] = hv[i].y; vel[3 * i + 2] = hv[i].z; }
            if (acc) { acc[3 * i] = ha[i].x; acc[3 * i + 1] = ha[i].y; acc[3 * i + 2] = ha[i].z; }
        }
    })
}

RRG_API rrg_status rrg_ensemble_tuning(const rrg_ensemble* e, int* variant, int* jchunk,
                                       int* num_items, double* force_ms) {
    if (!e) return RRG_ERR_INVALID;
    if (variant) *variant = e->variant;
    if (jchunk) *jchunk = e->jchunk;
    if (num_items) *num_items = e->num_items;
    if (force_ms) *force_ms = e->tuned_ms;
    return RRG_OK;
}

RRG_API rrg_status rrg_ensemble_synchronize(rrg_ensemble* e) {
    ENS_ENTRY(e, { RRG_CUDA(cudaStreamSynchronize(e->stream)); })
}

}  // extern "C"
