// One PM step's whole wave solve in one persistent kernel (FP32, periodic box without an
// absorbing layer, the reference's wired path): wave source from the deposit, `iterations`
// damped-wave substeps (wave_diss_iteration, wave.cu:106-193), then the gradient
// (calc_acceleration_field_, rm_p2mesh.cu:238-290).
//
// Decomposition: a block of 256 threads owns RB = 256 / W rows (y) x ZC planes (z) of whole
// x-rows, W = nx / 4 float4 per row; a thread owns one float4 column (four x-cells of one row,
// all ZC planes) and keeps its current and previous level in registers and its source in
// shared memory for the whole solve. The x neighbours are warp shuffles (a warp holds whole
// rows, periodic wrap inside the row), y neighbours come through a shared-memory tile, z
// neighbours inside the column are the thread's own registers.
//
// Only the block faces cross between blocks, through face buffers in L2: rows y0 and
// y0 + RB - 1 (faces 0 and 1) and planes z0 and z0 + ZC - 1 (faces 2 and 3). After a substep
// the block stores its faces and publishes the epoch with one release store of its counter;
// before the next substep it waits (acquire loads) until its four neighbours (y +- 1, z +- 1,
// periodic) have published the same epoch and copies their faces into its halo (cp.async).
// Face buffers are double-buffered by epoch parity: a block publishes epoch e + 2 only after
// reading its neighbours' e + 1, which they publish after reading its e. L2 traffic per substep
// is the faces written once and read once; the full levels are written to global memory once,
// at the end. A thread stores each face value as soon as it has computed it (the same time per
// launch as storing them all after the plane loop: 87.9 against 88.0 us under ncu).
//
// Where a substep's time goes on 128^3 (clock64 stamps in an instrumented copy, block-local
// time at 1.97 GHz, 3.6 us per substep): the stencil ~0.65 us; the face stores, the barrier and
// the release ~0.85 us; the wait for the neighbours' releases ~1.05 us; the halo copy ~0.6 us;
// the barriers the rest. The exchange, not the stencil, sets the period, and an SM moves its
// ~32 KB of face stores per substep to L2 at only ~40 B per clock. Measured and not kept:
// - a release per warp for its share of a face: every warp then waits for its stores to land;
// - the poll in every warp, to drop the barrier between the poll and the copy: no change;
// - the face cells first, then the interior while the edge warps wait and copy, with a second
//   own-rows buffer: 99 against 95 us per launch (the pointer selects and buffer lengthened the
//   stencil more than the overlap saved);
// - each face value as one 64-bit word (value, epoch) that the readers poll directly, with no
//   fence, counter or second copy: 114 against 95 us per launch (the doubled face bytes and the
//   re-polls saturate the SM's path to L2);
// - one block of 512 threads (16 rows) per SM on 128^3 instead of two of 256, for a quarter
//   fewer face bytes per SM: 98.8 against 93.6 us per launch.
//
// All blocks must be resident together: the launch is cooperative and the host checks capacity
// first. Every wait is bounded; one that runs out sets the error word and the block leaves (the
// step's results are then invalid), and later launches return at once until the host, which
// turns the word into an error, clears the sync memory. The arithmetic is that of
// wave_source_kernel<float>, wave_periodic_x4_kernel and gradient_x4_kernel, expression for
// expression, so the results are the same bits.
#include <cstdlib>
#include <mutex>

#include "kernels.cuh"

namespace rrg {
namespace {

constexpr int kThreads = 256;
constexpr int kZC = 8;                          // planes per block
constexpr double kPiW = 3.14159265358979;       // the reference's PI (co_info_structs.h:7)
constexpr long long kWaitCycles = 1ll << 28;    // ~0.14 s at 1.9 GHz per wait at most
constexpr int kCounterStride = 32;              // a block's epoch counter: 128 bytes apart
constexpr int kErrWord = 16383;                 // in the first 64 KB: counters, error word
constexpr size_t kFaceOffset = 65536;           // then the faces
constexpr int kFace4 = 256;                     // float4 per face: ZC x W or RB x W, at most 256

// Sync memory layout (bytes): [0, 65536) per block (stride 128 B) the epoch counter, then the
// error word (the last 4 bytes); then the faces [parity 2][block][face 4][kFace4] float4.
size_t sync_bytes_for(int64_t nblocks) {
    return kFaceOffset + static_cast<size_t>(nblocks) * 2 * 4 * kFace4 * sizeof(float4);
}

template <int W>
struct Shape {
    static constexpr int nx = 4 * W;
    static constexpr int RB = kThreads / W;           // rows per block
    static constexpr int Hy = kZC * W;                // float4 of a y face (ZC slots of W)
    static constexpr int Hz = RB * W;                 // float4 of a z face (RB slots) = 256
    static constexpr int Hn = 2 * Hy + 2 * Hz;        // a block's halo: y-, y+, z-, z+
    static constexpr int NH = (Hn + kThreads - 1) / kThreads;  // halo float4 per thread
    static constexpr int tileN = kZC * (RB + 2) * W;  // y tile: rows y0 - 1 .. y0 + RB
    static constexpr int zhN = 2 * RB * W;            // z halo planes z0 - 1 and z0 + ZC
    static constexpr size_t smem = (tileN + zhN + kZC * kThreads) * sizeof(float4);
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// 16-byte asynchronous copy global -> shared through L2 only (.cg)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned int sa = static_cast<unsigned int>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;" ::: "memory");
}

struct SolveArgs {
    float* phi0;
    float* phi1;
    int cur;                        // phi_cur at entry: 0 -> phi0 is the current level
    int iterations;
    const unsigned long long* mg;   // this step's deposit
    unsigned long long* mg_zero;    // the other deposit grid: cleared
    double inv_scale, inv_dx3, rho_sub;
    float km, ka, ko, kf, grad_coef;
    float* src;                     // nullptr, or where the source is also stored
    float4* acc4;                   // nullptr: no gradient
    unsigned int* sync;             // sync_bytes_for(blocks), zeroed before the first launch
};

template <int W>
__global__ void __launch_bounds__(kThreads, 2) wave_solve_kernel(const SolveArgs a) {
    using S = Shape<W>;
    constexpr int nx = S::nx, RB = S::RB, ZC = kZC;
    extern __shared__ __align__(16) float4 sm[];
    float4* const tile = sm;                  // [ZC][RB + 2][W]
    float4* const zh = sm + S::tileN;         // [2][RB][W]
    float4* const srcs = zh + S::zhN;         // [ZC][kThreads]
    __shared__ int fail_s;
    __shared__ unsigned int base_s;

    volatile unsigned int* const err = a.sync + kErrWord;
    unsigned int* const counters = a.sync + (blockIdx.y * gridDim.x + blockIdx.x) * kCounterStride;
    if (threadIdx.x == 0) {
        // an earlier launch failed: the state is invalid until the host resets the sync memory
        fail_s = *err != 0;
        // epochs published so far (the same in every block between launches)
        base_s = *reinterpret_cast<volatile unsigned int*>(counters);
    }
    __syncthreads();
    if (fail_s) return;
    const unsigned int base = base_s;

    const int tid = threadIdx.x, lane = tid & 31;
    const int r = tid / W, q = tid % W;
    const int gx = gridDim.x, gz = gridDim.y;
    const int bx = blockIdx.x, bz = blockIdx.y;
    const int y0 = bx * RB, z0 = bz * ZC, y = y0 + r;
    const int seg = lane - lane % W;
    const int lsrc = seg + (lane - seg + W - 1) % W;
    const int rsrc = seg + (lane - seg + 1) % W;
    const int me = bz * gx + bx;
    const int nblocks = gx * gz;
    // face numbers: 0 = row y0 (slot k), 1 = row y0 + RB - 1 (slot k), 2 = plane z0 (slot r),
    // 3 = plane z0 + ZC - 1 (slot r); a slot is W float4. The y- halo is the lower y
    // neighbour's face 1, y+ the upper one's face 0, z- the lower z neighbour's face 3, z+ the
    // upper one's face 2.
    const int nb_ym = bz * gx + (bx == 0 ? gx - 1 : bx - 1);
    const int nb_yp = bz * gx + (bx + 1 == gx ? 0 : bx + 1);
    const int nb_zm = (bz == 0 ? gz - 1 : bz - 1) * gx + bx;
    const int nb_zp = (bz + 1 == gz ? 0 : bz + 1) * gx + bx;
    float4* const faces = reinterpret_cast<float4*>(reinterpret_cast<char*>(a.sync) + kFaceOffset);
    auto face = [&](unsigned int e, int block, int f) {
        return faces + ((static_cast<size_t>(e & 1u) * nblocks + block) * 4 + f) * kFace4;
    };
    const size_t col = (static_cast<size_t>(z0) * nx + y) * W + q;  // float4 index, plane z0
    constexpr size_t plane4 = static_cast<size_t>(nx) * W;

    // ---- the column's levels and source --------------------------------------------------
    float4 cur[ZC], old[ZC];
    {
        const float4* c4 = reinterpret_cast<const float4*>(a.cur == 0 ? a.phi0 : a.phi1);
        const float4* p4 = reinterpret_cast<const float4*>(a.cur == 0 ? a.phi1 : a.phi0);
        const ulonglong2* m2 = reinterpret_cast<const ulonglong2*>(a.mg);
        ulonglong2* z2 = reinterpret_cast<ulonglong2*>(a.mg_zero);
#pragma unroll
        for (int k = 0; k < ZC; ++k) {
            const size_t o4 = col + k * plane4;
            cur[k] = __ldcg(c4 + o4);
            old[k] = __ldcg(p4 + o4);
            const ulonglong2 m01 = __ldcg(m2 + 2 * o4);
            const ulonglong2 m23 = __ldcg(m2 + 2 * o4 + 1);
            const unsigned long long mq[4] = {m01.x, m01.y, m23.x, m23.y};
            float sv[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const double mass = static_cast<double>(mq[e]) * a.inv_scale;
                const double rho = mass * a.inv_dx3 - a.rho_sub;
                sv[e] = static_cast<float>(1.0 * (4.0 * kPiW * 1.0 * rho));
            }
            const float4 s4 = make_float4(sv[0], sv[1], sv[2], sv[3]);
            srcs[k * kThreads + tid] = s4;
            if (a.src != nullptr) __stcg(reinterpret_cast<float4*>(a.src) + o4, s4);
            const ulonglong2 zz = make_ulonglong2(0ull, 0ull);
            __stcg(z2 + 2 * o4, zz);
            __stcg(z2 + 2 * o4 + 1, zz);
        }
    }
    // lanes 0-3 of warp 0 watch one neighbour's counter each
    const unsigned int* watched = nullptr;
    if (tid < 4)
        watched = a.sync + (tid == 0 ? nb_ym : tid == 1 ? nb_yp : tid == 2 ? nb_zm : nb_zp) *
                               kCounterStride;

    // ---- pieces of a substep ---------------------------------------------------------------
    // publish: the block barrier orders every thread's face stores (and its reads of the tile
    // and halo) before the release of epoch e
    // the face values of plane k of a level under epoch e, stored as soon as they are computed
    // so that the stores drain while the other planes are computed
    auto store_faces = [&](unsigned int e, int k, const float4& v) {
        if (r == 0) __stcg(face(e, me, 0) + k * W + q, v);
        else if (r == RB - 1) __stcg(face(e, me, 1) + k * W + q, v);
        if (k == 0) __stcg(face(e, me, 2) + tid, v);
        else if (k == ZC - 1) __stcg(face(e, me, 3) + tid, v);
    };
    auto publish = [&](unsigned int e) {
        __syncthreads();
        if (tid == 0) st_release(counters, e);
    };
    // own rows of the current level into the tile, then the neighbours' faces of epoch e into
    // the halo rows and planes; false for every thread when a wait ran out
    auto exchange = [&](unsigned int e) -> bool {
#pragma unroll
        for (int k = 0; k < ZC; ++k) tile[(k * (RB + 2) + r + 1) * W + q] = cur[k];
        if (tid < 4) {
            const long long t0 = clock64();
            for (unsigned int polls = 1; static_cast<int>(ld_acquire(watched) - e) < 0; ++polls) {
                // give up when the wait ran out, or another block already failed
                if (clock64() - t0 > kWaitCycles || ((polls & 255u) == 0 && *err != 0)) {
                    fail_s = 1;
                    atomicExch(a.sync + kErrWord, 1u);  // (the host clears it)
                    break;
                }
            }
        }
        __syncthreads();
        if (fail_s) return false;
#pragma unroll
        for (int j = 0; j < S::NH; ++j) {
            const int i = tid + j * kThreads;
            if (i >= S::Hn) break;
            if (i < 2 * S::Hy) {
                const int reg = i / S::Hy, off = i - reg * S::Hy;
                const int k = off / W, qq = off - k * W;
                cp_async16(tile + (k * (RB + 2) + (reg == 0 ? 0 : RB + 1)) * W + qq,
                           face(e, reg == 0 ? nb_ym : nb_yp, reg == 0 ? 1 : 0) + off);
            } else {
                const int jj = i - 2 * S::Hy;
                const int reg = jj / S::Hz, off = jj - reg * S::Hz;
                cp_async16(zh + reg * S::Hz + off,
                           face(e, reg == 0 ? nb_zm : nb_zp, reg == 0 ? 3 : 2) + off);
            }
        }
        cp_async_wait_all();
        __syncthreads();
        return true;
    };
    // the new value of cell k of the column from the level in cur / the tile / the halo
    auto cell = [&](int k, const float4& zm, const float4& zp) -> float4 {
        const float4 c = cur[k];
        const float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
        const float rgt = __shfl_sync(0xffffffffu, c.x, rsrc);
        const float4 ym = tile[(k * (RB + 2) + r) * W + q];
        const float4 yp = tile[(k * (RB + 2) + r + 2) * W + q];
        const float4 po = old[k], sv = srcs[k * kThreads + tid];
        float4 out;
        out.x = (lft + c.y + ym.x + yp.x + zm.x + zp.x) * a.km + c.x * a.ka + po.x * a.ko + sv.x * a.kf;
        out.y = (c.x + c.z + ym.y + yp.y + zm.y + zp.y) * a.km + c.y * a.ka + po.y * a.ko + sv.y * a.kf;
        out.z = (c.y + c.w + ym.z + yp.z + zm.z + zp.z) * a.km + c.z * a.ka + po.z * a.ko + sv.z * a.kf;
        out.w = (c.z + rgt + ym.w + yp.w + zm.w + zp.w) * a.km + c.w * a.ka + po.w * a.ko + sv.w * a.kf;
        return out;
    };

    // ---- substeps --------------------------------------------------------------------------
    const unsigned int e0 = base + 1;   // epoch of level 0; level t has e0 + t
#pragma unroll
    for (int k = 0; k < ZC; ++k) store_faces(e0, k, cur[k]);
    publish(e0);
    if (!exchange(e0)) return;
    for (int t = 0; t < a.iterations; ++t) {
        float4 zm = zh[r * W + q];
        const float4 ztop = zh[(RB + r) * W + q];
#pragma unroll
        for (int k = 0; k < ZC; ++k) {
            const float4 out = cell(k, zm, k + 1 < ZC ? cur[k + 1] : ztop);
            zm = cur[k];
            old[k] = cur[k];
            cur[k] = out;
            store_faces(e0 + t + 1, k, out);
        }
        const unsigned int e = e0 + t + 1;
        publish(e);  // (its barrier also ends this substep's reads of the tile and halo)
        if (t + 1 < a.iterations || a.acc4 != nullptr) {
            if (!exchange(e)) return;
        }
    }

    // ---- the levels to global memory (only this thread reads them in this launch) ---------
    {
        const bool fin0 = (a.cur ^ (a.iterations & 1)) == 0;
        float4* fin = reinterpret_cast<float4*>(fin0 ? a.phi0 : a.phi1);
        float4* prv = reinterpret_cast<float4*>(fin0 ? a.phi1 : a.phi0);
#pragma unroll
        for (int k = 0; k < ZC; ++k) {
            __stcg(fin + col + k * plane4, cur[k]);
            __stcg(prv + col + k * plane4, old[k]);
        }
    }

    // ---- gradient of the final level (its halo is in place): central inside, one-sided at
    // the faces
    if (a.acc4 != nullptr) {
        const int x = 4 * q;
#pragma unroll
        for (int k = 0; k < ZC; ++k) {
            const int z = z0 + k;
            const float4 c = cur[k];
            const float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
            const float rgt = __shfl_sync(0xffffffffu, c.x, rsrc);
            const float d0 = x == 0 ? c.y - c.x : 0.5f * (c.y - lft);
            const float d1 = 0.5f * (c.z - c.x);
            const float d2 = 0.5f * (c.w - c.y);
            const float d3 = x + 4 == nx ? c.w - c.z : 0.5f * (rgt - c.z);
            const float4 ym = tile[(k * (RB + 2) + r) * W + q];
            const float4 yp = tile[(k * (RB + 2) + r + 2) * W + q];
            float4 ey;
            if (y == 0) ey = make_float4(yp.x - c.x, yp.y - c.y, yp.z - c.z, yp.w - c.w);
            else if (y == nx - 1) ey = make_float4(c.x - ym.x, c.y - ym.y, c.z - ym.z, c.w - ym.w);
            else
                ey = make_float4(0.5f * (yp.x - ym.x), 0.5f * (yp.y - ym.y), 0.5f * (yp.z - ym.z),
                                 0.5f * (yp.w - ym.w));
            const float4 zm = k > 0 ? cur[k - 1] : zh[r * W + q];
            const float4 zp = k + 1 < ZC ? cur[k + 1] : zh[(RB + r) * W + q];
            float4 ez;
            if (z == 0) ez = make_float4(zp.x - c.x, zp.y - c.y, zp.z - c.z, zp.w - c.w);
            else if (z == nx - 1) ez = make_float4(c.x - zm.x, c.y - zm.y, c.z - zm.z, c.w - zm.w);
            else
                ez = make_float4(0.5f * (zp.x - zm.x), 0.5f * (zp.y - zm.y), 0.5f * (zp.z - zm.z),
                                 0.5f * (zp.w - zm.w));
            const float g = a.grad_coef;
            float4* o = a.acc4 + (static_cast<size_t>(z) * nx + y) * nx + x;
            o[0] = make_float4(d0 * g, ey.x * g, ez.x * g, c.x);
            o[1] = make_float4(d1 * g, ey.y * g, ez.y * g, c.y);
            o[2] = make_float4(d2 * g, ey.z * g, ez.z * g, c.z);
            o[3] = make_float4(d3 * g, ey.w * g, ez.w * g, c.w);
        }
    }
    // the counter ends at e0 + iterations in every block: the next launch starts from there
}

template <int W>
void set_smem_attr() {
    RRG_CUDA(cudaFuncSetAttribute(wave_solve_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(Shape<W>::smem)));
}

template <int W>
int blocks_per_sm() {
    int per_sm = 0;
    RRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wave_solve_kernel<W>,
                                                           kThreads, Shape<W>::smem));
    return per_sm;
}

int64_t block_count(int nx) {
    const int W = nx / 4, RB = kThreads / W;
    return static_cast<int64_t>(nx / RB) * (nx / kZC);
}

}  // namespace

bool wave_solve_applicable(int nx) {
    if (const char* e = std::getenv("RRG_WAVE_PERSIST"))
        if (std::atoi(e) == 0) return false;
    // instantiated for rows of 8, 16 and 32 float4: nx = 32, 64, 128
    return nx == 32 || nx == 64 || nx == 128;
}

size_t wave_solve_sync_bytes(int nx) {
    return (nx == 32 || nx == 64 || nx == 128) ? sync_bytes_for(block_count(nx)) : kFaceOffset;
}

bool launch_wave_solve(int nx, int iterations, float* phi0, float* phi1, int cur,
                       const unsigned long long* mg, unsigned long long* mg_zero, int shift_s,
                       double dx, double rho_sub, const WaveCoef& w, float* src, float4* acc4,
                       unsigned int* sync, size_t sync_bytes, cudaStream_t s) {
    if (!wave_solve_applicable(nx) || iterations < 1) return false;
    const int W = nx / 4, RB = kThreads / W;
    const dim3 grid(nx / RB, nx / kZC);
    const int64_t nblocks = static_cast<int64_t>(grid.x) * grid.y;
    RRG_REQUIRE(nblocks * kCounterStride < kErrWord && sync_bytes >= sync_bytes_for(nblocks),
                RRG_ERR_INVALID, "wave solve: sync memory too small for the grid");
    int dev = 0;
    RRG_CUDA(cudaGetDevice(&dev));
    {
        // the opt-in above 48 KB of shared memory is per device
        static std::mutex mu;
        static bool done[64] = {};
        std::lock_guard<std::mutex> lock(mu);
        if (dev < 0 || dev >= 64 || !done[dev]) {
            set_smem_attr<8>();
            set_smem_attr<16>();
            set_smem_attr<32>();
            if (dev >= 0 && dev < 64) done[dev] = true;
        }
    }
    const int per_sm = W == 8 ? blocks_per_sm<8>()
                              : (W == 16 ? blocks_per_sm<16>() : blocks_per_sm<32>());
    if (static_cast<int64_t>(per_sm) * num_sms(dev) < nblocks)
        return false;  // not all blocks could be resident at once
    SolveArgs a;
    a.phi0 = phi0;
    a.phi1 = phi1;
    a.cur = cur;
    a.iterations = iterations;
    a.mg = mg;
    a.mg_zero = mg_zero;
    a.inv_scale = ldexp(1.0, -shift_s);
    a.inv_dx3 = 1.0 / (dx * dx * dx);
    a.rho_sub = rho_sub;
    a.km = static_cast<float>(w.K_MAIN);
    a.ka = static_cast<float>(w.K_ACTUAL);
    a.ko = static_cast<float>(w.K_OLD);
    a.kf = static_cast<float>(w.K_F);
    a.grad_coef = static_cast<float>(-1.0 / dx);
    a.src = src;
    a.acc4 = acc4;
    a.sync = sync;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (W == 8) {
        cfg.dynamicSmemBytes = Shape<8>::smem;
        RRG_CUDA(cudaLaunchKernelEx(&cfg, wave_solve_kernel<8>, a));
    } else if (W == 16) {
        cfg.dynamicSmemBytes = Shape<16>::smem;
        RRG_CUDA(cudaLaunchKernelEx(&cfg, wave_solve_kernel<16>, a));
    } else {
        cfg.dynamicSmemBytes = Shape<32>::smem;
        RRG_CUDA(cudaLaunchKernelEx(&cfg, wave_solve_kernel<32>, a));
    }
    RRG_LAUNCHED();
    return true;
}

}  // namespace rrg
