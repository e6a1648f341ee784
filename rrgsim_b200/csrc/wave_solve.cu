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
//   fewer face bytes per SM: 98.8 against 93.6 us per launch;
// - an L2 prefetch of the deposit and the earlier level at entry: 100.2 against 98.0 us;
// - no counter: empty face slots hold the NaN pattern 0xffffffff (never an FP32 arithmetic
//   result), a thread per neighbour face polls one float4 until it has arrived, every thread
//   loads its share, re-reads any float4 still empty and empties the slot, and a fence per
//   thread orders those resets before its next face stores. The same bits, but 103-108 against
//   98 us per launch (the resets double the stores to L2; with face stores after the planes or
//   interleaved, with or without a back-off in the poll, all within 1%);
// - clusters of 4 x 2 blocks (y x z; 32 of them resident with the cooperative launch): faces
//   between partners pushed straight into the partner's tile and z halo between two cluster
//   barriers per substep, only the cluster's boundary faces through L2 (4 or 8 KB per block
//   instead of 16, one or two counters instead of four). The same bits, but 112.8 against 96.9
//   us per launch: the two cluster barriers add more than the smaller exchange saves;
// - relaxed loads in the poll and one acquire fence after it instead of acquire loads: 100.2
//   against 92.7 us per launch (the fence costs more than the acquire loads).
//
// Timing-only copies (results wrong on purpose) split the launch: without the stencil
// arithmetic it takes 79.8 us against 98.0, so the 20 exchanges, the prologue and the gradient
// cost ~80 us and the stencil ~18 us (0.9 us per substep). The two-substep kernel without its
// arithmetic takes 74.7 us: its 10 exchanges (two cells deep, eight neighbours) cost about as
// much as the 20 one-deep ones.
//
// All blocks must be resident together: the launch is cooperative and the host checks capacity
// first. Every wait is bounded; one that runs out sets the error word and the block leaves (the
// step's results are then invalid), and later launches return at once until the host, which
// turns the word into an error, clears the sync memory. The arithmetic is that of
// wave_source_kernel<float>, wave_periodic_x4_kernel and gradient_x4_kernel, expression for
// expression, so the results are the same bits.
#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "kernels.cuh"

namespace rrg {
namespace {

constexpr int kThreads = 256;
constexpr int kZC = 8;                          // planes per block
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
    float km, ka, ko, kf, grad_coef;  // kf = 1: the substeps run on increments (wave_inc_source)
    double kf_d, km_d, kao_d;         // K_F, K_MAIN, K_ACTUAL + K_OLD - 1 for the increments' source
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

    // ---- the column's level 0 (phi0); the deposit's FP64 sources -------------------------
    const float4* const c4 = reinterpret_cast<const float4*>(a.cur == 0 ? a.phi0 : a.phi1);
    const float4* const p4 = reinterpret_cast<const float4*>(a.cur == 0 ? a.phi1 : a.phi0);
    const ulonglong2* const m2 = reinterpret_cast<const ulonglong2*>(a.mg);
    float4 cur[ZC], old[ZC] = {};  // (old: set before the first substep)
#pragma unroll
    for (int k = 0; k < ZC; ++k) {
        cur[k] = __ldcg(c4 + col + k * plane4);
        tile[(k * (RB + 2) + r + 1) * W + q] = cur[k];
    }
    // phi0's halo straight from global memory (rows y0 - 1 and y0 + RB at the own planes, planes
    // z0 - 1 and z0 + ZC of the own rows, periodic): no exchange is needed for level 0
    for (int i = tid; i < 2 * S::Hy; i += kThreads) {
        const int reg = i / S::Hy, off = i - reg * S::Hy, k = off / W, qq = off - k * W;
        const int yy = reg == 0 ? (y0 == 0 ? nx - 1 : y0 - 1) : (y0 + RB == nx ? 0 : y0 + RB);
        tile[(k * (RB + 2) + (reg == 0 ? 0 : RB + 1)) * W + qq] =
            __ldcg(c4 + (static_cast<size_t>(z0 + k) * nx + yy) * W + qq);
    }
    for (int i = tid; i < 2 * S::Hz; i += kThreads) {
        const int reg = i / S::Hz, off = i - reg * S::Hz, rr = off / W, qq = off - rr * W;
        const int zz = reg == 0 ? (z0 == 0 ? nx - 1 : z0 - 1) : (z0 + ZC == nx ? 0 : z0 + ZC);
        zh[i] = __ldcg(c4 + (static_cast<size_t>(zz) * nx + y0 + rr) * W + qq);
    }
    auto source = [&](size_t o4, double sd[4]) {
        const ulonglong2 m01 = __ldcg(m2 + 2 * o4);
        const ulonglong2 m23 = __ldcg(m2 + 2 * o4 + 1);
        sd[0] = wave_source_value(m01.x, a.inv_scale, a.inv_dx3, a.rho_sub);
        sd[1] = wave_source_value(m01.y, a.inv_scale, a.inv_dx3, a.rho_sub);
        sd[2] = wave_source_value(m23.x, a.inv_scale, a.inv_dx3, a.rho_sub);
        sd[3] = wave_source_value(m23.y, a.inv_scale, a.inv_dx3, a.rho_sub);
    };
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
        return wave_cell4(c, lft, rgt, ym, yp, zm, zp, po, sv, a.km, a.ka, a.ko, a.kf);
    };

    // ---- substeps --------------------------------------------------------------------------
    // level t + 1 is published as epoch e0 + t + 1 (level 0 is not exchanged)
    const unsigned int e0 = base;
    __syncthreads();  // phi0 and its halo in the tile
    // the increments' source g from phi0 and its halo (wave_inc_source); the plain source stored
    // where asked, the other deposit cleared; then level 0 of the increments is zero everywhere
    // and the one before it phi_prev - phi0
    {
        ulonglong2* z2 = reinterpret_cast<ulonglong2*>(a.mg_zero);
        float4 zm = zh[r * W + q];
        const float4 ztop = zh[(RB + r) * W + q];
#pragma unroll
        for (int k = 0; k < ZC; ++k) {
            const size_t o4 = col + k * plane4;
            double sd[4];
            source(o4, sd);
            const float4 c = cur[k];
            const float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
            const float rgt = __shfl_sync(0xffffffffu, c.x, rsrc);
            srcs[k * kThreads + tid] = wave_inc_source4(
                sd, c, lft, rgt, tile[(k * (RB + 2) + r) * W + q],
                tile[(k * (RB + 2) + r + 2) * W + q], zm, k + 1 < ZC ? cur[k + 1] : ztop,
                a.kf_d, a.km_d, a.kao_d);
            zm = c;
            if (a.src != nullptr)
                __stcg(reinterpret_cast<float4*>(a.src) + o4,
                       make_float4(static_cast<float>(sd[0]), static_cast<float>(sd[1]),
                                   static_cast<float>(sd[2]), static_cast<float>(sd[3])));
            const ulonglong2 zz = make_ulonglong2(0ull, 0ull);
            __stcg(z2 + 2 * o4, zz);
            __stcg(z2 + 2 * o4 + 1, zz);
        }
#pragma unroll
        for (int k = 0; k < ZC; ++k) {
            old[k] = f4_sub(__ldcg(p4 + col + k * plane4), cur[k]);
            cur[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncthreads();
        for (int i = tid; i < S::tileN; i += kThreads) tile[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int i = tid; i < S::zhN; i += kThreads) zh[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
    }
    for (int t = 0; t < a.iterations; ++t) {
        const bool last = t + 1 == a.iterations;
        float4 zm = zh[r * W + q];
        const float4 ztop = zh[(RB + r) * W + q];
#pragma unroll
        for (int k = 0; k < ZC; ++k) {
            const float4 out = cell(k, zm, k + 1 < ZC ? cur[k + 1] : ztop);
            zm = cur[k];
            if (last) {
                // the solve's last substep: full levels, phi0 + d (phi0 read again: only this
                // block writes its cells, after its last exchange)
                const float4 p0 = __ldcg(c4 + col + k * plane4);
                old[k] = f4_add(p0, cur[k]);
                cur[k] = f4_add(p0, out);
            } else {
                old[k] = cur[k];
                cur[k] = out;
            }
            store_faces(e0 + t + 1, k, cur[k]);
        }
        const unsigned int e = e0 + t + 1;
        publish(e);  // (its barrier also ends this substep's reads of the tile and halo)
        // (the last exchange gives the gradient its halo; it also keeps every block's final
        // writes after its neighbours' reads of phi0's halo, even without a gradient)
        if (!exchange(e)) return;
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
            // a warp's 128 cells are contiguous (its rows are consecutive): staged through the
            // source area (idle now), then stored 512 contiguous bytes per instruction
            float4* const st = srcs + (tid >> 5) * 128;
            __syncwarp();
            st[4 * lane] = make_float4(d0 * g, ey.x * g, ez.x * g, c.x);
            st[4 * lane + 1] = make_float4(d1 * g, ey.y * g, ez.y * g, c.y);
            st[4 * lane + 2] = make_float4(d2 * g, ey.z * g, ez.z * g, c.z);
            st[4 * lane + 3] = make_float4(d3 * g, ey.w * g, ez.w * g, c.w);
            __syncwarp();
            float4* const o = a.acc4 + (static_cast<size_t>(z) * nx + (y - lane / W)) * nx;
#pragma unroll
            for (int i = 0; i < 4; ++i) o[i * 32 + lane] = st[i * 32 + lane];
        }
    }
    // the counter ends at e0 + iterations in every block: the next launch starts from there
}


// ================================================================================================
// Two substeps per exchange (nx = 128): temporal blocking with a halo two cells deep.
//
// A block of 512 threads (one block per SM, 128 blocks) owns RB = 16 rows x ZC = 8 planes of
// whole x-rows; a warp is one row. A thread keeps its row's float4 column over the planes
// z0 - 1 .. z0 + ZC (its own ZC planes and one on either side) in registers, current and
// previous level. One exchange brings level t of the neighbours two cells deep: rows
// y0 - 2 .. y0 - 1 and y0 + RB .. y0 + RB + 1 at the own planes, planes z0 - 2 .. z0 - 1 and
// z0 + ZC .. z0 + ZC + 1 of the own rows, and the four edge rows (y0 - 1 or y0 + RB, z0 - 1 or
// z0 + ZC) from the diagonal neighbours. Substep A then advances the ten-plane columns and the
// two rows just outside the block (y0 - 1 and y0 + RB at the own planes: one warp per row and
// plane, sixteen in all) to level t + 1; substep B advances the block's own cells to t + 2 from
// those. A cell outside the block is computed from the same values, by the same expression
// (wave_cell4), as its owner computes it, so the results are the bits of one exchange per
// substep. Per two substeps: one exchange instead of two, for 19 float4 updates per thread
// instead of 16, and 48 KB of faces stored per block (an SM of the one-exchange kernel stores
// 64 KB in two substeps).
//
// Shared memory (225,280 bytes): the level tile [KP planes][RB + 4 rows][W], the planes
// z0 - 2 and z0 + ZC + 1 of the own rows, the columns' source [KP][T], and for the two outer
// rows their source and, double-buffered, their previous level. An odd substep count ends with
// one substep B on its own. Every pass ends with an exchange, the last one giving the gradient
// its halo; a block writes its levels to global memory only after it, so every neighbour has
// read its initial halo from there by then.
namespace tb {
constexpr int T = 512;
constexpr int W = 32;
constexpr int NX = 4 * W;
constexpr int RB = T / W;                 // 16 rows
constexpr int ZC = kZC;                   // 8 planes
constexpr int KP = ZC + 2;                // planes of a thread's column: z0 - 1 .. z0 + ZC
constexpr int JR = RB + 4;                // tile rows: y0 - 2 .. y0 + RB + 1
constexpr int tileN = KP * JR * W;
constexpr int zhN = 2 * RB * W;
constexpr int srcN = KP * T;
constexpr int ringN = 2 * ZC * W;         // rows y0 - 1 (side 0) and y0 + RB (side 1)
constexpr size_t smem = static_cast<size_t>(tileN + zhN + srcN + 3 * ringN) * sizeof(float4);
constexpr int FY = 2 * ZC * W;            // y face: two rows x ZC planes, [row][plane][W]
constexpr int FZ = 2 * RB * W;            // z face: two planes x RB rows, [plane][row][W]
constexpr int FB = 2 * FY + 2 * FZ;       // a block's faces per epoch parity: F0 F1 F2 F3
constexpr int HALO = 2 * FY + 2 * FZ + 4 * W;  // float4 a block copies in per exchange
static_assert(2 * ZC == T / 32, "one warp per outer row and plane");
}  // namespace tb

size_t sync_bytes_tb(int64_t nblocks) {
    return kFaceOffset + static_cast<size_t>(nblocks) * 2 * tb::FB * sizeof(float4);
}

__global__ void __launch_bounds__(tb::T, 1) wave_solve_tb_kernel(const SolveArgs a) {
    using namespace tb;
    extern __shared__ __align__(16) float4 sm[];
    float4* const tile = sm;              // [KP][JR][W]: plane z0 - 1 + k, row y0 - 2 + j
    float4* const zh = tile + tileN;      // [2][RB][W]: planes z0 - 2, z0 + ZC + 1
    float4* const srcs = zh + zhN;        // [KP][T]
    float4* const rsrc = srcs + srcN;     // [2 sides][ZC][W]: the outer rows' source
    float4* const rold = rsrc + ringN;    // [2 parities][2 sides][ZC][W]: their earlier level
    __shared__ int fail_s;
    __shared__ unsigned int base_s;

    const int gx = gridDim.x, gz = gridDim.y, bx = blockIdx.x, bz = blockIdx.y;
    const int me = bz * gx + bx, nblocks = gx * gz;
    volatile unsigned int* const err = a.sync + kErrWord;
    unsigned int* const counter = a.sync + me * kCounterStride;
    if (threadIdx.x == 0) {
        fail_s = *err != 0;  // an earlier launch failed: invalid until the host resets
        base_s = *reinterpret_cast<volatile unsigned int*>(counter);
    }
    __syncthreads();
    if (fail_s) return;
    const unsigned int base = base_s;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r = warp, q = lane;
    const int y0 = bx * RB, z0 = bz * ZC;
    const int lsrc = (lane + 31) & 31, rsrcl = (lane + 1) & 31;
    const int bxm = bx == 0 ? gx - 1 : bx - 1, bxp = bx + 1 == gx ? 0 : bx + 1;
    const int bzm = bz == 0 ? gz - 1 : bz - 1, bzp = bz + 1 == gz ? 0 : bz + 1;
    float4* const faces = reinterpret_cast<float4*>(reinterpret_cast<char*>(a.sync) + kFaceOffset);
    auto face = [&](unsigned int e, int block) {
        return faces + (static_cast<size_t>(e & 1u) * nblocks + block) * FB;
    };
    auto T4 = [&](int k, int j) { return tile + (k * JR + j) * W; };
    auto g4 = [](int z, int yy) -> size_t {  // float4 index of (0, yy, z), periodic
        return (static_cast<size_t>(z & (NX - 1)) * NX + (yy & (NX - 1))) * W;
    };
    const float km = a.km, ka = a.ka, ko = a.ko, kf = a.kf;
    const float4* const c4 = reinterpret_cast<const float4*>(a.cur == 0 ? a.phi0 : a.phi1);
    const float4* const p4 = reinterpret_cast<const float4*>(a.cur == 0 ? a.phi1 : a.phi0);
    const ulonglong2* const m2 = reinterpret_cast<const ulonglong2*>(a.mg);
    // the FP64 sources of four cells from the deposit (wave_source_value)
    auto source = [&](size_t o4, double sd[4]) {
        const ulonglong2 m01 = __ldcg(m2 + 2 * o4);
        const ulonglong2 m23 = __ldcg(m2 + 2 * o4 + 1);
        sd[0] = wave_source_value(m01.x, a.inv_scale, a.inv_dx3, a.rho_sub);
        sd[1] = wave_source_value(m01.y, a.inv_scale, a.inv_dx3, a.rho_sub);
        sd[2] = wave_source_value(m23.x, a.inv_scale, a.inv_dx3, a.rho_sub);
        sd[3] = wave_source_value(m23.y, a.inv_scale, a.inv_dx3, a.rho_sub);
    };

    // ---- level 0 (phi0) and its halo from global memory into the tile ----------------------
#pragma unroll
    for (int k = 0; k < KP; ++k) T4(k, r + 2)[q] = __ldcg(c4 + g4(z0 - 1 + k, y0 + r) + q);
    for (int i = tid; i < 4 * ZC * W; i += T) {  // rows y0-2, y0-1, y0+RB, y0+RB+1, own planes
        const int jj = i / (ZC * W), rem = i - jj * (ZC * W), kk = rem / W, qq = rem - kk * W;
        const int j = jj < 2 ? jj : RB + jj;
        T4(kk + 1, j)[qq] = __ldcg(c4 + g4(z0 + kk, y0 - 2 + j) + qq);
    }
    for (int i = tid; i < 4 * W; i += T) {  // the four edge rows
        const int cc = i / W, qq = i - cc * W;
        const int j = (cc & 1) ? RB + 2 : 1, k = (cc & 2) ? KP - 1 : 0;
        T4(k, j)[qq] = __ldcg(c4 + g4(z0 - 1 + k, y0 - 2 + j) + qq);
    }
    for (int i = tid; i < zhN; i += T) {  // planes z0 - 2 and z0 + ZC + 1 of the own rows
        const int side = i / (RB * W), rem = i - side * (RB * W), rr = rem / W, qq = rem - rr * W;
        zh[i] = __ldcg(c4 + g4(side ? z0 + ZC + 1 : z0 - 2, y0 + rr) + qq);
    }
    for (int i = tid; i < ringN; i += T) {  // the outer rows' increment before level 0
        const int side = i / (ZC * W), rem = i - side * (ZC * W), kk = rem / W, qq = rem - kk * W;
        const size_t o4 = g4(z0 + kk, side ? y0 + RB : y0 - 1) + qq;
        rold[i] = f4_sub(__ldcg(p4 + o4), __ldcg(c4 + o4));
    }
    __syncthreads();

    // ---- the increments' source g of the columns and of the outer rows (from phi0 and its
    // halo); the plain source stored where asked, the other deposit cleared -------------------
    {
        const double kfd = a.kf_d, kmd = a.km_d, kao = a.kao_d;
#pragma unroll 1
        for (int k = 0; k < KP; ++k) {
            const size_t o4 = g4(z0 - 1 + k, y0 + r) + q;
            double sd[4];
            source(o4, sd);
            const float4 c = T4(k, r + 2)[q];
            const float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
            const float rgt = __shfl_sync(0xffffffffu, c.x, rsrcl);
            const float4 zm = k > 0 ? T4(k - 1, r + 2)[q] : zh[r * W + q];
            const float4 zp = k + 1 < KP ? T4(k + 1, r + 2)[q] : zh[(RB + r) * W + q];
            srcs[k * T + tid] = wave_inc_source4(sd, c, lft, rgt, T4(k, r + 1)[q],
                                                 T4(k, r + 3)[q], zm, zp, kfd, kmd, kao);
            if (k >= 1 && k <= ZC) {
                if (a.src != nullptr)
                    __stcg(reinterpret_cast<float4*>(a.src) + o4,
                           make_float4(static_cast<float>(sd[0]), static_cast<float>(sd[1]),
                                       static_cast<float>(sd[2]), static_cast<float>(sd[3])));
                ulonglong2* z2 = reinterpret_cast<ulonglong2*>(a.mg_zero);
                const ulonglong2 zz = make_ulonglong2(0ull, 0ull);
                __stcg(z2 + 2 * o4, zz);
                __stcg(z2 + 2 * o4 + 1, zz);
            }
        }
        const int side = warp / ZC, kk = warp - side * ZC, k = kk + 1;
        const int j = side ? RB + 2 : 1;
        double sd[4];
        source(g4(z0 + kk, side ? y0 + RB : y0 - 1) + q, sd);
        const float4 c = T4(k, j)[q];
        const float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
        const float rgt = __shfl_sync(0xffffffffu, c.x, rsrcl);
        rsrc[(side * ZC + kk) * W + q] =
            wave_inc_source4(sd, c, lft, rgt, T4(k, j - 1)[q], T4(k, j + 1)[q], T4(k - 1, j)[q],
                             T4(k + 1, j)[q], kfd, kmd, kao);
    }
    // ---- level 0 of the increments is zero everywhere; the one before is phi_prev - phi0 ---
    float4 cur[KP], old[KP];
#pragma unroll
    for (int k = 0; k < KP; ++k) {
        old[k] = f4_sub(__ldcg(p4 + g4(z0 - 1 + k, y0 + r) + q), T4(k, r + 2)[q]);
        cur[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    for (int i = tid; i < tileN; i += T) tile[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = tid; i < zhN; i += T) zh[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();

    // lanes 0-7 of warp 0 watch one neighbour's counter each: y-, y+, z-, z+, then the
    // diagonals (y-, z-), (y+, z-), (y-, z+), (y+, z+)
    const unsigned int* watched = nullptr;
    if (tid < 8) {
        const int nbx = (tid == 0 || tid == 4 || tid == 6) ? bxm
                        : (tid == 1 || tid == 5 || tid == 7) ? bxp : bx;
        const int nbz = (tid == 2 || tid == 4 || tid == 5) ? bzm
                        : (tid == 3 || tid == 6 || tid == 7) ? bzp : bz;
        watched = a.sync + (nbz * gx + nbx) * kCounterStride;
    }
    const int nb_ym = bz * gx + bxm, nb_yp = bz * gx + bxp;
    const int nb_zm = bzm * gx + bx, nb_zp = bzp * gx + bx;
    const int nb_mm = bzm * gx + bxm, nb_pm = bzm * gx + bxp;
    const int nb_mp = bzp * gx + bxm, nb_pp = bzp * gx + bxp;

    // ---- pieces of a pass ------------------------------------------------------------------
    // the block's face values of plane k (1 .. ZC) of the level of epoch e: F0 rows 0, 1;
    // F1 rows RB - 2, RB - 1; F2 planes 1, 2; F3 planes ZC - 1, ZC
    auto store_faces = [&](unsigned int e, int k, const float4& v) {
        float4* const f = face(e, me);
        if (r < 2) __stcg(f + (r * ZC + k - 1) * W + q, v);
        else if (r >= RB - 2) __stcg(f + FY + ((r - RB + 2) * ZC + k - 1) * W + q, v);
        if (k <= 2) __stcg(f + 2 * FY + ((k - 1) * RB + r) * W + q, v);
        else if (k >= ZC - 1) __stcg(f + 2 * FY + FZ + ((k - ZC + 1) * RB + r) * W + q, v);
    };
    // substep A: level t -> t + 1 on the ten-plane columns and the outer rows; the new levels
    // replace level t in the tile once every read of it is done. The outer rows' earlier level
    // is read from parity par and their new one written to the other.
    auto substep_a = [&](int par) {
        float4 zm = zh[r * W + q];
        const float4 ztop = zh[(RB + r) * W + q];
#pragma unroll
        for (int k = 0; k < KP; ++k) {
            const float4 c = cur[k];
            const float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
            const float rgt = __shfl_sync(0xffffffffu, c.x, rsrcl);
            const float4 zp = k + 1 < KP ? cur[k + 1] : ztop;
            const float4 out = wave_cell4(c, lft, rgt, T4(k, r + 1)[q], T4(k, r + 3)[q], zm, zp,
                                          old[k], srcs[k * T + tid], km, ka, ko, kf);
            zm = c;
            old[k] = c;
            cur[k] = out;
        }
        const int side = warp / ZC, kk = warp - side * ZC, k = kk + 1;
        const int j = side ? RB + 2 : 1;
        const int ri = (side * ZC + kk) * W + q;
        float4 ring;
        {
            const float4 c = T4(k, j)[q];
            const float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
            const float rgt = __shfl_sync(0xffffffffu, c.x, rsrcl);
            ring = wave_cell4(c, lft, rgt, T4(k, j - 1)[q], T4(k, j + 1)[q], T4(k - 1, j)[q],
                              T4(k + 1, j)[q], rold[par * ringN + ri], rsrc[ri], km, ka, ko, kf);
        }
        __syncthreads();
#pragma unroll
        for (int k2 = 0; k2 < KP; ++k2) T4(k2, r + 2)[q] = cur[k2];
        T4(k, j)[q] = ring;
        rold[(par ^ 1) * ringN + ri] = ring;
        __syncthreads();
    };
    // substep B: the own cells (planes 1 .. ZC) one level on, from the tile and the columns'
    // outer planes; faces stored under epoch e as they are computed. In the solve's last
    // substep the own levels become full levels, phi0 + d (phi0 read again from global memory:
    // only this block writes its cells, and only after its last exchange), so the last exchange
    // brings the neighbours' full final level for the gradient.
    auto substep_b = [&](unsigned int e, bool last) {
        float4 zm = cur[0];
#pragma unroll
        for (int k = 1; k <= ZC; ++k) {
            const float4 c = cur[k];
            const float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
            const float rgt = __shfl_sync(0xffffffffu, c.x, rsrcl);
            const float4 out = wave_cell4(c, lft, rgt, T4(k, r + 1)[q], T4(k, r + 3)[q], zm,
                                          cur[k + 1], old[k], srcs[k * T + tid], km, ka, ko, kf);
            zm = c;
            old[k] = c;
            cur[k] = out;
            if (!last) store_faces(e, k, out);
        }
        if (last) {
#pragma unroll
            for (int k = 1; k <= ZC; ++k) {
                const float4 p0 = __ldcg(c4 + g4(z0 - 1 + k, y0 + r) + q);
                old[k] = f4_add(p0, old[k]);
                cur[k] = f4_add(p0, cur[k]);
                store_faces(e, k, cur[k]);
            }
        }
    };
    // publish epoch e (the barrier orders every thread's face stores and its reads of the tile
    // before the release), then bring in the neighbours' faces of epoch e; false for every
    // thread when a wait ran out
    auto exchange = [&](unsigned int e) -> bool {
        __syncthreads();
        if (tid == 0) st_release(counter, e);
#pragma unroll
        for (int k = 1; k <= ZC; ++k) T4(k, r + 2)[q] = cur[k];
        if (tid < 8) {
            const long long t0 = clock64();
            for (unsigned int polls = 1; static_cast<int>(ld_acquire(watched) - e) < 0; ++polls) {
                if (clock64() - t0 > kWaitCycles || ((polls & 255u) == 0 && *err != 0)) {
                    fail_s = 1;
                    atomicExch(a.sync + kErrWord, 1u);  // (the host clears it)
                    break;
                }
            }
        }
        __syncthreads();
        if (fail_s) return false;
        for (int i = tid; i < HALO; i += T) {
            const float4* from;
            float4* to;
            if (i < 2 * FY) {
                // rows y0 - 2, y0 - 1 from the lower y neighbour's F1; rows y0 + RB,
                // y0 + RB + 1 from the upper one's F0
                const int side = i / FY, off = i - side * FY;
                const int rr = off / (ZC * W), rem = off - rr * (ZC * W);
                const int kk = rem / W, qq = rem - kk * W;
                from = face(e, side ? nb_yp : nb_ym) + (side ? 0 : FY) + off;
                to = T4(kk + 1, side ? RB + 2 + rr : rr) + qq;
            } else if (i < 2 * FY + 2 * FZ) {
                // planes z0 - 2, z0 - 1 from the lower z neighbour's F3; planes z0 + ZC,
                // z0 + ZC + 1 from the upper one's F2
                const int iz = i - 2 * FY;
                const int side = iz / FZ, off = iz - side * FZ;
                const int pp = off / (RB * W), rem = off - pp * (RB * W);
                const int rr = rem / W, qq = rem - rr * W;
                from = face(e, side ? nb_zp : nb_zm) + 2 * FY + (side ? 0 : FZ) + off;
                if (side == 0) to = pp == 0 ? zh + rr * W + qq : T4(0, rr + 2) + qq;
                else to = pp == 0 ? T4(KP - 1, rr + 2) + qq : zh + (RB + rr) * W + qq;
            } else {
                // the edge rows (y0 - 1 or y0 + RB, z0 - 1 or z0 + ZC) from the diagonal
                // neighbours: row RB - 1 is F1's second row, row 0 F0's first; plane ZC is
                // slot ZC - 1 of a y face, plane 1 slot 0
                const int ic = i - 2 * FY - 2 * FZ;
                const int cc = ic / W, qq = ic - cc * W;
                const bool up_y = (cc & 1) != 0, up_z = (cc & 2) != 0;
                const int nb = up_z ? (up_y ? nb_pp : nb_mp) : (up_y ? nb_pm : nb_mm);
                const int slot = up_z ? 0 : ZC - 1;
                from = face(e, nb) + (up_y ? slot * W : FY + (ZC + slot) * W) + qq;
                to = T4(up_z ? KP - 1 : 0, up_y ? RB + 2 : 1) + qq;
            }
            cp_async16(to, from);
        }
        cp_async_wait_all();
        __syncthreads();
        // the columns' outer planes: the level before, and level t from the halo
        old[0] = cur[0];
        cur[0] = T4(0, r + 2)[q];
        old[KP - 1] = cur[KP - 1];
        cur[KP - 1] = T4(KP - 1, r + 2)[q];
        return true;
    };

    // ---- passes of two substeps, then an odd one -------------------------------------------
    unsigned int e = base;
    int par = 0;
    const int npairs = a.iterations / 2;
    const int npasses = npairs + (a.iterations & 1);
    for (int p = 0; p < npasses; ++p) {
        if (p < npairs) {  // two substeps; an odd count ends with substep B alone
            substep_a(par);
            par ^= 1;
        }
        ++e;
        substep_b(e, p + 1 == npasses);
        if (!exchange(e)) return;
    }

    // ---- the levels to global memory ------------------------------------------------------
    {
        const bool fin0 = (a.cur ^ (a.iterations & 1)) == 0;
        float4* fin = reinterpret_cast<float4*>(fin0 ? a.phi0 : a.phi1);
        float4* prv = reinterpret_cast<float4*>(fin0 ? a.phi1 : a.phi0);
#pragma unroll
        for (int k = 1; k <= ZC; ++k) {
            const size_t o4 = g4(z0 - 1 + k, y0 + r) + q;
            __stcg(fin + o4, cur[k]);
            __stcg(prv + o4, old[k]);
        }
    }

    // ---- gradient of the final level (gradient_x4_kernel's expressions) -------------------
    if (a.acc4 != nullptr) {
        const int x = 4 * q, y = y0 + r;
#pragma unroll
        for (int k = 1; k <= ZC; ++k) {
            const int z = z0 - 1 + k;
            const float4 c = cur[k];
            const float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
            const float rgt = __shfl_sync(0xffffffffu, c.x, rsrcl);
            const float d0 = x == 0 ? c.y - c.x : 0.5f * (c.y - lft);
            const float d1 = 0.5f * (c.z - c.x);
            const float d2 = 0.5f * (c.w - c.y);
            const float d3 = x + 4 == NX ? c.w - c.z : 0.5f * (rgt - c.z);
            const float4 ym = T4(k, r + 1)[q];
            const float4 yp = T4(k, r + 3)[q];
            float4 ey;
            if (y == 0) ey = make_float4(yp.x - c.x, yp.y - c.y, yp.z - c.z, yp.w - c.w);
            else if (y == NX - 1) ey = make_float4(c.x - ym.x, c.y - ym.y, c.z - ym.z, c.w - ym.w);
            else
                ey = make_float4(0.5f * (yp.x - ym.x), 0.5f * (yp.y - ym.y), 0.5f * (yp.z - ym.z),
                                 0.5f * (yp.w - ym.w));
            const float4 zm = cur[k - 1];
            const float4 zp = cur[k + 1];
            float4 ez;
            if (z == 0) ez = make_float4(zp.x - c.x, zp.y - c.y, zp.z - c.z, zp.w - c.w);
            else if (z == NX - 1) ez = make_float4(c.x - zm.x, c.y - zm.y, c.z - zm.z, c.w - zm.w);
            else
                ez = make_float4(0.5f * (zp.x - zm.x), 0.5f * (zp.y - zm.y), 0.5f * (zp.z - zm.z),
                                 0.5f * (zp.w - zm.w));
            const float g = a.grad_coef;
            // the warp's row (128 cells) staged through the source area (idle now), then stored
            // 512 contiguous bytes per instruction
            float4* const st = srcs + warp * 128;
            __syncwarp();
            st[4 * lane] = make_float4(d0 * g, ey.x * g, ez.x * g, c.x);
            st[4 * lane + 1] = make_float4(d1 * g, ey.y * g, ez.y * g, c.y);
            st[4 * lane + 2] = make_float4(d2 * g, ey.z * g, ez.z * g, c.z);
            st[4 * lane + 3] = make_float4(d3 * g, ey.w * g, ez.w * g, c.w);
            __syncwarp();
            float4* const o = a.acc4 + (static_cast<size_t>(z) * NX + y) * NX;
#pragma unroll
            for (int i = 0; i < 4; ++i) o[i * 32 + lane] = st[i * 32 + lane];
        }
    }
    // the counter ends at base + (passes) in every block: the next launch starts from there
}

bool use_tb() {
    // RRG_WAVE_TB=1 runs the two-substeps-per-exchange kernel on 128^3 (same bits); read once per
    // process, since the two kernels lay out the synchronisation memory differently
    static const bool on = [] {
        const char* e = std::getenv("RRG_WAVE_TB");
        return e && std::atoi(e) != 0;
    }();
    return on;
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
    if (nx == 128) return std::max(sync_bytes_for(block_count(nx)), sync_bytes_tb(128));
    return (nx == 32 || nx == 64) ? sync_bytes_for(block_count(nx)) : kFaceOffset;
}

bool launch_wave_solve(int nx, int iterations, float* phi0, float* phi1, int cur,
                       const unsigned long long* mg, unsigned long long* mg_zero, int shift_s,
                       double dx, double rho_sub, const WaveCoef& w, float* src, float4* acc4,
                       unsigned int* sync, size_t sync_bytes, cudaStream_t s) {
    if (!wave_solve_applicable(nx) || iterations < 1) return false;
    const bool tbk = nx == 128 && use_tb();
    const int W = nx / 4, RB = (tbk ? tb::T : kThreads) / W;
    const dim3 grid(nx / RB, nx / kZC);
    const int64_t nblocks = static_cast<int64_t>(grid.x) * grid.y;
    RRG_REQUIRE(nblocks * kCounterStride < kErrWord &&
                    sync_bytes >= (tbk ? sync_bytes_tb(nblocks) : sync_bytes_for(nblocks)),
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
            RRG_CUDA(cudaFuncSetAttribute(wave_solve_tb_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(tb::smem)));
            if (dev >= 0 && dev < 64) done[dev] = true;
        }
    }
    int per_sm = 0;
    if (tbk)
        RRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wave_solve_tb_kernel,
                                                               tb::T, tb::smem));
    else
        per_sm = W == 8 ? blocks_per_sm<8>() : (W == 16 ? blocks_per_sm<16>() : blocks_per_sm<32>());
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
    a.kf = 1.0f;
    a.kf_d = w.K_F;
    a.km_d = w.K_MAIN;
    a.kao_d = w.K_ACTUAL + w.K_OLD - 1.0;
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
    if (tbk) {
        cfg.blockDim = dim3(tb::T);
        cfg.dynamicSmemBytes = tb::smem;
        RRG_CUDA(cudaLaunchKernelEx(&cfg, wave_solve_tb_kernel, a));
    } else if (W == 8) {
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
