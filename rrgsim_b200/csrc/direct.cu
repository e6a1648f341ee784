// Direct-sum softened gravity on sm_100a.
//
// Follows acceleration_kernel_blocked_ / grav_kernel_blocked_ (solver/lib/rrgsim_nbody/src/
// nbody.cu:19-114): every i sums over every j, self pair included, softening averaged as
// (soft2_i + soft2_j) / 2 (held here as h_i + h_j with h = soft2 / 2, which is the same value
// bit for bit). The reference's FP64 1/sqrt + cube becomes one SFU rsqrt and three multiplies.
//
// Layout: posm = float4 (x, y, z, m) per particle; j-tiles of 256 are staged through shared
// memory with a register prefetch of the next tile; each thread owns IPT i-particles so one
// shared-memory broadcast feeds IPT pair evaluations. Partial sums of one tile are formed in
// FP32 and folded into the running sum once per tile (blocked summation; Kahan-compensated in
// the MIXED precision). For small N the j-range is split over blockIdx.y and the partials are
// reduced in FP64 in a fixed order by a second kernel (deterministic).
#include <algorithm>
#include <cstdlib>

#include "kernels.cuh"

namespace rrg {
namespace {

constexpr int kBS = 256;         // threads per block = j-tile length
constexpr float kPadPos = 1e18f; // padding j: far away and massless -> contributes exactly 0

template <typename R>
struct EpiDev {
    int mode;
    R dt;
    V4<R>* acc;
    R* pot;
    V4<R>* vel;
    V4<R>* u;
    V4<R>* pos_out;
    V4<float>* lo_out;
};

template <typename R>
EpiDev<R> make_epi(const DirectEpi& e) {
    EpiDev<R> d;
    d.mode = e.mode;
    d.dt = static_cast<R>(e.dt);
    d.acc = static_cast<V4<R>*>(e.acc);
    d.pot = static_cast<R*>(e.pot);
    d.vel = static_cast<V4<R>*>(e.vel);
    d.u = static_cast<V4<R>*>(e.u);
    d.pos_out = static_cast<V4<R>*>(e.pos_out);
    d.lo_out = static_cast<V4<float>*>(e.lo_out);
    return d;
}

// Per-particle epilogue. Arithmetic order follows predict_step_ / correct_step_
// (nbody.cu:139-151, 175-180): v = 0.5 (u + dt a) with u = v_old + v*, v* = v + dt a,
// x += (dt 0.5) (v + v*).
template <typename R, bool MIXED>
__device__ __forceinline__ void apply_epi(const EpiDev<R>& e, int64_t i, R ax, R ay, R az,
                                          R phi, bool want_pot, const V4<R>* posm,
                                          const V4<float>* poslo) {
    if (want_pot && e.pot) e.pot[i] = phi;
    if (e.mode == EPI_STORE) {
        e.acc[i] = v4<R>(ax, ay, az, R(0));
        return;
    }
    const V4<R> u = e.u[i];
    const R dt = e.dt;
    const R vx = R(0.5) * (u.x + dt * ax);
    const R vy = R(0.5) * (u.y + dt * ay);
    const R vz = R(0.5) * (u.z + dt * az);
    if (e.mode == EPI_CORRECT) {
        e.vel[i] = v4<R>(vx, vy, vz, R(0));
        e.acc[i] = v4<R>(ax, ay, az, R(0));
        return;
    }
    // EPI_CORRECT_PREDICT: next step's predict on the corrected velocity; the synced (v, a)
    // of this step are stored too where the caller asks (checkpoints)
    if (e.vel) e.vel[i] = v4<R>(vx, vy, vz, R(0));
    if (e.acc) e.acc[i] = v4<R>(ax, ay, az, R(0));
    const R sx = vx + dt * ax, sy = vy + dt * ay, sz = vz + dt * az;  // v*
    const R ux = vx + sx, uy = vy + sy, uz = vz + sz;
    e.u[i] = v4<R>(ux, uy, uz, R(0));
    const R hdt = dt * R(0.5);
    const V4<R> p = posm[i];
    if constexpr (MIXED) {
        const V4<float> lo = poslo[i];
        float hx = p.x, lx = lo.x, hy = p.y, ly = lo.y, hz = p.z, lz = lo.z;
        df_add(hx, lx, hdt * ux);
        df_add(hy, ly, hdt * uy);
        df_add(hz, lz, hdt * uz);
        e.pos_out[i] = v4<R>(hx, hy, hz, p.w);
        e.lo_out[i] = v4<float>(lx, ly, lz, 0.f);
    } else {
        e.pos_out[i] = v4<R>(p.x + hdt * ux, p.y + hdt * uy, p.z + hdt * uz, p.w);
    }
}

struct F32Params {
    const V4<float>* posm;
    const V4<float>* poslo;
    const float* hsoft;
    float uniform_h;
    float uniform_m;     // every particle's mass when all are equal (UMASS kernels)
    int64_t n;
    int64_t jchunk;
    V4<float>* part_hi;  // [splits][n]
    V4<float>* part_lo;  // [splits][n] (MIXED)
    bool want_pot;
    EpiDev<float> epi;
};

template <int IPT, bool USOFT, bool MIXED, bool POT>
__global__ void __launch_bounds__(kBS, 2) direct_f32_kernel(const F32Params p) {
    __shared__ V4<float> s_pos[kBS];
    __shared__ float s_h[USOFT ? 1 : kBS];
    __shared__ V4<float> s_lo[MIXED ? kBS : 1];

    const int tid = threadIdx.x;
    const int64_t n = p.n;
    const int64_t ibase = static_cast<int64_t>(blockIdx.x) * (kBS * IPT);

    float xi[IPT], yi[IPT], zi[IPT], hi[IPT];
    float xl[IPT], yl[IPT], zl[IPT];
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
        const int64_t i = ibase + q * kBS + tid;
        V4<float> pi = v4<float>(0.f, 0.f, 0.f, 0.f);
        V4<float> li = v4<float>(0.f, 0.f, 0.f, 0.f);
        float h = p.uniform_h;
        if (i < n) {
            pi = p.posm[i];
            if constexpr (!USOFT) h = p.hsoft[i];
            if constexpr (MIXED) li = p.poslo[i];
        }
        xi[q] = pi.x; yi[q] = pi.y; zi[q] = pi.z;
        hi[q] = USOFT ? (p.uniform_h + p.uniform_h) : h;
        xl[q] = li.x; yl[q] = li.y; zl[q] = li.z;
    }

    float ax[IPT], ay[IPT], az[IPT], ap[IPT];
    float cx[IPT], cy[IPT], cz[IPT], cp[IPT];
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
        ax[q] = ay[q] = az[q] = ap[q] = 0.f;
        cx[q] = cy[q] = cz[q] = cp[q] = 0.f;
    }

    const int64_t jb = static_cast<int64_t>(blockIdx.y) * p.jchunk;
    const int64_t je = min(n, jb + p.jchunk);

    // register prefetch of the first tile
    V4<float> nxt_pos = v4<float>(kPadPos, kPadPos, kPadPos, 0.f);
    float nxt_h = 1.f;
    V4<float> nxt_lo = v4<float>(0.f, 0.f, 0.f, 0.f);
    {
        const int64_t j = jb + tid;
        if (j < je) {
            nxt_pos = p.posm[j];
            if constexpr (!USOFT) nxt_h = p.hsoft[j];
            if constexpr (MIXED) nxt_lo = p.poslo[j];
        }
    }

    for (int64_t j0 = jb; j0 < je; j0 += kBS) {
        __syncthreads();  // previous tile fully consumed
        s_pos[tid] = nxt_pos;
        if constexpr (!USOFT) s_h[tid] = nxt_h;
        if constexpr (MIXED) s_lo[tid] = nxt_lo;
        __syncthreads();
        {
            const int64_t j = j0 + kBS + tid;
            nxt_pos = v4<float>(kPadPos, kPadPos, kPadPos, 0.f);
            nxt_h = 1.f;
            nxt_lo = v4<float>(0.f, 0.f, 0.f, 0.f);
            if (j < je) {
                nxt_pos = p.posm[j];
                if constexpr (!USOFT) nxt_h = p.hsoft[j];
                if constexpr (MIXED) nxt_lo = p.poslo[j];
            }
        }

        float tx[IPT], ty[IPT], tz[IPT], tp[IPT];
#pragma unroll
        for (int q = 0; q < IPT; ++q) tx[q] = ty[q] = tz[q] = tp[q] = 0.f;

#pragma unroll 8
        for (int k = 0; k < kBS; ++k) {
            const V4<float> pj = s_pos[k];
            float hj = 0.f;
            if constexpr (!USOFT) hj = s_h[k];
            V4<float> lj;
            if constexpr (MIXED) lj = s_lo[k];
#pragma unroll
            for (int q = 0; q < IPT; ++q) {
                float dx = pj.x - xi[q];
                float dy = pj.y - yi[q];
                float dz = pj.z - zi[q];
                if constexpr (MIXED) {
                    dx += lj.x - xl[q];
                    dy += lj.y - yl[q];
                    dz += lj.z - zl[q];
                }
                const float s = USOFT ? hi[q] : (hi[q] + hj);
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, s)));
                const float inv = rsqrt_sfu(r2);
                const float minv = pj.w * inv;
                const float kk = minv * (inv * inv);
                tx[q] = fmaf(dx, kk, tx[q]);
                ty[q] = fmaf(dy, kk, ty[q]);
                tz[q] = fmaf(dz, kk, tz[q]);
                if constexpr (POT) tp[q] += minv;
            }
        }
#pragma unroll
        for (int q = 0; q < IPT; ++q) {
            if constexpr (MIXED) {
                kahan_add(ax[q], cx[q], tx[q]);
                kahan_add(ay[q], cy[q], ty[q]);
                kahan_add(az[q], cz[q], tz[q]);
                if constexpr (POT) kahan_add(ap[q], cp[q], tp[q]);
            } else {
                ax[q] += tx[q];
                ay[q] += ty[q];
                az[q] += tz[q];
                if constexpr (POT) ap[q] += tp[q];
            }
        }
    }

#pragma unroll
    for (int q = 0; q < IPT; ++q) {
        const int64_t i = ibase + q * kBS + tid;
        if (i >= n) continue;
        if (gridDim.y > 1) {
            const int64_t o = static_cast<int64_t>(blockIdx.y) * n + i;
            p.part_hi[o] = v4<float>(ax[q], ay[q], az[q], ap[q]);
            if constexpr (MIXED) p.part_lo[o] = v4<float>(-cx[q], -cy[q], -cz[q], -cp[q]);
        } else {
            float fx = ax[q], fy = ay[q], fz = az[q], fp = ap[q];
            if constexpr (MIXED) {
                fx -= cx[q];
                fy -= cy[q];
                fz -= cz[q];
                fp -= cp[q];
            }
            apply_epi<float, MIXED>(p.epi, i, fx, fy, fz, -fp, POT, p.posm, p.poslo);
        }
    }
}

// ----------------------------------------------------------------------------------------------
// Packed variant: Blackwell's paired FP32 instructions (add/mul/fma .f32x2) evaluate two pairs
// per instruction. Each thread owns 2 G i-particles held as G float2 lanes; the j-tile is
// staged pre-duplicated, (x, x, y, y) and (z, z, m, m), so every shared-memory broadcast
// lands directly in the register pairs the paired instructions read. Same arithmetic per pair
// as direct_f32_kernel (FP32 mode, tile-blocked summation).
// ----------------------------------------------------------------------------------------------
// UMASS: every particle has the mass p.uniform_m, which then multiplies the sums once at the
// end instead of every pair (11 FP32 operations per pair instead of 12). The massless padding
// of a last tile sits 1e18 away: its inv^3 flushes to zero and its inv adds below 1e-18.
template <int G, bool USOFT, bool POT, bool UMASS>
__global__ void __launch_bounds__(kBS, 2) direct_f32x2_kernel(const F32Params p) {
    __shared__ float4 s_xy[kBS];
    __shared__ float4 s_zm[kBS];
    __shared__ float2 s_h[USOFT ? 1 : kBS];
    constexpr int IPT = 2 * G;
    const int tid = threadIdx.x;
    const int64_t n = p.n;
    const int64_t ibase = static_cast<int64_t>(blockIdx.x) * (kBS * IPT);

    float2 nx[G], ny[G], nz[G], hs[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        float v[2][4];
        float h[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int64_t i = ibase + (2 * g + e) * kBS + tid;
            V4<float> pi = v4<float>(0.f, 0.f, 0.f, 0.f);
            h[e] = p.uniform_h;
            if (i < n) {
                pi = p.posm[i];
                if constexpr (!USOFT) h[e] = p.hsoft[i];
            }
            v[e][0] = pi.x;
            v[e][1] = pi.y;
            v[e][2] = pi.z;
        }
        nx[g] = make_float2(-v[0][0], -v[1][0]);
        ny[g] = make_float2(-v[0][1], -v[1][1]);
        nz[g] = make_float2(-v[0][2], -v[1][2]);
        hs[g] = USOFT ? make_float2(2.f * p.uniform_h, 2.f * p.uniform_h) : make_float2(h[0], h[1]);
    }
    float2 ax[G], ay[G], az[G], ap[G];
#pragma unroll
    for (int g = 0; g < G; ++g) ax[g] = ay[g] = az[g] = ap[g] = make_float2(0.f, 0.f);

    const int64_t jb = static_cast<int64_t>(blockIdx.y) * p.jchunk;
    const int64_t je = min(n, jb + p.jchunk);
    V4<float> nxt = v4<float>(kPadPos, kPadPos, kPadPos, 0.f);
    float nxt_h = 1.f;
    {
        const int64_t j = jb + tid;
        if (j < je) {
            nxt = p.posm[j];
            if constexpr (!USOFT) nxt_h = p.hsoft[j];
        }
    }
    for (int64_t j0 = jb; j0 < je; j0 += kBS) {
        __syncthreads();
        s_xy[tid] = make_float4(nxt.x, nxt.x, nxt.y, nxt.y);
        s_zm[tid] = make_float4(nxt.z, nxt.z, nxt.w, nxt.w);
        if constexpr (!USOFT) s_h[tid] = make_float2(nxt_h, nxt_h);
        __syncthreads();
        {
            const int64_t j = j0 + kBS + tid;
            nxt = v4<float>(kPadPos, kPadPos, kPadPos, 0.f);
            nxt_h = 1.f;
            if (j < je) {
                nxt = p.posm[j];
                if constexpr (!USOFT) nxt_h = p.hsoft[j];
            }
        }
        float2 tx[G], ty[G], tz[G], tp[G];
#pragma unroll
        for (int g = 0; g < G; ++g) tx[g] = ty[g] = tz[g] = tp[g] = make_float2(0.f, 0.f);
#pragma unroll 8
        for (int k = 0; k < kBS; ++k) {
            const float4 xy = s_xy[k];
            const float4 zm = s_zm[k];
            const float2 px = make_float2(xy.x, xy.y), py = make_float2(xy.z, xy.w);
            const float2 pz = make_float2(zm.x, zm.y), pm = make_float2(zm.z, zm.w);
            float2 hj = make_float2(0.f, 0.f);
            if constexpr (!USOFT) hj = s_h[k];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const float2 dx = __fadd2_rn(px, nx[g]);
                const float2 dy = __fadd2_rn(py, ny[g]);
                const float2 dz = __fadd2_rn(pz, nz[g]);
                const float2 s = USOFT ? hs[g] : __fadd2_rn(hs[g], hj);
                const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, s)));
                const float2 inv = make_float2(rsqrt_sfu(r2.x), rsqrt_sfu(r2.y));
                const float2 minv = UMASS ? inv : __fmul2_rn(pm, inv);
                const float2 kk = __fmul2_rn(minv, __fmul2_rn(inv, inv));
                tx[g] = __ffma2_rn(dx, kk, tx[g]);
                ty[g] = __ffma2_rn(dy, kk, ty[g]);
                tz[g] = __ffma2_rn(dz, kk, tz[g]);
                if constexpr (POT) tp[g] = __fadd2_rn(tp[g], minv);
            }
        }
#pragma unroll
        for (int g = 0; g < G; ++g) {
            ax[g] = __fadd2_rn(ax[g], tx[g]);
            ay[g] = __fadd2_rn(ay[g], ty[g]);
            az[g] = __fadd2_rn(az[g], tz[g]);
            if constexpr (POT) ap[g] = __fadd2_rn(ap[g], tp[g]);
        }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int64_t i = ibase + (2 * g + e) * kBS + tid;
            if (i >= n) continue;
            float fx = e ? ax[g].y : ax[g].x, fy = e ? ay[g].y : ay[g].x,
                  fz = e ? az[g].y : az[g].x, fp = e ? ap[g].y : ap[g].x;
            if constexpr (UMASS) {
                fx *= p.uniform_m;
                fy *= p.uniform_m;
                fz *= p.uniform_m;
                fp *= p.uniform_m;
            }
            if (gridDim.y > 1) {
                p.part_hi[static_cast<int64_t>(blockIdx.y) * n + i] = v4<float>(fx, fy, fz, fp);
            } else {
                apply_epi<float, false>(p.epi, i, fx, fy, fz, -fp, POT, p.posm, p.poslo);
            }
        }
    }
}

// Paired over j (variants 6 and 7): each thread holds G i-particles, and each f32x2 instruction
// takes one i against two consecutive j of the tile. One pair of shared-memory loads then feeds
// G x 2 pairs with G = 1 already (the i-paired kernel needs G = 2 for that, and so half as many
// blocks), and a block covers kBS x G particles. Shared layout per j-pair q:
// (x_2q, x_2q+1, y_2q, y_2q+1), (z_2q, z_2q+1, m_2q, m_2q+1), (h_2q, h_2q+1); each thread's two
// lanes (even and odd j) add at the end.
template <int G, bool USOFT, bool POT, bool UMASS>
__global__ void __launch_bounds__(kBS, 2) direct_f32jp_kernel(const F32Params p) {
    __shared__ float4 s_xy[kBS / 2];
    __shared__ float4 s_zm[kBS / 2];
    __shared__ float2 s_h[USOFT ? 1 : kBS / 2];
    const int tid = threadIdx.x;
    const int64_t n = p.n;
    const int64_t ibase = static_cast<int64_t>(blockIdx.x) * (kBS * G);

    float2 nx[G], ny[G], nz[G], hs[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int64_t i = ibase + g * kBS + tid;
        V4<float> pi = v4<float>(0.f, 0.f, 0.f, 0.f);
        float h = p.uniform_h;
        if (i < n) {
            pi = p.posm[i];
            if constexpr (!USOFT) h = p.hsoft[i];
        }
        nx[g] = make_float2(-pi.x, -pi.x);
        ny[g] = make_float2(-pi.y, -pi.y);
        nz[g] = make_float2(-pi.z, -pi.z);
        hs[g] = USOFT ? make_float2(2.f * p.uniform_h, 2.f * p.uniform_h) : make_float2(h, h);
    }
    float2 ax[G], ay[G], az[G], ap[G];
#pragma unroll
    for (int g = 0; g < G; ++g) ax[g] = ay[g] = az[g] = ap[g] = make_float2(0.f, 0.f);

    const int64_t jb = static_cast<int64_t>(blockIdx.y) * p.jchunk;
    const int64_t je = min(n, jb + p.jchunk);
    V4<float> nxt = v4<float>(kPadPos, kPadPos, kPadPos, 0.f);
    float nxt_h = 1.f;
    {
        const int64_t j = jb + tid;
        if (j < je) {
            nxt = p.posm[j];
            if constexpr (!USOFT) nxt_h = p.hsoft[j];
        }
    }
    float* const fxy = reinterpret_cast<float*>(s_xy);
    float* const fzm = reinterpret_cast<float*>(s_zm);
    float* const fh = reinterpret_cast<float*>(s_h);
    const int q0 = tid >> 1, e0 = tid & 1;
    for (int64_t j0 = jb; j0 < je; j0 += kBS) {
        __syncthreads();
        fxy[4 * q0 + e0] = nxt.x;
        fxy[4 * q0 + 2 + e0] = nxt.y;
        fzm[4 * q0 + e0] = nxt.z;
        fzm[4 * q0 + 2 + e0] = nxt.w;
        if constexpr (!USOFT) fh[2 * q0 + e0] = nxt_h;
        __syncthreads();
        {
            const int64_t j = j0 + kBS + tid;
            nxt = v4<float>(kPadPos, kPadPos, kPadPos, 0.f);
            nxt_h = 1.f;
            if (j < je) {
                nxt = p.posm[j];
                if constexpr (!USOFT) nxt_h = p.hsoft[j];
            }
        }
        float2 tx[G], ty[G], tz[G], tp[G];
#pragma unroll
        for (int g = 0; g < G; ++g) tx[g] = ty[g] = tz[g] = tp[g] = make_float2(0.f, 0.f);
#pragma unroll 8
        for (int q = 0; q < kBS / 2; ++q) {
            const float4 xy = s_xy[q];
            const float4 zm = s_zm[q];
            const float2 px = make_float2(xy.x, xy.y), py = make_float2(xy.z, xy.w);
            const float2 pz = make_float2(zm.x, zm.y), pm = make_float2(zm.z, zm.w);
            float2 hj = make_float2(0.f, 0.f);
            if constexpr (!USOFT) hj = s_h[q];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const float2 dx = __fadd2_rn(px, nx[g]);
                const float2 dy = __fadd2_rn(py, ny[g]);
                const float2 dz = __fadd2_rn(pz, nz[g]);
                const float2 s = USOFT ? hs[g] : __fadd2_rn(hs[g], hj);
                const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, s)));
                const float2 inv = make_float2(rsqrt_sfu(r2.x), rsqrt_sfu(r2.y));
                const float2 minv = UMASS ? inv : __fmul2_rn(pm, inv);
                const float2 kk = __fmul2_rn(minv, __fmul2_rn(inv, inv));
                tx[g] = __ffma2_rn(dx, kk, tx[g]);
                ty[g] = __ffma2_rn(dy, kk, ty[g]);
                tz[g] = __ffma2_rn(dz, kk, tz[g]);
                if constexpr (POT) tp[g] = __fadd2_rn(tp[g], minv);
            }
        }
#pragma unroll
        for (int g = 0; g < G; ++g) {
            ax[g] = __fadd2_rn(ax[g], tx[g]);
            ay[g] = __fadd2_rn(ay[g], ty[g]);
            az[g] = __fadd2_rn(az[g], tz[g]);
            if constexpr (POT) ap[g] = __fadd2_rn(ap[g], tp[g]);
        }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int64_t i = ibase + g * kBS + tid;
        if (i >= n) continue;
        float fx = ax[g].x + ax[g].y, fy = ay[g].x + ay[g].y, fz = az[g].x + az[g].y,
              fp = ap[g].x + ap[g].y;
        if constexpr (UMASS) {
            fx *= p.uniform_m;
            fy *= p.uniform_m;
            fz *= p.uniform_m;
            fp *= p.uniform_m;
        }
        if (gridDim.y > 1) {
            p.part_hi[static_cast<int64_t>(blockIdx.y) * n + i] = v4<float>(fx, fy, fz, fp);
        } else {
            apply_epi<float, false>(p.epi, i, fx, fy, fz, -fp, POT, p.posm, p.poslo);
        }
    }
}

// Fixed-order FP64 reduction of the split partials, then the epilogue.
template <bool MIXED>
__global__ void direct_f32_finish(const F32Params p, int splits) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    double sx = 0, sy = 0, sz = 0, sp = 0;
    for (int s = 0; s < splits; ++s) {
        const V4<float> h = p.part_hi[static_cast<int64_t>(s) * p.n + i];
        sx += h.x; sy += h.y; sz += h.z; sp += h.w;
        if constexpr (MIXED) {
            const V4<float> l = p.part_lo[static_cast<int64_t>(s) * p.n + i];
            sx += l.x; sy += l.y; sz += l.z; sp += l.w;
        }
    }
    apply_epi<float, MIXED>(p.epi, i, static_cast<float>(sx), static_cast<float>(sy),
                            static_cast<float>(sz), static_cast<float>(-sp), p.want_pot,
                            p.posm, p.poslo);
}

// ----------------------------------------------------------------------------------------------
// FP64: the reference arithmetic (1 / sqrt, cube), one i per thread.
// ----------------------------------------------------------------------------------------------
struct F64Params {
    const V4<double>* posm;
    const double* hsoft;
    double uniform_h;
    int64_t n;
    int64_t jchunk;
    V4<double>* part;
    bool want_pot;
    EpiDev<double> epi;
};

template <bool USOFT, bool POT>
__global__ void __launch_bounds__(kBS) direct_f64_kernel(const F64Params p) {
    __shared__ V4<double> s_pos[kBS];
    __shared__ double s_h[USOFT ? 1 : kBS];
    const int tid = threadIdx.x;
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kBS + tid;
    V4<double> pi = v4<double>(0, 0, 0, 0);
    double h = p.uniform_h;
    if (i < p.n) {
        pi = p.posm[i];
        if constexpr (!USOFT) h = p.hsoft[i];
    }
    double ax = 0, ay = 0, az = 0, ap = 0;
    const int64_t jb = static_cast<int64_t>(blockIdx.y) * p.jchunk;
    const int64_t je = min(p.n, jb + p.jchunk);
    for (int64_t j0 = jb; j0 < je; j0 += kBS) {
        const int64_t j = j0 + tid;
        __syncthreads();
        if (j < je) {
            s_pos[tid] = p.posm[j];
            if constexpr (!USOFT) s_h[tid] = p.hsoft[j];
        } else {
            s_pos[tid] = v4<double>(1e150, 1e150, 1e150, 0);
            if constexpr (!USOFT) s_h[tid] = 1.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < kBS; ++k) {
            const V4<double> pj = s_pos[k];
            const double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            const double hs = USOFT ? (h + h) : (h + s_h[k]);
            const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz + hs);
            const double kk = pj.w * (inv * inv * inv);
            ax += dx * kk;
            ay += dy * kk;
            az += dz * kk;
            if constexpr (POT) ap += pj.w * inv;
        }
    }
    if (i >= p.n) return;
    if (gridDim.y > 1) {
        p.part[static_cast<int64_t>(blockIdx.y) * p.n + i] = v4<double>(ax, ay, az, ap);
    } else {
        apply_epi<double, false>(p.epi, i, ax, ay, az, -ap, POT, p.posm, nullptr);
    }
}

__global__ void direct_f64_finish(const F64Params p, int splits) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    double sx = 0, sy = 0, sz = 0, sp = 0;
    for (int s = 0; s < splits; ++s) {
        const V4<double> h = p.part[static_cast<int64_t>(s) * p.n + i];
        sx += h.x; sy += h.y; sz += h.z; sp += h.w;
    }
    apply_epi<double, false>(p.epi, i, sx, sy, sz, -sp, p.want_pot, p.posm, nullptr);
}

// ----------------------------------------------------------------------------------------------
template <int IPT, bool MIXED, bool POT>
void dispatch_f32_soft(bool usoft, dim3 grid, const F32Params& p, cudaStream_t s) {
    if (usoft)
        direct_f32_kernel<IPT, true, MIXED, POT><<<grid, kBS, 0, s>>>(p);
    else
        direct_f32_kernel<IPT, false, MIXED, POT><<<grid, kBS, 0, s>>>(p);
}

template <int IPT>
void dispatch_f32(bool usoft, bool mixed, bool pot, dim3 grid, const F32Params& p,
                  cudaStream_t s) {
    if (mixed) {
        if (pot) dispatch_f32_soft<IPT, true, true>(usoft, grid, p, s);
        else dispatch_f32_soft<IPT, true, false>(usoft, grid, p, s);
    } else {
        if (pot) dispatch_f32_soft<IPT, false, true>(usoft, grid, p, s);
        else dispatch_f32_soft<IPT, false, false>(usoft, grid, p, s);
    }
}

// Kernel variants of the FP32 path: 1 = scalar, 1 i per thread; 2 = scalar, 2 i per thread;
// 3 = paired f32x2, 2 i per thread; 4 = paired f32x2, 4 i per thread; 5 = paired f32x2, 6 i
// per thread; 6 = paired over j, 1 i per thread; 7 = paired over j, 2 i per thread. MIXED and
// FP64 use the scalar kernels. RRG_DIRECT_VARIANT overrides the choice (for sweeps).
int env_variant() {
    static const int v = [] {
        const char* e = std::getenv("RRG_DIRECT_VARIANT");
        return e ? std::atoi(e) : 0;
    }();
    return v;
}

int variant_for(int prec, int64_t n) {
    if (prec == RRG_PREC_FP64) return 1;
    const int e = env_variant();
    if (prec == RRG_PREC_MIXED) return (e == 1 || e == 2) ? e : (n <= 16384 ? 1 : 2);
    if (e >= 1 && e <= 7) return e;
    // measured on B200 (Plummer, FP32, Gpairs/s at N = 16,384 / 65,536 / 262,144): paired
    // over i with 2 i-particles per thread 2220 / 2588 / 2607, with 4: 2057 / 2478 / 2669;
    // paired over j with 1: 2255 / 2672 / 2686, with 2: 2372 / 2722 / 2741
    return n < 16384 ? 3 : 7;
}

int ipt_of(int variant) {
    return variant == 1 || variant == 6 ? 1 : variant == 4 ? 4 : variant == 5 ? 6 : 2;
}

int ipt_for(int prec, int64_t n) { return ipt_of(variant_for(prec, n)); }

// Resident 256-thread blocks per SM of the kernel a variant launches (queried once).
int resident_blocks(int prec, int variant) {
    static int cache[3][8] = {};
    int& r = cache[prec][variant];
    if (r) return r;
    const void* k = nullptr;
    if (prec == RRG_PREC_FP64) k = reinterpret_cast<const void*>(&direct_f64_kernel<true, false>);
    else if (prec == RRG_PREC_MIXED)
        k = variant == 1 ? reinterpret_cast<const void*>(&direct_f32_kernel<1, true, true, false>)
                         : reinterpret_cast<const void*>(&direct_f32_kernel<2, true, true, false>);
    else if (variant == 1) k = reinterpret_cast<const void*>(&direct_f32_kernel<1, true, false, false>);
    else if (variant == 2) k = reinterpret_cast<const void*>(&direct_f32_kernel<2, true, false, false>);
    else if (variant == 3) k = reinterpret_cast<const void*>(&direct_f32x2_kernel<1, true, false, false>);
    else if (variant == 4) k = reinterpret_cast<const void*>(&direct_f32x2_kernel<2, true, false, false>);
    else if (variant == 5) k = reinterpret_cast<const void*>(&direct_f32x2_kernel<3, true, false, false>);
    else if (variant == 6) k = reinterpret_cast<const void*>(&direct_f32jp_kernel<1, true, false, false>);
    else k = reinterpret_cast<const void*>(&direct_f32jp_kernel<2, true, false, false>);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kBS, 0) != cudaSuccess || nb < 1) {
        (void)cudaGetLastError();
        nb = 1;
    }
    r = nb;
    return r;
}

}  // namespace

// j-split count: the smallest one whose block count fills whole waves of resident blocks to
// within 2% of the best achievable (wave quantisation is what costs at these sizes; each
// extra split only adds n x 16 B of partials and a tiny reduction). The count is a request:
// the launch rounds it to whole j-tile chunks, and on B200 that measured faster at N = 16,384
// than choosing among realisable counts only.
int direct_choose_splits(int prec, int64_t n, int sms) {
    const int variant = variant_for(prec, n);
    const int ipt = ipt_of(variant);
    const int64_t iblocks = (n + kBS * ipt - 1) / (kBS * ipt);
    const int64_t tiles = (n + kBS - 1) / kBS;
    const int64_t slots = static_cast<int64_t>(sms) * resident_blocks(prec, variant);
    double eff[65] = {};
    double best = 0.0;
    const int64_t top = std::min<int64_t>(tiles, 64);
    for (int64_t sp = 1; sp <= top; ++sp) {
        const int64_t total = iblocks * sp;
        const int64_t waves = (total + slots - 1) / slots;
        eff[sp] = static_cast<double>(total) / static_cast<double>(waves * slots);
        best = std::max(best, eff[sp]);
    }
    for (int64_t sp = 1; sp <= top; ++sp)
        if (eff[sp] >= best - 0.02) return static_cast<int>(sp);
    return 1;
}

size_t direct_scratch_bytes(int prec, int64_t n, int splits) {
    if (splits <= 1) return 0;
    const size_t per = (prec == RRG_PREC_FP64) ? sizeof(V4<double>)
                       : (prec == RRG_PREC_MIXED) ? 2 * sizeof(V4<float>)
                                                   : sizeof(V4<float>);
    return per * static_cast<size_t>(n) * static_cast<size_t>(splits);
}

void launch_direct(const DirectLaunch& L) {
    RRG_REQUIRE(L.n > 0, RRG_ERR_INVALID, "direct sum: n must be positive");
    const int splits = L.splits > 0 ? L.splits : 1;
    const int64_t tiles = (L.n + kBS - 1) / kBS;
    const int64_t tiles_per = (tiles + splits - 1) / splits;
    const int64_t jchunk = tiles_per * kBS;
    const int real_splits = static_cast<int>((tiles + tiles_per - 1) / tiles_per);
    RRG_REQUIRE(real_splits <= 1 || L.scratch_bytes >= direct_scratch_bytes(L.prec, L.n, real_splits),
                RRG_ERR_INVALID, "direct sum: scratch too small for the split count");
    RRG_REQUIRE(real_splits <= 1 || (reinterpret_cast<uintptr_t>(L.scratch) & 15u) == 0,
                RRG_ERR_INVALID, "direct sum: split partials must start on a 16-byte boundary");
    const bool usoft = (L.hsoft == nullptr);
    const int variant = (L.prec == RRG_PREC_FP32 && L.variant >= 1 && L.variant <= 7)
                            ? L.variant
                            : variant_for(L.prec, L.n);
    const int ipt = L.prec == RRG_PREC_FP64 ? 1 : ipt_of(variant);

    if (L.prec == RRG_PREC_FP64) {
        F64Params p;
        p.posm = static_cast<const V4<double>*>(L.posm);
        p.hsoft = static_cast<const double*>(L.hsoft);
        p.uniform_h = L.uniform_hsoft;
        p.n = L.n;
        p.jchunk = jchunk;
        p.part = static_cast<V4<double>*>(L.scratch);
        p.want_pot = L.want_pot;
        p.epi = make_epi<double>(L.epi);
        dim3 grid(static_cast<unsigned>((L.n + kBS - 1) / kBS), real_splits);
        if (usoft) {
            if (L.want_pot) direct_f64_kernel<true, true><<<grid, kBS, 0, L.stream>>>(p);
            else direct_f64_kernel<true, false><<<grid, kBS, 0, L.stream>>>(p);
        } else {
            if (L.want_pot) direct_f64_kernel<false, true><<<grid, kBS, 0, L.stream>>>(p);
            else direct_f64_kernel<false, false><<<grid, kBS, 0, L.stream>>>(p);
        }
        RRG_LAUNCHED();
        if (real_splits > 1) {
            direct_f64_finish<<<div_up(L.n, 256), 256, 0, L.stream>>>(p, real_splits);
            RRG_LAUNCHED();
        }
        return;
    }

    const bool mixed = (L.prec == RRG_PREC_MIXED);
    F32Params p;
    p.posm = static_cast<const V4<float>*>(L.posm);
    p.poslo = static_cast<const V4<float>*>(L.poslo);
    p.hsoft = static_cast<const float*>(L.hsoft);
    p.uniform_h = static_cast<float>(L.uniform_hsoft);
    p.n = L.n;
    p.jchunk = jchunk;
    p.part_hi = static_cast<V4<float>*>(L.scratch);
    p.part_lo = mixed && L.scratch
                    ? static_cast<V4<float>*>(L.scratch) + static_cast<size_t>(real_splits) * L.n
                    : nullptr;
    p.want_pot = L.want_pot;
    p.epi = make_epi<float>(L.epi);
    RRG_REQUIRE(!mixed || L.poslo != nullptr, RRG_ERR_INVALID,
                "direct sum: MIXED precision needs the low position parts");
    dim3 grid(static_cast<unsigned>((L.n + kBS * ipt - 1) / (kBS * ipt)), real_splits);
    if (variant >= 3) {
        const bool umass = L.uniform_mass >= 0.0;
        p.uniform_m = umass ? static_cast<float>(L.uniform_mass) : 0.f;
#define RRG_X2M(G, M)                                                                            \
    do {                                                                                         \
        if (usoft) {                                                                             \
            if (L.want_pot) direct_f32x2_kernel<G, true, true, M><<<grid, kBS, 0, L.stream>>>(p); \
            else direct_f32x2_kernel<G, true, false, M><<<grid, kBS, 0, L.stream>>>(p);          \
        } else {                                                                                 \
            if (L.want_pot) direct_f32x2_kernel<G, false, true, M><<<grid, kBS, 0, L.stream>>>(p);\
            else direct_f32x2_kernel<G, false, false, M><<<grid, kBS, 0, L.stream>>>(p);         \
        }                                                                                        \
    } while (0)
#define RRG_JPM(G, M)                                                                            \
    do {                                                                                         \
        if (usoft) {                                                                             \
            if (L.want_pot) direct_f32jp_kernel<G, true, true, M><<<grid, kBS, 0, L.stream>>>(p); \
            else direct_f32jp_kernel<G, true, false, M><<<grid, kBS, 0, L.stream>>>(p);          \
        } else {                                                                                 \
            if (L.want_pot) direct_f32jp_kernel<G, false, true, M><<<grid, kBS, 0, L.stream>>>(p);\
            else direct_f32jp_kernel<G, false, false, M><<<grid, kBS, 0, L.stream>>>(p);         \
        }                                                                                        \
    } while (0)
        if (variant == 3) {
            if (umass) RRG_X2M(1, true);
            else RRG_X2M(1, false);
        } else if (variant == 4) {
            if (umass) RRG_X2M(2, true);
            else RRG_X2M(2, false);
        } else if (variant == 5) {
            if (umass) RRG_X2M(3, true);
            else RRG_X2M(3, false);
        } else if (variant == 6) {
            if (umass) RRG_JPM(1, true);
            else RRG_JPM(1, false);
        } else {
            if (umass) RRG_JPM(2, true);
            else RRG_JPM(2, false);
        }
#undef RRG_X2M
#undef RRG_JPM
    } else if (ipt == 1) {
        dispatch_f32<1>(usoft, mixed, L.want_pot, grid, p, L.stream);
    } else {
        dispatch_f32<2>(usoft, mixed, L.want_pot, grid, p, L.stream);
    }
    RRG_LAUNCHED();
    if (real_splits > 1) {
        if (mixed) direct_f32_finish<true><<<div_up(L.n, 256), 256, 0, L.stream>>>(p, real_splits);
        else direct_f32_finish<false><<<div_up(L.n, 256), 256, 0, L.stream>>>(p, real_splits);
        RRG_LAUNCHED();
    }
}

}  // namespace rrg
