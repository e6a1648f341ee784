// Hand-written adjoint of the direct-sum leapfrog on sm_100a.
//
// Forward (nbody.cu:19-65): a_i = sum_j m_j d_ij f_ij, d_ij = x_j - x_i,
//   f_ij = (|d_ij|^2 + h_i + h_j)^(-3/2).
// With g_ij = -3 (|d_ij|^2 + h_i + h_j)^(-5/2) the Jacobian blocks are
//   da_i/dx_j = m_j (f_ij I + g_ij d_ij d_ij^T)   (j != i),   da_i/dx_i = -sum_j (same),
//   da_i/dm_j = d_ij f_ij.
// For a cotangent lam on a (vector-Jacobian product):
//   xbar_k = sum_j (f_kj u_kj + g_kj d_kj (d_kj . u_kj)),  u_kj = m_k lam_j - m_j lam_k
//   mbar_k = -sum_j f_kj (lam_j . d_kj)
// The self pair contributes exactly zero (d = 0, u = 0), so the loop runs over all j like the
// forward kernel: j-tiles of 256 through shared memory, split-j partials summed in FP64 in a
// fixed order.
//
// Leapfrog (predict_step_ / correct_step_, nbody.cu:122-181), one step n -> n+1:
//   x' = x + dt v + dt^2/2 a(x),   v' = v + dt/2 (a(x) + a(x')).
// Backward with cotangents (X, V) of (x_{n+1}, v_{n+1}), X already holding the path through
// a(x_{n+1}) into v_{n+1}:
//   V_n = dt X + V
//   c_n = dt^2/2 X + dt/2 V + dt/2 V_n      (the last term: v_n's own dependence on a(x_n),
//                                             absent for n = 0 where v_0 is an input)
//   X_n = X + J(x_n)^T c_n,   mbar += (da(x_n)/dm)^T c_n
// so each step costs one vector-Jacobian product at x_n. The forward keeps (x, v, a(x)) every
// K steps. Between checkpoints the states come back two ways:
//   FP64: recomputed forward from the checkpoint below (K - 2 force evaluations per K steps),
//         so the gradient is the exact adjoint of the forward trajectory;
//   FP32: the leapfrog run backwards from the checkpoint above (reverse_init_kernel,
//         vjp_reverse_finish), the force a(x_m) summed in the same pass over the pairs as the
//         VJP at x_m (3 more operations per pair instead of a separate force evaluation).
//         Each reversed step rounds once more than the forward did; every segment restarts
//         from an exact checkpoint.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "host_io.h"
#include "kernels.cuh"

namespace rrg {
namespace {

constexpr int kBS = 256;

template <typename R>
struct VjpParams {
    const V4<R>* posm;
    const R* hsoft;
    R uniform_h;
    int64_t n;
    int64_t jchunk;
    const V4<R>* lam;
    V4<R>* out;
    V4<R>* part;
    int accumulate;  // out += result instead of out = result
    V4<R>* part_a;   // force partials (kernels with FORCE)
};

// Backward elementwise update of one step (applied to X after the VJP of the step before):
//   V_n = dt X + V;  c = dt^2/2 X + dt/2 V + [n > 0] dt/2 V_n.  V == nullptr: none.
template <typename R>
struct AdjUpd {
    V4<R>* V = nullptr;
    V4<R>* c = nullptr;
    R dt = 0;
    int with_vn = 0;
};

template <typename R>
__device__ __forceinline__ void adjoint_update_at(int64_t i, R xx, R xy, R xz,
                                                  const AdjUpd<R>& u) {
    const V4<R> v = u.V[i];
    const R dt = u.dt, h = dt * R(0.5), h2 = dt * dt * R(0.5);
    const R vx = dt * xx + v.x, vy = dt * xy + v.y, vz = dt * xz + v.z;
    R cx = h2 * xx + h * v.x, cy = h2 * xy + h * v.y, cz = h2 * xz + h * v.z;
    if (u.with_vn) {
        cx += h * vx;
        cy += h * vy;
        cz += h * vz;
    }
    u.V[i] = v4<R>(vx, vy, vz, R(0));
    u.c[i] = v4<R>(cx, cy, cz, R(0));
}

// FP64: CUDA's rsqrt (within 1 ulp) instead of the forward's 1 / sqrt, whose square root and
// division each cost a Newton sequence; the VJP's pair loop is FP64-pipe bound, and the
// difference (a few 1e-16 relative per pair) is far below what any FP64 check resolves
template <typename R>
__device__ __forceinline__ R inv_sqrt(R x) {
    if constexpr (sizeof(R) == 4) return rsqrt_sfu(x);
    else return rsqrt(x);
}

// ----------------------------------------------------------------------------------------------
// FP32 VJP on Blackwell's paired FP32 instructions (add/mul/fma .f32x2): each thread owns two
// k-particles, k0 = base + tid and k1 = base + 256 + tid, as the two halves of float2 registers;
// the j-tile is staged pre-duplicated, (x, x, y, y) (z, z, m, m) (lx, lx, ly, ly) (lz, lz, h, h),
// so each shared-memory broadcast lands in the register pairs the paired instructions read.
// Per pair: d = x_j - x_k, r2 = |d|^2 + h_k + h_j, f = r2^-3/2, g3 = r2^-5/2,
//   u = m_k lam_j - m_j lam_k  (UMASS: lam_j - lam_k, the common mass applied once at the end),
//   A += f u,  B += g3 (d . u) d,  M += f (d . lam_j);
// then x-bar_k = A - 3 B (x m for UMASS), m-bar_k = -M. 26 FMA-pipe operations per pair with
// uniform mass and softening (29 in general) and one SFU reciprocal square root; the FMA pipe
// is the bound.
// Sums run tile-blocked (256 j) like the forward kernels; j-split partials are summed in FP64
// in a fixed order by vjp_finish. Padding j sits 1e18 away with zero mass and cotangent: its
// f and g3 flush to zero, so it adds exactly nothing.
constexpr float kVjpPad = 1e18f;

// MGRAD = false: the mass gradient is not wanted (w of the result is 0), 4 operations less.
// FORCE: the same pass also sums the force a_k = sum_j m_j f d (3 operations more, 4 with
// unequal masses) into p.part_a, and every result goes to the split partials (a finish pass
// always follows).
template <bool USOFT, bool UMASS, bool MGRAD, bool FORCE>
__global__ void __launch_bounds__(kBS, 2) vjp_f32x2_kernel(const VjpParams<float> p, float um) {
    __shared__ float4 s_xy[kBS];
    __shared__ float4 s_zm[kBS];
    __shared__ float4 s_lxy[kBS];
    __shared__ float4 s_lzh[kBS];
    const int tid = threadIdx.x;
    const int64_t n = p.n;
    const int64_t kbase = static_cast<int64_t>(blockIdx.x) * (2 * kBS);

    float2 nx, ny, nz, hs, mk, lkx, lky, lkz;
    {
        float v[2][4], l[2][3], h[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int64_t k = kbase + e * kBS + tid;
            V4<float> pk = v4<float>(0.f, 0.f, 0.f, 0.f), lk = pk;
            h[e] = p.uniform_h;
            if (k < n) {
                pk = p.posm[k];
                lk = p.lam[k];
                if constexpr (!USOFT) h[e] = p.hsoft[k];
            }
            v[e][0] = pk.x;
            v[e][1] = pk.y;
            v[e][2] = pk.z;
            v[e][3] = pk.w;
            l[e][0] = lk.x;
            l[e][1] = lk.y;
            l[e][2] = lk.z;
        }
        nx = make_float2(-v[0][0], -v[1][0]);
        ny = make_float2(-v[0][1], -v[1][1]);
        nz = make_float2(-v[0][2], -v[1][2]);
        mk = make_float2(v[0][3], v[1][3]);
        // lam_k enters u with a minus sign: keep it negated
        lkx = make_float2(-l[0][0], -l[1][0]);
        lky = make_float2(-l[0][1], -l[1][1]);
        lkz = make_float2(-l[0][2], -l[1][2]);
        hs = USOFT ? make_float2(2.f * p.uniform_h, 2.f * p.uniform_h) : make_float2(h[0], h[1]);
    }
    const float2 z2 = make_float2(0.f, 0.f);
    float2 Ax = z2, Ay = z2, Az = z2, Bx = z2, By = z2, Bz = z2, Mm = z2;
    float2 Fx = z2, Fy = z2, Fz = z2;

    const int64_t jb = static_cast<int64_t>(blockIdx.y) * p.jchunk;
    const int64_t je = min(n, jb + p.jchunk);
    V4<float> nxt = v4<float>(kVjpPad, kVjpPad, kVjpPad, 0.f), nxl = v4<float>(0.f, 0.f, 0.f, 0.f);
    float nxt_h = 1.f;
    {
        const int64_t j = jb + tid;
        if (j < je) {
            nxt = p.posm[j];
            nxl = p.lam[j];
            if constexpr (!USOFT) nxt_h = p.hsoft[j];
        }
    }
    for (int64_t j0 = jb; j0 < je; j0 += kBS) {
        __syncthreads();
        s_xy[tid] = make_float4(nxt.x, nxt.x, nxt.y, nxt.y);
        s_zm[tid] = make_float4(nxt.z, nxt.z, nxt.w, nxt.w);
        s_lxy[tid] = make_float4(nxl.x, nxl.x, nxl.y, nxl.y);
        s_lzh[tid] = make_float4(nxl.z, nxl.z, nxt_h, nxt_h);
        __syncthreads();
        {
            const int64_t j = j0 + kBS + tid;
            nxt = v4<float>(kVjpPad, kVjpPad, kVjpPad, 0.f);
            nxl = v4<float>(0.f, 0.f, 0.f, 0.f);
            nxt_h = 1.f;
            if (j < je) {
                nxt = p.posm[j];
                nxl = p.lam[j];
                if constexpr (!USOFT) nxt_h = p.hsoft[j];
            }
        }
        float2 tAx = z2, tAy = z2, tAz = z2, tBx = z2, tBy = z2, tBz = z2, tM = z2;
        float2 tFx = z2, tFy = z2, tFz = z2;
#pragma unroll 4
        for (int q = 0; q < kBS; ++q) {
            const float4 xy = s_xy[q], zm = s_zm[q], lxy = s_lxy[q], lzh = s_lzh[q];
            const float2 px = make_float2(xy.x, xy.y), py = make_float2(xy.z, xy.w);
            const float2 pz = make_float2(zm.x, zm.y);
            const float2 ljx = make_float2(lxy.x, lxy.y), ljy = make_float2(lxy.z, lxy.w);
            const float2 ljz = make_float2(lzh.x, lzh.y);
            const float2 dx = __fadd2_rn(px, nx);
            const float2 dy = __fadd2_rn(py, ny);
            const float2 dz = __fadd2_rn(pz, nz);
            const float2 s = USOFT ? hs : __fadd2_rn(hs, make_float2(lzh.z, lzh.w));
            const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, s)));
            // one SFU op per pair: a second (rcp for r2^-1) would make the SFU pipe the bound
            const float2 inv = make_float2(rsqrt_sfu(r2.x), rsqrt_sfu(r2.y));
            const float2 inv2 = __fmul2_rn(inv, inv);
            const float2 f = __fmul2_rn(inv, inv2);
            const float2 g3 = __fmul2_rn(f, inv2);
            float2 ux, uy, uz;
            if constexpr (UMASS) {
                ux = __fadd2_rn(ljx, lkx);
                uy = __fadd2_rn(ljy, lky);
                uz = __fadd2_rn(ljz, lkz);
            } else {
                const float2 mj = make_float2(zm.z, zm.w);
                ux = __ffma2_rn(mk, ljx, __fmul2_rn(mj, lkx));
                uy = __ffma2_rn(mk, ljy, __fmul2_rn(mj, lky));
                uz = __ffma2_rn(mk, ljz, __fmul2_rn(mj, lkz));
            }
            const float2 dot = __ffma2_rn(dz, uz, __ffma2_rn(dy, uy, __fmul2_rn(dx, ux)));
            const float2 t = __fmul2_rn(g3, dot);
            tAx = __ffma2_rn(f, ux, tAx);
            tAy = __ffma2_rn(f, uy, tAy);
            tAz = __ffma2_rn(f, uz, tAz);
            tBx = __ffma2_rn(t, dx, tBx);
            tBy = __ffma2_rn(t, dy, tBy);
            tBz = __ffma2_rn(t, dz, tBz);
            if constexpr (MGRAD) {
                const float2 dl = __ffma2_rn(dz, ljz, __ffma2_rn(dy, ljy, __fmul2_rn(dx, ljx)));
                tM = __ffma2_rn(f, dl, tM);
            }
            if constexpr (FORCE) {
                const float2 fm = UMASS ? f : __fmul2_rn(make_float2(zm.z, zm.w), f);
                tFx = __ffma2_rn(fm, dx, tFx);
                tFy = __ffma2_rn(fm, dy, tFy);
                tFz = __ffma2_rn(fm, dz, tFz);
            }
        }
        Ax = __fadd2_rn(Ax, tAx);
        Ay = __fadd2_rn(Ay, tAy);
        Az = __fadd2_rn(Az, tAz);
        Bx = __fadd2_rn(Bx, tBx);
        By = __fadd2_rn(By, tBy);
        Bz = __fadd2_rn(Bz, tBz);
        Mm = __fadd2_rn(Mm, tM);
        if constexpr (FORCE) {
            Fx = __fadd2_rn(Fx, tFx);
            Fy = __fadd2_rn(Fy, tFy);
            Fz = __fadd2_rn(Fz, tFz);
        }
    }
    const float sc = UMASS ? um : 1.f;
    const float gx[2] = {sc * (Ax.x - 3.f * Bx.x), sc * (Ax.y - 3.f * Bx.y)};
    const float gy[2] = {sc * (Ay.x - 3.f * By.x), sc * (Ay.y - 3.f * By.y)};
    const float gz[2] = {sc * (Az.x - 3.f * Bz.x), sc * (Az.y - 3.f * Bz.y)};
    const float gm[2] = {MGRAD ? -Mm.x : 0.f, MGRAD ? -Mm.y : 0.f};
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int64_t k = kbase + e * kBS + tid;
        if (k >= n) continue;
        if (FORCE || gridDim.y > 1) {
            const int64_t o = static_cast<int64_t>(blockIdx.y) * n + k;
            p.part[o] = v4<float>(gx[e], gy[e], gz[e], gm[e]);
            if constexpr (FORCE) {
                p.part_a[o] = e ? v4<float>(sc * Fx.y, sc * Fy.y, sc * Fz.y, 0.f)
                                : v4<float>(sc * Fx.x, sc * Fy.x, sc * Fz.x, 0.f);
            }
        } else if (p.accumulate) {
            const V4<float> o = p.out[k];
            p.out[k] = v4<float>(o.x + gx[e], o.y + gy[e], o.z + gz[e], o.w + gm[e]);
        } else {
            p.out[k] = v4<float>(gx[e], gy[e], gz[e], gm[e]);
        }
    }
}

// ----------------------------------------------------------------------------------------------
// Symmetric VJP: the pair term is antisymmetric (T_jk = -T_kj for x-bar), so each unordered
// pair of particles is evaluated once. Blocks run over tile pairs (a, b), a <= b, of 256
// particles: threads own k in tile a, tile b sits in shared memory. For a < b the j-side sums
// (x-bar_j -= T, m-bar_j += f (lam_k . d)) travel along the warp with the j they belong to (one
// shuffle per sum and step, see the kernel) and each warp adds its sums for a chunk of 32 j into
// a shared accumulator; block (a, b) then writes its tile-a sums to slot [a][b] and its
// tile-b sums to slot [b][a]. A finish pass adds the T slots of each particle in order
// (deterministic). Diagonal tiles evaluate only the k-side, as a non-symmetric pass would.
template <typename R>
struct VjpSymParams {
    const V4<R>* posm;
    const R* hsoft;
    R uniform_h;
    int64_t n;
    int tiles;
    const V4<R>* lam;
    V4<R>* slots;  // [tiles][tiles][256]
};


template <typename R, bool USOFT>
__global__ void __launch_bounds__(kBS) vjp_sym_kernel(const VjpSymParams<R> p) {
    __shared__ V4<R> s_pos[kBS];
    __shared__ V4<R> s_lam[kBS];
    __shared__ R s_h[USOFT ? 1 : kBS];
    __shared__ R s_acc[kBS][4];
    const int tid = threadIdx.x, lane = tid & 31;
    // upper-triangular (with diagonal) row-major tile-pair index -> (a, b)
    const int T = p.tiles;
    const int64_t t = blockIdx.x;
    auto S = [T](int64_t a) { return a * T - a * (a - 1) / 2; };
    const double B2 = 2.0 * T + 1.0;
    int64_t a = static_cast<int64_t>(floor((B2 - sqrt(B2 * B2 - 8.0 * static_cast<double>(t))) * 0.5));
    if (a < 0) a = 0;
    while (a + 1 < T && S(a + 1) <= t) ++a;
    while (a > 0 && S(a) > t) --a;
    const int64_t b = t - S(a) + a;

    const int64_t k = a * kBS + tid;
    V4<R> pk = v4<R>(R(1e18), R(1e18), R(1e18), R(0)), lk = v4<R>(0, 0, 0, 0);
    R hk = p.uniform_h;
    if (k < p.n) {
        pk = p.posm[k];
        lk = p.lam[k];
        if constexpr (!USOFT) hk = p.hsoft[k];
    }
    const int64_t j = b * kBS + tid;
    if (j < p.n) {
        s_pos[tid] = p.posm[j];
        s_lam[tid] = p.lam[j];
        if constexpr (!USOFT) s_h[tid] = p.hsoft[j];
    } else {
        s_pos[tid] = v4<R>(R(1e18), R(1e18), R(1e18), R(0));
        s_lam[tid] = v4<R>(0, 0, 0, 0);
        if constexpr (!USOFT) s_h[tid] = R(1);
    }
    s_acc[tid][0] = s_acc[tid][1] = s_acc[tid][2] = s_acc[tid][3] = R(0);
    __syncthreads();
    const bool sym = (a != b);
    R gx = 0, gy = 0, gz = 0, gm = 0;
    // one pair (k, j): its k-side terms into (gx, gy, gz, gm), its j-side ones returned
    auto pair = [&](int q, R& jx, R& jy, R& jz, R& jm) {
        const V4<R> pj = s_pos[q];
        const V4<R> lj = s_lam[q];
        const R dx = pj.x - pk.x, dy = pj.y - pk.y, dz = pj.z - pk.z;
        const R s = USOFT ? (hk + hk) : (hk + s_h[q]);
        const R r2 = dx * dx + dy * dy + dz * dz + s;
        const R inv = inv_sqrt(r2);
        const R inv2 = inv * inv;
        const R f = inv * inv2;
        const R g = R(-3) * f * inv2;
        const R ux = pk.w * lj.x - pj.w * lk.x;
        const R uy = pk.w * lj.y - pj.w * lk.y;
        const R uz = pk.w * lj.z - pj.w * lk.z;
        const R tt = g * (dx * ux + dy * uy + dz * uz);
        const R Tx = f * ux + tt * dx, Ty = f * uy + tt * dy, Tz = f * uz + tt * dz;
        gx += Tx;
        gy += Ty;
        gz += Tz;
        gm -= f * (dx * lj.x + dy * lj.y + dz * lj.z);
        jx = -Tx;
        jy = -Ty;
        jz = -Tz;
        jm = f * (dx * lk.x + dy * lk.y + dz * lk.z);
    };
    if (!sym) {
#pragma unroll 2
        for (int q = 0; q < kBS; ++q) {
            R jx, jy, jz, jm;
            pair(q, jx, jy, jz, jm);
        }
    } else {
        // the j-side terms ride along the warp: in step t of a chunk of 32 j, lane l takes
        // j = 32 c + (l + t) mod 32 and adds to the sums that lane l + 1 held for it, so after
        // 32 steps lane l holds its warp's sums for j = 32 c + l (one shuffle per sum and step,
        // and one shared add per chunk, instead of a warp reduction per j)
        for (int c = 0; c < kBS / 32; ++c) {
            R ax = 0, ay = 0, az = 0, am = 0;
#pragma unroll 4
            for (int t = 0; t < 32; ++t) {
                R jx, jy, jz, jm;
                pair(c * 32 + ((lane + t) & 31), jx, jy, jz, jm);
                const int from = (lane + 1) & 31;
                ax = __shfl_sync(0xffffffffu, ax + jx, from);
                ay = __shfl_sync(0xffffffffu, ay + jy, from);
                az = __shfl_sync(0xffffffffu, az + jz, from);
                am = __shfl_sync(0xffffffffu, am + jm, from);
            }
            atomicAdd(&s_acc[c * 32 + lane][0], ax);
            atomicAdd(&s_acc[c * 32 + lane][1], ay);
            atomicAdd(&s_acc[c * 32 + lane][2], az);
            atomicAdd(&s_acc[c * 32 + lane][3], am);
        }
    }
    p.slots[(a * T + b) * kBS + tid] = v4<R>(gx, gy, gz, gm);
    if (sym) {
        __syncthreads();
        p.slots[(b * T + a) * kBS + tid] =
            v4<R>(s_acc[tid][0], s_acc[tid][1], s_acc[tid][2], s_acc[tid][3]);
    }
}

template <typename R>
__global__ void vjp_sym_finish(int64_t n, int T, const V4<R>* __restrict__ slots,
                               V4<R>* __restrict__ out, int accumulate, const AdjUpd<R> upd) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t a = k / kBS, l = k % kBS;
    double sx = 0, sy = 0, sz = 0, sm = 0;
    for (int b = 0; b < T; ++b) {
        const V4<R> v = slots[(a * T + b) * kBS + l];
        sx += v.x;
        sy += v.y;
        sz += v.z;
        sm += v.w;
    }
    if (accumulate) {
        const V4<R> o = out[k];
        sx += o.x;
        sy += o.y;
        sz += o.z;
        sm += o.w;
    }
    const V4<R> r = v4<R>(static_cast<R>(sx), static_cast<R>(sy), static_cast<R>(sz),
                          static_cast<R>(sm));
    out[k] = r;
    if (upd.V) adjoint_update_at(k, r.x, r.y, r.z, upd);
}

template <typename R>
size_t vjp_sym_slot_bytes(int64_t n) {
    const int64_t T = (n + kBS - 1) / kBS;
    return sizeof(V4<R>) * static_cast<size_t>(T * T * kBS);
}

template <typename R>
void vjp_sym_launch(const void* posm, const void* hsoft, double uniform_h, int64_t n,
                    const void* lam, void* out, bool accumulate, void* slots,
                    cudaStream_t stream, const AdjUpd<R>& upd = AdjUpd<R>()) {
    const int T = static_cast<int>((n + kBS - 1) / kBS);
    VjpSymParams<R> p;
    p.posm = static_cast<const V4<R>*>(posm);
    p.hsoft = static_cast<const R*>(hsoft);
    p.uniform_h = static_cast<R>(uniform_h);
    p.n = n;
    p.tiles = T;
    p.lam = static_cast<const V4<R>*>(lam);
    p.slots = static_cast<V4<R>*>(slots);
    const unsigned blocks = static_cast<unsigned>(static_cast<int64_t>(T) * (T + 1) / 2);
    if (hsoft) vjp_sym_kernel<R, false><<<blocks, kBS, 0, stream>>>(p);
    else vjp_sym_kernel<R, true><<<blocks, kBS, 0, stream>>>(p);
    RRG_LAUNCHED();
    vjp_sym_finish<R><<<div_up(n, 256), 256, 0, stream>>>(n, T, p.slots, static_cast<V4<R>*>(out),
                                                          accumulate ? 1 : 0, upd);
    RRG_LAUNCHED();
}

template <typename R>
__global__ void vjp_finish(const VjpParams<R> p, int splits, const AdjUpd<R> upd) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= p.n) return;
    double sx = 0, sy = 0, sz = 0, sm = 0;
    for (int s = 0; s < splits; ++s) {
        const V4<R> v = p.part[static_cast<int64_t>(s) * p.n + k];
        sx += v.x;
        sy += v.y;
        sz += v.z;
        sm += v.w;
    }
    if (p.accumulate) {
        const V4<R> o = p.out[k];
        sx += o.x;
        sy += o.y;
        sz += o.z;
        sm += o.w;
    }
    const V4<R> r = v4<R>(static_cast<R>(sx), static_cast<R>(sy), static_cast<R>(sz),
                          static_cast<R>(sm));
    p.out[k] = r;
    if (upd.V) adjoint_update_at(k, r.x, r.y, r.z, upd);
}

// j-split count of the paired FP32 VJP: the smallest whose block count fills whole waves of
// resident blocks to within 2% of the best achievable (the rule of the forward kernels).
int vjp_f32x2_splits(int64_t n, int sms) {
    static int resident = 0;
    if (!resident) {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &nb, reinterpret_cast<const void*>(&vjp_f32x2_kernel<true, true, true, false>), kBS, 0) !=
                cudaSuccess ||
            nb < 1) {
            (void)cudaGetLastError();
            nb = 1;
        }
        resident = nb;
    }
    const int64_t kblocks = (n + 2 * kBS - 1) / (2 * kBS);
    const int64_t tiles = (n + kBS - 1) / kBS;
    const int64_t slots = static_cast<int64_t>(sms) * resident;
    double best = 0, eff[65] = {};
    const int64_t top = std::min<int64_t>(tiles, 64);
    for (int64_t sp = 1; sp <= top; ++sp) {
        const int64_t total = kblocks * sp;
        const int64_t waves = (total + slots - 1) / slots;
        eff[sp] = static_cast<double>(total) / static_cast<double>(waves * slots);
        best = std::max(best, eff[sp]);
    }
    for (int64_t sp = 1; sp <= top; ++sp)
        if (eff[sp] >= best - 0.02) return static_cast<int>(sp);
    return 1;
}

size_t vjp_f32x2_part_bytes(int64_t n, int splits) {
    return splits > 1 ? sizeof(V4<float>) * static_cast<size_t>(n) * splits : 0;
}

// uniform_m >= 0: every particle has this mass (the caller has checked).
void adjoint_update_launch(int64_t n, const void* X, const AdjUpd<float>& upd, cudaStream_t s);

// upd.V != nullptr: also applies the next step's adjoint update to out (= X) afterwards.
// mgrad = false: no mass gradient (the w slot gets 0, or keeps its value when accumulating).
void vjp_f32x2_launch(const void* posm, const void* hsoft, double uniform_h, double uniform_m,
                      int64_t n, const void* lam, void* out, bool accumulate, void* part,
                      int splits, cudaStream_t stream,
                      const AdjUpd<float>& upd = AdjUpd<float>(), bool mgrad = true) {
    const int64_t tiles = (n + kBS - 1) / kBS;
    const int64_t tiles_per = (tiles + splits - 1) / splits;
    const int real = static_cast<int>((tiles + tiles_per - 1) / tiles_per);
    VjpParams<float> p;
    p.posm = static_cast<const V4<float>*>(posm);
    p.hsoft = static_cast<const float*>(hsoft);
    p.uniform_h = static_cast<float>(uniform_h);
    p.n = n;
    p.jchunk = tiles_per * kBS;
    p.lam = static_cast<const V4<float>*>(lam);
    p.out = static_cast<V4<float>*>(out);
    p.part = static_cast<V4<float>*>(part);
    p.accumulate = accumulate ? 1 : 0;
    p.part_a = nullptr;
    RRG_REQUIRE(real == 1 || part != nullptr, RRG_ERR_STATE, "vjp: missing split partials");
    dim3 grid(static_cast<unsigned>((n + 2 * kBS - 1) / (2 * kBS)), real);
    const float um = uniform_m >= 0 ? static_cast<float>(uniform_m) : 1.f;
#define RRG_VJP2(US, UM, MG) vjp_f32x2_kernel<US, UM, MG, false><<<grid, kBS, 0, stream>>>(p, um)
#define RRG_VJP2_M(US, UM) \
    do {                   \
        if (mgrad)         \
            RRG_VJP2(US, UM, true); \
        else               \
            RRG_VJP2(US, UM, false); \
    } while (0)
    if (uniform_m >= 0) {
        if (hsoft) RRG_VJP2_M(false, true);
        else RRG_VJP2_M(true, true);
    } else {
        if (hsoft) RRG_VJP2_M(false, false);
        else RRG_VJP2_M(true, false);
    }
#undef RRG_VJP2_M
#undef RRG_VJP2
    RRG_LAUNCHED();
    if (real > 1) {
        vjp_finish<float><<<div_up(n, 256), 256, 0, stream>>>(p, real, upd);
        RRG_LAUNCHED();
    } else if (upd.V) {
        adjoint_update_launch(n, out, upd, stream);
    }
}

// ----------------------------------------------------------------------------------------------
// Reverse leapfrog between checkpoints (FP32 backward). The step x' = x + dt v + dt^2/2 a(x),
// v' = v + dt/2 (a(x) + a(x')) inverts exactly in real arithmetic:
//   w = v' - dt/2 a(x'),  x = x' - dt w,  v = w - dt/2 a(x),
// so the backward sweep rebuilds x_m from the state at m + 1, the force a(x_m) coming out of
// the same pass over the pairs as the VJP at x_m. In FP32 each reversed step rounds once more
// than the forward did, and every segment starts again from an exact checkpoint.
struct RevStep {
    const V4<float>* x;  // x_m (positions and masses)
    V4<float>* x_next;   // x_{m-1} out, or nullptr
    V4<float>* w;        // half-step velocity, updated in place: w -= dt a(x_m)
    float dt;
};

// Top of a segment: w = v - dt/2 a, x_out = x - dt w (mass carried).
__global__ void reverse_init_kernel(int64_t n, const V4<float>* __restrict__ x,
                                    const V4<float>* __restrict__ v,
                                    const V4<float>* __restrict__ a, V4<float>* __restrict__ w,
                                    V4<float>* __restrict__ x_out, float dt) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float h = 0.5f * dt;
    const V4<float> vi = v[i], ai = a[i], xi = x[i];
    const V4<float> wi = v4<float>(vi.x - h * ai.x, vi.y - h * ai.y, vi.z - h * ai.z, 0.f);
    w[i] = wi;
    x_out[i] = v4<float>(xi.x - dt * wi.x, xi.y - dt * wi.y, xi.z - dt * wi.z, xi.w);
}

// Finish of a FORCE pass at x_m: X += sum of the VJP partials (fixed order, FP64), a(x_m) from
// the force partials, w -= dt a, x_{m-1} = x_m - dt w, then the adjoint update of step m - 1.
__global__ void vjp_reverse_finish(const VjpParams<float> p, int splits, const AdjUpd<float> upd,
                                   const RevStep r) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= p.n) return;
    double sx = 0, sy = 0, sz = 0, sm = 0, ax = 0, ay = 0, az = 0;
    for (int s = 0; s < splits; ++s) {
        const int64_t o = static_cast<int64_t>(s) * p.n + k;
        const V4<float> v = p.part[o];
        sx += v.x;
        sy += v.y;
        sz += v.z;
        sm += v.w;
        const V4<float> a = p.part_a[o];
        ax += a.x;
        ay += a.y;
        az += a.z;
    }
    const V4<float> o = p.out[k];
    const V4<float> X = v4<float>(static_cast<float>(sx + o.x), static_cast<float>(sy + o.y),
                                  static_cast<float>(sz + o.z), static_cast<float>(sm + o.w));
    p.out[k] = X;
    V4<float> w = r.w[k];
    w.x -= r.dt * static_cast<float>(ax);
    w.y -= r.dt * static_cast<float>(ay);
    w.z -= r.dt * static_cast<float>(az);
    r.w[k] = w;
    if (r.x_next) {
        const V4<float> x = r.x[k];
        r.x_next[k] = v4<float>(x.x - r.dt * w.x, x.y - r.dt * w.y, x.z - r.dt * w.z, x.w);
    }
    if (upd.V) adjoint_update_at(k, X.x, X.y, X.z, upd);
}

// One reverse step at x_m = r.x: VJP with cotangent lam accumulated into out (= X), a(x_m),
// the reverse update of (w, positions) and the adjoint update upd. part / part_a hold
// [splits][n] V4 each.
void vjp_reverse_launch(const void* hsoft, double uniform_h, double uniform_m, int64_t n,
                        const void* lam, void* out, void* part, void* part_a, int splits,
                        cudaStream_t stream, const AdjUpd<float>& upd, const RevStep& r,
                        bool mgrad) {
    const int64_t tiles = (n + kBS - 1) / kBS;
    const int64_t tiles_per = (tiles + splits - 1) / splits;
    const int real = static_cast<int>((tiles + tiles_per - 1) / tiles_per);
    RRG_REQUIRE(part && part_a, RRG_ERR_STATE, "vjp: missing partials");
    VjpParams<float> p;
    p.posm = r.x;
    p.hsoft = static_cast<const float*>(hsoft);
    p.uniform_h = static_cast<float>(uniform_h);
    p.n = n;
    p.jchunk = tiles_per * kBS;
    p.lam = static_cast<const V4<float>*>(lam);
    p.out = static_cast<V4<float>*>(out);
    p.part = static_cast<V4<float>*>(part);
    p.accumulate = 1;
    p.part_a = static_cast<V4<float>*>(part_a);
    dim3 grid(static_cast<unsigned>((n + 2 * kBS - 1) / (2 * kBS)), real);
    const float um = uniform_m >= 0 ? static_cast<float>(uniform_m) : 1.f;
#define RRG_VJPF(US, UM, MG) vjp_f32x2_kernel<US, UM, MG, true><<<grid, kBS, 0, stream>>>(p, um)
#define RRG_VJPF_M(US, UM)          \
    do {                            \
        if (mgrad)                  \
            RRG_VJPF(US, UM, true); \
        else                        \
            RRG_VJPF(US, UM, false); \
    } while (0)
    if (uniform_m >= 0) {
        if (hsoft) RRG_VJPF_M(false, true);
        else RRG_VJPF_M(true, true);
    } else {
        if (hsoft) RRG_VJPF_M(false, false);
        else RRG_VJPF_M(true, false);
    }
#undef RRG_VJPF_M
#undef RRG_VJPF
    RRG_LAUNCHED();
    vjp_reverse_finish<<<div_up(n, 256), 256, 0, stream>>>(p, real, upd, r);
    RRG_LAUNCHED();
}

// Does every particle's mass equal posm[0].w?  flags[0] (zeroed by the caller) becomes 1 on a
// mismatch; flags[1] receives posm[0].w as double bits.
template <typename R>
__global__ void uniform_mass_kernel(int64_t n, const V4<R>* __restrict__ posm,
                                    unsigned long long* __restrict__ flags) {
    const R m0 = posm[0].w;
    bool same = true;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        same &= posm[i].w == m0;
    if (!__all_sync(0xffffffffu, same) && (threadIdx.x & 31) == 0) flags[0] = 1ull;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        flags[1] = static_cast<unsigned long long>(__double_as_longlong(static_cast<double>(m0)));
}

// ----------------------------------------------------------------------------------------------
// The adjoint update on its own (first step of the backward sweep, or no split finish to
// carry it)
template <typename R>
__global__ void adjoint_update_kernel(int64_t n, const V4<R>* __restrict__ X, const AdjUpd<R> upd) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V4<R> x = X[i];
    adjoint_update_at(i, x.x, x.y, x.z, upd);
}

void adjoint_update_launch(int64_t n, const void* X, const AdjUpd<float>& upd, cudaStream_t s) {
    adjoint_update_kernel<float><<<div_up(n, 256), 256, 0, s>>>(
        n, static_cast<const V4<float>*>(X), upd);
    RRG_LAUNCHED();
}

// c = s V (x, y, z; w = 0)
template <typename R>
__global__ void scale_xyz_kernel(int64_t n, const V4<R>* __restrict__ V, V4<R>* __restrict__ c,
                                 R s) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V4<R> v = V[i];
    c[i] = v4<R>(s * v.x, s * v.y, s * v.z, R(0));
}

struct ABuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~ABuf() {
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
            throw Error(RRG_ERR_NOMEM, std::string("adjoint: cudaMalloc failed: ") +
                                           cudaGetErrorString(e));
        }
        bytes = b;
    }
    char* c() const { return static_cast<char*>(p); }
};

}  // namespace

void launch_direct_vjp_f32(const void* posm, const void* hsoft, float uniform_hsoft, int64_t n,
                           const void* lam, void* out, cudaStream_t stream) {
    int dev = 0;
    RRG_CUDA(cudaGetDevice(&dev));
    const int splits = vjp_f32x2_splits(n, num_sms(dev));
    void* part = nullptr;
    const size_t pb = vjp_f32x2_part_bytes(n, splits);
    if (pb) RRG_CUDA(cudaMallocAsync(&part, pb, stream));
    try {
        vjp_f32x2_launch(posm, hsoft, uniform_hsoft, -1.0, n, lam, out, false, part, splits,
                         stream);
    } catch (...) {
        if (part) cudaFreeAsync(part, stream);
        throw;
    }
    if (part) RRG_CUDA(cudaFreeAsync(part, stream));
}

}  // namespace rrg

using namespace rrg;

// ================================================================================================
// Leapfrog adjoint object
// ================================================================================================
struct rrg_adjoint {
    int device = 0;
    int prec = RRG_PREC_FP32;
    size_t rsz = 4;
    int64_t n = 0;
    double dt = 0.0;
    int nsteps = 0;
    int every = 20;
    double uniform_h = 0.0;
    ABuf hsoft;
    ABuf ckpt_x, ckpt_v, ckpt_a;  // (nsteps / every + 1) x n x V4: state and a(x) there
    ABuf seg_x;            // (every + 1) x n x V4
    ABuf x, x2, v, a, u, X, V, c, g, xN, scratch, sym_slots;
    ABuf vjp_part;          // FP32: j-split partials of the paired VJP
    ABuf vjp_part_a;        // FP32: force partials of the reverse steps
    ABuf w;                 // FP32: half-step velocity of the reverse steps
    ABuf mflags;            // uniform-mass check: mismatch flag, mass bits
    int splits = 1;
    int vjp_splits = 1;
    double uniform_m = -1;  // >= 0 while every particle of the last forward has this mass
    bool mass_grad = true;  // compute dL/dm (the w slot of the position gradient)
    bool forward_done = false;
    std::string err;
};

namespace {

size_t vb(const rrg_adjoint* A) { return 4 * A->rsz * static_cast<size_t>(A->n); }

void forces(rrg_adjoint* A, const void* x, void* acc, cudaStream_t s) {
    DirectLaunch L;
    L.prec = A->prec;
    L.posm = x;
    L.hsoft = A->hsoft.p;
    L.uniform_hsoft = A->uniform_h;
    L.n = A->n;
    L.uniform_mass = A->uniform_m;
    L.epi.mode = EPI_STORE;
    L.epi.acc = acc;
    L.splits = A->splits;
    L.scratch = A->scratch.p;
    L.scratch_bytes = A->scratch.bytes;
    L.stream = s;
    launch_direct(L);
}

// Force evaluation at the positions `in` with the leapfrog epilogue. out != nullptr: correct,
// then the next step's predict (u, positions into out), storing the corrected v and a where
// vel / acc are given; out == nullptr: correct only, into vel and acc (both required).
void direct_step(rrg_adjoint* A, const void* in, void* out, void* vel, void* acc,
                 cudaStream_t s) {
    DirectLaunch L;
    L.prec = A->prec;
    L.posm = in;
    L.hsoft = A->hsoft.p;
    L.uniform_hsoft = A->uniform_h;
    L.uniform_mass = A->uniform_m;
    L.n = A->n;
    L.epi.mode = out ? EPI_CORRECT_PREDICT : EPI_CORRECT;
    L.epi.dt = A->dt;
    L.epi.u = A->u.p;
    L.epi.pos_out = out;
    L.epi.vel = vel;
    L.epi.acc = acc;
    L.splits = A->splits;
    L.scratch = A->scratch.p;
    L.scratch_bytes = A->scratch.bytes;
    L.stream = s;
    launch_direct(L);
}

// Where the forward keeps x_n: in its checkpoint slot on checkpoint steps, else in one of two
// work buffers (consecutive steps never share one).
char* forward_pos(rrg_adjoint* A, int n) {
    if (n % A->every == 0) return A->ckpt_x.c() + vb(A) * (n / A->every);
    return (n & 1) ? A->x.c() : A->x2.c();
}

// The adjoint update of step m (m < 0: none).
template <typename R>
AdjUpd<R> step_update(rrg_adjoint* A, int m) {
    AdjUpd<R> u;
    if (m < 0) return u;
    u.V = static_cast<V4<R>*>(A->V.p);
    u.c = static_cast<V4<R>*>(A->c.p);
    u.dt = static_cast<R>(A->dt);
    u.with_vn = m > 0 ? 1 : 0;
    return u;
}

// X += J(x)^T c, w slot += dm: the paired kernel in FP32, the symmetric one in FP64; then
// the update of step m (m >= 0) from the new X, in the same finish pass.
void vjp(rrg_adjoint* A, const void* x, int m, cudaStream_t s) {
    if (A->prec == RRG_PREC_FP64)
        vjp_sym_launch<double>(x, A->hsoft.p, A->uniform_h, A->n, A->c.p, A->X.p, true,
                               A->sym_slots.p, s, step_update<double>(A, m));
    else
        vjp_f32x2_launch(x, A->hsoft.p, A->uniform_h, A->uniform_m, A->n, A->c.p, A->X.p, true,
                         A->vjp_part.p, A->vjp_splits, s, step_update<float>(A, m),
                         A->mass_grad);
}

// Sets A->uniform_m from the masses in x (one small kernel and a 16-byte read-back).
void detect_uniform_mass(rrg_adjoint* A, const void* x, cudaStream_t s) {
    RRG_CUDA(cudaMemsetAsync(A->mflags.p, 0, 16, s));
    const int blocks = static_cast<int>(std::min<int64_t>(div_up(A->n, 256), 1184));
    if (A->prec == RRG_PREC_FP64)
        uniform_mass_kernel<double><<<blocks, 256, 0, s>>>(A->n, static_cast<const V4<double>*>(x),
                                                           static_cast<unsigned long long*>(A->mflags.p));
    else
        uniform_mass_kernel<float><<<blocks, 256, 0, s>>>(A->n, static_cast<const V4<float>*>(x),
                                                          static_cast<unsigned long long*>(A->mflags.p));
    RRG_LAUNCHED();
    unsigned long long f[2] = {1, 0};
    RRG_CUDA(cudaMemcpyAsync(f, A->mflags.p, 16, cudaMemcpyDeviceToHost, s));
    RRG_CUDA(cudaStreamSynchronize(s));
    double m = 0;
    std::memcpy(&m, &f[1], 8);
    A->uniform_m = (f[0] == 0 && m >= 0) ? m : -1.0;
}

#define ADJ_ENTRY(A, ...)                                                                    \
    try {                                                                                    \
        RRG_REQUIRE((A) != nullptr, RRG_ERR_INVALID, "null adjoint");                        \
        RRG_CUDA(cudaSetDevice((A)->device));                                               \
        __VA_ARGS__;                                                                         \
        return RRG_OK;                                                                       \
    } catch (const Error& x_) {                                                              \
        if (A) (A)->err = x_.what();                                                         \
        set_thread_error(x_.what());                                                         \
        return x_.code;                                                                      \
    }

}  // namespace

extern "C" {

RRG_API rrg_status rrg_dev_direct_vjp(const void* posm, const void* hsoft, double uniform_hsoft,
                                      int64_t n, const void* lam, void* out, int precision,
                                      void* stream) {
    try {
        RRG_REQUIRE(posm && lam && out && n > 0, RRG_ERR_INVALID, "rrg_dev_direct_vjp: bad args");
        RRG_REQUIRE(precision == RRG_PREC_FP32 || precision == RRG_PREC_FP64, RRG_ERR_INVALID,
                    "rrg_dev_direct_vjp: precision must be FP32 or FP64");
        int dev = 0;
        RRG_CUDA(cudaGetDevice(&dev));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (precision == RRG_PREC_FP32) {
            launch_direct_vjp_f32(posm, hsoft, static_cast<float>(uniform_hsoft), n, lam, out, s);
            return RRG_OK;
        }
        void* slots = nullptr;
        RRG_CUDA(cudaMallocAsync(&slots, vjp_sym_slot_bytes<double>(n), s));
        try {
            vjp_sym_launch<double>(posm, hsoft, uniform_hsoft, n, lam, out, false, slots, s);
        } catch (...) {
            cudaFreeAsync(slots, s);
            throw;
        }
        RRG_CUDA(cudaFreeAsync(slots, s));
        return RRG_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        return e.code;
    }
}

RRG_API rrg_status rrg_adjoint_create(int device, int precision, int64_t n, double dt,
                                      int nsteps, int checkpoint_every, const double* soft2,
                                      rrg_adjoint** out) {
    rrg_adjoint* A = nullptr;
    try {
        RRG_REQUIRE(out && soft2, RRG_ERR_INVALID, "rrg_adjoint_create: NULL argument");
        RRG_REQUIRE(precision == RRG_PREC_FP32 || precision == RRG_PREC_FP64, RRG_ERR_INVALID,
                    "rrg_adjoint_create: precision must be FP32 or FP64");
        RRG_REQUIRE(n >= 1 && n < (int64_t(1) << 31) && nsteps >= 1 && dt > 0,
                    RRG_ERR_INVALID, "rrg_adjoint_create: bad sizes or dt");
        RRG_CUDA(cudaSetDevice(device));
        A = new rrg_adjoint();
        A->device = device;
        A->prec = precision;
        A->rsz = precision == RRG_PREC_FP64 ? 8 : 4;
        A->n = n;
        A->dt = dt;
        A->nsteps = nsteps;
        A->every = checkpoint_every <= 0 ? nsteps : std::min(checkpoint_every, nsteps);
        bool uniform = true;
        for (int64_t i = 1; i < n && uniform; ++i) uniform = soft2[i] == soft2[0];
        A->uniform_h = 0.5 * soft2[0];
        if (!uniform) {
            A->hsoft.alloc(A->rsz * n);
            std::vector<double> h(n);
            for (int64_t i = 0; i < n; ++i) h[i] = 0.5 * soft2[i];
            if (A->rsz == 8) {
                RRG_CUDA(cudaMemcpy(A->hsoft.p, h.data(), 8 * n, cudaMemcpyHostToDevice));
            } else {
                std::vector<float> hf(h.begin(), h.end());
                RRG_CUDA(cudaMemcpy(A->hsoft.p, hf.data(), 4 * n, cudaMemcpyHostToDevice));
            }
        }
        const int nck = (nsteps + A->every - 1) / A->every + 1;
        A->ckpt_x.alloc(vb(A) * nck);
        A->ckpt_v.alloc(vb(A) * nck);
        A->ckpt_a.alloc(vb(A) * nck);
        if (precision == RRG_PREC_FP64) A->seg_x.alloc(vb(A) * (A->every + 1));
        for (ABuf* b : {&A->x, &A->x2, &A->v, &A->a, &A->u, &A->X, &A->V, &A->c, &A->g, &A->xN})
            b->alloc(vb(A));
        const int sms = num_sms(device);
        A->splits = direct_choose_splits(precision, n, sms);
        const size_t sb = direct_scratch_bytes(precision, n, A->splits);
        if (sb) A->scratch.alloc(sb);
        if (precision == RRG_PREC_FP64) {
            A->sym_slots.alloc(vjp_sym_slot_bytes<double>(n));
        } else {
            A->vjp_splits = vjp_f32x2_splits(n, sms);
            // the reverse steps write partials even with one split
            const size_t pb = sizeof(V4<float>) * static_cast<size_t>(n) *
                              static_cast<size_t>(std::max(1, A->vjp_splits));
            A->vjp_part.alloc(pb);
            A->vjp_part_a.alloc(pb);
            A->w.alloc(vb(A));
        }
        A->mflags.alloc(16);
        *out = A;
        return RRG_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        delete A;
        return e.code;
    }
}

RRG_API rrg_status rrg_adjoint_destroy(rrg_adjoint* A) {
    if (!A) return RRG_OK;
    cudaSetDevice(A->device);
    cudaDeviceSynchronize();
    delete A;
    return RRG_OK;
}

// Forward: nsteps leapfrog steps from (x0 = (x, y, z, m) per particle, v0), on caller device
// memory (V4 of the object's precision). Saves checkpoints; writes the final state.
RRG_API rrg_status rrg_adjoint_forward(rrg_adjoint* A, const void* x0, const void* v0,
                                       void* x_out, void* v_out, void* stream) {
    ADJ_ENTRY(A, {
        RRG_REQUIRE(x0 && v0, RRG_ERR_INVALID, "rrg_adjoint_forward: NULL input");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t b = vb(A);
        char* x_0 = A->ckpt_x.c();
        RRG_CUDA(cudaMemcpyAsync(x_0, x0, b, cudaMemcpyDeviceToDevice, s));
        RRG_CUDA(cudaMemcpyAsync(A->ckpt_v.p, v0, b, cudaMemcpyDeviceToDevice, s));
        detect_uniform_mass(A, x_0, s);
        forces(A, x_0, A->ckpt_a.p, s);
        // x_1 from (x_0, v_0, a_0); then one fused launch per step (correct + next predict),
        // checkpoints written by the epilogue itself
        char* x_1 = forward_pos(A, 1);
        RRG_CUDA(cudaMemcpyAsync(x_1, x_0, b, cudaMemcpyDeviceToDevice, s));
        launch_predict(A->prec, A->n, x_1, nullptr, A->ckpt_v.p, A->ckpt_a.p, A->u.p, A->dt, s);
        for (int n = 1; n < A->nsteps; ++n) {
            const bool ck = n % A->every == 0;
            const size_t k = static_cast<size_t>(n / A->every);
            direct_step(A, forward_pos(A, n), forward_pos(A, n + 1),
                        ck ? A->ckpt_v.c() + b * k : nullptr, ck ? A->ckpt_a.c() + b * k : nullptr,
                        s);
        }
        char* x_N = forward_pos(A, A->nsteps);
        direct_step(A, x_N, nullptr, A->v.p, A->a.p, s);
        RRG_CUDA(cudaMemcpyAsync(A->xN.p, x_N, b, cudaMemcpyDeviceToDevice, s));
        if (x_out) RRG_CUDA(cudaMemcpyAsync(x_out, x_N, b, cudaMemcpyDeviceToDevice, s));
        if (v_out) RRG_CUDA(cudaMemcpyAsync(v_out, A->v.p, b, cudaMemcpyDeviceToDevice, s));
        A->forward_done = true;
    })
}

// Backward: cotangents of the final (x, v) in, gradients of the initial (x, v, m) out.
// gx_out[i] = (dL/dx, dL/dy, dL/dz, dL/dm), gv_out[i] = (dL/dvx, dL/dvy, dL/dvz, 0).
RRG_API rrg_status rrg_adjoint_backward(rrg_adjoint* A, const void* gx_final,
                                        const void* gv_final, void* gx_out, void* gv_out,
                                        void* stream) {
    ADJ_ENTRY(A, {
        RRG_REQUIRE(A->forward_done, RRG_ERR_STATE, "rrg_adjoint_backward before forward");
        RRG_REQUIRE(gx_out && gv_out, RRG_ERR_INVALID, "rrg_adjoint_backward: NULL output");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t b = vb(A);
        // X (cotangent of x, w = accumulated mass gradient), V
        if (gx_final) RRG_CUDA(cudaMemcpyAsync(A->X.p, gx_final, b, cudaMemcpyDeviceToDevice, s));
        else RRG_CUDA(cudaMemsetAsync(A->X.p, 0, b, s));
        if (gv_final) RRG_CUDA(cudaMemcpyAsync(A->V.p, gv_final, b, cudaMemcpyDeviceToDevice, s));
        else RRG_CUDA(cudaMemsetAsync(A->V.p, 0, b, s));
        // the w slot of X accumulates dL/dm: start it at zero
        RRG_CUDA(cudaMemset2DAsync(A->X.c() + 3 * A->rsz, 4 * A->rsz, 0, A->rsz, A->n, s));
        if (gv_final) {
            // v_N = v_{N-1} + dt/2 (a_{N-1} + a(x_N)): the final velocity's own dependence on
            // a(x_N) reaches x_N (and m) through one product with cotangent dt/2 V_N
            const int bl = div_up(A->n, 256);
            if (A->prec == RRG_PREC_FP64)
                scale_xyz_kernel<double><<<bl, 256, 0, s>>>(A->n, static_cast<const V4<double>*>(A->V.p),
                                                            static_cast<V4<double>*>(A->c.p), 0.5 * A->dt);
            else
                scale_xyz_kernel<float><<<bl, 256, 0, s>>>(A->n, static_cast<const V4<float>*>(A->V.p),
                                                           static_cast<V4<float>*>(A->c.p),
                                                           static_cast<float>(0.5 * A->dt));
            RRG_LAUNCHED();
            vjp(A, A->xN.p, A->nsteps - 1, s);
        } else {
            const int bl = div_up(A->n, 256);
            const int m = A->nsteps - 1;
            if (A->prec == RRG_PREC_FP64)
                adjoint_update_kernel<double><<<bl, 256, 0, s>>>(
                    A->n, static_cast<const V4<double>*>(A->X.p), step_update<double>(A, m));
            else
                adjoint_update_kernel<float><<<bl, 256, 0, s>>>(
                    A->n, static_cast<const V4<float>*>(A->X.p), step_update<float>(A, m));
            RRG_LAUNCHED();
        }
        const int nseg = (A->nsteps + A->every - 1) / A->every;
        for (int seg = nseg - 1; seg >= 0 && A->prec == RRG_PREC_FP32; --seg) {
            // FP32: reverse steps from the state at the segment's top (the next checkpoint, or
            // the final state) down to n0 + 1, each one pass of the fused VJP + force kernel;
            // x_n0 is the checkpoint itself
            const int n0 = seg * A->every;
            const int n1 = std::min(A->nsteps, n0 + A->every);
            char* xc = A->ckpt_x.c() + b * seg;
            if (n1 - n0 > 1) {
                const bool last = seg == nseg - 1;
                const size_t top = static_cast<size_t>(seg + 1);
                const void* xt = last ? A->xN.p : A->ckpt_x.c() + b * top;
                const void* vt = last ? A->v.p : A->ckpt_v.c() + b * top;
                const void* at = last ? A->a.p : A->ckpt_a.c() + b * top;
                char* xbuf[2] = {A->x.c(), A->x2.c()};
                reverse_init_kernel<<<div_up(A->n, 256), 256, 0, s>>>(
                    A->n, static_cast<const V4<float>*>(xt), static_cast<const V4<float>*>(vt),
                    static_cast<const V4<float>*>(at), static_cast<V4<float>*>(A->w.p),
                    reinterpret_cast<V4<float>*>(xbuf[(n1 - 1) & 1]), static_cast<float>(A->dt));
                RRG_LAUNCHED();
                for (int m = n1 - 1; m > n0; --m) {
                    RevStep r;
                    r.x = reinterpret_cast<const V4<float>*>(xbuf[m & 1]);
                    r.x_next = m - 1 > n0 ? reinterpret_cast<V4<float>*>(xbuf[(m - 1) & 1]) : nullptr;
                    r.w = static_cast<V4<float>*>(A->w.p);
                    r.dt = static_cast<float>(A->dt);
                    vjp_reverse_launch(A->hsoft.p, A->uniform_h, A->uniform_m, A->n, A->c.p, A->X.p,
                                       A->vjp_part.p, A->vjp_part_a.p, A->vjp_splits, s,
                                       step_update<float>(A, m - 1), r, A->mass_grad);
                }
            }
            vjp(A, xc, n0 - 1, s);
        }
        for (int seg = nseg - 1; seg >= 0 && A->prec == RRG_PREC_FP64; --seg) {
            const int n0 = seg * A->every;
            const int n1 = std::min(A->nsteps, n0 + A->every);
            // FP64: recompute the segment from its checkpoint: x_n0 is the checkpoint itself, x_n for
            // n0 < n < n1 go to seg_x[n - n0] (a predict, then fused steps)
            char* xc = A->ckpt_x.c() + b * seg;
            if (n1 - n0 > 1) {
                char* x1 = A->seg_x.c() + b;
                RRG_CUDA(cudaMemcpyAsync(x1, xc, b, cudaMemcpyDeviceToDevice, s));
                launch_predict(A->prec, A->n, x1, nullptr, A->ckpt_v.c() + b * seg,
                               A->ckpt_a.c() + b * seg, A->u.p, A->dt, s);
                for (int jn = 1; jn + 1 < n1 - n0; ++jn)
                    direct_step(A, A->seg_x.c() + b * jn, A->seg_x.c() + b * (jn + 1), nullptr,
                                nullptr, s);
            }
            for (int n = n1 - 1; n >= n0; --n) {
                // X += J(x_n)^T c_n (and its w slot += dm), then step n - 1's update
                vjp(A, n == n0 ? xc : A->seg_x.c() + b * (n - n0), n - 1, s);
            }
        }
        if (!A->mass_grad)
            RRG_CUDA(cudaMemset2DAsync(A->X.c() + 3 * A->rsz, 4 * A->rsz, 0, A->rsz, A->n, s));
        RRG_CUDA(cudaMemcpyAsync(gx_out, A->X.p, b, cudaMemcpyDeviceToDevice, s));
        RRG_CUDA(cudaMemcpyAsync(gv_out, A->V.p, b, cudaMemcpyDeviceToDevice, s));
    })
}

RRG_API rrg_status rrg_adjoint_set_mass_gradient(rrg_adjoint* A, int enabled) {
    ADJ_ENTRY(A, { A->mass_grad = enabled != 0; })
}

}  // extern "C"
