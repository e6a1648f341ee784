// Leapfrog (predict/correct), FP64 diagnostics and state packing on sm_100a.
#include <cstdlib>

#include "kernels.cuh"
#include "sums.cuh"

namespace rrg {
namespace {

// predict_step_ (solver/lib/rrgsim_nbody/src/nbody.cu:122-152):
//   v* = v + dt a ;  x += dt 0.5 (v + v*)
// The sum v + v* is kept as u so correct_step_ (:159-181) can form 0.5 (v + v* + dt a_new).
template <typename R, bool MIXED>
__global__ void predict_kernel(int64_t n, V4<R>* __restrict__ posm, V4<float>* __restrict__ lo,
                               const V4<R>* __restrict__ vel, const V4<R>* __restrict__ acc,
                               V4<R>* __restrict__ u, R dt) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V4<R> v = vel[i];
    const V4<R> a = acc[i];
    const R sx = v.x + dt * a.x, sy = v.y + dt * a.y, sz = v.z + dt * a.z;
    const R ux = v.x + sx, uy = v.y + sy, uz = v.z + sz;
    u[i] = v4<R>(ux, uy, uz, R(0));
    const R hdt = dt * R(0.5);
    V4<R> p = posm[i];
    if constexpr (MIXED) {
        V4<float> l = lo[i];
        df_add(p.x, l.x, hdt * ux);
        df_add(p.y, l.y, hdt * uy);
        df_add(p.z, l.z, hdt * uz);
        lo[i] = l;
    } else {
        p.x = p.x + hdt * ux;
        p.y = p.y + hdt * uy;
        p.z = p.z + hdt * uz;
    }
    posm[i] = p;
}

template <typename R>
__global__ void correct_kernel(int64_t n, V4<R>* __restrict__ vel, const V4<R>* __restrict__ acc,
                               const V4<R>* __restrict__ u, R dt) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V4<R> a = acc[i];
    const V4<R> uu = u[i];
    vel[i] = v4<R>(R(0.5) * (uu.x + dt * a.x), R(0.5) * (uu.y + dt * a.y),
                   R(0.5) * (uu.z + dt * a.z), R(0));
}

// ---------------------------------------------------------------------------------------------
// FP64 reductions: per particle (promoted to double)
//   Ek2 += m v^2, Ep2 += m phi, P += m v, L += m (x cross v), M += m, Mx += m x
// Block partials are summed by one block in a fixed order.
// calc_conservation: nbody.cu:246-291; compute_center_of_mass_kernel: nbody.cu:293-396.
// ---------------------------------------------------------------------------------------------
constexpr int kRedThreads = 256;

// partial: [nblocks][kRedVals][2] (hi, lo). COM adds the four mass-centre sums (M, Mx); without
// it they stay 0.
template <typename R, bool MIXED, bool COM>
__global__ void __launch_bounds__(kRedThreads) conservation_kernel(
    int64_t n, const V4<R>* __restrict__ posm, const V4<float>* __restrict__ lo,
    const V4<R>* __restrict__ vel, const R* __restrict__ pot, double* __restrict__ partial) {
    constexpr int NV = COM ? kRedVals : 8;
    Casc acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = Casc{0.0, 0.0};
    // the next particle's loads are issued before this one's sums (a thread's FP64 chains
    // would otherwise wait out a memory latency per particle)
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    V4<R> pn{}, vn{};
    V4<float> ln{};
    R phn = R(0);
    if (i < n) {
        pn = posm[i];
        vn = vel[i];
        if constexpr (MIXED) ln = lo[i];
        if (pot) phn = pot[i];
    }
    for (; i < n; i += stride) {
        const V4<R> p = pn, v = vn;
        const V4<float> l = ln;
        const R ph = phn;
        const int64_t i2 = i + stride;
        if (i2 < n) {
            pn = posm[i2];
            vn = vel[i2];
            if constexpr (MIXED) ln = lo[i2];
            if (pot) phn = pot[i2];
        }
        double x = p.x, y = p.y, z = p.z;
        if constexpr (MIXED) {
            x += l.x;
            y += l.y;
            z += l.z;
        }
        const double m = p.w;
        const double vx = v.x, vy = v.y, vz = v.z;
        const double phd = pot ? static_cast<double>(ph) : 0.0;
#pragma unroll
        for (int k = 0; k < kConsTerms; ++k)
            casc_add(acc[k], cons_term(k, x, y, z, m, vx, vy, vz, phd));
        if constexpr (COM) {
            casc_add(acc[8], m);
            casc_add(acc[9], __dmul_rn(m, x));
            casc_add(acc[10], __dmul_rn(m, y));
            casc_add(acc[11], __dmul_rn(m, z));
        }
    }
    // block partials: every thread's sums go to shared memory, then warp w reduces values
    // w, w + 8, ...: each lane adds 8 threads' sums in order, then a fixed shuffle tree (about
    // a third of the FP64 work of a shuffle tree per value in every warp)
    __shared__ DD red[NV][kRedThreads];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) red[k][threadIdx.x] = dd_norm(acc[k].s, acc[k].c);
    __syncthreads();
    for (int k = w; k < kRedVals; k += kRedThreads / 32) {
        DD t{0.0, 0.0};
        if (k < NV) {
#pragma unroll
            for (int j = lane; j < kRedThreads; j += 32) t = dd_add(t, red[k][j]);
            t = warp_sum_dd(t);
        }
        if (lane == 0) {
            const int64_t o = (static_cast<int64_t>(blockIdx.x) * kRedVals + k) * 2;
            partial[o] = t.hi;
            partial[o + 1] = t.lo;
        }
    }
}

// One block per reduced value: thread t sums block partials t, t + 256, ... in order, then a
// fixed shuffle tree per warp and the warps in order, all in double-double; the result is its
// rounded high part. Value k of block b is the double-double at
// partial[(k kstride + b bstride) 2]; values from `nvals` on are zero. (Summing in the last
// block of the main kernel instead, with the other blocks counted by an atomic, measured
// slower: one block then does twelve blocks' work.)
__global__ void __launch_bounds__(kRedThreads) conservation_finish(
    const double* __restrict__ partial, int nblocks, int nvals, int64_t kstride,
    int64_t bstride, double* __restrict__ out) {
    const int k = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    DD t{0.0, 0.0};
    // eight records' loads are in flight before their additions (a thread that loaded one
    // record per addition waited out a memory latency per record)
    constexpr int U = 8;
    for (int b0 = threadIdx.x; b0 < nblocks && k < nvals; b0 += U * kRedThreads) {
        DD v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int b = b0 + u * kRedThreads;
            const int64_t o = (k * kstride + static_cast<int64_t>(b) * bstride) * 2;
            v[u] = b < nblocks ? DD{partial[o], partial[o + 1]} : DD{0.0, 0.0};
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (b0 + u * kRedThreads < nblocks) t = dd_add(t, v[u]);
    }
    t = warp_sum_dd(t);
    __shared__ DD s[kRedThreads / 32];
    if (lane == 0) s[w] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        DD r{0.0, 0.0};
        for (int ww = 0; ww < kRedThreads / 32; ++ww) r = dd_add(r, s[ww]);
        out[k] = r.hi;
    }
}

// Validity of uploaded particles, the largest mass and whether masses and softenings are
// uniform: grid-stride over the flat arrays (coalesced), one warp reduction and one atomic per
// warp and quantity.
__global__ void __launch_bounds__(256) check_state_kernel(
    int64_t n, const double* __restrict__ pos3, const double* __restrict__ vel3,
    const double* __restrict__ mass, const double* __restrict__ soft2, LoadCheck* chk) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    unsigned int bad_pv = 0, bad_m = 0, bad_s = 0, mv = 0, sv = 0;
    double mmax = 0.0;
    for (int64_t k = t0; k < 3 * n; k += stride) {
        if (!isfinite(__ldg(pos3 + k)) || !isfinite(__ldg(vel3 + k)))
            bad_pv = max(bad_pv, 0xffffffffu - static_cast<unsigned int>(k / 3));
    }
    const double m0 = __ldg(mass), s0 = __ldg(soft2);
    for (int64_t i = t0; i < n; i += stride) {
        const double m = __ldg(mass + i), h = __ldg(soft2 + i);
        if (!(isfinite(m) && m >= 0.0)) bad_m = max(bad_m, 0xffffffffu - static_cast<unsigned int>(i));
        else mmax = fmax(mmax, m);
        if (!(isfinite(h) && h >= 0.0)) bad_s = max(bad_s, 0xffffffffu - static_cast<unsigned int>(i));
        mv |= (m != m0);
        sv |= (h != s0);
    }
    bad_pv = __reduce_max_sync(0xffffffffu, bad_pv);
    bad_m = __reduce_max_sync(0xffffffffu, bad_m);
    bad_s = __reduce_max_sync(0xffffffffu, bad_s);
    mv = __reduce_or_sync(0xffffffffu, mv);
    sv = __reduce_or_sync(0xffffffffu, sv);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mmax = fmax(mmax, __shfl_xor_sync(0xffffffffu, mmax, o));
    if ((threadIdx.x & 31) == 0) {
        if (bad_pv) atomicMax(&chk->bad_pv, bad_pv);
        if (bad_m) atomicMax(&chk->bad_mass, bad_m);
        if (bad_s) atomicMax(&chk->bad_soft, bad_s);
        if (mv) atomicOr(&chk->mass_varies, 1u);
        if (sv) atomicOr(&chk->soft_varies, 1u);
        // non-negative doubles order as their bit patterns
        if (mmax > 0.0)
            atomicMax(&chk->mass_max_bits,
                      static_cast<unsigned long long>(__double_as_longlong(mmax)));
    }
}

// Host FP64 AoS -> device state.
template <typename R, bool MIXED>
__global__ void pack_kernel(int64_t n, const double* __restrict__ pos3,
                            const double* __restrict__ vel3, const double* __restrict__ mass,
                            const double* __restrict__ soft2, V4<R>* __restrict__ posm,
                            V4<float>* __restrict__ lo, V4<R>* __restrict__ vel,
                            R* __restrict__ hsoft) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = pos3[3 * i], y = pos3[3 * i + 1], z = pos3[3 * i + 2];
    posm[i] = v4<R>(static_cast<R>(x), static_cast<R>(y), static_cast<R>(z),
                    static_cast<R>(mass[i]));
    if constexpr (MIXED) {
        const float hx = static_cast<float>(x), hy = static_cast<float>(y),
                    hz = static_cast<float>(z);
        lo[i] = v4<float>(static_cast<float>(x - hx), static_cast<float>(y - hy),
                          static_cast<float>(z - hz), 0.f);
    }
    vel[i] = v4<R>(static_cast<R>(vel3[3 * i]), static_cast<R>(vel3[3 * i + 1]),
                   static_cast<R>(vel3[3 * i + 2]), R(0));
    if (hsoft) hsoft[i] = static_cast<R>(0.5 * soft2[i]);
}

template <typename R, bool MIXED>
__global__ void unpack_kernel(int64_t n, const int32_t* __restrict__ id,
                              const V4<R>* __restrict__ posm, const V4<float>* __restrict__ lo,
                              const V4<R>* __restrict__ vel, const V4<R>* __restrict__ acc,
                              const R* __restrict__ pot, double* __restrict__ pos3,
                              double* __restrict__ vel3, double* __restrict__ acc3,
                              double* __restrict__ grav) {
    const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t i = id ? static_cast<int64_t>(id[s]) : s;
    if (pos3) {
        const V4<R> p = posm[s];
        double x = p.x, y = p.y, z = p.z;
        if constexpr (MIXED) {
            const V4<float> l = lo[s];
            x += l.x;
            y += l.y;
            z += l.z;
        }
        pos3[3 * i] = x;
        pos3[3 * i + 1] = y;
        pos3[3 * i + 2] = z;
    }
    if (vel3) {
        const V4<R> v = vel[s];
        vel3[3 * i] = v.x;
        vel3[3 * i + 1] = v.y;
        vel3[3 * i + 2] = v.z;
    }
    if (acc3) {
        const V4<R> a = acc[s];
        acc3[3 * i] = a.x;
        acc3[3 * i + 1] = a.y;
        acc3[3 * i + 2] = a.z;
    }
    if (grav) grav[i] = pot[s];
}

}  // namespace

void launch_predict(int prec, int64_t n, void* posm, void* poslo, const void* vel,
                    const void* acc, void* u, double dt, cudaStream_t s) {
    const int b = div_up(n, 256);
    if (prec == RRG_PREC_FP64)
        predict_kernel<double, false><<<b, 256, 0, s>>>(
            n, static_cast<V4<double>*>(posm), nullptr, static_cast<const V4<double>*>(vel),
            static_cast<const V4<double>*>(acc), static_cast<V4<double>*>(u), dt);
    else if (prec == RRG_PREC_MIXED)
        predict_kernel<float, true><<<b, 256, 0, s>>>(
            n, static_cast<V4<float>*>(posm), static_cast<V4<float>*>(poslo),
            static_cast<const V4<float>*>(vel), static_cast<const V4<float>*>(acc),
            static_cast<V4<float>*>(u), static_cast<float>(dt));
    else
        predict_kernel<float, false><<<b, 256, 0, s>>>(
            n, static_cast<V4<float>*>(posm), nullptr, static_cast<const V4<float>*>(vel),
            static_cast<const V4<float>*>(acc), static_cast<V4<float>*>(u),
            static_cast<float>(dt));
    RRG_LAUNCHED();
}

void launch_correct(int prec, int64_t n, void* vel, const void* acc, const void* u, double dt,
                    cudaStream_t s) {
    const int b = div_up(n, 256);
    if (prec == RRG_PREC_FP64)
        correct_kernel<double><<<b, 256, 0, s>>>(n, static_cast<V4<double>*>(vel),
                                                 static_cast<const V4<double>*>(acc),
                                                 static_cast<const V4<double>*>(u), dt);
    else
        correct_kernel<float><<<b, 256, 0, s>>>(n, static_cast<V4<float>*>(vel),
                                                static_cast<const V4<float>*>(acc),
                                                static_cast<const V4<float>*>(u),
                                                static_cast<float>(dt));
    RRG_LAUNCHED();
}

// Two blocks per SM: the sums are FP64-bound, and few partials keep the final pass short.
// RRG_CONS_BLOCKS caps the block count (for sweeps; the partial buffer is sized from this).
// 592 (4 per SM) measured best at 2^20 particles: 296 left the FP64 chains latency-bound,
// more blocks cost more in the per-block epilogue than they gain.
int conservation_blocks(int64_t n) {
    static const int cap = [] {
        const char* e = std::getenv("RRG_CONS_BLOCKS");
        const int v = e ? std::atoi(e) : 0;
        return v > 0 ? v : 592;
    }();
    const int b = div_up(n, kRedThreads);
    return b < cap ? (b < 1 ? 1 : b) : cap;
}

void launch_conservation(int prec, int64_t n, const void* posm, const void* poslo,
                         const void* vel, const void* pot, double* partial, int nblocks,
                         double* out, cudaStream_t s, bool com) {
#define RRG_CONS(R, MX, C, LO)                                                               \
    conservation_kernel<R, MX, C><<<nblocks, kRedThreads, 0, s>>>(                            \
        n, static_cast<const V4<R>*>(posm), LO, static_cast<const V4<R>*>(vel),               \
        static_cast<const R*>(pot), partial)
    const V4<float>* lo = static_cast<const V4<float>*>(poslo);
    if (prec == RRG_PREC_FP64) {
        if (com) RRG_CONS(double, false, true, nullptr);
        else RRG_CONS(double, false, false, nullptr);
    } else if (prec == RRG_PREC_MIXED) {
        if (com) RRG_CONS(float, true, true, lo);
        else RRG_CONS(float, true, false, lo);
    } else {
        if (com) RRG_CONS(float, false, true, nullptr);
        else RRG_CONS(float, false, false, nullptr);
    }
#undef RRG_CONS
    RRG_LAUNCHED();
    conservation_finish<<<kRedVals, kRedThreads, 0, s>>>(partial, nblocks, kRedVals, 1,
                                                          kRedVals, out);
    RRG_LAUNCHED();
}

void launch_conservation_finish_value_major(const double* partial, int nblocks, int nvals,
                                            double* out, cudaStream_t s) {
    conservation_finish<<<kRedVals, kRedThreads, 0, s>>>(partial, nblocks, nvals, nblocks, 1,
                                                          out);
    RRG_LAUNCHED();
}

void launch_check_state(int64_t n, const double* pos3, const double* vel3, const double* mass,
                        const double* soft2, LoadCheck* chk, int sms, cudaStream_t s) {
    const int b = std::max(1, std::min(div_up(3 * n, 256), 4 * sms));
    check_state_kernel<<<b, 256, 0, s>>>(n, pos3, vel3, mass, soft2, chk);
    RRG_LAUNCHED();
}

void launch_pack_state(int prec, int64_t n, const double* pos3, const double* vel3,
                       const double* mass, const double* soft2, void* posm, void* poslo,
                       void* vel, void* hsoft, cudaStream_t s) {
    const int b = div_up(n, 256);
    if (prec == RRG_PREC_FP64)
        pack_kernel<double, false><<<b, 256, 0, s>>>(
            n, pos3, vel3, mass, soft2, static_cast<V4<double>*>(posm), nullptr,
            static_cast<V4<double>*>(vel), static_cast<double*>(hsoft));
    else if (prec == RRG_PREC_MIXED)
        pack_kernel<float, true><<<b, 256, 0, s>>>(
            n, pos3, vel3, mass, soft2, static_cast<V4<float>*>(posm),
            static_cast<V4<float>*>(poslo), static_cast<V4<float>*>(vel),
            static_cast<float*>(hsoft));
    else
        pack_kernel<float, false><<<b, 256, 0, s>>>(
            n, pos3, vel3, mass, soft2, static_cast<V4<float>*>(posm), nullptr,
            static_cast<V4<float>*>(vel), static_cast<float*>(hsoft));
    RRG_LAUNCHED();
}

void launch_unpack_state(int prec, int64_t n, const int32_t* id, const void* posm,
                         const void* poslo, const void* vel, const void* acc, const void* pot,
                         double* pos3, double* vel3, double* acc3, double* grav,
                         cudaStream_t s) {
    const int b = div_up(n, 256);
    if (prec == RRG_PREC_FP64)
        unpack_kernel<double, false><<<b, 256, 0, s>>>(
            n, id, static_cast<const V4<double>*>(posm), nullptr,
            static_cast<const V4<double>*>(vel), static_cast<const V4<double>*>(acc),
            static_cast<const double*>(pot), pos3, vel3, acc3, grav);
    else if (prec == RRG_PREC_MIXED)
        unpack_kernel<float, true><<<b, 256, 0, s>>>(
            n, id, static_cast<const V4<float>*>(posm), static_cast<const V4<float>*>(poslo),
            static_cast<const V4<float>*>(vel), static_cast<const V4<float>*>(acc),
            static_cast<const float*>(pot), pos3, vel3, acc3, grav);
    else
        unpack_kernel<float, false><<<b, 256, 0, s>>>(
            n, id, static_cast<const V4<float>*>(posm), nullptr,
            static_cast<const V4<float>*>(vel), static_cast<const V4<float>*>(acc),
            static_cast<const float*>(pot), pos3, vel3, acc3, grav);
    RRG_LAUNCHED();
}

}  // namespace rrg
