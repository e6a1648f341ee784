// Order-independent FP64 sums of the conservation diagnostics (calc_conservation,
// nbody.cu:246-291; compute_center_of_mass_kernel, nbody.cu:293-396), shared by the
// conservation kernels (integrate.cu) and the fused particle pass (pm.cu), which folds the same
// sums into the last pass of a step.
//
// The sums are double-double (Knuth TwoSum / Fast2Sum carried through every addition, rounded
// once at the end): each result is the correctly rounded sum of the per-particle terms unless
// that exact sum lies within about 2^-100 of its magnitude of a rounding boundary, so it does
// not depend on the order of the particles in memory, which the cell sort changes, nor on how
// the particles are split among threads and blocks.
#pragma once

#include "common.cuh"

namespace rrg {

// values per block record: Ek, Ep (x2), momentum (3), angular momentum (3), then the mass
// centre's M and M x (4) when requested
constexpr int kRedVals = 12;
constexpr int kConsTerms = 8;

struct DD {
    double hi, lo;
};

__device__ __forceinline__ DD dd_norm(double s, double e) {
    const double hi = __dadd_rn(s, e);
    return DD{hi, __dsub_rn(e, __dsub_rn(hi, s))};
}

__device__ __forceinline__ DD dd_add(DD a, double b) {
    const double s = __dadd_rn(a.hi, b);
    const double bb = __dsub_rn(s, a.hi);
    const double e = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b, bb));
    return dd_norm(s, __dadd_rn(e, a.lo));
}

__device__ __forceinline__ DD dd_add(DD a, DD b) {
    const double s = __dadd_rn(a.hi, b.hi);
    const double bb = __dsub_rn(s, a.hi);
    const double e = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b.hi, bb));
    return dd_norm(s, __dadd_rn(e, __dadd_rn(a.lo, b.lo)));
}

__device__ __forceinline__ DD warp_sum_dd(DD v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        DD w;
        w.hi = __shfl_down_sync(0xffffffffu, v.hi, o);
        w.lo = __shfl_down_sync(0xffffffffu, v.lo, o);
        v = dd_add(v, w);
    }
    return v;
}

// Per thread each sum is cascaded (Ogita, Rump and Oishi's Sum2): s += x by TwoSum, and the
// rounding errors add up in c, 7 FP64 operations per term; (s, c) becomes a double-double for
// the warp, block and final reductions.
struct Casc {
    double s, c;
};

__device__ __forceinline__ void casc_add(Casc& a, double x) {
    const double t = __dadd_rn(a.s, x);
    const double z = __dsub_rn(t, a.s);
    a.c = __dadd_rn(a.c, __dadd_rn(__dsub_rn(a.s, __dsub_rn(t, z)), __dsub_rn(x, z)));
    a.s = t;
}

// Term k of one particle (nbody.cu:246-291): m |v|^2, m phi, m v, m (x cross v). Each operation
// is rounded separately, so every kernel that sums these forms the same terms.
__device__ __forceinline__ double cons_term(int k, double x, double y, double z, double m,
                                            double vx, double vy, double vz, double ph) {
    switch (k) {
        case 0:
            return __dmul_rn(m, __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)),
                                          __dmul_rn(vz, vz)));
        case 1: return __dmul_rn(m, ph);
        case 2: return __dmul_rn(m, vx);
        case 3: return __dmul_rn(m, vy);
        case 4: return __dmul_rn(m, vz);
        case 5: return __dmul_rn(m, __dsub_rn(__dmul_rn(vz, y), __dmul_rn(vy, z)));
        case 6: return __dmul_rn(m, __dsub_rn(__dmul_rn(vx, z), __dmul_rn(vz, x)));
        default: return __dmul_rn(m, __dsub_rn(__dmul_rn(vy, x), __dmul_rn(vx, y)));
    }
}

}  // namespace rrg
