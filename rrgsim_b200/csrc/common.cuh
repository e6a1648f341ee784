// Shared definitions for the sm_100a kernels and the C-ABI implementation.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "rrg.h"

namespace rrg {

// ---------------------------------------------------------------------------------------------
// Errors: every C-ABI entry point catches rrg::Error and turns it into a status code.
// ---------------------------------------------------------------------------------------------
struct Error : std::runtime_error {
    rrg_status code;
    Error(rrg_status c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

#define RRG_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t rrg_e_ = (call);                                                          \
        if (rrg_e_ != cudaSuccess)                                                            \
            throw ::rrg::Error(RRG_ERR_CUDA,                                                  \
                               std::string(#call) + ": " + cudaGetErrorString(rrg_e_));       \
    } while (0)

#define RRG_REQUIRE(cond, code, msg)                                                          \
    do {                                                                                      \
        if (!(cond)) throw ::rrg::Error((code), (msg));                                       \
    } while (0)

// Launch accounting: every kernel launch goes through rrg_launched(), graph replays add
// their kernel-node count. The counter is process-wide.
void count_launches(uint64_t n);
bool capturing_now();  // true while this thread records a CUDA graph (launches not counted)
void set_capturing(bool on);

#define RRG_LAUNCHED()                                                                        \
    do {                                                                                      \
        RRG_CUDA(cudaGetLastError());                                                         \
        if (!::rrg::capturing_now()) ::rrg::count_launches(1);                                \
    } while (0)

// ---------------------------------------------------------------------------------------------
// 4-wide vectors of float or double with natural vector alignment (one 16 B or 32 B access).
// ---------------------------------------------------------------------------------------------
template <typename R>
struct alignas(4 * sizeof(R)) V4 {
    R x, y, z, w;
};

template <typename R>
__host__ __device__ __forceinline__ V4<R> v4(R x, R y, R z, R w) {
    V4<R> v;
    v.x = x;
    v.y = y;
    v.z = z;
    v.w = w;
    return v;
}

// SFU reciprocal square root (one MUFU.RSQ); |rel err| ~ 2^-23.
__device__ __forceinline__ float rsqrt_sfu(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Error-free transformations for double-float arithmetic (Knuth TwoSum, Dekker Fast2Sum).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
__device__ __forceinline__ void fast_two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    e = __fsub_rn(b, __fsub_rn(s, a));
}
// (hi, lo) += d, renormalised.
__device__ __forceinline__ void df_add(float& hi, float& lo, float d) {
    float s, e;
    two_sum(hi, d, s, e);
    e = __fadd_rn(e, lo);
    fast_two_sum(s, e, hi, lo);
}
// Kahan compensated accumulation: sum += v with running compensation c (true = sum - c).
__device__ __forceinline__ void kahan_add(float& sum, float& c, float v) {
    float y = __fsub_rn(v, c);
    float t = __fadd_rn(sum, y);
    c = __fsub_rn(__fsub_rn(t, sum), y);
    sum = t;
}

// ---------------------------------------------------------------------------------------------
// Grid description shared by the PM kernels (passed by value; no __constant__ globals).
// ---------------------------------------------------------------------------------------------
struct GridDev {
    int nx;
    double dx;
    double domain_min;
    double inv_dx;   // 1 / dx (CIC uses a multiply, rm_p2mesh.cu:185)
    double sim_l;
};

inline int div_up(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

int num_sms(int device);

}  // namespace rrg
