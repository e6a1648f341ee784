// Direct-sum forces for callers that cannot allocate device memory.
//
// rrg_dev_direct_forces_f32 takes its scratch (the per-particle potential and the partial sums
// of the j-splits) from the stream-ordered allocator on every call. Some callers cannot let a
// library allocate: a host application that reserves its whole device-memory budget up front,
// a plugin running inside another framework's memory manager, or a real-time loop that must
// not risk an allocation failing or stalling mid-run. This variant keeps its scratch in one
// file-scope device array of fixed size instead, so a call allocates nothing.
//
// The array is shared by every call on a device and keeps the previous call's contents; calls
// that overlap on the GPU (different streams, no ordering between them) race on it. Every
// scratch byte a call reads is written earlier in that same call, so nothing needs clearing.
#include <mutex>
#include <string>

#include "host_io.h"
#include "kernels.cuh"

namespace rrg {
namespace {

constexpr size_t kScratchBytes = size_t(4) << 20;  // 4 MiB per device, held until exit
constexpr int64_t kMaxN = int64_t(1) << 20;        // the potential alone fills 4 MiB at this n
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device. In host code the name g_scratch is only
// a host-side stand-in for the symbol, never a device address: it must be translated once per
// device, with that device current. The first call on a device does this.
void* scratch_address(int dev) {
    RRG_REQUIRE(dev >= 0 && dev < kMaxDevices, RRG_ERR_INVALID,
                "rrg_dev_direct_forces_f32_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        RRG_CUDA(cudaGetSymbolAddress(&p, g_scratch));
        g_addr[dev] = p;
    }
    return g_addr[dev];
}

}  // namespace
}  // namespace rrg

using namespace rrg;

extern "C" RRG_API rrg_status rrg_dev_direct_forces_f32_noalloc(const void* posm,
                                                                const void* hsoft,
                                                                float uniform_hsoft, int64_t n,
                                                                void* out, void* stream) {
    try {
        RRG_REQUIRE(posm && out, RRG_ERR_INVALID,
                    "rrg_dev_direct_forces_f32_noalloc: NULL pointer");
        RRG_REQUIRE(n >= 1 && n <= kMaxN, RRG_ERR_INVALID,
                    "rrg_dev_direct_forces_f32_noalloc: n = " + std::to_string(n) +
                        " is outside [1, 1048576], the size its fixed 4 MiB scratch serves");
        int dev = 0;
        RRG_CUDA(cudaGetDevice(&dev));
        char* base = static_cast<char*>(scratch_address(dev));
        cudaStream_t s = static_cast<cudaStream_t>(stream);

        // potential first (256-byte aligned), split partials behind it, all inside 4 MiB
        const size_t pot_bytes = (sizeof(float) * static_cast<size_t>(n) + 255) & ~size_t(255);
        int splits = direct_choose_splits(RRG_PREC_FP32, n, num_sms(dev));
        while (splits > 1 &&
               pot_bytes + direct_scratch_bytes(RRG_PREC_FP32, n, splits) > kScratchBytes)
            --splits;

        DirectLaunch L;
        L.prec = RRG_PREC_FP32;
        L.posm = posm;
        L.hsoft = hsoft;
        L.uniform_hsoft = uniform_hsoft;
        L.n = n;
        L.want_pot = true;
        L.epi.mode = EPI_STORE;
        L.epi.acc = out;
        L.epi.pot = base;
        L.splits = splits;
        L.scratch = splits > 1 ? base + pot_bytes : nullptr;
        L.scratch_bytes = splits > 1 ? kScratchBytes - pot_bytes : 0;
        L.stream = s;
        launch_direct(L);
        // out[i].w = potential[i]
        RRG_CUDA(cudaMemcpy2DAsync(static_cast<char*>(out) + 12, 16, base, 4, 4,
                                   static_cast<size_t>(n), cudaMemcpyDeviceToDevice, s));
        return RRG_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        return e.code;
    }
}
