// Counting sort of the particles by CIC base cell on sm_100a.
//
// Particles that share a base cell deposit into the same eight grid cells and gather from the
// same eight field cells. Stored next to each other, one warp's deposits collapse into a few
// atomics (cic_deposit_warp sums runs of equal cells) and its gathers hit the same cache
// lines. The sort is a counting sort: cell keys + histogram, an exclusive scan of the counts,
// a destination per particle, then one scatter per particle array. Results do not depend on
// the order (the deposit is integer, everything else is per particle); only memory order
// changes, and the `id` array keeps the original index for output.
#include <cub/device/device_scan.cuh>

#include "kernels.cuh"

namespace rrg {
namespace {

__device__ __forceinline__ int base_cell_axis(double x, double dmin, double inv_dx, int nx) {
    // the CIC base index of rm_p2mesh.cu:191-203 (same rounding as the deposit)
    double u = __dsub_rn(__dmul_rn(__dsub_rn(x, dmin), inv_dx), 0.5);
    const double hi = __dsub_rn(static_cast<double>(nx - 1), 1e-6);
    if (!(u >= 0.0)) u = 0.0;
    if (u > hi) u = hi;
    return static_cast<int>(floor(u));
}

template <typename R>
__global__ void __launch_bounds__(256) cell_keys_kernel(int64_t n, const void* __restrict__ posm,
                                                        const V4<float>* __restrict__ lo,
                                                        GridDev g, uint32_t* __restrict__ keys,
                                                        uint32_t* __restrict__ counts) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool active = i < n;
    uint32_t key = 0xffffffffu;
    if (active) {
        double x, y, z;
        if constexpr (sizeof(R) == 8) {
            const V4<double> p = static_cast<const V4<double>*>(posm)[i];
            x = p.x;
            y = p.y;
            z = p.z;
        } else {
            const V4<float> p = static_cast<const V4<float>*>(posm)[i];
            x = p.x;
            y = p.y;
            z = p.z;
            if (lo) {
                const V4<float> l = lo[i];
                x += l.x;
                y += l.y;
                z += l.z;
            }
        }
        const int nx = g.nx;
        const int a = base_cell_axis(x, g.domain_min, g.inv_dx, nx);
        const int b = base_cell_axis(y, g.domain_min, g.inv_dx, nx);
        const int c = base_cell_axis(z, g.domain_min, g.inv_dx, nx);
        key = static_cast<uint32_t>(a + nx * (b + nx * c));
        keys[i] = key;
    }
    // one atomic per group of lanes with the same key
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (active && (threadIdx.x & 31) == (__ffs(peers) - 1))
        atomicAdd(counts + key, static_cast<uint32_t>(__popc(peers)));
}

__global__ void __launch_bounds__(256) sort_dest_kernel(int64_t n, const uint32_t* __restrict__ keys,
                                                        const uint32_t* __restrict__ offsets,
                                                        uint32_t* __restrict__ cursor,
                                                        uint32_t* __restrict__ dest) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool active = i < n;
    const uint32_t key = active ? keys[i] : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (active && lane == leader) base = atomicAdd(cursor + key, static_cast<uint32_t>(__popc(peers)));
    base = __shfl_sync(peers, base, leader);
    if (active) {
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        dest[i] = offsets[key] + base + rank;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) permute_kernel(int64_t n, const uint32_t* __restrict__ dest,
                                                      const T* __restrict__ in,
                                                      T* __restrict__ out) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[dest[i]] = in[i];
}

__global__ void iota_kernel(int64_t n, int32_t* __restrict__ id) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) id[i] = static_cast<int32_t>(i);
}

}  // namespace

size_t sort_scan_temp_bytes(int64_t ncells) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, static_cast<const uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), static_cast<int>(ncells + 1));
    return bytes;
}

void launch_cell_keys(int prec, int64_t n, const void* posm, const void* poslo,
                      const GridDev& g, uint32_t* keys, uint32_t* counts, cudaStream_t s) {
    const int b = div_up(n, 256);
    if (prec == RRG_PREC_FP64)
        cell_keys_kernel<double><<<b, 256, 0, s>>>(n, posm, nullptr, g, keys, counts);
    else
        cell_keys_kernel<float><<<b, 256, 0, s>>>(
            n, posm, prec == RRG_PREC_MIXED ? static_cast<const V4<float>*>(poslo) : nullptr, g,
            keys, counts);
    RRG_LAUNCHED();
}

void launch_scan_counts(const uint32_t* counts, uint32_t* offsets, int64_t ncells, void* temp,
                        size_t temp_bytes, cudaStream_t s) {
    size_t bytes = temp_bytes;
    RRG_CUDA(cub::DeviceScan::ExclusiveSum(temp, bytes, counts, offsets,
                                           static_cast<int>(ncells + 1), s));
    // the scan is one or two library kernels
    if (!capturing_now()) count_launches(1);
}

void launch_sort_dest(int64_t n, const uint32_t* keys, const uint32_t* offsets,
                      uint32_t* cursor, uint32_t* dest, cudaStream_t s) {
    sort_dest_kernel<<<div_up(n, 256), 256, 0, s>>>(n, keys, offsets, cursor, dest);
    RRG_LAUNCHED();
}

void launch_permute(int64_t n, size_t elem_bytes, const uint32_t* dest, const void* in,
                    void* out, cudaStream_t s) {
    const int b = div_up(n, 256);
    switch (elem_bytes) {
        case 4:
            permute_kernel<uint32_t><<<b, 256, 0, s>>>(n, dest, static_cast<const uint32_t*>(in),
                                                       static_cast<uint32_t*>(out));
            break;
        case 8:
            permute_kernel<uint2><<<b, 256, 0, s>>>(n, dest, static_cast<const uint2*>(in),
                                                    static_cast<uint2*>(out));
            break;
        case 16:
            permute_kernel<uint4><<<b, 256, 0, s>>>(n, dest, static_cast<const uint4*>(in),
                                                    static_cast<uint4*>(out));
            break;
        case 32:
            permute_kernel<V4<double>><<<b, 256, 0, s>>>(
                n, dest, static_cast<const V4<double>*>(in), static_cast<V4<double>*>(out));
            break;
        default:
            throw Error(RRG_ERR_INVALID, "permute: unsupported element size");
    }
    RRG_LAUNCHED();
}

void launch_iota(int64_t n, int32_t* id, cudaStream_t s) {
    iota_kernel<<<div_up(n, 256), 256, 0, s>>>(n, id);
    RRG_LAUNCHED();
}

}  // namespace rrg
