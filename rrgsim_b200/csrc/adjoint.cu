// Hand-written adjoint (vector-Jacobian product) of the direct-sum acceleration on sm_100a.
//
// Forward (nbody.cu:19-65): a_i = sum_j m_j d_ij f_ij, d_ij = x_j - x_i,
//   f_ij = (|d_ij|^2 + h_i + h_j)^(-3/2).
// With g_ij = -3 (|d_ij|^2 + h_i + h_j)^(-5/2) the Jacobian blocks are
//   da_i/dx_j = m_j (f_ij I + g_ij d_ij d_ij^T)   (j != i),   da_i/dx_i = -sum_j (same),
//   da_i/dm_j = d_ij f_ij.
// For a cotangent lam on a:
//   xbar_k = sum_j (f_kj u_kj + g_kj d_kj (d_kj . u_kj)),  u_kj = m_k lam_j - m_j lam_k
//   mbar_k = -sum_j f_kj (lam_j . d_kj)
// The self pair contributes exactly zero (d = 0, u = 0), so the loop runs over all j like the
// forward kernel. Same tiling as the forward: j-tiles of 256 through shared memory, split-j
// partials reduced in FP64 in a fixed order.
#include "kernels.cuh"

namespace rrg {
namespace {

constexpr int kBS = 256;

struct VjpParams {
    const V4<float>* posm;
    const float* hsoft;
    float uniform_h;
    int64_t n;
    int64_t jchunk;
    const V4<float>* lam;
    V4<float>* out;
    V4<float>* part;
};

template <bool USOFT>
__global__ void __launch_bounds__(kBS, 2) vjp_kernel(const VjpParams p) {
    __shared__ V4<float> s_pos[kBS];
    __shared__ V4<float> s_lam[kBS];
    __shared__ float s_h[USOFT ? 1 : kBS];
    const int tid = threadIdx.x;
    const int64_t k = static_cast<int64_t>(blockIdx.x) * kBS + tid;
    V4<float> pk = v4<float>(0.f, 0.f, 0.f, 0.f), lk = v4<float>(0.f, 0.f, 0.f, 0.f);
    float hk = p.uniform_h;
    if (k < p.n) {
        pk = p.posm[k];
        lk = p.lam[k];
        if constexpr (!USOFT) hk = p.hsoft[k];
    }
    float gx = 0.f, gy = 0.f, gz = 0.f, gm = 0.f;
    const int64_t jb = static_cast<int64_t>(blockIdx.y) * p.jchunk;
    const int64_t je = min(p.n, jb + p.jchunk);
    for (int64_t j0 = jb; j0 < je; j0 += kBS) {
        const int64_t j = j0 + tid;
        __syncthreads();
        if (j < je) {
            s_pos[tid] = p.posm[j];
            s_lam[tid] = p.lam[j];
            if constexpr (!USOFT) s_h[tid] = p.hsoft[j];
        } else {
            s_pos[tid] = v4<float>(1e18f, 1e18f, 1e18f, 0.f);
            s_lam[tid] = v4<float>(0.f, 0.f, 0.f, 0.f);
            if constexpr (!USOFT) s_h[tid] = 1.f;
        }
        __syncthreads();
        float tx = 0.f, ty = 0.f, tz = 0.f, tm = 0.f;
#pragma unroll 4
        for (int q = 0; q < kBS; ++q) {
            const V4<float> pj = s_pos[q];
            const V4<float> lj = s_lam[q];
            const float dx = pj.x - pk.x, dy = pj.y - pk.y, dz = pj.z - pk.z;
            const float s = USOFT ? (hk + hk) : (hk + s_h[q]);
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, s)));
            const float inv = rsqrt_sfu(r2);
            const float inv2 = inv * inv;
            const float f = inv * inv2;
            const float g = -3.f * f * inv2;
            const float ux = pk.w * lj.x - pj.w * lk.x;
            const float uy = pk.w * lj.y - pj.w * lk.y;
            const float uz = pk.w * lj.z - pj.w * lk.z;
            const float du = fmaf(dz, uz, fmaf(dy, uy, dx * ux));
            const float t = g * du;
            tx = fmaf(f, ux, fmaf(t, dx, tx));
            ty = fmaf(f, uy, fmaf(t, dy, ty));
            tz = fmaf(f, uz, fmaf(t, dz, tz));
            const float ld = fmaf(dz, lj.z, fmaf(dy, lj.y, dx * lj.x));
            tm = fmaf(-f, ld, tm);
        }
        gx += tx;
        gy += ty;
        gz += tz;
        gm += tm;
    }
    if (k >= p.n) return;
    if (gridDim.y > 1) p.part[static_cast<int64_t>(blockIdx.y) * p.n + k] = v4<float>(gx, gy, gz, gm);
    else p.out[k] = v4<float>(gx, gy, gz, gm);
}

__global__ void vjp_finish(const VjpParams p, int splits) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= p.n) return;
    double sx = 0, sy = 0, sz = 0, sm = 0;
    for (int s = 0; s < splits; ++s) {
        const V4<float> v = p.part[static_cast<int64_t>(s) * p.n + k];
        sx += v.x; sy += v.y; sz += v.z; sm += v.w;
    }
    p.out[k] = v4<float>(static_cast<float>(sx), static_cast<float>(sy), static_cast<float>(sz),
                         static_cast<float>(sm));
}

}  // namespace

void launch_direct_vjp_f32(const void* posm, const void* hsoft, float uniform_hsoft, int64_t n,
                           const void* lam, void* out, cudaStream_t stream) {
    int dev = 0;
    RRG_CUDA(cudaGetDevice(&dev));
    const int splits_req = direct_choose_splits(RRG_PREC_FP32, n, num_sms(dev));
    const int64_t tiles = (n + kBS - 1) / kBS;
    const int64_t tiles_per = (tiles + splits_req - 1) / splits_req;
    const int splits = static_cast<int>((tiles + tiles_per - 1) / tiles_per);
    VjpParams p;
    p.posm = static_cast<const V4<float>*>(posm);
    p.hsoft = static_cast<const float*>(hsoft);
    p.uniform_h = uniform_hsoft;
    p.n = n;
    p.jchunk = tiles_per * kBS;
    p.lam = static_cast<const V4<float>*>(lam);
    p.out = static_cast<V4<float>*>(out);
    p.part = nullptr;
    if (splits > 1)
        RRG_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p.part),
                                 sizeof(V4<float>) * n * splits, stream));
    dim3 grid(static_cast<unsigned>((n + kBS - 1) / kBS), splits);
    if (hsoft) vjp_kernel<false><<<grid, kBS, 0, stream>>>(p);
    else vjp_kernel<true><<<grid, kBS, 0, stream>>>(p);
    RRG_LAUNCHED();
    if (splits > 1) {
        vjp_finish<<<div_up(n, 256), 256, 0, stream>>>(p, splits);
        RRG_LAUNCHED();
        RRG_CUDA(cudaFreeAsync(p.part, stream));
    }
}

}  // namespace rrg
