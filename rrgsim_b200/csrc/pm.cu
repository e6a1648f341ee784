// Particle-mesh kernels on sm_100a: CIC deposit into int64 fixed point, damped-wave potential
// relaxation, gradient, trilinear force interpolation, and the fused particle pass.
//
// Grid layout is the reference's AT(x, y, z) = x + y nx + z nx^2
// (solver/lib/rrgsim_common/include/co_device_utils.cuh:61), nx^3 cells, cell centres at
// domain_min + (i + 1/2) dx for CIC / interpolation and nodes at domain_min + i dx for the wave
// boundary terms (wave.cu:18-20), exactly as in the reference.
#include <cstdlib>

#include "kernels.cuh"
#include "sums.cuh"

namespace rrg {
namespace {

constexpr double kPi = 3.14159265358979;  // the reference's PI (co_info_structs.h:7)
static_assert(kPmSumValues == kConsTerms, "PM_SUMS records hold the 8 conservation terms");

__device__ __forceinline__ int wrap_mod(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

__device__ __forceinline__ double load_x(const V4<float>* posm, const V4<float>* lo, int64_t i,
                                         double& y, double& z, float& m) {
    const V4<float> p = posm[i];
    double x = p.x;
    y = p.y;
    z = p.z;
    if (lo) {
        const V4<float> l = lo[i];
        x += l.x;
        y += l.y;
        z += l.z;
    }
    m = p.w;
    return x;
}

// ----------------------------------------------------------------------------------------------
// CIC weights exactly as deposit_cell_mass_CIC_ (rm_p2mesh.cu:184-226), in FP64 with every
// operation rounded separately (no FMA contraction) so that the host oracle, compiled with
// -ffp-contract=off, produces the same bits:
//   u = (x - domain_min) * inv_dx - 0.5 ; clamp to [0, nx - 1 - 1e-6]
//   i0 = floor(u) ; i1 = min(i0 + 1, nx - 1) ; f = u - i0 ; w0 = 1 - f ; w1 = f
// A NaN coordinate is treated as u = 0 (the reference would index out of bounds).
// ----------------------------------------------------------------------------------------------
__device__ __forceinline__ void cic_axis(double x, double dmin, double inv_dx, int nx, int& i0,
                                         int& i1, double& w0, double& w1) {
    double u = __dsub_rn(__dmul_rn(__dsub_rn(x, dmin), inv_dx), 0.5);
    const double hi = __dsub_rn(static_cast<double>(nx - 1), 1e-6);
    if (!(u >= 0.0)) u = 0.0;  // also catches NaN
    if (u > hi) u = hi;
    i0 = static_cast<int>(floor(u));
    i1 = min(i0 + 1, nx - 1);
    const double f = __dsub_rn(u, static_cast<double>(i0));
    w0 = __dsub_rn(1.0, f);
    w1 = f;
}

// Deposits one particle (all lanes of the warp call this together, converged).
// Lanes with the same base cell form a run once they sit next to each other: particles sorted by
// cell make long runs, but as they drift from the sorted order a warp's cells interleave. A warp
// holding more than four runs therefore first sorts its (cell, lane) pairs with a bitonic
// network of full-warp shuffles (15 compare-exchange steps) and takes each lane's values along.
// Each of the 8 corner values is then summed over its run by a segmented warp scan (five
// full-warp shuffles), and the run's last lane adds the eight sums with 64-bit atomics: one set
// of atomics per distinct cell in the warp. Values fit in 27 bits (the scale S is chosen so that
// m_max 2^S <= 2^26), so a warp's sum fits 32 bits; integer sums are exact in any order, so the
// grid does not depend on how particles fall into runs. (Grouping lanes with __match_any_sync and
// summing each group with __reduce_add_sync cost more: every distinct group mask in a warp is a
// separate divergent pass. Without the warp sort the atomics multiply as runs fragment: at 2^20
// disk particles 0.3 cell off their sorted order, 51 us against 27. The hardware reduction with
// each lane's run mask taken from the run heads, for warps of up to 4, 8 or 32 runs instead of
// 2: 126.4, 131.6 and 144.9 against 124.7 us per PM step. Floors without conversion
// instructions (rounded-down additions of 2^52 and 1.5 2^23) in these weights and in the
// interpolation's: 124.6 against 124.6 us.)
__device__ __forceinline__ void cic_deposit_warp(bool active, double x, double y, double z,
                                                 double m, const GridDev& g, double scale,
                                                 unsigned long long* __restrict__ grid) {
    const int nx = g.nx;
    int i0 = 0, i1 = 0, j0 = 0, j1 = 0, k0 = 0, k1 = 0;
    double wx0 = 0, wx1 = 0, wy0 = 0, wy1 = 0, wz0 = 0, wz1 = 0;
    if (active) {
        cic_axis(x, g.domain_min, g.inv_dx, nx, i0, i1, wx0, wx1);
        cic_axis(y, g.domain_min, g.inv_dx, nx, j0, j1, wy0, wy1);
        cic_axis(z, g.domain_min, g.inv_dx, nx, k0, k1, wz0, wz1);
    }
    const int nx2 = nx * nx;  // nx^3 < 2^31 (nx <= 1024)
    const int lane = threadIdx.x & 31;
    const double ms = __dmul_rn(m, scale);
    // corner order and weight products as rm_p2mesh.cu:219-235
    const double wxs[2] = {wx0, wx1}, wys[2] = {wy0, wy1}, wzs[2] = {wz0, wz1};
    unsigned q[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        q[c] = 0;
        if (active) {
            const double w = __dmul_rn(__dmul_rn(wxs[c & 1], wys[(c >> 1) & 1]), wzs[c >> 2]);
            // round to the nearest integer, ties to even, as __double2ll_rn: adding 1.5 * 2^52
            // leaves the integer in the low mantissa bits (exact for 0 <= value < 2^31; values
            // here are below 2^27), an FP64 add instead of a conversion on the XU pipe
            q[c] = static_cast<unsigned>(
                __double2loint(__dadd_rn(__dmul_rn(ms, w), 6755399441055744.0)));
        }
    }
    // every lane takes part in every shuffle (none behind a short-circuit or a divergent branch)
    int key = active ? (i0 + j0 * nx + k0 * nx2) : -1;
    const int below0 = __shfl_up_sync(0xffffffffu, key, 1);
    const unsigned heads0 = __ballot_sync(0xffffffffu, lane == 0 || below0 != key);
    // a warp of 28 or more runs (sparse outskirts: nearly one cell per lane) skips the sort and
    // the scan, and every lane adds its own values (121.5 against 122.1 us per PM step; from 20
    // runs on the extra atomics cost more than the scan saves: 126.8; skipping the sort also for
    // warps whose lanes are already in cell order, one ballot: 121.6 against 121.8, not kept)
    constexpr int sparse = 28;
    if (__popc(heads0) > 4 && __popc(heads0) < sparse) {  // warp-uniform
        int src = lane;
        if (nx <= 406) {
            // (cell + 1, lane) packed into one int (nx^3 < 2^26): one shuffle per step
            int kv = ((key + 1) << 5) | lane;
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const int pk = __shfl_xor_sync(0xffffffffu, kv, j);
                    const bool ascending = (lane & k) == 0, lower = (lane & j) == 0;
                    if (lower == ascending ? pk < kv : pk > kv) kv = pk;
                }
            }
            key = (kv >> 5) - 1;
            src = kv & 31;
        } else {
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const int pk = __shfl_xor_sync(0xffffffffu, key, j);
                    const int ps = __shfl_xor_sync(0xffffffffu, src, j);
                    const bool ascending = (lane & k) == 0, lower = (lane & j) == 0;
                    const bool less = pk < key || (pk == key && ps < src);
                    if (lower == ascending ? less : !less) {
                        key = pk;
                        src = ps;
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) q[c] = __shfl_sync(0xffffffffu, q[c], src);
    }
    const int below = __shfl_up_sync(0xffffffffu, key, 1);
    const int above = __shfl_down_sync(0xffffffffu, key, 1);
    const bool head = lane == 0 || below != key;
    bool tail = lane == 31 || above != key;
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    unsigned sum[8];
    if (__popc(heads) >= sparse) {
        // (nearly) every lane its own cell: each adds its own values
#pragma unroll
        for (int c = 0; c < 8; ++c) sum[c] = q[c];
        tail = true;
    } else if (__popc(heads) <= 2) {
        // one or two runs (warp-uniform; the common case in dense regions of sorted
        // particles): one hardware reduction per run and corner instead of the scan
        const unsigned second = heads & ~1u;  // the second run's head lane bit, or 0
        const unsigned mask = second == 0u ? 0xffffffffu
                              : ((lane < __ffs(second) - 1) ? second - 1u : ~(second - 1u));
#pragma unroll
        for (int c = 0; c < 8; ++c) sum[c] = __reduce_add_sync(mask, q[c]);
    } else {
        const int first = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));  // the run's first lane
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            unsigned v = q[c];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned t = __shfl_up_sync(0xffffffffu, v, d);
                if (lane - d >= first) v += t;
            }
            sum[c] = v;  // at the run's last lane: the run's total
        }
    }
    if (key >= 0 && tail) {
        // the run's cell and its corners (clamped as cic_axis clamps)
        const int a0 = key % nx, b0 = (key / nx) % nx, c0 = key / nx2;
        const int a1 = min(a0 + 1, nx - 1), b1 = min(b0 + 1, nx - 1), c1 = min(c0 + 1, nx - 1);
        const int ii[8] = {a0, a1, a0, a1, a0, a1, a0, a1};
        const int jj[8] = {b0, b0, b1, b1, b0, b0, b1, b1};
        const int kk[8] = {c0, c0, c0, c0, c1, c1, c1, c1};
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            if (sum[c] != 0u)
                atomicAdd(grid + (kk[c] * nx + jj[c]) * nx + ii[c],
                          static_cast<unsigned long long>(sum[c]));
        }
    }
}

template <typename R>
__device__ __forceinline__ void load_pos(const void* posm, const V4<float>* lo, int64_t i,
                                         double& x, double& y, double& z, double& m) {
    if constexpr (sizeof(R) == 8) {
        const V4<double> p = static_cast<const V4<double>*>(posm)[i];
        x = p.x;
        y = p.y;
        z = p.z;
        m = p.w;
    } else {
        float mf;
        x = load_x(static_cast<const V4<float>*>(posm), lo, i, y, z, mf);
        m = mf;
    }
}

template <typename R>
__global__ void __launch_bounds__(256) cic_kernel(int64_t n, const void* __restrict__ posm,
                                                  const V4<float>* __restrict__ lo, GridDev g,
                                                  double scale,
                                                  unsigned long long* __restrict__ grid) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool active = i < n;
    double x = 0, y = 0, z = 0, m = 0;
    if (active) load_pos<R>(posm, lo, i, x, y, z, m);
    cic_deposit_warp(active, x, y, z, m, g, scale, grid);
}

// ----------------------------------------------------------------------------------------------
// Wave source: f = 4 pi G rho, rho = mass / dx^3 - rho_sub (wave.cu:150-153), mass from the
// fixed-point grid. Optionally clears the fixed-point grid for the next deposit.
// ----------------------------------------------------------------------------------------------
// FP64 divides by dx^3 as the reference does; FP32, whose source is rounded to float anyway,
// multiplies by the host's 1 / dx^3 (an FP64 division per cell made this pass instruction-bound).
template <typename R>
__global__ void wave_source_kernel(int64_t ncells, unsigned long long* __restrict__ mgrid,
                                   double inv_scale, double dx3, double inv_dx3, double rho_sub,
                                   double mult, R* __restrict__ src, bool zero_grid) {
    const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    const unsigned long long q = mgrid[c];
    if (zero_grid) mgrid[c] = 0ull;
    if constexpr (sizeof(R) == 8) {
        const double mass = static_cast<double>(q) * inv_scale;
        const double rho = mass / dx3 - rho_sub;
        src[c] = static_cast<R>(mult * (4.0 * kPi * 1.0 * rho));
    } else {
        src[c] = static_cast<R>(__dmul_rn(mult, wave_source_value(q, inv_scale, inv_dx3, rho_sub)));
    }
}

// The incremental solve's preparation and finish (wave_inc_source): one thread per cell,
// periodic neighbours.
__global__ void wave_inc_prep_kernel(int nx, const unsigned long long* __restrict__ mg,
                                     unsigned long long* __restrict__ mg_zero,
                                     double inv_scale, double inv_dx3, double rho_sub,
                                     const float* __restrict__ phi0,
                                     const float* __restrict__ phi_prev, double kf, double km,
                                     double kao, float* __restrict__ g, float* __restrict__ d,
                                     float* __restrict__ d_old, float* __restrict__ src) {
    const int64_t nc = static_cast<int64_t>(nx) * nx * nx;
    const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int x = static_cast<int>(c % nx), y = static_cast<int>((c / nx) % nx),
              z = static_cast<int>(c / (static_cast<int64_t>(nx) * nx));
    const int64_t row = c - x, plane = static_cast<int64_t>(nx) * nx;
    const int64_t cz = c - static_cast<int64_t>(z) * plane;
    const float p = phi0[c];
    const float l = phi0[row + (x == 0 ? nx - 1 : x - 1)];
    const float r = phi0[row + (x == nx - 1 ? 0 : x + 1)];
    const float ym = phi0[c + (y == 0 ? (nx - 1) * nx : -nx)];
    const float yp = phi0[c + (y == nx - 1 ? -(nx - 1) * nx : nx)];
    const float zm = phi0[cz + (z == 0 ? nx - 1 : z - 1) * plane];
    const float zp = phi0[cz + (z == nx - 1 ? 0 : z + 1) * plane];
    const double sd = wave_source_value(mg[c], inv_scale, inv_dx3, rho_sub);
    g[c] = wave_inc_source(sd, l, r, ym, yp, zm, zp, p, kf, km, kao);
    if (d) d[c] = 0.f;
    d_old[c] = __fsub_rn(phi_prev[c], p);
    if (src) src[c] = static_cast<float>(sd);
    if (mg_zero) mg_zero[c] = 0ull;
}

__global__ void wave_inc_finish_kernel(int64_t nc, const float* phi0, const float* d_fin,
                                       const float* d_prv, float* fin, float* prv) {
    const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const float p = phi0[c], a = d_fin[c], b = d_prv[c];
    fin[c] = __fadd_rn(p, a);
    prv[c] = __fadd_rn(p, b);
}

// ----------------------------------------------------------------------------------------------
// Damped wave substep (wave_diss_iteration, wave.cu:106-193).
//   phi_new = K_MAIN sum6 + K_ACTUAL phi + K_OLD phi_old + K_F f
// Every variant marches a thread through a chunk of z-planes with the z-neighbours in
// registers; phi_new overwrites phi_old in place (each cell's old value is read only by its own
// thread), so two grid buffers rotate instead of the reference's three.
// ----------------------------------------------------------------------------------------------
constexpr int kTX = 32, kTY = 8;

struct WaveDev {
    int nx;
    int zc;
    int bc;          // rrg_boundary_type
    int uniform;     // periodic without absorbing layer -> constant coefficients
    double K_MAIN, K_ACTUAL, K_OLD, K_F;
    double C, DT, DX, diss_base, diss_extra, sim_l, domain_min;
    double bc_mass, comx, comy, comz, r_min;
};

__device__ __forceinline__ double layer_diss(const WaveDev& w, double x) {
    const double x_in = 0.5 * w.sim_l;
    const double d = fabs(x) - x_in;
    return d > 0 ? w.diss_extra * d * d : 0.0;
}

__device__ __forceinline__ double monopole_phi(const WaveDev& w, double x, double y, double z) {
    const double rx = w.comx - x, ry = w.comy - y, rz = w.comz - z;
    const double dist = sqrt(rx * rx + ry * ry + rz * rz);
    const double r = fmax(dist, w.r_min);
    return -1.0 * w.bc_mass / r;
}

template <typename R>
__device__ __forceinline__ double psi_at(const WaveDev& w, const R* phi, int i, int j, int k) {
    const int64_t nx = w.nx;
    const double x = w.domain_min + i * w.DX, y = w.domain_min + j * w.DX,
                 z = w.domain_min + k * w.DX;
    return static_cast<double>(phi[i + j * nx + k * nx * nx]) - monopole_phi(w, x, y, z);
}

// Radiative boundary node (radiative_boundary / upwind_axis, wave.cu:51-104).
template <typename R>
__device__ double radiative_value(const WaveDev& w, const R* phi, int ix, int iy, int iz) {
    const double x = w.domain_min + ix * w.DX, y = w.domain_min + iy * w.DX,
                 z = w.domain_min + iz * w.DX;
    const double rx = x - w.comx, ry = y - w.comy, rz = z - w.comz;
    const double r = fmax(sqrt(rx * rx + ry * ry + rz * rz), w.r_min);
    const double n3[3] = {rx / r, ry / r, rz / r};
    const double psi0 = psi_at<R>(w, phi, ix, iy, iz);
    double dpsi_dr = 0.0;
    const int idx[3] = {ix, iy, iz};
    for (int axis = 0; axis < 3; ++axis) {
        const int i0 = idx[axis];
        int in = (n3[axis] > 0) ? i0 - 1 : i0 + 1;
        if (in < 0 || in >= w.nx) in = 2 * i0 - in;
        int jx = ix, jy = iy, jz = iz;
        if (axis == 0) jx = in;
        else if (axis == 1) jy = in;
        else jz = in;
        const double d = (psi0 - psi_at<R>(w, phi, jx, jy, jz)) / ((i0 - in) * w.DX);
        dpsi_dr += n3[axis] * d;
    }
    const double psi_new = psi0 - w.C * w.DT * (dpsi_dr + psi0 / r);
    return psi_new + monopole_phi(w, x, y, z);
}

__device__ __forceinline__ unsigned long long dbits(double v) {
    return static_cast<unsigned long long>(__double_as_longlong(v));
}

// Block-wide max of (dmax, amax) folded into maxbits[0..1] (non-negative doubles compare as
// their bit patterns).
__device__ __forceinline__ void block_max_to(double dmax, double amax, int tid,
                                             unsigned long long* maxbits) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dmax = fmax(dmax, __shfl_down_sync(0xffffffffu, dmax, o));
        amax = fmax(amax, __shfl_down_sync(0xffffffffu, amax, o));
    }
    __shared__ double sd[kTX * kTY / 32], sa[kTX * kTY / 32];  // blocks of up to 256 threads
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) {
        sd[wid] = dmax;
        sa[wid] = amax;
    }
    __syncthreads();
    if (tid == 0) {
        double d = 0, a = 0;
        const int warps = static_cast<int>((blockDim.x * blockDim.y + 31) / 32);
        for (int k = 0; k < warps; ++k) {
            d = fmax(d, sd[k]);
            a = fmax(a, sa[k]);
        }
        atomicMax(maxbits, dbits(d));
        atomicMax(maxbits + 1, dbits(a));
    }
}

// Periodic box without an absorbing layer (the reference's wired path, wave.cu:177-181):
// constant coefficients, wrapped neighbours, and a compile-time z-chunk so the column's
// ZC + 2 potential values are all requested before the first update (memory-level
// parallelism for a latency-bound stencil).
template <typename R, int ZC, bool CHECK>
__global__ void __launch_bounds__(kTX* kTY, 8) wave_periodic_kernel(
    const R* __restrict__ phi, R* __restrict__ phi_old, const R* __restrict__ src,
    const WaveDev w, unsigned long long* __restrict__ maxbits) {
    const int nx = w.nx;
    const int plane = nx * nx;
    const int tid = threadIdx.y * kTX + threadIdx.x;
    const int x = blockIdx.x * kTX + threadIdx.x;
    const int y = blockIdx.y * kTY + threadIdx.y;
    double dmax = 0.0, amax = 0.0;
    if (x < nx && y < nx) {
        const int oxm = x > 0 ? -1 : nx - 1;
        const int oxp = x < nx - 1 ? 1 : -(nx - 1);
        const int oym = y > 0 ? -nx : (nx - 1) * nx;
        const int oyp = y < nx - 1 ? nx : -(nx - 1) * nx;
        const int col = x + y * nx;
        const int z0 = blockIdx.z * ZC;
        const R km = static_cast<R>(w.K_MAIN), ka = static_cast<R>(w.K_ACTUAL),
                ko = static_cast<R>(w.K_OLD), kf = static_cast<R>(w.K_F);
        R pv[ZC + 2];  // phi at z0 - 1 ... z0 + ZC (wrapped)
#pragma unroll
        for (int k = 0; k < ZC + 2; ++k) {
            int z = z0 - 1 + k;
            z = z < 0 ? z + nx : (z >= nx ? z - nx : z);
            pv[k] = __ldg(phi + col + z * plane);
        }
#pragma unroll
        for (int k = 0; k < ZC; ++k) {
            const int z = z0 + k;
            if (z < nx) {
                const int c = col + z * plane;
                const R lap = __ldg(phi + c + oxm) + __ldg(phi + c + oxp) +
                              __ldg(phi + c + oym) + __ldg(phi + c + oyp) + pv[k] + pv[k + 2];
                const R out = lap * km + pv[k + 1] * ka + phi_old[c] * ko + src[c] * kf;
                phi_old[c] = out;
                if constexpr (CHECK) {
                    dmax = fmax(dmax, fabs(static_cast<double>(out) - static_cast<double>(pv[k + 1])));
                    amax = fmax(amax, fabs(static_cast<double>(out)));
                }
            }
        }
    }
    if constexpr (CHECK) block_max_to(dmax, amax, tid, maxbits);
}

// FP32 periodic box, four x-cells per thread as one float4 (nx % 4 == 0, and nx / 4 either
// divides 32 or is a multiple of 32): a warp covers whole rows (nx <= 128) or 32 consecutive
// float4 of one row, so the x - 1 / x + 4 neighbours are warp shuffles with the periodic wrap
// inside the row's lanes (a scalar load at the two warp edges only when rows are wider than a
// warp). Rows y +- 1 are coalesced float4 loads, the z neighbours a register pipeline of ZC + 2
// planes. About 1.5 memory instructions per cell instead of 7. Same arithmetic as
// wave_periodic_kernel: lap = x- + x+ + y- + y+ + z- + z+, out = lap K_MAIN + phi K_ACTUAL +
// phi_old K_OLD + src K_F.
// ADJ: the adjoint substep of the PM adjoint instead (phi the current cotangent C, phi_old the
// previous one P, no source): P <- K_MAIN L6(C) + K_ACTUAL C + K_OLD P and F += K_F C.
template <int ZC, bool CHECK, int BS, bool ADJ = false>
__global__ void __launch_bounds__(BS, 1024 / BS) wave_periodic_x4_kernel(
    const float* __restrict__ phi, float* __restrict__ phi_old, const float* __restrict__ src,
    const WaveDev w, unsigned long long* __restrict__ maxbits, float* __restrict__ fadj = nullptr) {
    const int nx = w.nx;
    const int W = nx >> 2;       // float4 per row
    const int plane4 = W * nx;   // float4 per plane
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int g = blockIdx.x * BS + tid;  // float4 index within a plane
    const bool valid = g < plane4;
    const int y = g / W, q = g - (g / W) * W;
    int lsrc, rsrc;
    bool lload = false, rload = false;
    if (W >= 32) {
        lsrc = (lane + 31) & 31;
        rsrc = (lane + 1) & 31;
        lload = W > 32 && lane == 0;
        rload = W > 32 && lane == 31;
    } else {
        const int seg = lane - lane % W;
        lsrc = seg + (lane - seg + W - 1) % W;
        rsrc = seg + (lane - seg + 1) % W;
    }
    const float4* phi4 = reinterpret_cast<const float4*>(phi);
    const float4* src4 = reinterpret_cast<const float4*>(src);
    float4* old4 = reinterpret_cast<float4*>(phi_old);
    const float km = static_cast<float>(w.K_MAIN), ka = static_cast<float>(w.K_ACTUAL),
                ko = static_cast<float>(w.K_OLD), kf = static_cast<float>(w.K_F);
    const int z0 = blockIdx.y * ZC;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 pv[ZC + 2];  // phi at z0 - 1 ... z0 + ZC (wrapped)
#pragma unroll
    for (int k = 0; k < ZC + 2; ++k) {
        int z = z0 - 1 + k;
        z = z < 0 ? z + nx : (z >= nx ? z - nx : z);
        pv[k] = valid ? __ldg(phi4 + g + z * plane4) : zero4;
    }
    const int gym = y > 0 ? g - W : g + (nx - 1) * W;
    const int gyp = y < nx - 1 ? g + W : g - (nx - 1) * W;
    const int xl = q == 0 ? nx - 1 : 4 * q - 1;      // row-local x of the left edge value
    const int xr = q == W - 1 ? 0 : 4 * q + 4;       // and of the right one
    double dmax = 0.0, amax = 0.0;
#pragma unroll
    for (int k = 0; k < ZC; ++k) {
        const int z = z0 + k;
        const float4 c = pv[k + 1];
        float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
        float rgt = __shfl_sync(0xffffffffu, c.x, rsrc);
        if (valid) {
            const int rowbase = z * nx * nx + y * nx;
            if (lload) lft = __ldg(phi + rowbase + xl);
            if (rload) rgt = __ldg(phi + rowbase + xr);
            const int o = g + z * plane4;
            const float4 ym = __ldg(phi4 + gym + z * plane4);
            const float4 yp = __ldg(phi4 + gyp + z * plane4);
            const float4 zm = pv[k], zp = pv[k + 2];
            const float4 po = old4[o];
            if constexpr (ADJ) {
                old4[o] = wave_cell4(c, lft, rgt, ym, yp, zm, zp, po, zero4, km, ka, ko, 0.f);
                float4* f4 = reinterpret_cast<float4*>(fadj) + o;
                float4 f = *f4;
                f.x = __fmaf_rn(kf, c.x, f.x);
                f.y = __fmaf_rn(kf, c.y, f.y);
                f.z = __fmaf_rn(kf, c.z, f.z);
                f.w = __fmaf_rn(kf, c.w, f.w);
                *f4 = f;
                continue;
            }
            const float4 s = __ldg(src4 + o);
            const float4 out = wave_cell4(c, lft, rgt, ym, yp, zm, zp, po, s, km, ka, ko, kf);
            old4[o] = out;
            if constexpr (CHECK) {
                // differences in FP64, as the scalar kernels take them
                const double d = fmax(fmax(fabs(double(out.x) - double(c.x)),
                                           fabs(double(out.y) - double(c.y))),
                                      fmax(fabs(double(out.z) - double(c.z)),
                                           fabs(double(out.w) - double(c.w))));
                const float a = fmaxf(fmaxf(fabsf(out.x), fabsf(out.y)),
                                      fmaxf(fabsf(out.z), fabsf(out.w)));
                dmax = fmax(dmax, d);
                amax = fmax(amax, static_cast<double>(a));
            }
        }
    }
    if constexpr (CHECK) block_max_to(dmax, amax, tid, maxbits);
}

// UNIFORM is the periodic box without an absorbing layer (the reference's wired path): the
// boundary code compiles away and the kernel fits 8 resident blocks per SM.
template <typename R, bool UNIFORM, bool CHECK>
__global__ void __launch_bounds__(kTX* kTY, UNIFORM ? 8 : 2) wave_step_kernel(
    const R* __restrict__ phi, R* __restrict__ phi_old, const R* __restrict__ src,
    const WaveDev w, unsigned long long* __restrict__ maxbits) {
    // One thread per (x, y) column marches through zc planes: phi(z - 1), phi(z), phi(z + 1)
    // stay in registers, the four in-plane neighbours come through L1 (adjacent threads share
    // their cache lines). No shared memory, no barriers. int32 indexing: nx <= 1024.
    const int nx = w.nx;
    const int plane = nx * nx;
    const int tid = threadIdx.y * kTX + threadIdx.x;
    const int x = blockIdx.x * kTX + threadIdx.x;
    const int y = blockIdx.y * kTY + threadIdx.y;
    const bool valid = (x < nx) && (y < nx);
    const bool periodic = UNIFORM ? true : (w.bc == RRG_BC_PERIODIC);
    double dmax = 0.0, amax = 0.0;
    if (valid) {
        // in-plane neighbour offsets: periodic wrap, or clamped (unused on the boundary nodes)
        const int oxm = x > 0 ? -1 : (periodic ? nx - 1 : 0);
        const int oxp = x < nx - 1 ? 1 : (periodic ? -(nx - 1) : 0);
        const int oym = y > 0 ? -nx : (periodic ? (nx - 1) * nx : 0);
        const int oyp = y < nx - 1 ? nx : (periodic ? -(nx - 1) * nx : 0);
        const bool xy_edge = x == 0 || x == nx - 1 || y == 0 || y == nx - 1;
        const int col = x + y * nx;
        const int z0 = blockIdx.z * w.zc;
        const int z1 = min(nx, z0 + w.zc);
        const int zm0 = z0 > 0 ? z0 - 1 : (periodic ? nx - 1 : 0);
        R pm = __ldg(phi + col + zm0 * plane);
        R pc = __ldg(phi + col + z0 * plane);
        for (int z = z0; z < z1; ++z) {
            const int zn = z < nx - 1 ? z + 1 : (periodic ? 0 : nx - 1);
            const R pn = __ldg(phi + col + zn * plane);
            const int c = col + z * plane;
            R out;
            if (!periodic && (xy_edge || z == 0 || z == nx - 1)) {
                double v = 0.0;
                if (w.bc == RRG_BC_MONOPOLE_DIRICHLET)
                    v = monopole_phi(w, w.domain_min + x * w.DX, w.domain_min + y * w.DX,
                                     w.domain_min + z * w.DX);
                else if (w.bc == RRG_BC_MONOPOLE_RADIATIVE)
                    v = radiative_value<R>(w, phi, x, y, z);
                out = static_cast<R>(v);
            } else {
                const R lap = __ldg(phi + c + oxm) + __ldg(phi + c + oxp) +
                              __ldg(phi + c + oym) + __ldg(phi + c + oyp) + pm + pn;
                R kmain, kact, kold, kf;
                if constexpr (UNIFORM) {
                    kmain = static_cast<R>(w.K_MAIN);
                    kact = static_cast<R>(w.K_ACTUAL);
                    kold = static_cast<R>(w.K_OLD);
                    kf = static_cast<R>(w.K_F);
                } else {
                    double diss = w.diss_base;
                    diss += layer_diss(w, w.domain_min + x * w.DX);
                    diss += layer_diss(w, w.domain_min + y * w.DX);
                    diss += layer_diss(w, w.domain_min + z * w.DX);
                    const double Q = diss * w.C * w.DT * 0.5;
                    const double W = 1 + Q;
                    const double K = w.C * w.C * w.DT * w.DT / (w.DX * w.DX);
                    kmain = static_cast<R>(K / W);
                    kf = static_cast<R>(-w.C * w.C * w.DT * w.DT / W);
                    kact = static_cast<R>(2 * (1 - 3 * K) / W);
                    kold = static_cast<R>((Q - 1) / W);
                }
                out = lap * kmain + pc * kact + phi_old[c] * kold + src[c] * kf;
            }
            phi_old[c] = out;
            if constexpr (CHECK) {
                dmax = fmax(dmax, fabs(static_cast<double>(out) - static_cast<double>(pc)));
                amax = fmax(amax, fabs(static_cast<double>(out)));
            }
            pm = pc;
            pc = pn;
        }
    }
    if constexpr (CHECK) {
        // warp max -> block max -> one atomicMax per block on the (non-negative) double bits
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dmax = fmax(dmax, __shfl_down_sync(0xffffffffu, dmax, o));
            amax = fmax(amax, __shfl_down_sync(0xffffffffu, amax, o));
        }
        __shared__ double sd[kTX * kTY / 32], sa[kTX * kTY / 32];
        const int lane = tid & 31, wid = tid >> 5;
        if (lane == 0) {
            sd[wid] = dmax;
            sa[wid] = amax;
        }
        __syncthreads();
        if (tid == 0) {
            double d = 0, a = 0;
            for (int k = 0; k < kTX * kTY / 32; ++k) {
                d = fmax(d, sd[k]);
                a = fmax(a, sa[k]);
            }
            atomicMax(maxbits, dbits(d));
            atomicMax(maxbits + 1, dbits(a));
        }
    }
}

// ----------------------------------------------------------------------------------------------
// Gradient (calc_acceleration_field_, rm_p2mesh.cu:238-290): central differences inside,
// one-sided at the faces, a = -dphi / dx. Output cell (ax, ay, az, phi).
// ----------------------------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kTX* kTY) gradient_kernel(int nx, R coef,
                                                            const R* __restrict__ phi,
                                                            V4<R>* __restrict__ acc4) {
    const int x = blockIdx.x * kTX + threadIdx.x;
    const int y = blockIdx.y * kTY + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= nx || y >= nx) return;
    const int64_t sx = 1, sy = nx, sz = static_cast<int64_t>(nx) * nx;
    const int64_t c = x + y * sy + z * sz;
    const R pc = phi[c];
    R dx, dy, dz;
    if (x == 0) dx = phi[c + sx] - pc;
    else if (x == nx - 1) dx = pc - phi[c - sx];
    else dx = R(0.5) * (phi[c + sx] - phi[c - sx]);
    if (y == 0) dy = phi[c + sy] - pc;
    else if (y == nx - 1) dy = pc - phi[c - sy];
    else dy = R(0.5) * (phi[c + sy] - phi[c - sy]);
    if (z == 0) dz = phi[c + sz] - pc;
    else if (z == nx - 1) dz = pc - phi[c - sz];
    else dz = R(0.5) * (phi[c + sz] - phi[c - sz]);
    acc4[c] = v4<R>(dx * coef, dy * coef, dz * coef, pc);
}

// FP32 gradient with four x-cells per thread (float4 rows, as wave_periodic_x4_kernel): x +- 1
// by warp shuffles (a scalar load at warp edges when a row is wider than a warp), rows y +- 1 as
// coalesced float4 loads, the z neighbours from a register pipeline over ZC planes, and the four
// (ax, ay, az, phi) cells written as four float4 stores. Same expressions, faces one-sided, as
// gradient_kernel. Needs nx % 4 == 0, nx % ZC == 0 and nx / 4 dividing 32 or a multiple of 32.
template <int ZC, int BS>
__global__ void __launch_bounds__(BS) gradient_x4_kernel(int nx, float coef,
                                                         const float* __restrict__ phi,
                                                         float4* __restrict__ acc4) {
    const int W = nx >> 2;
    const int plane4 = W * nx;
    const int tid = threadIdx.x, lane = tid & 31;
    const int g = blockIdx.x * BS + tid;
    const bool valid = g < plane4;
    const int y = g / W, q = g - (g / W) * W;
    int lsrc, rsrc;
    bool lload = false, rload = false;
    if (W >= 32) {
        lsrc = (lane + 31) & 31;
        rsrc = (lane + 1) & 31;
        lload = W > 32 && lane == 0 && q > 0;
        rload = W > 32 && lane == 31 && q < W - 1;
    } else {
        const int seg = lane - lane % W;
        lsrc = seg + (lane - seg + W - 1) % W;
        rsrc = seg + (lane - seg + 1) % W;
    }
    const float4* phi4 = reinterpret_cast<const float4*>(phi);
    const int z0 = blockIdx.y * ZC;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 pv[ZC + 2];  // phi at z0 - 1 ... z0 + ZC (clamped to the box; faces are one-sided)
#pragma unroll
    for (int k = 0; k < ZC + 2; ++k) {
        const int z = min(max(z0 - 1 + k, 0), nx - 1);
        pv[k] = valid ? __ldg(phi4 + g + z * plane4) : zero4;
    }
    const int gym = y > 0 ? g - W : g;
    const int gyp = y < nx - 1 ? g + W : g;
    const int x = 4 * q;
#pragma unroll
    for (int k = 0; k < ZC; ++k) {
        const int z = z0 + k;
        const float4 c = pv[k + 1];
        float lft = __shfl_sync(0xffffffffu, c.w, lsrc);
        float rgt = __shfl_sync(0xffffffffu, c.x, rsrc);
        if (!valid) continue;
        const int rowbase = z * nx * nx + y * nx;
        if (lload) lft = __ldg(phi + rowbase + x - 1);
        if (rload) rgt = __ldg(phi + rowbase + x + 4);
        // x: central inside, one-sided at x = 0 and x = nx - 1
        const float d0 = x == 0 ? c.y - c.x : 0.5f * (c.y - lft);
        const float d1 = 0.5f * (c.z - c.x);
        const float d2 = 0.5f * (c.w - c.y);
        const float d3 = x + 4 == nx ? c.w - c.z : 0.5f * (rgt - c.z);
        // y
        float4 ey;
        if (y == 0) {
            const float4 yp = __ldg(phi4 + gyp + z * plane4);
            ey = make_float4(yp.x - c.x, yp.y - c.y, yp.z - c.z, yp.w - c.w);
        } else if (y == nx - 1) {
            const float4 ym = __ldg(phi4 + gym + z * plane4);
            ey = make_float4(c.x - ym.x, c.y - ym.y, c.z - ym.z, c.w - ym.w);
        } else {
            const float4 yp = __ldg(phi4 + gyp + z * plane4);
            const float4 ym = __ldg(phi4 + gym + z * plane4);
            ey = make_float4(0.5f * (yp.x - ym.x), 0.5f * (yp.y - ym.y), 0.5f * (yp.z - ym.z),
                             0.5f * (yp.w - ym.w));
        }
        // z
        const float4 zm = pv[k], zp = pv[k + 2];
        float4 ez;
        if (z == 0) ez = make_float4(zp.x - c.x, zp.y - c.y, zp.z - c.z, zp.w - c.w);
        else if (z == nx - 1) ez = make_float4(c.x - zm.x, c.y - zm.y, c.z - zm.z, c.w - zm.w);
        else
            ez = make_float4(0.5f * (zp.x - zm.x), 0.5f * (zp.y - zm.y), 0.5f * (zp.z - zm.z),
                             0.5f * (zp.w - zm.w));
        float4* o = acc4 + (static_cast<size_t>(z) * nx + y) * nx + x;
        o[0] = make_float4(d0 * coef, ey.x * coef, ez.x * coef, c.x);
        o[1] = make_float4(d1 * coef, ey.y * coef, ez.y * coef, c.y);
        o[2] = make_float4(d2 * coef, ey.z * coef, ez.z * coef, c.z);
        o[3] = make_float4(d3 * coef, ey.w * coef, ez.w * coef, c.w);
    }
}

// ----------------------------------------------------------------------------------------------
// Trilinear gather (interpolate_acceleration_to_particles_kernel, rm_mesh2p.cu:48-114).
// Index selection as the reference: f = (x - domain_min) / dx - 0.5 in FP64, i0 = floorf(f)
// (the reference passes its double to floorf, i.e. floors the float-rounded value), weights
// from the unclamped fraction, indices clamped to [0, nx - 1]; summation order z, y, x.
// ----------------------------------------------------------------------------------------------
// DIV: divide by dx as the reference (FP64 path); else multiply by 1 / dx (FP32 and MIXED,
// whose weights are rounded to float: an FP64 division per axis dominated the particle pass).
template <bool DIV>
__device__ __forceinline__ void interp_axis(double x, double dmin, double dx, double inv_dx,
                                            int nx, int& i0, int& i1, double& w) {
    const double f = (DIV ? (x - dmin) / dx : (x - dmin) * inv_dx) - 0.5;
    int a = static_cast<int>(floorf(static_cast<float>(f)));
    w = f - a;
    i0 = max(0, min(a, nx - 1));
    i1 = max(0, min(a + 1, nx - 1));
}

template <typename R>
__device__ __forceinline__ void trilinear(const V4<R>* __restrict__ acc4, const GridDev& g,
                                          double x, double y, double z, R& ax, R& ay, R& az) {
    int i0, i1, j0, j1, k0, k1;
    double wxd, wyd, wzd;
    constexpr bool DIV = sizeof(R) == 8;
    interp_axis<DIV>(x, g.domain_min, g.dx, g.inv_dx, g.nx, i0, i1, wxd);
    interp_axis<DIV>(y, g.domain_min, g.dx, g.inv_dx, g.nx, j0, j1, wyd);
    interp_axis<DIV>(z, g.domain_min, g.dx, g.inv_dx, g.nx, k0, k1, wzd);
    const R wx = static_cast<R>(wxd), wy = static_cast<R>(wyd), wz = static_cast<R>(wzd);
    const int nx = g.nx;  // nx^3 < 2^31 (nx <= 1024)
    ax = ay = az = R(0);
#pragma unroll
    for (int k = 0; k <= 1; ++k) {
        const int kk = k == 0 ? k0 : k1;
        const R wk = k == 0 ? (R(1) - wz) : wz;
#pragma unroll
        for (int j = 0; j <= 1; ++j) {
            const int jj = j == 0 ? j0 : j1;
            const R wj = j == 0 ? (R(1) - wy) : wy;
#pragma unroll
            for (int i = 0; i <= 1; ++i) {
                const int ii = i == 0 ? i0 : i1;
                const R wi = i == 0 ? (R(1) - wx) : wx;
                const R weight = wi * wj * wk;
                const V4<R> f = acc4[(kk * nx + jj) * nx + ii];
                ax += weight * f.x;
                ay += weight * f.y;
                az += weight * f.z;
            }
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(256) interp_kernel(int64_t n, const void* __restrict__ posm,
                                                     const V4<float>* __restrict__ lo, GridDev g,
                                                     const V4<R>* __restrict__ acc4,
                                                     V4<R>* __restrict__ acc) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x, y, z, m;
    load_pos<R>(posm, lo, i, x, y, z, m);
    R ax, ay, az;
    trilinear<R>(acc4, g, x, y, z, ax, ay, az);
    acc[i] = v4<R>(ax, ay, az, R(0));
}

// NGP cell as assign_particles_to_cells_ (rm_p2mesh.cu:37-49): truncation, clamp.
__device__ __forceinline__ int ngp_axis(double x, double dmin, double dx, int nx) {
    const double f = (x - dmin) / dx;
    int a = (f == f) ? static_cast<int>(f) : 0;
    return max(0, min(a, nx - 1));
}

template <typename R>
__global__ void __launch_bounds__(256) ngp_phi_kernel(int64_t n, const void* __restrict__ posm,
                                                      const V4<float>* __restrict__ lo,
                                                      GridDev g, const R* __restrict__ phi,
                                                      R* __restrict__ pot) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x, y, z, m;
    load_pos<R>(posm, lo, i, x, y, z, m);
    const int64_t nx = g.nx;
    const int64_t c = ngp_axis(x, g.domain_min, g.dx, g.nx) +
                      ngp_axis(y, g.domain_min, g.dx, g.nx) * nx +
                      ngp_axis(z, g.domain_min, g.dx, g.nx) * nx * nx;
    pot[i] = phi[c];
}

// ----------------------------------------------------------------------------------------------
// NGP projections of particle values onto the grid (N-body strategy with a grid,
// rrgsim_integration_nbody.cuh:32-48): per-cell particle counts (assign_particles_to_cells_,
// rm_p2mesh.cu:25-66), then each particle adds value / count of its cell
// (deposit_cell_grav_NGP_ / deposit_cell_acc_NGP_, rm_p2mesh.cu:142-174).
template <typename R>
__device__ __forceinline__ int64_t ngp_cell(const void* posm, const V4<float>* lo, int64_t i,
                                            const GridDev& g) {
    double x, y, z, m;
    load_pos<R>(posm, lo, i, x, y, z, m);
    const int64_t nx = g.nx;
    return ngp_axis(x, g.domain_min, g.dx, g.nx) + ngp_axis(y, g.domain_min, g.dx, g.nx) * nx +
           ngp_axis(z, g.domain_min, g.dx, g.nx) * nx * nx;
}

template <typename R>
__global__ void __launch_bounds__(256) ngp_count_kernel(int64_t n, const void* __restrict__ posm,
                                                        const V4<float>* __restrict__ lo,
                                                        GridDev g, int* __restrict__ count) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    atomicAdd(count + ngp_cell<R>(posm, lo, i, g), 1);
}

template <typename R>
__global__ void __launch_bounds__(256) ngp_project_kernel(int64_t n, const void* __restrict__ posm,
                                                          const V4<float>* __restrict__ lo,
                                                          GridDev g, const int* __restrict__ count,
                                                          const R* __restrict__ pot,
                                                          const V4<R>* __restrict__ acc,
                                                          R* __restrict__ phi_grid,
                                                          R* __restrict__ acc_grid) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t c = ngp_cell<R>(posm, lo, i, g);
    const R cnt = static_cast<R>(count[c]);
    if (phi_grid) atomicAdd(phi_grid + c, pot[i] / cnt);
    if (acc_grid) {
        const V4<R> a = acc[i];
        const R inv = R(1) / cnt;
        atomicAdd(acc_grid + 4 * c, a.x * inv);
        atomicAdd(acc_grid + 4 * c + 1, a.y * inv);
        atomicAdd(acc_grid + 4 * c + 2, a.z * inv);
    }
}

// ----------------------------------------------------------------------------------------------
// Fused particle pass of the wave strategy (one launch per step):
//   [INTERP_CORRECT]  a = trilinear(x); v = (u + dt a) / 2                  (correct_step_)
//   [PREDICT_DEPOSIT] v* = v + dt a; u = v + v*; x += dt/2 u; CIC(x)        (predict_step_ +
//                                                                             deposit)
// ----------------------------------------------------------------------------------------------
template <typename R, bool MIXED, int MODE>
__global__ void __launch_bounds__(kPmThreads, 6) pm_particle_kernel(PmParticleArgs a, double scale) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool active = i < a.n;
    // PM_SUMS: every particle's 8 conservation terms, kept in shared memory until the block's
    // record is formed at the end of the pass (16 KB per block, reused by the reduction)
    constexpr bool SUMS = (MODE & PM_SUMS) != 0;
    __shared__ double terms[SUMS ? kConsTerms : 1][SUMS ? kPmThreads : 1];
    V4<R>* posm = static_cast<V4<R>*>(a.posm);
    V4<float>* lo = static_cast<V4<float>*>(a.poslo);
    V4<R>* vel = static_cast<V4<R>*>(a.vel);
    V4<R>* accp = static_cast<V4<R>*>(a.acc);
    V4<R>* u = static_cast<V4<R>*>(a.u);
    const R dt = static_cast<R>(a.dt);
    double x = 0, y = 0, z = 0, m = 0;
    if (active) load_pos<R>(a.posm, MIXED ? lo : nullptr, i, x, y, z, m);

    R vx = 0, vy = 0, vz = 0, ax = 0, ay = 0, az = 0;
    if (active) {
        if constexpr ((MODE & PM_INTERP_CORRECT) != 0) {
            trilinear<R>(static_cast<const V4<R>*>(a.acc4), a.g, x, y, z, ax, ay, az);
            const V4<R> uu = u[i];
            vx = R(0.5) * (uu.x + dt * ax);
            vy = R(0.5) * (uu.y + dt * ay);
            vz = R(0.5) * (uu.z + dt * az);
            if constexpr ((MODE & PM_WRITE_SYNC) != 0) {
                vel[i] = v4<R>(vx, vy, vz, R(0));
                accp[i] = v4<R>(ax, ay, az, R(0));
            }
        } else {
            const V4<R> v = vel[i];
            const V4<R> ac = accp[i];
            vx = v.x; vy = v.y; vz = v.z;
            ax = ac.x; ay = ac.y; az = ac.z;
        }
    }
    if constexpr (SUMS) {
        // the synced state's terms, formed as conservation_kernel forms them (x, v and phi
        // promoted to double); stored now, so the deposit below has the registers
        const double ph = active ? static_cast<double>(static_cast<const R*>(a.pot)[i]) : 0.0;
#pragma unroll
        for (int k = 0; k < kConsTerms; ++k)
            terms[k][threadIdx.x] =
                active ? cons_term(k, x, y, z, m, static_cast<double>(vx),
                                   static_cast<double>(vy), static_cast<double>(vz), ph)
                       : 0.0;
    }
    if constexpr ((MODE & PM_PREDICT_DEPOSIT) != 0) {
        if (active) {
            const R sx = vx + dt * ax, sy = vy + dt * ay, sz = vz + dt * az;
            const R ux = vx + sx, uy = vy + sy, uz = vz + sz;
            u[i] = v4<R>(ux, uy, uz, R(0));
            const R hdt = dt * R(0.5);
            V4<R> p = posm[i];
            if constexpr (MIXED) {
                V4<float> l = lo[i];
                df_add(p.x, l.x, hdt * ux);
                df_add(p.y, l.y, hdt * uy);
                df_add(p.z, l.z, hdt * uz);
                (a.lo_out ? static_cast<V4<float>*>(a.lo_out) : lo)[i] = l;
                x = static_cast<double>(p.x) + l.x;
                y = static_cast<double>(p.y) + l.y;
                z = static_cast<double>(p.z) + l.z;
            } else {
                p.x = p.x + hdt * ux;
                p.y = p.y + hdt * uy;
                p.z = p.z + hdt * uz;
                x = p.x;
                y = p.y;
                z = p.z;
            }
            (a.pos_out ? static_cast<V4<R>*>(a.pos_out) : posm)[i] = p;
        }
        cic_deposit_warp(active, x, y, z, m, a.g, scale, a.mgrid);
    }
    if constexpr (SUMS) {
        // the block's record, in three fixed-order stages (FP64 issue, not latency, is what
        // this costs, so every stage keeps its warps' lanes busy): warp k sums term k, each
        // lane 8 particles' terms (cascaded); two warps combine those 32 partials per term 4 at
        // a time; then one lane per term adds the last 8. Records are value-major,
        // partial[(k gridDim.x + block) 2 + {0, 1}], so the finishing kernel reads them
        // coalesced.
        static_assert(kPmThreads / 32 == kConsTerms, "one warp per term");
        static_assert(sizeof(DD) * kConsTerms * 40 <= sizeof(double) * kConsTerms * kPmThreads,
                      "the stages fit in the terms' shared memory");
        DD (*stage)[40] = reinterpret_cast<DD (*)[40]>(&terms[0][0]);
        __syncthreads();
        const int t = threadIdx.x;
        {
            const int k = t >> 5, lane = t & 31;
            Casc c{terms[k][lane], 0.0};
#pragma unroll
            for (int j = lane + 32; j < kPmThreads; j += 32) casc_add(c, terms[k][j]);
            __syncthreads();  // every term read before the stages overwrite them
            stage[k][lane] = dd_norm(c.s, c.c);
        }
        __syncthreads();
        if (t < 64) {
            const int k = t >> 3, q = t & 7;
            DD d = stage[k][4 * q];
#pragma unroll
            for (int j = 1; j < 4; ++j) d = dd_add(d, stage[k][4 * q + j]);
            stage[k][32 + q] = d;
        }
        __syncthreads();
        if (t < kConsTerms) {
            DD d = stage[t][32];
#pragma unroll
            for (int j = 1; j < 8; ++j) d = dd_add(d, stage[t][32 + j]);
            const int64_t o = (static_cast<int64_t>(t) * gridDim.x + blockIdx.x) * 2;
            a.partial[o] = d.hi;
            a.partial[o + 1] = d.lo;
        }
    }
}

template <typename R, bool MIXED>
void dispatch_pm(const PmParticleArgs& a, int mode, double scale, cudaStream_t s) {
    const int b = div_up(a.n, 256);
    switch (mode) {
        case PM_INTERP_CORRECT | PM_WRITE_SYNC:
            pm_particle_kernel<R, MIXED, PM_INTERP_CORRECT | PM_WRITE_SYNC><<<b, 256, 0, s>>>(a, scale);
            break;
        case PM_PREDICT_DEPOSIT:
            pm_particle_kernel<R, MIXED, PM_PREDICT_DEPOSIT><<<b, 256, 0, s>>>(a, scale);
            break;
        case PM_INTERP_CORRECT | PM_PREDICT_DEPOSIT:
            pm_particle_kernel<R, MIXED, PM_INTERP_CORRECT | PM_PREDICT_DEPOSIT><<<b, 256, 0, s>>>(a, scale);
            break;
        case PM_INTERP_CORRECT | PM_PREDICT_DEPOSIT | PM_WRITE_SYNC:
            pm_particle_kernel<R, MIXED, PM_INTERP_CORRECT | PM_PREDICT_DEPOSIT | PM_WRITE_SYNC>
                <<<b, 256, 0, s>>>(a, scale);
            break;
        case PM_INTERP_CORRECT | PM_PREDICT_DEPOSIT | PM_WRITE_SYNC | PM_SUMS:
            pm_particle_kernel<R, MIXED,
                               PM_INTERP_CORRECT | PM_PREDICT_DEPOSIT | PM_WRITE_SYNC | PM_SUMS>
                <<<b, 256, 0, s>>>(a, scale);
            break;
        default:
            throw Error(RRG_ERR_INVALID, "pm particle pass: unsupported mode");
    }
}

}  // namespace

// ----------------------------------------------------------------------------------------------
void launch_cic_deposit(int prec, int64_t n, const void* posm, const void* poslo,
                        const GridDev& g, int shift_s, unsigned long long* grid,
                        cudaStream_t s) {
    const double scale = ldexp(1.0, shift_s);
    const int b = div_up(n, 256);
    if (prec == RRG_PREC_FP64)
        cic_kernel<double><<<b, 256, 0, s>>>(n, posm, nullptr, g, scale, grid);
    else
        cic_kernel<float><<<b, 256, 0, s>>>(
            n, posm, prec == RRG_PREC_MIXED ? static_cast<const V4<float>*>(poslo) : nullptr, g,
            scale, grid);
    RRG_LAUNCHED();
}

void launch_wave_source(int prec, int nx, const unsigned long long* mgrid, int shift_s,
                        double dx, double rho_mean, double scale, void* src, bool zero_grid,
                        cudaStream_t s) {
    const int64_t nc = static_cast<int64_t>(nx) * nx * nx;
    const double inv_scale = ldexp(1.0, -shift_s);
    auto* mg = const_cast<unsigned long long*>(mgrid);
    const double dx3 = dx * dx * dx;
    if (prec == RRG_PREC_FP64)
        wave_source_kernel<double><<<div_up(nc, 256), 256, 0, s>>>(
            nc, mg, inv_scale, dx3, 1.0 / dx3, rho_mean, scale, static_cast<double*>(src),
            zero_grid);
    else
        wave_source_kernel<float><<<div_up(nc, 256), 256, 0, s>>>(
            nc, mg, inv_scale, dx3, 1.0 / dx3, rho_mean, scale, static_cast<float*>(src),
            zero_grid);
    RRG_LAUNCHED();
}

void launch_wave_inc_prep(int nx, const unsigned long long* mg, unsigned long long* mg_zero,
                          int shift_s, double dx, double rho_sub, const float* phi0,
                          const float* phi_prev, const WaveCoef& w, float* g, float* d,
                          float* d_old, float* src, cudaStream_t s) {
    const int64_t nc = static_cast<int64_t>(nx) * nx * nx;
    wave_inc_prep_kernel<<<div_up(nc, 256), 256, 0, s>>>(
        nx, mg, mg_zero, ldexp(1.0, -shift_s), 1.0 / (dx * dx * dx), rho_sub, phi0, phi_prev,
        w.K_F, w.K_MAIN, w.K_ACTUAL + w.K_OLD - 1.0, g, d, d_old, src);
    RRG_LAUNCHED();
}

void launch_wave_inc_finish(int nx, const float* phi0, const float* d_fin, const float* d_prv,
                            float* fin, float* prv, cudaStream_t s) {
    const int64_t nc = static_cast<int64_t>(nx) * nx * nx;
    wave_inc_finish_kernel<<<div_up(nc, 256), 256, 0, s>>>(nc, phi0, d_fin, d_prv, fin, prv);
    RRG_LAUNCHED();
}

// One adjoint substep of the PM adjoint with the float4 stencil (FP32, periodic): false,
// launching nothing, on grids whose rows do not tile into warps.
bool launch_wave_adjoint_step(int nx, const float* C, float* P, float* F, double km, double ka,
                              double beta, double kf, cudaStream_t s) {
    const int W4 = nx / 4;
    if (nx < 16 || nx % 8 != 0 || !(32 % W4 == 0 || W4 % 32 == 0)) return false;
    WaveDev w{};
    w.nx = nx;
    w.uniform = 1;
    w.bc = RRG_BC_PERIODIC;
    w.K_MAIN = km;
    w.K_ACTUAL = ka;
    w.K_OLD = beta;
    w.K_F = kf;
    // z-chunk as the forward stencil chooses it: the longest of 8, 4, 2 planes that still gives
    // two 256-thread blocks' worth of threads per SM
    int dev = 0;
    RRG_CUDA(cudaGetDevice(&dev));
    const int sms = num_sms(dev);
    const int bs = 128;
    const int rows_blocks = div_up(static_cast<int64_t>(W4) * nx, bs);
    int zx = 2;
    for (int cand : {8, 4})
        if (static_cast<int64_t>(rows_blocks) * (nx / cand) * bs >= 2 * 256 * sms) {
            zx = cand;
            break;
        }
    const dim3 g4(rows_blocks, nx / zx);
    if (zx == 8)
        wave_periodic_x4_kernel<8, false, 128, true><<<g4, bs, 0, s>>>(C, P, nullptr, w, nullptr, F);
    else if (zx == 4)
        wave_periodic_x4_kernel<4, false, 128, true><<<g4, bs, 0, s>>>(C, P, nullptr, w, nullptr, F);
    else
        wave_periodic_x4_kernel<2, false, 128, true><<<g4, bs, 0, s>>>(C, P, nullptr, w, nullptr, F);
    RRG_LAUNCHED();
    return true;
}

// RRG_WAVE_BS = 128 / 256 fixes the block size of the float4 stencil (for sweeps).
int wave_bs_override() {
    static const int v = [] {
        const char* e = std::getenv("RRG_WAVE_BS");
        return e ? std::atoi(e) : 0;
    }();
    return v;
}

// RRG_WAVE_ZC = 2 / 4 / 8 fixes the z-chunk of the float4 stencil (for sweeps).
int wave_zc_override() {
    static const int v = [] {
        const char* e = std::getenv("RRG_WAVE_ZC");
        return e ? std::atoi(e) : 0;
    }();
    return v;
}

void launch_wave_step(int prec, int nx, const void* phi, void* phi_old_inout, const void* src,
                      const WaveCoef& c, unsigned long long* maxbits, cudaStream_t s) {
    WaveDev w;
    w.nx = nx;
    w.bc = c.bc_type;
    w.uniform = (c.bc_type == RRG_BC_PERIODIC && !c.keep_layer) ? 1 : 0;
    w.K_MAIN = c.K_MAIN;
    w.K_ACTUAL = c.K_ACTUAL;
    w.K_OLD = c.K_OLD;
    w.K_F = c.K_F;
    w.C = c.C;
    w.DT = c.DT;
    w.DX = c.DX;
    w.diss_base = c.diss_base;
    w.diss_extra = c.diss_extra;
    w.sim_l = c.sim_l;
    w.domain_min = c.domain_min;
    w.bc_mass = c.bc_mass;
    w.comx = c.com[0];
    w.comy = c.com[1];
    w.comz = c.com[2];
    w.r_min = c.r_min;
    const int gx = div_up(nx, kTX), gy = div_up(nx, kTY);
    // z-chunk: trade wave efficiency (blocks against 8 resident 256-thread blocks per SM)
    // against the one extra plane each column loads per chunk
    int dev = 0;
    RRG_CUDA(cudaGetDevice(&dev));
    static int sms = 0;
    if (!sms) sms = num_sms(dev);
    const int64_t slots = static_cast<int64_t>(sms) * 8;
    int zc = 32;
    double best = -1.0;
    for (int cand : {2, 4, 8, 16, 32, 64}) {
        if (cand > nx && cand != 2) break;
        const int64_t blocks = static_cast<int64_t>(gx) * gy * div_up(nx, cand);
        const int64_t waves = (blocks + slots - 1) / slots;
        const double eff = static_cast<double>(blocks) / static_cast<double>(waves * slots) *
                           cand / (cand + 1.0);
        if (eff > best + 1e-9) {
            best = eff;
            zc = cand;
        }
    }
    w.zc = zc;
    dim3 grid(gx, gy, div_up(nx, zc));
    dim3 block(kTX, kTY);
    const bool check = maxbits != nullptr;
    const int W4 = nx / 4;
    if (w.uniform && prec != RRG_PREC_FP64 && nx >= 16 && nx % 4 == 0 &&
        (32 % W4 == 0 || W4 % 32 == 0)) {
        // float4 rows: z-chunk of 2, 4 or 8 planes (dividing nx), at least two blocks per SM
        // (at 128^3 that is 4, measured fastest inside the PM step on B200)
        // 128-thread blocks: at 128^3 with 4-plane chunks 1024 blocks fill 8 per SM to 99%
        // (256-thread blocks: 512 on 4 per SM, 86%); measured faster inside the PM step
        const int bs = wave_bs_override() == 256 ? 256 : 128;
        const int rows_blocks = div_up(static_cast<int64_t>(W4) * nx, bs);
        int zx = wave_zc_override();
        if (zx != 2 && zx != 4 && zx != 8) {
            zx = 2;
            for (int cand : {8, 4})
                if (nx % cand == 0 &&
                    static_cast<int64_t>(rows_blocks) * (nx / cand) * bs >= 2 * 256 * sms) {
                    zx = cand;
                    break;
                }
        }
        if (nx % zx != 0) zx = 2;
        dim3 g4(rows_blocks, nx / zx);
        const float* p = static_cast<const float*>(phi);
        float* po = static_cast<float*>(phi_old_inout);
        const float* sr = static_cast<const float*>(src);
#define RRG_WAVE_X4B(Z, B)                                                                   \
    do {                                                                                      \
        if (check) wave_periodic_x4_kernel<Z, true, B><<<g4, B, 0, s>>>(p, po, sr, w, maxbits); \
        else wave_periodic_x4_kernel<Z, false, B><<<g4, B, 0, s>>>(p, po, sr, w, maxbits);      \
    } while (0)
#define RRG_WAVE_X4(Z)                  \
    do {                                \
        if (bs == 128) RRG_WAVE_X4B(Z, 128); \
        else RRG_WAVE_X4B(Z, 256);      \
    } while (0)
        if (zx == 8) RRG_WAVE_X4(8);
        else if (zx == 4) RRG_WAVE_X4(4);
        else RRG_WAVE_X4(2);
#undef RRG_WAVE_X4
#undef RRG_WAVE_X4B
        RRG_LAUNCHED();
        return;
    }
    if (w.uniform) {
        // compile-time chunk of 2, 4 or 8 planes, the nearest the chooser's pick
        const int zcf = zc >= 8 ? 8 : (zc >= 4 ? 4 : 2);
        dim3 g2(gx, gy, div_up(nx, zcf));
#define RRG_WAVE_P(R, Z)                                                                      \
    do {                                                                                      \
        const R* p = static_cast<const R*>(phi);                                              \
        R* po = static_cast<R*>(phi_old_inout);                                               \
        const R* sr = static_cast<const R*>(src);                                             \
        if (check) wave_periodic_kernel<R, Z, true><<<g2, block, 0, s>>>(p, po, sr, w, maxbits); \
        else wave_periodic_kernel<R, Z, false><<<g2, block, 0, s>>>(p, po, sr, w, maxbits);      \
    } while (0)
        if (prec == RRG_PREC_FP64) {
            if (zcf == 8) RRG_WAVE_P(double, 8);
            else if (zcf == 4) RRG_WAVE_P(double, 4);
            else RRG_WAVE_P(double, 2);
        } else {
            if (zcf == 8) RRG_WAVE_P(float, 8);
            else if (zcf == 4) RRG_WAVE_P(float, 4);
            else RRG_WAVE_P(float, 2);
        }
#undef RRG_WAVE_P
        RRG_LAUNCHED();
        return;
    }
#define RRG_WAVE_LAUNCH(R)                                                                    \
    do {                                                                                      \
        const R* p = static_cast<const R*>(phi);                                              \
        R* po = static_cast<R*>(phi_old_inout);                                               \
        const R* sr = static_cast<const R*>(src);                                             \
        if (w.uniform) {                                                                      \
            if (check) wave_step_kernel<R, true, true><<<grid, block, 0, s>>>(p, po, sr, w, maxbits); \
            else wave_step_kernel<R, true, false><<<grid, block, 0, s>>>(p, po, sr, w, maxbits);     \
        } else {                                                                              \
            if (check) wave_step_kernel<R, false, true><<<grid, block, 0, s>>>(p, po, sr, w, maxbits); \
            else wave_step_kernel<R, false, false><<<grid, block, 0, s>>>(p, po, sr, w, maxbits);     \
        }                                                                                     \
    } while (0)
    if (prec == RRG_PREC_FP64) RRG_WAVE_LAUNCH(double);
    else RRG_WAVE_LAUNCH(float);
#undef RRG_WAVE_LAUNCH
    RRG_LAUNCHED();
}

void launch_gradient(int prec, int nx, double dx, const void* phi, void* acc4, cudaStream_t s) {
    const double coef = -1.0 / dx;
    const int W4 = nx / 4;
    if (prec != RRG_PREC_FP64 && nx >= 8 && nx % 4 == 0 && (32 % W4 == 0 || W4 % 32 == 0)) {
        dim3 g4(div_up(static_cast<int64_t>(W4) * nx, 128), nx / 4);
        gradient_x4_kernel<4, 128><<<g4, 128, 0, s>>>(nx, static_cast<float>(coef),
                                                      static_cast<const float*>(phi),
                                                      static_cast<float4*>(acc4));
        RRG_LAUNCHED();
        return;
    }
    dim3 grid(div_up(nx, kTX), div_up(nx, kTY), nx);
    dim3 block(kTX, kTY);
    if (prec == RRG_PREC_FP64)
        gradient_kernel<double><<<grid, block, 0, s>>>(nx, coef, static_cast<const double*>(phi),
                                                       static_cast<V4<double>*>(acc4));
    else
        gradient_kernel<float><<<grid, block, 0, s>>>(nx, static_cast<float>(coef),
                                                      static_cast<const float*>(phi),
                                                      static_cast<V4<float>*>(acc4));
    RRG_LAUNCHED();
}

void launch_interp(int prec, int64_t n, const void* posm, const void* poslo, const GridDev& g,
                   const void* acc4, void* acc, cudaStream_t s) {
    const int b = div_up(n, 256);
    if (prec == RRG_PREC_FP64)
        interp_kernel<double><<<b, 256, 0, s>>>(n, posm, nullptr, g,
                                                static_cast<const V4<double>*>(acc4),
                                                static_cast<V4<double>*>(acc));
    else
        interp_kernel<float><<<b, 256, 0, s>>>(
            n, posm, prec == RRG_PREC_MIXED ? static_cast<const V4<float>*>(poslo) : nullptr, g,
            static_cast<const V4<float>*>(acc4), static_cast<V4<float>*>(acc));
    RRG_LAUNCHED();
}

void launch_ngp_phi(int prec, int64_t n, const void* posm, const void* poslo, const GridDev& g,
                    const void* phi, void* pot, cudaStream_t s) {
    const int b = div_up(n, 256);
    if (prec == RRG_PREC_FP64)
        ngp_phi_kernel<double><<<b, 256, 0, s>>>(n, posm, nullptr, g,
                                                 static_cast<const double*>(phi),
                                                 static_cast<double*>(pot));
    else
        ngp_phi_kernel<float><<<b, 256, 0, s>>>(
            n, posm, prec == RRG_PREC_MIXED ? static_cast<const V4<float>*>(poslo) : nullptr, g,
            static_cast<const float*>(phi), static_cast<float*>(pot));
    RRG_LAUNCHED();
}

void launch_ngp_project(int prec, int64_t n, const void* posm, const void* poslo,
                        const GridDev& g, int* count, const void* pot, const void* acc,
                        void* phi_grid, void* acc4_grid, cudaStream_t s) {
    const int b = div_up(n, 256);
    const V4<float>* lo = prec == RRG_PREC_MIXED ? static_cast<const V4<float>*>(poslo) : nullptr;
    if (prec == RRG_PREC_FP64) {
        ngp_count_kernel<double><<<b, 256, 0, s>>>(n, posm, nullptr, g, count);
        RRG_LAUNCHED();
        ngp_project_kernel<double><<<b, 256, 0, s>>>(
            n, posm, nullptr, g, count, static_cast<const double*>(pot),
            static_cast<const V4<double>*>(acc), static_cast<double*>(phi_grid),
            static_cast<double*>(acc4_grid));
    } else {
        ngp_count_kernel<float><<<b, 256, 0, s>>>(n, posm, lo, g, count);
        RRG_LAUNCHED();
        ngp_project_kernel<float><<<b, 256, 0, s>>>(
            n, posm, lo, g, count, static_cast<const float*>(pot),
            static_cast<const V4<float>*>(acc), static_cast<float*>(phi_grid),
            static_cast<float*>(acc4_grid));
    }
    RRG_LAUNCHED();
}

void launch_pm_particles(const PmParticleArgs& a, int mode, cudaStream_t s) {
    const double scale = ldexp(1.0, a.shift_s);
    if (a.prec == RRG_PREC_FP64) dispatch_pm<double, false>(a, mode, scale, s);
    else if (a.prec == RRG_PREC_MIXED) dispatch_pm<float, true>(a, mode, scale, s);
    else dispatch_pm<float, false>(a, mode, scale, s);
    RRG_LAUNCHED();
}

}  // namespace rrg
