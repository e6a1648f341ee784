// Hand-written adjoint of the particle-mesh leapfrog (periodic wave potential) on sm_100a.
//
// Forward step (RectWaveIntegrationSolver::calc_step, rrgsim_integration_rect.cuh:99-112):
//   u  = 2 v + dt a;  x' = x + dt/2 u                       (predict_step_, nbody.cu:122-152)
//   M  = CIC(x', m)                                         (rm_p2mesh.cu:176-236)
//   f  = 4 pi (M / dx^3 - rho_mean)                         (wave.cu:150-153)
//   S substeps  phi_new = K_M L6(phi) + K_A phi + K_O phi_old + K_F f   (wave.cu:163-192)
//   g  = -D phi                                             (rm_p2mesh.cu:238-290)
//   a' = T(x') g                                            (rm_mesh2p.cu:48-114)
//   v' = (u + dt a') / 2                                    (correct_step_, nbody.cu:159-181)
// Every map but the two particle/grid couplings is linear, so the backward pass is:
//   - correct:  U = V'/2, A'' = A' + dt/2 V'
//   - interp:   gbar = T(x')^T A'' (a CIC-style scatter); x' gets sum_c dw_c/dx' (g_c . A'')
//   - gradient: Phi_cur += -D^T gbar
//   - substeps in reverse: (P, C) -> (K_O C, K_M L6 C + K_A C + P), F += K_F C (L6 is
//     symmetric on the periodic box, so the adjoint substep is the same stencil)
//   - source:   Mbar = 4 pi F / dx^3
//   - deposit:  m gets sum_c w_c Mbar_c (a trilinear gather, the CIC adjoint); x' gets
//               m sum_c dw_c/dx' Mbar_c (zero where the reference clamps)
//   - predict:  U += dt/2 X, V = 2 U, A = dt U, X passes through.
// The initial potential is a fixed input (the relaxation before the first step is not
// differentiated); a_0 = T(x_0) g_0 is, through x_0. The fixed-point rounding of the deposit
// is treated as the identity (its relative size is 2^-27).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "host_io.h"
#include "kernels.cuh"

namespace rrg {
namespace {

constexpr double kPi = 3.14159265358979;

__device__ __forceinline__ void interp_axis_w(double x, double dmin, double dx, int nx, int& i0,
                                              int& i1, double& w) {
    const double f = (x - dmin) / dx - 0.5;
    const int a = static_cast<int>(floorf(static_cast<float>(f)));
    w = f - a;
    i0 = max(0, min(a, nx - 1));
    i1 = max(0, min(a + 1, nx - 1));
}

// interp adjoint: gbar += T(x)^T A (atomics, when gbar != nullptr; gbar holds 4 values per
// cell, the fourth unused); X = sum dW/dx (g . A)
template <typename R>
__global__ void __launch_bounds__(256) interp_adjoint_kernel(int64_t n, const V4<R>* __restrict__ posm,
                                                             GridDev g, const V4<R>* __restrict__ acc4,
                                                             const V4<R>* __restrict__ A,
                                                             R* __restrict__ gbar,
                                                             V4<R>* __restrict__ X) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const V4<R> q = posm[p];
    const V4<R> a = A[p];
    int ii[2], jj[2], kk[2];
    double wx, wy, wz;
    interp_axis_w(q.x, g.domain_min, g.dx, g.nx, ii[0], ii[1], wx);
    interp_axis_w(q.y, g.domain_min, g.dx, g.nx, jj[0], jj[1], wy);
    interp_axis_w(q.z, g.domain_min, g.dx, g.nx, kk[0], kk[1], wz);
    const R wxs[2] = {R(1) - R(wx), R(wx)}, wys[2] = {R(1) - R(wy), R(wy)},
            wzs[2] = {R(1) - R(wz), R(wz)};
    const R inv = R(1.0 / g.dx);
    const R dws[2] = {-inv, inv};
    const int64_t nx = g.nx;
    R gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int64_t c = kk[k] * nx * nx + jj[j] * nx + ii[i];
                const V4<R> f = acc4[c];
                const R s = f.x * a.x + f.y * a.y + f.z * a.z;
                gx += dws[i] * wys[j] * wzs[k] * s;
                gy += wxs[i] * dws[j] * wzs[k] * s;
                gz += wxs[i] * wys[j] * dws[k] * s;
                if (gbar) {
                    const R W = wxs[i] * wys[j] * wzs[k];
                    if constexpr (sizeof(R) == 4) {
                        // one 16-byte vector atomic per corner instead of three scalar ones
                        atomicAdd(reinterpret_cast<float4*>(gbar) + c,
                                  make_float4(W * a.x, W * a.y, W * a.z, 0.f));
                    } else {
                        atomicAdd(gbar + 4 * c, W * a.x);
                        atomicAdd(gbar + 4 * c + 1, W * a.y);
                        atomicAdd(gbar + 4 * c + 2, W * a.z);
                    }
                }
            }
    X[p] = v4<R>(gx, gy, gz, R(0));
}

// gradient adjoint: phi += -1/dx D^T gbar (D: central inside, one-sided on the faces)
template <typename R>
__device__ __forceinline__ R dT_axis(const R* gb, int comp, int64_t c, int j, int n, int64_t st) {
    R s = 0;
    if (j - 1 >= 0) s += (j - 1 == 0 ? R(1) : R(0.5)) * gb[4 * (c - st) + comp];
    if (j + 1 <= n - 1) s -= (j + 1 == n - 1 ? R(1) : R(0.5)) * gb[4 * (c + st) + comp];
    if (j == 0) s -= gb[4 * c + comp];
    if (j == n - 1) s += gb[4 * c + comp];
    return s;
}

template <typename R>
__global__ void __launch_bounds__(256) gradient_adjoint_kernel(int nx, R coef, const R* __restrict__ gbar,
                                                               R* __restrict__ phi_bar) {
    const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t nc = static_cast<int64_t>(nx) * nx * nx;
    if (c >= nc) return;
    const int x = static_cast<int>(c % nx), y = static_cast<int>((c / nx) % nx),
              z = static_cast<int>(c / (static_cast<int64_t>(nx) * nx));
    const R s = dT_axis(gbar, 0, c, x, nx, 1) + dT_axis(gbar, 1, c, y, nx, nx) +
                dT_axis(gbar, 2, c, z, nx, static_cast<int64_t>(nx) * nx);
    phi_bar[c] += coef * s;
}

// adjoint substep on the periodic box: P <- K_M L6(C) + K_A C + beta P;  F += K_F C
template <typename R>
__global__ void __launch_bounds__(256) wave_adjoint_kernel(int nx, const R* __restrict__ C, R* __restrict__ P,
                                                           R* __restrict__ F, R km, R ka, R beta,
                                                           R kf) {
    const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t nc = static_cast<int64_t>(nx) * nx * nx;
    if (c >= nc) return;
    const int64_t plane = static_cast<int64_t>(nx) * nx;
    const int x = static_cast<int>(c % nx), y = static_cast<int>((c / nx) % nx),
              z = static_cast<int>(c / plane);
    const int64_t xm = x > 0 ? c - 1 : c + nx - 1, xp = x < nx - 1 ? c + 1 : c - (nx - 1);
    const int64_t ym = y > 0 ? c - nx : c + (nx - 1) * nx,
                  yp = y < nx - 1 ? c + nx : c - static_cast<int64_t>(nx - 1) * nx;
    const int64_t zm = z > 0 ? c - plane : c + (nx - 1) * plane,
                  zp = z < nx - 1 ? c + plane : c - (nx - 1) * plane;
    const R cc = C[c];
    const R lap = C[xm] + C[xp] + C[ym] + C[yp] + C[zm] + C[zp];
    P[c] = km * lap + ka * cc + beta * P[c];
    F[c] += kf * cc;
}

// deposit adjoint at x: m_bar += sum_c W_c Mbar_c; Xd = m sum_c dW_c/dx Mbar_c
// (CIC weights of rm_p2mesh.cu:191-216; derivative zero where u is clamped)
__device__ __forceinline__ void cic_axis_d(double x, double dmin, double inv_dx, int nx, int& i0,
                                           int& i1, double& w0, double& w1, double& du) {
    double u = (x - dmin) * inv_dx - 0.5;
    const double hi = static_cast<double>(nx - 1) - 1e-6;
    du = inv_dx;
    if (!(u >= 0.0)) {
        u = 0.0;
        du = 0.0;
    }
    if (u > hi) {
        u = hi;
        du = 0.0;
    }
    i0 = static_cast<int>(floor(u));
    i1 = min(i0 + 1, nx - 1);
    const double f = u - i0;
    w0 = 1.0 - f;
    w1 = f;
}

template <typename R>
__global__ void __launch_bounds__(256) deposit_adjoint_kernel(int64_t n, const V4<R>* __restrict__ posm,
                                                              GridDev g, const R* __restrict__ F,
                                                              R mscale, V4<R>* __restrict__ Xd) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const V4<R> q = posm[p];
    int ii[2], jj[2], kk[2];
    double wx[2], wy[2], wz[2], dux, duy, duz;
    cic_axis_d(q.x, g.domain_min, g.inv_dx, g.nx, ii[0], ii[1], wx[0], wx[1], dux);
    cic_axis_d(q.y, g.domain_min, g.inv_dx, g.nx, jj[0], jj[1], wy[0], wy[1], duy);
    cic_axis_d(q.z, g.domain_min, g.inv_dx, g.nx, kk[0], kk[1], wz[0], wz[1], duz);
    const double sgn[2] = {-1.0, 1.0};
    const int64_t nx = g.nx;
    double mb = 0, gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const double Mb = static_cast<double>(mscale) *
                                  static_cast<double>(F[kk[k] * nx * nx + jj[j] * nx + ii[i]]);
                mb += wx[i] * wy[j] * wz[k] * Mb;
                gx += sgn[i] * dux * wy[j] * wz[k] * Mb;
                gy += wx[i] * sgn[j] * duy * wz[k] * Mb;
                gz += wx[i] * wy[j] * sgn[k] * duz * Mb;
            }
    const double m = q.w;
    Xd[p] = v4<R>(static_cast<R>(m * gx), static_cast<R>(m * gy), static_cast<R>(m * gz),
                  static_cast<R>(mb));
}

// correct adjoint: U = V / 2, A += dt/2 V
template <typename R>
__global__ void correct_adjoint_kernel(int64_t n, const V4<R>* __restrict__ V, V4<R>* __restrict__ A,
                                       V4<R>* __restrict__ U, R dt) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const V4<R> v = V[p];
    V4<R> a = A[p];
    const R h = dt * R(0.5);
    a.x += h * v.x;
    a.y += h * v.y;
    a.z += h * v.z;
    A[p] = a;
    U[p] = v4<R>(R(0.5) * v.x, R(0.5) * v.y, R(0.5) * v.z, R(0));
}

// predict adjoint: Xt = X + Xi + Xd (w: m_bar accumulates Xd.w); U += dt/2 Xt; V = 2 U;
// A = dt U; X = Xt
template <typename R>
__global__ void predict_adjoint_kernel(int64_t n, V4<R>* __restrict__ X, const V4<R>* __restrict__ Xi,
                                       const V4<R>* __restrict__ Xd, const V4<R>* __restrict__ U,
                                       V4<R>* __restrict__ V, V4<R>* __restrict__ A, R dt) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const V4<R> x = X[p], xi = Xi[p], xd = Xd[p], u = U[p];
    const R tx = x.x + xi.x + xd.x, ty = x.y + xi.y + xd.y, tz = x.z + xi.z + xd.z;
    const R h = dt * R(0.5);
    const R ux = u.x + h * tx, uy = u.y + h * ty, uz = u.z + h * tz;
    X[p] = v4<R>(tx, ty, tz, x.w + xd.w);
    V[p] = v4<R>(R(2) * ux, R(2) * uy, R(2) * uz, R(0));
    A[p] = v4<R>(dt * ux, dt * uy, dt * uz, R(0));
}

template <typename R>
__global__ void add_xyz_kernel(int64_t n, V4<R>* __restrict__ X, const V4<R>* __restrict__ Y) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    V4<R> x = X[p];
    const V4<R> y = Y[p];
    x.x += y.x;
    x.y += y.y;
    x.z += y.z;
    X[p] = x;
}

template <typename R>
__global__ void scale_kernel(int64_t n, R* __restrict__ a, R s) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) a[i] *= s;
}

struct PBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~PBuf() {
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
            throw Error(RRG_ERR_NOMEM, std::string("pm adjoint: cudaMalloc failed: ") +
                                           cudaGetErrorString(e));
        }
        bytes = b;
    }
    char* c() const { return static_cast<char*>(p); }
};

}  // namespace
}  // namespace rrg

using namespace rrg;

struct rrg_pm_adjoint {
    int device = 0;
    int prec = RRG_PREC_FP32;
    size_t rsz = 4;
    int64_t n = 0;
    double dt = 0.0;
    int nsteps = 0, every = 20, substeps = 20;
    rrg_grid_info grid{};
    GridDev gdev{};
    WaveCoef wc{};
    double rho_mean = 0.0;
    int64_t nc = 0;
    int shift_s = 0;
    PBuf x, v, a, u, mg, src, phi[2], acc4;
    PBuf ck_x, ck_v, ck_a, ck_phi;     // per checkpoint: x, v, a, phi_prev, phi_cur
    PBuf seg_x, seg_phi;               // per step of a segment: x_{n+1}, phi_cur_{n+1}
    PBuf X, V, A, U, Xi, Xd, gbar, Cb, Pb, F;
    bool forward_done = false;
    std::string err;
};

namespace {

size_t pvb(const rrg_pm_adjoint* P) { return 4 * P->rsz * static_cast<size_t>(P->n); }
size_t gvb(const rrg_pm_adjoint* P) { return P->rsz * static_cast<size_t>(P->nc); }

// one PM step in place on (x, v, a, phi[0] = prev, phi[1] = cur)
void pm_step(rrg_pm_adjoint* P, cudaStream_t s) {
    launch_predict(P->prec, P->n, P->x.p, nullptr, P->v.p, P->a.p, P->u.p, P->dt, s);
    RRG_CUDA(cudaMemsetAsync(P->mg.p, 0, P->mg.bytes, s));
    launch_cic_deposit(P->prec, P->n, P->x.p, nullptr, P->gdev, P->shift_s,
                       static_cast<unsigned long long*>(P->mg.p), s);
    launch_wave_source(P->prec, P->grid.nx, static_cast<unsigned long long*>(P->mg.p), P->shift_s,
                       P->grid.dx, P->rho_mean, 1.0, P->src.p, false, s);
    for (int k = 0; k < P->substeps; ++k) {
        // phi[1] current, phi[0] previous: the new level overwrites phi[0], then roles swap
        launch_wave_step(P->prec, P->grid.nx, P->phi[1].p, P->phi[0].p, P->src.p, P->wc, nullptr, s);
        std::swap(P->phi[0].p, P->phi[1].p);
    }
    launch_gradient(P->prec, P->grid.nx, P->grid.dx, P->phi[1].p, P->acc4.p, s);
    launch_interp(P->prec, P->n, P->x.p, nullptr, P->gdev, P->acc4.p, P->a.p, s);
    launch_correct(P->prec, P->n, P->v.p, P->a.p, P->u.p, P->dt, s);
}

template <typename R>
void backward_step(rrg_pm_adjoint* P, const void* xn1, const void* phin1, cudaStream_t s) {
    const int64_t n = P->n, nc = P->nc;
    const int bp = div_up(n, 256), bg = div_up(nc, 256);
    auto* X = static_cast<V4<R>*>(P->X.p);
    auto* V = static_cast<V4<R>*>(P->V.p);
    auto* A = static_cast<V4<R>*>(P->A.p);
    auto* U = static_cast<V4<R>*>(P->U.p);
    auto* Xi = static_cast<V4<R>*>(P->Xi.p);
    auto* Xd = static_cast<V4<R>*>(P->Xd.p);
    const R dt = static_cast<R>(P->dt);
    correct_adjoint_kernel<R><<<bp, 256, 0, s>>>(n, V, A, U, dt);
    RRG_LAUNCHED();
    launch_gradient(P->prec, P->grid.nx, P->grid.dx, phin1, P->acc4.p, s);
    RRG_CUDA(cudaMemsetAsync(P->gbar.p, 0, P->gbar.bytes, s));
    interp_adjoint_kernel<R><<<bp, 256, 0, s>>>(n, static_cast<const V4<R>*>(xn1), P->gdev,
                                                static_cast<const V4<R>*>(P->acc4.p), A,
                                                static_cast<R*>(P->gbar.p), Xi);
    RRG_LAUNCHED();
    // Cb holds the cotangent of the current level (scale 1), Pb the previous one (scale 1)
    gradient_adjoint_kernel<R><<<bg, 256, 0, s>>>(P->grid.nx, static_cast<R>(-1.0 / P->grid.dx),
                                                  static_cast<const R*>(P->gbar.p),
                                                  static_cast<R*>(P->Cb.p));
    RRG_LAUNCHED();
    RRG_CUDA(cudaMemsetAsync(P->F.p, 0, P->F.bytes, s));
    R beta = R(1);
    for (int k = 0; k < P->substeps; ++k) {
        // FP32: the float4 stencil (x +- 1 by shuffles, z from a register pipeline)
        const bool x4 = sizeof(R) == 4 &&
                        launch_wave_adjoint_step(P->grid.nx, static_cast<const float*>(P->Cb.p),
                                                 static_cast<float*>(P->Pb.p),
                                                 static_cast<float*>(P->F.p), P->wc.K_MAIN,
                                                 P->wc.K_ACTUAL, static_cast<double>(beta),
                                                 P->wc.K_F, s);
        if (!x4) {
            wave_adjoint_kernel<R><<<bg, 256, 0, s>>>(
                P->grid.nx, static_cast<const R*>(P->Cb.p), static_cast<R*>(P->Pb.p),
                static_cast<R*>(P->F.p), static_cast<R>(P->wc.K_MAIN),
                static_cast<R>(P->wc.K_ACTUAL), beta, static_cast<R>(P->wc.K_F));
            RRG_LAUNCHED();
        }
        std::swap(P->Cb.p, P->Pb.p);  // the new current cotangent; old C becomes P / K_O
        beta = static_cast<R>(P->wc.K_OLD);
    }
    // leave Pb unscaled (Pb *= K_O) so the next step sees both cotangents with scale 1
    scale_kernel<R><<<bg, 256, 0, s>>>(nc, static_cast<R*>(P->Pb.p), static_cast<R>(P->wc.K_OLD));
    RRG_LAUNCHED();
    deposit_adjoint_kernel<R><<<bp, 256, 0, s>>>(n, static_cast<const V4<R>*>(xn1), P->gdev,
                                                 static_cast<const R*>(P->F.p),
                                                 static_cast<R>(4.0 * kPi / (P->grid.dx * P->grid.dx * P->grid.dx)),
                                                 Xd);
    RRG_LAUNCHED();
    predict_adjoint_kernel<R><<<bp, 256, 0, s>>>(n, X, Xi, Xd, U, V, A, dt);
    RRG_LAUNCHED();
}

#define PMA_ENTRY(P, ...)                                                                    \
    try {                                                                                    \
        RRG_REQUIRE((P) != nullptr, RRG_ERR_INVALID, "null pm adjoint");                     \
        RRG_CUDA(cudaSetDevice((P)->device));                                                \
        __VA_ARGS__;                                                                         \
        return RRG_OK;                                                                       \
    } catch (const Error& x_) {                                                              \
        if (P) (P)->err = x_.what();                                                         \
        set_thread_error(x_.what());                                                         \
        return x_.code;                                                                      \
    }

}  // namespace

extern "C" {

RRG_API rrg_status rrg_pm_adjoint_create(int device, int precision, int64_t n, double m_max,
                                         const rrg_grid_info* grid, const rrg_wave_params* wave,
                                         double total_mass_for_rho, double dt, int nsteps,
                                         int checkpoint_every, rrg_pm_adjoint** out) {
    rrg_pm_adjoint* P = nullptr;
    try {
        RRG_REQUIRE(out && grid && wave, RRG_ERR_INVALID, "rrg_pm_adjoint_create: NULL argument");
        RRG_REQUIRE(precision == RRG_PREC_FP32 || precision == RRG_PREC_FP64, RRG_ERR_INVALID,
                    "rrg_pm_adjoint_create: precision must be FP32 or FP64");
        RRG_REQUIRE(n >= 1 && nsteps >= 1 && dt > 0 && grid->nx >= 2 && grid->nx <= 1024,
                    RRG_ERR_INVALID, "rrg_pm_adjoint_create: bad sizes");
        RRG_CUDA(cudaSetDevice(device));
        P = new rrg_pm_adjoint();
        P->device = device;
        P->prec = precision;
        P->rsz = precision == RRG_PREC_FP64 ? 8 : 4;
        P->n = n;
        P->dt = dt;
        P->nsteps = nsteps;
        P->every = checkpoint_every <= 0 ? nsteps : std::min(checkpoint_every, nsteps);
        P->substeps = wave->iterations;
        P->grid = *grid;
        P->gdev.nx = grid->nx;
        P->gdev.dx = grid->dx;
        P->gdev.domain_min = grid->domain_min;
        P->gdev.inv_dx = 1.0 / grid->dx;
        P->gdev.sim_l = grid->sim_l;
        P->nc = static_cast<int64_t>(grid->nx) * grid->nx * grid->nx;
        const double L = grid->nx * grid->dx;
        P->rho_mean = total_mass_for_rho / (L * L * L);
        {
            int e = 0;
            std::frexp(m_max > 0 ? m_max : 1.0, &e);
            P->shift_s = 26 - e;
        }
        const double C = wave->wave_speed, DT = wave->dt, DX = grid->dx;
        const double Q = wave->diss_base * C * DT * 0.5, W = 1 + Q,
                     K = C * C * DT * DT / (DX * DX);
        P->wc.K_MAIN = K / W;
        P->wc.K_F = -C * C * DT * DT / W;
        P->wc.K_ACTUAL = 2 * (1 - 3 * K) / W;
        P->wc.K_OLD = (Q - 1) / W;
        P->wc.bc_type = RRG_BC_PERIODIC;
        P->wc.keep_layer = 0;
        P->wc.C = C;
        P->wc.DT = DT;
        P->wc.DX = DX;
        P->wc.domain_min = grid->domain_min;
        const size_t pb = pvb(P), gb = gvb(P);
        for (PBuf* b : {&P->x, &P->v, &P->a, &P->u, &P->X, &P->V, &P->A, &P->U, &P->Xi, &P->Xd})
            b->alloc(pb);
        P->mg.alloc(8 * P->nc);
        for (PBuf* b : {&P->src, &P->phi[0], &P->phi[1], &P->Cb, &P->Pb, &P->F}) b->alloc(gb);
        P->acc4.alloc(4 * gb);
        P->gbar.alloc(4 * gb);
        const int nck = (nsteps + P->every - 1) / P->every;
        P->ck_x.alloc(pb * nck);
        P->ck_v.alloc(pb * nck);
        P->ck_a.alloc(pb * nck);
        P->ck_phi.alloc(2 * gb * nck);
        P->seg_x.alloc(pb * P->every);
        P->seg_phi.alloc(gb * P->every);
        *out = P;
        return RRG_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        delete P;
        return e.code;
    }
}

RRG_API rrg_status rrg_pm_adjoint_destroy(rrg_pm_adjoint* P) {
    if (!P) return RRG_OK;
    cudaSetDevice(P->device);
    cudaDeviceSynchronize();
    delete P;
    return RRG_OK;
}

// Forward from x0[i] = (x, y, z, m), v0 (n x 4 of the precision) and the initial wave levels
// phi_prev0, phi_cur0 (nx^3): a_0 = T(x_0) g(phi_cur0), then nsteps PM steps. x_out / v_out /
// phi_out (may be NULL) receive the final positions, velocities and current level.
RRG_API rrg_status rrg_pm_adjoint_forward(rrg_pm_adjoint* P, const void* x0, const void* v0,
                                          const void* phi_prev0, const void* phi_cur0,
                                          void* x_out, void* v_out, void* phi_out,
                                          void* stream) {
    PMA_ENTRY(P, {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t pb = pvb(P), gb = gvb(P);
        RRG_CUDA(cudaMemcpyAsync(P->x.p, x0, pb, cudaMemcpyDeviceToDevice, s));
        RRG_CUDA(cudaMemcpyAsync(P->v.p, v0, pb, cudaMemcpyDeviceToDevice, s));
        RRG_CUDA(cudaMemcpyAsync(P->phi[0].p, phi_prev0, gb, cudaMemcpyDeviceToDevice, s));
        RRG_CUDA(cudaMemcpyAsync(P->phi[1].p, phi_cur0, gb, cudaMemcpyDeviceToDevice, s));
        launch_gradient(P->prec, P->grid.nx, P->grid.dx, P->phi[1].p, P->acc4.p, s);
        launch_interp(P->prec, P->n, P->x.p, nullptr, P->gdev, P->acc4.p, P->a.p, s);
        for (int k = 0; k < P->nsteps; ++k) {
            if (k % P->every == 0) {
                const int c = k / P->every;
                RRG_CUDA(cudaMemcpyAsync(P->ck_x.c() + pb * c, P->x.p, pb, cudaMemcpyDeviceToDevice, s));
                RRG_CUDA(cudaMemcpyAsync(P->ck_v.c() + pb * c, P->v.p, pb, cudaMemcpyDeviceToDevice, s));
                RRG_CUDA(cudaMemcpyAsync(P->ck_a.c() + pb * c, P->a.p, pb, cudaMemcpyDeviceToDevice, s));
                RRG_CUDA(cudaMemcpyAsync(P->ck_phi.c() + 2 * gb * c, P->phi[0].p, gb, cudaMemcpyDeviceToDevice, s));
                RRG_CUDA(cudaMemcpyAsync(P->ck_phi.c() + 2 * gb * c + gb, P->phi[1].p, gb, cudaMemcpyDeviceToDevice, s));
            }
            pm_step(P, s);
        }
        if (x_out) RRG_CUDA(cudaMemcpyAsync(x_out, P->x.p, pb, cudaMemcpyDeviceToDevice, s));
        if (v_out) RRG_CUDA(cudaMemcpyAsync(v_out, P->v.p, pb, cudaMemcpyDeviceToDevice, s));
        if (phi_out) RRG_CUDA(cudaMemcpyAsync(phi_out, P->phi[1].p, gb, cudaMemcpyDeviceToDevice, s));
        P->forward_done = true;
    })
}

// Backward: cotangents of the final x (n x 4, w ignored) and v in (NULL = zero); out gx[i] =
// (dL/dx, dL/dy, dL/dz, dL/dm) and gv[i] of the initial state. The initial potential is held
// fixed.
RRG_API rrg_status rrg_pm_adjoint_backward(rrg_pm_adjoint* P, const void* gx_final,
                                           const void* gv_final, void* gx_out, void* gv_out,
                                           void* stream) {
    PMA_ENTRY(P, {
        RRG_REQUIRE(P->forward_done, RRG_ERR_STATE, "rrg_pm_adjoint_backward before forward");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t pb = pvb(P), gb = gvb(P);
        if (gx_final) RRG_CUDA(cudaMemcpyAsync(P->X.p, gx_final, pb, cudaMemcpyDeviceToDevice, s));
        else RRG_CUDA(cudaMemsetAsync(P->X.p, 0, pb, s));
        if (gv_final) RRG_CUDA(cudaMemcpyAsync(P->V.p, gv_final, pb, cudaMemcpyDeviceToDevice, s));
        else RRG_CUDA(cudaMemsetAsync(P->V.p, 0, pb, s));
        RRG_CUDA(cudaMemset2DAsync(P->X.c() + 3 * P->rsz, 4 * P->rsz, 0, P->rsz, P->n, s));
        RRG_CUDA(cudaMemsetAsync(P->A.p, 0, pb, s));
        RRG_CUDA(cudaMemsetAsync(P->Cb.p, 0, gb, s));
        RRG_CUDA(cudaMemsetAsync(P->Pb.p, 0, gb, s));
        const int nseg = (P->nsteps + P->every - 1) / P->every;
        for (int seg = nseg - 1; seg >= 0; --seg) {
            const int n0 = seg * P->every, n1 = std::min(P->nsteps, n0 + P->every);
            RRG_CUDA(cudaMemcpyAsync(P->x.p, P->ck_x.c() + pb * seg, pb, cudaMemcpyDeviceToDevice, s));
            RRG_CUDA(cudaMemcpyAsync(P->v.p, P->ck_v.c() + pb * seg, pb, cudaMemcpyDeviceToDevice, s));
            RRG_CUDA(cudaMemcpyAsync(P->a.p, P->ck_a.c() + pb * seg, pb, cudaMemcpyDeviceToDevice, s));
            RRG_CUDA(cudaMemcpyAsync(P->phi[0].p, P->ck_phi.c() + 2 * gb * seg, gb, cudaMemcpyDeviceToDevice, s));
            RRG_CUDA(cudaMemcpyAsync(P->phi[1].p, P->ck_phi.c() + 2 * gb * seg + gb, gb, cudaMemcpyDeviceToDevice, s));
            for (int k = n0; k < n1; ++k) {
                pm_step(P, s);
                RRG_CUDA(cudaMemcpyAsync(P->seg_x.c() + pb * (k - n0), P->x.p, pb, cudaMemcpyDeviceToDevice, s));
                RRG_CUDA(cudaMemcpyAsync(P->seg_phi.c() + gb * (k - n0), P->phi[1].p, gb, cudaMemcpyDeviceToDevice, s));
            }
            for (int k = n1 - 1; k >= n0; --k) {
                const void* xk1 = P->seg_x.c() + pb * (k - n0);
                const void* pk1 = P->seg_phi.c() + gb * (k - n0);
                if (P->prec == RRG_PREC_FP64) backward_step<double>(P, xk1, pk1, s);
                else backward_step<float>(P, xk1, pk1, s);
            }
        }
        // a_0 = T(x_0) g(phi_cur0): its cotangent A reaches x_0 (the grid is held fixed)
        RRG_CUDA(cudaMemcpyAsync(P->x.p, P->ck_x.p, pb, cudaMemcpyDeviceToDevice, s));
        launch_gradient(P->prec, P->grid.nx, P->grid.dx, P->ck_phi.c() + gb, P->acc4.p, s);
        const int bp = div_up(P->n, 256);
        if (P->prec == RRG_PREC_FP64) {
            interp_adjoint_kernel<double><<<bp, 256, 0, s>>>(
                P->n, static_cast<const V4<double>*>(P->x.p), P->gdev,
                static_cast<const V4<double>*>(P->acc4.p), static_cast<const V4<double>*>(P->A.p),
                nullptr, static_cast<V4<double>*>(P->Xi.p));
            RRG_LAUNCHED();
            add_xyz_kernel<double><<<bp, 256, 0, s>>>(P->n, static_cast<V4<double>*>(P->X.p),
                                                     static_cast<const V4<double>*>(P->Xi.p));
        } else {
            interp_adjoint_kernel<float><<<bp, 256, 0, s>>>(
                P->n, static_cast<const V4<float>*>(P->x.p), P->gdev,
                static_cast<const V4<float>*>(P->acc4.p), static_cast<const V4<float>*>(P->A.p),
                nullptr, static_cast<V4<float>*>(P->Xi.p));
            RRG_LAUNCHED();
            add_xyz_kernel<float><<<bp, 256, 0, s>>>(P->n, static_cast<V4<float>*>(P->X.p),
                                                    static_cast<const V4<float>*>(P->Xi.p));
        }
        RRG_LAUNCHED();
        RRG_CUDA(cudaMemcpyAsync(gx_out, P->X.p, pb, cudaMemcpyDeviceToDevice, s));
        RRG_CUDA(cudaMemcpyAsync(gv_out, P->V.p, pb, cudaMemcpyDeviceToDevice, s));
    })
}

}  // extern "C"
