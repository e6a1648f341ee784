// Harness over the reference's own CUDA kernels and integration strategies — TEST
// INFRASTRUCTURE ONLY. Built by build_ref.sh together with the unmodified reference sources
// (solver/lib/**, solver/app/include/*.cuh) into oracle/_ref/librrgref.so, then used to
//   - make golden vectors from the reference itself (tests/golden/make_golden.py), and
//   - time the reference's step on the same GPU (bench.py).
// Every entry point drives the reference exactly as integrate() does
// (solver/app/src/rrgsim_integration.cu:19-146): initialize the contexts, pick the strategy,
// init -> precalc -> sync, then calc_step in a loop.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <co_grid_context.cuh>
#include <co_particles_context.cuh>
#include <nbody.cuh>
#include <rm_mesh2p.cuh>
#include <rm_p2mesh.cuh>
#include <wave.cuh>

#include "rrgsim_integration_nbody.cuh"
#include "rrgsim_integration_rect.cuh"

namespace {

thread_local std::string g_err;

rrgsim::common::ParticlesData make_particles(int64_t n, const double* pos, const double* vel,
                                             const double* mass, const double* soft2) {
    rrgsim::common::ParticlesData pd;
    pd.pos.resize(n);
    pd.vel.resize(n);
    pd.mass.assign(mass, mass + n);
    pd.soft2.assign(soft2, soft2 + n);
    for (int64_t i = 0; i < n; ++i) {
        pd.pos[i] = make_double3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        pd.vel[i] = make_double3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
    pd.info.ntotal = static_cast<int>(n);
    return pd;
}

// GridInfo exactly as from_json derives it (solver/lib/rrgsim_io/src/io_json.cpp:28-40)
rrgsim::common::GridInfo make_grid(int nx, double dx, double bc_frac) {
    rrgsim::common::GridInfo g;
    g.nx = nx;
    g.dx = dx;
    g.domain_l = g.dx * g.nx;
    g.sim_l = (1. - bc_frac) * g.domain_l;
    g.bc_l = 0.5 * bc_frac * g.domain_l;
    g.domain_max = 0.5 * g.domain_l;
    g.domain_min = -0.5 * g.domain_l;
    return g;
}

void copy3(const std::vector<double3>& v, double* out) {
    if (!out) return;
    for (size_t i = 0; i < v.size(); ++i) {
        out[3 * i] = v[i].x;
        out[3 * i + 1] = v[i].y;
        out[3 * i + 2] = v[i].z;
    }
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// NBodyIntegrationSolver: precalc (grav + acc), then nsteps calc_step.
// Outputs after precalc: acc0, grav0; after the steps: pos, vel, acc. ms_per_step from CUDA
// events around the step loop (default stream, as the reference runs).
int ref_nbody(int64_t n, const double* pos, const double* vel, const double* mass,
              const double* soft2, double dt, int nsteps, double* acc0, double* grav0,
              double* pos_out, double* vel_out, double* acc_out, double* ms_per_step) {
    try {
        auto pd = make_particles(n, pos, vel, mass, soft2);
        auto ctx_ = rrgsim::common::initialize_particles_context_(pd);
        rrgsim::integration::IntegrationParams params;
        params.sim_params.dt_dynamics = dt;
        std::shared_ptr<rrgsim::integration::IntegrationSolver> solver =
            std::make_shared<rrgsim::integration::NBodyIntegrationSolver>();
        solver->init(params, ctx_, nullptr);
        solver->precalc();
        copy3(ctx_->acc_.to_vector(), acc0);
        if (grav0) {
            auto g = ctx_->grav_.to_vector();
            std::memcpy(grav0, g.data(), sizeof(double) * n);
        }
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaDeviceSynchronize();
        cudaEventRecord(e0, 0);
        for (int s = 0; s < nsteps; ++s) solver->calc_step();
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms_per_step) *ms_per_step = nsteps ? ms / nsteps : 0.0;
        copy3(ctx_->pos_.to_vector(), pos_out);
        copy3(ctx_->vel_.to_vector(), vel_out);
        copy3(ctx_->acc_.to_vector(), acc_out);
        RR::CUDA::check(cudaGetLastError(), "ref_nbody");
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// RectWaveIntegrationSolver: precalc (CIC, periodic boundary with M = 1, setup relaxation,
// gradient), sync (NGP potential + trilinear acceleration), then nsteps calc_step.
// wave[] = {diss_base, diss_extra, wave_speed, setup_iterations, iterations, tolerance,
//           print_step, steady_check_step, steady_hold_steps}.
// Outputs after precalc+sync: mass0 (nx^3), phi0 (nx^3), acc0 (n x 3), grav0 (n);
// after the steps: pos, vel, acc, and phi (nx^3).
int ref_pm(int64_t n, const double* pos, const double* vel, const double* mass,
           const double* soft2, int nx, double dx, double bc_frac, const double* wave, double dt,
           int nsteps, double* mass0, double* phi0, double* acc0, double* grav0,
           double* pos_out, double* vel_out, double* acc_out, double* phi_out,
           double* ms_per_step) {
    try {
        auto pd = make_particles(n, pos, vel, mass, soft2);
        auto pctx = rrgsim::common::initialize_particles_context_(pd);
        auto grid = make_grid(nx, dx, bc_frac);
        auto gctx = rrgsim::common::initialize_grid_context_(grid);
        rrgsim::common::WaveParams wp{};
        wp.diss_base = wave[0];
        wp.diss_extra = wave[1];
        wp.wave_speed = wave[2];
        wp.setup_iterations = static_cast<int>(wave[3]);
        wp.iterations = static_cast<int>(wave[4]);
        wp.tolerance = wave[5];
        wp.print_step = static_cast<int>(wave[6]);
        wp.steady_check_step = static_cast<int>(wave[7]);
        wp.steady_hold_steps = static_cast<int>(wave[8]);
        wp.dt = 0.5 * dx / (wp.wave_speed * std::sqrt(3.0));  // io_json.cpp:178
        rrgsim::integration::IntegrationParams params;
        params.sim_params.dt_dynamics = dt;
        params.sim_params.use_wave_model = true;
        params.mb_grid_info = grid;
        params.mb_wave_params = wp;
        std::shared_ptr<rrgsim::integration::IntegrationSolver> solver =
            std::make_shared<rrgsim::integration::RectWaveIntegrationSolver>();
        solver->init(params, pctx, gctx);
        solver->precalc();
        solver->sync_particles_and_grid();
        const size_t nc = static_cast<size_t>(nx) * nx * nx;
        if (mass0) {
            auto m = gctx->mass_.to_vector();
            std::memcpy(mass0, m.data(), sizeof(double) * nc);
        }
        if (phi0) {
            auto p = gctx->grav_curr_.to_vector();
            std::memcpy(phi0, p.data(), sizeof(double) * nc);
        }
        copy3(pctx->acc_.to_vector(), acc0);
        if (grav0) {
            auto g = pctx->grav_.to_vector();
            std::memcpy(grav0, g.data(), sizeof(double) * n);
        }
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaDeviceSynchronize();
        cudaEventRecord(e0, 0);
        for (int s = 0; s < nsteps; ++s) solver->calc_step();
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms_per_step) *ms_per_step = nsteps ? ms / nsteps : 0.0;
        copy3(pctx->pos_.to_vector(), pos_out);
        copy3(pctx->vel_.to_vector(), vel_out);
        copy3(pctx->acc_.to_vector(), acc_out);
        if (phi_out) {
            auto p = gctx->grav_curr_.to_vector();
            std::memcpy(phi_out, p.data(), sizeof(double) * nc);
        }
        RR::CUDA::check(cudaGetLastError(), "ref_pm");
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// NBodyIntegrationSolver with a grid (rrgsim_integration_nbody.cuh:32-48): precalc, nsteps
// calc_step, then sync_particles_and_grid: CIC mass, the particle potential (recomputed), and
// the NGP cell averages of the particle potential and acceleration. Outputs: the grid's mass,
// potential (nx^3) and acceleration (nx^3 x 3); the particles' pos, vel, acc (n x 3) and
// potential (n).
int ref_nbody_grid(int64_t n, const double* pos, const double* vel, const double* mass,
                   const double* soft2, double dt, int nsteps, int nx, double dx,
                   double bc_frac, double* grid_mass, double* grid_grav, double* grid_acc,
                   double* pos_out, double* vel_out, double* acc_out, double* grav_out) {
    try {
        auto pd = make_particles(n, pos, vel, mass, soft2);
        auto pctx = rrgsim::common::initialize_particles_context_(pd);
        auto grid = make_grid(nx, dx, bc_frac);
        auto gctx = rrgsim::common::initialize_grid_context_(grid);
        rrgsim::integration::IntegrationParams params;
        params.sim_params.dt_dynamics = dt;
        params.sim_params.use_wave_model = false;
        params.mb_grid_info = grid;
        std::shared_ptr<rrgsim::integration::IntegrationSolver> solver =
            std::make_shared<rrgsim::integration::NBodyIntegrationSolver>();
        solver->init(params, pctx, gctx);
        solver->precalc();
        for (int s = 0; s < nsteps; ++s) solver->calc_step();
        solver->sync_particles_and_grid();
        const size_t nc = static_cast<size_t>(nx) * nx * nx;
        if (grid_mass) {
            auto m = gctx->mass_.to_vector();
            std::memcpy(grid_mass, m.data(), sizeof(double) * nc);
        }
        if (grid_grav) {
            auto g = gctx->grav_curr_.to_vector();
            std::memcpy(grid_grav, g.data(), sizeof(double) * nc);
        }
        copy3(gctx->acc_.to_vector(), grid_acc);
        copy3(pctx->pos_.to_vector(), pos_out);
        copy3(pctx->vel_.to_vector(), vel_out);
        copy3(pctx->acc_.to_vector(), acc_out);
        if (grav_out) {
            auto g = pctx->grav_.to_vector();
            std::memcpy(grav_out, g.data(), sizeof(double) * n);
        }
        RR::CUDA::check(cudaGetLastError(), "ref_nbody_grid");
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// The reference's wave solver under a non-periodic or layered boundary (wave.cu:18-104, set up
// by set_boundary_monopole / set_boundary_periodic, :196-228), which its precalc leaves
// commented out (rrgsim_integration_rect.cuh:57-64): CIC of the particles, the boundary
// (bc = 0: periodic keeping the absorbing layer, 1: monopole Dirichlet, 2: monopole radiative,
// with total_mass and com), both potential levels set to phi_init, then `iterations` substeps
// with no steady check. wave[] as for ref_pm. Outputs: mass (nx^3) and the final potential.
int ref_wave_bc(int64_t n, const double* pos, const double* vel, const double* mass,
                const double* soft2, int nx, double dx, double bc_frac, const double* wave,
                int bc, double total_mass, const double* com, const double* phi_init,
                int iterations, double* mass_out, double* phi_out) {
    try {
        auto pd = make_particles(n, pos, vel, mass, soft2);
        auto pctx = rrgsim::common::initialize_particles_context_(pd);
        auto grid = make_grid(nx, dx, bc_frac);
        auto gctx = rrgsim::common::initialize_grid_context_(grid);
        rrgsim::common::WaveParams wp{};
        wp.diss_base = wave[0];
        wp.diss_extra = wave[1];
        wp.wave_speed = wave[2];
        wp.setup_iterations = static_cast<int>(wave[3]);
        wp.iterations = static_cast<int>(wave[4]);
        wp.tolerance = wave[5];
        wp.print_step = static_cast<int>(wave[6]);
        wp.steady_check_step = static_cast<int>(wave[7]);
        wp.steady_hold_steps = static_cast<int>(wave[8]);
        wp.dt = 0.5 * dx / (wp.wave_speed * std::sqrt(3.0));  // io_json.cpp:178
        // grid_info_ came with the grid context; the wave parameters as the strategy's init
        // uploads them (rrgsim_integration_rect.cuh:35-40)
        RR::CUDA::CuCopyToSymbol(wp, rrgsim::common::wave_params_, RR::CUDA::ToDevice);
        rrgsim::rect_mesh::convert_particles_to_grid(pctx, gctx);
        if (bc == 0)
            rrgsim::wave::set_boundary_periodic(total_mass, grid, true);
        else
            rrgsim::wave::set_boundary_monopole(total_mass, make_double3(com[0], com[1], com[2]),
                                                bc == 2, dx);
        const size_t nc = static_cast<size_t>(nx) * nx * nx;
        std::vector<double> phi(phi_init, phi_init + nc);
        gctx->grav_prev_ = phi;
        gctx->grav_curr_ = phi;
        rrgsim::wave::solve_wave_equation(gctx, wp, iterations);
        if (mass_out) {
            auto m = gctx->mass_.to_vector();
            std::memcpy(mass_out, m.data(), sizeof(double) * nc);
        }
        if (phi_out) {
            auto p = gctx->grav_curr_.to_vector();
            std::memcpy(phi_out, p.data(), sizeof(double) * nc);
        }
        RR::CUDA::check(cudaGetLastError(), "ref_wave_bc");
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

}  // extern "C"
