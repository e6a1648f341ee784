"""The particle-mesh adjoint (csrc/pm_adjoint.cu) against torch autograd through a plain
FP64 torch restatement of the same step (CIC deposit, periodic damped-wave substeps,
one-sided-face gradient, trilinear interpolation, leapfrog)."""
import math

import numpy as np
import pytest

import rrgsim_b200 as rg
from helpers import disk

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rrgsim_b200.adjoint import PMEngine, pm_leapfrog  # noqa: E402

PI = 3.14159265358979


def torch_pm(x, v, m, phi_p, phi_c, g, coef, dt, steps, substeps):
    nx, dx, dmin = g.nx, g.dx, g.domain_min
    km, ka, ko, kf, rho_mean = coef

    def corners(i0, i1, j0, j1, k0, k1):
        out = []
        for kk in (k0, k1):
            for jj in (j0, j1):
                for ii in (i0, i1):
                    out.append(ii + jj * nx + kk * nx * nx)
        return out

    def cic(x):  # rm_p2mesh.cu:184-235
        u = torch.clamp((x - dmin) / dx - 0.5, 0.0, (nx - 1) - 1e-6)
        i0 = torch.floor(u).detach().long()
        f = u - i0
        i1 = torch.clamp(i0 + 1, max=nx - 1)
        w = [1 - f, f]
        M = torch.zeros(nx ** 3, dtype=x.dtype, device=x.device)
        idx = corners(i0[:, 0], i1[:, 0], i0[:, 1], i1[:, 1], i0[:, 2], i1[:, 2])
        c = 0
        for kz in range(2):
            for jy in range(2):
                for ix in range(2):
                    M = M.index_add(0, idx[c], m * w[ix][:, 0] * w[jy][:, 1] * w[kz][:, 2])
                    c += 1
        return M

    def substep(pp, pc, f):  # wave.cu:183-192, periodic
        a = pc.view(nx, nx, nx)
        lap = sum(torch.roll(a, s, d) for d in range(3) for s in (1, -1)).reshape(-1)
        return km * lap + ka * pc + ko * pp + kf * f

    def grad(phi):  # rm_p2mesh.cu:254-287
        a = phi.view(nx, nx, nx)  # [z, y, x]
        outs = []
        for d in (2, 1, 0):
            n = a.shape[d]
            sl = lambda s, e: [slice(None)] * d + [slice(s, e)]  # noqa: E731
            first = a[tuple(sl(1, 2))] - a[tuple(sl(0, 1))]
            mid = 0.5 * (a[tuple(sl(2, n))] - a[tuple(sl(0, n - 2))])
            last = a[tuple(sl(n - 1, n))] - a[tuple(sl(n - 2, n - 1))]
            outs.append(-(torch.cat([first, mid, last], d) / dx).reshape(-1))
        return torch.stack(outs, 1)

    def interp(x, gr):  # rm_mesh2p.cu:64-111
        f = (x - dmin) / dx - 0.5
        a = torch.floor(f.detach().float()).double().long()
        w = f - a
        i0 = torch.clamp(a, 0, nx - 1)
        i1 = torch.clamp(a + 1, 0, nx - 1)
        ws = [1 - w, w]
        idx = corners(i0[:, 0], i1[:, 0], i0[:, 1], i1[:, 1], i0[:, 2], i1[:, 2])
        out = 0
        c = 0
        for kz in range(2):
            for jy in range(2):
                for ix in range(2):
                    W = ws[ix][:, 0] * ws[jy][:, 1] * ws[kz][:, 2]
                    out = out + W[:, None] * gr[idx[c]]
                    c += 1
        return out

    a = interp(x, grad(phi_c.detach()))
    pp, pc = phi_p.detach(), phi_c.detach()
    for _ in range(steps):
        u = v + (v + dt * a)
        x = x + dt * 0.5 * u
        f = 4 * PI * (cic(x) / dx ** 3 - rho_mean)
        for _ in range(substeps):
            pp, pc = pc, substep(pp, pc, f)
        a = interp(x, grad(pc))
        v = 0.5 * (u + dt * a)
    return x, v


def _case(nx=16, n=512, substeps=5):
    pos, vel, m, s2 = disk(n, seed=31)
    grid = rg.GridInfo.from_values(nx, 16.0 / nx, 0.0)
    c = 10.0 * float(np.max(np.linalg.norm(vel, axis=1)))
    wave = rg.WaveParams.make(grid.dx, diss_base=1.0 / (4 * grid.dx), wave_speed=c,
                              iterations=substeps, setup_iterations=200, steady_check_step=10 ** 6)
    sim = rg.SimParams(time_max=1.0, dt_save=1.0, dt_dynamics=2e-3, saves_without_dump=0,
                       use_wave_model=1)
    with rg.Context(0, "fp64") as ctx:  # a relaxed potential to start from
        ctx.load_particles(pos, vel, m, s2)
        ctx.init_grid(grid)
        ctx.set_wave_params(wave)
        ctx.solver_init(sim)
        ctx.precalc()
        phi = ctx.get_grid()["grav"]
    DT, DX, C = wave.dt, grid.dx, wave.wave_speed
    Q = wave.diss_base * C * DT * 0.5
    W = 1 + Q
    K = C * C * DT * DT / (DX * DX)
    coef = (K / W, 2 * (1 - 3 * K) / W, (Q - 1) / W, -C * C * DT * DT / W,
            1.0 / (nx * DX) ** 3)
    return pos, vel, m, grid, wave, phi, coef


@pytest.mark.parametrize("every", [1, 3])
def test_pm_adjoint_matches_autograd_fp64(every):
    pos, vel, m, grid, wave, phi, coef = _case()
    steps, dt = 6, 2e-3
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
    x0, v0, mm, ph = t(pos), t(vel), t(m), t(phi)
    target = x0 + 1e-3 * torch.randn_like(x0)
    eng = PMEngine(len(m), float(m.max()), grid, wave, dt, steps, "fp64", every)
    grads = []
    for ours in (True, False):
        xr, vr, mr = (a.clone().requires_grad_(True) for a in (x0, v0, mm))
        if ours:
            xN, vN = pm_leapfrog(xr, vr, mr, ph, ph, eng)
        else:
            xN, vN = torch_pm(xr, vr, mr, ph, ph, grid, coef, dt, steps, wave.iterations)
        loss = ((xN - target) ** 2).sum(1).mean() + 0.2 * (vN ** 2).sum(1).mean()
        loss.backward()
        grads.append((xN.detach(), xr.grad, vr.grad, mr.grad))
    # forward states agree (the library deposits in int64 fixed point: 2^-27 per contribution)
    assert torch.max(torch.abs(grads[0][0] - grads[1][0])) <= 1e-10
    for a, b in zip(grads[0][1:], grads[1][1:]):
        rel = float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
        assert rel <= 1e-6, rel


def test_pm_adjoint_fp32_close_to_fp64():
    pos, vel, m, grid, wave, phi, _ = _case(nx=32, n=4096, substeps=10)
    steps, dt = 8, 2e-3
    out = []
    for prec, dtype in (("fp32", torch.float32), ("fp64", torch.float64)):
        t = lambda a: torch.tensor(a, dtype=dtype, device="cuda")  # noqa: E731
        x0, v0, mm, ph = t(pos), t(vel), t(m), t(phi)
        eng = PMEngine(len(m), float(m.max()), grid, wave, dt, steps, prec, 4)
        xr, vr, mr = (a.clone().requires_grad_(True) for a in (x0, v0, mm))
        xN, vN = pm_leapfrog(xr, vr, mr, ph, ph, eng)
        loss = ((xN - (x0 + 1e-3)) ** 2).sum(1).mean()
        loss.backward()
        out.append(torch.cat([xr.grad.ravel(), vr.grad.ravel(), mr.grad.ravel()]).double())
    rel = float(torch.linalg.norm(out[0] - out[1]) / torch.linalg.norm(out[1]))
    assert rel <= 2e-3, rel
