"""Differentiable direct N-body: a torch.autograd.Function over the hand-written adjoint.

    xN, vN = nbody_leapfrog(x0, v0, m, soft2, dt, nsteps, checkpoint_every=20)

runs the reference's leapfrog (predict / direct-sum acceleration / correct, nbody.cu:19-181)
nsteps times on the GPU. Its backward is the adjoint kernels of csrc/adjoint.cu: one
vector-Jacobian product of the direct-sum force per step, states recomputed from checkpoints
kept every `checkpoint_every` steps. Gradients flow to x0, v0 and the masses m. FP32 tensors
run the FP32 kernels, FP64 tensors the FP64 ones.
"""
from __future__ import annotations

import ctypes as C
import json
import time

import numpy as np
import torch

from . import PREC, RRGError, check, generate_plummer, lib

_d = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731


def _sig():
    L = lib()
    vp, i64 = C.c_void_p, C.c_int64
    L.rrg_adjoint_create.argtypes = [C.c_int, C.c_int, i64, C.c_double, C.c_int, C.c_int,
                                     C.POINTER(C.c_double), C.POINTER(vp)]
    L.rrg_adjoint_destroy.argtypes = [vp]
    L.rrg_adjoint_forward.argtypes = [vp, vp, vp, vp, vp, vp]
    L.rrg_adjoint_backward.argtypes = [vp, vp, vp, vp, vp, vp]
    L.rrg_adjoint_set_mass_gradient.argtypes = [vp, C.c_int]
    L.rrg_dev_direct_vjp.argtypes = [vp, vp, C.c_double, i64, vp, vp, C.c_int, vp]
    for f in ("rrg_adjoint_create", "rrg_adjoint_destroy", "rrg_adjoint_forward",
              "rrg_adjoint_backward", "rrg_adjoint_set_mass_gradient", "rrg_dev_direct_vjp"):
        getattr(L, f).restype = C.c_int
    return L


class LeapfrogEngine:
    """One rrg_adjoint object: fixed n, dt, step count, checkpoint spacing and softening."""

    def __init__(self, n: int, dt: float, nsteps: int, soft2, precision: str = "fp32",
                 checkpoint_every: int = 20, device: int = 0):
        self.L = _sig()
        s2 = np.ascontiguousarray(np.broadcast_to(np.asarray(soft2, dtype=np.float64), (n,)))
        self.h = C.c_void_p()
        self.n, self.precision = n, precision
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        check(self.L.rrg_adjoint_create(device, PREC[precision], n, float(dt), int(nsteps),
                                        int(checkpoint_every), _d(s2), C.byref(self.h)))

    def _stream(self):
        return torch.cuda.current_stream().cuda_stream

    def forward(self, x4, v4, x_out=None, v_out=None):
        check(self.L.rrg_adjoint_forward(self.h, x4.data_ptr(), v4.data_ptr(),
                                         x_out.data_ptr() if x_out is not None else None,
                                         v_out.data_ptr() if v_out is not None else None,
                                         self._stream()))

    def backward(self, gx4, gv4, gx_out, gv_out, mass_grad: bool = True):
        check(self.L.rrg_adjoint_set_mass_gradient(self.h, 1 if mass_grad else 0))
        check(self.L.rrg_adjoint_backward(self.h, gx4.data_ptr() if gx4 is not None else None,
                                          gv4.data_ptr() if gv4 is not None else None,
                                          gx_out.data_ptr(), gv_out.data_ptr(),
                                          self._stream()))

    def close(self):
        if self.h:
            self.L.rrg_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _pad4(a, w=None):
    col = torch.zeros((a.shape[0], 1), dtype=a.dtype, device=a.device) if w is None else w[:, None]
    return torch.cat([a, col], 1).contiguous()


class NBodyLeapfrog(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, m, engine: LeapfrogEngine):
        if x0.dtype != engine.dtype or not x0.is_cuda:
            raise RRGError(1, f"nbody_leapfrog: expected CUDA {engine.dtype} tensors")
        x4 = _pad4(x0.detach(), m.detach())
        v4 = _pad4(v0.detach())
        xo, vo = torch.empty_like(x4), torch.empty_like(v4)
        engine.forward(x4, v4, xo, vo)
        ctx.engine = engine
        return xo[:, :3].contiguous(), vo[:, :3].contiguous()

    @staticmethod
    def backward(ctx, gx, gv):
        e = ctx.engine
        gx4 = _pad4(gx.contiguous()) if gx is not None else None
        gv4 = _pad4(gv.contiguous()) if gv is not None else None
        out_x = torch.empty((e.n, 4), dtype=e.dtype, device="cuda")
        out_v = torch.empty((e.n, 4), dtype=e.dtype, device="cuda")
        want_m = ctx.needs_input_grad[2]
        e.backward(gx4, gv4, out_x, out_v, mass_grad=want_m)
        return out_x[:, :3], out_v[:, :3], (out_x[:, 3] if want_m else None), None


def nbody_leapfrog(x0, v0, m, soft2, dt, nsteps, checkpoint_every=20, engine=None):
    """Final (positions, velocities) after nsteps leapfrog steps, differentiable in x0, v0, m."""
    if engine is None:
        engine = LeapfrogEngine(x0.shape[0], dt, nsteps, soft2,
                                "fp64" if x0.dtype == torch.float64 else "fp32",
                                checkpoint_every, x0.device.index or 0)
    return NBodyLeapfrog.apply(x0, v0, m, engine)


class PMEngine:
    """One rrg_pm_adjoint object: differentiable particle-mesh steps on a periodic grid."""

    def __init__(self, n: int, m_max: float, grid, wave, dt: float, nsteps: int,
                 precision: str = "fp32", checkpoint_every: int = 20,
                 total_mass_for_rho: float = 1.0, device: int = 0):
        from . import GridInfo, WaveParams  # noqa: F401  (structure types)
        self.L = lib()
        vp, i64 = C.c_void_p, C.c_int64
        L = self.L
        L.rrg_pm_adjoint_create.argtypes = [C.c_int, C.c_int, i64, C.c_double,
                                            C.POINTER(type(grid)), C.POINTER(type(wave)),
                                            C.c_double, C.c_double, C.c_int, C.c_int,
                                            C.POINTER(vp)]
        L.rrg_pm_adjoint_forward.argtypes = [vp] * 9
        L.rrg_pm_adjoint_backward.argtypes = [vp] * 6
        L.rrg_pm_adjoint_destroy.argtypes = [vp]
        for f in ("rrg_pm_adjoint_create", "rrg_pm_adjoint_forward", "rrg_pm_adjoint_backward",
                  "rrg_pm_adjoint_destroy"):
            getattr(L, f).restype = C.c_int
        self.n, self.nc = n, grid.nx ** 3
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.h = C.c_void_p()
        check(L.rrg_pm_adjoint_create(device, PREC[precision], n, float(m_max), C.byref(grid),
                                      C.byref(wave), float(total_mass_for_rho), float(dt),
                                      int(nsteps), int(checkpoint_every), C.byref(self.h)))

    def forward(self, x4, v4, phi_prev, phi_cur, x_out, v_out, phi_out=None):
        s = torch.cuda.current_stream().cuda_stream
        check(self.L.rrg_pm_adjoint_forward(self.h, x4.data_ptr(), v4.data_ptr(),
                                            phi_prev.data_ptr(), phi_cur.data_ptr(),
                                            x_out.data_ptr(), v_out.data_ptr(),
                                            phi_out.data_ptr() if phi_out is not None else None,
                                            s))

    def backward(self, gx4, gv4, gx_out, gv_out):
        s = torch.cuda.current_stream().cuda_stream
        check(self.L.rrg_pm_adjoint_backward(self.h, gx4.data_ptr() if gx4 is not None else None,
                                             gv4.data_ptr() if gv4 is not None else None,
                                             gx_out.data_ptr(), gv_out.data_ptr(), s))

    def close(self):
        if self.h:
            self.L.rrg_pm_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PMLeapfrog(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, m, phi_prev, phi_cur, engine: PMEngine):
        x4 = _pad4(x0.detach(), m.detach())
        v4 = _pad4(v0.detach())
        xo, vo = torch.empty_like(x4), torch.empty_like(v4)
        engine.forward(x4, v4, phi_prev.contiguous(), phi_cur.contiguous(), xo, vo)
        ctx.engine = engine
        return xo[:, :3].contiguous(), vo[:, :3].contiguous()

    @staticmethod
    def backward(ctx, gx, gv):
        e = ctx.engine
        gx4 = _pad4(gx.contiguous()) if gx is not None else None
        gv4 = _pad4(gv.contiguous()) if gv is not None else None
        out_x = torch.empty((e.n, 4), dtype=e.dtype, device="cuda")
        out_v = torch.empty((e.n, 4), dtype=e.dtype, device="cuda")
        e.backward(gx4, gv4, out_x, out_v)
        return out_x[:, :3], out_v[:, :3], out_x[:, 3], None, None, None


def pm_leapfrog(x0, v0, m, phi_prev, phi_cur, engine: PMEngine):
    """Final (positions, velocities) after the engine's PM steps from the given wave levels;
    differentiable in x0, v0 and m (the initial potential is held fixed)."""
    return PMLeapfrog.apply(x0, v0, m, phi_prev, phi_cur, engine)


def direct_vjp(posm, lam, soft2_uniform: float):
    """(d<lam, a>/dx, d<lam, a>/dm) for the direct-sum acceleration; posm, lam n x 4."""
    L = _sig()
    out = torch.empty_like(posm)
    prec = PREC["fp64"] if posm.dtype == torch.float64 else PREC["fp32"]
    check(L.rrg_dev_direct_vjp(posm.data_ptr(), None, 0.5 * soft2_uniform, posm.shape[0],
                               lam.data_ptr(), out.data_ptr(), prec,
                               torch.cuda.current_stream().cuda_stream))
    return out


def bench_form(torch_mod=None, n=16384, nsteps=200, dt=1e-3, eps=0.02, every=20, fd_dirs=64):
    """Adjoint through 200 leapfrog steps of a Plummer sphere (N = 16,384, eps = 0.02): the
    loss is the mean squared distance of the final positions from targets that the forward
    model produces from initial conditions perturbed by sigma = 1e-3. Gradient w.r.t. initial
    positions, velocities and masses; wall-time ratio of the backward (recompute included) to
    the forward; central finite differences (h = 1e-4, FP64) on random directions."""
    pos, vel = generate_plummer(11, n, 1.0, 1.0, 20.0)
    m = np.full(n, 1.0 / n)
    rng = np.random.default_rng(12)
    dev = "cuda"
    res = {"form": "adjoint_nbody_16384", "n": n, "steps": nsteps, "checkpoint_every": every}
    # one target perturbation for both precisions, so their gradients are of the same loss
    pert = 1e-3 * rng.standard_normal((n, 3))
    grads = {}
    for prec, dt_ in (("fp32", torch.float32), ("fp64", torch.float64)):
        eng = LeapfrogEngine(n, dt, nsteps, eps * eps, prec, every)
        x0 = torch.tensor(pos, dtype=dt_, device=dev)
        v0 = torch.tensor(vel, dtype=dt_, device=dev)
        mm = torch.tensor(m, dtype=dt_, device=dev)
        with torch.no_grad():
            xt, _ = nbody_leapfrog(x0 + torch.tensor(pert, dtype=dt_, device=dev), v0, mm,
                                   eps * eps, dt, nsteps, engine=eng)
        x0r, v0r, mr = (t.clone().requires_grad_(True) for t in (x0, v0, mm))
        # warm-up pass, then timed forward and backward
        xN, _ = nbody_leapfrog(x0r, v0r, mr, eps * eps, dt, nsteps, engine=eng)
        loss = ((xN - xt) ** 2).sum(1).mean()
        loss.backward()
        torch.cuda.synchronize()
        for t in (x0r, v0r, mr):
            t.grad = None
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record()
        xN, _ = nbody_leapfrog(x0r, v0r, mr, eps * eps, dt, nsteps, engine=eng)
        loss = ((xN - xt) ** 2).sum(1).mean()
        b.record()
        loss.backward()
        c.record()
        torch.cuda.synchronize()
        fwd, bwd = a.elapsed_time(b), b.elapsed_time(c)
        grads[prec] = (x0r.grad.double().cpu().numpy(), v0r.grad.double().cpu().numpy(),
                       mr.grad.double().cpu().numpy())
        res[prec] = {"forward_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
                     "loss": float(loss.detach())}
        if prec == "fp64" and fd_dirs > 0:
            # central differences along random directions in (x0, v0, m), FP64 forward model
            fd_rel = []
            gvec = np.concatenate([g.ravel() for g in grads["fp64"]])
            g32 = np.concatenate([g.ravel() for g in grads["fp32"]])
            rel32 = []
            h = 1e-4
            with torch.no_grad():
                for k in range(fd_dirs):
                    d = rng.standard_normal(gvec.size)
                    d /= np.linalg.norm(d)
                    dx = torch.tensor(d[:3 * n].reshape(n, 3), dtype=dt_, device=dev)
                    dv = torch.tensor(d[3 * n:6 * n].reshape(n, 3), dtype=dt_, device=dev)
                    dm = torch.tensor(d[6 * n:], dtype=dt_, device=dev)
                    lp = ((nbody_leapfrog(x0 + h * dx, v0 + h * dv, mm + h * dm, eps * eps, dt,
                                          nsteps, engine=eng)[0] - xt) ** 2).sum(1).mean()
                    lm = ((nbody_leapfrog(x0 - h * dx, v0 - h * dv, mm - h * dm, eps * eps, dt,
                                          nsteps, engine=eng)[0] - xt) ** 2).sum(1).mean()
                    fd = float(lp - lm) / (2 * h)
                    fd_rel.append(abs(gvec @ d - fd) / max(abs(fd), 1e-300))
                    rel32.append(abs(g32 @ d - fd) / max(abs(fd), 1e-300))
            res["fd_check"] = {"directions": fd_dirs, "h": h,
                               "fp64_adjoint_rel_err_median": float(np.median(fd_rel)),
                               "fp64_adjoint_rel_err_max": float(np.max(fd_rel)),
                               "fp32_adjoint_rel_err_median": float(np.median(rel32)),
                               "fp32_adjoint_rel_err_max": float(np.max(rel32))}
        eng.close()
    g64 = np.concatenate([g.ravel() for g in grads["fp64"]])
    g32 = np.concatenate([g.ravel() for g in grads["fp32"]])
    res["fp32_vs_fp64_gradient_rel_l2"] = float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))
    # per particle: |g32 - g64| / |g64| of the position gradient
    p32, p64 = grads["fp32"][0], grads["fp64"][0]
    per = np.linalg.norm(p32 - p64, axis=1) / np.maximum(np.linalg.norm(p64, axis=1), 1e-300)
    res["fp32_vs_fp64_position_gradient_per_particle"] = {
        "median": float(np.median(per)), "p90": float(np.percentile(per, 90)),
        "p99": float(np.percentile(per, 99))}
    res["adjoint_over_forward_fp32"] = res["fp32"]["backward_over_forward"]
    # the same FP32 gradient keeping every step's state in HBM (no recompute)
    eng = LeapfrogEngine(n, dt, nsteps, eps * eps, "fp32", 1)
    x0r, v0r, mr = (torch.tensor(a, dtype=torch.float32, device=dev).requires_grad_(True)
                    for a in (pos, vel, m))
    for rep in range(2):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record()
        xN, _ = nbody_leapfrog(x0r, v0r, mr, eps * eps, dt, nsteps, engine=eng)
        loss = (xN ** 2).sum(1).mean()
        b.record()
        loss.backward()
        c.record()
        torch.cuda.synchronize()
    res["fp32_every_step_in_hbm"] = {"forward_ms": a.elapsed_time(b),
                                     "backward_ms": b.elapsed_time(c),
                                     "backward_over_forward": b.elapsed_time(c) / a.elapsed_time(b)}
    eng.close()
    # checkpoints every 20 steps, gradient w.r.t. positions and velocities only (fixed masses:
    # the VJP skips dL/dm)
    eng = LeapfrogEngine(n, dt, nsteps, eps * eps, "fp32", every)
    x0r, v0r = (torch.tensor(a, dtype=torch.float32, device=dev).requires_grad_(True)
                for a in (pos, vel))
    mm = torch.tensor(m, dtype=torch.float32, device=dev)
    for rep in range(2):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record()
        xN, _ = nbody_leapfrog(x0r, v0r, mm, eps * eps, dt, nsteps, engine=eng)
        loss = (xN ** 2).sum(1).mean()
        b.record()
        loss.backward()
        c.record()
        torch.cuda.synchronize()
    res["fp32_positions_velocities_only"] = {
        "forward_ms": a.elapsed_time(b), "backward_ms": b.elapsed_time(c),
        "backward_over_forward": b.elapsed_time(c) / a.elapsed_time(b)}
    eng.close()
    return res


def bench_form_vjp(torch_mod=None, sizes=(16384, 65536), reps=20):
    """One force VJP (rrg_dev_direct_vjp, masses spread so the general kernels run) against one
    force evaluation (rrg_dev_direct_forces_f32) at the same N, Plummer spheres, eps = 0.02."""
    from . import lib
    res = {"form": "direct_vjp", "reps": reps, "sizes": {}}
    s = torch.cuda.current_stream()
    for n in sizes:
        pos, _ = generate_plummer(5, n, 1.0, 1.0, 20.0)
        m = np.linspace(0.5, 2.0, n) / n
        row = {}
        for prec, dt_ in (("fp32", torch.float32), ("fp64", torch.float64)):
            posm = torch.tensor(np.c_[pos, m], dtype=dt_, device="cuda").contiguous()
            lam = torch.randn(n, 4, dtype=dt_, device="cuda")
            lam[:, 3] = 0
            for _ in range(3):
                direct_vjp(posm, lam, 4e-4)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                direct_vjp(posm, lam, 4e-4)
            b.record()
            torch.cuda.synchronize()
            ms = a.elapsed_time(b) / reps
            row[prec] = {"vjp_ms": ms, "vjp_gpairs_per_s": n * n / (ms * 1e-3) / 1e9}
            if prec == "fp32":
                out = torch.empty_like(posm)
                L = lib()
                for _ in range(3):
                    check(L.rrg_dev_direct_forces_f32(posm.data_ptr(), None, None, C.c_float(2e-4),
                                                      n, out.data_ptr(), PREC["fp32"],
                                                      s.cuda_stream))
                a.record()
                for _ in range(reps):
                    check(L.rrg_dev_direct_forces_f32(posm.data_ptr(), None, None, C.c_float(2e-4),
                                                      n, out.data_ptr(), PREC["fp32"],
                                                      s.cuda_stream))
                b.record()
                torch.cuda.synchronize()
                fms = a.elapsed_time(b) / reps
                row[prec]["forces_ms"] = fms
                row[prec]["vjp_over_forces"] = ms / fms
                # 28 FP32 operations per pair in the general-mass VJP kernel
                row[prec]["vjp_tflops_at_28_per_pair"] = n * n * 28 / (ms * 1e-3) / 1e12
        res["sizes"][str(n)] = row
    return res


def bench_form_pm(torch_mod=None, n=262144, nx=64, nsteps=200, dt=2e-3, substeps=20, every=20,
                  fd_dirs=8):
    """PM adjoint: N = 262,144 disk particles on a 64^3 periodic grid (+-8 Rd), 20 substeps
    per step, 200 steps, checkpoints every 20; loss and targets as in bench_form. Wall-time
    ratio of the backward (recompute included) to the forward, FP32 vs FP64 gradients, and
    central differences (h = 1e-3, FP64) along random directions."""
    from . import Context, GridInfo, SimParams, WaveParams, generate_exp_disk
    pos, vel = generate_exp_disk(21, n, 1.0, 1.0, 0.1, 7.5, 7.5, 0.1, 0.0, 0.0)
    m = np.full(n, 1.0 / n)
    grid = GridInfo.from_values(nx, 16.0 / nx, 0.0)
    c = 10.0 * float(np.max(np.linalg.norm(vel, axis=1)))
    wave = WaveParams.make(grid.dx, diss_base=1.0 / (4 * grid.dx), wave_speed=c,
                           iterations=substeps, setup_iterations=4000, tolerance=1e-6)
    sim = SimParams(time_max=1.0, dt_save=1.0, dt_dynamics=dt, saves_without_dump=0,
                    use_wave_model=1)
    with Context(0, "fp64") as ctx:
        ctx.load_particles(pos, vel, m, np.full(n, 1e-4))
        ctx.init_grid(grid)
        ctx.set_wave_params(wave)
        ctx.solver_init(sim)
        ctx.precalc()
        phi = ctx.get_grid()["grav"]
    rng = np.random.default_rng(22)
    res = {"form": "adjoint_pm_262144_64", "n": n, "grid": nx, "steps": nsteps,
           "substeps": substeps, "checkpoint_every": every}
    pert = 1e-3 * rng.standard_normal((n, 3))
    grads = {}
    for prec, dt_ in (("fp32", torch.float32), ("fp64", torch.float64)):
        t = lambda a: torch.tensor(a, dtype=dt_, device="cuda")  # noqa: E731
        x0, v0, mm, ph = t(pos), t(vel), t(m), t(phi)
        eng = PMEngine(n, float(m.max()), grid, wave, dt, nsteps, prec, every)
        with torch.no_grad():
            xt, _ = pm_leapfrog(x0 + t(pert), v0, mm, ph, ph, eng)
        xr, vr, mr = (a.clone().requires_grad_(True) for a in (x0, v0, mm))
        xN, _ = pm_leapfrog(xr, vr, mr, ph, ph, eng)
        ((xN - xt) ** 2).sum(1).mean().backward()
        torch.cuda.synchronize()
        for a in (xr, vr, mr):
            a.grad = None
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        xN, _ = pm_leapfrog(xr, vr, mr, ph, ph, eng)
        loss = ((xN - xt) ** 2).sum(1).mean()
        e1.record()
        loss.backward()
        e2.record()
        torch.cuda.synchronize()
        fwd, bwd = e0.elapsed_time(e1), e1.elapsed_time(e2)
        grads[prec] = np.concatenate([a.grad.double().cpu().numpy().ravel() for a in (xr, vr, mr)])
        res[prec] = {"forward_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
                     "loss": float(loss.detach())}
        if prec == "fp64" and fd_dirs > 0:
            h = 1e-3
            rel, rel32 = [], []
            with torch.no_grad():
                for _ in range(fd_dirs):
                    d = rng.standard_normal(grads["fp64"].size)
                    d /= np.linalg.norm(d)
                    dx_ = t(d[:3 * n].reshape(n, 3))
                    dv_ = t(d[3 * n:6 * n].reshape(n, 3))
                    dm_ = t(d[6 * n:])
                    lp = ((pm_leapfrog(x0 + h * dx_, v0 + h * dv_, mm + h * dm_, ph, ph, eng)[0]
                           - xt) ** 2).sum(1).mean()
                    lm = ((pm_leapfrog(x0 - h * dx_, v0 - h * dv_, mm - h * dm_, ph, ph, eng)[0]
                           - xt) ** 2).sum(1).mean()
                    fd = float(lp - lm) / (2 * h)
                    rel.append(abs(grads["fp64"] @ d - fd) / max(abs(fd), 1e-300))
                    rel32.append(abs(grads["fp32"] @ d - fd) / max(abs(fd), 1e-300))
            res["fd_check"] = {"directions": fd_dirs, "h": h,
                               "fp64_adjoint_rel_err_median": float(np.median(rel)),
                               "fp64_adjoint_rel_err_max": float(np.max(rel)),
                               "fp32_adjoint_rel_err_median": float(np.median(rel32))}
        eng.close()
    res["fp32_vs_fp64_gradient_rel_l2"] = float(np.linalg.norm(grads["fp32"] - grads["fp64"]) /
                                                np.linalg.norm(grads["fp64"]))
    res["adjoint_over_forward_fp32"] = res["fp32"]["backward_over_forward"]
    return res


if __name__ == "__main__":
    print(json.dumps(bench_form()))
    print(json.dumps(bench_form_pm()))
