"""The hand-written adjoint (csrc/adjoint.cu) against independent FP64 gradients: torch
autograd through a plain torch restatement of the same force and leapfrog, and central finite
differences."""
import numpy as np
import pytest

import rrgsim_b200 as rg
from helpers import plummer

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rrgsim_b200.adjoint import LeapfrogEngine, direct_vjp, nbody_leapfrog  # noqa: E402


def torch_acc(x, m, s2):
    d = x[None, :, :] - x[:, None, :]          # d_ij = x_j - x_i (nbody.cu:45-49)
    r2 = (d * d).sum(-1) + s2                   # + (soft2_i + soft2_j) / 2, uniform here
    f = r2 ** -1.5
    return (m[None, :, None] * d * f[..., None]).sum(1)


def torch_leapfrog(x, v, m, s2, dt, steps):
    a = torch_acc(x, m, s2)
    for _ in range(steps):                      # nbody.cu:139-151, 175-180
        vs = v + dt * a
        u = v + vs
        x = x + dt * 0.5 * u
        a = torch_acc(x, m, s2)
        v = 0.5 * (u + dt * a)
    return x, v


def _inputs(n, seed, dtype):
    pos, vel, m, _ = plummer(n, seed=seed)
    t = lambda a: torch.tensor(a, dtype=dtype, device="cuda")  # noqa: E731
    return t(pos), t(vel), t(m)


@pytest.mark.parametrize("n", [300, 1537])
@pytest.mark.parametrize("masses", ["equal", "spread"])
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 2e-4)])
def test_force_vjp_matches_autograd(dtype, tol, masses, n):
    s2 = 0.02 ** 2
    x, _, m = _inputs(n, 1, torch.float64)
    if masses == "spread":
        m = m * torch.linspace(0.5, 2.0, n, dtype=torch.float64, device="cuda")
    lam = torch.randn(n, 3, dtype=torch.float64, device="cuda")
    xr, mr = x.clone().requires_grad_(True), m.clone().requires_grad_(True)
    (torch_acc(xr, mr, s2) * lam).sum().backward()
    posm = torch.cat([x, m[:, None]], 1).to(dtype).contiguous()
    lam4 = torch.cat([lam, torch.zeros(n, 1, dtype=torch.float64, device="cuda")], 1).to(dtype)
    out = direct_vjp(posm, lam4.contiguous(), s2).double()
    gx, gm = xr.grad, mr.grad
    assert torch.linalg.norm(out[:, :3] - gx) / torch.linalg.norm(gx) <= tol
    assert torch.linalg.norm(out[:, 3] - gm) / torch.linalg.norm(gm) <= tol


@pytest.mark.parametrize("every", [1, 5, 0])
def test_leapfrog_adjoint_matches_autograd_fp64(every):
    n, s2, dt, steps = 64, 0.05 ** 2, 2e-3, 20
    x, v, m = _inputs(n, 2, torch.float64)
    target = x + 0.01 * torch.randn_like(x)
    grads = []
    for ours in (True, False):
        xr, vr, mr = (t.clone().requires_grad_(True) for t in (x, v, m))
        if ours:
            xN, vN = nbody_leapfrog(xr, vr, mr, s2, dt, steps, checkpoint_every=every)
        else:
            xN, vN = torch_leapfrog(xr, vr, mr, s2, dt, steps)
        loss = ((xN - target) ** 2).sum(1).mean() + 0.3 * (vN ** 2).sum(1).mean()
        loss.backward()
        grads.append((xr.grad, vr.grad, mr.grad))
    for a, b in zip(*grads):
        assert torch.linalg.norm(a - b) / torch.linalg.norm(b) <= 1e-10


def test_leapfrog_adjoint_central_differences_fp64():
    n, s2, dt, steps = 256, 0.02 ** 2, 1e-3, 40
    x, v, m = _inputs(n, 3, torch.float64)
    target = x + 1e-3 * torch.randn_like(x)
    eng = LeapfrogEngine(n, dt, steps, s2, "fp64", checkpoint_every=8)
    xr, vr, mr = (t.clone().requires_grad_(True) for t in (x, v, m))
    loss = ((nbody_leapfrog(xr, vr, mr, s2, dt, steps, engine=eng)[0] - target) ** 2).sum(1).mean()
    loss.backward()
    g = torch.cat([xr.grad.ravel(), vr.grad.ravel(), mr.grad.ravel()])
    rng = np.random.default_rng(0)
    h = 1e-4
    with torch.no_grad():
        for _ in range(6):
            d = torch.tensor(rng.standard_normal(g.numel()), dtype=torch.float64, device="cuda")
            d /= torch.linalg.norm(d)
            dx, dv, dm = d[:3 * n].view(n, 3), d[3 * n:6 * n].view(n, 3), d[6 * n:]
            f = lambda s: ((nbody_leapfrog(x + s * dx, v + s * dv, m + s * dm, s2, dt, steps,  # noqa: E731
                                           engine=eng)[0] - target) ** 2).sum(1).mean()
            fd = float(f(h) - f(-h)) / (2 * h)
            assert abs(float(g @ d) - fd) <= 1e-6 * abs(fd) + 1e-14


@pytest.mark.parametrize("n,masses", [(2048, "equal"), (3001, "spread")])
def test_fp32_adjoint_close_to_fp64(n, masses):
    """Equal masses take the uniform-mass kernels in FP32, a spread of masses the general ones;
    3001 particles leave ragged last tiles."""
    s2, dt, steps = 0.02 ** 2, 1e-3, 60
    out = []
    for dtype in (torch.float32, torch.float64):
        x, v, m = _inputs(n, 4, dtype)
        if masses == "spread":
            m = m * torch.linspace(0.5, 2.0, n, dtype=dtype, device="cuda")
        target = x + 1e-3
        xr, vr, mr = (t.clone().requires_grad_(True) for t in (x, v, m))
        loss = ((nbody_leapfrog(xr, vr, mr, s2, dt, steps, checkpoint_every=20)[0] - target) ** 2).sum(1).mean()
        loss.backward()
        out.append(torch.cat([xr.grad.ravel(), vr.grad.ravel(), mr.grad.ravel()]).double())
    rel = float(torch.linalg.norm(out[0] - out[1]) / torch.linalg.norm(out[1]))
    assert rel <= 1e-3, rel


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_adjoint_without_mass_gradient(dtype):
    """Masses that need no gradient: the same position and velocity gradients, none for m."""
    n, s2, dt, steps = 1000, 0.02 ** 2, 1e-3, 30
    x, v, m = _inputs(n, 6, dtype)
    target = x + 1e-3
    grads = []
    for m_grad in (True, False):
        xr, vr = x.clone().requires_grad_(True), v.clone().requires_grad_(True)
        mr = m.clone().requires_grad_(m_grad)
        loss = ((nbody_leapfrog(xr, vr, mr, s2, dt, steps, checkpoint_every=7)[0] - target) ** 2).sum(1).mean()
        loss.backward()
        grads.append((xr.grad, vr.grad, mr.grad))
    (gx1, gv1, gm1), (gx2, gv2, gm2) = grads
    assert gm1 is not None and gm2 is None
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    for a, b in ((gx1, gx2), (gv1, gv2)):
        assert float(torch.linalg.norm(a - b) / torch.linalg.norm(a)) <= tol
