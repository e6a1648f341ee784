"""Known-answer tests from physics: the reference ships no tests, so besides its own build's
golden vectors these pin the solver to exact or analytic answers. Each runs on the FP64 oracle
(CPU) and on the CUDA path (GPU, every precision it applies to).

- CIC deposit: the mass is conserved and, for a particle away from the faces, the cell-centre
  mean of the deposited mass is the particle's position (partition of unity, first moment).
- Wave solver: a density of one periodic Fourier mode relaxes to the exact solution of the
  discrete Poisson equation that the damped wave equation's steady state satisfies,
  L_h phi = 4 pi (rho - rho_mean), solved by FFT with the 7-point stencil's eigenvalues
  sum_a (2 cos(k_a dx) - 2) / dx^2 (for the grid actually deposited: the reference's clamp of
  u to nx - 1 - 1e-6 moves 1e-6 of each last-plane particle to its neighbour).
- Leapfrog: the kick-drift-kick scheme of predict_step / correct_step is time-reversible:
  stepping back with negated velocities returns to the initial positions.
- Kepler: a softened two-body circular orbit keeps its energy and separation over two orbits.
- Plummer sphere: the direct-sum potential and radial force of 8192 particles follow
  -M / sqrt(r^2 + a^2) and -M r / (r^2 + a^2)^(3/2) up to sampling noise.
"""
import numpy as np
import pytest

import oracle as orc
import rrgsim_b200 as rg
from helpers import plummer

PRECS = ["fp32", "mixed", "fp64"]


# ---- CIC ------------------------------------------------------------------------------------
def _cell_centres(nx, dx):
    c = -0.5 * nx * dx + (np.arange(nx) + 0.5) * dx
    z, y, x = np.meshgrid(c, c, c, indexing="ij")  # x fastest
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)


def _cic_particles(n, nx, dx, seed):
    rng = np.random.default_rng(seed)
    # inside the cell centres' span, where no weight is clamped
    half = 0.5 * nx * dx - dx
    pos = rng.uniform(-half, half, size=(n, 3))
    mass = rng.uniform(0.5, 1.5, size=n) / n
    return pos, mass


def _check_cic(grid_mass, pos, mass, nx, dx, atol):
    np.testing.assert_allclose(grid_mass.sum(), mass.sum(), rtol=0, atol=atol * len(mass) + 1e-15)
    assert grid_mass.min() >= 0.0
    centres = _cell_centres(nx, dx)
    first = centres.T @ grid_mass
    np.testing.assert_allclose(first, (pos * mass[:, None]).sum(axis=0), rtol=0,
                               atol=nx * dx * atol * len(mass) + 1e-14)


def test_oracle_cic_conserves_mass_and_first_moment():
    nx, dx = 16, 1.0
    g = orc.make_grid(nx, dx)
    for seed in range(4):
        pos, mass = _cic_particles(1 if seed == 0 else 1000, nx, dx, seed)
        gm = orc.cic_fp64(pos, mass, g)
        if seed == 0:
            assert np.count_nonzero(gm) <= 8
        _check_cic(gm, pos, mass, nx, dx, 1e-16)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PRECS)
def test_gpu_cic_conserves_mass_and_first_moment(prec):
    nx, dx = 32, 0.5
    grid = rg.GridInfo.from_values(nx, dx, 0.0)
    for seed, n in ((0, 1), (1, 50000)):
        pos, mass = _cic_particles(n, nx, dx, seed)
        if prec == "fp32":
            pos = pos.astype(np.float32).astype(np.float64)
            mass = mass.astype(np.float32).astype(np.float64)
        with rg.Context(0, prec) as c:
            c.load_particles(pos, np.zeros_like(pos), mass, np.full(n, 1e-4))
            c.init_grid(grid)
            c.convert_particles_to_grid()
            gm = c.get_grid()["mass"]
            shift = c.deposit_scale()
        # each of the 8 corner values is rounded to a multiple of 2^-S
        _check_cic(gm, pos, mass, nx, dx, 8 * 0.5 * 2.0 ** -shift)


# ---- one Fourier mode through the wave solver --------------------------------------------
def _fourier_case(nx, dx, amp=0.5, kx=1):
    """One particle at each cell centre, masses (1 + amp sin(kappa x)) / nx^3 (total 1)."""
    L = nx * dx
    pos = _cell_centres(nx, dx)
    kappa = 2.0 * np.pi * kx / L
    mass = (1.0 + amp * np.sin(kappa * pos[:, 0])) / nx ** 3
    return pos, mass


def _poisson_fft(mass_grid, nx, dx):
    """The periodic solution of L_h phi = 4 pi (rho - rho_mean) with zero mean (the damped
    wave keeps the mean of a zero start), rho = cell mass / dx^3, rho_mean = 1 / L^3."""
    rho_dev = mass_grid.reshape(nx, nx, nx) / dx ** 3 - 1.0 / (nx * dx) ** 3
    k = 2.0 * np.pi * np.fft.fftfreq(nx)
    ev = (2.0 * np.cos(k) - 2.0) / dx ** 2
    lam = ev[:, None, None] + ev[None, :, None] + ev[None, None, :]
    lam[0, 0, 0] = 1.0
    ph = np.fft.fftn(4.0 * np.pi * rho_dev) / lam
    ph[0, 0, 0] = 0.0
    return np.real(np.fft.ifftn(ph)).ravel()


def test_oracle_wave_relaxes_to_the_discrete_poisson_solution():
    nx, dx = 16, 1.0
    pos, mass = _fourier_case(nx, dx)
    g = orc.make_grid(nx, dx, wave_speed=1.0, diss_base=1.0 / (4 * dx), bc_type=1,
                      rho_mean=1.0 / (nx * dx) ** 3, tolerance=0.0, steady_check_step=10 ** 6)
    gm = orc.cic_fp64(pos, mass, g)
    phi = _poisson_fft(gm, nx, dx)
    st = orc.WaveState(nx)
    it, _ = st.solve(g, gm, 3000)
    assert it == 3000
    assert np.max(np.abs(st.curr - phi)) <= 1e-10 * np.max(np.abs(phi))


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("nx,dx,one_call", [(16, 1.0, False), (32, 0.5, True)])
def test_gpu_wave_relaxes_to_the_discrete_poisson_solution(prec, nx, dx, one_call):
    """(32^3 in one call runs the persistent solve in FP32 and MIXED.)"""
    pos, mass = _fourier_case(nx, dx)
    grid = rg.GridInfo.from_values(nx, dx, 0.0)
    wp = rg.WaveParams.make(dx, diss_base=1.0 / (4 * dx), wave_speed=1.0, tolerance=0.0,
                            steady_check_step=10 ** 6)
    n = len(mass)
    with rg.Context(0, prec) as c:
        c.load_particles(pos, np.zeros_like(pos), mass, np.full(n, 1e-4))
        c.init_grid(grid)
        c.set_wave_params(wp)
        c.convert_particles_to_grid()
        c.set_boundary_periodic(1.0)
        c.set_grid_potential(np.zeros(nx ** 3))
        if one_call:
            c.solve_wave_and_field(3000)
        else:
            c.solve_wave_equation(3000)
        out = c.get_grid()
    # a periodic potential is defined up to a constant: the deposit's fixed-point rounding
    # leaves the total mass 1 +- ~1e-13, and the damped wave lets the mean of phi drift by
    # that residue (a uniform ~1e-10 in FP64 after 3000 substeps)
    got = out["grav"] - out["grav"].mean()
    phi = _poisson_fft(out["mass"], nx, dx)  # of the grid this run deposited
    # FP32 levels: the steady state carries the stencil's rounding times the lowest mode's
    # conditioning (~6 / (2 pi / nx)^2)
    tol = 1e-9 if prec == "fp64" else 1e-4
    assert np.max(np.abs(got - phi)) <= tol * np.max(np.abs(phi))


# ---- leapfrog time reversal ------------------------------------------------------------------
def _reversal_case():
    return plummer(256, seed=5, soft=0.05)


def test_oracle_leapfrog_is_time_reversible():
    pos, vel, m, s2 = _reversal_case()
    dt, k = 1e-3, 50
    p1, v1, a1 = orc.nbody_steps(pos, vel, orc.direct_acc(pos, m, s2), m, s2, dt, k)
    p2, v2, _ = orc.nbody_steps(p1, -v1, a1, m, s2, dt, k)
    assert np.max(np.abs(p2 - pos)) <= 1e-12
    assert np.max(np.abs(v2 + vel)) <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PRECS)
def test_gpu_leapfrog_is_time_reversible(prec):
    pos, vel, m, s2 = _reversal_case()
    dt, k = 1e-3, 50
    sim = rg.SimParams(time_max=1.0, dt_save=1.0, dt_dynamics=dt, saves_without_dump=2 ** 63,
                       use_wave_model=0)

    def run(p, v):
        with rg.Context(0, prec) as c:
            c.load_particles(p, v, m, s2)
            c.solver_init(sim)
            c.precalc()
            c.calc_steps(k)
            out = c.get_particles()
        return out["pos"], out["vel"]

    p1, v1 = run(pos, vel)
    p2, v2 = run(p1, -v1)
    tol = {"fp64": 1e-12, "mixed": 1e-6, "fp32": 2e-5}[prec]
    assert np.max(np.abs(p2 - pos)) <= tol


# ---- Kepler two-body orbit -------------------------------------------------------------------
def _kepler():
    pos = np.array([[0.5, 0.0, 0.0], [-0.5, 0.0, 0.0]])
    vel = np.array([[0.0, 0.5, 0.0], [0.0, -0.5, 0.0]])
    mass = np.array([0.5, 0.5])
    soft2 = np.full(2, 1e-10)
    return pos, vel, mass, soft2


def _circular(t):
    p = np.array([0.5 * np.cos(t), 0.5 * np.sin(t), 0.0])
    return np.stack([p, -p])


def _energy(pos, vel, mass, soft2):
    d2 = np.sum((pos[0] - pos[1]) ** 2) + 0.5 * (soft2[0] + soft2[1])
    return 0.5 * np.sum(mass * np.sum(vel ** 2, axis=1)) - mass[0] * mass[1] / np.sqrt(d2)


def test_oracle_kepler_orbit_keeps_energy_and_separation():
    pos, vel, mass, soft2 = _kepler()
    e0 = _energy(pos, vel, mass, soft2)
    dt = 1e-3
    acc = orc.direct_acc(pos, mass, soft2)
    per = int(round(2 * np.pi / dt))
    for _ in range(2):
        pos, vel, acc = orc.nbody_steps(pos, vel, acc, mass, soft2, dt, per)
        assert abs(_energy(pos, vel, mass, soft2) / e0 - 1.0) <= 1e-6
        assert abs(np.linalg.norm(pos[0] - pos[1]) - 1.0) <= 1e-6
    # on the exact circular orbit (angular speed 1) at the end time: the leapfrog's phase
    # error is O(dt^2) per unit time
    assert np.max(np.abs(pos - _circular(2 * per * dt))) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PRECS)
def test_gpu_kepler_orbit_keeps_energy_and_separation(prec):
    pos, vel, mass, soft2 = _kepler()
    e0 = _energy(pos, vel, mass, soft2)
    dt = 1e-3
    per = int(round(2 * np.pi / dt))
    sim = rg.SimParams(time_max=100.0, dt_save=100.0, dt_dynamics=dt,
                       saves_without_dump=2 ** 63, use_wave_model=0)
    # energy and separation; position on the exact orbit. FP32 velocities (FP32 and MIXED) walk
    # by their rounding over the 12,566 steps
    tol, ptol = {"fp64": (1e-6, 1e-5), "mixed": (1e-4, 1e-3), "fp32": (3e-4, 3e-3)}[prec]
    with rg.Context(0, prec) as c:
        c.load_particles(pos, vel, mass, soft2)
        c.solver_init(sim)
        c.precalc()
        for _ in range(2):
            c.calc_steps(per)
            s = c.get_particles()
            assert abs(_energy(s["pos"], s["vel"], mass, soft2) / e0 - 1.0) <= tol
            assert abs(np.linalg.norm(s["pos"][0] - s["pos"][1]) - 1.0) <= tol
    assert np.max(np.abs(s["pos"] - _circular(2 * per * dt))) <= ptol


# ---- Plummer sphere mean field ---------------------------------------------------------------
def _plummer_field(pos, acc, grav):
    r = np.linalg.norm(pos, axis=1)
    inner = r < 3.0
    phi_a = -1.0 / np.sqrt(r ** 2 + 1.0)
    ar_a = -r / (r ** 2 + 1.0) ** 1.5
    ar = np.sum(acc * pos, axis=1) / np.maximum(r, 1e-300)
    return inner, phi_a, ar_a, ar


def _check_plummer(pos, acc, grav, m, s2):
    inner, phi_a, ar_a, ar = _plummer_field(pos, acc, grav)
    # the self term -m_i / sqrt(soft2_i) of the reference's potential, removed
    phi = grav + m / np.sqrt(s2)
    assert np.median(np.abs(phi[inner] / phi_a[inner] - 1.0)) <= 0.02
    ratio = ar[inner] / ar_a[inner]
    assert np.median(np.abs(ratio - 1.0)) <= 0.1
    assert abs(np.median(ratio) - 1.0) <= 0.03


def test_oracle_plummer_sphere_follows_its_mean_field():
    pos, vel, m, s2 = plummer(8192, seed=7, soft=0.01)
    _check_plummer(pos, orc.direct_acc(pos, m, s2), orc.direct_grav(pos, m, s2), m, s2)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PRECS)
def test_gpu_plummer_sphere_follows_its_mean_field(prec):
    pos, vel, m, s2 = plummer(8192, seed=7, soft=0.01)
    with rg.Context(0, prec) as c:
        c.load_particles(pos, vel, m, s2)
        c.nbody_acceleration()
        c.nbody_grav()
        s = c.get_particles()
    _check_plummer(s["pos"], s["acc"], s["grav"], m, s2)
