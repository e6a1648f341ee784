"""Particle-mesh path on the GPU against the FP64 oracle.

CIC: the int64 fixed-point grid is bit-exact to the oracle's fixed-point deposit of the same
(FP32-held) particles, and equals the reference's FP64 deposit to within the fixed-point step.
Wave, gradient, interpolation and NGP lookups follow the reference within FP32 rounding.
"""
import numpy as np
import pytest

import oracle as orc
import rrgsim_b200 as rg
from helpers import disk, f32, rel_err

pytestmark = pytest.mark.gpu


def _grid(nx, half_width=8.0, bc_frac=0.2):
    return rg.GridInfo.from_values(nx, 2 * half_width / nx, bc_frac)


def _orc_grid(g: rg.GridInfo, **kw):
    bc_frac = 1.0 - g.sim_l / g.domain_l
    return orc.make_grid(g.nx, g.dx, bc_frac=bc_frac, **kw)


def _ctx(prec, pos, vel, m, s2, grid):
    c = rg.Context(0, prec)
    c.load_particles(pos, vel, m, s2)
    c.init_grid(grid)
    return c


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("n,nx", [(1, 8), (300, 8), (20000, 32), (200000, 64)])
def test_cic_fixed_point_bit_exact(prec, n, nx):
    pos, vel, m, s2 = disk(n, seed=n)
    # particles outside the domain and on its faces exercise the reference's clamp
    if n >= 300:
        pos[:5] = [[9.0, 0, 0], [-9.0, -9.0, 9.0], [8.0, 8.0, -8.0], [0.0625, 0.0625, 0.0625],
                   [-8.0, 0.0, 7.999]]
    g = _grid(nx)
    with _ctx(prec, pos, vel, m, s2, g) as c:
        c.convert_particles_to_grid()
        mass = c.get_grid()["mass"]
        shift = c.deposit_scale()
    held_pos = pos if prec != "fp32" else f32(pos)
    held_m = m if prec == "fp64" else f32(m)
    og = _orc_grid(g)
    q = orc.cic_fixed(held_pos, held_m, og, shift)
    np.testing.assert_array_equal(mass, q.astype(np.float64) * 2.0 ** -shift)
    # against the reference's FP64 deposit: within 8 half-steps of 2^-S per particle
    ref = orc.cic_fp64(held_pos, held_m, og)
    assert np.max(np.abs(mass - ref)) <= 8 * n * 2.0 ** -shift
    assert abs(mass.sum() - held_m.sum()) <= 8 * n * 2.0 ** -shift


def test_cic_run_to_run_deterministic():
    pos, vel, m, s2 = disk(100000, seed=9)
    g = _grid(64)
    grids = []
    for _ in range(2):
        with _ctx("fp32", pos, vel, m, s2, g) as c:
            c.convert_particles_to_grid()
            grids.append(c.get_grid()["mass"])
    np.testing.assert_array_equal(grids[0], grids[1])


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_cic_same_grid_in_any_particle_order(prec):
    """The deposit sums runs of equal cells per warp, sorting a warp's cells first when they
    interleave: particles sorted by cell (few runs per warp), sorted then moved a little (runs
    broken up), and shuffled (a warp sort in nearly every warp) give the same fixed-point grid,
    the oracle's."""
    rng = np.random.default_rng(17)
    pos, vel, m, s2 = disk(200000, seed=17)
    g = _grid(64)
    key = np.floor((pos + 8.0) / g.dx - 0.5).clip(0, 63).astype(np.int64)
    order = np.argsort((key[:, 2] * 64 + key[:, 1]) * 64 + key[:, 0], kind="stable")
    moved = pos[order] + 0.3 * g.dx * rng.uniform(-1, 1, (len(pos), 3))
    shuffled = rng.permutation(len(pos))
    cases = [(pos[order], m[order]), (moved, m[order]), (pos[shuffled], m[shuffled]),
             (moved[::-1].copy(), m[order][::-1].copy())]
    grids = []
    for p, mm in cases:
        with _ctx(prec, p, vel[: len(p)], mm, s2, g) as c:
            c.convert_particles_to_grid()
            grids.append(c.get_grid()["mass"])
            shift = c.deposit_scale()
    np.testing.assert_array_equal(grids[0], grids[2])
    np.testing.assert_array_equal(grids[1], grids[3])
    held_pos = (lambda a: a) if prec != "fp32" else f32
    held_m = (lambda a: a) if prec == "fp64" else f32
    og = _orc_grid(g)
    for (p, mm), got in zip(cases[:2], grids[:2]):
        q = orc.cic_fixed(held_pos(p), held_m(mm), og, shift)
        np.testing.assert_array_equal(got, q.astype(np.float64) * 2.0 ** -shift)


def _wave_setup(nx, prec, seed=11):
    rng = np.random.default_rng(seed)
    pos, vel, m, s2 = disk(20000, seed=seed)
    g = _grid(nx)
    vmax = np.max(np.linalg.norm(vel, axis=1))
    c_speed = 10 * vmax
    wp = rg.WaveParams.make(g.dx, diss_base=1.0 / (4 * g.dx), wave_speed=c_speed,
                            iterations=20, setup_iterations=400, steady_check_step=30)
    phi0 = -1.0 + 0.1 * rng.standard_normal(nx ** 3)
    return pos, vel, m, s2, g, wp, phi0


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("nx", [8, 33, 64, 128])
def test_wave_iteration_matches_oracle(prec, nx):
    pos, vel, m, s2, g, wp, phi0 = _wave_setup(nx, prec)
    with _ctx(prec, pos, vel, m, s2, g) as c:
        c.set_wave_params(wp)
        c.convert_particles_to_grid()
        c.set_boundary_periodic(1.0)
        c.set_grid_potential(phi0)
        it, _ = c.solve_wave_equation(3)
        got = c.get_grid()
    assert it == 3
    og = _orc_grid(g, wave_speed=wp.wave_speed, diss_base=wp.diss_base, bc_type=1,
                   rho_mean=1.0 / (nx * g.dx) ** 3)
    phi = phi0 if prec == "fp64" else f32(phi0)
    st = orc.WaveState(nx)
    st.set_all(phi)
    st.solve(og, got["mass"], 3)
    ref = st.curr
    tol = 1e-12 if prec == "fp64" else 2e-6
    assert np.max(np.abs(got["grav"] - ref)) <= tol * np.max(np.abs(ref))


@pytest.mark.parametrize("bc", ["zero", "monopole", "radiative", "periodic_layer"])
def test_wave_boundaries_match_oracle(bc):
    nx = 24
    pos, vel, m, s2, g, wp, phi0 = _wave_setup(nx, "fp64")
    wp.diss_extra = 0.3
    com = np.array([0.1, -0.05, 0.02])
    with _ctx("fp64", pos, vel, m, s2, g) as c:
        c.set_wave_params(wp)
        c.convert_particles_to_grid()
        if bc == "zero":
            c.set_boundary_zero()
            kw = dict(bc_type=0)
        elif bc == "periodic_layer":
            c.set_boundary_periodic(1.0, keep_layer=True)
            kw = dict(bc_type=1, rho_mean=1.0 / (nx * g.dx) ** 3, keep_layer=1)
        else:
            c.set_boundary_monopole(1.0, com, radiative=(bc == "radiative"))
            kw = dict(bc_type=3 if bc == "radiative" else 2, bc_mass=1.0, com=tuple(com))
        c.set_grid_potential(phi0)
        c.solve_wave_equation(4)
        got = c.get_grid()
    og = _orc_grid(g, wave_speed=wp.wave_speed, diss_base=wp.diss_base,
                   diss_extra=wp.diss_extra, **kw)
    st = orc.WaveState(nx)
    st.set_all(phi0)
    st.solve(og, got["mass"], 4)
    np.testing.assert_allclose(got["grav"], st.curr, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_steady_state_relaxation(prec):
    nx = 32
    pos, vel, m, s2, g, wp, _ = _wave_setup(nx, prec)
    wp.tolerance = 1e-4
    wp.steady_check_step = 10
    with _ctx(prec, pos, vel, m, s2, g) as c:
        c.set_wave_params(wp)
        c.convert_particles_to_grid()
        c.set_boundary_periodic(1.0)
        it, rel = c.solve_wave_equation(3000)
        got = c.get_grid()
    og = _orc_grid(g, wave_speed=wp.wave_speed, diss_base=wp.diss_base, bc_type=1,
                   rho_mean=1.0 / (nx * g.dx) ** 3, tolerance=1e-4, steady_check_step=10)
    st = orc.WaveState(nx)
    rit, rrel = st.solve(og, got["mass"], 3000)
    if prec == "fp64":
        assert it == rit
        assert abs(rel - rrel) <= 1e-9 * rrel
    else:
        assert abs(it - rit) <= 20
    ref = st.curr
    assert np.max(np.abs(got["grav"] - ref)) <= (1e-12 if prec == "fp64" else 1e-3) * np.max(np.abs(ref))


@pytest.mark.parametrize("nx", [40, 32, 64, 128])
@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_gradient_and_interpolation(prec, nx):
    """nx = 40 runs the scalar gradient, 32 / 64 / 128 the float4-row one in FP32 and MIXED."""
    rng = np.random.default_rng(5)
    pos, vel, m, s2 = disk(30000, seed=5)
    pos[:4] = [[9.5, 0, 0], [-8.0, -8.0, -8.0], [7.99, 7.99, 7.99], [0.1, -0.1, 0.2]]
    g = _grid(nx)
    phi = np.sin(np.arange(nx ** 3) * 0.37) + 0.1 * rng.standard_normal(nx ** 3)
    with _ctx(prec, pos, vel, m, s2, g) as c:
        c.set_grid_potential(phi)
        c.calc_acceleration_field()
        c.project_grid_acceleration_on_particles()
        c.project_grid_grav_on_particles()
        grid = c.get_grid()
        part = c.get_particles()
    og = _orc_grid(g)
    held_phi = phi if prec == "fp64" else f32(phi)
    held_pos = f32(pos) if prec == "fp32" else pos
    acc3 = orc.gradient(og, held_phi)
    tol = 1e-12 if prec == "fp64" else 1e-5
    assert np.max(np.abs(grid["acc"] - acc3)) <= tol * np.max(np.abs(acc3))
    ref = orc.interp(held_pos, og, acc3)
    assert np.max(np.abs(part["acc"] - ref)) <= tol * np.max(np.abs(acc3))
    np.testing.assert_array_equal(part["grav"], orc.ngp_phi(held_pos, og, grid["grav"]))


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_pm_steps_match_oracle(prec):
    """Disk N=20000 on a 32^3 periodic wave grid: precalc + 10 fused steps of 20 substeps."""
    nx, n, dt, steps = 32, 20000, 2e-3, 10
    pos, vel, m, s2 = disk(n, seed=1)
    g = _grid(nx)
    vmax = np.max(np.linalg.norm(vel, axis=1))
    wp = rg.WaveParams.make(g.dx, diss_base=1.0 / (4 * g.dx), wave_speed=10 * vmax,
                            iterations=20, setup_iterations=600, steady_check_step=1000)
    sim = rg.SimParams(time_max=1.0, dt_save=0.1, dt_dynamics=dt, saves_without_dump=2 ** 63,
                       use_wave_model=1)
    with _ctx(prec, pos, vel, m, s2, g) as c:
        c.set_wave_params(wp)
        c.solver_init(sim)
        c.precalc()
        c.sync_particles_and_grid()
        a0 = c.get_particles()["acc"]
        c.calc_steps(steps)
        got = c.get_particles()
    og = _orc_grid(g, wave_speed=wp.wave_speed, diss_base=wp.diss_base, bc_type=1,
                   rho_mean=1.0 / (nx * g.dx) ** 3, steady_check_step=1000)
    st = orc.WaveState(nx)
    mgrid = orc.cic_fp64(pos, m, og)
    st.solve(og, mgrid, 600)
    ra0 = orc.interp(pos, og, orc.gradient(og, st.curr))
    # the deposit is int64 fixed point in every precision (2^-27 relative per contribution),
    # so even the FP64 path differs from the reference's FP64 atomics at the 1e-8 level.
    # Measured: precalc accelerations FP32 / MIXED 2.2e-6 / 2.3e-6 (the relaxations differ by the
    # steady state's FP32 rounding), FP64 3.4e-10; after 10 steps accelerations 1.1e-7 / 9.6e-8 /
    # 3.6e-10, positions 4.8e-8 / 4.7e-10 / 2.6e-15, velocities 9.0e-8 / 9.0e-8 / 6.2e-13.
    tol_a = 1e-8 if prec == "fp64" else 1e-5
    assert np.median(rel_err(a0, ra0)) <= tol_a
    rp, rv, ra = orc.pm_steps(pos, vel, ra0, m, og, 20, dt, st, steps)
    print(f"\n{prec}: precalc acc {np.median(rel_err(a0, ra0)):.3e}; after {steps} steps: acc "
          f"{np.median(rel_err(got['acc'], ra)):.3e}, pos {np.median(rel_err(got['pos'], rp)):.3e}, "
          f"vel {np.median(rel_err(got['vel'], rv)):.3e}")
    assert np.median(rel_err(got["pos"], rp)) <= {"fp64": 1e-12, "mixed": 5e-9, "fp32": 3e-7}[prec]
    assert np.max(np.abs(got["pos"] - rp)) <= (1e-9 if prec == "fp64" else 2e-5)
    assert np.median(rel_err(got["vel"], rv)) <= (1e-10 if prec == "fp64" else 1e-6)
    assert np.median(rel_err(got["acc"], ra)) <= (1e-8 if prec == "fp64" else 1e-6)


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_sorting_by_cell_changes_nothing_but_memory_order(prec):
    """The counting sort between fused chunks permutes memory only (the synced state and a
    pending prediction alike): results are bit-identical with and without it, and particles
    come back in their original order."""
    nx, n, dt = 32, 30000, 2e-3
    pos, vel, m, s2 = disk(n, seed=2)
    g = _grid(nx)
    vmax = np.max(np.linalg.norm(vel, axis=1))
    wp = rg.WaveParams.make(g.dx, diss_base=1.0 / (4 * g.dx), wave_speed=10 * vmax,
                            iterations=20, setup_iterations=200, steady_check_step=1000)
    sim = rg.SimParams(time_max=1.0, dt_save=0.1, dt_dynamics=dt, saves_without_dump=2 ** 63,
                       use_wave_model=1)
    out = []
    for interval in (0, 7):
        with _ctx(prec, pos, vel, m, s2, g) as c:
            c.set_sort_interval(interval)
            c.set_wave_params(wp)
            c.solver_init(sim)
            c.precalc()
            c.sync_particles_and_grid()
            c.calc_steps(23)
            c.calc_steps(9)
            c.sync_particles_and_grid()
            out.append((c.get_particles(), c.get_grid()))
    (p0, g0), (p1, g1) = out
    for k in ("pos", "vel", "acc", "grav"):
        np.testing.assert_array_equal(p0[k], p1[k])
    np.testing.assert_array_equal(g0["mass"], g1["mass"])
    np.testing.assert_array_equal(g0["grav"], g1["grav"])


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_nbody_sync_projects_particles_on_grid(prec):
    """N-body strategy with a grid (rrgsim_integration_nbody.cuh:32-48): the sync deposits the
    CIC mass and writes NGP cell averages of the particle potential and acceleration."""
    n, nx, dt = 6000, 16, 1e-3
    pos, vel, m, s2 = disk(n, seed=21)
    pos[:3] = [[9.5, 0, 0], [-8.0, -8.0, 8.0], [0.0, 0.0, 0.0]]  # clamped and face cells
    g = _grid(nx)
    sim = rg.SimParams(time_max=1.0, dt_save=0.1, dt_dynamics=dt, saves_without_dump=2 ** 63,
                       use_wave_model=0)
    with _ctx(prec, pos, vel, m, s2, g) as c:
        c.solver_init(sim)
        c.precalc()
        c.calc_steps(3)
        c.sync_particles_and_grid()
        p = c.get_particles()
        grid = c.get_grid()
        shift = c.deposit_scale()
    og = _orc_grid(g)
    held_m = m if prec == "fp64" else f32(m)
    held_pos = p["pos"] if prec == "fp64" else f32(p["pos"])
    q = orc.cic_fixed(held_pos, held_m, og, shift)
    np.testing.assert_array_equal(grid["mass"], q.astype(np.float64) * 2.0 ** -shift)
    want_phi = orc.ngp_project(held_pos, og, p["grav"])
    want_acc = orc.ngp_project(held_pos, og, p["acc"])
    # cell sums of value / count: the order of the device's atomics only
    tol = 1e-12 if prec == "fp64" else 2e-6
    scale_phi = np.max(np.abs(want_phi))
    scale_acc = np.max(np.abs(want_acc))
    assert np.max(np.abs(grid["grav"] - want_phi)) <= tol * scale_phi
    assert np.max(np.abs(grid["acc"] - want_acc)) <= tol * scale_acc
    occupied = np.bincount(orc.ngp_cell(held_pos, og), minlength=nx ** 3) > 0
    assert np.all(grid["grav"][~occupied] == 0.0)
    assert np.all(grid["grav"][occupied] < 0.0)


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("interval", [0, 4])
def test_step_by_step_calls_equal_one_long_call(prec, interval):
    """Each calc_steps call ends by predicting the next step (kept pending, adopted by the next
    call); reads in between see the synced state. One call of 12 steps, 12 calls of one step
    and calls split around reads give the same bits."""
    nx, n, dt = 32, 20000, 2e-3
    pos, vel, m, s2 = disk(n, seed=5)
    g = _grid(nx)
    vmax = np.max(np.linalg.norm(vel, axis=1))
    wp = rg.WaveParams.make(g.dx, diss_base=1.0 / (4 * g.dx), wave_speed=10 * vmax,
                            iterations=20, setup_iterations=200, steady_check_step=1000)
    sim = rg.SimParams(time_max=1.0, dt_save=0.1, dt_dynamics=dt, saves_without_dump=2 ** 63,
                       use_wave_model=1)
    out = []
    for plan in ("long", "single", "split", "prepared"):
        with _ctx(prec, pos, vel, m, s2, g) as c:
            c.set_sort_interval(interval)
            c.set_wave_params(wp)
            c.solver_init(sim)
            c.precalc()
            if plan == "long":
                c.calc_steps(12)
            elif plan == "single":
                for _ in range(12):
                    c.calc_steps(1)
            elif plan == "prepared":
                # recording the graphs of the next call ahead of it runs nothing and changes
                # nothing
                c.calc_steps(3)
                before = c.get_particles()
                c.prepare_steps(9)
                c.prepare_steps(9)
                after = c.get_particles()
                for k in ("pos", "vel", "acc"):
                    np.testing.assert_array_equal(before[k], after[k])
                assert c.time()[1] == 3
                c.calc_steps(9)
            else:
                c.calc_steps(5)
                mid = c.get_particles()
                c.calc_conservation()
                c.get_grid()
                c.calc_steps(7)
            out.append((c.get_particles(), c.get_grid()))
            if plan == "split":
                with _ctx(prec, pos, vel, m, s2, g) as r:
                    r.set_sort_interval(interval)
                    r.set_wave_params(wp)
                    r.solver_init(sim)
                    r.precalc()
                    r.calc_steps(5)
                    ref_mid = r.get_particles()
                for k in ("pos", "vel", "acc"):
                    np.testing.assert_array_equal(mid[k], ref_mid[k])
    for p, gr in out[1:]:
        for k in ("pos", "vel", "acc"):
            np.testing.assert_array_equal(p[k], out[0][0][k])
        np.testing.assert_array_equal(gr["mass"], out[0][1]["mass"])
        np.testing.assert_array_equal(gr["grav"], out[0][1]["grav"])


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_step_sums_equal_a_pass_over_the_particles(prec):
    """With set_step_sums the last particle pass of each calc_steps call also forms the
    conservation sums (nbody.cu:246-291) of the state it leaves, and a calc_conservation or
    calc_conservation_async right after the call only combines them: one kernel instead of two.
    The sums equal those of the pass over the particles bit for bit, the steps do not change,
    and a call that may change the state in between (here the sync, which rewrites the
    particles' potential) makes the sums come from the particles again."""
    torch = pytest.importorskip("torch")
    nx, n, dt = 32, 20000, 2e-3
    pos, vel, m, s2 = disk(n, seed=5)
    m = m * np.linspace(0.5, 1.5, n)
    g = _grid(nx)
    vmax = np.max(np.linalg.norm(vel, axis=1))
    wp = rg.WaveParams.make(g.dx, diss_base=1.0 / (4 * g.dx), wave_speed=10 * vmax,
                            iterations=20, setup_iterations=200, steady_check_step=1000)
    sim = rg.SimParams(time_max=1.0, dt_save=0.1, dt_dynamics=dt, saves_without_dump=2 ** 63,
                       use_wave_model=1)
    calls = [1, 1, 3, 1, 6, 1]  # sorts (every 4 steps) fall inside and between calls
    res = {}
    for on in (False, True):
        sums = torch.full((len(calls), 12), float("nan"), dtype=torch.float64).pin_memory().numpy()
        rows, launches = [], []
        with _ctx(prec, pos, vel, m, s2, g) as c:
            c.set_sort_interval(4)
            c.set_wave_params(wp)
            c.solver_init(sim)
            c.precalc()
            c.sync_particles_and_grid()  # a potential on the particles: Ep is not zero
            c.set_step_sums(on)
            for k, steps in enumerate(calls):
                c.calc_steps(steps)
                if k == 3:
                    c.sync_particles_and_grid()
                l0 = rg.kernel_launch_count()
                c.calc_conservation_async(sums[k])
                rows.append(c.calc_conservation())
                launches.append(rg.kernel_launch_count() - l0)
            c.synchronize()
            res[on] = (rows, launches, sums.copy(), c.get_particles())
    rows_off, launches_off, sums_off, p_off = res[False]
    rows_on, launches_on, sums_on, p_on = res[True]
    assert launches_off == [4] * len(calls)
    assert launches_on == [2, 2, 2, 4, 2, 2]
    assert rows_on[0]["Ep"] != 0.0
    for a, b in zip(rows_off, rows_on):
        assert a["Ek"] == b["Ek"] and a["Ep"] == b["Ep"]
        np.testing.assert_array_equal(a["momentum"], b["momentum"])
        np.testing.assert_array_equal(a["angular"], b["angular"])
    np.testing.assert_array_equal(sums_off, sums_on)
    for k in ("pos", "vel", "acc"):
        np.testing.assert_array_equal(p_off[k], p_on[k])


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
@pytest.mark.parametrize("nx,iterations", [(32, 20), (64, 7), (64, 1), (128, 20), (128, 7),
                                           (128, 1)])
def test_persistent_wave_solve_equals_one_launch_per_substep(monkeypatch, prec, nx, iterations):
    """Periodic FP32 grids of 32, 64 and 128 cells run each step's source, substeps and
    gradient as one persistent kernel; RRG_WAVE_PERSIST=0 launches them one by one. Same bits
    for the particles, the potential levels and the field, over steps with sorts in between,
    odd substep counts (the level parity flips every step; one substep swaps the final and the
    previous level within the launch) and split calls."""
    n, dt = 60000, 2e-3
    pos, vel, m, s2 = disk(n, seed=nx + iterations)
    g = _grid(nx)
    vmax = np.max(np.linalg.norm(vel, axis=1))
    wp = rg.WaveParams.make(g.dx, diss_base=1.0 / (4 * g.dx), wave_speed=10 * vmax,
                            iterations=iterations, setup_iterations=100,
                            steady_check_step=1000)
    sim = rg.SimParams(time_max=1.0, dt_save=0.1, dt_dynamics=dt, saves_without_dump=2 ** 63,
                       use_wave_model=1)
    out, launches = [], []
    for persist in ("1", "0"):
        monkeypatch.setenv("RRG_WAVE_PERSIST", persist)
        with _ctx(prec, pos, vel, m, s2, g) as c:
            c.set_sort_interval(3)
            c.set_wave_params(wp)
            c.solver_init(sim)
            c.precalc()
            k0 = rg.kernel_launch_count()
            c.calc_steps(4)
            mid = c.get_particles()
            c.calc_steps(5)
            c.synchronize()
            launches.append(rg.kernel_launch_count() - k0)
            out.append((mid, c.get_particles(), c.get_grid(), c.get_wave_state()))
    (mid1, p1, g1, w1), (mid0, p0, g0, w0) = out
    for k in ("pos", "vel", "acc"):
        np.testing.assert_array_equal(mid1[k], mid0[k])
        np.testing.assert_array_equal(p1[k], p0[k])
    for k in g1:
        np.testing.assert_array_equal(g1[k], g0[k])
    for a, b in zip(w1, w0):
        np.testing.assert_array_equal(a, b)
    # one kernel instead of the increments' preparation, the substeps, the finish and the
    # gradient in each of the 9 steps
    assert launches[0] + 9 * (iterations + 2) == launches[1]


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("nx", [64, 40, 128])
def test_solve_wave_and_field_against_separate_calls(monkeypatch, prec, nx):
    """The one-call solve (the fused steps' solve). FP64: the same bits as
    solve_wave_equation + calc_acceleration_field. FP32 / MIXED on periodic grids: the
    incremental form (each solve advances increments over its first level, rounded into the
    level once at the end), the same bits from the persistent kernels (64^3, 128^3) and from one
    launch per substep (RRG_WAVE_PERSIST=0; 40^3 always), and against the FP64 oracle within
    the bound of the separate calls, which advance the full levels in FP32."""
    pos, vel, m, s2, g, wp, phi0 = _wave_setup(nx, prec)
    wp.steady_check_step = 10 ** 6  # no steady checks inside the 7 substeps

    def run(fused):
        with _ctx(prec, pos, vel, m, s2, g) as c:
            c.set_wave_params(wp)
            c.convert_particles_to_grid()
            c.set_boundary_periodic(1.0)
            c.set_grid_potential(phi0)
            if fused:
                c.solve_wave_and_field(7)
            else:
                it, _ = c.solve_wave_equation(7)
                assert it == 7
                c.calc_acceleration_field()
            return c.get_grid(), c.get_wave_state()

    (g1, w1), (g0, w0) = run(True), run(False)
    if prec == "fp64":
        for k in g1:
            np.testing.assert_array_equal(g1[k], g0[k])
        for a, b in zip(w1, w0):
            np.testing.assert_array_equal(a, b)
        return
    monkeypatch.setenv("RRG_WAVE_PERSIST", "0")
    g2, w2 = run(True)
    for k in g1:
        np.testing.assert_array_equal(g1[k], g2[k])
    for a, b in zip(w1, w2):
        np.testing.assert_array_equal(a, b)
    og = _orc_grid(g, wave_speed=wp.wave_speed, diss_base=wp.diss_base, bc_type=1,
                   rho_mean=1.0 / (nx * g.dx) ** 3)
    st = orc.WaveState(nx)
    st.set_all(f32(phi0))
    st.solve(og, g1["mass"], 7)
    scale = np.max(np.abs(st.curr))
    e_inc = np.max(np.abs(g1["grav"] - st.curr)) / scale
    e_plain = np.max(np.abs(g0["grav"] - st.curr)) / scale
    assert e_inc <= 2e-6 and e_inc <= 1.5 * e_plain + 1e-9
    np.testing.assert_allclose(g1["grav"], g0["grav"], rtol=0, atol=4e-6 * scale)


@pytest.mark.parametrize("nx", [64, 128])
def test_persistent_solve_reports_a_wait_that_ran_out(nx):
    """Every wait between the persistent solve's thread blocks is bounded (~0.14 s). Rewinding
    one block's epoch counter makes its neighbours wait for epochs it never publishes: the
    waits run out, the kernel sets its error word and returns, the next synchronising call
    raises, and after that the context computes the same bits as a fresh one. (128^3 runs the
    two-substeps-per-exchange kernel, 64^3 the one-exchange-per-substep kernel.)"""
    from cuda.bindings import runtime as cudart

    pos, vel, m, s2, g, wp, phi0 = _wave_setup(nx, "fp32")

    def fresh_solve(c):
        c.set_wave_params(wp)
        c.convert_particles_to_grid()
        c.set_boundary_periodic(1.0)
        c.set_grid_potential(phi0)
        c.solve_wave_and_field(5)
        return c.get_grid()

    with _ctx("fp32", pos, vel, m, s2, g) as ref:
        want = fresh_solve(ref)
    with _ctx("fp32", pos, vel, m, s2, g) as c:
        fresh_solve(c)
        c.synchronize()
        ptr, nbytes = c.wave_solve_sync()
        assert ptr != 0 and nbytes >= 65536
        zero = np.zeros(1, dtype=np.uint32)
        err, = cudart.cudaMemcpy(ptr, zero.ctypes.data, 4, cudart.cudaMemcpyKind.cudaMemcpyHostToDevice)
        assert err == cudart.cudaError_t.cudaSuccess
        c.solve_wave_and_field(5)
        with pytest.raises(rg.RRGError, match="timed out"):
            c.synchronize()
        # the sync memory is clear again and the context usable
        got = fresh_solve(c)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k])


def test_load_particles_rejects_bad_input_on_the_device():
    """The upload is checked on the device: the lowest offending particle is named, positions
    and velocities before masses before softenings, and the context keeps its particles."""
    pos, vel, m, s2 = disk(5000, seed=4)
    g = _grid(16)
    with _ctx("fp32", pos, vel, m, s2, g) as c:
        keep = c.get_particles()
        cases = []
        p = pos.copy()
        p[1234, 1] = np.nan
        v = vel.copy()
        v[3000, 2] = np.inf
        cases.append(((p, v, m, s2), "non-finite position/velocity at particle 1234"))
        mm = m.copy()
        mm[77] = -1.0
        ss = s2.copy()
        ss[77] = np.nan
        cases.append(((pos, vel, mm, ss), "bad mass at particle 77"))
        ss = s2.copy()
        ss[4999] = -1e-4
        cases.append(((pos, vel, m, ss), "bad soft2 at particle 4999"))
        for args, msg in cases:
            with pytest.raises(rg.RRGError) as e:
                c.load_particles(*args)
            assert msg in str(e.value)
        got = c.get_particles()
        for k in ("pos", "vel"):
            np.testing.assert_array_equal(got[k], keep[k])
        # uniform and non-uniform masses / softenings both load
        mm = m.copy()
        mm[::3] *= 2.0
        ss = s2.copy()
        ss[::2] = 4e-4
        c.load_particles(pos, vel, mm, ss)
        c.convert_particles_to_grid()
        assert abs(c.get_grid()["mass"].sum() - f32(mm).sum()) <= 1e-6 * mm.sum()
