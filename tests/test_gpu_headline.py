"""Parity at the measured sizes: the particle-mesh step of the benchmark workload (2^20 disk
particles, 128^3, 20 substeps, dt = 2e-3) against the FP64 oracle from the same state, and the
int64 CIC deposit of 8,388,608 disk particles on 256^3 against the oracle's fixed-point deposit.

The step is RectWaveIntegrationSolver::calc_step (rrgsim_integration_rect.cuh:99-112): predict,
CIC deposit (rm_p2mesh.cu:176-236), 20 damped-wave substeps (wave.cu:106-193), gradient
(rm_p2mesh.cu:238-290), trilinear interpolation (rm_mesh2p.cu:48-114), correct. The context's
synced state (positions, velocities, accelerations and both wave levels) is read back and the
oracle steps it in FP64, so each comparison measures the error of the fused steps alone.
"""
import numpy as np
import pytest

import oracle as orc
import rrgsim_b200 as rg
from helpers import disk, f32, rel_err

pytestmark = pytest.mark.gpu

N, NX, DT, SUB = 1 << 20, 128, 2e-3, 20


def _setup(prec):
    pos, vel, m, s2 = disk(N, seed=1)
    g = rg.GridInfo.from_values(NX, 16.0 / NX, 0.0)
    vmax = float(np.max(np.linalg.norm(vel, axis=1)))
    wp = rg.WaveParams.make(g.dx, diss_base=1.0 / (4 * g.dx), wave_speed=10 * vmax,
                            iterations=SUB, setup_iterations=400, steady_check_step=10 ** 6)
    sim = rg.SimParams(time_max=1e9, dt_save=1e9, dt_dynamics=DT, saves_without_dump=0,
                       use_wave_model=1)
    c = rg.Context(0, prec)
    c.load_particles(pos, vel, m, s2)
    c.init_grid(g)
    c.set_wave_params(wp)
    c.solver_init(sim)
    c.precalc()
    og = orc.make_grid(NX, g.dx, wave_speed=wp.wave_speed, diss_base=wp.diss_base, bc_type=1,
                       rho_mean=1.0 / (NX * g.dx) ** 3, steady_check_step=10 ** 9)
    return c, m, og


# Median relative error of the accelerations after one and after three fused steps from the
# same state (the bar: 1e-5), and of the positions after three. The solves advance increments
# over each step's first level (measured 2.1e-7 after one step, 2.9e-7 after three, in FP32 and
# MIXED; full FP32 levels gave 4.2e-6 after one step and 1.3e-5 after three); MIXED keeps
# double-float positions (measured 1.0e-10 against 3.1e-8 in FP32).
ACC_TOL = {"fp32": 1e-6, "mixed": 1e-6}
POS_TOL = {"fp32": 1e-7, "mixed": 1e-9}


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_headline_pm_steps_match_oracle(prec):
    c, m, og = _setup(prec)
    with c:
        c.calc_steps(2)  # into the fused regime: a pending prediction, sorted particles
        s0 = c.get_particles()
        cur, prev = c.get_wave_state()
        c.calc_steps(1)
        s1 = c.get_particles()
        c.calc_steps(2)
        s3 = c.get_particles()
    st = orc.WaveState(NX)
    st.bufs[0][:] = prev
    st.bufs[1][:] = cur
    held_m = f32(m)
    rp1, rv1, ra1 = orc.pm_steps(s0["pos"], s0["vel"], s0["acc"], held_m, og, SUB, DT, st, 1)
    rp3, rv3, ra3 = orc.pm_steps(rp1, rv1, ra1, held_m, og, SUB, DT, st, 2)
    e_acc1 = float(np.median(rel_err(s1["acc"], ra1)))
    e_acc3 = float(np.median(rel_err(s3["acc"], ra3)))
    e_pos3 = float(np.median(rel_err(s3["pos"], rp3)))
    print(f"\n{prec}: acc median rel err after 1 step {e_acc1:.3e}, after 3 {e_acc3:.3e}; "
          f"positions after 3 {e_pos3:.3e}")
    assert e_acc1 <= ACC_TOL[prec]
    assert e_acc3 <= ACC_TOL[prec]
    assert e_pos3 <= POS_TOL[prec]
    assert np.max(np.abs(s3["pos"] - rp3)) <= 1e-5


def test_cic_8M_particles_on_256_bit_exact():
    """int64 fixed-point CIC of 8,388,608 disk particles on 256^3 spanning +-8 Rd: the grid is
    bit-exact to the oracle's fixed-point deposit of the same FP32-held particles, and within
    the fixed-point step of the reference's FP64 deposit (rm_p2mesh.cu:176-236)."""
    n, nx = 8388608, 256
    pos, vel, m, s2 = disk(n, seed=2)
    g = rg.GridInfo.from_values(nx, 16.0 / nx, 0.0)
    with rg.Context(0, "fp32") as c:
        c.load_particles(pos, vel, m, s2)
        c.init_grid(g)
        c.convert_particles_to_grid()
        mass = c.get_grid()["mass"]
        shift = c.deposit_scale()
    og = orc.make_grid(nx, g.dx)
    hp, hm = f32(pos), f32(m)
    q = orc.cic_fixed(hp, hm, og, shift)
    np.testing.assert_array_equal(mass, q.astype(np.float64) * 2.0 ** -shift)
    # each of a particle's 8 contributions is rounded to the nearest 2^-S
    ref = orc.cic_fp64(hp, hm, og)
    assert np.max(np.abs(mass - ref)) <= 8 * n * 2.0 ** -shift
    assert abs(mass.sum() - hm.sum()) <= 8 * n * 2.0 ** -shift
