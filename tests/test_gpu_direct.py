"""Direct-sum gravity and leapfrog on the GPU against the FP64 oracle.

Bar: per-step accelerations within a median relative error of 1e-5 (FP32), 1e-6 (MIXED) and
1e-12 (FP64) of the oracle on the same FP64 inputs; positions after 10 steps within 1e-4.
"""
import numpy as np
import pytest

import oracle as orc
import rrgsim_b200 as rg
from helpers import f32, plummer, rel_err

pytestmark = pytest.mark.gpu

TOL_MEDIAN = {"fp32": 1e-5, "mixed": 1e-6, "fp64": 1e-12}


def _ctx(prec, pos, vel, m, s2):
    c = rg.Context(0, prec)
    c.load_particles(pos, vel, m, s2)
    return c


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("n", [1, 257, 4096, 20000])
def test_acceleration_matches_oracle(prec, n):
    pos, vel, m, s2 = plummer(n, seed=n)
    with _ctx(prec, pos, vel, m, s2) as c:
        c.nbody_acceleration()
        got = c.get_particles()["acc"]
    ref = orc.direct_acc(pos, m, s2)
    if n == 1:
        np.testing.assert_allclose(got, 0.0, atol=0)
        return
    err = rel_err(got, ref)
    assert np.median(err) <= TOL_MEDIAN[prec], np.median(err)
    assert np.max(err) <= (1e-3 if prec != "fp64" else 1e-10)


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_potential_matches_oracle(prec):
    n = 3000
    pos, vel, m, s2 = plummer(n, seed=7)
    with _ctx(prec, pos, vel, m, s2) as c:
        c.nbody_grav()
        got = c.get_particles()["grav"]
    ref = orc.direct_grav(pos, m, s2)
    err = np.abs(got - ref) / np.abs(ref)
    assert np.median(err) <= TOL_MEDIAN[prec]
    # self term kept (nbody.cu:108-113): a lone particle has phi = -m / sqrt(soft2)
    with _ctx(prec, pos[:1], vel[:1], m[:1], s2[:1]) as c:
        c.nbody_grav()
        g1 = c.get_particles()["grav"][0]
    assert abs(g1 - (-m[0] / np.sqrt(s2[0]))) <= 1e-6 * abs(g1)


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_two_softening_components(prec):
    # star + dark components with different softening and masses (the reference's two ICs)
    n1, n2 = 1500, 700
    p1, v1, m1, _ = plummer(n1, seed=1)
    p2, v2, m2, _ = plummer(n2, seed=2, mass=3.0, a=2.0)
    pos = np.vstack([p1, p2])
    vel = np.vstack([v1, v2])
    m = np.concatenate([m1, m2])
    s2 = np.concatenate([np.full(n1, 0.004 ** 2), np.full(n2, 0.05 ** 2)])
    with _ctx(prec, pos, vel, m, s2) as c:
        c.nbody_acceleration()
        got = c.get_particles()["acc"]
    err = rel_err(got, orc.direct_acc(pos, m, s2))
    assert np.median(err) <= TOL_MEDIAN[prec]


def test_zero_mass_particles_are_inert():
    pos, vel, m, s2 = plummer(600, seed=3)
    m[::3] = 0.0
    with _ctx("fp32", pos, vel, m, s2) as c:
        c.nbody_acceleration()
        got = c.get_particles()["acc"]
    keep = m > 0
    with _ctx("fp32", pos[keep], vel[keep], m[keep], s2[keep]) as c:
        c.nbody_acceleration()
        got2 = c.get_particles()["acc"]
    np.testing.assert_allclose(got[keep], got2, rtol=2e-5, atol=1e-6)


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_predict_correct_operators(prec):
    n = 777
    pos, vel, m, s2 = plummer(n, seed=4)
    dt = 1e-3
    with _ctx(prec, pos, vel, m, s2) as c:
        c.nbody_acceleration()
        a0 = c.get_particles()["acc"]
        c.predict_step(dt)
        c.nbody_acceleration()
        c.correct_step(dt)
        got = c.get_particles()
    # oracle from the same a0 (rounded as the device holds it)
    rp, vstar = orc.predict(pos, vel, a0, dt)
    ra = orc.direct_acc(rp, m, s2)
    rv = orc.correct(vel, vstar, ra, dt)
    tol = {"fp32": 1e-6, "mixed": 1e-6, "fp64": 1e-13}[prec]
    assert np.max(rel_err(got["pos"], rp)) <= tol
    assert np.median(rel_err(got["vel"], rv)) <= 10 * tol


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_ten_fused_steps_match_oracle(prec):
    """Plummer N=4096, eps=0.01, dt=1e-3 (the small direct-sum configuration), 10 steps."""
    n, dt = 4096, 1e-3
    pos, vel, m, s2 = plummer(n, seed=0)
    sim = rg.SimParams(time_max=1.0, dt_save=0.01, dt_dynamics=dt,
                       saves_without_dump=2 ** 63, use_wave_model=0)
    with _ctx(prec, pos, vel, m, s2) as c:
        c.solver_init(sim)
        c.precalc()
        c.calc_steps(10)
        got = c.get_particles()
        t, it = c.time()
    rp, rv, ra = orc.nbody_steps(pos, vel, orc.direct_acc(pos, m, s2), m, s2, dt, 10)
    assert it == 10 and abs(t - 10 * dt) < 1e-15
    assert np.median(rel_err(got["pos"], rp)) <= 1e-4
    assert np.max(rel_err(got["pos"], rp)) <= (1e-4 if prec != "fp64" else 1e-12)
    assert np.median(rel_err(got["vel"], rv)) <= 1e-4
    assert np.median(rel_err(got["acc"], ra)) <= TOL_MEDIAN[prec] * 10


def test_fused_steps_equal_operator_steps():
    n, dt = 2048, 1e-3
    pos, vel, m, s2 = plummer(n, seed=5)
    sim = rg.SimParams(time_max=1.0, dt_save=0.01, dt_dynamics=dt,
                       saves_without_dump=2 ** 63, use_wave_model=0)
    with _ctx("fp32", pos, vel, m, s2) as c:
        c.solver_init(sim)
        c.precalc()
        for _ in range(3):  # graph recorded once, then replayed
            c.calc_steps(4)
        fused = c.get_particles()
    with _ctx("fp32", pos, vel, m, s2) as c:
        c.nbody_acceleration()
        for _ in range(12):
            c.predict_step(dt)
            c.nbody_acceleration()
            c.correct_step(dt)
        ops = c.get_particles()
    np.testing.assert_allclose(fused["pos"], ops["pos"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(fused["vel"], ops["vel"], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_conservation_reductions(prec):
    n = 5000
    pos, vel, m, s2 = plummer(n, seed=6)
    with _ctx(prec, pos, vel, m, s2) as c:
        c.nbody_grav()
        cons = c.calc_conservation()
        com, mt = c.calc_mass_center()
        grav = c.get_particles()["grav"]
    if prec == "fp32":
        pos_r, vel_r, m_r = f32(pos), f32(vel), f32(m)
    else:
        pos_r, vel_r, m_r = pos, vel, m
    ref = orc.conservation(pos_r, vel_r, m_r, grav)
    assert abs(cons["Ek"] - ref["Ek"]) <= 1e-12 * abs(ref["Ek"])
    assert abs(cons["Ep"] - ref["Ep"]) <= 1e-12 * abs(ref["Ep"])
    np.testing.assert_allclose(cons["momentum"], ref["momentum"], rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(cons["angular"], ref["angular"], rtol=1e-9, atol=1e-15)
    rc, rm = orc.mass_center(pos_r, m_r)
    np.testing.assert_allclose(com, rc, rtol=1e-9, atol=1e-14)
    assert abs(mt - rm) <= 1e-12


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_conservation_sums_do_not_depend_on_particle_order(prec):
    """The reductions are double-double and round once, so the order of the particles in
    memory (which the cell sort changes) does not change a bit of the result."""
    n = 20000
    pos, vel, m, s2 = plummer(n, seed=9)
    m = m * np.linspace(0.5, 1.5, n)
    perm = np.random.default_rng(4).permutation(n)
    out = []
    for order in (np.arange(n), perm):
        with _ctx(prec, pos[order], vel[order], m[order], s2[order]) as c:
            out.append((c.calc_conservation(), c.calc_mass_center()))
    (a, (ca, ma)), (b, (cb, mb)) = out
    assert a["Ek"] == b["Ek"]
    np.testing.assert_array_equal(a["momentum"], b["momentum"])
    np.testing.assert_array_equal(a["angular"], b["angular"])
    np.testing.assert_array_equal(ca, cb)
    assert ma == mb


@pytest.mark.parametrize("memory", ["pageable", "pinned"])
def test_asynchronous_conservation_sums_equal_the_synchronous_ones(memory):
    """Pageable memory gets a copy; pinned memory the device can address gets the sums from
    the reduction kernel itself."""
    n = 3000
    pos, vel, m, s2 = plummer(n, seed=8)
    if memory == "pinned":
        torch = pytest.importorskip("torch")
        sums = torch.full((3, 12), float("nan"), dtype=torch.float64).pin_memory().numpy()
    else:
        sums = np.full((3, 12), np.nan)
    with _ctx("fp32", pos, vel, m, s2) as c:
        c.nbody_grav()
        ref = c.calc_conservation()
        for k in range(3):  # several in flight, the stream orders them
            c.calc_conservation_async(sums[k])
        c.synchronize()
    for k in range(3):
        got = rg.conservation_from_sums(sums[k])
        assert got["Ek"] == ref["Ek"] and got["Ep"] == ref["Ep"]
        np.testing.assert_array_equal(got["momentum"], ref["momentum"])
        np.testing.assert_array_equal(got["angular"], ref["angular"])


_VARIANT_SCRIPT = r"""
import json, sys
import numpy as np
sys.path[:0] = sys.argv[1:3]
import oracle as orc
import rrgsim_b200 as rg
from helpers import plummer, rel_err
out = {}
for n, uniform in ((1000, True), (20000, True), (5001, False)):
    pos, vel, m, s2 = plummer(n, seed=n)
    if not uniform:  # masses and softenings vary: the kernels without the uniform shortcuts
        m = m * np.linspace(0.5, 1.5, n)
        s2 = s2 * np.linspace(0.5, 2.0, n)
    c = rg.Context(0, "fp32")
    c.load_particles(pos, vel, m, s2)
    c.nbody_acceleration()
    acc = c.get_particles()["acc"]
    c.nbody_grav()
    grav = c.get_particles()["grav"]
    c.close()
    g = orc.direct_grav(pos, m, s2)
    out[f"{n}"] = [float(np.median(rel_err(acc, orc.direct_acc(pos, m, s2)))),
                   float(np.median(np.abs(grav - g) / np.abs(g)))]
print(json.dumps(out))
"""


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6, 7])
def test_every_fp32_kernel_variant_matches_oracle(variant):
    """Each FP32 direct-sum kernel (scalar with 1 or 2 i-particles per thread; paired over i
    with 2, 4 or 6; paired over j with 1 or 2), chosen by RRG_DIRECT_VARIANT, which is read once
    per process: accelerations and potentials at sizes with one and several j-splits, with
    uniform and with varying masses and softenings, against the FP64 oracle."""
    import json
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    env = dict(os.environ, RRG_DIRECT_VARIANT=str(variant))
    r = subprocess.run([sys.executable, "-c", _VARIANT_SCRIPT, here, os.path.dirname(here)],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    errs = json.loads(r.stdout.strip().splitlines()[-1])
    for n, (ea, eg) in errs.items():
        assert ea <= 1e-5 and eg <= 1e-5, (variant, n, ea, eg)


@pytest.mark.parametrize("n", [3000, 3001, 65537])
def test_raw_device_entry_points_match_context(n):
    # n = 3001 and 65537 (n % 4 != 0, several j-splits): the split partials must still start
    # on a 16-byte boundary behind the n-float potential
    torch = pytest.importorskip("torch")
    pos, vel, m, s2 = plummer(n, seed=8)
    posm = torch.tensor(np.hstack([pos, m[:, None]]), dtype=torch.float32, device="cuda")
    out = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rg.check(rg.lib().rrg_dev_direct_forces_f32(posm.data_ptr(), None, None,
                                                float(np.float32(0.5 * s2[0])), n,
                                                out.data_ptr(), 0, stream))
    torch.cuda.synchronize()
    o = out.cpu().numpy().astype(np.float64)
    assert np.median(rel_err(o[:, :3], orc.direct_acc(pos, m, s2))) <= 1e-5
    g = orc.direct_grav(pos, m, s2)
    assert np.median(np.abs(o[:, 3] - g) / np.abs(g)) <= 1e-5


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_precision_configuration_against_fp64_oracle(prec):
    """The precision configuration (bulge: Plummer M = 0.2, a = 0.2; disk: M = 0.8, Rd = 1;
    N = 65,536, soft2 = 1e-4): initial accelerations against the FP64 oracle's direct sum
    (nbody.cu:19-65), then 50 fused steps at dt = 1e-3, whose energy stays within 1e-6 of
    its start. MIXED sums tiles with Kahan compensation and keeps double-float positions."""
    from rrgsim_b200.bench_forms import _bulge_disk
    n, dt = 65536, 1e-3
    pos, vel, m, s2 = _bulge_disk(n)
    sim = rg.SimParams(time_max=10.0, dt_save=1.0, dt_dynamics=dt, saves_without_dump=0,
                       use_wave_model=0)
    with rg.Context(0, prec) as c:
        c.load_particles(pos, vel, m, s2)
        c.solver_init(sim)
        c.precalc()
        acc = c.get_particles()["acc"]
        e0 = c.calc_conservation()
        c.calc_steps(50)
        c.sync_particles_and_grid()
        e1 = c.calc_conservation()
    held = pos if prec == "mixed" else f32(pos)
    ref = orc.direct_acc(held, f32(m), s2)
    err = rel_err(acc, ref)
    print(f"\n{prec}: N = 65536 acceleration median rel err {np.median(err):.3e}, "
          f"p99 {np.percentile(err, 99):.3e}")
    assert np.median(err) <= 1e-6
    assert np.percentile(err, 99) <= 1e-5
    E0, E1 = e0["Ek"] + e0["Ep"], e1["Ek"] + e1["Ep"]
    assert abs(E1 / E0 - 1.0) <= 1e-6
