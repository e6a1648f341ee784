"""Batched ensemble of galaxies: one persistent force launch over a work-list must give each
galaxy the same trajectory as stepping it alone, and match the FP64 oracle."""
import numpy as np
import pytest

import oracle as orc
import rrgsim_b200 as rg
from helpers import rel_err

pytestmark = pytest.mark.gpu


def _small_ensemble():
    return rg.make_ensemble(ngal=9, nmin=256, nmax=6000, seed=5)


@pytest.mark.parametrize("autotune", [False, True])
def test_ensemble_matches_single_galaxy_contexts_and_oracle(autotune):
    counts, pos, vel, mass, s2 = _small_ensemble()
    dt, steps = 1e-3, 7
    with rg.Ensemble(counts, pos, vel, mass, s2, dt, autotune=autotune) as e:
        a0 = e.get()["acc"]
        e.step(3)
        e.step(4)
        got = e.get()
        tune = e.tuning()
    assert tune["items"] >= len(counts)
    off = np.concatenate([[0], np.cumsum(counts)])
    sim = rg.SimParams(time_max=1.0, dt_save=1.0, dt_dynamics=dt, saves_without_dump=0,
                       use_wave_model=0)
    for g in range(len(counts)):
        sl = slice(off[g], off[g + 1])
        soft2 = np.full(counts[g], s2[g])
        ra0 = orc.direct_acc(pos[sl], mass[sl], soft2)
        assert np.median(rel_err(a0[sl], ra0)) <= 1e-5
        with rg.Context(0, "fp32") as c:
            c.load_particles(pos[sl], vel[sl], mass[sl], soft2)
            c.solver_init(sim)
            c.precalc()
            c.calc_steps(steps)
            one = c.get_particles()
        np.testing.assert_allclose(got["pos"][sl], one["pos"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(got["vel"][sl], one["vel"], rtol=1e-4, atol=1e-5)
        rp, rv, ra = orc.nbody_steps(pos[sl], vel[sl], ra0, mass[sl], soft2, dt, steps)
        assert np.median(rel_err(got["pos"][sl], rp)) <= 1e-5
        assert np.median(rel_err(got["acc"][sl], ra)) <= 1e-4


@pytest.mark.parametrize("plain", [False, True])
def test_sequential_baseline_gives_the_same_state(plain):
    counts, pos, vel, mass, s2 = _small_ensemble()
    out = []
    for seq in (False, True):
        with rg.Ensemble(counts, pos, vel, mass, s2, 1e-3, autotune=False) as e:
            if seq:
                e.step_sequential(5, plain=plain)
            else:
                e.step(5)
            out.append(e.get())
    np.testing.assert_allclose(out[0]["pos"], out[1]["pos"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(out[0]["vel"], out[1]["vel"], rtol=1e-4, atol=1e-5)


def test_ensemble_rejects_bad_input():
    counts, pos, vel, mass, s2 = _small_ensemble()
    bad = pos.copy()
    bad[3, 1] = np.nan
    with pytest.raises(rg.RRGError):
        rg.Ensemble(counts, bad, vel, mass, s2, 1e-3)
    with pytest.raises(rg.RRGError):
        rg.Ensemble(counts, pos, vel, mass, s2, -1.0)
