"""The `rrgsim <work_dir>` executable end to end: params.json + IC text in, snapshot dumps and
CSV tables out (solver/app/src/rrgsim.cu:12-62, rrgsim_integration.cu:19-146)."""
import json
import struct
import subprocess

import numpy as np
import pytest

import oracle as orc
import rrgsim_b200 as rg
from helpers import disk, f32, plummer, rel_err

pytestmark = pytest.mark.gpu


def _write_case(tmp_path, pos, vel, sim, grid=None, wave=None, soft=0.01):
    (tmp_path / "ini").mkdir()
    rg.write_ic_text(tmp_path / "ini" / "S.txt", pos, vel)
    params = {
        "ini_params": {"mass_star": 1.0, "mass_dark": 1.0, "soft_star": soft,
                       "soft_dark": soft, "ini_file_star": "ini\\S.txt", "ini_file_dark": None},
        "sim_params": sim,
    }
    if grid:
        params["grid_params"] = grid
    if wave:
        params["wave_params"] = wave
    (tmp_path / "params.json").write_text(json.dumps(params, indent=2))


def _run(tmp_path, precision="fp32", extra=()):
    r = subprocess.run([str(rg.BIN_PATH), str(tmp_path), *extra], capture_output=True, text=True,
                       env={"RRGSIM_QUIET": "1", "RRGSIM_PRECISION": precision,
                            "PATH": "/usr/bin:/bin"}, timeout=600)
    assert r.returncode == 0, r.stderr
    return r


def _read_dump(path):
    raw = path.read_bytes()
    n, t = struct.unpack("<Qd", raw[:16])
    body = np.frombuffer(raw[16:], dtype="<f8")
    return t, body[:3 * n].reshape(n, 3), body[3 * n:].reshape(n, 3)


def test_rrgsim_nbody_dumps_match_oracle(tmp_path):
    n, dt = 512, 1e-3
    pos, vel, m, s2 = plummer(n, seed=21)
    _write_case(tmp_path, pos, vel, {"time_max": 0.02, "dt_save": 0.005, "dt_dynamics": dt,
                                     "saves_without_dump": 3})
    _run(tmp_path)
    dumps = sorted(p.name for p in (tmp_path / "dump").iterdir() if p.name.startswith("S_"))
    # saves at iterations 5, 10, 15, 20; dumps while the save counter is below 3
    assert dumps == ["S_    5.bin", "S_   10.bin"]
    acc = orc.direct_acc(pos, m, s2)
    p, v = pos, vel
    done = 0
    for it, name in [(5, "S_    5.bin"), (10, "S_   10.bin")]:
        p, v, acc = orc.nbody_steps(p, v, acc, m, s2, dt, it - done)
        done = it
        t, dp, dv = _read_dump(tmp_path / "dump" / name)
        assert abs(t - it * dt) < 1e-12
        assert np.max(rel_err(dp, p)) <= 1e-5
        assert np.median(rel_err(dv, v)) <= 1e-5
    # conservation tables: header once, one row per save
    rows = (tmp_path / "data" / "delta_energy.csv").read_text().splitlines()
    assert rows[0] == "t, E, E_rel_signed, E_rel, Ek, Ep"
    assert len(rows) == 1 + 4
    e_rel = np.array([float(r.split(",")[3]) for r in rows[1:]])
    assert np.all(e_rel < 1e-3)
    for tab in ("delta_momentum", "delta_ang_z", "delta_ang_norm", "sample_particle"):
        assert (tmp_path / "data" / f"{tab}.csv").exists()
    assert any((tmp_path / "logs").iterdir())


def _table(path):
    rows = path.read_text().splitlines()
    head = [h.strip() for h in rows[0].split(",")]
    vals = np.array([[float(x) for x in r.split(",")] for r in rows[1:]])
    return head, vals


def test_rrgsim_tables_follow_the_reference_formulas(tmp_path):
    """The conservation and sample tables (print_conservation, print_sample_particle:
    rrgsim_conservation.cu:9-98, 334-359) recomputed from the dumped snapshots with the FP64
    oracle: E = Ek + Ep with Ep = sum m phi / 2, |P|, L_z and |L|, each with its relative change
    against the start; the sample row is particle 0."""
    n, dt = 512, 1e-3
    pos, vel, m, s2 = plummer(n, seed=23)
    _write_case(tmp_path, pos, vel, {"time_max": 0.02, "dt_save": 0.005, "dt_dynamics": dt,
                                     "saves_without_dump": 3})
    _run(tmp_path)
    data = tmp_path / "data"

    def cons(p, v):
        c = orc.conservation(p, v, m, orc.direct_grav(p, m, s2))
        L = c["angular"]
        return {"E": c["Ek"] + c["Ep"], "Ek": c["Ek"], "Ep": c["Ep"],
                "P": np.linalg.norm(c["momentum"]), "Lz": L[2], "L": np.linalg.norm(L)}

    c0 = cons(f32(pos), f32(vel))
    he, te = _table(data / "delta_energy.csv")
    hp, tp = _table(data / "delta_momentum.csv")
    hz, tz = _table(data / "delta_ang_z.csv")
    hn, tn = _table(data / "delta_ang_norm.csv")
    hs, ts = _table(data / "sample_particle.csv")
    assert hp == ["t", "momentum_norm", "momentum_diff", "momentum_rel_signed", "momentum_rel"]
    assert hz == ["t", "ang_z", "ang_z_rel_signed", "ang_z_rel"]
    assert hn == ["t", "ang_norm", "ang_norm_rel_signed", "ang_norm_rel"]
    assert hs == ["i", "x", "y", "z", "vx", "vy", "vz", "grav", "ax", "ay", "az"]
    assert len(ts) == 1 + 4  # the start, then every save
    for row, name in ((0, "S_    5.bin"), (1, "S_   10.bin")):
        t, dp, dv = _read_dump(tmp_path / "dump" / name)
        c = cons(dp, dv)
        e_rel = c["E"] / c0["E"] - 1
        assert abs(te[row, 0] - t) < 1e-8
        np.testing.assert_allclose(te[row, [1, 4, 5]], [c["E"], c["Ek"], c["Ep"]], rtol=1e-5)
        assert abs(te[row, 2] - e_rel) < 5e-6 and abs(te[row, 3] - abs(e_rel)) < 5e-6
        p_rel = c["P"] / c0["P"] - 1
        np.testing.assert_allclose(tp[row, 1], c["P"], rtol=1e-9)
        np.testing.assert_allclose(tp[row, 2], c["P"] - c0["P"], atol=1e-12)
        assert abs(tp[row, 3] - p_rel) < 1e-8 and abs(tp[row, 4] - abs(p_rel)) < 1e-8
        lz_rel = c["Lz"] / c0["Lz"] - 1
        np.testing.assert_allclose(tz[row, 1], c["Lz"], rtol=1e-9)
        assert abs(tz[row, 2] - lz_rel) < 1e-8 and abs(tz[row, 3] - abs(lz_rel)) < 1e-8
        ln_rel = c["L"] / c0["L"] - 1
        np.testing.assert_allclose(tn[row, 1], c["L"], rtol=1e-9)
        assert abs(tn[row, 2] - ln_rel) < 1e-8
        # sample particle: index 0 at this save, 8 decimals
        s = ts[row + 1]
        assert s[0] == 0
        np.testing.assert_allclose(s[1:4], dp[0], atol=1e-8)
        np.testing.assert_allclose(s[4:7], dv[0], atol=1e-8)
        np.testing.assert_allclose(s[7], orc.direct_grav(dp, m, s2)[0], rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(s[8:11], orc.direct_acc(dp, m, s2)[0], rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(ts[0, 1:4], f32(pos)[0], atol=1e-8)
    np.testing.assert_allclose(ts[0, 4:7], f32(vel)[0], atol=1e-8)


def test_rrgsim_wave_mode_runs_and_matches_library(tmp_path):
    n, nx, dt = 4096, 16, 2e-3
    pos, vel, m, s2 = disk(n, seed=22)
    c = 10.0 * float(np.max(np.linalg.norm(vel, axis=1)))
    dx = 1.0
    wave = {"diss_base": 1.0 / (4 * dx), "diss_extra": 0.0, "wave_speed": c,
            "setup_iterations": 300, "iterations": 20, "steady_check_step": 1000}
    _write_case(tmp_path, pos, vel,
                {"time_max": 0.01, "dt_save": 0.004, "dt_dynamics": dt, "saves_without_dump": 5},
                grid={"nx": nx, "dx": dx, "bc_frac": 0.2}, wave=wave, soft=0.01)
    _run(tmp_path)
    names = sorted(p.name for p in (tmp_path / "dump").iterdir())
    # snapshots, the wave levels beside them, the base conservation
    assert names == ["C0.bin", "S_    2.bin", "S_    4.bin", "W_    2.bin", "W_    4.bin"]
    # same run through the library API
    grid = rg.GridInfo.from_values(nx, dx, 0.2)
    wp = rg.WaveParams.make(dx, diss_base=wave["diss_base"], wave_speed=c, iterations=20,
                            setup_iterations=300, steady_check_step=1000)
    sim = rg.SimParams(time_max=0.01, dt_save=0.004, dt_dynamics=dt, saves_without_dump=5,
                       use_wave_model=1)
    with rg.Context(0, "fp32") as ctx:
        ctx.load_particles(pos, vel, m, s2)
        ctx.init_grid(grid)
        ctx.set_wave_params(wp)
        ctx.solver_init(sim)
        ctx.precalc()
        ctx.sync_particles_and_grid()
        ctx.calc_steps(2)
        s = ctx.get_particles()
        gr = ctx.get_grid()
    t, dp, dv = _read_dump(tmp_path / "dump" / "S_    2.bin")
    np.testing.assert_array_equal(dp, s["pos"])
    np.testing.assert_array_equal(dv, s["vel"])
    for sub in ("a_grid", "grav_grid", "mass_grid"):
        assert any((tmp_path / "data" / sub).iterdir())
    # the axis profiles through the centre at t = 2 dt (print_acc_projection and friends,
    # rrgsim_conservation.cu:360-424), 8 decimals, against the library's grid at that step
    h = nx // 2
    at = lambda x, y, z: x + y * nx + z * nx * nx  # noqa: E731
    xs = -0.5 * nx * dx + dx * np.arange(nx)
    ha, ta = _table(tmp_path / "data" / "a_grid" / "a_grid_center_0.00400000.csv")
    assert ha == ["x", "ax", "ay", "az"]
    np.testing.assert_allclose(ta[:, 0], xs, atol=1e-8)
    np.testing.assert_allclose(ta[:, 1:], gr["acc"][[at(i, h, h) for i in range(nx)]], atol=1e-8)
    hg, tg = _table(tmp_path / "data" / "grav_grid" / "grav_axis_center_0.0040000000.csv")
    assert hg == ["r", "gx", "gy", "gz"]
    for col, idx in ((1, [at(i, h, h) for i in range(nx)]), (2, [at(h, i, h) for i in range(nx)]),
                     (3, [at(h, h, i) for i in range(nx)])):
        np.testing.assert_allclose(tg[:, col], gr["grav"][idx], atol=1e-8)
    hm, tm = _table(tmp_path / "data" / "mass_grid" / "mass_axis_center_0.0040000000.csv")
    assert hm == ["r", "mx", "my", "mz"]
    np.testing.assert_allclose(tm[:, 1], gr["mass"][[at(i, h, h) for i in range(nx)]], atol=1e-8)


@pytest.mark.parametrize("mode,precision", [("nbody", "fp32"), ("wave", "fp32"),
                                            ("wave", "mixed")])
def test_resume_from_dump_continues_bit_exactly(tmp_path, mode, precision):
    """A run to t = 0.0161 and a run to t = 0.0081 resumed from its iteration-4 dump with
    `--resume 4` produce the same later snapshots, wave levels and conservation tables."""
    dt = 2e-3
    if mode == "nbody":
        pos, vel, _, _ = plummer(1024, seed=31)
        extra = {}
    else:
        pos, vel, _, _ = disk(8192, seed=32)
        c = 10.0 * float(np.max(np.linalg.norm(vel, axis=1)))
        extra = {"grid": {"nx": 16, "dx": 1.0, "bc_frac": 0.2},
                 "wave": {"diss_base": 0.25, "diss_extra": 0.0, "wave_speed": c,
                          "setup_iterations": 300, "iterations": 20,
                          "steady_check_step": 1000}}
    sim = {"dt_save": 0.004, "dt_dynamics": dt, "saves_without_dump": 100}
    full, part = tmp_path / "full", tmp_path / "part"
    full.mkdir()
    part.mkdir()
    _write_case(full, pos, vel, dict(sim, time_max=0.0161), **extra)
    _run(full, precision)
    _write_case(part, pos, vel, dict(sim, time_max=0.0081), **extra)
    _run(part, precision)
    assert not (part / "dump" / "S_    6.bin").exists()
    (part / "params.json").write_text((full / "params.json").read_text())
    _run(part, precision, extra=("--resume", "4"))
    for it in (6, 8):
        a = (full / "dump" / f"S_    {it}.bin").read_bytes()
        b = (part / "dump" / f"S_    {it}.bin").read_bytes()
        assert a == b, f"snapshot {it} differs"
        if mode == "wave":
            assert (full / "dump" / f"W_    {it}.bin").read_bytes() == \
                (part / "dump" / f"W_    {it}.bin").read_bytes()
    for tab in ("delta_energy", "delta_momentum", "delta_ang_z"):
        assert (full / "data" / f"{tab}.csv").read_text() == \
            (part / "data" / f"{tab}.csv").read_text(), tab
