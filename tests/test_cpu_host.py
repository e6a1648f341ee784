"""CPU-only tests: the C-ABI library loads and exports every declared symbol, and the host
boundary (params.json, IC text, snapshot dumps, IC generators) behaves like the reference's."""
import ctypes as C
import json
import re
import struct
from pathlib import Path

import numpy as np
import pytest

import rrgsim_b200 as rg

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "rrg.h").read_text()
    return sorted(set(re.findall(r"RRG_API[^;(]*?\b(rrg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 40
    L = C.CDLL(str(rg.LIB_PATH))
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert rg.version().startswith("rrgsim-b200")


def test_no_gpu_calls_fail_cleanly_without_device():
    # creating a context is the first GPU call; on a CPU box it must fail with a status
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(rg.RRGError):
        rg.Context(0, "fp32")


SAMPLE = {
    "ini_params": {"mass_star": 1.0, "mass_dark": 1.0, "soft_star": 0.004, "soft_dark": 0.004,
                   "ini_file_star": "ini\\S.txt", "ini_file_dark": None},
    "sim_params": {"time_max": 1.0, "dt_save": 0.01, "dt_dynamics": 0.002,
                   "saves_without_dump": 10, "acceleration_model": "Wave"},
    "grid_params": {"nx": 512, "dx": 0.025, "bc_frac": 0.2},
    "wave_params": {"diss_base": 0.1, "diss_extra": 0.01, "wave_speed": 4574.337022617616,
                    "setup_iterations": 30000, "iterations": 3000, "tolerance": 1E-6,
                    "print_step": 500, "steady_check_step": 30, "steady_hold_steps": 3},
}


def test_parse_params_json_like_reference(tmp_path):
    p = tmp_path / "params.json"
    p.write_text(json.dumps(SAMPLE, indent=4))
    pp = rg.parse_params_json(p)
    assert pp.ini.ini_file_star == b"ini\\S.txt" and pp.ini.ini_file_dark == b""
    assert pp.sim.dt_dynamics == 0.002 and pp.sim.saves_without_dump == 10
    assert pp.has_grid and pp.has_wave and pp.sim.use_wave_model == 1
    # io_json.cpp:28-40
    assert pp.grid.nx == 512 and pp.grid.domain_l == 0.025 * 512
    assert pp.grid.domain_min == -0.5 * 0.025 * 512
    assert abs(pp.grid.sim_l - 0.8 * 12.8) < 1e-12
    assert abs(pp.grid.bc_l - 0.5 * 0.2 * 12.8) < 1e-12
    # io_json.cpp:178: dt = 0.5 dx / (c sqrt 3)
    assert pp.wave.dt == 0.5 * 0.025 / (4574.337022617616 * np.sqrt(3.0))


def test_parse_params_defaults_and_modes(tmp_path):
    d = json.loads(json.dumps(SAMPLE))
    del d["wave_params"]["setup_iterations"], d["wave_params"]["tolerance"]
    del d["sim_params"]["saves_without_dump"]
    p = tmp_path / "params.json"
    p.write_text(json.dumps(d))
    pp = rg.parse_params_json(p)
    assert pp.wave.setup_iterations == 30000 and pp.wave.tolerance == 1e-6
    assert pp.sim.saves_without_dump == 2 ** 64 - 1
    del d["wave_params"]
    p.write_text(json.dumps(d))
    pp = rg.parse_params_json(p)
    assert pp.has_grid and not pp.has_wave and pp.sim.use_wave_model == 0


@pytest.mark.parametrize("mutate", ["missing_sim", "missing_key", "bad_type", "bad_json",
                                    "missing_file"])
def test_parse_params_errors(tmp_path, mutate):
    d = json.loads(json.dumps(SAMPLE))
    p = tmp_path / "params.json"
    if mutate == "missing_sim":
        del d["sim_params"]
    elif mutate == "missing_key":
        del d["ini_params"]["mass_star"]
    elif mutate == "bad_type":
        d["sim_params"]["dt_dynamics"] = "fast"
    text = json.dumps(d)
    if mutate == "bad_json":
        text = text[:-5]
    if mutate != "missing_file":
        p.write_text(text)
    with pytest.raises(rg.RRGError) as e:
        rg.parse_params_json(p)
    assert e.value.status == 4


def test_ic_text_round_trip_and_cumulative_mass(tmp_path):
    rng = np.random.default_rng(0)
    pos, vel = rng.standard_normal((300, 3)), rng.standard_normal((300, 3))
    f = tmp_path / "S.txt"
    rg.write_ic_text(f, pos, vel)
    p2, v2, m, s2 = rg.read_ic(f, 2.0, 0.01)
    np.testing.assert_array_equal(p2, pos)
    np.testing.assert_array_equal(v2, vel)
    assert np.all(m == 2.0 / 300) and np.all(s2 == 0.01 * 0.01)
    # second component: mass divided by the cumulative count (io_particles_csv.cpp:37)
    _, _, m2, _ = rg.read_ic(f, 3.0, 0.02, n_before=100)
    assert np.all(m2 == 3.0 / 400)


def test_ic_errors(tmp_path):
    f = tmp_path / "bad.txt"
    f.write_text("3 0.0\n1 2 3 4 5 6\n1 2 3 4 5 6\n")
    with pytest.raises(rg.RRGError, match="mismatch"):
        rg.read_ic(f, 1.0, 0.01)
    f.write_text("2 0.0\n1 2 3 4 5\n1 2 3 4 5 6\n")
    with pytest.raises(rg.RRGError, match="fewer than 6"):
        rg.read_ic(f, 1.0, 0.01)
    f.write_text("abc\n")
    with pytest.raises(rg.RRGError, match="header"):
        rg.read_ic(f, 1.0, 0.01)


def test_dump_format_matches_reference(tmp_path):
    rng = np.random.default_rng(1)
    pos, vel = rng.standard_normal((5, 3)), rng.standard_normal((5, 3))
    rg.write_dump(tmp_path, 42, 0.084, pos, vel)
    f = tmp_path / "S_   42.bin"  # fmt "S_{:>5d}.bin" (io_particles_bin.cu:18)
    raw = f.read_bytes()
    assert len(raw) == 8 + 8 + 5 * 24 * 2
    n, t = struct.unpack("<Qd", raw[:16])
    assert n == 5 and t == 0.084
    body = np.frombuffer(raw[16:], dtype="<f8")
    np.testing.assert_array_equal(body[:15].reshape(5, 3), pos)
    np.testing.assert_array_equal(body[15:].reshape(5, 3), vel)
    t2, p2, v2 = rg.read_dump(f)
    assert t2 == 0.084
    np.testing.assert_array_equal(p2, pos)
    with pytest.raises(rg.RRGError):
        rg.write_dump(tmp_path / "no" / "such" / "dir", 1, 0.0, pos, vel)


def test_generators_deterministic_and_shaped():
    p1, v1 = rg.generate_plummer(0, 4096)
    p2, v2 = rg.generate_plummer(0, 4096)
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(v1, v2)
    r = np.linalg.norm(p1, axis=1)
    assert r.max() <= 20.0
    # half-mass radius of a Plummer sphere: a / sqrt(2^(2/3) - 1) ~ 1.305 a
    assert abs(np.median(r) - 1.305) < 0.06
    # virial equilibrium: 2 T ~ |W| = 3 pi / 32 for M = a = 1
    T = 0.5 * np.mean(np.sum(v1 * v1, axis=1))
    assert abs(2 * T - 3 * np.pi / 32) < 0.03
    pd, vd = rg.generate_exp_disk(1, 20000)
    R = np.hypot(pd[:, 0], pd[:, 1])
    assert R.max() <= 7.5 and np.abs(pd[:, 2]).max() < 7.5
    # median radius of an exponential disk: 1.678 Rd
    assert abs(np.median(R) - 1.678) < 0.05
    assert abs(np.median(np.abs(pd[:, 2])) - 0.1 * np.arctanh(0.5)) < 0.01


def test_oracle_disk_generator_gives_the_library_bits():
    """The timed CPU arm of the benchmark makes its inputs with the oracle's restatement of the
    disk generator (so it loads nothing of the product): the same bits for the same seed."""
    import oracle as orc
    for seed, n in ((1, 30000), (7, 1000)):
        po, vo = orc.exp_disk(seed, n, 1.0, 1.0, 0.1, 7.5, 7.5, 0.1)
        pl, vl = rg.generate_exp_disk(seed, n, 1.0, 1.0, 0.1, 7.5, 7.5, 0.1)
        np.testing.assert_array_equal(po, pl)
        np.testing.assert_array_equal(vo, vl)


@pytest.mark.parametrize("fault", ["no_params", "bad_json", "missing_ic", "truncated_ic",
                                   "short_row"])
def test_rrgsim_executable_reports_host_faults(tmp_path, fault):
    """Failures on the host side end the run with exit code 1 and a message, before any GPU
    work (the reference logs them and exits 0)."""
    import subprocess
    rng = np.random.default_rng(0)
    pos, vel = rng.standard_normal((8, 3)), rng.standard_normal((8, 3))
    (tmp_path / "ini").mkdir()
    rg.write_ic_text(tmp_path / "ini" / "S.txt", pos, vel)
    d = json.loads(json.dumps(SAMPLE))
    d.pop("grid_params")
    d.pop("wave_params")
    if fault == "missing_ic":
        d["ini_params"]["ini_file_star"] = "ini/none.txt"
    if fault == "truncated_ic":
        lines = (tmp_path / "ini" / "S.txt").read_text().splitlines()
        (tmp_path / "ini" / "S.txt").write_text("\n".join(lines[:5]) + "\n")
    if fault == "short_row":
        lines = (tmp_path / "ini" / "S.txt").read_text().splitlines()
        lines[3] = "1 2 3"
        (tmp_path / "ini" / "S.txt").write_text("\n".join(lines) + "\n")
    if fault != "no_params":
        text = json.dumps(d)
        (tmp_path / "params.json").write_text(text[:-3] if fault == "bad_json" else text)
    r = subprocess.run([str(rg.BIN_PATH), str(tmp_path)], capture_output=True, text=True,
                       env={"RRGSIM_QUIET": "1", "PATH": "/usr/bin:/bin"}, timeout=120)
    assert r.returncode == 1
    assert "rrgsim:" in r.stderr
    assert not (tmp_path / "dump").exists()
