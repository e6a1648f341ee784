"""Measurements of the secondary forms of the hot path (one JSON line per form).

    python -m rrgsim_b200.bench_forms [plummer|precision|ensemble|adjoint|adjoint_pm|vjp|all]

plummer   : Plummer N = 4096, eps = 0.01, dt = 1e-3, 100 steps, a snapshot every 10 steps.
precision : bulge (Plummer M = 0.2, a = 0.2) + disk (M = 0.8, Rd = 1), N = 65,536 direct sum over
            1000 steps at dt = 1e-3 in FP32, MIXED and FP64 (the FP64 run is the error
            reference: the library's FP64 path, held to the host oracle by the tests), plus
            8,388,608 disk particles through the int64 CIC deposit on 256^3.
ensemble  : 64 galaxies, N log-uniform in [1024, 65536] (seed 3), 500 steps batched vs one
            launch per galaxy.
adjoint   : gradient of the mean squared final-position error through 200 leapfrog steps
            (N = 16,384 Plummer, eps = 0.02, dt = 1e-3, checkpoints every 20 steps) vs the
            forward pass.
adjoint_pm: the same through the particle-mesh step (N = 262,144 disk, 64^3, 20 substeps).
vjp       : one force vector-Jacobian product vs one force evaluation, N = 16,384 and 65,536.
All inputs are synthetic (the reference ships no benchmark data). Times are CUDA events on
the stream the library launches on.
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np

import rrgsim_b200 as rg


def _events(torch, stream):
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    return a, b


def _fp32_peak_tflops():
    return 148 * 128 * 2 * 1965e6 / 1e12


def form_plummer(torch):
    n, dt = 4096, 1e-3
    pos, vel = rg.generate_plummer(0, n, 1.0, 1.0, 20.0)
    m, s2 = np.full(n, 1.0 / n), np.full(n, 1e-4)
    sim = rg.SimParams(time_max=0.1, dt_save=0.01, dt_dynamics=dt, saves_without_dump=11,
                       use_wave_model=0)
    s = torch.cuda.Stream()
    out = {}
    for prec in ("fp32", "fp64"):
        with rg.Context(0, prec) as c:
            c.set_stream(s.cuda_stream)
            c.load_particles(pos, vel, m, s2)
            c.solver_init(sim)
            c.precalc()
            c.calc_steps(10)  # warm-up: records the graph
            c.load_particles(pos, vel, m, s2)
            c.precalc()
            c.synchronize()
            a, b = _events(torch, s)
            t0 = time.perf_counter()
            a.record(s)
            snaps = []
            for _ in range(10):
                c.calc_steps(10)
                snaps.append(c.get_particles()["pos"])  # the snapshot download
            b.record(s)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            out[prec] = {"ms_total_device": a.elapsed_time(b), "wall_s": wall,
                         "final_pos": snaps[-1], "pos10": snaps[0]}
    steps = 100
    ms = out["fp32"]["ms_total_device"]
    err10 = np.linalg.norm(out["fp32"]["pos10"] - out["fp64"]["pos10"], axis=1) / \
        np.linalg.norm(out["fp64"]["pos10"], axis=1)
    return {"form": "plummer_4096", "steps": steps, "snapshots": 10,
            "ms_per_step_incl_snapshots": ms / steps,
            "gpairs_per_s_incl_snapshots": n * n * steps / (ms * 1e-3) / 1e9,
            "wall_s": out["fp32"]["wall_s"],
            "pos_rel_err_after_10_steps_vs_fp64": {"median": float(np.median(err10)),
                                                    "max": float(np.max(err10))}}


def _bulge_disk(n):
    nb = n // 5
    pb, vb = rg.generate_plummer(7, nb, 0.2, 0.2, 4.0)
    pd, vd = rg.generate_exp_disk(8, n - nb, 0.8, 1.0, 0.1, 7.5, 7.5, 0.1, 0.2, 0.2)
    pos, vel = np.vstack([pb, pd]), np.vstack([vb, vd])
    return pos, vel, np.full(n, 1.0 / n), np.full(n, 1e-4)


def form_precision(torch, steps=1000):
    n, dt = 65536, 1e-3
    pos, vel, m, s2 = _bulge_disk(n)
    sim = rg.SimParams(time_max=10.0, dt_save=1.0, dt_dynamics=dt, saves_without_dump=0,
                       use_wave_model=0)
    s = torch.cuda.Stream()
    res = {}
    for prec in ("fp64", "fp32", "mixed"):
        with rg.Context(0, prec) as c:
            c.set_stream(s.cuda_stream)
            c.load_particles(pos, vel, m, s2)
            c.solver_init(sim)
            c.precalc()
            st0 = c.get_particles()
            e0 = c.calc_conservation()
            E0 = e0["Ek"] + e0["Ep"]
            c.calc_steps(10)
            p10 = c.get_particles()["pos"]
            a, b = _events(torch, s)
            a.record(s)
            c.calc_steps(steps - 10)
            b.record(s)
            torch.cuda.synchronize()
            c.sync_particles_and_grid()
            e1 = c.calc_conservation()
            res[prec] = {"acc0": st0["acc"], "p10": p10, "ms_per_step": a.elapsed_time(b) / (steps - 10),
                         "E_drift": (e1["Ek"] + e1["Ep"]) / E0 - 1.0}
    ref = res["fp64"]
    out = {"form": "precision_bulge_disk_65536", "steps": steps, "dt": dt}
    for prec in ("fp32", "mixed", "fp64"):
        r = res[prec]
        ea = np.linalg.norm(r["acc0"] - ref["acc0"], axis=1) / np.linalg.norm(ref["acc0"], axis=1)
        ep = np.linalg.norm(r["p10"] - ref["p10"], axis=1) / np.linalg.norm(ref["p10"], axis=1)
        out[prec] = {"acc_rel_err_median": float(np.median(ea)), "acc_rel_err_p99": float(np.percentile(ea, 99)),
                     "pos10_rel_err_median": float(np.median(ep)),
                     "energy_drift_after_steps": float(r["E_drift"]),
                     "gpairs_per_s": n * n / (r["ms_per_step"] * 1e-3) / 1e9}
    # int64 fixed-point CIC of 8,388,608 disk particles on 256^3 (+-8 Rd)
    nd, nx = 8388608, 256
    pd, vd = rg.generate_exp_disk(9, nd, 1.0, 1.0, 0.1, 7.5, 7.5, 0.1, 0.0, 0.0)
    md = np.full(nd, 1.0 / nd)
    grid = rg.GridInfo.from_values(nx, 16.0 / nx, 0.0)
    masses = []
    with rg.Context(0, "fp32") as c:
        c.set_stream(s.cuda_stream)
        c.load_particles(pd, vd, md, np.full(nd, 1e-4))
        c.init_grid(grid)
        c.convert_particles_to_grid()
        c.synchronize()
        a, b = _events(torch, s)
        a.record(s)
        for _ in range(5):
            c.convert_particles_to_grid()
        b.record(s)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / 5
        masses.append(c.get_grid()["mass"])
        c.convert_particles_to_grid()
        masses.append(c.get_grid()["mass"])
        shift = c.deposit_scale()
    out["cic_8M_256"] = {"particles": nd, "grid": nx, "ms_per_deposit": ms,
                         "particles_per_s": nd / (ms * 1e-3),
                         "run_to_run_bit_identical": bool(np.array_equal(masses[0], masses[1])),
                         "mass_sum_error": float(abs(masses[0].sum() - 1.0)),
                         "fixed_point_shift": shift}
    return out


def form_ensemble(torch, steps=500):
    counts, pos, vel, mass, s2 = rg.make_ensemble()
    pairs = float((counts.astype(np.float64) ** 2).sum())
    s = torch.cuda.Stream()
    res = {}
    for mode in ("batched", "sequential", "sequential_plain"):
        with rg.Ensemble(counts, pos, vel, mass, s2, 1e-3, autotune=(mode == "batched")) as e:
            e.set_stream(s.cuda_stream)
            if mode == "batched":
                run = e.step
            elif mode == "sequential":
                run = e.step_sequential
            else:
                run = lambda k: e.step_sequential(k, plain=True)  # noqa: E731
            k = steps if mode == "batched" else 20
            run(2)
            e.synchronize()
            a, b = _events(torch, s)
            a.record(s)
            run(k)
            b.record(s)
            torch.cuda.synchronize()
            res[mode] = {"ms_per_step": a.elapsed_time(b) / k, "steps_timed": k}
            if mode == "batched":
                res[mode]["tuning"] = e.tuning()
    b_ms, s_ms = res["batched"]["ms_per_step"], res["sequential"]["ms_per_step"]
    p_ms = res["sequential_plain"]["ms_per_step"]
    return {"form": "ensemble_64", "galaxies": len(counts), "particles": int(counts.sum()),
            "pairs_per_step": pairs, "batched_ms_per_step": b_ms,
            "sequential_ms_per_step": s_ms, "speedup_vs_sequential": s_ms / b_ms,
            "sequential_plain_ms_per_step": p_ms,
            "speedup_vs_plain_per_galaxy_launches": p_ms / b_ms,
            "batched_gpairs_per_s": pairs / (b_ms * 1e-3) / 1e9,
            "frac_fp32_peak": pairs / (b_ms * 1e-3) * 20 / 1e12 / _fp32_peak_tflops(),
            "tuning": res["batched"]["tuning"]}


def bench_line_forms(torch, precision_steps=1000, ensemble_steps=50):
    """The secondary forms in brief, for the benchmark's JSON line (about half a minute):
    c3: the bulge + disk N = 65,536 in FP32, MIXED and FP64 (initial accelerations returned as
        arrays for the caller's error check; energy drift over `precision_steps` steps);
    c4: the 64-galaxy ensemble batched against 64 sequential launches;
    c5: adjoint / forward wall time, N-body and particle mesh (no finite differences)."""
    from . import adjoint
    t0 = time.perf_counter()
    n, dt = 65536, 1e-3
    pos, vel, m, s2 = _bulge_disk(n)
    sim = rg.SimParams(time_max=10.0, dt_save=1.0, dt_dynamics=dt, saves_without_dump=0,
                       use_wave_model=0)
    s = torch.cuda.Stream()
    c3 = {"particles": n, "steps": precision_steps, "dt": dt, "acc0": {}}
    for prec in ("fp32", "mixed", "fp64"):
        with rg.Context(0, prec) as c:
            c.set_stream(s.cuda_stream)
            c.load_particles(pos, vel, m, s2)
            c.solver_init(sim)
            c.precalc()
            c3["acc0"][prec] = c.get_particles()["acc"]
            if prec == "fp64":
                continue
            e0 = c.calc_conservation()
            a, b = _events(torch, s)
            c.prepare_steps(precision_steps)
            a.record(s)
            c.calc_steps(precision_steps)
            b.record(s)
            torch.cuda.synchronize()
            c.sync_particles_and_grid()
            e1 = c.calc_conservation()
            c3[prec] = {"energy_drift": (e1["Ek"] + e1["Ep"]) / (e0["Ek"] + e0["Ep"]) - 1.0,
                        "gpairs_per_s": n * n * precision_steps /
                        (a.elapsed_time(b) * 1e-3) / 1e9}
    c3["inputs"] = (pos, m, s2)
    c4 = form_ensemble(torch, steps=ensemble_steps)
    c4.pop("tuning", None)
    an = adjoint.bench_form(fd_dirs=0)
    ap = adjoint.bench_form_pm(fd_dirs=0)
    c5 = {"nbody_16384_200_steps": {p: an[p]["backward_over_forward"] for p in ("fp32", "fp64")},
          "pm_262144_64_200_steps": {p: ap[p]["backward_over_forward"] for p in ("fp32", "fp64")},
          "target": "<= 3"}
    return {"precision_c3": c3, "ensemble_c4": c4, "adjoint_c5": c5,
            "seconds": time.perf_counter() - t0}


def main(argv):
    import torch
    which = argv[1] if len(argv) > 1 else "all"
    forms = {"plummer": form_plummer, "precision": form_precision, "ensemble": form_ensemble}
    try:
        from rrgsim_b200 import adjoint
        forms["adjoint"] = adjoint.bench_form
        forms["adjoint_pm"] = adjoint.bench_form_pm
        forms["vjp"] = adjoint.bench_form_vjp
    except ImportError:
        pass
    for name, f in forms.items():
        if which in ("all", name):
            print(json.dumps(f(torch)), flush=True)


if __name__ == "__main__":
    main(sys.argv)
