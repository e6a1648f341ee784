#!/usr/bin/env python
"""Times the reference's own CUDA build (oracle/_ref/librrgref.so) on this GPU — TEST
INFRASTRUCTURE, run by hand for the comparison tables (not by bench.py).

Drives the reference's RectWave and NBody integration strategies exactly as integrate() does,
on the same synthetic workloads as the benchmark, and prints one JSON line:
  pm:     N = 2^20 exponential disk, 128^3 periodic wave grid, 20 substeps, dt = 2e-3
  nbody:  Plummer N = 4096 and N = 65,536, eps = 0.01, dt = 1e-3
The relaxation before the timed PM steps is cut short (a step costs the same either way).
"""
from __future__ import annotations

import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import rrgsim_b200 as rg  # noqa: E402  (host-side IC generators only)
from oracle import ref_lib as load_ref  # noqa: E402

d = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(d)


def time_pm(L, steps: int = 10):
    n, nx = 1 << 20, 128
    pos, vel = rg.generate_exp_disk(1, n, 1.0, 1.0, 0.1, 7.5, 7.5, 0.1, 0.0, 0.0)
    mass, soft2 = np.full(n, 1.0 / n), np.full(n, 1e-4)
    dx = 16.0 / nx
    c = 10.0 * float(np.max(np.linalg.norm(vel, axis=1)))
    wave = np.array([1.0 / (4 * dx), 0.0, c, 200, 20, 1e-6, 500, 30, 3], dtype=np.float64)
    outs = [np.empty(nx ** 3), np.empty(nx ** 3), np.empty((n, 3)), np.empty(n),
            np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3)), np.empty(nx ** 3)]
    ms = C.c_double()
    rc = L.ref_pm(n, _p(pos), _p(vel), _p(mass), _p(soft2), nx, dx, 0.0, _p(wave), 2e-3, steps,
                  *[_p(o) for o in outs], C.byref(ms))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    return {"particles": n, "grid": nx, "substeps": 20, "steps": steps,
            "ms_per_step": ms.value, "particle_steps_per_s": n / (ms.value * 1e-3)}


def time_nbody(L, n: int, steps: int):
    pos, vel = rg.generate_plummer(0, n, 1.0, 1.0, 20.0)
    mass, soft2 = np.full(n, 1.0 / n), np.full(n, 1e-4)
    outs = [np.empty((n, 3)), np.empty(n), np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))]
    ms = C.c_double()
    rc = L.ref_nbody(n, _p(pos), _p(vel), _p(mass), _p(soft2), 1e-3, steps,
                     *[_p(o) for o in outs], C.byref(ms))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    return {"n": n, "steps": steps, "ms_per_step": ms.value,
            "gpairs_per_s": n * n / (ms.value * 1e-3) / 1e9}


def main():
    L = load_ref()
    out = {"impl": "reference CUDA (unmodified sources, FP64 default, sm_100a)",
           "pm": time_pm(L),
           "nbody_4096": time_nbody(L, 4096, 100),
           "nbody_65536": time_nbody(L, 65536, 5)}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
