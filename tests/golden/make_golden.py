#!/usr/bin/env python
"""Generates the golden fixtures of tests/golden/ from the reference's own CUDA build.

Runs on a CUDA machine with oracle/_ref/librrgref.so built (oracle/build_ref.sh compiles the
reference's unmodified solver sources with stand-ins for its empty submodules). Each fixture
stores the seeded inputs and what the reference's NBody / RectWave integration strategies
produce from them, in the reference's default FP64 arithmetic.

    python tests/golden/make_golden.py [out_dir]
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import rrgsim_b200 as rg  # noqa: E402  (host-side IC generators only)

d = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(d)


def load_ref():
    import oracle
    return oracle.ref_lib()


def nbody_case(L, name, pos, vel, mass, soft2, dt, steps, out: Path):
    n = len(mass)
    acc0, grav0 = np.empty((n, 3)), np.empty(n)
    p1, v1, a1 = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
    ms = C.c_double()
    rc = L.ref_nbody(n, _p(pos), _p(vel), _p(mass), _p(soft2), dt, steps, _p(acc0), _p(grav0),
                     _p(p1), _p(v1), _p(a1), C.byref(ms))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    np.savez_compressed(out / f"{name}.npz", pos=pos, vel=vel, mass=mass, soft2=soft2,
                        dt=dt, steps=steps, acc0=acc0, grav0=grav0, pos_n=p1, vel_n=v1,
                        acc_n=a1)


def pm_case(L, name, pos, vel, mass, soft2, nx, dx, bc_frac, wave, dt, steps, out: Path):
    n = len(mass)
    nc = nx ** 3
    mass0, phi0, phi_n = np.empty(nc), np.empty(nc), np.empty(nc)
    acc0, grav0 = np.empty((n, 3)), np.empty(n)
    p1, v1, a1 = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
    ms = C.c_double()
    w = np.asarray(wave, dtype=np.float64)
    rc = L.ref_pm(n, _p(pos), _p(vel), _p(mass), _p(soft2), nx, dx, bc_frac, _p(w), dt, steps,
                  _p(mass0), _p(phi0), _p(acc0), _p(grav0), _p(p1), _p(v1), _p(a1), _p(phi_n),
                  C.byref(ms))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    np.savez_compressed(out / f"{name}.npz", pos=pos, vel=vel, mass=mass, soft2=soft2, nx=nx,
                        dx=dx, bc_frac=bc_frac, wave=w, dt=dt, steps=steps, mass0=mass0,
                        phi0=phi0, acc0=acc0, grav0=grav0, pos_n=p1, vel_n=v1, acc_n=a1,
                        phi_n=phi_n)


def wave_bc_case(L, name, pos, vel, mass, soft2, nx, dx, bc_frac, wave, bc, total_mass, com,
                 phi_init, iterations, out: Path):
    n = len(mass)
    nc = nx ** 3
    mass0, phi = np.empty(nc), np.empty(nc)
    w = np.asarray(wave, dtype=np.float64)
    com = np.asarray(com, dtype=np.float64)
    rc = L.ref_wave_bc(n, _p(pos), _p(vel), _p(mass), _p(soft2), nx, dx, bc_frac, _p(w), bc,
                       total_mass, _p(com), _p(phi_init), iterations, _p(mass0), _p(phi))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    np.savez_compressed(out / f"{name}.npz", pos=pos, vel=vel, mass=mass, soft2=soft2, nx=nx,
                        dx=dx, bc_frac=bc_frac, wave=w, bc=bc, total_mass=total_mass, com=com,
                        phi_init=phi_init, iterations=iterations, mass0=mass0, phi=phi)


def nbody_grid_case(L, name, pos, vel, mass, soft2, dt, steps, nx, dx, bc_frac, out: Path):
    n = len(mass)
    nc = nx ** 3
    gm, gg, ga = np.empty(nc), np.empty(nc), np.empty((nc, 3))
    p1, v1, a1, g1 = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3)), np.empty(n)
    rc = L.ref_nbody_grid(n, _p(pos), _p(vel), _p(mass), _p(soft2), dt, steps, nx, dx, bc_frac,
                          _p(gm), _p(gg), _p(ga), _p(p1), _p(v1), _p(a1), _p(g1))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    np.savez_compressed(out / f"{name}.npz", pos=pos, vel=vel, mass=mass, soft2=soft2, dt=dt,
                        steps=steps, nx=nx, dx=dx, bc_frac=bc_frac, grid_mass=gm, grid_grav=gg,
                        grid_acc=ga, pos_n=p1, vel_n=v1, acc_n=a1, grav_n=g1)


def main():
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent
    out.mkdir(parents=True, exist_ok=True)
    L = load_ref()

    # 1. Plummer sphere, N = 512 (a multiple of the reference's 256-thread blocks), eps = 0.01
    pos, vel = rg.generate_plummer(0, 512, 1.0, 1.0, 20.0)
    nbody_case(L, "ref_nbody_plummer512", pos, vel, np.full(512, 1 / 512),
               np.full(512, 1e-4), 1e-3, 10, out)

    # 2. two components (star + dark) with different masses and softening, N = 256 + 256
    p1, v1 = rg.generate_plummer(1, 256, 1.0, 1.0, 20.0)
    p2, v2 = rg.generate_plummer(2, 256, 3.0, 2.0, 20.0)
    pos = np.vstack([p1, p2])
    vel = np.vstack([v1, v2])
    mass = np.concatenate([np.full(256, 1.0 / 256), np.full(256, 3.0 / 512)])
    soft2 = np.concatenate([np.full(256, 0.004 ** 2), np.full(256, 0.05 ** 2)])
    nbody_case(L, "ref_nbody_two_components512", pos, vel, mass, soft2, 1e-3, 10, out)

    # 2b. the Plummer configuration at N = 4096 (eps = 0.01, dt = 1e-3), 20 steps
    pos, vel = rg.generate_plummer(0, 4096, 1.0, 1.0, 20.0)
    nbody_case(L, "ref_nbody_plummer4096", pos, vel, np.full(4096, 1 / 4096),
               np.full(4096, 1e-4), 1e-3, 20, out)

    # 3. exponential disk on a 16^3 periodic wave grid spanning +-8 (dx = 1)
    n, nx = 2048, 16
    pos, vel = rg.generate_exp_disk(1, n, 1.0, 1.0, 0.1, 7.5, 7.5, 0.1, 0.0, 0.0)
    dx = 16.0 / nx
    c = 10.0 * float(np.max(np.linalg.norm(vel, axis=1)))
    # diss_base, diss_extra, c, setup_iterations, iterations, tolerance, print, check, hold
    wave = [1.0 / (4 * dx), 0.0, c, 400, 20, 1e-6, 500, 30, 3]
    pm_case(L, "ref_pm_disk2048_nx16", pos, vel, np.full(n, 1.0 / n), np.full(n, 1e-4), nx,
            dx, 0.2, wave, 2e-3, 5, out)

    # 4. the same disk on a 32^3 grid with a dissipative layer value and an early steady stop
    nx = 32
    dx = 16.0 / nx
    wave = [1.0 / (4 * dx), 0.01, c, 3000, 20, 1e-5, 500, 10, 3]
    pm_case(L, "ref_pm_disk2048_nx32_steady", pos, vel, np.full(n, 1.0 / n),
            np.full(n, 1e-4), nx, dx, 0.2, wave, 2e-3, 3, out)

    # 5. a larger disk on a 32^3 grid without a steady check inside the step (the fused steps'
    # whole per-step solve), and 6. on a 64^3 grid with an odd substep count
    n = 8192
    pos, vel = rg.generate_exp_disk(2, n, 1.0, 1.0, 0.1, 7.5, 7.5, 0.1, 0.0, 0.0)
    c = 10.0 * float(np.max(np.linalg.norm(vel, axis=1)))
    nx = 32
    dx = 16.0 / nx
    wave = [1.0 / (4 * dx), 0.0, c, 1000, 20, 1e-6, 5000, 1000, 3]
    pm_case(L, "ref_pm_disk8192_nx32", pos, vel, np.full(n, 1.0 / n), np.full(n, 1e-4), nx, dx,
            0.2, wave, 2e-3, 6, out)
    nx = 64
    dx = 16.0 / nx
    wave = [1.0 / (4 * dx), 0.0, c, 1000, 7, 1e-6, 5000, 1000, 3]
    pm_case(L, "ref_pm_disk8192_nx64_odd", pos, vel, np.full(n, 1.0 / n), np.full(n, 1e-4), nx,
            dx, 0.2, wave, 2e-3, 5, out)
    # 7. the reference's other boundaries, which its precalc leaves commented out: periodic
    # keeping the absorbing layer, monopole Dirichlet and monopole radiative, from a seeded
    # potential on 24^3 with a dissipative layer, 30 substeps
    n, nx = 2048, 24
    pos, vel = rg.generate_exp_disk(3, n, 1.0, 1.0, 0.1, 7.5, 7.5, 0.1, 0.0, 0.0)
    dx = 16.0 / nx
    c = 10.0 * float(np.max(np.linalg.norm(vel, axis=1)))
    wave = [1.0 / (4 * dx), 0.3, c, 0, 0, 1e-6, 10 ** 6, 10 ** 6, 3]
    phi_init = -1.0 + 0.1 * np.random.default_rng(3).standard_normal(nx ** 3)
    for bc, tag in ((0, "periodic_layer"), (1, "monopole"), (2, "radiative")):
        wave_bc_case(L, f"ref_wave_bc_{tag}", pos, vel, np.full(n, 1.0 / n), np.full(n, 1e-4),
                     nx, dx, 0.2, wave, bc, 1.0, (0.1, -0.05, 0.02), phi_init, 30, out)
    # 8. the N-body strategy with a grid: the sync's CIC mass and NGP cell averages of the
    # particle potential and acceleration (a disk on 16^3 spanning +-8), after 3 steps
    n, nx = 4096, 16
    pos, vel = rg.generate_exp_disk(4, n, 1.0, 1.0, 0.1, 7.5, 7.5, 0.1, 0.0, 0.0)
    nbody_grid_case(L, "ref_nbody_grid_disk4096_nx16", pos, vel, np.full(n, 1.0 / n),
                    np.full(n, 1e-4), 1e-3, 3, nx, 16.0 / nx, 0.2, out)
    for f in sorted(out.glob("ref_*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
