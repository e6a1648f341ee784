"""FP64 CPU oracle of the galaxy-dynamics hot path — TEST INFRASTRUCTURE ONLY.

numpy wrappers over liboracle.so (oracle.c). Only tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py use this module; the product (rrgsim_b200) never imports it.
Every function follows the reference kernel cited in oracle.h.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"


class Grid(C.Structure):
    """GridInfo + WaveParams + BoundaryParams of the reference, as the oracle takes them."""

    _fields_ = [
        ("nx", C.c_int32), ("dx", C.c_double), ("domain_min", C.c_double),
        ("sim_l", C.c_double), ("wave_speed", C.c_double), ("dt", C.c_double),
        ("diss_base", C.c_double), ("diss_extra", C.c_double), ("bc_type", C.c_int32),
        ("bc_mass", C.c_double), ("com", C.c_double * 3), ("r_min", C.c_double),
        ("rho_mean", C.c_double), ("keep_layer", C.c_int32), ("tolerance", C.c_double),
        ("steady_check_step", C.c_int32), ("steady_hold_steps", C.c_int32),
    ]


def build() -> Path:
    src = [HERE / "oracle.c", HERE / "oracle.h"]
    if not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in src):
        subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True,
                       capture_output=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB_PATH))
        d = C.POINTER(C.c_double)
        i64 = C.c_int64
        g = C.POINTER(Grid)
        pd = C.POINTER(d)
        sig = {
            "orc_num_threads": (C.c_int, []),
            "orc_set_threads": (None, [C.c_int]),
            "orc_direct_acc": (None, [i64, d, d, d, d]),
            "orc_direct_grav": (None, [i64, d, d, d, d]),
            "orc_predict": (None, [i64, d, d, d, d, C.c_double]),
            "orc_correct": (None, [i64, d, d, d, C.c_double]),
            "orc_nbody_steps": (None, [i64, d, d, d, d, d, C.c_double, C.c_int]),
            "orc_cic_fp64": (None, [i64, d, d, g, d]),
            "orc_cic_fixed": (None, [i64, d, d, g, C.c_int, C.POINTER(C.c_uint64)]),
            "orc_wave_iteration": (None, [g, d, d, d, d]),
            "orc_steady_rel_diff": (C.c_double, [i64, d, d]),
            "orc_solve_wave": (C.c_int, [g, pd, pd, pd, d, C.c_int, d]),
            "orc_gradient": (None, [g, d, d]),
            "orc_interp": (None, [i64, d, g, d, d]),
            "orc_ngp_cell": (None, [i64, d, g, C.POINTER(i64)]),
            "orc_ngp_phi": (None, [i64, d, g, d, d]),
            "orc_pm_steps": (None, [i64, d, d, d, d, g, C.c_int, C.c_double, pd, pd, pd, d, d,
                                    C.c_int]),
            "orc_conservation": (None, [i64, d, d, d, d, d]),
            "orc_mass_center": (None, [i64, d, d, d]),
            "orc_exp_disk": (None, [C.c_uint64, i64, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_double, d, d]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def make_grid(nx: int, dx: float, bc_frac: float = 0.0, wave_speed: float = 1.0,
              diss_base: float = 0.0, diss_extra: float = 0.0, bc_type: int = 1,
              rho_mean: float = 0.0, keep_layer: int = 0, bc_mass: float = 0.0,
              com=(0.0, 0.0, 0.0), tolerance: float = 1e-6, steady_check_step: int = 30,
              steady_hold_steps: int = 3) -> Grid:
    """Grid values as io_json.cpp:28-40 and :170-179 derive them (dt from the CFL rule)."""
    domain_l = dx * nx
    g = Grid()
    g.nx = nx
    g.dx = dx
    g.domain_min = -0.5 * domain_l
    g.sim_l = (1.0 - bc_frac) * domain_l
    g.wave_speed = wave_speed
    g.dt = 0.5 * dx / (wave_speed * np.sqrt(3.0))
    g.diss_base = diss_base
    g.diss_extra = diss_extra
    g.bc_type = bc_type
    g.bc_mass = bc_mass
    for k in range(3):
        g.com[k] = com[k]
    g.r_min = 0.5 * dx
    g.rho_mean = rho_mean
    g.keep_layer = keep_layer
    g.tolerance = tolerance
    g.steady_check_step = steady_check_step
    g.steady_hold_steps = steady_hold_steps
    return g


def ref_lib():
    """The reference's own CUDA build (oracle/_ref/librrgref.so, made by build_ref.sh)."""
    dp = C.POINTER(C.c_double)
    L = C.CDLL(str(HERE / "_ref" / "librrgref.so"))
    L.ref_last_error.restype = C.c_char_p
    L.ref_nbody.argtypes = [C.c_int64, dp, dp, dp, dp, C.c_double, C.c_int, dp, dp, dp, dp, dp,
                            dp]
    L.ref_pm.argtypes = [C.c_int64, dp, dp, dp, dp, C.c_int, C.c_double, C.c_double, dp,
                         C.c_double, C.c_int, dp, dp, dp, dp, dp, dp, dp, dp, dp]
    L.ref_wave_bc.argtypes = [C.c_int64, dp, dp, dp, dp, C.c_int, C.c_double, C.c_double, dp,
                              C.c_int, C.c_double, dp, dp, C.c_int, dp, dp]
    L.ref_nbody_grid.argtypes = [C.c_int64, dp, dp, dp, dp, C.c_double, C.c_int, C.c_int,
                                 C.c_double, C.c_double, dp, dp, dp, dp, dp, dp, dp]
    return L


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def direct_acc(pos, mass, soft2) -> np.ndarray:
    pos, mass, soft2 = _f64(pos), _f64(mass), _f64(soft2)
    out = np.empty_like(pos)
    lib().orc_direct_acc(len(mass), _d(pos), _d(mass), _d(soft2), _d(out))
    return out


def direct_grav(pos, mass, soft2) -> np.ndarray:
    pos, mass, soft2 = _f64(pos), _f64(mass), _f64(soft2)
    out = np.empty_like(mass)
    lib().orc_direct_grav(len(mass), _d(pos), _d(mass), _d(soft2), _d(out))
    return out


def nbody_steps(pos, vel, acc, mass, soft2, dt, nsteps):
    """Returns (pos, vel, acc) after nsteps of predict / acceleration / correct."""
    pos, vel, acc = _f64(pos).copy(), _f64(vel).copy(), _f64(acc).copy()
    mass, soft2 = _f64(mass), _f64(soft2)
    lib().orc_nbody_steps(len(mass), _d(pos), _d(vel), _d(acc), _d(mass), _d(soft2),
                          float(dt), int(nsteps))
    return pos, vel, acc


def predict(pos, vel, acc, dt):
    pos, vel, acc = _f64(pos).copy(), _f64(vel), _f64(acc)
    vstar = np.empty_like(vel)
    lib().orc_predict(vel.shape[0], _d(acc), _d(vel), _d(pos), _d(vstar), float(dt))
    return pos, vstar


def correct(vel, vstar, acc, dt):
    vel, vstar, acc = _f64(vel).copy(), _f64(vstar), _f64(acc)
    lib().orc_correct(vel.shape[0], _d(acc), _d(vel), _d(vstar), float(dt))
    return vel


def cic_fp64(pos, mass, g: Grid) -> np.ndarray:
    pos, mass = _f64(pos), _f64(mass)
    out = np.empty(g.nx ** 3, dtype=np.float64)
    lib().orc_cic_fp64(len(mass), _d(pos), _d(mass), C.byref(g), _d(out))
    return out


def cic_fixed(pos, mass, g: Grid, shift: int) -> np.ndarray:
    pos, mass = _f64(pos), _f64(mass)
    out = np.empty(g.nx ** 3, dtype=np.uint64)
    lib().orc_cic_fixed(len(mass), _d(pos), _d(mass), C.byref(g), int(shift),
                        out.ctypes.data_as(C.POINTER(C.c_uint64)))
    return out


def wave_iteration(g: Grid, phi, phi_old, mass) -> np.ndarray:
    phi, phi_old, mass = _f64(phi), _f64(phi_old), _f64(mass)
    out = np.empty_like(phi)
    lib().orc_wave_iteration(C.byref(g), _d(phi), _d(phi_old), _d(mass), _d(out))
    return out


def steady_rel_diff(u_new, u_old) -> float:
    u_new, u_old = _f64(u_new), _f64(u_old)
    return float(lib().orc_steady_rel_diff(u_new.size, _d(u_new), _d(u_old)))


class WaveState:
    """Three rotating potential levels, as GridContext_ holds them (co_grid_context.cuh:35-38)."""

    def __init__(self, nx: int):
        self.bufs = [np.zeros(nx ** 3) for _ in range(3)]
        self.p = [C.cast(b.ctypes.data, C.POINTER(C.c_double)) for b in self.bufs]
        self.ptrs = (C.POINTER(C.c_double) * 3)(*self.p)

    def _addr(self, k):
        return C.cast(C.byref(self.ptrs, k * C.sizeof(C.POINTER(C.c_double))),
                      C.POINTER(C.POINTER(C.c_double)))

    def array(self, k) -> np.ndarray:
        addr = C.cast(self.ptrs[k], C.c_void_p).value
        for b in self.bufs:
            if b.ctypes.data == addr:
                return b
        raise RuntimeError("lost buffer")

    @property
    def curr(self) -> np.ndarray:
        return self.array(1)

    @property
    def prev_level(self) -> np.ndarray:
        return self.array(0)

    def set_all(self, phi) -> None:
        for b in self.bufs:
            b[:] = phi

    def solve(self, g: Grid, mass, max_iterations: int):
        mass = _f64(mass)
        rel = C.c_double(0.0)
        it = lib().orc_solve_wave(C.byref(g), self._addr(0), self._addr(1), self._addr(2),
                                  _d(mass), int(max_iterations), C.byref(rel))
        return it, rel.value


def gradient(g: Grid, phi) -> np.ndarray:
    phi = _f64(phi)
    out = np.empty((phi.size, 3))
    lib().orc_gradient(C.byref(g), _d(phi), _d(out))
    return out


def interp(pos, g: Grid, acc3) -> np.ndarray:
    pos, acc3 = _f64(pos), _f64(acc3)
    out = np.empty_like(pos)
    lib().orc_interp(pos.shape[0], _d(pos), C.byref(g), _d(acc3), _d(out))
    return out


def ngp_cell(pos, g: Grid) -> np.ndarray:
    pos = _f64(pos)
    out = np.empty(pos.shape[0], dtype=np.int64)
    lib().orc_ngp_cell(pos.shape[0], _d(pos), C.byref(g), out.ctypes.data_as(C.POINTER(C.c_int64)))
    return out


def ngp_phi(pos, g: Grid, phi) -> np.ndarray:
    pos, phi = _f64(pos), _f64(phi)
    out = np.empty(pos.shape[0])
    lib().orc_ngp_phi(pos.shape[0], _d(pos), C.byref(g), _d(phi), _d(out))
    return out


def ngp_project(pos, g: Grid, values) -> np.ndarray:
    """NGP cell average of per-particle values: every particle adds value / (particles in its
    cell) to its cell (deposit_cell_grav_NGP_ / deposit_cell_acc_NGP_, rm_p2mesh.cu:142-174,
    cell counts from assign_particles_to_cells_, rm_p2mesh.cu:25-66). values is (n,) or (n, k);
    the result is (nx^3,) or (nx^3, k). Summation order is numpy's; the reference's is that of
    its atomics."""
    values = _f64(values)
    cell = ngp_cell(pos, g)
    count = np.bincount(cell, minlength=g.nx ** 3).astype(np.float64)
    share = values / (count[cell] if values.ndim == 1 else count[cell][:, None])
    out = np.zeros((g.nx ** 3,) + values.shape[1:])
    np.add.at(out, cell, share)
    return out


def pm_steps(pos, vel, acc, mass, g: Grid, iterations: int, dt: float, wave: WaveState,
             nsteps: int):
    """RectWaveIntegrationSolver::calc_step, nsteps times. Returns (pos, vel, acc)."""
    pos, vel, acc = _f64(pos).copy(), _f64(vel).copy(), _f64(acc).copy()
    mass = _f64(mass)
    mgrid = np.empty(g.nx ** 3)
    acc3 = np.empty((g.nx ** 3, 3))
    lib().orc_pm_steps(pos.shape[0], _d(pos), _d(vel), _d(acc), _d(mass), C.byref(g),
                       int(iterations), float(dt), wave._addr(0), wave._addr(1), wave._addr(2),
                       _d(mgrid), _d(acc3), int(nsteps))
    return pos, vel, acc


def conservation(pos, vel, mass, grav) -> dict:
    pos, vel, mass, grav = _f64(pos), _f64(vel), _f64(mass), _f64(grav)
    out = np.empty(8)
    lib().orc_conservation(len(mass), _d(pos), _d(vel), _d(mass), _d(grav), _d(out))
    return {"Ek": out[0], "Ep": out[1], "momentum": out[2:5].copy(), "angular": out[5:8].copy()}


def mass_center(pos, mass):
    pos, mass = _f64(pos), _f64(mass)
    out = np.empty(4)
    lib().orc_mass_center(len(mass), _d(pos), _d(mass), _d(out))
    return out[:3].copy(), float(out[3])


def exp_disk(seed: int, n: int, disk_mass: float = 1.0, scale_length: float = 1.0,
             z0: float = 0.1, r_max: float = 7.5, z_max: float = 7.5, disp_frac: float = 0.1):
    """The benchmark's synthetic exponential disk: the same bits as
    rrgsim_b200.generate_exp_disk with the same arguments and no bulge."""
    pos, vel = np.empty((n, 3)), np.empty((n, 3))
    lib().orc_exp_disk(int(seed), int(n), float(disk_mass), float(scale_length), float(z0),
                       float(r_max), float(z_max), float(disp_frac), _d(pos), _d(vel))
    return pos, vel
