"""rrgsim_b200 — Blackwell (sm_100a) galaxy-dynamics hot path of RRGalaxSim.

Thin Python binding over the C ABI of librrg.so (include/rrg.h). Names follow the reference
solver's free functions (solver/lib/rrgsim_nbody/include/nbody.cuh, rm_p2mesh.cuh,
rm_mesh2p.cuh, wave.cuh) and its IntegrationSolver strategy (rrgsim_integration.cuh:22-42).
There is no CPU fallback: if librrg.so is missing, or no CUDA device is present, the calls fail
with RRGError.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "librrg.so"
BIN_PATH = PKG / "bin" / "rrgsim"

PREC = {"fp32": 0, "mixed": 1, "fp64": 2}
BC_ZERO_DIRICHLET, BC_PERIODIC, BC_MONOPOLE_DIRICHLET, BC_MONOPOLE_RADIATIVE = 0, 1, 2, 3

STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "NOMEM", 4: "IO", 5: "STATE", 6: "UNSUPPORTED"}


class RRGError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{STATUS.get(status, status)}] {message}")
        self.status = status


class SimParams(C.Structure):
    _fields_ = [("time_max", C.c_double), ("dt_save", C.c_double), ("dt_dynamics", C.c_double),
                ("saves_without_dump", C.c_uint64), ("use_wave_model", C.c_int32)]


class GridInfo(C.Structure):
    _fields_ = [("nx", C.c_int32), ("dx", C.c_double), ("domain_l", C.c_double),
                ("domain_min", C.c_double), ("domain_max", C.c_double), ("bc_l", C.c_double),
                ("sim_l", C.c_double)]

    @classmethod
    def from_values(cls, nx: int, dx: float, bc_frac: float = 0.0) -> "GridInfo":
        """As from_json(GridInfo) derives the domain (solver/lib/rrgsim_io/src/io_json.cpp:28-40)."""
        g = cls()
        g.nx = int(nx)
        g.dx = float(dx)
        g.domain_l = g.dx * g.nx
        g.sim_l = (1.0 - bc_frac) * g.domain_l
        g.bc_l = 0.5 * bc_frac * g.domain_l
        g.domain_max = 0.5 * g.domain_l
        g.domain_min = -0.5 * g.domain_l
        return g


class WaveParams(C.Structure):
    _fields_ = [("diss_base", C.c_double), ("diss_extra", C.c_double), ("wave_speed", C.c_double),
                ("dt", C.c_double), ("setup_iterations", C.c_int32), ("iterations", C.c_int32),
                ("tolerance", C.c_double), ("print_step", C.c_int32),
                ("steady_check_step", C.c_int32), ("steady_hold_steps", C.c_int32)]

    @classmethod
    def make(cls, dx: float, diss_base: float, wave_speed: float, diss_extra: float = 0.0,
             setup_iterations: int = 30000, iterations: int = 3000, tolerance: float = 1e-6,
             print_step: int = 500, steady_check_step: int = 30,
             steady_hold_steps: int = 3) -> "WaveParams":
        """Defaults of io_json.cpp:53-99; dt from the CFL rule of io_json.cpp:170-179."""
        w = cls()
        w.diss_base, w.diss_extra, w.wave_speed = diss_base, diss_extra, wave_speed
        w.dt = 0.5 * dx / (wave_speed * np.sqrt(3.0))
        w.setup_iterations, w.iterations, w.tolerance = setup_iterations, iterations, tolerance
        w.print_step, w.steady_check_step = print_step, steady_check_step
        w.steady_hold_steps = steady_hold_steps
        return w


class Conservation(C.Structure):
    _fields_ = [("time", C.c_double), ("Ek", C.c_double), ("Ep", C.c_double),
                ("momentum", C.c_double * 3), ("angular", C.c_double * 3)]

    def as_dict(self) -> dict:
        return {"time": self.time, "Ek": self.Ek, "Ep": self.Ep,
                "momentum": np.array(self.momentum[:]), "angular": np.array(self.angular[:])}


class IniParams(C.Structure):
    _fields_ = [("mass_star", C.c_double), ("mass_dark", C.c_double), ("soft_star", C.c_double),
                ("soft_dark", C.c_double), ("ini_file_star", C.c_char * 1024),
                ("ini_file_dark", C.c_char * 1024)]


class ParsedParams(C.Structure):
    _fields_ = [("ini", IniParams), ("sim", SimParams), ("has_grid", C.c_int32),
                ("grid", GridInfo), ("has_wave", C.c_int32), ("wave", WaveParams)]


_lib = None


def lib() -> C.CDLL:
    """Loads librrg.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RRGError(2, f"{LIB_PATH} is missing: build it with `python -m rrgsim_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    vp, d, i64, i32 = C.c_void_p, C.POINTER(C.c_double), C.c_int64, C.c_int
    st = C.c_int
    sig = {
        "rrg_version": (C.c_char_p, []),
        "rrg_last_error": (C.c_char_p, [vp]),
        "rrg_kernel_launch_count": (C.c_uint64, []),
        "rrg_create": (st, [i32, i32, C.POINTER(vp)]),
        "rrg_destroy": (st, [vp]),
        "rrg_set_stream": (st, [vp, vp]),
        "rrg_synchronize": (st, [vp]),
        "rrg_load_particles": (st, [vp, i64, d, d, d, d]),
        "rrg_num_particles": (i64, [vp]),
        "rrg_get_particles": (st, [vp, d, d, d, d]),
        "rrg_get_time": (st, [vp, d, C.POINTER(C.c_uint64)]),
        "rrg_init_grid": (st, [vp, C.POINTER(GridInfo)]),
        "rrg_set_wave_params": (st, [vp, C.POINTER(WaveParams)]),
        "rrg_get_grid": (st, [vp, d, d, d]),
        "rrg_set_grid_potential": (st, [vp, d]),
        "rrg_get_deposit_scale": (st, [vp, C.POINTER(C.c_int32)]),
        "rrg_predict_step": (st, [vp, C.c_double]),
        "rrg_nbody_acceleration": (st, [vp]),
        "rrg_nbody_grav": (st, [vp]),
        "rrg_correct_step": (st, [vp, C.c_double]),
        "rrg_convert_particles_to_grid": (st, [vp]),
        "rrg_set_boundary_periodic": (st, [vp, C.c_double, i32]),
        "rrg_set_boundary_monopole": (st, [vp, C.c_double, d, i32]),
        "rrg_set_boundary_zero": (st, [vp]),
        "rrg_solve_wave_equation": (st, [vp, i32, C.POINTER(C.c_int), d]),
        "rrg_solve_wave_and_field": (st, [vp, i32]),
        "rrg_wave_solve_sync": (st, [vp, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
        "rrg_calc_acceleration_field": (st, [vp]),
        "rrg_project_grid_acceleration_on_particles": (st, [vp]),
        "rrg_project_grid_grav_on_particles": (st, [vp]),
        "rrg_calc_conservation": (st, [vp, C.POINTER(Conservation)]),
        "rrg_calc_conservation_async": (st, [vp, vp]),
        "rrg_conservation_from_sums": (st, [vp, C.c_double, C.POINTER(Conservation)]),
        "rrg_calc_mass_center": (st, [vp, d, d]),
        "rrg_solver_init": (st, [vp, C.POINTER(SimParams)]),
        "rrg_solver_precalc": (st, [vp]),
        "rrg_solver_calc_steps": (st, [vp, i32]),
        "rrg_solver_prepare": (st, [vp, i32]),
        "rrg_solver_sync": (st, [vp]),
        "rrg_solver_resume": (st, [vp]),
        "rrg_get_wave_state": (st, [vp, d, d]),
        "rrg_set_wave_state": (st, [vp, d, d]),
        "rrg_set_sort_interval": (st, [vp, i32]),
        "rrg_set_step_sums": (st, [vp, i32]),
        "rrg_parse_params_json": (st, [C.c_char_p, C.POINTER(ParsedParams)]),
        "rrg_read_ic_component": (st, [C.c_char_p, C.c_double, C.c_double, i64, i64, d, d, d, d,
                                       C.POINTER(i64)]),
        "rrg_ic_header_count": (st, [C.c_char_p, C.POINTER(i64)]),
        "rrg_write_ic_text": (st, [C.c_char_p, i64, C.c_double, d, d]),
        "rrg_write_dump": (st, [C.c_char_p, C.c_uint64, C.c_double, i64, d, d]),
        "rrg_read_dump": (st, [C.c_char_p, i64, C.POINTER(i64), d, d, d]),
        "rrg_run": (st, [C.c_char_p, i32, i32]),
        "rrg_run_resume": (st, [C.c_char_p, C.c_uint64, i32, i32]),
        "rrg_write_wave_state": (st, [C.c_char_p, C.c_uint64, C.c_double, i32, d, d]),
        "rrg_read_wave_state": (st, [C.c_char_p, i32, d, d, d]),
        "rrg_generate_plummer": (st, [C.c_uint64, i64, C.c_double, C.c_double, C.c_double, d, d]),
        "rrg_generate_exp_disk": (st, [C.c_uint64, i64, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, d, d]),
        "rrg_dev_direct_forces_f32": (st, [vp, vp, vp, C.c_float, i64, vp, i32, vp]),
        "rrg_dev_direct_vjp_f32": (st, [vp, vp, C.c_float, i64, vp, vp, vp]),
        "rrg_dev_direct_forces_f32_noalloc": (st, [vp, vp, C.c_float, i64, vp, vp]),
        "rrg_ensemble_create": (st, [i32, i32, C.POINTER(i64), d, d, d, d, C.c_double, i32,
                                     C.POINTER(vp)]),
        "rrg_ensemble_destroy": (st, [vp]),
        "rrg_ensemble_set_stream": (st, [vp, vp]),
        "rrg_ensemble_step": (st, [vp, i32]),
        "rrg_ensemble_step_sequential": (st, [vp, i32, i32]),
        "rrg_ensemble_synchronize": (st, [vp]),
        "rrg_ensemble_get": (st, [vp, d, d, d]),
        "rrg_ensemble_tuning": (st, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), d]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _d(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def check(status: int, ctx=None) -> None:
    if status != 0:
        msg = lib().rrg_last_error(ctx)
        raise RRGError(status, msg.decode() if msg else "")


def kernel_launch_count() -> int:
    return int(lib().rrg_kernel_launch_count())


class Context:
    """A simulation context on one GPU (particles, optional grid, solver state)."""

    def __init__(self, device: int = 0, precision: str = "fp32"):
        self._h = C.c_void_p()
        check(lib().rrg_create(int(device), PREC[precision], C.byref(self._h)))
        self.precision = precision
        self.n = 0
        self.grid = None

    # -- lifecycle ---------------------------------------------------------------------------
    def close(self) -> None:
        if self._h:
            lib().rrg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, status: int) -> None:
        check(status, self._h)

    def set_stream(self, stream_ptr: int | None) -> None:
        self._c(lib().rrg_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def synchronize(self) -> None:
        self._c(lib().rrg_synchronize(self._h))

    # -- particles ---------------------------------------------------------------------------
    def load_particles(self, pos, vel, mass, soft2) -> None:
        pos, vel, mass, soft2 = _f64(pos), _f64(vel), _f64(mass), _f64(soft2)
        n = mass.shape[0]
        if pos.shape != (n, 3) or vel.shape != (n, 3) or soft2.shape != (n,):
            raise RRGError(1, "load_particles: pos/vel must be (n, 3), mass/soft2 (n,)")
        self._c(lib().rrg_load_particles(self._h, n, _d(pos), _d(vel), _d(mass), _d(soft2)))
        self.n = n

    def get_particles(self, out: dict | None = None) -> dict:
        """The particle state in the original order. With `out`, only the arrays it holds
        ("pos", "vel", "acc": float64 (n, 3) C-contiguous; "grav": float64 (n,)) are
        written, in place (pinned host arrays make the copies direct)."""
        n = self.n
        if out is None:
            out = {"pos": np.empty((n, 3)), "vel": np.empty((n, 3)), "acc": np.empty((n, 3)),
                   "grav": np.empty(n)}
        for k, a in out.items():
            want = (n,) if k == "grav" else (n, 3)
            if (k not in ("pos", "vel", "acc", "grav") or a.dtype != np.float64 or
                    a.shape != want or not a.flags.c_contiguous):
                raise RRGError(1, f"get_particles: out[{k!r}] must be float64 {want}, contiguous")
        self._c(lib().rrg_get_particles(self._h, *(_d(out[k]) if k in out else None
                                                   for k in ("pos", "vel", "acc", "grav"))))
        return out

    def time(self):
        t = C.c_double()
        it = C.c_uint64()
        self._c(lib().rrg_get_time(self._h, C.byref(t), C.byref(it)))
        return t.value, it.value

    # -- grid --------------------------------------------------------------------------------
    def init_grid(self, grid: GridInfo) -> None:
        self._c(lib().rrg_init_grid(self._h, C.byref(grid)))
        self.grid = grid

    def set_wave_params(self, wave: WaveParams) -> None:
        self._c(lib().rrg_set_wave_params(self._h, C.byref(wave)))

    def get_grid(self) -> dict:
        nc = self.grid.nx ** 3
        mass, grav, acc = np.empty(nc), np.empty(nc), np.empty((nc, 3))
        self._c(lib().rrg_get_grid(self._h, _d(mass), _d(grav), _d(acc)))
        return {"mass": mass, "grav": grav, "acc": acc}

    def set_grid_potential(self, phi) -> None:
        phi = _f64(phi)
        self._c(lib().rrg_set_grid_potential(self._h, _d(phi)))

    def deposit_scale(self) -> int:
        s = C.c_int32()
        self._c(lib().rrg_get_deposit_scale(self._h, C.byref(s)))
        return s.value

    # -- operators (reference free functions) ------------------------------------------------
    def predict_step(self, dt: float) -> None:
        self._c(lib().rrg_predict_step(self._h, float(dt)))

    def nbody_acceleration(self) -> None:
        self._c(lib().rrg_nbody_acceleration(self._h))

    def nbody_grav(self) -> None:
        self._c(lib().rrg_nbody_grav(self._h))

    def correct_step(self, dt: float) -> None:
        self._c(lib().rrg_correct_step(self._h, float(dt)))

    def convert_particles_to_grid(self) -> None:
        self._c(lib().rrg_convert_particles_to_grid(self._h))

    def set_boundary_periodic(self, total_mass: float, keep_layer: bool = False) -> None:
        self._c(lib().rrg_set_boundary_periodic(self._h, float(total_mass), int(keep_layer)))

    def set_boundary_monopole(self, total_mass: float, center_of_mass, radiative: bool) -> None:
        com = _f64(center_of_mass)
        self._c(lib().rrg_set_boundary_monopole(self._h, float(total_mass), _d(com),
                                                int(radiative)))

    def set_boundary_zero(self) -> None:
        self._c(lib().rrg_set_boundary_zero(self._h))

    def solve_wave_equation(self, max_iterations: int):
        it = C.c_int()
        rel = C.c_double()
        self._c(lib().rrg_solve_wave_equation(self._h, int(max_iterations), C.byref(it),
                                              C.byref(rel)))
        return it.value, rel.value

    def calc_acceleration_field(self) -> None:
        self._c(lib().rrg_calc_acceleration_field(self._h))

    def solve_wave_and_field(self, iterations: int) -> None:
        """solve_wave_equation for exactly `iterations` substeps (no steady checks), then
        calc_acceleration_field, as one call: one persistent kernel on periodic FP32 / MIXED
        grids of 32, 64 or 128 cells without an absorbing layer."""
        self._c(lib().rrg_solve_wave_and_field(self._h, int(iterations)))

    def wave_solve_sync(self) -> tuple[int, int]:
        """(device address, bytes) of the persistent wave solve's synchronisation memory:
        per-block epoch counters 128 bytes apart, the error word at byte 65532, the faces."""
        p, n = C.c_void_p(), C.c_size_t()
        self._c(lib().rrg_wave_solve_sync(self._h, C.byref(p), C.byref(n)))
        return int(p.value or 0), int(n.value)

    def project_grid_acceleration_on_particles(self) -> None:
        self._c(lib().rrg_project_grid_acceleration_on_particles(self._h))

    def project_grid_grav_on_particles(self) -> None:
        self._c(lib().rrg_project_grid_grav_on_particles(self._h))

    def calc_conservation(self) -> dict:
        c = Conservation()
        self._c(lib().rrg_calc_conservation(self._h, C.byref(c)))
        return c.as_dict()

    def calc_conservation_async(self, sums: np.ndarray) -> None:
        """Enqueue the conservation sums into `sums` (12 float64, ideally pinned); no wait.
        Read them once the context stream has passed this point (conservation_from_sums)."""
        if sums.dtype != np.float64 or sums.size < 12 or not sums.flags["C_CONTIGUOUS"]:
            raise RRGError(1, "calc_conservation_async: needs 12 contiguous float64")
        self._c(lib().rrg_calc_conservation_async(self._h, sums.ctypes.data))

    def calc_mass_center(self):
        com = np.empty(3)
        m = C.c_double()
        self._c(lib().rrg_calc_mass_center(self._h, _d(com), C.byref(m)))
        return com, m.value

    # -- integration strategy ----------------------------------------------------------------
    def solver_init(self, sim: SimParams) -> None:
        self._c(lib().rrg_solver_init(self._h, C.byref(sim)))

    def precalc(self) -> None:
        self._c(lib().rrg_solver_precalc(self._h))

    def calc_steps(self, nsteps: int) -> None:
        self._c(lib().rrg_solver_calc_steps(self._h, int(nsteps)))

    def prepare_steps(self, nsteps: int) -> None:
        """Records the CUDA graphs the next calc_steps(nsteps) replays; runs nothing."""
        self._c(lib().rrg_solver_prepare(self._h, int(nsteps)))

    def sync_particles_and_grid(self) -> None:
        self._c(lib().rrg_solver_sync(self._h))

    def resume(self) -> None:
        """Precalc for a restored state: forces from the loaded positions and, in wave mode,
        the potential set by set_wave_state (no setup relaxation)."""
        self._c(lib().rrg_solver_resume(self._h))

    def get_wave_state(self):
        nc = self.grid.nx ** 3
        cur, prev = np.empty(nc), np.empty(nc)
        self._c(lib().rrg_get_wave_state(self._h, _d(cur), _d(prev)))
        return cur, prev

    def set_wave_state(self, cur, prev) -> None:
        cur, prev = _f64(cur), _f64(prev)
        self._c(lib().rrg_set_wave_state(self._h, _d(cur), _d(prev)))

    def set_sort_interval(self, interval: int) -> None:
        self._c(lib().rrg_set_sort_interval(self._h, int(interval)))

    def set_step_sums(self, enable: bool) -> None:
        """Wave mode: the last particle pass of each calc_steps call also forms the
        conservation sums, so a calc_conservation(_async) right after it only combines them."""
        self._c(lib().rrg_set_step_sums(self._h, 1 if enable else 0))


class Ensemble:
    """Independent galaxies stepped together (one persistent force launch per step)."""

    def __init__(self, counts, pos, vel, mass, soft2_per_galaxy, dt: float, device: int = 0,
                 autotune: bool = True):
        counts = np.ascontiguousarray(counts, dtype=np.int64)
        pos, vel, mass = _f64(pos), _f64(vel), _f64(mass)
        s2 = _f64(soft2_per_galaxy)
        self.counts = counts
        self.ntot = int(counts.sum())
        if pos.shape != (self.ntot, 3) or vel.shape != (self.ntot, 3) or mass.shape != (self.ntot,):
            raise RRGError(1, "Ensemble: arrays must hold sum(counts) particles")
        self._h = C.c_void_p()
        check(lib().rrg_ensemble_create(int(device), len(counts),
                                        counts.ctypes.data_as(C.POINTER(C.c_int64)), _d(pos),
                                        _d(vel), _d(mass), _d(s2), float(dt), int(autotune),
                                        C.byref(self._h)))

    def _c(self, status):
        check(status, None)

    def step(self, nsteps: int) -> None:
        self._c(lib().rrg_ensemble_step(self._h, int(nsteps)))

    def step_sequential(self, nsteps: int, plain: bool = False) -> None:
        """One force launch per galaxy; plain=True in the reference's launch shape."""
        self._c(lib().rrg_ensemble_step_sequential(self._h, int(nsteps), int(plain)))

    def set_stream(self, stream_ptr) -> None:
        self._c(lib().rrg_ensemble_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def synchronize(self) -> None:
        self._c(lib().rrg_ensemble_synchronize(self._h))

    def get(self) -> dict:
        pos, vel, acc = (np.empty((self.ntot, 3)) for _ in range(3))
        self._c(lib().rrg_ensemble_get(self._h, _d(pos), _d(vel), _d(acc)))
        return {"pos": pos, "vel": vel, "acc": acc}

    def tuning(self) -> dict:
        v, j, k = C.c_int(), C.c_int(), C.c_int()
        ms = C.c_double()
        self._c(lib().rrg_ensemble_tuning(self._h, C.byref(v), C.byref(j), C.byref(k),
                                          C.byref(ms)))
        return {"variant": v.value, "jchunk": j.value, "items": k.value, "force_ms": ms.value}

    def close(self) -> None:
        if self._h:
            lib().rrg_ensemble_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def make_ensemble(ngal: int = 64, nmin: int = 1024, nmax: int = 65536, seed: int = 3,
                  base_mass: float = 1.0, base_scale: float = 1.0, base_soft: float = 0.01):
    """The batched-form galaxies: N log-uniform in [nmin, nmax], each a Plummer sphere or an
    exponential disk by coin flip, mass / scale radius / softening each uniform in
    [0.5, 2] x base. Returns counts, pos, vel, mass, soft2 per galaxy."""
    rng = np.random.default_rng(seed)
    counts, P, V, M, S2 = [], [], [], [], []
    for g in range(ngal):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        disk_kind = rng.random() < 0.5
        mass, scale, soft = (base_mass * rng.uniform(0.5, 2.0), base_scale * rng.uniform(0.5, 2.0),
                             base_soft * rng.uniform(0.5, 2.0))
        gseed = int(rng.integers(1 << 62))
        if disk_kind:
            p, v = generate_exp_disk(gseed, n, mass, scale, 0.1 * scale, 7.5 * scale,
                                     7.5 * scale, 0.1)
        else:
            p, v = generate_plummer(gseed, n, mass, scale, 20.0 * scale)
        counts.append(n)
        P.append(p)
        V.append(v)
        M.append(np.full(n, mass / n))
        S2.append(soft * soft)
    return (np.array(counts, dtype=np.int64), np.vstack(P), np.vstack(V), np.concatenate(M),
            np.array(S2))


# -- host I/O --------------------------------------------------------------------------------
def conservation_from_sums(sums: np.ndarray, time: float = 0.0) -> dict:
    """Ek, Ep, momentum and angular momentum from the 12 sums of calc_conservation_async."""
    s = np.ascontiguousarray(sums, dtype=np.float64)
    c = Conservation()
    check(lib().rrg_conservation_from_sums(s.ctypes.data, float(time), C.byref(c)))
    return c.as_dict()


def parse_params_json(path) -> ParsedParams:
    p = ParsedParams()
    check(lib().rrg_parse_params_json(str(path).encode(), C.byref(p)))
    return p


def read_ic(path, component_mass: float, component_soft: float, n_before: int = 0):
    """One IC component; arrays sized for this file only (mass divides by n_before + N)."""
    n = C.c_int64()
    check(lib().rrg_ic_header_count(str(path).encode(), C.byref(n)))
    total = n_before + n.value
    pos, vel = np.zeros((total, 3)), np.zeros((total, 3))
    mass, soft2 = np.zeros(total), np.zeros(total)
    got = C.c_int64()
    check(lib().rrg_read_ic_component(str(path).encode(), float(component_mass),
                                      float(component_soft), int(n_before), total, _d(pos),
                                      _d(vel), _d(mass), _d(soft2), C.byref(got)))
    return pos[n_before:], vel[n_before:], mass[n_before:], soft2[n_before:]


def write_ic_text(path, pos, vel, t: float = 0.0) -> None:
    pos, vel = _f64(pos), _f64(vel)
    check(lib().rrg_write_ic_text(str(path).encode(), pos.shape[0], float(t), _d(pos), _d(vel)))


def write_dump(dump_dir, iteration: int, time: float, pos, vel) -> None:
    pos, vel = _f64(pos), _f64(vel)
    check(lib().rrg_write_dump(str(dump_dir).encode(), int(iteration), float(time), pos.shape[0],
                               _d(pos), _d(vel)))


def read_dump(path):
    n = C.c_int64()
    t = C.c_double()
    check(lib().rrg_read_dump(str(path).encode(), 0, C.byref(n), C.byref(t), None, None))
    pos, vel = np.empty((n.value, 3)), np.empty((n.value, 3))
    check(lib().rrg_read_dump(str(path).encode(), n.value, C.byref(n), C.byref(t), _d(pos),
                              _d(vel)))
    return t.value, pos, vel


def run(work_dir, device: int = 0, precision: str = "fp32", resume: int | None = None) -> None:
    """The rrgsim run of work_dir; resume=<iteration> continues from that dump."""
    if resume is None:
        check(lib().rrg_run(str(work_dir).encode(), int(device), PREC[precision]))
    else:
        check(lib().rrg_run_resume(str(work_dir).encode(), int(resume), int(device),
                                   PREC[precision]))


def read_wave_state(path, nx: int):
    cur, prev = np.empty(nx ** 3), np.empty(nx ** 3)
    t = C.c_double()
    check(lib().rrg_read_wave_state(str(path).encode(), int(nx), C.byref(t), _d(cur), _d(prev)))
    return t.value, cur, prev


def generate_plummer(seed: int, n: int, total_mass: float = 1.0, scale_radius: float = 1.0,
                     r_max: float = 20.0):
    pos, vel = np.empty((n, 3)), np.empty((n, 3))
    check(lib().rrg_generate_plummer(int(seed), int(n), float(total_mass), float(scale_radius),
                                     float(r_max), _d(pos), _d(vel)))
    return pos, vel


def generate_exp_disk(seed: int, n: int, disk_mass: float = 1.0, scale_length: float = 1.0,
                      z0: float = 0.1, r_max: float = 7.5, z_max: float = 7.5,
                      disp_frac: float = 0.1, bulge_mass: float = 0.0, bulge_a: float = 0.0):
    pos, vel = np.empty((n, 3)), np.empty((n, 3))
    check(lib().rrg_generate_exp_disk(int(seed), int(n), float(disk_mass), float(scale_length),
                                      float(z0), float(r_max), float(z_max), float(disp_frac),
                                      float(bulge_mass), float(bulge_a), _d(pos), _d(vel)))
    return pos, vel


def version() -> str:
    return lib().rrg_version().decode()
