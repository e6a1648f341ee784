"""Shared helpers of the tests: synthetic inputs and error metrics."""
import numpy as np

import rrgsim_b200 as rg


def plummer(n, seed=0, mass=1.0, a=1.0, soft=0.01):
    pos, vel = rg.generate_plummer(seed, n, mass, a, 20.0 * a)
    m = np.full(n, mass / n)
    s2 = np.full(n, soft * soft)
    return pos, vel, m, s2


def disk(n, seed=1, mass=1.0, rd=1.0, z0=0.1, rmax=7.5, disp=0.1):
    pos, vel = rg.generate_exp_disk(seed, n, mass, rd, z0, rmax, rmax, disp, 0.0, 0.0)
    m = np.full(n, mass / n)
    s2 = np.full(n, 1e-4)
    return pos, vel, m, s2


def f32(a):
    """The values an FP32 state holds, as float64."""
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def rel_err(a, b):
    """Per-row relative error |a - b| / |b| (rows are 3-vectors)."""
    a = np.asarray(a).reshape(len(b), -1)
    b = np.asarray(b).reshape(len(b), -1)
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)
