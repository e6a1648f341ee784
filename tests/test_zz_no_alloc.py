"""The allocation-free direct-sum entry point (rrg_dev_direct_forces_f32_noalloc).

It exists for callers that cannot let the library allocate device memory: it keeps its
scratch in a fixed 4 MiB device array per GPU instead of asking the allocator on each call.
These tests call it through the C ABI and check that two calls in a row give what the
allocating entry point (rrg_dev_direct_forces_f32) gives, within the FP32 tolerance used for
the direct sum elsewhere, and that sizes beyond its limit are refused. This file is collected
last so a failure here cannot hide the result of any other test.
"""
import numpy as np
import pytest

import oracle as orc
import rrgsim_b200 as rg
from helpers import plummer

pytestmark = pytest.mark.gpu


def _posm(torch, pos, m):
    return torch.tensor(np.hstack([pos, m[:, None]]), dtype=torch.float32, device="cuda")


@pytest.mark.parametrize("n", [1, 3000, 3001, 4096, 65536, 65537])
def test_noalloc_matches_allocating_entry_point(n):
    torch = pytest.importorskip("torch")
    L = rg.lib()
    pos, vel, m, s2 = plummer(n, seed=n)
    posm = _posm(torch, pos, m)
    h = float(np.float32(0.5 * s2[0]))
    stream = torch.cuda.current_stream().cuda_stream
    ref = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    rg.check(L.rrg_dev_direct_forces_f32(posm.data_ptr(), None, None, h, n, ref.data_ptr(), 0,
                                         stream))
    outs = []
    for _ in range(2):  # two calls in a row share (and reuse) the fixed scratch
        out = torch.full((n, 4), float("nan"), dtype=torch.float32, device="cuda")
        rg.check(L.rrg_dev_direct_forces_f32_noalloc(posm.data_ptr(), None, h, n,
                                                     out.data_ptr(), stream))
        outs.append(out)
    torch.cuda.synchronize()
    r = ref.cpu().numpy().astype(np.float64)
    for out in outs:
        o = out.cpu().numpy().astype(np.float64)
        assert np.isfinite(o).all()
        # same kernels; only the number of j-splits may differ, so the FP32 sums may differ
        # in the last bits: hold them to the direct-sum FP32 tolerance
        np.testing.assert_allclose(o, r, rtol=1e-5, atol=1e-6 * np.abs(r).max())
        # and against the FP64 oracle: the direct sum's median relative error bar
        if 2 <= n <= 4096:  # (n = 1: the self pair alone, zero force)
            acc = orc.direct_acc(pos, m, s2)
            err = np.linalg.norm(o[:, :3] - acc, axis=1) / np.linalg.norm(acc, axis=1)
            assert np.median(err) <= 1e-5


def test_noalloc_with_per_particle_softening():
    torch = pytest.importorskip("torch")
    L = rg.lib()
    n = 2000
    pos, vel, m, s2 = plummer(n, seed=3)
    s2[::2] = 0.05 ** 2
    posm = _posm(torch, pos, m)
    hs = torch.tensor(0.5 * s2, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    ref = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    out = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    rg.check(L.rrg_dev_direct_forces_f32(posm.data_ptr(), None, hs.data_ptr(), 0.0, n,
                                         ref.data_ptr(), 0, stream))
    rg.check(L.rrg_dev_direct_forces_f32_noalloc(posm.data_ptr(), hs.data_ptr(), 0.0, n,
                                                 out.data_ptr(), stream))
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_noalloc_refuses_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    L = rg.lib()
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for n in (0, (1 << 20) + 1):
        st = L.rrg_dev_direct_forces_f32_noalloc(dummy.data_ptr(), None, 1e-4, n,
                                                 dummy.data_ptr(), stream)
        assert st == 1  # RRG_ERR_INVALID, before any launch
        assert b"1048576" in L.rrg_last_error(None)
