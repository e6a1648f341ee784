"""The persisting L2 window over a context's deposit grids and wave levels.

A context with a grid puts an access-policy window (persisting hits) over its grid arena on the
stream it launches on; the window follows the context to another stream and leaves a caller's
stream when the context does (rrg_set_stream, rrg_destroy). These tests read the window back
from the stream with cudaStreamGetAttribute.
"""
import pytest

import rrgsim_b200 as rg
from helpers import disk

pytestmark = pytest.mark.gpu


def _window(cudart, stream_ptr):
    err, v = cudart.cudaStreamGetAttribute(stream_ptr,
                                           cudart.cudaStreamAttrID.cudaLaunchAttributeAccessPolicyWindow)
    assert err == cudart.cudaError_t.cudaSuccess
    return v.accessPolicyWindow


def test_l2_window_follows_the_context_stream():
    torch = pytest.importorskip("torch")
    from cuda.bindings import runtime as cudart
    err, maxp = cudart.cudaDeviceGetAttribute(
        cudart.cudaDeviceAttr.cudaDevAttrMaxPersistingL2CacheSize, 0)
    assert err == cudart.cudaError_t.cudaSuccess
    if maxp == 0:
        pytest.skip("no persisting L2 on this device")
    pos, vel, m, s2 = disk(1000, seed=5)
    s1, s2_ = torch.cuda.Stream(), torch.cuda.Stream()
    c = rg.Context(0, "fp32")
    c.load_particles(pos, vel, m, s2)
    c.set_stream(s1.cuda_stream)
    assert _window(cudart, s1.cuda_stream).num_bytes == 0  # no grid yet: no window
    nx = 32
    c.init_grid(rg.GridInfo.from_values(nx, 16.0 / nx, 0.2))
    w = _window(cudart, s1.cuda_stream)
    # two int64 deposit grids and two FP32 levels
    assert w.num_bytes == 2 * nx ** 3 * 8 + 2 * nx ** 3 * 4
    assert w.hitProp == cudart.cudaAccessProperty.cudaAccessPropertyPersisting
    assert 0.0 < w.hitRatio <= 1.0
    c.set_stream(s2_.cuda_stream)  # the window moves with the context
    assert _window(cudart, s1.cuda_stream).num_bytes == 0
    assert _window(cudart, s2_.cuda_stream).num_bytes == w.num_bytes
    c.close()  # and leaves the caller's stream with it
    assert _window(cudart, s2_.cuda_stream).num_bytes == 0
