"""The allocation-free loss/gradient entry point of the warm-start network.

Some callers cannot call cudaMalloc: a host framework that hands all device memory to its own
pool, or code running at a point where allocating is not allowed.  For them the library offers
lp_mlp_loss_grad_noalloc, which takes caller-owned device buffers and keeps its work space in a
fixed static device array.  This file is collected last so that a run stopping at the first
failure has already run every other test; it must pass on its own in a fresh process too.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5  # same FP32 kernels on both paths: agreement to FP32 reduction-order level


def _host_loss_grad(L, w, x, y):
    F = C.POINTER(C.c_float)
    loss = C.c_float()
    g = np.zeros_like(w)
    L.check(L.lib().lp_mlp_loss_grad(w.ctypes.data_as(F), w.size, x.ctypes.data_as(F), y.ctypes.data_as(F), len(y),
                                     C.byref(loss), g.ctypes.data_as(F)))
    return loss.value, g


def test_noalloc_loss_grad_matches_allocating_entry_point():
    import torch

    from litter_physics_b200 import _lib as L
    from litter_physics_b200 import warmstart

    L.build()
    w = warmstart.init_weights(seed=3)
    dw = torch.from_numpy(w).cuda()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(11)
    for n in (3000, 4096):  # two calls in a row, different sizes
        x = rng.normal(size=(n, 6)).astype(np.float32)
        y = rng.normal(size=n).astype(np.float32)
        dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
        dloss = torch.zeros(1, device="cuda")
        dgrad = torch.zeros(w.size, device="cuda")
        L.check(L.lib().lp_mlp_loss_grad_noalloc(dw.data_ptr(), dx.data_ptr(), dy.data_ptr(), n, dloss.data_ptr(),
                                                 dgrad.data_ptr(), stream.cuda_stream))
        torch.cuda.synchronize()
        ref_loss, ref_grad = _host_loss_grad(L, w, x, y)
        got = dgrad.cpu().numpy()
        assert abs(dloss.item() - ref_loss) <= TOL * abs(ref_loss)
        assert np.abs(got - ref_grad).max() <= TOL * np.abs(ref_grad).max()


def test_noalloc_call_on_a_side_stream_allocates_nothing():
    """After the first call has set the work space up, a call queued on another stream leaves
    the device's free memory unchanged and still matches the allocating entry point."""
    import torch

    from litter_physics_b200 import _lib as L
    from litter_physics_b200 import warmstart

    L.build()
    w = warmstart.init_weights(seed=5)
    rng = np.random.default_rng(12)
    n = 2048
    x = rng.normal(size=(n, 6)).astype(np.float32)
    y = rng.normal(size=n).astype(np.float32)
    dw, dx, dy = torch.from_numpy(w).cuda(), torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    dloss = torch.zeros(1, device="cuda")
    dgrad = torch.zeros(w.size, device="cuda")
    side = torch.cuda.Stream()
    args = (dw.data_ptr(), dx.data_ptr(), dy.data_ptr(), n, dloss.data_ptr(), dgrad.data_ptr(), side.cuda_stream)
    L.check(L.lib().lp_mlp_loss_grad_noalloc(*args))  # set-up call (may be the first on this device)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        L.check(L.lib().lp_mlp_loss_grad_noalloc(*args))
    side.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    ref_loss, ref_grad = _host_loss_grad(L, w, x, y)
    assert abs(dloss.item() - ref_loss) <= TOL * abs(ref_loss)
    assert np.abs(dgrad.cpu().numpy() - ref_grad).max() <= TOL * np.abs(ref_grad).max()


def test_noalloc_rejects_sizes_beyond_its_work_space():
    import torch

    from litter_physics_b200 import _lib as L

    L.build()
    dummy = torch.zeros(8, device="cuda")
    st = L.lib().lp_mlp_loss_grad_noalloc(dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), 4097,
                                          dummy.data_ptr(), dummy.data_ptr(), None)
    assert st == 1
    assert b"outside 1..4096" in L.lib().lp_last_error()
