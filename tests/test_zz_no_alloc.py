"""gdf_train_loss_static: the allocation-free loss entry point.

Callers that cannot allocate device memory while they run (a renderer whose
device memory is a fixed arena, a host that forbids cudaMalloc after start-
up) evaluate the training loss through this entry point; its intermediates
live in a fixed array inside the library. This file is collected last so a
failure here never hides the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

import pygdf
from gdf_testutil import dev, gen_weights
from pygdf import workload as W

pytestmark = pytest.mark.gpu


def _static_loss(ctx, a, b, t, n, stream=None):
    import torch
    loss = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    dropped = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    sp = stream.cuda_stream if stream is not None else None
    pygdf.check(pygdf.lib().gdf_train_loss_static(ctx.h, a.data_ptr(), b.data_ptr(), t.data_ptr(), n,
                                                  loss.data_ptr(), dropped.data_ptr(), sp))
    torch.cuda.synchronize()
    return float(loss.item()), int(dropped.item())


def test_static_loss_matches_train_step_on_two_calls_in_a_row():
    cfg = pygdf.default_config(pygdf.PRESET_SMALL)
    ctx = pygdf.Context(cfg)
    ctx.set_params(0, gen_weights(cfg, 0, 31))
    ctx.set_params(1, gen_weights(cfg, 1, 32))
    n = 8192
    a, b, t = W.training_batch(n, 13, cfg.n_bins_theta)
    t = t.copy()
    t[5, 5] = 0.0  # one rejected record: the counter must restart at zero on every call
    da, db, dt = dev(a), dev(b), dev(t)
    for _ in range(2):
        loss, dropped = _static_loss(ctx, da, db, dt, n)
        # gdf_train_step reports the loss of the weights it starts from, then updates them
        st = ctx.train_step(da, db, dt)
        ctx.sync()
        assert dropped == st.n_dropped == 1
        assert np.isfinite(loss)
        assert abs(loss - st.loss) <= 1e-6 * abs(st.loss), (loss, st.loss)
    ctx.close()


def test_static_loss_rejects_batches_beyond_its_capacity():
    cfg = pygdf.default_config(pygdf.PRESET_SMALL)
    ctx = pygdf.Context(cfg)
    import torch
    x = torch.zeros((4, 10), dtype=torch.float32, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    L = pygdf.lib()
    st = L.gdf_train_loss_static(ctx.h, x.data_ptr(), x.data_ptr(), x.data_ptr(), 65537, out.data_ptr(),
                                 out.data_ptr(), None)
    assert st == 1 and b"65536" in L.gdf_last_error()
    assert L.gdf_train_loss_static(ctx.h, x.data_ptr(), x.data_ptr(), x.data_ptr(), 0, out.data_ptr(),
                                   out.data_ptr(), None) == 1
    ctx.close()


def test_static_loss_at_full_capacity_on_a_side_stream():
    """n = 65,536 fills the array exactly; two calls in a row on a stream
    other than the default one (the counter reset and the kernels are
    ordered on the caller's stream)."""
    import torch
    cfg = pygdf.default_config(pygdf.PRESET_SMALL)
    ctx = pygdf.Context(cfg)
    ctx.set_params(0, gen_weights(cfg, 0, 41))
    ctx.set_params(1, gen_weights(cfg, 1, 42))
    n = 65536
    a, b, t = W.training_batch(n, 17, cfg.n_bins_theta)
    t = t.copy()
    t[[3, n - 1], 5] = 0.0  # two rejected records, one in the array's last slot
    da, db, dt = dev(a), dev(b), dev(t)
    side = torch.cuda.Stream()
    for _ in range(2):
        loss, dropped = _static_loss(ctx, da, db, dt, n, stream=side)
        st = ctx.train_step(da, db, dt)
        ctx.sync()
        assert dropped == st.n_dropped == 2
        assert abs(loss - st.loss) <= 1e-6 * abs(st.loss), (loss, st.loss)
    ctx.close()
