"""GPU parity of the DF training step (gdf_train_step) against the oracle.

After one step from a zero optimizer state Adam's first moment is
m = (1 - beta1) * g with g = grad / loss_scale (+ l2_reg * w for MLP
weights), so the kernel's gradient is recovered exactly from m and compared
with the oracle's FP64 gradient of the same batch. Adam + EMA are then
checked in isolation by applying the oracle's optimizer to the kernel's own
gradient.
"""
import numpy as np
import pytest

import oracle as O
import pygdf
from gdf_testutil import dev, gen_weights
from pygdf import workload as W

pytestmark = pytest.mark.gpu


def _setup(preset, seed=1, n=4096, gain=1.2, amp=0.2):
    cfg = pygdf.default_config(preset)
    ctx = pygdf.Context(cfg)
    pt = gen_weights(cfg, 0, seed, gain, amp)
    pp = gen_weights(cfg, 1, seed + 1, gain, amp)
    ctx.set_params(0, pt)
    ctx.set_params(1, pp)
    a, b, t = W.training_batch(n, seed + 7, cfg.n_bins_theta, cfg.pdf_interp == 0)
    return cfg, ctx, pt, pp, a, b, t


def _kernel_gradient(ctx, net, cfg, w_before):
    m, v, steps, opt_step = ctx.get_optimizer_state(net)
    d = O.df_cfg_from(cfg)
    n_mlp = O.df_mlp_params(d, net)
    g = m.astype(np.float64) / (1.0 - np.float64(np.float32(cfg.adam_df.beta1)))
    g[:n_mlp] -= np.float64(cfg.adam_df.l2_reg) * w_before[:n_mlp]
    return g, m, v, steps, opt_step, n_mlp


def _rel(a, b):
    return float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30))


@pytest.mark.parametrize("preset", [pygdf.PRESET_SMALL, pygdf.PRESET_FULL, pygdf.PRESET_REFERENCE])
def test_train_step_gradients_match_oracle(preset):
    cfg, ctx, pt, pp, a, b, t = _setup(preset)
    st = ctx.train_step(dev(a), dev(b), dev(t))
    ctx.sync()
    d = O.df_cfg_from(cfg)
    ref = O.df_train_grads(d, pt, pp, a, b, t, cfg.loss_scale)
    loss_ref = float(np.mean(ref["likelihood"].astype(np.float64)))
    assert st.n_dropped == 0 and st.n_records == a.shape[0]
    assert abs(st.loss - loss_ref) <= 1e-3 * abs(loss_ref) + 1e-6, (st.loss, loss_ref)
    for net, w0, gref in ((0, pt, ref["grad_theta"]), (1, pp, ref["grad_phi"])):
        g, m, v, steps, opt_step, n_mlp = _kernel_gradient(ctx, net, cfg, w0)
        assert opt_step == 1
        gref = gref / cfg.loss_scale
        # MLP weight gradients: matrix by matrix
        assert _rel(g[:n_mlp], gref[:n_mlp]) < 5e-3, (net, _rel(g[:n_mlp], gref[:n_mlp]))
        # grid: identical set of touched entries, then values
        touched_ref = gref[n_mlp:] != 0.0
        touched = steps[n_mlp:] > 0
        assert np.array_equal(touched, touched_ref), (net, int((touched != touched_ref).sum()))
        assert _rel(g[n_mlp:], gref[n_mlp:]) < 5e-3, (net, _rel(g[n_mlp:], gref[n_mlp:]))
        # every MLP weight is stepped each call (matrix parameters, adam.h:73-80)
        assert np.all(steps[:n_mlp] == 1)
    gn = np.sqrt(sum(np.sum((r / cfg.loss_scale) ** 2) for r in (ref["grad_theta"], ref["grad_phi"])))
    assert abs(st.grad_norm - gn) <= 5e-3 * gn, (st.grad_norm, gn)
    ctx.close()


def test_adam_ema_match_oracle_on_kernel_gradient():
    cfg, ctx, pt, pp, a, b, t = _setup(pygdf.PRESET_SMALL, seed=5)
    ctx.train_step(dev(a), dev(b), dev(t))
    ctx.sync()
    for net, w0 in ((0, pt), (1, pp)):
        g, m, v, steps, opt_step, n_mlp = _kernel_gradient(ctx, net, cfg, w0)
        # the kernel's (scaled) gradient, fed to the oracle optimizer
        grad_scaled = m.astype(np.float64) / (1.0 - np.float64(np.float32(cfg.adam_df.beta1)))
        grad_scaled[:n_mlp] -= np.float64(cfg.adam_df.l2_reg) * w0[:n_mlp]
        grad_scaled *= cfg.loss_scale
        n = w0.size
        z = np.zeros(n, np.float32)
        master, w16, ema, m2, v2, s2 = O.adam_ema(grad_scaled, n_mlp, cfg.loss_scale, cfg.adam_df, 1,
                                                  w0, O.round_f16(w0), z, z, np.zeros(n, np.uint32))
        got_master = ctx.get_params(net)
        got_ema = ctx.get_inference_params(net)
        assert np.array_equal(s2, steps)
        assert np.allclose(v, v2, rtol=1e-4, atol=1e-30)
        assert np.allclose(got_master, master, rtol=0, atol=2e-6 * max(1.0, np.abs(master).max()))
        assert np.allclose(got_ema, ema, rtol=2e-3, atol=1e-7)
    ctx.close()


def test_dropped_records_are_filtered_and_counted():
    cfg, ctx, pt, pp, a, b, t = _setup(pygdf.PRESET_SMALL, seed=9, n=2048)
    a = a.copy()
    t = t.copy()
    a[3, 0] = np.nan
    t[10, 5] = 0.0          # wiPdf == 0 is rejected like a NaN record
    t[11, 2] = np.nan
    st = ctx.train_step(dev(a), dev(b), dev(t))
    ctx.sync()
    assert st.n_dropped == 3
    ref = O.df_train_grads(O.df_cfg_from(cfg), pt, pp, a, b, t, cfg.loss_scale)
    assert ref["dropped"] == 3
    assert np.isfinite(st.loss)
    assert abs(st.loss - float(np.mean(ref["likelihood"].astype(np.float64)))) < 1e-3 * abs(st.loss) + 1e-6
    for net in (0, 1):
        assert np.all(np.isfinite(ctx.get_params(net)))
    ctx.close()


def test_training_reduces_loss_and_inference_uses_ema():
    cfg = pygdf.default_config(pygdf.PRESET_SMALL)
    ctx = pygdf.Context(cfg)
    a, b, t = W.training_batch(65536, 3, cfg.n_bins_theta)
    da, db, dt = dev(a), dev(b), dev(t)
    losses = []
    for _ in range(30):
        losses.append(ctx.train_step(da, db, dt).loss)
    ctx.sync()
    assert losses[-1] < losses[0] * 0.9, losses
    # EMA inference weights differ from the raw training weights
    assert not np.array_equal(ctx.get_inference_params(0), O.round_f16(ctx.get_params(0)))
    ctx.close()


def test_optimizer_state_round_trip():
    cfg, ctx, pt, pp, a, b, t = _setup(pygdf.PRESET_SMALL, seed=2, n=1024)
    ctx.train_step(dev(a), dev(b), dev(t))
    m, v, s, k = ctx.get_optimizer_state(1)
    ctx.set_optimizer_state(1, m * 2, v * 3, s + 5, k + 7)
    m2, v2, s2, k2 = ctx.get_optimizer_state(1)
    assert np.array_equal(m2, m * 2) and np.array_equal(v2, v * 3)
    assert np.array_equal(s2, s + 5) and k2 == k + 7
    ctx.close()
