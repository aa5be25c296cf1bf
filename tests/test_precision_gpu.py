"""Inference forms by MLP operand format (gdf_config.precision).

* BF16 and FP8 forms against the oracle run with the same storage points
  (bf16: weights, encoded inputs and hidden activations rounded to bf16;
  FP8: e4m3 hidden matrices with a power-of-two scale per matrix and per
  activation row, fp16 first and output matrices): no worse than an
  FP32-accumulating forward of the same form, as the coarse rounding steps
  make rounding flips between FP32 and FP64 accumulation common.
* All forms against the unrounded oracle (FP64 accumulation, no rounding of
  activations; the fp16 EMA weights are the network): the pdf, sampled
  direction and divergence-loss error each format carries, reported and
  bounded.
* The BF16 form also trains in bf16 (MLP weights, encoded inputs,
  activations and gradients; fp32 accumulation and optimizer): one step's
  loss and gradients against the FP64 oracle, next to the FP16 form's.
"""
import numpy as np
import pytest

import oracle as O
import pygdf
from gdf_testutil import dev, make_ctx, run_infer_pair
from pygdf import workload as W

pytestmark = pytest.mark.gpu


FORMS = [(pygdf.PREC_BF16, "bf16"), (pygdf.PREC_FP8, "fp8")]


@pytest.mark.parametrize("form", FORMS, ids=["bf16", "fp8"])
@pytest.mark.parametrize("preset", [pygdf.PRESET_SMALL, pygdf.PRESET_FULL, pygdf.PRESET_REFERENCE])
def test_form_infer_no_worse_than_fp32_accumulation(preset, form):
    """At bf16's and e4m3's rounding steps, rounding flips between FP32 and
    FP64 accumulation are common, so the per-row criteria of the fp16 tests
    do not apply; as for fp16 with large weights, the kernel's deviation from
    the FP64-accumulating oracle of the same form must stay within a small
    multiple of an FP32-accumulating forward's, for theta directions (max and
    99th percentile) and for pdfs at the kernel's directions."""
    prec, storage = form
    ctx, pt, pp = make_ctx(preset, seed=11, precision=prec)
    n = 3000
    got, _, _, guided, ref_pdf, q, _ = run_infer_pair(ctx, pt, pp, n, seed=5, storage=storage)
    d = O.df_cfg_from(ctx.cfg)
    wi, _ = W.wi_init(n, 5, 0.8, 0.2)
    u = W.uniforms(n, 5)
    L = O.lib()
    L.go_set_accumulation(1)
    try:
        ref32 = O.infer(d, pt, pp, q, wi, guided, u, storage=storage)
        b = O.eval_pdf(d, pt, pp, q, got[:, :2], storage=storage)
    finally:
        L.go_set_accumulation(0)
    ref64 = O.infer(d, pt, pp, q, wi, guided, u, storage=storage)
    a = O.eval_pdf(d, pt, pp, q, got[:, :2], storage=storage)
    g = guided.astype(bool)
    dg = np.abs(got[g, 0] - ref64[g, 0])
    de = np.abs(ref32[g, 0] - ref64[g, 0])
    print(storage, "theta direction deviation (max, p99): kernel", dg.max(), np.percentile(dg, 99),
          "fp32 emulation", de.max(), np.percentile(de, 99))
    # the largest deviation is one rounding flip on a row whose quadratic
    # root is ill-conditioned, so it gets a wider allowance than the bulk
    assert dg.max() <= 4 * de.max() + 3e-4, (dg.max(), de.max())
    assert np.percentile(dg, 99) <= 3 * np.percentile(de, 99) + 2e-5
    spread = np.abs(a - b) / (np.abs(a) + 1e-6)
    rel = np.abs(got[:, 2:4] - ref_pdf) / (np.abs(ref_pdf) + 1e-6)
    print(storage, "pdf deviation (max): kernel", rel.max(), "fp32 emulation", spread.max())
    if storage == "bf16":
        # a bf16 activation that rounds the other way (a 2^-8 step) moves a
        # pdf by up to ~2e-3; the bulk must match the FP32 forward's
        assert np.percentile(rel, 99) <= 3 * np.percentile(spread, 99) + 1e-4
        assert rel.max() <= 5e-3 and np.mean(rel > 1e-3) <= 2e-3, (rel.max(), np.mean(rel > 1e-3))
    else:
        # one e4m3 activation that rounds the other way (a 2^-3 step) moves a
        # pdf by up to a few percent; such rows are rare and both forwards have
        # them, on different rows, so the bulk and the count are compared
        assert np.percentile(rel, 99) <= 3 * np.percentile(spread, 99) + 1e-4
        assert np.mean(rel > 5e-3) <= 2e-3 and rel.max() < 0.1, (np.mean(rel > 5e-3), rel.max())
    ctx.close()


def _errors(precision, preset=pygdf.PRESET_FULL, n=8192):
    """Errors of one inference form against the unrounded FP64 oracle on the
    same weights and inputs: relative error of pdf_theta * pdf_phi at fixed
    directions, |delta u| of guided samples (theta; phi conditioned on the
    oracle's theta), and the relative error of the divergence loss
    mean(-L / wi_pdf * log(pdf_theta * pdf_phi)) over a synthetic batch."""
    ctx, pt, pp = make_ctx(preset, seed=13, precision=precision)
    d = O.df_cfg_from(ctx.cfg)
    q = W.queries(n, 8)
    u = np.random.default_rng(9).random((n, 2), dtype=np.float32)
    out = dev(np.zeros((n, 2), np.float32))
    ctx.eval_pdf(dev(q), dev(u), out)
    ctx.sync()
    got = out.cpu().numpy().astype(np.float64)
    ref = O.eval_pdf(d, pt, pp, q, u, storage="none", weights="fp16").astype(np.float64)
    g, r = got[:, 0] * got[:, 1], ref[:, 0] * ref[:, 1]
    rel = np.abs(g - r) / np.abs(r)
    # sampled directions, every query guided
    wi, _ = W.wi_init(n, 21, 1.0, 0.0)
    uu = W.uniforms(n, 21)
    guided = np.ones(n, np.uint8)
    wi_dev = dev(wi)
    ctx.infer(dev(q), wi_dev, guided=dev(guided), uniforms=dev(uu))
    ctx.sync()
    gw = wi_dev.cpu().numpy()
    rw = O.infer(d, pt, pp, q, wi, guided, uu, storage="none")
    du = np.abs(gw[:, 0].astype(np.float64) - rw[:, 0])
    # divergence loss over the pdfs at fixed directions: radiance L and
    # sampling pdf wi_pdf of a synthetic record batch
    rng = np.random.default_rng(17)
    li, wpdf = rng.exponential(1.0, n), rng.uniform(0.05, 2.0, n)
    loss_g = np.mean(-li / wpdf * np.log(np.abs(g) + 1e-5))
    loss_r = np.mean(-li / wpdf * np.log(np.abs(r) + 1e-5))
    ctx.close()
    return {"pdf": (np.percentile(rel, 50), np.percentile(rel, 99), rel.max()),
            "dir": (np.percentile(du, 50), np.percentile(du, 99), du.max()),
            "loss": abs(loss_g - loss_r) / abs(loss_r)}


def test_errors_against_unrounded_oracle():
    e = {name: _errors(prec) for name, prec in
         (("fp16", pygdf.PREC_FP16), ("bf16", pygdf.PREC_BF16), ("fp8", pygdf.PREC_FP8))}
    for name, v in e.items():
        print(name, "vs unrounded FP64 oracle: pdf_theta*pdf_phi rel (p50, p99, max)", v["pdf"],
              "theta sample |du| (p50, p99, max)", v["dir"], "loss rel", v["loss"])
    # measured on a B200 (pdf p50 / p99 / max, theta |du| p99, loss):
    #   fp16 7.8e-5 / 3.2e-4 / 5.2e-4, 1.2e-5, 1.3e-4
    #   bf16 8.7e-4 / 3.5e-3 / 5.7e-3, 1.1e-4, 5.3e-4
    #   fp8  1.1e-2 / 4.8e-2 / 8.2e-2, 1.6e-3, 1.1e-2
    assert e["fp16"]["pdf"][1] < 2e-3 and e["fp16"]["pdf"][2] < 2e-3
    assert e["bf16"]["pdf"][1] < 1e-2 and e["bf16"]["pdf"][2] < 2e-2
    assert e["fp8"]["pdf"][1] < 0.1 and e["fp8"]["pdf"][2] < 0.2
    # the coarser format carries the larger error
    assert e["fp16"]["pdf"][1] < e["bf16"]["pdf"][1] < e["fp8"]["pdf"][1]
    assert e["fp16"]["loss"] < 1e-3 and e["bf16"]["loss"] < 5e-3 and e["fp8"]["loss"] < 0.05
    assert e["fp16"]["dir"][1] < e["bf16"]["dir"][1] < e["fp8"]["dir"][1] < 1e-2


@pytest.mark.parametrize("form", FORMS, ids=["bf16", "fp8"])
def test_form_compensated_scans(form):
    """The BF16 / FP8 forms keep softmax, CDF and interpolation in fp32 with
    Neumaier-compensated sums: the FP64 normalisation check of their pdfs
    (|1 - sum p_i / N| per row and network) stays at the few roundings left
    after the compensated sum -- below the plain FP16 form's bound of a
    64-term fp32 sum -- and their sampled directions still invert their
    own CDFs (parity with the oracle of the same form is checked above)."""
    import torch
    prec, storage = form
    ctx, pt, pp = make_ctx(pygdf.PRESET_FULL, seed=4, precision=prec)
    n = 6000
    q = dev(W.queries(n, 2))
    wi0, guided = W.wi_init(n, 2, 0.8, 0.2)
    wi = dev(wi0)
    err = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.infer_ex(wi, queries=q, guided=dev(guided), seed=3, offset=9, norm_err=err)
    ctx.sync()
    e = float(err.cpu().item())
    print(storage, "max |1 - sum p / N| with compensated sums:", e)
    assert 0.0 <= e <= 4 * 2.0 ** -24, e
    ctx.close()


def _step_gradients(preset, prec, seed=3, n=8192):
    from gdf_testutil import gen_weights
    cfg = pygdf.default_config(preset)
    cfg.precision = prec
    ctx = pygdf.Context(cfg)
    pt, pp = gen_weights(cfg, 0, seed, 1.2, 0.2), gen_weights(cfg, 1, seed + 1, 1.2, 0.2)
    ctx.set_params(0, pt)
    ctx.set_params(1, pp)
    a, b, t = W.training_batch(n, seed + 7, cfg.n_bins_theta, cfg.pdf_interp == 0)
    st = ctx.train_step(dev(a), dev(b), dev(t))
    ctx.sync()
    d = O.df_cfg_from(cfg)
    beta1 = np.float64(np.float32(cfg.adam_df.beta1))
    grads = []
    for net, w0 in ((0, pt), (1, pp)):
        m = ctx.get_optimizer_state(net)[0].astype(np.float64)
        g = m / (1.0 - beta1)
        n_mlp = O.df_mlp_params(d, net)
        g[:n_mlp] -= np.float64(cfg.adam_df.l2_reg) * w0[:n_mlp]
        grads.append((g, n_mlp))
    ctx.close()
    return cfg, st, grads, (pt, pp, a, b, t)


@pytest.mark.parametrize("preset", [pygdf.PRESET_SMALL, pygdf.PRESET_FULL])
def test_bf16_training_step(preset):
    """One training step of the BF16 form: loss and gradients (recovered from
    Adam's first moment) against the oracle run with the same storage points
    (bf16 MLP matrices, encoded inputs, activations, dL/dlogits and backward
    activations; fp16 pdf tables), as tight as the FP16 form against its
    own; and, reported beside the FP16 form's, against the FP16 oracle (the
    reference's storage points): the error the format carries. The weight
    gradient sums records of both signs, so bf16's coarser storage (8
    significand bits to fp16's 11) shows up there several times larger than
    in any one term."""
    cfg, st16, g16, data = _step_gradients(preset, pygdf.PREC_FP16)
    _, stbf, gbf, _ = _step_gradients(preset, pygdf.PREC_BF16)
    pt, pp, a, b, t = data
    d = O.df_cfg_from(cfg)
    ref16 = O.df_train_grads(d, pt, pp, a, b, t, cfg.loss_scale)
    refbf = O.df_train_grads(d, pt, pp, a, b, t, cfg.loss_scale, storage="bf16")

    def rel(x, y):
        return float(np.linalg.norm(x - y) / (np.linalg.norm(y) + 1e-30))

    def loss_err(st, ref):
        lr = float(np.mean(ref["likelihood"].astype(np.float64)))
        return abs(st.loss - lr) / abs(lr)

    e16, ebf, ebf_fmt = loss_err(st16, ref16), loss_err(stbf, refbf), loss_err(stbf, ref16)
    print(f"loss rel error: fp16 form vs its oracle {e16:.2e}; bf16 form vs its oracle {ebf:.2e}, "
          f"vs the fp16 oracle {ebf_fmt:.2e}")
    assert e16 < 1e-4 and ebf < 1e-4, (e16, ebf)
    for net, key in ((0, "grad_theta"), (1, "grad_phi")):
        (x16, n_mlp), (xbf, _) = g16[net], gbf[net]
        r16g, rbfg = ref16[key] / cfg.loss_scale, refbf[key] / cfg.loss_scale
        for part, name in ((slice(0, n_mlp), "mlp"), (slice(n_mlp, None), "grid")):
            a16, abf, fmt = rel(x16[part], r16g[part]), rel(xbf[part], rbfg[part]), rel(xbf[part], r16g[part])
            print(f"net {net} {name} gradient rel error: fp16 form {a16:.2e}, bf16 form {abf:.2e} "
                  f"(vs the fp16 oracle {fmt:.2e})")
            assert a16 < 5e-3 and abf < 5e-3, (net, name, a16, abf)
    assert stbf.n_records == st16.n_records and stbf.n_dropped == st16.n_dropped


def test_bf16_training_reduces_loss():
    """Steps of the BF16 form on one batch lower its loss, as the FP16 form's do."""
    from gdf_testutil import gen_weights
    cfg = pygdf.default_config(pygdf.PRESET_SMALL)
    cfg.precision = pygdf.PREC_BF16
    ctx = pygdf.Context(cfg)
    ctx.set_params(0, gen_weights(cfg, 0, 5, 1.2, 0.2))
    ctx.set_params(1, gen_weights(cfg, 1, 6, 1.2, 0.2))
    a, b, t = (dev(x) for x in W.training_batch(8192, 9, cfg.n_bins_theta, cfg.pdf_interp == 0))
    losses = [ctx.train_step(a, b, t).loss for _ in range(30)]
    print("bf16 losses:", losses[0], losses[-1])
    assert np.all(np.isfinite(losses)) and losses[-1] < losses[0]
    ctx.close()
