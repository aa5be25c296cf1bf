"""GPU parity of the fused DF inference kernel against the oracle.

Each test drives the product through the C ABI (libgdf_b200.so via ctypes)
and checks it against the CPU oracle on the same seeded inputs and weights.
"""
import numpy as np
import pytest

import oracle as O
import pygdf
from gdf_testutil import (check_directions, check_pdfs, compare_infer, dev, expected_edge_ties,
                          fp32_emulation_spread, make_ctx, run_infer_pair)
from pygdf import workload as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("preset,n", [(pygdf.PRESET_SMALL, 8192), (pygdf.PRESET_FULL, 4096),
                                      (pygdf.PRESET_REFERENCE, 4096)])
def test_infer_matches_oracle(preset, n):
    ctx, pt, pp = make_ctx(preset, seed=11)
    got, ref, gap, guided, ref_pdf, _, exact = run_infer_pair(ctx, pt, pp, n, seed=5)
    stats = compare_infer(ctx, got, ref, gap, guided, ref_pdf, exact)
    # rows whose uniform lies within EDGE_TOL_E2E of a CDF edge are excluded;
    # their number must be what uniform uniforms give, not more
    n_g = int(guided.sum())
    expected = expected_edge_ties(ctx.cfg, n_g)
    print(f"edge ties skipped: {stats['edge_skipped']} of {n_g} guided rows "
          f"({stats['edge_skipped'] / n_g:.4%}), expected {expected:.1f}")
    assert stats["edge_skipped"] <= 2 * expected + 8
    ctx.close()


@pytest.mark.parametrize("preset", [pygdf.PRESET_SMALL, pygdf.PRESET_FULL])
def test_infer_phi_unchained_matches_oracle(preset):
    """phi end to end: the oracle samples theta itself and conditions its phi
    network on its own u_theta. Where both sides' u_theta agree to 2e-7 (the
    TriangleWave's 2^11 top frequency then moves the phi input by < 5e-4),
    the phi bins must agree except within 1e-4 of an edge of the oracle's
    phi CDF."""
    ctx, pt, pp = make_ctx(preset, seed=13)
    n = 8192
    q = W.queries(n, 8)
    wi, guided = W.wi_init(n, 8, 1.0, 0.0)
    u = W.uniforms(n, 8)
    wd = dev(wi)
    ctx.infer(dev(q), wd, uniforms=dev(u))
    ctx.sync()
    got = wd.cpu().numpy()
    d = O.df_cfg_from(ctx.cfg)
    ref, gap = O.infer(d, pt, pp, q, wi, None, u, edge_gap=True)
    close = np.abs(got[:, 0].astype(np.float64) - ref[:, 0]) <= 2e-7
    assert close.mean() > 0.2, close.mean()
    nb = ctx.cfg.n_bins_phi
    b_got = np.floor(got[:, 1] * nb + 0.5).astype(int)
    b_ref = np.floor(ref[:, 1] * nb + 0.5).astype(int)
    decided = close & (gap[:, 1] > 1e-4)
    assert np.array_equal(b_got[decided], b_ref[decided])
    print(f"unchained phi: {int(decided.sum())} of {n} rows decided")
    ctx.close()


@pytest.mark.parametrize("preset", [pygdf.PRESET_FULL, pygdf.PRESET_REFERENCE])
def test_infer_peaky_weights_no_worse_than_fp32_accumulation(preset):
    """Large weights make fp16 activation-rounding flips visible. The kernel's
    deviation from the FP64 oracle must stay within a small multiple of that
    of an FP32-accumulating forward (the oracle with sequential fp32 sums;
    the tensor cores sum in a different order), for directions (max and 99th
    percentile) and pdfs."""
    import oracle as O
    ctx, pt, pp = make_ctx(preset, seed=21, gain=2.5, amp=0.5)
    got, ref, gap, guided, ref_pdf, q, exact = run_infer_pair(ctx, pt, pp, 3000, seed=6)
    d = O.df_cfg_from(ctx.cfg)
    from pygdf import workload as W
    wi, _ = W.wi_init(3000, 6, 0.8, 0.2)
    u = W.uniforms(3000, 6)
    L = O.lib()
    L.go_set_accumulation(1)
    try:
        ref32 = O.infer(d, pt, pp, q, wi, guided, u)
    finally:
        L.go_set_accumulation(0)
    ref64 = O.infer(d, pt, pp, q, wi, guided, u)
    g = guided.astype(bool)
    dg = np.abs(got[g, 0] - ref64[g, 0])
    de = np.abs(ref32[g, 0] - ref64[g, 0])
    assert dg.max() <= 4 * de.max() + 3e-4, (dg.max(), de.max())
    assert np.percentile(dg, 99) <= 3 * np.percentile(de, 99) + 2e-5
    spread = fp32_emulation_spread(d, pt, pp, q, got[:, :2])
    rel = np.abs(got[:, 2:4] - ref_pdf) / (np.abs(ref_pdf) + 1e-6)
    assert rel.max() <= 3 * spread.max() + 1e-4, (rel.max(), spread.max())
    ctx.close()


def test_infer_nearest_interpolation():
    ctx, pt, pp = make_ctx(pygdf.PRESET_SMALL, seed=3, pdf_interp=pygdf.PDF_NEAREST)
    got, ref, gap, guided, ref_pdf, _, exact = run_infer_pair(ctx, pt, pp, 4096, seed=9)
    compare_infer(ctx, got, ref, gap, guided, ref_pdf, exact)
    ctx.close()


@pytest.mark.parametrize("n", [1, 7, 127, 128, 129, 513, 1000])
def test_infer_ragged_sizes(n):
    ctx, pt, pp = make_ctx(pygdf.PRESET_SMALL, seed=4)
    got, ref, gap, guided, ref_pdf, _, exact = run_infer_pair(ctx, pt, pp, n, seed=n)
    compare_infer(ctx, got, ref, gap, guided, ref_pdf, exact)
    ctx.close()


def test_infer_in_kernel_philox_matches_oracle_philox():
    ctx, pt, pp = make_ctx(pygdf.PRESET_SMALL, seed=6)
    got, ref, gap, guided, ref_pdf, _, exact = run_infer_pair(ctx, pt, pp, 3000, seed=2,
                                                       philox=(0xC0FFEE1234, 77))
    compare_infer(ctx, got, ref, gap, guided, ref_pdf, exact)
    ctx.close()


def test_infer_is_deterministic_and_writes_every_row():
    import torch
    from pygdf import workload as W
    ctx, pt, pp = make_ctx(pygdf.PRESET_FULL, seed=8)
    n = 20000
    q = dev(W.queries(n, 1))
    wi0, guided = W.wi_init(n, 1, 1.0, 0.0)
    outs = []
    for _ in range(2):
        wi = dev(wi0)
        wi[:, 0:2] = float("nan")  # guided rows must overwrite the directions
        ctx.infer(q, wi, guided=dev(guided), seed=5, offset=1)
        ctx.sync()
        outs.append(wi.cpu().numpy())
    assert np.all(np.isfinite(outs[0]))
    assert np.array_equal(outs[0], outs[1])
    assert outs[0][:, :2].min() >= 0.0 and outs[0][:, :2].max() < 1.0
    ctx.close()


@pytest.mark.parametrize("preset", [pygdf.PRESET_SMALL, pygdf.PRESET_FULL])
def test_cdf_normalisation_check(preset):
    """gdf_infer_args.cdf_norm_err_dev: the FP64 normalisation check of every
    row's theta and phi pdfs. The fp32 pdfs p_i = e_i * (N / sum e) sum to N
    up to a few fp32 roundings of the 64-term sum (<= ~N * 2^-24 relative),
    as do the oracle's tables (softmax x N) of the same rows. The check must
    not change the guiding data."""
    import torch
    from pygdf import workload as W
    ctx, pt, pp = make_ctx(preset, seed=4)
    n = 6000
    q = dev(W.queries(n, 2))
    wi0, guided = W.wi_init(n, 2, 0.8, 0.2)
    g = dev(guided)
    wi_a, wi_b = dev(wi0), dev(wi0)
    err = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.infer_ex(wi_a, queries=q, guided=g, seed=3, offset=9, norm_err=err)
    ctx.infer_ex(wi_b, queries=q, guided=g, seed=3, offset=9)
    ctx.sync()
    e = float(err.cpu().item())
    nb = max(ctx.cfg.n_bins_theta, ctx.cfg.n_bins_phi)
    print("max |1 - sum p / N| over rows (theta and phi):", e)
    assert 0.0 <= e <= 4 * nb * 2.0 ** -24
    assert np.array_equal(wi_a.cpu().numpy(), wi_b.cpu().numpy())
    # the oracle's tables at the kernel's thetas sum to N as well
    d = O.df_cfg_from(ctx.cfg)
    tt, tp = O.pdf_tables(d, pt, pp, W.queries(200, 2), wi_a.cpu().numpy()[:200, 0])
    assert np.abs(tt.sum(1) / tt.shape[1] - 1).max() < 1e-5 and np.abs(tp.sum(1) / tp.shape[1] - 1).max() < 1e-5
    ctx.close()


def test_eval_pdf_matches_oracle():
    from pygdf import workload as W
    ctx, pt, pp = make_ctx(pygdf.PRESET_FULL, seed=12)
    n = 3000
    q = W.queries(n, 3)
    u = np.random.default_rng(4).random((n, 2), dtype=np.float32)
    out = dev(np.zeros((n, 2), np.float32))
    ctx.eval_pdf(dev(q), dev(u), out)
    ctx.sync()
    got = out.cpu().numpy()
    ref = O.eval_pdf(O.df_cfg_from(ctx.cfg), pt, pp, q, u)
    rel = np.abs(got - ref) / (np.abs(ref) + 1e-6)
    assert rel.max() < 1e-3, rel.max()
    ctx.close()


@pytest.mark.parametrize("preset", [pygdf.PRESET_SMALL, pygdf.PRESET_FULL, pygdf.PRESET_REFERENCE])
def test_post_inference_matches_oracle(preset):
    cfg = pygdf.default_config(preset)
    ctx = pygdf.Context(cfg)
    rng = np.random.default_rng(7)
    n = 5000
    lt = rng.normal(0, 2.5, (n, cfg.n_bins_theta)).astype(np.float32)
    lp = rng.normal(0, 2.5, (n, cfg.n_bins_phi)).astype(np.float32)
    u = rng.random((n, 4), dtype=np.float32)
    wi = np.concatenate([rng.random((n, 2), dtype=np.float32), np.ones((n, 2), np.float32)], 1)
    guided = (rng.random(n) < 0.7).astype(np.uint8)
    wi_dev = dev(wi)
    ctx.post_inference(dev(lt), dev(lp), dev(u), wi_dev, guided=dev(guided))
    ctx.sync()
    got = wi_dev.cpu().numpy()
    d = O.df_cfg_from(cfg)
    ref, gap = O.post_inference(d, lt, lp, u, wi, guided, edge_gap=True)
    check_directions(cfg, got, ref, gap, guided, edge_tol=1e-6)
    # same logits: the oracle's pdfs at the kernel's directions differ only by
    # the libm ulps of expf/logf
    at = wi.copy()
    at[:, :2] = got[:, :2]
    ref_at = O.post_inference(d, lt, lp, u, at, np.zeros(n, np.uint8))
    check_pdfs(got[:, 2:], ref_at[:, 2:], rtol=2e-5)
    ctx.close()


def test_sync_status_clean_after_runs():
    ctx, _, _ = make_ctx(pygdf.PRESET_SMALL)
    ctx.sync()
    ctx.close()


def test_stage_events_time_the_two_launches_and_change_nothing():
    """gdf_infer_args.stage_events: the call records the two events after its
    grid-feature and fused launches; the guiding data is the same as without
    them, and the two stage times add up to the call."""
    import torch
    ctx, _, _ = make_ctx(pygdf.PRESET_FULL, seed=8)
    n = 200000
    q = dev(W.queries(n, 4))
    wi0, guided = W.wi_init(n, 4, 0.7, 0.1)
    g = dev(guided)
    wa, wb = dev(wi0), dev(wi0)
    ctx.infer_ex(wa, queries=q, guided=g, seed=2, offset=3)
    stream = torch.cuda.current_stream()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    mid = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for m in mid:
        m.record(stream)
    s.record(stream)
    ctx.infer_ex(wb, queries=q, guided=g, seed=2, offset=3, stream=stream, stage_events=mid)
    e.record(stream)
    e.synchronize()
    np.testing.assert_array_equal(wa.cpu().numpy(), wb.cpu().numpy())
    t_feat, t_fused, t_all = s.elapsed_time(mid[0]), mid[0].elapsed_time(mid[1]), s.elapsed_time(e)
    print(f"grid features {t_feat:.3f} ms, fused {t_fused:.3f} ms, call {t_all:.3f} ms")
    assert t_feat > 0 and t_fused > 0 and t_feat + t_fused <= t_all * 1.001 + 1e-3
    ctx.close()
