"""Distribution-inspection workloads (LearnedDistribution::mouseOverInference
and mouseOverSampling, src/render/guided/learnedDistribution.cpp:386-656):

* gdf_pdf_image equals pdf_theta * pdf_phi / (4 pi) from gdf_eval_pdf at the
  pixel centres the integrator writes (integrator.cpp:721-731), bit for bit;
* the image integrates to one over the sphere;
* a histogram of gdf_sample_histogram draws matches the learned pdf
  integrated over each histogram pixel, within 5 Poisson sigma.
"""
import numpy as np
import pytest
import torch

import pygdf
from gdf_testutil import dev, gen_weights, make_ctx, mlp_dims
from pygdf import workload as W

pytestmark = pytest.mark.gpu
INV_4PI = np.float32(0.0795774715459476678844)


def _query(seed):
    return W.queries(1, seed)[0]


def _centres(w, h):
    x = np.arange(w * h) % w
    y = np.arange(w * h) // w
    u = x.astype(np.float32) / np.float32(w) + np.float32(0.5) / np.float32(w)
    v = y.astype(np.float32) / np.float32(h) + np.float32(0.5) / np.float32(h)
    return np.stack([u, v], axis=1).astype(np.float32)


@pytest.mark.parametrize("preset", [pygdf.PRESET_SMALL, pygdf.PRESET_FULL])
def test_pdf_image_equals_eval_pdf(preset):
    ctx, _, _ = make_ctx(preset, seed=3, gain=2.0)
    q = _query(7)
    w, h = 96, 64
    img = dev(np.zeros(w * h, np.float32))
    ctx.pdf_image(q, w, h, img)
    uv = _centres(w, h)
    out = dev(np.zeros((w * h, 2), np.float32))
    ctx.eval_pdf(dev(np.tile(q, (w * h, 1))), dev(uv), out)
    torch.cuda.synchronize()
    p = out.cpu().numpy()
    ref = (p[:, 0] * p[:, 1]) * INV_4PI
    np.testing.assert_array_equal(img.cpu().numpy(), ref.astype(np.float32))
    ctx.close()


def test_pdf_image_integrates_to_one():
    ctx, _, _ = make_ctx(pygdf.PRESET_FULL, seed=4, gain=2.0)
    w = h = 512
    img = dev(np.zeros(w * h, np.float32))
    ctx.pdf_image(_query(8), w, h, img)
    torch.cuda.synchronize()
    total = float(img.cpu().numpy().astype(np.float64).sum()) * 4.0 * np.pi / (w * h)
    assert abs(total - 1.0) < 5e-3, total
    ctx.close()


def test_sample_histogram_follows_pdf():
    """With the phi network's TriangleWave(theta) input columns zeroed, the
    learned distribution is separable, p(u, v) = p_theta(u) p_phi(v), and the
    expected count of a histogram pixel is n times the product of the two
    marginals integrated over it. The marginals are evaluated at 128 points
    per pixel; their kinks (bin centres) lie on those cell edges, so the
    midpoint sums are exact for the piecewise-linear pdfs."""
    cfg = pygdf.default_config(pygdf.PRESET_FULL)
    ctx = pygdf.Context(cfg)
    pt = gen_weights(cfg, 0, 5, 2.0)
    pp = gen_weights(cfg, 1, 6, 2.0)
    lf = cfg.grid_phi.n_levels * cfg.grid_phi.n_features_per_level
    k0 = mlp_dims(cfg, 1)[0][1]
    layer0 = pp[:64 * k0].reshape(64, k0)
    layer0[:, lf + 28:lf + 40] = 0.0          # phi input: grid | SH 16 | OneBlob 12 | TW 12 | pad
    ctx.set_params(0, pt)
    ctx.set_params(1, pp)
    q = _query(9)
    n = 1 << 22
    w = h = 32
    counts = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    dirs = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    ctx.sample_histogram(q, n, 77, w, h, counts, dirs)
    sub = 128
    m = w * sub
    cen = ((np.arange(m) + 0.5) / m).astype(np.float32)
    half = np.full(m, 0.5, np.float32)
    out_t = dev(np.zeros((m, 2), np.float32))
    out_p = dev(np.zeros((m, 2), np.float32))
    rows = dev(np.tile(q, (m, 1)))
    ctx.eval_pdf(rows, dev(np.stack([cen, half], 1)), out_t)
    ctx.eval_pdf(rows, dev(np.stack([half, cen], 1)), out_p)
    torch.cuda.synchronize()
    p_theta = out_t.cpu().numpy()[:, 0].astype(np.float64).reshape(w, sub).sum(1) / m
    p_phi = out_p.cpu().numpy()[:, 1].astype(np.float64).reshape(h, sub).sum(1) / m
    assert abs(p_theta.sum() - 1) < 1e-4 and abs(p_phi.sum() - 1) < 1e-4
    e = n * np.outer(p_phi, p_theta)                     # [y][x]
    c = counts.cpu().numpy().view(np.uint32).astype(np.float64).reshape(h, w)
    assert c.sum() == n
    d = dirs.cpu().numpy()
    assert d.min() >= 0.0 and d.max() < 1.0
    bad = np.abs(c - e) > 5.0 * np.sqrt(e) + 2.0
    assert not bad.any(), (np.argwhere(bad)[:5], c[bad][:5], e[bad][:5])
    ctx.close()
