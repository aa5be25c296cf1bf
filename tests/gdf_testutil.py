"""Helpers shared by the GPU parity tests: contexts with test weights, device
buffers, and the parity criteria of the DF path.

Parity criteria (inference):
  * sampled bin (CDF segment) identical to the oracle's, except where the
    oracle's uniform lies within EDGE_TOL of the segment's CDF edge;
  * pdf_theta, pdf_phi within PDF_RTOL relative (plus a tiny absolute floor);
  * sampled directions within DIR_ATOL.
"""
import numpy as np

import oracle as O
import pygdf
from pygdf import workload as W

EDGE_TOL = 1e-6
PDF_RTOL = 1e-3
PDF_ATOL = 1e-6
DIR_ATOL = 1e-3


def test_weights(ctx: pygdf.Context, net: int, seed: int, mlp_gain: float = 2.5, grid_amp: float = 0.5):
    """Weights with peaky distributions: Xavier-scaled MLP x gain, grid U(-amp, amp)."""
    rng = np.random.default_rng(seed)
    n = ctx.n_params(net)
    p = ctx.get_params(net)  # Xavier init from the library, rescaled
    cfg = ctx.cfg
    d = O.df_cfg_from(cfg)
    n_mlp = O.df_mlp_params(d, net) if net < 2 else n
    p[:n_mlp] *= mlp_gain
    p[n_mlp:] = rng.uniform(-grid_amp, grid_amp, n - n_mlp).astype(np.float32)
    ctx.set_params(net, p)
    return p


def make_ctx(preset: int, seed: int = 0, **overrides):
    cfg = pygdf.default_config(preset)
    for k, v in overrides.items():
        setattr(cfg, k, v)
    ctx = pygdf.Context(cfg)
    pt = test_weights(ctx, 0, seed)
    pp = test_weights(ctx, 1, seed + 1)
    return ctx, pt, pp


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def bins_of(u, n, linear):
    u = np.asarray(u, dtype=np.float64)
    return np.floor(u * n + (0.5 if linear else 0.0)).astype(np.int64)


def compare_infer(cfg, got, ref, gap, guided):
    """Returns a dict of error statistics; asserts the parity criteria."""
    linear = cfg.pdf_interp == 0
    g = guided.astype(bool)
    res = {}
    for k, nb, col in ((0, cfg.n_bins_theta, 0), (1, cfg.n_bins_phi, 1)):
        ok_edge = gap[:, k] > EDGE_TOL
        if k == 1:
            # phi is conditioned on theta: a theta tie changes phi's inputs
            ok_edge &= gap[:, 0] > EDGE_TOL
        sel = g & ok_edge
        bg, br = bins_of(got[:, col], nb, linear), bins_of(ref[:, col], nb, linear)
        mism = np.nonzero(sel & (bg != br))[0]
        assert mism.size == 0, f"net {k}: {mism.size} bin mismatches, e.g. rows {mism[:5]}"
        du = np.abs(got[sel, col] - ref[sel, col])
        res[f"dir{k}_max_abs"] = float(du.max()) if du.size else 0.0
        assert res[f"dir{k}_max_abs"] <= DIR_ATOL, res
        # pdf: compare all rows whose direction agrees (non-guided rows always)
        pg, pr = got[:, 2 + k], ref[:, 2 + k]
        use = (~g) | sel
        rel = np.abs(pg[use] - pr[use]) / (np.abs(pr[use]) + PDF_ATOL)
        res[f"pdf{k}_max_rel"] = float(rel.max()) if rel.size else 0.0
        assert res[f"pdf{k}_max_rel"] <= PDF_RTOL, res
    res["edge_skipped"] = int((g & ~((gap[:, 0] > EDGE_TOL) & (gap[:, 1] > EDGE_TOL))).sum())
    return res


def run_infer_pair(ctx, pt, pp, n, seed, guided_frac=0.8, one_sided=0.2, philox=None):
    import torch
    cfg = ctx.cfg
    q = W.queries(n, seed)
    wi, guided = W.wi_init(n, seed, guided_frac, one_sided)
    if philox is None:
        u = W.uniforms(n, seed)
        u_dev = dev(u)
    else:
        u = O.philox_uniforms(philox[0], philox[1], n)
        u_dev = None
    q_dev, wi_dev, g_dev = dev(q), dev(wi), dev(guided)
    ctx.infer(q_dev, wi_dev, guided=g_dev, uniforms=u_dev,
              seed=philox[0] if philox else 0, offset=philox[1] if philox else 0)
    ctx.sync()
    got = wi_dev.cpu().numpy()
    d = O.df_cfg_from(cfg)
    ref, gap = O.infer(d, pt, pp, q, wi, guided, u, edge_gap=True)
    return got, ref, gap, guided
