"""Helpers shared by the GPU parity tests: contexts with test weights, device
buffers, and the parity criteria of the DF path.

Parity criteria (inference), all against the CPU oracle on identical inputs,
weights and uniforms:
  * sampled bin (bin of the direction) identical, except where the oracle's
    uniform lies within the edge tolerance of a CDF edge (EDGE_TOL on
    identical logits; EDGE_TOL_E2E through the networks, whose pdf tables
    differ from the FP64 oracle by up to ~1e-4 relative) or where the
    direction lies within DIR_ATOL of a bin boundary;
  * sampled directions within DIR_ATOL. The reference's inversion formula
    (train.h:490-501) solves a quadratic whose float evaluation loses up to
    ~1e-3 when |A| is just above its 1e-5 threshold, so ulp-level input
    differences move the root by that much in the reference itself;
  * pdf_theta, pdf_phi at the kernel's directions within PDF_RTOL relative of
    the oracle's pdf at the same directions (PDF_ATOL absolute floor).
"""
import ctypes as C

import numpy as np

import oracle as O
import pygdf
from pygdf import workload as W

EDGE_TOL = 1e-6        # identical logits (epilogue-only tests)
EDGE_TOL_E2E = 3e-5    # through the MLPs: this library's CDF error against FP64 stays below ~1e-5


def expected_edge_ties(cfg, n_guided: int, tol: float = EDGE_TOL_E2E) -> float:
    """Expected number of guided rows whose theta or phi uniform falls within
    `tol` of one of the N + 1 CDF edges of its table (uniform u)."""
    p = 1.0 - (1.0 - 2 * tol * (cfg.n_bins_theta + 1)) * (1.0 - 2 * tol * (cfg.n_bins_phi + 1))
    return n_guided * p
PDF_RTOL = 1e-3
PDF_ATOL = 1e-6
DIR_ATOL = 2e-3
DIR_TIGHT = 2e-4


def mlp_dims(cfg, net: int):
    """(rows, cols) of each FullyFusedMLP matrix of a network, tcnn order."""
    if net == 2:
        k0 = O.lib().go_nrc_input_width(C.byref(O.nrc_cfg_from(cfg)))
        h, out = cfg.mlp_nrc.n_hidden_layers, 16
    else:
        d = O.df_cfg_from(cfg)
        k0 = O.lib().go_df_input_width(C.byref(d), net)
        h = cfg.mlp_theta.n_hidden_layers if net == 0 else cfg.mlp_phi.n_hidden_layers
        nb = cfg.n_bins_theta if net == 0 else cfg.n_bins_phi
        out = (nb + 15) // 16 * 16
    return [(64, k0)] + [(64, 64)] * (h - 1) + [(out, 64)]


def gen_weights(cfg, net: int, seed: int, mlp_gain: float = 1.2, grid_amp: float = 0.2):
    """Xavier-uniform MLP matrices x `mlp_gain`, grid tables U(-amp, amp); numpy
    only, so a failed GPU comparison can be replayed on the CPU."""
    rng = np.random.default_rng(seed)
    parts = []
    for r, c in mlp_dims(cfg, net):
        s = np.sqrt(6.0 / (r + c)) * mlp_gain
        parts.append(rng.uniform(-s, s, r * c))
    if net < 2:
        d = O.df_cfg_from(cfg)
        n_grid = O.df_n_params(d, net) - O.df_mlp_params(d, net)
        parts.append(rng.uniform(-grid_amp, grid_amp, n_grid))
    return np.concatenate(parts).astype(np.float32)


def make_ctx(preset: int, seed: int = 0, gain: float = 1.2, amp: float = 0.2, **overrides):
    cfg = pygdf.default_config(preset)
    for k, v in overrides.items():
        setattr(cfg, k, v)
    ctx = pygdf.Context(cfg)
    pt = gen_weights(cfg, 0, seed, gain, amp)
    pp = gen_weights(cfg, 1, seed + 1, gain, amp)
    ctx.set_params(0, pt)
    ctx.set_params(1, pp)
    return ctx, pt, pp


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def bins_of(u, n, linear):
    u = np.asarray(u, dtype=np.float64)
    return np.floor(u * n + (0.5 if linear else 0.0)).astype(np.int64)


def near_boundary(u, n, linear, tol):
    x = np.asarray(u, dtype=np.float64) * n + (0.5 if linear else 0.0)
    return np.abs(x - np.round(x)) < np.asarray(tol) * n


def exact_directions(cfg, tables_theta, tables_phi, uniforms):
    """FP64 inverse-CDF samples (go_sample_dir_f64) of the oracle's tables."""
    n = tables_theta.shape[0]
    lin = int(cfg.pdf_interp == 0)
    ex = np.empty((n, 2), dtype=np.float64)
    f = O.lib().go_sample_dir_f64
    for i in range(n):
        ex[i, 0] = f(O._p(tables_theta[i]), tables_theta.shape[1], lin, float(uniforms[i, 0]),
                     float(uniforms[i, 1]))
        ex[i, 1] = f(O._p(tables_phi[i]), tables_phi.shape[1], lin, float(uniforms[i, 2]),
                     float(uniforms[i, 3]))
    return ex


def check_directions(cfg, got, ref, gap, guided, edge_tol=EDGE_TOL_E2E, exact=None):
    """Bins and directions of guided rows. With `exact` (FP64 inverse-CDF
    samples), a direction passes when it is within DIR_TIGHT of the oracle's,
    or no further from the exact sample than twice the oracle's own float
    error (the reference formula's conditioning) plus DIR_TIGHT."""
    linear = cfg.pdf_interp == 0
    g = guided.astype(bool)
    res = {}
    for k, nb in ((0, cfg.n_bins_theta), (1, cfg.n_bins_phi)):
        sel = g & (gap[:, k] > edge_tol)
        du = np.abs(got[:, k].astype(np.float64) - ref[:, k])
        if exact is not None:
            allow = np.maximum(DIR_TIGHT, 2.0 * np.abs(ref[:, k] - exact[:, k]) + DIR_TIGHT)
            ok = (du <= DIR_TIGHT) | (np.abs(got[:, k] - exact[:, k]) <= allow)
        else:
            allow = np.full(du.shape, DIR_ATOL)
            ok = du <= DIR_ATOL
        bad = np.nonzero(sel & ~ok)[0]
        assert bad.size == 0, f"net {k}: direction off on rows {bad[:5]}: {got[bad[:5], k]} vs {ref[bad[:5], k]}"
        bg, br = bins_of(got[:, k], nb, linear), bins_of(ref[:, k], nb, linear)
        ambiguous = near_boundary(ref[:, k], nb, linear, allow)
        mism = np.nonzero(sel & ~ambiguous & (bg != br))[0]
        assert mism.size == 0, f"net {k}: {mism.size} bin mismatches, e.g. rows {mism[:5]}"
        res[f"dir{k}_max_abs"] = float(du[sel].max()) if sel.any() else 0.0
        # non-guided rows keep the caller's direction bit for bit
        assert np.array_equal(got[~g, k], ref[~g, k])
    res["edge_skipped"] = int((g & ~((gap[:, 0] > edge_tol) & (gap[:, 1] > edge_tol))).sum())
    return res


def check_pdfs(got_pdf, ref_pdf, rtol=PDF_RTOL):
    rel = np.abs(got_pdf - ref_pdf) / (np.abs(ref_pdf) + PDF_ATOL)
    worst = float(rel.max()) if rel.size else 0.0
    assert worst <= rtol, (worst, np.unravel_index(np.argmax(rel), rel.shape))
    return worst


def run_infer_pair(ctx, pt, pp, n, seed, guided_frac=0.8, one_sided=0.2, philox=None, storage="fp16"):
    """Runs gdf_infer and the oracle on identical inputs.

    theta is compared with the oracle directly. phi is compared *chained*: the
    oracle's phi network is conditioned on the kernel's own u_theta, because
    the phi input encodes u_theta with a 12-frequency TriangleWave whose top
    frequency turns a 1e-6 difference in u_theta into ~4e-3 in the input.
    Returns got, ref (chained), gap, guided, ref_pdf_at_got, q, exact.
    """
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
    ref, gap = O.infer(d, pt, pp, q, wi, guided, u, edge_gap=True, storage=storage)
    # chained phi: oracle phi tables conditioned on the kernel's u_theta
    tt, tp = O.pdf_tables(d, pt, pp, q, got[:, 0], storage=storage)
    lin = cfg.pdf_interp == 0
    gsel = guided.astype(bool)
    for i in np.nonzero(gsel)[0]:
        _, ref[i, 1], gap[i, 1] = O.sample_dir(tp[i], lin, float(u[i, 2]), float(u[i, 3]))
    exact = exact_directions(cfg, tt, tp, u)
    # oracle pdfs at the kernel's directions (phi conditioned on the kernel's theta)
    ref_pdf_at_got = O.eval_pdf(d, pt, pp, q, got[:, :2], storage=storage) * wi[:, 2:4]
    dump("infer", q=q, wi=wi, guided=guided, u=u, got=got, ref=ref, gap=gap, ref_pdf=ref_pdf_at_got,
         exact=exact)
    return got, ref, gap, guided, ref_pdf_at_got, q, exact


def dump(tag, **arrays):
    """Saves the last compared arrays when GDF_DUMP_DIR is set (post-mortem of
    a failed GPU run without re-running it)."""
    import os
    d = os.environ.get("GDF_DUMP_DIR")
    if not d:
        return
    os.makedirs(d, exist_ok=True)
    import inspect
    caller = "unknown"
    for fr in inspect.stack():
        if fr.function.startswith("test_"):
            caller = fr.function
            break
    np.savez_compressed(os.path.join(d, f"{caller}_{tag}_{arrays['q'].shape[0]}.npz"), **arrays)


def compare_infer(ctx, got, ref, gap, guided, ref_pdf_at_got, exact, rtol=PDF_RTOL):
    res = check_directions(ctx.cfg, got, ref, gap, guided, exact=exact)
    res["pdf_max_rel"] = check_pdfs(got[:, 2:4], ref_pdf_at_got, rtol)
    return res


def fp32_emulation_spread(d, pt, pp, q, u):
    """Per-row pdf deviation of an FP32-accumulating forward from the FP64 oracle."""
    L = O.lib()
    L.go_set_accumulation.argtypes = [C.c_int]
    a = O.eval_pdf(d, pt, pp, q, u)
    L.go_set_accumulation(1)
    try:
        b = O.eval_pdf(d, pt, pp, q, u)
    finally:
        L.go_set_accumulation(0)
    return np.abs(a - b) / (np.abs(a) + PDF_ATOL)
