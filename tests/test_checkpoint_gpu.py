"""Checkpoints: gdf_save_network / gdf_load_network against the reference's
format (LearnedDistribution::saveNetwork / loadNetwork,
learnedDistribution.cpp:295-384; NRC::saveNetwork / loadNetwork,
nrc.cpp:62-112): one raw fp32 file per network, the Trainer's full-precision
parameters in tiny-cuda-nn order, no header.

The interop case loads the files this library writes into the reference's
own networks (tiny-cuda-nn rebuilt from the reference tree, oracle/_ref) the
way loadNetwork does -- the raw floats into Trainer::set_params_full_precision
-- and checks that the reference then infers what this library infers.
"""
import os

import numpy as np
import pytest

import oracle as O
import pygdf
from gdf_testutil import dev, gen_weights
from pygdf import workload as W

pytestmark = pytest.mark.gpu

FILES = ("AR_network_theta.bin", "AR_network_phi.bin", "NRC_network.bin")


def _ctx(preset, seed):
    cfg = pygdf.default_config(preset)
    ctx = pygdf.Context(cfg)
    params = [gen_weights(cfg, net, seed + net) for net in (0, 1, 2)]
    for net in (0, 1, 2):
        ctx.set_params(net, params[net])
    return cfg, ctx, params


@pytest.mark.parametrize("preset", [pygdf.PRESET_SMALL, pygdf.PRESET_REFERENCE])
def test_save_writes_raw_fp32_params_and_load_round_trips(preset, tmp_path):
    cfg, ctx, params = _ctx(preset, 3)
    prefix = str(tmp_path) + os.sep
    ctx.save(prefix)
    for net, name in enumerate(FILES):
        raw = np.fromfile(prefix + name, dtype=np.float32)
        assert raw.size == ctx.n_params(net)
        assert os.path.getsize(prefix + name) == 4 * ctx.n_params(net)  # no header
        np.testing.assert_array_equal(raw, params[net])
    # a fresh context with other weights takes the files' weights, and its
    # inference copy is fp16 of them (loadNetwork -> set_params_full_precision)
    ctx2 = pygdf.Context(cfg)
    ctx2.load(prefix)
    for net in (0, 1, 2):
        np.testing.assert_array_equal(ctx2.get_params(net), params[net])
        np.testing.assert_array_equal(ctx2.get_inference_params(net), O.round_f16(params[net]))
    # and infers exactly what the saving context infers
    n = 3000
    q = dev(W.queries(n, 1))
    wi0, guided = W.wi_init(n, 1, 0.8, 0.2)
    a, b = dev(wi0), dev(wi0)
    ctx.infer(q, a, guided=dev(guided), seed=5, offset=1)
    ctx2.infer(q, b, guided=dev(guided), seed=5, offset=1)
    ctx.sync()
    ctx2.sync()
    np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
    ctx.close()
    ctx2.close()


def test_load_rejects_short_file(tmp_path):
    cfg, ctx, params = _ctx(pygdf.PRESET_SMALL, 4)
    prefix = str(tmp_path) + os.sep
    ctx.save(prefix)
    raw = np.fromfile(prefix + FILES[1], dtype=np.float32)
    raw[:-1].tofile(prefix + FILES[1])
    ctx2 = pygdf.Context(cfg)
    with pytest.raises(pygdf.GdfError):
        ctx2.load(prefix)
    ctx.close()
    ctx2.close()


@pytest.mark.parametrize("preset", [pygdf.PRESET_SMALL, pygdf.PRESET_REFERENCE])
def test_saved_files_load_into_the_reference_networks(preset, tmp_path):
    """The reference's loadNetwork reads the raw floats into
    set_params_full_precision; done here with the files this library saved,
    the reference's networks reproduce this library's pdfs at the
    reference's sampled directions (within the fp16-accumulation spread of
    the reference, 1e-2 relative) and tiny-cuda-nn's parameter counts equal
    the files' sizes."""
    import tcnnref as T
    cfg = pygdf.default_config(preset)
    if not T.available(cfg.n_bins_theta, cfg.n_bins_phi):
        pytest.skip("reference GPU harness not built")
    import torch
    cfg, ctx, params = _ctx(preset, 5)
    prefix = str(tmp_path) + os.sep
    ctx.save(prefix)
    R = T.DfRef(cfg)
    for net in (0, 1):
        raw = np.fromfile(prefix + FILES[net], dtype=np.float32)
        assert raw.size == R.n_params(net)
        R.set_params(net, raw)
        np.testing.assert_array_equal(R.get_params(net), raw)
    n = 4096
    q = dev(W.queries(n, 2))
    wi0, guided = W.wi_init(n, 2, 0.8, 0.0)
    u = dev(W.uniforms(n, 2))
    wr = dev(wi0)
    R.infer(wr, u, queries=q, guided=dev(guided))
    torch.cuda.synchronize()
    got_ref = wr.cpu().numpy()
    pdf = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    ctx.eval_pdf(q, dev(got_ref[:, :2].copy()), pdf)
    ctx.sync()
    ours = pdf.cpu().numpy() * wi0[:, 2:4]
    rel = np.abs(ours - got_ref[:, 2:4]) / (np.abs(got_ref[:, 2:4]) + 1e-6)
    assert np.percentile(rel, 99) < 5e-3 and rel.max() < 1e-2, (np.percentile(rel, 99), rel.max())
    R.close()
    ctx.close()
