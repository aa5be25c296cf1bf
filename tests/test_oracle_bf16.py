"""The oracle's bf16 rounding of the BF16 inference form, pinned on the CPU:
the C routine (go_round_bf16, used inside the oracle's forward) and the
numpy one (round_bf16, used for the weights) both equal PyTorch's bfloat16
conversion (round to nearest even) on random values across the float range,
on every tie between neighbouring bf16 values, and on infinities."""
import numpy as np
import torch

import oracle as O


def _torch_bf16(x):
    return torch.from_numpy(np.asarray(x, dtype=np.float32)).to(torch.bfloat16).float().numpy()


def test_round_bf16_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(4000) * 10.0 ** rng.uniform(-30, 30, 4000),
                        rng.uniform(-1, 1, 4000)]).astype(np.float32)
    # ties: halfway between neighbouring bf16 values (low 16 bits 0x8000)
    hi = (rng.integers(0x0080, 0x7f00, 2000, dtype=np.uint32) << 16) | 0x8000
    ties = hi.view(np.float32)
    x = np.concatenate([x, ties, -ties, np.array([np.inf, -np.inf, 0.0, -0.0], np.float32)])
    ref = _torch_bf16(x)
    assert np.array_equal(O.round_bf16(x), ref)
    L = O.lib()
    got = np.array([L.go_round_bf16(float(v)) for v in x], dtype=np.float32)
    assert np.array_equal(got, ref)


def test_training_oracle_storage_switch():
    """The training oracle's storage switch (the bf16 training form's storage
    points): it changes the gradients by the format's error -- more than
    fp32 noise, much less than the gradients -- is deterministic, and leaves
    the default fp16 model untouched afterwards."""
    import pygdf
    from gdf_testutil import gen_weights
    from pygdf import workload as W
    cfg = pygdf.default_config(pygdf.PRESET_SMALL)
    d = O.df_cfg_from(cfg)
    pt, pp = gen_weights(cfg, 0, 3), gen_weights(cfg, 1, 4)
    a, b, t = W.training_batch(1024, 10, cfg.n_bins_theta, cfg.pdf_interp == 0)
    g16 = O.df_train_grads(d, pt, pp, a, b, t, cfg.loss_scale)
    gbf = O.df_train_grads(d, pt, pp, a, b, t, cfg.loss_scale, storage="bf16")
    gbf2 = O.df_train_grads(d, pt, pp, a, b, t, cfg.loss_scale, storage="bf16")
    g16b = O.df_train_grads(d, pt, pp, a, b, t, cfg.loss_scale)
    for key in ("grad_theta", "grad_phi"):
        assert np.array_equal(gbf[key], gbf2[key]) and np.array_equal(g16[key], g16b[key])
        rel = np.linalg.norm(gbf[key] - g16[key]) / np.linalg.norm(g16[key])
        assert 1e-4 < rel < 0.3, (key, rel)
