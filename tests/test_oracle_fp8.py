"""The oracle's e4m3 arithmetic of the FP8 inference form, pinned on the CPU.

go_round_e4m3 (OCP E4M3: bias 7, 3 mantissa bits, largest finite 448,
round to nearest even) is checked against PyTorch's float8_e4m3fn
conversion on every finite e4m3 value, every midpoint between neighbours
(ties to even) and random values across the range, subnormals included;
go_e4m3_scale_exp against its definition (largest 2^k with amax * 2^k <= 448).
"""
import numpy as np
import torch

import oracle as O


def test_round_e4m3_matches_torch_float8():
    L = O.lib()
    codes = torch.arange(256, dtype=torch.uint8).view(torch.float8_e4m3fn).float().numpy()
    fin = np.unique(codes[np.isfinite(codes)])
    mids = (fin[:-1] + fin[1:]) / 2
    rng = np.random.default_rng(0)
    xs = np.concatenate([fin, mids, rng.uniform(-448, 448, 3000), rng.uniform(-0.05, 0.05, 3000),
                         np.exp(rng.uniform(-14, 6, 3000)) * rng.choice([-1.0, 1.0], 3000)])
    xs = xs[np.abs(xs) <= 448].astype(np.float32)
    got = np.array([L.go_round_e4m3(float(x)) for x in xs])
    ref = torch.from_numpy(xs).to(torch.float8_e4m3fn).float().numpy()
    assert np.array_equal(got, ref), xs[got != ref][:8]
    # saturation above the largest finite value
    assert L.go_round_e4m3(470.0) == 448.0 and L.go_round_e4m3(-1e6) == -448.0


def test_e4m3_scale_exp():
    L = O.lib()
    rng = np.random.default_rng(1)
    for amax in np.concatenate([np.exp(rng.uniform(-40, 40, 2000)), [448.0, 449.0, 1.75, 1.7500001, 1.0, 2.0]]):
        k = L.go_e4m3_scale_exp(float(amax))
        assert amax * 2.0 ** k <= 448.0 and amax * 2.0 ** (k + 1) > 448.0, (amax, k)
    assert L.go_e4m3_scale_exp(0.0) == 0 and L.go_e4m3_scale_exp(float("inf")) == 0
    assert L.go_e4m3_scale_exp(1e-40) == 100 and L.go_e4m3_scale_exp(1e40) == -100


def _e4m3(x):
    x = np.asarray(x, dtype=np.float64)
    return torch.from_numpy(x.astype(np.float32)).to(torch.float8_e4m3fn).double().numpy()


def _scale_exp(amax):
    """Largest k with amax * 2^k <= 448, found by search (0 for amax = 0)."""
    if amax == 0.0:
        return 0
    k = int(np.floor(np.log2(448.0 / amax)))
    while amax * 2.0 ** (k + 1) <= 448.0:
        k += 1
    while amax * 2.0 ** k > 448.0:
        k -= 1
    return max(-100, min(100, k))


def _fp8_forward(w, k0, width, n_hidden, n_out, x):
    """The FP8 inference form written out in numpy: matrix 0 over the fp16
    inputs, each hidden matrix as e4m3(W * 2^kw) over e4m3(relu(h) * 2^kr)
    with kw from max|W| and kr from the row's max, descaled by 2^-(kw+kr),
    the last activations rounded to fp16 for the output matrix."""
    mats, o = [], 0
    for rows, cols in [(width, k0)] + [(width, width)] * (n_hidden - 1) + [(n_out, width)]:
        mats.append(w[o:o + rows * cols].astype(np.float64).reshape(rows, cols))
        o += rows * cols
    acc = mats[0] @ x.astype(np.float64)
    d = 1.0
    for l in range(1, n_hidden + 1):
        v = np.maximum(acc * d, 0.0)
        if l < n_hidden:
            kr = _scale_exp(v.max())
            kw = _scale_exp(np.abs(mats[l]).max())
            acc = _e4m3(mats[l] * 2.0 ** kw) @ _e4m3(v * 2.0 ** kr)
            d = 2.0 ** -(kw + kr)
        else:
            h = v.astype(np.float16).astype(np.float64)
            return mats[l] @ h


def test_oracle_fp8_forward_matches_an_independent_restatement():
    rng = np.random.default_rng(3)
    k0, width, n_hidden, n_out = 64, 64, 4, 64
    n_w = width * k0 + (n_hidden - 1) * width * width + n_out * width
    worst = 0.0
    for trial in range(20):
        scale = 10.0 ** rng.uniform(-2, 1)  # weights of very different magnitudes
        w = (rng.standard_normal(n_w) * scale / 8).astype(np.float16).astype(np.float32)
        x = rng.uniform(-1, 1, k0).astype(np.float16).astype(np.float32)
        got = O.mlp_forward(w, k0, width, n_hidden, n_out, x, storage="fp8").astype(np.float64)
        ref = _fp8_forward(w, k0, width, n_hidden, n_out, x)
        err = np.abs(got - ref) / (np.abs(ref).max() + 1e-30)
        worst = max(worst, err.max())
    # the oracle returns fp32 logits of an FP64 computation
    assert worst < 1e-6, worst
