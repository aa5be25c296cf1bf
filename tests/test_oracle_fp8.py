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
