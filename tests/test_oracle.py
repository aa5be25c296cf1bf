"""CPU checks of the oracle against known answers and analytic identities.

The reference ships no tests or golden vectors for this path, so the oracle
is pinned here by (a) published known-answer vectors (Philox), (b) analytic
properties of each restated function, and (c) the reference's own host-
compilable functions (test_reference_pin.py).
"""
import math

import numpy as np
import pytest

import oracle as O


def test_philox_known_answers():
    # Random123 known-answer vectors for Philox4x32-10 (Salmon et al., SC'11).
    assert O.philox_block([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    f = 0xFFFFFFFF
    assert O.philox_block([f, f, f, f], [f, f]) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox_block([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_philox_uniform_range_and_mean():
    u = O.philox_uniforms(1234, 7, 50000)
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.005
    # 23-bit mantissa trick: every value is a multiple of 2^-23
    assert np.all(np.mod(u.astype(np.float64) * 2 ** 23, 1.0) == 0.0)


def test_fp16_rounding_matches_ieee():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.normal(0, 1, 2000), rng.normal(0, 1e-5, 500), rng.normal(0, 3e4, 200),
                         [65504.0, 65519.0, 65520.0, 6.1e-5, 5.96e-8, 2.98e-8, 0.0, -0.0]])
    with np.errstate(over="ignore"):
        for x in xs:
            assert O.round_f16_scalar(x) == np.float32(np.float16(x)), x


def test_softmax_times_n():
    v = O.softmax_times_n(np.zeros(32))
    assert np.allclose(v, 1.0, atol=1e-6)
    rng = np.random.default_rng(1)
    v = O.softmax_times_n(rng.normal(0, 3, 64))
    assert abs(v.sum() - 64.0) < 1e-3
    # max starts at 0 (train.h:846): all-negative logits are not shifted by
    # their own max. Moderate ones are fine ...
    v = O.softmax_times_n(np.full(16, -50.0))
    assert np.allclose(v, 1.0, atol=1e-5)
    # ... but once every exp underflows the reference's softmax2 divides by a
    # zero sum; the restatement keeps that behaviour (non-finite pdfs).
    v = O.softmax_times_n(np.full(16, -200.0))
    assert not np.any(np.isfinite(v))


@pytest.mark.parametrize("linear", [True, False])
@pytest.mark.parametrize("n", [16, 32, 64])
def test_uniform_pdf_sampling_is_identity(linear, n):
    pdf = np.ones(n, dtype=np.float32)
    for u in np.linspace(0.0, 0.999, 97):
        _, d, _ = O.sample_dir(pdf, linear, float(u), 0.5)
        assert abs(d - min(u, 1 - 1e-5)) < 2e-6, (u, d)


@pytest.mark.parametrize("linear", [True, False])
def test_one_hot_pdf_samples_inside_bin(linear):
    n = 32
    rng = np.random.default_rng(2)
    for b in range(n):
        logits = np.full(n, -30.0)
        logits[b] = 30.0
        pdf = O.softmax_times_n(logits)
        for u in rng.random(8):
            _, d, _ = O.sample_dir(pdf, linear, float(u), 0.5)
            lo = (b - 0.5) / n if linear else b / n
            hi = (b + 1.5) / n if linear else (b + 1) / n
            assert lo - 1e-5 <= d <= hi + 1e-5, (b, u, d)


@pytest.mark.parametrize("linear", [True, False])
def test_sampling_float_matches_double_twin(linear):
    rng = np.random.default_rng(3)
    worst = 0.0
    for _ in range(2000):
        n = int(rng.choice([16, 32, 64]))
        pdf = O.softmax_times_n(rng.normal(0, 2, n))
        u, u2 = rng.random(2)
        _, d, gap = O.sample_dir(pdf, linear, float(u), float(u2))
        pdf32 = O.f32(pdf)  # alive across the call
        dd = O.lib().go_sample_dir_f64(O._p(pdf32), n, int(linear), float(np.float32(u)),
                                        float(np.float32(u2)))
        if gap > 1e-5:
            worst = max(worst, abs(d - dd))
    assert worst < 2e-3, worst


def test_sample_pdf_interpolation():
    n = 16
    pdf = np.arange(1, n + 1, dtype=np.float32)
    for i in range(n):
        assert O.sample_pdf(pdf, (i + 0.5) / n, True) == pytest.approx(pdf[i], rel=1e-6)
        assert O.sample_pdf(pdf, (i + 0.25) / n, False) == pdf[i]
    # outer half bins: nearest, no wrap-around
    assert O.sample_pdf(pdf, 0.1 / n, True) == pdf[0]
    assert O.sample_pdf(pdf, 1 - 0.1 / n, True) == pdf[-1]
    # midpoint between two centres
    assert O.sample_pdf(pdf, 1.0 / n, True) == pytest.approx(1.5, rel=1e-6)


@pytest.mark.parametrize("linear", [True, False])
def test_interpolated_pdf_integrates_to_one(linear):
    rng = np.random.default_rng(4)
    n = 32
    pdf = O.softmax_times_n(rng.normal(0, 2, n))
    xs = (np.arange(20000) + 0.5) / 20000
    integral = np.mean([O.sample_pdf(pdf, float(x), linear) for x in xs])
    assert abs(integral - 1.0) < 2e-3


def test_sh_orthonormal():
    rng = np.random.default_rng(5)
    m = 100000
    z = 1 - 2 * rng.random(m)
    phi = 2 * np.pi * rng.random(m)
    r = np.sqrt(1 - z * z)
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    Y = O.sh_encode(4, ((d + 1) * 0.5).astype(np.float32)[:4000])
    G = 4 * np.pi * (Y.T @ Y) / Y.shape[0]
    assert np.abs(G - np.eye(16)).max() < 0.12


def test_oneblob_partition_of_unity():
    x = np.linspace(0, 1, 101).astype(np.float32)
    e = O.oneblob_encode(4, x)
    assert np.allclose(e.sum(1), 1.0, atol=1e-6)
    assert e.min() >= -1e-7


@pytest.mark.parametrize("preset,expected", [(0, 860_160), (1, 14_229_504), (2, 4_133_152)])
def test_grid_parameter_counts(preset, expected):
    import pygdf
    cfg = pygdf.default_config(preset)
    d = O.df_cfg_from(cfg)
    assert O.df_n_params(d, 0) - O.df_mlp_params(d, 0) == expected


def test_grid_trilinear_reproduces_linear_function():
    gc = O.GridCfg(1, 1, 2, 19, 9, 2.0, 0)  # dense, one level, linear
    g = O.grid_tables(gc)
    res = g.resolution[0]
    n_entries = g.offset[1]
    table = np.zeros(n_entries * 2, dtype=np.float32)
    for idx in range(n_entries):
        x, y, z = idx % res, (idx // res) % res, idx // (res * res)
        table[idx * 2] = x + 2 * y + 4 * z
        table[idx * 2 + 1] = 1.0
    rng = np.random.default_rng(6)
    # corners stay inside the level (index wrap-around is a tcnn quirk, tested elsewhere)
    for p in rng.random((200, 3)).astype(np.float32) * 0.9:
        gp = p.astype(np.float64) * g.scale[0] + 0.5
        out = O.grid_encode(g, table, p)
        assert out[0] == pytest.approx(gp[0] + 2 * gp[1] + 4 * gp[2], rel=1e-5)
        assert out[1] == pytest.approx(1.0, rel=1e-6)
