"""Pins the oracle to the reference's own code, bit for bit.

oracle/_ref/libgdf_refpin.so is src/render/guided/train.h (with AR.h,
parameters.h, guideditem.h, workqueue.h) from the reference tree compiled
for the host, built by oracle/build_ref.py. Each test feeds identical inputs
to a reference function and to its oracle restatement and requires identical
float results. Skipped when the reference tree is not available.
"""
import numpy as np
import pytest

import oracle as O

REF = O.ref_lib()
pytestmark = pytest.mark.skipif(REF is None, reason="reference tree not available to build the pin")


def _tables(rng, n_rows, n, scale=2.5):
    return [O.softmax_times_n(rng.normal(0, scale, n)) for _ in range(n_rows)]


@pytest.mark.parametrize("n", [16, 32, 64])
def test_softmax_times_n_bit_exact(n):
    rng = np.random.default_rng(n)
    for _ in range(300):
        z = rng.normal(0, 4, n).astype(np.float32)
        a = z.copy()
        b = z.copy()
        assert REF.ref_softmax_times_n(O._p(a), n) == 0
        O.lib().go_softmax2_times_n(O._p(b), n)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def _edge_pdfs(n, rng):
    """Uniform, one-hot, nearly flat (|A| around the 1e-5 threshold), and
    zero-mass bins (CDF ties and the fallback uniform)."""
    out = [np.ones(n, np.float32)]
    z = np.full(n, -30.0)
    z[rng.integers(n)] = 30.0
    out.append(O.softmax_times_n(z))
    flat = np.ones(n, np.float32)
    flat[1::2] += np.float32(1e-5) * rng.uniform(0.5, 3.0, n // 2).astype(np.float32)
    out.append(flat)
    sparse = np.zeros(n, np.float32)
    sparse[rng.integers(n, size=3)] = np.float32(n) / 3
    out.append(sparse)
    return out


@pytest.mark.parametrize("n", [16, 32, 64])
@pytest.mark.parametrize("is_theta", [1, 0])
def test_inversion_sampling_bit_exact(n, is_theta):
    rng = np.random.default_rng(100 + n + is_theta)
    tables = _tables(rng, 200, n) + _edge_pdfs(n, rng)
    for pdf in tables:
        for u, u2 in rng.random((20, 2), dtype=np.float32):
            pdf32 = O.f32(pdf)
            ref = REF.ref_sample_dir(O._p(pdf32), n, is_theta, float(u), float(u2))
            _, got, _ = O.sample_dir(pdf, True, float(u), float(u2))
            assert np.float32(ref).view(np.uint32) == np.float32(got).view(np.uint32), (n, u, u2, ref, got)


@pytest.mark.parametrize("n", [16, 32, 64])
def test_pdf_interpolation_bit_exact(n):
    rng = np.random.default_rng(200 + n)
    for pdf in _tables(rng, 100, n):
        for u in np.concatenate([rng.random(30, dtype=np.float32), [0.0, 1e-7, 0.5 / n, 1 - 1e-5]]):
            for is_theta in (1, 0):
                pdf32 = O.f32(pdf)
                ref = REF.ref_sample_pdf(O._p(pdf32), float(u), n, is_theta)
                got = O.sample_pdf(pdf, float(u), True)
                assert np.float32(ref) == np.float32(got), (u, ref, got)


def test_theta_condition_bit_exact():
    rng = np.random.default_rng(3)
    for u in np.concatenate([rng.random(2000, dtype=np.float32), [0.0, 1 - 1e-5, 0.5, 1 / 16]]):
        ref = REF.ref_theta_condition16(float(u))
        got = O.lib().go_theta_condition(float(u), 16, 1)
        assert np.float32(ref) == np.float32(got)


@pytest.mark.parametrize("n", [16, 32, 64])
def test_logit_gradients_bit_exact(n):
    rng = np.random.default_rng(300 + n)
    for pdf in _tables(rng, 150, n):
        tab16 = pdf.astype(np.float16)
        bits = tab16.view(np.uint16)
        u, other = rng.random(2, dtype=np.float32)
        prefix = np.float32(-rng.uniform(0.01, 50.0))
        out_ref = np.zeros(n, np.uint16)
        for is_theta in (1, 0):
            assert REF.ref_grads_linear(float(u), float(other), float(prefix), O._p(bits), n, is_theta,
                                        O._p(out_ref)) == 0
            out = np.zeros(n, np.float32)
            tab32 = tab16.astype(np.float32)  # keep the array alive across the call
            O.lib().go_dlogits(O._p(tab32), n, 1, float(u), float(other), float(prefix), O._p(out))
            assert np.array_equal(out_ref.view(np.float16).astype(np.float32), out)


def test_divergence_loss_and_gradients_bit_exact():
    """combine_AR_pdf_and_dl_doutput with the reference's 16 / 32 bins."""
    rng = np.random.default_rng(7)
    n = 512
    tt = np.stack(_tables(rng, n, 16)).astype(np.float16)
    tp = np.stack(_tables(rng, n, 32)).astype(np.float16)
    target = np.empty((n, 9), np.float32)
    target[:, 0:2] = rng.random((n, 2), dtype=np.float32)
    target[:, 2:5] = rng.random((n, 3), dtype=np.float32) * 3
    target[:, 5] = rng.uniform(0.01, 1.0, n).astype(np.float32)
    target[:, 6:9] = 1.0
    dlt_ref = np.zeros((n, 16), np.uint16)
    dlp_ref = np.zeros((n, 32), np.uint16)
    lik_ref = np.zeros(n, np.float32)
    REF.ref_combine(O._p(target), n, O._p(tt.view(np.uint16)), O._p(tp.view(np.uint16)), O._p(dlt_ref),
                    O._p(dlp_ref), O._p(lik_ref), 1024.0)
    dlt = np.zeros((n, 16), np.float32)
    dlp = np.zeros((n, 32), np.float32)
    lik = np.zeros(n, np.float32)
    tt32, tp32 = tt.astype(np.float32), tp.astype(np.float32)  # alive across the call
    O.lib().go_combine(O._p(target), n, O._p(tt32), 16, O._p(tp32), 32, 1, 1024.0, O._p(dlt), O._p(dlp),
                       O._p(lik))
    assert np.array_equal(lik_ref.view(np.uint32), lik.view(np.uint32))
    assert np.array_equal(dlt_ref.view(np.float16).astype(np.float32), dlt)
    assert np.array_equal(dlp_ref.view(np.float16).astype(np.float32), dlp)
