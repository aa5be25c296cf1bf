"""Pins the oracle to the reference's own code, bit for bit.

oracle/_ref/libgdf_refpin.so is src/render/guided/train.h (with AR.h,
parameters.h, guideditem.h, workqueue.h) from the reference tree compiled
for the host, built by oracle/build_ref.py. Each test feeds identical inputs
to a reference function and to its oracle restatement and requires identical
float results. Skipped when the reference tree is not available.
"""
import ctypes as C

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


# --------------------------------------------------------------------------
# train.cu / train.h / AR.h / workqueue.h helpers, compiled from the reference
# tree for the host (the kernels run as host loops over the thread index).

from pygdf import workload as W  # noqa: E402

AABB = ((-2.0, -1.0, -3.0), (4.0, 2.0, 1.0))


def _aabb6():
    return np.asarray(list(AABB[0]) + list(AABB[1]), np.float32)


def _shading(n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(AABB[0], np.float32), np.asarray(AABB[1], np.float32)
    pos = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    wo = rng.normal(size=(n, 3)).astype(np.float32) * rng.uniform(0.2, 3.0, (n, 1)).astype(np.float32)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    rough = rng.exponential(0.5, n).astype(np.float32)
    return pos, wo, nrm, rough


def test_generate_inference_data_bit_exact():
    """generate_inference_data_AR (train.cu:334-362): normalizeSpatialCoord,
    warp_direction_for_sh, cartesianToSphericalNormalized of the normal,
    warp_roughness_for_ob (train.h:272-276, 1243-1249)."""
    n = 20000
    pos, wo, nrm, rough = _shading(n, 1)
    # axis-aligned and pole normals, zero roughness
    nrm[:6] = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float32)
    rough[:3] = 0.0
    a = np.full((n, 9), np.nan, np.float32)
    b = np.full((n, 10), np.nan, np.float32)
    REF.ref_generate_inference_data(O._p(pos), O._p(wo), O._p(nrm), O._p(rough), n, O._p(_aabb6()), O._p(a),
                                    O._p(b))
    q = O.prepare_queries(pos, wo, nrm, rough, AABB)
    assert np.array_equal(a.view(np.uint32), q.view(np.uint32))
    assert np.array_equal(b[:, :9].view(np.uint32), q.view(np.uint32))
    w = np.empty((n, 7), np.float32)
    REF.ref_input_warps(O._p(pos), O._p(wo), O._p(rough), n, O._p(_aabb6()), O._p(w))
    assert np.array_equal(w[:, :3], q[:, :3])
    # warp_direction_for_sh takes the direction as given: (wo + 1) / 2
    assert np.array_equal(w[:, 3:6], ((wo + np.float32(1)) * np.float32(0.5)).astype(np.float32))
    assert np.array_equal(w[:, 6], q[:, 8])


def test_autoregressive_view_bit_exact():
    """AutoRegressive::pdf / sample (AR.h:25-48) with squareToUniformSphere
    (math_utils.h:226-231), the consumer view of a guiding record."""
    rng = np.random.default_rng(2)
    n = 50000
    wi = np.empty((n, 4), np.float32)
    wi[:, :2] = rng.random((n, 2), dtype=np.float32)
    wi[:, 2:] = rng.exponential(1.0, (n, 2)).astype(np.float32)
    wi[:4, :2] = [[0, 0], [1 - 1e-5, 1 - 1e-5], [0.5, 0.25], [1, 1]]
    a = np.empty((n, 4), np.float32)
    REF.ref_autoregressive(O._p(wi), n, O._p(a))
    b = O.autoregressive(wi)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def _path_arrays(n, seed, defects=True):
    fields, depth = W.path_state(n, seed, aabb=AABB, defects=defects)
    fields = {k: np.ascontiguousarray(v) for k, v in fields.items()}
    return fields, depth


@pytest.mark.parametrize("offset,stride", [(0, 1), (3, 2)])
def test_generate_training_data_bit_exact(offset, stride):
    """generate_training_data_AR (train.cu:6-96) with the reference's 16 theta
    bins: record inputs, the phi net's theta condition and GuidedOutput,
    invalid records dropped; records in thread order (pixel, then depth)."""
    n_px = 6000
    fields, depth = _path_arrays(n_px, 3)
    n_train = (n_px - offset) // stride
    cap = n_train * 5
    ra = np.empty((cap, 9), np.float32)
    rb = np.empty((cap, 10), np.float32)
    rt = np.empty((cap, 9), np.float32)
    d_ref = depth.copy()  # the struct holds raw pointers: keep the arrays alive
    s = O._paths(fields, d_ref)
    k = REF.ref_generate_training_data(C.byref(s), O._p(_aabb6()), n_train, offset, stride, O._p(ra), O._p(rb),
                                       O._p(rt), cap)
    oa, ob, ot = O.build_df_records(fields, depth.copy(), AABB, n_train, offset, stride, 16, True)
    assert k == oa.shape[0] and k > 0.5 * n_train
    assert np.array_equal(ra[:k].view(np.uint32), oa.view(np.uint32))
    assert np.array_equal(rb[:k].view(np.uint32), ob.view(np.uint32))
    assert np.array_equal(rt[:k].view(np.uint32), ot.view(np.uint32))


@pytest.mark.parametrize("with_training", [1, 0])
def test_generate_nrc_records_bit_exact(with_training):
    """generate_training_data_nrc_with_inference / generate_NRCinput_from_
    training_data (train.cu:156-262): NRC query rows with (depth, pixel),
    training rows and targets, and the depth counters decremented."""
    n_px = 5000
    fields, depth = _path_arrays(n_px, 4)
    cap = n_px * 5
    q = np.empty((cap, 15), np.float32)
    qd = np.empty(cap, np.int32)
    qp = np.empty(cap, np.int32)
    ti = np.empty((cap, 15), np.float32)
    tt = np.empty((cap, 3), np.float32)
    counts = (C.c_int64 * 2)()
    d_ref = depth.copy()
    s = O._paths(fields, d_ref)
    REF.ref_generate_nrc_records(C.byref(s), O._p(_aabb6()), n_px, 0, 1, with_training, O._p(q), O._p(qd), O._p(qp),
                                 cap, O._p(ti), O._p(tt), cap, counts)
    d_or = depth.copy()
    r = O.build_nrc_records(fields, d_or, AABB, n_px, 0, 1, bool(with_training))
    kq, kt = counts[0], counts[1]
    assert kq == r["q_in"].shape[0] and kt == r["t_in"].shape[0] and kq > n_px
    assert np.array_equal(q[:kq].view(np.uint32), r["q_in"].view(np.uint32))
    assert np.array_equal(qd[:kq], r["q_depth"]) and np.array_equal(qp[:kq], r["q_pixel"])
    assert np.array_equal(ti[:kt].view(np.uint32), r["t_in"].view(np.uint32))
    assert np.array_equal(tt[:kt].view(np.uint32), r["t_target"].view(np.uint32))
    assert np.array_equal(d_ref, d_or)


def test_nrc_substitution_bit_exact():
    """apply_NRCoutput_to_training_data + divide_training_data_by_NRCoutput
    (train.cu:265-308, OPTIMIZE_ON_NRC = 4) through
    replaceIndirectRadianceSkipDelta / divideRadiance (workqueue.h:113-136)."""
    n_px = 4000
    fields, depth = _path_arrays(n_px, 5, defects=False)
    depth = depth - 1  # after the producer's decrement
    r = O.build_nrc_records({k: v.copy() for k, v in fields.items()}, (depth + 1).astype(np.uint32), AABB, n_px,
                            0, 1, True)
    m = r["q_depth"].shape[0]
    rng = np.random.default_rng(6)
    out = rng.exponential(1.0, (m, 3)).astype(np.float32)
    out[rng.random((m, 3)) < 0.05] = 1e-6  # below M_EPSILON: divideRadiance leaves the channel
    f_ref = {k: v.copy() for k, v in fields.items()}
    f_or = {k: v.copy() for k, v in fields.items()}
    d_ref, d_or = depth.astype(np.uint32), depth.astype(np.uint32)
    s = O._paths(f_ref, d_ref)
    REF.ref_apply_nrc(C.byref(s), O._p(out), O._p(r["q_depth"]), O._p(r["q_pixel"]), m)
    O.apply_nrc(f_or, d_or, out, r["q_depth"], r["q_pixel"])
    assert not np.array_equal(f_ref["L"], fields["L"])
    assert np.array_equal(f_ref["L"].view(np.uint32), f_or["L"].view(np.uint32))


@pytest.mark.parametrize("preset", [0, 1])
def test_cpu_baseline_equals_oracle_fp32_path(preset):
    """The CPU baseline bench.py times (oracle/ref_cpu.cpp: the reference's
    thetaPostInference / phiPostInference compiled for the host after the
    oracle's fp32 encodings and MLP forward) gives the oracle fp32 path's
    guiding data bit for bit."""
    import pygdf
    from gdf_testutil import gen_weights
    cfg = pygdf.default_config(preset)
    d = O.df_cfg_from(cfg)
    if not O.refcpu_available(cfg.n_bins_theta, cfg.n_bins_phi):
        pytest.skip("CPU baseline library not built")
    pt, pp = O.round_f16(gen_weights(cfg, 0, 3)), O.round_f16(gen_weights(cfg, 1, 4))
    n = 3000
    q = W.queries(n, 1)
    wi, g = W.wi_init(n, 1, 0.8, 0.2)
    u = W.uniforms(n, 1)
    a = O.refcpu_infer(d, pt, pp, q, wi, g, u, 4)
    b = O.infer_fp32(d, pt, pp, q, wi, g, u, 4)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
