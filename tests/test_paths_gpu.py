"""GPU parity of the path-record stages against the oracle:

* gdf_prepare_queries / gdf_infer_ex(shading): generate_inference_data_AR
  (src/render/guided/train.cu:334-362);
* gdf_build_train_records: generate_training_data_AR (train.cu:6-96);
* gdf_build_nrc_records: generate_training_data_nrc_with_inference and
  generate_NRCinput_from_training_data (train.cu:156-262);
* gdf_apply_nrc / gdf_nrc_substitute_paths: apply + divide of the NRC
  output (train.cu:265-308, workqueue.h:100-129);
* gdf_train_paths / gdf_nrc_train_paths: the frame-level batch loops
  (learnedDistribution.cpp:208-293, nrc.cpp:114-170);
* gdf_infer_ex(dir_pdf): the AutoRegressive consumer view (AR.h:25-48).

Tolerances: values made only of +,-,*,/ and sqrt are compared bit-exactly
(the kernels are compiled without FMA contraction, the oracle with
-ffp-contract=off); values through sinf/cosf/acosf/atan2f/expf, where CUDA's
functions and the host libm may differ by an ulp or two, within 2e-6
absolute (all such values lie in [0, 1] or [-1, 1]). Record counts, order,
depths and pixel ids are exact.
"""
import numpy as np
import pytest
import torch

import oracle as O
import pygdf
from gdf_testutil import dev
from pygdf import workload as W

pytestmark = pytest.mark.gpu

AABB = ((-2.0, -1.0, -3.0), (4.0, 2.0, 1.0))
TOL = 2e-6


def _state_dev(fields, depth):
    f = {k: dev(np.ascontiguousarray(v)) for k, v in fields.items()}
    cd = dev(depth.view(np.int32).copy())
    return f, cd, pygdf.path_state(f, cd)


def _host(t):
    return t.cpu().numpy()


def _ctx(preset=pygdf.PRESET_SMALL, **kw):
    cfg = pygdf.default_config(preset)
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg, pygdf.Context(cfg)


def _px(n, offset=0, stride=1):
    return pygdf.TrainPixels(n, offset, stride)


def test_prepare_queries_matches_oracle():
    rng = np.random.default_rng(0)
    n = 10000
    pos = (np.array(AABB[0]) + (np.array(AABB[1]) - np.array(AABB[0])) * rng.random((n, 3))).astype(np.float32)
    wo = (rng.normal(size=(n, 3)) * 3).astype(np.float32)       # not unit length
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    rough = rng.random(n, dtype=np.float32) * 2
    q = dev(np.zeros((n, 9), np.float32))
    pygdf.prepare_queries(pygdf.shading(dev(pos), dev(wo), dev(nrm), dev(rough)),
                          pygdf.Aabb.of(*AABB), q)
    torch.cuda.synchronize()
    got = _host(q)
    ref = O.prepare_queries(pos, wo, nrm, rough, AABB)
    np.testing.assert_array_equal(got[:, :6], ref[:, :6])
    np.testing.assert_allclose(got[:, 6:], ref[:, 6:], rtol=0, atol=TOL)


@pytest.mark.parametrize("offset,stride", [(0, 1), (2, 3)])
@pytest.mark.parametrize("linear", [True, False])
def test_build_train_records_match_oracle(offset, stride, linear):
    fields, depth = W.path_state(7000, 11)
    cfg, ctx = _ctx(pdf_interp=pygdf.PDF_LINEAR if linear else pygdf.PDF_NEAREST)
    f, cd, st = _state_dev(fields, depth)
    px = _px(7000, offset, stride)
    n_train = 7000 // stride
    cap = n_train * 5
    a, b, t = (dev(np.zeros((cap, k), np.float32)) for k in (9, 10, 9))
    k = ctx.build_train_records(st, pygdf.Aabb.of(*AABB), px, a, b, t)
    ra, rb, rt = O.build_df_records(fields, depth.copy(), AABB, n_train, offset, stride,
                                    cfg.n_bins_theta, linear)
    assert k == ra.shape[0] and k > 0
    ga, gb, gt = _host(a)[:k], _host(b)[:k], _host(t)[:k]
    np.testing.assert_array_equal(ga[:, :3], ra[:, :3])
    np.testing.assert_allclose(ga[:, 3:], ra[:, 3:], rtol=0, atol=TOL)
    np.testing.assert_array_equal(gb[:, :9], ga)
    np.testing.assert_allclose(gb[:, 9], rb[:, 9], rtol=0, atol=TOL)
    np.testing.assert_allclose(gt[:, :2], rt[:, :2], rtol=0, atol=TOL)
    np.testing.assert_array_equal(gt[:, 2:], rt[:, 2:])
    assert not np.isnan(ga).any() and not np.isnan(gt).any()
    ctx.close()


def test_build_train_records_capacity_is_enforced():
    fields, depth = W.path_state(500, 2)
    _, ctx = _ctx()
    _, _, st = _state_dev(fields, depth)
    cap = 10
    a, b, t = (dev(np.zeros((cap, k), np.float32)) for k in (9, 10, 9))
    with pytest.raises(pygdf.GdfError):
        ctx.build_train_records(st, pygdf.Aabb.of(*AABB), _px(500), a, b, t)
    ctx.close()


@pytest.mark.parametrize("with_training", [True, False])
def test_build_nrc_records_match_oracle(with_training):
    fields, depth = W.path_state(6000, 12)
    _, ctx = _ctx()
    f, cd, st = _state_dev(fields, depth)
    cap = 6000 * 5
    qi, ti = dev(np.zeros((cap, 15), np.float32)), dev(np.zeros((cap, 15), np.float32))
    qd, qp = (dev(np.zeros(cap, np.int32)) for _ in range(2))
    tt = dev(np.zeros((cap, 3), np.float32))
    kq, kt = ctx.build_nrc_records(st, pygdf.Aabb.of(*AABB), _px(6000), with_training, qi, qd, qp,
                                   ti, tt)
    rdepth = depth.copy()
    r = O.build_nrc_records(fields, rdepth, AABB, 6000, 0, 1, with_training)
    assert kq == r["q_in"].shape[0] and kt == r["t_in"].shape[0]
    assert kq > 0 and (kt > 0) == with_training
    np.testing.assert_array_equal(_host(qd)[:kq], r["q_depth"])
    np.testing.assert_array_equal(_host(qp)[:kq], r["q_pixel"])
    g = _host(qi)[:kq]
    np.testing.assert_array_equal(g[:, :3], r["q_in"][:, :3])
    np.testing.assert_allclose(g[:, 3:9], r["q_in"][:, 3:9], rtol=0, atol=TOL)
    np.testing.assert_array_equal(g[:, 9:], r["q_in"][:, 9:])
    if with_training:
        np.testing.assert_allclose(_host(ti)[:kt], r["t_in"], rtol=0, atol=TOL)
        np.testing.assert_array_equal(_host(tt)[:kt], r["t_target"])
    np.testing.assert_array_equal(_host(cd).view(np.uint32), rdepth)
    ctx.close()


def test_apply_nrc_matches_oracle():
    fields, depth = W.path_state(5000, 13, defects=False)
    _, ctx = _ctx()
    f, cd, st = _state_dev(fields, depth)
    r = O.build_nrc_records(fields, depth, AABB, 5000, 0, 1, True)   # depth decremented
    cd.copy_(torch.from_numpy(depth.view(np.int32)).cuda())
    m = r["q_depth"].shape[0]
    rng = np.random.default_rng(5)
    out = rng.exponential(1.0, (m, 3)).astype(np.float32)
    out[rng.random((m, 3)) < 0.05] = 1e-6                              # below M_EPSILON: no divide
    ctx.apply_nrc(st, dev(out), dev(r["q_depth"]), dev(r["q_pixel"]))
    torch.cuda.synchronize()
    O.apply_nrc(fields, depth, out, r["q_depth"], r["q_pixel"])
    np.testing.assert_array_equal(_host(f["L"]), fields["L"])
    ctx.close()


def _nrc_rows_dev(ctx, fields, depth, n_pixels):
    """GPU-built NRC rows of a fresh device copy of the state."""
    _, _, st = _state_dev(fields, depth)
    cap = n_pixels * 5
    qi, ti = dev(np.zeros((cap, 15), np.float32)), dev(np.zeros((cap, 15), np.float32))
    qd, qp = (dev(np.zeros(cap, np.int32)) for _ in range(2))
    tt = dev(np.zeros((cap, 3), np.float32))
    kq, kt = ctx.build_nrc_records(st, pygdf.Aabb.of(*AABB), _px(n_pixels), True, qi, qd, qp, ti, tt)
    return qi[:kq], qd[:kq], qp[:kq], ti[:kt], tt[:kt]


def test_nrc_train_then_substitute_matches_oracle():
    """NRC::trainStep followed by inferenceStepFromTrainingData on the rows it
    built (the integrator's OPTIMIZE_ON_NRC = 4 order, integrator.cpp:1202-1232)."""
    # no injected defects: a zero wiPdf turns into a 1e5 x NRC target
    # (train.cu:197), which overflows the fp16 loss gradient as in tcnn
    fields, depth = W.path_state(60000, 14, defects=False)
    cfg, ctx = _ctx(min_train_batch=8192)
    f, cd, st = _state_dev(fields, depth)
    qi, qd, qp, ti, _ = _nrc_rows_dev(ctx, fields, depth, 60000)
    loss, n = ctx.nrc_train_paths(st, pygdf.Aabb.of(*AABB), _px(60000))
    rdepth = depth.copy()
    r = O.build_nrc_records(fields, rdepth, AABB, 60000, 0, 1, True)
    assert n == r["t_in"].shape[0] == ti.shape[0]
    np.testing.assert_array_equal(_host(cd).view(np.uint32), rdepth)
    assert np.isfinite(loss) and loss > 0
    # outputs of the trained NRC on the same rows the library built
    out = dev(np.zeros((qi.shape[0], 3), np.float32))
    ctx.nrc_query(qi, out)
    torch.cuda.synchronize()
    ctx.nrc_substitute_paths(st, pygdf.Aabb.of(*AABB), _px(60000), skip_generation=True)
    O.apply_nrc(fields, rdepth, _host(out), _host(qd), _host(qp))
    np.testing.assert_array_equal(_host(f["L"]), fields["L"])
    ctx.close()


def test_nrc_train_paths_batch_loop():
    """nrc.cpp:129-168: batches = max(n / bs + 1, batchPerFrame), effective
    size min(n / batches, bs) rounded down to 128, row offset iter * local,
    loss = sum / batches."""
    fields, depth = W.path_state(70000, 15, defects=False)
    cfg, ctx = _ctx(nrc_batches_per_frame=2, min_train_batch=8192)
    _, ctx2 = _ctx(nrc_batches_per_frame=2, min_train_batch=8192)
    _, _, st = _state_dev(fields, depth)
    loss, n = ctx.nrc_train_paths(st, pygdf.Aabb.of(*AABB), _px(70000))
    _, _, _, ti, tt = _nrc_rows_dev(ctx2, fields, depth, 70000)
    assert n == ti.shape[0]
    bs = cfg.nrc_batch_size
    batches = max(n // bs + 1, 2)
    eff = min(n // batches, bs)
    exp = 0.0
    for it in range(batches):
        local = min(n - it * eff, eff)
        local -= local % 128
        if local < cfg.min_train_batch:
            break
        exp += ctx2.nrc_train_step(ti[it * local:], tt[it * local:], n=local).loss
    exp /= batches
    assert exp > 0
    assert abs(loss - exp) <= 1e-6 * exp, (loss, exp)
    ctx.close()
    ctx2.close()


def test_train_paths_batch_loop():
    """learnedDistribution.cpp:227-290: batches = min(n / bs + 1,
    batchPerFrame), batch i at row i * bs, size rounded down to 128, stop
    below MIN_TRAIN_BATCH_SIZE, loss = sum / batches."""
    fields, depth = W.path_state(60000, 16)
    cfg, ctx = _ctx()
    _, ctx2 = _ctx()
    _, _, st = _state_dev(fields, depth)
    loss, n = ctx.train_paths(st, pygdf.Aabb.of(*AABB), _px(60000))
    cap = 60000 * 5
    a, b, t = (dev(np.zeros((cap, k), np.float32)) for k in (9, 10, 9))
    k = ctx2.build_train_records(st, pygdf.Aabb.of(*AABB), _px(60000), a, b, t)
    assert k == n and n > 2 * cfg.df_batch_size
    bs = cfg.df_batch_size
    batches = min(n // bs + 1, cfg.df_batches_per_frame)
    exp, used = 0.0, 0
    for it in range(batches):
        local = min(n - it * bs, bs)
        local -= local % 128
        if local < cfg.min_train_batch:
            break
        o = it * bs
        exp += ctx2.train_step(a[o:], b[o:], t[o:], n=local).loss
        used += 1
    exp /= batches
    assert used >= 2
    assert abs(loss - exp) <= 1e-5 * abs(exp), (loss, exp)
    ctx.close()
    ctx2.close()


def test_train_paths_async_captures_into_a_graph():
    """gdf_train_paths_async keeps the record count on the device, so the
    frame's producer and batch loop capture into one CUDA graph. Each replay
    trains a frame: its loss and record count equal gdf_train_paths' on a
    context with the same weights (batches after the first see grid weights
    whose gradients were summed by float atomics: 1e-5 relative), and only
    the batches the loop reaches take an optimizer step."""
    fields, depth = W.path_state(60000, 16)
    cfg, ctx = _ctx()
    _, ctx2 = _ctx()
    _, _, st = _state_dev(fields, depth)
    box, px = pygdf.Aabb.of(*AABB), _px(60000)
    init = [ctx.get_params(k) for k in (0, 1)]
    loss_d = torch.zeros(1, dtype=torch.float32, device="cuda")
    n_d = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.train_paths_async(st, box, px, loss_d, n_d)  # allocates the frame buffers
    torch.cuda.synchronize()
    for k in (0, 1):  # back to the initial weights and optimizer state
        ctx.set_params(k, init[k])
        z = np.zeros(init[k].size, np.float32)
        ctx.set_optimizer_state(k, z, z, np.zeros(init[k].size, np.uint32), 0)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
            ctx.train_paths_async(st, box, px, loss_d, n_d, stream=s)
    torch.cuda.synchronize()
    loss_ref, n_ref = ctx2.train_paths(st, box, px)
    bs = cfg.df_batch_size
    batches = min(n_ref // bs + 1, cfg.df_batches_per_frame)
    used = 0
    for it in range(batches):
        local = min(n_ref - it * bs, bs)
        if local - local % 128 < cfg.min_train_batch:
            break
        used += 1
    assert 2 <= used < cfg.df_batches_per_frame  # launched batches that train nothing are covered
    for frame in (1, 2):
        g.replay()
        torch.cuda.synchronize()
        assert int(n_d.item()) == n_ref
        for k in (0, 1):
            assert ctx.get_optimizer_state(k)[3] == frame * used
        if frame == 1:
            loss = float(loss_d.item())
            assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref), (loss, loss_ref)
            assert ctx2.get_optimizer_state(0)[3] == used
    del g
    ctx.close()
    ctx2.close()


def test_train_paths_below_min_batch_trains_nothing():
    """A frame with fewer records than min_train_batch: the batch loop breaks
    at once (learnedDistribution.cpp:232-233), so the weights and the
    optimizer step stay as they were and the loss is 0 / batches = 0."""
    fields, depth = W.path_state(2000, 17)
    cfg, ctx = _ctx()
    _, _, st = _state_dev(fields, depth)
    before = [ctx.get_params(k) for k in (0, 1)]
    loss, n = ctx.train_paths(st, pygdf.Aabb.of(*AABB), _px(2000))
    assert 0 < n < cfg.min_train_batch and loss == 0.0
    for k in (0, 1):
        np.testing.assert_array_equal(ctx.get_params(k), before[k])
        assert ctx.get_optimizer_state(k)[3] == 0
    ctx.close()


def test_infer_ex_shading_equals_prepared_queries():
    cfg, ctx = _ctx(pygdf.PRESET_FULL)
    rng = np.random.default_rng(3)
    n = 50000
    pos = (np.array(AABB[0]) + (np.array(AABB[1]) - np.array(AABB[0])) * rng.random((n, 3))).astype(np.float32)
    wo = rng.normal(size=(n, 3)).astype(np.float32)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    rough = rng.random(n, dtype=np.float32)
    sh = pygdf.shading(dev(pos), dev(wo), dev(nrm), dev(rough))
    box = pygdf.Aabb.of(*AABB)
    q = dev(np.zeros((n, 9), np.float32))
    pygdf.prepare_queries(sh, box, q)
    wi0 = W.wi_init(n, 4, guided_frac=0.8, one_sided_frac=0.2)[0]
    w_a, w_b = dev(wi0), dev(wi0)
    ctx.infer(q, w_a, seed=9, offset=2)
    ctx.infer_ex(w_b, shading=sh, aabb=box, seed=9, offset=2)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_host(w_a), _host(w_b))
    ctx.close()


def test_infer_ex_dir_pdf_is_the_autoregressive_view():
    cfg, ctx = _ctx(pygdf.PRESET_FULL)
    n = 40000
    q = dev(W.queries(n, 5))
    wi0, guided = W.wi_init(n, 6, guided_frac=0.7, one_sided_frac=0.3)
    wi = dev(wi0)
    dp = dev(np.zeros((n, 4), np.float32))
    ctx.infer_ex(wi, queries=q, guided=dev(guided), seed=1, offset=0, dir_pdf=dp)
    torch.cuda.synchronize()
    w, d = _host(wi), _host(dp)
    # the oracle's AutoRegressive view, bit-exact to AR.h:25-48 compiled from
    # the reference (test_reference_pin.py): squareToUniformSphere and
    # pdf = |pt| |pp| / (4 pi); directions within the sinf/cosf difference
    # between the GPU and the host C library
    ref = O.autoregressive(w)
    np.testing.assert_array_equal(d[:, 3], ref[:, 0])
    np.testing.assert_allclose(d[:, :3], ref[:, 1:], rtol=0, atol=4e-6)
    np.testing.assert_allclose(np.linalg.norm(d[:, :3], axis=1), 1.0, atol=4e-6)
    ctx.close()


@pytest.mark.parametrize("kind", ["df", "nrc"])
def test_dense_paths_match_oracle(kind):
    """Every pixel five vertices deep, no delta or miss vertices: each warp
    emits 160 records, more than the producer stages in shared memory, so
    the direct-write path is exercised too."""
    fields, depth = W.path_state(4000, 17, defects=False)
    fields["delta"][:] = 0
    fields["miss"][:] = 0
    depth[:] = 5
    cfg, ctx = _ctx()
    f, cd, st = _state_dev(fields, depth)
    cap = 4000 * 5
    if kind == "df":
        a, b, t = (dev(np.zeros((cap, k), np.float32)) for k in (9, 10, 9))
        k = ctx.build_train_records(st, pygdf.Aabb.of(*AABB), _px(4000), a, b, t)
        ra, rb, rt = O.build_df_records(fields, depth.copy(), AABB, 4000, 0, 1, cfg.n_bins_theta, True)
        assert k == ra.shape[0] == cap
        np.testing.assert_allclose(_host(a), ra, rtol=0, atol=TOL)
        np.testing.assert_allclose(_host(b), rb, rtol=0, atol=TOL)
        np.testing.assert_allclose(_host(t), rt, rtol=0, atol=TOL)
    else:
        qi, ti = dev(np.zeros((cap, 15), np.float32)), dev(np.zeros((cap, 15), np.float32))
        qd, qp = (dev(np.zeros(cap, np.int32)) for _ in range(2))
        tt = dev(np.zeros((cap, 3), np.float32))
        kq, kt = ctx.build_nrc_records(st, pygdf.Aabb.of(*AABB), _px(4000), True, qi, qd, qp, ti, tt)
        r = O.build_nrc_records(fields, depth.copy(), AABB, 4000, 0, 1, True)
        assert kq == cap and kt == 4000 * 4
        np.testing.assert_array_equal(_host(qd), r["q_depth"])
        np.testing.assert_array_equal(_host(qp), r["q_pixel"])
        np.testing.assert_allclose(_host(qi), r["q_in"], rtol=0, atol=TOL)
        np.testing.assert_allclose(_host(ti)[:kt], r["t_in"], rtol=0, atol=TOL)
        np.testing.assert_array_equal(_host(tt)[:kt], r["t_target"])
    ctx.close()
