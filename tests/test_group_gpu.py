"""Grouped inference (gdf_group_infer): every job of a grouped call gets
exactly what gdf_infer gives it alone -- same guiding data bit for bit --
for jobs with their own weights, mixed bin counts (32 and 64), ragged
wavefronts, with and without caller uniforms and guided masks; on the
first call (autotuning on scratch copies) and on later calls that reuse the
captured graph with other job sizes."""
import numpy as np
import pytest
import torch

import pygdf
from gdf_testutil import dev, make_ctx
from pygdf import workload as W

pytestmark = pytest.mark.gpu


def _contexts():
    ctxs = []
    for k in range(6):
        bins = 64 if k % 2 == 0 else 32
        ctx, _, _ = make_ctx(pygdf.PRESET_FULL, seed=100 + k, n_bins_theta=bins, n_bins_phi=bins)
        ctxs.append(ctx)
    return ctxs


def _jobs(ctxs, sizes, seed):
    jobs = []
    for k, (ctx, n) in enumerate(zip(ctxs, sizes)):
        q = W.queries(n, seed + k)
        wi, guided = W.wi_init(n, seed + k, guided_frac=0.7, one_sided_frac=0.2)
        j = {"ctx": ctx, "queries": dev(q), "wi": dev(wi), "wi0": wi, "n": n,
             "seed": 11 + k, "offset": 3 * k}
        if k % 3 == 1:
            j["uniforms"] = dev(W.uniforms(n, seed + k))
        if k % 3 != 2:
            j["guided"] = dev(guided)
        jobs.append(j)
    return jobs


def _check(jobs):
    for j in jobs:
        ref = dev(j["wi0"])
        j["ctx"].infer(j["queries"], ref, guided=j.get("guided"), uniforms=j.get("uniforms"),
                       seed=j["seed"], offset=j["offset"])
        torch.cuda.synchronize()
        np.testing.assert_array_equal(j["wi"].cpu().numpy(), ref.cpu().numpy())


def test_group_equals_separate_calls():
    ctxs = _contexts()
    g = pygdf.Group(max_jobs=16)
    jobs = _jobs(ctxs, [20000, 14000, 129, 9800, 1, 6860], seed=40)
    g.infer(jobs)
    g.sync()
    wgs, fb, ms = g.tuning()
    assert wgs in (2, 4) and fb in (128, 256) and (ms > 0).all()
    _check(jobs)
    # other sizes, same signature bucket or not: graphs are reused or built
    jobs = _jobs(ctxs, [16384, 127, 9000, 4802, 3361, 255], seed=70)
    g.infer(jobs)
    g.sync()
    _check(jobs)
    jobs = _jobs(ctxs[:3], [5000, 0, 700], seed=90)
    g.infer(jobs)
    g.sync()
    _check(jobs)
    g.close()
    for c in ctxs:
        c.close()


def test_sm_cap_keeps_results_across_plans():
    """A capped fused launch gives the same rows. The cap is applied to each
    captured graph when it is replayed; the plan with 64-bin jobs (the most
    shared memory) is replayed capped after a plan of 32-bin jobs only was
    captured, which must not invalidate its launch."""
    ctxs = _contexts()
    g = pygdf.Group(max_jobs=16)
    g.set_shape(4, 256)
    big = _jobs(ctxs, [9000, 7000, 5000, 3000, 2000, 1000], seed=70)
    g.infer(big)
    small = _jobs(ctxs[1::2], [4000, 3000, 2000], seed=80)  # 32-bin jobs only
    g.infer(small)
    g.sync()
    _check(big)
    _check(small)
    for cap in (20, 1, 0):
        g.set_sm_cap(cap)
        again = _jobs(ctxs, [9000, 7000, 5000, 3000, 2000, 1000], seed=90 + cap)
        g.infer(again)
        g.sync()
        _check(again)
    with pytest.raises(pygdf.GdfError):
        g.set_sm_cap(-1)
    g.close()
    for c in ctxs:
        c.close()


def test_job_done_flags():
    """gdf_group_job_done: off by default; with tracking on, after a call
    has finished every job reports done; a new call's jobs start over (its
    flags carry the new call's number), an empty job is done at once, and
    indexes outside the last call are not."""
    ctxs = _contexts()
    g = pygdf.Group(max_jobs=16)
    g.set_shape(4, 256)
    g.infer(_jobs(ctxs[:1], [1000], seed=110))
    g.sync()
    assert not g.job_done(0)
    g.track_jobs(True)
    jobs = _jobs(ctxs, [1000, 30000, 0, 5000], seed=120)
    g.infer(jobs)
    g.sync()
    assert all(g.job_done(k) for k in range(4))
    assert not g.job_done(4) and not g.job_done(-1)
    again = _jobs(ctxs[:2], [70000, 2000], seed=130)
    g.infer(again)
    g.sync()
    assert g.job_done(0) and g.job_done(1) and not g.job_done(2)
    _check(jobs)
    _check(again)
    g.close()
    for c in ctxs:
        c.close()
