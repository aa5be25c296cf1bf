"""Known-answer tests of the oracle's path-record semantics (CPU).

They pin the oracle to the reference's rules on hand-built single-pixel
states:
  - replaceIndirectRadianceSkipDelta (src/render/guided/workqueue.h:122-129)
    writes thp[d-1] * (nrc + Le[d-1]) into the nearest non-delta record at or
    below d-1, and divideRadiance (workqueue.h:104-111) divides only valid
    records (depth < curDepth) and only channels with nrc > M_EPSILON; all
    applies happen before all divides (two kernels, train.cu:265-308);
  - generate_training_data_AR (train.cu:6-96) skips delta vertices and drops
    records with wiPdf == 0; its target radiance is L / thp * misWeight *
    bsdfVal with channels of thp <= M_EPSILON set to zero;
  - generate_training_data_nrc_with_inference (train.cu:156-214) emits query
    rows for every non-delta, non-miss vertex, training rows for all but the
    last, and decrements curDepth.
"""
import numpy as np

import oracle as O
from pygdf import workload as W

AABB = ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))


def _single_pixel(depth, delta=(), miss=()):
    fields, _ = W.path_state(1, 0, defects=False)
    for d in delta:
        fields["delta"][d, 0] = 1
    for d in range(5):
        if d not in delta:
            fields["delta"][d, 0] = 0
        fields["miss"][d, 0] = 1 if d in miss else 0
    return fields, np.array([depth], np.uint32)


def test_apply_then_divide_known_answer():
    fields, cd = _single_pixel(3, delta=(1,))
    L0 = fields["L"].copy()
    thp, Le = fields["thp"], fields["Le"]
    # query rows at depths 0, 2, 3 (1 is a delta vertex), curDepth already 3
    depth = np.array([0, 2, 3], np.int32)
    pixel = np.zeros(3, np.int32)
    out = np.array([[2.0, 4.0, 1e-6], [0.5, 0.25, 8.0], [3.0, 1.0, 2.0]], np.float32)
    O.apply_nrc(fields, cd, out, depth, pixel)
    f32 = np.float32
    exp0 = thp[1, 0] * (out[1] + Le[1, 0])           # row d=2: d-1 = 1 is delta -> record 0
    exp2 = thp[2, 0] * (out[2] + Le[2, 0])           # row d=3: record 2
    exp0 = np.where(out[0] > f32(1e-5), exp0 / out[0], exp0)   # divide record 0 by row d=0
    exp2 = np.where(out[1] > f32(1e-5), exp2 / out[1], exp2)   # divide record 2 by row d=2
    np.testing.assert_array_equal(fields["L"][0, 0], exp0.astype(np.float32))
    np.testing.assert_array_equal(fields["L"][2, 0], exp2.astype(np.float32))
    np.testing.assert_array_equal(fields["L"][1, 0], L0[1, 0])  # delta record untouched
    np.testing.assert_array_equal(fields["L"][3, 0], L0[3, 0])  # depth 3 >= curDepth: invalid


def test_df_records_skip_delta_and_zero_pdf():
    fields, cd = _single_pixel(4, delta=(1,))
    fields["wi_pdf"][2, 0] = 0.0
    fields["thp"][3, 0, 1] = 1e-6
    a, b, t = O.build_df_records(fields, cd, AABB, 1, 0, 1, 32, True)
    assert a.shape[0] == 2                     # depths 0 and 3
    L = fields["L"][3, 0] / fields["thp"][3, 0]
    L[1] = 0.0
    L = L * fields["mis_weight"][3, 0] * fields["bsdf_val"][3, 0]
    np.testing.assert_array_equal(t[1, 2:5], L.astype(np.float32))
    assert t[1, 5] == fields["wi_pdf"][3, 0]
    np.testing.assert_array_equal(b[:, :9], a)


def test_nrc_rows_and_depth_decrement():
    fields, cd = _single_pixel(4, delta=(0,), miss=(3,))
    r = O.build_nrc_records(fields, cd, AABB, 1, 0, 1, True)
    np.testing.assert_array_equal(r["q_depth"], [1, 2])  # 0 delta, 3 miss
    assert r["t_in"].shape[0] == 2                         # d < depth - 1 = 3
    assert cd[0] == 3
    cd0 = np.array([0], np.uint32)
    O.build_nrc_records(fields, cd0, AABB, 1, 0, 1, False)
    assert cd0[0] == 0xFFFFFFFF                            # unsigned decrement, as the reference


def test_records_ordered_by_pixel_then_depth():
    fields, cd = W.path_state(300, 4, defects=False)
    r = O.build_nrc_records(fields, cd.copy(), AABB, 300, 0, 1, False)
    key = r["q_pixel"].astype(np.int64) * 8 + r["q_depth"]
    assert np.all(np.diff(key) > 0)
