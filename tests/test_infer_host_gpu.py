"""gdf_infer_host (host buffers, chunked pipeline over two streams) returns
exactly what gdf_infer returns on the same data: the grid features and the
in-kernel Philox counters continue across chunks."""
import numpy as np
import pytest
import torch

import pygdf
from gdf_testutil import dev
from pygdf import workload as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,with_uniforms", [(300001, False), (131072, True), (77, False)])
def test_infer_host_equals_infer(n, with_uniforms):
    cfg = pygdf.default_config(pygdf.PRESET_FULL)
    ctx = pygdf.Context(cfg)
    q = W.queries(n, 21)
    wi0, guided = W.wi_init(n, 22, guided_frac=0.75, one_sided_frac=0.25)
    uni = W.uniforms(n, 23) if with_uniforms else None
    wi_d = dev(wi0)
    ctx.infer(dev(q), wi_d, guided=dev(guided), uniforms=dev(uni) if uni is not None else None,
              seed=5, offset=9)
    torch.cuda.synchronize()
    qp = torch.from_numpy(q).pin_memory()
    gp = torch.from_numpy(guided).pin_memory()
    up = torch.from_numpy(uni).pin_memory() if uni is not None else None
    wp = torch.from_numpy(wi0.copy()).pin_memory()
    out = torch.empty_like(wp).pin_memory()
    ctx.infer_host(qp, wp, out, guided=gp, uniforms=up, seed=5, offset=9)
    ctx.sync()
    np.testing.assert_array_equal(out.numpy(), wi_d.cpu().numpy())
    ctx.close()
