"""The request server (gdf_server_*): each result is the same alone and in
the mix. Two instances serve inference requests and two train (one step and
three steps), all submitted interleaved so that grouped inference launches
and training steps overlap on the device; then the same per-instance
sequences run directly on fresh copies of the instances. Inference results
must be identical bit for bit; a first training step's loss is identical,
later ones within 1e-4 relative (they see weights updated by the earlier
steps). After one step the MLP matrices are identical; grid gradients are
summed with float atomics in no fixed order and Adam normalises each step,
so a near-zero gradient whose sum changes sign moves its weight by up to the
learning rate: grid weights must mostly agree within 1e-5 relative, and
every weight within 2 x lr per step."""
import numpy as np
import pytest
import torch

import pygdf
from gdf_testutil import dev, make_ctx
from pygdf import workload as W

pytestmark = pytest.mark.gpu

SIZES = [3000, 17000, 512, 9000, 25000, 1000]


def _instances():
    return [make_ctx(pygdf.PRESET_SMALL, seed=200 + k)[0] for k in range(4)]


def _infer_requests():
    reqs = []
    for k in range(2):
        for i, n in enumerate(SIZES):
            q = W.queries(n, 10 * k + i)
            wi, guided = W.wi_init(n, 10 * k + i, guided_frac=0.8, one_sided_frac=0.2)
            reqs.append(dict(inst=k, q=q, wi=wi, guided=guided, seed=k + 1, offset=i))
    return reqs


# training steps of instances 2 and 3: one step shows what a step alone
# changes, three show the drift after steps that saw other grid weights
TRAIN_STEPS = (1, 3)


def _train_batches(cfg):
    return [[W.training_batch(16384, 50 + 7 * k + s, cfg.n_bins_theta) for s in range(TRAIN_STEPS[k])]
            for k in range(2)]


@pytest.mark.parametrize("reserve", [0, 32])
def test_results_same_alone_and_in_the_mix(reserve):
    """reserve > 0: training's persistent kernels run on (SMs - reserve) CTAs
    and inference beside a training step on `reserve` CTAs. Rows do not
    depend on the CTA count; the MLP gradient partials are reduced over a
    different number of CTAs, which the weight criteria below absorb."""
    insts = _instances()
    cfg = insts[0].cfg
    budget = sum(pygdf.ctx_bytes(c) for c in insts) + (1 << 30)
    srv = pygdf.Server(budget, slots=4, max_batch=8, train_sm_reserve=reserve)
    for c in insts:
        srv.add_instance(c)
    ireqs = _infer_requests()
    tb = _train_batches(cfg)
    # interleave: inference of instances 0/1 and training of instances 2/3
    order = []
    for i in range(len(SIZES)):
        order += [("i", i), ("i", len(SIZES) + i)]
        if i < 3:
            order += [("t", (k, i)) for k in range(2) if i < TRAIN_STEPS[k]]
    tickets, outs, keep = [], {}, []
    for kind, key in order:
        if kind == "i":
            r = ireqs[key]
            wi_d = dev(r["wi"])
            q_d, g_d = dev(r["q"]), dev(r["guided"])
            keep += [q_d, g_d]
            outs[("i", key)] = wi_d
            tickets.append((("i", key), srv.submit_infer(insts[r["inst"]], q_d, wi_d, guided=g_d,
                                                         seed=r["seed"], offset=r["offset"])))
        else:
            k, s = key
            a, b, t = (dev(x) for x in tb[k][s])
            keep += [a, b, t]
            tickets.append((("t", key), srv.submit_train(insts[2 + k], a, b, t)))
    losses = {}
    for key, t in tickets:
        st, lat = srv.wait(t)
        assert lat > 0
        if key[0] == "t":
            losses[key[1]] = st.loss
    stats = srv.stats()
    assert stats.requests == len(tickets) and stats.p50_ms <= stats.p99_ms
    srv.close()
    mix_params = [insts[2 + k].get_params(n) for k in range(2) for n in (0, 1)]

    # alone: fresh instances with the same initial weights, direct calls;
    # the training sequences run twice alone to measure run-to-run spread
    alone = _instances()
    for key, _ in tickets:
        if key[0] == "i":
            r = ireqs[key[1]]
            wi_d = dev(r["wi"])
            alone[r["inst"]].infer(dev(r["q"]), wi_d, guided=dev(r["guided"]), seed=r["seed"], offset=r["offset"])
            torch.cuda.synchronize()
            np.testing.assert_array_equal(outs[key].cpu().numpy(), wi_d.cpu().numpy())
        else:
            k, s = key[1]
            a, b, t = (dev(x) for x in tb[k][s])
            st = alone[2 + k].train_step(a, b, t)
            if s == 0:  # no earlier step: the forward has no atomics, the loss is exact
                assert st.loss == losses[(k, s)], (st.loss, losses[(k, s)])
            else:  # measured on a B200: up to 2.4e-5 relative
                assert abs(st.loss - losses[(k, s)]) <= 1e-4 * abs(st.loss), (st.loss, losses[(k, s)])
    again = _instances()[2:]
    for k in range(2):
        for s in range(TRAIN_STEPS[k]):
            again[k].train_step(*(dev(x) for x in tb[k][s]))
    alone_params = [alone[2 + k].get_params(n) for k in range(2) for n in (0, 1)]
    again_params = [again[k].get_params(n) for k in range(2) for n in (0, 1)]
    lr = cfg.adam_df.learning_rate
    import oracle as O
    d = O.df_cfg_from(cfg)

    def agree(x, y, rtol=1e-5):
        return np.isclose(x, y, rtol=rtol, atol=rtol * 1e-2).mean()

    for i, (x, y, z) in enumerate(zip(mix_params, alone_params, again_params)):
        n_mlp = O.df_mlp_params(d, i % 2)
        mlp, grid = slice(0, n_mlp), slice(n_mlp, None)
        if i < 2:
            # one step from the same weights: the MLP gradients are per-CTA
            # partials reduced in a fixed order, so the matrices are identical
            # on the same CTA count and differ by the reduction order alone
            # on another (reserve > 0); the grid gradient is a float-atomic
            # sum in no fixed order, which Adam's normalisation makes visible
            # only where it is near zero
            if reserve == 0:
                np.testing.assert_array_equal(x[mlp], y[mlp])
            else:
                assert agree(x[mlp], y[mlp], 1e-6) >= 0.999, agree(x[mlp], y[mlp], 1e-6)
            assert agree(x[grid], y[grid]) >= 0.97, agree(x[grid], y[grid])
        else:
            # after the first step every weight depends on grid weights that
            # the float-atomic order changed: measured on a B200, 0.80 to 1.0
            # of the matrices' and 0.97 to 1.0 of the grid tables' weights
            # agree, between the mix and a run alone and between two runs
            # alone alike. Weights of the wrong instance agree on ~none.
            for part in (mlp, grid):
                a_mix, a_rep = agree(x[part], y[part]), agree(z[part], y[part])
                print(f"net {i} {'mlp' if part is mlp else 'grid'}: mix {a_mix:.4f}, two runs alone {a_rep:.4f}")
                assert a_mix >= 0.6 and a_rep >= 0.6, (a_mix, a_rep)
        # near-zero gradients whose float-atomic sum changed sign move a
        # weight by at most about lr per Adam step
        assert np.abs(x - y).max() <= 2 * TRAIN_STEPS[i // 2] * lr, np.abs(x - y).max()
    for c in insts + alone + again:
        c.close()


def test_budget_is_enforced():
    insts = _instances()[:2]
    one = pygdf.ctx_bytes(insts[0])
    srv = pygdf.Server(one + (1 << 20), slots=2, max_batch=4)
    srv.add_instance(insts[0])
    with pytest.raises(pygdf.GdfError):
        srv.add_instance(insts[1])
    q = dev(W.queries(1 << 16, 3))
    wi = dev(W.wi_init(1 << 16, 3)[0])
    with pytest.raises(pygdf.GdfError):          # 64K queries need 8 MiB of feature tiles
        srv.submit_infer(insts[0], q, wi)
    srv.close()
    for c in insts:
        c.close()


def test_sm_reserve_is_validated():
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for bad in (-1, sms):
        with pytest.raises(pygdf.GdfError):
            pygdf.Server(1 << 30, slots=2, max_batch=4, train_sm_reserve=bad)
    pygdf.Server(1 << 30, slots=2, max_batch=4, train_sm_reserve=sms - 1).close()


def test_training_orders_the_inference_of_its_instance():
    """Per instance: inference requests before a training request see the
    weights before it, those after see the weights after it, and inference
    requests between two training requests may run together. Before the
    first step the results equal the same sequence run directly bit for
    bit; after it the weights carry the step's float-atomic grid sums, so
    at least 99 % of the rows must agree; and the last request, a repeat of
    the first, must see other weights than the first."""
    insts = _instances()[:1]
    c = insts[0]
    srv = pygdf.Server(pygdf.ctx_bytes(c) + (1 << 30), slots=4, max_batch=8)
    srv.add_instance(c)
    reqs = _infer_requests()[:4]
    batch = _train_batches(c.cfg)[1][:2]
    seq = [("i", 0), ("i", 1), ("t", 0), ("i", 2), ("i", 3), ("t", 1), ("i", 0)]
    outs, tickets, keep = [], [], []
    for kind, k in seq:
        if kind == "i":
            r = reqs[k]
            wi_d, q_d, g_d = dev(r["wi"]), dev(r["q"]), dev(r["guided"])
            keep += [q_d, g_d]
            outs.append(wi_d)
            tickets.append(srv.submit_infer(c, q_d, wi_d, guided=g_d, seed=r["seed"], offset=r["offset"]))
        else:
            a, b, t = (dev(x) for x in batch[k])
            keep += [a, b, t]
            outs.append(None)
            tickets.append(srv.submit_train(c, a, b, t))
    for t in tickets:
        srv.wait(t)
    srv.close()
    alone = _instances()[0]
    trained = False
    for (kind, k), got in zip(seq, outs):
        if kind == "i":
            r = reqs[k]
            wi_d = dev(r["wi"])
            alone.infer(dev(r["q"]), wi_d, guided=dev(r["guided"]), seed=r["seed"], offset=r["offset"])
            torch.cuda.synchronize()
            x, y = got.cpu().numpy(), wi_d.cpu().numpy()
            if not trained:
                np.testing.assert_array_equal(x, y)
            else:
                same = np.all(x == y, axis=1).mean()
                assert same >= 0.99, same
        else:
            alone.train_step(*(dev(x) for x in batch[k]))
            trained = True
    first, last = outs[0].cpu().numpy(), outs[-1].cpu().numpy()
    guided = reqs[0]["guided"].astype(bool)
    assert np.all(first[guided] == last[guided], axis=1).mean() < 0.5
    c.close()
    alone.close()
