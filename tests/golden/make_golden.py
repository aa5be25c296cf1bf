"""Generates the golden vectors of tests/golden/ from the reference's own GPU
path (tiny-cuda-nn v1.6 + the reference DF kernels, oracle/build_ref_gpu.py),
on a CUDA GPU:

    python tests/golden/make_golden.py [out_dir]

Inputs and weights come from seeded numpy generators (gdf_testutil.gen_weights,
pygdf.workload), so only the reference's outputs are stored; tests/
test_golden.py regenerates the inputs and checks the FP64 oracle against
them on the CPU. Written: reference_<preset>.npz for the 65,536-query
configuration (hash grid 8x2, 32/32 bins) and the reference's own layout
(base_product_df.json: dense grid 8x4 smoothstep, 16/32 bins).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "guiding-df_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

import pygdf  # noqa: E402
import tcnnref as T  # noqa: E402
from gdf_testutil import gen_weights  # noqa: E402
from pygdf import workload as W  # noqa: E402

# Seeds and sizes; tests/test_golden.py reads them from the files.
N_QUERIES, SEED_Q, SEED_W = 512, 5, 11
N_TRAIN, SEED_T = 1024, 7


def main(out_dir: str) -> None:
    import torch
    torch.cuda.set_device(0)
    os.makedirs(out_dir, exist_ok=True)
    for preset, name in ((pygdf.PRESET_SMALL, "small"), (pygdf.PRESET_REFERENCE, "reference")):
        cfg = pygdf.default_config(preset)
        R = T.DfRef(cfg)
        pt, pp = gen_weights(cfg, 0, SEED_W, 1.2, 0.2), gen_weights(cfg, 1, SEED_W + 1, 1.2, 0.2)
        R.set_params(0, pt)
        R.set_params(1, pp)
        q = W.queries(N_QUERIES, SEED_Q)
        wi, guided = W.wi_init(N_QUERIES, SEED_Q, 0.8, 0.2)
        u = W.uniforms(N_QUERIES, SEED_Q)
        wr = torch.from_numpy(wi).cuda()
        R.infer(wr, torch.from_numpy(u).cuda(), queries=torch.from_numpy(q).cuda(),
                guided=torch.from_numpy(guided).cuda())
        torch.cuda.synchronize()
        tt, tp, _ = R.last_pdfs(N_QUERIES)
        a, b, t = W.training_batch(N_TRAIN, SEED_T, cfg.n_bins_theta, cfg.pdf_interp == 0)
        loss, gt, gp, lr = R.train_step(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                                        torch.from_numpy(t).cuda(), step=False, grads=True, per_record=True)
        n_mlp = [_mlp(cfg, k) for k in (0, 1)]
        np.savez_compressed(
            os.path.join(out_dir, f"reference_{name}.npz"),
            preset=preset, n_queries=N_QUERIES, seed_q=SEED_Q, seed_w=SEED_W, n_train=N_TRAIN, seed_t=SEED_T,
            wi=wr.cpu().numpy(), table_theta=tt, table_phi=tp, loss=np.float32(loss), loss_per_record=lr,
            grad_mlp_theta=gt[:n_mlp[0]], grad_mlp_phi=gp[:n_mlp[1]],
            grad_grid_norm=np.array([np.linalg.norm(gt[n_mlp[0]:]), np.linalg.norm(gp[n_mlp[1]:])]))
        R.close()
        print(name, "loss", loss)


def _mlp(cfg, net: int) -> int:
    from gdf_testutil import mlp_dims
    return sum(r * c for r, c in mlp_dims(cfg, net))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
