"""Python driver of the C oracle (oracle/gdf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker. The product never imports it.

The shared object is built on demand with gcc into oracle/_build/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
SO = os.path.join(BUILD, "libgdf_oracle.so")
SRCS = [os.path.join(HERE, "gdf_oracle.c"), os.path.join(HERE, "gdf_oracle_train.c"),
        os.path.join(HERE, "gdf_oracle_paths.c")]
HDR = os.path.join(HERE, "gdf_oracle.h")


def build(force: bool = False) -> str:
    srcs = [s for s in SRCS if os.path.exists(s)]
    newest = max(os.path.getmtime(p) for p in srcs + [HDR])
    if not force and os.path.exists(SO) and os.path.getmtime(SO) >= newest:
        return SO
    os.makedirs(BUILD, exist_ok=True)
    tmp = SO + ".tmp"
    cmd = ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
           "-shared", "-o", tmp, *srcs, "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, SO)
    return SO


class GridCfg(C.Structure):
    _fields_ = [("type", C.c_int32), ("n_levels", C.c_int32), ("n_features_per_level", C.c_int32),
                ("log2_hashmap_size", C.c_int32), ("base_resolution", C.c_int32),
                ("per_level_scale", C.c_float), ("interpolation", C.c_int32)]


class DfCfg(C.Structure):
    _fields_ = [("n_bins_theta", C.c_int32), ("n_bins_phi", C.c_int32), ("pdf_interp", C.c_int32),
                ("grid_theta", GridCfg), ("grid_phi", GridCfg), ("sh_degree", C.c_int32),
                ("oneblob_bins", C.c_int32), ("tw_frequencies", C.c_int32), ("width", C.c_int32),
                ("hidden_theta", C.c_int32), ("hidden_phi", C.c_int32)]


class NrcCfg(C.Structure):
    _fields_ = [("frequencies", C.c_int32), ("oneblob_bins", C.c_int32), ("width", C.c_int32),
                ("hidden", C.c_int32)]


class Grid(C.Structure):
    _fields_ = [("c", GridCfg), ("scale", C.c_float * 24), ("resolution", C.c_uint32 * 24),
                ("offset", C.c_uint32 * 25), ("n_params", C.c_int64)]


_lib = None
P = C.c_void_p


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        for name, args, res in [
            ("go_philox_uniforms", [C.c_uint64, C.c_uint64, C.c_int64, P], None),
            ("go_philox4x32_10", [P, P, P], None),
            ("go_grid_init", [C.POINTER(Grid), C.POINTER(GridCfg)], C.c_int),
            ("go_df_n_params", [C.POINTER(DfCfg), C.c_int], C.c_int64),
            ("go_df_mlp_params", [C.POINTER(DfCfg), C.c_int], C.c_int64),
            ("go_df_input_width", [C.POINTER(DfCfg), C.c_int], C.c_int32),
            ("go_nrc_n_params", [C.POINTER(NrcCfg)], C.c_int64),
            ("go_nrc_input_width", [C.POINTER(NrcCfg)], C.c_int32),
            ("go_df_encode", [C.POINTER(DfCfg), C.POINTER(Grid), C.c_int, P, P, C.c_float, P], None),
            ("go_nrc_encode", [C.POINTER(NrcCfg), P, P], None),
            ("go_sh_encode", [C.c_int, P, P], None),
            ("go_oneblob_encode", [C.c_int, P, C.c_int, P], None),
            ("go_post_inference", [C.POINTER(DfCfg), P, P, P, P, P, P, C.c_int64], None),
            ("go_infer", [C.POINTER(DfCfg), P, P, P, P, P, P, P, C.c_int64, C.c_int], None),
            ("go_infer_fp32", [C.POINTER(DfCfg), P, P, P, P, P, P, C.c_int64, C.c_int], None),
            ("go_eval_pdf", [C.POINTER(DfCfg), P, P, P, P, P, C.c_int64, C.c_int], None),
            ("go_nrc_query", [C.POINTER(NrcCfg), P, P, P, C.c_int64, C.c_int], None),
            ("go_sample_dir", [P, C.c_int, C.c_int, C.c_float, C.c_float, P, P], C.c_int),
            ("go_sample_dir_f64", [P, C.c_int, C.c_int, C.c_double, C.c_double], C.c_double),
            ("go_sample_pdf", [P, C.c_float, C.c_int, C.c_int], C.c_float),
            ("go_softmax2_times_n", [P, C.c_int], None),
            ("go_round_f16", [C.c_double], C.c_float),
            ("go_round_e4m3", [C.c_double], C.c_double),
            ("go_round_bf16", [C.c_float], C.c_float),
            ("go_mlp_forward", [P, C.c_int, C.c_int, C.c_int, C.c_int, P, P, P], None),
            ("go_e4m3_scale_exp", [C.c_double], C.c_int),
            ("go_df_pdf_tables", [C.POINTER(DfCfg), P, P, P, P, P, P, C.c_int64], None),
            ("go_set_accumulation", [C.c_int], None),
            ("go_set_storage", [C.c_int], None),
            ("go_df_train_grads", [C.POINTER(DfCfg), P, P, P, P, P, C.c_int64, C.c_float, P, P, P, P, P, P],
             C.c_int64),
            ("go_dlogits", [P, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, P], None),
            ("go_combine", [P, C.c_int64, P, C.c_int, P, C.c_int, C.c_int, C.c_float, P, P, P], None),
            ("go_theta_condition", [C.c_float, C.c_int, C.c_int], C.c_float),
            ("go_nrc_train_grads", [C.POINTER(NrcCfg), P, P, P, C.c_int64, C.c_float, P, P], None),
            ("go_adam_ema", [C.c_int64, C.c_int64, P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                             C.c_float, C.c_float, C.c_uint32, P, P, P, P, P, P], None),
            ("go_grid_encode", [C.POINTER(Grid), P, P, P], None),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def df_cfg_from(cfg) -> DfCfg:
    """gdf_config (pygdf.Config) -> oracle config."""
    d = DfCfg()
    d.n_bins_theta, d.n_bins_phi, d.pdf_interp = cfg.n_bins_theta, cfg.n_bins_phi, cfg.pdf_interp
    for dst, src in ((d.grid_theta, cfg.grid_theta), (d.grid_phi, cfg.grid_phi)):
        for f, _ in GridCfg._fields_:
            setattr(dst, f, getattr(src, f))
    d.sh_degree, d.oneblob_bins, d.tw_frequencies = cfg.sh_degree, cfg.oneblob_bins, cfg.tw_frequencies
    d.width = cfg.mlp_theta.n_neurons
    d.hidden_theta, d.hidden_phi = cfg.mlp_theta.n_hidden_layers, cfg.mlp_phi.n_hidden_layers
    return d


def nrc_cfg_from(cfg) -> NrcCfg:
    n = NrcCfg()
    n.frequencies, n.oneblob_bins = cfg.nrc_frequencies, cfg.nrc_oneblob_bins
    n.width, n.hidden = cfg.mlp_nrc.n_neurons, cfg.mlp_nrc.n_hidden_layers
    return n


def round_f16(a) -> np.ndarray:
    return np.asarray(a, dtype=np.float32).astype(np.float16).astype(np.float32)


def philox_uniforms(seed: int, offset: int, n: int) -> np.ndarray:
    out = np.empty((n, 4), dtype=np.float32)
    lib().go_philox_uniforms(seed, offset, n, _p(out))
    return out


def philox_block(ctr, key) -> list[int]:
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.empty(4, dtype=np.uint32)
    lib().go_philox4x32_10(_p(c), _p(k), _p(o))
    return [int(x) for x in o]


def df_n_params(d: DfCfg, net: int) -> int:
    return int(lib().go_df_n_params(C.byref(d), net))


def df_mlp_params(d: DfCfg, net: int) -> int:
    return int(lib().go_df_mlp_params(C.byref(d), net))


STORAGE = {"fp16": 0, "bf16": 1, "none": 2, "fp8": 3}


def round_bf16(a) -> np.ndarray:
    """Round to nearest even bf16, as cvt.rn.bf16.f32."""
    x = np.ascontiguousarray(a, dtype=np.float32).copy()
    u = x.view(np.uint32)
    fin = (u & 0x7F800000) != 0x7F800000
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    u[fin] = r[fin].astype(np.uint32)
    return x


def df_weights(d: DfCfg, net: int, params, storage: str = "fp16") -> np.ndarray:
    """Inference weights of one DF network: the fp16 EMA copy; in bf16 the
    MLP matrices are that copy rounded to bf16 (the grid tables stay fp16)."""
    w = round_f16(params)
    if storage == "bf16":
        m = df_mlp_params(d, net)
        w[:m] = round_bf16(w[:m])
    return w


class _storage:
    def __init__(self, fmt: str):
        self.fmt = STORAGE[fmt]

    def __enter__(self):
        lib().go_set_storage(self.fmt)

    def __exit__(self, *exc):
        lib().go_set_storage(0)


def infer(d: DfCfg, p_theta, p_phi, queries, wi, guided=None, uniforms=None, n_threads=0,
          edge_gap=False, storage: str = "fp16"):
    """gdf_infer restated; params are fp32 and rounded to the inference
    format here (fp16 EMA copy, bf16 MLP matrices in the bf16 form)."""
    pt, pp = df_weights(d, 0, p_theta, storage), df_weights(d, 1, p_phi, storage)
    q = f32(queries)
    w = f32(wi).copy()
    g = None if guided is None else np.ascontiguousarray(guided, dtype=np.uint8)
    u = f32(uniforms)
    n = q.shape[0]
    gap = np.empty((n, 2), dtype=np.float32) if edge_gap else None
    with _storage(storage):
        lib().go_infer(C.byref(d), _p(pt), _p(pp), _p(q), _p(g), _p(u), _p(w), _p(gap), n, n_threads)
    return (w, gap) if edge_gap else w


def infer_fp32(d: DfCfg, p_theta16, p_phi16, queries, wi, guided, uniforms, n_threads=0):
    w = f32(wi).copy()
    n = queries.shape[0]
    lib().go_infer_fp32(C.byref(d), _p(p_theta16), _p(p_phi16), _p(queries), _p(guided),
                        _p(uniforms), _p(w), n, n_threads)
    return w


def eval_pdf(d: DfCfg, p_theta, p_phi, queries, u, n_threads=0, storage: str = "fp16",
             weights: str | None = None):
    """pdfs at given directions; `storage` rounds the activations, `weights`
    (default: storage) selects the weight format."""
    wf = storage if weights is None else weights
    pt, pp = df_weights(d, 0, p_theta, wf), df_weights(d, 1, p_phi, wf)
    q, uu = f32(queries), f32(u)
    out = np.empty((q.shape[0], 2), dtype=np.float32)
    with _storage(storage):
        lib().go_eval_pdf(C.byref(d), _p(pt), _p(pp), _p(q), _p(uu), _p(out), q.shape[0], n_threads)
    return out


def mlp_forward(w16, k0: int, width: int, n_hidden: int, n_out_pad: int, x16, storage: str = "fp16"):
    """One row through go_mlp_forward: w16 the MLP matrices (row-major,
    back to back), x16 the k0 encoded inputs; returns the n_out_pad logits."""
    w, x = f32(w16), f32(x16)
    out = np.empty(n_out_pad, dtype=np.float32)
    with _storage(storage):
        lib().go_mlp_forward(_p(w), k0, width, n_hidden, n_out_pad, _p(x), _p(out), None)
    return out


def post_inference(d: DfCfg, lt, lp, uniforms, wi, guided=None, edge_gap=False):
    lt, lp, u = f32(lt), f32(lp), f32(uniforms)
    w = f32(wi).copy()
    g = None if guided is None else np.ascontiguousarray(guided, dtype=np.uint8)
    gap = np.empty((lt.shape[0], 2), dtype=np.float32)
    lib().go_post_inference(C.byref(d), _p(lt), _p(lp), _p(g), _p(u), _p(w), _p(gap), lt.shape[0])
    return (w, gap) if edge_gap else w


def post_inference_tables(d: DfCfg, table_theta, table_phi, uniforms, wi, guided=None):
    """thetaPostInference / phiPostInference (train.h:896-929) from given pdf
    tables (softmax x N already applied): guided rows sample u_theta from
    uniforms[:, 0:2] and u_phi from uniforms[:, 2:4]; every row's pdfs at its
    directions multiply into wi[:, 2:4]."""
    lin = d.pdf_interp == 0
    w = f32(wi).copy()
    u = f32(uniforms)
    for i in range(w.shape[0]):
        if guided is None or guided[i]:
            w[i, 0] = sample_dir(table_theta[i], lin, float(u[i, 0]), float(u[i, 1]))[1]
            w[i, 1] = sample_dir(table_phi[i], lin, float(u[i, 2]), float(u[i, 3]))[1]
        w[i, 2] *= np.float32(sample_pdf(table_theta[i], float(w[i, 0]), lin))
        w[i, 3] *= np.float32(sample_pdf(table_phi[i], float(w[i, 1]), lin))
    return w


def nrc_query(nc: NrcCfg, params, inp, n_threads=0):
    p = round_f16(params)
    x = f32(inp)
    out = np.empty((x.shape[0], 3), dtype=np.float32)
    lib().go_nrc_query(C.byref(nc), _p(p), _p(x), _p(out), x.shape[0], n_threads)
    return out


def df_encode(d: DfCfg, net: int, params, q, theta_cond=0.0) -> np.ndarray:
    g = Grid()
    lib().go_grid_init(C.byref(g), C.byref(d.grid_theta if net == 0 else d.grid_phi))
    pr = round_f16(params)
    k0 = int(lib().go_df_input_width(C.byref(d), net))
    out = np.empty(k0, dtype=np.float32)
    qq = f32(q)
    lib().go_df_encode(C.byref(d), C.byref(g), net, _p(pr), _p(qq), theta_cond, _p(out))
    return out


def grid_tables(gc: GridCfg) -> Grid:
    g = Grid()
    lib().go_grid_init(C.byref(g), C.byref(gc))
    return g


def sh_encode(degree: int, dirs01: np.ndarray) -> np.ndarray:
    out = np.empty((dirs01.shape[0], degree * degree), dtype=np.float64)
    for i in range(dirs01.shape[0]):
        v = f32(dirs01[i])
        lib().go_sh_encode(degree, _p(v), _p(out[i]))
    return out


def oneblob_encode(n_bins: int, x: np.ndarray) -> np.ndarray:
    x = f32(x)
    out = np.empty(x.shape[0] * n_bins, dtype=np.float64)
    lib().go_oneblob_encode(n_bins, _p(x), x.shape[0], _p(out))
    return out.reshape(x.shape[0], n_bins)


def sample_dir(pdf, linear: bool, u: float, u2: float):
    p = f32(pdf)
    d = np.zeros(1, dtype=np.float32)
    gap = np.zeros(1, dtype=np.float32)
    seg = lib().go_sample_dir(_p(p), p.size, int(linear), u, u2, _p(d), _p(gap))
    return int(seg), float(d[0]), float(gap[0])


def sample_pdf(pdf, u: float, linear: bool) -> float:
    p = f32(pdf)
    return float(lib().go_sample_pdf(_p(p), u, p.size, int(linear)))


def softmax_times_n(v) -> np.ndarray:
    a = f32(v).copy()
    lib().go_softmax2_times_n(_p(a), a.size)
    return a


def round_f16_scalar(x: float) -> float:
    return float(lib().go_round_f16(float(x)))


def grid_encode(g: Grid, table, pos) -> np.ndarray:
    t = f32(table)
    p = f32(pos)
    out = np.empty(g.c.n_levels * g.c.n_features_per_level, dtype=np.float64)
    lib().go_grid_encode(C.byref(g), _p(t), _p(p), _p(out))
    return out


def pdf_tables(d: DfCfg, p_theta, p_phi, queries, u_theta, storage: str = "fp16"):
    pt, pp = df_weights(d, 0, p_theta, storage), df_weights(d, 1, p_phi, storage)
    q, ut = f32(queries), f32(u_theta)
    n = q.shape[0]
    a = np.empty((n, d.n_bins_theta), dtype=np.float32)
    b = np.empty((n, d.n_bins_phi), dtype=np.float32)
    with _storage(storage):
        lib().go_df_pdf_tables(C.byref(d), _p(pt), _p(pp), _p(q), _p(ut), _p(a), _p(b), n)
    return a, b


def df_train_grads(d: DfCfg, w_theta, w_phi, in_theta, in_phi, target, loss_scale=1024.0,
                   storage: str = "fp16"):
    """Gradients (scaled by loss_scale, FP64) of one DF training batch; the
    weights are the fp32 masters, rounded here to the fp16 training copies.
    storage "bf16": the bf16 training form's storage points (MLP matrices
    bf16(fp16 copy), encoded inputs, activations, dL/dlogits and backward
    activations in bf16; the pdf tables stay fp16)."""
    wt, wp = df_weights(d, 0, w_theta, storage), df_weights(d, 1, w_phi, storage)
    a, b, t = f32(in_theta), f32(in_phi), f32(target)
    n = a.shape[0]
    gt = np.zeros(wt.size, np.float64)
    gp = np.zeros(wp.size, np.float64)
    lik = np.empty(n, np.float32)
    pdf = np.empty((n, 2), np.float32)
    dlt = np.empty((n, d.n_bins_theta), np.float32)
    dlp = np.empty((n, d.n_bins_phi), np.float32)
    with _storage(storage):
        dropped = lib().go_df_train_grads(C.byref(d), _p(wt), _p(wp), _p(a), _p(b), _p(t), n, loss_scale,
                                          _p(gt), _p(gp), _p(lik), _p(pdf), _p(dlt), _p(dlp))
    return dict(grad_theta=gt, grad_phi=gp, likelihood=lik, pdf=pdf, dlog_theta=dlt, dlog_phi=dlp,
                dropped=int(dropped))


def adam_ema(grad_scaled, n_matrix, loss_scale, adam, step, master, ema16, m, v, steps):
    """One Adam + EMA step (adam.h / ema.h); returns updated copies."""
    master = f32(master).copy()
    w16 = round_f16(master)
    ema = f32(ema16).copy()
    m = f32(m).copy()
    v = f32(v).copy()
    steps = np.ascontiguousarray(steps, np.uint32).copy()
    g = np.ascontiguousarray(grad_scaled, np.float64)
    lib().go_adam_ema(master.size, n_matrix, _p(g), loss_scale, adam.learning_rate, adam.beta1, adam.beta2,
                      adam.epsilon, adam.l2_reg, adam.ema_decay, step, _p(master), _p(w16), _p(ema), _p(m),
                      _p(v), _p(steps))
    return master, w16, ema, m, v, steps


REF_SO = os.path.join(HERE, "_ref", "libgdf_refpin.so")
_ref = None


def ref_lib():
    """The reference's own DF functions compiled for the host (oracle/_ref),
    or None when they could not be built (no reference tree)."""
    global _ref
    if _ref is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("build_ref", os.path.join(HERE, "build_ref.py"))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        so = m.build()
        if not so or not os.path.exists(so):
            return None
        L = C.CDLL(so)
        for name, args, res in [
            ("ref_softmax_times_n", [P, C.c_int], C.c_int),
            ("ref_sample_dir", [P, C.c_int, C.c_int, C.c_float, C.c_float], C.c_float),
            ("ref_sample_pdf", [P, C.c_float, C.c_int, C.c_int], C.c_float),
            ("ref_theta_condition16", [C.c_float], C.c_float),
            ("ref_grads_linear", [C.c_float, C.c_float, C.c_float, P, C.c_int, C.c_int, P], C.c_int),
            ("ref_combine", [P, C.c_int64, P, P, P, P, P, C.c_float], None),
            ("ref_input_warps", [P, P, P, C.c_int64, P, P], None),
            ("ref_autoregressive", [P, C.c_int64, P], None),
            ("ref_generate_inference_data", [P, P, P, P, C.c_int64, P, P, P], None),
            ("ref_generate_training_data", [C.c_void_p, P, C.c_int64, C.c_uint32, C.c_uint32, P, P, P,
                                            C.c_int64], C.c_int64),
            ("ref_generate_nrc_records", [C.c_void_p, P, C.c_int64, C.c_uint32, C.c_uint32, C.c_int, P, P, P,
                                          C.c_int64, P, P, C.c_int64, P], None),
            ("ref_apply_nrc", [C.c_void_p, P, P, P, C.c_int64], None),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _ref = L
    return _ref


def nrc_train_grads(nc: NrcCfg, w, inp, target, loss_scale=1024.0):
    """NRC batch: per-record loss values and the FP64 gradient (scaled)."""
    w16 = round_f16(w)
    x, y = f32(inp), f32(target)
    m = x.shape[0]
    g = np.zeros(w16.size, np.float64)
    loss = np.empty(m, np.float32)
    lib().go_nrc_train_grads(C.byref(nc), _p(w16), _p(x), _p(y), m, loss_scale, _p(g), _p(loss))
    return g, loss


# ---- path records (gdf_oracle_paths.c) ------------------------------------

PATH_FIELDS = ["L", "thp", "Le", "pos", "dir", "wi_pdf", "mis_weight", "delta", "miss", "bsdf_val",
               "wo", "normal", "roughness", "diffuse", "specular"]


class GoPaths(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(f, C.c_void_p) for f in PATH_FIELDS] + [("cur_depth", C.c_void_p)]


def _paths(fields: dict, cur_depth: np.ndarray):
    """go_paths over numpy arrays (modified in place by the oracle)."""
    s = GoPaths()
    s.n = cur_depth.shape[0]
    for f in PATH_FIELDS:
        a = fields[f]
        assert a.flags.c_contiguous
        setattr(s, f, a.ctypes.data)
    s.cur_depth = cur_depth.ctypes.data
    return s


def _aabb6(aabb):
    return (C.c_float * 6)(*[float(x) for x in list(aabb[0]) + list(aabb[1])])


def prepare_queries(pos, wo, nrm, rough, aabb):
    n = pos.shape[0]
    q = np.empty((n, 9), np.float32)
    L = lib()
    L.go_prepare_queries.argtypes = [C.c_void_p] * 4 + [C.c_void_p, C.c_void_p, C.c_int64]
    p, w, m, r = f32(pos), f32(wo), f32(nrm), f32(rough)
    L.go_prepare_queries(_p(p), _p(w), _p(m), _p(r), _aabb6(aabb), _p(q), n)
    return q


def build_df_records(fields, cur_depth, aabb, n_train, offset, stride, bins, linear):
    cap = n_train * 5
    a = np.empty((cap, 9), np.float32)
    b = np.empty((cap, 10), np.float32)
    t = np.empty((cap, 9), np.float32)
    L = lib()
    L.go_build_df_records.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_uint32, C.c_uint32,
                                      C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
    L.go_build_df_records.restype = C.c_int64
    s = _paths(fields, cur_depth)
    k = L.go_build_df_records(C.byref(s), _aabb6(aabb), n_train, offset, stride, bins, int(linear),
                              _p(a), _p(b), _p(t), cap)
    return a[:k], b[:k], t[:k]


def build_nrc_records(fields, cur_depth, aabb, n_train, offset, stride, with_training):
    """Returns dict(q_in, q_depth, q_pixel, t_in, t_target); decrements cur_depth in place."""
    cap = n_train * 5
    q = np.empty((cap, 15), np.float32)
    qd = np.empty(cap, np.int32)
    qp = np.empty(cap, np.int32)
    ti = np.empty((cap, 15), np.float32)
    tt = np.empty((cap, 3), np.float32)
    counts = (C.c_int64 * 2)()
    L = lib()
    L.go_build_nrc_records.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_uint32, C.c_uint32,
                                       C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                       C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    s = _paths(fields, cur_depth)
    L.go_build_nrc_records(C.byref(s), _aabb6(aabb), n_train, offset, stride, int(with_training),
                           _p(q), _p(qd), _p(qp), cap, _p(ti), _p(tt), cap, counts)
    kq, kt = counts[0], counts[1]
    return dict(q_in=q[:kq], q_depth=qd[:kq], q_pixel=qp[:kq], t_in=ti[:kt], t_target=tt[:kt])


def apply_nrc(fields, cur_depth, out, depth, pixel):
    """Modifies fields['L'] in place."""
    L = lib()
    L.go_apply_nrc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
    s = _paths(fields, cur_depth)
    o, d, p = f32(out), np.ascontiguousarray(depth, np.int32), np.ascontiguousarray(pixel, np.int32)
    L.go_apply_nrc(C.byref(s), _p(o), _p(d), _p(p), o.shape[0])


_refcpu = {}


def refcpu_available(bins_theta: int, bins_phi: int) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libgdf_refcpu_{bins_theta}x{bins_phi}.so"))


def refcpu_infer(d: DfCfg, p_theta16, p_phi16, queries, wi, guided=None, uniforms=None, n_threads=0):
    """The CPU baseline: the reference's thetaPostInference / phiPostInference
    compiled for the host (oracle/ref_cpu.cpp) after the oracle's fp32
    encodings + MLP forward. Returns the guiding data [n x 4]."""
    key = (d.n_bins_theta, d.n_bins_phi)
    if key not in _refcpu:
        path = os.path.join(HERE, "_ref", f"libgdf_refcpu_{key[0]}x{key[1]}.so")
        L = C.CDLL(path)
        L.refcpu_infer.argtypes = [C.c_void_p, P, P, P, P, P, P, C.c_int64, C.c_int]
        L.refcpu_infer.restype = C.c_int
        _refcpu[key] = L
    q = f32(queries)
    out = f32(wi).copy()
    g = None if guided is None else np.ascontiguousarray(guided, np.uint8)
    u = f32(uniforms)
    rc = _refcpu[key].refcpu_infer(C.byref(d), _p(f32(p_theta16)), _p(f32(p_phi16)), _p(q), _p(g), _p(u),
                                   _p(out), q.shape[0], n_threads)
    if rc != 0:
        raise ValueError("refcpu_infer: configuration differs from the library's bin counts")
    return out


def autoregressive(wi4) -> np.ndarray:
    """AutoRegressive view (AR.h:25-48) of guiding records [n x 4]:
    [n x 4] = (solid-angle pdf, world direction)."""
    w = f32(wi4)
    out = np.empty((w.shape[0], 4), np.float32)
    L = lib()
    L.go_autoregressive.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
    L.go_autoregressive(_p(w), w.shape[0], _p(out))
    return out
