"""ctypes binding of the gdf C ABI (include/gdf.h) for tests and the bench.

This module only forwards to libgdf_b200.so; it computes nothing itself and
raises if the library is missing, so a missing build can never fall back to
another implementation.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libgdf_b200.so")

GDF_ABI_VERSION = 2
MAX_TRAIN_DEPTH = 5
GDF_OK = 0
STATUS = {0: "OK", 1: "INVALID_ARG", 2: "OOM_BUDGET", 3: "CUDA", 4: "TIMEOUT", 5: "NUMERIC",
          6: "UNSUPPORTED", 7: "STATE"}
PRESET_SMALL, PRESET_FULL, PRESET_REFERENCE = 0, 1, 2
NET_THETA, NET_PHI, NET_NRC = 0, 1, 2
PDF_LINEAR, PDF_NEAREST = 0, 1
PREC_FP16, PREC_BF16, PREC_FP8 = 0, 1, 2


class GridConfig(C.Structure):
    _fields_ = [("type", C.c_int32), ("n_levels", C.c_int32), ("n_features_per_level", C.c_int32),
                ("log2_hashmap_size", C.c_int32), ("base_resolution", C.c_int32),
                ("per_level_scale", C.c_float), ("interpolation", C.c_int32)]


class MlpConfig(C.Structure):
    _fields_ = [("n_neurons", C.c_int32), ("n_hidden_layers", C.c_int32)]


class AdamConfig(C.Structure):
    _fields_ = [("learning_rate", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
                ("epsilon", C.c_float), ("l2_reg", C.c_float), ("ema_decay", C.c_float)]


class Config(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("n_bins_theta", C.c_int32), ("n_bins_phi", C.c_int32),
                ("pdf_interp", C.c_int32), ("grid_theta", GridConfig), ("grid_phi", GridConfig),
                ("sh_degree", C.c_int32), ("oneblob_bins", C.c_int32), ("tw_frequencies", C.c_int32),
                ("mlp_theta", MlpConfig), ("mlp_phi", MlpConfig), ("adam_df", AdamConfig),
                ("loss_scale", C.c_float), ("nrc_enable", C.c_int32), ("nrc_frequencies", C.c_int32),
                ("nrc_oneblob_bins", C.c_int32), ("mlp_nrc", MlpConfig), ("adam_nrc", AdamConfig),
                ("nrc_loss_scale", C.c_float), ("precision", C.c_int32), ("seed", C.c_uint32),
                ("max_queries", C.c_int64), ("max_train_batch", C.c_int64),
                ("df_batch_size", C.c_int64), ("nrc_batch_size", C.c_int64),
                ("min_train_batch", C.c_int64), ("df_batches_per_frame", C.c_int32),
                ("nrc_batches_per_frame", C.c_int32)]


class Aabb(C.Structure):
    _fields_ = [("lo", C.c_float * 3), ("hi", C.c_float * 3)]

    @staticmethod
    def of(lo, hi) -> "Aabb":
        a = Aabb()
        for k in range(3):
            a.lo[k] = float(lo[k])
            a.hi[k] = float(hi[k])
        return a


class Shading(C.Structure):
    _fields_ = [("pos", C.c_void_p), ("wo", C.c_void_p), ("normal", C.c_void_p),
                ("roughness", C.c_void_p)]


# gdf_record_fields member order, with components per pixel and element type
RECORD_FIELDS = [("L", 3, "f4"), ("thp", 3, "f4"), ("Le", 3, "f4"), ("pos", 3, "f4"),
                 ("dir", 2, "f4"), ("wi_pdf", 1, "f4"), ("mis_weight", 1, "f4"),
                 ("delta", 1, "u1"), ("miss", 1, "u1"), ("bsdf_val", 3, "f4"), ("wo", 2, "f4"),
                 ("normal", 2, "f4"), ("roughness", 1, "f4"), ("diffuse", 3, "f4"),
                 ("specular", 3, "f4")]


class RecordFields(C.Structure):
    _fields_ = [(name, C.c_void_p) for name, _, _ in RECORD_FIELDS]


class PathState(C.Structure):
    _fields_ = [("depth", RecordFields * MAX_TRAIN_DEPTH), ("cur_depth", C.c_void_p)]


class TrainPixels(C.Structure):
    _fields_ = [("max_queue_size", C.c_int64), ("offset", C.c_uint32), ("stride", C.c_uint32)]


class InferArgs(C.Structure):
    _fields_ = [("queries_dev", C.c_void_p), ("shading", C.POINTER(Shading)), ("aabb", Aabb),
                ("guided_dev", C.c_void_p), ("uniforms_dev", C.c_void_p),
                ("philox_seed", C.c_uint64), ("philox_offset", C.c_uint64),
                ("wi_dev", C.c_void_p), ("dir_pdf_dev", C.c_void_p), ("n", C.c_int64),
                ("cdf_norm_err_dev", C.c_void_p), ("stage_events", C.c_void_p)]


def path_state(fields: dict, cur_depth) -> PathState:
    """gdf_path_state over device tensors: fields[name] is [depth, pixel(, k)]
    contiguous, cur_depth is [pixel] uint32 (int32 storage)."""
    st = PathState()
    for name, k, _ in RECORD_FIELDS:
        t = fields[name]
        per_depth = t[0].numel() * t.element_size()
        for d in range(MAX_TRAIN_DEPTH):
            setattr(st.depth[d], name, t.data_ptr() + d * per_depth)
    st.cur_depth = cur_depth.data_ptr()
    st._keep = (fields, cur_depth)  # the struct holds raw pointers into these tensors
    return st


class Job(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("queries_dev", C.c_void_p), ("guided_dev", C.c_void_p),
                ("uniforms_dev", C.c_void_p), ("philox_seed", C.c_uint64), ("philox_offset", C.c_uint64),
                ("wi_dev", C.c_void_p), ("n", C.c_int64)]


class Request(C.Structure):
    _fields_ = [("kind", C.c_int32), ("instance", C.c_void_p), ("n", C.c_int64),
                ("queries_dev", C.c_void_p), ("guided_dev", C.c_void_p), ("uniforms_dev", C.c_void_p),
                ("philox_seed", C.c_uint64), ("philox_offset", C.c_uint64), ("wi_dev", C.c_void_p),
                ("in_theta_dev", C.c_void_p), ("in_phi_dev", C.c_void_p), ("target_dev", C.c_void_p)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("slots", C.c_int32), ("max_batch", C.c_int32),
                ("max_train_slots", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("train_sm_reserve", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("requests", C.c_int64), ("queries", C.c_int64), ("pending", C.c_int64),
                ("resident_bytes", C.c_int64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("max_ms", C.c_double), ("queries_per_s", C.c_double)]


class TrainStats(C.Structure):
    _fields_ = [("loss", C.c_double), ("grad_norm", C.c_double), ("n_records", C.c_int64),
                ("n_dropped", C.c_int64)]


class GdfError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"gdf status {STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None
P = C.c_void_p


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libgdf_b200.so not built at {LIB_PATH}; run guiding-df_b200/build.py")
        L = C.CDLL(LIB_PATH)
        sig = {
            "gdf_default_config": [C.c_int32, C.POINTER(Config)],
            "gdf_create": [C.POINTER(Config), C.POINTER(C.c_void_p)],
            "gdf_destroy": [P],
            "gdf_reset_training": [P, C.c_uint32],
            "gdf_n_params": [P, C.c_int32, C.POINTER(C.c_int64)],
            "gdf_set_params": [P, C.c_int32, P, C.c_int64],
            "gdf_get_params": [P, C.c_int32, P, C.c_int64],
            "gdf_get_inference_params": [P, C.c_int32, P, C.c_int64],
            "gdf_save_network": [P, C.c_char_p],
            "gdf_load_network": [P, C.c_char_p],
            "gdf_infer": [P, P, P, P, C.c_uint64, C.c_uint64, P, C.c_int64, P],
            "gdf_eval_pdf": [P, P, P, P, C.c_int64, P],
            "gdf_post_inference": [P, P, P, P, P, P, C.c_int64, P],
            "gdf_train_step": [P, P, P, P, C.c_int64, C.POINTER(TrainStats), P],
            "gdf_nrc_query": [P, P, P, C.c_int64, P],
            "gdf_nrc_train_step": [P, P, P, C.c_int64, C.POINTER(TrainStats), P],
            "gdf_sync_status": [P, P],
            "gdf_get_optimizer_state": [P, C.c_int32, P, P, P, C.c_int64, P],
            "gdf_set_optimizer_state": [P, C.c_int32, P, P, P, C.c_int64, C.c_uint32],
            "gdf_train_loss_static": [P, P, P, P, C.c_int64, P, P, P],
            "gdf_infer_ex": [P, C.POINTER(InferArgs), P],
            "gdf_infer_host": [P, P, P, P, C.c_uint64, C.c_uint64, P, P, C.c_int64, P],
            "gdf_pdf_image": [P, P, C.c_int32, C.c_int32, P, P],
            "gdf_group_create": [C.c_int32, C.POINTER(C.c_void_p)],
            "gdf_group_destroy": [P],
            "gdf_group_infer": [P, P, C.c_int32, P],
            "gdf_group_tuning": [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), P],
            "gdf_group_sync_status": [P, P],
            "gdf_group_set_shape": [P, C.c_int32, C.c_int32],
            "gdf_group_set_sm_cap": [P, C.c_int32],
            "gdf_group_job_done": [P, C.c_int32],
            "gdf_group_track_jobs": [P, C.c_int32],
            "gdf_ctx_bytes": [P, C.POINTER(C.c_int64)],
            "gdf_server_create": [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)],
            "gdf_server_destroy": [P],
            "gdf_server_add_instance": [P, P],
            "gdf_server_submit": [P, C.POINTER(Request), C.POINTER(C.c_uint64)],
            "gdf_server_wait": [P, C.c_uint64, C.POINTER(TrainStats), C.POINTER(C.c_double)],
            "gdf_server_get_stats": [P, C.POINTER(ServerStats), C.c_int32],
            "gdf_sample_histogram": [P, P, C.c_int64, C.c_uint64, C.c_int32, C.c_int32, P, P, P],
            "gdf_prepare_queries": [C.POINTER(Shading), C.POINTER(Aabb), P, C.c_int64, P],
            "gdf_build_train_records": [P, C.POINTER(PathState), C.POINTER(Aabb), C.POINTER(TrainPixels),
                                        P, P, P, C.c_int64, C.POINTER(C.c_int64), P],
            "gdf_build_nrc_records": [P, C.POINTER(PathState), C.POINTER(Aabb), C.POINTER(TrainPixels),
                                      C.c_int32, P, P, P, C.c_int64, P, P, C.c_int64,
                                      C.POINTER(C.c_int64 * 2), P],
            "gdf_apply_nrc": [P, C.POINTER(PathState), P, P, P, C.c_int64, P],
            "gdf_nrc_train_paths": [P, C.POINTER(PathState), C.POINTER(Aabb), C.POINTER(TrainPixels),
                                    C.POINTER(C.c_float), C.POINTER(C.c_int64), P],
            "gdf_nrc_substitute_paths": [P, C.POINTER(PathState), C.POINTER(Aabb),
                                         C.POINTER(TrainPixels), C.c_int32, P],
            "gdf_train_paths_async": [P, C.POINTER(PathState), C.POINTER(Aabb), C.POINTER(TrainPixels),
                                      P, P, P],
            "gdf_train_paths": [P, C.POINTER(PathState), C.POINTER(Aabb), C.POINTER(TrainPixels),
                                C.POINTER(C.c_float), C.POINTER(C.c_int64), P],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.gdf_last_error.restype = C.c_char_p
        L.gdf_last_error.argtypes = []
        L.gdf_status_string.restype = C.c_char_p
        L.gdf_status_string.argtypes = [C.c_int]
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != GDF_OK:
        raise GdfError(status, lib().gdf_last_error().decode())


def default_config(preset: int) -> Config:
    c = Config()
    check(lib().gdf_default_config(preset, C.byref(c)))
    return c


def _ptr(x):
    """Device/host pointer of a torch tensor, numpy array or int (None -> NULL)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(type(x))


def shading(pos, wo, normal, roughness) -> Shading:
    sh = Shading(_ptr(pos), _ptr(wo), _ptr(normal), _ptr(roughness))
    sh._keep = (pos, wo, normal, roughness)  # raw pointers into these tensors
    return sh


def prepare_queries(sh: Shading, aabb: Aabb, queries, n=None, stream=None):
    n = queries.shape[0] if n is None else n
    check(lib().gdf_prepare_queries(C.byref(sh), C.byref(aabb), _ptr(queries), n, _stream(stream)))


def _stream(s):
    if s is None:
        return None
    if isinstance(s, int):
        return s
    return s.cuda_stream


class Context:
    """Owns one gdf_ctx (LearnedDistribution + NRC state on the current device)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        h = C.c_void_p()
        check(lib().gdf_create(C.byref(cfg), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().gdf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def n_params(self, net: int) -> int:
        n = C.c_int64()
        check(lib().gdf_n_params(self.h, net, C.byref(n)))
        return n.value

    def set_params(self, net: int, params):
        import numpy as np
        a = np.ascontiguousarray(params, dtype=np.float32)
        check(lib().gdf_set_params(self.h, net, a.ctypes.data, a.size))

    def get_params(self, net: int):
        import numpy as np
        a = np.empty(self.n_params(net), dtype=np.float32)
        check(lib().gdf_get_params(self.h, net, a.ctypes.data, a.size))
        return a

    def get_inference_params(self, net: int):
        import numpy as np
        a = np.empty(self.n_params(net), dtype=np.float32)
        check(lib().gdf_get_inference_params(self.h, net, a.ctypes.data, a.size))
        return a

    def save(self, prefix: str):
        check(lib().gdf_save_network(self.h, prefix.encode()))

    def load(self, prefix: str):
        check(lib().gdf_load_network(self.h, prefix.encode()))

    def infer(self, queries, wi, guided=None, uniforms=None, seed=0, offset=0, n=None, stream=None):
        n = queries.shape[0] if n is None else n
        check(lib().gdf_infer(self.h, _ptr(queries), _ptr(guided), _ptr(uniforms), seed, offset,
                              _ptr(wi), n, _stream(stream)))

    def infer_host(self, queries, wi_in, wi_out, guided=None, uniforms=None, seed=0, offset=0,
                   n=None, stream=None):
        n = queries.shape[0] if n is None else n
        check(lib().gdf_infer_host(self.h, _ptr(queries), _ptr(guided), _ptr(uniforms), seed, offset,
                                   _ptr(wi_in), _ptr(wi_out), n, _stream(stream)))

    def pdf_image(self, query, width, height, image, stream=None):
        import numpy as np
        q = np.ascontiguousarray(query, dtype=np.float32)
        check(lib().gdf_pdf_image(self.h, q.ctypes.data, width, height, _ptr(image), _stream(stream)))

    def sample_histogram(self, query, n_samples, seed, width, height, counts, dirs=None, stream=None):
        import numpy as np
        q = np.ascontiguousarray(query, dtype=np.float32)
        check(lib().gdf_sample_histogram(self.h, q.ctypes.data, n_samples, seed, width, height,
                                         _ptr(counts), _ptr(dirs), _stream(stream)))

    def eval_pdf(self, queries, u, pdf_out, n=None, stream=None):
        n = queries.shape[0] if n is None else n
        check(lib().gdf_eval_pdf(self.h, _ptr(queries), _ptr(u), _ptr(pdf_out), n, _stream(stream)))

    def post_inference(self, logits_theta, logits_phi, uniforms, wi, guided=None, n=None, stream=None):
        n = logits_theta.shape[0] if n is None else n
        check(lib().gdf_post_inference(self.h, _ptr(logits_theta), _ptr(logits_phi), _ptr(guided),
                                       _ptr(uniforms), _ptr(wi), n, _stream(stream)))

    def train_step(self, in_theta, in_phi, target, n=None, stream=None, stats=True):
        n = in_theta.shape[0] if n is None else n
        st = TrainStats()
        check(lib().gdf_train_step(self.h, _ptr(in_theta), _ptr(in_phi), _ptr(target), n,
                                   C.byref(st) if stats else None, _stream(stream)))
        return st

    def nrc_query(self, inp, out, n=None, stream=None):
        n = inp.shape[0] if n is None else n
        check(lib().gdf_nrc_query(self.h, _ptr(inp), _ptr(out), n, _stream(stream)))

    def nrc_train_step(self, inp, target, n=None, stream=None, stats=True):
        n = inp.shape[0] if n is None else n
        st = TrainStats()
        check(lib().gdf_nrc_train_step(self.h, _ptr(inp), _ptr(target), n,
                                       C.byref(st) if stats else None, _stream(stream)))
        return st

    def infer_ex(self, wi, n=None, queries=None, shading: "Shading | None" = None, aabb=None,
                 guided=None, uniforms=None, seed=0, offset=0, dir_pdf=None, norm_err=None, stream=None,
                 stage_events=None):
        """stage_events: two recorded torch.cuda.Event objects (timing) that
        the call re-records after the grid-feature and the fused launch."""
        n = wi.shape[0] if n is None else n
        a = InferArgs()
        a.queries_dev = _ptr(queries)
        a.shading = C.pointer(shading) if shading is not None else None
        a._keep = shading
        if aabb is not None:
            a.aabb = aabb
        a.guided_dev = _ptr(guided)
        a.uniforms_dev = _ptr(uniforms)
        a.philox_seed = seed
        a.philox_offset = offset
        a.wi_dev = _ptr(wi)
        a.dir_pdf_dev = _ptr(dir_pdf)
        a.n = n
        a.cdf_norm_err_dev = _ptr(norm_err)
        if stage_events is not None:
            if any(not e.cuda_event for e in stage_events):
                raise ValueError("stage_events must be recorded once before use (torch creates them lazily)")
            evs = (C.c_void_p * 2)(*[e.cuda_event for e in stage_events])
            a.stage_events = C.cast(evs, C.c_void_p)
            a._keep_events = evs
        check(lib().gdf_infer_ex(self.h, C.byref(a), _stream(stream)))

    def build_train_records(self, st: PathState, aabb: Aabb, px: TrainPixels, in_theta, in_phi,
                            target, capacity=None, stream=None) -> int:
        cap = in_theta.shape[0] if capacity is None else capacity
        cnt = C.c_int64()
        check(lib().gdf_build_train_records(self.h, C.byref(st), C.byref(aabb), C.byref(px),
                                            _ptr(in_theta), _ptr(in_phi), _ptr(target), cap,
                                            C.byref(cnt), _stream(stream)))
        return cnt.value

    def build_nrc_records(self, st: PathState, aabb: Aabb, px: TrainPixels, with_training: bool,
                          q_in, q_depth, q_pixel, t_in=None, t_target=None, stream=None):
        counts = (C.c_int64 * 2)()
        qcap = q_in.shape[0]
        tcap = t_in.shape[0] if t_in is not None else 0
        check(lib().gdf_build_nrc_records(self.h, C.byref(st), C.byref(aabb), C.byref(px),
                                          int(with_training), _ptr(q_in), _ptr(q_depth),
                                          _ptr(q_pixel), qcap, _ptr(t_in), _ptr(t_target), tcap,
                                          C.byref(counts), _stream(stream)))
        return counts[0], counts[1]

    def apply_nrc(self, st: PathState, nrc_out, depth, pixel, m=None, stream=None):
        m = depth.shape[0] if m is None else m
        check(lib().gdf_apply_nrc(self.h, C.byref(st), _ptr(nrc_out), _ptr(depth), _ptr(pixel), m,
                                  _stream(stream)))

    def nrc_train_paths(self, st: PathState, aabb: Aabb, px: TrainPixels, stream=None):
        loss = C.c_float()
        n = C.c_int64()
        check(lib().gdf_nrc_train_paths(self.h, C.byref(st), C.byref(aabb), C.byref(px),
                                        C.byref(loss), C.byref(n), _stream(stream)))
        return loss.value, n.value

    def nrc_substitute_paths(self, st: PathState, aabb: Aabb, px: TrainPixels,
                             skip_generation=False, stream=None):
        check(lib().gdf_nrc_substitute_paths(self.h, C.byref(st), C.byref(aabb), C.byref(px),
                                             int(skip_generation), _stream(stream)))

    def train_paths(self, st: PathState, aabb: Aabb, px: TrainPixels, stream=None):
        loss = C.c_float()
        n = C.c_int64()
        check(lib().gdf_train_paths(self.h, C.byref(st), C.byref(aabb), C.byref(px),
                                    C.byref(loss), C.byref(n), _stream(stream)))
        return loss.value, n.value

    def train_paths_async(self, st: PathState, aabb: Aabb, px: TrainPixels, loss_dev=None, n_dev=None,
                          stream=None):
        """Stream-ordered frame training; results land in device tensors
        (float32 loss, int64 record count)."""
        check(lib().gdf_train_paths_async(self.h, C.byref(st), C.byref(aabb), C.byref(px), _ptr(loss_dev),
                                          _ptr(n_dev), _stream(stream)))

    def get_optimizer_state(self, net: int):
        import numpy as np
        n = self.n_params(net)
        m = np.empty(n, np.float32)
        v = np.empty(n, np.float32)
        st = np.empty(n, np.uint32)
        step = C.c_uint32()
        check(lib().gdf_get_optimizer_state(self.h, net, m.ctypes.data, v.ctypes.data, st.ctypes.data, n,
                                            C.byref(step)))
        return m, v, st, step.value

    def set_optimizer_state(self, net: int, m, v, steps, opt_step: int):
        import numpy as np
        m = np.ascontiguousarray(m, np.float32)
        v = np.ascontiguousarray(v, np.float32)
        s = np.ascontiguousarray(steps, np.uint32)
        check(lib().gdf_set_optimizer_state(self.h, net, m.ctypes.data, v.ctypes.data, s.ctypes.data, m.size,
                                            opt_step))

    def sync(self, stream=None):
        check(lib().gdf_sync_status(self.h, _stream(stream)))


class Group:
    """A grouped inference engine (gdf_group): one launch pair for many jobs."""

    def __init__(self, max_jobs: int = 64):
        h = C.c_void_p()
        check(lib().gdf_group_create(max_jobs, C.byref(h)))
        self.h = h

    def infer(self, jobs, stream=None):
        """jobs: list of dicts with ctx, queries, wi and optional guided,
        uniforms, seed, offset, n."""
        arr = (Job * len(jobs))()
        for a, j in zip(arr, jobs):
            a.ctx = j["ctx"].h
            a.queries_dev = _ptr(j["queries"])
            a.guided_dev = _ptr(j.get("guided"))
            a.uniforms_dev = _ptr(j.get("uniforms"))
            a.philox_seed = j.get("seed", 0)
            a.philox_offset = j.get("offset", 0)
            a.wi_dev = _ptr(j["wi"])
            a.n = j.get("n", j["queries"].shape[0])
        check(lib().gdf_group_infer(self.h, arr, len(jobs), _stream(stream)))

    def set_shape(self, warpgroups: int, feature_block: int):
        check(lib().gdf_group_set_shape(self.h, warpgroups, feature_block))

    def track_jobs(self, on: bool = True):
        check(lib().gdf_group_track_jobs(self.h, int(on)))

    def job_done(self, job: int) -> bool:
        return bool(lib().gdf_group_job_done(self.h, job))

    def set_sm_cap(self, ctas: int):
        check(lib().gdf_group_set_sm_cap(self.h, ctas))

    def tuning(self):
        import numpy as np
        w, b = C.c_int32(), C.c_int32()
        ms = np.zeros(4, np.float32)
        check(lib().gdf_group_tuning(self.h, C.byref(w), C.byref(b), ms.ctypes.data))
        return w.value, b.value, ms

    def sync(self, stream=None):
        check(lib().gdf_group_sync_status(self.h, _stream(stream)))

    def close(self):
        if self.h:
            lib().gdf_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


REQ_INFER, REQ_TRAIN = 0, 1


def ctx_bytes(ctx) -> int:
    b = C.c_int64()
    check(lib().gdf_ctx_bytes(ctx.h, C.byref(b)))
    return b.value


class Server:
    """gdf_server: resident instances, continuous admission and batching."""

    def __init__(self, budget_bytes: int, slots: int = 4, max_batch: int = 16, device: int = 0,
                 max_train_slots: int = 0, train_sm_reserve: int = 0):
        cfg = ServerConfig(device, slots, max_batch, max_train_slots, budget_bytes, train_sm_reserve)
        h = C.c_void_p()
        check(lib().gdf_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self._keep = {}

    def add_instance(self, ctx):
        check(lib().gdf_server_add_instance(self.h, ctx.h))

    def submit_infer(self, ctx, queries, wi, guided=None, uniforms=None, seed=0, offset=0, n=None) -> int:
        r = Request(REQ_INFER, ctx.h, queries.shape[0] if n is None else n, _ptr(queries), _ptr(guided),
                    _ptr(uniforms), seed, offset, _ptr(wi), None, None, None)
        return self._submit(r, (queries, wi, guided, uniforms))

    def submit_train(self, ctx, in_theta, in_phi, target, n=None) -> int:
        r = Request(REQ_TRAIN, ctx.h, in_theta.shape[0] if n is None else n, None, None, None, 0, 0, None,
                    _ptr(in_theta), _ptr(in_phi), _ptr(target))
        return self._submit(r, (in_theta, in_phi, target))

    def _submit(self, r, keep) -> int:
        t = C.c_uint64()
        check(lib().gdf_server_submit(self.h, C.byref(r), C.byref(t)))
        self._keep[t.value] = keep
        return t.value

    def wait(self, ticket: int):
        st = TrainStats()
        lat = C.c_double()
        try:
            check(lib().gdf_server_wait(self.h, ticket, C.byref(st), C.byref(lat)))
        finally:
            self._keep.pop(ticket, None)
        return st, lat.value

    def stats(self, reset: bool = False) -> ServerStats:
        st = ServerStats()
        check(lib().gdf_server_get_stats(self.h, C.byref(st), int(reset)))
        return st

    def close(self):
        if self.h:
            lib().gdf_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
