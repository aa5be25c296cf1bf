"""ctypes driver of the reference GPU harness (oracle/ref_gpu/harness.cu).

TEST INFRASTRUCTURE ONLY. The harness runs the reference's own GPU path --
tiny-cuda-nn v1.6 and the reference DF kernels, built for sm_100a by
oracle/build_ref_gpu.py into oracle/_ref/libgdf_tcnnref_<theta>x<phi>.so --
on device buffers. Tests use it as the checker of the CUDA path on identical
weights, inputs and uniforms; bench.py times it as the reference GPU
baseline. Nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes as C
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_libs: dict[tuple[int, int], C.CDLL] = {}


def lib_path(theta: int, phi: int) -> str:
    return os.path.join(REF_DIR, f"libgdf_tcnnref_{theta}x{phi}.so")


def available(theta: int, phi: int) -> bool:
    return os.path.exists(lib_path(theta, phi))


def lib(theta: int, phi: int) -> C.CDLL:
    key = (theta, phi)
    if key in _libs:
        return _libs[key]
    path = lib_path(theta, phi)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (oracle/build_ref_gpu.py)")
    L = C.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
    vp, i64, i32, fp = C.c_void_p, C.c_int64, C.c_int32, C.POINTER(C.c_float)
    L.tref_last_error.restype = C.c_char_p
    L.tref_set_scrub.argtypes = [i32]
    L.tref_set_scrub.restype = None
    L.tref_bins.argtypes = [C.POINTER(i32), C.POINTER(i32)]
    L.tref_df_create.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.tref_df_destroy.argtypes = [vp]
    L.tref_df_destroy.restype = None
    L.tref_df_n_params.argtypes = [vp, i32]
    L.tref_df_n_params.restype = i64
    L.tref_df_encoded_width.argtypes = [vp, i32]
    L.tref_df_encoded_width.restype = i64
    for f in (L.tref_df_set_params, L.tref_df_get_params, L.tref_df_get_inference_params):
        f.argtypes = [vp, i32, vp, i64]
    L.tref_df_infer.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, vp]
    L.tref_df_last_pdfs.argtypes = [vp, vp, vp, vp, i64]
    L.tref_df_train_step.argtypes = [vp, vp, vp, vp, i64, i32, fp, vp, vp, vp, vp]
    L.tref_nrc_create.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.tref_nrc_destroy.argtypes = [vp]
    L.tref_nrc_destroy.restype = None
    L.tref_nrc_n_params.argtypes = [vp]
    L.tref_nrc_n_params.restype = i64
    L.tref_nrc_set_params.argtypes = [vp, vp, i64]
    L.tref_nrc_get_params.argtypes = [vp, vp, i64]
    L.tref_nrc_query.argtypes = [vp, vp, vp, i64, vp]
    L.tref_nrc_train_step.argtypes = [vp, vp, vp, i64, i32, fp, vp, vp]
    t, p = C.c_int32(), C.c_int32()
    L.tref_bins(C.byref(t), C.byref(p))
    if (t.value, p.value) != key:
        raise RuntimeError(f"{path} was compiled for {t.value}x{p.value} bins")
    _libs[key] = L
    return L


def _check(L, rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what}: {L.tref_last_error().decode()}")


_GRID_OTYPE = {0: "HashGrid", 1: "DenseGrid", 2: "TiledGrid"}
_GRID_INTERP = {0: "Linear", 1: "Smoothstep", 2: "Nearest"}


def _grid_json(g) -> dict:
    return {"otype": _GRID_OTYPE[g.type], "n_levels": g.n_levels, "n_features_per_level": g.n_features_per_level,
            "log2_hashmap_size": g.log2_hashmap_size, "base_resolution": g.base_resolution,
            "per_level_scale": float(g.per_level_scale), "interpolation": _GRID_INTERP[g.interpolation],
            "n_dims_to_encode": 3}


def _adam_json(a) -> dict:
    return {"otype": "Ema", "decay": float(a.ema_decay),
            "nested": {"otype": "Adam", "learning_rate": float(a.learning_rate), "beta1": float(a.beta1),
                       "beta2": float(a.beta2), "epsilon": float(a.epsilon), "l2_reg": float(a.l2_reg),
                       "adabound": False}}


def df_nn_json(cfg) -> dict:
    """The "nn" object of a DF config (base_product_df.json layout) that
    describes the same networks as a gdf_config (pygdf.Config)."""
    def enc(grid, phi: bool) -> dict:
        nested = [_grid_json(grid),
                  {"otype": "SphericalHarmonics", "degree": cfg.sh_degree, "n_dims_to_encode": 3},
                  {"otype": "OneBlob", "n_bins": cfg.oneblob_bins, "n_dims_to_encode": 3}]
        if phi:
            nested.append({"otype": "TriangleWave", "n_frequencies": cfg.tw_frequencies, "n_dims_to_encode": 1})
        return {"otype": "Composite", "nested": nested}

    def net(m) -> dict:
        return {"otype": "FullyFusedMLP", "activation": "ReLU", "output_activation": "None",
                "n_neurons": m.n_neurons, "n_hidden_layers": m.n_hidden_layers}

    return {"loss": {"otype": "L2"}, "optimizer": _adam_json(cfg.adam_df),
            "theta_encoding": enc(cfg.grid_theta, False), "phi_encoding": enc(cfg.grid_phi, True),
            "theta_network": net(cfg.mlp_theta), "phi_network": net(cfg.mlp_phi)}


def nrc_nn_json(cfg) -> dict:
    """The "nn" object of base_hashgrid_nrc_df.json for a gdf_config's NRC."""
    return {"loss": {"otype": "RelativeL2Luminance"}, "optimizer": _adam_json(cfg.adam_nrc),
            "encoding": {"otype": "Composite", "nested": [
                {"n_dims_to_encode": 3, "otype": "Frequency", "n_frequencies": cfg.nrc_frequencies},
                {"otype": "OneBlob", "n_bins": cfg.nrc_oneblob_bins, "n_dims_to_encode": 6},
                {"n_dims_to_encode": 6, "otype": "Identity"}]},
            "network": {"otype": "FullyFusedMLP", "activation": "ReLU", "output_activation": "None",
                        "n_neurons": cfg.mlp_nrc.n_neurons, "n_hidden_layers": cfg.mlp_nrc.n_hidden_layers}}


def _ptr(t) -> int | None:
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


class DfRef:
    """LearnedDistribution on tiny-cuda-nn (the reference GPU path).

    scrub: zero the start of the workspace arenas before every call, so the
    four theta-input columns the reference never writes (tiny-cuda-nn's
    OneBlob misplaces its padding, encodings/oneblob.h:223-226) read 0, as
    on the reference's first call, instead of stale workspace contents. The
    parity tests scrub; the speed baseline does not."""

    def __init__(self, cfg, scrub: bool = True):
        self.bins = (cfg.n_bins_theta, cfg.n_bins_phi)
        self.L = lib(*self.bins)
        self.L.tref_set_scrub(int(scrub))
        h = C.c_void_p()
        _check(self.L, self.L.tref_df_create(json.dumps(df_nn_json(cfg)).encode(), C.byref(h)), "tref_df_create")
        self.h = h

    def close(self) -> None:
        if self.h:
            self.L.tref_df_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def n_params(self, net: int) -> int:
        return int(self.L.tref_df_n_params(self.h, net))

    def encoded_width(self, net: int) -> int:
        return int(self.L.tref_df_encoded_width(self.h, net))

    def set_params(self, net: int, p) -> None:
        import numpy as np
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(self.L, self.L.tref_df_set_params(self.h, net, p.ctypes.data, p.size), "set_params")

    def get_params(self, net: int, inference: bool = False):
        import numpy as np
        out = np.empty(self.n_params(net), np.float32)
        f = self.L.tref_df_get_inference_params if inference else self.L.tref_df_get_params
        _check(self.L, f(self.h, net, out.ctypes.data, out.size), "get_params")
        return out

    def infer(self, wi, uniforms, queries=None, shading=None, aabb=None, guided=None, stream=0) -> None:
        """inferenceStep on device tensors; wi [n x 4] in/out. Either
        queries [n x 9] or shading = (pos, wo, normal, rough) with aabb
        (lo3 + hi3, host floats)."""
        n = wi.shape[0]
        a6 = None
        if shading is not None:
            a6 = (C.c_float * 6)(*[float(x) for x in aabb])
            pos, wo, nrm, rough = (_ptr(t) for t in shading)
        else:
            pos = wo = nrm = rough = None
        _check(self.L, self.L.tref_df_infer(self.h, _ptr(queries), pos, wo, nrm, rough,
                                            C.cast(a6, C.c_void_p) if a6 is not None else None, _ptr(guided),
                                            _ptr(uniforms), _ptr(wi), n, stream), "tref_df_infer")

    def last_pdfs(self, n: int):
        import numpy as np
        t = np.empty((n, self.bins[0]), np.float32)
        p = np.empty((n, self.bins[1]), np.float32)
        ip = np.empty((n, 10), np.float32)
        _check(self.L, self.L.tref_df_last_pdfs(self.h, t.ctypes.data, p.ctypes.data, ip.ctypes.data, n),
               "last_pdfs")
        return t, p, ip

    def train_step(self, in_theta, in_phi, target, step: bool = True, grads: bool = False,
                   per_record: bool = False, stream=0):
        """One reference training batch; returns (loss, grad_theta, grad_phi,
        loss per record), the last three None unless asked for."""
        import numpy as np
        n = in_theta.shape[0]
        loss = C.c_float()
        gt = np.empty(self.n_params(0), np.float32) if grads else None
        gp = np.empty(self.n_params(1), np.float32) if grads else None
        lr = np.empty(n, np.float32) if per_record else None
        _check(self.L, self.L.tref_df_train_step(self.h, _ptr(in_theta), _ptr(in_phi), _ptr(target), n, int(step),
                                                 C.byref(loss), _ptr(gt), _ptr(gp), _ptr(lr), stream),
               "tref_df_train_step")
        return loss.value, gt, gp, lr


class NrcRef:
    """NRC on tiny-cuda-nn (the reference GPU path). Needs any built
    harness library; the NRC does not depend on the bin counts."""

    def __init__(self, cfg, bins: tuple[int, int] = (64, 64)):
        self.L = lib(*bins)
        h = C.c_void_p()
        _check(self.L, self.L.tref_nrc_create(json.dumps(nrc_nn_json(cfg)).encode(), C.byref(h)), "tref_nrc_create")
        self.h = h

    def close(self) -> None:
        if self.h:
            self.L.tref_nrc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def n_params(self) -> int:
        return int(self.L.tref_nrc_n_params(self.h))

    def set_params(self, p) -> None:
        import numpy as np
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(self.L, self.L.tref_nrc_set_params(self.h, p.ctypes.data, p.size), "nrc set_params")

    def get_params(self):
        import numpy as np
        out = np.empty(self.n_params(), np.float32)
        _check(self.L, self.L.tref_nrc_get_params(self.h, out.ctypes.data, out.size), "nrc get_params")
        return out

    def query(self, inp, out, stream=0) -> None:
        _check(self.L, self.L.tref_nrc_query(self.h, _ptr(inp), _ptr(out), inp.shape[0], stream), "tref_nrc_query")

    def train_step(self, inp, target, step: bool = True, grads: bool = False, stream=0):
        import numpy as np
        loss = C.c_float()
        g = np.empty(self.n_params(), np.float32) if grads else None
        _check(self.L, self.L.tref_nrc_train_step(self.h, _ptr(inp), _ptr(target), inp.shape[0], int(step),
                                                  C.byref(loss), _ptr(g), stream), "tref_nrc_train_step")
        return loss.value, g
