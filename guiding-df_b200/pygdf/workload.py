"""Seeded synthetic workloads standing in for the reference's scenes.

The reference evaluates on downloaded scenes that are not available; these
generators produce query and training records with the shapes and value
distributions of the benchmark configurations:

* query record: position uniform in [0,1]^3, shading normal and outgoing
  direction uniform on the sphere, roughness 0.5;
* training target: a radiance field of 4 von Mises-Fisher lobes per cell of
  an 8^3 grid over [0,1]^3 (lobe means uniform on S^2, kappa log-uniform in
  [1, 200], RGB weights uniform in [0,1]^3), evaluated with the vMF density of
  src/lib/src/util/vmf.h:22-27.

The record -> network-input mapping restates generate_inference_data_AR
(src/render/guided/train.cu:334-362) and generate_training_data_AR
(train.cu:6-96) in numpy float32.
"""
from __future__ import annotations

import numpy as np

INV_PI = np.float32(0.318309886183790671538)
INV_2PI = np.float32(0.15915494309189533577)


def _unit_sphere(rng: np.random.Generator, n: int) -> np.ndarray:
    z = 1.0 - 2.0 * rng.random(n)
    phi = 2.0 * np.pi * rng.random(n)
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1).astype(np.float32)


def query_records(n: int, seed: int) -> dict:
    rng = np.random.default_rng(seed)
    return {
        "pos": rng.random((n, 3), dtype=np.float32),
        "wo": _unit_sphere(rng, n),
        "normal": _unit_sphere(rng, n),
        "roughness": np.full(n, 0.5, dtype=np.float32),
    }


def normalize_spatial(pos: np.ndarray, aabb_min=(0, 0, 0), aabb_max=(1, 1, 1)) -> np.ndarray:
    """normalizeSpatialCoord (train.h:272-276): AABB inflated by 0.5% of its diagonal."""
    lo = np.asarray(aabb_min, dtype=np.float32)
    hi = np.asarray(aabb_max, dtype=np.float32)
    infl = np.float32(np.linalg.norm(hi - lo) * 0.005)
    lo, hi = lo - infl, hi + infl
    center = (lo + hi) * np.float32(0.5)
    diag = hi - lo
    return (np.float32(0.5) + (pos - center) / diag).astype(np.float32)


def spherical_normalized(v: np.ndarray) -> np.ndarray:
    """cartesianToSphericalNormalized (math_utils.h:183-196)."""
    vn = v / np.linalg.norm(v, axis=1, keepdims=True)
    theta = np.arccos(np.clip(vn[:, 2], -1.0, 1.0))
    phi = np.arctan2(vn[:, 1], vn[:, 0])
    phi = np.where(phi < 0, phi + 2 * np.pi, phi)
    return np.stack([theta / np.pi, phi / (2 * np.pi)], axis=1).astype(np.float32)


def queries_from_records(rec: dict) -> np.ndarray:
    """Network input rows [n x 9] of generate_inference_data_AR."""
    n = rec["pos"].shape[0]
    q = np.empty((n, 9), dtype=np.float32)
    q[:, 0:3] = normalize_spatial(rec["pos"])
    wo = rec["wo"] / np.linalg.norm(rec["wo"], axis=1, keepdims=True)
    q[:, 3:6] = (wo + 1.0) * 0.5  # warp_direction_for_sh (train.h:1243)
    q[:, 6:8] = spherical_normalized(rec["normal"])
    q[:, 8] = 1.0 - np.exp(-rec["roughness"])  # warp_roughness_for_ob (train.h:1247)
    return q


def queries(n: int, seed: int) -> np.ndarray:
    return queries_from_records(query_records(n, seed))


def wi_init(n: int, seed: int, guided_frac: float = 1.0, one_sided_frac: float = 0.0):
    """Initial guiding-data rows and the guided mask.

    Non-guided rows carry a BSDF-sampled square direction in slots 0,1; slots
    2,3 carry the caller's sign (-1 for one-sided BSDFs, integrator.cpp:383-384).
    """
    rng = np.random.default_rng(seed + 1)
    wi = np.empty((n, 4), dtype=np.float32)
    wi[:, 0:2] = rng.random((n, 2), dtype=np.float32)
    sign = np.where(rng.random(n) < one_sided_frac, -1.0, 1.0).astype(np.float32)
    wi[:, 2] = sign
    wi[:, 3] = sign
    guided = (rng.random(n) < guided_frac).astype(np.uint8)
    return wi, guided


def uniforms(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed + 2)
    return rng.random((n, 4), dtype=np.float32)


class VmfField:
    """4 vMF lobes per cell of an 8^3 grid over [0,1]^3."""

    def __init__(self, seed: int, cells: int = 8, lobes: int = 4):
        rng = np.random.default_rng(seed + 3)
        self.cells, self.lobes = cells, lobes
        m = cells ** 3 * lobes
        self.mu = _unit_sphere(rng, m).reshape(cells ** 3, lobes, 3)
        self.kappa = np.exp(rng.uniform(np.log(1.0), np.log(200.0), m)).astype(np.float32)
        self.kappa = self.kappa.reshape(cells ** 3, lobes)
        self.w = rng.random((cells ** 3, lobes, 3), dtype=np.float32)

    def radiance(self, pos: np.ndarray, wi: np.ndarray) -> np.ndarray:
        c = np.clip((pos * self.cells).astype(np.int64), 0, self.cells - 1)
        cell = (c[:, 0] * self.cells + c[:, 1]) * self.cells + c[:, 2]
        mu, k, w = self.mu[cell], self.kappa[cell], self.w[cell]
        cos = np.einsum("nld,nd->nl", mu, wi)
        # VMFDistribution::eval (vmf.h:22-27)
        val = np.exp(k * np.minimum(0.0, cos - 1.0)) * k / (2 * np.pi * (1 - np.exp(-2 * k)))
        return np.einsum("nl,nlc->nc", val, w).astype(np.float32)


def uniform_sphere_to_square(v: np.ndarray) -> np.ndarray:
    """uniformSphereToSquare (math_utils.h:233-240)."""
    vn = v / np.linalg.norm(v, axis=1, keepdims=True)
    phi = np.arctan2(vn[:, 1], vn[:, 0]) * INV_2PI
    return np.stack([(1.0 - vn[:, 2]) * 0.5, np.where(phi < 0, phi + 1.0, phi)], axis=1).astype(np.float32)


def training_batch(n: int, seed: int, n_bins_theta: int, linear: bool = True):
    """(GuidedInput [n x 9], GuidedInputPhi [n x 10], GuidedOutput [n x 9]) of
    generate_training_data_AR with omega_i uniform, p_wi = 1/(4 pi),
    bsdfVal = 1, misWeight = 1, thp = 1."""
    rec = query_records(n, seed)
    q = queries_from_records(rec)
    rng = np.random.default_rng(seed + 4)
    wi_dir = _unit_sphere(rng, n)
    field = VmfField(seed)
    L = field.radiance(rec["pos"], wi_dir)
    u = uniform_sphere_to_square(wi_dir)
    nb = np.float32(n_bins_theta)
    fl = np.minimum(np.floor(u[:, 0] * nb).astype(np.int32), n_bins_theta - 1).astype(np.float32)
    if linear:
        cond = (fl + (u[:, 0] * nb - fl)) / nb
    else:
        cond = fl / nb
    in_phi = np.concatenate([q, cond[:, None].astype(np.float32)], axis=1)
    out = np.empty((n, 9), dtype=np.float32)
    out[:, 0:2] = u
    out[:, 2:5] = L
    out[:, 5] = np.float32(1.0 / (4.0 * np.pi))
    out[:, 6:9] = 1.0
    return q, in_phi.astype(np.float32), out


def nrc_batch(n: int, seed: int):
    """GuidedInputNRC rows [n x 15] and RGB targets [n x 3]."""
    rec = query_records(n, seed)
    q = queries_from_records(rec)
    rng = np.random.default_rng(seed + 5)
    x = np.empty((n, 15), dtype=np.float32)
    x[:, 0:9] = q
    x[:, 9:12] = rng.random((n, 3), dtype=np.float32)   # diffuse
    x[:, 12:15] = rng.random((n, 3), dtype=np.float32)  # specular
    wo = rec["wo"]
    field = VmfField(seed)
    y = field.radiance(rec["pos"], wo)
    return x, y


def path_state(n_pixels: int, seed: int, aabb=((-2.0, -1.0, -3.0), (4.0, 2.0, 1.0)),
               defects: bool = True) -> tuple[dict, np.ndarray]:
    """Per-pixel vertex records of one frame, laid out like
    GuidedPixelStateBuffer (workqueue.h:16-145, RadianceRecordItem in
    guideditem.h:23-44): fields[name] is [MAX_TRAIN_DEPTH, n_pixels(, k)].

    Path lengths follow a survival of 0.7 per bounce; about 15 % of the
    vertices are delta-lobe samples and 5 % NRC alignment records of misses.
    With `defects`, a few per mille of positions, directions and radiances
    are NaN, some throughputs are below M_EPSILON and some pdfs are zero, so
    the producers' filters are exercised."""
    rng = np.random.default_rng(seed)
    d, n = 5, n_pixels
    lo = np.asarray(aabb[0], np.float32)
    hi = np.asarray(aabb[1], np.float32)
    f32 = np.float32

    def sph(shape):
        t = np.arccos(1.0 - 2.0 * rng.random(shape)).astype(f32)
        p = (2.0 * np.pi * rng.random(shape)).astype(f32)
        return np.stack([t, p], axis=-1)

    thp = (0.05 + 0.95 * rng.random((d, n, 3))).astype(f32)
    fields = {
        # accumulated radiance carries the vertex throughput (recordRadiance,
        # workqueue.h:84-92), so L / thp is a local radiance of order one
        "L": (thp * rng.exponential(1.0, (d, n, 3))).astype(f32),
        "thp": thp,
        "Le": (0.1 * rng.random((d, n, 3))).astype(f32),
        "pos": (lo + (hi - lo) * rng.random((d, n, 3))).astype(f32),
        "dir": sph((d, n)),
        "wi_pdf": (0.05 + 2.0 * rng.random((d, n))).astype(f32),
        "mis_weight": rng.random((d, n), dtype=f32),
        "delta": (rng.random((d, n)) < 0.15).astype(np.uint8),
        "miss": (rng.random((d, n)) < 0.05).astype(np.uint8),
        "bsdf_val": rng.random((d, n, 3), dtype=f32),
        "wo": sph((d, n)),
        "normal": sph((d, n)),
        "roughness": rng.random((d, n), dtype=f32),
        "diffuse": rng.random((d, n, 3), dtype=f32),
        "specular": rng.random((d, n, 3), dtype=f32),
    }
    depth = np.zeros(n, np.uint32)
    alive = np.ones(n, bool)
    for k in range(d):
        depth += alive
        alive &= rng.random(n) < 0.7
    if defects:
        def poke(name, frac, value):
            a = fields[name]
            m = rng.random(a.shape[:2]) < frac
            a[m] = value
        poke("pos", 0.004, np.nan)
        poke("dir", 0.003, np.nan)
        poke("wo", 0.002, np.nan)
        poke("wo", 0.001, np.inf)
        poke("dir", 0.001, -np.inf)
        poke("L", 0.004, np.nan)
        poke("thp", 0.02, 1e-6)
        poke("wi_pdf", 0.01, 0.0)
    return fields, depth
