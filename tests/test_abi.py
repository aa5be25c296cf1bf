"""The C-ABI library builds, loads and exports every declared entry point.

Runs without a GPU: only host-side entry points are called.
"""
import ctypes as C
import os
import re
import subprocess

import pytest

import pygdf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gdf.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(gdf_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["gdf_create", "gdf_infer", "gdf_eval_pdf", "gdf_train_step", "gdf_nrc_query",
                 "gdf_nrc_train_step", "gdf_set_params", "gdf_get_params", "gdf_save_network",
                 "gdf_load_network", "gdf_post_inference", "gdf_sync_status"]:
        assert must in names


def test_library_exports_every_declared_symbol(built_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", built_lib], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (gdf_\w+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing


def test_library_is_built_for_sm100a_only(built_lib):
    out = subprocess.run(["cuobjdump", "--list-elf", built_lib], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    archs = set(re.findall(r"sm_(\d+a?)", out.stdout))
    assert archs == {"100a"}, archs


def test_default_configs(built_lib):
    small = pygdf.default_config(pygdf.PRESET_SMALL)
    assert (small.n_bins_theta, small.grid_theta.n_levels, small.grid_theta.log2_hashmap_size) == (32, 8, 16)
    assert small.mlp_theta.n_hidden_layers == 3
    full = pygdf.default_config(pygdf.PRESET_FULL)
    assert (full.n_bins_phi, full.grid_phi.n_levels, full.grid_phi.log2_hashmap_size) == (64, 16, 19)
    assert full.mlp_phi.n_hidden_layers == 4 and full.mlp_nrc.n_hidden_layers == 5
    assert full.max_queries == 1920 * 1080
    ref = pygdf.default_config(pygdf.PRESET_REFERENCE)
    assert (ref.n_bins_theta, ref.n_bins_phi) == (16, 32)
    assert ref.grid_theta.type == 1 and ref.grid_theta.interpolation == 1
    assert abs(ref.grid_theta.per_level_scale - 1.405) < 1e-6
    assert abs(ref.adam_df.learning_rate - 3e-2) < 1e-9 and abs(ref.adam_df.ema_decay - 0.95) < 1e-7
    assert abs(ref.adam_nrc.learning_rate - 8e-3) < 1e-9 and abs(ref.adam_nrc.ema_decay - 0.99) < 1e-7
    with pytest.raises(pygdf.GdfError):
        pygdf.default_config(99)


def test_create_rejects_bad_configs(built_lib):
    L = pygdf.lib()
    c = pygdf.default_config(pygdf.PRESET_SMALL)
    c.abi_version = 0
    h = C.c_void_p()
    assert L.gdf_create(C.byref(c), C.byref(h)) == 1 and not h
    c = pygdf.default_config(pygdf.PRESET_SMALL)
    c.n_bins_theta = 24
    assert L.gdf_create(C.byref(c), C.byref(h)) == 1
    c = pygdf.default_config(pygdf.PRESET_SMALL)
    c.sh_degree = 3
    assert L.gdf_create(C.byref(c), C.byref(h)) == 6
    assert b"SH" in L.gdf_last_error()
    assert L.gdf_create(None, C.byref(h)) == 1


def test_null_context_is_an_error_not_a_crash(built_lib):
    L = pygdf.lib()
    assert L.gdf_infer(None, None, None, None, 0, 0, None, 1, None) == 1
    assert L.gdf_nrc_query(None, None, None, 1, None) != 0
    n = C.c_int64()
    assert L.gdf_n_params(None, 0, C.byref(n)) == 1
    assert L.gdf_destroy(None) == 0
    assert L.gdf_status_string(4) == b"device wait timed out"
