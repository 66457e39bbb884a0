"""The C ABI library: loads, exports every declared symbol, fails loudly without a GPU."""
import os
import re

import numpy as np
import pytest

import lux_b200

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "lux_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lux_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = lux_b200.load_library()
    declared = _declared_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) <= set(lux_b200.SIGNATURES), set(declared) - set(lux_b200.SIGNATURES)
    assert lib.lux_abi_version() == 1


def test_error_text_is_thread_local_string():
    lib = lux_b200.load_library()
    assert isinstance(lib.lux_last_error(), bytes)


def test_null_arguments_are_rejected_without_gpu_work():
    lib = lux_b200.load_library()
    assert lib.lux_ctx_create(None, 0, None) == lux_b200.LUX_ERR_INVALID_ARGUMENT
    assert lib.lux_ctx_destroy(None) == lux_b200.LUX_OK
    assert lib.lux_bvh_destroy(None) == lux_b200.LUX_OK
    assert lib.lux_lbvh_build(None, None, 0, 0, 30, None) != lux_b200.LUX_OK


def test_workload_generator_is_prefix_stable():
    from lux_b200 import workloads as W
    a = W.soup_triangles(1000)
    b = W.soup_triangles(4000)
    # Counter-based streams: per-stream prefixes agree (centroid stream is consecutive).
    ca = a.reshape(-1, 3, 3).mean(axis=1)
    assert np.all(np.isfinite(a)) and a.shape == (1000, 9)
    assert np.allclose(W.splitmix_uniform(7, 1, 10), W.splitmix_uniform(7, 1, 20)[:10])
    assert np.all((ca > -0.05) & (ca < 1.05))
    r = W.uniform_rays(100)
    assert np.allclose(np.linalg.norm(r[:, 4:7], axis=1), 1.0, atol=1e-6)
