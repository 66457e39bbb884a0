"""lux_lbvh_morton_sort_static, the allocation-free Morton sort, against lux_lbvh_build +
lux_bvh_download on the same inputs (B200).

Collected last so that it also runs after every other test has used the library; it
passes alone in a fresh process too.  Integer outputs: the bar is bit-exact."""
import numpy as np
import pytest

import lux_b200
from lux_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAX_PRIMS = 1048576


def _static_sort(ctx, prims: np.ndarray, kind: int, bits: int):
    import torch
    n = prims.shape[0]
    d_prims = torch.from_numpy(np.ascontiguousarray(prims, np.float32)).cuda()
    codes = torch.empty(n, dtype=torch.int64, device="cuda")
    ids = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()  # the context's stream is not ordered after torch's
    lib = lux_b200.load_library()
    st = lib.lux_lbvh_morton_sort_static(ctx.handle, d_prims.data_ptr(), n, kind, bits,
                                         codes.data_ptr(), ids.data_ptr())
    assert st == lux_b200.LUX_OK, lib.lux_last_error()
    return codes.cpu().numpy().view(np.uint64), ids.cpu().numpy()


def _existing(ctx, prims: np.ndarray, kind: int, bits: int):
    tree = ctx.build_lbvh(np.ascontiguousarray(prims, np.float32), kind, bits).download()
    return tree.sorted_codes, tree.sorted_ids


def _inputs():
    wide = W.soup_triangles(300_000, 5) * np.float32(4.0) - np.float32(1.5)
    return [(wide, lux_b200.PRIM_TRIANGLES, 30),
            (W.query_boxes(100_000, 9, half_extent=2e-3), lux_b200.PRIM_AABBS, 63),
            (W.soup_triangles(200_000, 6), lux_b200.PRIM_TRIANGLES, 63),
            (W.soup_triangles(4097, 8), lux_b200.PRIM_TRIANGLES, 30)]


def test_two_calls_in_a_row_match_the_build(ctx):
    import torch
    cases = _inputs()
    # The array keeps the previous call's contents: alternate wide and narrow inputs,
    # larger and smaller counts, and both key widths.
    for prims, kind, bits in cases + cases[:2]:
        got_codes, got_ids = _static_sort(ctx, prims, kind, bits)
        want_codes, want_ids = _existing(ctx, prims, kind, bits)
        assert np.array_equal(got_codes, want_codes)
        assert np.array_equal(got_ids, want_ids)
    # Repeated calls take no device memory (the first call on the device has already
    # looked up the static array).
    prims, kind, bits = cases[2]
    d_prims = torch.from_numpy(prims).cuda()
    codes = torch.empty(prims.shape[0], dtype=torch.int64, device="cuda")
    ids = torch.empty(prims.shape[0], dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    lib = lux_b200.load_library()
    free_before = torch.cuda.mem_get_info()[0]
    held = [ctx.get_option(lux_b200.OPT_SCRATCH_BYTES), ctx.get_option(lux_b200.OPT_STAGING_BYTES)]
    for _ in range(2):
        assert lib.lux_lbvh_morton_sort_static(ctx.handle, d_prims.data_ptr(), prims.shape[0],
                                               kind, bits, codes.data_ptr(),
                                               ids.data_ptr()) == lux_b200.LUX_OK
    assert torch.cuda.mem_get_info()[0] == free_before
    # Nor does it grow the context's own reusable scratch or staging.
    assert [ctx.get_option(lux_b200.OPT_SCRATCH_BYTES),
            ctx.get_option(lux_b200.OPT_STAGING_BYTES)] == held
    want_codes, want_ids = _existing(ctx, prims, kind, bits)
    assert np.array_equal(codes.cpu().numpy().view(np.uint64), want_codes)
    assert np.array_equal(ids.cpu().numpy(), want_ids)


def test_matches_the_reference_builders_own_order(ctx, golden_lbvh):
    """Directly against the reference: the fixtures the reference's own host LBVH wrote
    (build_cpu_lbvh_tree, bvh/cpu_lbvh_builder.h:163-259; tests/golden/make_golden.py) give
    the 30-bit codes and the stable sorted primitive order; two passes over all of them in
    a row, so each call starts from the previous one's array contents."""
    for _ in range(2):
        for name, case in golden_lbvh.items():
            prims = case["prims"]
            if len(prims) < 2:   # one primitive: no order to check, its code is unused
                continue
            codes, ids = _static_sort(ctx, prims, int(case["kind"]), 30)
            assert np.array_equal(ids, case["sorted_ids"]), name
            assert np.array_equal(codes, case["sorted_codes"].astype(np.uint64)), name


def test_limits_and_pointer_kinds_are_checked(ctx):
    import torch
    lib = lux_b200.load_library()
    dev = torch.zeros(16, dtype=torch.int64, device="cuda")
    st = lib.lux_lbvh_morton_sort_static(ctx.handle, dev.data_ptr(), MAX_PRIMS + 1,
                                         lux_b200.PRIM_TRIANGLES, 30, dev.data_ptr(),
                                         dev.data_ptr())
    assert st == lux_b200.LUX_ERR_INVALID_ARGUMENT
    assert b"LUX_STATIC_SORT_MAX_PRIMS" in lib.lux_last_error()
    host = np.zeros(64, np.float32)
    st = lib.lux_lbvh_morton_sort_static(ctx.handle, host.ctypes.data, 4,
                                         lux_b200.PRIM_TRIANGLES, 30, dev.data_ptr(),
                                         dev.data_ptr())
    assert st == lux_b200.LUX_ERR_INVALID_ARGUMENT
    assert lib.lux_lbvh_morton_sort_static(ctx.handle, None, 0, lux_b200.PRIM_TRIANGLES, 30,
                                           None, None) == lux_b200.LUX_OK
    assert lib.lux_lbvh_morton_sort_static(ctx.handle, None, 0, lux_b200.PRIM_TRIANGLES, 31,
                                           None, None) == lux_b200.LUX_ERR_INVALID_ARGUMENT
