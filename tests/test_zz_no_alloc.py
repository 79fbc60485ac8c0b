"""bt_density_noalloc: the density blur for callers that may not allocate.

Such callers (a plugin whose host application owns every device allocation,
or a frame loop that cannot take cudaMalloc's synchronisation) hand in device
buffers they were given; the entry point keeps its intermediate image in a
static device array instead of allocating. Its output must equal the density
that the allocating path (bt_upload) computes from the same splat counts, on
two calls in a row that share the static array.
"""
import ctypes

import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

pytestmark = pytest.mark.gpu

DENSITY_RTOL = 1e-5   # the density tolerance of the parity tests


def _reference_density(w):
    opts = bt.Options(width=w.width, height=w.height, sample_spacing=w.spacing, blur_sigma=w.sigma)
    gpu = bt.Gpu(opts)
    gpu.upload((w.xy, w.starts))
    counts, density = gpu.read_counts(), gpu.read_density()
    gpu.close()
    return counts, density


def test_noalloc_density_matches_the_allocating_path():
    import torch

    lib = bt.library()
    cases = [synthetic.small(), synthetic.small(seed_offset=7)]
    expected = [_reference_density(w) for w in cases]
    assert not np.array_equal(expected[0][1], expected[1][1])
    # Two calls in a row: the second reuses the static array the first left
    # behind (its running maximum must be cleared, not carried over).
    for w, (counts, density) in zip(cases, expected):
        dev_counts = torch.from_numpy(counts.view(np.int32)).cuda()
        dev_out = torch.full((w.width * w.height,), float("nan"), dtype=torch.float32, device="cuda")
        status = lib.bt_density_noalloc(ctypes.c_void_p(dev_counts.data_ptr()), ctypes.c_void_p(dev_out.data_ptr()),
                                        w.width, w.height, ctypes.c_float(w.sigma), None)
        assert status == 0, lib.bt_last_error(None)
        torch.cuda.synchronize()
        got = dev_out.cpu().numpy()
        np.testing.assert_allclose(got, density, rtol=DENSITY_RTOL, atol=DENSITY_RTOL)
        np.testing.assert_array_equal(got, density)


def test_noalloc_rejects_maps_beyond_the_static_scratch():
    lib = bt.library()
    status = lib.bt_density_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), 1025, 1024, ctypes.c_float(0.0), None)
    assert status == 3
    assert "exceeds the static scratch" in lib.bt_last_error(None).decode()


def test_noalloc_rejects_misaligned_buffers_before_launching():
    # The output is written four texels at a time and the counts are read as
    # whole words: misaligned buffers are refused on the host, so nothing is
    # launched (the addresses below are never dereferenced).
    lib = bt.library()
    status = lib.bt_density_noalloc(ctypes.c_void_p(256), ctypes.c_void_p(256 + 4), 64, 64, ctypes.c_float(0.0), None)
    assert status == 3
    assert "16-byte aligned" in lib.bt_last_error(None).decode()
    status = lib.bt_density_noalloc(ctypes.c_void_p(256 + 2), ctypes.c_void_p(256), 64, 64, ctypes.c_float(0.0), None)
    assert status == 3
    assert "4-byte aligned" in lib.bt_last_error(None).decode()
