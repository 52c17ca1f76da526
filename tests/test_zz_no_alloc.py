"""The allocation-free median fill (pct_regularize_device_noalloc) against the handle-based entry
point, through the C ABI.

That entry point exists for callers that may not allocate GPU memory while they run (their
device memory belongs to their own pool, or allocation after start-up is forbidden); its scratch
is a fixed array inside the library instead of handle-owned buffers. This file is collected
last on purpose, so that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import pseudoctimaging_b200 as pct
from conftest import load_golden

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name", ["nan_rich_nh7", "small_nh7_2atlas", "nh3_tiny"])
def test_noalloc_fill_matches_handle_fill_on_two_calls_in_a_row(name):
    g = load_golden(name)
    nh = int(g["nh"])
    nz, nx, ny = g["out"].shape
    stream = torch.cuda.current_stream().cuda_stream
    with pct.Handle(0) as h:
        ref = torch.from_numpy(g["out"].copy()).cuda()
        ref_fills = h.regularize_device(ref.data_ptr(), nx, ny, nz, nh, stream)
    expected = ref.cpu().numpy()
    # Two calls in a row: the second one starts from whatever the first left in the shared array.
    for _ in range(2):
        vol = torch.from_numpy(g["out"].copy()).cuda()
        fills = ctypes.c_int64(-1)
        st = pct.lib.pct_regularize_device_noalloc(vol.data_ptr(), nx, ny, nz, nh,
                                                   ctypes.byref(fills), stream)
        assert st == 0, pct.lib.pct_strerror(st)
        torch.cuda.synchronize()
        got = vol.cpu().numpy()
        # Same kernels on the same data: the results must agree bit for bit (and so within the
        # 1e-4 relative tolerance the parity tests use).
        assert np.array_equal(_bits(got), _bits(expected))
        assert fills.value == ref_fills
        assert not np.isnan(got).any()


def test_noalloc_fill_rejects_volumes_beyond_its_fixed_scratch():
    small = torch.zeros(8, device="cuda")
    fills = ctypes.c_int64(-1)
    # 256^3 = 2^24 voxels, twice the 2^23 limit: rejected before anything runs on the GPU.
    st = pct.lib.pct_regularize_device_noalloc(small.data_ptr(), 256, 256, 256, 7,
                                               ctypes.byref(fills), None)
    assert st == -8
    assert fills.value == -1
    assert b"fixed scratch" in pct.lib.pct_strerror(st)
