"""C ABI surface and host-side logic of libpct_b200.so (no GPU needed)."""
import ctypes
import re

import numpy as np
import pytest

import pseudoctimaging_b200 as pct
from conftest import REPO

HEADER = REPO / "include" / "pct_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pct_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for required in ("pct_create", "pct_destroy", "pct_synthesize", "pct_synthesize_device",
                     "pct_strerror", "pct_run_pipeline", "pct_regularize_device"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(pct.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_python_bindings_cover_the_header():
    assert sorted(pct.SIGNATURES) == declared_functions()


def test_abi_version_and_strerror():
    assert pct.lib.pct_abi_version() == 1
    for code, name in pct.STATUS.items():
        s = pct.lib.pct_strerror(code)
        assert isinstance(s, bytes) and s
    assert pct.lib.pct_strerror(12345) == b"unknown status"


def test_null_handle_is_rejected():
    null = None
    assert pct.lib.pct_destroy(null) == -1
    assert pct.lib.pct_set_memory_limit(null, 0) == -1
    out = np.zeros(8, np.float32)
    p = out.ctypes.data
    assert pct.lib.pct_synthesize(null, p, p, p, p, 2, 2, 2, 1, 7, 1.0, 3) == -1
    assert pct.lib.pct_synthesize_device(null, p, p, p, p, 2, 2, 2, 1, 7, 1.0, 3, None) == -1
    assert pct.lib.pct_last_error_message(null) == b""
    assert pct.lib.pct_set_kernel_timing(null, 1) == -1
    ms, n = ctypes.c_double(), ctypes.c_int()
    assert pct.lib.pct_kernel_time(null, ctypes.byref(ms), ctypes.byref(n)) == -1


def test_create_rejects_bad_device_index():
    h = ctypes.c_void_p()
    assert pct.lib.pct_create(-1, ctypes.byref(h)) == -5
    assert pct.lib.pct_create(10_000, ctypes.byref(h)) == -5
    assert h.value is None


def test_synth_is_deterministic_and_seeded():
    a = pct.synth_subject(20, 18, 12, 2, n_blobs=5, seed=3)
    b = pct.synth_subject(20, 18, 12, 2, n_blobs=5, seed=3)
    c = pct.synth_subject(20, 18, 12, 2, n_blobs=5, seed=4)
    for x, y in ((a.img, b.img), (a.atlas_mri, b.atlas_mri), (a.atlas_ct, b.atlas_ct)):
        assert np.array_equal(x, y)
    assert not np.array_equal(a.img, c.img)
    assert a.img.shape == (12, 20, 18) and a.atlas_mri.shape == (2, 12, 20, 18)


def test_synth_value_ranges_follow_the_recipe():
    s = pct.synth_subject(48, 40, 24, 2, n_blobs=20, seed=0)
    # CT = clip(map, -1000, 2000) + N(0, 20): a few sigma outside the clip range at most
    assert s.atlas_ct.min() > -1000 - 8 * 20 and s.atlas_ct.max() < 2000 + 8 * 20
    # both ends of the HU map are populated: air between blobs, bone at blob peaks
    assert (s.atlas_ct < -900).mean() > 0.01 and (s.atlas_ct > 300).mean() > 0.01
    # atlas MRI is a displaced copy of the input: strongly correlated but not identical
    r = np.corrcoef(s.img.ravel(), s.atlas_mri[0].ravel())[0, 1]
    assert 0.8 < r < 0.9999


def test_synth_rejects_bad_params():
    p = pct.SynthParams()
    assert pct.lib.pct_synth_default_params(ctypes.byref(p), 0, 4, 4, 1, 3, 0) == 0
    assert pct.lib.pct_synth_generate(ctypes.byref(p), None, None, None) == -1
    assert pct.lib.pct_synth_generate(None, None, None, None) == -1


def test_div_and_host_label_normalisation():
    assert pct.div_from(2.5, 1.0) == 337.5
    ct = np.array([-1024.0, 0.0, 3071.0], np.float32)
    np.testing.assert_array_equal(pct.normalize_labels(ct), np.float32(255.0) * ((ct + 1024) / np.float32(4095.0)))


@pytest.mark.parametrize("dims", [(1 << 21, 1 << 21, 1 << 21),   # product 2^63 wraps negative
                                  ((1 << 31) - 1, (1 << 31) - 1, 4),
                                  (3, 1 << 30, 1 << 30),
                                  (2048, 2048, 3)])                # 12.6M > 2^23, no overflow
def test_noalloc_fill_rejects_oversized_shapes_before_any_device_work(dims):
    """The size check of the allocation-free fill compares factor by factor, so shapes whose
    voxel count overflows 64 bits are rejected too. Run only where no GPU is visible: the
    rejection must come before any CUDA call, and without a GPU nothing could run if it did not."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("host-only check; shapes like these are never sent to a GPU entry point")
    fills = ctypes.c_int64(-1)
    st = pct.lib.pct_regularize_device_noalloc(ctypes.c_void_p(16), *dims, 7,
                                               ctypes.byref(fills), None)
    assert st == -8, pct.STATUS.get(st, st)  # PCT_ERR_TOO_LARGE
    assert fills.value == -1
