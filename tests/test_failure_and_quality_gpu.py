"""Failure detection and the quality metric on the GPU, through the C ABI.

Failure detection uses no GPU fault: the fusion kernel's waits on its TMA copies are bounded, and
a testing hook makes the first CTA withhold the copies its first wait expects, so that wait runs
out after a short limit; the kernel records the timeout and stops, the call reports
PCT_ERR_TIMEOUT, and the same context then runs normally.
"""
import time

import numpy as np
import pytest
import torch

import oracle
import pseudoctimaging_b200 as pct
from conftest import compare_fused, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    h = pct.Handle(0)
    yield h
    h.close()


def test_bounded_wait_timeout_is_reported_and_context_survives(handle):
    g = load_golden("nh9_3atlas")
    nh, div = int(g["nh"]), float(g["div"])
    handle.test_wait_timeout(100.0)
    t0 = time.perf_counter()
    with pytest.raises(pct.PctError) as e:
        handle.synthesize(g["img"], g["atlas_mri"], g["label"], nh, div)
    assert e.value.status == -6
    assert time.perf_counter() - t0 >= 0.1
    # the hook is one-shot and the context is still usable
    out = handle.synthesize(g["img"], g["atlas_mri"], g["label"], nh, div)
    _, prod, sumw = oracle.fuse_port(g["img"], g["atlas_mri"], g["label"], nh, div, with_sums=True)
    compare_fused(out, g["out"], nh, 1e-4, prod, sumw)


def test_timeout_surfaces_through_device_status(handle):
    g = load_golden("small_nh7_2atlas")
    dev = torch.device("cuda:0")
    img = torch.from_numpy(g["img"]).to(dev)
    atl = torch.from_numpy(g["atlas_mri"]).to(dev)
    lab = torch.from_numpy(g["label"]).to(dev)
    out = torch.zeros_like(img)
    nz, nx, ny = img.shape
    stream = torch.cuda.current_stream().cuda_stream
    handle.test_wait_timeout(50.0)
    handle.synthesize_device(img.data_ptr(), atl.data_ptr(), lab.data_ptr(), out.data_ptr(), nx, ny,
                             nz, 2, 7, float(g["div"]), pct.EXEC_B200_FP32, stream)
    with pytest.raises(pct.PctError) as e:
        handle.device_status(stream)
    assert e.value.status == -6
    handle.device_status(stream)  # cleared
    handle.synthesize_device(img.data_ptr(), atl.data_ptr(), lab.data_ptr(), out.data_ptr(), nx, ny,
                             nz, 2, 7, float(g["div"]), pct.EXEC_B200_FP32, stream)
    handle.device_status(stream)
    compare_fused(out.cpu().numpy(), g["out"], 7, 1e-4)


def _ncc_numpy(a, b, nh):
    lo = (nh - 1) // 2 + 1
    a = a[lo:-lo, lo:-lo, lo:-lo].astype(np.float64)
    b = b[lo:-lo, lo:-lo, lo:-lo].astype(np.float64)
    m = ~np.isnan(a) & ~np.isnan(b)
    a, b = a[m], b[m]
    return float(np.corrcoef(a, b)[0, 1]), int(m.sum())


def test_ncc_matches_float64_reference(handle):
    g = load_golden("small_nh7_2atlas")
    a = g["out"]
    rng = np.random.default_rng(3)
    b = (a + rng.normal(0, 5, a.shape)).astype(np.float32)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    nz, nx, ny = a.shape
    v, n = handle.ncc_device(da.data_ptr(), db.data_ptr(), nx, ny, nz, 7)
    ref, nref = _ncc_numpy(a, b, 7)
    assert n == nref
    assert v == pytest.approx(ref, abs=1e-9)
    one, _ = handle.ncc_device(da.data_ptr(), da.data_ptr(), nx, ny, nz, 7)
    assert one == pytest.approx(1.0, abs=1e-12)
    neg = torch.from_numpy((-3 * a + 7).astype(np.float32)).cuda()
    m1, _ = handle.ncc_device(da.data_ptr(), neg.data_ptr(), nx, ny, nz, 7)
    assert m1 == pytest.approx(-1.0, abs=1e-6)


def test_ncc_of_fused_pseudo_ct_beats_a_single_atlas(handle):
    """Quality, the reference's way (NCC against a reference CT): fusing four displaced, noisy
    atlases correlates better with their consensus CT than a single atlas's CT does."""
    s = pct.synth_subject(48, 44, 36, 4, n_blobs=10, seed=21)
    label = pct.normalize_labels(s.atlas_ct)
    fused = handle.synthesize(s.img, s.atlas_mri, label, 7, 337.5)
    consensus = np.median(label, axis=0).astype(np.float32)
    nz, nx, ny = s.img.shape
    d_c = torch.from_numpy(consensus).cuda()
    ncc_fused, n = handle.ncc_device(torch.from_numpy(fused).cuda().data_ptr(), d_c.data_ptr(),
                                     nx, ny, nz, 7)
    single = [handle.ncc_device(torch.from_numpy(label[a].copy()).cuda().data_ptr(),
                                d_c.data_ptr(), nx, ny, nz, 7)[0] for a in range(4)]
    assert n > 0 and np.isfinite(ncc_fused)
    assert ncc_fused > min(single)
