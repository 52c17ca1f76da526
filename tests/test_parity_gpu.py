"""CUDA path against the reference (golden fixtures) and the oracle, through the C ABI.

Tolerance: the plain FP32 path must match the reference's FP64 output within 1e-4 relative per
voxel (RTOL below); NaN masks must agree except for voxels whose FP64 sums sit within 0.1% of
DBL_EPSILON, where FP32 may fall on the other side of the reference's threshold.
"""
import numpy as np
import pytest
import torch

import oracle
import pseudoctimaging_b200 as pct
from conftest import compare_fused, golden_names, load_golden

pytestmark = pytest.mark.gpu
RTOL = 1e-4


@pytest.fixture(scope="module")
def handle():
    h = pct.Handle(0)
    yield h
    h.close()


def interior_slices(nh):
    lo = (nh - 1) // 2 + 1
    return (slice(lo, -lo),) * 3, lo


@pytest.mark.parametrize("name", golden_names())
def test_golden_fusion(handle, name):
    g = load_golden(name)
    nh, div = int(g["nh"]), float(g["div"])
    out = handle.synthesize(g["img"], g["atlas_mri"], g["label"], nh, div)
    _, prod, sumw = oracle.fuse_port(g["img"], g["atlas_mri"], g["label"], nh, div, with_sums=True)
    stats = compare_fused(out, g["out"], nh, RTOL, prod, sumw)
    # border voxels are zero, as the reference leaves them after its device memset
    border = np.ones(out.shape, bool)
    sl, _ = interior_slices(nh)
    border[sl] = False
    assert np.all(out[border] == 0)
    print(name, stats)


@pytest.mark.parametrize("nh,num", [(7, 1), (9, 2), (11, 2), (5, 1), (3, 2)])
def test_config0_against_oracle(handle, nh, num):
    """Config 0 (64x64x32, 20 blobs, sigma 2.5, beta 1) at every compiled window size."""
    s = pct.synth_subject(64, 64, 32, num, n_blobs=20, seed=0)
    label = pct.normalize_labels(s.atlas_ct)
    div = pct.div_from(2.5, 1.0)
    out = handle.synthesize(s.img, s.atlas_mri, label, nh, div)
    ref, prod, sumw = oracle.fuse_port(s.img, s.atlas_mri, label, nh, div, with_sums=True)
    print(nh, num, compare_fused(out, ref, nh, RTOL, prod, sumw))


@pytest.mark.parametrize("shape,nh,num", [
    ((13, 20, 40), 11, 2),   # one interior plane: direct form
    ((14, 19, 37), 11, 1),   # two interior planes: direct form
    ((15, 18, 35), 11, 2),   # three planes (one half-tile): tiled, half 1 shifted onto half 0
    ((9, 16, 33), 7, 1),     # one plane at NH7
    ((11, 17, 12), 7, 2),    # three planes, four interior rows along y
    ((23, 9, 45), 7, 1),     # one interior row along x
    ((21, 24, 9), 5, 2),     # one interior column along y
    ((12, 12, 12), 3, 3),    # NH3 cube
])
def test_thin_and_degenerate_volumes(handle, shape, nh, num):
    nz, nx, ny = shape
    s = pct.synth_subject(nx, ny, nz, num, n_blobs=4, seed=nz * 100 + nx)
    label = pct.normalize_labels(s.atlas_ct)
    out = handle.synthesize(s.img, s.atlas_mri, label, nh, 337.5)
    ref, prod, sumw = oracle.fuse_port(s.img, s.atlas_mri, label, nh, 337.5, with_sums=True)
    compare_fused(out, ref, nh, RTOL, prod, sumw)
    sl, _ = interior_slices(nh)
    border = np.ones(out.shape, bool)
    border[sl] = False
    assert np.all(out[border] == 0)


def test_reference_exec_choices_run_the_same_kernel(handle):
    g = load_golden("small_nh7_2atlas")
    outs = [handle.synthesize(g["img"], g["atlas_mri"], g["label"], 7, float(g["div"]), c)
            for c in (pct.EXEC_GM, pct.EXEC_GM2, pct.EXEC_SM, pct.EXEC_B200_FP32)]
    for o in outs[1:]:
        assert np.array_equal(o.view(np.uint32), outs[0].view(np.uint32))


def test_repeat_calls_are_deterministic_and_reuse_buffers(handle):
    g = load_golden("nh9_3atlas")
    a = handle.synthesize(g["img"], g["atlas_mri"], g["label"], 9, float(g["div"]))
    b = handle.synthesize(g["img"], g["atlas_mri"], g["label"], 9, float(g["div"]))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("nh", [2, 1, 0, -3, 8])
def test_bad_window_rejected(handle, nh):
    g = load_golden("small_nh7_2atlas")
    with pytest.raises(pct.PctError) as e:
        handle.synthesize(g["img"], g["atlas_mri"], g["label"], nh, 337.5)
    assert e.value.status == -1


def test_window_beyond_compiled_range_is_unsupported(handle):
    g = load_golden("nh11_2atlas")
    with pytest.raises(pct.PctError) as e:
        handle.synthesize(g["img"], g["atlas_mri"], g["label"], 13, 337.5)
    assert e.value.status == -4


@pytest.mark.parametrize("div", [0.0, -1.0, float("nan"), float("inf")])
def test_bad_div_rejected(handle, div):
    g = load_golden("small_nh7_2atlas")
    with pytest.raises(pct.PctError) as e:
        handle.synthesize(g["img"], g["atlas_mri"], g["label"], 7, div)
    assert e.value.status == -1


def test_unknown_exec_choice_rejected(handle):
    g = load_golden("small_nh7_2atlas")
    with pytest.raises(pct.PctError) as e:
        handle.synthesize(g["img"], g["atlas_mri"], g["label"], 7, 337.5, 42)
    assert e.value.status == -1


def test_memory_limit_reports_out_of_memory():
    g = load_golden("nh9_3atlas")
    with pct.Handle(0) as h:
        h.set_memory_limit(1024)
        with pytest.raises(pct.PctError) as e:
            h.synthesize(g["img"], g["atlas_mri"], g["label"], 9, 337.5)
        assert e.value.status == -3
        h.set_memory_limit(0)
        h.synthesize(g["img"], g["atlas_mri"], g["label"], 9, 337.5)


def test_device_api_writes_interior_only(handle):
    g = load_golden("nh9_3atlas")
    nh, div = 9, float(g["div"])
    dev = torch.device("cuda:0")
    img = torch.from_numpy(g["img"]).to(dev)
    atl = torch.from_numpy(g["atlas_mri"]).to(dev)
    lab = torch.from_numpy(g["label"]).to(dev)
    out = torch.full_like(img, 7.0)
    nz, nx, ny = img.shape
    stream = torch.cuda.current_stream().cuda_stream
    handle.synthesize_device(img.data_ptr(), atl.data_ptr(), lab.data_ptr(), out.data_ptr(),
                             nx, ny, nz, atl.shape[0], nh, div, pct.EXEC_B200_FP32, stream)
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    sl, _ = interior_slices(nh)
    border = np.ones(o.shape, bool)
    border[sl] = False
    assert np.all(o[border] == 7.0)
    host = handle.synthesize(g["img"], g["atlas_mri"], g["label"], nh, div)
    assert np.array_equal(o[sl].view(np.uint32), host[sl].view(np.uint32))


def test_kernel_timing_counts_fusion_launches():
    """The fusion kernel's own device time, as the benchmark's roofline reads it: one timed
    launch per plain call while timing is on, each inside the call's own span on the stream,
    none while it is off, and a read starts the count over."""
    g = load_golden("nh9_3atlas")
    nh, div = 9, float(g["div"])
    dev = torch.device("cuda:0")
    img, atl, lab = (torch.from_numpy(g[k]).to(dev) for k in ("img", "atlas_mri", "label"))
    out = torch.zeros_like(img)
    nz, nx, ny = img.shape
    stream = torch.cuda.current_stream()
    with pct.Handle(0) as h:
        def call():
            h.synthesize_device(img.data_ptr(), atl.data_ptr(), lab.data_ptr(), out.data_ptr(),
                                nx, ny, nz, atl.shape[0], nh, div, pct.EXEC_B200_FP32,
                                stream.cuda_stream)
        call()
        assert h.kernel_time() == (0.0, 0)
        h.set_kernel_timing(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms, n = h.kernel_time()
        assert n == 3 and 0.0 < ms <= e0.elapsed_time(e1)
        assert h.kernel_time() == (0.0, 0)
        # a volume with no interior voxel launches no fusion kernel and times nothing
        flat = np.zeros((2 * 5, 12, 12), np.float32)
        h.synthesize(flat, flat[None], flat[None], nh, div)
        assert h.kernel_time() == (0.0, 0)
        h.set_kernel_timing(False)
        call()
        torch.cuda.synchronize()
        assert h.kernel_time() == (0.0, 0)


@pytest.fixture(scope="module")
def full_subject():
    """Config 1 inputs: 222x222x112, 60 blobs, 10 atlases (seed 1)."""
    s = pct.synth_subject(222, 222, 112, 10, n_blobs=60, seed=1)
    return s, pct.normalize_labels(s.atlas_ct)


@pytest.mark.parametrize("nh", [7, 9, 11])
def test_full_size_sampled_voxels(handle, full_subject, nh):
    """Full config-1 volume on the GPU; the oracle recomputes 1500 random interior voxels."""
    s, label = full_subject
    div = pct.div_from(2.5, 1.0)
    out = handle.synthesize(s.img, s.atlas_mri, label, nh, div)
    nz, nx, ny = s.img.shape
    lo = (nh - 1) // 2 + 1
    rng = np.random.default_rng(nh)
    z = rng.integers(lo, nz - lo, 1500)
    x = rng.integers(lo, nx - lo, 1500)
    y = rng.integers(lo, ny - lo, 1500)
    vox = z * nx * ny + x * ny + y
    ref, prod, sumw = oracle.fuse_port_voxels(s.img, s.atlas_mri, label, nh, div, vox)
    got = out.reshape(-1)[vox]
    gn, rn = np.isnan(got), np.isnan(ref)
    mism = gn != rn
    if mism.any():
        near = (np.abs(np.abs(prod[mism]) / 2.220446049250313e-16 - 1) < 1e-3) | \
               (np.abs(np.abs(sumw[mism]) / 2.220446049250313e-16 - 1) < 1e-3)
        assert near.all()
    both = ~gn & ~rn
    rel = np.abs(got[both].astype(np.float64) - ref[both]) / np.maximum(np.abs(ref[both]), 1e-30)
    assert rel.max() <= RTOL, rel.max()


def test_full_size_properties(handle, full_subject):
    """Size-independent properties at the full config-1 size (NH=11):
    the fused value is a weighted mean of atlas CT labels, so (1) permuting the atlases leaves
    it unchanged, (2) scaling every label by c scales it by c, (3) adding a constant to every
    label adds that constant, and (4) it lies within the range of the labels."""
    s, label = full_subject
    div = pct.div_from(2.5, 1.0)
    nh = 11
    sl, _ = interior_slices(nh)
    base = handle.synthesize(s.img, s.atlas_mri, label, nh, div)[sl]
    fin = ~np.isnan(base)
    perm = np.array([3, 7, 0, 9, 1, 5, 2, 8, 6, 4])
    p = handle.synthesize(s.img, s.atlas_mri[perm], label[perm], nh, div)[sl]
    assert np.array_equal(np.isnan(p), ~fin)
    np.testing.assert_allclose(p[fin], base[fin], rtol=2e-5, atol=1e-5)
    sc = handle.synthesize(s.img, s.atlas_mri, label * np.float32(2.0), nh, div)[sl]
    np.testing.assert_allclose(sc[fin], 2 * base[fin], rtol=2e-5, atol=1e-5)
    sh = handle.synthesize(s.img, s.atlas_mri, label + np.float32(100.0), nh, div)[sl]
    np.testing.assert_allclose(sh[fin], base[fin] + 100, rtol=2e-5, atol=2e-3)
    assert base[fin].min() >= label.min() - 1e-3 and base[fin].max() <= label.max() + 1e-3


def test_identical_atlas_with_constant_ct_returns_the_constant(handle):
    """An atlas equal to the input with CT c everywhere fuses to c wherever weights survive."""
    s = pct.synth_subject(40, 36, 30, 1, n_blobs=8, seed=11)
    label = np.full_like(s.atlas_mri, 123.25)
    out = handle.synthesize(s.img, s.img[None], label, 7, 337.5)
    sl, _ = interior_slices(7)
    v = out[sl]
    assert not np.isnan(v).any()   # the zero-offset candidate has weight 1
    np.testing.assert_allclose(v, 123.25, rtol=1e-5)
