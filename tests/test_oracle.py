"""The CPU oracles against the reference's own outputs (no GPU).

The C restatement (oracle/pct_oracle.c) must reproduce the golden fixtures, which were produced
by the unmodified reference routines, bit for bit; where the reference library is built it is
also cross-checked live on fresh seeds.
"""
import numpy as np
import pytest

import oracle
from conftest import golden_names, load_golden

NAMES = golden_names()


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", NAMES)
def test_port_matches_golden_fusion(name):
    g = load_golden(name)
    out = oracle.fuse_port(g["img"], g["atlas_mri"], g["label"], int(g["nh"]), float(g["div"]))
    assert np.array_equal(bits(out), bits(g["out"]))


@pytest.mark.parametrize("name", NAMES)
def test_port_matches_golden_post(name):
    g = load_golden(name)
    nh = int(g["nh"])
    reg, _ = oracle.regularize_port(g["out"], nh)
    assert np.array_equal(bits(reg), bits(g["regularized"]))
    assert np.array_equal(bits(oracle.finalize_port(reg)), bits(g["hu"]))


@pytest.mark.parametrize("name", NAMES)
def test_label_normalisation_matches(name):
    g = load_golden(name)
    assert np.array_equal(bits(oracle.normalize_labels_port(g["atlas_ct_hu"])), bits(g["label"]))


def test_div_formula():
    assert oracle.div_port(2.5, 1.0) == 337.5
    assert oracle.div_port(1.0, 1.0) == 54.0


def test_voxel_sampling_matches_full_volume():
    g = load_golden("nh9_3atlas")
    nh, div = int(g["nh"]), float(g["div"])
    full, prod, sumw = oracle.fuse_port(g["img"], g["atlas_mri"], g["label"], nh, div, with_sums=True)
    rng = np.random.default_rng(0)
    vox = rng.integers(0, full.size, 300)
    out, p, s = oracle.fuse_port_voxels(g["img"], g["atlas_mri"], g["label"], nh, div, vox)
    assert np.array_equal(bits(out), bits(full.reshape(-1)[vox]))
    inside = p != 0
    assert np.array_equal(p[inside], prod.reshape(-1)[vox][inside])
    assert np.array_equal(s[inside], sumw.reshape(-1)[vox][inside])


@pytest.mark.skipif(not oracle.has_reference(), reason="reference library not built here")
@pytest.mark.parametrize("seed,shape,num,nh", [(7, (21, 19, 25), 2, 7), (8, (24, 26, 22), 1, 9),
                                               (9, (26, 25, 27), 1, 11)])
def test_port_matches_reference_live(seed, shape, num, nh):
    import pseudoctimaging_b200 as pct

    nz, nx, ny = shape
    s = pct.synth_subject(nx, ny, nz, num, n_blobs=6, seed=seed)
    label = pct.normalize_labels(s.atlas_ct)
    ref = oracle.fuse_reference(s.img, s.atlas_mri, label, nh, 337.5)
    port = oracle.fuse_port(s.img, s.atlas_mri, label, nh, 337.5)
    assert np.array_equal(bits(ref), bits(port))
    # single-core reference routine agrees with its OpenMP twin
    single = oracle.fuse_reference(s.img, s.atlas_mri, label, nh, 337.5, multicore=False)
    assert np.array_equal(bits(single), bits(ref))


def test_planted_error_is_detected():
    """The checker catches a wrong value: perturb one oracle voxel and compare."""
    from conftest import compare_fused

    g = load_golden("small_nh7_2atlas")
    ref = g["out"]
    bad = ref.copy()
    lo = 4
    finite = np.argwhere(~np.isnan(bad[lo:-lo, lo:-lo, lo:-lo]))[0] + lo
    bad[tuple(finite)] *= 1.001
    with pytest.raises(AssertionError):
        compare_fused(bad, ref, 7, rtol=1e-4)
    nan_bad = ref.copy()
    nan_bad[tuple(finite)] = np.nan
    with pytest.raises(AssertionError):
        compare_fused(nan_bad, ref, 7, rtol=1e-4)
