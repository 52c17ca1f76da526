"""The host-pointer path with overlapped uploads: when the plan splits the atlases into two or
more groups, pct_synthesize and pct_run_pipeline launch the first group while the rest upload.
The same items run in the same group order and the combine adds the groups in the same order,
so the result must equal the device-pointer path (one launch) bit for bit; under a memory cap
too small for the double staging area the call falls back to the single upload."""
import numpy as np
import pytest
import torch

import pseudoctimaging_b200 as pct

pytestmark = pytest.mark.gpu


def device_run(h, img, atl, lab, nh, div):
    d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (img, atl, lab)]
    out = torch.zeros_like(d[0])
    nz, nx, ny = img.shape
    h.synthesize_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), out.data_ptr(), nx, ny,
                        nz, atl.shape[0], nh, div, pct.EXEC_B200_FP32)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def first_group_split(plan, nx, ny, nz, nh):
    """Whether the first atlas group uploads in plane ranges: the z-tiles that give every CTA of
    the grid an item read fewer planes than the volume has."""
    lo = (nh - 1) // 2 + 1
    tiles_xy = -(-(ny - 2 * lo) // 30) * -(-(nx - 2 * lo) // (4 * plan["tile_rows"]))
    zt = 2 * plan["tile_planes"]
    tiles_z = -(-(nz - 2 * lo) // zt)
    first = -(-plan["ctas"] // tiles_xy)
    return first < tiles_z and first * zt + 2 + 2 * (lo - 1) < nz


@pytest.mark.parametrize("shape,nh,min_groups,split",
                         [((64, 70, 48, 6), 11, 2, False), ((90, 61, 40, 4), 7, 2, False),
                          ((40, 45, 30, 10), 11, 3, False), ((222, 222, 112, 4), 11, 3, True),
                          ((64, 70, 252, 4), 7, 3, True)])
def test_pipelined_host_path_equals_device_path(shape, nh, min_groups, split):
    """Every atlas group after the first runs in a launch of its own as soon as it has landed;
    on volumes with more z-tiles than one round of the grid needs, the first group's first
    z-tiles start before the rest of its planes have landed."""
    nx, ny, nz, num = shape
    plan = pct.query_plan(nx, ny, nz, num, nh)
    assert plan["groups"] >= min_groups, plan  # the shape must take the pipelined path
    assert first_group_split(plan, nx, ny, nz, nh) == split, plan
    s = pct.synth_subject(nx, ny, nz, num, n_blobs=10, seed=nh)
    lab = pct.normalize_labels(s.atlas_ct)
    div = pct.div_from(2.5, 1.0)
    with pct.Handle(0) as h:
        host = h.synthesize(s.img, s.atlas_mri, lab, nh, div, pct.EXEC_B200_FP32)
        dev = device_run(h, s.img, s.atlas_mri, lab, nh, div)
        np.testing.assert_array_equal(np.isnan(host), np.isnan(dev))
        np.testing.assert_array_equal(np.nan_to_num(host), np.nan_to_num(dev))
        # the pipeline entry point normalises on the device: same fused volume before the fill
        piped = h.run_pipeline(s.img, s.atlas_mri, s.atlas_ct, nh, 2.5, 1.0,
                               pct.EXEC_B200_FP32, regularize=False)
        np.testing.assert_array_equal(np.isnan(piped), np.isnan(host))
        np.testing.assert_array_equal(np.nan_to_num(piped), np.nan_to_num(host))


def test_memory_cap_falls_back_to_single_upload():
    nx, ny, nz, num, nh = 64, 70, 48, 6, 11
    s = pct.synth_subject(nx, ny, nz, num, n_blobs=10, seed=3)
    lab = pct.normalize_labels(s.atlas_ct)
    div = pct.div_from(2.5, 1.0)
    with pct.Handle(0) as h:
        ref = h.synthesize(s.img, s.atlas_mri, lab, nh, div, pct.EXEC_B200_FP32)
    vox = nx * ny * nz * 4
    pitch = (ny + 3) // 4 * 4
    stacks = 2 * num * nz * nx * pitch * 4
    partial = pct.query_plan(nx, ny, nz, num, nh)["scratch_bytes"]
    # room for everything the single upload needs (img, out, stacks, one staging stack,
    # partial sums, status word), not for the pipelined path's second staging stack
    cap = 2 * vox + stacks + num * vox + partial + 4096
    with pct.Handle(0) as h:
        h.set_memory_limit(cap)
        got = h.synthesize(s.img, s.atlas_mri, lab, nh, div, pct.EXEC_B200_FP32)
    np.testing.assert_array_equal(np.nan_to_num(got), np.nan_to_num(ref))
