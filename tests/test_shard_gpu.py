"""Z-slab sharding with the CUDA path, as passes on one GPU: each slab's sub-volume (slab plus
hw+1 halo planes) through pct_synthesize, stitched, against the unsharded run of the same
kernel and against the FP64 oracle. The atlas-group split of a sub-volume can differ from the
whole volume's, so the two CUDA runs agree within the cross-path tolerance (2e-5), not bitwise."""
import numpy as np
import pytest

import oracle
import pseudoctimaging_b200 as pct
from conftest import compare_fused
from pseudoctimaging_b200 import shard

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nh,parts,choice", [(7, 3, pct.EXEC_B200_FP32), (11, 2, pct.EXEC_B200_FP32),
                                             (9, 4, pct.EXEC_B200_FP32)])
def test_sharded_passes_match_whole_volume(nh, parts, choice):
    s = pct.synth_subject(46, 37, 41, 3, n_blobs=8, seed=60 + nh)
    lab = pct.normalize_labels(s.atlas_ct)
    div = pct.div_from(2.5, 1.0)
    with pct.Handle(0) as h:
        whole = h.synthesize(s.img, s.atlas_mri, lab, nh, div, choice)
        out = np.zeros_like(whole)
        for sl in shard.slab_plan(s.img.shape[0], nh, parts):
            out[sl.z_begin:sl.z_end] = shard.synthesize_part(s.img, s.atlas_mri, lab, nh, div, sl,
                                                             handle=h, exec_choice=choice)
    ref, prod, sumw = oracle.fuse_port(s.img, s.atlas_mri, lab, nh, div, with_sums=True)
    compare_fused(out, whole, nh, 2e-5)
    compare_fused(out, ref, nh, 1e-4, prod, sumw)
    lo = (nh - 1) // 2 + 1
    assert np.all(out[:lo] == 0) and np.all(out[-lo:] == 0)


def test_sharded_learned_form_matches_whole_volume():
    from pseudoctimaging_b200 import learned
    s = pct.synth_subject(40, 47, 44, 2, n_blobs=8, seed=71)
    lab = pct.normalize_labels(s.atlas_ct)
    div = pct.div_from(2.5, 1.0)
    with pct.Handle(0) as h, learned.LearnedModel.load(learned.CHECKPOINT) as m:
        h.attach_model(m, 0.0)
        h.set_learned_block(1)  # per-row proposals: independent of where the slabs start
        whole = h.synthesize(s.img, s.atlas_mri, lab, 11, div, pct.EXEC_LEARNED)
        out = np.zeros_like(whole)
        for sl in shard.slab_plan(s.img.shape[0], 11, 3):
            out[sl.z_begin:sl.z_end] = shard.synthesize_part(s.img, s.atlas_mri, lab, 11, div, sl,
                                                             handle=h,
                                                             exec_choice=pct.EXEC_LEARNED)
    # the network sees zeros beyond the sub-volume only outside the interior's receptive field,
    # and the rows and their proposals are the same: the slabs reproduce the whole run exactly
    np.testing.assert_array_equal(np.isnan(out), np.isnan(whole))
    np.testing.assert_array_equal(np.nan_to_num(out), np.nan_to_num(whole))
