"""Z-slab sharding (multi-GPU host logic) on the CPU: the slab plan, and world-size 2 and 3 gloo
process groups where each rank computes its slab with the FP64 oracle and the slabs are
all-gathered. The assembled volume must equal the unsharded oracle run exactly, since every
voxel's arithmetic is the same in a sub-volume."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
import pseudoctimaging_b200 as pct
from pseudoctimaging_b200 import shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(nz=26, seed=4):
    s = pct.synth_subject(24, 21, nz, 2, n_blobs=6, seed=seed)
    return s.img, s.atlas_mri, pct.normalize_labels(s.atlas_ct)


def _oracle_compute(nh, div):
    def compute(img, atlas, label):
        return oracle.fuse_port(img, atlas, label, nh, div)
    return compute


def _rank_main(rank, world, port, outdir, nh, div):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        img, atl, lab = _case()
        out = shard.synthesize_sharded(img, atl, lab, nh, div, compute=_oracle_compute(nh, div))
        np.save(os.path.join(outdir, f"r{rank}.npy"), out)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nz,nh,parts", [(32, 7, 1), (32, 7, 3), (30, 11, 4), (17, 5, 2),
                                         (20, 7, 9), (13, 11, 2)])
def test_slab_plan_covers_the_interior(nz, nh, parts):
    lo = (nh - 1) // 2 + 1
    plan = shard.slab_plan(nz, nh, parts)
    covered = []
    for s in plan:
        covered += list(range(s.z_begin, s.z_end))
        if s.planes:
            assert s.src_begin == s.z_begin - lo and s.src_end == s.z_end + lo
            assert 0 <= s.src_begin and s.src_end <= nz
    assert covered == list(range(lo, max(lo, nz - lo)))
    sizes = [s.planes for s in plan]
    assert max(sizes) - min(sizes) <= 1


def test_slab_plan_rejects_bad_arguments():
    with pytest.raises(pct.PctError):
        shard.slab_plan(30, 6, 2)
    with pytest.raises(pct.PctError):
        shard.slab_plan(30, 7, 0)
    import ctypes
    v = [ctypes.c_int() for _ in range(4)]
    refs = [ctypes.byref(x) for x in v]
    assert pct.lib.pct_slab_plan(30, 7, 0, 0, *refs) == -1
    assert pct.lib.pct_slab_plan(30, 7, 2, 2, *refs) == -1
    assert pct.lib.pct_slab_plan(0, 7, 2, 0, *refs) == -1
    assert pct.lib.pct_slab_plan(30, 7, 2, 1, *refs) == 0


@pytest.mark.parametrize("parts", [1, 2, 3, 5])
def test_passes_stitch_to_the_whole_volume(parts):
    img, atl, lab = _case()
    nh, div = 7, 337.5
    full = oracle.fuse_port(img, atl, lab, nh, div)
    out = np.zeros_like(img)
    for s in shard.slab_plan(img.shape[0], nh, parts):
        out[s.z_begin:s.z_end] = shard.synthesize_part(img, atl, lab, nh, div, s,
                                                       compute=_oracle_compute(nh, div))
    np.testing.assert_array_equal(np.isnan(out), np.isnan(full))
    np.testing.assert_array_equal(np.nan_to_num(out), np.nan_to_num(full))


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_assemble_the_whole_volume(tmp_path, world):
    nh, div = 7, 337.5
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), nh, div),
                       nprocs=world, join=True, start_method="spawn")
    img, atl, lab = _case()
    full = oracle.fuse_port(img, atl, lab, nh, div)
    for r in range(world):
        got = np.load(tmp_path / f"r{r}.npy")
        np.testing.assert_array_equal(np.isnan(got), np.isnan(full))
        np.testing.assert_array_equal(np.nan_to_num(got), np.nan_to_num(full))
