"""Learned-proposal form, host side (no GPU): checkpoint format, the committed checkpoint, the
kept-set rule and the training samplers."""
import numpy as np
import pytest

import pseudoctimaging_b200 as pct
from pseudoctimaging_b200 import learned


def test_checkpoint_round_trip(tmp_path):
    p = np.random.default_rng(0).standard_normal(learned.NUM_PARAMS).astype(np.float32)
    learned.save_params(tmp_path / "a.pctl", p)
    raw = (tmp_path / "a.pctl").read_bytes()
    assert raw[:8] == b"PCTLRN01" and len(raw) == 16 + 4 * learned.NUM_PARAMS
    np.testing.assert_array_equal(learned.load_params(tmp_path / "a.pctl"), p)


def test_checkpoint_rejects_bad_files(tmp_path):
    (tmp_path / "bad.pctl").write_bytes(b"NOTMODEL" + bytes(8) + bytes(4 * learned.NUM_PARAMS))
    with pytest.raises(ValueError):
        learned.load_params(tmp_path / "bad.pctl")
    short = b"PCTLRN01" + np.array([10, 0], "<u4").tobytes() + bytes(40)
    (tmp_path / "short.pctl").write_bytes(short)
    with pytest.raises(ValueError):
        learned.load_params(tmp_path / "short.pctl")
    with pytest.raises(ValueError):
        learned.save_params(tmp_path / "x.pctl", np.zeros(5, np.float32))


def test_committed_checkpoint_loads():
    p = learned.load_params(learned.CHECKPOINT)
    assert p.shape == (learned.NUM_PARAMS,) and np.isfinite(p).all()
    assert np.abs(p).max() < 100


def test_rank_sum_set():
    top = np.array([[0, -1, 1, -2], [0, 1, -1, 2], [3, 2, 4, 1]])
    s = learned.rank_sum_set(top)
    assert len(s) == 32 and len({tuple(o) for o in s}) == 32
    assert tuple(s[0]) == (0, 0, 3)  # ranks (0, 0, 0) first
    # every rank triple with i + j + k <= 4 and nothing else
    ranks = {(list(top[0]).index(a), list(top[1]).index(b), list(top[2]).index(c)) for a, b, c in s}
    assert ranks == {(i, j, k) for i in range(4) for j in range(4) for k in range(4)
                     if i + j + k <= 4}


@pytest.mark.parametrize("k,level", [(10, 2), (20, 3), (32, 4)])
def test_rank_sum_set_sizes_nest(k, level):
    """The smaller kept sets are the rank triples of lower rank sum, each inside the next."""
    top = np.array([[0, -1, 1, -2], [0, 1, -1, 2], [3, 2, 4, 1]])
    s = {tuple(o) for o in learned.rank_sum_set(top, k)}
    assert len(s) == k and learned.KEPT_LEVEL[k] == level
    ranks = {(list(top[0]).index(a), list(top[1]).index(b), list(top[2]).index(c)) for a, b, c in s}
    assert ranks == {(i, j, l) for i in range(4) for j in range(4) for l in range(4)
                     if i + j + l <= level}
    bigger = {10: 20, 20: 32, 32: 32}[k]
    assert s <= {tuple(o) for o in learned.rank_sum_set(top, bigger)}
    with pytest.raises(KeyError):
        learned.rank_sum_set(top, 16)


def test_samplers_stay_in_the_interior():
    shapes = [(40, 44, 30, 3), (36, 50, 28, 2)]
    smp = learned.random_samples(shapes, 5000, 1)
    for s, a, v in smp:
        nx, ny, nz, num = shapes[s]
        z, x, y = v // (nx * ny), (v % (nx * ny)) // ny, v % ny
        assert 0 <= a < num and 6 <= z < nz - 6 and 6 <= x < nx - 6 and 6 <= y < ny - 6
    subj = pct.synth_subject(40, 44, 30, 2, n_blobs=6, seed=3)
    st = learned.structured_samples([subj.img], 2, 3000, 2)
    nz, nx, ny = subj.img.shape
    z, x, y = st[:, 2] // (nx * ny), (st[:, 2] % (nx * ny)) // ny, st[:, 2] % ny
    assert (z >= 6).all() and (z < nz - 6).all() and (x >= 6).all() and (x < nx - 6).all()
    assert (y >= 6).all() and (y < ny - 6).all() and set(np.unique(st[:, 1])) <= {0, 1}
    # gradient-weighted: the sampled voxels have a larger mean gradient than the interior's
    g = np.sqrt(sum(d.astype(np.float64) ** 2 for d in np.gradient(subj.img)))
    assert g.ravel()[st[:, 2]].mean() > 1.5 * g[6:-6, 6:-6, 6:-6].mean()


def test_prior_params_shape():
    p = learned.prior_params()
    assert p.shape == (learned.NUM_PARAMS,)
    assert np.count_nonzero(p) == 30  # 3 axes x 10 offsets off the centre
