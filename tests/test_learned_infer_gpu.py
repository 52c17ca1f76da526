"""Learned-proposal form, inference side, on the GPU (EXEC_CHOICE 7).

* With every pair forced to the full search (threshold above 1) the form is the plain method and
  must match the FP64 oracle within the plain gate (1e-4 relative).
* With a fixed "prior" network (zero convolutions, head biases only) every voxel and every row
  gets the same k offsets (32, 20 or 10), so the output has an exact float64 restatement: the
  fusion over those offsets.
* The committed trained network beats the same-k baselines without it (the centre prior and an
  untrained network) in recall of the plain method's top-32 and in error against the plain
  method.
* The tensor-core convolutions and the proposal step are checked voxel by voxel against a float64
  restatement of the network on the BF16 weights.
"""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

import learned_ref
import oracle
import pseudoctimaging_b200 as pct
from conftest import DBL_EPS, compare_fused
from pseudoctimaging_b200 import learned

pytestmark = pytest.mark.gpu
NH = 11
LO = 6
DIV = 337.5


def subject(nx, ny, nz, num, seed):
    s = pct.synth_subject(nx, ny, nz, num, n_blobs=12, seed=seed)
    return s.img, s.atlas_mri, pct.normalize_labels(s.atlas_ct)


prior_params = learned.prior_params


def prior_proposal(scales=(0.7, 0.5, 0.3), k=32):
    """Offsets in rank order per axis and the confidence of the k kept offsets, in float64 (ties:
    lower offset first)."""
    top, probs = [], []
    for c in scales:
        logits = np.array([-c * (j - 5) ** 2 for j in range(11)], np.float64)
        p = np.exp(logits - logits.max())
        p /= p.sum()
        order = sorted(range(11), key=lambda j: (-p[j], j))[:4]
        top.append([j - 5 for j in order])
        probs.append([p[j] for j in order])
    level = learned.KEPT_LEVEL[k]
    conf = sum(probs[0][i] * probs[1][j] * probs[2][l] for i in range(4) for j in range(4)
               for l in range(4) if i + j + l <= level)
    return np.array(top), conf


def fuse_offsets_f64(img, atlas, label, offsets, div, LO=LO):
    """Float64 fusion over a fixed offset list at every interior voxel (interior from LO);
    (out, prod, sumw)."""
    nz, nx, ny = img.shape
    I = img.astype(np.float64)
    shape = (nz - 2 * LO, nx - 2 * LO, ny - 2 * LO)
    P, W = np.zeros(shape), np.zeros(shape)

    def win(vol, dz, dx, dy):
        return vol[LO + dz:nz - LO + dz, LO + dx:nx - LO + dx, LO + dy:ny - LO + dy]

    for a in range(atlas.shape[0]):
        A = atlas[a].astype(np.float64)
        L = label[a].astype(np.float64)
        for dw, du, dv in offsets:
            ssd = np.zeros(shape)
            for dz in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        ssd += (win(I, dz, dx, dy) - win(A, dz + dw, dx + du, dy + dv)) ** 2
            w = np.exp(-ssd / div)
            P += w * win(L, dw, du, dv)
            W += w
    out = np.zeros_like(img)
    prod, sumw = np.zeros(img.shape), np.zeros(img.shape)
    core = (slice(LO, nz - LO), slice(LO, nx - LO), slice(LO, ny - LO))
    ok = (np.abs(P) > DBL_EPS) & (np.abs(W) > DBL_EPS)
    out[core] = np.where(ok, P / np.where(ok, W, 1.0), np.nan)
    prod[core], sumw[core] = P, W
    return out, prod, sumw


def rows_of(nx, ny, nz, lo=LO):
    return (nz - 2 * lo) * (nx - 2 * lo) * -(-(ny - 2 * lo) // 30)


def interior(nx, ny, nz, lo=LO):
    return (nz - 2 * lo) * (nx - 2 * lo) * (ny - 2 * lo)


def test_attach_rules():
    img, atl, lab = subject(30, 31, 28, 1, 5)
    with pct.Handle(0) as h:
        with pytest.raises(pct.PctError) as e:
            h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        assert e.value.status == -4
        with learned.LearnedModel(0, seed=1) as m:
            with pytest.raises(pct.PctError) as e:
                h.attach_model(m, -0.5)
            assert e.value.status == -1
            h.attach_model(m, 0.0)
            with pytest.raises(pct.PctError) as e:  # NH 7, 9 and 11 only
                h.synthesize(img, atl, lab, 5, DIV, pct.EXEC_LEARNED)
            assert e.value.status == -4
            out = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
            assert np.all(out[:LO] == 0) and np.all(out[:, :, -LO:] == 0)
            h.attach_model(None)
            with pytest.raises(pct.PctError):
                h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        for bad in (0, 16, 33):
            with pytest.raises(pct.PctError) as e:
                h.set_learned_k(bad)
            assert e.value.status == -1


@pytest.mark.parametrize("shape", [(36, 41, 30, 2), (44, 70, 33, 3)])
def test_full_fallback_is_the_plain_method(shape):
    nx, ny, nz, num = shape
    img, atl, lab = subject(nx, ny, nz, num, 11)
    ref, prod, sumw = oracle.fuse_port(img, atl, lab, NH, DIV, with_sums=True)
    with pct.Handle(0) as h, learned.LearnedModel(0, seed=2) as m:
        h.attach_model(m, 2.0)
        got = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        st = h.learned_stats()
    compare_fused(got, ref, NH, 1e-4, prod, sumw)
    assert st["fallback_pairs"] == interior(nx, ny, nz) * num
    assert st["row_offsets"] == rows_of(nx, ny, nz) * 1331 * num


def centre_offsets(k):
    """The k offsets of the 11^3 window nearest its centre, by squared distance, ties in
    (dw, du, dv) order (a stable sort of the lexicographic enumeration)."""
    import itertools
    return sorted(itertools.product(range(-5, 6), repeat=3),
                  key=lambda o: o[0] ** 2 + o[1] ** 2 + o[2] ** 2)[:k]


@pytest.mark.parametrize("k", [1, 7, 32, 57, 125])
def test_centre_prior_without_network_exact(k):
    """The no-network baseline (pct_set_learned_prior): no convolutions, no proposal, every voxel
    rescores the k centre offsets; exact against the float64 fusion over those offsets."""
    nx, ny, nz, num = 36, 41, 30, 2
    img, atl, lab = subject(nx, ny, nz, num, 21)
    ref, prod, sumw = fuse_offsets_f64(img, atl, lab, centre_offsets(k), DIV)
    with pct.Handle(0) as h:
        h.set_learned_prior(k)  # no model attached: the prior needs none
        got = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        st = h.learned_stats()
        with learned.LearnedModel(0, seed=3) as m:  # an attached model does not change it
            h.attach_model(m, 0.5)
            again = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
            h.attach_model(None)
        h.set_learned_prior(0)
        with pytest.raises(pct.PctError) as e:  # back to the network, which is not attached
            h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        assert e.value.status == -4
        for bad in (-1, 126):
            with pytest.raises(pct.PctError) as e:
                h.set_learned_prior(bad)
            assert e.value.status == -1
    compare_fused(got, ref, NH, 1e-4, prod, sumw)
    assert np.array_equal(got.view(np.uint32), again.view(np.uint32))
    assert st["fallback_pairs"] == 0
    assert st["row_offsets"] == rows_of(nx, ny, nz) * k * num


@pytest.mark.parametrize("k,block", [(32, 4), (20, 4), (10, 4), (20, 1)])
def test_prior_proposal_exact(k, block):
    nx, ny, nz, num = 40, 47, 32, 2
    img, atl, lab = subject(nx, ny, nz, num, 21)
    top, conf = prior_proposal(k=k)
    offsets = learned.rank_sum_set(top, k)
    assert len({tuple(o) for o in offsets}) == k
    ref, prod, sumw = fuse_offsets_f64(img, atl, lab, offsets, DIV)
    with pct.Handle(0) as h, learned.LearnedModel(0, params=prior_params()) as m:
        h.attach_model(m, 0.0)
        h.set_learned_k(k)
        h.set_learned_block(block)
        got = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        st = h.learned_stats()
    compare_fused(got, ref, NH, 1e-4, prod, sumw)
    assert st["fallback_pairs"] == 0
    assert st["row_offsets"] == rows_of(nx, ny, nz) * k * num


@pytest.mark.parametrize("k", [32, 20])
def test_confidence_threshold(k):
    nx, ny, nz, num = 34, 37, 29, 1
    img, atl, lab = subject(nx, ny, nz, num, 31)
    _, conf = prior_proposal(k=k)
    ref = oracle.fuse_port(img, atl, lab, NH, DIV)
    with pct.Handle(0) as h, learned.LearnedModel(0, params=prior_params()) as m:
        h.set_learned_k(k)
        h.attach_model(m, conf * (1 - 1e-3))
        h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        assert h.learned_stats()["fallback_pairs"] == 0
        h.attach_model(m, conf * (1 + 1e-3))
        got = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        assert h.learned_stats()["fallback_pairs"] == interior(nx, ny, nz) * num
    compare_fused(got, ref, NH, 1e-4)


def test_partial_fallback_runs_whole_tiles_through_the_plain_kernel():
    """Low-confidence voxels send their whole tile of the plain kernel (30 y x 12 x x 8 z voxels
    from the first interior voxel, tile set 0 at NH = 11) to its full search: every tile of the
    result equals either the no-fallback run bit for bit or the FP64 oracle within the plain gate,
    and the fallback count is the interior voxels of the tiles that fell back."""
    nx, ny, nz, num = 40, 70, 36, 1
    img, atl, lab = subject(nx, ny, nz, num, 51)
    ref, prod, sumw = oracle.fuse_port(img, atl, lab, NH, DIV, with_sums=True)
    core = (slice(LO, nz - LO), slice(LO, nx - LO), slice(LO, ny - LO))
    with pct.Handle(0) as h, learned.LearnedModel(0, seed=9) as m:
        h.attach_model(m, 0.0)
        base = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        partial = None
        for thr in np.geomspace(1e-3, 0.5, 40):
            h.attach_model(m, float(thr))
            got = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
            st = h.learned_stats()
            if 0 < st["fallback_pairs"] < interior(nx, ny, nz) * num:
                partial = (got, st)
                break
    assert partial is not None, "no threshold gave a partial fallback"
    got, st = partial
    iz, ix, iy = nz - 2 * LO, nx - 2 * LO, ny - 2 * LO
    g, b, r = got[core], base[core], ref[core]
    fell = 0
    for tz in range(0, iz, 8):
        for tx in range(0, ix, 12):
            for ty in range(0, iy, 30):
                t = (slice(tz, tz + 8), slice(tx, tx + 12), slice(ty, ty + 30))
                if np.array_equal(g[t].view(np.uint32), b[t].view(np.uint32)):
                    continue
                fin = np.isfinite(r[t])
                assert np.array_equal(np.isnan(g[t]), np.isnan(r[t]))
                rel = np.abs(g[t][fin] - r[t][fin]) / np.abs(r[t][fin])
                assert rel.max() <= 1e-4
                fell += g[t].size
    assert fell * num == st["fallback_pairs"]


def tiles_of(nx, ny, nz):
    """Interior-relative slices of the plain kernel's tiles (30 y x 12 x x 8 z at NH = 11)."""
    iz, ix, iy = nz - 2 * LO, nx - 2 * LO, ny - 2 * LO
    return [(slice(tz, tz + 8), slice(tx, tx + 12), slice(ty, ty + 30))
            for tz in range(0, iz, 8) for tx in range(0, ix, 12) for ty in range(0, iy, 30)]


def test_full_fallback_over_blocks_of_atlases():
    """A threshold above every confidence sends every (tile, atlas) pair to the plain kernel's full
    search: 35 atlases run as a block of 32 (16 pairs) and a block of 3 (a pair and a single), and
    the result is the full search of every atlas, within the plain gate of the FP64 oracle."""
    nx, ny, nz, num = 30, 45, 30, 35
    img, atl, lab = subject(nx, ny, nz, num, 61)
    ref = oracle.fuse_port(img, atl, lab, NH, DIV)
    core = (slice(LO, nz - LO), slice(LO, nx - LO), slice(LO, ny - LO))
    with pct.Handle(0) as h, learned.LearnedModel(0, seed=9) as m:
        h.attach_model(m, 2.0)
        got = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        st = h.learned_stats()
    assert st["fallback_pairs"] == interior(nx, ny, nz) * num
    g, r = got[core], ref[core]
    assert np.array_equal(np.isnan(g), np.isnan(r))
    fin = np.isfinite(r)
    assert (np.abs(g[fin] - r[fin]) / np.abs(r[fin])).max() <= 1e-4


def test_mixed_fallback_tiles_per_atlas():
    """With several atlases each atlas flags its own tiles: a tile no atlas flags equals the run
    without fallback bit for bit, a tile every atlas flags is the full search (FP64 oracle within
    the plain gate), and the fallback count is the sum of the atlases' own counts (each atlas run
    alone at the same threshold shows which tiles it flags)."""
    nx, ny, nz, num = 40, 70, 36, 3
    img, atl, lab = subject(nx, ny, nz, num, 53)
    ref = oracle.fuse_port(img, atl, lab, NH, DIV)
    core = (slice(LO, nz - LO), slice(LO, nx - LO), slice(LO, ny - LO))
    tiles = tiles_of(nx, ny, nz)
    with pct.Handle(0) as h, learned.LearnedModel(0, seed=9) as m:
        h.attach_model(m, 0.0)
        base = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)[core]
        singles0 = [h.synthesize(img, atl[a:a + 1], lab[a:a + 1], NH, DIV,
                                 pct.EXEC_LEARNED)[core] for a in range(num)]
        found = None
        for thr in np.geomspace(1e-3, 0.5, 40):
            h.attach_model(m, float(thr))
            got = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)[core]
            st = h.learned_stats()
            if 0 < st["fallback_pairs"] < interior(nx, ny, nz) * num:
                flagged, count = [], 0
                for a in range(num):
                    one = h.synthesize(img, atl[a:a + 1], lab[a:a + 1], NH, DIV,
                                       pct.EXEC_LEARNED)[core]
                    count += h.learned_stats()["fallback_pairs"]
                    flagged.append({i for i, t in enumerate(tiles) if not np.array_equal(
                        one[t].view(np.uint32), singles0[a][t].view(np.uint32))})
                found = (got, st, flagged, count)
                break
    assert found is not None, "no threshold gave a partial fallback"
    got, st, flagged, count = found
    assert st["fallback_pairs"] == count
    assert sum(len(f) for f in flagged) > 0
    r = ref[core]
    for i, t in enumerate(tiles):
        hit = sum(i in f for f in flagged)
        if hit == 0:
            assert np.array_equal(got[t].view(np.uint32), base[t].view(np.uint32))
        elif hit == num:
            fin = np.isfinite(r[t])
            assert np.array_equal(np.isnan(got[t]), np.isnan(r[t]))
            assert (np.abs(got[t][fin] - r[t][fin]) / np.abs(r[t][fin])).max() <= 1e-4


def test_probe_matches_float64_network():
    nx, ny, nz = 38, 45, 31
    img, atl, _ = subject(nx, ny, nz, 1, 41)
    rng = np.random.default_rng(0)
    z = rng.integers(LO, nz - LO, 48)
    x = rng.integers(LO, nx - LO, 48)
    y = rng.integers(LO, ny - LO, 48)
    vox = (z * nx + x) * ny + y
    with learned.LearnedModel(0, seed=7) as m:
        # larger head weights than the initialisation, so that the proposals are not ties
        p = m.get_params()
        p[-33 - 33 * 16:-33] *= 20.0
        m.set_params(p)
        wb = m.get_params(inference_precision=True)
        d_img = torch.from_numpy(img).cuda()
        d_atl = torch.from_numpy(atl[0]).cuda()
        feats, top, conf = m.probe(d_img.data_ptr(), d_atl.data_ptr(), nx, ny, nz, vox)
    ps = {k: torch.tensor(v, dtype=torch.float64) for k, v in learned_ref.unflatten(
        wb.astype(np.float64)).items()}
    x64 = torch.tensor(learned_ref.patches([img], [atl], [(0, 0, int(v)) for v in vox],
                                           None))
    h = x64
    for i in range(1, 5):
        h = F.relu(F.conv3d(h, ps[f"W{i}"], ps[f"B{i}"]))
    ref = h.reshape(len(vox), 16).numpy()
    scale = np.abs(ref).max()
    err = np.abs(feats - ref)
    assert err.max() <= 0.03 * scale + 1e-6, (err.max(), scale)
    # proposals from the GPU's own features, in float64: same top-4 per axis, same confidence
    logits = feats.astype(np.float64) @ ps["H"].numpy().T + ps["HB"].numpy()
    for i in range(len(vox)):
        probs = []
        for a in range(3):
            lg = logits[i, a * 11:(a + 1) * 11]
            pr = np.exp(lg - lg.max())
            pr /= pr.sum()
            order = sorted(range(11), key=lambda j: (-pr[j], j))[:4]
            got = [int(t) + 5 for t in top[i, a]]
            # equal up to near-ties in FP32
            for r in range(4):
                assert got[r] == order[r] or abs(pr[got[r]] - pr[order[r]]) < 1e-5
            probs.append([pr[j] for j in got])
        c = sum(probs[0][a] * probs[1][b] * probs[2][k] for a in range(4) for b in range(4)
                for k in range(4) if a + b + k <= 4)
        assert abs(c - conf[i]) < 1e-4


def test_host_device_and_pipeline_paths_agree():
    nx, ny, nz, num = 33, 42, 30, 2
    img, atl, lab = subject(nx, ny, nz, num, 51)
    with pct.Handle(0) as h, learned.LearnedModel(0, seed=9) as m:
        h.attach_model(m, 0.3)
        host = h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED)
        d = [torch.from_numpy(a).cuda() for a in (img, atl, lab)]
        out = torch.zeros_like(d[0])
        h.synthesize_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), out.data_ptr(), nx,
                            ny, nz, num, NH, DIV, pct.EXEC_LEARNED)
        torch.cuda.synchronize()
        dev = out.cpu().numpy()
    np.testing.assert_array_equal(np.isnan(host), np.isnan(dev))
    np.testing.assert_array_equal(np.nan_to_num(host), np.nan_to_num(dev))


@pytest.mark.parametrize("block,shape,nh", [(4, (47, 53, 35), 11), (3, (41, 70, 30), 11),
                                            (1, (33, 42, 29), 11), (5, (26, 40, 22), 11),
                                            (4, (39, 44, 27), 7), (1, (30, 37, 25), 9)])
def test_restricted_convs_match_every_voxel(block, shape, nh):
    """The convolutions compute only what the anchor rows need (conv4 on the anchor rows, each
    earlier layer one row, plane and y further out); every needed value must be the one the
    whole-volume convolutions give, so the results are bit-identical (also with the interior of
    the smaller windows, which starts 4 and 5 voxels from the faces)."""
    nx, ny, nz = shape
    lo = (nh - 1) // 2 + 1
    img, atl, lab = subject(nx, ny, nz, 2, 60 + block)
    with pct.Handle(0) as h, learned.LearnedModel.load(learned.CHECKPOINT) as m:
        h.attach_model(m, 0.2)
        h.set_learned_block(block)
        sparse = h.synthesize(img, atl, lab, nh, DIV, pct.EXEC_LEARNED)
        st_sparse = h.learned_stats()
        h.set_learned_convs(True)
        full = h.synthesize(img, atl, lab, nh, DIV, pct.EXEC_LEARNED)
        st_full = h.learned_stats()
        h.set_learned_convs(False)
    np.testing.assert_array_equal(np.isnan(sparse), np.isnan(full))
    np.testing.assert_array_equal(np.nan_to_num(sparse), np.nan_to_num(full))
    assert st_sparse == st_full
    assert np.isfinite(sparse[lo:-lo, lo:-lo, lo:-lo]).mean() > 0.5


def test_checkpoint_round_trip(tmp_path):
    with learned.LearnedModel(0, seed=4) as m:
        p = m.get_params()
        m.save(tmp_path / "m.pctl")
    q = learned.load_params(tmp_path / "m.pctl")
    np.testing.assert_array_equal(p, q)
    with learned.LearnedModel.load(tmp_path / "m.pctl") as m2:
        np.testing.assert_array_equal(m2.get_params(), p)


def _structured_voxels(img, n, seed):
    rng = np.random.default_rng(seed)
    nz, nx, ny = img.shape
    g = np.sqrt(sum(d.astype(np.float64) ** 2 for d in np.gradient(img)))
    w = g[LO:nz - LO, LO:nx - LO, LO:ny - LO].ravel()
    flat = rng.choice(w.size, n, replace=False, p=w / w.sum())
    iz, ix, iy = np.unravel_index(flat, (nz - 2 * LO, nx - 2 * LO, ny - 2 * LO))
    return ((iz + LO) * nx + ix + LO) * ny + iy + LO


def test_trained_network_gain():
    """The committed network against the same-k baselines without it, on a held-out subject:
    the centre prior (no network) and an untrained network. Per-voxel recall of the plain
    method's exact top-32 (float64) at structured voxels, and the fused result's error against
    the plain FP32 method."""
    nx, ny, nz, num = 128, 128, 80, 4
    subj = pct.synth_subject(nx, ny, nz, num, n_blobs=14, seed=7001)
    trained = learned.load_params(learned.CHECKPOINT)
    with learned.LearnedModel(0, seed=7001) as m:
        untrained = m.get_params()
    models = {"trained": trained, "prior": learned.prior_params(), "untrained": untrained}
    # recall of the exact top-32 by each voxel's own 32
    vox = _structured_voxels(subj.img, 150, 3)
    d_img = torch.from_numpy(subj.img).cuda()
    d_atl = torch.from_numpy(subj.atlas_mri[0]).cuda()
    truth = []
    for v in vox:
        ssd = learned_ref.top32_float64(subj.img, subj.atlas_mri[0], int(v))
        truth.append(set(np.argsort(ssd, kind="stable")[:32].tolist()))
    recall = {}
    for name, p in models.items():
        with learned.LearnedModel(0, params=p) as m:
            _, top, _ = m.probe(d_img.data_ptr(), d_atl.data_ptr(), nx, ny, nz, vox)
        hits = 0
        for i in range(len(vox)):
            kept = {(dw + 5) * 121 + (du + 5) * 11 + dv + 5
                    for dw, du, dv in learned.rank_sum_set(top[i])}
            hits += len(kept & truth[i])
        recall[name] = hits / (32 * len(vox))
    # fused error against the plain method, k = 32 (no fallback)
    res = {name: learned.evaluate(p, [subj], thresholds=(0.0,), reps=1)[0]
           for name, p in models.items()}
    print("recall", recall, "mae", {k: v["mae_hu"] for k, v in res.items()})
    assert recall["trained"] > recall["prior"] > recall["untrained"]
    assert res["trained"]["mae_hu"] < res["prior"]["mae_hu"] < res["untrained"]["mae_hu"]
    assert res["trained"]["mae_hu"] <= 5.0
    assert res["trained"]["offsets_per_row"] == 32.0


@pytest.mark.parametrize("mode,nh", [("network", 11), ("network_conf", 11), ("prior", 11),
                                     ("network_conf", 9), ("prior", 7)])
def test_runtime_compiled_rescoring_matches_library_build(mode, nh, monkeypatch):
    """The rescoring runs from a module compiled at run time for the volume's x extent and row
    pitch; PCT_RESCORE_JIT=0 keeps the library's own build of the same code. Both give the same
    output bit for bit (odd sizes; with a confidence threshold the atlas rows are repacked to a
    16-byte pitch, a second geometry)."""
    nx, ny, nz, num = 41, 53, 31, 2
    img, atl, lab = subject(nx, ny, nz, num, 61)
    outs = []
    for jit in ("1", "0"):
        monkeypatch.setenv("PCT_RESCORE_JIT", jit)
        with pct.Handle(0) as h, learned.LearnedModel(0, seed=5) as m:
            if mode == "prior":
                h.set_learned_prior(32)
            else:
                h.attach_model(m, 0.02 if mode == "network_conf" else 0.0)
            outs.append((h.synthesize(img, atl, lab, nh, DIV, pct.EXEC_LEARNED), h.learned_stats()))
    (a, sa), (b, sb) = outs
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert sa == sb



@pytest.mark.parametrize("mode", ["network", "prior"])
@pytest.mark.parametrize("nz", [13, 14, 15, 17])
def test_pair_items_on_thin_volumes(nz, mode, monkeypatch):
    """The rescoring's z-pair items (two planes of a proposal block per warp) against the one-plane
    items, bit for bit, on 1 to 5 interior planes: one plane keeps the one-plane items, an odd
    count shifts the last pair back by a plane that it does not own."""
    nx, ny, num = 20, 37, 2
    img, atl, lab = subject(nx, ny, nz, num, 70 + nz)
    outs = []
    for pairs in ("1", "0"):
        monkeypatch.setenv("PCT_RS_PAIRS", pairs)
        with pct.Handle(0) as h, learned.LearnedModel(0, seed=5) as m:
            if mode == "prior":
                h.set_learned_prior(32)
            else:
                h.attach_model(m, 0.0)
            outs.append((h.synthesize(img, atl, lab, NH, DIV, pct.EXEC_LEARNED), h.learned_stats()))
    (a, sa), (b, sb) = outs
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert sa == sb
    assert sa["row_offsets"] == rows_of(nx, ny, nz) * 32 * num


def window_proposal(nh, k, scales=(0.7, 0.5, 0.3)):
    """The prior network's proposal for an NH window: per axis the softmax of its biases over the
    window's offsets, the 4 most probable (ties: lower offset first), the kept rank triples and
    their probability mass, in float64."""
    hw = (nh - 1) // 2
    top, probs = [], []
    for c in scales:
        d = np.arange(-hw, hw + 1)
        logits = -c * d.astype(np.float64) ** 2
        p = np.exp(logits - logits.max())
        p /= p.sum()
        order = sorted(range(len(d)), key=lambda j: (-p[j], j))[:4]
        top.append([int(d[j]) for j in order])
        probs.append([p[j] for j in order])
    level = learned.KEPT_LEVEL[k]
    conf = sum(probs[0][i] * probs[1][j] * probs[2][l] for i in range(4) for j in range(4)
               for l in range(4) if i + j + l <= level)
    return np.array(top), conf


@pytest.mark.parametrize("nh,k,block", [(7, 32, 4), (9, 32, 4), (9, 20, 1), (7, 10, 4)])
def test_prior_proposal_exact_small_windows(nh, k, block):
    """NH 7 and 9: the network's softmaxes run over the window's offsets only; with the prior
    network every row keeps the same k offsets, exactly the float64 fusion over them, on the
    larger interior of the smaller window."""
    lo = (nh - 1) // 2 + 1
    nx, ny, nz, num = 38, 45, 30, 2
    img, atl, lab = subject(nx, ny, nz, num, 23)
    top, _ = window_proposal(nh, k)
    offsets = learned.rank_sum_set(top, k)
    assert len({tuple(o) for o in offsets}) == k
    ref, prod, sumw = fuse_offsets_f64(img, atl, lab, offsets, DIV, LO=lo)
    with pct.Handle(0) as h, learned.LearnedModel(0, params=prior_params()) as m:
        h.attach_model(m, 0.0)
        h.set_learned_k(k)
        h.set_learned_block(block)
        got = h.synthesize(img, atl, lab, nh, DIV, pct.EXEC_LEARNED)
        st = h.learned_stats()
    compare_fused(got, ref, nh, 1e-4, prod, sumw)
    assert np.all(got[:lo] == 0) and np.all(got[:, :, -lo:] == 0)
    assert st["fallback_pairs"] == 0
    assert st["row_offsets"] == rows_of(nx, ny, nz, lo) * k * num


@pytest.mark.parametrize("nh", [7, 9])
def test_confidence_and_full_fallback_small_windows(nh):
    """Below the prior's own confidence nothing falls back; above 1 every pair takes the full
    NH^3 window, which is the plain method."""
    lo = (nh - 1) // 2 + 1
    nx, ny, nz, num = 34, 37, 29, 2
    img, atl, lab = subject(nx, ny, nz, num, 33)
    _, conf = window_proposal(nh, 32)
    ref, prod, sumw = oracle.fuse_port(img, atl, lab, nh, DIV, with_sums=True)
    with pct.Handle(0) as h, learned.LearnedModel(0, params=prior_params()) as m:
        h.attach_model(m, conf * (1 - 1e-3))
        h.synthesize(img, atl, lab, nh, DIV, pct.EXEC_LEARNED)
        assert h.learned_stats()["fallback_pairs"] == 0
        h.attach_model(m, 2.0)
        got = h.synthesize(img, atl, lab, nh, DIV, pct.EXEC_LEARNED)
        st = h.learned_stats()
    compare_fused(got, ref, nh, 1e-4, prod, sumw)
    assert st["fallback_pairs"] == interior(nx, ny, nz, lo) * num
    assert st["row_offsets"] == rows_of(nx, ny, nz, lo) * nh ** 3 * num


@pytest.mark.parametrize("nh", [7, 9])
def test_centre_prior_small_windows(nh):
    """The no-network centre prior at NH 7 and 9: the 32 and 57 offsets nearest the centre of the
    window, exactly the float64 fusion over them."""
    import itertools
    lo, hw = (nh - 1) // 2 + 1, (nh - 1) // 2
    nx, ny, nz, num = 36, 41, 30, 2
    img, atl, lab = subject(nx, ny, nz, num, 21)
    with pct.Handle(0) as h:
        for k in (32, 57):
            offs = sorted(itertools.product(range(-hw, hw + 1), repeat=3),
                          key=lambda o: o[0] ** 2 + o[1] ** 2 + o[2] ** 2)[:k]
            ref, prod, sumw = fuse_offsets_f64(img, atl, lab, offs, DIV, LO=lo)
            h.set_learned_prior(k)
            got = h.synthesize(img, atl, lab, nh, DIV, pct.EXEC_LEARNED)
            compare_fused(got, ref, nh, 1e-4, prod, sumw)
            assert h.learned_stats()["row_offsets"] == rows_of(nx, ny, nz, lo) * k * num


def sampled_fusion_f64(img, atlas, label, offsets, div, vox):
    """Float64 fusion over a fixed offset list at the flat voxels `vox` only; (out, prod, sumw)."""
    nz, nx, ny = img.shape
    z, r = np.divmod(vox, nx * ny)
    x, y = np.divmod(r, ny)
    taps = [(dz, dx, dy) for dz in (-1, 0, 1) for dx in (-1, 0, 1) for dy in (-1, 0, 1)]
    I = np.stack([img[z + dz, x + dx, y + dy] for dz, dx, dy in taps]).astype(np.float64)
    P = np.zeros(len(vox))
    W = np.zeros(len(vox))
    for a in range(atlas.shape[0]):
        A, L = atlas[a], label[a]
        for dw, du, dv in offsets:
            Ab = np.stack([A[z + dw + dz, x + du + dx, y + dv + dy] for dz, dx, dy in taps])
            ssd = ((I - Ab.astype(np.float64)) ** 2).sum(axis=0)
            w = np.exp(-ssd / div)
            P += w * L[z + dw, x + du, y + dv]
            W += w
    ok = (np.abs(P) > DBL_EPS) & (np.abs(W) > DBL_EPS)
    return np.where(ok, P / np.where(ok, W, 1.0), np.nan), P, W


@pytest.mark.parametrize("k", [32, 10])
def test_full_size_prior_network_sampled_voxels(k):
    """The learned form at the full config-1 geometry (222x222x112, 10 atlases, the run-time
    compiled rescoring for nx = 222 and pitch 222) with the prior network: every row keeps the
    same k offsets, so 1,500 sampled interior voxels must equal the float64 fusion over them."""
    s = pct.synth_subject(222, 222, 112, 10, n_blobs=60, seed=1)
    lab = pct.normalize_labels(s.atlas_ct)
    top, _ = prior_proposal(k=k)
    offsets = learned.rank_sum_set(top, k)
    with pct.Handle(0) as h, learned.LearnedModel(0, params=prior_params()) as m:
        h.attach_model(m, 0.0)
        h.set_learned_k(k)
        got = h.synthesize(s.img, s.atlas_mri, lab, NH, DIV, pct.EXEC_LEARNED)
    nz, nx, ny = s.img.shape
    rng = np.random.default_rng(k)
    vox = (rng.integers(LO, nz - LO, 1500) * nx * ny + rng.integers(LO, nx - LO, 1500) * ny
           + rng.integers(LO, ny - LO, 1500))
    ref, P, W = sampled_fusion_f64(s.img, s.atlas_mri, lab, offsets, DIV, vox)
    g = got.reshape(-1)[vox]
    gn, rn = np.isnan(g), np.isnan(ref)
    mism = gn != rn
    if mism.any():  # only where a float64 sum sits at the DBL_EPSILON threshold
        near = (np.abs(np.abs(P[mism]) / DBL_EPS - 1) < 1e-3) | (np.abs(np.abs(W[mism]) / DBL_EPS - 1) < 1e-3)
        assert near.all()
    both = ~gn & ~rn
    rel = np.abs(g[both].astype(np.float64) - ref[both]) / np.maximum(np.abs(ref[both]), 1e-30)
    assert rel.max() <= 1e-4, rel.max()


def test_full_size_centre_prior_sampled_voxels():
    """The no-network centre prior at the full config-1 geometry (k = 57): 1,500 sampled interior
    voxels against the float64 fusion over the 57 offsets nearest the window's centre."""
    s = pct.synth_subject(222, 222, 112, 10, n_blobs=60, seed=1)
    lab = pct.normalize_labels(s.atlas_ct)
    with pct.Handle(0) as h:
        h.set_learned_prior(57)
        got = h.synthesize(s.img, s.atlas_mri, lab, NH, DIV, pct.EXEC_LEARNED)
    nz, nx, ny = s.img.shape
    rng = np.random.default_rng(57)
    vox = (rng.integers(LO, nz - LO, 1500) * nx * ny + rng.integers(LO, nx - LO, 1500) * ny
           + rng.integers(LO, ny - LO, 1500))
    ref, P, W = sampled_fusion_f64(s.img, s.atlas_mri, lab, centre_offsets(57), DIV, vox)
    g = got.reshape(-1)[vox]
    both = ~np.isnan(g) & ~np.isnan(ref)
    mism = np.isnan(g) != np.isnan(ref)
    if mism.any():
        near = (np.abs(np.abs(P[mism]) / DBL_EPS - 1) < 1e-3) | (np.abs(np.abs(W[mism]) / DBL_EPS - 1) < 1e-3)
        assert near.all()
    rel = np.abs(g[both].astype(np.float64) - ref[both]) / np.maximum(np.abs(ref[both]), 1e-30)
    assert rel.max() <= 1e-4, rel.max()
