"""Batched form: many subjects of uneven size, atlas count and NH in one persistent launch, a CUDA
graph replaying it, and the tile-shape autotuner (through the C ABI)."""
import json

import numpy as np
import pytest
import torch

import oracle
import pseudoctimaging_b200 as pct
from conftest import compare_fused

pytestmark = pytest.mark.gpu

# (nx, ny, nz, num_atlas, nh, seed): uneven sizes (incl. ny % 4 != 0 and == 0), atlas counts, NH
SPECS = [(52, 46, 40, 3, 11, 1), (40, 44, 36, 2, 7, 2), (61, 37, 30, 1, 9, 3),
         (36, 48, 42, 4, 9, 4), (45, 50, 33, 2, 7, 5), (30, 29, 31, 1, 11, 6)]


def make_batch(specs=SPECS):
    subs, host, dev = [], [], []
    for nx, ny, nz, num, nh, seed in specs:
        s = pct.synth_subject(nx, ny, nz, num, n_blobs=8, seed=seed)
        lab = pct.normalize_labels(s.atlas_ct)
        d = [torch.from_numpy(x).cuda() for x in (s.img, s.atlas_mri, lab)]
        out = torch.zeros_like(d[0])
        dev.append((d, out))
        host.append((s, lab))
        subs.append(pct.SubjectDesc(img=d[0].data_ptr(), atlas=d[1].data_ptr(),
                                    atlas_label=d[2].data_ptr(), out=out.data_ptr(), nx=nx, ny=ny,
                                    nz=nz, num_atlas=num, nh=nh, div=337.5))
    return subs, host, dev


@pytest.fixture(scope="module")
def handle():
    h = pct.Handle(0)
    yield h
    h.close()


def test_batch_matches_single_subject_path_and_oracle(handle):
    subs, host, dev = make_batch()
    stream = torch.cuda.current_stream().cuda_stream
    handle.synthesize_batch(subs, stream)
    handle.device_status(stream)
    for k, ((s, lab), (d, out)) in enumerate(zip(host, dev)):
        nx, ny, nz, num, nh, _ = SPECS[k]
        got = out.cpu().numpy()
        single = handle.synthesize(s.img, s.atlas_mri, lab, nh, 337.5)
        lo = (nh - 1) // 2 + 1
        sl = (slice(lo, -lo),) * 3
        assert np.array_equal(np.isnan(got[sl]), np.isnan(single[sl]))
        fin = ~np.isnan(single[sl])
        # the single-subject path may split atlases into groups (another summation order)
        np.testing.assert_allclose(got[sl][fin], single[sl][fin], rtol=2e-5, atol=1e-5)
        if k < 3:
            ref, prod, sumw = oracle.fuse_port(s.img, s.atlas_mri, lab, nh, 337.5, with_sums=True)
            compare_fused(got, ref, nh, 1e-4, prod, sumw)


def test_graph_replays_on_updated_inputs(handle):
    subs, host, dev = make_batch(SPECS[:4])
    stream = torch.cuda.current_stream().cuda_stream
    handle.synthesize_batch(subs, stream)
    direct = [out.clone() for _, out in dev]
    with handle.batch_graph(subs, stream) as g:
        for _ in range(2):
            for _, out in dev:
                out.zero_()
            g.launch(stream)
            g.status(stream)
            for (_, out), ref in zip(dev, direct):
                assert torch.equal(out.isnan(), ref.isnan())
                m = ~ref.isnan()
                assert torch.equal(out[m], ref[m])
        # the graph reads the buffers at replay time: doubled labels give doubled outputs
        for (d, _), _r in zip(dev, direct):
            d[2].mul_(2.0)
        g.launch(stream)
        g.status(stream)
        for (_, out), ref in zip(dev, direct):
            m = ~ref.isnan()
            torch.testing.assert_close(out[m], 2 * ref[m], rtol=1e-6, atol=1e-5)


def test_autotuner_picks_a_set_caches_it_and_sets_agree(handle, tmp_path):
    subs, host, dev = make_batch(SPECS[:4])
    cache = tmp_path / "tune.jsonl"
    chosen, ms = handle.autotune(subs, cache)
    assert chosen in range(pct.lib.pct_tile_sets()) and handle.tile_set == chosen
    assert all(t > 0 for t in ms) and ms[chosen] == min(ms)
    line = json.loads(cache.read_text().splitlines()[-1])
    assert line["set"] == chosen and len(line["ms"]) == len(ms)
    again, ms2 = handle.autotune(subs, cache)
    assert again == chosen and all(t == -1 for t in ms2)
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for k in range(pct.lib.pct_tile_sets()):
        handle.set_tile_set(k)
        handle.synthesize_batch(subs, stream)
        handle.device_status(stream)
        outs.append([out.cpu().numpy() for _, out in dev])
    handle.set_tile_set(0)
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(np.isnan(a), np.isnan(b))
        fin = ~np.isnan(a)
        np.testing.assert_allclose(a[fin], b[fin], rtol=2e-5, atol=1e-5)


def test_batch_rejects_windows_it_does_not_compile(handle):
    subs, _, _ = make_batch([(30, 30, 30, 1, 7, 9)])
    subs[0].nh = 5
    with pytest.raises(pct.PctError) as e:
        handle.synthesize_batch(subs)
    assert e.value.status == -4
