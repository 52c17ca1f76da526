"""Tensor-core form (EXEC_CHOICE 5 FP16, 6 BF16) on the GPU.

* Selection: the 16 survivors the tcgen05 correlation keeps per voxel are checked against a
  float64 restatement of the same ranking (the subject's rounded mean removed, 16-bit rounding of
  both patches, |b|^2/2 of the rounded patch): every survivor must rank among the restatement's
  best 16 up to FP32 accumulation near-ties and the 2^-12 relative key packing.
* Result: the fused output against the FP64 oracle (the plain method) and against the exact
  top-16 fusion (the best this form can do), as MAE and max-abs error in HU.
"""
import numpy as np
import pytest
import torch

import oracle
import pseudoctimaging_b200 as pct
from conftest import DBL_EPS

pytestmark = pytest.mark.gpu
LO = 6
DIV = 337.5
HU = 4095.0 / 255.0


def subject(nx, ny, nz, num, seed):
    s = pct.synth_subject(nx, ny, nz, num, n_blobs=10, seed=seed)
    return s.img, s.atlas_mri, pct.normalize_labels(s.atlas_ct)


def round16(x, bf16):
    x = np.asarray(x, np.float32)
    if not bf16:
        return x.astype(np.float16).astype(np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32)


def subject_offset(img):
    """The kernel's offset mu: rint of the input MRI's mean, with its FP32 summation order (1024
    threads, thread t summing elements t, t + 1024, ... in order, then a halving tree)."""
    flat = np.ascontiguousarray(img, np.float32).ravel()
    part = np.zeros(1024, np.float32)
    for t in range(1024):
        acc = np.float32(0)
        for v in flat[t::1024]:
            acc = np.float32(acc + v)
        part[t] = acc
    h = 512
    while h > 0:
        part[:h] = (part[:h] + part[h:2 * h]).astype(np.float32)
        h //= 2
    return np.float32(np.rint(np.float32(part[0] / np.float32(flat.size))))


def ranking_f64(img, atl, z, x, y, bf16, mu):
    """D' = a.b - |b|^2/2 of the rounded patches for the 1331 offsets of voxel (z, x, y)."""
    s = np.float32(1.0 / 64.0)
    a = round16((img[z - 1:z + 2, x - 1:x + 2, y - 1:y + 2].astype(np.float32) - mu) * s, bf16)
    out = np.empty(1331)
    o = 0
    for dz in range(-5, 6):
        for dx in range(-5, 6):
            for dy in range(-5, 6):
                b = atl[z + dz - 1:z + dz + 2, x + dx - 1:x + dx + 2, y + dy - 1:y + dy + 2]
                b = round16((b.astype(np.float32) - mu) * s, bf16)
                h = np.float32(0.5) * np.float32((b.astype(np.float32) ** 2).sum(dtype=np.float32))
                out[o] = (a.astype(np.float64) * b).sum() - float(h)
                o += 1
    return out


def exact_top16_fusion(img, atl, lab, k=16):
    """Float64 fusion where each (voxel, atlas) keeps only its k smallest exact SSDs."""
    nz, nx, ny = img.shape
    shape = (nz - 2 * LO, nx - 2 * LO, ny - 2 * LO)
    I = img.astype(np.float64)
    P, W = np.zeros(shape), np.zeros(shape)

    def win(vol, dz, dx, dy):
        return vol[LO + dz:nz - LO + dz, LO + dx:nx - LO + dx, LO + dy:ny - LO + dy]

    offs = [(dz, dx, dy) for dz in range(-5, 6) for dx in range(-5, 6) for dy in range(-5, 6)]
    for a in range(atl.shape[0]):
        A = atl[a].astype(np.float64)
        ssd = np.empty((len(offs),) + shape)
        for i, (dw, du, dv) in enumerate(offs):
            acc = np.zeros(shape)
            for dz in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        acc += (win(I, dz, dx, dy) - win(A, dz + dw, dx + du, dy + dv)) ** 2
            ssd[i] = acc
        keep = np.argsort(ssd, axis=0, kind="stable")[:k]
        for i, (dw, du, dv) in enumerate(offs):
            sel = (keep == i).any(axis=0)
            w = np.where(sel, np.exp(-ssd[i] / DIV), 0.0)
            P += w * win(lab[a].astype(np.float64), dw, du, dv)
            W += w
    out = np.zeros(img.shape)
    ok = (np.abs(P) > DBL_EPS) & (np.abs(W) > DBL_EPS)
    out[LO:nz - LO, LO:nx - LO, LO:ny - LO] = np.where(ok, P / np.where(ok, W, 1), np.nan)
    return out


def err_hu(got, ref):
    core = (slice(LO, -LO),) * 3
    g, r = got[core].astype(np.float64), ref[core].astype(np.float64)
    both = np.isfinite(g) & np.isfinite(r)
    e = np.abs(g[both] - r[both]) * HU
    return float(e.mean()), float(e.max()), int((np.isnan(g) != np.isnan(r)).sum())


@pytest.mark.parametrize("choice", [pct.EXEC_TC_FP16, pct.EXEC_TC_BF16])
def test_survivors_match_the_rounded_ranking(choice):
    bf16 = choice == pct.EXEC_TC_BF16
    nx, ny, nz = 29, 35, 27
    img, atl, lab = subject(nx, ny, nz, 1, 81)
    d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (img, atl, lab)]
    out = torch.zeros_like(d[0])
    top = torch.zeros((nz * nx * ny, 16), dtype=torch.int16, device="cuda")
    with pct.Handle(0) as h:
        h._check(pct.lib.pct_tc_survivors(h.ptr, choice, d[0].data_ptr(), d[1].data_ptr(),
                                          d[2].data_ptr(), out.data_ptr(), nx, ny, nz, DIV,
                                          top.data_ptr(), None), "pct_tc_survivors")
    top = top.cpu().numpy().astype(np.int64)
    rng = np.random.default_rng(1)
    hits = worst = 0
    checked = 60
    mu = subject_offset(img)
    for _ in range(checked):
        z, x, y = (int(rng.integers(LO, n - LO)) for n in (nz, nx, ny))
        dp = ranking_f64(img, atl[0], z, x, y, bf16, mu)
        best16 = np.sort(dp)[::-1][15]
        sel = top[(z * nx + x) * ny + y]
        assert len(set(sel.tolist())) == 16
        tol = 2e-3 + 1e-6 * np.abs(dp).max()
        assert (dp[sel] >= best16 - tol).all(), (z, x, y, dp[sel].min(), best16)
        hits += len(set(sel.tolist()) & set(np.argsort(-dp, kind="stable")[:16].tolist()))
        worst = max(worst, float(best16 - dp[sel].min()))
    assert hits / (16 * checked) > 0.9


@pytest.mark.parametrize("choice", [pct.EXEC_TC_FP16, pct.EXEC_TC_BF16])
def test_error_against_fp64_and_exact_top16(choice):
    nx, ny, nz, num = 32, 37, 30, 2
    img, atl, lab = subject(nx, ny, nz, num, 91)
    ref = oracle.fuse_port(img, atl, lab, 11, DIV)
    top16 = exact_top16_fusion(img, atl, lab)
    with pct.Handle(0) as h:
        got = h.synthesize(img, atl, lab, 11, DIV, choice)
        plain = h.synthesize(img, atl, lab, 11, DIV, pct.EXEC_B200_FP32)
    mae_fp64, max_fp64, nan_fp64 = err_hu(got, ref)
    mae_top, max_top, nan_top = err_hu(got, top16)
    mae_plain, _, _ = err_hu(got, plain)
    print(f"choice {choice}: vs FP64 MAE {mae_fp64:.3f} HU max {max_fp64:.1f}; vs exact top-16 "
          f"MAE {mae_top:.4f} max {max_top:.2f}; vs plain MAE {mae_plain:.3f}")
    assert mae_top < 0.5 and mae_fp64 < 5.0
    assert abs(mae_plain - mae_fp64) < 0.05
    assert np.all(got[:LO] == 0)


def test_rejects_other_windows():
    img, atl, lab = subject(30, 30, 28, 1, 3)
    with pct.Handle(0) as h:
        with pytest.raises(pct.PctError) as e:
            h.synthesize(img, atl, lab, 9, DIV, pct.EXEC_TC_FP16)
    assert e.value.status == -4
