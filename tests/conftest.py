import pathlib
import sys

import numpy as np
import pytest

REPO = pathlib.Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


def golden_names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


# DBL_EPSILON, the reference's threshold on both sums (NewPatchedBrainPureC.cpp:1325).
DBL_EPS = 2.220446049250313e-16


def compare_fused(got: np.ndarray, ref: np.ndarray, nh: int, rtol: float, prod=None, sumw=None,
                  eps_margin: float = 1e-3) -> dict:
    """Compares two fused volumes over the interior.

    Voxels finite in both must satisfy |got-ref| <= rtol*|ref|. NaN masks must agree, except for
    voxels whose reference sums lie within a relative `eps_margin` of DBL_EPSILON (when the
    oracle's product/sum_weight are supplied), where FP32 and FP64 may fall on either side.
    Returns statistics; raises AssertionError on a violation.
    """
    lo = (nh - 1) // 2 + 1
    sl = (slice(lo, -lo), slice(lo, -lo), slice(lo, -lo))
    g, r = got[sl], ref[sl]
    gn, rn = np.isnan(g), np.isnan(r)
    mism = gn != rn
    if mism.any():
        if prod is None or sumw is None:
            raise AssertionError(f"{int(mism.sum())} NaN-mask mismatches")
        p, s = np.abs(prod[sl][mism]), np.abs(sumw[sl][mism])
        near = (np.abs(p / DBL_EPS - 1) < eps_margin) | (np.abs(s / DBL_EPS - 1) < eps_margin)
        assert near.all(), f"{int((~near).sum())} NaN-mask mismatches away from the threshold"
    both = ~gn & ~rn
    d = np.abs(g[both].astype(np.float64) - r[both].astype(np.float64))
    rel = d / np.maximum(np.abs(r[both].astype(np.float64)), 1e-30)
    worst = float(rel.max()) if rel.size else 0.0
    assert worst <= rtol, f"max relative error {worst:.3e} > {rtol:.1e}"
    return {"max_rel": worst, "max_abs": float(d.max()) if d.size else 0.0,
            "nan": int(rn.sum()), "nan_mismatch": int(mism.sum()), "compared": int(both.sum())}
