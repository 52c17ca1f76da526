"""Regenerates the golden fixtures in this folder from the reference's own CPU code.

    python tests/golden/make_golden.py

Inputs come from the library's seeded generator (pct_synth_generate) at small sizes; outputs come
from the UNMODIFIED reference routines compiled into oracle/_ref/libpctref.so
(MultiAtlasPatchBasedSegmentationOpenMP, RegularizationStep, RoundMatrix;
src/CPU/NewPatchedBrainPureC.cpp:1350-1449,1059-1106,1221-1227) and the reference's HU map
(:1732-1738, float arithmetic as written there). The reference has no test vectors of its own,
so these fixtures pin the oracle and the CUDA path to the reference's actual outputs.
"""
from __future__ import annotations

import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import oracle  # noqa: E402
import pseudoctimaging_b200 as pct  # noqa: E402

# name: (nz, nx, ny, num_atlas, nh, sigma, beta, n_blobs, seed)
CASES = {
    "small_nh7_2atlas": (18, 20, 24, 2, 7, 2.5, 1.0, 6, 101),
    "odd_nh7_1atlas": (19, 17, 23, 1, 7, 2.5, 1.0, 5, 102),
    "nh9_3atlas": (26, 28, 30, 3, 9, 2.5, 1.0, 8, 103),
    "nh11_2atlas": (30, 32, 34, 2, 11, 2.5, 1.0, 8, 104),
    "nh3_tiny": (12, 13, 14, 1, 3, 2.5, 1.0, 3, 105),
    # small sigma: most weights underflow the DBL_EPSILON rule, many NaNs to regularise
    "nan_rich_nh7": (20, 22, 26, 1, 7, 0.6, 1.0, 6, 106),
    # window larger than the volume allows: no interior voxel at all
    "no_interior_nh11": (11, 12, 40, 1, 11, 2.5, 1.0, 3, 107),
}


def to_hu_reference(v: np.ndarray) -> np.ndarray:
    """NewPatchedBrainPureC.cpp:1735-1738: round(4095.0f*(v/255.0f)) - 1024.0f in float."""
    v = v.astype(np.float32)
    return (np.round(np.float32(4095.0) * (v / np.float32(255.0))) - np.float32(1024.0)).astype(np.float32)


def make_case(name: str, spec) -> dict:
    nz, nx, ny, num, nh, sigma, beta, blobs, seed = spec
    s = pct.synth_subject(nx, ny, nz, num, n_blobs=blobs, seed=seed)
    label = pct.normalize_labels(s.atlas_ct)
    div = 2 * 27 * beta * sigma ** 2
    out = oracle.fuse_reference(s.img, s.atlas_mri, label, nh, div, multicore=True)
    reg = oracle.regularize_reference(out, nh)
    rounded = reg.copy()
    oracle.reference().pctref_round(rounded.ctypes.data, rounded.size)
    hu = to_hu_reference(rounded)
    return dict(img=s.img, atlas_mri=s.atlas_mri, atlas_ct_hu=s.atlas_ct, label=label,
                nh=np.int32(nh), sigma=np.float64(sigma), beta=np.float64(beta),
                div=np.float64(div), seed=np.int64(seed), out=out, regularized=reg, hu=hu)


def main() -> None:
    if not oracle.has_reference():
        raise SystemExit("oracle/_ref/libpctref.so missing: build it with `make -C oracle all`")
    for name, spec in CASES.items():
        d = make_case(name, spec)
        np.savez_compressed(HERE / f"{name}.npz", **d)
        nan = int(np.isnan(d["out"]).sum())
        print(f"{name}: shape {d['img'].shape} atlases {d['atlas_mri'].shape[0]} nh {int(d['nh'])} "
              f"nan {nan}")


if __name__ == "__main__":
    main()
