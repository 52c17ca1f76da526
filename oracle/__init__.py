"""Parity oracles for the pseudo-CT path (TEST INFRASTRUCTURE ONLY).

Two CPU implementations, both double precision:

* ``port``: our C restatement, ``oracle/pct_oracle.c`` -> ``oracle/libpct_oracle.so``.
* ``reference``: the reference's own ``src/CPU/NewPatchedBrainPureC.cpp``, compiled unmodified by
  ``oracle/Makefile`` into ``oracle/_ref/libpctref.so`` (only where the reference checkout was
  available at build time; the built file travels with the repository).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline arm use this module, and only
as the checker or as the timed CPU baseline; the product library never calls it.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
PORT_LIB = HERE / "libpct_oracle.so"
REF_LIB = HERE / "_ref" / "libpctref.so"

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double


# Where the build container keeps the reference checkout (read-only); PCT_REFERENCE_DIR overrides.
_DEFAULT_REF_DIR = "/root/reference"


def build() -> None:
    """Builds the restatement and, where the reference checkout exists, the reference library."""
    make = "/usr/bin/make" if os.path.exists("/usr/bin/make") else "make"
    ref = os.environ.get("PCT_REFERENCE_DIR") or _DEFAULT_REF_DIR
    args = [make, "-s", "-C", str(HERE), "all"]
    if os.path.isdir(ref):
        args.append(f"REF={ref}")
    subprocess.run(args, check=True)


def _load(path: pathlib.Path) -> ctypes.CDLL:
    if not path.exists():
        raise FileNotFoundError(f"{path} not built (run `make -C oracle all`)")
    return ctypes.CDLL(str(path))


_port = None
_ref = None


def port() -> ctypes.CDLL:
    global _port
    if _port is None:
        lib = _load(PORT_LIB)
        lib.pct_oracle_div.restype = _D
        lib.pct_oracle_div.argtypes = [_D, _D]
        lib.pct_oracle_fuse.restype = ctypes.c_int64
        lib.pct_oracle_fuse.argtypes = [_P, _P, _P, _P, _I, _I, _I, _I, _I, _D, _P, _P, _I]
        lib.pct_oracle_fuse_voxels.restype = _I
        lib.pct_oracle_fuse_voxels.argtypes = [_P, _P, _P, _I, _I, _I, _I, _I, _D, _P,
                                               ctypes.c_int64, _P, _P, _P, _I]
        lib.pct_oracle_regularize.restype = ctypes.c_int64
        lib.pct_oracle_regularize.argtypes = [_I, _I, _I, _I, _I, _P]
        lib.pct_oracle_round.argtypes = [_P, ctypes.c_size_t]
        lib.pct_oracle_to_hu.argtypes = [_P, ctypes.c_size_t]
        lib.pct_oracle_normalize_labels.argtypes = [_P, ctypes.c_size_t]
        _port = lib
    return _port


def has_reference() -> bool:
    return REF_LIB.exists()


def reference() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        lib = _load(REF_LIB)
        lib.pctref_fuse.restype = _I
        lib.pctref_fuse.argtypes = [_P, _P, _P, _P, _I, _I, _I, _I, _I, _D, _I, _I, _I]
        lib.pctref_regularize.restype = _I
        lib.pctref_regularize.argtypes = [_I, _I, _I, _I, _I, _P, _I]
        lib.pctref_round.restype = _I
        lib.pctref_round.argtypes = [_P, _I]
        lib.pctref_max_threads.restype = _I
        _ref = lib
    return _ref


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _dims(img: np.ndarray):
    nz, nx, ny = img.shape
    return nx, ny, nz


def fuse_port(img, atlas, label, nh: int, div: float, threads: int = 0, with_sums: bool = False):
    """Restatement of MultiAtlasPatchBasedSegmentationOpenMP; border voxels are 0."""
    img, atlas, label = _c(img), _c(atlas), _c(label)
    if atlas.ndim == 3:
        atlas, label = atlas[None], label[None]
    nx, ny, nz = _dims(img)
    out = np.zeros_like(img)
    prod = np.zeros(img.shape, np.float64) if with_sums else None
    sumw = np.zeros(img.shape, np.float64) if with_sums else None
    n = port().pct_oracle_fuse(img.ctypes.data, atlas.ctypes.data, label.ctypes.data,
                               out.ctypes.data, nx, ny, nz, atlas.shape[0], nh, float(div),
                               prod.ctypes.data if with_sums else None,
                               sumw.ctypes.data if with_sums else None, threads)
    if n < 0:
        raise ValueError("pct_oracle_fuse rejected its arguments")
    return (out, prod, sumw) if with_sums else out


def fuse_port_voxels(img, atlas, label, nh: int, div: float, voxels, threads: int = 0):
    """Oracle values (out, product, sum_weight) at flat voxel indices z*nx*ny + x*ny + y."""
    img, atlas, label = _c(img), _c(atlas), _c(label)
    if atlas.ndim == 3:
        atlas, label = atlas[None], label[None]
    nx, ny, nz = _dims(img)
    vox = np.ascontiguousarray(voxels, dtype=np.int64)
    out = np.zeros(vox.shape, np.float32)
    prod = np.zeros(vox.shape, np.float64)
    sumw = np.zeros(vox.shape, np.float64)
    st = port().pct_oracle_fuse_voxels(img.ctypes.data, atlas.ctypes.data, label.ctypes.data, nx,
                                       ny, nz, atlas.shape[0], nh, float(div), vox.ctypes.data,
                                       vox.size, out.ctypes.data, prod.ctypes.data,
                                       sumw.ctypes.data, threads)
    if st != 0:
        raise ValueError("pct_oracle_fuse_voxels rejected its arguments")
    return out, prod, sumw


def fuse_reference(img, atlas, label, nh: int, div: float, multicore: bool = True,
                   threads: int = 0) -> np.ndarray:
    """The reference's own MultiAtlasPatchBasedSegmentation[OpenMP]; border voxels are 0."""
    img, atlas, label = _c(img), _c(atlas), _c(label)
    if atlas.ndim == 3:
        atlas, label = atlas[None], label[None]
    nx, ny, nz = _dims(img)
    out = np.zeros_like(img)
    st = reference().pctref_fuse(img.ctypes.data, atlas.ctypes.data, label.ctypes.data,
                                 out.ctypes.data, nx, ny, nz, atlas.shape[0], nh, float(div),
                                 int(multicore), threads, 1)
    if st != 0:
        raise ValueError("pctref_fuse rejected its arguments")
    return out


def regularize_port(vol, nh: int) -> tuple[np.ndarray, int]:
    v = _c(vol).copy()
    nz, nx, ny = v.shape
    fills = port().pct_oracle_regularize((nh - 1) // 2, 1, nx, ny, nz, v.ctypes.data)
    return v, int(fills)


def regularize_reference(vol, nh: int) -> np.ndarray:
    v = _c(vol).copy()
    nz, nx, ny = v.shape
    reference().pctref_regularize((nh - 1) // 2, 1, nx, ny, nz, v.ctypes.data, 1)
    return v


def finalize_port(vol) -> np.ndarray:
    v = _c(vol).copy()
    port().pct_oracle_round(v.ctypes.data, v.size)
    port().pct_oracle_to_hu(v.ctypes.data, v.size)
    return v


def normalize_labels_port(ct_hu) -> np.ndarray:
    v = _c(ct_hu).copy()
    port().pct_oracle_normalize_labels(v.ctypes.data, v.size)
    return v


def div_port(sigma: float, beta: float) -> float:
    return float(port().pct_oracle_div(sigma, beta))
