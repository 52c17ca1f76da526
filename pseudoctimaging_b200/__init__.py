"""pct_b200: B200-native patch-based multi-atlas pseudo-CT synthesis.

Python mirror of the reference's operator interface for this path, over the C ABI of
``lib/libpct_b200.so`` (declared in ``include/pct_b200.h``):

* :func:`multi_patch_based_segmentation_gpu` follows ``MultiPatchBasedSegmentationGpu``
  (PatchBasedPseudoCT.cu:1635-1750): host arrays in the reference layout ``[atlas][z][x][y]``,
  an EXEC_CHOICE and ``div``; returns the synthesised label volume (NaN where the weights
  vanish, 0 on the border).
* :class:`Handle` exposes the device-pointer entry points (``synthesize_device`` etc.) for
  buffers that already live on the GPU (for instance ``torch`` tensors, via ``data_ptr()``).
* :func:`run_pipeline` is the reference ``main`` flow: label normalisation, the path,
  regularisation, rounding and the map back to HU.

There is no CPU fallback: every call goes to the CUDA library, and importing this module
raises if the library has not been built.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
from dataclasses import dataclass

import numpy as np

_PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = _PKG / "lib" / "libpct_b200.so"

# EXEC_CHOICE (PatchBasedPseudoCT.cu:71-78 for 0..2; the rest are this library's).
EXEC_GM, EXEC_GM2, EXEC_SM = 0, 1, 2
EXEC_B200_FP32 = 3
EXEC_TC_FP16, EXEC_TC_BF16 = 5, 6
EXEC_LEARNED, EXEC_BATCHED = 7, 8

PCT_OK = 0
STATUS = {
    0: "PCT_OK", -1: "PCT_ERR_INVALID_ARG", -2: "PCT_ERR_CUDA", -3: "PCT_ERR_OUT_OF_MEMORY",
    -4: "PCT_ERR_UNSUPPORTED", -5: "PCT_ERR_NO_DEVICE", -6: "PCT_ERR_TIMEOUT",
    -7: "PCT_ERR_INTERNAL", -8: "PCT_ERR_TOO_LARGE",
}


class PctError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        name = STATUS.get(status, str(status))
        super().__init__(f"{name}: {message}" if message else name)


class ErrorStats(ctypes.Structure):
    _fields_ = [("mae_hu", ctypes.c_double), ("max_abs_hu", ctypes.c_double),
                ("max_rel", ctypes.c_double), ("compared", ctypes.c_int64),
                ("nan_mismatch", ctypes.c_int64), ("nan_both", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SynthParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("num_atlas", ctypes.c_int), ("n_blobs", ctypes.c_int),
                ("amp_lo", ctypes.c_float), ("amp_hi", ctypes.c_float),
                ("std_lo", ctypes.c_float), ("std_hi", ctypes.c_float),
                ("mri_noise", ctypes.c_float), ("ct_noise", ctypes.c_float),
                ("max_disp", ctypes.c_float), ("seed", ctypes.c_uint64)]


class SubjectDesc(ctypes.Structure):
    """pct_subject: one subject of a batch (device pointers)."""
    _fields_ = [("img", ctypes.c_void_p), ("atlas", ctypes.c_void_p),
                ("atlas_label", ctypes.c_void_p), ("out", ctypes.c_void_p),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("num_atlas", ctypes.c_int), ("nh", ctypes.c_int), ("div", ctypes.c_double)]


class TrainSubject(ctypes.Structure):
    """pct_train_subject: a device-resident subject for building a training set."""
    _fields_ = [("img", ctypes.c_void_p), ("atlas", ctypes.c_void_p), ("nx", ctypes.c_int),
                ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("num_atlas", ctypes.c_int)]


class Plan(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int), ("groups", ctypes.c_int), ("tiles", ctypes.c_int),
                ("ctas", ctypes.c_int), ("tile_rows", ctypes.c_int),
                ("tile_planes", ctypes.c_int), ("scratch_bytes", ctypes.c_size_t)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_SZ = ctypes.c_size_t

# name -> (restype, argtypes); one entry per function of include/pct_b200.h.
SIGNATURES = {
    "pct_abi_version": (_I, []),
    "pct_strerror": (ctypes.c_char_p, [_I]),
    "pct_last_error_message": (ctypes.c_char_p, [_P]),
    "pct_create": (_I, [_I, ctypes.POINTER(_P)]),
    "pct_destroy": (_I, [_P]),
    "pct_set_memory_limit": (_I, [_P, _SZ]),
    "pct_set_stream": (_I, [_P, _P]),
    "pct_synthesize": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _D, _I]),
    "pct_synthesize_device": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _D, _I, _P]),
    "pct_device_status": (_I, [_P, _P]),
    "pct_query_plan": (_I, [_I, _I, _I, _I, _I, _I, ctypes.POINTER(Plan)]),
    "pct_slab_plan": (_I, [_I, _I, _I, _I] + [ctypes.POINTER(_I)] * 4),
    "pct_synthesize_batch": (_I, [_P, ctypes.POINTER(SubjectDesc), _I, _P]),
    "pct_batch_create": (_I, [_P, ctypes.POINTER(SubjectDesc), _I, _P, ctypes.POINTER(_P)]),
    "pct_batch_launch": (_I, [_P, _P]),
    "pct_batch_status": (_I, [_P, _P]),
    "pct_batch_destroy": (_I, [_P]),
    "pct_tile_sets": (_I, []),
    "pct_set_tile_set": (_I, [_P, _I]),
    "pct_set_kernel_timing": (_I, [_P, _I]),
    "pct_kernel_time": (_I, [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]),
    "pct_get_tile_set": (_I, [_P]),
    "pct_autotune": (_I, [_P, ctypes.POINTER(SubjectDesc), _I, ctypes.c_char_p,
                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]),
    "pct_normalize_labels_device": (_I, [_P, _P, _SZ, _P]),
    "pct_regularize_device": (_I, [_P, _P, _I, _I, _I, _I, ctypes.POINTER(ctypes.c_int64), _P]),
    "pct_regularize_device_noalloc": (_I, [_P, _I, _I, _I, _I, ctypes.POINTER(ctypes.c_int64),
                                            _P]),
    "pct_finalize_hu_device": (_I, [_P, _P, _SZ, _P]),
    "pct_run_pipeline": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _D, _D, _I, _I]),
    "pct_error_stats_device": (_I, [_P, _P, _P, _I, _I, _I, _I, ctypes.POINTER(ErrorStats), _P]),
    "pct_matrixio_dims": (_I, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]),
    "pct_matrixio_read": (_I, [ctypes.c_char_p, _P, _SZ]),
    "pct_matrixio_write": (_I, [ctypes.c_char_p, _P, _I, _I, _I, _I]),
    "pct_raw_read": (_I, [ctypes.c_char_p, _P, _SZ]),
    "pct_raw_write": (_I, [ctypes.c_char_p, _P, _SZ]),
    "pct_mat_dims": (_I, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]),
    "pct_mat_read": (_I, [ctypes.c_char_p, _P, _P, _P, _SZ, _SZ]),
    "pct_mat_write": (_I, [ctypes.c_char_p, ctypes.c_char_p, _P, _I, _I, _I]),
    "pct_ncc_device": (_I, [_P, _P, _P, _I, _I, _I, _I, ctypes.POINTER(ctypes.c_double),
                            ctypes.POINTER(ctypes.c_int64), _P]),
    "pct_test_wait_timeout": (_I, [_P, _D]),
    "pct_model_num_params": (_I, []),
    "pct_model_create": (_I, [_I, ctypes.c_uint64, ctypes.POINTER(_P)]),
    "pct_model_destroy": (_I, [_P]),
    "pct_model_last_error": (ctypes.c_char_p, [_P]),
    "pct_model_set_params": (_I, [_P, _P]),
    "pct_model_get_params": (_I, [_P, _P, _I]),
    "pct_model_load_file": (_I, [_P, ctypes.c_char_p]),
    "pct_model_save_file": (_I, [_P, ctypes.c_char_p]),
    "pct_train_set_create": (_I, [_I, ctypes.POINTER(TrainSubject), _I, _P, _I,
                                  ctypes.POINTER(_P)]),
    "pct_train_set_targets": (_I, [_P, _P, _P]),
    "pct_train_set_destroy": (_I, [_P]),
    "pct_model_gradients": (_I, [_P, _P, _I, _I, _P, ctypes.POINTER(ctypes.c_float)]),
    "pct_model_train": (_I, [_P, _P, _I, _I, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]),
    "pct_attach_model": (_I, [_P, _P, ctypes.c_float]),
    "pct_set_learned_block": (_I, [_P, _I]),
    "pct_set_learned_convs": (_I, [_P, _I]),
    "pct_set_learned_k": (_I, [_P, _I]),
    "pct_set_learned_prior": (_I, [_P, _I]),
    "pct_tc_survivors": (_I, [_P, _I, _P, _P, _P, _P, _I, _I, _I, _D, _P, _P]),
    "pct_learned_stats": (_I, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "pct_model_probe": (_I, [_P, _P, _P, _I, _I, _I, _P, _I, _P, _P, _P]),
    "pct_synth_default_params": (_I, [ctypes.POINTER(SynthParams), _I, _I, _I, _I, _I,
                                      ctypes.c_uint64]),
    "pct_synth_generate": (_I, [ctypes.POINTER(SynthParams), _P, _P, _P]),
}


def load_library(path: os.PathLike | str | None = None) -> ctypes.CDLL:
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python pseudoctimaging_b200/build.py` "
            "(the CUDA library is required; there is no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load_library()


def query_plan(nx: int, ny: int, nz: int, num: int, nh: int, device: int = 0) -> dict:
    """How the device entry point would run this shape (launches, atlas groups, tiles, grid)."""
    p = Plan()
    st = lib.pct_query_plan(device, nx, ny, nz, num, nh, ctypes.byref(p))
    if st != PCT_OK:
        raise PctError(st, "pct_query_plan")
    return p.as_dict()


def div_from(sigma: float, beta: float) -> float:
    """div = 2*27*beta*sigma^2 (PatchBasedPseudoCT.cu:2154)."""
    return 2 * 27 * beta * sigma ** 2


def normalize_labels(ct_hu: np.ndarray) -> np.ndarray:
    """Host copy of the reference's label scale, 255*((L+1024)/4095) in float32."""
    ct = np.asarray(ct_hu, dtype=np.float32)
    return (np.float32(255.0) * ((ct + np.float32(1024.0)) / np.float32(4095.0))).astype(np.float32)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _f32c(a, name: str) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a


def _shape3(img: np.ndarray) -> tuple[int, int, int]:
    if img.ndim != 3:
        raise ValueError("img must be a 3-D array [z][x][y]")
    nz, nx, ny = img.shape
    return nx, ny, nz


class Handle:
    """A device context with cached buffers (one per host thread)."""

    def __init__(self, device: int = 0):
        h = _P()
        st = lib.pct_create(device, ctypes.byref(h))
        if st != PCT_OK:
            raise PctError(st, f"pct_create(device={device})")
        self._h = h

    @property
    def ptr(self) -> int:
        return self._h.value

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib.pct_destroy(self._h)
            self._h = _P()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str) -> None:
        if st != PCT_OK:
            msg = lib.pct_last_error_message(self._h) or b""
            raise PctError(st, f"{what}: {msg.decode(errors='replace')}")

    def set_stream(self, stream: int | None) -> None:
        """cudaStream_t (as an int) for host-pointer calls; None/0 = the handle's own stream."""
        self._check(lib.pct_set_stream(self._h, stream or None), "pct_set_stream")

    def set_memory_limit(self, nbytes: int) -> None:
        self._check(lib.pct_set_memory_limit(self._h, nbytes), "pct_set_memory_limit")

    def set_learned_block(self, block: int) -> None:
        """Rows per proposal block along z and x for EXEC_LEARNED (default 4; 1 = per row
        segment)."""
        self._check(lib.pct_set_learned_block(self._h, int(block)), "pct_set_learned_block")

    def set_learned_k(self, k: int) -> None:
        """Offsets rescored per proposal for EXEC_LEARNED: 32 (default; rank triples i + j + k <=
        4 of the 4 best offsets per axis), 20 (<= 3) or 10 (<= 2)."""
        self._check(lib.pct_set_learned_k(self._h, int(k)), "pct_set_learned_k")

    def set_learned_prior(self, k: int) -> None:
        """k > 0: EXEC_CHOICE 7 runs the no-network centre prior with k offsets; 0: the network."""
        self._check(lib.pct_set_learned_prior(self._h, k), "pct_set_learned_prior")

    def set_learned_convs(self, every_voxel: bool) -> None:
        """Diagnostic: True = EXEC_LEARNED's convolutions over every voxel instead of only the
        outputs the anchor rows need (bit-identical result)."""
        self._check(lib.pct_set_learned_convs(self._h, int(bool(every_voxel))),
                    "pct_set_learned_convs")

    def attach_model(self, model, conf_threshold: float = 0.0) -> None:
        """Makes EXEC_LEARNED available (NH 7, 9, 11) with a :class:`learned.LearnedModel` (None
        detaches). Pairs whose 32 proposals hold less than ``conf_threshold`` of the proposal's
        probability mass fall back to the full search. The model must outlive its use."""
        self._model = model
        self._check(lib.pct_attach_model(self._h, model.ptr if model is not None else None,
                                         float(conf_threshold)), "pct_attach_model")

    def learned_stats(self) -> dict:
        """Counters of the last learned run: ``fallback_pairs`` ((voxel, atlas) pairs that took
        the full search) and ``row_offsets`` (offsets evaluated, summed over 30-voxel rows)."""
        f, r = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(lib.pct_learned_stats(self._h, ctypes.byref(f), ctypes.byref(r)),
                    "pct_learned_stats")
        return {"fallback_pairs": int(f.value), "row_offsets": int(r.value)}

    def synthesize(self, img, atlas, atlas_label, nh: int, div: float,
                   exec_choice: int = EXEC_B200_FP32) -> np.ndarray:
        """Host arrays in, host label volume out (the drop-in entry point)."""
        img = _f32c(img, "img")
        atlas = _f32c(atlas, "atlas")
        atlas_label = _f32c(atlas_label, "atlas_label")
        nx, ny, nz = _shape3(img)
        if atlas.ndim == 3:
            atlas = atlas[None]
        if atlas_label.ndim == 3:
            atlas_label = atlas_label[None]
        num = atlas.shape[0]
        if atlas.shape != (num, nz, nx, ny) or atlas_label.shape != atlas.shape:
            raise ValueError("atlas / atlas_label must be [num][z][x][y] matching img")
        out = np.empty_like(img)
        self._check(lib.pct_synthesize(self._h, _ptr(img), _ptr(atlas), _ptr(atlas_label), _ptr(out),
                                       nx, ny, nz, num, nh, float(div), exec_choice),
                    "pct_synthesize")
        return out

    def synthesize_device(self, d_img: int, d_atlas: int, d_label: int, d_out: int, nx: int,
                          ny: int, nz: int, num: int, nh: int, div: float,
                          exec_choice: int = EXEC_B200_FP32, stream: int = 0) -> None:
        self._check(lib.pct_synthesize_device(self._h, d_img, d_atlas, d_label, d_out, nx, ny, nz,
                                              num, nh, float(div), exec_choice, stream or None),
                    "pct_synthesize_device")

    def device_status(self, stream: int = 0) -> None:
        """Drains `stream` and raises PctError if a kernel's bounded wait gave up."""
        self._check(lib.pct_device_status(self._h, stream or None), "pct_device_status")

    def normalize_labels_device(self, d_label: int, n: int, stream: int = 0) -> None:
        self._check(lib.pct_normalize_labels_device(self._h, d_label, n, stream or None),
                    "pct_normalize_labels_device")

    def regularize_device(self, d_vol: int, nx: int, ny: int, nz: int, nh: int,
                          stream: int = 0) -> int:
        fills = ctypes.c_int64(0)
        self._check(lib.pct_regularize_device(self._h, d_vol, nx, ny, nz, nh, ctypes.byref(fills),
                                              stream or None), "pct_regularize_device")
        return fills.value

    def finalize_hu_device(self, d_vol: int, n: int, stream: int = 0) -> None:
        self._check(lib.pct_finalize_hu_device(self._h, d_vol, n, stream or None),
                    "pct_finalize_hu_device")

    def error_stats_device(self, d_a: int, d_b: int, nx: int, ny: int, nz: int, nh: int,
                           stream: int = 0) -> dict:
        st = ErrorStats()
        self._check(lib.pct_error_stats_device(self._h, d_a, d_b, nx, ny, nz, nh, ctypes.byref(st),
                                               stream or None), "pct_error_stats_device")
        return st.as_dict()

    @staticmethod
    def _subjects(subjects) -> "ctypes.Array":
        arr = (SubjectDesc * len(subjects))()
        for i, sd in enumerate(subjects):
            arr[i] = sd if isinstance(sd, SubjectDesc) else SubjectDesc(**sd)
        return arr

    def synthesize_batch(self, subjects, stream: int = 0) -> None:
        """One persistent launch over `subjects` (SubjectDesc or dicts of its fields)."""
        arr = self._subjects(subjects)
        self._check(lib.pct_synthesize_batch(self._h, arr, len(arr), stream or None),
                    "pct_synthesize_batch")

    def batch_graph(self, subjects, stream: int = 0) -> "BatchGraph":
        return BatchGraph(self, subjects, stream)

    def set_kernel_timing(self, on: bool) -> None:
        """Record CUDA events around every fusion launch of the plain path from now on."""
        self._check(lib.pct_set_kernel_timing(self._h, int(bool(on))), "pct_set_kernel_timing")

    def kernel_time(self) -> tuple[float, int]:
        """(summed device ms, launches) of the fusion launches timed since the last read."""
        ms, n = ctypes.c_double(), ctypes.c_int()
        self._check(lib.pct_kernel_time(self._h, ctypes.byref(ms), ctypes.byref(n)),
                    "pct_kernel_time")
        return float(ms.value), int(n.value)

    def set_tile_set(self, k: int) -> None:
        self._check(lib.pct_set_tile_set(self._h, k), "pct_set_tile_set")

    @property
    def tile_set(self) -> int:
        return lib.pct_get_tile_set(self._h)

    def autotune(self, subjects, cache_path=None) -> tuple[int, list[float]]:
        """Times every compiled tile set on the batch; keeps the fastest on this handle."""
        arr = self._subjects(subjects)
        n = lib.pct_tile_sets()
        ms = (ctypes.c_double * n)()
        chosen = ctypes.c_int(-1)
        path = str(cache_path).encode() if cache_path else None
        self._check(lib.pct_autotune(self._h, arr, len(arr), path, ms, ctypes.byref(chosen)),
                    "pct_autotune")
        return chosen.value, list(ms)

    def ncc_device(self, d_a: int, d_b: int, nx: int, ny: int, nz: int, nh: int,
                   stream: int = 0) -> tuple[float, int]:
        v, n = ctypes.c_double(0.0), ctypes.c_int64(0)
        self._check(lib.pct_ncc_device(self._h, d_a, d_b, nx, ny, nz, nh, ctypes.byref(v),
                                       ctypes.byref(n), stream or None), "pct_ncc_device")
        return v.value, n.value

    def test_wait_timeout(self, timeout_ms: float) -> None:
        """Arms the one-shot bounded-wait test of the next fusion launch."""
        self._check(lib.pct_test_wait_timeout(self._h, float(timeout_ms)), "pct_test_wait_timeout")

    def run_pipeline(self, img, atlas_mri, atlas_ct_hu, nh: int, sigma: float, beta: float,
                     exec_choice: int = EXEC_B200_FP32, regularize: bool = True) -> np.ndarray:
        img = _f32c(img, "img")
        atlas_mri = _f32c(atlas_mri, "atlas_mri")
        atlas_ct_hu = _f32c(atlas_ct_hu, "atlas_ct_hu")
        nx, ny, nz = _shape3(img)
        num = atlas_mri.shape[0]
        out = np.empty_like(img)
        self._check(lib.pct_run_pipeline(self._h, _ptr(img), _ptr(atlas_mri), _ptr(atlas_ct_hu),
                                         _ptr(out), nx, ny, nz, num, nh, float(sigma), float(beta),
                                         exec_choice, int(bool(regularize))), "pct_run_pipeline")
        return out


class BatchGraph:
    """A batch captured into a CUDA graph (pct_batch_create); launch() replays it."""

    def __init__(self, handle: Handle, subjects, stream: int = 0):
        self._handle = handle
        self._arr = Handle._subjects(subjects)
        b = _P()
        handle._check(lib.pct_batch_create(handle._h, self._arr, len(self._arr), stream or None,
                                           ctypes.byref(b)), "pct_batch_create")
        self._b = b

    def launch(self, stream: int = 0) -> None:
        st = lib.pct_batch_launch(self._b, stream or None)
        if st != PCT_OK:
            raise PctError(st, "pct_batch_launch")

    def status(self, stream: int = 0) -> None:
        st = lib.pct_batch_status(self._b, stream or None)
        if st != PCT_OK:
            raise PctError(st, "pct_batch_status")

    def close(self) -> None:
        if getattr(self, "_b", None) and self._b.value:
            lib.pct_batch_destroy(self._b)
            self._b = _P()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


_default_handle: Handle | None = None


def default_handle() -> Handle:
    global _default_handle
    if _default_handle is None:
        _default_handle = Handle(0)
    return _default_handle


def multi_patch_based_segmentation_gpu(img, atlas, atlas_label, choice: int, div: float,
                                       nh: int) -> np.ndarray:
    """Mirror of MultiPatchBasedSegmentationGpu(img, atlas, atlas_label, out, choice, div)
    (PatchBasedPseudoCT.cu:1635) with the reference's global ``nh`` as an argument and the
    output returned. ``atlas_label`` must already be label-normalised."""
    return default_handle().synthesize(img, atlas, atlas_label, nh, div, choice)


def run_pipeline(img, atlas_mri, atlas_ct_hu, nh: int, sigma: float = 1.0, beta: float = 1.0,
                 exec_choice: int = EXEC_B200_FP32, regularize: bool = True) -> np.ndarray:
    return default_handle().run_pipeline(img, atlas_mri, atlas_ct_hu, nh, sigma, beta,
                                         exec_choice, regularize)


def read_matrixio(path) -> np.ndarray:
    """A MatrixIO text volume as float32 [num][depth][rows][cols] (= [num][nz][nx][ny])."""
    dims = (ctypes.c_int * 4)()
    st = lib.pct_matrixio_dims(str(path).encode(), dims)
    if st != PCT_OK:
        raise PctError(st, f"pct_matrixio_dims({path})")
    num, rows, cols, depth = dims
    out = np.empty((num, depth, rows, cols), np.float32)
    st = lib.pct_matrixio_read(str(path).encode(), _ptr(out), out.size)
    if st != PCT_OK:
        raise PctError(st, f"pct_matrixio_read({path})")
    return out


def write_matrixio(path, vol) -> None:
    """Writes [num][nz][nx][ny] (or [nz][nx][ny]) float32 data in the MatrixIO text format."""
    v = np.ascontiguousarray(vol, np.float32)
    if v.ndim == 3:
        v = v[None]
    num, depth, rows, cols = v.shape
    st = lib.pct_matrixio_write(str(path).encode(), _ptr(v), num, rows, cols, depth)
    if st != PCT_OK:
        raise PctError(st, f"pct_matrixio_write({path})")


def read_mat(path):
    """The reference's MAT data file (img, atlas, atlas_label): (img [z][x][y], atlas MRI
    [num][z][x][y], atlas CT [num][z][x][y]) as float32, x = MATLAB dimension 1."""
    dims = (ctypes.c_int * 4)()
    st = lib.pct_mat_dims(str(path).encode(), dims)
    if st != PCT_OK:
        raise PctError(st, f"pct_mat_dims({path})")
    num, nx, ny, nz = dims
    img = np.empty((nz, nx, ny), np.float32)
    atl = np.empty((num, nz, nx, ny), np.float32)
    ct = np.empty((num, nz, nx, ny), np.float32)
    st = lib.pct_mat_read(str(path).encode(), _ptr(img), _ptr(atl), _ptr(ct), img.size, atl.size)
    if st != PCT_OK:
        raise PctError(st, f"pct_mat_read({path})")
    return img, atl, ct


def write_mat(path, variable: str, vol) -> None:
    """Writes a [z][x][y] float32 volume as one [nx ny nz] single variable of a MAT-file, as the
    reference writes its result."""
    v = np.ascontiguousarray(vol, np.float32)
    nz, nx, ny = v.shape
    st = lib.pct_mat_write(str(path).encode(), variable.encode(), _ptr(v), nx, ny, nz)
    if st != PCT_OK:
        raise PctError(st, f"pct_mat_write({path})")


@dataclass
class Subject:
    img: np.ndarray        # [z][x][y] input MRI
    atlas_mri: np.ndarray  # [num][z][x][y]
    atlas_ct: np.ndarray   # [num][z][x][y] CT in HU

    @property
    def shape(self):
        return self.img.shape


def synth_subject(nx: int, ny: int, nz: int, num_atlas: int, n_blobs: int = 20, seed: int = 0,
                  **overrides) -> Subject:
    """Seeded synthetic subject (pct_synth_generate); arrays are [z][x][y] / [num][z][x][y]."""
    p = SynthParams()
    st = lib.pct_synth_default_params(ctypes.byref(p), nx, ny, nz, num_atlas, n_blobs, seed)
    if st != PCT_OK:
        raise PctError(st, "pct_synth_default_params")
    for k, v in overrides.items():
        setattr(p, k, v)
    img = np.empty((nz, nx, ny), np.float32)
    mri = np.empty((num_atlas, nz, nx, ny), np.float32)
    ct = np.empty((num_atlas, nz, nx, ny), np.float32)
    st = lib.pct_synth_generate(ctypes.byref(p), _ptr(img), _ptr(mri), _ptr(ct))
    if st != PCT_OK:
        raise PctError(st, "pct_synth_generate")
    return Subject(img, mri, ct)


__all__ = [
    "EXEC_GM", "EXEC_GM2", "EXEC_SM", "EXEC_B200_FP32", "EXEC_TC_FP16", "EXEC_TC_BF16",
    "EXEC_LEARNED", "EXEC_BATCHED", "Handle", "BatchGraph", "SubjectDesc", "Plan", "PctError", "ErrorStats", "SynthParams", "Subject",
    "lib", "load_library", "div_from", "normalize_labels", "multi_patch_based_segmentation_gpu",
    "run_pipeline", "synth_subject", "default_handle", "LIB_PATH", "SIGNATURES",
]
