"""Learned-proposal form (EXEC_CHOICE 7): the network, its training set, training and checkpoints.

The network (``csrc/pct_learned.h``) is a small 3D CNN over the co-located 9x9x9 patches of the
input MRI and one atlas MRI: conv 2->16 and three conv 16->16 (3x3x3 valid, ReLU), then three
linear heads 16->11 that score the offsets dw, du and dv of the 11^3 search window (a softmax
per axis). The inference kernels propose per row segment of 30 voxels along y and per atlas:
the per-axis probabilities of the segment's voxels are summed, the 4 most probable offsets per
axis kept and, of their 64 combinations, the 32 whose per-axis ranks sum to at most 4; only those
32 offsets get the exact FP32 SSD and a weight. Rows share the proposal of their block's anchor
row (blocks of 4 x 4 rows in z and x by default, ``Handle.set_learned_block``). A voxel whose
probability mass on the 32 (measured on the anchor row) is below a confidence threshold takes
the full 11^3 search instead.

Training targets come from the plain method itself: for a sampled (subject, atlas, voxel) the
exact FP32 SSD of all 1331 offsets, the 32 smallest, as one distribution per axis. Forward,
backward and Adam are this library's own CUDA kernels.

Checkpoints are a 16-byte header (``b"PCTLRN01"``, uint32 parameter count, uint32 0) followed by
the FP32 master weights, little-endian, in the flat order of ``csrc/pct_learned.h``.

Command line (training, then evaluation on held-out subjects against the plain method)::

    python -m pseudoctimaging_b200.learned --out model.pctl --subjects 8 --atlases 10 \\
        --size 222 222 112 --samples 2000000 --epochs 20
    python -m pseudoctimaging_b200.learned evaluate model.pctl --thresholds 0 0.3 0.5
"""
from __future__ import annotations

import argparse
import ctypes
import json
import pathlib
import sys
import time

import numpy as np

from . import PctError, TrainSubject, lib, synth_subject

NUM_PARAMS = lib.pct_model_num_params()
MAGIC = b"PCTLRN01"
# The network trained on 8 synthetic 222x222x112 subjects with 10 atlases (NH = 11); its training
# command and held-out evaluation sit beside it in learned_nh11.json.
CHECKPOINT = pathlib.Path(__file__).resolve().parent / "checkpoints" / "learned_nh11.pctl"
AXIS = 11
TOP_K = 32


def _check(st: int, what: str, model=None) -> None:
    if st != 0:
        msg = ""
        if model is not None:
            msg = (lib.pct_model_last_error(model) or b"").decode(errors="replace")
        raise PctError(st, f"{what}: {msg}")


class LearnedModel:
    """FP32 master weights + Adam state + the BF16 copy the kernels use, on one device."""

    def __init__(self, device: int = 0, seed: int = 0, params: np.ndarray | None = None):
        m = ctypes.c_void_p()
        _check(lib.pct_model_create(device, seed, ctypes.byref(m)), "pct_model_create")
        self._m = m
        self.device = device
        if params is not None:
            self.set_params(params)

    @property
    def ptr(self):
        return self._m

    def close(self) -> None:
        if getattr(self, "_m", None) and self._m.value:
            lib.pct_model_destroy(self._m)
            self._m = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(params, np.float32)
        if p.shape != (NUM_PARAMS,):
            raise ValueError(f"expected {NUM_PARAMS} parameters, got {p.shape}")
        _check(lib.pct_model_set_params(self._m, p.ctypes.data), "pct_model_set_params", self._m)

    def get_params(self, inference_precision: bool = False) -> np.ndarray:
        p = np.empty(NUM_PARAMS, np.float32)
        _check(lib.pct_model_get_params(self._m, p.ctypes.data, int(inference_precision)),
               "pct_model_get_params", self._m)
        return p

    def gradients(self, ts: "TrainSet", begin: int, count: int) -> tuple[np.ndarray, float]:
        g = np.empty(NUM_PARAMS, np.float32)
        loss = ctypes.c_float()
        _check(lib.pct_model_gradients(self._m, ts.ptr, begin, count, g.ctypes.data,
                                       ctypes.byref(loss)), "pct_model_gradients", self._m)
        return g, float(loss.value)

    def train(self, ts: "TrainSet", batch: int, steps: int, lr: float) -> float:
        loss = ctypes.c_float()
        _check(lib.pct_model_train(self._m, ts.ptr, batch, steps, float(lr), ctypes.byref(loss)),
               "pct_model_train", self._m)
        return float(loss.value)

    def probe(self, d_img: int, d_atlas: int, nx: int, ny: int, nz: int, voxels):
        """conv4 features [n][16], proposal offsets [n][3][4] (rank order) and confidence [n]."""
        v = np.ascontiguousarray(voxels, np.int64)
        n = len(v)
        feats = np.empty((n, 16), np.float32)
        top = np.empty((n, 3, 4), np.int8)
        conf = np.empty(n, np.float32)
        _check(lib.pct_model_probe(self._m, d_img, d_atlas, nx, ny, nz, v.ctypes.data, n,
                                   feats.ctypes.data, top.ctypes.data, conf.ctypes.data),
               "pct_model_probe", self._m)
        return feats, top, conf

    def save(self, path) -> None:
        _check(lib.pct_model_save_file(self._m, str(path).encode()), "pct_model_save_file",
               self._m)

    @classmethod
    def load(cls, path, device: int = 0) -> "LearnedModel":
        m = cls(device=device)
        _check(lib.pct_model_load_file(m._m, str(path).encode()), "pct_model_load_file", m._m)
        return m


def save_params(path, params: np.ndarray) -> None:
    p = np.ascontiguousarray(params, "<f4")
    if p.shape != (NUM_PARAMS,):
        raise ValueError("wrong parameter count")
    with open(path, "wb") as f:
        f.write(MAGIC + np.array([NUM_PARAMS, 0], "<u4").tobytes() + p.tobytes())


def load_params(path) -> np.ndarray:
    raw = pathlib.Path(path).read_bytes()
    if raw[:8] != MAGIC:
        raise ValueError(f"{path}: not a learned-proposal checkpoint")
    n = int(np.frombuffer(raw[8:12], "<u4")[0])
    if n != NUM_PARAMS or len(raw) != 16 + 4 * n:
        raise ValueError(f"{path}: {n} parameters, this build has {NUM_PARAMS}")
    return np.frombuffer(raw[16:], "<f4").astype(np.float32)


class TrainSet:
    """Samples (subject, atlas, voxel) over device-resident subjects, with targets computed on the
    GPU from the plain method. ``subjects``: list of (d_img, d_atlas, nx, ny, nz, num_atlas)."""

    def __init__(self, subjects, samples, device: int = 0):
        arr = (TrainSubject * len(subjects))(
            *[TrainSubject(img=s[0], atlas=s[1], nx=s[2], ny=s[3], nz=s[4], num_atlas=s[5])
              for s in subjects])
        smp = np.ascontiguousarray(samples, np.int32)
        ts = ctypes.c_void_p()
        _check(lib.pct_train_set_create(device, arr, len(subjects), smp.ctypes.data, len(smp),
                                        ctypes.byref(ts)), "pct_train_set_create")
        self.ptr, self.n = ts, len(smp)

    def targets(self) -> tuple[np.ndarray, np.ndarray]:
        t = np.empty((self.n, 3 * AXIS), np.float32)
        top = np.empty((self.n, TOP_K), np.int16)
        _check(lib.pct_train_set_targets(self.ptr, t.ctypes.data, top.ctypes.data),
               "pct_train_set_targets")
        return t, top

    def close(self) -> None:
        if self.ptr and self.ptr.value:
            lib.pct_train_set_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def random_samples(shapes, n: int, seed: int) -> np.ndarray:
    """n samples (subject, atlas, flat voxel) uniform over subjects, atlases and the NH=11
    interior; shapes: list of (nx, ny, nz, num_atlas)."""
    rng = np.random.default_rng(seed)
    s = rng.integers(0, len(shapes), n)
    out = np.empty((n, 3), np.int64)
    for k, (nx, ny, nz, num) in enumerate(shapes):
        idx = np.nonzero(s == k)[0]
        z = rng.integers(6, nz - 6, len(idx))
        x = rng.integers(6, nx - 6, len(idx))
        y = rng.integers(6, ny - 6, len(idx))
        out[idx, 0] = k
        out[idx, 1] = rng.integers(0, num, len(idx))
        out[idx, 2] = (z * nx + x) * ny + y
    return out.astype(np.int32)


def structured_samples(images, num_atlas: int, n: int, seed: int) -> np.ndarray:
    """n samples drawn with probability proportional to the input MRI's gradient magnitude over
    the NH=11 interior (the regions where the SSD landscape has a shape to learn); images: one
    [nz][nx][ny] input MRI per subject, each with num_atlas atlases."""
    rng = np.random.default_rng(seed)
    per = np.bincount(rng.integers(0, len(images), n), minlength=len(images))
    out = []
    for k, img in enumerate(images):
        nz, nx, ny = img.shape
        g = np.sqrt(sum(d.astype(np.float64) ** 2 for d in np.gradient(img.astype(np.float32))))
        w = g[6:nz - 6, 6:nx - 6, 6:ny - 6].ravel()
        flat = rng.choice(w.size, per[k], p=w / w.sum())
        iz, ix, iy = np.unravel_index(flat, (nz - 12, nx - 12, ny - 12))
        vox = ((iz + 6) * nx + (ix + 6)) * ny + (iy + 6)
        out.append(np.stack([np.full(per[k], k), rng.integers(0, num_atlas, per[k]), vox], 1))
    smp = np.concatenate(out)
    return smp[rng.permutation(len(smp))].astype(np.int32)


KEPT_LEVEL = {10: 2, 20: 3, 32: 4}


def rank_sum_set(top: np.ndarray, k: int = 32) -> np.ndarray:
    """The kept offsets of one proposal, top [3][4] (dw, du, dv in rank order): rank triples
    (i, j, l) with i + j + l <= 4 for k = 32 (3 for k = 20, 2 for k = 10). Returns [k][3]
    offsets in -5..5."""
    level = KEPT_LEVEL[k]
    out = [(top[0][i], top[1][j], top[2][l]) for i in range(4) for j in range(4) for l in range(4)
           if i + j + l <= level]
    return np.array(out, np.int64)


def train_driver(argv=None) -> dict:
    """Generates synthetic subjects on the host, moves them to the GPU, builds the training set
    (targets from the plain method) and trains; writes the checkpoint and a JSON summary line."""
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--subjects", type=int, default=8)
    ap.add_argument("--atlases", type=int, default=10)
    ap.add_argument("--size", type=int, nargs=3, default=[222, 222, 112], metavar=("NX", "NY", "NZ"))
    ap.add_argument("--blobs", type=int, default=60)
    ap.add_argument("--samples", type=int, default=2_000_000)
    ap.add_argument("--structured", type=float, default=0.5,
                    help="share of samples drawn in proportion to the MRI gradient magnitude")
    ap.add_argument("--epochs", type=float, default=1.0)
    ap.add_argument("--batch", type=int, default=1184)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--lr-final", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--max-seconds", type=float, default=0.0, help="stop training after this")
    ap.add_argument("--init", default=None, help="start from this checkpoint")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)

    import torch

    torch.cuda.set_device(a.device)
    nx, ny, nz = a.size
    t0 = time.time()
    keep, subs, images = [], [], []
    for k in range(a.subjects):
        s = synth_subject(nx, ny, nz, a.atlases, n_blobs=a.blobs, seed=a.seed + k)
        images.append(s.img)
        d_img = torch.from_numpy(s.img).cuda()
        d_atl = torch.from_numpy(s.atlas_mri).cuda()
        keep.append((d_img, d_atl))
        subs.append((d_img.data_ptr(), d_atl.data_ptr(), nx, ny, nz, a.atlases))
    t_gen = time.time() - t0
    n_struct = int(round(a.structured * a.samples))
    samples = np.concatenate([
        random_samples([(nx, ny, nz, a.atlases)] * a.subjects, a.samples - n_struct, a.seed),
        structured_samples(images, a.atlases, n_struct, a.seed + 1)])
    samples = samples[np.random.default_rng(a.seed + 2).permutation(len(samples))]
    t0 = time.time()
    ts = TrainSet(subs, samples, a.device)
    t_targets = time.time() - t0
    model = LearnedModel(a.device, seed=a.seed)
    if a.init:
        model.set_params(load_params(a.init))
    steps_per_epoch = max(1, a.samples // a.batch)
    total = max(1, int(round(a.epochs * steps_per_epoch)))
    chunk = max(1, min(100, total // 20 or 1))
    log, done, t0 = [], 0, time.time()
    while done < total:
        n = min(chunk, total - done)
        frac = done / total
        lr = a.lr * (a.lr_final / a.lr) ** frac  # exponential decay from lr to lr_final
        loss = model.train(ts, a.batch, n, lr)
        done += n
        log.append((done, round(time.time() - t0, 2), lr, loss))
        print(json.dumps({"step": done, "of": total, "lr": lr, "loss": loss,
                          "seconds": round(time.time() - t0, 1)}), flush=True)
        if a.max_seconds and time.time() - t0 > a.max_seconds:
            break
    t_train = time.time() - t0
    model.save(a.out)
    summary = {"checkpoint": str(a.out), "subjects": a.subjects, "atlases": a.atlases,
               "size": [nx, ny, nz], "samples": a.samples, "batch": a.batch, "steps": done,
               "samples_seen": done * a.batch, "seconds_generate": round(t_gen, 1),
               "seconds_targets": round(t_targets, 2), "seconds_train": round(t_train, 1),
               "samples_per_second": round(done * a.batch / max(t_train, 1e-9)),
               "first_loss": log[0][3], "final_loss": log[-1][3]}
    print(json.dumps(summary), flush=True)
    ts.close()
    model.close()
    return summary


def prior_params(scales=(0.7, 0.5, 0.3)) -> np.ndarray:
    """A network without learned features: zero convolutions and head biases -c*(d)^2 per axis,
    so every voxel is proposed the same 32 offsets around the centre of the window (the
    proposal baseline "no network, same k")."""
    p = np.zeros(NUM_PARAMS, np.float32)
    hb = NUM_PARAMS - 3 * AXIS
    for a, c in enumerate(scales):
        for j in range(AXIS):
            p[hb + a * AXIS + j] = -c * (j - 5) ** 2
    return p


def evaluate(params: np.ndarray, subjects, thresholds=(0.0,), nh: int = 11, sigma: float = 2.5,
             beta: float = 1.0, reps: int = 3, device: int = 0) -> list[dict]:
    """Learned form against the plain method on device-resident subjects: per threshold, the mean
    absolute error in HU over voxels finite in both, the largest error, NaN-mask differences,
    the share of (voxel, atlas) pairs that fell back, offsets evaluated per 30-voxel row, and the
    CUDA-event time of both paths. ``subjects``: host Subjects (img, atlas_mri, atlas_ct in HU)."""
    import torch

    from . import EXEC_B200_FP32, EXEC_LEARNED, Handle, div_from, normalize_labels

    div = div_from(sigma, beta)
    stream = torch.cuda.Stream(device)
    out = []
    with Handle(device) as h, LearnedModel(device, params=params) as m:
        for si, s in enumerate(subjects):
            nz, nx, ny = s.img.shape
            num = s.atlas_mri.shape[0]
            d = [torch.from_numpy(np.ascontiguousarray(a)).cuda(device)
                 for a in (s.img, s.atlas_mri, normalize_labels(s.atlas_ct))]
            o_plain = torch.zeros_like(d[0])
            o_learn = torch.zeros_like(d[0])

            def run(choice, o):
                h.synthesize_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), o.data_ptr(),
                                    nx, ny, nz, num, nh, div, choice, stream.cuda_stream)

            def timed(choice, o):
                with torch.cuda.stream(stream):
                    run(choice, o)
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    for _ in range(reps):
                        run(choice, o)
                    e1.record(stream)
                    stream.synchronize()
                h.device_status(stream.cuda_stream)
                return e0.elapsed_time(e1) / reps

            ms_plain = timed(EXEC_B200_FP32, o_plain)
            ref = o_plain.cpu().numpy()[6:-6, 6:-6, 6:-6].astype(np.float64)
            pairs = (nz - 12) * (nx - 12) * (ny - 12) * num
            rows = (nz - 12) * (nx - 12) * -(-(ny - 12) // 30) * num
            for thr in thresholds:
                h.attach_model(m, thr)
                ms = timed(EXEC_LEARNED, o_learn)
                st = h.learned_stats()
                got = o_learn.cpu().numpy()[6:-6, 6:-6, 6:-6].astype(np.float64)
                both = np.isfinite(got) & np.isfinite(ref)
                err_hu = np.abs(got[both] - ref[both]) * (4095.0 / 255.0)
                out.append({"subject": si, "threshold": thr, "mae_hu": float(err_hu.mean()),
                            "max_abs_hu": float(err_hu.max()),
                            "nan_mismatch": int((np.isnan(got) != np.isnan(ref)).sum()),
                            "fallback_share": st["fallback_pairs"] / pairs,
                            "offsets_per_row": st["row_offsets"] / rows,
                            "ms_learned": ms, "ms_plain": ms_plain, "speedup": ms_plain / ms})
            h.attach_model(None)
    return out


def evaluate_driver(argv=None) -> list[dict]:
    ap = argparse.ArgumentParser(description="evaluate a learned-proposal checkpoint")
    ap.add_argument("checkpoint", help="checkpoint file, 'prior' (the same 32 offsets around the "
                    "window centre everywhere) or 'random' (an untrained network)")
    ap.add_argument("--subjects", type=int, default=2)
    ap.add_argument("--atlases", type=int, default=10)
    ap.add_argument("--size", type=int, nargs=3, default=[222, 222, 112])
    ap.add_argument("--blobs", type=int, default=60)
    ap.add_argument("--seed", type=int, default=5000, help="held-out subjects use seeds from here")
    ap.add_argument("--thresholds", type=float, nargs="+", default=[0.0])
    a = ap.parse_args(argv)
    if a.checkpoint == "prior":
        params = prior_params()
    elif a.checkpoint == "random":  # an untrained network: proposals without learned content
        with LearnedModel(0, seed=a.seed) as m:
            params = m.get_params()
    else:
        params = load_params(a.checkpoint)
    nx, ny, nz = a.size
    subs = [synth_subject(nx, ny, nz, a.atlases, n_blobs=a.blobs, seed=a.seed + k)
            for k in range(a.subjects)]
    res = evaluate(params, subs, a.thresholds)
    for r in res:
        print(json.dumps(r), flush=True)
    return res


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "evaluate":
        evaluate_driver(sys.argv[2:])
    else:
        train_driver(sys.argv[1:])
