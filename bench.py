#!/usr/bin/env python
"""Benchmark of the pseudo-CT path: voxels/s at 222x222x112, 10 atlases, NH=11.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With --gpus N > 1 and no launcher around it, the command re-runs itself as N ranks under
torch.distributed.run; every arm checks that the ranks launched equal --gpus.

One step = one pass of the path (patch SSD -> exp weights -> weighted CT fusion) over one
synthetic subject (seeded generator; the reference's subject data is not public): one
pct_synthesize_device call on inputs resident in HBM. Timed with CUDA events on the launching
stream, W warm-up steps, K timed steps, barrier + synchronize on both sides, max over ranks.
Under torchrun each rank processes its own subject (weak scaling, no data-path collective).

`e2e` times the drop-in host-pointer entry point (pct_synthesize): pinned host inputs copied
in, the path, the volume copied out, every step.

`--impl reference` times the reference's own OpenMP CPU routine
(MultiAtlasPatchBasedSegmentationOpenMP, compiled unmodified into oracle/_ref) on all host
threads over a bounded slab of the same workload, extrapolated to the full volume by its
measured candidates/s (the per-voxel work is identical everywhere).
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

# Workload: config 1 at the metric's window (222x222x112, 10 atlases, NH=11, sigma 2.5, beta 1).
NX, NY, NZ, NUM, NH = 222, 222, 112, 10, 11
SIGMA, BETA = 2.5, 1.0
N_BLOBS = 60
METRIC = "pseudo-CT voxels/s at 222x222x112, 10 atlases, NH=11"
UNIT = "voxels/s"
# The reference's best published number for this metric: CUDA-SM on one V100 (DGX Station),
# 10.30 s for the 222x222x112 subject with 10 atlases at NH=11, transfers included.
PUBLISHED_NH11_VOXELS_PER_S = 535826.0
# Algorithmic FP32 lane-operations per candidate (voxel, atlas, offset): 1 sub + 1 mul for the
# squared difference, 6 adds for the separable 3x3x3 box sum, 1 scale, 1 FMA + 1 add for the two
# accumulators; plus 1 MUFU ex2.
OPS_PER_CANDIDATE = 11
FP32_LANES_PER_SM = 128
MUFU_LANES_PER_SM = 16
PROFILE_SUMMARY = REPO / "profiles" / "fuse_tma_nh11_222x222x112_10atlas.md"


def interior(n: int, nh: int) -> int:
    return max(0, n - 2 * ((nh - 1) // 2 + 1))


def candidates(nx=None, ny=None, nz=None, num=None, nh=None) -> int:
    """Candidates (voxel, atlas, offset) of one pass; defaults are the current workload."""
    nx = NX if nx is None else nx
    ny = NY if ny is None else ny
    nz = NZ if nz is None else nz
    num = NUM if num is None else num
    nh = NH if nh is None else nh
    return interior(nx, nh) * interior(ny, nh) * interior(nz, nh) * num * nh ** 3


class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self._t:
            self._t.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0, "fallback": True}


def profiled_traffic() -> float | None:
    """Per-launch DRAM bytes of the fusion kernel from the committed ncu summary, if any."""
    if not PROFILE_SUMMARY.exists():
        return None
    for line in PROFILE_SUMMARY.read_text().splitlines():
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------------- CPU side

def reference_inputs(sub_nz: int, seed: int = 1) -> dict:
    """The config-1 subject cropped to sub_nz planes, made by the seeded generator in a child
    process (which loads libpct_b200.so), handed over through a temporary .npz; the caller then
    loads only the oracle. Labels are normalised and div is computed by the oracle restatement."""
    import tempfile

    import oracle

    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "subject.npz")
        code = ("import sys, numpy as np; sys.path.insert(0, sys.argv[1]); "
                "import pseudoctimaging_b200 as pct; "
                "s = pct.synth_subject(*map(int, sys.argv[2:6]), n_blobs=int(sys.argv[6]), "
                "seed=int(sys.argv[7])); "
                "np.savez(sys.argv[8], img=s.img, mri=s.atlas_mri, ct=s.atlas_ct)")
        subprocess.run([sys.executable, "-c", code, str(REPO), str(NX), str(NY), str(sub_nz),
                        str(NUM), str(N_BLOBS), str(seed), path], check=True, timeout=600)
        with np.load(path) as z:
            img, mri, ct = z["img"], z["mri"], z["ct"]
    return {"img": img, "mri": mri, "label": oracle.normalize_labels_port(ct),
            "div": oracle.div_port(SIGMA, BETA)}


def cpu_reference_rate(target_s: float, threads: int = 0, subject: dict | None = None) -> dict:
    """Times the reference's OpenMP routine on a z/x-cropped slab of the workload (1 interior
    z-plane, enough interior x-rows for about target_s seconds); returns candidates/s."""
    import oracle

    lo = (NH - 1) // 2 + 1
    sub_nz = 2 * lo + 1
    s = subject if subject is not None else reference_inputs(sub_nz)

    def run(xrows: int) -> tuple[float, int]:
        nx = 2 * lo + xrows
        img = np.ascontiguousarray(s["img"][:, :nx, :])
        mri = np.ascontiguousarray(s["mri"][:, :, :nx, :])
        lab = np.ascontiguousarray(s["label"][:, :, :nx, :])
        t = time.perf_counter()
        oracle.fuse_reference(img, mri, lab, NH, s["div"], multicore=True, threads=threads)
        dt = time.perf_counter() - t
        return dt, candidates(nx, NY, sub_nz, NUM, NH)

    dt, c = run(2)  # calibration
    rate = c / dt
    rows = int(max(2, min(interior(NX, NH), round(target_s * rate / candidates(2 * lo + 1, NY, sub_nz, NUM, NH)))))
    dt, c = run(rows)
    cores = threads if threads > 0 else oracle.reference().pctref_max_threads()
    return {"cand_per_s": c / dt, "seconds": dt, "candidates": c, "cores": cores,
            "sample": f"{NY}x{rows}x1 interior voxels (slab {2 * lo + rows}x{NY}x{sub_nz} of the "
                      f"222x222x112 config-1 subject, seed 1), {NUM} atlases, NH={NH}"}


def run_reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle

    if not oracle.has_reference():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libpctref.so was not built (reference sources absent at build time)"}))
        return
    full = candidates()
    step_s = []
    last = None
    subject = reference_inputs(2 * ((NH - 1) // 2 + 1) + 1)
    for i in range(args.warmup + args.steps):
        r = cpu_reference_rate(args.ref_step_seconds, subject=subject)
        if i >= args.warmup:
            step_s.append(full / r["cand_per_s"])
            last = r
    t = statistics.median(step_s)
    value = NX * NY * NZ / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded blobs/displacement generator, config 1)",
        "config": {"workload": "222x222x112 subject, 10 atlases, NH=11, sigma 2.5, beta 1; "
                               "each step a bounded slab, extrapolated by candidates/s",
                   "nh": NH, "atlases": NUM, "volume": [NX, NY, NZ]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": last["cores"], "kind": "reference",
                         "sample": last["sample"], "cand_per_s": last["cand_per_s"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------------- GPU side

FP64_SAMPLE = 4000  # interior voxels per subject checked against the FP64 oracle


def sample_interior(nx: int, ny: int, nz: int, nh: int, n: int = FP64_SAMPLE,
                    seed: int = 7) -> np.ndarray:
    """Seeded uniform sample of interior voxels, as flat indices z*nx*ny + x*ny + y."""
    lo = (nh - 1) // 2 + 1
    rng = np.random.default_rng(seed)
    z = rng.integers(lo, nz - lo, n)
    x = rng.integers(lo, nx - lo, n)
    y = rng.integers(lo, ny - lo, n)
    return np.unique(z.astype(np.int64) * nx * ny + x.astype(np.int64) * ny + y)


class Fp64Check:
    """The FP64 CPU oracle (the restatement of MultiAtlasPatchBasedSegmentationOpenMP, bit-exact
    against the reference's own routine) at sampled interior voxels of one subject, and the error
    of any output volume against it: MAE and max abs in HU, max relative, NaN-mask mismatches."""

    def __init__(self, img, mri, label, nh, div, n=FP64_SAMPLE):
        import oracle

        nz, nx, ny = img.shape
        self.vox = sample_interior(nx, ny, nz, nh, n)
        t = time.perf_counter()
        out, prod, sumw = oracle.fuse_port_voxels(img, mri, label, nh, div, self.vox)
        self.seconds = time.perf_counter() - t
        self.nan = np.isnan(out)
        with np.errstate(invalid="ignore", divide="ignore"):
            self.ref = np.where(self.nan, np.nan, prod / sumw)

    def errors(self, vol) -> dict:
        a = np.asarray(vol).reshape(-1)[self.vox].astype(np.float64)
        both = np.isfinite(a) & ~self.nan
        d = np.abs(a[both] - self.ref[both])
        return {"mae_hu_vs_fp64": float(d.mean() * 4095.0 / 255.0),
                "max_abs_hu_vs_fp64": float(d.max() * 4095.0 / 255.0),
                "max_rel_vs_fp64": float((d / np.maximum(np.abs(self.ref[both]), 1e-30)).max()),
                "nan_mismatch_vs_fp64": int((np.isnan(a) != self.nan).sum()),
                "fp64_voxels": int(self.vox.size)}



def measure_e2e(h, s, label, div, sptr, stream, steps, world, dev) -> dict:
    """The drop-in host-pointer entry point (pct_synthesize) on pinned host buffers: every step
    copies the subject in, runs the path and copies the volume out, on `stream`."""
    import torch
    import torch.distributed as dist

    import pseudoctimaging_b200 as pct

    p_img = torch.from_numpy(s.img).pin_memory()
    p_mri = torch.from_numpy(s.atlas_mri).pin_memory()
    p_lab = torch.from_numpy(label).pin_memory()
    p_out = torch.empty_like(p_img).pin_memory()
    nz, nx, ny = s.img.shape
    h.set_stream(sptr)

    def e2e_step():
        st = pct.lib.pct_synthesize(h.ptr, p_img.data_ptr(), p_mri.data_ptr(), p_lab.data_ptr(),
                                    p_out.data_ptr(), nx, ny, nz, NUM, NH, div, pct.EXEC_B200_FP32)
        if st != 0:
            raise pct.PctError(st, "pct_synthesize")

    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    h.set_stream(None)
    nvox = nx * ny * nz
    return {"value": world * nvox / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "steps": steps, "h2d_bytes_per_step": int(4 * nvox * (1 + 2 * NUM)),
            "d2h_bytes_per_step": int(4 * nvox), "out": p_out}


def run_b200_arm(args) -> None:
    import torch
    import torch.distributed as dist

    import pseudoctimaging_b200 as pct

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    s = pct.synth_subject(NX, NY, NZ, NUM, n_blobs=N_BLOBS, seed=1 + rank)
    label = pct.normalize_labels(s.atlas_ct)
    div = pct.div_from(SIGMA, BETA)
    d_img = torch.from_numpy(s.img).to(dev)
    d_mri = torch.from_numpy(s.atlas_mri).to(dev)
    d_lab = torch.from_numpy(label).to(dev)
    d_out = torch.zeros_like(d_img)
    h = pct.Handle(local)
    if args.tile_set is not None:
        h.set_tile_set(args.tile_set)
    stream = torch.cuda.Stream(dev)  # a real stream handle, so events and kernels share it
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream

    def step():
        h.synthesize_device(d_img.data_ptr(), d_mri.data_ptr(), d_lab.data_ptr(),
                            d_out.data_ptr(), NX, NY, NZ, NUM, NH, div, pct.EXEC_B200_FP32, sptr)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h.kernel_time()  # drop anything recorded before the timed region
    h.set_kernel_timing(True)  # events around each fusion launch, on the same stream
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    h.set_kernel_timing(False)
    kernel_total_ms, kernel_launches = h.kernel_time()
    barrier()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    kernel_ms = kernel_total_ms / kernel_launches if kernel_launches else ms
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    nvox = NX * NY * NZ
    value = world * nvox / (ms / 1e3)

    e2e = None
    if not args.no_e2e:
        e2e = measure_e2e(h, s, label, div, sptr, stream, max(1, min(args.steps, 5)), world, dev)
        out = e2e.pop("out")
        assert np.array_equal(np.isnan(out.numpy()), np.isnan(d_out.cpu().numpy())), \
            "host-pointer and device-pointer runs disagree"

    plan = pct.query_plan(NX, NY, NZ, NUM, NH, local)
    clocks = clk.summary()
    check = Fp64Check(s.img, s.atlas_mri, label, NH, div)
    plain_fp64 = check.errors(d_out.cpu().numpy())
    forms = None
    if world == 1 and NH == 11 and not args.no_forms:
        forms = time_other_forms(pct, h, d_img, d_mri, d_lab, d_out, div, stream, args, check)
        fb = forms["learned_conf0.05"]
        # what the fallback may cost: its share of the plain method's time plus the learned form
        fb["bound_ms"] = fb["fallback_share"] * ms + forms["learned"]["ms_per_step"]
        forms["batch"] = measure_batch(args, max(3, args.steps // 4), 1)
    peaks = measured_peaks()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = clocks["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)
    cand = candidates()
    fp32_peak = sms * FP32_LANES_PER_SM * mhz * 1e6  # lane-ops/s at the sampled clock
    mufu_peak = sms * MUFU_LANES_PER_SM * mhz * 1e6
    # the roofline is the fusion kernel's: its own launches' device time in the timed region
    achieved = cand * OPS_PER_CANDIDATE / (kernel_ms / 1e3)
    traffic = profiled_traffic() if (NZ == 112 and NH == 11) else None
    hbm_achieved = (traffic / (kernel_ms / 1e3) / 1e9) if traffic else None

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": (value / PUBLISHED_NH11_VOXELS_PER_S
                        if (NZ == 112 and NH == 11) else None),
        "vs_baseline_ref": "reference's best published: CUDA-SM, 1x V100, 10.30 s incl. "
                           "transfers = 535,826 voxels/s (NH=11)",
        "dtype": "f32",
        "data": "synthetic (seeded blobs/displacement generator, config 1; one subject per GPU)",
        "config": {"workload": f"{NX}x{NY}x{NZ} subject, 10 atlases, NH={NH}, sigma 2.5, beta 1, "
                               "plain FP32 kernel (EXEC_CHOICE 3)",
                   "nh": NH, "atlases": NUM, "volume": [NX, NY, NZ],
                   "l2": f"inputs larger than L2 ({1 + 2 * NUM} volumes, "
                         f"{4 * nvox * (1 + 2 * NUM) / 1e6:.0f} MB per subject)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "tile_set": h.tile_set},
        "candidates_per_s": world * cand / (ms / 1e3),
        "gpu_launches": args.steps * plan["launches"],
        "plan": plan,
        "roofline": {
            "bound": "fp32", "unit": "TFLOP/s",
            "achieved": achieved / 1e12, "peak": fp32_peak / 1e12, "frac": achieved / fp32_peak,
            "traffic": traffic,
            "kernel": "fuse_tma_kernel", "kernel_ms": kernel_ms, "kernel_launches": kernel_launches,
            "note": (f"{OPS_PER_CANDIDATE} FP32 lane-ops per candidate x {cand:.3e} candidates per "
                     f"launch / the kernel's mean launch time ({kernel_launches} launches timed "
                     f"with CUDA events on the step's stream; the step adds the repack and the "
                     f"group combine); peak = {sms} SMs x {FP32_LANES_PER_SM} FP32 lanes x "
                     f"sampled SM clock {mhz:.0f} MHz; MUFU ex2 roof "
                     f"{cand / mufu_peak * 1e3:.2f} ms"),
            "mufu_frac": (cand / (kernel_ms / 1e3)) / mufu_peak,
            "hbm": {"achieved_gbs": hbm_achieved, "peak_gbs": peaks.get("hbm_gbs"),
                    "frac": (hbm_achieved / peaks["hbm_gbs"]) if hbm_achieved else None},
        },
        "e2e": e2e,
        "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "quality": dict(plain_fp64, fp64_seconds=check.seconds,
                        note="plain FP32 output vs the FP64 CPU oracle at sampled interior "
                             "voxels of the full-size subject"),
    }
    if forms:
        line["forms"] = forms
    h.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_rate(args.cpu_seconds)
        cpu_value = nvox / (cand / r["cand_per_s"])
        line["cpu_baseline"] = {"value": cpu_value, "unit": UNIT, "cores": r["cores"],
                                "kind": "reference", "sample": r["sample"],
                                "seconds": r["seconds"], "cand_per_s": r["cand_per_s"]}
    if rank == 0:
        print(json.dumps(line))


def time_other_forms(pct, h, d_img, d_mri, d_lab, d_plain, div, stream, args, check) -> dict:
    """The learned proposal (EXEC_CHOICE 7, committed network) and the tensor-core forms
    (5 FP16, 6 BF16) on the same resident subject as the plain kernel: CUDA-event time per step
    with its own clock record, the error against the plain kernel's output and against the FP64
    oracle at sampled voxels (HU), so one bench line carries every form."""
    import torch

    from pseudoctimaging_b200 import learned

    core = (slice(6, -6),) * 3
    ref = d_plain.cpu().numpy()[core].astype(np.float64)
    nvox = NX * NY * NZ
    model = learned.LearnedModel.load(learned.CHECKPOINT, torch.cuda.current_device())
    h.attach_model(model, 0.0)
    out = {}
    steps_fast = max(5, args.steps // 2)
    # prior_kN: the same rescoring without the network (the N window offsets nearest the
    # centre for every voxel), for comparing what the network buys at equal time
    # learned_conf0.05: the confidence fallback (tiles holding a voxel below the threshold run
    # the plain full search)
    for name, choice, steps, k, prior, conf in (
            ("learned", pct.EXEC_LEARNED, steps_fast, 32, 0, 0.0),
            ("learned_k20", pct.EXEC_LEARNED, steps_fast, 20, 0, 0.0),
            ("learned_k10", pct.EXEC_LEARNED, steps_fast, 10, 0, 0.0),
            ("learned_conf0.05", pct.EXEC_LEARNED, 3, 32, 0, 0.05),
            ("prior_k32", pct.EXEC_LEARNED, steps_fast, 0, 32, 0.0),
            ("prior_k57", pct.EXEC_LEARNED, steps_fast, 0, 57, 0.0),
            ("prior_k81", pct.EXEC_LEARNED, steps_fast, 0, 81, 0.0),
            ("prior_k123", pct.EXEC_LEARNED, steps_fast, 0, 123, 0.0),
            ("tc_fp16", pct.EXEC_TC_FP16, 5, 0, 0, 0.0),
            ("tc_bf16", pct.EXEC_TC_BF16, 5, 0, 0, 0.0)):
        o = torch.zeros_like(d_img)
        if k:
            h.set_learned_k(k)
        h.set_learned_prior(prior)
        h.attach_model(model, conf)

        def step():
            h.synthesize_device(d_img.data_ptr(), d_mri.data_ptr(), d_lab.data_ptr(), o.data_ptr(),
                                NX, NY, NZ, NUM, NH, div, choice, stream.cuda_stream)
        step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record(stream)
            for _ in range(steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize()
        h.device_status(stream.cuda_stream)
        ms = e0.elapsed_time(e1) / steps
        vol = o.cpu().numpy()
        g = vol[core].astype(np.float64)
        both = np.isfinite(g) & np.isfinite(ref)
        e = np.abs(g[both] - ref[both]) * (4095.0 / 255.0)
        c = clk.summary()
        out[name] = {"ms_per_step": ms, "value": nvox / (ms / 1e3), "steps": steps,
                     "mae_hu_vs_plain": float(e.mean()), "max_abs_hu_vs_plain": float(e.max()),
                     "nan_mismatch": int((np.isnan(g) != np.isnan(ref)).sum()),
                     **check.errors(vol),
                     "clocks": {kk: c[kk] for kk in ("sm_mhz", "sm_max_mhz", "reasons")}}
        if k or prior:
            st = h.learned_stats()
            out[name]["offsets_per_row"] = st["row_offsets"] / (
                (NZ - 12) * (NX - 12) * -(-(NY - 12) // 30) * NUM)
            out[name]["fallback_share"] = st["fallback_pairs"] / (
                (NZ - 12) * (NX - 12) * (NY - 12) * NUM)
    h.set_learned_prior(0)
    h.set_learned_k(32)
    h.attach_model(None)
    model.close()
    return out


def config3_specs(n: int = 16, seed: int = 3) -> list[tuple[int, int, int, int, int]]:
    """Config 3: subjects of uneven size (x, y in 96..222, z in 64..112), 5..20 atlases, NH in
    {7, 9, 11}, drawn from a seeded generator: (nx, ny, nz, num_atlas, nh)."""
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(96, 223)), int(rng.integers(96, 223)), int(rng.integers(64, 113)),
             int(rng.integers(5, 21)), int(rng.choice([7, 9, 11]))) for _ in range(n)]


def measure_batch(args, steps: int, warmup: int) -> dict:
    """Config 3: all subjects in one persistent launch captured in a CUDA graph, tile set chosen
    by the autotuner over every compiled set (timings per set reported); one step = one graph
    replay over every subject. The first subject is checked against the FP64 oracle at sampled
    voxels."""
    import tempfile

    import torch

    import pseudoctimaging_b200 as pct

    dev = torch.device("cuda", torch.cuda.current_device())
    specs = config3_specs(args.batch_subjects)
    subs, keep = [], []
    nvox = cand = 0
    check = None
    div = pct.div_from(SIGMA, BETA)
    for i, (nx, ny, nz, num, nh) in enumerate(specs):
        s = pct.synth_subject(nx, ny, nz, num, n_blobs=N_BLOBS, seed=100 + i)
        lab = pct.normalize_labels(s.atlas_ct)
        if i == 0:
            check = (Fp64Check(s.img, s.atlas_mri, lab, nh, div, n=1000), (nz, nx, ny))
        d = [torch.from_numpy(x).to(dev) for x in (s.img, s.atlas_mri, lab)]
        out = torch.zeros_like(d[0])
        keep.append((d, out))
        subs.append(pct.SubjectDesc(img=d[0].data_ptr(), atlas=d[1].data_ptr(),
                                    atlas_label=d[2].data_ptr(), out=out.data_ptr(), nx=nx, ny=ny,
                                    nz=nz, num_atlas=num, nh=nh, div=div))
        nvox += nx * ny * nz
        cand += candidates(nx, ny, nz, num, nh)
        del s
    h = pct.Handle(dev.index)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    cache = os.path.join(tempfile.gettempdir(), f"pct_b200_tune_{os.getpid()}.jsonl")
    chosen, tune_ms = h.autotune(subs, cache)
    g = h.batch_graph(subs, stream.cuda_stream)
    for _ in range(warmup):
        g.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        ev0.record(stream)
        for _ in range(steps):
            g.launch(stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
    g.status(stream.cuda_stream)
    ms = ev0.elapsed_time(ev1) / steps
    clocks = clk.summary()
    fp64 = check[0].errors(keep[0][1].cpu().numpy())
    g.close()
    h.close()
    try:
        os.remove(cache)
    except OSError:
        pass
    return {"workload": f"config 3: {len(specs)} subjects (x, y 96..222, z 64..112, 5..20 atlases, "
                        "NH 7/9/11), one persistent launch replayed as a CUDA graph",
            "ms_per_step": ms, "value": nvox / (ms / 1e3), "unit": UNIT, "steps": steps,
            "voxels": nvox, "candidates": cand, "candidates_per_s": cand / (ms / 1e3),
            "tile_set": chosen, "autotune_ms_per_set": tune_ms, "subjects": specs,
            "fp64_subject0": fp64,
            "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")}}


def run_batch_arm(args) -> None:
    """Config 3 as its own bench line (see measure_batch)."""
    b = measure_batch(args, args.steps, args.warmup)
    line = {
        "metric": f"pseudo-CT voxels/s, config 3 batch ({args.batch_subjects} subjects, one "
                  "persistent launch in a CUDA graph)",
        "value": b["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": b["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator, config 3)",
        "config": {"workload": "config 3 batch", "subjects": b["subjects"], "voxels": b["voxels"],
                   "candidates": b["candidates"], "tile_set": b["tile_set"],
                   "autotune_ms_per_set": b["autotune_ms_per_set"]},
        "candidates_per_s": b["candidates_per_s"],
        "fp64_subject0": b["fp64_subject0"],
        "gpu_launches": args.steps * 1,
        "clocks": b["clocks"],
    }
    print(json.dumps(line))


def run_sharded_arm(args) -> None:
    """One config-1 subject split into z slabs over the N ranks (one GPU each, strong scaling):
    each rank holds its slab plus hw+1 halo planes of every input volume in its own HBM and runs
    the plain kernel on that sub-volume; value = the whole subject's voxels / the slowest rank's
    time. The outputs are disjoint; an untimed NCCL all-gather assembles them once at the end
    and rank 0 checks the result against a whole-volume run on its GPU."""
    import datetime

    import torch
    import torch.distributed as dist

    import pseudoctimaging_b200 as pct
    from pseudoctimaging_b200 import shard

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    s = pct.synth_subject(NX, NY, NZ, NUM, n_blobs=N_BLOBS, seed=1)
    label = pct.normalize_labels(s.atlas_ct)
    div = pct.div_from(SIGMA, BETA)
    sl = shard.slab_plan(NZ, NH, world)[rank]
    sub = shard.extract(s.img, s.atlas_mri, label, sl)
    d = [torch.from_numpy(x).to(dev) for x in sub]
    d_out = torch.zeros_like(d[0])
    nzs = sl.src_planes
    h = pct.Handle(local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def step():
        h.synthesize_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d_out.data_ptr(),
                            NX, NY, nzs, NUM, NH, div, pct.EXEC_B200_FP32, stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    h.device_status(stream.cuda_stream)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1) / args.steps], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    # assemble once (untimed) and check on rank 0
    mine = d_out[sl.z_begin - sl.src_begin:sl.z_end - sl.src_begin]
    plan = shard.slab_plan(NZ, NH, world)
    biggest = max(p.planes for p in plan)
    buf = torch.zeros((biggest, NX, NY), device=dev)
    buf[:mine.shape[0]] = mine
    parts = [torch.empty_like(buf) for _ in range(world)]
    if world > 1:
        dist.all_gather(parts, buf)
    else:
        parts = [buf]
    check = None
    if rank == 0:
        whole = np.zeros((NZ, NX, NY), np.float32)
        for p, tt in zip(plan, parts):
            whole[p.z_begin:p.z_end] = tt[:p.planes].cpu().numpy()
        ref = h.synthesize(s.img, s.atlas_mri, label, NH, div, pct.EXEC_B200_FP32)
        both = np.isfinite(ref) & np.isfinite(whole)
        check = {"nan_mask_equal": bool(np.array_equal(np.isnan(ref), np.isnan(whole))),
                 "max_rel_vs_whole_volume": float(np.max(np.abs(whole[both] - ref[both]) /
                                                         np.maximum(np.abs(ref[both]), 1e-30)))}
    clocks = clk.summary()
    nvox = NX * NY * NZ
    line = {
        "metric": f"pseudo-CT voxels/s at {NX}x{NY}x{NZ}, 10 atlases, NH={NH}, one subject "
                  "z-sharded over the GPUs",
        "value": nvox / (ms / 1e3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, config 1)",
        "config": {"workload": "config 1 subject, z slabs + halo per GPU, plain FP32 kernel",
                   "slabs": [[p.z_begin, p.z_end] for p in plan], "parallelism": f"z-slab x{world}"},
        "check": check,
        "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
    }
    h.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def run_tc_arm(args) -> None:
    """Config 2: the tensor-core form (EXEC_CHOICE 5 FP16 and 6 BF16: tcgen05 correlation, top-16
    per (voxel, atlas), exact FP32 rescoring) on a 222x222x112 subject with 20 atlases, NH = 11,
    against the plain FP32 kernel on the same inputs: voxels/s of each, the error against the
    plain method in HU, and the error of every form against the FP64 CPU oracle at sampled
    interior voxels of the full-size subject."""
    import torch

    import pseudoctimaging_b200 as pct

    num = 20
    dev = torch.device("cuda", 0)
    s = pct.synth_subject(NX, NY, NZ, num, n_blobs=N_BLOBS, seed=2)
    label = pct.normalize_labels(s.atlas_ct)
    div = pct.div_from(SIGMA, BETA)
    d = [torch.from_numpy(x).to(dev) for x in (s.img, s.atlas_mri, label)]
    h = pct.Handle(0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    outs, times = {}, {}
    with ClockSampler(0) as clk:
        for choice, steps in ((pct.EXEC_B200_FP32, max(1, args.steps // 2)),
                              (pct.EXEC_TC_FP16, args.steps), (pct.EXEC_TC_BF16, args.steps)):
            o = torch.zeros_like(d[0])

            def step():
                h.synthesize_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), o.data_ptr(),
                                    NX, NY, NZ, num, 11, div, choice, stream.cuda_stream)
            for _ in range(args.warmup):
                step()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize()
            h.device_status(stream.cuda_stream)
            times[choice] = e0.elapsed_time(e1) / steps
            outs[choice] = o.cpu().numpy()
    core = (slice(6, -6),) * 3
    ref = outs[pct.EXEC_B200_FP32][core].astype(np.float64)
    nvox = NX * NY * NZ
    check = Fp64Check(s.img, s.atlas_mri, label, 11, div)
    forms = {}
    for choice, name in ((pct.EXEC_TC_FP16, "fp16"), (pct.EXEC_TC_BF16, "bf16")):
        g = outs[choice][core].astype(np.float64)
        both = np.isfinite(g) & np.isfinite(ref)
        e = np.abs(g[both] - ref[both]) * (4095.0 / 255.0)
        forms[name] = {"ms_per_step": times[choice], "value": nvox / (times[choice] / 1e3),
                       "mae_hu_vs_plain": float(e.mean()), "max_abs_hu_vs_plain": float(e.max()),
                       "nan_mismatch": int((np.isnan(g) != np.isnan(ref)).sum()),
                       **check.errors(outs[choice])}
    # tensor work: three K = 16 MMAs of 128 x 128 per chunk (the patch taps and norms, then the
    # window penalty and the voxel norm), 28 chunks per tile and atlas
    tiles = -(-(NZ - 12) // 4) * -(-(NX - 12) // 4) * -(-(NY - 12) // 8)
    flop = 2.0 * 128 * 128 * 48 * 28 * tiles * num
    peaks = measured_peaks()
    clocks = clk.summary()
    ms = times[pct.EXEC_TC_FP16]
    line = {
        "metric": f"pseudo-CT voxels/s at {NX}x{NY}x{NZ}, 20 atlases, NH=11, tensor-core form "
                  "(EXEC_CHOICE 5 FP16; BF16 beside it)",
        "value": forms["fp16"]["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp16/bf16 correlation, f32 rescoring",
        "data": "synthetic (seeded generator, config 2, seed 2)",
        "config": {"workload": "config 2: tensor-core correlation, top-16 per (voxel, atlas)",
                   "volume": [NX, NY, NZ], "atlases": num, "nh": 11},
        "forms": forms,
        "plain": {"ms_per_step": times[pct.EXEC_B200_FP32],
                  "value": nvox / (times[pct.EXEC_B200_FP32] / 1e3),
                  **check.errors(outs[pct.EXEC_B200_FP32])},
        # per FP16 step: the input mean, per atlas the patch rows and the main launch, per atlas
        # after the first the redo launch, and the finalisation
        "gpu_launches": args.steps * (3 * num + 1),
        "roofline": {"bound": "tensor", "unit": "TFLOP/s", "achieved": flop / (ms / 1e3) / 1e12,
                     "peak": peaks.get("bf16_tflops"),
                     "frac": flop / (ms / 1e3) / 1e12 / peaks["bf16_tflops"]
                     if peaks.get("bf16_tflops") else None,
                     "traffic": None,
                     "note": "dense correlation FLOPs (128 x 128 x 48 per chunk, 28 chunks per "
                             "tile and atlas) over the FP16 step; MMAs of N = 128 are issue-rate "
                             "bound, and the selection epilogue runs beside them"},
        "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
    }
    h.close()
    print(json.dumps(line))


def learned_conv_flops(nx: int, ny: int, nz: int, block: int = 4) -> float:
    """Algorithmic FLOPs of the learned form's convolutions for one atlas, over the outputs the
    restricted plan computes: conv4 on the anchor rows of the row blocks, conv(4 - r) within r
    rows and planes of them, conv1 over the box 3 rows and planes around the anchors (y within
    3 of the interior); 2 * 16 output channels * (16 * 27 or 2 * 27) MACs per output voxel."""
    def anchors(extent):
        return [6 + min(b * block + block // 2, extent - 1) for b in range(-(-extent // block))]

    az, ax = anchors(nz - 12), anchors(nx - 12)
    flop = 0.0
    for r in (2, 1, 0):  # conv2, conv3, conv4
        zs = {a + d for a in az for d in range(-r, r + 1)}
        xs = {a + d for a in ax for d in range(-r, r + 1)}
        flop += len(zs) * len(xs) * (ny - 12 + 2 * r) * 2.0 * 16 * 16 * 27
    c1 = (az[-1] - az[0] + 7) * (ax[-1] - ax[0] + 7) * (ny - 6)
    return flop + c1 * 2.0 * 16 * 2 * 27


def run_learned_arm(args) -> None:
    """Config 4: the learned-proposal form (EXEC_CHOICE 7, the committed trained network) on a
    held-out 222x222x112 subject with 10 atlases, NH = 11, against the plain FP32 kernel on the
    same inputs in the same run: voxels/s of both, the speed-up, and the learned form's error
    against the plain method in HU."""
    import torch

    import pseudoctimaging_b200 as pct
    from pseudoctimaging_b200 import learned

    dev = torch.device("cuda", 0)
    s = pct.synth_subject(NX, NY, NZ, NUM, n_blobs=N_BLOBS, seed=5000)  # held out from training
    label = pct.normalize_labels(s.atlas_ct)
    div = pct.div_from(SIGMA, BETA)
    d = [torch.from_numpy(x).to(dev) for x in (s.img, s.atlas_mri, label)]
    o_plain, o_learn = torch.zeros_like(d[0]), torch.zeros_like(d[0])
    h = pct.Handle(0)
    model = learned.LearnedModel.load(learned.CHECKPOINT)
    h.attach_model(model, args.conf)
    h.set_learned_k(args.k)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def timed(choice, out, steps, warmup):
        def step():
            h.synthesize_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), out.data_ptr(),
                                NX, NY, NZ, NUM, 11, div, choice, stream.cuda_stream)
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        h.device_status(stream.cuda_stream)
        return e0.elapsed_time(e1) / steps

    ms_plain = timed(pct.EXEC_B200_FP32, o_plain, max(1, args.steps // 2), 1)
    with ClockSampler(0) as clk:
        ms = timed(pct.EXEC_LEARNED, o_learn, args.steps, args.warmup)
    st = h.learned_stats()
    core = (slice(6, -6),) * 3
    check = Fp64Check(s.img, s.atlas_mri, label, 11, div)
    vol_learn, vol_plain = o_learn.cpu().numpy(), o_plain.cpu().numpy()
    a = vol_learn[core].astype(np.float64)
    b = vol_plain[core].astype(np.float64)
    both = np.isfinite(a) & np.isfinite(b)
    err = np.abs(a[both] - b[both]) * (4095.0 / 255.0)
    nvox = NX * NY * NZ
    pairs = (NZ - 12) * (NX - 12) * (NY - 12) * NUM
    rows = (NZ - 12) * (NX - 12) * -(-(NY - 12) // 30) * NUM
    # tensor work of the convolutions over the outputs the restricted plan computes
    conv_flop = learned_conv_flops(NX, NY, NZ) * NUM
    peaks = measured_peaks()
    bf16 = peaks.get("bf16_tflops")
    clocks = clk.summary()
    line = {
        "metric": f"pseudo-CT voxels/s at {NX}x{NY}x{NZ}, 10 atlases, NH=11, learned proposal "
                  "(EXEC_CHOICE 7)",
        "value": nvox / (ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 network, f32 rescoring",
        "data": "synthetic (seeded generator, config 4 held-out subject, seed 5000)",
        "config": {"workload": f"config 4: learned proposal, k = {args.k} per row segment",
                   "checkpoint": learned.CHECKPOINT.name, "conf_threshold": args.conf,
                   "volume": [NX, NY, NZ], "atlases": NUM, "nh": 11},
        "plain": {"ms_per_step": ms_plain, "value": nvox / (ms_plain / 1e3),
                  **check.errors(vol_plain)},
        "speedup_vs_plain": ms_plain / ms,
        "quality_vs_plain": {"mae_hu": float(err.mean()), "max_abs_hu": float(err.max()),
                             "nan_mismatch": int((np.isnan(a) != np.isnan(b)).sum())},
        "quality_vs_fp64": check.errors(vol_learn),
        "fallback_share": st["fallback_pairs"] / pairs,
        "offsets_per_row": st["row_offsets"] / rows,
        "gpu_launches": args.steps * (7 + 6 * NUM + 1),
        "roofline": {"bound": "tensor", "unit": "TFLOP/s",
                     "achieved": conv_flop / (ms / 1e3) / 1e12, "peak": bf16,
                     "frac": (conv_flop / (ms / 1e3) / 1e12 / bf16) if bf16 else None,
                     "traffic": None,
                     "note": "algorithmic convolution FLOPs (conv1..conv4 over the outputs the "
                             "anchor rows need) over the whole step, which also holds the "
                             "proposal and the rescoring"},
        "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
    }
    h.attach_model(None)
    model.close()
    h.close()
    print(json.dumps(line))


def spawn_ranks(n: int) -> int:
    """Re-runs this command as n ranks under torch.distributed.run (one process per GPU) when
    --gpus asks for more than one GPU and no launcher started us; returns its exit code."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = ["timeout", "-k", "60", "1800", sys.executable, "-m", "torch.distributed.run",
           "--nnodes=1", f"--nproc-per-node={n}", "--master-addr", "127.0.0.1",
           "--master-port", str(port), str(pathlib.Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def run_dry_arm(args) -> None:
    """The launcher and rank logic without a GPU: every rank joins a gloo group, takes the same
    barrier and max-reduction as the timed arms, and rank 0 prints n_gpus and the ranks seen."""
    import datetime

    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        dist.barrier()
    t = torch.tensor([float(rank)], dtype=torch.float64)
    ranks = torch.zeros(world, dtype=torch.float64)
    ranks[rank] = 1.0
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(ranks, op=dist.ReduceOp.SUM)
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"dry": True, "n_gpus": world, "gpus_requested": args.gpus,
                          "max_rank": int(t.item()), "ranks_seen": int(ranks.sum().item())}))


def main() -> None:
    global NZ, NH, METRIC
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["single", "batch", "learned", "sharded", "tc"],
                    default="single",
                    help="single: config 1 subject (the metric); batch: config 3 subjects; "
                         "learned: config 4, the learned proposal against the plain kernel; "
                         "sharded: one config 1 subject split into z slabs over the GPUs; "
                         "tc: config 2, the tensor-core form against the plain kernel")
    ap.add_argument("--conf", type=float, default=0.0,
                    help="learned workload: confidence threshold of the full-search fallback")
    ap.add_argument("--k", type=int, default=32, choices=[10, 20, 32],
                    help="learned workload: offsets rescored per proposal")
    ap.add_argument("--batch-subjects", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-pointer end-to-end leg")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip timing the learned and tensor-core forms beside the plain kernel")
    ap.add_argument("--nh", type=int, default=NH, choices=[3, 5, 7, 9, 11],
                    help="search window (default 11, the metric's; 7 and 9 are config-1 sweeps)")
    ap.add_argument("--nz", type=int, default=NZ,
                    help="z extent of the subject (default 112; smaller only for profiling runs)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="CPU-baseline sample length (rank 0, N=1 only)")
    ap.add_argument("--ref-step-seconds", type=float, default=4.0,
                    help="length of each reference-arm step")
    ap.add_argument("--tile-set", type=int, default=None,
                    help="single workload: the plain kernel's register-tile set (default: the "
                         "handle's, set 0)")
    ap.add_argument("--dry", action="store_true",
                    help="launcher and rank logic only (gloo, no GPU work)")
    args = ap.parse_args()
    if args.gpus < 1:
        ap.error("--gpus must be at least 1")
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(spawn_ranks(args.gpus))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but {world} rank(s) were launched")
    NZ = args.nz
    NH = args.nh
    METRIC = f"pseudo-CT voxels/s at {NX}x{NY}x{NZ}, 10 atlases, NH={NH}"
    if args.dry:
        run_dry_arm(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "batch":
        run_batch_arm(args)
    elif args.workload == "learned":
        run_learned_arm(args)
    elif args.workload == "sharded":
        run_sharded_arm(args)
    elif args.workload == "tc":
        run_tc_arm(args)
    else:
        run_b200_arm(args)


if __name__ == "__main__":
    main()
