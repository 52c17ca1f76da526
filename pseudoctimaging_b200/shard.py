"""Z-slab sharding of one subject over ranks (one process per GPU) or over passes on one GPU.

Every interior voxel is independent, so the path shards without a data-path collective: the
interior z planes are split into contiguous slabs (``pct_slab_plan``); each part copies its slab
plus ``hw + 1`` halo planes of the input MRI and of every atlas MRI and CT into its own device
memory and runs the ordinary synthesis on that sub-volume, whose interior is exactly the slab.
The outputs are disjoint. ``synthesize_sharded`` assembles the whole volume on every rank with one
all-gather (NCCL between GPUs, gloo between CPU processes); the reference has no counterpart (it
runs one subject on one device).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import EXEC_B200_FP32, PctError, lib


@dataclass(frozen=True)
class Slab:
    part: int
    z_begin: int    # first output plane of this part (global index)
    z_end: int      # one past the last output plane
    src_begin: int  # first input plane this part needs
    src_end: int

    @property
    def planes(self) -> int:
        return self.z_end - self.z_begin

    @property
    def src_planes(self) -> int:
        return self.src_end - self.src_begin


def slab_plan(nz: int, nh: int, parts: int) -> list[Slab]:
    if parts < 1:
        raise PctError(-1, f"slab_plan: parts must be >= 1, got {parts}")
    out = []
    for p in range(parts):
        v = [ctypes.c_int() for _ in range(4)]
        st = lib.pct_slab_plan(nz, nh, parts, p, *[ctypes.byref(x) for x in v])
        if st != 0:
            raise PctError(st, f"pct_slab_plan(nz={nz}, nh={nh}, parts={parts}, part={p})")
        out.append(Slab(p, *(x.value for x in v)))
    return out


def extract(img: np.ndarray, atlas: np.ndarray, label: np.ndarray, slab: Slab):
    """The sub-volume a part needs, as contiguous arrays [nz'][nx][ny] / [num][nz'][nx][ny]."""
    sl = slice(slab.src_begin, slab.src_end)
    return (np.ascontiguousarray(img[sl]), np.ascontiguousarray(atlas[:, sl]),
            np.ascontiguousarray(label[:, sl]))


def slab_planes(sub_out: np.ndarray, slab: Slab) -> np.ndarray:
    """The slab's own output planes out of the sub-volume's result."""
    o = slab.z_begin - slab.src_begin
    return sub_out[o:o + slab.planes]


def _cuda_compute(handle, nh: int, div: float, exec_choice: int):
    def compute(img, atlas, label):
        return handle.synthesize(img, atlas, label, nh, div, exec_choice)
    return compute


def synthesize_part(img, atlas, label, nh: int, div: float, slab: Slab, compute=None, handle=None,
                    exec_choice: int = EXEC_B200_FP32) -> np.ndarray:
    """Output planes [slab.z_begin, slab.z_end) of the subject. ``compute(img, atlas, label)``
    maps a sub-volume to its fused result; by default the CUDA path on ``handle``."""
    if slab.planes == 0:
        return np.zeros((0,) + img.shape[1:], np.float32)
    if compute is None:
        if handle is None:
            from . import default_handle
            handle = default_handle()
        compute = _cuda_compute(handle, nh, div, exec_choice)
    return slab_planes(compute(*extract(img, atlas, label, slab)), slab)


def synthesize_sharded(img, atlas, label, nh: int, div: float, exec_choice: int = EXEC_B200_FP32,
                       compute=None, handle=None, group=None) -> np.ndarray:
    """The whole fused volume on every rank of ``group`` (torch.distributed), each rank computing
    one z slab. Without an initialised process group this is one part on this process."""
    import torch
    import torch.distributed as dist

    img = np.ascontiguousarray(img, np.float32)
    atlas = np.ascontiguousarray(atlas, np.float32)
    label = np.ascontiguousarray(label, np.float32)
    if atlas.ndim == 3:
        atlas, label = atlas[None], label[None]
    nz, nx, ny = img.shape
    ranked = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if ranked else 0
    world = dist.get_world_size(group) if ranked else 1
    plan = slab_plan(nz, nh, world)
    mine = synthesize_part(img, atlas, label, nh, div, plan[rank], compute, handle, exec_choice)
    out = np.zeros_like(img)
    if world == 1:
        out[plan[0].z_begin:plan[0].z_end] = mine
        return out
    # one all-gather of equally padded slabs; the plan tells each rank where the others' go
    biggest = max(s.planes for s in plan)
    dev = (torch.device("cuda", torch.cuda.current_device())
           if dist.get_backend(group) == "nccl" else torch.device("cpu"))
    buf = torch.zeros((biggest, nx, ny), dtype=torch.float32, device=dev)
    if mine.shape[0]:
        buf[:mine.shape[0]] = torch.from_numpy(np.ascontiguousarray(mine)).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    for s, t in zip(plan, parts):
        if s.planes:
            out[s.z_begin:s.z_end] = t[:s.planes].cpu().numpy()
    return out
