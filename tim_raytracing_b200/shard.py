"""Splitting one trace job across GPUs (one process per GPU).

Rays are independent, so a job shards without any exchange during tracing:
every rank holds its own copy of the scene (uploaded to its own GPU) and traces
a contiguous range of the job's units -- rays of a batch, output rows of a
frame, probes of a field -- and the results are put back together in input
order afterwards, only where a single consumer wants them in one place. For
serving, scenes instead have an affinity rank: each resident scene lives on one
GPU and every job on it is routed there.

The reference renders on one device only (one Vulkan queue, single render
thread, src/rtDevice/private/RenderContext.cpp:23-31); its unit of work is one
independent ray per shader invocation (src/Shaders/cameraPass.comp:43-56,
src/Shaders/genLightProbField.comp:41-50), which is what makes these splits
exact: the reassembled records equal those of one GPU tracing everything.

The process group is the caller's (torch.distributed, NCCL between GPUs, gloo
on the host); the reassembly is one all-gather of equal-sized padded slices.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np

# Frame rows are split on the 8x4-pixel tile rows of the camera kernels.
ROW_ALIGN = 4


def contiguous_ranges(n: int, parts: int, align: int = 1, weights: Sequence[float] | None = None) -> list:
    """Splits [0, n) into `parts` contiguous ranges [b, e) in order, each boundary
    a multiple of `align` (the last range ends at n). Without weights the ranges
    hold equal numbers of units (up to the alignment); with per-unit weights
    (an estimate of each unit's cost, e.g. rays per frame row) the boundaries sit
    where the cumulative weight crosses k/parts of the total, so that every rank
    gets about the same work. Ranges may be empty when n is small."""
    if parts < 1 or align < 1 or n < 0:
        raise ValueError("contiguous_ranges: parts and align must be >= 1 and n >= 0")
    if weights is not None:
        w = np.asarray(weights, np.float64)
        if w.shape != (n,) or np.any(w < 0) or not np.all(np.isfinite(w)):
            raise ValueError("contiguous_ranges: weights must be n finite non-negative values")
        cum = np.concatenate([[0.0], np.cumsum(w)])
        total = cum[-1]
    cuts = [0]
    for k in range(1, parts):
        if weights is not None and total > 0:
            target = total * k / parts
            c = int(np.searchsorted(cum, target, side="left"))   # first prefix reaching the target
            # pick the nearer of the two unit boundaries around the target
            if c > 0 and target - cum[c - 1] < cum[min(c, n)] - target:
                c -= 1
        else:
            c = (n * k) // parts
        c = int(round(c / align)) * align
        c = min(max(c, cuts[-1]), n)
        cuts.append(c)
    cuts.append(n)
    return [(cuts[k], cuts[k + 1]) for k in range(parts)]


def row_bands(height: int, parts: int, weights: Sequence[float] | None = None) -> list:
    """Contiguous bands of output rows [b, e) for `parts` ranks, boundaries on the
    camera kernels' 4-row tile boundaries; optional per-row cost weights."""
    return contiguous_ranges(height, parts, ROW_ALIGN, weights)


def frame_row_weights(records: np.ndarray, width: int, height: int, tile_counts=None, tile: int = 16,
                      bounce: bool = True) -> np.ndarray:
    """Per-row cost estimate of a camera frame from a previous frame's records
    (tracingData, [W*H, 8] u32): every traced pixel costs its primary ray, and a
    hit pixel also its secondary rays -- the sun ray, one ray per tile-culled light
    of its tile (or 1 without tile lists) and the bounce ray. Row 0 is never traced
    (cameraPass.comp:46) and weighs 0."""
    rec = np.asarray(records, np.uint32).reshape(height, width, 8)
    hit = rec[:, :, 3] != np.float32(100.0).view(np.uint32)
    sec = np.full((height, width), 1.0 + (1.0 if bounce else 0.0))
    if tile_counts is not None:
        tx = (width + tile - 1) // tile
        tc = np.asarray(tile_counts, np.float64).reshape(-1, tx)
        sec += np.repeat(np.repeat(tc, tile, axis=0), tile, axis=1)[:height, :width]
    else:
        sec += 1.0
    w = (1.0 + hit * sec).sum(axis=1)
    w[0] = 0.0
    return w


def gather_in_order(local, ranges: Sequence, group=None):
    """All-gathers each rank's slice (a torch tensor whose first dimension is its
    range's length, in the order of `ranges`) and returns the concatenation in
    input order on every rank. Slices are padded to the longest range, so one
    collective of equal sizes does it (NCCL on GPUs, gloo on the host)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if len(ranges) != world:
        raise ValueError("gather_in_order: one range per rank")
    longest = max(e - b for b, e in ranges)
    rank = dist.get_rank(group)
    b, e = ranges[rank]
    if local.shape[0] != e - b:
        raise ValueError(f"gather_in_order: rank {rank} holds {local.shape[0]} units, its range has {e - b}")
    pad = torch.zeros((longest,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: e - b] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([parts[k][: ranges[k][1] - ranges[k][0]] for k in range(world)], 0)


def trace_sharded(trace: Callable, n: int, group=None, weights=None, align: int = 1):
    """Runs `trace(begin, end)` on this rank's contiguous range of the n units
    of one job and returns (all results in input order, this rank's range).
    `trace` returns a torch tensor with one row per unit of [begin, end) -- a
    GPU trace of those rays or rows on this rank's device (or any stand-in
    with the same result, e.g. a host restatement in tests)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    ranges = contiguous_ranges(n, world, align, weights)
    b, e = ranges[rank]
    local = trace(b, e)
    return gather_in_order(local, ranges, group), ranges[rank]


class SceneRouter:
    """Scene affinity for serving on several GPUs: each resident scene is
    assigned to one rank -- largest device footprint first, each onto the rank
    with the least bytes so far (ties: the lower rank) -- and every job on a scene
    is routed to that scene's rank, where its BVH already sits. The assignment
    depends only on the scene sizes, so every rank computes the same one."""

    def __init__(self, scene_bytes: dict, world: int):
        if world < 1:
            raise ValueError("SceneRouter: world must be >= 1")
        self.world = world
        self.load = [0] * world
        self.rank_of_scene = {}
        for sid in sorted(scene_bytes, key=lambda s: (-int(scene_bytes[s]), s)):
            r = min(range(world), key=lambda k: (self.load[k], k))
            self.rank_of_scene[sid] = r
            self.load[r] += int(scene_bytes[sid])

    def rank_of(self, scene) -> int:
        try:
            return self.rank_of_scene[scene]
        except KeyError:
            raise KeyError(f"SceneRouter: scene {scene!r} is not resident") from None

    def scenes_of(self, rank: int) -> list:
        return sorted(s for s, r in self.rank_of_scene.items() if r == rank)

    def route(self, jobs: Sequence) -> list:
        """Splits jobs [(scene, ...), ...] into per-rank lists of job indices in
        submission order."""
        out = [[] for _ in range(self.world)]
        for j, job in enumerate(jobs):
            out[self.rank_of(job[0])].append(j)
        return out
