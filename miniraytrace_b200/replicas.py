"""Sample-striped replicas: one process per GPU renders a disjoint share of
the samples of the same frame, and the FP64 accumulation buffers are summed.

The reference renders on one device, sample k of a pixel with the random
stream of frame index k (pathtrace.comp:105). With N ranks, rank r renders
its s-th sample with frame index ``s * N + r`` (``Engine.set_sample_stream(r,
N)``), so the union of all ranks' samples is exactly the single-device sample
set; the accumulation layout (r, g, b sums and the sample count per pixel,
FP64) adds across ranks without any rescaling. The combine is one reduce of
that buffer per step; there is no other data exchange.
"""
from __future__ import annotations


def sample_stream(rank: int, world: int) -> tuple[int, int]:
    """(offset, stride) of rank's sample stream for Engine.set_sample_stream."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return rank, world


def frames_of(rank: int, world: int, first_sample: int, count: int) -> list[int]:
    """Frame indices of samples first_sample .. first_sample + count - 1 of
    rank's stream (the kernels' frame index: offset + sample * stride)."""
    offset, stride = sample_stream(rank, world)
    return [offset + s * stride for s in range(first_sample, first_sample + count)]


def combine_accumulation(buf, dist, dst: int = 0):
    """Sums every rank's FP64 accumulation tensor (H, W, 4) into rank dst's.
    Every rank must call it at the same point of its step sequence."""
    dist.reduce(buf, dst=dst)
    return buf


def max_over_ranks(value: float, dist, device) -> float:
    """The largest of the ranks' values (step times are reported as the
    slowest rank's); returns value unchanged without a process group."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
