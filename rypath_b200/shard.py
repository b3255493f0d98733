"""Splitting one progressive render across ranks (one process per GPU) and merging their films.

The render shards by independent lanes: every (pixel, absolute sample) lane of a film is
computed from its own indices alone (begin_sample, shaders/render.metal:2424-2469), so ranks
that render disjoint ranges of absolute sample indices of the same film need no exchange while
they render.  Their films merge by adding the FP64 accumulators and counts pixel by pixel, the
fold rypath's progressive driver applies batch by batch (PacketFilmBatch, src/packet_film.cpp:
198-265; render_progressive, src/render_driver.cpp:287-316).

``merge_film`` is the one collective: an all-gather of the ranks' films over
torch.distributed (NCCL between GPUs, gloo on CPU), then, on every rank, a compensated sum of
the films in rank order, so the merged film is the same on every rank and does not depend on
the order a reduction tree would add them in.
"""

from __future__ import annotations

import numpy as np

from . import abi


def sample_range(sample_count: int, rank: int, world: int, sample_begin: int = 0) -> tuple[int, int]:
    """The rank's contiguous share ``(begin, count)`` of samples [sample_begin, sample_begin + sample_count).

    Shares differ by at most one sample; lower ranks take the remainder."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if sample_count < 0 or sample_begin < 0:
        raise ValueError("sample ranges are nonnegative")
    base, extra = divmod(sample_count, world)
    begin = sample_begin + rank * base + min(rank, extra)
    return begin, base + (1 if rank < extra else 0)


def _two_sum(a: np.ndarray, b: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Knuth's TwoSum: s + e == a + b exactly, s = fl(a + b)."""
    s = a + b
    bb = s - a
    e = (a - (s - bb)) + (b - bb)
    return s, e


def add_films(films: list[np.ndarray]) -> np.ndarray:
    """Sum of films (rp_film_pixel rows) in list order.

    Each compensated pair (sum, correction) and (weight_sum, weight_correction) is added with
    TwoSum, its rounding error folded into the correction; second moments and counts add
    plainly."""
    if not films:
        raise ValueError("no films to add")
    out = films[0].copy()
    for f in films[1:]:
        if f.shape != out.shape or f.dtype != out.dtype:
            raise ValueError("films differ in size or layout")
        for value, corr in (("sum", "correction"), ("weight_sum", "weight_correction")):
            s, e = _two_sum(out[value], f[value])
            out[value] = s
            out[corr] = out[corr] + f[corr] + e
        out["square"] = out["square"] + f["square"]
        out["count"] = out["count"] + f["count"]
    return out


def merge_film(film: np.ndarray, group=None) -> np.ndarray:
    """All ranks' films added in rank order (``add_films``), returned on every rank.

    ``film`` is this rank's host film (rp_film_pixel rows, ``abi.film_dtype()``).  The films
    travel as bytes: a CUDA tensor when the group's backend is NCCL, a CPU tensor otherwise."""
    import torch
    import torch.distributed as dist

    film = np.ascontiguousarray(film)
    if film.dtype != abi.film_dtype():
        raise ValueError("merge_film takes rp_film_pixel rows")
    world = dist.get_world_size(group)
    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    mine = torch.from_numpy(film.view(np.uint8).reshape(-1)).to(device)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    films = [p.cpu().numpy().view(abi.film_dtype()) for p in parts]
    return add_films(films)
