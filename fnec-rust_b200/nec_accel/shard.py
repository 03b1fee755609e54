"""Sharding of independent Hallen solve units across GPUs (one process per GPU).

The reference solves the frequencies of a sweep independently and, in its
hybrid mode, spreads them over host threads with rayon
(apps/nec-cli/src/solve_session.rs:1794-1815); its worker solves each
(deck, config, frequency) request on its own.  Units -- (antenna, frequency,
right-hand side) tuples -- never exchange data, so a job of many antennas is
split across ranks with no collective on the data path: each rank plans and
solves its own sub-batch, and the small per-unit results (feedpoint rows and
currents, a few KB per solve) are gathered on the host of rank 0 in the job's
unit order.

`partition` is a greedy longest-processing-time split: antennas are taken
largest estimated cost first and each goes to the rank with the least cost so
far (ties to the lower rank), which keeps every rank within one antenna's cost
of the mean.  Costs come from the work model of the solve (Z fill samples,
Gram, factor, refinement) computed from the deck on the host, so the split
needs no device.  `gather_units` collects per-unit results on rank 0 over any
torch.distributed process group (gloo on the host, or NCCL).
"""
from __future__ import annotations

from typing import Any, List, Sequence

import numpy as np


def antenna_sizes(antenna) -> tuple:
    """(N segments, S unknowns upper bound, frequencies, right-hand sides,
    pattern points, ground) of an Antenna, from its cards alone.  S counts
    one homogeneous column per GW card (the most the solve can have before
    collinear merging or path grouping lowers it)."""
    wires = antenna.wires
    n = int(np.sum(wires["segments"])) if len(wires) else 0
    s = n + len(wires)
    nf = len(antenna.freqs_hz)
    n_rhs = max(len(antenna.sources), 1) if antenna.separate_sources else 1
    if antenna.rp_points is not None:
        pts = len(antenna.rp_points)
    elif antenna.rp is not None:
        pts = int(antenna.rp[0]) * int(antenna.rp[1])
    else:
        pts = 0
    return n, s, nf, n_rhs, pts, int(antenna.ground)


def unit_cost(n: int, s: int, n_freq: int = 1, n_rhs: int = 1, n_points: int = 0, ground: int = 0,
              mixed: bool = True) -> float:
    """Estimated work of one antenna's solves in real flops: 60 per Z
    sample (8 N^2, twice over a PEC ground), the Gram 8 N^3, the factor
    (8/3) S^3, the refinement or substitution (about 6 operator passes of
    16 N^2 in the mixed form; 8 S^2 per right-hand side in the plain one)
    and the far field 8 N per direction (the power grid of 64,800 or
    32,760 directions plus the requested points)."""
    fill = 60.0 * 8.0 * n * n * (2 if ground == 1 else 1)
    gram = 8.0 * n ** 3
    factor = 8.0 * s ** 3 / 3.0
    solve = n_rhs * (6 * 16.0 * n * n if mixed else 8.0 * s * s)
    ff = 0.0
    if n_points:
        ff = n_rhs * 8.0 * n * (n_points + (32760 if ground == 1 else 64800))
    return float(n_freq * (fill + gram + factor + solve + ff))


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Split unit indices over `world` ranks, largest cost first onto the
    least-loaded rank (ties: lower rank, then lower index).  Each rank's list
    is returned in ascending index order, so a rank's results come back in
    the job's order.  Every index appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.asarray(costs, np.float64)
    order = sorted(range(len(c)), key=lambda i: (-c[i], i))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(c[i])
    return [sorted(p) for p in parts]


def partition_antennas(antennas: Sequence[Any], world: int, mixed: bool = True) -> List[List[int]]:
    """`partition` of a list of Antenna by the work model."""
    costs = []
    for a in antennas:
        n, s, nf, nr, pts, g = antenna_sizes(a)
        costs.append(unit_cost(n, s, nf, nr, pts, g, mixed))
    return partition(costs, world)


def loads(costs: Sequence[float], parts: Sequence[Sequence[int]]) -> List[float]:
    c = np.asarray(costs, np.float64)
    return [float(c[list(p)].sum()) if len(p) else 0.0 for p in parts]


def gather_units(local: Sequence[Any], index: Sequence[int], n_total: int, group=None, dst: int = 0):
    """Gather per-unit results on rank `dst`.  Every rank passes its results
    `local[k]` for job units `index[k]`; rank `dst` returns the list of all
    n_total results in job order (other ranks return None).  A unit that no
    rank returned, or that two ranks returned, raises ValueError."""
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    payload = (list(index), list(local))
    got = [None] * world if rank == dst else None
    dist.gather_object(payload, got, dst=dst, group=group)
    if rank != dst:
        return None
    out: List[Any] = [None] * n_total
    seen = np.zeros(n_total, np.int64)
    for idx, vals in got:
        if len(idx) != len(vals):
            raise ValueError("a rank returned a different number of indices and results")
        for i, v in zip(idx, vals):
            if not 0 <= i < n_total:
                raise ValueError(f"unit index {i} outside the job of {n_total}")
            seen[i] += 1
            out[i] = v
    if np.any(seen != 1):
        bad = np.nonzero(seen != 1)[0][:8].tolist()
        raise ValueError(f"units not gathered exactly once: {bad}")
    return out
