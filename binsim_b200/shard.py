"""Sharding over ranks (one process per GPU): sigma by column bands, the pool
gradient by ranges of pool groups.

sigma = H c is split by beta columns: rank r computes sigma[:, lo_r:hi_r] for
every alpha row (``bsim_hvec_cols``), then the bands are exchanged so that every
rank holds the whole sigma.  The exchange is needed because the next operator
application (the next Davidson expansion vector, the next VQE step) reads all of
its input: the source determinants of any destination column lie in every
column.  The exchange is one all-gather of equal-size packed bands over the
process group — NCCL over NVLink on GPUs, gloo on CPU.

Column bands (rather than alpha-row bands) keep every stage of the structured
sigma local to the band: the pure-alpha row AXPYs, the mixed GEMM's column
chunks, the gather and the final combine all restrict to the band's columns,
and the pure-beta stage restricts to the band's rows of the transposed vector.
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Tuple


def column_bands(nb: int, world: int, align: int = 128) -> List[Tuple[int, int]]:
    """Contiguous bands [lo, hi) covering [0, nb) once, each start a multiple of
    `align`, sizes as equal as the alignment allows (trailing bands may be empty)."""
    if nb < 0 or world < 1 or align < 1:
        raise ValueError("need nb >= 0, world >= 1, align >= 1")
    nblk = math.ceil(nb / align)
    out = []
    for r in range(world):
        b0 = nblk * r // world
        b1 = nblk * (r + 1) // world
        out.append((min(nb, b0 * align), min(nb, b1 * align)))
    return out


class ColumnShardedSigma:
    """sigma over a process group, split by beta-column bands.

    compute(x, y, lo, hi) must write columns [lo, hi) of H x into y (a full-size
    vector, alpha-major: index a * nb + b) and leave the rest of y alone; on GPUs
    it is ``CuOTFFunctions.hvec_cols``.  After the call every rank holds the whole
    sigma in y."""

    def __init__(self, compute: Callable, na: int, nb: int, group=None, align: int = 128):
        import torch.distributed as dist
        self.compute = compute
        self.na, self.nb = na, nb
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.bands = column_bands(nb, self.world, align)
        self.width = max(hi - lo for lo, hi in self.bands)
        self._send = None
        self._recv = None

    @property
    def band(self) -> Tuple[int, int]:
        return self.bands[self.rank]

    def exchange_bytes(self) -> int:
        """Bytes this rank receives per sigma (the all-gather of packed bands)."""
        return (self.world - 1) * self.na * self.width * 8

    def __call__(self, x, y, mixed: bool = False) -> None:
        import torch
        import torch.distributed as dist
        lo, hi = self.band
        if hi > lo:
            if mixed:
                self.compute(x, y, lo, hi, mixed=True)
            else:
                self.compute(x, y, lo, hi)
        if self.world == 1:
            return
        if self._send is None or self._send.device != y.device:
            self._send = torch.zeros((self.na, self.width), dtype=y.dtype, device=y.device)
            self._recv = [torch.empty_like(self._send) for _ in range(self.world)]
        y2 = y.view(self.na, self.nb)
        self._send[:, : hi - lo].copy_(y2[:, lo:hi])
        dist.all_gather(self._recv, self._send, group=self.group)
        for r, (l2, h2) in enumerate(self.bands):
            if r != self.rank and h2 > l2:
                y2[:, l2:h2].copy_(self._recv[r][:, : h2 - l2])


def group_ranges(costs, world: int) -> List[Tuple[int, int]]:
    """Contiguous ranges [lo, hi) of groups covering [0, len(costs)) once, one per rank,
    cut where the running sum of `costs` (work per group, e.g. its connected pairs)
    crosses multiples of total / world."""
    import numpy as np
    if world < 1:
        raise ValueError("need world >= 1")
    c = np.asarray(costs, dtype=np.float64)
    n = len(c)
    cum = np.concatenate([[0.0], np.cumsum(c)])
    tot = cum[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum, tot * r / world, side="left")) if tot > 0 else n * r // world)
    cuts.append(n)
    cuts = [min(max(x, 0), n) for x in cuts]
    for i in range(1, len(cuts)):   # monotone
        cuts[i] = max(cuts[i], cuts[i - 1])
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


class PoolShardedGradient:
    """The pool gradient (ADAPT screening) over a process group: every rank holds the
    state and H psi and computes the gradients of its range of pool groups, then the
    ranges are all-gathered so that every rank holds all of them.  The pool work is
    independent per group, so the only exchange is the gradient vector itself.

    compute(lo, hi, out) must write the gradients of groups [lo, hi) into `out`
    (a length hi - lo vector); on GPUs it is ``CuOTFFunctions.batchgrad`` of the
    rank's ``network.group_range`` sub-network."""

    def __init__(self, compute: Callable, ngs: int, costs=None, group=None):
        import torch.distributed as dist
        self.compute = compute
        self.ngs = ngs
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.ranges = group_ranges([1.0] * ngs if costs is None else costs, self.world)
        self.width = max(1, max(hi - lo for lo, hi in self.ranges))
        self._send = None
        self._recv = None

    @property
    def range(self) -> Tuple[int, int]:
        return self.ranges[self.rank]

    def __call__(self, grads) -> None:
        import torch
        import torch.distributed as dist
        lo, hi = self.range
        if self._send is None or self._send.device != grads.device:
            self._send = torch.zeros(self.width, dtype=grads.dtype, device=grads.device)
            self._recv = [torch.empty_like(self._send) for _ in range(self.world)]
        if hi > lo:
            self.compute(lo, hi, self._send[: hi - lo])
        if self.world == 1:
            grads[lo:hi].copy_(self._send[: hi - lo])
            return
        dist.all_gather(self._recv, self._send, group=self.group)
        for r, (l2, h2) in enumerate(self.ranges):
            if h2 > l2:
                grads[l2:h2].copy_(self._recv[r][: h2 - l2])
