"""Column-band sharding of sigma over ranks (one process per GPU).

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
