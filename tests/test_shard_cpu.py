"""Column-band sharding of sigma (the N > 1 path) on CPU: band arithmetic, and a
world-size-2 gloo run of the exchange with the oracle as the per-band compute."""
import math
import os
import socket
from datetime import timedelta

import numpy as np
import pytest


def test_column_bands_cover_once_and_align():
    from binsim_b200.shard import column_bands
    for nb in (0, 1, 35, 127, 128, 129, 3432, 12870, 43758):
        for world in (1, 2, 3, 4, 8):
            bands = column_bands(nb, world)
            assert len(bands) == world
            cover = np.zeros(nb, np.int64)
            prev = 0
            for lo, hi in bands:
                assert lo == prev and lo <= hi      # contiguous, in order
                assert lo % 128 == 0 or lo == nb    # every non-empty band starts aligned
                cover[lo:hi] += 1
                prev = hi
            assert prev == nb and (cover == 1).all()
            widths = [hi - lo for lo, hi in bands]
            assert max(widths) - min(widths) <= 2 * 128   # balanced to within the alignment (plus a ragged end)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, norb, na, nb, outdir):
    import torch
    import torch.distributed as dist
    from binsim_b200 import network as nw
    from binsim_b200.shard import ColumnShardedSigma
    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        O = Oracle()
        Bo = O.basis(norb, na, nb)
        No = O.network(nw.hamiltonian_network(norb, seed=5))
        nA, nB = math.comb(norb, na), math.comb(norb, nb)
        x = np.random.default_rng(3).normal(size=nA * nB)   # the same input on every rank
        ref = O.hvec(Bo, No, x)
        calls = []

        def compute(xt, yt, lo, hi):
            calls.append((lo, hi))
            full = O.hvec(Bo, No, xt.numpy()).reshape(nA, nB)
            yt.view(nA, nB)[:, lo:hi] = torch.from_numpy(np.ascontiguousarray(full[:, lo:hi]))

        S = ColumnShardedSigma(compute, nA, nB, align=8)
        y = torch.full((nA * nB,), float("nan"), dtype=torch.float64)
        S(torch.from_numpy(x), y)
        ok = bool(np.array_equal(y.numpy(), ref))
        np.save(os.path.join(outdir, f"rank{rank}.npy"),
                np.array([ok, calls == [S.band] if S.band[1] > S.band[0] else calls == [], S.exchange_bytes()],
                         dtype=np.float64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_sigma_gloo_matches_oracle(tmp_path, world):
    import torch.multiprocessing as mp
    norb, na, nb = 7, 3, 4          # 35 x 35 determinants: bands of 8 columns
    mp.spawn(_worker, args=(world, _free_port(), norb, na, nb, str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        ok, band_only, nbytes = np.load(tmp_path / f"rank{r}.npy")
        assert ok == 1.0, f"rank {r}: gathered sigma differs from the oracle"
        assert band_only == 1.0, f"rank {r}: computed outside its band"
        assert nbytes > 0
