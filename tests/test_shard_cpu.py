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


def test_group_ranges_cover_once_and_balance():
    from binsim_b200.shard import group_ranges
    rng = np.random.default_rng(0)
    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            costs = rng.integers(1, 50, size=n)
            rs = group_ranges(costs, world)
            assert len(rs) == world and rs[0][0] == 0 and rs[-1][1] == n
            assert all(rs[i][1] == rs[i + 1][0] for i in range(world - 1))
            if n >= world:
                loads = [costs[lo:hi].sum() for lo, hi in rs]
                assert max(loads) - min(loads) <= 2 * costs.max()


def test_group_range_subnetwork_acts_like_the_slice(oracle):
    from binsim_b200 import network as nw
    norb = 6
    pool = nw.ucc_pool(norb).network
    B = oracle.basis(norb, 3, 3)
    N = oracle.network(pool)
    lo, hi = 101, 173
    S = oracle.network(nw.group_range(pool, lo, hi))
    v = np.random.default_rng(2).normal(size=B.dim)
    for g in (0, 17, hi - lo - 1):
        assert np.array_equal(oracle.expm(B, S, g, 0.3, v), oracle.expm(B, N, lo + g, 0.3, v))


def _pool_worker(rank, world, port, norb, na, nb, outdir):
    import torch
    import torch.distributed as dist
    from binsim_b200 import network as nw
    from binsim_b200.shard import PoolShardedGradient
    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        O = Oracle()
        Bo = O.basis(norb, na, nb)
        pool = nw.ucc_pool(norb).network
        rng = np.random.default_rng(4)
        psi, hpsi = rng.normal(size=Bo.dim), rng.normal(size=Bo.dim)   # the same state on every rank
        ref = O.batchgrad(Bo, O.network(pool), np.zeros(pool.ngs), psi, hpsi)
        calls = []

        def compute(lo, hi, out):
            calls.append((lo, hi))
            sub = O.network(nw.group_range(pool, lo, hi))
            out.copy_(torch.from_numpy(O.batchgrad(Bo, sub, np.zeros(hi - lo), psi, hpsi)))
        costs = np.asarray(pool.num_zas) + np.asarray(pool.num_zbs)   # any positive work estimate
        S = PoolShardedGradient(compute, pool.ngs, costs=costs)
        g = torch.full((pool.ngs,), float("nan"), dtype=torch.float64)
        S(g)
        # the oracle's OpenMP reductions round in thread order: equal to 1e-12 relative
        ok = bool(np.abs(g.numpy() - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()))
        np.save(os.path.join(outdir, f"pool{rank}.npy"),
                np.array([ok, calls == [S.range] if S.range[1] > S.range[0] else calls == []], dtype=np.float64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_pool_gradient_gloo_matches_oracle(tmp_path, world):
    """The pool gradient split by ranges of pool groups over world ranks (gloo), every
    rank ending with the whole gradient vector, equal to the unsplit oracle."""
    import torch.multiprocessing as mp
    mp.spawn(_pool_worker, args=(world, _free_port(), 6, 3, 3, str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        ok, own_only = np.load(tmp_path / f"pool{r}.npy")
        assert ok == 1.0, f"rank {r}: gathered pool gradient differs from the oracle"
        assert own_only == 1.0, f"rank {r}: computed outside its range"
