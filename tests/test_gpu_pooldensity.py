"""GPU parity of the transition-density pool gradient (bsim_pooldensity_*) against the
reference's batch_tran outputs (golden) and the pair-list batch gradient, and of
bsim_batchgrad's theta = 0 route through it (every theta zero, decided on the
device) against the oracle's batch gradient (op/batchgrad.hpp:529-540)."""
import numpy as np
import pytest

from binsim_b200 import cuotf, network as nw
from conftest import dev, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["h6_3a3b", "h8_4a4b"])
def test_pooldensity_matches_golden_trans_pool(cuda, case):
    z, _, pool = load_golden(case)
    B = cuotf.CuBasis(int(z["norb"]), int(z["na"]), int(z["nb"]))
    pd = cuotf.PoolDensity(B, pool)
    x, y = dev(cuda, z["x"]), dev(cuda, z["y"])
    g = cuda.empty(pool.ngs, dtype=cuda.float64, device="cuda")
    for _ in range(2):   # the tables are cleared on every call
        pd.grad(x, y, g)
        cuda.cuda.synchronize()
        ref = z["trans_pool"]
        assert np.abs(g.cpu().numpy() - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("norb,na,nb,bits", [(10, 4, 3, 32), (12, 3, 3, 64), (28, 2, 2, 64)])
def test_pooldensity_matches_batchgrad(cuda, norb, na, nb, bits):
    pool = nw.ucc_pool(norb, native=True)
    B = cuotf.CuBasis(norb, na, nb, string_bits=bits)
    net = cuotf.CuNetwork(pool.network, string_bits=bits)
    f = cuotf.CuOTFFunctions(B, net, net)
    rng = np.random.default_rng(norb)
    l, r = dev(cuda, rng.normal(size=B.dim)), dev(cuda, rng.normal(size=B.dim))
    ref = cuda.empty(pool.network.ngs, dtype=cuda.float64, device="cuda")
    f.batchgrad(l, r, ref, cuda.zeros_like(ref))
    pd = cuotf.PoolDensity(B, pool.network)
    g = cuda.empty_like(ref)
    pd.grad(l, r, g)
    cuda.cuda.synchronize()
    a, b = g.cpu().numpy(), ref.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_pooldensity_on_symmetry_blocks(cuda):
    """A blocked basis runs in the dense array over all alpha and beta strings."""
    norb, orbsym = 8, [0, 1, 2, 3, 0, 1, 2, 3]
    pool = nw.ucc_pool(norb)
    pool.network.orbsym = np.asarray(orbsym, np.int64)
    B = cuotf.CuBasis(norb, 4, 3, orbsym=orbsym, total_sym=1, num_irreps=4)
    net = cuotf.CuNetwork(pool.network)
    f = cuotf.CuOTFFunctions(B, net, net)
    rng = np.random.default_rng(5)
    l, r = dev(cuda, rng.normal(size=B.dim)), dev(cuda, rng.normal(size=B.dim))
    ref = cuda.empty(pool.network.ngs, dtype=cuda.float64, device="cuda")
    f.batchgrad(l, r, ref, cuda.zeros_like(ref))
    g = cuda.empty_like(ref)
    pd = cuotf.PoolDensity(B, pool.network)   # held until the kernels have finished
    pd.grad(l, r, g)
    cuda.cuda.synchronize()
    a, b = g.cpu().numpy(), ref.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def _mixed_network(norb, seed):
    """Pool groups with Hamiltonian groups between them: the Hamiltonian's groups
    match no single excitation, so one batchgrad call runs both the density route
    and the pair lists."""
    pool = nw.ucc_pool(norb).network
    ham = nw.hamiltonian_network(norb, seed=seed)
    groups, hams = [], list(range(0, ham.ngs, 5))
    for g in range(pool.ngs):
        groups.append(pool.group(g))
        if g % 7 == 0 and hams:
            groups.append(ham.group(hams.pop()))
    return nw._pack(groups, norb)


@pytest.mark.parametrize("orbsym,tsym", [(None, 0), ([0, 1, 0, 1, 0, 1, 0, 1], 1)])
def test_batchgrad_route_matches_oracle(cuda, oracle, orbsym, tsym):
    """theta = 0: planned groups through the densities, the rest through the pair
    lists (single block) or the tile kernel (symmetry blocks); then one nonzero
    theta, which sends every group to the general kernels; then theta = 0 again."""
    norb, na, nb = 8, 4, 3
    net = _mixed_network(norb, 2)
    if orbsym is not None:
        net.orbsym = np.asarray(orbsym, np.int64)
    kind, _, _ = cuotf.pool_plan(net)
    assert (kind < 0).any() and (kind > 0).any()
    Bo = oracle.basis(norb, na, nb, orbsym=orbsym, total_sym=tsym, num_irreps=2 if orbsym else 16)
    No = oracle.network(net)
    B = cuotf.CuBasis(norb, na, nb, orbsym=orbsym, total_sym=tsym, num_irreps=2 if orbsym else 16)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net), cuotf.CuNetwork(net))
    rng = np.random.default_rng(11)
    l, r = rng.normal(size=B.dim), rng.normal(size=B.dim)
    th = np.zeros(net.ngs)
    th1 = th.copy()
    th1[net.ngs // 2] = 0.3
    g = cuda.empty(net.ngs, dtype=cuda.float64, device="cuda")
    for t in (th, th1, th):
        f.batchgrad(dev(cuda, l), dev(cuda, r), g, dev(cuda, t))
        ref = oracle.batchgrad(Bo, No, t, l, r)
        assert np.abs(g.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
