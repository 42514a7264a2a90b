"""GPU parity of the transition-density pool gradient (bsim_pooldensity_*) against the
reference's batch_tran outputs (golden) and the pair-list batch gradient.

Opt-in: these kernels have not yet run on a GPU, so the tests run only with
BSIM_TEST_POOLDENSITY=1 until they have passed once."""
import os

import numpy as np
import pytest

from binsim_b200 import cuotf, network as nw
from conftest import dev, load_golden

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("BSIM_TEST_POOLDENSITY") != "1",
                                 reason="density kernels not yet run on a GPU: set BSIM_TEST_POOLDENSITY=1")]


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
