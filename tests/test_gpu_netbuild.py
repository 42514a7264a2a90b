"""Device-side network construction (bsim_netbuild_compress_device): every group's
one-sided Jacobi SVD in one batched GPU launch gives the host builder's groups, Z
lists and ranks, the same group matrices M = wa wb^T (the compression of
jl/network.jl:158-301), and the same sigma / expm on the GPU.

Tolerances: group matrices 1e-12 absolute (the two builders rotate column pairs
in different orders); sigma 1e-12 x max|sigma|; expm 1e-13 absolute on a unit
vector."""
import numpy as np
import pytest

from conftest import dev

pytestmark = pytest.mark.gpu


def _same_network(a, b):
    for k in ("axs", "bxs", "ranks", "num_zas", "num_zbs", "flat_zas", "flat_zbs"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    oa = ob = 0
    for gi in range(a.ngs):
        na, nb, r = int(a.num_zas[gi]), int(a.num_zbs[gi]), int(a.ranks[gi])
        Ma = a.flat_wa[oa:oa + na * r].reshape(r, na).T @ a.flat_wb[ob:ob + nb * r].reshape(r, nb)
        Mb = b.flat_wa[oa:oa + na * r].reshape(r, na).T @ b.flat_wb[ob:ob + nb * r].reshape(r, nb)
        assert np.abs(Ma - Mb).max() < 1e-12, gi
        oa += na * r
        ob += nb * r


@pytest.mark.parametrize("norb", [8, 16])
def test_device_hamiltonian_builder_matches_host(cuda, norb):
    """16 orbitals: the diagonal group's matrix is 137 x 137 (a 512-thread CTA)."""
    from binsim_b200 import cuotf, network as nw
    h, g, e = nw.synthetic_integrals(norb, 3)
    x, z, c = nw.jw_hamiltonian_terms(h, g, e)
    ax, az, bx, bz = nw.split_aabb(x, z, norb)
    a = cuotf.compress_groups_native(ax, az, bx, bz, c, norb)
    b = cuotf.compress_groups_native(ax, az, bx, bz, c, norb, device=True)
    _same_network(a, b)
    assert int(np.minimum(b.num_zas, b.num_zbs).max()) > 8   # some group took the 512-thread path
    if norb == 8:
        B = cuotf.CuBasis(norb, 4, 4)
        fa = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(a))
        fb = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(b))
        v = dev(cuda, np.random.default_rng(0).normal(size=B.dim))
        ya, yb = cuda.empty_like(v), cuda.empty_like(v)
        fa.hvec(v, ya)
        fb.hvec(v, yb)
        assert float((ya - yb).abs().max()) <= 1e-12 * float(ya.abs().max())


def test_device_pool_builder_matches_host(cuda):
    """One group per generator component (the run form), as ucc_pool builds them."""
    from binsim_b200 import cuotf, network as nw
    norb = 9
    a = nw.ucc_pool(norb, native=True).network
    b = nw.ucc_pool(norb, device=True).network
    _same_network(a, b)
    B = cuotf.CuBasis(norb, 4, 4)
    fa = cuotf.CuOTFFunctions(B, None, cuotf.CuNetwork(a))
    fb = cuotf.CuOTFFunctions(B, None, cuotf.CuNetwork(b))
    v0 = np.random.default_rng(1).normal(size=B.dim)
    v0 /= np.linalg.norm(v0)
    for gi in range(0, a.ngs, 211):
        va, vb = dev(cuda, v0), dev(cuda, v0)
        fa.expm(gi + 1, 0.4, va)
        fb.expm(gi + 1, 0.4, vb)
        assert float((va - vb).abs().max()) <= 1e-13


def test_device_builder_planted_rank(cuda):
    """A planted rank-1 group (outer product) and a rank-0 group come back exact."""
    from binsim_b200 import cuotf
    za, zb = np.array([1, 2, 4], np.uint64), np.array([1, 8], np.uint64)
    u, w = np.array([0.3, -1.2, 0.5]), np.array([2.0, -0.7])
    AZ, BZ = np.meshgrid(za, zb, indexing="ij")
    coef = np.outer(u, w).ravel()
    n = coef.size
    ax = np.concatenate([np.full(n, 3, np.uint64), [6]]).astype(np.uint64)
    bx = np.concatenate([np.full(n, 5, np.uint64), [0]]).astype(np.uint64)
    net = cuotf.compress_groups_native(ax, np.concatenate([AZ.ravel(), [1]]).astype(np.uint64), bx,
                                       np.concatenate([BZ.ravel(), [0]]).astype(np.uint64),
                                       np.concatenate([coef, [0.0]]), 4, device=True)
    assert net.ngs == 2 and int(net.ranks[0]) == 1 and int(net.ranks[1]) == 0
    M = net.flat_wa[:3].reshape(1, 3).T @ net.flat_wb[:2].reshape(1, 2)
    np.testing.assert_allclose(M, np.outer(u, w), atol=1e-14)
