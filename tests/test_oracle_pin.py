"""Pin the C restatement (oracle/otf_oracle.c) against the reference.

* against the golden fixtures made by the reference's own libraries
  (tests/golden/gen_golden.py) -- runs everywhere;
* against the reference libraries directly (oracle/_ref) on fresh seeded
  inputs -- runs where they are built.
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden

TOL = 1e-12


def _basis(oracle, z):
    return oracle.basis(int(z["norb"]), int(z["na"]), int(z["nb"]), orbsym=z["orbsym"],
                        total_sym=int(z["total_sym"]), num_irreps=int(z["num_irreps"]))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_golden(oracle, name):
    z, ham, pool = load_golden(name)
    B = _basis(oracle, z)
    assert B.dim == int(z["dim"])
    H, P = oracle.network(ham), oracle.network(pool)
    x, y = z["x"], z["y"]
    scale = np.abs(z["sigma"]).max()
    np.testing.assert_allclose(oracle.hvec(B, H, x), z["sigma"], rtol=0, atol=TOL * scale)
    np.testing.assert_allclose(oracle.diag(B, H), z["diag"], rtol=0, atol=TOL * np.abs(z["diag"]).max())
    for k, (i, t) in enumerate(zip(z["ops"], z["thetas"])):
        np.testing.assert_allclose(oracle.expm(B, P, int(i), t, x), z["expm"][k], rtol=0, atol=1e-14)
        assert abs(oracle.grad(B, P, int(i), t, x, y) - z["grad"][k]) < 1e-13
        g, l2, r2 = oracle.backgrad(B, P, int(i), t, x, y)
        assert abs(g - z["backgrad"][k]) < 1e-13
        np.testing.assert_allclose(l2, z["backgrad_l"][k], rtol=0, atol=1e-14)
        np.testing.assert_allclose(r2, z["backgrad_r"][k], rtol=0, atol=1e-14)
    bg = oracle.batchgrad(B, P, z["batch_thetas"], x, z["sigma"])
    np.testing.assert_allclose(bg, z["batchgrad"], rtol=0, atol=TOL * max(1.0, np.abs(z["batchgrad"]).max()))
    assert B.det_index((1 << int(z["na"])) - 1, (1 << int(z["nb"])) - 1) == int(z["hf"])


@pytest.mark.parametrize("norb,na,nb,orbsym,tsym", [
    (5, 2, 3, None, 0),
    (7, 3, 3, [0, 1, 2, 3, 0, 1, 2], 2),
    (8, 4, 4, [0, 1, 1, 0, 2, 3, 3, 2], 0),
])
def test_oracle_matches_reference_libs(oracle, reflibs, norb, na, nb, orbsym, tsym):
    from binsim_b200 import network as nw
    osym = np.zeros(norb, np.int64) if orbsym is None else np.asarray(orbsym, np.int64)
    ham = nw.hamiltonian_network(norb, seed=norb * 7 + 1)
    pool = nw.ucc_pool(norb).network
    ham.orbsym = osym; pool.orbsym = osym
    rb, dim = reflibs.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    B = oracle.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    assert B.dim == dim
    rh, rp = reflibs.network(ham), reflibs.network(pool)
    H, P = oracle.network(ham), oracle.network(pool)
    rng = np.random.default_rng(norb)
    x, y = rng.normal(size=dim), rng.normal(size=dim)
    s_ref = reflibs.hvec(rb, rh, x, dim)
    np.testing.assert_allclose(oracle.hvec(B, H, x), s_ref, rtol=0, atol=1e-12 * np.abs(s_ref).max())
    np.testing.assert_allclose(oracle.diag(B, H), reflibs.diag_elems(rb, rh, dim), rtol=0, atol=1e-12)
    for i in rng.choice(pool.ngs, 25, replace=False):
        t = rng.normal()
        np.testing.assert_allclose(oracle.expm(B, P, int(i), t, x), reflibs.expm(rb, rp, int(i), t, x), atol=1e-13)
        assert abs(oracle.grad(B, P, int(i), t, x, y) - reflibs.grad(rb, rp, int(i), t, x, y)) < 1e-11
    th = rng.normal(size=pool.ngs)
    np.testing.assert_allclose(oracle.batchgrad(B, P, th, x, y), reflibs.batchgrad(rb, rp, th, x, y, pool.ngs),
                               atol=1e-10)


def test_oracle_davidson_helpers_match_libdiag(oracle, reflibs):
    import ctypes as C
    rng = np.random.default_rng(5)
    n, k = 3001, 5
    Q = np.linalg.qr(rng.normal(size=(n, k)))[0]
    V = [np.ascontiguousarray(Q[:, j]) for j in range(k)]
    AV = [rng.normal(size=n) for _ in range(k)]
    c = rng.normal(size=k)
    d = rng.normal(size=n)
    arr = lambda vs: (C.c_void_p * len(vs))(*[v.ctypes.data for v in vs])
    out = np.zeros(n)
    nr = reflibs.diag.build_ritz_and_residual_f64(n, k, c.ctypes.data, 0.3, arr(V), arr(AV), out.ctypes.data)
    nr2, out2 = oracle.ritz_residual(c, 0.3, V, AV)
    assert abs(nr - nr2) < 1e-10 and np.abs(out - out2).max() < 1e-12
    r = rng.normal(size=n); r1 = r.copy()
    reflibs.diag.apply_preconditioner_inplace_f64(n, r1.ctypes.data, d.ctypes.data, 0.1, 0.05)
    np.testing.assert_allclose(oracle.precondition(r, d, 0.1, 0.05), r1, rtol=1e-15)
    v = rng.normal(size=n); v1 = v.copy()
    m1 = reflibs.diag.mgs_orthogonalize_f64(n, k, arr(V), v1.ctypes.data)
    m2, v2 = oracle.mgs(V, v)
    assert abs(m1 - m2) < 1e-12 * m1 and np.abs(v1 - v2).max() < 1e-12
    col = np.zeros(k)
    reflibs.diag.compute_heff_col_f64(n, k, arr(V), AV[0].ctypes.data, col.ctypes.data)
    np.testing.assert_allclose(oracle.heff_col(V, AV[0]), col, rtol=1e-12)


@pytest.mark.parametrize("norb,na,nb,orbsym,tsym", [
    (6, 3, 2, None, 0),
    (7, 3, 3, [0, 1, 2, 3, 0, 1, 2], 2),
])
def test_oracle_tvec_backtran_batch_ops_match_reference_libs(oracle, reflibs, norb, na, nb, orbsym, tsym):
    """tvec, backtran, batch_expm and batch_tran (the reference CPU library's
    tvec_contract_otf, backtran_contract_otf, batch_expm_contract_otf and
    batch_tran_contract_otf) against the C restatement, on Hamiltonian groups
    (including the diagonal group) and on pool generators."""
    from binsim_b200 import network as nw
    osym = np.zeros(norb, np.int64) if orbsym is None else np.asarray(orbsym, np.int64)
    ham = nw.hamiltonian_network(norb, seed=norb * 3 + 2)
    pool = nw.ucc_pool(norb).network
    ham.orbsym = osym; pool.orbsym = osym
    rb, dim = reflibs.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    B = oracle.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    rng = np.random.default_rng(norb + 100)
    x, y = rng.normal(size=dim), rng.normal(size=dim)
    for net in (ham, pool):
        rn, N = reflibs.network(net), oracle.network(net)
        for i in sorted(set([0] + list(rng.choice(net.ngs, 12, replace=False)))):
            i = int(i)
            np.testing.assert_allclose(oracle.tvec(B, N, i, x), reflibs.tvec(rb, rn, i, x, dim), rtol=0, atol=1e-13)
            t = rng.normal()
            for a, b in zip(oracle.backtran(B, N, i, t, x, y), reflibs.backtran(rb, rn, i, t, x, y, dim)):
                np.testing.assert_allclose(a, b, rtol=0, atol=1e-13)
            M = rng.normal(size=(dim, 4))
            np.testing.assert_allclose(oracle.batchexpm(B, N, i, t, M, 3), reflibs.batchexpm(rb, rn, i, t, M, 3),
                                       rtol=0, atol=1e-13)
        tr = reflibs.batchtran(rb, rn, x, y, net.ngs)
        np.testing.assert_allclose(oracle.batchtran(B, N, x, y), tr, rtol=0, atol=1e-11 * max(1.0, np.abs(tr).max()))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_tvec_backtran_batch_ops_match_golden(oracle, name):
    """The restated tvec / backtran / batch_expm / batch_tran against the reference's
    outputs stored in the golden fixtures."""
    z, ham, pool = load_golden(name)
    B = _basis(oracle, z)
    H, P = oracle.network(ham), oracle.network(pool)
    x, y = z["x"], z["y"]
    for k, i in enumerate(z["ops"][:4]):
        np.testing.assert_allclose(oracle.tvec(B, P, int(i), x), z["tvec"][k], rtol=0, atol=1e-14)
        l2, r2, b2 = oracle.backtran(B, P, int(i), z["thetas"][k], x, y)
        np.testing.assert_allclose(l2, z["backtran_l"][k], rtol=0, atol=1e-14)
        np.testing.assert_allclose(r2, z["backtran_r"][k], rtol=0, atol=1e-14)
        np.testing.assert_allclose(b2, z["backtran_b"][k], rtol=0, atol=1e-14)
    np.testing.assert_allclose(oracle.tvec(B, H, 0, x), z["tvec_ham0"], rtol=0, atol=1e-13)
    for a, b in zip(oracle.backtran(B, H, 0, 0.4, x, y), z["backtran_ham0"]):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-13)
    np.testing.assert_allclose(oracle.batchexpm(B, P, int(z["ops"][0]), z["thetas"][0], z["batchexpm_in"], 2),
                               z["batchexpm"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(oracle.batchtran(B, P, x, y), z["trans_pool"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(oracle.batchtran(B, H, x, y), z["trans_ham"], rtol=0,
                               atol=1e-12 * max(1.0, np.abs(z["trans_ham"]).max()))


def complex_weights(net, seed):
    """Complex weights for a real network's groups: each real weight times a seeded
    phase and modulus (the networks of the reference's complex interface)."""
    rng = np.random.default_rng(seed)
    wa = np.asarray(net.flat_wa) * rng.uniform(0.5, 1.5, len(net.flat_wa)) * np.exp(1j * rng.uniform(0, 6.3, len(net.flat_wa)))
    wb = np.asarray(net.flat_wb) * rng.uniform(0.5, 1.5, len(net.flat_wb)) * np.exp(1j * rng.uniform(0, 6.3, len(net.flat_wb)))
    return wa, wb


@pytest.mark.parametrize("norb,na,nb,orbsym,tsym", [
    (6, 3, 2, None, 0),
    (7, 3, 3, [0, 1, 2, 3, 0, 1, 2], 2),
])
def test_oracle_c64_ops_match_reference_libs(oracle, reflibs, norb, na, nb, orbsym, tsym):
    """The complex restatement against the reference CPU library's _c64 entry points:
    sigma, diagonal, expm, grad, backgrad, tvec, backtran, batch_expm, batch_grad and
    batch_tran, on a Hamiltonian with complex weights (diagonal group included) and on
    pool generators with complex weights."""
    from binsim_b200 import network as nw
    osym = np.zeros(norb, np.int64) if orbsym is None else np.asarray(orbsym, np.int64)
    ham = nw.hamiltonian_network(norb, seed=norb + 40)
    pool = nw.ucc_pool(norb).network
    ham.orbsym = osym; pool.orbsym = osym
    rb, dim = reflibs.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    B = oracle.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    rng = np.random.default_rng(norb + 7)
    x = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    y = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    for k, net in enumerate((ham, pool)):
        wa, wb = complex_weights(net, seed=norb + k)
        rn, N = reflibs.network_c64(net, wa, wb), oracle.network_c64(net, wa, wb)
        if k == 0:
            s = reflibs.hvec_c64(rb, rn, x, dim)
            np.testing.assert_allclose(oracle.hvec_c64(B, N, x), s, rtol=0, atol=1e-12 * np.abs(s).max())
            np.testing.assert_allclose(oracle.diag_c64(B, N), reflibs.diag_c64(rb, rn, dim), rtol=0, atol=1e-12)
        for i in sorted(set([0] + list(rng.choice(net.ngs, 8, replace=False)))):
            i, t = int(i), float(rng.normal())
            np.testing.assert_allclose(oracle.expm_c64(B, N, i, t, x), reflibs.expm_c64(rb, rn, i, t, x), atol=1e-13)
            assert abs(oracle.grad_c64(B, N, i, t, x, y) - reflibs.grad_c64(rb, rn, i, t, x, y)) < 1e-11
            g0, l0, r0 = reflibs.backgrad_c64(rb, rn, i, t, x, y)
            g1, l1, r1 = oracle.backgrad_c64(B, N, i, t, x, y)
            assert abs(g0 - g1) < 1e-11
            np.testing.assert_allclose(l1, l0, atol=1e-13); np.testing.assert_allclose(r1, r0, atol=1e-13)
            np.testing.assert_allclose(oracle.tvec_c64(B, N, i, x), reflibs.tvec_c64(rb, rn, i, x, dim), atol=1e-13)
            for a, b in zip(oracle.backtran_c64(B, N, i, t, x, y), reflibs.backtran_c64(rb, rn, i, t, x, y, dim)):
                np.testing.assert_allclose(a, b, atol=1e-13)
            M = rng.normal(size=(dim, 3)) + 1j * rng.normal(size=(dim, 3))
            np.testing.assert_allclose(oracle.batchexpm_c64(B, N, i, t, M, 2), reflibs.batchexpm_c64(rb, rn, i, t, M, 2),
                                       atol=1e-13)
        th = rng.normal(size=net.ngs)
        gr = reflibs.batchgrad_c64(rb, rn, th, x, y, net.ngs)
        np.testing.assert_allclose(oracle.batchgrad_c64(B, N, th, x, y), gr, atol=1e-10 * max(1.0, np.abs(gr).max()))
        tr = reflibs.batchtran_c64(rb, rn, x, y, net.ngs)
        np.testing.assert_allclose(oracle.batchtran_c64(B, N, x, y), tr, atol=1e-10 * max(1.0, np.abs(tr).max()))


@pytest.mark.parametrize("norb,na,nb,orbsym,tsym", [
    (8, 4, 3, None, 0),
    (7, 3, 3, [0, 1, 2, 3, 0, 1, 2], 2),
])
def test_oracle_matches_reference_ui64_operators(oracle, reflibs, norb, na, nb, orbsym, tsym):
    """The reference's uint64 operators (_ui64_f64, over its basis interface instantiated
    for uint64) against the oracle, which keeps every string as a 64-bit word: sigma,
    diagonal, expm, grad, backgrad, batch grad, tvec and batch tran."""
    from oracle.oracle import RefLibsU64, ref_u64_available
    from binsim_b200 import network as nw
    if not ref_u64_available():
        pytest.skip("oracle/_ref/libbasis_ui64.so not built")
    ref = RefLibsU64(reflibs)
    osym = np.zeros(norb, np.int64) if orbsym is None else np.asarray(orbsym, np.int64)
    ham = nw.hamiltonian_network(norb, seed=norb * 5 + 2)
    pool = nw.ucc_pool(norb).network
    ham.orbsym = osym; pool.orbsym = osym
    rb, dim = ref.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    B = oracle.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    assert B.dim == dim
    rh, rp = ref.network(ham), ref.network(pool)
    H, Pn = oracle.network(ham), oracle.network(pool)
    rng = np.random.default_rng(norb + 100)
    x, y = rng.normal(size=dim), rng.normal(size=dim)
    s = ref.hvec(rb, rh, x, dim)
    np.testing.assert_allclose(oracle.hvec(B, H, x), s, rtol=0, atol=TOL * np.abs(s).max())
    d = ref.diag_elems(rb, rh, dim)
    np.testing.assert_allclose(oracle.diag(B, H), d, rtol=0, atol=TOL * np.abs(d).max())
    for i in rng.choice(pool.ngs, 8, replace=False):
        t = rng.normal(0, 0.7)
        np.testing.assert_allclose(oracle.expm(B, Pn, int(i), t, x), ref.expm(rb, rp, int(i), t, x), rtol=0,
                                   atol=1e-13)
        assert abs(oracle.grad(B, Pn, int(i), t, x, y) - ref.grad(rb, rp, int(i), t, x, y)) < 1e-12
        g1, l1, r1 = oracle.backgrad(B, Pn, int(i), t, x, y)
        g2, l2, r2 = ref.backgrad(rb, rp, int(i), t, x, y)
        assert abs(g1 - g2) < 1e-12
        np.testing.assert_allclose(l1, l2, rtol=0, atol=1e-13)
        np.testing.assert_allclose(r1, r2, rtol=0, atol=1e-13)
        np.testing.assert_allclose(oracle.tvec(B, Pn, int(i), x), ref.tvec(rb, rp, int(i), x, dim), rtol=0,
                                   atol=1e-13)
    th = rng.normal(0, 0.3, size=pool.ngs)
    bg = ref.batchgrad(rb, rp, th, x, y, pool.ngs)
    np.testing.assert_allclose(oracle.batchgrad(B, Pn, th, x, y), bg, rtol=0, atol=TOL * np.abs(bg).max())
    bt = ref.batchtran(rb, rp, x, y, pool.ngs)
    np.testing.assert_allclose(oracle.batchtran(B, Pn, x, y), bt, rtol=0, atol=TOL * np.abs(bt).max())


@pytest.mark.parametrize("norb,na,nb,orbsym,tsym", [
    (6, 3, 2, None, 0),
    (7, 3, 3, [0, 1, 2, 3, 0, 1, 2], 2),
])
def test_oracle_c64_matches_reference_ui64_c64_operators(oracle, reflibs, norb, na, nb, orbsym, tsym):
    """The complex restatement against the reference's uint64 complex operators
    (_ui64_c64): the checks of the uint32 complex pin, on the uint64 basis."""
    from oracle.oracle import RefLibsU64, ref_u64_available
    if not ref_u64_available():
        pytest.skip("oracle/_ref/libbasis_ui64.so not built")
    view = RefLibsU64(reflibs).complex_view(reflibs)
    test_oracle_c64_ops_match_reference_libs(oracle, view, norb, na, nb, orbsym, tsym)
