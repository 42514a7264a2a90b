"""Complex (c64) operators on the GPU against the reference CPU library's _c64 outputs
(golden fixture tests/golden/c64_h6_3a2b.npz) and the oracle's complex restatement."""
import numpy as np
import pytest

from conftest import GOLDEN, load_golden  # noqa: F401

pytestmark = pytest.mark.gpu


def cdev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, np.complex128), device="cuda")


def _setup(z, ham, pool, bits=32):
    from binsim_b200 import cuotf
    B = cuotf.CuBasis(int(z["norb"]), int(z["na"]), int(z["nb"]), orbsym=z["orbsym"],
                      total_sym=int(z["total_sym"]), num_irreps=int(z["num_irreps"]), string_bits=bits)
    H = cuotf.CuNetworkC64(ham, z["ham_wa"], z["ham_wb"], string_bits=bits)
    P = cuotf.CuNetworkC64(pool, z["pool_wa"], z["pool_wb"], string_bits=bits)
    return B, cuotf.CuOTFC64(B, H), cuotf.CuOTFC64(B, P)


@pytest.mark.parametrize("bits", [32, 64])
def test_c64_ops_match_golden(cuda, bits):
    z, ham, pool = load_golden("c64_h6_3a2b")
    B, fh, fp = _setup(z, ham, pool, bits)
    assert B.dim == int(z["dim"])
    x, y = z["x"], z["y"]
    tol = 1e-12
    out = cuda.full((B.dim,), 3.0 + 1j, dtype=cuda.complex128, device="cuda")
    fh.hvec(cdev(cuda, x), out)
    np.testing.assert_allclose(out.cpu().numpy(), z["sigma"], rtol=0, atol=tol * np.abs(z["sigma"]).max())
    d = cuda.zeros(B.dim, dtype=cuda.complex128, device="cuda")
    fh.get_diags(d)
    np.testing.assert_allclose(d.cpu().numpy(), z["diag"], rtol=0, atol=tol * np.abs(z["diag"]).max())
    v = cdev(cuda, x)
    fh.expm(0, 0.6, v)   # the diagonal group: exp(i theta Im vt) factors
    np.testing.assert_allclose(v.cpu().numpy(), z["expm_ham0"], rtol=0, atol=1e-13)
    assert abs(fh.grad(0, 0.6, cdev(cuda, x), cdev(cuda, y)) - complex(z["grad_ham0"])) < 1e-11
    fh.tvec(0, cdev(cuda, x), out)
    np.testing.assert_allclose(out.cpu().numpy(), z["tvec_ham0"], rtol=0, atol=1e-13)
    for k, (i, t) in enumerate(zip(z["ops"], z["thetas"])):
        i, t = int(i), float(t)
        v = cdev(cuda, x)
        fp.expm(i, t, v)
        np.testing.assert_allclose(v.cpu().numpy(), z["expm"][k], rtol=0, atol=1e-13)
        assert abs(fp.grad(i, t, cdev(cuda, x), cdev(cuda, y)) - complex(z["grad"][k])) < 1e-11
        l, r = cdev(cuda, x), cdev(cuda, y)
        g = fp.backgrad(i, t, l, r)
        assert abs(g - complex(z["backgrad"][k])) < 1e-11
        np.testing.assert_allclose(l.cpu().numpy(), z["backgrad_l"][k], rtol=0, atol=1e-13)
        np.testing.assert_allclose(r.cpu().numpy(), z["backgrad_r"][k], rtol=0, atol=1e-13)
        fp.tvec(i, cdev(cuda, x), out)
        np.testing.assert_allclose(out.cpu().numpy(), z["tvec"][k], rtol=0, atol=1e-13)
        l, r, b = cdev(cuda, x), cdev(cuda, y), cuda.full_like(out, 5.0)
        fp.backtran(i, t, l, r, b)
        for a, ref in zip((l, r, b), (z["backtran_l"][k], z["backtran_r"][k], z["backtran_b"][k])):
            np.testing.assert_allclose(a.cpu().numpy(), ref, rtol=0, atol=1e-13)
    M = cdev(cuda, z["batchexpm_in"])
    fp.batchexpm(int(z["ops"][0]), float(z["thetas"][0]), M, 3, 2)
    np.testing.assert_allclose(M.cpu().numpy(), z["batchexpm"], rtol=0, atol=1e-13)
    g = cuda.zeros(pool.ngs, dtype=cuda.complex128, device="cuda")
    fp.batchgrad(z["batch_thetas"], cdev(cuda, x), cdev(cuda, y), g)
    np.testing.assert_allclose(g.cpu().numpy(), z["batchgrad"], rtol=0,
                               atol=1e-11 * max(1.0, np.abs(z["batchgrad"]).max()))
    t = cuda.zeros(pool.ngs, dtype=cuda.complex128, device="cuda")
    fp.batchtran(cdev(cuda, x), cdev(cuda, y), t)
    np.testing.assert_allclose(t.cpu().numpy(), z["trans_pool"], rtol=0, atol=1e-12)
    th = cuda.zeros(ham.ngs, dtype=cuda.complex128, device="cuda")
    fh.batchtran(cdev(cuda, x), cdev(cuda, y), th)
    np.testing.assert_allclose(th.cpu().numpy(), z["trans_ham"], rtol=0,
                               atol=1e-11 * max(1.0, np.abs(z["trans_ham"]).max()))


def test_c64_sigma_and_pool_ops_match_oracle(cuda, oracle):
    """9 orbitals 4a+4b (15,876 dets): complex-weight Hamiltonian sigma and pool
    operators against the oracle's complex restatement; real networks are refused by
    the c64 calls and c64 networks by the real ones."""
    from binsim_b200 import cuotf, network as nw
    from test_oracle_pin import complex_weights
    norb, na, nb = 9, 4, 4
    ham = nw.hamiltonian_network(norb, seed=12)
    pool = nw.ucc_pool(norb).network
    hw, pw = complex_weights(ham, 3), complex_weights(pool, 4)
    Bo = oracle.basis(norb, na, nb)
    Ho, Po = oracle.network_c64(ham, *hw), oracle.network_c64(pool, *pw)
    B = cuotf.CuBasis(norb, na, nb)
    fh = cuotf.CuOTFC64(B, cuotf.CuNetworkC64(ham, *hw))
    fp = cuotf.CuOTFC64(B, cuotf.CuNetworkC64(pool, *pw))
    rng = np.random.default_rng(6)
    x = rng.normal(size=B.dim) + 1j * rng.normal(size=B.dim)
    y = rng.normal(size=B.dim) + 1j * rng.normal(size=B.dim)
    out = cuda.empty(B.dim, dtype=cuda.complex128, device="cuda")
    fh.hvec(cdev(cuda, x), out)
    ref = oracle.hvec_c64(Bo, Ho, x)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    for i in rng.choice(pool.ngs, 10, replace=False):
        i, t = int(i), float(rng.normal())
        v = cdev(cuda, x)
        fp.expm(i, t, v)
        np.testing.assert_allclose(v.cpu().numpy(), oracle.expm_c64(Bo, Po, i, t, x), rtol=0, atol=1e-13)
        l, r = cdev(cuda, x), cdev(cuda, y)
        g = fp.backgrad(i, t, l, r)
        g0, l0, r0 = oracle.backgrad_c64(Bo, Po, i, t, x, y)
        assert abs(g - g0) < 1e-10 * max(1.0, abs(g0))
        np.testing.assert_allclose(l.cpu().numpy(), l0, rtol=0, atol=1e-13)
    th = rng.normal(size=pool.ngs)
    gd = cuda.zeros(pool.ngs, dtype=cuda.complex128, device="cuda")
    fp.batchgrad(th, cdev(cuda, x), cdev(cuda, y), gd)
    gref = oracle.batchgrad_c64(Bo, Po, th, x, y)
    np.testing.assert_allclose(gd.cpu().numpy(), gref, rtol=0, atol=1e-10 * max(1.0, np.abs(gref).max()))
    # handle kinds do not mix
    Hreal = cuotf.CuNetwork(ham)
    with pytest.raises(cuotf.CuOTFError):
        cuotf.CuOTFC64(B, Hreal).hvec(cdev(cuda, x), out)
    with pytest.raises(cuotf.CuOTFError):
        cuotf.CuOTFFunctions(B, fh.net).hvec(cuda.zeros(B.dim, dtype=cuda.float64, device="cuda"),
                                              cuda.zeros(B.dim, dtype=cuda.float64, device="cuda"))


def test_real_and_complex_reductions_share_a_basis(cuda, oracle):
    """Real grad after complex grads on the same basis handle (they share its reduction
    scratch): both keep their own partial slots and ticket words."""
    from binsim_b200 import cuotf, network as nw
    from test_oracle_pin import complex_weights
    norb, na, nb = 7, 3, 3
    pool = nw.ucc_pool(norb).network
    B = cuotf.CuBasis(norb, na, nb)
    Bo, Po = oracle.basis(norb, na, nb), oracle.network(pool)
    fr = cuotf.CuOTFFunctions(B, None, cuotf.CuNetwork(pool))
    fc = cuotf.CuOTFC64(B, cuotf.CuNetworkC64(pool, *complex_weights(pool, 9)))
    rng = np.random.default_rng(2)
    x, y = rng.normal(size=B.dim), rng.normal(size=B.dim)
    xc, yc = cdev(cuda, x + 1j * y), cdev(cuda, y - 0.5j * x)
    xd, yd = cuda.as_tensor(x, device="cuda"), cuda.as_tensor(y, device="cuda")
    for i in (3, 11, 40):
        fc.grad(i, 0.3, xc, yc)
        g = fr.grad(i + 1, 0.3, xd, yd)
        assert abs(g - oracle.grad(Bo, Po, i, 0.3, x, y)) < 1e-11
        fc.backgrad(i, 0.2, xc.clone(), yc.clone())
