"""expm / grad / backgrad / batchgrad on the GPU against golden fixtures and the oracle."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, cu_setup, dev, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_pair_ops_match_golden(cuda, name):
    z, ham, pool = load_golden(name)
    B, H, P, f = cu_setup(z, ham, pool)
    x, y = z["x"], z["y"]
    for k, (i, t) in enumerate(zip(z["ops"], z["thetas"])):
        v = dev(cuda, x)
        f.expm(int(i) + 1, t, v)
        np.testing.assert_allclose(v.cpu().numpy(), z["expm"][k], rtol=0, atol=1e-14)
        g = f.grad(int(i) + 1, t, dev(cuda, x), dev(cuda, y))
        assert abs(g - z["grad"][k]) < 1e-12 * max(1.0, abs(z["grad"][k]))
        l, r = dev(cuda, x), dev(cuda, y)
        g = f.backgrad(int(i) + 1, t, l, r)
        assert abs(g - z["backgrad"][k]) < 1e-12 * max(1.0, abs(z["backgrad"][k]))
        np.testing.assert_allclose(l.cpu().numpy(), z["backgrad_l"][k], rtol=0, atol=1e-14)
        np.testing.assert_allclose(r.cpu().numpy(), z["backgrad_r"][k], rtol=0, atol=1e-14)
    grads = cuda.full((pool.ngs,), 7.0, dtype=cuda.float64, device="cuda")   # overwritten
    f.batchgrad(dev(cuda, x), dev(cuda, z["sigma"]), grads, dev(cuda, z["batch_thetas"]))
    np.testing.assert_allclose(grads.cpu().numpy(), z["batchgrad"], rtol=0,
                               atol=1e-12 * max(1.0, np.abs(z["batchgrad"]).max()))


def test_legacy_pair_entry_points(cuda):
    z, ham, pool = load_golden("h8_4a3b_sym")
    B, H, P, f = cu_setup(z, ham, pool)
    from binsim_b200.cuotf import lib
    L = lib()
    i, t = int(z["ops"][0]), float(z["thetas"][0])
    v = dev(cuda, z["x"])
    L.expm_cuda(B.h, P.h, i, t, v.data_ptr())
    L.sync_device_cuda()
    np.testing.assert_allclose(v.cpu().numpy(), z["expm"][0], atol=1e-14)
    xd, yd = dev(cuda, z["x"]), dev(cuda, z["y"])   # held: distinct device pointers
    g = L.grad_cuda(B.h, P.h, i, t, xd.data_ptr(), yd.data_ptr())
    assert abs(g - z["grad"][0]) < 1e-12
    g2 = L.grad_cuda_2d(B.h, P.h, i, t, xd.data_ptr(), yd.data_ptr())
    assert g2 == g
    l, r = dev(cuda, z["x"]), dev(cuda, z["y"])
    g = L.backgrad_cuda(B.h, P.h, i, t, l.data_ptr(), r.data_ptr())
    assert abs(g - z["backgrad"][0]) < 1e-12
    # an out-of-range index is reported and leaves the vector untouched
    w = dev(cuda, z["x"])
    L.expm_cuda(B.h, P.h, 10 ** 9, 0.3, w.data_ptr())
    assert np.array_equal(w.cpu().numpy(), z["x"])
    assert b"out of range" in L.bsim_last_error()


def test_expm_sequence_and_orthogonality(cuda, oracle):
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 9, 4, 4
    pool = nw.ucc_pool(norb).network
    Bo, Po = oracle.basis(norb, na, nb), oracle.network(pool)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, None, cuotf.CuNetwork(pool))
    rng = np.random.default_rng(1)
    idx = rng.integers(0, pool.ngs, size=40)
    th = rng.normal(0, 0.3, size=40)
    x = rng.normal(size=B.dim)
    ref = x.copy()
    for i, t in zip(idx, th):
        ref = oracle.expm(Bo, Po, int(i), t, ref)
    v = dev(cuda, x)
    f.expm_seq(idx + 1, th, v)
    np.testing.assert_allclose(v.cpu().numpy(), ref, rtol=0, atol=1e-13)
    assert abs(float(v.norm()) - np.linalg.norm(x)) < 1e-11
    # inverse sequence returns the input
    f.expm_seq(idx[::-1] + 1, -th[::-1], v)
    np.testing.assert_allclose(v.cpu().numpy(), x, atol=1e-12)


def test_batchgrad_matches_oracle_at_theta_zero(cuda, oracle):
    """ADAPT screening (jl/vqe.jl:235-238): batchgrad(psi, H psi, 0)."""
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 9, 4, 5
    ham, pool = nw.hamiltonian_network(norb, seed=5), nw.ucc_pool(norb).network
    Bo, Ho, Po = oracle.basis(norb, na, nb), oracle.network(ham), oracle.network(pool)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(ham), cuotf.CuNetwork(pool))
    psi = np.random.default_rng(3).normal(size=B.dim)
    hpsi = oracle.hvec(Bo, Ho, psi)
    ref = oracle.batchgrad(Bo, Po, np.zeros(pool.ngs), psi, hpsi)
    g = cuda.empty(pool.ngs, dtype=cuda.float64, device="cuda")
    f.batchgrad(dev(cuda, psi), dev(cuda, hpsi), g, cuda.zeros(pool.ngs, dtype=cuda.float64, device="cuda"))
    np.testing.assert_allclose(g.cpu().numpy(), ref, rtol=0, atol=1e-11 * np.abs(ref).max())


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_tvec_backtran_batch_ops_match_golden(cuda, name):
    """GPU tvec / backtran / batchexpm / batchtran (CPU-only in the reference) against
    the reference CPU library's outputs stored in the golden fixtures: pool generators,
    the Hamiltonian's diagonal group and every group's transition element."""
    from binsim_b200 import cuotf
    z, ham, pool = load_golden(name)
    B, H, P, f = cu_setup(z, ham, pool)
    fh = cuotf.CuOTFFunctions(B, H, H)
    x, y = z["x"], z["y"]
    out = cuda.full((B.dim,), 3.0, dtype=cuda.float64, device="cuda")   # overwritten
    for k, i in enumerate(z["ops"][:4]):
        f.tvec(int(i) + 1, dev(cuda, x), out)
        np.testing.assert_allclose(out.cpu().numpy(), z["tvec"][k], rtol=0, atol=1e-14)
        l, r, b = dev(cuda, x), dev(cuda, y), cuda.full_like(out, 5.0)
        f.backtran(int(i) + 1, float(z["thetas"][k]), l, r, b)
        np.testing.assert_allclose(l.cpu().numpy(), z["backtran_l"][k], rtol=0, atol=1e-14)
        np.testing.assert_allclose(r.cpu().numpy(), z["backtran_r"][k], rtol=0, atol=1e-14)
        np.testing.assert_allclose(b.cpu().numpy(), z["backtran_b"][k], rtol=0, atol=1e-14)
    fh.tvec(1, dev(cuda, x), out)   # the diagonal group
    np.testing.assert_allclose(out.cpu().numpy(), z["tvec_ham0"], rtol=0, atol=1e-13)
    l, r, b = dev(cuda, x), dev(cuda, y), cuda.zeros_like(out)
    fh.backtran(1, 0.4, l, r, b)
    for a, ref in zip((l, r, b), z["backtran_ham0"]):
        np.testing.assert_allclose(a.cpu().numpy(), ref, rtol=0, atol=1e-13)
    M = dev(cuda, z["batchexpm_in"])
    f.batchexpm(int(z["ops"][0]) + 1, float(z["thetas"][0]), M, 3, 2)
    np.testing.assert_allclose(M.cpu().numpy(), z["batchexpm"], rtol=0, atol=1e-14)
    tp = cuda.full((pool.ngs,), 9.0, dtype=cuda.float64, device="cuda")
    f.batchtran(dev(cuda, x), dev(cuda, y), tp)
    np.testing.assert_allclose(tp.cpu().numpy(), z["trans_pool"], rtol=0, atol=1e-13)
    th = cuda.full((ham.ngs,), 9.0, dtype=cuda.float64, device="cuda")
    fh.batchtran(dev(cuda, x), dev(cuda, y), th)
    np.testing.assert_allclose(th.cpu().numpy(), z["trans_ham"], rtol=0,
                               atol=1e-12 * max(1.0, np.abs(z["trans_ham"]).max()))


def test_tvec_backtran_legacy_names_and_u64(cuda, oracle):
    """The void-returning names (tvec_cuda, backtran_cuda, batchexpm_cuda, batchtran_cuda)
    and UInt64 handles at 28 orbitals (ranked string addressing) against the oracle."""
    from binsim_b200 import cuotf, network as nw
    from binsim_b200.cuotf import lib
    from test_gpu_u64 import random_network
    norb, na, nb = 28, 2, 2
    net = random_network(norb, seed=4, ngroups=30)
    Bo, No = oracle.basis(norb, na, nb), oracle.network(net)
    B = cuotf.CuBasis(norb, na, nb, string_bits=64)
    N = cuotf.CuNetwork(net, string_bits=64)
    rng = np.random.default_rng(8)
    x, y = rng.normal(size=B.dim), rng.normal(size=B.dim)
    L = lib()
    xd, yd = dev(cuda, x), dev(cuda, y)   # held: the raw pointers below must stay distinct
    for g in (0, 1, 2, 3, 7):
        out = cuda.zeros(B.dim, dtype=cuda.float64, device="cuda")
        L.tvec_cuda(B.h, N.h, g, xd.data_ptr(), out.data_ptr())
        L.sync_device_cuda()
        np.testing.assert_allclose(out.cpu().numpy(), oracle.tvec(Bo, No, g, x), rtol=0, atol=1e-12)
        l, r, b = dev(cuda, x), dev(cuda, y), cuda.zeros_like(out)
        L.backtran_cuda(B.h, N.h, g, 0.7, l.data_ptr(), r.data_ptr(), b.data_ptr())
        L.sync_device_cuda()
        for a, ref in zip((l, r, b), oracle.backtran(Bo, No, g, 0.7, x, y)):
            np.testing.assert_allclose(a.cpu().numpy(), ref, rtol=0, atol=1e-12)
        M = rng.normal(size=(B.dim, 2))
        Md = dev(cuda, M)
        L.batchexpm_cuda(B.h, N.h, g, -0.3, Md.data_ptr(), 2, 2)
        L.sync_device_cuda()
        np.testing.assert_allclose(Md.cpu().numpy(), oracle.batchexpm(Bo, No, g, -0.3, M, 2), rtol=0, atol=1e-12)
    t = cuda.zeros(net.ngs, dtype=cuda.float64, device="cuda")
    L.batchtran_cuda(B.h, N.h, xd.data_ptr(), yd.data_ptr(), t.data_ptr())
    L.sync_device_cuda()
    tr = oracle.batchtran(Bo, No, x, y)
    np.testing.assert_allclose(t.cpu().numpy(), tr, rtol=0, atol=1e-11 * max(1.0, np.abs(tr).max()))
    with pytest.raises(cuotf.CuOTFError):   # num_vecs > ld
        cuotf.CuOTFFunctions(B, N, N).batchexpm(2, 0.1, Md, 1, 2)
