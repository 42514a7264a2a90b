"""Davidson on device: libdiag's helpers (Part 3 of the C-ABI) and the drivers."""
import ctypes as C

import numpy as np
import pytest

from conftest import dev

pytestmark = pytest.mark.gpu


def _ptrs(ts):
    return (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def test_device_helpers_match_oracle(cuda, oracle):
    from binsim_b200.cuotf import lib
    L = lib()
    rng = np.random.default_rng(0)
    n, k = 200_003, 6
    Q = np.linalg.qr(rng.normal(size=(n, k)))[0]
    V = [np.ascontiguousarray(Q[:, j]) for j in range(k)]
    AV = [rng.normal(size=n) for _ in range(k)]
    c, d = rng.normal(size=k), rng.normal(size=n)
    Vd, AVd = [dev(cuda, v) for v in V], [dev(cuda, v) for v in AV]
    out = cuda.empty(n, dtype=cuda.float64, device="cuda")
    nr = L.build_ritz_and_residual_cuda(n, k, c.ctypes.data, 0.25, _ptrs(Vd), _ptrs(AVd), out.data_ptr())
    nr2, out2 = oracle.ritz_residual(c, 0.25, V, AV)
    assert abs(nr - nr2) < 1e-12 * nr2
    np.testing.assert_allclose(out.cpu().numpy(), out2, atol=1e-12)
    x = cuda.empty(n, dtype=cuda.float64, device="cuda")
    L.build_ritz_vector_cuda(n, k, c.ctypes.data, _ptrs(Vd), x.data_ptr())
    np.testing.assert_allclose(x.cpu().numpy(), oracle.ritz_vector(c, V), atol=1e-12)
    r = rng.normal(size=n)
    rd = dev(cuda, r)
    L.apply_preconditioner_inplace_cuda(n, rd.data_ptr(), dev(cuda, d).data_ptr(), 0.1, 0.05)
    np.testing.assert_allclose(rd.cpu().numpy(), oracle.precondition(r, d, 0.1, 0.05), rtol=1e-15)
    v = rng.normal(size=n)
    vd = dev(cuda, v)
    m = L.mgs_orthogonalize_cuda(n, k, _ptrs(Vd), vd.data_ptr())
    m2, v2 = oracle.mgs(V, v)
    assert abs(m - m2) < 1e-12 * m2
    np.testing.assert_allclose(vd.cpu().numpy(), v2, atol=1e-12)
    assert abs(L.fast_dot_cuda(n, Vd[0].data_ptr(), AVd[1].data_ptr()) - V[0] @ AV[1]) < 1e-11
    w = dev(cuda, v)
    nrm = L.inplace_normalize_cuda(n, w.data_ptr())
    assert abs(nrm - np.linalg.norm(v)) < 1e-10 and abs(float(w.norm()) - 1) < 1e-14
    col = np.zeros(k)
    L.compute_heff_col_cuda(n, k, _ptrs(Vd), AVd[2].data_ptr(), col.ctypes.data)
    np.testing.assert_allclose(col, oracle.heff_col(V, AV[2]), atol=1e-11)
    heff = np.zeros((k, k), order="F")
    L.rebuild_heff_cuda(n, k, _ptrs(Vd), _ptrs(AVd), heff.ctypes.data, k)
    np.testing.assert_allclose(heff, np.array([[V[i] @ AV[j] for j in range(k)] for i in range(k)]), atol=1e-11)


def _lowest(oracle, Bo, No, k=1):
    from scipy.sparse.linalg import LinearOperator, eigsh
    op = LinearOperator((Bo.dim, Bo.dim), matvec=lambda x: oracle.hvec(Bo, No, x), dtype=np.float64)
    return np.sort(eigsh(op, k=k, which="SA", tol=1e-13)[0])


@pytest.mark.parametrize("maxspace", [12, 5])
def test_davidson_fp64_and_mixed(cuda, oracle, maxspace):
    """The device-resident drivers against eigsh; maxspace 5 restarts every few steps."""
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 9, 4, 4
    net = nw.hamiltonian_network(norb, seed=21)
    Bo, No = oracle.basis(norb, na, nb), oracle.network(net)
    e_ref = _lowest(oracle, Bo, No)[0]
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    diags = cuda.zeros(B.dim, dtype=cuda.float64, device="cuda")
    f.get_diags(diags)
    v0 = cuda.zeros_like(diags)
    v0[B.hf_index()] = 1.0
    x = cuda.empty_like(diags)
    st = f.davidson(v0.clone(), diags, x, tol=1e-6, maxiter=300, ncv=3, maxspace=maxspace)
    assert abs(st["energy"] - e_ref) < 1e-9, (st, e_ref)
    assert st["residual"] < 1e-6
    # the eigenvector: H x = E x
    hx = cuda.empty_like(x)
    f.hvec(x, hx)
    assert float((hx - st["energy"] * x).norm()) < 1e-5
    xm = cuda.empty_like(diags)
    sm = f.davidson(v0.clone(), diags, xm, tol=1e-6, maxiter=300, maxspace=maxspace, mixed=True)
    assert abs(sm["energy"] - e_ref) < 1e-8, (sm, e_ref)
    assert sm["sigma_fp32"] > 0 and sm["residual"] < 1e-6


@pytest.mark.parametrize("mixed,diag32", [(False, False), (True, False), (True, True)])
def test_block_davidson_lowest_two_roots(cuda, oracle, mixed, diag32):
    """Block Davidson for 2 roots (FP64, and FP32 storage with FP64 refinement, with an
    FP64 or FP32 diagonal) against the oracle's two lowest eigenvalues (scipy eigsh over
    the oracle sigma): energies within 1e-9, H x_i = E_i x_i, orthonormal Ritz vectors."""
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 9, 4, 4
    net = nw.hamiltonian_network(norb, seed=21)
    Bo, No = oracle.basis(norb, na, nb), oracle.network(net)
    e_ref = _lowest(oracle, Bo, No, k=2)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    diags = cuda.zeros(B.dim, dtype=cuda.float64, device="cuda")
    f.get_diags(diags)
    X = cuda.zeros((2, B.dim), dtype=cuda.float64, device="cuda")
    low = cuda.argsort(diags)[:2]
    X[0, low[0]] = 1.0
    X[1, low[1]] = 1.0
    d = diags.float() if diag32 else diags
    st = f.davidson_block(X, d, 2, tol=1e-6, maxiter=400, ncv=2, maxspace=8, mixed=mixed)
    assert st["converged"], st
    np.testing.assert_allclose(st["energies"], e_ref, rtol=0, atol=1e-9)
    if mixed:
        assert st["sigma_fp32"] > st["sigma_fp64"] > 0
    else:
        assert st["sigma_fp32"] == 0
    G = (X @ X.T).cpu().numpy()
    np.testing.assert_allclose(G, np.eye(2), atol=1e-10)
    for i in range(2):
        hx = cuda.empty_like(diags)
        f.hvec(X[i].contiguous(), hx)
        r = float((hx - st["energies"][i] * X[i]).norm())
        assert r < 2e-6, (i, r)


def test_block_davidson_rejects_bad_shapes(cuda):
    from binsim_b200 import cuotf, network as nw
    B = cuotf.CuBasis(6, 3, 3)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(nw.hamiltonian_network(6, seed=1)))
    d = cuda.ones(B.dim, dtype=cuda.float64, device="cuda")
    X = cuda.zeros((2, B.dim), dtype=cuda.float64, device="cuda")
    with pytest.raises(cuotf.CuOTFError):   # maxspace < ncv + nroots
        f.davidson_block(X, d, 2, ncv=2, maxspace=3)
    with pytest.raises(cuotf.CuOTFError):   # linearly dependent start vectors
        f.davidson_block(X, d, 2)
