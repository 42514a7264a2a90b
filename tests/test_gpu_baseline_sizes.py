"""Parity at the benchmark sizes, against the reference's own compiled CPU library
(libotf_native built from the reference sources into oracle/_ref).

* 12 orbitals 6a+6b (853,776 determinants, the plain FP64 FCI Davidson size):
  sigma (FP64 and FP32 bulk) and diag(H) of the seeded synthetic Hamiltonian,
  through the library's own handles and through the reference's host handles
  (build_basisdev_f64 / build_networkdev_f64), against hvec_gather_contract_otf_f64
  and get_diags_elements_f64 (op/hvec.hpp:481-554).
* 14 orbitals 7a+7b (11,778,624 determinants, the VQE size): expm, grad and
  backgrad of pool generators of every excitation kind against
  expm_contract_otf_f64, grad_contract_otf_f64 and backgrad_contract_otf_f64
  (op/expm.hpp:374-438, op/grad.hpp:397-465, op/backgrad.hpp:406-474).

Tolerances: FP64 sigma and diagonal 1e-12 x max|sigma|; FP32-bulk sigma
2e-6 x max|sigma|; the Givens updates 1e-13 absolute on unit vectors; gradients
1e-12 relative (1e-12 absolute floor).
"""
import numpy as np
import pytest

from conftest import dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h12(reflibs):
    from binsim_b200 import network as nw
    net = nw.hamiltonian_network(12, seed=0)
    rb, dim = reflibs.basis(12, 6, 6)
    rn = reflibs.network(net)
    x = np.random.default_rng(1).normal(size=dim)
    x /= np.linalg.norm(x)
    return net, rb, rn, dim, x, reflibs.hvec(rb, rn, x, dim), reflibs.diag_elems(rb, rn, dim)


def test_sigma_and_diag_match_reference_at_12_orbitals(cuda, h12):
    from binsim_b200 import cuotf
    net, rb, rn, dim, x, yref, dref = h12
    assert dim == 924 ** 2
    B = cuotf.CuBasis(12, 6, 6)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    xd = dev(cuda, x)
    y = cuda.empty_like(xd)
    scale = np.abs(yref).max()
    f.hvec(xd, y)
    assert np.abs(y.cpu().numpy() - yref).max() <= 1e-12 * scale
    f.hvec_mixed(xd, y)
    assert np.abs(y.cpu().numpy() - yref).max() <= 2e-6 * scale
    d = cuda.zeros_like(xd)
    f.get_diags(d)
    assert np.abs(d.cpu().numpy() - dref).max() <= 1e-12 * np.abs(dref).max()


def test_reference_host_handles_at_12_orbitals(cuda, h12):
    """The drop-in path: the reference's host BasisManager / Network_OTF handles
    through the legacy entry points, as jl/cuda/cunetwork.jl calls them."""
    from binsim_b200 import cuotf
    net, rb, rn, dim, x, yref, dref = h12
    L = cuotf.lib()
    db, dn = L.build_basisdev_f64(rb), L.build_networkdev_f64(rn)
    assert db and dn
    try:
        xd = dev(cuda, x)
        y = cuda.empty_like(xd)
        L.hvec_cuda(db, dn, xd.data_ptr(), y.data_ptr())
        d = cuda.zeros_like(xd)
        L.get_diags_elements_cuda(db, dn, d.data_ptr())
        L.sync_device_cuda()
        assert np.abs(y.cpu().numpy() - yref).max() <= 1e-12 * np.abs(yref).max()
        assert np.abs(d.cpu().numpy() - dref).max() <= 1e-12 * np.abs(dref).max()
    finally:
        L.destroy_networkdev_f64(dn)
        L.destroy_basisdev_f64(db)


def test_pair_operators_match_reference_at_14_orbitals(cuda, reflibs):
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 14, 7, 7
    pool = nw.ucc_pool(norb, native=True).network
    rb, dim = reflibs.basis(norb, na, nb)
    rp = reflibs.network(pool)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, None, cuotf.CuNetwork(pool))
    rng = np.random.default_rng(3)
    l = rng.normal(size=dim)
    l /= np.linalg.norm(l)
    r = rng.normal(size=dim)
    r /= np.linalg.norm(r)
    types = pool.type_codes()
    # two groups of each kind: pure alpha, pure beta, mixed
    picks = []
    for t in (1, 2, 3):
        g = np.flatnonzero(types == t)
        picks += [int(g[0]), int(g[len(g) // 2])]
    for k, g in enumerate(picks):
        theta = 0.3 - 0.11 * k
        v = dev(cuda, l)
        f.expm(g + 1, theta, v)                          # 1-based, as the Julia closures
        assert np.abs(v.cpu().numpy() - reflibs.expm(rb, rp, g, theta, l)).max() <= 1e-13
        gr = f.grad(g + 1, theta, dev(cuda, l), dev(cuda, r))
        gref = reflibs.grad(rb, rp, g, theta, l, r)
        assert abs(gr - gref) <= 1e-12 * max(1.0, abs(gref))
        lv, rv = dev(cuda, l), dev(cuda, r)
        bg = f.backgrad(g + 1, theta, lv, rv)
        bref, lref, rref = reflibs.backgrad(rb, rp, g, theta, l, r)
        assert abs(bg - bref) <= 1e-12 * max(1.0, abs(bref))
        assert np.abs(lv.cpu().numpy() - lref).max() <= 1e-13
        assert np.abs(rv.cpu().numpy() - rref).max() <= 1e-13
