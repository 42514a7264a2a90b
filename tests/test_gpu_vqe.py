"""VQE energy + adjoint gradient against the oracle sweep and finite differences."""
import numpy as np
import pytest

from conftest import dev

pytestmark = pytest.mark.gpu


def _oracle_energy_grad(oracle, Bo, Ho, Po, op_idx, param_idx, thetas, ref_idx, ref_val):
    """energy_objective, jl/vqe.jl:1-21, on the oracle."""
    lv = np.zeros(Bo.dim)
    lv[ref_idx] = ref_val
    for i, p in zip(op_idx, param_idx):
        lv = oracle.expm(Bo, Po, int(i), thetas[p], lv)
    rv = oracle.hvec(Bo, Ho, lv)
    ll = lv @ lv
    E = (lv @ rv) / ll
    grad = np.zeros(len(thetas))
    for i, p in zip(op_idx[::-1], param_idx[::-1]):
        g, lv, rv = oracle.backgrad(Bo, Po, int(i), thetas[p], lv, rv)
        grad[p] += 2 * g / ll
    return E, grad


@pytest.mark.parametrize("ckpt", [0, 4])
def test_adjoint_gradient_matches_oracle(cuda, oracle, ckpt):
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 8, 4, 4
    ham, pool = nw.hamiltonian_network(norb, seed=3), nw.ucc_pool(norb)
    op_idx, param_idx, th = nw.draw_generators(pool, 30, seed=7, amp_sigma=0.2)
    Bo, Ho, Po = oracle.basis(norb, na, nb), oracle.network(ham), oracle.network(pool.network)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(ham), cuotf.CuNetwork(pool.network))
    ref_idx, ref_val = np.array([B.hf_index()]), np.array([1.0])
    E0, g0 = _oracle_energy_grad(oracle, Bo, Ho, Po, op_idx, param_idx, th, ref_idx, ref_val)
    lv = cuda.empty(B.dim, dtype=cuda.float64, device="cuda")
    rv = cuda.empty_like(lv)
    E, g, var = f.energy_grad(op_idx, param_idx, th, ref_idx, ref_val, lv, rv, ckpt_every=ckpt)
    assert abs(E - E0) < 1e-12
    np.testing.assert_allclose(g, g0, rtol=0, atol=1e-11)
    assert var >= 0.0
    # after the sweep lv holds the uncomputed reference state
    ref = np.zeros(B.dim); ref[ref_idx] = ref_val
    assert np.abs(lv.cpu().numpy() - ref).max() < 1e-12


def test_adjoint_gradient_matches_central_differences(cuda):
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 7, 3, 4
    ham, pool = nw.hamiltonian_network(norb, seed=8), nw.ucc_pool(norb)
    op_idx, param_idx, th = nw.draw_generators(pool, 12, seed=2, amp_sigma=0.3)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(ham), cuotf.CuNetwork(pool.network))
    ref_idx, ref_val = np.array([B.hf_index()]), np.array([1.0])
    lv = cuda.empty(B.dim, dtype=cuda.float64, device="cuda")
    rv = cuda.empty_like(lv)
    E, g, _ = f.energy_grad(op_idx, param_idx, th, ref_idx, ref_val, lv, rv, ckpt_every=3)

    def energy(t):
        f.prepare_state(op_idx, param_idx, t, ref_idx, ref_val, lv)
        f.hvec(lv, rv)
        return float(lv @ rv) / float(lv @ lv)
    h = 1e-5
    for p in range(len(th)):
        tp, tm = th.copy(), th.copy()
        tp[p] += h; tm[p] -= h
        fd = (energy(tp) - energy(tm)) / (2 * h)
        assert abs(fd - g[p]) < 1e-7, (p, fd, g[p])
