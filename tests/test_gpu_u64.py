"""UInt64 strings: the same operators on UInt64 handles, including bases above
26 orbitals where strings are addressed by their colex rank (the reference's
dense 2^norb map does not exist there), against the oracle (whose basis
searches sorted UInt64 string lists, the reference's find_index rule)."""
import numpy as np
import pytest

from conftest import dev

pytestmark = pytest.mark.gpu


def random_network(norb, seed, ngroups=60, orbsym=None):
    """Seeded OTF network with groups of every type: X masks of 2 or 4 orbitals per
    spin, random Z masks and rank-1/2 weights."""
    from binsim_b200 import network as nw
    rng = np.random.default_rng(seed)

    def mask(k):
        bits = rng.choice(norb, size=k, replace=False)
        return int(sum(1 << int(b) for b in bits))

    def zs(n):
        return np.array([mask(int(rng.integers(0, 4))) for _ in range(n)], np.uint64)
    groups = [(0, 0, 2, zs(3), zs(3), rng.normal(size=(3, 2)), rng.normal(size=(3, 2)))]   # diagonal
    for g in range(ngroups):
        t = g % 3
        ax = mask(int(rng.choice([2, 4]))) if t in (0, 2) else 0
        bx = mask(int(rng.choice([2, 4]))) if t in (1, 2) else 0
        r = int(rng.integers(1, 3))
        na, nb = int(rng.integers(1, 4)), int(rng.integers(1, 4))
        groups.append((ax, bx, r, zs(na), zs(nb), rng.normal(size=(na, r)), rng.normal(size=(nb, r))))
    return nw._pack(groups, norb, orbsym)


def _check_all(cuda, oracle, norb, na, nb, net, orbsym=None, tsym=0, bits=64):
    from binsim_b200 import cuotf
    Bo = oracle.basis(norb, na, nb, orbsym=orbsym, total_sym=tsym)
    No = oracle.network(net)
    B = cuotf.CuBasis(norb, na, nb, orbsym=orbsym, total_sym=tsym, string_bits=bits)
    H = cuotf.CuNetwork(net, string_bits=bits)
    f = cuotf.CuOTFFunctions(B, H, H)
    assert B.dim == Bo.dim
    rng = np.random.default_rng(1)
    x, yv = rng.normal(size=B.dim), rng.normal(size=B.dim)
    xd = dev(cuda, x)
    y = cuda.empty_like(xd)
    f.hvec(xd, y)
    ref = oracle.hvec(Bo, No, x)
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))
    d = cuda.zeros_like(xd)
    f.get_diags(d)
    dref = oracle.diag(Bo, No)
    np.testing.assert_allclose(d.cpu().numpy(), dref, rtol=0, atol=1e-12 * max(1.0, np.abs(dref).max()))
    for g in range(1, net.ngs, 7):
        t = 0.37 + 0.01 * g
        v = dev(cuda, x)
        f.expm(g + 1, t, v)
        np.testing.assert_allclose(v.cpu().numpy(), oracle.expm(Bo, No, g, t, x), rtol=0, atol=1e-12)
        gr = f.grad(g + 1, t, dev(cuda, x), dev(cuda, yv))
        g0 = oracle.grad(Bo, No, g, t, x, yv)
        assert abs(gr - g0) < 1e-11 * max(1.0, abs(g0))
        l, r = dev(cuda, x), dev(cuda, yv)
        gb = f.backgrad(g + 1, t, l, r)
        gb0, l0, r0 = oracle.backgrad(Bo, No, g, t, x, yv)
        assert abs(gb - gb0) < 1e-11 * max(1.0, abs(gb0))
        np.testing.assert_allclose(l.cpu().numpy(), l0, rtol=0, atol=1e-12)
        np.testing.assert_allclose(r.cpu().numpy(), r0, rtol=0, atol=1e-12)
    th = rng.normal(size=net.ngs) * 0.3
    grads = cuda.zeros(net.ngs, dtype=cuda.float64, device="cuda")
    f.batchgrad(dev(cuda, x), dev(cuda, yv), grads, dev(cuda, th))
    gref = oracle.batchgrad(Bo, No, th, x, yv)
    np.testing.assert_allclose(grads.cpu().numpy(), gref, rtol=0, atol=1e-11 * max(1.0, np.abs(gref).max()))
    return B, f


def test_u64_handles_match_oracle_small(cuda, oracle):
    """UInt64 handles on a 10-orbital space (dense maps) give the oracle's results."""
    _check_all(cuda, oracle, 10, 4, 5, random_network(10, seed=3))


def test_u64_ranked_strings_above_32_orbitals(cuda, oracle):
    """34 orbitals, 2a+2b (561^2 determinants): UInt64 strings addressed by colex rank."""
    B, f = _check_all(cuda, oracle, 34, 2, 2, random_network(34, seed=5, ngroups=90))
    # the HF determinant and a high-orbital determinant are found by their strings
    assert B.find_det(0b11, 0b11) == 0
    assert B.find_det((1 << 33) | (1 << 32), (1 << 33) | 1) >= 0


def test_u64_ranked_strings_with_symmetry_blocks(cuda, oracle):
    """28 orbitals (ranked addressing) split into irreps: indices inside each irrep's list."""
    norb = 28
    orbsym = np.array([p % 4 for p in range(norb)], np.int64)
    _check_all(cuda, oracle, norb, 2, 3, random_network(norb, seed=9, ngroups=60, orbsym=orbsym),
               orbsym=orbsym, tsym=1)


def test_u64_rejects_mixed_string_types(cuda):
    from binsim_b200 import cuotf
    B64 = cuotf.CuBasis(10, 4, 4, string_bits=64)
    H32 = cuotf.CuNetwork(random_network(10, seed=1), string_bits=32)
    x = cuda.zeros(B64.dim, dtype=cuda.float64, device="cuda")
    f = cuotf.CuOTFFunctions(B64, H32)
    with pytest.raises(cuotf.CuOTFError):
        f.hvec(x, x.clone())
