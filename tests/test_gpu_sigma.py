"""sigma = H c and diag(H) on the GPU against the oracle and the golden fixtures."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, cu_setup, dev, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_sigma_and_diag_match_golden(cuda, name):
    z, ham, pool = load_golden(name)
    B, H, P, f = cu_setup(z, ham, None)
    assert B.dim == int(z["dim"])
    x = dev(cuda, z["x"])
    y = cuda.empty_like(x)
    f.hvec(x, y)
    scale = np.abs(z["sigma"]).max()
    np.testing.assert_allclose(y.cpu().numpy(), z["sigma"], rtol=0, atol=1e-12 * scale)
    d = cuda.zeros_like(x)
    f.get_diags(d)
    np.testing.assert_allclose(d.cpu().numpy(), z["diag"], rtol=0, atol=1e-12 * np.abs(z["diag"]).max())
    assert B.hf_index() == int(z["hf"])


@pytest.mark.parametrize("norb,na,nb,orbsym,tsym", [
    (10, 5, 5, None, 0),
    (10, 4, 5, [0, 1, 2, 3, 0, 1, 2, 3, 0, 1], 3),
    (11, 3, 6, None, 0),
])
def test_sigma_matches_oracle(cuda, oracle, norb, na, nb, orbsym, tsym):
    from binsim_b200 import cuotf, network as nw
    osym = np.zeros(norb, np.int64) if orbsym is None else np.asarray(orbsym, np.int64)
    net = nw.hamiltonian_network(norb, seed=norb + na)
    net.orbsym = osym
    Bo = oracle.basis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    No = oracle.network(net)
    B = cuotf.CuBasis(norb, na, nb, orbsym=osym, total_sym=tsym, num_irreps=4)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    assert B.dim == Bo.dim
    path, why, nres = f.sigma_path()
    assert path == (0 if orbsym is not None else 1), (path, why)
    x = np.random.default_rng(norb).normal(size=B.dim)
    ref = oracle.hvec(Bo, No, x)
    y = cuda.empty(B.dim, dtype=cuda.float64, device="cuda")
    f.hvec(dev(cuda, x), y)
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    # FP32 bulk: per-chunk FP32 sums, FP64 across chunks
    ym = cuda.empty_like(y)
    f.hvec_mixed(dev(cuda, x), ym)
    err = np.abs(ym.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 2e-6, err
    # FP32 input variant
    from binsim_b200.cuotf import lib
    y32 = cuda.empty_like(y)
    assert lib().bsim_hvec_f32in(B.h, f.ham.h, dev(cuda, x, cuda.float32).data_ptr(), y32.data_ptr(), None) == 0
    cuda.cuda.synchronize()
    assert np.abs(y32.cpu().numpy() - ref).max() / np.abs(ref).max() < 2e-6


def test_sigma_is_symmetric_operator(cuda):
    """<u|H v> == <H u|v> on a 12-orbital case (size-independent property)."""
    from binsim_b200 import cuotf, network as nw
    net = nw.hamiltonian_network(12, seed=0)
    B = cuotf.CuBasis(12, 6, 6)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    g = cuda.Generator(device="cuda").manual_seed(0)
    u = cuda.randn(B.dim, dtype=cuda.float64, device="cuda", generator=g)
    v = cuda.randn(B.dim, dtype=cuda.float64, device="cuda", generator=g)
    hu, hv = cuda.empty_like(u), cuda.empty_like(v)
    f.hvec(u, hu)
    f.hvec(v, hv)
    a, b = float(u @ hv), float(hu @ v)
    assert abs(a - b) < 1e-10 * max(abs(a), 1.0)
    # linearity: H(2u + 3v) = 2Hu + 3Hv
    w = 2 * u + 3 * v
    hw = cuda.empty_like(w)
    f.hvec(w, hw)
    assert float((hw - 2 * hu - 3 * hv).abs().max()) < 1e-10 * float(hw.abs().max())


def test_reference_host_handles(cuda, reflibs):
    """build_basisdev_f64 / build_networkdev_f64 accept the reference's host handles."""
    from binsim_b200 import cuotf, network as nw
    L = cuotf.lib()
    norb, na, nb = 8, 4, 3
    osym = np.array([0, 1, 0, 1, 2, 3, 2, 3], np.int64)
    net = nw.hamiltonian_network(norb, seed=4)
    net.orbsym = osym
    rb, dim = reflibs.basis(norb, na, nb, orbsym=osym, total_sym=2, num_irreps=4)
    rn = reflibs.network(net)
    db = L.build_basisdev_f64(rb)
    dn = L.build_networkdev_f64(rn)
    assert db and dn
    x = np.random.default_rng(2).normal(size=dim)
    xd = dev(cuda, x)
    yd = cuda.zeros_like(xd)
    L.hvec_cuda(db, dn, xd.data_ptr(), yd.data_ptr())
    L.sync_device_cuda()
    ref = reflibs.hvec(rb, rn, x, dim)
    np.testing.assert_allclose(yd.cpu().numpy(), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    d = cuda.zeros_like(xd)
    L.get_diags_elements_cuda(db, dn, d.data_ptr())
    L.sync_device_cuda()
    np.testing.assert_allclose(d.cpu().numpy(), reflibs.diag_elems(rb, rn, dim), atol=1e-12)
    L.destroy_networkdev_f64(dn)
    L.destroy_basisdev_f64(db)


@pytest.mark.parametrize("mixed", [False, True])
def test_column_bands_reassemble_sigma(cuda, mixed):
    """Column-band sigma (the per-rank unit of the sharded path): bands computed
    separately reproduce the whole sigma (to rounding: a band sums the same-spin
    doubles of the beta side through the row lists, a whole sigma through the
    intermediate strings), every split gives the same bits, and a call leaves the
    columns outside its band untouched."""
    import math
    from binsim_b200 import cuotf, network as nw
    from binsim_b200.shard import column_bands
    norb, na, nb = 11, 4, 5                      # 330 x 462 determinants
    net = nw.hamiltonian_network(norb, seed=12)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    assert f.sigma_path()[0] == 1
    nA, nB = math.comb(norb, na), math.comb(norb, nb)
    x = dev(cuda, np.random.default_rng(4).normal(size=B.dim))
    full = cuda.empty_like(x)
    (f.hvec_mixed if mixed else f.hvec)(x, full)
    first = None
    for world in (2, 3, 4):
        y = cuda.full_like(x, float("nan"))
        for lo, hi in column_bands(nB, world):
            before = y.clone()
            f.hvec_cols(x, y, lo, hi, mixed=mixed)
            changed = (y != before) & ~(y.isnan() & before.isnan())
            outside = changed.view(nA, nB).clone()
            outside[:, lo:hi] = False
            assert not bool(outside.any()), "wrote outside its column band"
        tol = (2e-6 if mixed else 1e-13) * float(full.abs().max())
        assert float((y - full).abs().max()) <= tol
        if first is None:
            first = y.clone()
        assert cuda.equal(y, first)
    # misaligned band start is an argument error
    with pytest.raises(cuotf.CuOTFError):
        f.hvec_cols(x, y, 5, 40)


def sparse_hamiltonian_network(norb, seed, nquads=1500):
    """Jordan-Wigner network of a Hamiltonian with a random symmetric one-body part and
    a few random 8-fold-symmetric two-body integrals (quick to build at any norb)."""
    from binsim_b200 import network as nw
    rng = np.random.default_rng(seed)
    h = rng.normal(scale=0.1, size=(norb, norb))
    h = h + h.T
    g = np.zeros((norb,) * 4)
    for _ in range(nquads):
        p, q, r, s = rng.integers(0, norb, size=4)
        v = rng.normal(scale=0.05)
        for (a, b, c, d) in ((p, q, r, s), (q, p, s, r), (r, s, p, q), (s, r, q, p),
                             (q, p, r, s), (p, q, s, r), (s, r, p, q), (r, s, q, p)):
            g[a, b, c, d] = v   # (pq|rs) symmetric under the chemist's 8-fold permutations
    eri = np.einsum("psqr->pqrs", g)   # passed as g[p,q,r,s] = (ps|qr)
    x, z, c = nw.jw_hamiltonian_terms(h, eri, 0.0)
    ax, az, bx, bz = nw.split_aabb(x, z, norb)
    return nw.compress_groups(ax, az, bx, bz, c, norb)


@pytest.mark.parametrize("norb,na,nb,bits", [(18, 5, 2, 32), (28, 3, 1, 32), (28, 3, 1, 64)])
def test_structured_sigma_two_passes_and_streamed_lam(cuda, norb, na, nb, bits):
    """More than 64 connected alpha singles per string (two GEMM passes), and at 28
    orbitals a Lam too large for shared memory (streamed per F chunk) with ranked string
    addressing, against the generic tile kernel (itself oracle-tested)."""
    from binsim_b200 import cuotf
    net = sparse_hamiltonian_network(norb, seed=norb + na)
    B = cuotf.CuBasis(norb, na, nb, string_bits=bits)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net, string_bits=bits))
    path = f.sigma_path()
    assert path[0] == 1, path
    x = dev(cuda, np.random.default_rng(2).normal(size=B.dim))
    y = cuda.empty_like(x)
    y_ref = cuda.empty_like(x)
    f.hvec(x, y)
    f.hvec_tiles(x, y_ref, 0, f.num_tiles())
    scale = float(y_ref.abs().max())
    assert float((y - y_ref).abs().max()) <= 1e-12 * scale
    f.hvec_mixed(x, y)
    assert float((y - y_ref).abs().max()) <= 2e-6 * scale


@pytest.mark.parametrize("mixed", [False, True])
def test_mixed_gemm_source_row_in_global_memory(cuda, oracle, monkeypatch, mixed):
    """The mixed GEMM reading its source row from global memory (the kernel shape used
    when a beta row exceeds shared memory: FP64 at 18 orbitals, 8 electrons) against
    the row staged on chip and the oracle's sigma.  FP64: the same bits (both run the
    same DMMA sums in the same order).  FP32 bulk: the on-chip shape runs on the
    tcgen05 tensor cores (TF32 hi/lo products) and the global-row shape on the CUDA
    cores, so they agree to the FP32-bulk tolerance, 2e-6 x max|sigma|."""
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 11, 5, 5
    net = nw.hamiltonian_network(norb, seed=5)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    assert f.sigma_path()[0] == 1
    xh = np.random.default_rng(3).normal(size=B.dim)
    x = dev(cuda, xh)
    y_chip, y_glob = cuda.empty_like(x), cuda.empty_like(x)
    run = f.hvec_mixed if mixed else f.hvec
    run(x, y_chip)
    monkeypatch.setenv("BSIM_MIXED_ROW_SMEM", "1")
    run(x, y_glob)
    monkeypatch.delenv("BSIM_MIXED_ROW_SMEM")
    ref = oracle.hvec(oracle.basis(norb, na, nb), oracle.network(net), xh)
    tol = 2e-6 if mixed else 1e-12
    if mixed:
        assert float((y_chip - y_glob).abs().max()) <= tol * np.abs(ref).max()
    else:
        assert cuda.equal(y_chip, y_glob)
    assert np.abs(y_glob.cpu().numpy() - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("norb,na,nb", [(11, 5, 5), (12, 6, 5), (13, 3, 4)])
@pytest.mark.parametrize("row_on_chip", [True, False])
def test_fp64_mixed_gemm_kernels_agree(cuda, oracle, monkeypatch, norb, na, nb, row_on_chip):
    """The FP64 mixed GEMM with per-warp B fragments (default; m16n8k4 DMMA tiles)
    against the kernel with a shared X slice (BSIM_MIXED_DMMA=0; m8n8k4 tiles):
    the same products in the same K order, to 1e-13 x max|sigma| (the two MMA
    shapes may round their 4-term sums differently); both against the oracle at
    1e-12 x max|sigma|.  row_on_chip False reads the source row from global
    memory (BSIM_MIXED_ROW_SMEM=1).  Connected rows per pass 30, 36 / 30 and 30:
    partial 16-row tiles."""
    from binsim_b200 import cuotf, network as nw
    net = nw.hamiltonian_network(norb, seed=9)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    assert f.sigma_path()[0] == 1
    xh = np.random.default_rng(norb).normal(size=B.dim)
    x = dev(cuda, xh)
    if not row_on_chip:
        monkeypatch.setenv("BSIM_MIXED_ROW_SMEM", "1")
    y_new, y_old = cuda.empty_like(x), cuda.empty_like(x)
    f.hvec(x, y_new)
    monkeypatch.setenv("BSIM_MIXED_DMMA", "0")
    f.hvec(x, y_old)
    ref = oracle.hvec(oracle.basis(norb, na, nb), oracle.network(net), xh)
    assert float((y_new - y_old).abs().max()) <= 1e-13 * np.abs(ref).max()
    assert np.abs(y_new.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("norb,na,nb", [(11, 5, 5), (12, 6, 5), (12, 2, 4)])
def test_fp64_intermediate_gemm_kernels_agree(cuda, oracle, monkeypatch, norb, na, nb):
    """The FP64 intermediate-string GEMM with per-warp B fragments (the default)
    against the shared-slice kernel (BSIM_RI_DMMA=0), both against the oracle at
    1e-12 x max|sigma|.  Pairs outside an intermediate 28 / 28, 28 / 36 and 66 / 45:
    the per-warp kernel's m16n8k8 steps with an m16n8k4 step for an odd last group
    of 4 rows (28, 36, 66) and without one (45); both kernels add over the same K
    order (the shared-slice kernel computes rows 64.. with scalar FMAs)."""
    from binsim_b200 import cuotf, network as nw
    net = nw.hamiltonian_network(norb, seed=11)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    path = f.sigma_path()
    assert path[0] == 1 and "ri-alpha" in path[1], path
    xh = np.random.default_rng(norb + 1).normal(size=B.dim)
    x = dev(cuda, xh)
    y_new, y_old = cuda.empty_like(x), cuda.empty_like(x)
    monkeypatch.delenv("BSIM_RI_DMMA", raising=False)
    f.hvec(x, y_new)
    monkeypatch.setenv("BSIM_RI_DMMA", "0")
    f.hvec(x, y_old)
    ref = oracle.hvec(oracle.basis(norb, na, nb), oracle.network(net), xh)
    scale = np.abs(ref).max()
    assert float((y_new - y_old).abs().max()) <= 1e-12 * scale
    assert np.abs(y_new.cpu().numpy() - ref).max() <= 1e-12 * scale


@pytest.mark.parametrize("norb,na,nb", [(13, 3, 3), (13, 3, 4), (14, 4, 4)])
def test_intermediate_string_gemm_beyond_64_pairs(cuda, oracle, norb, na, nb):
    """66 pairs outside each (n-2)-electron intermediate string (the count at 18 orbitals,
    8 electrons): rows 64-65 of the intermediate-string GEMM come from the tail FMAs.
    Against the oracle, and against the same sigma with those doubles in the row lists."""
    from binsim_b200 import cuotf, network as nw
    net = nw.hamiltonian_network(norb, seed=norb + nb)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    path, why, _ = f.sigma_path()
    assert path == 1 and "ri-alpha" in why and "ri-beta" in why, why
    xh = np.random.default_rng(norb).normal(size=B.dim)
    x = dev(cuda, xh)
    y = cuda.empty_like(x)
    f.hvec(x, y)
    ref = oracle.hvec(oracle.basis(norb, na, nb), oracle.network(net), xh)
    scale = np.abs(ref).max()
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=0, atol=1e-12 * scale)
    ym = cuda.empty_like(x)
    f.hvec_mixed(x, ym)
    assert np.abs(ym.cpu().numpy() - ref).max() <= 2e-6 * scale


def test_hvec_host_pipeline(cuda):
    """bsim_hvec_host over several distinct host vectors (pinned and pageable, the same
    output buffer twice) gives the device sigma of each, bit for bit."""
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 10, 5, 4
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(nw.hamiltonian_network(norb, seed=3)))
    rng = np.random.default_rng(0)
    xs = [rng.normal(size=B.dim) for _ in range(5)]
    srcs = [cuda.from_numpy(xs[0]).pin_memory(), cuda.from_numpy(xs[1]).pin_memory(), xs[2], xs[3],
            cuda.from_numpy(xs[4]).pin_memory()]
    outs = [cuda.empty(B.dim, dtype=cuda.float64).pin_memory() for _ in range(3)] + [np.zeros(B.dim)]
    dsts = [outs[0], outs[1], outs[2], outs[3], outs[0]]   # slot 0 is written twice, last by step 4
    for mixed in (False, True):
        f.hvec_host(srcs, dsts, mixed=mixed)
        for k in (1, 2, 3, 4):
            y = cuda.empty(B.dim, dtype=cuda.float64, device="cuda")
            (f.hvec_mixed if mixed else f.hvec)(dev(cuda, xs[k]), y)
            got = dsts[k].numpy() if hasattr(dsts[k], "numpy") else dsts[k]
            assert np.array_equal(got, y.cpu().numpy()), (mixed, k)
    f.hvec_host([], [])


def test_fp32_mixed_gemm_80_row_tile_matches_64_row_passes(cuda, monkeypatch):
    """65..80 connected alpha singles (18 orbitals, 5 alpha electrons: 65): the FP32 80-row
    tile gives the same bits as a 64-row and a 16-row pass (each output accumulates the
    same FMAs in the same order).  CUDA-core kernels (BSIM_MIXED_TC=0): the tensor-core
    kernel takes this size otherwise."""
    from binsim_b200 import cuotf
    monkeypatch.setenv("BSIM_MIXED_TC", "0")
    net = sparse_hamiltonian_network(18, seed=23)
    B = cuotf.CuBasis(18, 5, 2)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    assert f.sigma_path()[0] == 1
    x = dev(cuda, np.random.default_rng(4).normal(size=B.dim))
    y80, y64 = cuda.empty_like(x), cuda.empty_like(x)
    f.hvec_mixed(x, y80)
    monkeypatch.setenv("BSIM_MIXED_ROWS80", "0")
    f.hvec_mixed(x, y64)
    monkeypatch.delenv("BSIM_MIXED_ROWS80")
    assert cuda.equal(y80, y64)
