"""bsim_grad_noalloc: the gradient entry point that never allocates device
memory, for hosts that cannot call cudaMalloc while running (their memory pool
already owns the device, or an allocation's implicit synchronisation is not
acceptable).  It must give the same result as bsim_grad, call after call, even
though every call reuses one fixed scratch array inside the library.

Each case calls it FIRST on freshly created handles (before any bsim_grad could
have built per-network pair lists) and reads the library's allocation counter
around those calls: it must not move.  Then bsim_grad runs on the same inputs
for comparison, and a further no-allocation call (which may now use the lists
bsim_grad built) must agree as well.

Kept in a file that pytest collects last, so a failure here cannot hide the
results of the other GPU tests.
"""
import numpy as np
import pytest

from conftest import cu_setup, dev, load_golden

pytestmark = pytest.mark.gpu


def _compare_first_calls(cuda, L, B, P, x, y, cases):
    out = cuda.zeros(3 * len(cases), dtype=cuda.float64, device="cuda")
    stream = cuda.cuda.current_stream().cuda_stream
    cuda.cuda.synchronize()
    before = L.bsim_device_alloc_count()
    for k, (idx, theta) in enumerate(cases):     # consecutive calls through the C-ABI, fresh handles
        assert L.bsim_grad_noalloc(B.h, P.h, idx, theta, x.data_ptr(), y.data_ptr(), out.data_ptr() + 8 * k,
                                   stream) == 0, L.bsim_last_error()
    cuda.cuda.synchronize()
    assert L.bsim_device_alloc_count() == before, "bsim_grad_noalloc allocated device memory"
    n = len(cases)
    for k, (idx, theta) in enumerate(cases):
        assert L.bsim_grad(B.h, P.h, idx, theta, x.data_ptr(), y.data_ptr(), out.data_ptr() + 8 * (n + k),
                           stream) == 0
    before = L.bsim_device_alloc_count()
    for k, (idx, theta) in enumerate(cases):     # again, after bsim_grad may have built pair lists
        assert L.bsim_grad_noalloc(B.h, P.h, idx, theta, x.data_ptr(), y.data_ptr(),
                                   out.data_ptr() + 8 * (2 * n + k), stream) == 0
    cuda.cuda.synchronize()
    assert L.bsim_device_alloc_count() == before
    g = out.cpu().numpy().reshape(3, n)
    tol = 1e-12 * np.maximum(1.0, np.abs(g[1]))
    assert np.all(np.abs(g[0] - g[1]) <= tol), g
    assert np.all(np.abs(g[2] - g[1]) <= tol), g


@pytest.mark.parametrize("case", ["h8_4a4b", "h8_4a3b_sym"])
def test_noalloc_grad_first_call_matches_grad(cuda, case):
    """Single-block basis (the pair-list path after bsim_grad) and a symmetry-
    blocked basis (the row kernel, one partial sum per alpha string and block)."""
    from binsim_b200.cuotf import lib
    L = lib()
    z, ham, pool = load_golden(case)
    B, H, P, f = cu_setup(z, None, pool)
    x, y = dev(cuda, z["x"]), dev(cuda, z["y"])
    ops, th = z["ops"], z["thetas"]
    cases = [(int(ops[i]), float(th[i])) for i in range(min(4, len(ops)))]
    _compare_first_calls(cuda, L, B, P, x, y, cases)


def test_noalloc_grad_uint64_strings(cuda):
    """UInt64 handles above the dense-map limit (28 orbitals, colex-ranked strings)."""
    from binsim_b200 import cuotf, network as nw
    L = cuotf.lib()
    norb, na, nb = 28, 2, 2
    # spin-orbital generators t - t^dagger (alpha = 2p, beta = 2p + 1): two
    # singles, an alpha-beta double and two same-spin doubles
    comps = [([40], [6]), ([41], [7]), ([50, 9], [2, 53]), ([54, 44], [4, 10]), ([55, 47], [27, 5])]
    parts = [nw._component(c, a, norb) for c, a in comps]
    cat = lambda k: np.concatenate([p[k] for p in parts])
    pool = nw._compress_each(cat(0), cat(1), cat(2), cat(3), cat(4), [len(p[4]) for p in parts], norb)
    B = cuotf.CuBasis(norb, na, nb, string_bits=64)
    P = cuotf.CuNetwork(pool, string_bits=64)
    rng = np.random.default_rng(5)
    x, y = dev(cuda, rng.normal(size=B.dim)), dev(cuda, rng.normal(size=B.dim))
    cases = [(g, 0.1 + 0.05 * g) for g in range(pool.ngs)]
    _compare_first_calls(cuda, L, B, P, x, y, cases)


def test_noalloc_rejects_oversized_basis(cuda):
    from binsim_b200 import cuotf, network as nw
    L = cuotf.lib()
    # C(20, 10) = 184756 alpha strings: more partial sums than the fixed scratch holds
    B = cuotf.CuBasis(20, 10, 1)
    P = cuotf.CuNetwork(nw.ucc_pool(4).network)
    v = cuda.zeros(B.dim, dtype=cuda.float64, device="cuda")
    out = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    st = L.bsim_grad_noalloc(B.h, P.h, 0, 0.1, v.data_ptr(), v.data_ptr(), out.data_ptr(), None)
    assert st == -7
    assert b"fixed scratch" in L.bsim_last_error()
