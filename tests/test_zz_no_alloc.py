"""bsim_grad_noalloc: the gradient entry point that never allocates device
memory, for hosts that cannot call cudaMalloc while running (their memory pool
already owns the device, or an allocation's implicit synchronisation is not
acceptable).  It must give the same result as bsim_grad, call after call, even
though every call reuses one fixed scratch array inside the library.

Kept in a file that pytest collects last, so a failure here cannot hide the
results of the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cu_setup, dev, load_golden

pytestmark = pytest.mark.gpu


def test_noalloc_grad_matches_grad_on_consecutive_calls(cuda):
    from binsim_b200.cuotf import lib
    L = lib()
    z, ham, pool = load_golden("h8_4a4b")
    B, H, P, f = cu_setup(z, None, pool)
    x, y = dev(cuda, z["x"]), dev(cuda, z["y"])
    out = cuda.zeros(2, dtype=cuda.float64, device="cuda")
    stream = cuda.cuda.current_stream().cuda_stream
    cases = [(int(z["ops"][0]), float(z["thetas"][0])), (int(z["ops"][1]), float(z["thetas"][1]))]
    for idx, theta in cases:     # two calls in a row through the C-ABI
        assert L.bsim_grad(B.h, P.h, idx, theta, x.data_ptr(), y.data_ptr(), out.data_ptr(), stream) == 0
        assert L.bsim_grad_noalloc(B.h, P.h, idx, theta, x.data_ptr(), y.data_ptr(), out.data_ptr() + 8,
                                   stream) == 0
        cuda.cuda.synchronize()
        g, g_noalloc = out.cpu().numpy()
        assert abs(g_noalloc - g) <= 1e-12 * max(1.0, abs(g)), (idx, g, g_noalloc)


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
