"""FP32-bulk sigma whose mixed part and intermediate-string (same-spin doubles)
product run on the tcgen05 tensor cores (kind::tf32
with every operand split into TF32 hi + lo, FP32 accumulation in tensor memory),
against the oracle's FP64 sigma.  The sizes cover ragged K slices (F excitations
not a multiple of the 40-row slice or of the MMA's K step of 8), ragged column
chunks (beta strings not a multiple of 128) and unequal alpha / beta counts.

The kernel runs with the source row staged on chip and, selected by
BSIM_MIXED_TC, read from global memory with 64 or 80 excitations per pass.

Tolerance: 2e-6 x max|sigma|, the FP32-bulk bar of the other sigma tests.  The
kernels' bounded waits must never have given up (bsim_tensor_core_timeouts)."""
import ctypes as C

import numpy as np
import pytest

from conftest import dev

pytestmark = pytest.mark.gpu


def _timeouts(L, reset=False):
    n = C.c_int32()
    assert L.bsim_tensor_core_timeouts(C.byref(n), 1 if reset else 0) == 0
    return n.value


@pytest.mark.parametrize("mode", ["", "global64", "global80"])
@pytest.mark.parametrize("norb,na,nb", [(8, 4, 4), (10, 5, 5), (11, 5, 6), (12, 6, 6)])
def test_fp32_bulk_sigma_on_tensor_cores_matches_oracle(cuda, oracle, monkeypatch, norb, na, nb, mode):
    """mode: the automatic kernel choice (source row on chip at these sizes), or
    the source row read from global memory with 64 or 80 excitations per pass
    (the 18-orbital shapes, where the row does not fit on chip)."""
    from binsim_b200 import cuotf, network as nw
    monkeypatch.setenv("BSIM_MIXED_TC", mode)
    L = cuotf.lib()
    _timeouts(L, reset=True)
    net = nw.hamiltonian_network(norb, seed=2)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    assert f.sigma_path()[0] == 1   # the structured path, whose mixed GEMM this is
    x = np.random.default_rng(norb).normal(size=B.dim)
    x /= np.linalg.norm(x)
    ref = oracle.hvec(oracle.basis(norb, na, nb), oracle.network(net), x)
    xd = dev(cuda, x)
    y = cuda.empty_like(xd)
    for _ in range(2):   # a second call reuses the plan and the scratch
        f.hvec_mixed(xd, y)
        cuda.cuda.synchronize()
        assert np.abs(y.cpu().numpy() - ref).max() <= 2e-6 * np.abs(ref).max()
    assert _timeouts(L) == 0


def test_tensor_core_and_cuda_core_fp32_paths_agree(cuda, monkeypatch):
    """The same FP32-bulk sigma through the tensor-core kernel and through the
    CUDA-core kernel (BSIM_MIXED_TC=0) agree to the FP32-bulk tolerance, and both
    agree with the FP64 sigma to it."""
    from binsim_b200 import cuotf, network as nw
    norb, na, nb = 12, 6, 5
    net = nw.hamiltonian_network(norb, seed=7)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    x = dev(cuda, np.random.default_rng(2).normal(size=B.dim))
    y_tc, y_cc, y64 = (cuda.empty_like(x) for _ in range(3))
    f.hvec_mixed(x, y_tc)
    f.hvec(x, y64)
    monkeypatch.setenv("BSIM_MIXED_TC", "0")
    f.hvec_mixed(x, y_cc)
    scale = float(y64.abs().max())
    assert float((y_tc - y_cc).abs().max()) <= 2e-6 * scale
    assert float((y_tc - y64).abs().max()) <= 2e-6 * scale
    assert float((y_cc - y64).abs().max()) <= 2e-6 * scale


@pytest.mark.parametrize("norb,na,nb", [(8, 4, 4), (10, 5, 5), (11, 3, 3), (12, 3, 3), (13, 3, 3), (12, 2, 4)])
def test_intermediate_string_gemm_on_tensor_cores(cuda, oracle, monkeypatch, norb, na, nb):
    """The same-spin doubles through intermediate strings on the tensor cores, at
    every accumulator width: pairs outside an intermediate 15 (N = 16), 21 (32),
    45 (48), 55 (64), 66 (80; alpha of 12o 2a+4b, whose beta side has 45).  FP32
    bulk against the oracle's FP64 sigma, and against the CUDA-core kernel
    (BSIM_RI_TC=0)."""
    from binsim_b200 import cuotf, network as nw
    L = cuotf.lib()
    _timeouts(L, reset=True)
    net = nw.hamiltonian_network(norb, seed=5)
    B = cuotf.CuBasis(norb, na, nb)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    path = f.sigma_path()
    assert path[0] == 1 and "ri-alpha" in path[1] and "ri-beta" in path[1], path
    x = np.random.default_rng(norb + na).normal(size=B.dim)
    x /= np.linalg.norm(x)
    ref = oracle.hvec(oracle.basis(norb, na, nb), oracle.network(net), x)
    scale = np.abs(ref).max()
    xd = dev(cuda, x)
    y_tc, y_cc = cuda.empty_like(xd), cuda.empty_like(xd)
    f.hvec_mixed(xd, y_tc)
    cuda.cuda.synchronize()
    assert np.abs(y_tc.cpu().numpy() - ref).max() <= 2e-6 * scale
    monkeypatch.setenv("BSIM_RI_TC", "0")
    f.hvec_mixed(xd, y_cc)
    assert float((y_tc - y_cc).abs().max()) <= 2e-6 * scale
    assert _timeouts(L) == 0
