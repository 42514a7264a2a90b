import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["h6_3a3b", "h8_4a3b_sym", "h8_4a4b"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of libcuotf")


def load_golden(name):
    """Fixture dict plus the two OTFNetwork objects it stores."""
    from binsim_b200 import network as nw
    z = dict(np.load(os.path.join(GOLDEN, name + ".npz")))

    def net(prefix):
        return nw.OTFNetwork(norb=int(z[f"{prefix}_norb"]), orbsym=z[f"{prefix}_orbsym"], axs=z[f"{prefix}_axs"],
                             bxs=z[f"{prefix}_bxs"], ranks=z[f"{prefix}_ranks"], num_zas=z[f"{prefix}_num_zas"],
                             num_zbs=z[f"{prefix}_num_zbs"], flat_zas=z[f"{prefix}_flat_zas"],
                             flat_zbs=z[f"{prefix}_flat_zbs"], flat_wa=z[f"{prefix}_flat_wa"],
                             flat_wb=z[f"{prefix}_flat_wb"])
    return z, net("ham"), net("pool")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reflibs():
    from oracle.oracle import RefLibs, ref_available
    if not ref_available():
        pytest.skip("oracle/_ref (the reference's compiled CPU libraries) not built")
    return RefLibs()


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; GPU tests fail (not skip) without one."""
    import torch
    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    return torch


def dev(torch, a, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda", dtype=dtype or torch.float64)


def cu_setup(z, ham, pool):
    from binsim_b200 import cuotf
    B = cuotf.CuBasis(int(z["norb"]), int(z["na"]), int(z["nb"]), orbsym=z["orbsym"],
                      total_sym=int(z["total_sym"]), num_irreps=int(z["num_irreps"]))
    H = cuotf.CuNetwork(ham) if ham is not None else None
    P = cuotf.CuNetwork(pool) if pool is not None else None
    return B, H, P, cuotf.CuOTFFunctions(B, H, P)
