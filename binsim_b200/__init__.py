"""binsim_b200 -- BinSim's on-the-fly (OTF) operator path on B200 (sm_100a).

* ``binsim_b200.cuotf``    -- ctypes binding of libcuotf (include/binsim_cuotf.h)
  and the host layer mirroring the reference's CuOTF_Functions.
* ``binsim_b200.network``  -- host-side construction of OTF networks (JW
  Hamiltonian, SVD grouping, UCC pools).
* ``binsim_b200.build``    -- compiles libcuotf in-tree.
"""
from . import network  # noqa: F401

__all__ = ["network"]
