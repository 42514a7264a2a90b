"""Times the reference's own GPU library on this GPU (test infrastructure).

The reference CUDA library (src/extern/cuotf.cu, built unchanged for sm_100a by
`make -C oracle ref-gpu` into oracle/_ref/libcuotf_ref.so) is driven through its
own C-ABI with host handles from the reference CPU libraries (oracle/_ref), the
way jl/cuda/cunetwork.jl drives it:

  python oracle/time_ref_gpu.py sigma 16   # hvec_cuda, norb 16 8a+8b (14: 7a+7b)
  python oracle/time_ref_gpu.py vqe        # energy_objective (jl/vqe.jl:1-21) on
                                           # expm_cuda / hvec_cuda / backgrad_cuda

Each result is checked against this repository's library on the same inputs and
printed as one JSON line.  Nothing in the product imports this file.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this directory heads sys.path and its oracle.py would shadow
# the oracle package of the repository root
sys.path = [ROOT] + [p for p in sys.path if os.path.abspath(p or ".") != HERE]

import numpy as np  # noqa: E402

vp, i64, dbl = C.c_void_p, C.c_int64, C.c_double


def ref_gpu_lib():
    path = os.path.join(HERE, "_ref", "libcuotf_ref.so")
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run make -C oracle ref-gpu")
    L = C.CDLL(path)
    L.sync_device_cuda.argtypes = []
    L.build_basisdev_f64.restype = vp
    L.build_basisdev_f64.argtypes = [vp]
    L.build_networkdev_f64.restype = vp
    L.build_networkdev_f64.argtypes = [vp]
    L.hvec_cuda.argtypes = [vp, vp, vp, vp]
    L.expm_cuda.argtypes = [vp, vp, i64, dbl, vp]
    L.backgrad_cuda.restype = dbl
    L.backgrad_cuda.argtypes = [vp, vp, i64, dbl, vp, vp]
    return L


def time_sigma(norb, compare=True):
    """hvec_cuda of the reference GPU library at norb orbitals (norb/2 + norb/2
    electrons); with compare, also this library's sigma on the same input."""
    import torch
    from binsim_b200 import network as nw
    from oracle.oracle import RefLibs
    ne = norb // 2
    R, L = RefLibs(), ref_gpu_lib()
    net = nw.hamiltonian_network(norb, seed=0)
    hb, dim = R.basis(norb, ne, ne)
    hn = R.network(net)
    db, dn = L.build_basisdev_f64(hb), L.build_networkdev_f64(hn)
    x = torch.randn(dim, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    x /= x.norm()
    y = torch.empty_like(x)
    L.hvec_cuda(db, dn, x.data_ptr(), y.data_ptr())
    L.sync_device_cuda()
    reps = 3 if norb <= 14 else 1
    t0 = time.perf_counter()
    for _ in range(reps):
        L.hvec_cuda(db, dn, x.data_ptr(), y.data_ptr())
    L.sync_device_cuda()
    ref_s = (time.perf_counter() - t0) / reps
    if not compare:
        return {"what": f"hvec_cuda, {norb} orbitals {ne}a+{ne}b, dim {dim}", "reference_gpu_s": ref_s,
                "reps": reps}
    from binsim_b200 import cuotf
    B = cuotf.CuBasis(norb, ne, ne)
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(net))
    y2 = torch.empty_like(x)
    f.hvec(x, y2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        f.hvec(x, y2)
    torch.cuda.synchronize()
    own_s = (time.perf_counter() - t0) / reps
    err = float((y - y2).abs().max() / y.abs().max())
    return {"what": f"hvec_cuda, {norb} orbitals {ne}a+{ne}b, dim {dim}", "reference_gpu_s": ref_s,
            "this_library_s": own_s, "speedup": ref_s / own_s, "max_rel_diff": err, "reps": reps}


def time_vqe():
    import torch
    import bench
    from binsim_b200 import cuotf
    from oracle.oracle import RefLibs
    cfg = bench.VQE_CFG
    ham, pool, op_idx, param_idx, th = bench.vqe_problem(cfg)
    R, L = RefLibs(), ref_gpu_lib()
    hb, dim = R.basis(cfg["norb"], cfg["na"], cfg["nb"])
    hh, hp = R.network(ham), R.network(pool.network)
    db, dh, dp = L.build_basisdev_f64(hb), L.build_networkdev_f64(hh), L.build_networkdev_f64(hp)
    hf = R.det_index(hb, (1 << cfg["na"]) - 1, (1 << cfg["nb"]) - 1, dim)
    lv = torch.zeros(dim, dtype=torch.float64, device="cuda")
    rv = torch.empty_like(lv)

    def objective():   # jl/vqe.jl:1-21 on the reference kernels
        lv.zero_()
        lv[hf] = 1.0
        for i, p in zip(op_idx, param_idx):
            L.expm_cuda(db, dp, int(i), float(th[p]), lv.data_ptr())
        L.hvec_cuda(db, dh, lv.data_ptr(), rv.data_ptr())
        L.sync_device_cuda()
        ln = float(lv @ lv)
        e = float(lv @ rv) / ln
        g = np.zeros(len(th))
        for i, p in zip(op_idx[::-1], param_idx[::-1]):
            g[p] += L.backgrad_cuda(db, dp, int(i), float(th[p]), lv.data_ptr(), rv.data_ptr()) * 2 / ln
        return e, g
    objective()
    t0 = time.perf_counter()
    e_ref, g_ref = objective()
    ref_s = time.perf_counter() - t0
    B = cuotf.CuBasis(cfg["norb"], cfg["na"], cfg["nb"])
    f = cuotf.CuOTFFunctions(B, cuotf.CuNetwork(ham), cuotf.CuNetwork(pool.network))
    ri, rvv = np.array([B.hf_index()]), np.array([1.0])
    f.energy_grad(op_idx, param_idx, th, ri, rvv, lv, rv, ckpt_every=cfg["ckpt"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e, g, _ = f.energy_grad(op_idx, param_idx, th, ri, rvv, lv, rv, ckpt_every=cfg["ckpt"])
    own_s = time.perf_counter() - t0
    return {"what": f"energy_objective, {cfg['norb']} orbitals, {len(op_idx)} components, dim {dim}",
            "reference_gpu_s": ref_s, "this_library_s": own_s, "speedup": ref_s / own_s,
            "energy_diff": abs(e - e_ref), "max_grad_diff": float(np.abs(g - g_ref).max())}


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "sigma"
    out = time_sigma(int(sys.argv[2]) if len(sys.argv) > 2 else 14) if what == "sigma" else time_vqe()
    print(json.dumps(out))
