"""TEST INFRASTRUCTURE ONLY -- ctypes drivers for the checkers.

* ``Oracle`` drives ``oracle/liboracle.so``, the plain-C restatement of the
  OTF operator path (``oracle/otf_oracle.c``).
* ``RefLibs`` drives the reference's own CPU libraries compiled by
  ``oracle/Makefile`` into ``oracle/_ref`` (libotf_native, libbasis, libdiag,
  libham_real), restating the Julia glue that calls them
  (``jl/network.jl:17-48, 313-375, 483-608``, ``jl/davidson.jl``).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# Where the reference's sources lie (read-only; only oracle/Makefile compiles
# them).  The one place this location is read: environment variable
# BINSIM_REF_SRC, default /root/reference.  oracle/Makefile takes the same
# variable with the same default.
REF_SRC = os.environ.get("BINSIM_REF_SRC", "/root/reference")


def ref_sources_present() -> bool:
    """The reference's C++ headers are present (its CPU libraries can be built)."""
    return os.path.isdir(os.path.join(REF_SRC, "src", "include"))


def make_ref(target: str = "ref") -> None:
    """Run oracle/Makefile's target with this module's reference location."""
    subprocess.run(["make", "-s", "-C", HERE, target, f"BINSIM_REF_SRC={REF_SRC}"], check=True)
_lock = threading.Lock()

P = lambda a: a.ctypes.data_as(C.c_void_p)
i64 = C.c_int64
dbl = C.c_double
vp = C.c_void_p


def build_oracle(force: bool = False) -> str:
    """Compile liboracle.so (gcc, a second or two) if it is missing."""
    path = os.path.join(HERE, "liboracle.so")
    with _lock:
        if force or not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(
                os.path.join(HERE, "otf_oracle.c")):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return path


def _ptr_array(vecs):
    arr = (C.c_void_p * len(vecs))()
    for i, v in enumerate(vecs):
        arr[i] = v.ctypes.data
    return arr


class Oracle:
    """The C restatement: basis/network handles and every operator of the path."""

    def __init__(self):
        lib = C.CDLL(build_oracle())
        lib.oracle_basis_create.restype = vp
        lib.oracle_basis_create.argtypes = [i64, i64, i64, i64, vp, i64]
        lib.oracle_basis_dim.restype = i64
        lib.oracle_basis_dim.argtypes = [vp]
        lib.oracle_basis_num_blocks.restype = i64
        lib.oracle_basis_num_blocks.argtypes = [vp]
        lib.oracle_basis_blocks.argtypes = [vp, vp]
        lib.oracle_basis_strings.argtypes = [vp, i64, C.c_int, vp]
        lib.oracle_basis_destroy.argtypes = [vp]
        lib.oracle_net_create.restype = vp
        lib.oracle_net_create.argtypes = [vp, i64, i64] + [vp] * 9
        lib.oracle_net_destroy.argtypes = [vp]
        lib.oracle_hvec.argtypes = [vp, vp, vp, vp]
        lib.oracle_diag.argtypes = [vp, vp, vp]
        lib.oracle_expm.argtypes = [vp, vp, i64, dbl, vp]
        lib.oracle_grad.restype = dbl
        lib.oracle_grad.argtypes = [vp, vp, i64, dbl, vp, vp]
        lib.oracle_backgrad.restype = dbl
        lib.oracle_backgrad.argtypes = [vp, vp, i64, dbl, vp, vp]
        lib.oracle_batchgrad.argtypes = [vp, vp, vp, vp, vp, vp]
        lib.oracle_tvec.argtypes = [vp, vp, i64, vp, vp]
        lib.oracle_net_create_c64.restype = vp
        lib.oracle_net_create_c64.argtypes = [vp, i64, i64] + [vp] * 9
        for name, args in (("oracle_hvec_c64", [vp, vp, vp, vp]), ("oracle_diag_c64", [vp, vp, vp]),
                           ("oracle_expm_c64", [vp, vp, i64, dbl, vp]),
                           ("oracle_grad_c64", [vp, vp, i64, dbl, vp, vp, vp]),
                           ("oracle_backgrad_c64", [vp, vp, i64, dbl, vp, vp, vp]),
                           ("oracle_tvec_c64", [vp, vp, i64, vp, vp]),
                           ("oracle_backtran_c64", [vp, vp, i64, dbl, vp, vp, vp]),
                           ("oracle_batchexpm_c64", [vp, vp, i64, dbl, vp, C.c_int, C.c_int]),
                           ("oracle_batchgrad_c64", [vp, vp, vp, vp, vp, vp]),
                           ("oracle_batchtran_c64", [vp, vp, vp, vp, vp])):
            getattr(lib, name).argtypes = args
        lib.oracle_backtran.argtypes = [vp, vp, i64, dbl, vp, vp, vp]
        lib.oracle_batchexpm.argtypes = [vp, vp, i64, dbl, vp, C.c_int, C.c_int]
        lib.oracle_batchtran.argtypes = [vp, vp, vp, vp, vp]
        lib.oracle_ritz_residual.restype = dbl
        lib.oracle_ritz_residual.argtypes = [i64, C.c_int, vp, dbl, vp, vp, vp]
        lib.oracle_ritz_vector.argtypes = [i64, C.c_int, vp, vp, vp]
        lib.oracle_precondition.argtypes = [i64, vp, vp, dbl, dbl]
        lib.oracle_mgs.restype = dbl
        lib.oracle_mgs.argtypes = [i64, C.c_int, vp, vp]
        lib.oracle_normalize.restype = dbl
        lib.oracle_normalize.argtypes = [i64, vp]
        lib.oracle_dot.restype = dbl
        lib.oracle_dot.argtypes = [i64, vp, vp]
        lib.oracle_heff_col.argtypes = [i64, C.c_int, vp, vp, vp]
        self.lib = lib

    # -- handles ---------------------------------------------------------
    def basis(self, norb, na, nb, orbsym=None, total_sym=0, num_irreps=16):
        orbsym = np.zeros(norb, np.int64) if orbsym is None else np.ascontiguousarray(orbsym, np.int64)
        h = self.lib.oracle_basis_create(norb, na, nb, total_sym, P(orbsym), num_irreps)
        return OracleBasis(self, h, norb)

    def network(self, net):
        a = dict(orbsym=np.ascontiguousarray(net.orbsym, np.int64),
                 axs=np.ascontiguousarray(net.axs, np.uint64), bxs=np.ascontiguousarray(net.bxs, np.uint64),
                 ranks=np.ascontiguousarray(net.ranks, np.int64),
                 nza=np.ascontiguousarray(net.num_zas, np.int64), nzb=np.ascontiguousarray(net.num_zbs, np.int64),
                 za=np.ascontiguousarray(net.flat_zas, np.uint64), zb=np.ascontiguousarray(net.flat_zbs, np.uint64),
                 wa=np.ascontiguousarray(net.flat_wa, np.float64), wb=np.ascontiguousarray(net.flat_wb, np.float64))
        h = self.lib.oracle_net_create(P(a["orbsym"]), net.norb, net.ngs, P(a["axs"]), P(a["bxs"]), P(a["ranks"]),
                                       P(a["nza"]), P(a["nzb"]), P(a["za"]), P(a["zb"]), P(a["wa"]), P(a["wb"]))
        return OracleNet(self, h, net.ngs, a)

    def network_c64(self, net, wa, wb):
        """Complex-weight network (the reference's Tv = complex<double>): wa, wb are
        complex128 arrays in the order of net.flat_wa / net.flat_wb."""
        a = dict(orbsym=np.ascontiguousarray(net.orbsym, np.int64),
                 axs=np.ascontiguousarray(net.axs, np.uint64), bxs=np.ascontiguousarray(net.bxs, np.uint64),
                 ranks=np.ascontiguousarray(net.ranks, np.int64),
                 nza=np.ascontiguousarray(net.num_zas, np.int64), nzb=np.ascontiguousarray(net.num_zbs, np.int64),
                 za=np.ascontiguousarray(net.flat_zas, np.uint64), zb=np.ascontiguousarray(net.flat_zbs, np.uint64),
                 wa=np.ascontiguousarray(wa, np.complex128), wb=np.ascontiguousarray(wb, np.complex128))
        h = self.lib.oracle_net_create_c64(P(a["orbsym"]), net.norb, net.ngs, P(a["axs"]), P(a["bxs"]),
                                           P(a["ranks"]), P(a["nza"]), P(a["nzb"]), P(a["za"]), P(a["zb"]),
                                           P(a["wa"]), P(a["wb"]))
        return OracleNet(self, h, net.ngs, a)

    # complex operators on complex128 arrays
    def hvec_c64(self, B, N, x):
        x = np.ascontiguousarray(x, np.complex128); y = np.zeros(B.dim, np.complex128)
        self.lib.oracle_hvec_c64(B.h, N.h, P(x), P(y))
        return y

    def diag_c64(self, B, N):
        d = np.zeros(B.dim, np.complex128)
        self.lib.oracle_diag_c64(B.h, N.h, P(d))
        return d

    def expm_c64(self, B, N, idx, theta, v):
        v = np.array(v, np.complex128, copy=True)
        self.lib.oracle_expm_c64(B.h, N.h, idx, theta, P(v))
        return v

    def grad_c64(self, B, N, idx, theta, l, r):
        out = np.zeros(2)
        self.lib.oracle_grad_c64(B.h, N.h, idx, theta, P(np.ascontiguousarray(l, np.complex128)),
                                 P(np.ascontiguousarray(r, np.complex128)), P(out))
        return complex(out[0], out[1])

    def backgrad_c64(self, B, N, idx, theta, l, r):
        l = np.array(l, np.complex128, copy=True); r = np.array(r, np.complex128, copy=True)
        out = np.zeros(2)
        self.lib.oracle_backgrad_c64(B.h, N.h, idx, theta, P(l), P(r), P(out))
        return complex(out[0], out[1]), l, r

    def tvec_c64(self, B, N, idx, src):
        dst = np.zeros(B.dim, np.complex128)
        self.lib.oracle_tvec_c64(B.h, N.h, idx, P(np.ascontiguousarray(src, np.complex128)), P(dst))
        return dst

    def backtran_c64(self, B, N, idx, theta, l, r):
        l = np.array(l, np.complex128, copy=True); r = np.array(r, np.complex128, copy=True)
        b = np.zeros(B.dim, np.complex128)
        self.lib.oracle_backtran_c64(B.h, N.h, idx, theta, P(l), P(r), P(b))
        return l, r, b

    def batchexpm_c64(self, B, N, idx, theta, M, nv):
        M = np.array(M, np.complex128, copy=True, order="C")
        self.lib.oracle_batchexpm_c64(B.h, N.h, idx, theta, P(M), M.shape[1], nv)
        return M

    def batchgrad_c64(self, B, N, thetas, l, r):
        g = np.zeros(N.ngs, np.complex128)
        self.lib.oracle_batchgrad_c64(B.h, N.h, P(np.ascontiguousarray(thetas, np.float64)),
                                      P(np.ascontiguousarray(l, np.complex128)),
                                      P(np.ascontiguousarray(r, np.complex128)), P(g))
        return g

    def batchtran_c64(self, B, N, l, r):
        t = np.zeros(N.ngs, np.complex128)
        self.lib.oracle_batchtran_c64(B.h, N.h, P(np.ascontiguousarray(l, np.complex128)),
                                      P(np.ascontiguousarray(r, np.complex128)), P(t))
        return t

    # -- operators --------------------------------------------------------
    def hvec(self, B, N, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(B.dim)
        self.lib.oracle_hvec(B.h, N.h, P(x), P(y))
        return y

    def diag(self, B, N):
        d = np.zeros(B.dim)
        self.lib.oracle_diag(B.h, N.h, P(d))
        return d

    def expm(self, B, N, idx, theta, v):
        v = np.array(v, np.float64, copy=True)
        self.lib.oracle_expm(B.h, N.h, idx, theta, P(v))
        return v

    def grad(self, B, N, idx, theta, l, r):
        l = np.ascontiguousarray(l, np.float64); r = np.ascontiguousarray(r, np.float64)
        return self.lib.oracle_grad(B.h, N.h, idx, theta, P(l), P(r))

    def backgrad(self, B, N, idx, theta, l, r):
        """Returns (g, l_new, r_new); inputs are not modified."""
        l = np.array(l, np.float64, copy=True); r = np.array(r, np.float64, copy=True)
        g = self.lib.oracle_backgrad(B.h, N.h, idx, theta, P(l), P(r))
        return g, l, r

    def batchgrad(self, B, N, thetas, l, r):
        thetas = np.ascontiguousarray(thetas, np.float64)
        l = np.ascontiguousarray(l, np.float64); r = np.ascontiguousarray(r, np.float64)
        g = np.zeros(N.ngs)
        self.lib.oracle_batchgrad(B.h, N.h, P(thetas), P(l), P(r), P(g))
        return g

    def tvec(self, B, N, idx, src):
        src = np.ascontiguousarray(src, np.float64)
        dst = np.zeros(B.dim)
        self.lib.oracle_tvec(B.h, N.h, idx, P(src), P(dst))
        return dst

    def backtran(self, B, N, idx, theta, l, r):
        """Returns (l_new, r_new, b); inputs are not modified."""
        l = np.array(l, np.float64, copy=True); r = np.array(r, np.float64, copy=True)
        b = np.zeros(B.dim)
        self.lib.oracle_backtran(B.h, N.h, idx, theta, P(l), P(r), P(b))
        return l, r, b

    def batchexpm(self, B, N, idx, theta, M, nv):
        """M: (dim, ld) row-major; the first nv columns are rotated (a copy is returned)."""
        M = np.array(M, np.float64, copy=True, order="C")
        self.lib.oracle_batchexpm(B.h, N.h, idx, theta, P(M), M.shape[1], nv)
        return M

    def batchtran(self, B, N, l, r):
        l = np.ascontiguousarray(l, np.float64); r = np.ascontiguousarray(r, np.float64)
        t = np.zeros(N.ngs)
        self.lib.oracle_batchtran(B.h, N.h, P(l), P(r), P(t))
        return t

    # -- Davidson helpers -------------------------------------------------
    def ritz_residual(self, coeffs, e, V, AV):
        n = len(V[0]); out = np.zeros(n)
        c = np.ascontiguousarray(coeffs, np.float64)
        nr = self.lib.oracle_ritz_residual(n, len(V), P(c), e, _ptr_array(V), _ptr_array(AV), P(out))
        return nr, out

    def ritz_vector(self, coeffs, V):
        n = len(V[0]); out = np.zeros(n)
        c = np.ascontiguousarray(coeffs, np.float64)
        self.lib.oracle_ritz_vector(n, len(V), P(c), _ptr_array(V), P(out))
        return out

    def precondition(self, r, d, e, shift):
        r = np.array(r, np.float64, copy=True)
        self.lib.oracle_precondition(len(r), P(r), P(np.ascontiguousarray(d, np.float64)), e, shift)
        return r

    def mgs(self, V, v):
        v = np.array(v, np.float64, copy=True)
        nrm = self.lib.oracle_mgs(len(v), len(V), _ptr_array(V), P(v))
        return nrm, v

    def normalize(self, v):
        v = np.array(v, np.float64, copy=True)
        nrm = self.lib.oracle_normalize(len(v), P(v))
        return nrm, v

    def heff_col(self, V, av):
        out = np.zeros(len(V))
        self.lib.oracle_heff_col(len(av), len(V), _ptr_array(V), P(np.ascontiguousarray(av)), P(out))
        return out


class OracleBasis:
    def __init__(self, owner, h, norb):
        self.o, self.h, self.norb = owner, h, norb
        self.dim = owner.lib.oracle_basis_dim(h)
        self.num_blocks = owner.lib.oracle_basis_num_blocks(h)
        blk = np.zeros(5 * max(1, self.num_blocks), np.int64)
        owner.lib.oracle_basis_blocks(h, P(blk))
        self.blocks = blk[: 5 * self.num_blocks].reshape(-1, 5)

    def strings(self, k, spin):
        n = int(self.blocks[k, 2 + spin])
        out = np.zeros(max(1, n), np.uint64)
        self.o.lib.oracle_basis_strings(self.h, k, spin, P(out))
        return out[:n]

    def det_index(self, astr, bstr):
        for k in range(self.num_blocks):
            A, Bs = self.strings(k, 0), self.strings(k, 1)
            ia = np.searchsorted(A, astr); ib = np.searchsorted(Bs, bstr)
            if ia < len(A) and A[ia] == astr and ib < len(Bs) and Bs[ib] == bstr:
                return int(self.blocks[k, 4] + ia * len(Bs) + ib)
        return -1

    def __del__(self):
        try:
            self.o.lib.oracle_basis_destroy(self.h)
        except Exception:
            pass


class OracleNet:
    def __init__(self, owner, h, ngs, keep):
        self.o, self.h, self.ngs, self._keep = owner, h, ngs, keep

    def __del__(self):
        try:
            self.o.lib.oracle_net_destroy(self.h)
        except Exception:
            pass


# ---------------------------------------------------------------------------
# the reference's own libraries (built here from its sources)
# ---------------------------------------------------------------------------

class HamResult(C.Structure):
    """binsim::ham::HamResult<double>, ham.hpp:482-490."""
    _fields_ = [("axs", vp), ("azs", vp), ("bxs", vp), ("bzs", vp),
                ("cs", C.POINTER(C.c_double)), ("ncs", C.c_size_t)]


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f)) for f in
               ("libotf_native.so", "libbasis.so", "libdiag.so", "libham_real.so"))


def ref_u64_available() -> bool:
    """The reference's uint64 basis interface (ref_basis_ui64.cpp) next to its libraries."""
    return ref_available() and os.path.exists(os.path.join(REF_DIR, "libbasis_ui64.so"))


def build_ref() -> bool:
    """Compile oracle/_ref from the reference sources when they are present."""
    if ref_u64_available():
        return True
    if not ref_sources_present():
        return False
    make_ref("ref")
    return ref_available()


class Cplx(C.Structure):
    """std::complex<double> returned by value (two doubles)."""
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class RefLibs:
    """ctypes access to the reference's compiled CPU libraries (uint32 strings)."""

    def __init__(self):
        if not ref_available():
            raise RuntimeError("oracle/_ref libraries are not built")
        L = lambda n: C.CDLL(os.path.join(REF_DIR, n))
        self.otf, self.bas, self.diag, self.ham = (L("libotf_native.so"), L("libbasis.so"),
                                                   L("libdiag.so"), L("libham_real.so"))
        f = self.ham.generate_hamiltonian_real_64_128_f64
        f.restype = HamResult
        f.argtypes = [dbl, vp, vp, C.c_int, dbl, C.c_bool]
        self.otf.build_network_otf_f64.restype = vp
        self.otf.build_network_otf_f64.argtypes = [vp, i64, i64] + [vp] * 9
        self.otf.destroy_network_otf_f64.argtypes = [vp]
        self.otf.hvec_gather_contract_otf_f64.argtypes = [vp, vp, vp, vp]
        self.otf.get_diags_elements_f64.argtypes = [vp, vp, vp]
        self.otf.expm_contract_otf_f64.argtypes = [vp, vp, i64, dbl, vp]
        self.otf.grad_contract_otf_f64.restype = dbl
        self.otf.grad_contract_otf_f64.argtypes = [vp, vp, i64, dbl, vp, vp]
        self.otf.backgrad_contract_otf_f64.restype = dbl
        self.otf.backgrad_contract_otf_f64.argtypes = [vp, vp, i64, dbl, vp, vp]
        self.otf.batch_grad_contract_otf_f64.argtypes = [vp, vp, vp, vp, vp, vp]
        self.otf.tvec_contract_otf_f64.argtypes = [vp, vp, i64, vp, vp]
        self.otf.backtran_contract_otf_f64.argtypes = [vp, vp, i64, dbl, vp, vp, vp]
        self.otf.batch_expm_contract_otf_f64.argtypes = [vp, vp, i64, dbl, vp, C.c_int, C.c_int]
        self.otf.batch_tran_contract_otf_f64.argtypes = [vp, vp, vp, vp, vp]
        # complex interface (Tv = complex<double>, otf_native.cpp:4): complex results
        # come back as two doubles (the layout of std::complex<double>)
        self.otf.build_network_otf_c64.restype = vp
        self.otf.build_network_otf_c64.argtypes = [vp, i64, i64] + [vp] * 9
        self.otf.hvec_gather_contract_otf_c64.argtypes = [vp, vp, vp, vp]
        self.otf.get_diags_elements_c64.argtypes = [vp, vp, vp]
        self.otf.expm_contract_otf_c64.argtypes = [vp, vp, i64, dbl, vp]
        self.otf.grad_contract_otf_c64.restype = Cplx
        self.otf.grad_contract_otf_c64.argtypes = [vp, vp, i64, dbl, vp, vp]
        self.otf.backgrad_contract_otf_c64.restype = Cplx
        self.otf.backgrad_contract_otf_c64.argtypes = [vp, vp, i64, dbl, vp, vp]
        self.otf.tvec_contract_otf_c64.argtypes = [vp, vp, i64, vp, vp]
        self.otf.backtran_contract_otf_c64.argtypes = [vp, vp, i64, dbl, vp, vp, vp]
        self.otf.batch_expm_contract_otf_c64.argtypes = [vp, vp, i64, dbl, vp, C.c_int, C.c_int]
        self.otf.batch_grad_contract_otf_c64.argtypes = [vp, vp, vp, vp, vp, vp]
        self.otf.batch_tran_contract_otf_c64.argtypes = [vp, vp, vp, vp, vp]
        self.bas.create_basis_manager.restype = vp
        self.bas.create_basis_manager.argtypes = [i64, i64, i64, i64, vp, i64]
        self.bas.get_subspace_dim.restype = i64
        self.bas.get_subspace_dim.argtypes = [vp]
        self.bas.get_num_symmetry_blocks.restype = i64
        self.bas.get_num_symmetry_blocks.argtypes = [vp]
        self.bas.destroy_basis_manager.argtypes = [vp]
        self.bas.set_det_coeff_f64.argtypes = [vp, C.c_uint32, C.c_uint32, dbl, vp]
        for name in ("build_ritz_and_residual_f64", "mgs_orthogonalize_f64", "inplace_normalize_f64",
                     "fast_dot_f64"):
            getattr(self.diag, name).restype = dbl
        self.diag.build_ritz_and_residual_f64.argtypes = [i64, C.c_int, vp, dbl, vp, vp, vp]
        self.diag.build_ritz_vector_f64.argtypes = [i64, C.c_int, vp, vp, vp]
        self.diag.apply_preconditioner_inplace_f64.argtypes = [i64, vp, vp, dbl, dbl]
        self.diag.mgs_orthogonalize_f64.argtypes = [i64, C.c_int, vp, vp]
        self.diag.inplace_normalize_f64.argtypes = [i64, vp]
        self.diag.fast_dot_f64.argtypes = [i64, vp, vp]
        self.diag.compute_heff_col_f64.argtypes = [i64, C.c_int, vp, vp, vp]
        self._keep = []

    def hamiltonian_terms(self, h, g, e_nuc=0.0, tol=1e-12):
        """Raw (ax, az, bx, bz, cs) from generate_hamiltonian_real_64_128_f64
        (integrals passed column-major as Julia does, ham.hpp:214-241)."""
        h1 = np.asfortranarray(h, np.float64); g4 = np.asfortranarray(g, np.float64)
        r = self.ham.generate_hamiltonian_real_64_128_f64(e_nuc, h1.ctypes.data, g4.ctypes.data,
                                                          h.shape[0], tol, False)
        n = r.ncs
        U = lambda p: np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint32)), (n,)).astype(np.uint64)
        cs = np.ctypeslib.as_array(r.cs, (n,)).copy() if n else np.zeros(0)
        return U(r.axs), U(r.azs), U(r.bxs), U(r.bzs), cs

    def basis(self, norb, na, nb, orbsym=None, total_sym=0, num_irreps=16):
        orbsym = np.zeros(norb, np.int64) if orbsym is None else np.ascontiguousarray(orbsym, np.int64)
        h = self.bas.create_basis_manager(norb, na, nb, total_sym, P(orbsym), num_irreps)
        self._keep.append(orbsym)
        return h, self.bas.get_subspace_dim(h)

    def network(self, net):
        a = [np.ascontiguousarray(net.orbsym, np.int64)]
        arrs = [np.ascontiguousarray(net.axs, np.uint32), np.ascontiguousarray(net.bxs, np.uint32),
                np.ascontiguousarray(net.ranks, np.int64), np.ascontiguousarray(net.num_zas, np.int64),
                np.ascontiguousarray(net.num_zbs, np.int64), np.ascontiguousarray(net.flat_zas, np.uint32),
                np.ascontiguousarray(net.flat_zbs, np.uint32), np.ascontiguousarray(net.flat_wa, np.float64),
                np.ascontiguousarray(net.flat_wb, np.float64)]
        h = self.otf.build_network_otf_f64(P(a[0]), net.norb, net.ngs, *[P(x) for x in arrs])
        self._keep.append((a, arrs))
        return h

    def hvec(self, b, n, x, dim):
        x = np.ascontiguousarray(x, np.float64); y = np.zeros(dim)
        self.otf.hvec_gather_contract_otf_f64(b, n, P(x), P(y))
        return y

    def diag_elems(self, b, n, dim):
        d = np.zeros(dim)
        self.otf.get_diags_elements_f64(b, n, P(d))
        return d

    def expm(self, b, n, idx, theta, v):
        v = np.array(v, np.float64, copy=True)
        self.otf.expm_contract_otf_f64(b, n, idx, theta, P(v))
        return v

    def grad(self, b, n, idx, theta, l, r):
        return self.otf.grad_contract_otf_f64(b, n, idx, theta, P(np.ascontiguousarray(l)), P(np.ascontiguousarray(r)))

    def backgrad(self, b, n, idx, theta, l, r):
        l = np.array(l, np.float64, copy=True); r = np.array(r, np.float64, copy=True)
        g = self.otf.backgrad_contract_otf_f64(b, n, idx, theta, P(l), P(r))
        return g, l, r

    def batchgrad(self, b, n, thetas, l, r, ngs):
        g = np.zeros(ngs)
        self.otf.batch_grad_contract_otf_f64(b, n, P(np.ascontiguousarray(thetas, np.float64)),
                                             P(np.ascontiguousarray(l)), P(np.ascontiguousarray(r)), P(g))
        return g

    def tvec(self, b, n, idx, src, dim):
        dst = np.zeros(dim)
        self.otf.tvec_contract_otf_f64(b, n, idx, P(np.ascontiguousarray(src, np.float64)), P(dst))
        return dst

    def backtran(self, b, n, idx, theta, l, r, dim):
        l = np.array(l, np.float64, copy=True); r = np.array(r, np.float64, copy=True)
        bv = np.zeros(dim)
        self.otf.backtran_contract_otf_f64(b, n, idx, theta, P(l), P(r), P(bv))
        return l, r, bv

    def batchexpm(self, b, n, idx, theta, M, nv):
        M = np.array(M, np.float64, copy=True, order="C")
        self.otf.batch_expm_contract_otf_f64(b, n, idx, theta, P(M), M.shape[1], nv)
        return M

    def batchtran(self, b, n, l, r, ngs):
        t = np.zeros(ngs)
        self.otf.batch_tran_contract_otf_f64(b, n, P(np.ascontiguousarray(l)), P(np.ascontiguousarray(r)), P(t))
        return t

    def network_c64(self, net, wa, wb):
        a = [np.ascontiguousarray(net.orbsym, np.int64)]
        arrs = [np.ascontiguousarray(net.axs, np.uint32), np.ascontiguousarray(net.bxs, np.uint32),
                np.ascontiguousarray(net.ranks, np.int64), np.ascontiguousarray(net.num_zas, np.int64),
                np.ascontiguousarray(net.num_zbs, np.int64), np.ascontiguousarray(net.flat_zas, np.uint32),
                np.ascontiguousarray(net.flat_zbs, np.uint32), np.ascontiguousarray(wa, np.complex128),
                np.ascontiguousarray(wb, np.complex128)]
        h = self.otf.build_network_otf_c64(P(a[0]), net.norb, net.ngs, *[P(x) for x in arrs])
        self._keep.append((a, arrs))
        return h

    def hvec_c64(self, b, n, x, dim):
        x = np.ascontiguousarray(x, np.complex128); y = np.zeros(dim, np.complex128)
        self.otf.hvec_gather_contract_otf_c64(b, n, P(x), P(y))
        return y

    def diag_c64(self, b, n, dim):
        d = np.zeros(dim, np.complex128)
        self.otf.get_diags_elements_c64(b, n, P(d))
        return d

    def expm_c64(self, b, n, idx, theta, v):
        v = np.array(v, np.complex128, copy=True)
        self.otf.expm_contract_otf_c64(b, n, idx, theta, P(v))
        return v

    def grad_c64(self, b, n, idx, theta, l, r):
        z = self.otf.grad_contract_otf_c64(b, n, idx, theta, P(np.ascontiguousarray(l, np.complex128)),
                                           P(np.ascontiguousarray(r, np.complex128)))
        return complex(z.re, z.im)

    def backgrad_c64(self, b, n, idx, theta, l, r):
        l = np.array(l, np.complex128, copy=True); r = np.array(r, np.complex128, copy=True)
        z = self.otf.backgrad_contract_otf_c64(b, n, idx, theta, P(l), P(r))
        return complex(z.re, z.im), l, r

    def tvec_c64(self, b, n, idx, src, dim):
        dst = np.zeros(dim, np.complex128)
        self.otf.tvec_contract_otf_c64(b, n, idx, P(np.ascontiguousarray(src, np.complex128)), P(dst))
        return dst

    def backtran_c64(self, b, n, idx, theta, l, r, dim):
        l = np.array(l, np.complex128, copy=True); r = np.array(r, np.complex128, copy=True)
        bv = np.zeros(dim, np.complex128)
        self.otf.backtran_contract_otf_c64(b, n, idx, theta, P(l), P(r), P(bv))
        return l, r, bv

    def batchexpm_c64(self, b, n, idx, theta, M, nv):
        M = np.array(M, np.complex128, copy=True, order="C")
        self.otf.batch_expm_contract_otf_c64(b, n, idx, theta, P(M), M.shape[1], nv)
        return M

    def batchgrad_c64(self, b, n, thetas, l, r, ngs):
        g = np.zeros(ngs, np.complex128)
        self.otf.batch_grad_contract_otf_c64(b, n, P(np.ascontiguousarray(thetas, np.float64)),
                                             P(np.ascontiguousarray(l, np.complex128)),
                                             P(np.ascontiguousarray(r, np.complex128)), P(g))
        return g

    def batchtran_c64(self, b, n, l, r, ngs):
        t = np.zeros(ngs, np.complex128)
        self.otf.batch_tran_contract_otf_c64(b, n, P(np.ascontiguousarray(l, np.complex128)),
                                             P(np.ascontiguousarray(r, np.complex128)), P(t))
        return t

    def det_index(self, b, astr, bstr, dim):
        v = np.zeros(dim)
        self.bas.set_det_coeff_f64(b, astr, bstr, 1.0, P(v))
        nz = np.flatnonzero(v)
        return int(nz[0]) if len(nz) else -1

    def davidson(self, b, n, v0, diags, tol=1e-5, ncv=3, maxspace=23, maxiter=100000):
        """Lowest eigenpair by the reference driver jl/davidson.jl:1-160 over the
        reference's libdiag helpers and hvec_gather_contract_otf_f64.

        Returns (energy, vector, iterations, sigma_calls)."""
        N = len(v0)
        vpp = C.c_void_p * maxspace
        V, AV = [np.array(v0, np.float64, copy=True)], [np.empty(N)]
        Vp, AVp = vpp(), vpp()
        Vp[0], AVp[0] = V[0].ctypes.data, AV[0].ctypes.data
        axt = np.empty(N)
        heff = np.zeros((maxspace, maxspace), order="F")
        col = np.empty(maxspace)
        d = self.diag
        d.rebuild_heff_f64.argtypes = [i64, C.c_int, vp, vp, vp, C.c_int]
        d.inplace_normalize_f64(N, P(V[0]))
        nsig = 0

        def aop(x, y):
            nonlocal nsig
            y[:] = 0.0
            self.otf.hvec_gather_contract_otf_f64(b, n, P(x), P(y))
            nsig += 1

        aop(V[0], AV[0])
        heff[0, 0] = d.fast_dot_f64(N, P(V[0]), P(AV[0]))
        dim = 1
        e_best = heff[0, 0]
        Vt, AVt = [], []
        for it in range(1, maxiter + 1):
            es, vs = np.linalg.eigh(heff[:dim, :dim])
            k = int(np.argmin(es))
            e_best = float(es[k])
            coeffs = np.ascontiguousarray(vs[:, k])
            norm_r = d.build_ritz_and_residual_f64(N, dim, P(coeffs), e_best, Vp, AVp, P(axt))
            if norm_r < tol:
                xt = np.empty(N)
                d.build_ritz_vector_f64(N, dim, P(coeffs), Vp, P(xt))
                return e_best, xt, it, nsig
            if dim >= maxspace:
                nsave = min(ncv, dim)
                order = np.argsort(es)
                while len(Vt) < nsave:
                    Vt.append(np.empty(N)); AVt.append(np.empty(N))
                for i in range(nsave):
                    c = vs[:, order[i]]
                    Vt[i][:] = 0.0; AVt[i][:] = 0.0
                    for j in range(dim):
                        Vt[i] += c[j] * V[j]
                        AVt[i] += c[j] * AV[j]
                for i in range(nsave):
                    V[i][:] = Vt[i]; AV[i][:] = AVt[i]
                dim = nsave
                d.rebuild_heff_f64(N, dim, Vp, AVp, heff.ctypes.data, maxspace)
            shift = max(norm_r * 1e-2, 1e-4)
            d.apply_preconditioner_inplace_f64(N, P(axt), P(diags), e_best, shift)
            nb_ = float(np.linalg.norm(axt))
            na_ = d.mgs_orthogonalize_f64(N, dim, Vp, P(axt))
            if na_ < 0.717 * nb_:
                na_ = d.mgs_orthogonalize_f64(N, dim, Vp, P(axt))
            if na_ < 1e-12:
                xt = np.empty(N)
                d.build_ritz_vector_f64(N, dim, P(coeffs), Vp, P(xt))
                return e_best, xt, it, nsig
            d.inplace_normalize_f64(N, P(axt))
            dim += 1
            if len(V) < dim:
                V.append(np.empty(N)); AV.append(np.empty(N))
                Vp[dim - 1], AVp[dim - 1] = V[-1].ctypes.data, AV[-1].ctypes.data
            V[dim - 1][:] = axt
            aop(V[dim - 1], AV[dim - 1])
            d.compute_heff_col_f64(N, dim, Vp, P(AV[dim - 1]), P(col))
            heff[:dim, dim - 1] = col[:dim]
            heff[dim - 1, :dim] = col[:dim]
        es, vs = np.linalg.eigh(heff[:dim, :dim])
        coeffs = np.ascontiguousarray(vs[:, int(np.argmin(es))])
        xt = np.empty(N)
        d.build_ritz_vector_f64(N, dim, P(coeffs), Vp, P(xt))
        return e_best, xt, maxiter, nsig


class RefLibsU64:
    """The reference's uint64 operators (the _ui64_f64 exports of libotf_native,
    src/extern/otf_native.cpp:5) over a BasisManager<uint64> from the reference's own
    basis interface instantiated for uint64 (ref_basis_ui64.cpp).  The reference's
    dense string map (basis.hpp:271) limits this to small norb."""

    def __init__(self, ref: "RefLibs"):
        if not ref_u64_available():
            raise RuntimeError("oracle/_ref/libbasis_ui64.so is not built")
        self.otf = ref.otf
        self.bas = C.CDLL(os.path.join(REF_DIR, "libbasis_ui64.so"))
        self.bas.create_basis_manager_ui64.restype = vp
        self.bas.create_basis_manager_ui64.argtypes = [i64, i64, i64, i64, vp, i64]
        self.bas.get_subspace_dim_ui64.restype = i64
        self.bas.get_subspace_dim_ui64.argtypes = [vp]
        self.bas.destroy_basis_manager_ui64.argtypes = [vp]
        o = self.otf
        o.build_network_otf_ui64_f64.restype = vp
        o.build_network_otf_ui64_f64.argtypes = [vp, i64, i64] + [vp] * 9
        o.destroy_network_otf_ui64_f64.argtypes = [vp]
        o.hvec_gather_contract_otf_ui64_f64.argtypes = [vp, vp, vp, vp]
        o.get_diags_elements_ui64_f64.argtypes = [vp, vp, vp]
        o.expm_contract_otf_ui64_f64.argtypes = [vp, vp, i64, dbl, vp]
        o.grad_contract_otf_ui64_f64.restype = dbl
        o.grad_contract_otf_ui64_f64.argtypes = [vp, vp, i64, dbl, vp, vp]
        o.backgrad_contract_otf_ui64_f64.restype = dbl
        o.backgrad_contract_otf_ui64_f64.argtypes = [vp, vp, i64, dbl, vp, vp]
        o.batch_grad_contract_otf_ui64_f64.argtypes = [vp, vp, vp, vp, vp, vp]
        o.tvec_contract_otf_ui64_f64.argtypes = [vp, vp, i64, vp, vp]
        o.batch_tran_contract_otf_ui64_f64.argtypes = [vp, vp, vp, vp, vp]
        self._keep = []

    def basis(self, norb, na, nb, orbsym=None, total_sym=0, num_irreps=16):
        orbsym = np.zeros(norb, np.int64) if orbsym is None else np.ascontiguousarray(orbsym, np.int64)
        h = self.bas.create_basis_manager_ui64(norb, na, nb, total_sym, P(orbsym), num_irreps)
        self._keep.append(orbsym)
        return h, self.bas.get_subspace_dim_ui64(h)

    def network(self, net):
        a = [np.ascontiguousarray(net.orbsym, np.int64)]
        arrs = [np.ascontiguousarray(net.axs, np.uint64), np.ascontiguousarray(net.bxs, np.uint64),
                np.ascontiguousarray(net.ranks, np.int64), np.ascontiguousarray(net.num_zas, np.int64),
                np.ascontiguousarray(net.num_zbs, np.int64), np.ascontiguousarray(net.flat_zas, np.uint64),
                np.ascontiguousarray(net.flat_zbs, np.uint64), np.ascontiguousarray(net.flat_wa, np.float64),
                np.ascontiguousarray(net.flat_wb, np.float64)]
        h = self.otf.build_network_otf_ui64_f64(P(a[0]), net.norb, net.ngs, *[P(x) for x in arrs])
        self._keep.append((a, arrs))
        return h

    def hvec(self, b, n, x, dim):
        y = np.zeros(dim)
        self.otf.hvec_gather_contract_otf_ui64_f64(b, n, P(np.ascontiguousarray(x, np.float64)), P(y))
        return y

    def diag_elems(self, b, n, dim):
        d = np.zeros(dim)
        self.otf.get_diags_elements_ui64_f64(b, n, P(d))
        return d

    def expm(self, b, n, idx, theta, v):
        v = np.array(v, np.float64, copy=True)
        self.otf.expm_contract_otf_ui64_f64(b, n, idx, theta, P(v))
        return v

    def grad(self, b, n, idx, theta, l, r):
        return self.otf.grad_contract_otf_ui64_f64(b, n, idx, theta, P(np.ascontiguousarray(l, np.float64)),
                                                   P(np.ascontiguousarray(r, np.float64)))

    def backgrad(self, b, n, idx, theta, l, r):
        l = np.array(l, np.float64, copy=True); r = np.array(r, np.float64, copy=True)
        g = self.otf.backgrad_contract_otf_ui64_f64(b, n, idx, theta, P(l), P(r))
        return g, l, r

    def batchgrad(self, b, n, thetas, l, r, ngs):
        g = np.zeros(ngs)
        self.otf.batch_grad_contract_otf_ui64_f64(b, n, P(np.ascontiguousarray(thetas, np.float64)),
                                                  P(np.ascontiguousarray(l, np.float64)),
                                                  P(np.ascontiguousarray(r, np.float64)), P(g))
        return g

    def tvec(self, b, n, idx, src, dim):
        dst = np.zeros(dim)
        self.otf.tvec_contract_otf_ui64_f64(b, n, idx, P(np.ascontiguousarray(src, np.float64)), P(dst))
        return dst

    def batchtran(self, b, n, l, r, ngs):
        t = np.zeros(ngs)
        self.otf.batch_tran_contract_otf_ui64_f64(b, n, P(np.ascontiguousarray(l, np.float64)),
                                                  P(np.ascontiguousarray(r, np.float64)), P(t))
        return t

    def complex_view(self, ref: "RefLibs"):
        """A RefLibs whose basis is the uint64 one and whose _c64 operators call the
        reference's _ui64_c64 exports (otf_native.cpp:6), masks passed as uint64."""
        import copy
        o = self.otf
        for name in ("build_network_otf", "destroy_network_otf", "hvec_gather_contract_otf", "get_diags_elements",
                     "expm_contract_otf", "grad_contract_otf", "backgrad_contract_otf", "tvec_contract_otf",
                     "backtran_contract_otf", "batch_expm_contract_otf", "batch_grad_contract_otf",
                     "batch_tran_contract_otf"):
            src, dst = getattr(o, name + "_c64"), getattr(o, name + "_ui64_c64")
            dst.argtypes, dst.restype = src.argtypes, src.restype

        class _Suffix:
            def __getattr__(_, name):
                return getattr(o, name[:-4] + "_ui64_c64") if name.endswith("_c64") else getattr(o, name)

        view = copy.copy(ref)
        view.otf = _Suffix()
        view.basis = self.basis
        keep = self._keep

        def network_c64(net, wa, wb):
            a = [np.ascontiguousarray(net.orbsym, np.int64)]
            arrs = [np.ascontiguousarray(net.axs, np.uint64), np.ascontiguousarray(net.bxs, np.uint64),
                    np.ascontiguousarray(net.ranks, np.int64), np.ascontiguousarray(net.num_zas, np.int64),
                    np.ascontiguousarray(net.num_zbs, np.int64), np.ascontiguousarray(net.flat_zas, np.uint64),
                    np.ascontiguousarray(net.flat_zbs, np.uint64), np.ascontiguousarray(wa, np.complex128),
                    np.ascontiguousarray(wb, np.complex128)]
            h = o.build_network_otf_ui64_c64(P(a[0]), net.norb, net.ngs, *[P(x) for x in arrs])
            keep.append((a, arrs))
            return h
        view.network_c64 = network_c64
        return view
