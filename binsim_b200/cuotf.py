"""ctypes binding of libcuotf and a host layer mirroring the reference's
``CuOTF_Functions`` (``jl/cuda/cunetwork.jl:74-160``).

Device vectors are ``torch`` CUDA tensors (float64); torch provides device
memory and streams only -- all arithmetic runs in libcuotf's kernels.  Work is
enqueued on torch's current stream.  The library is loaded from
``binsim_b200/lib/libcuotf.so``; a missing library raises immediately (there
is no fallback path).
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import Optional, Sequence

import numpy as np

from . import network as nw

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcuotf.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "binsim_cuotf.h")

vp, i64, dbl, ci = C.c_void_p, C.c_int64, C.c_double, C.c_int
_lib = None


class CuOTFError(RuntimeError):
    """A libcuotf entry point returned a non-zero status."""

    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


def header_symbols() -> list:
    """Every function name declared in include/binsim_cuotf.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt)) -
                  {"extern", "if", "defined", "sizeof"})


def lib() -> C.CDLL:
    """Load libcuotf (once).  Raises FileNotFoundError when it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: run __graft_entry__.build() "
                                "(or python binsim_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    sig = {
        # part 1
        "sync_device_cuda": (None, []),
        "build_basisdev_f64": (vp, [vp]), "destroy_basisdev_f64": (None, [vp]),
        "build_networkdev_f64": (vp, [vp]), "destroy_networkdev_f64": (None, [vp]),
        "hvec_cuda": (None, [vp, vp, vp, vp]), "get_diags_elements_cuda": (None, [vp, vp, vp]),
        "expm_cuda": (None, [vp, vp, i64, dbl, vp]), "grad_cuda": (dbl, [vp, vp, i64, dbl, vp, vp]),
        "backgrad_cuda": (dbl, [vp, vp, i64, dbl, vp, vp]), "batchgrad_cuda": (None, [vp, vp, vp, vp, vp, vp]),
        "expm_cuda_2d": (None, [vp, vp, i64, dbl, vp]), "grad_cuda_2d": (dbl, [vp, vp, i64, dbl, vp, vp]),
        "backgrad_cuda_2d": (dbl, [vp, vp, i64, dbl, vp, vp]),
        # part 2
        "bsim_last_error": (C.c_char_p, []), "bsim_version": (C.c_char_p, []),
        "bsim_device_alloc_count": (i64, []),
        "bsim_release_cached_memory": (ci, []),
        "bsim_tensor_core_timeouts": (ci, [vp, ci]),
        "bsim_basis_create_u32": (ci, [i64, i64, i64, i64, vp, i64, vp]),
        "bsim_basis_create_u64": (ci, [i64, i64, i64, i64, vp, i64, vp]),
        "bsim_network_create_u64": (ci, [vp, i64, i64] + [vp] * 9 + [vp]),
        "bsim_basis_from_host": (ci, [vp, vp]), "bsim_basis_destroy": (ci, [vp]),
        "bsim_basis_dim": (i64, [vp]), "bsim_basis_find_det": (i64, [vp, C.c_uint64, C.c_uint64]),
        "bsim_network_create_u32": (ci, [vp, i64, i64] + [vp] * 9 + [vp]),
        "bsim_network_from_host": (ci, [vp, vp]), "bsim_network_destroy": (ci, [vp]),
        "bsim_network_ngs": (i64, [vp]),
        "bsim_hvec": (ci, [vp, vp, vp, vp, vp]), "bsim_hvec_mixed": (ci, [vp, vp, vp, vp, vp]),
        "bsim_hvec_f32in": (ci, [vp, vp, vp, vp, vp]),
        "bsim_hvec_path": (ci, [vp, vp, C.c_char_p, ci, vp]),
        "bsim_hvec_stage_times": (ci, [vp, vp, vp, vp, ci, vp, vp, ci, vp]),
        "bsim_hvec_cols": (ci, [vp, vp, vp, vp, i64, i64, ci, vp]),
        "bsim_fma_peak": (ci, [ci, vp, vp]),
        "bsim_hvec_num_tiles": (i64, [vp]), "bsim_hvec_tiles": (ci, [vp, vp, vp, vp, i64, i64, ci, vp]), "bsim_diag": (ci, [vp, vp, vp, vp]),
        "bsim_expm": (ci, [vp, vp, i64, dbl, vp, vp]), "bsim_expm_seq": (ci, [vp, vp, i64, vp, vp, vp, vp]),
        "bsim_grad": (ci, [vp, vp, i64, dbl, vp, vp, vp, vp]),
        "bsim_backgrad": (ci, [vp, vp, i64, dbl, vp, vp, vp, vp]),
        "bsim_grad_noalloc": (ci, [vp, vp, i64, dbl, vp, vp, vp, vp]),
        "bsim_batchgrad": (ci, [vp, vp, vp, vp, vp, vp, vp]),
        "bsim_hvec_host": (ci, [vp, vp, i64, vp, vp, ci, vp]),
        "bsim_netbuild_compress": (ci, [i64, vp, vp, vp, vp, vp, dbl, vp]),
        "bsim_netbuild_compress_runs": (ci, [i64, vp, vp, vp, vp, vp, dbl, i64, vp, vp]),
        "bsim_netbuild_compress_device": (ci, [i64, vp, vp, vp, vp, vp, dbl, i64, vp, vp, vp]),
        "bsim_netbuild_sizes": (ci, [vp, vp, vp, vp, vp, vp]),
        "bsim_netbuild_export": (ci, [vp] * 10),
        "bsim_netbuild_destroy": (ci, [vp]),
        "bsim_poolplan_classify": (ci, [i64, i64] + [vp] * 12),
        "bsim_pooldensity_hole_table": (ci, [i64, i64, i64, vp, vp, vp]),
        "bsim_pooldensity_create": (ci, [vp, i64, vp, vp, vp, vp]),
        "bsim_pooldensity_grad": (ci, [vp, vp, vp, vp, vp]),
        "bsim_pooldensity_destroy": (ci, [vp]),
        "bsim_network_create_c64": (ci, [vp, i64, i64] + [vp] * 10),
        "bsim_network_create_c64_u64": (ci, [vp, i64, i64] + [vp] * 10),
        "bsim_hvec_c64": (ci, [vp, vp, vp, vp, vp]),
        "bsim_diag_c64": (ci, [vp, vp, vp, vp]),
        "bsim_expm_c64": (ci, [vp, vp, i64, dbl, vp, vp]),
        "bsim_grad_c64": (ci, [vp, vp, i64, dbl, vp, vp, vp, vp]),
        "bsim_backgrad_c64": (ci, [vp, vp, i64, dbl, vp, vp, vp, vp]),
        "bsim_tvec_c64": (ci, [vp, vp, i64, vp, vp, vp]),
        "bsim_backtran_c64": (ci, [vp, vp, i64, dbl, vp, vp, vp, vp]),
        "bsim_batchexpm_c64": (ci, [vp, vp, i64, dbl, vp, ci, ci, vp]),
        "bsim_batchgrad_c64": (ci, [vp, vp, vp, vp, vp, vp, vp]),
        "bsim_batchtran_c64": (ci, [vp, vp, vp, vp, vp, vp]),
        "bsim_tvec": (ci, [vp, vp, i64, vp, vp, vp]),
        "bsim_backtran": (ci, [vp, vp, i64, dbl, vp, vp, vp, vp]),
        "bsim_batchexpm": (ci, [vp, vp, i64, dbl, vp, ci, ci, vp]),
        "bsim_batchtran": (ci, [vp, vp, vp, vp, vp, vp]),
        "tvec_cuda": (None, [vp, vp, i64, vp, vp]),
        "backtran_cuda": (None, [vp, vp, i64, dbl, vp, vp, vp]),
        "batchexpm_cuda": (None, [vp, vp, i64, dbl, vp, ci, ci]),
        "batchtran_cuda": (None, [vp, vp, vp, vp, vp]),
        "bsim_prepare_state": (ci, [vp, vp, i64, vp, vp, vp, vp, vp, i64, vp, vp]),
        "bsim_vqe_energy_grad": (ci, [vp, vp, vp, i64, vp, vp, i64, vp, vp, vp, i64, i64, vp, vp, vp, vp, vp, vp]),
        "bsim_davidson": (ci, [vp, vp, vp, vp, dbl, ci, ci, ci, ci, vp, vp, vp, vp, vp, vp, ci, vp]),
        "bsim_davidson_block": (ci, [vp, vp, ci, vp, vp, ci, dbl, ci, ci, ci, ci, vp, vp, vp, vp, vp, ci, vp]),
        # part 3
        "build_ritz_and_residual_cuda": (dbl, [i64, ci, vp, dbl, vp, vp, vp]),
        "build_ritz_vector_cuda": (None, [i64, ci, vp, vp, vp]),
        "apply_preconditioner_inplace_cuda": (None, [i64, vp, vp, dbl, dbl]),
        "mgs_orthogonalize_cuda": (dbl, [i64, ci, vp, vp]),
        "inplace_normalize_cuda": (dbl, [i64, vp]),
        "fast_dot_cuda": (dbl, [i64, vp, vp]),
        "compute_heff_col_cuda": (None, [i64, ci, vp, vp, vp]),
        "rebuild_heff_cuda": (None, [i64, ci, vp, vp, vp, ci]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(st: int, where: str):
    if st != 0:
        raise CuOTFError(st, where, lib().bsim_last_error().decode())


def _ptr(x) -> int:
    """Device pointer of a torch tensor, or host pointer of a numpy array."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return x.ctypes.data


def _stream(stream=None):
    if stream is not None:
        return stream
    import torch
    return torch.cuda.current_stream().cuda_stream


def _host(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def compress_groups_native(ax, az, bx, bz, c, norb: int, tol: float = 1e-12, orbsym=None,
                           run_sizes=None, device: bool = False, stream=None) -> nw.OTFNetwork:
    """The grouping and SVD compression of network.compress_groups (jl/network.jl:158-246)
    in the library's native builder (host threads); groups in order of first appearance,
    or with run_sizes one group per run of consecutive terms (the pool form).  device:
    every group's SVD in one batched launch on the current GPU (or the given stream)."""
    L = lib()
    arrs = [_host(ax, np.uint64), _host(az, np.uint64), _host(bx, np.uint64), _host(bz, np.uint64),
            _host(c, np.float64)]
    h = vp()
    if device:
        rs = _host(run_sizes if run_sizes is not None else [], np.int64)
        _check(L.bsim_netbuild_compress_device(len(arrs[4]), *[a.ctypes.data for a in arrs], tol, len(rs),
                                               rs.ctypes.data if len(rs) else None, _stream(stream),
                                               C.byref(h)), "bsim_netbuild_compress_device")
    elif run_sizes is None:
        _check(L.bsim_netbuild_compress(len(arrs[4]), *[a.ctypes.data for a in arrs], tol, C.byref(h)),
               "bsim_netbuild_compress")
    else:
        rs = _host(run_sizes, np.int64)
        _check(L.bsim_netbuild_compress_runs(len(arrs[4]), *[a.ctypes.data for a in arrs], tol, len(rs),
                                             rs.ctypes.data, C.byref(h)), "bsim_netbuild_compress_runs")
    try:
        n = [C.c_int64() for _ in range(5)]
        _check(L.bsim_netbuild_sizes(h, *[C.byref(x) for x in n]), "bsim_netbuild_sizes")
        ngs, tza, tzb, twa, twb = [x.value for x in n]
        out = dict(axs=np.zeros(ngs, np.uint64), bxs=np.zeros(ngs, np.uint64), ranks=np.zeros(ngs, np.int64),
                   num_zas=np.zeros(ngs, np.int64), num_zbs=np.zeros(ngs, np.int64),
                   flat_zas=np.zeros(tza, np.uint64), flat_zbs=np.zeros(tzb, np.uint64),
                   flat_wa=np.zeros(twa, np.float64), flat_wb=np.zeros(twb, np.float64))
        _check(L.bsim_netbuild_export(h, *[out[k].ctypes.data for k in
                                           ("axs", "bxs", "ranks", "num_zas", "num_zbs", "flat_zas", "flat_zbs",
                                            "flat_wa", "flat_wb")]), "bsim_netbuild_export")
    finally:
        L.bsim_netbuild_destroy(h)
    osym = np.zeros(norb, np.int64) if orbsym is None else np.asarray(orbsym, np.int64)
    return nw.OTFNetwork(norb=norb, orbsym=osym, **out)


POOL_KINDS = {"general": -1, "zero": 0, "d1a": 1, "d1b": 2, "tab": 3, "gaa": 4, "gbb": 5}


def pool_plan(net: nw.OTFNetwork):
    """Per group of a generator network: (kind, idx[ngs, 4], coef) from the library's
    pool-gradient plan (bsim_poolplan_classify, host code): group g is
    coef[g] / (alpha-first reordering sign) * (t - t^dagger) for the excitation whose
    transition-density entry idx[g] of table kind[g] it names; kind -1 matches no
    excitation, 0 has a zero gradient for real vectors."""
    L = lib()
    n = net.ngs
    arrs = [_host(net.axs, np.uint64), _host(net.bxs, np.uint64), _host(net.ranks, np.int64),
            _host(net.num_zas, np.int64), _host(net.num_zbs, np.int64), _host(net.flat_zas, np.uint64),
            _host(net.flat_zbs, np.uint64), _host(net.flat_wa, np.float64), _host(net.flat_wb, np.float64)]
    kind = np.zeros(n, np.int32)
    idx = np.zeros((n, 4), np.int32)
    coef = np.zeros(n, np.float64)
    _check(L.bsim_poolplan_classify(net.norb, n, *[a.ctypes.data for a in arrs], kind.ctypes.data,
                                    idx.ctypes.data, coef.ctypes.data), "bsim_poolplan_classify")
    return kind, idx, coef


def hole_table(strs, norb: int, holes: int):
    """(number of hole strings, table[nh, norb or norb (norb - 1) / 2]) of
    bsim_pooldensity_hole_table (host code): entries (index << 1) | sign or -1."""
    L = lib()
    s = _host(strs, np.uint64)
    nh = C.c_int64()
    _check(L.bsim_pooldensity_hole_table(norb, holes, len(s), s.ctypes.data, C.byref(nh), None),
           "bsim_pooldensity_hole_table")
    w = norb if holes == 1 else norb * (norb - 1) // 2
    tab = np.zeros((nh.value, w), np.int32)
    _check(L.bsim_pooldensity_hole_table(norb, holes, len(s), s.ctypes.data, C.byref(nh), tab.ctypes.data),
           "bsim_pooldensity_hole_table")
    return nh.value, tab


class PoolDensity:
    """Pool gradient at theta = 0 through transition densities on the GPU
    (bsim_pooldensity_*): plan from pool_plan(net), device vectors l, r."""

    def __init__(self, basis: "CuBasis", net: nw.OTFNetwork):
        self.kind, self.idx, self.coef = pool_plan(net)
        self.ngs = net.ngs
        self._h = vp()
        _check(lib().bsim_pooldensity_create(basis.h, self.ngs, self.kind.ctypes.data, self.idx.ctypes.data,
                                             self.coef.ctypes.data, C.byref(self._h)), "bsim_pooldensity_create")

    def grad(self, l, r, grads, stream=None):
        _check(lib().bsim_pooldensity_grad(self._h, _ptr(l), _ptr(r), _ptr(grads), _stream(stream)),
               "bsim_pooldensity_grad")

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().bsim_pooldensity_destroy(self._h)
            self._h = vp()


def fma_peak(fp64: bool = True, stream=None, dmma: bool = False) -> float:
    """CUDA-core FMA throughput of the current GPU (FP64 or FP32), or with dmma the
    FP64 tensor-core MMA throughput, TFLOP/s."""
    t = C.c_double()
    _check(lib().bsim_fma_peak(2 if dmma else (1 if fp64 else 0), C.byref(t), _stream(stream)), "fma_peak")
    return t.value


class CuBasis:
    """Device determinant space (``BasisManager`` + ``upload_basis``)."""

    def __init__(self, norb: int, na: int, nb: int, orbsym=None, total_sym: int = 0, num_irreps: int = 16,
                 host_handle: Optional[int] = None, string_bits: Optional[int] = None):
        """string_bits: 32 (UInt32 strings, the reference GPU library's type) or 64
        (UInt64, up to 63 orbitals); default 32 up to 32 orbitals, else 64."""
        L = lib()
        out = vp()
        self.string_bits = 32
        if host_handle is not None:
            _check(L.bsim_basis_from_host(host_handle, C.byref(out)), "bsim_basis_from_host")
        else:
            bits = string_bits or (32 if norb <= 32 else 64)
            if bits not in (32, 64):
                raise ValueError("string_bits must be 32 or 64")
            self.string_bits = bits
            self._orbsym = _host(np.zeros(norb) if orbsym is None else orbsym, np.int64)
            create = L.bsim_basis_create_u32 if bits == 32 else L.bsim_basis_create_u64
            _check(create(norb, na, nb, total_sym, self._orbsym.ctypes.data, num_irreps, C.byref(out)),
                   f"bsim_basis_create_u{bits}")
        self.h = out.value
        self.norb, self.nelec = norb, (na, nb)
        self.dim = L.bsim_basis_dim(self.h)

    def find_det(self, astr: int, bstr: int) -> int:
        return lib().bsim_basis_find_det(self.h, astr, bstr)

    def hf_index(self) -> int:
        """Index of the Hartree-Fock determinant (``get_hf``, jl/network.jl:81-116)."""
        na, nb = self.nelec
        return self.find_det((1 << na) - 1, (1 << nb) - 1)

    def close(self):
        if getattr(self, "h", None):
            lib().bsim_basis_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CuNetwork:
    """Device OTF network (``Network_OTF`` + ``upload_network``)."""

    def __init__(self, net: Optional[nw.OTFNetwork] = None, host_handle: Optional[int] = None,
                 string_bits: Optional[int] = None):
        """string_bits must match the basis the network is used with (default: 32
        up to 32 orbitals, else 64)."""
        L = lib()
        out = vp()
        if host_handle is not None:
            _check(L.bsim_network_from_host(host_handle, C.byref(out)), "bsim_network_from_host")
        else:
            bits = string_bits or (32 if net.norb <= 32 else 64)
            if bits == 32:
                a = net.as_uint32()
            else:
                a = {k: _host(getattr(net, k), np.uint64) for k in ("axs", "bxs", "flat_zas", "flat_zbs")}
            self._keep = [
                _host(net.orbsym, np.int64), a["axs"], a["bxs"], _host(net.ranks, np.int64),
                _host(net.num_zas, np.int64), _host(net.num_zbs, np.int64), a["flat_zas"], a["flat_zbs"],
                _host(net.flat_wa, np.float64), _host(net.flat_wb, np.float64)]
            k = self._keep
            create = L.bsim_network_create_u32 if bits == 32 else L.bsim_network_create_u64
            _check(create(k[0].ctypes.data, net.norb, net.ngs, *[x.ctypes.data for x in k[1:]], C.byref(out)),
                   f"bsim_network_create_u{bits}")
        self.h = out.value
        self.ngs = L.bsim_network_ngs(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().bsim_network_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CuNetworkC64:
    """Device OTF network with complex weights (the reference's _c64 networks):
    ``wa``, ``wb`` are complex128 arrays in the order of ``net.flat_wa`` /
    ``net.flat_wb`` (the real ``net`` supplies masks, ranks and counts)."""

    def __init__(self, net: nw.OTFNetwork, wa, wb, string_bits: Optional[int] = None):
        L = lib()
        out = vp()
        bits = string_bits or (32 if net.norb <= 32 else 64)
        if bits == 32:
            a = net.as_uint32()
        else:
            a = {k: _host(getattr(net, k), np.uint64) for k in ("axs", "bxs", "flat_zas", "flat_zbs")}
        self._keep = [
            _host(net.orbsym, np.int64), a["axs"], a["bxs"], _host(net.ranks, np.int64),
            _host(net.num_zas, np.int64), _host(net.num_zbs, np.int64), a["flat_zas"], a["flat_zbs"],
            np.ascontiguousarray(wa, np.complex128), np.ascontiguousarray(wb, np.complex128)]
        k = self._keep
        create = L.bsim_network_create_c64 if bits == 32 else L.bsim_network_create_c64_u64
        _check(create(k[0].ctypes.data, net.norb, net.ngs, *[x.ctypes.data for x in k[1:]], C.byref(out)),
               "bsim_network_create_c64")
        self.h = out.value
        self.ngs = L.bsim_network_ngs(self.h)

    close = CuNetwork.close
    __del__ = CuNetwork.__del__


class CuOTFC64:
    """Complex operators on complex128 torch tensors (the reference CPU library's
    _c64 interface, jl/network.jl:516-556, on the GPU); group indices 0-based."""

    def __init__(self, basis: "CuBasis", net: CuNetworkC64):
        self.basis, self.net = basis, net
        import torch
        self._slot = torch.zeros(2, dtype=torch.float64, device="cuda")

    def _c(self, name, *args):
        _check(getattr(lib(), name)(self.basis.h, self.net.h, *args), name)

    def hvec(self, src, dst, stream=None):
        self._c("bsim_hvec_c64", _ptr(src), _ptr(dst), _stream(stream))

    def get_diags(self, d, stream=None):
        self._c("bsim_diag_c64", _ptr(d), _stream(stream))

    def expm(self, idx: int, theta: float, v, stream=None):
        self._c("bsim_expm_c64", idx, theta, _ptr(v), _stream(stream))

    def grad(self, idx: int, theta: float, l, r, stream=None) -> complex:
        self._c("bsim_grad_c64", idx, theta, _ptr(l), _ptr(r), _ptr(self._slot), _stream(stream))
        re, im = self._slot.tolist()
        return complex(re, im)

    def backgrad(self, idx: int, theta: float, l, r, stream=None) -> complex:
        self._c("bsim_backgrad_c64", idx, theta, _ptr(l), _ptr(r), _ptr(self._slot), _stream(stream))
        re, im = self._slot.tolist()
        return complex(re, im)

    def tvec(self, idx: int, src, dst, stream=None):
        self._c("bsim_tvec_c64", idx, _ptr(src), _ptr(dst), _stream(stream))

    def backtran(self, idx: int, theta: float, l, r, b, stream=None):
        self._c("bsim_backtran_c64", idx, theta, _ptr(l), _ptr(r), _ptr(b), _stream(stream))

    def batchexpm(self, idx: int, theta: float, mat, ld: int, nv: int, stream=None):
        self._c("bsim_batchexpm_c64", idx, theta, _ptr(mat), ld, nv, _stream(stream))

    def batchgrad(self, thetas, l, r, grads, stream=None):
        th = _host(thetas, np.float64)
        self._c("bsim_batchgrad_c64", th.ctypes.data, _ptr(l), _ptr(r), _ptr(grads), _stream(stream))

    def batchtran(self, l, r, trans, stream=None):
        self._c("bsim_batchtran_c64", _ptr(l), _ptr(r), _ptr(trans), _stream(stream))


class CuOTFFunctions:
    """The operator closures of ``CuOTF_Functions`` (jl/cuda/cunetwork.jl:74-160).

    Generator indices are 1-based as in the Julia closures (they pass idx-1 to
    the C-ABI).  Vectors are float64 torch CUDA tensors of length ``basis.dim``.
    """

    def __init__(self, basis: CuBasis, ham: Optional[CuNetwork] = None, pool: Optional[CuNetwork] = None):
        self.basis, self.ham, self.pool = basis, ham, pool
        import torch
        self._scalar = torch.zeros(1, dtype=torch.float64, device="cuda")

    # -- jl/cuda/cunetwork.jl:105-150 --------------------------------------
    def hvec(self, v, Hv, stream=None):
        _check(lib().bsim_hvec(self.basis.h, self.ham.h, _ptr(v), _ptr(Hv), _stream(stream)), "hvec")

    def hvec_mixed(self, v, Hv, stream=None):
        _check(lib().bsim_hvec_mixed(self.basis.h, self.ham.h, _ptr(v), _ptr(Hv), _stream(stream)), "hvec_mixed")

    def hvec_tiles(self, v, Hv, tile_lo: int, tile_hi: int, mixed=False, stream=None):
        """sigma on destination tiles [tile_lo, tile_hi) only (row sharding)."""
        _check(lib().bsim_hvec_tiles(self.basis.h, self.ham.h, _ptr(v), _ptr(Hv), tile_lo, tile_hi,
                                     1 if mixed else 0, _stream(stream)), "hvec_tiles")

    def sigma_path(self):
        """(path, reason, residual groups): path 1 structured, 2 structured with the FP64
        source row in global memory, 0 generic."""
        buf = C.create_string_buffer(256)
        nres = C.c_int()
        r = lib().bsim_hvec_path(self.basis.h, self.ham.h, buf, 256, C.byref(nres))
        if r < 0:
            _check(r, "hvec_path")
        return r, buf.value.decode(), nres.value

    def hvec_host(self, srcs, dsts, mixed=False, stream=None):
        """dsts[k] = H srcs[k] for host tensors/arrays (dim float64 each), the copies of
        neighbouring steps overlapped with sigma; pinned host memory lets them overlap."""
        n = len(srcs)
        if len(dsts) != n:
            raise ValueError("srcs and dsts differ in length")
        sp = (C.c_void_p * max(n, 1))(*[_ptr(x) for x in srcs])
        dp = (C.c_void_p * max(n, 1))(*[_ptr(x) for x in dsts])
        _check(lib().bsim_hvec_host(self.basis.h, self.ham.h, n, sp, dp, 1 if mixed else 0, _stream(stream)),
               "hvec_host")

    def hvec_cols(self, v, Hv, col_lo: int, col_hi: int, mixed=False, stream=None):
        """sigma on beta columns [col_lo, col_hi) only (column-band sharding)."""
        _check(lib().bsim_hvec_cols(self.basis.h, self.ham.h, _ptr(v), _ptr(Hv), col_lo, col_hi, 1 if mixed else 0,
                                    _stream(stream)), "hvec_cols")

    STAGES = ("frame_transpose", "pure_alpha", "pure_beta", "mixed_gemm", "mixed_gather", "final", "residual",
              "ri_gemm", "ri_gather")

    def sigma_stage_times(self, v, Hv, mixed=False, stream=None):
        """One structured sigma with CUDA events per launch: {stage: (ms, launches)}."""
        n = len(self.STAGES)
        ms, nl = (C.c_double * n)(), (C.c_int * n)()
        _check(lib().bsim_hvec_stage_times(self.basis.h, self.ham.h, _ptr(v), _ptr(Hv), 1 if mixed else 0, ms, nl, n,
                                           _stream(stream)), "hvec_stage_times")
        return {k: (ms[i], nl[i]) for i, k in enumerate(self.STAGES)}

    def num_tiles(self) -> int:
        return lib().bsim_hvec_num_tiles(self.basis.h)

    def get_diags(self, dv, stream=None):
        _check(lib().bsim_diag(self.basis.h, self.ham.h, _ptr(dv), _stream(stream)), "get_diags")

    def expm(self, idx: int, theta: float, v, stream=None):
        _check(lib().bsim_expm(self.basis.h, self.pool.h, idx - 1, theta, _ptr(v), _stream(stream)), "expm")

    def grad(self, idx: int, theta: float, lv, rv, stream=None) -> float:
        _check(lib().bsim_grad(self.basis.h, self.pool.h, idx - 1, theta, _ptr(lv), _ptr(rv),
                               _ptr(self._scalar), _stream(stream)), "grad")
        return float(self._scalar.item())

    def backgrad(self, idx: int, theta: float, lv, rv, stream=None) -> float:
        _check(lib().bsim_backgrad(self.basis.h, self.pool.h, idx - 1, theta, _ptr(lv), _ptr(rv),
                                   _ptr(self._scalar), _stream(stream)), "backgrad")
        return float(self._scalar.item())

    def batchgrad(self, lv, rv, grads, x, stream=None):
        _check(lib().bsim_batchgrad(self.basis.h, self.pool.h, _ptr(x), _ptr(lv), _ptr(rv), _ptr(grads),
                                    _stream(stream)), "batchgrad")

    # the CPU-only operators of the reference (jl/network.jl:451-466)
    def tvec(self, idx: int, lv, rv, stream=None):
        """|rv> = T_idx |lv> (1-based idx)."""
        _check(lib().bsim_tvec(self.basis.h, self.pool.h, idx - 1, _ptr(lv), _ptr(rv), _stream(stream)), "tvec")

    def backtran(self, idx: int, theta: float, lv, rv, tlv, stream=None):
        """lv, rv <- exp(theta T_idx) lv, rv; tlv = T_idx lv (rotated)."""
        _check(lib().bsim_backtran(self.basis.h, self.pool.h, idx - 1, theta, _ptr(lv), _ptr(rv), _ptr(tlv),
                                   _stream(stream)), "backtran")

    def batchexpm(self, idx: int, theta: float, mat, N: int, j: int, stream=None):
        """exp(theta T_idx) on the first j of the N entries each determinant holds in mat
        (Julia's N x dim column-major matrix, i.e. a row-major dim x N array)."""
        _check(lib().bsim_batchexpm(self.basis.h, self.pool.h, idx - 1, theta, _ptr(mat), N, j, _stream(stream)),
               "batchexpm")

    def batchtran(self, lv, rv, trans, stream=None):
        """trans[g] = <lv|T_g|rv> for every pool group."""
        _check(lib().bsim_batchtran(self.basis.h, self.pool.h, _ptr(lv), _ptr(rv), _ptr(trans), _stream(stream)),
               "batchtran")

    # -- sequence-level entry points ------------------------------------------
    def expm_seq(self, idxs: Sequence[int], thetas: Sequence[float], v, stream=None):
        """Apply exp(theta_i G_{idx_i}) for i in order (1-based idx)."""
        ii = _host(np.asarray(idxs) - 1, np.int64)
        tt = _host(thetas, np.float64)
        _check(lib().bsim_expm_seq(self.basis.h, self.pool.h, len(ii), ii.ctypes.data, tt.ctypes.data, _ptr(v),
                                   _stream(stream)), "expm_seq")

    def prepare_state(self, op_idx, param_idx, thetas, ref_idx, ref_val, v, stream=None):
        """v = prod exp(thetas[param_idx[i]] G_{op_idx[i]}) |ref> (0-based indices)."""
        o, p = _host(op_idx, np.int64), _host(param_idx, np.int64)
        t, ri, rv = _host(thetas, np.float64), _host(ref_idx, np.int64), _host(ref_val, np.float64)
        _check(lib().bsim_prepare_state(self.basis.h, self.pool.h, len(o), o.ctypes.data, p.ctypes.data,
                                        t.ctypes.data, ri.ctypes.data, rv.ctypes.data, len(ri), _ptr(v),
                                        _stream(stream)), "prepare_state")

    def energy_grad(self, op_idx, param_idx, thetas, ref_idx, ref_val, lv, rv, ckpt_every: int = 64, stream=None):
        """(energy, gradient[n_params], variance) by the adjoint sweep (jl/vqe.jl:1-21)."""
        o, p = _host(op_idx, np.int64), _host(param_idx, np.int64)
        t, ri, rvv = _host(thetas, np.float64), _host(ref_idx, np.int64), _host(ref_val, np.float64)
        g = np.zeros(len(t))
        e, var = C.c_double(), C.c_double()
        _check(lib().bsim_vqe_energy_grad(self.basis.h, self.ham.h, self.pool.h, len(o), o.ctypes.data,
                                          p.ctypes.data, len(t), t.ctypes.data, ri.ctypes.data, rvv.ctypes.data,
                                          len(ri), ckpt_every, _ptr(lv), _ptr(rv), C.byref(e), C.byref(var),
                                          g.ctypes.data, _stream(stream)), "vqe_energy_grad")
        return e.value, g, var.value

    def davidson(self, v0, diags, x_out, tol=1e-5, maxiter=200, ncv=3, maxspace=23, mixed=False, verbose=False,
                 stream=None):
        """Lowest eigenpair (jl/davidson.jl:1-185).  Returns a stats dict."""
        e, r = C.c_double(), C.c_double()
        it, s64, s32 = C.c_int(), C.c_int(), C.c_int()
        _check(lib().bsim_davidson(self.basis.h, self.ham.h, _ptr(v0), _ptr(diags), tol, maxiter, ncv, maxspace,
                                   1 if mixed else 0, _ptr(x_out), C.byref(e), C.byref(r), C.byref(it),
                                   C.byref(s64), C.byref(s32), 1 if verbose else 0, _stream(stream)), "davidson")
        return dict(energy=e.value, residual=r.value, iterations=it.value, sigma_fp64=s64.value,
                    sigma_fp32=s32.value)

    def davidson_block(self, X, diags, nroots, tol=1e-5, maxiter=200, ncv=None, maxspace=None, mixed=False,
                       verbose=False, stream=None):
        """Lowest ``nroots`` eigenpairs by block Davidson.  X (device, nroots x dim FP64):
        start vectors in, Ritz vectors out; diags FP64 or FP32 (device).  Returns a
        stats dict with per-root energies and FP64 residual norms."""
        ncv = nroots if ncv is None else ncv
        maxspace = ncv + 2 * nroots if maxspace is None else maxspace
        d32 = 1 if str(diags.dtype).endswith("float32") else 0
        en, rs = (C.c_double * nroots)(), (C.c_double * nroots)()
        it, s64, s32 = C.c_int(), C.c_int(), C.c_int()
        _check(lib().bsim_davidson_block(self.basis.h, self.ham.h, nroots, _ptr(X), _ptr(diags), d32, tol, maxiter,
                                         ncv, maxspace, 1 if mixed else 0, en, rs, C.byref(it), C.byref(s64),
                                         C.byref(s32), 1 if verbose else 0, _stream(stream)), "davidson_block")
        return dict(energies=list(en), residuals=list(rs), iterations=it.value, sigma_fp64=s64.value,
                    sigma_fp32=s32.value, converged=all(r < tol for r in rs))
