"""The C-ABI library without a GPU: it loads, exports every symbol the header
declares, and rejects bad arguments with status codes (no compute calls)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from binsim_b200 import cuotf
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_symbol():
    L = cuotf.lib()
    syms = cuotf.header_symbols()
    assert len(syms) >= 40
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_reference_entry_points_present():
    # names bound by jl/cuda/cunetwork.jl
    L = cuotf.lib()
    for s in ["sync_device_cuda", "build_basisdev_f64", "destroy_basisdev_f64", "build_networkdev_f64",
              "destroy_networkdev_f64", "hvec_cuda", "get_diags_elements_cuda", "expm_cuda", "grad_cuda",
              "backgrad_cuda", "batchgrad_cuda", "expm_cuda_2d", "grad_cuda_2d", "backgrad_cuda_2d"]:
        assert hasattr(L, s)


def test_bad_handles_are_rejected():
    L = cuotf.lib()
    assert L.bsim_hvec(None, None, None, None, None) == cuotf.CuOTFError.__init__.__code__.co_argcount * 0 - 2
    junk = np.zeros(64, np.uint8)   # valid memory, wrong magic word
    assert L.bsim_hvec(junk.ctypes.data, None, None, None, None) == -2
    assert b"invalid basis handle" in L.bsim_last_error()
    assert L.bsim_basis_dim(None) == -1
    assert L.bsim_network_ngs(junk.ctypes.data) == -1
    assert L.bsim_basis_destroy(None) == -2


def test_out_pointer_null_is_rejected():
    L = cuotf.lib()
    o = np.zeros(4, np.int64)
    assert L.bsim_basis_create_u32(4, 2, 2, 0, o.ctypes.data, 16, None) == -1
    assert L.bsim_network_create_u32(o.ctypes.data, 4, 0, *([None] * 10)) == -1


def test_legacy_entry_points_do_not_exit_on_bad_handles(capfd):
    L = cuotf.lib()
    L.hvec_cuda(None, None, None, None)
    assert L.grad_cuda(None, None, 0, 0.1, None, None) == 0.0
    err = capfd.readouterr().err
    assert "hvec_cuda" in err and "grad_cuda" in err


@pytest.mark.skipif(not orc.ref_sources_present(), reason="reference headers absent")
def test_host_handle_layout_mirror_matches_reference(tmp_path):
    """refmirror.h reproduces the field offsets of the reference's host objects."""
    prog = r'''
#include <cstddef>
#include <cstdio>
#include "basis/basis.hpp"
#include "ham/otf.hpp"
#include "refmirror.h"
#define P(a,b,f) printf("%zu %zu\n", offsetof(a,f), offsetof(b,f))
int main(){
  using RB = BasisManager<uint32>; using MB = bsim::refmirror::BasisManager32;
  P(RB,MB,blocks); P(RB,MB,num_blocks); P(RB,MB,orbsym); P(RB,MB,num_irreps); P(RB,MB,total_sym);
  P(RB,MB,dim); P(RB,MB,norb); P(RB,MB,a_idx_map);
  using RD = BlockDesc<uint32>; using MD = bsim::refmirror::BlockDesc32;
  P(RD,MD,astrs); P(RD,MD,bstrs); P(RD,MD,offset);
  printf("%zu %zu\n", sizeof(RD), sizeof(MD));
  using RG = SVDGroup_OTF<uint32,double>; using MG = bsim::refmirror::SVDGroup32;
  P(RG,MG,rank); P(RG,MG,original_idx); P(RG,MG,num_za); P(RG,MG,unique_zas); P(RG,MG,num_zb);
  P(RG,MG,unique_zbs); P(RG,MG,wa); P(RG,MG,wb);
  printf("%zu %zu\n", sizeof(RG), sizeof(MG));
  using RN = Network_OTF<uint32,double>; using MN = bsim::refmirror::NetworkOTF32;
  P(RN,MN,diag_groups); P(RN,MN,pure_a_groups); P(RN,MN,pure_b_groups); P(RN,MN,mixed_groups);
  P(RN,MN,sorted_idxs); P(RN,MN,excit_types); P(RN,MN,orbsym);
  return 0; }
'''
    src = tmp_path / "layout.cpp"
    src.write_text(prog)
    exe = tmp_path / "layout"
    subprocess.run(["g++", "-std=c++20", "-fopenmp", "-Wno-invalid-offsetof", "-I" + os.path.join(orc.REF_SRC, "src", "include"),
                    "-I" + os.path.join(ROOT, "binsim_b200", "csrc"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in filter(None, out):
        a, b = line.split()
        assert a == b, out
