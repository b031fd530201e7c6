"""CPU tests of the C ABI: the libraries load and export every function the headers declare,
the drop-in structs have the reference's layout, and the host-side coefficient code matches
the reference's coefficients() bit for bit.  No kernel is launched (no GPU here)."""
import ctypes as C
import os
import re
import subprocess
import textwrap

import numpy as np
import pytest
from conftest import ROOT

import hackathon_b200 as hh

INCLUDE = os.path.join(ROOT, "include")


def declared_functions(header: str) -> list[str]:
    text = open(os.path.join(INCLUDE, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-zA-Z_]\w*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "defined")))


def exported(lib_path: str) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_libhh_exports_every_declared_symbol():
    names = declared_functions("hh.h")
    assert len(names) >= 25
    syms = exported(hh.LIB_PATH)
    missing = [n for n in names if n not in syms]
    assert not missing, missing
    assert set(names) <= set(hh.SIGNATURES), set(names) - set(hh.SIGNATURES)
    hh.lib()  # every declared symbol resolves through ctypes


@pytest.mark.parametrize("header,lib,expect", [
    ("hh_dropin2d.h", hh.DROPIN2D_PATH, {"solver", "forwardDST", "reverseDST", "hh2d_status"}),
    ("hh_dropin3d.h", hh.DROPIN3D_PATH, {"solver", "DST", "hh3d_status"}),
])
def test_dropin_libraries_export_reference_entry_points(header, lib, expect):
    assert set(declared_functions(header)) == expect
    assert expect <= exported(lib)
    C.CDLL(lib)  # loads (and pulls libhh.so through its rpath)


def _compile_run(src: str, d) -> str:
    c = os.path.join(str(d), "abi_probe.c")
    exe = os.path.join(str(d), "abi_probe")
    open(c, "w").write(src)
    r = subprocess.run(["/usr/bin/gcc", "-I", INCLUDE, c, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return subprocess.run([exe], capture_output=True, text=True).stdout


def test_dropin_struct_layouts_match_reference(tmp_path):
    """192-byte 2D System / 312-byte 3D System with the reference's field offsets
    (2D_Program/headers/structs.h:20-30, 3D_Program/headers/structs.h:46-58)."""
    out = _compile_run(textwrap.dedent("""
        #include <stdio.h>
        #include <stddef.h>
        #include "hh_dropin2d.h"
        #define hh2d_order hh3d_order_unused
        int main(void) {
            printf("%zu %zu %zu %zu %zu\\n", sizeof(hh2d_System), sizeof(hh2d_Lattice),
                   offsetof(hh2d_System, order), offsetof(hh2d_System, k), offsetof(hh2d_System, am));
            printf("%zu\\n", sizeof(hh2d_DSTN));
            return 0;
        }"""), tmp_path)
    assert out.split() == ["192", "64", "68", "72", "184", "16"]
    out3 = _compile_run(textwrap.dedent("""
        #include <stdio.h>
        #include <stddef.h>
        #include "hh_dropin3d.h"
        int main(void) {
            printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(hh3d_System), sizeof(hh3d_Lattice),
                   offsetof(hh3d_System, order), offsetof(hh3d_System, a), offsetof(hh3d_System, A),
                   offsetof(hh3d_System, sol), offsetof(hh3d_System, error));
            return 0;
        }"""), tmp_path)
    assert out3.split() == ["312", "88", "88", "96", "208", "288", "304"]


def test_ctypes_mirrors_have_reference_sizes():
    from oracle import System2D, System3D
    assert C.sizeof(System2D) == 192 and C.sizeof(System3D) == 312


@pytest.mark.parametrize("order", [2, 4, 6])
@pytest.mark.parametrize("k", [10.0, 50.0, 3.0 + 0.5j])
def test_host_coefficients_match_reference_2d(oracle, order, k):
    n = 37
    ours = hh.coefficients(2, n, order, k)
    pb, keep = oracle.problem2d(n, order, k, np.zeros((n + 2, n + 2), dtype=complex))
    ref = oracle.coefficients_2d(pb)
    for nm in ("bp", "ap", "b", "a", "bm", "am"):
        assert np.array_equal(ours[nm], ref[nm]), nm


@pytest.mark.parametrize("order", [2, 4, 6])
def test_host_coefficients_match_reference_3d(oracle, order):
    n, k = 21, 30.0
    h = 1.0 / (n + 1)
    ours = hh.coefficients(3, n, order, k)
    pb, keep = oracle.problem3d(n, order, np.full(n + 2, complex(k) ** 2), np.zeros((n + 2,) * 3, complex), h)
    ref = oracle.coefficients_3d(pb)
    for nm in ref:
        assert np.array_equal(ours[nm], ref[nm]), nm


def test_invalid_arguments_are_rejected_without_a_gpu():
    L = hh.lib()
    assert L.hh_coefficients2d(0, 6, 1.0, 0.0, None) == 1
    arr = [np.zeros(4, complex) for _ in range(6)]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arr])
    assert L.hh_coefficients2d(4, 5, 1.0, 0.0, ptrs) == 1  # order 5: HH_ERR_INVALID
    assert L.hh_dst1_rows(None, 7, 1, None, 7, None, 7) == 1
    assert L.hh_solve(None, None, None, 1) == 1
    assert b"invalid" in L.hh_last_error()
    assert L.hh_server_inject_error(None, 1) == 1
