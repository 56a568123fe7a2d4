"""The C-ABI library loads without a GPU and exports every declared symbol."""

import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "psipm_b200.h")
LIB = os.path.join(ROOT, "mf-psipm_b200", "psipm_b200", "libpsipm_b200.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(psipm_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("psipm_create", "psipm_destroy", "psipm_set_theta", "psipm_scores",
                     "psipm_refresh_core", "psipm_factor", "psipm_apply", "psipm_matvec",
                     "psipm_pcg", "psipm_solve"):
        assert required in names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build the library first: make -C mf-psipm_b200"
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_signatures_cover_header():
    from psipm_b200 import _lib

    assert set(_lib.SIGNATURES) == set(declared_functions())


def test_header_compiles_as_c_and_links(tmp_path):
    """include/psipm_b200.h is plain C99: a C caller compiles against it, links
    the library and gets the documented argument error (no GPU involved)."""
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        import pytest

        pytest.skip("gcc not available")
    src = tmp_path / "caller.c"
    src.write_text(r'''
#include <stdio.h>
#include "psipm_b200.h"
int main(void) {
    psipm_handle* h = 0;
    int64_t colptr[2] = {0, 0};
    int rc = psipm_create(0, 1, 0, colptr, 0, 0, 0, PSIPM_FP64, &h);
    int rc2 = psipm_solve(0, 0, 0, 1e-8, 10, PSIPM_PCG_SPECTRAL, 100, 0.1, 0, 0, 0, 0, 0, 0, 0);
    printf("%d %d %lld\n", rc, rc2, (long long)psipm_num_candidates(0));
    psipm_destroy(0);
    return (rc == PSIPM_ERR_ARGUMENT && rc2 == PSIPM_ERR_ARGUMENT) ? 0 : 1;
}
''')
    exe = tmp_path / "caller"
    libdir = os.path.dirname(LIB)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe), "-L", libdir, "-lpsipm_b200", f"-Wl,-rpath,{libdir}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.split() == ["-1", "-1", "-1"]
