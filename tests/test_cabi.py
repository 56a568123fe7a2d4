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
