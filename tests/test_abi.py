"""The C-ABI library loads and exports every symbol include/chfsi.h declares."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "chfsi.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(chfsi_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("chfsi_create", "chfsi_destroy", "chfsi_chebyshev_filter", "chfsi_rayleigh_ritz",
                 "chfsi_diagonalize", "chfsi_apply_h", "chfsi_scf_run"):
        assert must in names


def test_library_exports_every_declared_symbol(chfsi):
    lib = ctypes.CDLL(chfsi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_sm100a_only():
    import subprocess
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf",
                          os.path.join(ROOT, "chemrust-scf_b200", "libchfsi_b200.so")],
                         capture_output=True, text=True).stdout
    archs = set(re.findall(r"sm_(\d+a?)", out))
    assert archs == {"100a"}, archs


def test_no_device_is_an_error_not_a_fallback(chfsi):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    s = chfsi.SyntheticSystem(config_index=0)
    with pytest.raises(chfsi.NoDevice):
        chfsi.Context(s)


def test_bad_input_rejected(chfsi):
    d = chfsi.Dims()
    d.n_pw = 0
    h = ctypes.c_void_p()
    assert chfsi.lib().chfsi_create(ctypes.byref(d), None, ctypes.byref(h)) == chfsi.BAD_INPUT
