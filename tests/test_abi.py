"""The C-ABI library loads and exports every entry point include/defmm_b200.h
declares (no compute call: these tests run without a GPU)."""
import ctypes
import os
import re

import pytest

from defmm_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "defmm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(defmm_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ["defmm_create", "defmm_destroy", "defmm_prcmpt", "defmm_gemv", "defmm_gemv_device",
              "defmm_gemv_batched", "defmm_check_full", "defmm_load_inp", "defmm_add_source_particle",
              "defmm_add_target_particle"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(api._LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_create_destroy_without_device():
    A = api.IBFMM_Mat()
    assert A.info("n_sources") == 0
    del A


def test_argument_checks_without_device():
    # calls that must be rejected before touching a device
    A = api.IBFMM_Mat()
    for nt, bps in ((64, 16), (128, -1), (256, 65)):
        with pytest.raises(api.DefmmError):
            A.set_launch(nt, bps)
    A.set_launch(256, 8)  # valid choices are recorded without a device
    with pytest.raises(api.DefmmError):
        A._check(api.lib().defmm_set_m2l_pairing(A._h, 2))
    A.set_m2l_pairing(True)
    A.set_m2l_pairing(False)
    for rb, g in ((0, 0), (33, 0), (4, -1)):
        with pytest.raises(api.DefmmError):
            A.set_blocking(rb, g)
    A.set_blocking(8, 3)
    for rb in (0, 3, 16, -4):
        with pytest.raises(api.DefmmError):
            A.set_rhs_per_cta(rb)
    A.set_rhs_per_cta(4)
    with pytest.raises(api.DefmmError):
        A._check(api.lib().defmm_set_m2l_staging(A._h, 2))
    A.set_m2l_staging(False)
    A.set_m2l_staging(True)
    with pytest.raises(api.DefmmError):
        A.autotune(reps=0)
    with pytest.raises(api.DefmmError):
        A.autotune(reps=1)  # before prcmpt
    L = api.lib()
    assert L.defmm_mlp_forward(None, None, 1, None, None, None, None) == api.lib().defmm_mlp_forward(
        None, None, 0, None, None, None, None) != 0
    assert L.defmm_mlp_adam(None, None, None, None, 0, 1e-3, 0.0, None) != 0
