"""The C-ABI library loads and exports every entry point of include/mslice.h
(runs without a GPU; no compute call is made)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "mslice.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ms_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def libpath():
    from cudamultislice_b200 import build

    return build.build(verbose=False)


def test_header_declares_the_reference_method_list():
    names = header_functions()
    # one entry per method of UnmanagedMultisliceSimulation's public API
    # (unmanagedGUISimulation.cuh:154-195) plus the managed wrapper getters
    for n in ["ms_import_atoms", "ms_upload_binned_atoms", "ms_upload_binned_atoms_tds", "ms_get_parameterisation",
              "ms_apply_microscope_parameters", "ms_set_calculation_variables", "ms_stem_set_calculation_variables",
              "ms_precalculate_frequencies", "ms_initialise_wavefunctions", "ms_initialise_wavefunctions_dz",
              "ms_stem_initialise_wavefunctions", "ms_alloc_tds", "ms_multislice_step_fd",
              "ms_multislice_step_conventional", "ms_alloc_host_image", "ms_simulate_image", "ms_get_exit_wave",
              "ms_get_stem_exit_wave", "ms_free_exit_wave", "ms_add_tds_waves", "ms_get_ew_value_abs",
              "ms_get_ew_value_re", "ms_get_ew_value_im", "ms_get_im_value", "ms_get_dqe_im_value", "ms_get_tds_min", "ms_get_tds_max",
              "ms_get_tds_val", "ms_get_image_contrast", "ms_get_size_x", "ms_get_size_y", "ms_get_size_z",
              "ms_get_slices", "ms_get_kmax", "ms_get_im_min", "ms_get_im_max", "ms_get_ew_min", "ms_get_ew_max"]:
        assert n in names, n


def test_library_exports_every_declared_symbol(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (ms_[a-z0-9_]+)\b", out))
    missing = [n for n in header_functions() if n not in exported]
    assert not missing, missing


def test_ctypes_signatures_cover_the_header(libpath):
    from cudamultislice_b200 import _lib

    assert sorted(_lib.SIGNATURES) == header_functions()
    L = _lib.lib()
    for n in header_functions():
        assert getattr(L, n) is not None


def test_library_links_no_torch(libpath):
    out = subprocess.run(["ldd", libpath], capture_output=True, text=True).stdout
    assert "torch" not in out
    assert "libcufft" in out


def test_version_string(libpath):
    from cudamultislice_b200 import _lib

    assert b"sm_100a" in _lib.lib().ms_version()


def test_null_handle_is_rejected(libpath):
    from cudamultislice_b200 import _lib

    L = _lib.lib()
    assert L.ms_multislice_step_conventional(None, 1) == 1
    assert L.ms_destroy(None) == 1
    out = C.c_float()
    assert L.ms_get_kmax(None, C.byref(out)) == 1
