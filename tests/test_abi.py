"""C-ABI boundary (CPU): the library loads, exports every entry point that
include/glst_c.h declares, and reports errors as status codes."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, cuda_available

HEADER = os.path.join(ROOT, "include", "glst_c.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(glst_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for n in ("glst_create", "glst_create_ncell", "glst_init", "glst_destroy", "glst_compute",
              "glst_assign_atoms", "glst_calc_sf", "glst_sum_rmt_sf", "glst_calc_lr_ef",
              "glst_calc_sr_ef", "glst_comm_ef", "glst_get_ef", "glst_energy"):
        assert n in names


def test_library_exports_every_declared_symbol(pkg):
    lib = ctypes.CDLL(pkg.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_the_header(pkg):
    from glst_b200 import _SIGNATURES
    assert set(declared_functions()) <= set(_SIGNATURES)


def test_status_strings_and_version(pkg):
    lib = pkg.load_library()
    assert lib.glst_status_string(0) == b"ok"
    assert lib.glst_status_string(4).startswith(b"spherical")
    assert b"sm_100a" in lib.glst_version()
    assert lib.glst_max_atoms_per_cell() == 8192


def test_bad_arguments_return_status(pkg):
    lib = pkg.load_library()
    assert lib.glst_create(None, 10, 1e-6, 10.0, 10.0, 10.0, 5.0, 0) == 1
    assert lib.glst_compute(None, None, None, None, None, None) == 1
    assert b"null" in lib.glst_last_error()
    with pytest.raises(pkg.GlstError):
        pkg.plan(10, -1.0, (10.0, 10.0, 10.0), 5.0)
    with pytest.raises(pkg.GlstError):
        pkg.plan(10, 1e-6, (0.0, 1.0, 1.0), 5.0)


@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly(pkg):
    with pytest.raises(pkg.GlstError) as e:
        pkg.GlstForce(648, 1.676e-6, 18.63, 18.63, 18.63, rcut=9.0)
    assert e.value.status == 3  # GLST_ERR_NO_DEVICE
