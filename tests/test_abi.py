"""The C-ABI library loads and exports every symbol include/newton_b200.h declares (no GPU needed)."""

import ctypes as C
import os
import re
import subprocess

import pytest

from newton_custom_contact_b200 import _abi, _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_lib.LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "newton_custom_contact_b200", "csrc")], check=True)
    return _lib.load()


def declared_functions():
    src = open(os.path.join(ROOT, "include", "newton_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|int32_t|int64_t)\s+(nb_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert set(names) == set(_lib.EXPORTS)


def test_library_exports_all_symbols(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.nb_abi_version() == _abi.NB_ABI_VERSION


def test_struct_sizes_match_header():
    # pointer-sized fields after the int header; sizes must be multiples of 8
    assert C.sizeof(_abi.NbModelDesc) == 12 * 4 + 8 + 8 * (len(_abi.NbModelDesc._fields_) - 13)
    assert C.sizeof(_abi.NbContactSeg) == 9 * 8
    assert C.sizeof(_abi.NbXpbdParams) == 4 * 4 + 6 * 4
    assert C.sizeof(_abi.NbStepIO) == 9 * 8


def test_invalid_arguments_rejected_without_gpu(lib):
    # a NULL descriptor is rejected before any CUDA call
    assert lib.nb_collide(None, None, None, 0, None) == _abi.NB_ERR_INVALID
    assert lib.nb_xpbd_step(None, None, None, None, 0.01, 0, None) == _abi.NB_ERR_INVALID
    assert lib.nb_publish_contacts(None, None, None, None) == _abi.NB_ERR_INVALID
    assert lib.nb_ingest_contacts(None, None, None, None) == _abi.NB_ERR_INVALID
