"""The C-ABI library loads and exports every symbol include/newton_b200.h declares (no GPU needed)."""

import ctypes as C
import os
import re
import subprocess

import pytest

from newton_custom_contact_b200 import _abi, _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", params=sorted(_lib.BUILDS))
def lib(request):
    """Both builds of the library (product and parity) export the same ABI."""
    if not all(os.path.exists(p) for p in _lib.BUILDS.values()):
        subprocess.run(["make", "-s", "-j", "8", "-C", os.path.join(ROOT, "newton_custom_contact_b200", "csrc")],
                       check=True)
    return _lib.load(_lib.BUILDS[request.param])


def declared_functions():
    src = open(os.path.join(ROOT, "include", "newton_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|int32_t|int64_t|const char\*)\s+(nb_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert set(names) == set(_lib.EXPORTS)


def test_library_exports_all_symbols(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.nb_abi_version() == _abi.NB_ABI_VERSION


def test_struct_layouts_match_header(tmp_path):
    """sizeof / offsetof of every struct, compiled from the header, equal the ctypes mirrors."""
    structs = {"NbModelDesc": _abi.NbModelDesc, "NbContactSeg": _abi.NbContactSeg,
               "NbContactsPublic": _abi.NbContactsPublic, "NbXpbdParams": _abi.NbXpbdParams,
               "NbStepIO": _abi.NbStepIO, "NbParticleDesc": _abi.NbParticleDesc,
               "NbSoftContacts": _abi.NbSoftContacts, "NbParticleIO": _abi.NbParticleIO}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "newton_b200.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    c_vals = dict(line.split() for line in out if line.strip())
    for name, cls in structs.items():
        assert int(c_vals[name]) == C.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(c_vals[f"{name}.{fname}"]) == getattr(cls, fname).offset, f"{name}.{fname}"


def test_invalid_arguments_rejected_without_gpu(lib):
    # a NULL descriptor is rejected before any CUDA call
    assert lib.nb_collide(None, None, None, 0, None) == _abi.NB_ERR_INVALID
    assert lib.nb_xpbd_step(None, None, None, None, 0.01, 0, None) == _abi.NB_ERR_INVALID
    assert lib.nb_publish_contacts(None, None, None, None) == _abi.NB_ERR_INVALID
    assert lib.nb_ingest_contacts(None, None, None, None) == _abi.NB_ERR_INVALID
