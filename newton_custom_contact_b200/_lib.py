"""Loader for the in-tree CUDA library libnewton_b200.so (C ABI in include/newton_b200.h).

There is no fallback: if the library or a CUDA device is missing, every entry
point raises.
"""

from __future__ import annotations

import ctypes as C
import os

from ._abi import (
    NB_ABI_VERSION,
    NB_ERR_CAPACITY,
    NB_ERR_CUDA,
    NB_ERR_INVALID,
    NB_ERR_UNSUPPORTED,
    NbAdjointIO,
    NbContactSeg,
    NbContactsPublic,
    NbMatchState,
    NbModelDesc,
    NbStepIO,
    NbWsNet,
    NbWsTrain,
    NbXpbdParams,
)

LIB_NAME = "libnewton_b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

EXPORTS = (
    "nb_abi_version",
    "nb_default_grid",
    "nb_collide",
    "nb_publish_contacts",
    "nb_xpbd_step",
    "nb_ingest_contacts",
    "nb_publish_contacts_static",
    "nb_contact_forces",
    "nb_match_contacts",
    "nb_ws_features",
    "nb_ws_targets",
    "nb_ws_infer",
    "nb_ws_grads",
    "nb_ws_adam",
    "nb_xpbd_step_adjoint",
    "nb_step_scratch_size",
    "nb_xpbd_substeps",
)

_lib = None


class NbError(RuntimeError):
    """A libnewton_b200 entry point returned a non-zero status."""

    _names = {
        NB_ERR_INVALID: "invalid argument",
        NB_ERR_CUDA: "CUDA error",
        NB_ERR_UNSUPPORTED: "unsupported by this build",
        NB_ERR_CAPACITY: "capacity exceeded",
    }

    def __init__(self, fn: str, code: int):
        super().__init__(f"{fn} failed: {self._names.get(code, 'error')} (code {code})")
        self.code = code


def load(path: str | None = None) -> C.CDLL:
    """Load (once) and type the library; raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{LIB_NAME} not found at {p}; build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `make -C newton_custom_contact_b200/csrc`"
        )
    lib = C.CDLL(p)
    lib.nb_abi_version.restype = C.c_int
    lib.nb_default_grid.restype = C.c_int32
    lib.nb_collide.restype = C.c_int
    lib.nb_collide.argtypes = [C.POINTER(NbModelDesc), C.c_void_p, C.POINTER(NbContactSeg), C.c_int32, C.c_void_p]
    lib.nb_publish_contacts.restype = C.c_int
    lib.nb_publish_contacts.argtypes = [C.POINTER(NbModelDesc), C.POINTER(NbContactSeg), C.POINTER(NbContactsPublic),
                                        C.c_void_p]
    lib.nb_xpbd_step.restype = C.c_int
    lib.nb_xpbd_step.argtypes = [C.POINTER(NbModelDesc), C.POINTER(NbXpbdParams), C.POINTER(NbStepIO),
                                 C.POINTER(NbContactSeg), C.c_float, C.c_int32, C.c_void_p]
    lib.nb_ingest_contacts.restype = C.c_int
    lib.nb_ingest_contacts.argtypes = [C.POINTER(NbModelDesc), C.POINTER(NbContactsPublic), C.POINTER(NbContactSeg),
                                       C.c_void_p]
    lib.nb_match_contacts.restype = C.c_int
    lib.nb_match_contacts.argtypes = [C.POINTER(NbModelDesc), C.c_void_p, C.POINTER(NbContactsPublic),
                                      C.POINTER(NbContactSeg), C.POINTER(NbMatchState), C.c_void_p]
    lib.nb_contact_forces.restype = C.c_int
    lib.nb_contact_forces.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_float, C.c_void_p, C.c_void_p]
    lib.nb_publish_contacts_static.restype = C.c_int
    lib.nb_publish_contacts_static.argtypes = [C.POINTER(NbModelDesc), C.POINTER(NbContactSeg),
                                               C.POINTER(NbContactsPublic), C.c_void_p]
    lib.nb_ws_features.restype = C.c_int
    lib.nb_ws_features.argtypes = [C.POINTER(NbModelDesc), C.c_void_p, C.c_void_p, C.POINTER(NbContactsPublic),
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p]
    lib.nb_ws_targets.restype = C.c_int
    lib.nb_ws_targets.argtypes = [C.POINTER(NbContactsPublic), C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    lib.nb_ws_infer.restype = C.c_int
    lib.nb_ws_infer.argtypes = [C.POINTER(NbWsNet), C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                C.c_void_p]
    lib.nb_ws_grads.restype = C.c_int
    lib.nb_ws_grads.argtypes = [C.POINTER(NbWsTrain), C.c_void_p]
    lib.nb_ws_adam.restype = C.c_int
    lib.nb_ws_adam.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float,
                               C.c_float, C.c_float, C.c_float, C.c_int32, C.c_void_p]
    lib.nb_xpbd_substeps.restype = C.c_int
    lib.nb_xpbd_substeps.argtypes = [C.POINTER(NbModelDesc), C.POINTER(NbXpbdParams), C.POINTER(NbStepIO),
                                     C.POINTER(NbContactSeg), C.POINTER(NbContactsPublic), C.c_float, C.c_int32,
                                     C.c_int32, C.c_void_p]
    lib.nb_step_scratch_size.restype = C.c_int64
    lib.nb_step_scratch_size.argtypes = [C.POINTER(NbModelDesc)]
    lib.nb_xpbd_step_adjoint.restype = C.c_int
    lib.nb_xpbd_step_adjoint.argtypes = [C.POINTER(NbModelDesc), C.POINTER(NbXpbdParams), C.POINTER(NbAdjointIO),
                                         C.POINTER(NbContactSeg), C.c_float, C.c_void_p]
    v = lib.nb_abi_version()
    if v != NB_ABI_VERSION:
        raise RuntimeError(f"{LIB_NAME} ABI version {v} != {NB_ABI_VERSION}; rebuild the library")
    if path is None:
        _lib = lib
    return lib


def check(fn: str, rc: int) -> None:
    if rc != 0:
        raise NbError(fn, rc)


def require_cuda(device) -> None:
    import torch

    if torch.device(device).type != "cuda":
        raise RuntimeError(
            "the rigid-contact XPBD kernels run on CUDA devices only; create the model with device='cuda'"
        )
    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device is available")


def stream_handle(device=None) -> int:
    import torch

    return int(torch.cuda.current_stream(device).cuda_stream)
