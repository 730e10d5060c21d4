"""Loader for the in-tree CUDA library (C ABI in include/newton_b200.h).

Two builds of the same sources export the same ABI:

* ``libnewton_b200.so`` -- the product build (the compiler contracts a*b+c
  into fused multiply-adds); used unless another build is selected;
* ``libnewton_b200_exact.so`` -- the parity build (``--fmad=false``): every
  fp32 expression rounds in source order, exactly like the CPU oracle, so the
  two agree bit for bit.

``use_build("exact")`` / ``with build("exact"):`` select the parity build for
the calls that follow (the environment variable ``NEWTON_B200_BUILD`` sets the
initial choice).  There is no fallback: if the library or a CUDA device is
missing, every entry point raises.
"""

from __future__ import annotations

import contextlib
import ctypes as C
import os

from ._abi import (
    NB_ABI_VERSION,
    NB_ERR_CAPACITY,
    NB_ERR_CUDA,
    NB_ERR_INVALID,
    NB_ERR_UNSUPPORTED,
    NbAdjointIO,
    NbParticleDesc,
    NbParticleIO,
    NbSoftContacts,
    NbContactSeg,
    NbContactsPublic,
    NbMatchState,
    NbModelDesc,
    NbStepIO,
    NbWsNet,
    NbWsTrain,
    NbXpbdParams,
)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libnewton_b200.so"
LIB_PATH = os.path.join(_HERE, LIB_NAME)
BUILDS = {"product": LIB_PATH, "exact": os.path.join(_HERE, "libnewton_b200_exact.so")}

EXPORTS = (
    "nb_abi_version",
    "nb_last_cuda_error",
    "nb_cuda_error_string",
    "nb_default_grid",
    "nb_clear_forces",
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
    "nb_xpbd_substeps",
    "nb_soft_collide",
    "nb_particle_step",
)

_libs: dict = {}
_active = os.environ.get("NEWTON_B200_BUILD", "product")
if _active not in BUILDS:
    raise ValueError(f"NEWTON_B200_BUILD must be one of {sorted(BUILDS)}, got {_active!r}")


def use_build(name: str) -> str:
    """Select the build ("product" or "exact") that load() returns from now on; returns the previous one."""
    global _active
    if name not in BUILDS:
        raise ValueError(f"unknown build {name!r}; expected one of {sorted(BUILDS)}")
    prev, _active = _active, name
    return prev


def active_build() -> str:
    return _active


@contextlib.contextmanager
def build(name: str):
    """Run the enclosed calls on one build of the library."""
    prev = use_build(name)
    try:
        yield load()
    finally:
        use_build(prev)


class NbError(RuntimeError):
    """A libnewton_b200 entry point returned a non-zero status."""

    _names = {
        NB_ERR_INVALID: "invalid argument",
        NB_ERR_CUDA: "CUDA error",
        NB_ERR_UNSUPPORTED: "unsupported by this build",
        NB_ERR_CAPACITY: "capacity exceeded",
    }

    def __init__(self, fn: str, code: int, cuda_error: int = 0, cuda_message: str = ""):
        msg = f"{fn} failed: {self._names.get(code, 'error')} (code {code})"
        if cuda_error:
            msg += f": cudaError {cuda_error} ({cuda_message})"
        super().__init__(msg)
        self.code = code
        self.cuda_error = cuda_error


def load(path: str | None = None) -> C.CDLL:
    """Load (once per build) and type the active build of the library; raises if it is missing."""
    if path is None and _active in _libs:
        return _libs[_active]
    p = path or BUILDS[_active]
    if not os.path.exists(p):
        raise RuntimeError(
            f"{os.path.basename(p)} not found at {p}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` or `make -j -C newton_custom_contact_b200/csrc`"
        )
    lib = C.CDLL(p)
    lib.nb_abi_version.restype = C.c_int
    lib.nb_last_cuda_error.restype = C.c_int
    lib.nb_cuda_error_string.restype = C.c_char_p
    lib.nb_cuda_error_string.argtypes = [C.c_int]
    lib.nb_default_grid.restype = C.c_int32
    lib.nb_clear_forces.restype = C.c_int
    lib.nb_clear_forces.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
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
    lib.nb_xpbd_step_adjoint.restype = C.c_int
    lib.nb_xpbd_step_adjoint.argtypes = [C.POINTER(NbModelDesc), C.POINTER(NbXpbdParams), C.POINTER(NbAdjointIO),
                                         C.POINTER(NbContactSeg), C.c_float, C.c_void_p]
    lib.nb_soft_collide.restype = C.c_int
    lib.nb_soft_collide.argtypes = [C.POINTER(NbParticleDesc), C.c_void_p, C.c_void_p, C.POINTER(NbSoftContacts),
                                    C.c_void_p]
    lib.nb_particle_step.restype = C.c_int
    lib.nb_particle_step.argtypes = [C.POINTER(NbParticleDesc), C.POINTER(NbParticleIO), C.POINTER(NbSoftContacts),
                                     C.c_float, C.c_int32, C.c_float, C.c_void_p]
    v = lib.nb_abi_version()
    if v != NB_ABI_VERSION:
        raise RuntimeError(f"{LIB_NAME} ABI version {v} != {NB_ABI_VERSION}; rebuild the library")
    if path is None:
        _libs[_active] = lib
    return lib


def check(fn: str, rc: int) -> None:
    if rc != 0:
        cuda_error, message = 0, ""
        if rc == NB_ERR_CUDA and _active in _libs:
            lib = _libs[_active]
            cuda_error = int(lib.nb_last_cuda_error())
            message = (lib.nb_cuda_error_string(cuda_error) or b"").decode(errors="replace")
        raise NbError(fn, rc, cuda_error, message)


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
