"""nb_publish_contacts_static (allocation-free publish) against nb_publish_contacts.

Both entry points are called through the C ABI on the same collision
segments; the static one gets no world-offset buffer.  Outputs are index and
copied-float data, so the tolerance is exact equality (bit patterns for
floats).  Two calls in a row check that nothing from the first call leaks
into the second.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, _lib, scenes
from newton_custom_contact_b200._abi import NB_ERR_CAPACITY, NbModelDesc, ptr

pytestmark = pytest.mark.gpu

MAX_WORLDS = 65536  # NB_PUBLISH_STATIC_MAX_WORLDS
_FLOAT = ("point0", "point1", "offset0", "offset1", "normal", "margin0", "margin1")
_INT = ("shape0", "shape1", "sort_key")


def _snapshot(pipe, c):
    torch.cuda.synchronize()
    n = int(c.rigid_contact_count.item())
    out = {"count": n}
    for k in _FLOAT + _INT:
        out[k] = getattr(c, f"rigid_contact_{k}")[:n].cpu().numpy().copy()
    W = pipe.model.world_count
    out["world_count"] = c._seg["world_count"][:W].cpu().numpy().copy()
    out["world_base"] = c._seg["world_base"][:W].cpu().numpy().copy()
    out["rec"] = c._seg["rec"][:n].cpu().numpy().view(np.uint32).copy()
    return out


def _poison(c):
    for k in _FLOAT:
        getattr(c, f"rigid_contact_{k}").fill_(float("nan"))
    for k in _INT:
        getattr(c, f"rigid_contact_{k}").fill_(-7)
    c.rigid_contact_count.fill_(-1)
    c._seg["rec"].fill_(float("nan"))
    c._seg["world_base"].fill_(-1)


def test_static_publish_matches_publish(cuda):
    model, _ = scenes.scene_c2(seed=5, worlds=48, nmin=8, nmax=40, device="cuda")
    pipe = CollisionPipeline(model)
    state = model.state()
    ref = pipe.contacts()
    pipe.collide(state, ref)  # nb_collide + nb_publish_contacts
    want = _snapshot(pipe, ref)
    assert want["count"] > 0

    lib = _lib.load()
    desc = pipe.desc()
    stream = C.c_void_p(_lib.stream_handle(model.device))
    got_c = pipe.contacts()
    seg = pipe.seg_struct(got_c)
    sentinel = torch.full_like(got_c._world_offset, -5)
    for call in range(2):
        _poison(got_c)
        assert lib.nb_collide(C.byref(desc), C.c_void_p(ptr(state.body_q)), C.byref(seg), 0, stream) == 0
        pub = pipe.public_struct(got_c)
        # the static entry point needs no scan buffer: the first call passes none, the second a
        # sentinel buffer that must come back untouched
        pub.world_offset = None if call == 0 else ptr(sentinel)
        assert lib.nb_publish_contacts_static(C.byref(desc), C.byref(seg), C.byref(pub), stream) == 0
        got = _snapshot(pipe, got_c)
        assert bool((sentinel == -5).all().item()), f"call {call}: caller's world_offset was written"
        assert got["count"] == want["count"], f"call {call}"
        for k in _INT + ("world_count", "world_base", "rec"):
            assert np.array_equal(got[k], want[k]), f"call {call}: {k}"
        for k in _FLOAT:
            assert np.array_equal(got[k].view(np.uint32), want[k].view(np.uint32)), f"call {call}: {k}"


def test_static_publish_rejects_too_many_worlds(cuda):
    model, _ = scenes.scene_c2(seed=5, worlds=4, nmin=8, nmax=12, device="cuda")
    pipe = CollisionPipeline(model)
    c = pipe.contacts()
    lib = _lib.load()
    big = NbModelDesc.from_buffer_copy(pipe.desc())
    big.world_count = MAX_WORLDS + 1
    seg = pipe.seg_struct(c)
    pub = pipe.public_struct(c)
    rc = lib.nb_publish_contacts_static(C.byref(big), C.byref(seg), C.byref(pub),
                                        C.c_void_p(_lib.stream_handle(model.device)))
    assert rc == NB_ERR_CAPACITY
