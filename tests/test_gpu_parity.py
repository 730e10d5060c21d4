"""CUDA path vs the CPU oracle on identical seeded scenes.

Both sides are compiled without fp contraction and sum per-body deltas in
the same 2^-32 fixed point, so contacts and body states are compared for
exact equality (the parity bar of 1e-5 rel / 1e-6 m is asserted as well, to
report the size of any difference).
"""

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, scenes

pytestmark = pytest.mark.gpu


def _small_c2(worlds=48, seed=7):
    return scenes.scene_c2(seed=seed, worlds=worlds, nmin=8, nmax=40, device="cuda")


def _segments_gpu(contacts):
    seg = contacts._seg
    return [seg[f"rec{k}"].cpu().numpy() for k in range(5)], seg["world_count"].cpu().numpy()


def _assert_segments_equal(model, layout, gpu_rec, gpu_wc, segs):
    assert np.array_equal(gpu_wc, segs.world_count), "per-world contact counts differ"
    cs = layout.contact_cap_start
    for w in range(model.world_count):
        n = int(segs.world_count[w])
        sl = slice(int(cs[w]), int(cs[w]) + n)
        for k in range(5):
            a = gpu_rec[k][sl].view(np.uint32)
            b = segs.rec[k][sl].view(np.uint32)
            assert np.array_equal(a, b), f"world {w} rec{k} differs"


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("scene", ["c1", "c2"])
def test_collide_bit_exact(cuda, orc, scene):
    model, info = scenes.scene_c1(device="cuda") if scene == "c1" else _small_c2()
    pipe = CollisionPipeline(model)
    state = model.state()
    contacts = pipe.contacts()
    pipe.collide(state, contacts)
    torch.cuda.synchronize()
    segs = orc.collide(model, pipe.layout, model.host("body_q"))
    rec, wc = _segments_gpu(contacts)
    assert wc.sum() > 0
    _assert_segments_equal(model, pipe.layout, rec, wc, segs)


def test_public_contacts_match_segments(cuda, orc):
    model, _ = _small_c2(worlds=16)
    pipe = CollisionPipeline(model, deterministic=True)
    contacts = pipe.contacts()
    pipe.collide(model.state(), contacts)
    torch.cuda.synchronize()
    n = int(contacts.rigid_contact_count.item())
    table = orc.contacts_table(model, pipe.layout, orc.collide(model, pipe.layout, model.host("body_q")))
    assert n == table.shape[0]
    s0 = contacts.rigid_contact_shape0[:n].cpu().numpy()
    s1 = contacts.rigid_contact_shape1[:n].cpu().numpy()
    assert np.array_equal(s0, table[:, 1].astype(np.int32))
    assert np.array_equal(s1, table[:, 2].astype(np.int32))
    assert _bits_equal(contacts.rigid_contact_point0[:n].cpu().numpy(), table[:, 4:7])
    assert _bits_equal(contacts.rigid_contact_normal[:n].cpu().numpy(), table[:, 10:13])
    keys = contacts.rigid_contact_sort_key[:n].cpu().numpy()
    # within a world the contacts are in deterministic key order
    wid = table[:, 0].astype(np.int64)
    for w in np.unique(wid):
        k = keys[wid == w]
        assert np.all(np.diff(k) > 0)
    # canonical sort of (shape0, shape1, sub) reproduces the oracle set exactly
    ref = np.lexsort((table[:, 3], table[:, 2], table[:, 1]))
    got = np.argsort(keys, kind="stable")
    assert np.array_equal(keys[got], (table[ref, 1].astype(np.int64) << 43) | (table[ref, 2].astype(np.int64) << 23)
                          | table[ref, 3].astype(np.int64))


def _run_loop(model, info, substeps, orc, iterations=None):
    """collide + step loop on the GPU (drop-in API) and on the oracle; returns both trajectories' end states."""
    it = iterations or info["iterations"]
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=it)
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    dt = info["dt"] / info["substeps"]
    for _ in range(substeps):
        s0.clear_forces()
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, dt)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy()
    f = np.zeros((model.body_count, 6), np.float32)
    p = solver.params()
    jt = model.host("joint_target_pos")
    jv = model.host("joint_target_vel")
    for _ in range(substeps):
        segs = orc.collide(model, pipe.layout, q)
        q, qd, _ = orc.step(model, pipe.layout, p, q, qd, f, segs, dt, joint_target_pos=jt, joint_target_vel=jv,
                            joint_f=np.zeros(model.joint_dof_count, np.float32))
    return s0.body_q.cpu().numpy(), s0.body_qd.cpu().numpy(), q, qd


@pytest.mark.parametrize("substeps", [1, 16])
def test_step_parity_c1(cuda, orc, substeps):
    model, info = scenes.scene_c1(device="cuda")
    gq, gqd, q, qd = _run_loop(model, info, substeps, orc)
    np.testing.assert_allclose(gq, q, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(gqd, qd, rtol=1e-5, atol=1e-6)
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)


@pytest.mark.parametrize("substeps", [1, 16])
def test_step_parity_c2(cuda, orc, substeps):
    model, info = _small_c2()
    gq, gqd, q, qd = _run_loop(model, info, substeps, orc)
    np.testing.assert_allclose(gq, q, rtol=1e-5, atol=1e-6)
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)


def test_step_without_contacts(cuda, orc):
    model, info = scenes.scene_c1(device="cuda")
    solver = SolverXPBD(model, iterations=4)
    s0, s1 = model.state(), model.state()
    solver.step(s0, s1, None, None, 1.0 / 600.0)
    torch.cuda.synchronize()
    from newton_custom_contact_b200.collide import PairLayout

    lay = PairLayout(model, model.host("shape_contact_pairs"))
    q, qd, _ = orc.step(model, lay, solver.params(), model.host("body_q"), model.host("body_qd"),
                        np.zeros((model.body_count, 6), np.float32), None, 1.0 / 600.0)
    assert _bits_equal(s1.body_q.cpu().numpy(), q)


def test_custom_contacts_ingested(cuda, orc):
    """Contacts written into the dense arrays (custom writer) give the same step as pipeline contacts."""
    model, info = _small_c2(worlds=8)
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=4)
    s0 = model.state()
    c1 = pipe.contacts()
    pipe.collide(s0, c1)
    out_a = model.state()
    solver.step(s0, out_a, None, c1, 1.0 / 480.0)
    # same contacts, written "by hand" in reversed order into a fresh buffer
    c2 = pipe.contacts()
    n = int(c1.rigid_contact_count.item())
    idx = torch.arange(n - 1, -1, -1, device="cuda")
    for name in ("shape0", "shape1", "point0", "point1", "offset0", "offset1", "normal", "margin0", "margin1"):
        getattr(c2, f"rigid_contact_{name}")[:n] = getattr(c1, f"rigid_contact_{name}")[:n][idx]
    c2.rigid_contact_count.fill_(n)
    c2.mark_dense_modified()
    out_b = model.state()
    solver.step(s0, out_b, None, c2, 1.0 / 480.0)
    torch.cuda.synchronize()
    assert torch.equal(out_a.body_q, out_b.body_q)
    assert torch.equal(out_a.body_qd, out_b.body_qd)
