"""CUDA path vs the CPU oracle on identical seeded scenes.

Both sides are compiled without fp contraction (the library's parity build)
and sum per-body deltas in float in contact / joint order, so contacts and
body states are compared for exact equality (the parity bar of 1e-5 rel /
1e-6 m is asserted as well, to report the size of any difference).
"""

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, scenes

pytestmark = pytest.mark.gpu


def _small_c2(worlds=48, seed=7):
    return scenes.scene_c2(seed=seed, worlds=worlds, nmin=8, nmax=40, device="cuda")


def _landed_c2(worlds, seed=11, frames=25, force=False):
    """A small C2 drop advanced `frames` frames through the pipeline (bodies landed: penetrating
    contacts; the first poses hold contacts inside the gap only)."""
    model, info = scenes.scene_c2(seed=seed, worlds=worlds, device="cuda")
    if force:
        model.request_contact_attributes("force")
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=4)
    contacts = pipe.contacts()
    s0, s1 = model.state(), model.state()
    dt = info["dt"] / info["substeps"]
    for _ in range(frames * info["substeps"]):
        s0.clear_forces()
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, dt)
        s0, s1 = s1, s0
    pipe.collide(s0, contacts)
    return model, pipe, solver, contacts, s0


def _published(contacts):
    n = int(contacts.rigid_contact_count.item())
    out = {k: getattr(contacts, f"rigid_contact_{k}")[:n].cpu().numpy()
           for k in ("shape0", "shape1", "point0", "point1", "offset0", "offset1", "normal", "margin0", "margin1")}
    return n, out


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def _assert_contacts_equal(model, pipe, contacts, segs, orc):
    """GPU dense contacts (world, key order) == oracle contacts, bit for bit."""
    assert np.array_equal(contacts._seg["world_count"].cpu().numpy(), segs.world_count), "per-world counts differ"
    table = orc.contacts_table(model, pipe.layout, segs)
    n, got = _published(contacts)
    assert n == table.shape[0] and n > 0
    assert np.array_equal(got["shape0"], table[:, 1].astype(np.int32))
    assert np.array_equal(got["shape1"], table[:, 2].astype(np.int32))
    for name, cols in (("point0", slice(4, 7)), ("point1", slice(7, 10)), ("normal", slice(10, 13)),
                       ("offset0", slice(13, 16)), ("offset1", slice(16, 19))):
        assert _bits_equal(got[name], table[:, cols]), name
    assert _bits_equal(got["margin0"], table[:, 19]) and _bits_equal(got["margin1"], table[:, 20])
    return table


@pytest.mark.parametrize("scene", ["c1", "c2"])
def test_collide_bit_exact(cuda, orc, scene):
    model, info = scenes.scene_c1(device="cuda") if scene == "c1" else _small_c2()
    pipe = CollisionPipeline(model)
    state = model.state()
    contacts = pipe.contacts()
    pipe.collide(state, contacts)
    torch.cuda.synchronize()
    segs = orc.collide(model, pipe.layout, model.host("body_q"))
    _assert_contacts_equal(model, pipe, contacts, segs, orc)


def test_public_contacts_sorted_keys(cuda, orc):
    model, _ = _small_c2(worlds=16)
    pipe = CollisionPipeline(model, deterministic=True)
    contacts = pipe.contacts()
    pipe.collide(model.state(), contacts)
    torch.cuda.synchronize()
    segs = orc.collide(model, pipe.layout, model.host("body_q"))
    table = _assert_contacts_equal(model, pipe, contacts, segs, orc)
    n = table.shape[0]
    keys = contacts.rigid_contact_sort_key[:n].cpu().numpy()
    wid = table[:, 0].astype(np.int64)
    for w in np.unique(wid):
        assert np.all(np.diff(keys[wid == w]) > 0), "contacts of a world are not in key order"
    expect = (table[:, 1].astype(np.int64) << 43) | (table[:, 2].astype(np.int64) << 23) | table[:, 3].astype(np.int64)
    assert np.array_equal(np.sort(keys), np.sort(expect))


def test_collide_all_group_sizes_and_nxn(cuda, orc):
    """The NxN candidate set equals the explicit list; contacts identical."""
    model, _ = _small_c2(worlds=12)
    a = CollisionPipeline(model, broad_phase="explicit")
    b = CollisionPipeline(model, broad_phase="nxn")
    ca, cb = a.contacts(), b.contacts()
    s = model.state()
    a.collide(s, ca)
    b.collide(s, cb)
    torch.cuda.synchronize()
    na, pa = _published(ca)
    nb, pb = _published(cb)
    assert na == nb
    for k in pa:
        assert np.array_equal(pa[k], pb[k]), k


def _run_loop(model, info, substeps, orc, iterations=None, group_threads=None, mode=None):
    """collide + step loop on the GPU (drop-in API) and on the oracle; returns both trajectories' end states."""
    it = iterations or info["iterations"]
    pipe = CollisionPipeline(model)
    if group_threads or mode:
        pipe.set_step_schedule(group_threads, mode=mode)
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


@pytest.mark.parametrize("substeps,group,mode", [(1, None, None), (16, None, None), (4, 32, "groups"),
                                                  (4, 32, "groups_compact"), (16, 32, "groups_compact"),
                                                  (4, 64, "groups"), (4, 64, "groups_compact"), (4, 128, "groups"),
                                                  (4, 32, "batch"), (4, 64, "batch"), (4, 128, "batch"),
                                                  (4, 256, "batch")])
def test_step_parity_c2(cuda, orc, substeps, group, mode):
    model, info = _small_c2()
    gq, gqd, q, qd = _run_loop(model, info, substeps, orc, group_threads=group, mode=mode)
    np.testing.assert_allclose(gq, q, rtol=1e-5, atol=1e-6)
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)


def test_step_without_contacts(cuda, orc):
    _check_step_without_contacts(scenes.scene_c1(device="cuda")[0], orc)


def _check_step_without_contacts(model, orc):
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
    """Contacts written into the dense arrays (custom writer): in the pipeline's own order they give the
    pipeline's step bit for bit (records follow the public order within each world); in reversed order
    the same step up to the rounding of the per-body sums, and the same bits on every call."""
    model, pipe, solver, c1, s0 = _landed_c2(worlds=8)
    out_a = model.state()
    solver.step(s0, out_a, None, c1, 1.0 / 480.0)
    n = int(c1.rigid_contact_count.item())
    names = ("shape0", "shape1", "point0", "point1", "offset0", "offset1", "normal", "margin0", "margin1")

    def ingested(order):
        c2 = pipe.contacts()
        for name in names:
            getattr(c2, f"rigid_contact_{name}")[:n] = getattr(c1, f"rigid_contact_{name}")[:n][order]
        c2.rigid_contact_count.fill_(n)
        c2.mark_dense_modified()
        out = model.state()
        solver.step(s0, out, None, c2, 1.0 / 480.0)
        torch.cuda.synchronize()
        return out

    same = ingested(torch.arange(n, device="cuda"))
    assert torch.equal(out_a.body_q, same.body_q) and torch.equal(out_a.body_qd, same.body_qd)
    rev = torch.arange(n - 1, -1, -1, device="cuda")
    out_b, out_c = ingested(rev), ingested(rev)
    torch.testing.assert_close(out_b.body_q, out_a.body_q, rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(out_b.body_qd, out_a.body_qd, rtol=1e-5, atol=1e-6 * 480.0)
    assert torch.equal(out_b.body_q, out_c.body_q) and torch.equal(out_b.body_qd, out_c.body_qd)


def test_capacity_overflow_solves_the_held_contacts(cuda, orc):
    """rigid_contact_max below the contact count: collide keeps the first `capacity` contacts in
    public order and flags the overflow; the solver records hold exactly those (min(5 x pairs,
    capacity) rows), so the step equals a step over those contacts written by hand (the reference's
    solver reads rigid_contact_count clamped to rigid_contact_max), per-contact forces included, and
    ingesting a count past the capacity takes the same contacts."""
    from newton_custom_contact_b200._abi import NB_STATUS_CONTACT_OVERFLOW

    model, full_pipe, solver, full, s0 = _landed_c2(worlds=8, force=True)
    n = int(full.rigid_contact_count.item())
    cap = n // 2 + 3
    assert 0 < cap < n
    pipe = CollisionPipeline(model, rigid_contact_max=cap)
    small = pipe.contacts()
    assert small._seg["rec"].shape[0] == cap and small._seg["impulse_scratch"].shape[0] == cap
    pipe.collide(s0, small)
    assert int(small.rigid_contact_count.item()) == n
    assert pipe.status(small) & NB_STATUS_CONTACT_OVERFLOW
    names = ("shape0", "shape1", "point0", "point1", "offset0", "offset1", "normal", "margin0", "margin1")
    for name in names:
        assert torch.equal(getattr(small, f"rigid_contact_{name}"), getattr(full, f"rigid_contact_{name}")[:cap])
    out_a = model.state()
    solver.step(s0, out_a, None, small, 1.0 / 480.0)
    solver.update_contacts(small)
    force_a = small.force.clone()

    def ingested(count):
        c = pipe.contacts()
        for name in names:
            getattr(c, f"rigid_contact_{name}").copy_(getattr(full, f"rigid_contact_{name}")[:cap])
        c.rigid_contact_count.fill_(count)
        c.mark_dense_modified()
        out = model.state()
        solver.step(s0, out, None, c, 1.0 / 480.0)
        solver.update_contacts(c)
        torch.cuda.synchronize()
        return out, c.force.clone()

    for count in (cap, n):
        out_b, force_b = ingested(count)
        assert torch.equal(out_a.body_q, out_b.body_q) and torch.equal(out_a.body_qd, out_b.body_qd), count
        assert torch.equal(force_a, force_b), count
    # the step did use the held contacts: some are penetrating and carry a force, and without
    # contacts the bodies move differently
    assert float(force_a.abs().max()) > 0
    out_free = model.state()
    solver.step(s0, out_free, None, None, 1.0 / 480.0)
    torch.cuda.synchronize()
    assert not torch.equal(out_free.body_qd, out_a.body_qd)


def test_collide_bit_exact_in_piled_state(cuda, orc):
    """Contacts after 25 frames of a 96-world drop (bodies landed and piled up,
    many box-box / box-capsule pairs near contact) equal the oracle's on the
    same poses: the MPR/GJK separation prefilter drops no contact."""
    model, info = scenes.scene_c2(seed=11, worlds=96, device="cuda")
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=info["iterations"])
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    dt = info["dt"] / info["substeps"]
    for _ in range(25 * info["substeps"]):
        s0.clear_forces()
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, dt)
        s0, s1 = s1, s0
    pipe.collide(s0, contacts)
    torch.cuda.synchronize()
    assert pipe.status(contacts) == 0
    segs = orc.collide(model, pipe.layout, s0.body_q.cpu().numpy())
    table = _assert_contacts_equal(model, pipe, contacts, segs, orc)
    assert table.shape[0] > 5000


def test_bench_scene_bit_exact(cuda, orc):
    """The benchmark scene itself (4096 uneven worlds, seed 1, 8 substeps x 8 iterations): six frames of
    collide + step free-running on the CUDA path and in the oracle end in bit-identical states, and the
    contacts of frame 6's first substep are bit-identical too."""
    model, info = scenes.scene_c2(seed=1, worlds=4096, device="cuda")
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=info["iterations"])
    params = solver.params()
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    dt = info["dt"] / info["substeps"]
    q, qd = model.host("body_q"), model.host("body_qd")
    f = np.zeros((model.body_count, 6), np.float32)
    for k in range(6 * info["substeps"]):
        s0.clear_forces()
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, dt)
        s0, s1 = s1, s0
        segs = orc.collide(model, pipe.layout, q)
        q, qd, st = orc.step(model, pipe.layout, params, q, qd, f, segs, dt)
        assert st == 0
    torch.cuda.synchronize()
    assert _bits_equal(s0.body_q.cpu().numpy(), q), "body_q after 6 frames"
    assert _bits_equal(s0.body_qd.cpu().numpy(), qd), "body_qd after 6 frames"
    pipe.collide(s0, contacts)
    torch.cuda.synchronize()
    assert pipe.status(contacts) == 0
    segs = orc.collide(model, pipe.layout, q)
    table = _assert_contacts_equal(model, pipe, contacts, segs, orc)
    assert table.shape[0] > 100000


@pytest.mark.parametrize("n", [1, 4, 5])
def test_substeps_entry_matches_host_loop(cuda, n):
    """nb_xpbd_substeps (SolverXPBD.step_substeps) against the host loop of collide + step, bit for bit,
    for odd and even substep counts (the state ping-pongs between the two buffers)."""
    model, info = _small_c2(worlds=24)
    dt = info["dt"] / info["substeps"]
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=info["iterations"])
    s0, s1 = model.state(), model.state()
    c = pipe.contacts()
    for _ in range(n):
        s0.clear_forces()
        pipe.collide(s0, c)
        solver.step(s0, s1, None, c, dt)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    ref_q, ref_qd = s0.body_q.cpu().numpy(), s0.body_qd.cpu().numpy()
    ref_count = int(c.rigid_contact_count.item())
    a, b = model.state(), model.state()
    c2 = pipe.contacts()
    a.clear_forces()
    solver.step_substeps(a, b, c2, dt, n)
    torch.cuda.synchronize()
    assert _bits_equal(b.body_q.cpu().numpy(), ref_q) and _bits_equal(b.body_qd.cpu().numpy(), ref_qd)
    assert int(c2.rigid_contact_count.item()) == ref_count
    assert pipe.status(c2) == 0


def test_contact_generation_bumped_by_collide(cuda):
    """Contacts.contact_generation advances once per collide inside the library's publish, with the
    reference's wraparound after INT32_MAX (compute_shape_aabbs, collide.py:211-218)."""
    model, _ = _small_c2(worlds=4)
    pipe = CollisionPipeline(model)
    c = pipe.contacts()
    s = model.state()
    g0 = int(c.contact_generation.item())
    for _ in range(3):
        pipe.collide(s, c)
    assert int(c.contact_generation.item()) == g0 + 3
    c.contact_generation.fill_(2147483647)
    pipe.collide(s, c)
    assert int(c.contact_generation.item()) == 0


def test_clear_forces_zeroes_body_f(cuda):
    model, _ = _small_c2(worlds=4)
    s = model.state()
    s.body_f.fill_(3.0)
    s.clear_forces()
    torch.cuda.synchronize()
    assert bool((s.body_f == 0).all().item())


@pytest.mark.parametrize("scene", ["c2", "c1", "c3", "large"])
def test_sap_broad_phase_same_contacts(cuda, scene):
    """broad_phase="sap" (per-world sort along x and sweep) finds the same candidates as testing every
    listed pair, so the published contacts are identical bit for bit, over a few substeps of motion."""
    if scene == "c2":
        model, info = _small_c2()
    elif scene == "c1":
        model, info = scenes.scene_c1(device="cuda")
    elif scene == "c3":
        model, info = scenes.scene_c3(worlds=4, device="cuda")
    else:
        # worlds of 200..300 bodies in the same 1 x 1 x 2 m column: those over the sweep's 256 shape
        # slots, and those under it with more than its 512 overlap slots, fall back to the pair test
        model, info = scenes.scene_c2(seed=9, worlds=4, nmin=200, nmax=300, device="cuda")
    dt = info["dt"] / info["substeps"]
    solver = SolverXPBD(model, iterations=info["iterations"])
    pipes = {mode: CollisionPipeline(model, broad_phase=mode) for mode in ("nxn", "sap")}
    cs = {mode: p.contacts() for mode, p in pipes.items()}
    s0, s1 = model.state(), model.state()
    for k in range(12):
        pubs = {}
        for mode, p in pipes.items():
            p.collide(s0, cs[mode])
            pubs[mode] = _published(cs[mode])
        assert pubs["nxn"][0] == pubs["sap"][0] > 0
        for f, v in pubs["nxn"][1].items():
            assert np.array_equal(np.asarray(v).view(np.uint32) if v.dtype == np.float32 else v,
                                  np.asarray(pubs["sap"][1][f]).view(np.uint32) if v.dtype == np.float32
                                  else pubs["sap"][1][f]), f"{f} at substep {k}"
        solver.step(s0, s1, None, cs["nxn"], dt)
        s0, s1 = s1, s0
