"""The particle path on the GPU (nb_soft_collide + nb_particle_step through CollisionPipeline and
SolverXPBD) against the numpy oracle (oracle/oracle_particles.py).

Scene: a spring cloth and loose particles dropped on a ground plane, a box, a sphere and a capsule
(scenes.scene_particles), dt 1/240, 8 iterations.  The parity build agrees with the oracle bit for bit
at every substep (soft contacts, positions, velocities); the product build (FMA contraction) agrees
within 1e-5 relative / 1e-6 m after one substep.
"""

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, particles, scenes
from oracle import oracle_particles as op

pytestmark = pytest.mark.gpu

DT = 1.0 / 240.0
ITERS = 8


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _gpu_run(model, substeps, q0=None, qd0=None, record=None, restitution=False):
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=ITERS, soft_contact_relaxation=0.9, enable_restitution=restitution)
    s0, s1 = model.state(), model.state()
    if q0 is not None:
        s0.particle_q.copy_(torch.from_numpy(q0))
        s0.particle_qd.copy_(torch.from_numpy(qd0))
    contacts = pipe.contacts()
    for k in range(substeps):
        pipe.collide(s0, contacts)
        if record is not None:
            n = int(contacts.soft_contact_count.item())
            m = min(n, contacts.soft_contact_max)
            record.append((n, contacts.soft_contact_particle[:m].cpu().numpy(),
                           contacts.soft_contact_shape[:m].cpu().numpy(),
                           contacts.soft_contact_body_pos[:m].cpu().numpy(),
                           contacts.soft_contact_body_vel[:m].cpu().numpy(),
                           contacts.soft_contact_normal[:m].cpu().numpy(),
                           s0.particle_q.cpu().numpy(), s0.particle_qd.cpu().numpy()))
        solver.step(s0, s1, None, contacts, DT)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    return s0, solver, pipe


def _oracle_substep(model, q, qd, margin, smax, restitution=False):
    soft = op.soft_collide(model._host, q, None, margin, smax)
    q, qd = op.step(model._host, particles.params(model), q, qd, None, soft, DT, ITERS, 0.9, restitution)
    return soft, q, qd


def test_particle_trajectory_bit_exact(cuda):
    model, _ = scenes.scene_particles(seed=7, device=cuda)
    record = []
    steps = 48
    s, solver, pipe = _gpu_run(model, steps, record=record)
    q, qd = model.host("particle_q").copy(), model.host("particle_qd").copy()
    smax = pipe.soft_contact_max
    total_contacts = 0
    for k in range(steps):
        n, cp, cs, bpos, bvel, cn, gq, gqd = record[k]
        assert np.array_equal(_bits(gq), _bits(q)), f"positions differ before substep {k}"
        assert np.array_equal(_bits(gqd), _bits(qd)), f"velocities differ before substep {k}"
        soft, q, qd = _oracle_substep(model, q, qd, pipe.soft_contact_margin, smax)
        assert n == soft[0], f"soft contact count differs at substep {k}: {n} vs {soft[0]}"
        assert np.array_equal(cp, soft[1]) and np.array_equal(cs, soft[2]), f"contact pairs differ at {k}"
        for name, g, o in (("body_pos", bpos, soft[3]), ("body_vel", bvel, soft[4]), ("normal", cn, soft[5])):
            assert np.array_equal(_bits(g), _bits(o)), f"soft_contact_{name} differs at substep {k}"
        total_contacts += n
    assert np.array_equal(_bits(s.particle_q.cpu().numpy()), _bits(q))
    assert np.array_equal(_bits(s.particle_qd.cpu().numpy()), _bits(qd))
    # the drop reached the shapes, every shape type was touched and nothing overflowed
    assert total_contacts > 1000
    shapes_hit = set(np.concatenate([r[2] for r in record]).tolist())
    assert shapes_hit == {0, 1, 2, 3}, shapes_hit
    assert solver._particles.status() == 0


def _prerolled(cuda, steps=40):
    model, _ = scenes.scene_particles(seed=9, device=cuda)
    s, _, _ = _gpu_run(model, steps)
    return model, s.particle_q.cpu().numpy(), s.particle_qd.cpu().numpy()


def test_particle_substep_exact_after_contact(cuda):
    """From a landed state: 1 and 16 substeps, bit for bit."""
    model, q0, qd0 = _prerolled(cuda)
    for n in (1, 16):
        s, _, pipe = _gpu_run(model, n, q0, qd0)
        q, qd = q0.copy(), qd0.copy()
        for _ in range(n):
            _, q, qd = _oracle_substep(model, q, qd, pipe.soft_contact_margin, pipe.soft_contact_max)
        assert np.array_equal(_bits(s.particle_q.cpu().numpy()), _bits(q)), n
        assert np.array_equal(_bits(s.particle_qd.cpu().numpy()), _bits(qd)), n


@pytest.mark.product_build
def test_particle_substep_product_build_tolerance(cuda):
    model, q0, qd0 = _prerolled(cuda)
    s, _, pipe = _gpu_run(model, 1, q0, qd0)
    _, q, qd = _oracle_substep(model, q0.copy(), qd0.copy(), pipe.soft_contact_margin, pipe.soft_contact_max)
    np.testing.assert_allclose(s.particle_q.cpu().numpy(), q, rtol=1e-5, atol=1e-6)
    # velocity = position / dt: the position bar over dt
    np.testing.assert_allclose(s.particle_qd.cpu().numpy(), qd, rtol=1e-5, atol=1e-6 / DT)


@pytest.mark.product_build
def test_particle_step_deterministic(cuda):
    model, _ = scenes.scene_particles(seed=11, device=cuda)
    a, _, _ = _gpu_run(model, 40)
    b, _, _ = _gpu_run(model, 40)
    assert torch.equal(a.particle_q, b.particle_q) and torch.equal(a.particle_qd, b.particle_qd)


def test_particles_beside_rigid_bodies(cuda):
    """A free box body (not colliding with particles) falls while the particles run: both halves of the
    substep in one solver call, the particles bit for bit."""
    model, _ = scenes.scene_particles(seed=3, cloth=6, loose=40, device=cuda, body_shapes=True)
    s, _, pipe = _gpu_run(model, 24)
    q, qd = model.host("particle_q").copy(), model.host("particle_qd").copy()
    for _ in range(24):
        _, q, qd = _oracle_substep(model, q, qd, pipe.soft_contact_margin, pipe.soft_contact_max)
    assert np.array_equal(_bits(s.particle_q.cpu().numpy()), _bits(q))
    z0 = float(model.body_q[0, 2])
    assert float(s.body_q[0, 2]) < z0 - 0.01  # the body fell


def test_large_particle_drop_stays_above_the_ground(cuda):
    """5.6k particles dropped on the ground and the static shapes: finite, no deep penetration, no overflow."""
    model, _ = scenes.scene_particles(seed=5, cloth=40, loose=4000, device=cuda)
    s, solver, pipe = _gpu_run(model, 120)
    q = s.particle_q.cpu().numpy()
    r = model.host("particle_radius")
    assert np.isfinite(q).all()
    active = (model.host("particle_flags") & 1) != 0
    assert float((q[active, 2] - r[active]).min()) > -1e-2
    assert solver._particles.status() == 0


def test_particle_restitution_bit_exact(cuda):
    """enable_restitution with soft_contact_restitution 0.6: apply_particle_shape_restitution after the
    iterations, bit for bit over 24 substeps from a landing state."""
    model, q0, qd0 = _prerolled(cuda, steps=30)
    model.soft_contact_restitution = 0.6
    s, solver, pipe = _gpu_run(model, 24, q0, qd0, restitution=True)
    q, qd = q0.copy(), qd0.copy()
    for _ in range(24):
        _, q, qd = _oracle_substep(model, q, qd, pipe.soft_contact_margin, pipe.soft_contact_max, True)
    assert np.array_equal(_bits(s.particle_q.cpu().numpy()), _bits(q))
    assert np.array_equal(_bits(s.particle_qd.cpu().numpy()), _bits(qd))
    # restitution changed the trajectory
    s2, _, _ = _gpu_run(model, 24, q0, qd0, restitution=False)
    assert not torch.equal(s.particle_qd, s2.particle_qd)


def _soft_block(cuda):
    """A 3 x 3 x 3 lattice of particles cut into 5 tetrahedra per cube, dropped tilted onto the ground."""
    from newton_custom_contact_b200 import ModelBuilder

    b = ModelBuilder()
    b.add_ground_plane()
    n, h = 3, 0.05
    idx = {}
    for i in range(n):
        for j in range(n):
            for k in range(n):
                p = (i * h + 0.3 * k * h, j * h, 0.08 + k * h + 0.2 * i * h)
                idx[i, j, k] = b.add_particle(p, (0.0, 0.0, -0.5), 0.02, radius=0.01)
    for i in range(n - 1):
        for j in range(n - 1):
            for k in range(n - 1):
                c = [idx[i + (v & 1), j + ((v >> 1) & 1), k + ((v >> 2) & 1)] for v in range(8)]
                for t in ((0, 1, 2, 4), (1, 3, 2, 7), (1, 4, 5, 7), (2, 7, 6, 4), (1, 2, 4, 7)):
                    a, bb, cc, d = (c[x] for x in t)
                    if b.add_tetrahedron(a, bb, cc, d, 1e3, 1e3) <= 0:
                        b.add_tetrahedron(a, cc, bb, d, 1e3, 1e3)
    return b.finalize(device=cuda)


def test_tetrahedral_block_bit_exact(cuda):
    model = _soft_block(cuda)
    assert model.tet_count == 40
    s, solver, pipe = _gpu_run(model, 48)
    q, qd = model.host("particle_q").copy(), model.host("particle_qd").copy()
    for _ in range(48):
        soft = op.soft_collide(model._host, q, None, pipe.soft_contact_margin, pipe.soft_contact_max)
        q, qd = op.step(model._host, particles.params(model), q, qd, None, soft, DT, ITERS, 0.9,
                        soft_body_relaxation=solver.soft_body_relaxation)
    assert np.array_equal(_bits(s.particle_q.cpu().numpy()), _bits(q))
    assert np.array_equal(_bits(s.particle_qd.cpu().numpy()), _bits(qd))
    assert float(q[:, 2].min()) < 0.02  # it reached the ground
