"""Generate golden fixtures from the reference's own rigid-contact code -- TEST INFRASTRUCTURE.

The reference (Newton on NVIDIA Warp) cannot run in this image: warp-lang is not installed and
there is no network.  This script runs the reference's unmodified Python/Warp source for the path
on the CPU through the Warp-language emulation in ``warp_emulation/`` (see ``reference_loader``):

* ``CollisionPipeline(model, broad_phase="explicit").collide(state, contacts)``
  (newton/_src/sim/collide.py:483-1124: compute_shape_aabbs, BroadPhaseExplicit,
  NarrowPhase.launch_custom_write -> narrow_phase_primitive_kernel and narrow_phase_kernel_gjk_mpr
  with collide.py's write_contact), and
* ``SolverXPBD(model, iterations).step(state_in, state_out, control, contacts, dt)``
  (newton/_src/solvers/xpbd/solver_xpbd.py:259-764 with kernels.py and solvers/solver.py),

on small seeded scenes built by this package's scene generators (the same ModelBuilder semantics
the tests use), with ``deterministic=True`` (contacts sorted by the reference's key before the
solver), and writes, per scene, to ``tests/golden/<scene>.npz``:

* the body state before each of 16 substeps of collide + step and after the last, and the
  contacts (in key order) of the first and the last substep;
* per substep, the reference's own spread: the largest change of that substep's result when every
  kernel runs its threads in another order (five seeded permutations) -- its sensitivity to the
  order of its float atomic sums, which a GPU leaves unspecified;
* for scenes with joint constraints, the same for a second rollout whose wp.asin / wp.acos are the
  library's own fp32 functions (``*_library_asin``).

Every fp32 operation of the emulation rounds to float32 in source order and kernels run their
threads in index order, so the fixtures are deterministic.

    python tests/golden/make_golden.py [--reference PATH] [--scenes NAME ...]

Run it in a container that holds the reference tree; the fixtures it writes are committed and
the tests read only them.
"""

from __future__ import annotations

import argparse
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if HERE not in sys.path:
    sys.path.insert(0, HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_SUBSTEPS = 16
PERMUTATION_SEEDS = (1234, 5678, 9012, 3456, 7890)


# ----------------------------------------------------------------------------- scenes
def scenes(device="cpu"):
    """Small seeded scenes of the path (name -> (model, info)); the tests rebuild them on the GPU."""
    from newton_custom_contact_b200 import scenes as sc

    out = {}
    # C2-style uneven worlds: boxes, spheres, capsules dropped on a ground plane
    m, info = sc.scene_c2(seed=21, worlds=2, nmin=8, nmax=12, device=device)
    out["c2_small"] = (m, info)
    # the same scene advanced into contact: bodies start resting / penetrating
    out["c2_small_landed"] = (m, dict(info, advance_frames=24))
    # C1: 64 boxes in one world (box-box manifolds through MPR/GJK)
    m1, info1 = sc.scene_c1(seed=0, device=device)
    out["c1"] = (m1, info1)
    # C3-style arm: revolute joints with limits and drives among boxes
    m3, info3 = sc.scene_c3(seed=7, worlds=1, device=device)
    out["c3_arm"] = (m3, info3)
    return out


# ----------------------------------------------------------------------------- reference objects
def reference_model(ref, model):
    """A namespace with the reference Model fields the path reads, as emulated Warp arrays."""
    wp = ref.warp
    h = model.host_arrays()
    B, S, J, D, W = model.body_count, model.shape_count, model.joint_count, model.joint_dof_count, \
        model.world_count
    A = wp.array
    m = types.SimpleNamespace()
    m.device = "cpu"
    m.requires_grad = False
    m.body_count, m.shape_count, m.joint_count, m.joint_dof_count = B, S, J, D
    m.world_count = W
    m.particle_count = 0
    m.particle_grid = None
    m.spring_count = m.edge_count = m.tet_count = 0
    m.body_q = A(h["body_q"], dtype=wp.transform)
    m.body_qd = A(h["body_qd"], dtype=wp.spatial_vector)
    m.body_com = A(h["body_com"], dtype=wp.vec3)
    m.body_mass = A(h["body_mass"], dtype=wp.float32)
    m.body_inv_mass = A(h["body_inv_mass"], dtype=wp.float32)
    m.body_inertia = A(h["body_inertia"].reshape(B, 3, 3), dtype=wp.mat33)
    m.body_inv_inertia = A(h["body_inv_inertia"].reshape(B, 3, 3), dtype=wp.mat33)
    m.body_flags = A(h["body_flags"], dtype=wp.int32)
    m.body_world = A(h["body_world"], dtype=wp.int32)
    m.gravity = A(h["gravity"], dtype=wp.vec3)
    m.shape_body = A(h["shape_body"], dtype=wp.int32)
    m.shape_type = A(h["shape_type"], dtype=wp.int32)
    m.shape_transform = A(h["shape_transform"], dtype=wp.transform)
    m.shape_scale = A(h["shape_scale"], dtype=wp.vec3)
    m.shape_margin = A(h["shape_margin"], dtype=wp.float32)
    m.shape_gap = A(h["shape_gap"], dtype=wp.float32)
    m.shape_collision_radius = A(h["shape_collision_radius"], dtype=wp.float32)
    m.shape_material_mu = A(h["shape_material_mu"], dtype=wp.float32)
    m.shape_material_mu_torsional = A(h["shape_material_mu_torsional"], dtype=wp.float32)
    m.shape_material_mu_rolling = A(h["shape_material_mu_rolling"], dtype=wp.float32)
    m.shape_material_restitution = A(h["shape_material_restitution"], dtype=wp.float32)
    m.shape_world = A(h["shape_world"], dtype=wp.int32)
    m.shape_flags = A(h["shape_flags"], dtype=wp.int32)
    m.shape_collision_group = A(h["shape_collision_group"], dtype=wp.int32)
    m.shape_source_ptr = A(np.zeros(S, np.uint64), dtype=wp.uint64)
    m.shape_collision_aabb_lower = A(np.zeros((S, 3), np.float32), dtype=wp.vec3)
    m.shape_collision_aabb_upper = A(np.zeros((S, 3), np.float32), dtype=wp.vec3)
    m.shape_sdf_index = A(np.full(S, -1, np.int32), dtype=wp.int32)
    m.shape_heightfield_index = A(np.full(S, -1, np.int32), dtype=wp.int32)
    m._shape_voxel_resolution = A(np.zeros((S, 3), np.int32), dtype=wp.vec3i)
    m.texture_sdf_data = None
    m.heightfield_data = None
    m.heightfield_elevations = None
    m.mesh_edge_indices = None
    m.shape_edge_range = None
    pairs = model.host("shape_contact_pairs")
    m.shape_contact_pairs = A(np.asarray(pairs, np.int32).reshape(-1, 2), dtype=wp.vec2i)
    m.shape_contact_pair_count = int(m.shape_contact_pairs.shape[0])
    m.shape_collision_filter_pairs = set(model.shape_collision_filter_pairs or ())
    m.rigid_contact_max = 0
    m.joint_type = A(h["joint_type"], dtype=wp.int32)
    m.joint_enabled = A(h["joint_enabled"], dtype=wp.int32)
    m.joint_parent = A(h["joint_parent"], dtype=wp.int32)
    m.joint_child = A(h["joint_child"], dtype=wp.int32)
    m.joint_X_p = A(h["joint_X_p"], dtype=wp.transform)
    m.joint_X_c = A(h["joint_X_c"], dtype=wp.transform)
    m.joint_qd_start = A(h["joint_qd_start"], dtype=wp.int32)
    m.joint_dof_dim = A(h["joint_dof_dim"].reshape(J, 2), dtype=wp.int32)
    m.joint_axis = A(h["joint_axis"].reshape(D, 3), dtype=wp.vec3)
    m.joint_limit_lower = A(h["joint_limit_lower"], dtype=wp.float32)
    m.joint_limit_upper = A(h["joint_limit_upper"], dtype=wp.float32)
    m.joint_target_ke = A(h["joint_target_ke"], dtype=wp.float32)
    m.joint_target_kd = A(h["joint_target_kd"], dtype=wp.float32)
    m._joint_target_pos = h["joint_target_pos"]
    m._joint_target_vel = h["joint_target_vel"]
    m.particle_q = m.particle_qd = None
    m.soft_contact_restitution = 0.0

    def control(clone_variables=True):
        import newton._src.sim as sim

        c = sim.Control()
        c.joint_f = A(np.zeros(D, np.float32), dtype=wp.float32)
        c.joint_target_pos = A(m._joint_target_pos, dtype=wp.float32)
        c.joint_target_vel = A(m._joint_target_vel, dtype=wp.float32)
        return c

    m.control = control
    m.get_requested_contact_attributes = lambda: set()
    m.request_contact_attributes = lambda *a: None
    m._add_custom_attributes = lambda *a, **k: None
    return m


def reference_state(ref, m, body_q, body_qd):
    import newton._src.sim as sim

    wp = ref.warp
    s = sim.State()
    s.body_q = wp.array(np.asarray(body_q, np.float32), dtype=wp.transform)
    s.body_qd = wp.array(np.asarray(body_qd, np.float32), dtype=wp.spatial_vector)
    s.body_f = wp.array(np.zeros((m.body_count, 6), np.float32), dtype=wp.spatial_vector)
    return s


def contacts_sorted(ref, c):
    """Live contacts of a reference Contacts buffer, ordered by the reference sort key
    (contact_data.py:59-83) -- the order of CollisionPipeline(deterministic=True)."""
    n = int(c.rigid_contact_count.numpy()[0])
    n = min(n, c.rigid_contact_max)
    out = {
        "shape0": c.rigid_contact_shape0.numpy()[:n].copy(),
        "shape1": c.rigid_contact_shape1.numpy()[:n].copy(),
        "point0": c.rigid_contact_point0.numpy()[:n].copy(),
        "point1": c.rigid_contact_point1.numpy()[:n].copy(),
        "offset0": c.rigid_contact_offset0.numpy()[:n].copy(),
        "offset1": c.rigid_contact_offset1.numpy()[:n].copy(),
        "normal": c.rigid_contact_normal.numpy()[:n].copy(),
        "margin0": c.rigid_contact_margin0.numpy()[:n].copy(),
        "margin1": c.rigid_contact_margin1.numpy()[:n].copy(),
    }
    return out


def run_scene(ref, model, info, log=print):
    """Reference collide + XPBD step on `model` with deterministic=True (contacts sorted by key before
    the solver), N_SUBSTEPS substeps after the scene's optional advance.  Returns:

    * ``body_q_all`` / ``body_qd_all`` [N_SUBSTEPS + 1, B, .]: the state before every substep and
      after the last;
    * ``contact_<field>_s1`` / ``_s16``: the contacts the first and the last substep solve;
    * ``spread_q`` / ``spread_qd`` [N_SUBSTEPS + 1]: for substep k, the largest change of the state
      after k when that one substep, from the same state k - 1, runs every kernel's threads in
      another order (seeded permutations) -- the reference's own sensitivity to the order of its
      float atomic sums (contact and joint deltas), which a GPU leaves unspecified.
    """
    m = reference_model(ref, model)
    pipe = ref.collide.CollisionPipeline(m, broad_phase="explicit", deterministic=True, verify_buffers=False)
    solver = ref.solver_xpbd.SolverXPBD(m, iterations=info["iterations"])
    dt = np.float32(info["dt"] / info["substeps"])
    q0 = model.host("body_q").astype(np.float32)
    qd0 = model.host("body_qd").astype(np.float32)
    s_in = reference_state(ref, m, q0, qd0)
    s_out = reference_state(ref, m, q0, qd0)
    contacts = ref.sim.Contacts(pipe.rigid_contact_max, 0, device="cpu")
    control = m.control()
    t0 = time.time()

    def substep(a, b):
        a.body_f.zero_()
        pipe.collide(a, contacts)
        solver.step(a, b, control, contacts, float(dt))

    adv = int(info.get("advance_frames", 0)) * int(info["substeps"])
    for k in range(adv):
        substep(s_in, s_out)
        s_in, s_out = s_out, s_in
    qs = [s_in.body_q.numpy().copy()]
    qds = [s_in.body_qd.numpy().copy()]
    spread_q = np.zeros(N_SUBSTEPS + 1, np.float32)
    spread_qd = np.zeros(N_SUBSTEPS + 1, np.float32)
    out = {"dt": np.float32(dt), "iterations": np.int32(info["iterations"])}
    for k in range(1, N_SUBSTEPS + 1):
        substep(s_in, s_out)
        if k in (1, N_SUBSTEPS):
            for key, v in contacts_sorted(ref, contacts).items():
                out[f"contact_{key}_s{k}"] = v
        q_new, qd_new = s_out.body_q.numpy().copy(), s_out.body_qd.numpy().copy()
        for seed in PERMUTATION_SEEDS:
            rng = np.random.default_rng(seed + k)
            ref.warp.launch_order = lambda n, rng=rng: rng.permutation(n)
            a = reference_state(ref, m, qs[-1], qds[-1])
            b = reference_state(ref, m, qs[-1], qds[-1])
            try:
                substep(a, b)
            finally:
                ref.warp.launch_order = None
            spread_q[k] = max(spread_q[k], np.abs(b.body_q.numpy() - q_new).max())
            spread_qd[k] = max(spread_qd[k], np.abs(b.body_qd.numpy() - qd_new).max())
        s_in, s_out = s_out, s_in
        qs.append(q_new)
        qds.append(qd_new)
        if k % 8 == 0:
            log(f"  substep {k}/{N_SUBSTEPS} ({time.time() - t0:.0f} s)")
    out["body_q_all"] = np.stack(qs)
    out["body_qd_all"] = np.stack(qds)
    out["spread_q"] = spread_q
    out["spread_qd"] = spread_qd
    return out


class library_asin:
    """Within the block, the emulated wp.asin / wp.acos are the library's own fp32 functions (called
    from the CPU oracle, which shares them with the CUDA kernels)."""

    def __init__(self, ref):
        self.wp = ref.warp

    def __enter__(self):
        import oracle

        lib = oracle.load()
        self.saved = (self.wp.asin, self.wp.acos)
        self.wp.asin = lambda x: np.float32(lib.orc_asin(float(x)))
        self.wp.acos = lambda x: np.float32(lib.orc_acos(float(x)))

    def __exit__(self, *exc):
        self.wp.asin, self.wp.acos = self.saved


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--scenes", nargs="*", default=None)
    args = ap.parse_args()
    import reference_loader

    ref = reference_loader.load(args.reference)
    import newton._src.sim as sim

    ref.sim = sim
    all_scenes = scenes()
    names = args.scenes or list(all_scenes)
    for name in names:
        model, info = all_scenes[name]
        print(f"{name}: {model.body_count} bodies, {model.shape_count} shapes, {model.joint_count} joints")
        fx = run_scene(ref, model, info)
        if model.joint_count and np.any(model.host("joint_type") != 4):
            # the joint solve's swing/twist angles call asin/acos; the library (and the oracle) use
            # their own fp32 asin/acos, so a second rollout with those pins everything else bit for bit
            with library_asin(ref):
                alt = run_scene(ref, model, info, log=lambda *a: None)
            for k, v in alt.items():
                if k not in ("dt", "iterations"):
                    fx[k + "_library_asin"] = v
        fx["scene"] = np.array(name)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **fx)
        print(f"  wrote {path}: {len(fx['contact_shape0_s1'])} contacts at substep 1, "
              f"{len(fx[f'contact_shape0_s{N_SUBSTEPS}'])} at substep {N_SUBSTEPS}")


if __name__ == "__main__":
    main()
