"""ctypes mirrors of the structs in include/newton_b200.h.

The field order and types must match the header exactly; ``test_abi_layout``
checks the sizes against the compiled library.
"""

from __future__ import annotations

import ctypes as C
import enum

NB_ABI_VERSION = 19

NB_OK = 0
NB_ERR_INVALID = 1
NB_ERR_CUDA = 2
NB_ERR_UNSUPPORTED = 3
NB_ERR_CAPACITY = 4

NB_STATUS_CONTACT_OVERFLOW = 1 << 0
NB_STATUS_NONFINITE = 1 << 1
NB_STATUS_FIXED_OVERFLOW = 1 << 2
NB_STATUS_QUEUE_TIMEOUT = 1 << 3
NB_STATUS_WORLD_TOO_LARGE = 1 << 4

NB_WS_KEEP_ALL = 1


class GeoType(enum.IntEnum):
    """Shape types (newton/_src/geometry/types.py:46-77)."""

    NONE = 0
    PLANE = 1
    HFIELD = 2
    SPHERE = 3
    CAPSULE = 4
    ELLIPSOID = 5
    CYLINDER = 6
    BOX = 7
    MESH = 8
    CONE = 9
    CONVEX_MESH = 10


SUPPORTED_GEO = (GeoType.PLANE, GeoType.SPHERE, GeoType.CAPSULE, GeoType.BOX)


class JointType(enum.IntEnum):
    """Joint types (newton/_src/sim/enums.py:29-55)."""

    PRISMATIC = 0
    REVOLUTE = 1
    BALL = 2
    FIXED = 3
    FREE = 4
    DISTANCE = 5
    D6 = 6
    CABLE = 7


class BodyFlags(enum.IntFlag):
    """Body state flags (newton/_src/sim/enums.py:8-25)."""

    DYNAMIC = 1 << 0
    KINEMATIC = 1 << 1
    ALL = DYNAMIC | KINEMATIC


class ShapeFlags(enum.IntFlag):
    """Shape flags (newton/_src/geometry/flags.py:18-36)."""

    VISIBLE = 1 << 0
    COLLIDE_SHAPES = 1 << 1
    COLLIDE_PARTICLES = 1 << 2
    SITE = 1 << 3
    HYDROELASTIC = 1 << 4


_fp = C.c_void_p


class NbModelDesc(C.Structure):
    _fields_ = [
        ("body_count", C.c_int32),
        ("shape_count", C.c_int32),
        ("joint_count", C.c_int32),
        ("joint_dof_count", C.c_int32),
        ("world_count", C.c_int32),
        ("global_shape_count", C.c_int32),
        ("pair_count", C.c_int32),
        ("max_world_bodies", C.c_int32),
        ("max_world_shapes", C.c_int32),
        ("max_world_joints", C.c_int32),
        ("max_world_pairs", C.c_int32),
        ("all_joints_free", C.c_int32),
        ("broad_phase", C.c_int32),
        ("pad_bp", C.c_int32),
        ("contact_capacity", C.c_int64),
        ("body_com", _fp),
        ("body_mass", _fp),
        ("body_inv_mass", _fp),
        ("body_inertia", _fp),
        ("body_inv_inertia", _fp),
        ("body_flags", _fp),
        ("body_world", _fp),
        ("gravity", _fp),
        ("shape_body", _fp),
        ("shape_type", _fp),
        ("shape_transform", _fp),
        ("shape_scale", _fp),
        ("shape_margin", _fp),
        ("shape_gap", _fp),
        ("shape_radius", _fp),
        ("shape_mu", _fp),
        ("shape_mu_torsional", _fp),
        ("shape_mu_rolling", _fp),
        ("shape_restitution", _fp),
        ("joint_type", _fp),
        ("joint_enabled", _fp),
        ("joint_parent", _fp),
        ("joint_child", _fp),
        ("joint_X_p", _fp),
        ("joint_X_c", _fp),
        ("joint_qd_start", _fp),
        ("joint_dof_dim", _fp),
        ("joint_axis", _fp),
        ("joint_limit_lower", _fp),
        ("joint_limit_upper", _fp),
        ("joint_target_ke", _fp),
        ("joint_target_kd", _fp),
        ("world_body_start", _fp),
        ("world_shape_start", _fp),
        ("world_joint_start", _fp),
        ("global_shapes", _fp),
        ("world_pair_start", _fp),
        ("pair_shapes", _fp),
        ("world_order", _fp),
        ("batch_count", C.c_int32),
        ("worlds_per_group", C.c_int32),
        ("group_threads", C.c_int32),
        ("cta_threads", C.c_int32),
        ("smem_floats_per_batch", C.c_int32),
        ("step_mode", C.c_int32),
        ("batch_world", _fp),
        ("batch_slab", _fp),
        ("body_pack", _fp),
        ("pair_table", _fp),
        ("world_table_start", _fp),
    ]


class NbContactSeg(C.Structure):
    _fields_ = [
        ("slots", _fp),
        ("rec", _fp),
        ("world_base", _fp),
        ("cand", _fp),
        ("cand_count", _fp),
        ("counts", _fp),
        ("queue", _fp),
        ("world_count", _fp),
        ("geom", _fp),
        ("work_counter", _fp),
        ("status", _fp),
        ("rec_index", _fp),
    ]


class NbMatchState(C.Structure):
    _fields_ = [
        ("capacity", C.c_int32),
        ("sticky", C.c_int32),
        ("pos_threshold_sq", C.c_float),
        ("normal_dot_threshold", C.c_float),
        ("prev_count", _fp),
        ("prev_world_offset", _fp),
        ("prev_keys", _fp),
        ("prev_mid", _fp),
        ("prev_normal", _fp),
        ("prev_claim", _fp),
        ("prev_was_matched", _fp),
        ("prev_point0", _fp),
        ("prev_point1", _fp),
        ("prev_offset0", _fp),
        ("prev_offset1", _fp),
        ("prev_normal_sticky", _fp),
        ("match_index", _fp),
        ("new_indices", _fp),
        ("new_count", _fp),
        ("broken_indices", _fp),
        ("broken_count", _fp),
    ]


class NbContactsPublic(C.Structure):
    _fields_ = [
        ("capacity", C.c_int32),
        ("pad0", C.c_int32),
        ("count", _fp),
        ("shape0", _fp),
        ("shape1", _fp),
        ("point0", _fp),
        ("point1", _fp),
        ("offset0", _fp),
        ("offset1", _fp),
        ("normal", _fp),
        ("margin0", _fp),
        ("margin1", _fp),
        ("sort_key", _fp),
        ("world_offset", _fp),
        ("generation", _fp),
    ]


class NbXpbdParams(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("rigid_contact_con_weighting", C.c_int32),
        ("enable_restitution", C.c_int32),
        ("pad0", C.c_int32),
        ("joint_linear_relaxation", C.c_float),
        ("joint_angular_relaxation", C.c_float),
        ("joint_linear_compliance", C.c_float),
        ("joint_angular_compliance", C.c_float),
        ("rigid_contact_relaxation", C.c_float),
        ("angular_damping", C.c_float),
    ]


class NbStepIO(C.Structure):
    _fields_ = [
        ("body_q_in", _fp),
        ("body_qd_in", _fp),
        ("body_f_in", _fp),
        ("body_q_out", _fp),
        ("body_qd_out", _fp),
        ("joint_target_pos", _fp),
        ("joint_target_vel", _fp),
        ("joint_f", _fp),
        ("contact_impulse", _fp),
        ("impulse_scratch", _fp),
        ("contact_impulse_capacity", C.c_int32),
        ("pad0", C.c_int32),
        ("body_parent_f", _fp),
        ("joint_impulse", _fp),
        ("ws_lambda", _fp),
        ("ws_capacity", C.c_int32),
        ("ws_flags", C.c_int32),
        ("ws_fallback", _fp),
    ]


class NbParticleDesc(C.Structure):
    _fields_ = [
        ("particle_count", C.c_int32),
        ("spring_count", C.c_int32),
        ("shape_count", C.c_int32),
        ("world_count", C.c_int32),
        ("particle_max_velocity", C.c_float),
        ("particle_max_radius", C.c_float),
        ("particle_mu", C.c_float),
        ("particle_cohesion", C.c_float),
        ("particle_adhesion", C.c_float),
        ("soft_contact_mu", C.c_float),
    ] + [(k, _fp) for k in ("particle_inv_mass", "particle_radius", "particle_flags", "particle_world", "gravity",
                            "spring_indices", "spring_rest_length", "spring_stiffness", "spring_damping",
                            "particle_spring_start", "particle_spring_list", "shape_body", "shape_type",
                            "shape_transform", "shape_scale", "shape_world", "shape_flags", "shape_mu")] + [
        ("edge_count", C.c_int32),
        ("soft_contact_restitution", C.c_float),
    ] + [(k, _fp) for k in ("edge_indices", "edge_rest_angle", "edge_bending_properties", "particle_edge_start",
                            "particle_edge_list")] + [
        ("tet_count", C.c_int32),
        ("soft_body_relaxation", C.c_float),
    ] + [(k, _fp) for k in ("tet_indices", "tet_poses", "particle_tet_start", "particle_tet_list")]


class NbSoftContacts(C.Structure):
    _fields_ = [(k, _fp) for k in ("count", "particle", "shape", "body_pos", "body_vel", "normal")] + [
        ("max", C.c_int32),
        ("margin", C.c_float),
        ("particle_start", _fp),
    ]


class NbParticleIO(C.Structure):
    _fields_ = [(k, _fp) for k in ("particle_q", "particle_qd", "particle_f", "particle_q_out", "particle_qd_out",
                                   "delta", "grid_head", "grid_next")] + [
        ("grid_size", C.c_int32),
        ("enable_restitution", C.c_int32),
        ("status", _fp),
    ]


NB_PARTICLE_ACTIVE = 1
NB_STATUS_PARTICLE_BODY_CONTACT = 1 << 7
NB_STATUS_NEIGHBOR_OVERFLOW = 1 << 8
NB_PARTICLE_MAX_NEIGHBORS = 32


class NbWsNet(C.Structure):
    _fields_ = [(k, _fp) for k in ("w1", "b1", "w2", "b2", "w3", "b3", "in_mean", "in_inv_std", "out_scale")]


class NbAdjointIO(C.Structure):
    _fields_ = [
        ("body_q_in", _fp),
        ("body_qd_in", _fp),
        ("body_f_in", _fp),
        ("grad_q_out", _fp),
        ("grad_qd_out", _fp),
        ("grad_q_in", _fp),
        ("grad_qd_in", _fp),
        ("grad_f_in", _fp),
        ("body_q_out", _fp),
        ("body_qd_out", _fp),
        ("tape_state", _fp),
        ("tape_delta", _fp),
        ("tape_weight", _fp),
        ("grad_acc", _fp),
        ("delta_acc", _fp),
        ("count_acc", _fp),
        ("active", _fp),
        ("active_count", _fp),
        ("active_capacity", C.c_int32),
        ("pad0", C.c_int32),
        ("status", _fp),
        ("grad_shape_mu", _fp),
        ("branch_contact", _fp),
        ("branch_body", _fp),
        ("branch_mode", C.c_int32),
        ("forward_only", C.c_int32),
    ]


class NbWsTrain(C.Structure):
    _fields_ = [("rows", C.c_int32), ("pad0", C.c_int32)] + [
        (k, _fp) for k in ("x", "t", "in_mean", "in_inv_std", "out_scale", "w1", "b1", "w2", "b2", "w3", "b3",
                           "g_w1", "g_b1", "g_w2", "g_b2", "g_w3", "g_b3", "xn", "z1", "h1", "z2", "h2", "y", "dy",
                           "dh", "dh2", "scratch_wq", "loss", "status")]


def ptr(a) -> int | None:
    """Raw address of a numpy array or torch tensor (None for None / empty)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if a.numel() == 0:
            return None
        return int(a.data_ptr())
    if a.size == 0:
        return None
    return int(a.ctypes.data)
