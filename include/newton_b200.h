/*
 * newton_b200.h -- C ABI of the B200-native rigid-contact XPBD step.
 *
 * The library replaces the hot path of Newton's rigid-body pipeline:
 *   Model.collide(state, contacts)              newton/_src/sim/model.py:996-1022
 *     -> CollisionPipeline.collide               newton/_src/sim/collide.py:902-1124
 *   SolverXPBD.step(s_in, s_out, ctl, c, dt)    newton/_src/solvers/xpbd/solver_xpbd.py:259-764
 *
 * Every pointer inside the descriptor structs is a DEVICE pointer (CUDA global
 * memory on the current device).  The structs themselves live in host memory
 * and are read by the entry points before launching; nothing is retained
 * between calls.  All launches go to the stream passed in (cudaStream_t given
 * as void* so the header needs no CUDA include); no entry point synchronises
 * the device, so every call can be captured into a CUDA graph.
 *
 * Return value of every entry point: 0 on success, a positive NB_ERR_* code
 * otherwise (launch errors are reported as NB_ERR_CUDA).  Device-side
 * conditions (contact overflow, non-finite state) are written as bits into
 * the status word `status` (NB_STATUS_*), read back by the caller when it
 * chooses to synchronise.
 *
 * Layouts (fp32 unless noted, "world" = independent scene, bodies / shapes /
 * joints of a world are contiguous index ranges):
 *   transform  7 floats  (px, py, pz, qx, qy, qz, qw)  -- wp.transform
 *   twist      6 floats  (vx, vy, vz, wx, wy, wz)      -- wp.spatial_vector
 *   mat33      9 floats  row-major
 * Contacts live in per-candidate slots: each candidate pair (a world's pair
 * that passed the AABB test) owns 5 contact slots of 5 float4 (80 bytes):
 *   f4[0] = (point0.xyz, margin0)        point0 in body frame of shape0's body
 *   f4[1] = (point1.xyz, margin1)
 *   f4[2] = (normal.xyz, bits(shape0))   normal points from shape0 to shape1
 *   f4[3] = (offset0.xyz, bits(shape1))
 *   f4[4] = (offset1.xyz, bits(tag))     tag = (body_a_local+1) | (body_b_local+1)<<12
 *                                        | sort_sub_key<<24 (local = index within the
 *                                        world's body range, -1 for static shapes)
 * Candidate c of world w is one of [world_pair_start[w], world_pair_start[w] +
 * cand_count[w]), ordered by the deterministic key (shape0, shape1) of
 * newton/_src/geometry/contact_data.py:59-83; its counts[c] contacts are in
 * sort_sub_key order, so walking candidates then slots gives key order.
 * The solver reads dense records (NbContactSeg.rec) with the same fields,
 * regrouped so a penetration test reads the first 48 bytes:
 *   f4[0] = (point0.xyz, margin0)   f4[1] = (point1.xyz, margin1)
 *   f4[2] = (normal.xyz, bits(tag)) f4[3] = (offset0.xyz, bits(shape0))
 *   f4[4] = (offset1.xyz, bits(shape1))
 */
#ifndef NEWTON_B200_H
#define NEWTON_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NB_ABI_VERSION 19

enum {
    NB_OK = 0,
    NB_ERR_INVALID = 1,     /* bad argument / descriptor */
    NB_ERR_CUDA = 2,        /* a CUDA call failed */
    NB_ERR_UNSUPPORTED = 3, /* model feature not supported by this build */
    NB_ERR_CAPACITY = 4     /* a fixed capacity is too small */
};

enum {
    NB_STATUS_CONTACT_OVERFLOW = 1u << 0, /* public contact buffer too small   */
    NB_STATUS_NONFINITE = 1u << 1,        /* NaN/Inf body state after a step   */
    NB_STATUS_FIXED_OVERFLOW = 1u << 2,   /* reserved (no longer produced)     */
    NB_STATUS_QUEUE_TIMEOUT = 1u << 3,    /* work-queue wait hit its bound     */
    NB_STATUS_WORLD_TOO_LARGE = 1u << 4,  /* world exceeds shared staging      */
    NB_STATUS_ADJOINT_UNSUPPORTED = 1u << 5, /* adjoint skipped a world with an enabled non-free joint */
    NB_STATUS_MODE_UNSUPPORTED = 1u << 6  /* reserved (no longer produced)     */
};

/* Geometry types (newton/_src/geometry/types.py:46-77). */
enum { NB_GEO_PLANE = 1, NB_GEO_SPHERE = 3, NB_GEO_CAPSULE = 4, NB_GEO_BOX = 7 };
/* Joint types (newton/_src/sim/enums.py:29-55). */
enum {
    NB_JOINT_PRISMATIC = 0, NB_JOINT_REVOLUTE = 1, NB_JOINT_BALL = 2, NB_JOINT_FIXED = 3,
    NB_JOINT_FREE = 4, NB_JOINT_DISTANCE = 5, NB_JOINT_D6 = 6
};
/* Body flags (newton/_src/sim/enums.py:8-25). */
enum { NB_BODY_DYNAMIC = 1, NB_BODY_KINEMATIC = 2 };

/* Static model description.  Mirrors the Model arrays the reference kernels
 * read (newton/_src/sim/model.py) plus the per-world partition and the
 * per-world candidate pair lists built once on the host. */
typedef struct NbModelDesc {
    int32_t body_count;
    int32_t shape_count;
    int32_t joint_count;
    int32_t joint_dof_count;
    int32_t world_count;
    int32_t global_shape_count;   /* shapes with world == -1 (static) */
    int32_t pair_count;           /* total candidate pairs over all worlds */
    int32_t max_world_bodies;     /* max bodies in one world */
    int32_t max_world_shapes;     /* max world shapes + global shapes */
    int32_t max_world_joints;
    int32_t max_world_pairs;
    int32_t all_joints_free;      /* 1: every joint is FREE (no joint constraints: the step may use its
                                     lean kernel); 0: unknown or not */
    int32_t broad_phase;          /* 0: test every pair of the world's pair list; 1: sweep and prune
                                     (broad_phase_sap.py): sort the world's AABBs along x, sweep, and
                                     keep the overlaps that are in the pair list -- the same candidate
                                     set, O(n log n + overlaps) per world of up to 256 shape slots
                                     (larger worlds test every pair) */
    int32_t pad_bp;
    int64_t contact_capacity;     /* contact slots = 5 * pair_count */

    /* bodies [B] */
    const float* body_com;          /* [B,3] */
    const float* body_mass;         /* [B]   */
    const float* body_inv_mass;     /* [B]   */
    const float* body_inertia;      /* [B,9] */
    const float* body_inv_inertia;  /* [B,9] */
    const int32_t* body_flags;      /* [B]   */
    const int32_t* body_world;      /* [B]   */
    const float* gravity;           /* [W,3] */

    /* shapes [S] */
    const int32_t* shape_body;      /* [S] (-1 = static) */
    const int32_t* shape_type;      /* [S] */
    const float* shape_transform;   /* [S,7] shape in body frame */
    const float* shape_scale;       /* [S,3] */
    const float* shape_margin;      /* [S] */
    const float* shape_gap;         /* [S] */
    const float* shape_radius;      /* [S] bounding radius (1e6 for an infinite plane) */
    const float* shape_mu;          /* [S] */
    const float* shape_mu_torsional;/* [S] */
    const float* shape_mu_rolling;  /* [S] */
    const float* shape_restitution; /* [S] */

    /* joints [J], dofs [D] */
    const int32_t* joint_type;      /* [J] */
    const int32_t* joint_enabled;   /* [J] */
    const int32_t* joint_parent;    /* [J] */
    const int32_t* joint_child;     /* [J] */
    const float* joint_X_p;         /* [J,7] */
    const float* joint_X_c;         /* [J,7] */
    const int32_t* joint_qd_start;  /* [J] */
    const int32_t* joint_dof_dim;   /* [J,2] (linear, angular) */
    const float* joint_axis;        /* [D,3] */
    const float* joint_limit_lower; /* [D] */
    const float* joint_limit_upper; /* [D] */
    const float* joint_target_ke;   /* [D] */
    const float* joint_target_kd;   /* [D] */

    /* world partition */
    const int32_t* world_body_start;   /* [W+1] */
    const int32_t* world_shape_start;  /* [W+1] world-local shapes only */
    const int32_t* world_joint_start;  /* [W+1] */
    const int32_t* global_shapes;      /* [G] global shape indices */
    const int32_t* world_pair_start;   /* [W+1] */
    const uint32_t* pair_shapes;       /* [P+4] packed world-local shape slots a | b<<16 after the
                                          type ordering of narrow_phase.py:207-210,
                                          sorted by contact key within each world.
                                          Slot i < n_local is shape world_shape_start[w]+i,
                                          slot n_local+g is global_shapes[g]. */
    const int32_t* world_order;        /* [W] worlds by decreasing cost (broad phase order) */
    /* solver schedule: batches of worlds that share one CTA's shared memory */
    int32_t batch_count;
    int32_t worlds_per_group;          /* 1 = one world per thread group */
    int32_t group_threads;             /* threads per world group: 32 (warp) ... 256 (CTA) */
    int32_t cta_threads;               /* threads per CTA of nb_xpbd_step */
    int32_t smem_floats_per_batch;     /* shared-memory arena of one CTA, in 4-byte words */
    int32_t step_mode;                 /* 0: batches of worlds (group_threads per world, batch_* arrays);
                                          1: independent groups of group_threads (32/64/128), full
                                             body slab (43 words/body);
                                          2: as 1 with a compact slab (21 words/body, mass
                                             properties read from body_pack); modes 1-2 pull worlds
                                             in world_order, each group owning
                                             arena * group_threads / cta_threads words */
    const int32_t* batch_world;        /* [batch_count, cta_threads/group_threads] world ids, -1 = none */
    const int32_t* batch_slab;         /* [batch_count, cta_threads/group_threads] arena offsets (words) */
    const float* body_pack;            /* [B,24], 16-byte aligned: per body com (3), effective inverse mass,
                                          inertia (9, row-major), effective inverse inertia (9), 2 zeros;
                                          "effective": zero for kinematic bodies (the solver's
                                          _update_effective_inv_mass_inertia, solver.py:160-174); the
                                          caller refreshes it when the model's mass properties or flags
                                          change.  Required by step_mode 2. */
    const int32_t* pair_table;         /* broad_phase 1, optional: per world a dense ns x ns table of
                                          pair indices (ns = the world's shapes + the global shapes;
                                          -1 = no listed pair; both orientations), at
                                          world_table_start[w]; NULL: binary search of the pair list */
    const int64_t* world_table_start;  /* [W+1] offsets into pair_table */
} NbModelDesc;

/* Contact slots and the per-substep collision work buffers (written by
 * nb_collide, read by nb_publish_contacts), and the solver's dense contact
 * records (written by nb_publish_contacts or nb_ingest_contacts, read by
 * nb_xpbd_step): world w's contacts are rec[world_base[w] + k],
 * k < world_count[w], in the solver record layout.  pair_count is
 * NbModelDesc.pair_count; rec_rows = min(pair_count*5, the public capacity
 * rigid_contact_max): the records hold the contacts the public arrays hold
 * (publish keeps the first `capacity` in public order and clamps the worlds'
 * counts past it; ingest takes at most the public count), and never more
 * than 5 per candidate pair. */
typedef struct NbContactSeg {
    float* slots;                /* [pair_count*5, 20] contact slots (5 float4 each), 16-byte aligned */
    float* rec;                  /* [rec_rows, 20] dense solver contact records, 16-byte aligned */
    int64_t* world_base;         /* [W] first rec index of each world */
    int32_t* cand;               /* [pair_count] pair index of each candidate (world-major, key order) */
    int32_t* cand_count;         /* [W] candidates per world */
    uint8_t* counts;             /* [pair_count] contacts written by each candidate (0..5) */
    int32_t* queue;              /* [2*pair_count, 2] narrow-phase work items (candidate, world):
                                    analytic queue from the front, MPR/GJK queue from the back */
    int32_t* world_count;        /* [W] contacts per world */
    float* geom;                 /* [shape_count, 20] world-space shape geometry staged per substep */
    int32_t* work_counter;       /* [8] device counters, zeroed by the entry points */
    uint32_t* status;            /* [1] NB_STATUS_* bits (sticky, cleared by the caller) */
    int32_t* rec_index;          /* [rec_rows] public contact index of each record, or NULL;
                                    needed only for per-contact impulses (written by publish / ingest) */
} NbContactSeg;

/* Public Contacts arrays in the reference layout (newton/_src/sim/contacts.py:43-186). */
typedef struct NbContactsPublic {
    int32_t capacity;            /* rigid_contact_max */
    int32_t pad0;
    int32_t* count;              /* [1] rigid_contact_count (may exceed capacity on overflow) */
    int32_t* shape0;             /* [cap] */
    int32_t* shape1;             /* [cap] */
    float* point0;               /* [cap,3] */
    float* point1;               /* [cap,3] */
    float* offset0;              /* [cap,3] */
    float* offset1;              /* [cap,3] */
    float* normal;               /* [cap,3] */
    float* margin0;              /* [cap] */
    float* margin1;              /* [cap] */
    int64_t* sort_key;           /* [cap] or NULL */
    int64_t* world_offset;       /* [W+1] scratch for the world scan */
    int32_t* generation;         /* [1] Contacts.contact_generation, bumped by every publish (wraps to 0 after
                                    INT32_MAX, as compute_shape_aabbs does, collide.py:211-218), or NULL */
} NbContactsPublic;

/* Frame-to-frame contact matching state (CollisionPipeline contact_matching,
 * newton/_src/geometry/contact_match.py).  All arrays are device memory owned
 * by the caller and persist between calls; prev_count must start at 0.
 * match_index rows past the live count hold -1 (rows the previous call wrote
 * are reset), so a buffer must start filled with -1. */
typedef struct NbMatchState {
    int32_t capacity;            /* rigid_contact_max (rows of every per-contact array) */
    int32_t sticky;              /* 0: "latest", 1: "sticky" (replay matched rows) */
    float pos_threshold_sq;      /* contact_matching_pos_threshold^2 [m^2] */
    float normal_dot_threshold;  /* contact_matching_normal_dot_threshold */
    int32_t* prev_count;         /* [2] contacts saved from the previous call; match_index rows
                                    the previous call wrote (start both at 0; a reset zeroes [0]) */
    int64_t* prev_world_offset;  /* [W+1] the previous call's per-world public offsets */
    int64_t* prev_keys;          /* [cap] previous sort keys */
    float* prev_mid;             /* [cap,3] previous world-space contact midpoints */
    float* prev_normal;          /* [cap,3] previous normals */
    int64_t* prev_claim;         /* [cap] scratch */
    int32_t* prev_was_matched;   /* [cap] scratch, required with new_indices, else NULL */
    float* prev_point0;          /* [cap,3] sticky only (else NULL): body-frame point0 */
    float* prev_point1;          /* [cap,3] */
    float* prev_offset0;         /* [cap,3] */
    float* prev_offset1;         /* [cap,3] */
    float* prev_normal_sticky;   /* [cap,3] */
    int32_t* match_index;        /* [cap] out: previous index, -1 not found, -2 broken */
    int32_t* new_indices;        /* [cap] out (contact_report) or NULL */
    int32_t* new_count;          /* [1] */
    int32_t* broken_indices;     /* [cap] out: previous indices nobody matched */
    int32_t* broken_count;       /* [1] */
} NbMatchState;

/* Learned warm start network (no counterpart in the reference): BF16 MLP
 * 24 -> 128 -> 128 -> 3 with SiLU, weights row-major [out, in] as raw bf16
 * bits; w1 is padded to 32 inputs and w3 to 16 outputs with zeros.  The
 * network predicts ratios y of the contact's velocity correction to a prior
 * (feature row column 26: the previous substep's correction of the matched
 * contact, else the velocity that removes the expected depth):
 * c = prior * y, lambda = c / w with w the generalised inverse mass along
 * the normal (column 24) or the tangents (column 25); lambda_n >= 0 and
 * |lambda_t| <= mu lambda_n (mu: column 17).  A feature row holds
 * NB_WS_FEATURES floats: the 24 network inputs, then w_n, w_t, prior. */
#define NB_WS_INPUTS 24
#define NB_WS_FEATURES 27
#define NB_WS_HIDDEN 128
#define NB_WS_OUTPUTS 3
typedef struct NbWsNet {
    const uint16_t* w1;          /* [128, 32] */
    const float* b1;             /* [128] */
    const uint16_t* w2;          /* [128, 128] */
    const float* b2;             /* [128] */
    const uint16_t* w3;          /* [16, 128] */
    const float* b3;             /* [16] */
    const float* in_mean;        /* [24] feature normalisation: x' = (x - mean) * inv_std */
    const float* in_inv_std;     /* [24] */
    const float* out_scale;      /* [3] y = network output * out_scale */
} NbWsNet;

/* One training step's buffers (forward + backward of the MLP on `rows`
 * samples, FP32 masters; weights row-major [out, in] without padding). */
typedef struct NbWsTrain {
    int32_t rows;
    int32_t pad0;
    const float* x;              /* [rows, 24] raw network inputs */
    const float* t;              /* [rows, 3] target ratios y = lambda * w / prior */
    const float* in_mean;        /* [24] */
    const float* in_inv_std;     /* [24] */
    const float* out_scale;      /* [3] */
    const float* w1; const float* b1;   /* [128,24], [128] */
    const float* w2; const float* b2;   /* [128,128], [128] */
    const float* w3; const float* b3;   /* [3,128], [3] */
    float* g_w1; float* g_b1; float* g_w2; float* g_b2; float* g_w3; float* g_b3;  /* gradients */
    float* xn;                   /* [rows, 24] scratch */
    float* z1; float* h1; float* z2; float* h2;  /* [rows, 128] scratch */
    float* y; float* dy;         /* [rows, 3] scratch */
    float* dh; float* dh2;       /* [rows, 128] scratch */
    float* scratch_wq;           /* [128*24 + 128*128 + 3*128] scratch */
    float* loss;                 /* [1] mean squared error of the normalised outputs */
    uint32_t* status;            /* [1] NB_STATUS_* bits (a tensor-core wait that timed out) */
} NbWsTrain;

/* SolverXPBD constructor arguments (newton/_src/solvers/xpbd/solver_xpbd.py:95-109). */
typedef struct NbXpbdParams {
    int32_t iterations;
    int32_t rigid_contact_con_weighting;
    int32_t enable_restitution;
    int32_t pad0;
    float joint_linear_relaxation;
    float joint_angular_relaxation;
    float joint_linear_compliance;
    float joint_angular_compliance;
    float rigid_contact_relaxation;
    float angular_damping;
} NbXpbdParams;

/* Per-step state buffers (State / Control arrays). */
typedef struct NbStepIO {
    const float* body_q_in;      /* [B,7] */
    const float* body_qd_in;     /* [B,6] */
    const float* body_f_in;      /* [B,6] */
    float* body_q_out;           /* [B,7] */
    float* body_qd_out;          /* [B,6] */
    const float* joint_target_pos; /* [D] (may be NULL when no joint drives) */
    const float* joint_target_vel; /* [D] */
    const float* joint_f;          /* [D] */
    float* contact_impulse;      /* [cap,6] accumulated weighted A-side impulse per public contact, or
                                    NULL; the caller zeroes it before the step (solver_xpbd.py:286-291) */
    float* impulse_scratch;      /* [rec_rows, 6] zero-filled scratch (one row per solver record of
                                    NbContactSeg), required with contact_impulse;
                                    left zero-filled on return */
    int32_t contact_impulse_capacity; /* rows of contact_impulse (rigid_contact_max) */
    int32_t pad0;
    float* body_parent_f;        /* [B,6] incoming joint wrench per body (State.body_parent_f) or NULL */
    float* joint_impulse;        /* [J,6] zero-filled scratch, required with body_parent_f; left
                                    zero-filled on return */
    const float* ws_lambda;      /* [ws_capacity,3] learned warm start: predicted impulse of each public
                                    contact in its contact frame (n, t1, t2), or NULL (plain solve) */
    int32_t ws_capacity;         /* rows of ws_lambda */
    int32_t ws_flags;            /* NB_WS_KEEP_ALL: keep every world's prediction (no fallback) */
    int32_t* ws_fallback;        /* [1] worlds whose warm start was rejected (counter) or NULL */
} NbStepIO;
#define NB_WS_KEEP_ALL 1

/* ABI version of the loaded library (NB_ABI_VERSION). */
int nb_abi_version(void);

/* The cudaError_t behind the last NB_ERR_CUDA an entry point returned on the
 * calling host thread (0 if none), and CUDA's description of a cudaError_t. */
int nb_last_cuda_error(void);
const char* nb_cuda_error_string(int code);


/* Number of CTAs the persistent kernels launch on the current device. */
int32_t nb_default_grid(void);

/*
 * State.clear_forces (newton/_src/sim/state.py:156): zero body_f [n_bodies, 6]
 * with a memset on the stream (no kernel launch).
 */
int nb_clear_forces(float* body_f, int32_t n_bodies, void* stream);

/*
 * Collision detection for all worlds: shape world transforms + AABBs
 * (replaces compute_shape_aabbs, collide.py:150-275), candidate-pair AABB test
 * (BroadPhaseExplicit, broad_phase_nxn.py:28-66; the NxN pair set of
 * broad_phase_nxn.py:129-214 is the same list), primitive and MPR/GJK narrow
 * phase with write_contact semantics (narrow_phase.py:153-776, collide.py:62-147)
 * and deterministic key-ordered compaction (contact_sort.py).
 * Writes the solver-format segments in `seg`.
 */
int nb_collide(const NbModelDesc* model, const float* body_q, const NbContactSeg* seg,
               int32_t grid_ctas, void* stream);  /* grid_ctas: narrow-phase CTAs, <= 0 = library default */

/*
 * Publish solver-format segments into the reference's dense Contacts arrays
 * ordered by (world, key); replaces the Contacts writes of write_contact
 * (collide.py:62-147) and ContactSorter.sort_full (contact_sort.py:305-400).
 */
int nb_publish_contacts(const NbModelDesc* model, const NbContactSeg* seg,
                        const NbContactsPublic* pub, void* stream);

/*
 * One XPBD substep for all worlds: apply_joint_forces, integrate_bodies,
 * `iterations` x (solve_body_contact_positions, apply_body_deltas,
 * solve_body_joints, apply_body_deltas), optional restitution and the
 * kinematic pass-through.  Replaces SolverXPBD.step (solver_xpbd.py:259-764).
 * With model->all_joints_free == 1 and neither restitution nor per-contact
 * impulses requested, a lean kernel without the joint solve runs (same
 * results); 0 always selects the full kernel.
 */
int nb_xpbd_step(const NbModelDesc* model, const NbXpbdParams* params, const NbStepIO* io,
                 const NbContactSeg* seg, float dt, int32_t grid_ctas, void* stream);

/*
 * n_substeps x (nb_collide, nb_publish_contacts, nb_xpbd_step) in one call --
 * the frame loop of the reference's examples (collide + SolverXPBD.step per
 * substep, e.g. newton/examples/contacts/example_pyramid.py:155-161) without a host round
 * trip per substep.  The state ping-pongs between io's input and output
 * buffers: body_q_in / body_qd_in hold the initial state and are overwritten
 * (as the reference's state_in is), body_q_out / body_qd_out receive the
 * final state; body_f_in is applied at every substep.  The plain solve only:
 * contact_impulse, body_parent_f and ws_lambda must be NULL
 * (NB_ERR_UNSUPPORTED).  pub receives the last substep's contacts.
 */
int nb_xpbd_substeps(const NbModelDesc* model, const NbXpbdParams* params, const NbStepIO* io,
                     const NbContactSeg* seg, const NbContactsPublic* pub, float dt, int32_t n_substeps,
                     int32_t grid_ctas, void* stream);

/*
 * Match the contacts nb_publish_contacts just wrote (with sort keys) against
 * the previous call's, then (sticky) replay matched rows, build the report and
 * save this frame for the next call.  Replaces ContactMatcher.match /
 * replay_matched / build_report / save_sorted_state
 * (newton/_src/geometry/contact_match.py:720-990) as called from
 * CollisionPipeline.collide (collide.py:1083-1182).  body_q: the poses the
 * contacts were generated at.
 */
int nb_match_contacts(const NbModelDesc* model, const float* body_q, const NbContactsPublic* pub,
                      const NbContactSeg* seg, const NbMatchState* state, void* stream);

/*
 * Learned warm start (no counterpart in the reference).
 * nb_ws_features: NB_WS_FEATURES floats per published contact from the
 * pre-step state: matched flag, ratios to the prior of the depth estimate,
 * the previous substep's corrections (through match_index), the relative
 * velocity, depth, gravity and thickness; normal, inverse-mass shares,
 * friction, body contact counts, log2 prior, direction to the other body,
 * static side; then w_n, w_t, prior.  body_count: [B] scratch.
 * nb_ws_targets: contact-frame lambdas of accumulated A-side impulses
 * ([cap,6] as written by nb_xpbd_step's contact_impulse); clear_impulse != 0
 * zeroes the live rows after reading, leaving the buffer ready for the next
 * step.
 * nb_ws_infer: the MLP on tensor cores (tcgen05), lambda [cap,3] for the
 * first min(count, cap) contacts (zero where the prior is zero).
 * nb_ws_grads / nb_ws_adam: training (gradients of the mean squared error,
 * GEMMs on tensor cores with FP32 accumulation; Adam update of an FP32
 * master array).
 */
int nb_ws_features(const NbModelDesc* model, const float* body_q, const float* body_qd,
                   const NbContactsPublic* pub, const float* prev_lambda, const int32_t* match_index,
                   int32_t* body_count, float dt, float* features, void* stream);
int nb_ws_targets(const NbContactsPublic* pub, float* contact_impulse, float* lambda, int32_t clear_impulse,
                  void* stream);
int nb_ws_infer(const NbWsNet* net, const float* features, const int32_t* count, int32_t capacity,
                float* lambda, uint32_t* status, void* stream);
int nb_ws_grads(const NbWsTrain* args, void* stream);
int nb_ws_adam(float* w, const float* grad, float* m1, float* m2, int64_t count, float lr, float beta1,
               float beta2, float eps, float weight_decay, int32_t step, void* stream);

/*
 * Adjoint of one substep (no counterpart in the reference's compiled code:
 * the reference differentiates SolverXPBD.step with wp.Tape over its Warp
 * kernels, solver_xpbd.py).  Given the step's inputs and the cotangents of
 * its outputs, writes the cotangents of body_q, body_qd and body_f.  Free
 * rigid bodies with contacts: the contact records of `seg` (as the step used
 * them) are held fixed, kinematic bodies are constants; a world with an
 * enabled non-free joint is skipped with NB_STATUS_ADJOINT_UNSUPPORTED;
 * restitution returns NB_ERR_UNSUPPORTED.  The forward pass is recomputed
 * inside (optionally written to body_q_out / body_qd_out).
 *
 * Branches.  The substep is piecewise smooth: per iteration, which contacts
 * are active (depth < 0), whether friction, torsional and rolling friction
 * are clamped to their cones, and whether a body's speeds fall under the
 * 1e-4 rest threshold.  The cotangents are those of the piece the forward
 * pass is on.  branch_mode 1 writes the forward pass's branches (one byte per
 * contact record and iteration, one per body and iteration); branch_mode 2
 * takes them from those arrays instead of evaluating them, so that a finite
 * difference around a recorded substep stays on its piece; it requires
 * forward_only, which runs the forward pass alone (body_q_out / body_qd_out
 * required; the cotangent pointers and grad_acc may be NULL).
 */
typedef struct NbAdjointIO {
    const float* body_q_in;      /* [B,7] the step's input state */
    const float* body_qd_in;     /* [B,6] */
    const float* body_f_in;      /* [B,6] */
    const float* grad_q_out;     /* [B,7] cotangent of the output body_q */
    const float* grad_qd_out;    /* [B,6] cotangent of the output body_qd */
    float* grad_q_in;            /* [B,7] out */
    float* grad_qd_in;           /* [B,6] out */
    float* grad_f_in;            /* [B,6] out, or NULL */
    float* body_q_out;           /* [B,7] out (the recomputed forward state), or NULL */
    float* body_qd_out;          /* [B,6] out, or NULL with body_q_out */
    float* tape_state;           /* [(iterations+1)*B*13] scratch */
    float* tape_delta;           /* [iterations*B*6] scratch */
    float* tape_weight;          /* [iterations*B] scratch */
    double* grad_acc;            /* [B*13] scratch */
    float* delta_acc;            /* [B*6] scratch */
    int32_t* count_acc;          /* [B] scratch */
    int32_t* active;             /* [iterations * active_capacity * 2] scratch: (record, world) of active contacts */
    int32_t* active_count;       /* [iterations] scratch */
    int32_t active_capacity;     /* active contacts per iteration (>= the contact count; overflow sets
                                    NB_STATUS_CONTACT_OVERFLOW) */
    int32_t pad0;
    uint32_t* status;            /* [1] NB_STATUS_* bits (sticky) */
    double* grad_shape_mu;       /* [S] accumulated (+=) cotangent of shape_mu (the friction coefficient a
                                    contact uses is the mean of its shapes'), or NULL */
    uint8_t* branch_contact;     /* [iterations * model->contact_capacity] branches of each contact record
                                    (bit 0 active, 1/2 friction error > 0 / clamped, 3/4/5 torsion error != 0
                                    / clamped low / high, 6/7 rolling error > 0 / clamped), or NULL */
    uint8_t* branch_body;        /* [iterations * B] rest thresholds of each body update (bits 0/1 linear /
                                    angular speed zeroed; 2/3 the same in the joint pass's update), or NULL */
    int32_t branch_mode;         /* 0 evaluate, 1 evaluate and record, 2 replay the recorded branches */
    int32_t forward_only;        /* nonzero: the forward pass only */
} NbAdjointIO;
int nb_xpbd_step_adjoint(const NbModelDesc* model, const NbXpbdParams* params, const NbAdjointIO* io,
                         const NbContactSeg* seg, float dt, void* stream);

/*
 * contacts.force from the impulses a step accumulated: force = impulse / dt for
 * rows < count[0] (read on the device), zero for the rest of `capacity` rows.
 * Replaces convert_contact_impulse_to_force (xpbd/kernels.py:2363-2393) as
 * launched by SolverXPBD.update_contacts (solver_xpbd.py:766-821).
 */
int nb_contact_forces(const float* contact_impulse, const int32_t* count, int32_t capacity, float dt,
                      float* force, void* stream);

/*
 * Move contacts a caller wrote into the dense public arrays (custom contact
 * writers) into solver records, bucketed by world.  Replaces nothing in the
 * reference (its solver reads the dense arrays directly,
 * xpbd/kernels.py:2062-2298).  Records keep the public order within each
 * world (public indices are bucketed by world, then ranked; the buckets use
 * seg->slots as scratch, which nb_collide rewrites anyway), and the solver
 * sums each body's deltas in record order: the pipeline's own contacts
 * ingested in their published order give the collide path's step bit for
 * bit, and a caller that writes the same contacts in another order changes
 * the bodies' sums by float rounding only, the same on every call.
 */
int nb_ingest_contacts(const NbModelDesc* model, const NbContactsPublic* pub,
                       const NbContactSeg* seg, void* stream);

/*
 * nb_publish_contacts without the caller's scan scratch: same outputs, but
 * pub->world_offset is ignored (may be NULL) and the world offsets live in a
 * file-scope device array of NB_PUBLISH_STATIC_MAX_WORLDS + 1 entries.  It
 * allocates nothing, for callers that cannot allocate device memory or hold
 * only the reference Contacts arrays (which have no per-world offsets).  No
 * counterpart in the reference.  Returns NB_ERR_CAPACITY when
 * model->world_count > NB_PUBLISH_STATIC_MAX_WORLDS.  One scratch array per
 * device: calls that may overlap in time on one device race; calls on one
 * stream are ordered.  Nothing in the scratch must start at zero.  The first
 * call on a device looks up the array's address (cudaGetSymbolAddress); make
 * it before any stream capture.  The address is kept for the life of the
 * process: cudaDeviceReset between calls is not supported (the next call
 * would write through the address of the destroyed context).
 * The caller's pub->world_offset is neither read nor written, so this call
 * cannot feed the consumer of per-world offsets: nb_match_contacts (contact
 * matching) reads pub->world_offset and needs nb_publish_contacts.
 */
#define NB_PUBLISH_STATIC_MAX_WORLDS 65536
int nb_publish_contacts_static(const NbModelDesc* model, const NbContactSeg* seg,
                               const NbContactsPublic* pub, void* stream);

/* ------------------------------------------------------------------------
 * Particles: the XPBD particle path (newton/_src/solvers/xpbd/kernels.py:
 * 114-357, 776-807; newton/_src/solvers/solver.py:11-47) and the soft
 * contacts between particles and shapes (newton/_src/geometry/kernels.py:
 * 1000-1140).  Particles are independent of the rigid-body step: they
 * collide with each other and with shapes, and the solver accepts particle
 * contacts with static shapes only (shape_body == -1).
 * ------------------------------------------------------------------------ */

/* Particle flag bit (newton/_src/sim/enums.py ParticleFlags.ACTIVE). */
#define NB_PARTICLE_ACTIVE 1
/* Status bits of the particle step (sticky, in NbParticleIO.status). */
#define NB_STATUS_PARTICLE_BODY_CONTACT (1u << 7)  /* a soft contact with a body-attached shape was skipped */
#define NB_STATUS_NEIGHBOR_OVERFLOW (1u << 8)      /* a particle touched more than NB_PARTICLE_MAX_NEIGHBORS others */
/* Particle-particle contacts summed per particle and iteration; more are dropped with
 * NB_STATUS_NEIGHBOR_OVERFLOW (twelve equal spheres can touch one). */
#define NB_PARTICLE_MAX_NEIGHBORS 32

/* Particles, springs and the shapes particles collide with: the Model arrays of
 * the same names (newton/_src/sim/model.py particle_*, spring_*, shape_*). */
typedef struct NbParticleDesc {
    int32_t particle_count;
    int32_t spring_count;
    int32_t shape_count;
    int32_t world_count;              /* rows of gravity */
    float particle_max_velocity;      /* Model.particle_max_velocity */
    float particle_max_radius;        /* Model.particle_max_radius */
    float particle_mu;                /* Model.particle_mu: particle-particle friction */
    float particle_cohesion;          /* Model.particle_cohesion */
    float particle_adhesion;          /* Model.particle_adhesion: particle-shape contact distance */
    float soft_contact_mu;            /* Model.soft_contact_mu */
    const float* particle_inv_mass;   /* [P]   */
    const float* particle_radius;     /* [P]   */
    const int32_t* particle_flags;    /* [P]   NB_PARTICLE_ACTIVE */
    const int32_t* particle_world;    /* [P]   (-1 = global) */
    const float* gravity;             /* [W,3] */
    const int32_t* spring_indices;    /* [S,2] */
    const float* spring_rest_length;  /* [S]   */
    const float* spring_stiffness;    /* [S]   */
    const float* spring_damping;      /* [S]   */
    const int32_t* particle_spring_start; /* [P+1] springs of particle p: particle_spring_list[start[p]..start[p+1]) */
    const int32_t* particle_spring_list;  /* [2S]  spring indices, ascending per particle */
    const int32_t* shape_body;        /* [Sh]  (-1 = static) */
    const int32_t* shape_type;        /* [Sh]  NB_GEO_* */
    const float* shape_transform;     /* [Sh,7] shape in body frame */
    const float* shape_scale;         /* [Sh,3] */
    const int32_t* shape_world;       /* [Sh]  */
    const int32_t* shape_flags;       /* [Sh]  bit 2 = COLLIDE_PARTICLES */
    const float* shape_mu;            /* [Sh]  */
    int32_t edge_count;               /* bending edges */
    float soft_contact_restitution;   /* Model.soft_contact_restitution */
    const int32_t* edge_indices;      /* [E,4] (i, j, k, l): opposite vertices i, j of the hinge edge k-l */
    const float* edge_rest_angle;     /* [E]   */
    const float* edge_bending_properties; /* [E,2] (ke, kd) */
    const int32_t* particle_edge_start;   /* [P+1] edges of particle p: particle_edge_list[start[p]..start[p+1]) */
    const int32_t* particle_edge_list;    /* edge indices, ascending per particle */
    int32_t tet_count;                /* tetrahedra */
    float soft_body_relaxation;       /* SolverXPBD.soft_body_relaxation: the tetrahedra's compliance */
    const int32_t* tet_indices;       /* [T,4] */
    const float* tet_poses;           /* [T,9] inverse rest matrices (row-major mat33) */
    const int32_t* particle_tet_start;    /* [P+1] tetrahedra of particle p: particle_tet_list[start[p]..start[p+1]) */
    const int32_t* particle_tet_list;     /* tetrahedron indices, ascending per particle */
} NbParticleDesc;

/* Soft contacts (newton/_src/sim/contacts.py soft_contact_* arrays), in
 * (particle, shape) order. */
typedef struct NbSoftContacts {
    int32_t* count;           /* [1] contacts found; may exceed max, the first max are stored */
    int32_t* particle;        /* [max] */
    int32_t* shape;           /* [max] */
    float* body_pos;          /* [max,3] contact point in the shape's body frame */
    float* body_vel;          /* [max,3] */
    float* normal;            /* [max,3] world frame */
    int32_t max;
    float margin;             /* contact when the shape's signed distance < margin + radius */
    int32_t* particle_start;  /* [P + 2 + ceil(P/1024)] scratch written by nb_soft_collide: the first
                                 contact of every particle ([0, P]), then per-block counts; read
                                 back by nb_particle_step */
} NbSoftContacts;

/* Work buffers of one particle substep. */
typedef struct NbParticleIO {
    const float* particle_q;   /* [P,3] state_in positions (read only) */
    const float* particle_qd;  /* [P,3] state_in velocities (read only) */
    const float* particle_f;   /* [P,3] state_in forces, or NULL for none */
    float* particle_q_out;     /* [P,3] state_out positions */
    float* particle_qd_out;    /* [P,3] state_out velocities */
    float* delta;              /* [P,3] scratch: the iteration's position corrections */
    int32_t* grid_head;        /* [2*grid_size] scratch: two hashed cell tables (first particle, -1 empty) */
    int32_t* grid_next;        /* [P] scratch: next particle of the same cell */
    int32_t grid_size;         /* cells per table, a power of two */
    int32_t enable_restitution; /* 1: apply_particle_shape_restitution (kernels.py:34-112) after the iterations */
    uint32_t* status;          /* [1] NB_STATUS_* bits (sticky, cleared by the caller) */
} NbParticleIO;

/*
 * Soft contacts of every active particle with every particle-colliding shape
 * of its world (create_soft_contacts, newton/_src/geometry/kernels.py:1000-
 * 1140; launched from newton/_src/sim/collide.py:1194-1230) for plane,
 * sphere, capsule and box shapes.  The reference appends contacts with an
 * atomic counter; here every particle's contacts follow one exclusive scan,
 * so the list is in (particle, shape) order, the order of the reference's
 * thread ids, on every run.  body_q may be NULL when no shape is attached to
 * a body.
 */
int nb_soft_collide(const NbParticleDesc* pd, const float* particle_q, const float* body_q,
                    const NbSoftContacts* sc, void* stream);

/*
 * One XPBD substep of the particles (SolverXPBD.step's particle branch,
 * newton/_src/solvers/xpbd/solver_xpbd.py:303-320, 377-505, 657-660):
 * integrate_particles (solver.py:11-47), then `iterations` times the
 * particle-shape contacts (kernels.py:114-222), particle-particle contacts
 * (kernels.py:225-289), springs (kernels.py:292-356), bending edges
 * (bending_constraint, kernels.py:358-457; the dihedral angle through an
 * atan2 built on the library's own asin, so that the oracle can match it bit
 * for bit), tetrahedra (solve_tetrahedra, kernels.py:459-628) and
 * apply_particle_deltas (kernels.py:776-807).  Each particle gathers its
 * corrections in a fixed order (its soft contacts, then its particle
 * neighbours in ascending index, then its springs, then its bending edges,
 * each in ascending index)
 * instead of the reference's atomic adds, so results do not change from run
 * to run.  sc may be NULL (no soft contacts); sc->particle_start must come
 * from nb_soft_collide on the same contacts.  Soft contacts with a
 * body-attached shape are skipped (NB_STATUS_PARTICLE_BODY_CONTACT).  With
 * io->enable_restitution, every particle then adds the restitution velocity
 * change of each of its soft contacts, in list order, all computed from its
 * velocity after the iterations.
 */
int nb_particle_step(const NbParticleDesc* pd, const NbParticleIO* io, const NbSoftContacts* sc, float dt,
                     int32_t iterations, float relaxation, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NEWTON_B200_H */
