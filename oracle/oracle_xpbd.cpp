// TEST INFRASTRUCTURE ONLY -- CPU oracle of Newton's SolverXPBD rigid substep.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it.
//
// Sequential restatement of:
//   integrate_rigid_body / integrate_bodies   newton/_src/solvers/solver.py:50-157
//   apply_joint_forces                        newton/_src/solvers/xpbd/kernels.py:890-1003
//   solve_body_contact_positions              newton/_src/solvers/xpbd/kernels.py:2062-2298
//   compute_contact_constraint_delta          newton/_src/solvers/xpbd/kernels.py:1945-1979
//   solve_body_joints                         newton/_src/solvers/xpbd/kernels.py:1441-1942
//   compute_positional/angular_correction     newton/_src/solvers/xpbd/kernels.py:1982-2059
//   apply_body_deltas                         newton/_src/solvers/xpbd/kernels.py:809-878
//   accumulate_weighted_contact_impulse       newton/_src/solvers/xpbd/kernels.py:2301-2360
//   apply_rigid_restitution                   newton/_src/solvers/xpbd/kernels.py:2471-2620
//   apply_body_delta_velocities               newton/_src/solvers/xpbd/kernels.py:881-887
//   SolverXPBD.step orchestration             newton/_src/solvers/xpbd/solver_xpbd.py:259-764
//
// The reference sums per-body deltas with float atomics, i.e. in an unspecified
// order on a GPU.  This oracle offers two accumulation modes:
//   ORC_ACC_FLOAT  -- plain fp32 sums in contact-index (joint-index) order: the
//                     reference run sequentially, and what the CUDA kernels
//                     compute (their ordered accumulation), so the two agree
//                     bit for bit;
//   ORC_ACC_FIXED  -- each contribution is rounded to a 2^-32 fixed-point
//                     int64 and summed exactly (order-independent); kept to
//                     measure how far another summation rule lands from the
//                     reference.
#include "oracle_math.h"
#include "../include/newton_b200.h"

#include <cstring>
#include <vector>

namespace orc {

enum { ORC_ACC_FIXED = 0, ORC_ACC_FLOAT = 1 };

static const float FX_SCALE = 4294967296.0f;        // 2^32
static const float FX_INV = 1.0f / 4294967296.0f;   // 2^-32 (exact)
static const float FX_LIMIT = 9.0e18f;

struct Acc {
    int mode;
    uint32_t* status;
    std::vector<int64_t> fx;   // [nb*6]
    std::vector<float> fl;     // [nb*6]
    std::vector<float> cnt;    // [nb]
    void reset(int nb) {
        fx.assign((size_t)nb * 6, 0);
        fl.assign((size_t)nb * 6, 0.0f);
        cnt.assign((size_t)nb, 0.0f);
    }
    int64_t q(float x) {
        float y = x * FX_SCALE;
        if (!(std::fabs(y) < FX_LIMIT)) {
            *status |= NB_STATUS_FIXED_OVERFLOW;
            if (y != y) y = 0.0f;
            else y = y > 0.0f ? FX_LIMIT : -FX_LIMIT;
        }
        return (int64_t)std::llrint(y);
    }
    void add(int b, V3 lin, V3 ang) {
        float v[6] = {lin.x, lin.y, lin.z, ang.x, ang.y, ang.z};
        for (int k = 0; k < 6; ++k) {
            if (mode == ORC_ACC_FIXED) fx[(size_t)b * 6 + k] += q(v[k]);
            else fl[(size_t)b * 6 + k] = fl[(size_t)b * 6 + k] + v[k];
        }
    }
    void get(int b, V3& lin, V3& ang) const {
        float v[6];
        for (int k = 0; k < 6; ++k) {
            if (mode == ORC_ACC_FIXED) v[k] = (float)fx[(size_t)b * 6 + k] * FX_INV;
            else v[k] = fl[(size_t)b * 6 + k];
        }
        lin = V3{v[0], v[1], v[2]};
        ang = V3{v[3], v[4], v[5]};
    }
};

struct BodyState {
    TF q;
    V3 v, w;
};

// solver.py:50-94
static void integrate_rigid_body(BodyState& s, V3 f0, V3 t0, V3 com, const M33& I, float inv_mass,
                                 const M33& inv_I, V3 g, float angular_damping, float dt) {
    V3 x0 = s.q.p;
    Q4 r0 = s.q.q;
    V3 w0 = s.w, v0 = s.v;
    V3 x_com = add(x0, qrot(r0, com));
    float nz = inv_mass != 0.0f ? 1.0f : 0.0f;
    V3 v1 = add(v0, mul(add(mul(f0, inv_mass), mul(g, nz)), dt));
    V3 x1 = add(x_com, mul(v1, dt));
    V3 wb = qrot_inv(r0, w0);
    V3 tb = sub(qrot_inv(r0, t0), cross(wb, mv(I, wb)));
    V3 w1 = qrot(r0, add(wb, mul(mv(inv_I, tb), dt)));
    Q4 r1 = qnormalize(qadd(r0, qscale(qscale(qmul(Q4{w1.x, w1.y, w1.z, 0.0f}, r0), 0.5f), dt)));
    w1 = mul(w1, 1.0f - angular_damping * dt);
    s.q = TF{sub(x1, qrot(r1, com)), r1};
    s.v = v1;
    s.w = w1;
}

// kernels.py:809-878 (weight already resolved: 1.0 or 1/count)
static void apply_body_delta(BodyState& s, V3 dlin, V3 dang, float weight, V3 com, const M33& I, float inv_m,
                             const M33& inv_I, float dt) {
    if (inv_m == 0.0f) return;
    V3 v0 = s.v, w0 = s.w;
    V3 p0 = s.q.p;
    Q4 q0 = s.q.q;
    V3 dp = mul(dlin, inv_m * weight);
    V3 dq = mul(dang, weight);
    V3 wb = qrot_inv(q0, w0);
    V3 dwb = mv(inv_I, qrot_inv(q0, dq));
    V3 tb = add(cross(dwb, mv(I, add(wb, dwb))), cross(wb, mv(I, dwb)));
    V3 dw1 = qrot(q0, sub(dwb, mv(mscale(dt, inv_I), tb)));
    Q4 dq4 = qscale(Q4{dw1.x * dt, dw1.y * dt, dw1.z * dt, 0.0f}, 0.5f);
    Q4 q1 = qadd(q0, qmul(dq4, q0));
    q1 = qnormalize(q1);
    V3 x_com = add(p0, qrot(q0, com));
    V3 p1 = add(x_com, mul(dp, dt));
    p1 = sub(p1, qrot(q1, com));
    s.q = TF{p1, q1};
    V3 v1 = add(v0, dp);
    V3 w1 = add(w0, dw1);
    if (length(v1) < 1e-4f) v1 = V3{0.0f, 0.0f, 0.0f};
    if (length(w1) < 1e-4f) w1 = V3{0.0f, 0.0f, 0.0f};
    s.v = v1;
    s.w = w1;
}

// kernels.py:1945-1979
static float contact_constraint_delta(float err, Q4 qa, Q4 qb, float m_inv_a, float m_inv_b, const M33& Ia,
                                      const M33& Ib, V3 la, V3 lb, V3 aa, V3 ab, float relaxation, float dt) {
    float denom = 0.0f;
    denom += length_sq(la) * m_inv_a;
    denom += length_sq(lb) * m_inv_b;
    V3 ra = qrot_inv(qa, aa);
    V3 rb = qrot_inv(qb, ab);
    denom += dot(ra, mv(Ia, ra));
    denom += dot(rb, mv(Ib, rb));
    float dl = -err;
    if (denom > 0.0f) dl /= dt * denom;
    return dl * relaxation;
}

// kernels.py:1982-2022
static float positional_correction(float err, float derr, Q4 qa, Q4 qb, float m_inv_a, float m_inv_b,
                                   const M33& Ia, const M33& Ib, V3 la, V3 lb, V3 aa, V3 ab, float lambda_in,
                                   float compliance, float damping, float dt) {
    float denom = 0.0f;
    denom += length_sq(la) * m_inv_a;
    denom += length_sq(lb) * m_inv_b;
    V3 ra = qrot_inv(qa, aa);
    V3 rb = qrot_inv(qb, ab);
    denom += dot(ra, mv(Ia, ra));
    denom += dot(rb, mv(Ib, rb));
    float alpha = compliance;
    float gamma = compliance * damping;
    float dl = -(err + alpha * lambda_in + gamma * derr);
    if (denom + alpha > 0.0f) dl /= (dt + gamma) * denom + alpha / dt;
    return dl;
}

// kernels.py:2025-2059
static float angular_correction(float err, float derr, Q4 qa, Q4 qb, const M33& Ia, const M33& Ib, V3 aa, V3 ab,
                                float lambda_in, float compliance, float damping, float dt) {
    float denom = 0.0f;
    V3 ra = qrot_inv(qa, aa);
    V3 rb = qrot_inv(qb, ab);
    denom += dot(ra, mv(Ia, ra));
    denom += dot(rb, mv(Ib, rb));
    float alpha = compliance;
    float gamma = compliance * damping;
    float dl = -(err + alpha * lambda_in + gamma * derr);
    if (denom + alpha > 0.0f) dl /= (dt + gamma) * denom + alpha / dt;
    return dl;
}

struct World {
    const NbModelDesc* m;
    int b0, nb;                      // body range
    std::vector<BodyState> st;       // current state
    std::vector<M33> I, invI;        // effective (kinematic -> 0)
    std::vector<float> inv_m;
    std::vector<V3> com;
    std::vector<int> flags;
    int local(int gb) const { return gb < 0 ? -1 : gb - b0; }
};

struct ContactIn {
    V3 p0, p1, n, o0, o1;
    float m0, m1;
    int s0, s1;
};

static ContactIn load_contact(const OrcSeg* seg, int64_t k) {
    ContactIn c;
    const float* r0 = seg->rec0 + 4 * k;
    const float* r1 = seg->rec1 + 4 * k;
    const float* r2 = seg->rec2 + 4 * k;
    const float* r3 = seg->rec3 + 4 * k;
    const float* r4 = seg->rec4 + 4 * k;
    c.p0 = V3{r0[0], r0[1], r0[2]}; c.m0 = r0[3];
    c.p1 = V3{r1[0], r1[1], r1[2]}; c.m1 = r1[3];
    c.n = V3{r2[0], r2[1], r2[2]}; std::memcpy(&c.s0, &r2[3], 4);
    c.o0 = V3{r3[0], r3[1], r3[2]}; std::memcpy(&c.s1, &r3[3], 4);
    c.o1 = V3{r4[0], r4[1], r4[2]};
    return c;
}

// kernels.py:2062-2298 for one contact; returns false when inactive.
// impulse (optional) receives the A-side spatial delta (contact_impulse_iter).
static bool solve_contact(World& W, const ContactIn& c, const float* body_qd_kin, float relaxation, float dt,
                          Acc& acc, bool weighting, float* impulse6) {
    const NbModelDesc* m = W.m;
    int sa = c.s0, sb = c.s1;
    if (sa == sb) return false;
    int ba = sa >= 0 ? m->shape_body[sa] : -1;
    int bb = sb >= 0 ? m->shape_body[sb] : -1;
    if (ba == bb) return false;
    int la = W.local(ba), lb = W.local(bb);
    TF Xa = la >= 0 ? W.st[la].q : tf_identity();
    TF Xb = lb >= 0 ? W.st[lb].q : tf_identity();
    V3 bx_a = tf_point(Xa, c.p0);
    V3 bx_b = tf_point(Xb, c.p1);
    float thickness = c.m0 + c.m1;
    V3 n = c.n;
    float d = dot(n, sub(bx_b, bx_a)) - thickness;
    if (d >= 0.0f) return false;
    float m_inv_a = 0.0f, m_inv_b = 0.0f;
    M33 Ia = zero_m33(), Ib = zero_m33();
    V3 com_a{0, 0, 0}, com_b{0, 0, 0};
    V3 om_a{0, 0, 0}, om_b{0, 0, 0};
    V3 off_a = c.o0, off_b = c.o1;
    if (la >= 0) { com_a = W.com[la]; m_inv_a = W.inv_m[la]; Ia = W.invI[la]; om_a = W.st[la].w; }
    if (lb >= 0) { com_b = W.com[lb]; m_inv_b = W.inv_m[lb]; Ib = W.invI[lb]; om_b = W.st[lb].w; }
    int nz = 0;
    float mu = 0.0f, mut = 0.0f, mur = 0.0f;
    if (sa >= 0) { nz += 1; mu += m->shape_mu[sa]; mut += m->shape_mu_torsional[sa]; mur += m->shape_mu_rolling[sa]; }
    if (sb >= 0) { nz += 1; mu += m->shape_mu[sb]; mut += m->shape_mu_torsional[sb]; mur += m->shape_mu_rolling[sb]; }
    if (nz > 0) { mu /= (float)nz; mut /= (float)nz; mur /= (float)nz; }
    V3 r_a = sub(bx_a, tf_point(Xa, com_a));
    V3 r_b = sub(bx_b, tf_point(Xb, com_b));
    V3 ang_a = neg(cross(r_a, n));
    V3 ang_b = cross(r_b, n);
    if (weighting) {
        if (la >= 0) acc.cnt[la] += 1.0f;
        if (lb >= 0) acc.cnt[lb] += 1.0f;
    }
    float lambda_n = contact_constraint_delta(d, Xa.q, Xb.q, m_inv_a, m_inv_b, Ia, Ib, neg(n), n, ang_a, ang_b,
                                              relaxation, dt);
    V3 lin_da = mul(neg(n), lambda_n);
    V3 lin_db = mul(n, lambda_n);
    V3 ang_da = mul(ang_a, lambda_n);
    V3 ang_db = mul(ang_b, lambda_n);
    if (mu > 0.0f) {
        bx_a = add(bx_a, tf_vector(Xa, off_a));
        bx_b = add(bx_b, tf_vector(Xb, off_b));
        V3 delta = sub(bx_b, bx_a);
        V3 fd = sub(delta, smul(dot(n, delta), n));
        r_a = sub(bx_a, tf_point(Xa, com_a));
        r_b = sub(bx_b, tf_point(Xb, com_b));
        V3 rvk{0.0f, 0.0f, 0.0f};
        if (la >= 0 && (W.flags[la] & NB_BODY_KINEMATIC)) {
            const float* qd = body_qd_kin + 6 * (size_t)ba;
            V3 va = add(cross(V3{qd[3], qd[4], qd[5]}, r_a), V3{qd[0], qd[1], qd[2]});
            rvk = sub(rvk, sub(va, smul(dot(n, va), n)));
        }
        if (lb >= 0 && (W.flags[lb] & NB_BODY_KINEMATIC)) {
            const float* qd = body_qd_kin + 6 * (size_t)bb;
            V3 vb = add(cross(V3{qd[3], qd[4], qd[5]}, r_b), V3{qd[0], qd[1], qd[2]});
            rvk = add(rvk, sub(vb, smul(dot(n, vb), n)));
        }
        fd = add(fd, mul(rvk, dt));
        V3 perp = normalize(fd);
        ang_a = neg(cross(r_a, perp));
        ang_b = cross(r_b, perp);
        float err = length(fd);
        if (err > 0.0f) {
            float lf = contact_constraint_delta(err, Xa.q, Xb.q, m_inv_a, m_inv_b, Ia, Ib, neg(perp), perp, ang_a,
                                                ang_b, relaxation, dt);
            lf = fmaxw(lf, -lambda_n * mu);
            lin_da = sub(lin_da, mul(perp, lf));
            lin_db = add(lin_db, mul(perp, lf));
            ang_da = add(ang_da, mul(ang_a, lf));
            ang_db = add(ang_db, mul(ang_b, lf));
        }
    }
    V3 dom = sub(om_b, om_a);
    if (mut > 0.0f) {
        float err = dot(dom, n) * dt;
        if (std::fabs(err) > 0.0f) {
            V3 z{0.0f, 0.0f, 0.0f};
            float lt = contact_constraint_delta(err, Xa.q, Xb.q, m_inv_a, m_inv_b, Ia, Ib, z, z, neg(n), n,
                                                relaxation, dt);
            lt = clampw(lt, -lambda_n * mut, lambda_n * mut);
            ang_da = sub(ang_da, mul(n, lt));
            ang_db = add(ang_db, mul(n, lt));
        }
    }
    if (mur > 0.0f) {
        dom = sub(dom, smul(dot(n, dom), n));
        float err = length(dom) * dt;
        if (err > 0.0f) {
            V3 z{0.0f, 0.0f, 0.0f};
            V3 rn = normalize(dom);
            float lr = contact_constraint_delta(err, Xa.q, Xb.q, m_inv_a, m_inv_b, Ia, Ib, z, z, neg(rn), rn,
                                                relaxation, dt);
            lr = fmaxw(lr, -lambda_n * mur);
            ang_da = sub(ang_da, mul(rn, lr));
            ang_db = add(ang_db, mul(rn, lr));
        }
    }
    if (la >= 0) acc.add(la, lin_da, ang_da);
    if (lb >= 0) acc.add(lb, lin_db, ang_db);
    if (impulse6) {
        impulse6[0] = lin_da.x; impulse6[1] = lin_da.y; impulse6[2] = lin_da.z;
        impulse6[3] = ang_da.x; impulse6[4] = ang_da.y; impulse6[5] = ang_da.z;
    }
    return true;
}

static V3 vabs(V3 a) { return V3{std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }

// update_joint_axis_weighted_target (kernels.py:1021-1033)
static void weighted_target(V3 axis, float target, float weight, V3& tgt, V3& wts) {
    V3 wa = mul(axis, weight);
    tgt = add(tgt, mul(wa, target));
    wts = add(wts, vabs(wa));
}

// Gather limit box + weighted targets of up to 3 axes starting at dof `start`
// (kernels.py:1594-1653 and 1815-1874).
static void joint_axes(const NbModelDesc* m, int start, int count, const float* tpos, const float* tvel, V3& lo,
                       V3& hi, V3& tp, V3& stiff, V3& tv, V3& damp) {
    lo = V3{0, 0, 0}; hi = V3{0, 0, 0};
    tp = V3{0, 0, 0}; stiff = V3{0, 0, 0}; tv = V3{0, 0, 0}; damp = V3{0, 0, 0};
    for (int k = 0; k < count && k < 3; ++k) {
        int i = start + k;
        V3 axis = load_v3(m->joint_axis + 3 * i);
        V3 lt = mul(axis, m->joint_limit_lower[i]);
        V3 ut = mul(axis, m->joint_limit_upper[i]);
        if (k == 0) {
            lo = vmin(lt, ut);
            hi = vmax(lt, ut);
        } else {
            V3 l2 = vmin(lt, ut), u2 = vmax(lt, ut);
            lo = vmin(lo, l2);
            hi = vmax(hi, u2);
        }
        float ke = m->joint_target_ke[i], kd = m->joint_target_kd[i];
        float tpi = tpos ? tpos[i] : 0.0f, tvi = tvel ? tvel[i] : 0.0f;
        if (ke > 0.0f) weighted_target(axis, tpi, ke, tp, stiff);
        if (kd > 0.0f) weighted_target(axis, tvi, kd, tv, damp);
    }
    for (int i = 0; i < 3; ++i)
        if (comp(stiff, i) > 0.0f) set_comp(tp, i, comp(tp, i) / comp(stiff, i));
    for (int i = 0; i < 3; ++i)
        if (comp(damp, i) > 0.0f) set_comp(tv, i, comp(tv, i) / comp(damp, i));
}

// solve_body_joints for one joint (kernels.py:1441-1942).
static void solve_joint(World& W, int j, const float* tpos, const float* tvel, const NbXpbdParams* p, float dt,
                        Acc& acc, float* imp = nullptr) {
    const NbModelDesc* m = W.m;
    int type = m->joint_type[j];
    if (!m->joint_enabled[j]) return;
    if (type == NB_JOINT_FREE) return;
    int id_c = m->joint_child[j], id_p = m->joint_parent[j];
    int lc = W.local(id_c), lp = W.local(id_p);
    TF X_pj = load_tf(m->joint_X_p + 7 * j);
    TF X_cj = load_tf(m->joint_X_c + 7 * j);
    TF X_wp = X_pj;
    float m_inv_p = 0.0f;
    M33 I_inv_p = zero_m33();
    TF pose_p = X_pj;
    V3 com_p{0, 0, 0}, vel_p{0, 0, 0}, om_p{0, 0, 0};
    if (id_p >= 0) {
        pose_p = W.st[lp].q;
        X_wp = tf_mul(pose_p, X_wp);
        com_p = W.com[lp];
        m_inv_p = W.inv_m[lp];
        I_inv_p = W.invI[lp];
        vel_p = W.st[lp].v;
        om_p = W.st[lp].w;
    }
    TF pose_c = W.st[lc].q;
    TF X_wc = tf_mul(pose_c, X_cj);
    V3 com_c = W.com[lc];
    float m_inv_c = W.inv_m[lc];
    M33 I_inv_c = W.invI[lc];
    V3 vel_c = W.st[lc].v, om_c = W.st[lc].w;
    if (m_inv_p == 0.0f && m_inv_c == 0.0f) return;
    V3 ldp{0, 0, 0}, adp{0, 0, 0}, ldc{0, 0, 0}, adc{0, 0, 0};
    TF rel = tf_mul(tf_inverse(X_wp), X_wc);
    V3 rel_p = rel.p;
    V3 x_c = X_wc.p;
    float lin_comp = p->joint_linear_compliance, ang_comp = p->joint_angular_compliance;
    float ang_relax = p->joint_angular_relaxation, lin_relax = p->joint_linear_relaxation;
    int axis_start = m->joint_qd_start[j];
    int lin_count = m->joint_dof_dim[2 * j], ang_count = m->joint_dof_dim[2 * j + 1];
    V3 wcom_p = tf_point(pose_p, com_p);
    V3 wcom_c = tf_point(pose_c, com_c);
    if (type == NB_JOINT_DISTANCE) {
        V3 r_p = sub(X_wp.p, wcom_p);
        V3 r_c = sub(X_wc.p, wcom_c);
        float lower = m->joint_limit_lower[axis_start], upper = m->joint_limit_upper[axis_start];
        if (lower < 0.0f && upper < 0.0f) return;
        float d = length(rel_p);
        float err = 0.0f;
        if (lower >= 0.0f && d < lower) {
            err = d - lower;
            rel_p = smul(err, normalize(sub(wcom_c, wcom_p)));
        } else if (upper >= 0.0f && d > upper) {
            err = d - upper;
        }
        if (std::fabs(err) > 1e-9f) {
            V3 lin_c = rel_p;
            V3 lin_p = neg(lin_c);
            r_c = sub(x_c, wcom_c);
            V3 ang_p = neg(cross(r_p, lin_c));
            V3 ang_c = cross(r_c, lin_c);
            float derr = dot(lin_p, vel_p) + dot(lin_c, vel_c) + dot(ang_p, om_p) + dot(ang_c, om_c);
            float compliance = lin_comp;
            float ke = m->joint_target_ke[axis_start];
            if (ke > 0.0f) compliance = 1.0f / ke;
            float damping = m->joint_target_kd[axis_start];
            float dl = positional_correction(err, derr, pose_p.q, pose_c.q, m_inv_p, m_inv_c, I_inv_p, I_inv_c,
                                             lin_p, lin_c, ang_p, ang_c, 0.0f, compliance, damping, dt);
            ldp = add(ldp, mul(lin_p, dl * lin_relax));
            adp = add(adp, mul(ang_p, dl * ang_relax));
            ldc = add(ldc, mul(lin_c, dl * lin_relax));
            adc = add(adc, mul(ang_c, dl * ang_relax));
        }
    } else {
        V3 lo, hi, tp, stiff, tv, damp;
        joint_axes(m, axis_start, lin_count, tpos, tvel, lo, hi, tp, stiff, tv, damp);
        M33 frame_p = quat_to_matrix(X_wp.q);
        V3 r_p = sub(x_c, wcom_p);
        V3 r_c = sub(x_c, tf_point(pose_c, com_c));
        for (int dim = 0; dim < 3; ++dim) {
            float e = comp(rel_p, dim);
            V3 lin_c{frame_p.m[0][dim], frame_p.m[1][dim], frame_p.m[2][dim]};
            V3 lin_p = neg(lin_c);
            V3 ang_p = neg(cross(r_p, lin_c));
            V3 ang_c = cross(r_c, lin_c);
            float derr = dot(lin_p, vel_p) + dot(lin_c, vel_c) + dot(ang_p, om_p) + dot(ang_c, om_c);
            float err = 0.0f, compliance = lin_comp, damping = 0.0f;
            float target_vel = comp(tv, dim);
            float derr_rel = derr - target_vel;
            float lower = comp(lo, dim), upper = comp(hi, dim);
            if (e < lower) err = e - lower;
            else if (e > upper) err = e - upper;
            else {
                float target_pos = clampw(comp(tp, dim), lower, upper);
                if (comp(stiff, dim) > 0.0f) {
                    err = e - target_pos;
                    compliance = 1.0f / comp(stiff, dim);
                    damping = comp(damp, dim);
                } else if (comp(damp, dim) > 0.0f) {
                    compliance = 1.0f / comp(damp, dim);
                    damping = comp(damp, dim);
                }
            }
            if (std::fabs(err) > 1e-9f || std::fabs(derr_rel) > 1e-9f) {
                float dl = positional_correction(err, derr_rel, pose_p.q, pose_c.q, m_inv_p, m_inv_c, I_inv_p,
                                                 I_inv_c, lin_p, lin_c, ang_p, ang_c, 0.0f, compliance, damping, dt);
                ldp = add(ldp, mul(lin_p, dl * lin_relax));
                adp = add(adp, mul(ang_p, dl * ang_relax));
                ldc = add(ldc, mul(lin_c, dl * lin_relax));
                adc = add(adc, mul(ang_c, dl * ang_relax));
            }
        }
    }
    if (type == NB_JOINT_FIXED || type == NB_JOINT_PRISMATIC || type == NB_JOINT_REVOLUTE || type == NB_JOINT_D6) {
        Q4 q_p = X_wp.q, q_c = X_wc.q;
        if (qdot(q_p, q_c) < 0.0f) q_c = qscale(q_c, -1.0f);
        Q4 rq = qmul(qinv(q_p), q_c);
        Q4 qtwist = qnormalize(Q4{rq.x, 0.0f, 0.0f, rq.w});
        Q4 qswing = qmul(rq, qinv(qtwist));
        float s = std::sqrt(rq.x * rq.x + rq.w * rq.w);
        float invs = 1.0f / s;
        float invscube = invs * invs * invs;
        float err0 = 2.0f * nb_asin(clampw(qtwist.x, -1.0f, 1.0f));
        float err1 = qswing.y, err2 = qswing.z;
        Q4 g0{invs - rq.x * rq.x * invscube, 0.0f, 0.0f, -(rq.w * rq.x) * invscube};
        Q4 g1{-rq.w * (rq.w * rq.z + rq.x * rq.y) * invscube, rq.w * invs, -rq.x * invs,
              rq.x * (rq.w * rq.z + rq.x * rq.y) * invscube};
        Q4 g2{rq.w * (rq.w * rq.y - rq.x * rq.z) * invscube, rq.x * invs, rq.w * invs,
              rq.x * (rq.z * rq.x - rq.w * rq.y) * invscube};
        g0 = qscale(g0, 2.0f / std::fabs(qtwist.w));
        float swing_sq = qswing.w * qswing.w;
        if (swing_sq + 1.0e-4f < 1.0f) {
            float d = std::sqrt(1.0f - qswing.w * qswing.w);
            float theta = 2.0f * nb_acos(clampw(qswing.w, -1.0f, 1.0f));
            float scale = theta / d;
            err1 *= scale;
            err2 *= scale;
            g1 = qscale(g1, scale);
            g2 = qscale(g2, scale);
        }
        float errs[3] = {err0, err1, err2};
        Q4 grads[3] = {g0, g1, g2};
        V3 lo, hi, tp, stiff, tv, damp;
        joint_axes(m, axis_start + lin_count, ang_count, tpos, tvel, lo, hi, tp, stiff, tv, damp);
        for (int dim = 0; dim < 3; ++dim) {
            float e = errs[dim];
            Q4 grad = grads[dim];
            Q4 qc4 = qmul(qmul(qscale(q_p, 0.5f), grad), qinv(q_c));
            V3 ang_c{qc4.x, qc4.y, qc4.z};
            V3 ang_p = neg(ang_c);
            float derr = dot(ang_p, om_p) + dot(ang_c, om_c);
            float err = 0.0f, compliance = ang_comp, damping = 0.0f;
            float target_vel = comp(tv, dim);
            float acl = length(ang_c);
            float derr_rel = derr - target_vel * acl;
            float lower = comp(lo, dim), upper = comp(hi, dim);
            if (e < lower) err = e - lower;
            else if (e > upper) err = e - upper;
            else {
                float target_pos = clampw(comp(tp, dim), lower, upper);
                if (comp(stiff, dim) > 0.0f) {
                    err = e - target_pos;
                    compliance = 1.0f / comp(stiff, dim);
                    damping = comp(damp, dim);
                } else if (comp(damp, dim) > 0.0f) {
                    damping = comp(damp, dim);
                    compliance = 1.0f / comp(damp, dim);
                }
            }
            float dl = angular_correction(err, derr_rel, pose_p.q, pose_c.q, I_inv_p, I_inv_c, ang_p, ang_c, 0.0f,
                                          compliance, damping, dt) *
                       ang_relax;
            adp = add(adp, mul(ang_p, dl));
            adc = add(adc, mul(ang_c, dl));
        }
    }
    if (id_p >= 0) acc.add(lp, ldp, adp);
    if (id_c >= 0) acc.add(lc, ldc, adc);
    if (imp) {  // joint_impulse row of joint j (kernels.py:1941-1942)
        float* r = imp;
        r[0] = r[0] + ldc.x; r[1] = r[1] + ldc.y; r[2] = r[2] + ldc.z;
        r[3] = r[3] + adc.x; r[4] = r[4] + adc.y; r[5] = r[5] + adc.z;
    }
}

// apply_joint_forces (kernels.py:890-1003), sequential in joint order.
static void joint_forces(const NbModelDesc* m, int j0, int j1, const float* body_q, const float* joint_f,
                         std::vector<float>& body_f) {
    if (!joint_f) return;
    for (int j = j0; j < j1; ++j) {
        int type = m->joint_type[j];
        if (!m->joint_enabled[j]) continue;
        if (type == NB_JOINT_FIXED) continue;
        int id_c = m->joint_child[j], id_p = m->joint_parent[j];
        TF X_pj = load_tf(m->joint_X_p + 7 * j), X_cj = load_tf(m->joint_X_c + 7 * j);
        TF X_wp = X_pj, pose_p = X_pj;
        V3 com_p{0, 0, 0};
        if (id_p >= 0) {
            pose_p = load_tf(body_q + 7 * id_p);
            X_wp = tf_mul(pose_p, X_wp);
            com_p = load_v3(m->body_com + 3 * id_p);
        }
        V3 r_p = sub(X_wp.p, tf_point(pose_p, com_p));
        TF pose_c = load_tf(body_q + 7 * id_c);
        TF X_wc = tf_mul(pose_c, X_cj);
        V3 com_c = load_v3(m->body_com + 3 * id_c);
        V3 r_c = sub(X_wc.p, tf_point(pose_c, com_c));
        int qs = m->joint_qd_start[j];
        int lin = m->joint_dof_dim[2 * j], ang = m->joint_dof_dim[2 * j + 1];
        V3 t_total{0, 0, 0}, f_total{0, 0, 0};
        auto addw = [&](int b, V3 f, V3 t, float sgn) {
            float* bf = body_f.data() + 6 * (size_t)b;
            float v[6] = {f.x, f.y, f.z, t.x, t.y, t.z};
            for (int k = 0; k < 6; ++k) bf[k] = sgn > 0 ? bf[k] + v[k] : bf[k] - v[k];
        };
        if (type == NB_JOINT_FREE || type == NB_JOINT_DISTANCE) {
            f_total = V3{joint_f[qs + 0], joint_f[qs + 1], joint_f[qs + 2]};
            t_total = V3{joint_f[qs + 3], joint_f[qs + 4], joint_f[qs + 5]};
            addw(id_c, f_total, t_total, 1.0f);
            if (id_p >= 0) addw(id_p, f_total, t_total, -1.0f);
            continue;
        } else if (type == NB_JOINT_BALL) {
            t_total = V3{joint_f[qs + 0], joint_f[qs + 1], joint_f[qs + 2]};
        } else {
            for (int k = 0; k < lin && k < 3; ++k)
                f_total = add(f_total, smul(joint_f[qs + k], tf_vector(X_wp, load_v3(m->joint_axis + 3 * (qs + k)))));
            for (int k = 0; k < ang && k < 3; ++k)
                t_total = add(t_total, smul(joint_f[qs + lin + k],
                                            tf_vector(X_wp, load_v3(m->joint_axis + 3 * (qs + lin + k)))));
        }
        if (id_p >= 0) addw(id_p, f_total, add(t_total, cross(r_p, f_total)), -1.0f);
        addw(id_c, f_total, add(t_total, cross(r_c, f_total)), 1.0f);
    }
}

}  // namespace orc

namespace orc {

// velocity_at_point (newton/_src/math/spatial.py:54-80): v + w x r
static V3 velocity_at(V3 v, V3 w, V3 r) { return add(cross(w, r), v); }

// apply_rigid_restitution (kernels.py:2471-2620) for one contact.  Poses and
// twists from before the step (q_prev, qd_prev), current twists from the
// world state; velocity deltas go to `acc`.
static void restitution_contact(World& W, const ContactIn& c, const float* q_prev, const float* qd_prev, float dt,
                                Acc& acc) {
    const NbModelDesc* m = W.m;
    int sa = c.s0, sb = c.s1;
    if (sa == sb) return;
    int ba = -1, bb = -1;
    int nz = 0;
    float rest = 0.0f;
    if (sa >= 0) { nz += 1; rest += m->shape_restitution[sa]; ba = m->shape_body[sa]; }
    if (sb >= 0) { nz += 1; rest += m->shape_restitution[sb]; bb = m->shape_body[sb]; }
    if (nz > 0) rest /= (float)nz;
    if (ba == bb) return;
    int la = W.local(ba), lb = W.local(bb);
    float m_inv_a = 0.0f, m_inv_b = 0.0f;
    M33 Ia = zero_m33(), Ib = zero_m33();
    TF Xa = tf_identity(), Xb = tf_identity();
    V3 com_a{0, 0, 0}, com_b{0, 0, 0};
    V3 v_a{0, 0, 0}, v_b{0, 0, 0}, v_a_new{0, 0, 0}, v_b_new{0, 0, 0};
    float inv_mass = 0.0f;
    if (ba >= 0) { Xa = load_tf(q_prev + 7 * (size_t)ba); m_inv_a = W.inv_m[la]; Ia = W.invI[la]; com_a = W.com[la]; }
    if (bb >= 0) { Xb = load_tf(q_prev + 7 * (size_t)bb); m_inv_b = W.inv_m[lb]; Ib = W.invI[lb]; com_b = W.com[lb]; }
    V3 bx_a = tf_point(Xa, add(c.p0, c.o0));
    V3 bx_b = tf_point(Xb, add(c.p1, c.o1));
    float thickness = c.m0 + c.m1;
    V3 n = c.n;
    float d = dot(n, sub(bx_b, bx_a)) - thickness;
    if (d >= 0.0f) return;
    V3 r_a = sub(bx_a, tf_point(Xa, com_a));
    V3 r_b = sub(bx_b, tf_point(Xb, com_b));
    V3 rxn_a{0, 0, 0}, rxn_b{0, 0, 0};
    if (ba >= 0) {
        int wi = m->body_world[ba];
        V3 g = load_v3(m->gravity + 3 * (size_t)(wi > 0 ? wi : 0));
        const float* qd = qd_prev + 6 * (size_t)ba;
        v_a = add(velocity_at(V3{qd[0], qd[1], qd[2]}, V3{qd[3], qd[4], qd[5]}, r_a), mul(g, dt));
        v_a_new = velocity_at(W.st[la].v, W.st[la].w, r_a);
        rxn_a = qrot_inv(Xa.q, cross(r_a, n));
        inv_mass += m_inv_a + dot(rxn_a, mv(Ia, rxn_a));
    }
    if (bb >= 0) {
        int wi = m->body_world[bb];
        V3 g = load_v3(m->gravity + 3 * (size_t)(wi > 0 ? wi : 0));
        const float* qd = qd_prev + 6 * (size_t)bb;
        v_b = add(velocity_at(V3{qd[0], qd[1], qd[2]}, V3{qd[3], qd[4], qd[5]}, r_b), mul(g, dt));
        v_b_new = velocity_at(W.st[lb].v, W.st[lb].w, r_b);
        rxn_b = qrot_inv(Xb.q, cross(r_b, n));
        inv_mass += m_inv_b + dot(rxn_b, mv(Ib, rxn_b));
    }
    if (inv_mass == 0.0f) return;
    float rel_old = dot(n, sub(v_b, v_a));
    float rel_new = dot(n, sub(v_b_new, v_a_new));
    if (rel_old >= 0.0f) return;
    float dv = (-rel_new - rest * rel_old) / inv_mass;
    if (ba >= 0) {
        float dva = -dv;
        V3 dq = qrot(Xa.q, mul(mv(Ia, rxn_a), dva));
        acc.add(la, mul(mul(n, m_inv_a), dva), dq);
    }
    if (bb >= 0) {
        float dvb = dv;
        V3 dq = qrot(Xb.q, mul(mv(Ib, rxn_b), dvb));
        acc.add(lb, mul(mul(n, m_inv_b), dvb), dq);
    }
}

}  // namespace orc

using namespace orc;

extern "C" {

// One SolverXPBD.step over all worlds (host pointers).  seg == NULL means no
// contacts.  `acc_mode` selects ORC_ACC_FIXED (0) or ORC_ACC_FLOAT (1).
// `status` receives NB_STATUS_* bits.
// the shared asin / acos (for the accuracy test)
float orc_asin(float x) { return nb_asin(x); }
float orc_acos(float x) { return nb_acos(x); }

int orc_step(const NbModelDesc* m, const NbXpbdParams* p, const NbStepIO* io, const OrcSeg* seg, float dt,
             int acc_mode, uint32_t* status) {
    int B = m->body_count;
    std::vector<float> body_f(io->body_f_in, io->body_f_in + 6 * (size_t)B);
    joint_forces(m, 0, m->joint_count, io->body_q_in, io->joint_f, body_f);
    uint32_t st_all = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : st_all)
    for (int w = 0; w < m->world_count; ++w) {
        uint32_t st = 0;
        World W;
        W.m = m;
        W.b0 = m->world_body_start[w];
        W.nb = m->world_body_start[w + 1] - W.b0;
        W.st.resize(W.nb);
        W.I.resize(W.nb);
        W.invI.resize(W.nb);
        W.inv_m.resize(W.nb);
        W.com.resize(W.nb);
        W.flags.resize(W.nb);
        for (int i = 0; i < W.nb; ++i) {
            int b = W.b0 + i;
            W.flags[i] = m->body_flags[b];
            bool kin = (W.flags[i] & NB_BODY_KINEMATIC) != 0;
            W.inv_m[i] = kin ? 0.0f : m->body_inv_mass[b];
            W.invI[i] = kin ? zero_m33() : load_m33(m->body_inv_inertia + 9 * (size_t)b);
            W.I[i] = load_m33(m->body_inertia + 9 * (size_t)b);
            W.com[i] = load_v3(m->body_com + 3 * (size_t)b);
            // integrate_bodies (solver.py:97-157)
            BodyState s;
            s.q = load_tf(io->body_q_in + 7 * (size_t)b);
            const float* qd = io->body_qd_in + 6 * (size_t)b;
            s.v = V3{qd[0], qd[1], qd[2]};
            s.w = V3{qd[3], qd[4], qd[5]};
            if (!kin) {
                const float* f = body_f.data() + 6 * (size_t)b;
                int wi = m->body_world[b];
                if (wi < 0) wi = 0;
                V3 g = load_v3(m->gravity + 3 * (size_t)wi);
                integrate_rigid_body(s, V3{f[0], f[1], f[2]}, V3{f[3], f[4], f[5]}, W.com[i], W.I[i],
                                     m->body_inv_mass[b], load_m33(m->body_inv_inertia + 9 * (size_t)b), g,
                                     p->angular_damping, dt);
            }
            W.st[i] = s;
        }
        Acc acc;
        acc.mode = acc_mode;
        acc.status = &st;
        int64_t c0 = 0;
        int nc = 0;
        if (seg) {
            c0 = 5 * (int64_t)m->world_pair_start[w];
            nc = seg->world_count[w];
        }
        int j0 = m->world_joint_start[w], j1 = m->world_joint_start[w + 1];
        std::vector<float> jimp(io->body_parent_f ? 6 * (size_t)(j1 - j0) : 0, 0.0f);
        for (int it = 0; it < p->iterations; ++it) {
            if (seg) {
                acc.reset(W.nb);
                for (int c = 0; c < nc; ++c) {
                    ContactIn ci = load_contact(seg, c0 + c);
                    float imp[6];
                    bool active = solve_contact(W, ci, io->body_qd_in, p->rigid_contact_relaxation, dt, acc,
                                                p->rigid_contact_con_weighting != 0,
                                                io->contact_impulse ? imp : nullptr);
                    (void)active;
                    if (io->contact_impulse && active) {
                        // accumulate_weighted_contact_impulse needs the final counts:
                        // deferred below (second pass) to keep the weights complete.
                    }
                }
                if (io->contact_impulse) {
                    // kernels.py:2301-2360 -- weights use this iteration's counts.
                    for (int c = 0; c < nc; ++c) {
                        ContactIn ci = load_contact(seg, c0 + c);
                        Acc dummy;
                        dummy.mode = acc_mode;
                        dummy.status = &st;
                        dummy.reset(W.nb);
                        float imp[6];
                        if (!solve_contact(W, ci, io->body_qd_in, p->rigid_contact_relaxation, dt, dummy, false, imp))
                            continue;
                        float weight = 1.0f;
                        if (p->rigid_contact_con_weighting) {
                            float na = 0.0f, nb2 = 0.0f;
                            int ba = ci.s0 >= 0 ? m->shape_body[ci.s0] : -1;
                            int bb = ci.s1 >= 0 ? m->shape_body[ci.s1] : -1;
                            if (ba >= 0) na = acc.cnt[W.local(ba)];
                            if (bb >= 0) nb2 = acc.cnt[W.local(bb)];
                            float ns = na + nb2;
                            if (ns > 0.0f) {
                                if (na == 0.0f) weight = 1.0f / nb2;
                                else if (nb2 == 0.0f) weight = 1.0f / na;
                                else weight = 2.0f / ns;
                            }
                        }
                        float* ci6 = io->contact_impulse + 6 * (size_t)(c0 + c);
                        for (int k = 0; k < 6; ++k) ci6[k] = ci6[k] + imp[k] * weight;
                    }
                }
                for (int i = 0; i < W.nb; ++i) {
                    V3 dl, da;
                    acc.get(i, dl, da);
                    float weight = 1.0f;
                    if (p->rigid_contact_con_weighting) {
                        float iw = acc.cnt[i];
                        if (iw > 0.0f) weight = 1.0f / iw;
                    }
                    apply_body_delta(W.st[i], dl, da, weight, W.com[i], W.I[i], W.inv_m[i], W.invI[i], dt);
                }
            }
            if (m->joint_count > 0) {
                acc.reset(W.nb);
                for (int j = j0; j < j1; ++j)
                    solve_joint(W, j, io->joint_target_pos, io->joint_target_vel, p, dt, acc,
                                io->body_parent_f ? jimp.data() + 6 * (size_t)(j - j0) : nullptr);
                for (int i = 0; i < W.nb; ++i) {
                    V3 dl, da;
                    acc.get(i, dl, da);
                    apply_body_delta(W.st[i], dl, da, 1.0f, W.com[i], W.I[i], W.inv_m[i], W.invI[i], dt);
                }
            }
        }
        if (seg && p->enable_restitution) {
            // solver_xpbd.py:685-755: after the iterations, from the pre-step state
            acc.reset(W.nb);
            for (int c = 0; c < nc; ++c)
                restitution_contact(W, load_contact(seg, c0 + c), io->body_q_in, io->body_qd_in, dt, acc);
            for (int i = 0; i < W.nb; ++i) {
                V3 dl, da;
                acc.get(i, dl, da);
                W.st[i].v = add(W.st[i].v, dl);
                W.st[i].w = add(W.st[i].w, da);
            }
        }
        if (io->body_parent_f) {
            // solver_xpbd.py:636-655 with convert_joint_impulse_to_parent_f (kernels.py:2396-2436)
            for (int i = 0; i < W.nb; ++i)
                for (int k = 0; k < 6; ++k) io->body_parent_f[6 * (size_t)(W.b0 + i) + k] = 0.0f;
            const float inv_dt = 1.0f / dt;
            for (int j = j0; j < j1; ++j) {
                const int c = m->joint_child[j];
                if (!m->joint_enabled[j] || m->joint_type[j] == NB_JOINT_FREE || c < 0) continue;
                for (int k = 0; k < 6; ++k)
                    io->body_parent_f[6 * (size_t)c + k] = jimp[6 * (size_t)(j - j0) + k] * inv_dt;
            }
        }
        for (int i = 0; i < W.nb; ++i) {
            int b = W.b0 + i;
            if (W.flags[i] & NB_BODY_KINEMATIC) {
                std::memcpy(io->body_q_out + 7 * (size_t)b, io->body_q_in + 7 * (size_t)b, 7 * sizeof(float));
                std::memcpy(io->body_qd_out + 6 * (size_t)b, io->body_qd_in + 6 * (size_t)b, 6 * sizeof(float));
                continue;
            }
            store_tf(io->body_q_out + 7 * (size_t)b, W.st[i].q);
            float* qd = io->body_qd_out + 6 * (size_t)b;
            qd[0] = W.st[i].v.x; qd[1] = W.st[i].v.y; qd[2] = W.st[i].v.z;
            qd[3] = W.st[i].w.x; qd[4] = W.st[i].w.y; qd[5] = W.st[i].w.z;
            for (int k = 0; k < 7; ++k)
                if (!std::isfinite(io->body_q_out[7 * (size_t)b + k])) st |= NB_STATUS_NONFINITE;
        }
        st_all |= st;
    }
    if (status) *status |= st_all;
    return 0;
}

}  // extern "C"
