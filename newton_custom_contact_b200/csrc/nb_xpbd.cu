// One XPBD substep for many independent worlds.
//
// Worlds are processed by thread groups of G threads (G = 32: one warp per
// world, up to G = 256: one CTA per world for scenes with few, large worlds).
// A host-side scheduler packs worlds of similar size into batches that share
// one CTA's shared-memory arena; each world's body poses, twists and mass
// properties live in its own slab for the whole substep, so the `iterations`
// constraint-projection passes never touch HBM for body state (the reference
// re-reads body arrays in ~7 launches per iteration,
// newton/_src/solvers/xpbd/solver_xpbd.py:371-630).  Per iteration:
//   contacts: the group tests the world's dense contact records in order,
//             compacts the penetrating ones in order and solves them
//             (solve_body_contact_positions, newton/_src/solvers/xpbd/kernels.py:2062-2298);
//             each body's delta is the float sum of its contacts' deltas in
//             contact order (nb_ordered.cuh) -- the reference's sum run
//             sequentially, deterministic on the GPU;
//   bodies:   weighted apply_body_deltas (kernels.py:809-878), then the joint
//             pass (solve_body_joints, kernels.py:1441-1942, summed in joint
//             order the same way) and the unweighted apply of
//             solver_xpbd.py:590-630.
// Group barriers are __syncwarp (G = 32), named barriers (G = 64, 128) or
// __syncthreads (G = 256).
#include <cuda_runtime.h>

#include "nb_kernels.cuh"
#include "nb_math.cuh"
#include "nb_ordered.cuh"

namespace {

constexpr int kST = NB_STEP_THREADS;  // threads per CTA

// entries of one ordered batch per group: at least one test round of G items,
// sized so that 8 warp groups' batches (21.5 KB) leave room for two CTAs' arenas per SM
template <int G>
struct BatchCap {
    static constexpr int value = G == 32 ? 48 : (G == 256 ? 256 : 128);
};
template <int G>
using Batch = nb::OrderedBatch<BatchCap<G>::value>;

// Per-world body state in shared memory.  kCompact = false: everything the
// substep touches is staged (43 words per body); kCompact = true: only the
// mutable part (pose, twist, delta accumulators, flags, contact count: 21
// words per body) is staged and the static mass properties are read from the
// model (read-only path), so worlds of up to 128 bodies fit one warp's share
// of the arena.
template <bool kCompact>
struct SBodiesT {
    static constexpr bool compact = kCompact;
    int nb;                    // bodies of this world (also the SoA stride)
    int b0;                    // global index of the world's first body
    float* f;                  // [13][nb] pose (7) + twist (6)
    float* c;                  // [4][nb]  com (3), effective inv mass          (full layout)
    float* I;                  // [9][nb]                                         (full layout)
    float* iI;                 // [9][nb]  effective inverse inertia              (full layout)
    const float4* g_pack;      // NbModelDesc.body_pack, 6 float4 per body        (compact layout)
    float* frc;                // [6][nb]  body_f + joint forces (aliases acc before integration)
    int* flags;                // [nb]
    float* acc;                // [6][nb]  delta accumulators (linear 3, angular 3)
    int* cnt;                  // [nb]     active contacts of the iteration

    __device__ TF q(int i) const {
        return TF{V3{f[0 * nb + i], f[1 * nb + i], f[2 * nb + i]},
                  Q4{f[3 * nb + i], f[4 * nb + i], f[5 * nb + i], f[6 * nb + i]}};
    }
    __device__ V3 v(int i) const { return V3{f[7 * nb + i], f[8 * nb + i], f[9 * nb + i]}; }
    __device__ V3 w(int i) const { return V3{f[10 * nb + i], f[11 * nb + i], f[12 * nb + i]}; }
    __device__ void set(int i, TF t, V3 lv, V3 aw) {
        f[0 * nb + i] = t.p.x; f[1 * nb + i] = t.p.y; f[2 * nb + i] = t.p.z;
        f[3 * nb + i] = t.q.x; f[4 * nb + i] = t.q.y; f[5 * nb + i] = t.q.z; f[6 * nb + i] = t.q.w;
        f[7 * nb + i] = lv.x; f[8 * nb + i] = lv.y; f[9 * nb + i] = lv.z;
        f[10 * nb + i] = aw.x; f[11 * nb + i] = aw.y; f[12 * nb + i] = aw.z;
    }
    __device__ bool kinematic(int i) const { return (flags[i] & NB_BODY_KINEMATIC) != 0; }
    // compact layout: body i's packed mass properties, floats 0..23 in 6 float4 (read-only path)
    __device__ const float4* pack(int i) const { return g_pack + 6 * (size_t)(b0 + i); }
    __device__ V3 com(int i) const {
        if constexpr (kCompact) {
            const float4 a = __ldg(pack(i));
            return V3{a.x, a.y, a.z};
        } else {
            return V3{c[i], c[nb + i], c[2 * nb + i]};
        }
    }
    __device__ float inv_m(int i) const {
        if constexpr (kCompact) return __ldg(pack(i)).w;
        else return c[3 * nb + i];
    }
    __device__ M33 inertia(int i) const {
        M33 r;
        if constexpr (kCompact) {
            // floats 4..12
            const float4 a = __ldg(pack(i) + 1), b = __ldg(pack(i) + 2), c3 = __ldg(pack(i) + 3);
            r.m[0][0] = a.x; r.m[0][1] = a.y; r.m[0][2] = a.z;
            r.m[1][0] = a.w; r.m[1][1] = b.x; r.m[1][2] = b.y;
            r.m[2][0] = b.z; r.m[2][1] = b.w; r.m[2][2] = c3.x;
        } else {
#pragma unroll
            for (int k = 0; k < 9; ++k) r.m[k / 3][k % 3] = I[k * nb + i];
        }
        return r;
    }
    __device__ M33 inv_inertia(int i) const {
        M33 r;
        if constexpr (kCompact) {
            // floats 13..21
            const float4 a = __ldg(pack(i) + 3), b = __ldg(pack(i) + 4), c5 = __ldg(pack(i) + 5);
            r.m[0][0] = a.y; r.m[0][1] = a.z; r.m[0][2] = a.w;
            r.m[1][0] = b.x; r.m[1][1] = b.y; r.m[1][2] = b.z;
            r.m[2][0] = b.w; r.m[2][1] = c5.x; r.m[2][2] = c5.y;
        } else {
#pragma unroll
            for (int k = 0; k < 9; ++k) r.m[k / 3][k % 3] = iI[k * nb + i];
        }
        return r;
    }
    // the reference's atomic_add(deltas, i, spatial_vector(lin, ang)): old + value, per component
    // (only body i's owner thread of the ordered pass calls this)
    __device__ __forceinline__ void add(int i, const float* d6) {
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k * nb + i] = acc[k * nb + i] + d6[k];
    }
    // read and clear the accumulated delta of body i; false when nothing was added
    __device__ bool take(int i, V3& lin, V3& ang) {
        float v[6];
        unsigned any = 0u;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            v[k] = acc[k * nb + i];
            any |= __float_as_uint(v[k]);
            acc[k * nb + i] = 0.0f;
        }
        lin = V3{v[0], v[1], v[2]};
        ang = V3{v[3], v[4], v[5]};
        return any != 0u;
    }
};

// 4-byte words of one world's slab: acc 6, f 13, [c 4, I 9, iI 9,] flags 1, cnt 1
template <bool kCompact>
__host__ __device__ constexpr int slab_words_per_body() { return kCompact ? 6 + 13 + 1 + 1 : 6 + 13 + 4 + 9 + 9 + 1 + 1; }

template <bool kCompact>
__device__ SBodiesT<kCompact> sbodies_carve(unsigned char* slab, const NbModelDesc& m, int b0, int nb) {
    SBodiesT<kCompact> s;
    s.nb = nb;
    s.b0 = b0;
    float* a = reinterpret_cast<float*>(slab);
    s.acc = a;
    s.frc = a;  // used only before integration
    float* fl = a + 6 * (size_t)nb;
    s.f = fl;
    s.g_pack = reinterpret_cast<const float4*>(m.body_pack);
    float* after;
    if constexpr (kCompact) {
        s.c = s.I = s.iI = nullptr;
        after = s.f + 13 * nb;
    } else {
        s.c = fl + 13 * nb;
        s.I = s.c + 4 * nb;
        s.iI = s.I + 9 * nb;
        after = s.iI + 9 * nb;
    }
    int* ip = reinterpret_cast<int*>(after);
    s.flags = ip;
    s.cnt = ip + nb;
    return s;
}

template <int G>
__device__ __forceinline__ void group_sync(int g) {
    if constexpr (G == 32) {
        __syncwarp();
    } else if constexpr (G == kST) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(G) : "memory");
    }
}

// solver.py:50-94
__device__ void integrate_rigid_body(TF& q, V3& v, V3& w, V3 f0, V3 t0, V3 com, const M33& I, float inv_mass,
                                     const M33& inv_I, V3 g, float angular_damping, float dt) {
    V3 x0 = q.p;
    Q4 r0 = q.q;
    V3 w0 = w, v0 = v;
    V3 x_com = add(x0, qrot(r0, com));
    float nz = inv_mass != 0.0f ? 1.0f : 0.0f;
    V3 v1 = add(v0, mul(add(mul(f0, inv_mass), mul(g, nz)), dt));
    V3 x1 = add(x_com, mul(v1, dt));
    V3 wb = qrot_inv(r0, w0);
    V3 tb = sub(qrot_inv(r0, t0), cross(wb, mv(I, wb)));
    V3 w1 = qrot(r0, add(wb, mul(mv(inv_I, tb), dt)));
    Q4 r1 = qnormalize(qadd(r0, qscale(qscale(qmul(Q4{w1.x, w1.y, w1.z, 0.0f}, r0), 0.5f), dt)));
    w1 = mul(w1, 1.0f - angular_damping * dt);
    q = TF{sub(x1, qrot(r1, com)), r1};
    v = v1;
    w = w1;
}

// kernels.py:809-878 with the weight already resolved
__device__ void apply_body_delta(TF& q, V3& v, V3& w, V3 dlin, V3 dang, float weight, V3 com, const M33& I,
                                 float inv_m, const M33& inv_I, float dt) {
    if (inv_m == 0.0f) return;
    V3 v0 = v, w0 = w;
    V3 p0 = q.p;
    Q4 q0 = q.q;
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
    q = TF{p1, q1};
    V3 v1 = add(v0, dp);
    V3 w1 = add(w0, dw1);
    if (length(v1) < 1e-4f) v1 = V3{0.0f, 0.0f, 0.0f};
    if (length(w1) < 1e-4f) w1 = V3{0.0f, 0.0f, 0.0f};
    v = v1;
    w = w1;
}

// apply_body_delta with a zero delta and weight 1 (the apply the joint pass runs after a world whose
// joints are all free), bit for bit.  With a zero delta and finite inertia the angular terms are signed
// zeros, and adding a signed zero changes no nonzero value: when every quaternion component is nonzero
// and finite, no angular velocity component is -0 (the only value a signed zero can flip) or
// non-finite, and the inertia and inverse inertia are finite, the result is the renormalised
// quaternion, the position re-expressed about the com, the velocities with +0 added and the rest
// thresholds -- the inertia terms are skipped.  Otherwise the general form runs.
__device__ void apply_zero_delta(TF& q, V3& v, V3& w, V3 com, const M33& I, float inv_m, const M33& inv_I,
                                 float dt) {
    if (inv_m == 0.0f) return;
    const Q4 q0 = q.q;
    const bool q_ok = q0.x != 0.0f && q0.y != 0.0f && q0.z != 0.0f && q0.w != 0.0f && isfinite(q0.x) &&
                      isfinite(q0.y) && isfinite(q0.z) && isfinite(q0.w);
    const bool w_ok = isfinite(w.x) && isfinite(w.y) && isfinite(w.z) && !(w.x == 0.0f && signbit(w.x)) &&
                      !(w.y == 0.0f && signbit(w.y)) && !(w.z == 0.0f && signbit(w.z));
    // x * 0 is 0 for every finite x and NaN otherwise
    float inert = 0.0f;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) inert += I.m[r][c] * 0.0f + inv_I.m[r][c] * 0.0f;
    const V3 zero{0.0f, 0.0f, 0.0f};
    if (!(q_ok && w_ok && inert == 0.0f)) {
        apply_body_delta(q, v, w, zero, zero, 1.0f, com, I, inv_m, inv_I, dt);
        return;
    }
    const V3 dp = mul(zero, inv_m * 1.0f);  // +0: the general form's dp
    const Q4 q1 = qnormalize(q0);
    V3 p1 = add(add(q.p, qrot(q0, com)), mul(dp, dt));
    p1 = sub(p1, qrot(q1, com));
    q = TF{p1, q1};
    V3 v1 = add(v, dp);
    V3 w1 = w;
    if (length(v1) < 1e-4f) v1 = zero;
    if (length(w1) < 1e-4f) w1 = zero;
    v = v1;
    w = w1;
}

// kernels.py:1945-1979
__device__ float contact_constraint_delta(float err, Q4 qa, Q4 qb, float m_inv_a, float m_inv_b, const M33& Ia,
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
__device__ float positional_correction(float err, float derr, Q4 qa, Q4 qb, float m_inv_a, float m_inv_b,
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
__device__ float angular_correction(float err, float derr, Q4 qa, Q4 qb, const M33& Ia, const M33& Ib, V3 aa, V3 ab,
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

// Penetration depth of one solver record (the first test of
// solve_body_contact_positions, kernels.py:2100-2130); reads 48 bytes.
template <class SB>
__device__ __forceinline__ float contact_depth(const SB& S, float4 r0, float4 r1, float4 r2, int la, int lb,
                                               TF& Xa, TF& Xb, V3& bx_a, V3& bx_b) {
    Xa = la >= 0 ? S.q(la) : tf_identity();
    Xb = lb >= 0 ? S.q(lb) : tf_identity();
    bx_a = tf_point(Xa, V3{r0.x, r0.y, r0.z});
    bx_b = tf_point(Xb, V3{r1.x, r1.y, r1.z});
    const float thickness = r0.w + r1.w;
    return dot(V3{r2.x, r2.y, r2.z}, sub(bx_b, bx_a)) - thickness;
}

// true when the reference's solve_body_contact_positions adds deltas for this
// record: distinct bodies (equal shapes imply equal bodies) and depth < 0 (NaN
// depths count, so they propagate exactly as in the reference); ends receives
// the two world-local bodies for the ordered accumulation
template <class SB>
__device__ __forceinline__ bool contact_active(const SB& S, float4 r0, float4 r1, float4 r2, int& ends) {
    const int tag = __float_as_int(r2.w);
    const int la = (tag & 0xFFF) - 1, lb = ((tag >> 12) & 0xFFF) - 1;
    if (la == lb) return false;
    TF Xa, Xb;
    V3 bx_a, bx_b;
    ends = nb::ends_pack(la, lb);
    return !(contact_depth(S, r0, r1, r2, la, lb, Xa, Xb, bx_a, bx_b) >= 0.0f);
}

// solve_body_contact_positions for one active contact (kernels.py:2062-2298):
// d12 receives the deltas the reference adds to body A (linear, angular) and
// body B; imp (optional) the A-side spatial delta (the contact_impulse_iter
// entry of the reference).  The caller has established that the contact is
// active (contact_active: distinct bodies, depth < 0 or NaN; equal shapes
// imply equal bodies).
template <class SB>
__device__ void solve_contact(const NbModelDesc& m, const SB& S, float4 r0, float4 r1, float4 r2, float4 r3,
                              float4 r4, float relaxation, float dt, float* d12, float* imp) {
    const int sa = __float_as_int(r3.w), sb = __float_as_int(r4.w);
    const int tag = __float_as_int(r2.w);
    const int la = (tag & 0xFFF) - 1, lb = ((tag >> 12) & 0xFFF) - 1;
    TF Xa, Xb;
    V3 bx_a, bx_b;
    const float d = contact_depth(S, r0, r1, r2, la, lb, Xa, Xb, bx_a, bx_b);
    const V3 n{r2.x, r2.y, r2.z};
    float m_inv_a = 0.0f, m_inv_b = 0.0f;
    M33 Ia = zero_m33(), Ib = zero_m33();
    V3 com_a{0, 0, 0}, com_b{0, 0, 0};
    V3 om_a{0, 0, 0}, om_b{0, 0, 0};
    V3 off_a{r3.x, r3.y, r3.z}, off_b{r4.x, r4.y, r4.z};
    if (la >= 0) { com_a = S.com(la); m_inv_a = S.inv_m(la); Ia = S.inv_inertia(la); om_a = S.w(la); }
    if (lb >= 0) { com_b = S.com(lb); m_inv_b = S.inv_m(lb); Ib = S.inv_inertia(lb); om_b = S.w(lb); }
    int nz = 0;
    float mu = 0.0f, mut = 0.0f, mur = 0.0f;
    if (sa >= 0) { nz += 1; mu += __ldg(m.shape_mu + sa); mut += __ldg(m.shape_mu_torsional + sa); mur += __ldg(m.shape_mu_rolling + sa); }
    if (sb >= 0) { nz += 1; mu += __ldg(m.shape_mu + sb); mut += __ldg(m.shape_mu_torsional + sb); mur += __ldg(m.shape_mu_rolling + sb); }
    if (nz > 0) { mu /= (float)nz; mut /= (float)nz; mur /= (float)nz; }
    V3 r_a = sub(bx_a, tf_point(Xa, com_a));
    V3 r_b = sub(bx_b, tf_point(Xb, com_b));
    V3 ang_a = neg(cross(r_a, n));
    V3 ang_b = cross(r_b, n);
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
        if (la >= 0 && (S.flags[la] & NB_BODY_KINEMATIC)) {
            V3 va = add(cross(S.w(la), r_a), S.v(la));
            rvk = sub(rvk, sub(va, smul(dot(n, va), n)));
        }
        if (lb >= 0 && (S.flags[lb] & NB_BODY_KINEMATIC)) {
            V3 vb = add(cross(S.w(lb), r_b), S.v(lb));
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
        if (fabsf(err) > 0.0f) {
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
    d12[0] = lin_da.x; d12[1] = lin_da.y; d12[2] = lin_da.z;
    d12[3] = ang_da.x; d12[4] = ang_da.y; d12[5] = ang_da.z;
    d12[6] = lin_db.x; d12[7] = lin_db.y; d12[8] = lin_db.z;
    d12[9] = ang_db.x; d12[10] = ang_db.y; d12[11] = ang_db.z;
    if (imp) {
        imp[0] = lin_da.x; imp[1] = lin_da.y; imp[2] = lin_da.z;
        imp[3] = ang_da.x; imp[4] = ang_da.y; imp[5] = ang_da.z;
    }
}

// velocity_at_point (newton/_src/math/spatial.py:54-80): v + w x r
__device__ __forceinline__ V3 velocity_at(V3 v, V3 w, V3 r) { return add(cross(w, r), v); }

// apply_rigid_restitution (kernels.py:2471-2620) for one solver record:
// pre-step poses / twists from the step's inputs, current twists from the
// slab.  Returns whether the reference adds velocity deltas for the record;
// if so, d12 receives them (body A linear, angular; body B linear, angular)
// and ends the two bodies.
template <class SB>
__device__ __noinline__ bool restitution_contact(const NbModelDesc& m, const SB& S, const float4* r, int b0,
                                                 const float* __restrict__ q_prev, const float* __restrict__ qd_prev,
                                                 float dt, float* d12, int& ends) {
    const float4 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4];
    const int sa = __float_as_int(r3.w), sb = __float_as_int(r4.w);
    if (sa == sb) return false;
    int nz = 0;
    float rest = 0.0f;
    if (sa >= 0) { nz += 1; rest += __ldg(m.shape_restitution + sa); }
    if (sb >= 0) { nz += 1; rest += __ldg(m.shape_restitution + sb); }
    if (nz > 0) rest /= (float)nz;
    const int tag = __float_as_int(r2.w);
    const int la = (tag & 0xFFF) - 1, lb = ((tag >> 12) & 0xFFF) - 1;
    if (la == lb) return false;
    float m_inv_a = 0.0f, m_inv_b = 0.0f;
    M33 Ia = zero_m33(), Ib = zero_m33();
    TF Xa = tf_identity(), Xb = tf_identity();
    V3 com_a{0, 0, 0}, com_b{0, 0, 0};
    V3 v_a{0, 0, 0}, v_b{0, 0, 0}, v_a_new{0, 0, 0}, v_b_new{0, 0, 0};
    float inv_mass = 0.0f;
    if (la >= 0) { Xa = load_tf(q_prev + 7 * (size_t)(b0 + la)); m_inv_a = S.inv_m(la); Ia = S.inv_inertia(la); com_a = S.com(la); }
    if (lb >= 0) { Xb = load_tf(q_prev + 7 * (size_t)(b0 + lb)); m_inv_b = S.inv_m(lb); Ib = S.inv_inertia(lb); com_b = S.com(lb); }
    const V3 n{r2.x, r2.y, r2.z};
    V3 bx_a = tf_point(Xa, add(V3{r0.x, r0.y, r0.z}, V3{r3.x, r3.y, r3.z}));
    V3 bx_b = tf_point(Xb, add(V3{r1.x, r1.y, r1.z}, V3{r4.x, r4.y, r4.z}));
    const float thickness = r0.w + r1.w;
    const float d = dot(n, sub(bx_b, bx_a)) - thickness;
    if (d >= 0.0f) return false;
    V3 r_a = sub(bx_a, tf_point(Xa, com_a));
    V3 r_b = sub(bx_b, tf_point(Xb, com_b));
    V3 rxn_a{0, 0, 0}, rxn_b{0, 0, 0};
    if (la >= 0) {
        const int wi = m.body_world[b0 + la];
        const V3 g = load_v3(m.gravity + 3 * (size_t)(wi > 0 ? wi : 0));
        const float* qd = qd_prev + 6 * (size_t)(b0 + la);
        v_a = add(velocity_at(V3{qd[0], qd[1], qd[2]}, V3{qd[3], qd[4], qd[5]}, r_a), mul(g, dt));
        v_a_new = velocity_at(S.v(la), S.w(la), r_a);
        rxn_a = qrot_inv(Xa.q, cross(r_a, n));
        inv_mass += m_inv_a + dot(rxn_a, mv(Ia, rxn_a));
    }
    if (lb >= 0) {
        const int wi = m.body_world[b0 + lb];
        const V3 g = load_v3(m.gravity + 3 * (size_t)(wi > 0 ? wi : 0));
        const float* qd = qd_prev + 6 * (size_t)(b0 + lb);
        v_b = add(velocity_at(V3{qd[0], qd[1], qd[2]}, V3{qd[3], qd[4], qd[5]}, r_b), mul(g, dt));
        v_b_new = velocity_at(S.v(lb), S.w(lb), r_b);
        rxn_b = qrot_inv(Xb.q, cross(r_b, n));
        inv_mass += m_inv_b + dot(rxn_b, mv(Ib, rxn_b));
    }
    if (inv_mass == 0.0f) return false;
    const float rel_old = dot(n, sub(v_b, v_a));
    const float rel_new = dot(n, sub(v_b_new, v_a_new));
    if (rel_old >= 0.0f) return false;
    const float dv = (-rel_new - rest * rel_old) / inv_mass;
    V3 la_v{0, 0, 0}, aa_v{0, 0, 0}, lb_v{0, 0, 0}, ab_v{0, 0, 0};
    if (la >= 0) {
        const float dva = -dv;
        la_v = mul(mul(n, m_inv_a), dva);
        aa_v = qrot(Xa.q, mul(mv(Ia, rxn_a), dva));
    }
    if (lb >= 0) {
        const float dvb = dv;
        lb_v = mul(mul(n, m_inv_b), dvb);
        ab_v = qrot(Xb.q, mul(mv(Ib, rxn_b), dvb));
    }
    d12[0] = la_v.x; d12[1] = la_v.y; d12[2] = la_v.z; d12[3] = aa_v.x; d12[4] = aa_v.y; d12[5] = aa_v.z;
    d12[6] = lb_v.x; d12[7] = lb_v.y; d12[8] = lb_v.z; d12[9] = ab_v.x; d12[10] = ab_v.y; d12[11] = ab_v.z;
    ends = nb::ends_pack(la, lb);
    return true;
}

// accumulate_weighted_contact_impulse (kernels.py:2301-2360) for the world's
// records: raw iteration impulses from the scratch (all zero for contacts
// that were not active), weighted by this iteration's body contact counts,
// added to the public contact's row; the scratch is cleared again.
template <int G, class SB>
__device__ __forceinline__ void accumulate_impulses(const SB& S, const float4* __restrict__ R, int nc,
                                                    int64_t rec_base, const int32_t* __restrict__ rec_index,
                                                    float* __restrict__ scratch, float* __restrict__ out, int cap,
                                                    bool weighting, int t) {
    for (int k = t; k < nc; k += G) {
        float* sc = scratch + (size_t)(rec_base + k) * 6;
        float raw[6];
        unsigned bits = 0u;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            raw[i] = sc[i];
            bits |= __float_as_uint(raw[i]);
        }
        if (bits == 0u) continue;
        const int tag = __float_as_int(R[(size_t)k * 5 + 2].w);
        const int la = (tag & 0xFFF) - 1, lb = ((tag >> 12) & 0xFFF) - 1;
        float weight = 1.0f;
        if (weighting) {
            const float na = la >= 0 ? (float)S.cnt[la] : 0.0f;
            const float nb = lb >= 0 ? (float)S.cnt[lb] : 0.0f;
            const float ns = na + nb;
            if (ns > 0.0f) {
                if (na == 0.0f) weight = 1.0f / nb;
                else if (nb == 0.0f) weight = 1.0f / na;
                else weight = 2.0f / ns;
            }
        }
        const int64_t pub = rec_index ? (int64_t)rec_index[rec_base + k] : rec_base + k;
        if (pub >= 0 && pub < cap) {
            float* o = out + (size_t)pub * 6;
#pragma unroll
            for (int i = 0; i < 6; ++i) o[i] = o[i] + raw[i] * weight;
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) sc[i] = 0.0f;
    }
}

__device__ V3 vabs(V3 a) { return V3{fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }

__device__ void weighted_target(V3 axis, float target, float weight, V3& tgt, V3& wts) {
    V3 wa = mul(axis, weight);
    tgt = add(tgt, mul(wa, target));
    wts = add(wts, vabs(wa));
}

__device__ void joint_axes(const NbModelDesc& m, int start, int count, const float* tpos, const float* tvel, V3& lo,
                           V3& hi, V3& tp, V3& stiff, V3& tv, V3& damp) {
    lo = V3{0, 0, 0}; hi = V3{0, 0, 0};
    tp = V3{0, 0, 0}; stiff = V3{0, 0, 0}; tv = V3{0, 0, 0}; damp = V3{0, 0, 0};
    for (int k = 0; k < count && k < 3; ++k) {
        int i = start + k;
        V3 axis = load_v3(m.joint_axis + 3 * (size_t)i);
        V3 lt = mul(axis, m.joint_limit_lower[i]);
        V3 ut = mul(axis, m.joint_limit_upper[i]);
        if (k == 0) {
            lo = vmin(lt, ut);
            hi = vmax(lt, ut);
        } else {
            V3 l2 = vmin(lt, ut), u2 = vmax(lt, ut);
            lo = vmin(lo, l2);
            hi = vmax(hi, u2);
        }
        float ke = m.joint_target_ke[i], kd = m.joint_target_kd[i];
        float tpi = tpos ? tpos[i] : 0.0f, tvi = tvel ? tvel[i] : 0.0f;
        if (ke > 0.0f) weighted_target(axis, tpi, ke, tp, stiff);
        if (kd > 0.0f) weighted_target(axis, tvi, kd, tv, damp);
    }
    for (int i = 0; i < 3; ++i)
        if (comp(stiff, i) > 0.0f) set_comp(tp, i, comp(tp, i) / comp(stiff, i));
    for (int i = 0; i < 3; ++i)
        if (comp(damp, i) > 0.0f) set_comp(tv, i, comp(tv, i) / comp(damp, i));
}

// Whether the reference's solve_body_joints adds deltas for joint j
// (kernels.py:1441-1942: enabled, not FREE, some body moves); ends receives
// the parent (side A) and child (side B) bodies.
template <class SB>
__device__ __forceinline__ bool joint_active(const NbModelDesc& m, const SB& S, int b0, int j, int& ends) {
    if (!m.joint_enabled[j] || m.joint_type[j] == NB_JOINT_FREE) return false;
    const int id_c = m.joint_child[j], id_p = m.joint_parent[j];
    const int lc = id_c - b0, lp = id_p < 0 ? -1 : id_p - b0;
    if ((id_p < 0 || S.inv_m(lp) == 0.0f) && S.inv_m(lc) == 0.0f) return false;
    ends = nb::ends_pack(lp, lc);
    return true;
}

// solve_body_joints for one active joint (kernels.py:1441-1942): d12
// receives the parent's delta (linear, angular) and the child's.  imp
// (optional) accumulates the child-side spatial delta (joint_impulse,
// kernels.py:1941-1942); only this thread touches joint j's row.
template <class SB>
__device__ __noinline__ void solve_joint(const NbModelDesc& m, const SB& S, int b0, int j, const float* tpos,
                                         const float* tvel, const NbXpbdParams& p, float dt, float* d12,
                                         float* imp) {
    // a joint that returns before its deltas contributes zeros: adding +0 leaves every accumulator
    // unchanged (an accumulator that starts at +0 never holds -0)
#pragma unroll
    for (int k = 0; k < 12; ++k) d12[k] = 0.0f;
    int type = m.joint_type[j];
    int id_c = m.joint_child[j], id_p = m.joint_parent[j];
    int lc = id_c - b0, lp = id_p < 0 ? -1 : id_p - b0;
    TF X_pj = load_tf(m.joint_X_p + 7 * (size_t)j);
    TF X_cj = load_tf(m.joint_X_c + 7 * (size_t)j);
    TF X_wp = X_pj;
    float m_inv_p = 0.0f;
    M33 I_inv_p = zero_m33();
    TF pose_p = X_pj;
    V3 com_p{0, 0, 0}, vel_p{0, 0, 0}, om_p{0, 0, 0};
    if (id_p >= 0) {
        pose_p = S.q(lp);
        X_wp = tf_mul(pose_p, X_wp);
        com_p = S.com(lp);
        m_inv_p = S.inv_m(lp);
        I_inv_p = S.inv_inertia(lp);
        vel_p = S.v(lp);
        om_p = S.w(lp);
    }
    TF pose_c = S.q(lc);
    TF X_wc = tf_mul(pose_c, X_cj);
    V3 com_c = S.com(lc);
    float m_inv_c = S.inv_m(lc);
    M33 I_inv_c = S.inv_inertia(lc);
    V3 vel_c = S.v(lc), om_c = S.w(lc);
    V3 ldp{0, 0, 0}, adp{0, 0, 0}, ldc{0, 0, 0}, adc{0, 0, 0};
    TF rel = tf_mul(tf_inverse(X_wp), X_wc);
    V3 rel_p = rel.p;
    V3 x_c = X_wc.p;
    float lin_comp = p.joint_linear_compliance, ang_comp = p.joint_angular_compliance;
    float ang_relax = p.joint_angular_relaxation, lin_relax = p.joint_linear_relaxation;
    int axis_start = m.joint_qd_start[j];
    int lin_count = m.joint_dof_dim[2 * j], ang_count = m.joint_dof_dim[2 * j + 1];
    V3 wcom_p = tf_point(pose_p, com_p);
    V3 wcom_c = tf_point(pose_c, com_c);
    if (type == NB_JOINT_DISTANCE) {
        V3 r_p = sub(X_wp.p, wcom_p);
        V3 r_c = sub(X_wc.p, wcom_c);
        float lower = m.joint_limit_lower[axis_start], upper = m.joint_limit_upper[axis_start];
        if (lower < 0.0f && upper < 0.0f) return;
        float d = length(rel_p);
        float err = 0.0f;
        if (lower >= 0.0f && d < lower) {
            err = d - lower;
            rel_p = smul(err, normalize(sub(wcom_c, wcom_p)));
        } else if (upper >= 0.0f && d > upper) {
            err = d - upper;
        }
        if (fabsf(err) > 1e-9f) {
            V3 lin_c = rel_p;
            V3 lin_p = neg(lin_c);
            r_c = sub(x_c, wcom_c);
            V3 ang_p = neg(cross(r_p, lin_c));
            V3 ang_c = cross(r_c, lin_c);
            float derr = dot(lin_p, vel_p) + dot(lin_c, vel_c) + dot(ang_p, om_p) + dot(ang_c, om_c);
            float compliance = lin_comp;
            float ke = m.joint_target_ke[axis_start];
            if (ke > 0.0f) compliance = 1.0f / ke;
            float damping = m.joint_target_kd[axis_start];
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
            if (fabsf(err) > 1e-9f || fabsf(derr_rel) > 1e-9f) {
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
        float s = sqrtf(rq.x * rq.x + rq.w * rq.w);
        float invs = 1.0f / s;
        float invscube = invs * invs * invs;
        float err0 = 2.0f * nb_asin(clampw(qtwist.x, -1.0f, 1.0f));
        float err1 = qswing.y, err2 = qswing.z;
        Q4 g0{invs - rq.x * rq.x * invscube, 0.0f, 0.0f, -(rq.w * rq.x) * invscube};
        Q4 g1{-rq.w * (rq.w * rq.z + rq.x * rq.y) * invscube, rq.w * invs, -rq.x * invs,
              rq.x * (rq.w * rq.z + rq.x * rq.y) * invscube};
        Q4 g2{rq.w * (rq.w * rq.y - rq.x * rq.z) * invscube, rq.x * invs, rq.w * invs,
              rq.x * (rq.z * rq.x - rq.w * rq.y) * invscube};
        g0 = qscale(g0, 2.0f / fabsf(qtwist.w));
        float swing_sq = qswing.w * qswing.w;
        if (swing_sq + 1.0e-4f < 1.0f) {
            float d = sqrtf(1.0f - qswing.w * qswing.w);
            float theta = 2.0f * nb_acos(clampw(qswing.w, -1.0f, 1.0f));
            float scale = theta / d;
            err1 *= scale;
            err2 *= scale;
            g1 = qscale(g1, scale);
            g2 = qscale(g2, scale);
        }
        V3 lo, hi, tp, stiff, tv, damp;
        joint_axes(m, axis_start + lin_count, ang_count, tpos, tvel, lo, hi, tp, stiff, tv, damp);
        for (int dim = 0; dim < 3; ++dim) {
            float e = dim == 0 ? err0 : (dim == 1 ? err1 : err2);
            Q4 grad = dim == 0 ? g0 : (dim == 1 ? g1 : g2);
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
    d12[0] = ldp.x; d12[1] = ldp.y; d12[2] = ldp.z; d12[3] = adp.x; d12[4] = adp.y; d12[5] = adp.z;
    d12[6] = ldc.x; d12[7] = ldc.y; d12[8] = ldc.z; d12[9] = adc.x; d12[10] = adc.y; d12[11] = adc.z;
    if (imp) {
        float* r = imp + 6 * (size_t)j;
        r[0] = r[0] + ldc.x; r[1] = r[1] + ldc.y; r[2] = r[2] + ldc.z;
        r[3] = r[3] + adc.x; r[4] = r[4] + adc.y; r[5] = r[5] + adc.z;
    }
}

// apply_joint_forces (kernels.py:890-1003) for the world's joints, in joint order
template <class SB>
__device__ void joint_forces(const NbModelDesc& m, SB& S, int b0, int j0, int j1, const float* joint_f) {
    for (int j = j0; j < j1; ++j) {
        int type = m.joint_type[j];
        if (!m.joint_enabled[j]) continue;
        if (type == NB_JOINT_FIXED) continue;
        int id_c = m.joint_child[j], id_p = m.joint_parent[j];
        int lc = id_c - b0, lp = id_p < 0 ? -1 : id_p - b0;
        TF X_pj = load_tf(m.joint_X_p + 7 * (size_t)j), X_cj = load_tf(m.joint_X_c + 7 * (size_t)j);
        TF X_wp = X_pj, pose_p = X_pj;
        V3 com_p{0, 0, 0};
        if (id_p >= 0) {
            pose_p = S.q(lp);
            X_wp = tf_mul(pose_p, X_wp);
            com_p = S.com(lp);
        }
        V3 r_p = sub(X_wp.p, tf_point(pose_p, com_p));
        TF pose_c = S.q(lc);
        TF X_wc = tf_mul(pose_c, X_cj);
        V3 r_c = sub(X_wc.p, tf_point(pose_c, S.com(lc)));
        int qs = m.joint_qd_start[j];
        int lin = m.joint_dof_dim[2 * j], ang = m.joint_dof_dim[2 * j + 1];
        V3 t_total{0, 0, 0}, f_total{0, 0, 0};
        float* F = S.frc;
        const int nb = S.nb;
        auto addw = [&](int b, V3 f, V3 t, bool plus) {
            float v[6] = {f.x, f.y, f.z, t.x, t.y, t.z};
            for (int k = 0; k < 6; ++k) F[k * nb + b] = plus ? F[k * nb + b] + v[k] : F[k * nb + b] - v[k];
        };
        if (type == NB_JOINT_FREE || type == NB_JOINT_DISTANCE) {
            f_total = V3{joint_f[qs + 0], joint_f[qs + 1], joint_f[qs + 2]};
            t_total = V3{joint_f[qs + 3], joint_f[qs + 4], joint_f[qs + 5]};
            addw(lc, f_total, t_total, true);
            if (id_p >= 0) addw(lp, f_total, t_total, false);
            continue;
        } else if (type == NB_JOINT_BALL) {
            t_total = V3{joint_f[qs + 0], joint_f[qs + 1], joint_f[qs + 2]};
        } else {
            for (int k = 0; k < lin && k < 3; ++k)
                f_total = add(f_total, smul(joint_f[qs + k], tf_vector(X_wp, load_v3(m.joint_axis + 3 * (size_t)(qs + k)))));
            for (int k = 0; k < ang && k < 3; ++k)
                t_total = add(t_total, smul(joint_f[qs + lin + k],
                                            tf_vector(X_wp, load_v3(m.joint_axis + 3 * (size_t)(qs + lin + k)))));
        }
        if (id_p >= 0) addw(lp, f_total, add(t_total, cross(r_p, f_total)), false);
        addw(lc, f_total, add(t_total, cross(r_c, f_total)), true);
    }
}

// Contact pass of one iteration for one world (solve_body_contact_positions
// over the world's records, kernels.py:2062-2298): the group tests the
// records in order (48-byte reads), solves the penetrating ones in batches
// with every thread busy, and each body's owner adds its contacts' deltas in
// record order (nb_ordered.cuh); with weighting, the owner also counts them
// (the reference's contact_inv_weight).  imp_scratch (optional) receives each
// active record's A-side delta.
template <int G, class SB>
__device__ __forceinline__ void contact_pass(const NbModelDesc& m, SB& S, const float4* __restrict__ R, int nc,
                                             Batch<G>& B, int g, int t, float relaxation, float dt, bool weighting,
                                             float* imp_scratch) {
    auto test = [&](int k, int& ends) -> bool {
        const float4* r = R + (size_t)k * 5;
        return contact_active(S, r[0], r[1], r[2], ends);
    };
    auto solve = [&](int k, float* d12) {
        const float4* r = R + (size_t)k * 5;
        solve_contact(m, S, r[0], r[1], r[2], r[3], r[4], relaxation, dt, d12,
                      imp_scratch ? imp_scratch + (size_t)k * 6 : nullptr);
    };
    auto add = [&](int i, int, const float* d6) {
        S.add(i, d6);
        if (weighting) S.cnt[i] += 1;
    };
    nb::ordered_pass<G, kST>(B, nc, g, t, test, solve, add);
}

// world's largest penetration max(-d, 0) over its contacts (group reduction
// in *slot, an int holding the float's bits; non-negative floats order as ints)
template <int G, class SB>
__device__ __forceinline__ float world_penetration(const SB& S, const float4* __restrict__ R, int nc, int g, int t,
                                                   int* slot) {
    if (t == 0) *slot = 0;
    group_sync<G>(g);
    float worst = 0.0f;
    for (int k = t; k < nc; k += G) {
        const float4* r = R + (size_t)k * 5;
        const int tag = __float_as_int(r[2].w);
        const int la = (tag & 0xFFF) - 1, lb = ((tag >> 12) & 0xFFF) - 1;
        if (la == lb) continue;
        TF Xa, Xb;
        V3 bx_a, bx_b;
        const float d = contact_depth(S, r[0], r[1], r[2], la, lb, Xa, Xb, bx_a, bx_b);
        worst = fmaxf(worst, -d);  // NaN depths do not count
    }
    if (worst > 0.0f) atomicMax(slot, __float_as_int(worst));
    group_sync<G>(g);
    const float v = __int_as_float(*slot);
    group_sync<G>(g);
    return v;
}

// Learned warm start (no counterpart in the reference): before the plain
// iterations, every contact's predicted impulse (io.ws_lambda, contact frame
// n, t1, t2 as built by nb_ws_features) is applied to its two bodies as one
// combined delta -- linear L on A, -L on B, angular r x L at the contact
// points -- summed per body in record order like the solver's deltas.
// Bodies that receive nothing are left untouched, so an all-zero prediction
// reproduces the plain step exactly.  The world falls back to no warm start
// (state restored from a snapshot kept in the step's output rows) when the
// warm start makes its largest penetration worse.
template <int G, class SB>
__device__ __forceinline__ void warm_start(const NbModelDesc& m, const NbStepIO& io, const NbContactSeg& seg, SB& S,
                                        const float4* __restrict__ R, int nc, int64_t rec_base, int b0, int g,
                                        int t, int* scratch, Batch<G>& B, float dt) {
    const int nb = S.nb;
    const float pen0 = world_penetration<G>(S, R, nc, g, t, scratch);
    // snapshot pose + twist into this world's output rows (overwritten by the write-back)
    for (int i = t; i < nb; i += G) {
        float* qo = io.body_q_out + 7 * (size_t)(b0 + i);
        float* qdo = io.body_qd_out + 6 * (size_t)(b0 + i);
        for (int k = 0; k < 7; ++k) qo[k] = S.f[k * nb + i];
        for (int k = 0; k < 6; ++k) qdo[k] = S.f[(7 + k) * nb + i];
    }
    auto prediction = [&](int k, float& ln, float& l1, float& l2) -> bool {
        const int64_t pub = seg.rec_index ? (int64_t)seg.rec_index[rec_base + k] : rec_base + k;
        if (pub < 0 || pub >= io.ws_capacity) return false;
        const float* lam = io.ws_lambda + 3 * (size_t)pub;
        ln = lam[0];
        l1 = lam[1];
        l2 = lam[2];
        if (ln == 0.0f && l1 == 0.0f && l2 == 0.0f) return false;
        return isfinite(ln) && isfinite(l1) && isfinite(l2);  // a non-finite prediction counts as none
    };
    auto test = [&](int k, int& ends) -> bool {
        float ln, l1, l2;
        if (!prediction(k, ln, l1, l2)) return false;
        const float4* r = R + (size_t)k * 5;
        const int tag = __float_as_int(r[2].w);
        const int la = (tag & 0xFFF) - 1, lb = ((tag >> 12) & 0xFFF) - 1;
        if (la == lb || __float_as_int(r[3].w) == __float_as_int(r[4].w)) return false;
        ends = nb::ends_pack(la, lb);
        return true;
    };
    auto solve = [&](int k, float* d12) {
        float ln, l1, l2;
        prediction(k, ln, l1, l2);
        const float4* r = R + (size_t)k * 5;
        const int tag = __float_as_int(r[2].w);
        const int la = (tag & 0xFFF) - 1, lb = ((tag >> 12) & 0xFFF) - 1;
        const V3 nrm{r[2].x, r[2].y, r[2].z};
        const V3 a = fabsf(nrm.x) < 0.9f ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 1.0f, 0.0f};
        const V3 t1 = normalize(cross(nrm, a));
        const V3 t2 = cross(nrm, t1);
        const V3 L = add(add(mul(nrm, -ln), mul(t1, l1)), mul(t2, l2));
        V3 aa{0, 0, 0}, ab{0, 0, 0};
        if (la >= 0) {
            const TF Xa = S.q(la);
            aa = cross(sub(tf_point(Xa, V3{r[0].x, r[0].y, r[0].z}), tf_point(Xa, S.com(la))), L);
        }
        const V3 Lb = neg(L);
        if (lb >= 0) {
            const TF Xb = S.q(lb);
            ab = cross(sub(tf_point(Xb, V3{r[1].x, r[1].y, r[1].z}), tf_point(Xb, S.com(lb))), Lb);
        }
        d12[0] = L.x; d12[1] = L.y; d12[2] = L.z; d12[3] = aa.x; d12[4] = aa.y; d12[5] = aa.z;
        d12[6] = Lb.x; d12[7] = Lb.y; d12[8] = Lb.z; d12[9] = ab.x; d12[10] = ab.y; d12[11] = ab.z;
    };
    auto add_row = [&](int i, int, const float* d6) { S.add(i, d6); };
    nb::ordered_pass<G, kST>(B, nc, g, t, test, solve, add_row);
    group_sync<G>(g);
    for (int i = t; i < nb; i += G) {
        V3 dl, da;
        if (!S.take(i, dl, da)) continue;  // untouched bodies stay bit-identical
        TF q = S.q(i);
        V3 v = S.v(i), wv = S.w(i);
        apply_body_delta(q, v, wv, dl, da, 1.0f, S.com(i), S.inertia(i), S.inv_m(i), S.inv_inertia(i), dt);
        S.set(i, q, v, wv);
    }
    group_sync<G>(g);
    const float pen1 = world_penetration<G>(S, R, nc, g, t, scratch);
    if (!(io.ws_flags & NB_WS_KEEP_ALL) && !(pen1 <= pen0)) {
        for (int i = t; i < nb; i += G) {
            const float* qo = io.body_q_out + 7 * (size_t)(b0 + i);
            const float* qdo = io.body_qd_out + 6 * (size_t)(b0 + i);
            for (int k = 0; k < 7; ++k) S.f[k * nb + i] = qo[k];
            for (int k = 0; k < 6; ++k) S.f[(7 + k) * nb + i] = qdo[k];
        }
        if (t == 0 && io.ws_fallback) atomicAdd(io.ws_fallback, 1);
    } else if (io.contact_impulse) {
        // the applied prediction is part of the contact's reported impulse (A side)
        for (int k = t; k < nc; k += G) {
            const int64_t pub = seg.rec_index ? (int64_t)seg.rec_index[rec_base + k] : rec_base + k;
            if (pub < 0 || pub >= io.ws_capacity || pub >= io.contact_impulse_capacity) continue;
            const float* lam = io.ws_lambda + 3 * (size_t)pub;
            const float ln = lam[0], l1 = lam[1], l2 = lam[2];
            if (ln == 0.0f && l1 == 0.0f && l2 == 0.0f) continue;
            if (!(isfinite(ln) && isfinite(l1) && isfinite(l2))) continue;
            const float4* r = R + (size_t)k * 5;
            const int tag = __float_as_int(r[2].w);
            const int la = (tag & 0xFFF) - 1, lb = ((tag >> 12) & 0xFFF) - 1;
            if (la == lb || __float_as_int(r[3].w) == __float_as_int(r[4].w)) continue;
            const V3 nrm{r[2].x, r[2].y, r[2].z};
            const V3 a = fabsf(nrm.x) < 0.9f ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 1.0f, 0.0f};
            const V3 t1 = normalize(cross(nrm, a));
            const V3 t2 = cross(nrm, t1);
            const V3 L = add(add(mul(nrm, -ln), mul(t1, l1)), mul(t2, l2));
            V3 A{0.0f, 0.0f, 0.0f};
            if (la >= 0) {
                const TF Xa = S.q(la);
                A = cross(sub(tf_point(Xa, V3{r[0].x, r[0].y, r[0].z}), tf_point(Xa, S.com(la))), L);
            }
            float* o = io.contact_impulse + (size_t)pub * 6;
            o[0] += L.x; o[1] += L.y; o[2] += L.z;
            o[3] += A.x; o[4] += A.y; o[5] += A.z;
        }
    }
    group_sync<G>(g);
}

// A world's bodies are a contiguous block of every per-body array, so the
// group stages them with linear loads: element e of a K-float-per-body block
// (body e / K, component e % K) lands in the structure-of-arrays slab at
// dst[(e % K) * nb + e / K].  The block is read as float4 from its first
// 16-byte boundary on (head and tail elements one by one), so consecutive
// threads read consecutive 16-byte words.
template <int G, int K>
__device__ __forceinline__ void stage_block(const float* __restrict__ src, int nb, float* dst, int t) {
    const int n = K * nb;
    const int head = min((int)(((16u - ((unsigned)(uintptr_t)src & 15u)) & 15u) >> 2), n);
    auto put = [&](int e, float v) { dst[(e % K) * nb + e / K] = v; };
    if (t < head) put(t, __ldg(src + t));
    const float4* s4 = reinterpret_cast<const float4*>(src + head);
    const int n4 = (n - head) >> 2;
    for (int j = t; j < n4; j += G) {
        const float4 v = __ldg(s4 + j);
        const int e = head + 4 * j;
        put(e, v.x);
        put(e + 1, v.y);
        put(e + 2, v.z);
        put(e + 3, v.w);
    }
    for (int e = head + 4 * n4 + t; e < n; e += G) put(e, __ldg(src + e));
}

// The write-back of a K-float-per-body block from the slab (component k of
// body i at src[k * nb + i]) with float4 stores from the first 16-byte boundary
// on.  Kinematic bodies keep their input row (keep[e] from `in`); a non-finite
// value of another body sets *bad.
template <int G, int K, class SB>
__device__ __forceinline__ void write_block(const SB& S, const float* src, const float* __restrict__ in, float* dst,
                                            int t, unsigned* bad) {
    const int nb = S.nb;
    const int n = K * nb;
    const int head = min((int)(((16u - ((unsigned)(uintptr_t)dst & 15u)) & 15u) >> 2), n);
    auto get = [&](int e) -> float {
        const int i = e / K;
        if (S.flags[i] & NB_BODY_KINEMATIC) return in[e];
        const float x = src[(e % K) * nb + i];
        if (!isfinite(x)) *bad |= 2u;
        return x;
    };
    if (t < head) dst[t] = get(t);
    float4* d4 = reinterpret_cast<float4*>(dst + head);
    const int n4 = (n - head) >> 2;
    for (int j = t; j < n4; j += G) {
        const int e = head + 4 * j;
        d4[j] = make_float4(get(e), get(e + 1), get(e + 2), get(e + 3));
    }
    for (int e = head + 4 * n4 + t; e < n; e += G) dst[e] = get(e);
}

// One world's substep with a group of G threads: stage, joint forces,
// integrate, `iterations` x (contacts, weighted apply, joints, apply),
// restitution, write-back.  The caller carved the world's slab into S.
// kLean: the variant for models whose joints are all FREE, called without
// restitution.  It drops that pass and the joint solve at compile time (each
// of them would be a no-op for such a call), which keeps the world's
// shared-memory view in registers instead of on the stack; the arithmetic of
// what remains is the same code.  kWarm: the warm-start pass (inlined) is
// compiled in; kImp: the per-contact impulse accumulation (contact forces,
// the warm start's targets) is compiled in.  The lean variant is built with
// and without each, so that plain calls carry neither.
template <int G, bool kLean, bool kWarm, bool kImp, class SB>
__device__ __forceinline__ void step_world(const NbModelDesc& m, const NbXpbdParams& p, const NbStepIO& io,
                                           const NbContactSeg& seg, bool has_contacts, float dt, int w, SB& S,
                                           int g, int t, int* flag, int* pen_slot, Batch<G>& B,
                                           unsigned* s_bad) {
    const bool weighting = p.rigid_contact_con_weighting != 0;
    const bool model_joints = m.joint_count > 0;
    const float4* rec = reinterpret_cast<const float4*>(seg.rec);
    const int b0 = S.b0;
    const int nb = S.nb;
    // ---- stage bodies (body_f + joint forces go to frc, aliased on acc): the
    // world's pose, twist and force blocks with linear, coalesced loads
    stage_block<G, 7>(io.body_q_in + 7 * (size_t)b0, nb, S.f, t);
    stage_block<G, 6>(io.body_qd_in + 6 * (size_t)b0, nb, S.f + 7 * nb, t);
    stage_block<G, 6>(io.body_f_in + 6 * (size_t)b0, nb, S.frc, t);
    for (int i = t; i < nb; i += G) {
        const int bi = b0 + i;
        const int fl = m.body_flags[bi];
        S.flags[i] = fl;
        if constexpr (!SB::compact) {
            const bool kin = (fl & NB_BODY_KINEMATIC) != 0;
            for (int k = 0; k < 3; ++k) S.c[k * nb + i] = m.body_com[3 * (size_t)bi + k];
            S.c[3 * nb + i] = kin ? 0.0f : m.body_inv_mass[bi];
            for (int k = 0; k < 9; ++k) {
                S.I[k * nb + i] = m.body_inertia[9 * (size_t)bi + k];
                S.iI[k * nb + i] = kin ? 0.0f : m.body_inv_inertia[9 * (size_t)bi + k];
            }
        }
        S.cnt[i] = 0;
    }
    const int j0 = m.world_joint_start[w], j1 = m.world_joint_start[w + 1];
    // bit 0: the world has a non-free enabled joint (needs a real joint pass);
    // bit 1: some joint of the world has a non-zero joint_f entry
    if (t == 0) flag[0] = 0;
    group_sync<G>(g);
    for (int j = j0 + t; j < j1; j += G) {
        if (m.joint_type[j] != NB_JOINT_FREE && m.joint_enabled[j]) atomicOr(&flag[0], 1);
        if (io.joint_f) {
            const int qs = m.joint_qd_start[j];
            const int nd = m.joint_dof_dim[2 * j] + m.joint_dof_dim[2 * j + 1];
            for (int k = 0; k < nd; ++k)
                if (io.joint_f[qs + k] != 0.0f) atomicOr(&flag[0], 2);
        }
    }
    group_sync<G>(g);
    // apply_joint_forces adds joint_f in joint order; all-zero forces change nothing
    if ((flag[0] & 2) && t == 0) joint_forces(m, S, b0, j0, j1, io.joint_f);
    group_sync<G>(g);
    const bool world_joints = (flag[0] & 1) != 0;
    // ---- integrate_bodies (state in registers, frc read before acc is zeroed)
    for (int i = t; i < nb; i += G) {
        const V3 f0{S.frc[0 * nb + i], S.frc[1 * nb + i], S.frc[2 * nb + i]};
        const V3 t0{S.frc[3 * nb + i], S.frc[4 * nb + i], S.frc[5 * nb + i]};
        if (!(S.flags[i] & NB_BODY_KINEMATIC)) {
            const int bi = b0 + i;
            int wi = m.body_world[bi];
            if (wi < 0) wi = 0;
            V3 gv = load_v3(m.gravity + 3 * (size_t)wi);
            TF q = S.q(i);
            V3 v = S.v(i), wv = S.w(i);
            integrate_rigid_body(q, v, wv, f0, t0, S.com(i), S.inertia(i), m.body_inv_mass[bi],
                                 load_m33(m.body_inv_inertia + 9 * (size_t)bi), gv, p.angular_damping, dt);
            S.set(i, q, v, wv);
        }
    }
    group_sync<G>(g);
    for (int i = t; i < nb; i += G)
        for (int k = 0; k < 6; ++k) S.acc[k * nb + i] = 0.0f;
    group_sync<G>(g);
    const int nc = has_contacts ? seg.world_count[w] : 0;
    const int64_t rec_base = has_contacts ? seg.world_base[w] : 0;
    const float4* R = rec + (size_t)rec_base * 5;
    const bool want_imp = (!kLean || kImp) && has_contacts && io.contact_impulse != nullptr;
    unsigned bad = 0u;
    if constexpr (kWarm) {
        if (has_contacts && io.ws_lambda) warm_start<G>(m, io, seg, S, R, nc, rec_base, b0, g, t, pen_slot, B, dt);
    }
    const V3 zero3{0.0f, 0.0f, 0.0f};
    for (int it = 0; it < p.iterations; ++it) {
        if (has_contacts) {
            contact_pass<G>(m, S, R, nc, B, g, t, p.rigid_contact_relaxation, dt, weighting,
                            want_imp ? io.impulse_scratch + (size_t)rec_base * 6 : nullptr);
            if constexpr (!kLean || kImp) {
                if (want_imp) {
                    accumulate_impulses<G>(S, R, nc, rec_base, seg.rec_index, io.impulse_scratch,
                                           io.contact_impulse, io.contact_impulse_capacity, weighting, t);
                    group_sync<G>(g);
                }
            }
            // apply_body_deltas over every body (kernels.py:809-878), weighted by the contact count;
            // in a world whose joints are all free the joint pass that follows adds nothing, so its
            // apply (again every body, zero delta) is fused here
            for (int i = t; i < nb; i += G) {
                V3 dl, da;
                S.take(i, dl, da);
                float weight = 1.0f;
                if (weighting) {
                    const float iw = (float)S.cnt[i];
                    S.cnt[i] = 0;
                    if (iw > 0.0f) weight = 1.0f / iw;
                }
                TF q = S.q(i);
                V3 v = S.v(i), wv = S.w(i);
                const V3 com = S.com(i);
                const float im = S.inv_m(i);
                const M33 I = S.inertia(i), iI = S.inv_inertia(i);
                apply_body_delta(q, v, wv, dl, da, weight, com, I, im, iI, dt);
                if (model_joints && !world_joints) apply_zero_delta(q, v, wv, com, I, im, iI, dt);
                S.set(i, q, v, wv);
            }
            group_sync<G>(g);
        }
        if (model_joints && (world_joints || !has_contacts)) {
            if constexpr (!kLean) {
                if (world_joints) {
                    float* jimp = io.body_parent_f ? io.joint_impulse : nullptr;
                    auto jtest = [&](int k, int& ends) -> bool { return joint_active(m, S, b0, j0 + k, ends); };
                    auto jsolve = [&](int k, float* d12) {
                        solve_joint(m, S, b0, j0 + k, io.joint_target_pos, io.joint_target_vel, p, dt, d12, jimp);
                    };
                    auto jadd = [&](int i, int, const float* d6) { S.add(i, d6); };
                    nb::ordered_pass<G, kST>(B, j1 - j0, g, t, jtest, jsolve, jadd);
                }
            }
            for (int i = t; i < nb; i += G) {
                V3 dl, da;
                S.take(i, dl, da);
                TF q = S.q(i);
                V3 v = S.v(i), wv = S.w(i);
                apply_body_delta(q, v, wv, dl, da, 1.0f, S.com(i), S.inertia(i), S.inv_m(i),
                                 S.inv_inertia(i), dt);
                S.set(i, q, v, wv);
            }
            group_sync<G>(g);
        }
    }
    // ---- restitution (solver_xpbd.py:685-755), after all iterations
    if constexpr (!kLean) {
        if (has_contacts && p.enable_restitution) {
            auto rtest = [&](int k, int& ends) -> bool {
                float tmp[12];
                return restitution_contact(m, S, R + (size_t)k * 5, b0, io.body_q_in, io.body_qd_in, dt, tmp, ends);
            };
            auto rsolve = [&](int k, float* d12) {
                int ends;
                restitution_contact(m, S, R + (size_t)k * 5, b0, io.body_q_in, io.body_qd_in, dt, d12, ends);
            };
            auto radd = [&](int i, int, const float* d6) { S.add(i, d6); };
            nb::ordered_pass<G, kST>(B, nc, g, t, rtest, rsolve, radd);
            // apply_body_delta_velocities (kernels.py:881-887) over every body
            for (int i = t; i < nb; i += G) {
                V3 dl, da;
                S.take(i, dl, da);
                const V3 v = S.v(i), wv = S.w(i);
                S.set(i, S.q(i), add(v, dl), add(wv, da));
            }
            group_sync<G>(g);
        }
    }
    // ---- body_parent_f (solver_xpbd.py:636-655, convert_joint_impulse_to_parent_f,
    // kernels.py:2396-2436): zero for every body of the world, then the
    // child-side impulse / dt of each enabled non-free joint
    if (io.body_parent_f) {
        for (int i = t; i < nb; i += G)
            for (int k = 0; k < 6; ++k) io.body_parent_f[6 * (size_t)(b0 + i) + k] = 0.0f;
        group_sync<G>(g);
        const float inv_dt = 1.0f / dt;
        for (int j = j0 + t; j < j1; j += G) {
            float* r = io.joint_impulse + 6 * (size_t)j;
            const int c = m.joint_child[j];
            if (m.joint_enabled[j] && m.joint_type[j] != NB_JOINT_FREE && c >= 0)
                for (int k = 0; k < 6; ++k) io.body_parent_f[6 * (size_t)c + k] = r[k] * inv_dt;
            for (int k = 0; k < 6; ++k) r[k] = 0.0f;
        }
        group_sync<G>(g);
    }
    // ---- write back with linear, coalesced stores (kinematic bodies pass through unchanged)
    group_sync<G>(g);
    write_block<G, 7>(S, S.f, io.body_q_in + 7 * (size_t)b0, io.body_q_out + 7 * (size_t)b0, t, &bad);
    write_block<G, 6>(S, S.f + 7 * nb, io.body_qd_in + 6 * (size_t)b0, io.body_qd_out + 6 * (size_t)b0, t, &bad);
    if (bad) atomicOr(s_bad, bad);
}

// Batch mode: a CTA takes a batch of worlds (host-packed into one arena, one
// world per group of G threads) from a device counter; the CTA waits for all
// of a batch's worlds before the next batch reuses the arena.
template <int G, bool kLean, bool kWarm, bool kImp>
__global__ void __launch_bounds__(kST, 2)
xpbd_step_kernel(NbModelDesc m, NbXpbdParams p, NbStepIO io, NbContactSeg seg, int has_contacts, float dt) {
    extern __shared__ __align__(16) unsigned char arena[];
    constexpr int kGroups = kST / G;
    __shared__ int s_batch;
    __shared__ unsigned s_bad;
    __shared__ int s_flag[kGroups];
    __shared__ int s_pen[kGroups];
    __shared__ Batch<G> s_ob[kGroups];
    const int g = threadIdx.x / G;   // group within the CTA
    const int t = threadIdx.x % G;   // thread within the group
    if (threadIdx.x == 0) s_bad = 0u;
    for (;;) {
        if (threadIdx.x == 0) s_batch = atomicAdd(&seg.work_counter[4], 1);
        __syncthreads();
        const int b = s_batch;
        if (b >= m.batch_count) break;
        const int w = m.batch_world[b * kGroups + g];
        if (w >= 0) {
            const int b0 = m.world_body_start[w];
            const int nb = m.world_body_start[w + 1] - b0;
            SBodiesT<false> S = sbodies_carve<false>(arena + 4 * (size_t)m.batch_slab[b * kGroups + g], m, b0, nb);
            step_world<G, kLean, kWarm, kImp>(m, p, io, seg, has_contacts != 0, dt, w, S, g, t, &s_flag[g], &s_pen[g],
                                        s_ob[g], &s_bad);
        }
        __syncthreads();  // every group is done with the arena before the next batch
    }
    if (threadIdx.x == 0 && s_bad) atomicOr(seg.status, (unsigned)NB_STATUS_NONFINITE);
}

// Group mode: the CTA's threads form 256 / G independent groups of G threads;
// every group owns a fixed share of the arena and pulls whole worlds (largest
// first) from a device counter on its own -- no CTA-wide barrier, so a group
// never waits for another group's world.  The host picks G and the slab
// layout so that the largest world fits one share (kCompact stages only the
// mutable body state).
template <int G, bool kCompact, bool kLean, bool kWarm, bool kImp>
__global__ void __launch_bounds__(kST, 2)
xpbd_step_group_kernel(NbModelDesc m, NbXpbdParams p, NbStepIO io, NbContactSeg seg, int has_contacts, float dt) {
    extern __shared__ __align__(16) unsigned char arena[];
    constexpr int kGroups = kST / G;
    __shared__ unsigned s_bad;
    __shared__ int s_world[kGroups];
    __shared__ int s_flag[kGroups];
    __shared__ int s_pen[kGroups];
    __shared__ Batch<G> s_ob[kGroups];
    const int g = threadIdx.x / G;
    const int t = threadIdx.x % G;
    if (threadIdx.x == 0) s_bad = 0u;
    __syncthreads();
    const int share = (m.smem_floats_per_batch / kGroups) & ~1;  // words per group, 8-byte aligned
    unsigned char* region = arena + 4 * (size_t)share * g;
    for (;;) {
        int k;
        if constexpr (G == 32) {
            k = 0;
            if (t == 0) k = atomicAdd(&seg.work_counter[4], 1);
            k = __shfl_sync(0xffffffffu, k, 0);
        } else {
            if (t == 0) s_world[g] = atomicAdd(&seg.work_counter[4], 1);
            group_sync<G>(g);
            k = s_world[g];
            group_sync<G>(g);  // everyone read it before the next pull overwrites it
        }
        if (k >= m.world_count) break;
        const int w = m.world_order[k];
        const int b0 = m.world_body_start[w];
        const int nb = m.world_body_start[w + 1] - b0;
        if (nb * slab_words_per_body<kCompact>() > share) {  // the host guarantees this never happens
            if (t == 0) atomicOr(seg.status, (unsigned)NB_STATUS_WORLD_TOO_LARGE);
            continue;
        }
        SBodiesT<kCompact> S = sbodies_carve<kCompact>(region, m, b0, nb);
        step_world<G, kLean, kWarm, kImp>(m, p, io, seg, has_contacts != 0, dt, w, S, g, t, &s_flag[g], &s_pen[g],
                                    s_ob[g], &s_bad);
        group_sync<G>(g);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_bad) atomicOr(seg.status, (unsigned)NB_STATUS_NONFINITE);
}

}  // namespace

size_t nb_step_smem_bytes(const NbModelDesc* m) { return (size_t)m->smem_floats_per_batch * 4; }

namespace {
// convert_contact_impulse_to_force (kernels.py:2363-2393)
__global__ void contact_force_kernel(const float* __restrict__ imp, const int32_t* __restrict__ count, int cap,
                                     float dt, float* __restrict__ force) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= cap) return;
    float* f = force + (size_t)tid * 6;
    if (tid >= count[0]) {
#pragma unroll
        for (int i = 0; i < 6; ++i) f[i] = 0.0f;
        return;
    }
    const float inv_dt = 1.0f / dt;
    const float* p = imp + (size_t)tid * 6;
#pragma unroll
    for (int i = 0; i < 6; ++i) f[i] = p[i] * inv_dt;
}
}  // namespace

cudaError_t nb_launch_contact_forces(const float* imp, const int32_t* count, int cap, float dt, float* force,
                                     cudaStream_t stream) {
    if (cap <= 0) return cudaSuccess;
    contact_force_kernel<<<(cap + 255) / 256, 256, 0, stream>>>(imp, count, cap, dt, force);
    return cudaGetLastError();
}

namespace {
// the lean step kernel applies: every joint is FREE and the call asks for no
// restitution (per-contact impulses select its kImp variant)
bool step_is_lean(const NbModelDesc* m, const NbXpbdParams* p, const NbStepIO*) {
    return m->all_joints_free == 1 && p->enable_restitution == 0;
}

template <int G, bool kLean, bool kWarm, bool kImp>
cudaError_t launch_step_variant(const NbModelDesc* m, const NbXpbdParams* p, const NbStepIO* io,
                                const NbContactSeg* seg, float dt, int grid, cudaStream_t stream) {
    const size_t smem = nb_step_smem_bytes(m);
    cudaError_t e = nb_raise_dynamic_smem((const void*)xpbd_step_kernel<G, kLean, kWarm, kImp>, smem);
    if (e != cudaSuccess) return e;
    const int has_contacts = seg->rec != nullptr && seg->world_count != nullptr && seg->world_base != nullptr;
    xpbd_step_kernel<G, kLean, kWarm, kImp><<<grid, kST, smem, stream>>>(*m, *p, *io, *seg, has_contacts, dt);
    return cudaGetLastError();
}

template <int G>
cudaError_t launch_step(const NbModelDesc* m, const NbXpbdParams* p, const NbStepIO* io, const NbContactSeg* seg,
                        float dt, int grid, cudaStream_t stream) {
    if (!step_is_lean(m, p, io)) return launch_step_variant<G, false, true, true>(m, p, io, seg, dt, grid, stream);
    if (io->contact_impulse)
        return io->ws_lambda ? launch_step_variant<G, true, true, true>(m, p, io, seg, dt, grid, stream)
                             : launch_step_variant<G, true, false, true>(m, p, io, seg, dt, grid, stream);
    return io->ws_lambda ? launch_step_variant<G, true, true, false>(m, p, io, seg, dt, grid, stream)
                         : launch_step_variant<G, true, false, false>(m, p, io, seg, dt, grid, stream);
}

template <int G, bool kCompact, bool kLean, bool kWarm, bool kImp>
cudaError_t launch_step_group_variant(const NbModelDesc* m, const NbXpbdParams* p, const NbStepIO* io,
                                      const NbContactSeg* seg, float dt, int grid, cudaStream_t stream) {
    const size_t smem = nb_step_smem_bytes(m);
    cudaError_t e = nb_raise_dynamic_smem((const void*)xpbd_step_group_kernel<G, kCompact, kLean, kWarm, kImp>, smem);
    if (e != cudaSuccess) return e;
    const int has_contacts = seg->rec != nullptr && seg->world_count != nullptr && seg->world_base != nullptr;
    xpbd_step_group_kernel<G, kCompact, kLean, kWarm, kImp><<<grid, kST, smem, stream>>>(*m, *p, *io, *seg, has_contacts,
                                                                                 dt);
    return cudaGetLastError();
}

template <int G, bool kCompact>
cudaError_t launch_step_group(const NbModelDesc* m, const NbXpbdParams* p, const NbStepIO* io,
                              const NbContactSeg* seg, float dt, int grid, cudaStream_t stream) {
    if (!step_is_lean(m, p, io))
        return launch_step_group_variant<G, kCompact, false, true, true>(m, p, io, seg, dt, grid, stream);
    if (io->contact_impulse)
        return io->ws_lambda
                   ? launch_step_group_variant<G, kCompact, true, true, true>(m, p, io, seg, dt, grid, stream)
                   : launch_step_group_variant<G, kCompact, true, false, true>(m, p, io, seg, dt, grid, stream);
    return io->ws_lambda ? launch_step_group_variant<G, kCompact, true, true, false>(m, p, io, seg, dt, grid, stream)
                         : launch_step_group_variant<G, kCompact, true, false, false>(m, p, io, seg, dt, grid, stream);
}

template <bool kCompact>
cudaError_t launch_step_groups(const NbModelDesc* m, const NbXpbdParams* p, const NbStepIO* io,
                               const NbContactSeg* seg, float dt, int grid, cudaStream_t stream) {
    switch (m->group_threads) {
        case 32: return launch_step_group<32, kCompact>(m, p, io, seg, dt, grid, stream);
        case 64: return launch_step_group<64, kCompact>(m, p, io, seg, dt, grid, stream);
        case 128: return launch_step_group<128, kCompact>(m, p, io, seg, dt, grid, stream);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace

int nb_step_slab_words(int compact) { return compact ? slab_words_per_body<true>() : slab_words_per_body<false>(); }

cudaError_t nb_launch_step(const NbModelDesc* m, const NbXpbdParams* p, const NbStepIO* io, const NbContactSeg* seg,
                           float dt, int grid, cudaStream_t stream) {
    if (m->cta_threads != kST) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(seg->work_counter + 4, 0, sizeof(int32_t), stream);
    if (e != cudaSuccess) return e;
    if (m->step_mode == 1) return launch_step_groups<false>(m, p, io, seg, dt, grid, stream);
    if (m->step_mode == 2) return launch_step_groups<true>(m, p, io, seg, dt, grid, stream);
    switch (m->group_threads) {
        case 32: return launch_step<32>(m, p, io, seg, dt, grid, stream);
        case 64: return launch_step<64>(m, p, io, seg, dt, grid, stream);
        case 128: return launch_step<128>(m, p, io, seg, dt, grid, stream);
        case 256: return launch_step<256>(m, p, io, seg, dt, grid, stream);
        default: return cudaErrorInvalidValue;
    }
}
