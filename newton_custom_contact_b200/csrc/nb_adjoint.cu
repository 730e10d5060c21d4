// Adjoint (reverse-mode gradient) of one XPBD substep for free rigid bodies
// with contacts.  The reference differentiates SolverXPBD.step by recording
// its Warp kernels on a wp.Tape (newton/_src/solvers/xpbd/solver_xpbd.py,
// requires_grad path) and replaying their generated adjoints; this file is a
// hand-written adjoint of the same substep:
//
//   state_in --integrate--> S_0 --iteration 0--> S_1 ... --iteration K-1--> S_K = state_out
//   iteration it:  D_it(i) = sum over active contacts k of body i: C_k(S_it(a_k), S_it(b_k))
//                  S_it+1(i) = A(S_it(i), D_it(i), w_it(i))     (apply_body_delta, weight 1/count)
//
// The forward pass (adjoint_forward_kernel, one CTA per world) re-runs the
// substep in FP32 with the solver's formulas and its ordered float delta sums
// (nb_ordered.cuh) and records S_0..S_K, D_it, w_it and each iteration's active contacts (a
// tape in global scratch).  The reverse pass walks the iterations backwards
// with two flat kernels per iteration over all worlds at once:
// adjoint_bodies_kernel (per body, the vector-Jacobian product of the body
// update: cotangents of S_it(i) and of D_it(i)) and adjoint_contacts_kernel
// (per active contact, the VJP of C_k added into its two bodies' pose and
// angular-velocity cotangents with FP64 atomics); adjoint_integrate_kernel
// finally gives d/d state_in and d/d body_f.  The body update and the
// integration are reversed by hand; a contact's local Jacobian (20 inputs)
// comes from the same generic code evaluated on forward-mode dual numbers,
// 4 directions per pass.
//
// Held fixed (piecewise constant in the reference's own gradient as well):
// the contact set and each record's body-frame points, offsets, normal and
// margins; which contacts are active; the per-body contact counts of the
// weighting; the friction-cone and velocity-threshold branches.  Kinematic
// bodies are constants.  Restitution and enabled non-free joints are not
// differentiated (the kernel flags a world with such a joint and skips it).
#include <cuda_runtime.h>

#include "nb_kernels.cuh"
#include "nb_math.cuh"
#include "nb_ordered.cuh"

namespace {

constexpr int kThreads = 128;
constexpr int kDirs = 4;  // forward-mode directions per pass

// ---------------------------------------------------------------- dual numbers

template <int N>
struct Dual {
    float v;
    float d[N];
    __device__ Dual() {}
    __device__ Dual(float x) : v(x) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0.0f;
    }
};

template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, float s) {
    Dual<N> r;
    r.v = a.v * s;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(float s, const Dual<N>& a) {
    return a * s;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v / b.v;
    const float ib = 1.0f / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, float s) {
    Dual<N> r = a;
    r.v = a.v + s;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(float s, const Dual<N>& a) {
    return a + s;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, float s) {
    Dual<N> r = a;
    r.v = a.v - s;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(float s, const Dual<N>& a) {
    return -a + s;
}

__device__ __forceinline__ float val(float x) { return x; }
template <int N>
__device__ __forceinline__ float val(const Dual<N>& x) {
    return x.v;
}
__device__ __forceinline__ float sqrt_t(float x) { return sqrtf(x); }
template <int N>
__device__ __forceinline__ Dual<N> sqrt_t(const Dual<N>& x) {
    Dual<N> r;
    r.v = sqrtf(x.v);
    const float g = r.v > 0.0f ? 0.5f / r.v : 0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = x.d[i] * g;
    return r;
}

// ---------------------------------------------------------------- generic vector math
// The solver's formulas (Warp builtin semantics), on a scalar type T.

template <class T>
struct V3T {
    T x, y, z;
};
template <class T>
struct Q4T {
    T x, y, z, w;
};

template <class T>
__device__ __forceinline__ V3T<T> vc(V3 a) {
    return V3T<T>{T(a.x), T(a.y), T(a.z)};
}
template <class T>
__device__ __forceinline__ V3T<T> operator+(const V3T<T>& a, const V3T<T>& b) {
    return V3T<T>{a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class T>
__device__ __forceinline__ V3T<T> operator-(const V3T<T>& a, const V3T<T>& b) {
    return V3T<T>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class T>
__device__ __forceinline__ V3T<T> operator-(const V3T<T>& a) {
    return V3T<T>{-a.x, -a.y, -a.z};
}
template <class T, class S>
__device__ __forceinline__ V3T<T> vmul(const V3T<T>& a, const S& s) {
    return V3T<T>{a.x * s, a.y * s, a.z * s};
}
template <class T>
__device__ __forceinline__ T vdot(const V3T<T>& a, const V3T<T>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class T>
__device__ __forceinline__ V3T<T> vcross(const V3T<T>& a, const V3T<T>& b) {
    return V3T<T>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T>
__device__ __forceinline__ T vlength(const V3T<T>& a) {
    return sqrt_t(vdot(a, a));
}
template <class T>
__device__ __forceinline__ V3T<T> vnormalize(const V3T<T>& a) {
    const T l = vlength(a);
    if (val(l) > 0.0f) return V3T<T>{a.x / l, a.y / l, a.z / l};
    return V3T<T>{T(0.0f), T(0.0f), T(0.0f)};
}
template <class T>
__device__ __forceinline__ V3T<T> mvt(const M33& a, const V3T<T>& v) {
    return V3T<T>{v.x * a.m[0][0] + v.y * a.m[0][1] + v.z * a.m[0][2],
                  v.x * a.m[1][0] + v.y * a.m[1][1] + v.z * a.m[1][2],
                  v.x * a.m[2][0] + v.y * a.m[2][1] + v.z * a.m[2][2]};
}
template <class T>
__device__ __forceinline__ Q4T<T> qmult(const Q4T<T>& a, const Q4T<T>& b) {
    return Q4T<T>{a.w * b.x + b.w * a.x + a.y * b.z - b.y * a.z, a.w * b.y + b.w * a.y + a.z * b.x - b.z * a.x,
                  a.w * b.z + b.w * a.z + a.x * b.y - b.x * a.y, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
template <class T>
__device__ __forceinline__ Q4T<T> qnormalizet(const Q4T<T>& q) {
    const T l = sqrt_t(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (val(l) > 0.0f) return Q4T<T>{q.x / l, q.y / l, q.z / l, q.w / l};
    return Q4T<T>{T(0.0f), T(0.0f), T(0.0f), T(1.0f)};
}
template <class T>
__device__ __forceinline__ V3T<T> qrott(const Q4T<T>& q, const V3T<T>& v) {
    const T c = 2.0f * q.w * q.w - 1.0f;
    const T d = 2.0f * (q.x * v.x + q.y * v.y + q.z * v.z);
    return V3T<T>{v.x * c + q.x * d + (q.y * v.z - q.z * v.y) * q.w * 2.0f,
                  v.y * c + q.y * d + (q.z * v.x - q.x * v.z) * q.w * 2.0f,
                  v.z * c + q.z * d + (q.x * v.y - q.y * v.x) * q.w * 2.0f};
}
template <class T>
__device__ __forceinline__ V3T<T> qrot_invt(const Q4T<T>& q, const V3T<T>& v) {
    const T c = 2.0f * q.w * q.w - 1.0f;
    const T d = 2.0f * (q.x * v.x + q.y * v.y + q.z * v.z);
    return V3T<T>{v.x * c + q.x * d - (q.y * v.z - q.z * v.y) * q.w * 2.0f,
                  v.y * c + q.y * d - (q.z * v.x - q.x * v.z) * q.w * 2.0f,
                  v.z * c + q.z * d - (q.x * v.y - q.y * v.x) * q.w * 2.0f};
}

// a body's substep state: pose (p, r), linear and angular velocity; 13 scalars
template <class T>
struct BodyT {
    V3T<T> p;
    Q4T<T> r;
    V3T<T> v, w;
};

// ---------------------------------------------------------------- generic substep pieces

// The branch decisions of one contact or one body update.  Evaluated, each
// decision that holds sets its bit; replayed, the bits decide instead of the
// state (the forward pass of a finite difference that must stay on the piece
// of a recorded substep).
struct Branches {
    unsigned bits = 0;
    bool replay = false;
    __device__ __forceinline__ bool take(int bit, bool cond) {
        if (replay) return ((bits >> bit) & 1u) != 0u;
        if (cond) bits |= 1u << bit;
        return cond;
    }
};

// integrate_bodies (newton/_src/solvers/solver.py:50-94)
template <class T>
__device__ __forceinline__ void integrate_g(BodyT<T>& b, const V3T<T>& f0, const V3T<T>& t0, V3 com, const M33& I, float inv_mass,
                            const M33& inv_I, V3 g, float angular_damping, float dt) {
    const V3T<T> x0 = b.p, w0 = b.w, v0 = b.v;
    const Q4T<T> r0 = b.r;
    const V3T<T> x_com = x0 + qrott(r0, vc<T>(com));
    const float nz = inv_mass != 0.0f ? 1.0f : 0.0f;
    const V3T<T> v1 = v0 + vmul(vmul(f0, inv_mass) + vc<T>(mul(g, nz)), dt);
    const V3T<T> x1 = x_com + vmul(v1, dt);
    const V3T<T> wb = qrot_invt(r0, w0);
    const V3T<T> tb = qrot_invt(r0, t0) - vcross(wb, mvt(I, wb));
    V3T<T> w1 = qrott(r0, wb + vmul(mvt(inv_I, tb), dt));
    const Q4T<T> wq{w1.x, w1.y, w1.z, T(0.0f)};
    const Q4T<T> dq = qmult(wq, r0);
    const Q4T<T> r1 = qnormalizet(Q4T<T>{r0.x + dq.x * 0.5f * dt, r0.y + dq.y * 0.5f * dt, r0.z + dq.z * 0.5f * dt,
                                         r0.w + dq.w * 0.5f * dt});
    w1 = vmul(w1, 1.0f - angular_damping * dt);
    b.p = x1 - qrott(r1, vc<T>(com));
    b.r = r1;
    b.v = v1;
    b.w = w1;
}

// apply_body_deltas (newton/_src/solvers/xpbd/kernels.py:809-878), weight resolved
template <class T>
__device__ __forceinline__ void apply_delta_g(BodyT<T>& b, const V3T<T>& dlin, const V3T<T>& dang, float weight, V3 com,
                              const M33& I, float inv_m, const M33& inv_I, float dt, Branches& br, int bit0) {
    if (inv_m == 0.0f) return;
    const V3T<T> v0 = b.v, w0 = b.w, p0 = b.p;
    const Q4T<T> q0 = b.r;
    const V3T<T> dp = vmul(dlin, inv_m * weight);
    const V3T<T> dq = vmul(dang, weight);
    const V3T<T> wb = qrot_invt(q0, w0);
    const V3T<T> dwb = mvt(inv_I, qrot_invt(q0, dq));
    const V3T<T> tb = vcross(dwb, mvt(I, wb + dwb)) + vcross(wb, mvt(I, dwb));
    const V3T<T> dw1 = qrott(q0, dwb - mvt(mscale(dt, inv_I), tb));
    const Q4T<T> dq4{dw1.x * dt * 0.5f, dw1.y * dt * 0.5f, dw1.z * dt * 0.5f, T(0.0f)};
    const Q4T<T> m = qmult(dq4, q0);
    const Q4T<T> q1 = qnormalizet(Q4T<T>{q0.x + m.x, q0.y + m.y, q0.z + m.z, q0.w + m.w});
    const V3T<T> x_com = p0 + qrott(q0, vc<T>(com));
    V3T<T> p1 = x_com + vmul(dp, dt);
    p1 = p1 - qrott(q1, vc<T>(com));
    V3T<T> v1 = v0 + dp;
    V3T<T> w1 = w0 + dw1;
    if (br.take(bit0, val(vlength(v1)) < 1e-4f)) v1 = V3T<T>{T(0.0f), T(0.0f), T(0.0f)};
    if (br.take(bit0 + 1, val(vlength(w1)) < 1e-4f)) w1 = V3T<T>{T(0.0f), T(0.0f), T(0.0f)};
    b.p = p1;
    b.r = q1;
    b.v = v1;
    b.w = w1;
}

// One iteration's update of a body: the weighted apply of the contact deltas
// (when the step has contact arrays), then -- when the model has joints, all
// free in a differentiated world -- the joint pass's apply of a zero delta,
// which only renormalises (solver_xpbd.py:554-630 as the solver kernel runs it)
template <class T>
__device__ __forceinline__ void body_update_g(BodyT<T>& b, const V3T<T>& dlin, const V3T<T>& dang, float weight, bool contacts,
                              bool joints, V3 com, const M33& I, float inv_m, const M33& inv_I, float dt,
                              Branches& br) {
    if (contacts) apply_delta_g(b, dlin, dang, weight, com, I, inv_m, inv_I, dt, br, 0);
    if (joints) {
        const V3T<T> z{T(0.0f), T(0.0f), T(0.0f)};
        apply_delta_g(b, z, z, 1.0f, com, I, inv_m, inv_I, dt, br, 2);
    }
}

// compute_contact_constraint_delta (kernels.py:1945-1979)
template <class T>
__device__ __forceinline__ T constraint_delta_g(const T& err, const Q4T<T>& qa, const Q4T<T>& qb, float m_inv_a, float m_inv_b,
                                const M33& Ia, const M33& Ib, const V3T<T>& la, const V3T<T>& lb,
                                const V3T<T>& aa, const V3T<T>& ab, float relaxation, float dt) {
    T denom = vdot(la, la) * m_inv_a;
    denom = denom + vdot(lb, lb) * m_inv_b;
    const V3T<T> ra = qrot_invt(qa, aa);
    const V3T<T> rb = qrot_invt(qb, ab);
    denom = denom + vdot(ra, mvt(Ia, ra));
    denom = denom + vdot(rb, mvt(Ib, rb));
    T dl = -err;
    if (val(denom) > 0.0f) dl = dl / (denom * dt);
    return dl * relaxation;
}


// constants of one contact record
struct ContactC {
    V3 p0, p1, n, off0, off1;
    float thickness;
    int la, lb;  // world-local bodies (-1: static)
    float mu, mut, mur;
    V3 com_a, com_b;
    float m_inv_a, m_inv_b;
    M33 Ia, Ib;
    bool kin_a, kin_b;
    V3 kv_a, kw_a, kv_b, kw_b;  // kinematic twists (constants)
};

// solve_body_contact_positions (kernels.py:2062-2298) for one contact:
// deltas (linear, angular) of A and B; false when the contact is inactive
// (mu: the contact's friction coefficient c.mu, as a T so that its derivative can be carried)
template <class T>
__device__ __forceinline__ bool contact_g(const ContactC& c, const BodyT<T>& A, const BodyT<T>& B, float relaxation, float dt,
                          V3T<T>& lin_da, V3T<T>& ang_da, V3T<T>& lin_db, V3T<T>& ang_db, const T& mu,
                          Branches& br) {
    const V3T<T> bxa0 = qrott(A.r, vc<T>(c.p0)) + A.p;
    const V3T<T> bxb0 = qrott(B.r, vc<T>(c.p1)) + B.p;
    const V3T<T> n = vc<T>(c.n);
    const T d = vdot(n, bxb0 - bxa0) - c.thickness;
    if (!br.take(0, val(d) < 0.0f)) return false;  // d >= 0 (NaN counts as active in the solver; not differentiated)
    const V3T<T> r_a0 = bxa0 - (qrott(A.r, vc<T>(c.com_a)) + A.p);
    const V3T<T> r_b0 = bxb0 - (qrott(B.r, vc<T>(c.com_b)) + B.p);
    V3T<T> ang_a = -vcross(r_a0, n);
    V3T<T> ang_b = vcross(r_b0, n);
    const T lambda_n =
        constraint_delta_g(d, A.r, B.r, c.m_inv_a, c.m_inv_b, c.Ia, c.Ib, -n, n, ang_a, ang_b, relaxation, dt);
    lin_da = vmul(-n, lambda_n);
    lin_db = vmul(n, lambda_n);
    ang_da = vmul(ang_a, lambda_n);
    ang_db = vmul(ang_b, lambda_n);
    if (c.mu > 0.0f) {
        const V3T<T> bxa = bxa0 + qrott(A.r, vc<T>(c.off0));
        const V3T<T> bxb = bxb0 + qrott(B.r, vc<T>(c.off1));
        const V3T<T> delta = bxb - bxa;
        V3T<T> fd = delta - vmul(n, vdot(n, delta));
        const V3T<T> r_a = bxa - (qrott(A.r, vc<T>(c.com_a)) + A.p);
        const V3T<T> r_b = bxb - (qrott(B.r, vc<T>(c.com_b)) + B.p);
        V3 rvk{0.0f, 0.0f, 0.0f};
        if (c.kin_a) {
            const V3T<T> va = vcross(vc<T>(c.kw_a), r_a) + vc<T>(c.kv_a);
            const V3T<T> vt = va - vmul(n, vdot(n, va));
            rvk = sub(rvk, V3{val(vt.x), val(vt.y), val(vt.z)});
        }
        if (c.kin_b) {
            const V3T<T> vb = vcross(vc<T>(c.kw_b), r_b) + vc<T>(c.kv_b);
            const V3T<T> vt = vb - vmul(n, vdot(n, vb));
            rvk = add(rvk, V3{val(vt.x), val(vt.y), val(vt.z)});
        }
        fd = fd + vc<T>(mul(rvk, dt));
        const V3T<T> perp = vnormalize(fd);
        ang_a = -vcross(r_a, perp);
        ang_b = vcross(r_b, perp);
        const T err = vlength(fd);
        if (br.take(1, val(err) > 0.0f)) {
            T lf = constraint_delta_g(err, A.r, B.r, c.m_inv_a, c.m_inv_b, c.Ia, c.Ib, -perp, perp, ang_a, ang_b,
                                      relaxation, dt);
            const T cap = -lambda_n * mu;
            if (br.take(2, !(val(lf) > val(cap)))) lf = cap;  // lf = max(lf, cap)
            lin_da = lin_da - vmul(perp, lf);
            lin_db = lin_db + vmul(perp, lf);
            ang_da = ang_da + vmul(ang_a, lf);
            ang_db = ang_db + vmul(ang_b, lf);
        }
    }
    V3T<T> dom = B.w - A.w;
    const V3T<T> z{T(0.0f), T(0.0f), T(0.0f)};
    if (c.mut > 0.0f) {
        const T err = vdot(dom, n) * dt;
        if (br.take(3, fabsf(val(err)) > 0.0f)) {
            T lt = constraint_delta_g(err, A.r, B.r, c.m_inv_a, c.m_inv_b, c.Ia, c.Ib, z, z, -n, n, relaxation, dt);
            const T lo = -lambda_n * c.mut, hi = lambda_n * c.mut;
            if (br.take(4, !(val(lt) > val(lo)))) lt = lo;  // lt = min(max(lt, lo), hi)
            if (br.take(5, !(val(lt) < val(hi)))) lt = hi;
            ang_da = ang_da - vmul(n, lt);
            ang_db = ang_db + vmul(n, lt);
        }
    }
    if (c.mur > 0.0f) {
        dom = dom - vmul(n, vdot(n, dom));
        const T err = vlength(dom) * dt;
        if (br.take(6, val(err) > 0.0f)) {
            const V3T<T> rn = vnormalize(dom);
            T lr = constraint_delta_g(err, A.r, B.r, c.m_inv_a, c.m_inv_b, c.Ia, c.Ib, z, z, -rn, rn, relaxation, dt);
            const T cap = -lambda_n * c.mur;
            if (br.take(7, !(val(lr) > val(cap)))) lr = cap;  // lr = max(lr, cap)
            ang_da = ang_da - vmul(rn, lr);
            ang_db = ang_db + vmul(rn, lr);
        }
    }
    return true;
}

// ---------------------------------------------------------------- state packing

// 13 floats per body: p (3), r (4, xyzw), v (3), w (3)
template <class T>
__device__ __forceinline__ BodyT<T> body_from(const float* s) {
    return BodyT<T>{V3T<T>{T(s[0]), T(s[1]), T(s[2])}, Q4T<T>{T(s[3]), T(s[4]), T(s[5]), T(s[6])},
                    V3T<T>{T(s[7]), T(s[8]), T(s[9])}, V3T<T>{T(s[10]), T(s[11]), T(s[12])}};
}
__device__ __forceinline__ void body_to(const BodyT<float>& b, float* s) {
    s[0] = b.p.x; s[1] = b.p.y; s[2] = b.p.z;
    s[3] = b.r.x; s[4] = b.r.y; s[5] = b.r.z; s[6] = b.r.w;
    s[7] = b.v.x; s[8] = b.v.y; s[9] = b.v.z;
    s[10] = b.w.x; s[11] = b.w.y; s[12] = b.w.z;
}
template <int N>
__device__ __forceinline__ void body_out(const BodyT<Dual<N>>& b, Dual<N>* o) {
    o[0] = b.p.x; o[1] = b.p.y; o[2] = b.p.z;
    o[3] = b.r.x; o[4] = b.r.y; o[5] = b.r.z; o[6] = b.r.w;
    o[7] = b.v.x; o[8] = b.v.y; o[9] = b.v.z;
    o[10] = b.w.x; o[11] = b.w.y; o[12] = b.w.z;
}
// seeds a dual input: value x, unit derivative in direction j - j0 when j is in [j0, j0 + N)
template <int N>
__device__ __forceinline__ Dual<N> seed(float x, int j, int j0) {
    Dual<N> r(x);
    if (j >= j0 && j < j0 + N) r.d[j - j0] = 1.0f;
    return r;
}

// ---------------------------------------------------------------- local vector-Jacobian products

// ---- hand-written reverse mode of the per-body pieces (float)

struct Q4f {
    float x, y, z, w;
};

// cotangent of q for v' = qrot(q, v) = v (2w^2 - 1) + 2 q (q.v) + 2 w (q x v) (any q, unit or not);
// `sgn` = -1 for qrot_inv (the cross term flips)
__device__ __forceinline__ void qrot_vjp_q(Q4 q, V3 v, V3 g, float sgn, Q4f& gq) {
    const V3 qv{q.x, q.y, q.z};
    const float qdv = dot(qv, v), qdg = dot(qv, g);
    const V3 vxg = cross(v, g);
    gq.x += 2.0f * qdv * g.x + 2.0f * v.x * qdg + sgn * 2.0f * q.w * vxg.x;
    gq.y += 2.0f * qdv * g.y + 2.0f * v.y * qdg + sgn * 2.0f * q.w * vxg.y;
    gq.z += 2.0f * qdv * g.z + 2.0f * v.z * qdg + sgn * 2.0f * q.w * vxg.z;
    gq.w += dot(g, add(mul(v, 4.0f * q.w), mul(cross(qv, v), 2.0f * sgn)));
}
// cotangents of a and b for m = qmul(a, b)
__device__ __forceinline__ void qmul_vjp(Q4 a, Q4 b, Q4f g, Q4f& ga, Q4f& gb) {
    ga.x += g.x * b.w - g.y * b.z + g.z * b.y - g.w * b.x;
    ga.y += g.x * b.z + g.y * b.w - g.z * b.x - g.w * b.y;
    ga.z += -g.x * b.y + g.y * b.x + g.z * b.w - g.w * b.z;
    ga.w += g.x * b.x + g.y * b.y + g.z * b.z + g.w * b.w;
    gb.x += g.x * a.w + g.y * a.z - g.z * a.y - g.w * a.x;
    gb.y += -g.x * a.z + g.y * a.w + g.z * a.x - g.w * a.y;
    gb.z += g.x * a.y - g.y * a.x + g.z * a.w - g.w * a.z;
    gb.w += g.x * a.x + g.y * a.y + g.z * a.z + g.w * a.w;
}
// cotangent of u for q = normalize(u) (the solver's qnormalize; zero u maps to the identity)
__device__ __forceinline__ Q4f qnormalize_vjp(Q4 u, Q4f g) {
    const float l = sqrtf(qdot(u, u));
    if (!(l > 0.0f)) return Q4f{0.0f, 0.0f, 0.0f, 0.0f};
    const Q4 q{u.x / l, u.y / l, u.z / l, u.w / l};
    const float d = q.x * g.x + q.y * g.y + q.z * g.z + q.w * g.w;
    return Q4f{(g.x - q.x * d) / l, (g.y - q.y * d) / l, (g.z - q.z * d) / l, (g.w - q.w * d) / l};
}
// cotangents of x and y for c = x cross y
__device__ __forceinline__ void cross_vjp(V3 x, V3 y, V3 g, V3& gx, V3& gy) {
    gx = add(gx, cross(y, g));
    gy = add(gy, cross(g, x));
}

// apply_delta_g(float) reversed: cotangents of the body state (13) and of the delta (6)
__device__ void apply_delta_rev(const float* s, const float* dl, float weight, V3 com, const M33& I, float inv_m,
                                const M33& inv_I, float dt, const float* gout, float* gs, float* gd) {
    for (int k = 0; k < 13; ++k) gs[k] = gout[k];
    for (int k = 0; k < 6; ++k) gd[k] = 0.0f;
    if (inv_m == 0.0f) return;
    // forward recomputation
    const V3 p0{s[0], s[1], s[2]}, v0{s[7], s[8], s[9]}, w0{s[10], s[11], s[12]};
    const Q4 q0{s[3], s[4], s[5], s[6]};
    const float c1 = inv_m * weight;
    const V3 dp = mul(V3{dl[0], dl[1], dl[2]}, c1);
    const V3 dq = mul(V3{dl[3], dl[4], dl[5]}, weight);
    const V3 wb = qrot_inv(q0, w0);
    const V3 z = qrot_inv(q0, dq);
    const V3 dwb = mv(inv_I, z);
    const V3 y1 = mv(I, add(wb, dwb)), y2 = mv(I, dwb);
    const V3 tb = add(cross(dwb, y1), cross(wb, y2));
    const M33 dtiI = mscale(dt, inv_I);
    const V3 u = sub(dwb, mv(dtiI, tb));
    const V3 dw1 = qrot(q0, u);
    const Q4 dq4{dw1.x * dt * 0.5f, dw1.y * dt * 0.5f, dw1.z * dt * 0.5f, 0.0f};
    const Q4 mq = qmul(dq4, q0);
    const Q4 q1u{q0.x + mq.x, q0.y + mq.y, q0.z + mq.z, q0.w + mq.w};
    const Q4 q1 = qnormalize(q1u);
    const V3 v1 = add(v0, dp), w1 = add(w0, dw1);
    // reverse
    V3 gp1{gout[0], gout[1], gout[2]}, gv1{gout[7], gout[8], gout[9]}, gw1{gout[10], gout[11], gout[12]};
    Q4f gq1{gout[3], gout[4], gout[5], gout[6]};
    if (length(v1) < 1e-4f) gv1 = V3{0.0f, 0.0f, 0.0f};
    if (length(w1) < 1e-4f) gw1 = V3{0.0f, 0.0f, 0.0f};
    V3 gv0 = gv1, gdp = gv1, gw0 = gw1, gdw1 = gw1;
    // p1 = p0 + qrot(q0, com) + dp dt - qrot(q1, com)
    V3 gp0 = gp1;
    gdp = add(gdp, mul(gp1, dt));
    Q4f gq0{0.0f, 0.0f, 0.0f, 0.0f};
    qrot_vjp_q(q0, com, gp1, 1.0f, gq0);
    qrot_vjp_q(q1, com, neg(gp1), 1.0f, gq1);
    // q1 = normalize(q0 + qmul(dq4, q0))
    const Q4f gq1u = qnormalize_vjp(q1u, gq1);
    gq0.x += gq1u.x; gq0.y += gq1u.y; gq0.z += gq1u.z; gq0.w += gq1u.w;
    Q4f gdq4{0.0f, 0.0f, 0.0f, 0.0f};
    qmul_vjp(dq4, q0, gq1u, gdq4, gq0);
    gdw1 = add(gdw1, mul(V3{gdq4.x, gdq4.y, gdq4.z}, dt * 0.5f));
    // dw1 = qrot(q0, u), u = dwb - dt inv_I tb
    qrot_vjp_q(q0, u, gdw1, 1.0f, gq0);
    const V3 gu = qrot_inv(q0, gdw1);
    V3 gdwb = gu;
    const V3 gtb = neg(mtv(dtiI, gu));
    // tb = dwb x (I (wb + dwb)) + wb x (I dwb)
    V3 gwb{0.0f, 0.0f, 0.0f}, gy1{0.0f, 0.0f, 0.0f}, gy2{0.0f, 0.0f, 0.0f};
    cross_vjp(dwb, y1, gtb, gdwb, gy1);
    cross_vjp(wb, y2, gtb, gwb, gy2);
    const V3 ty1 = mtv(I, gy1), ty2 = mtv(I, gy2);
    gwb = add(gwb, ty1);
    gdwb = add(gdwb, add(ty1, ty2));
    // dwb = inv_I qrot_inv(q0, dq)
    const V3 gz = mtv(inv_I, gdwb);
    qrot_vjp_q(q0, dq, gz, -1.0f, gq0);
    const V3 gdq = qrot(q0, gz);
    // wb = qrot_inv(q0, w0)
    qrot_vjp_q(q0, w0, gwb, -1.0f, gq0);
    gw0 = add(gw0, qrot(q0, gwb));
    gs[0] = gp0.x; gs[1] = gp0.y; gs[2] = gp0.z;
    gs[3] = gq0.x; gs[4] = gq0.y; gs[5] = gq0.z; gs[6] = gq0.w;
    gs[7] = gv0.x; gs[8] = gv0.y; gs[9] = gv0.z;
    gs[10] = gw0.x; gs[11] = gw0.y; gs[12] = gw0.z;
    gd[0] = gdp.x * c1; gd[1] = gdp.y * c1; gd[2] = gdp.z * c1;
    gd[3] = gdq.x * weight; gd[4] = gdq.y * weight; gd[5] = gdq.z * weight;
}

// body update (body_update_g) reversed: the optional zero-delta renormalisation,
// then the weighted apply
__device__ void vjp_apply(const float* s, const float* dl, float weight, bool contacts, bool joints, V3 com,
                          const M33& I, float inv_m, const M33& inv_I, float dt, const float* gout, float* gs,
                          float* gd) {
    float g[13];
    for (int k = 0; k < 13; ++k) g[k] = gout[k];
    float mid[13];
    for (int k = 0; k < 13; ++k) mid[k] = s[k];
    if (contacts) {
        BodyT<float> b = body_from<float>(s);
        Branches br;
        apply_delta_g(b, V3T<float>{dl[0], dl[1], dl[2]}, V3T<float>{dl[3], dl[4], dl[5]}, weight, com, I, inv_m,
                      inv_I, dt, br, 0);
        body_to(b, mid);
    }
    if (joints) {
        const float zero[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        float gz[6];
        apply_delta_rev(mid, zero, 1.0f, com, I, inv_m, inv_I, dt, gout, g, gz);
    }
    if (contacts) {
        apply_delta_rev(s, dl, weight, com, I, inv_m, inv_I, dt, g, gs, gd);
    } else {
        for (int k = 0; k < 13; ++k) gs[k] = g[k];
        for (int k = 0; k < 6; ++k) gd[k] = 0.0f;
    }
}

// integrate_g(float) reversed: cotangents of the state (13) and of the force / torque (6)
__device__ void vjp_integrate(const float* s, const float* f, V3 com, const M33& I, float inv_mass, const M33& inv_I,
                              V3 g, float damping, float dt, const float* gout, float* gs, float* gf) {
    (void)g;
    const V3 x0{s[0], s[1], s[2]}, w0{s[10], s[11], s[12]};
    const Q4 r0{s[3], s[4], s[5], s[6]};
    const V3 t0{f[3], f[4], f[5]};
    const V3 wb = qrot_inv(r0, w0);
    const V3 y = mv(I, wb);
    const V3 tb = sub(qrot_inv(r0, t0), cross(wb, y));
    const V3 sv = add(wb, mul(mv(inv_I, tb), dt));
    const V3 w1a = qrot(r0, sv);
    const Q4 wq{w1a.x, w1a.y, w1a.z, 0.0f};
    const Q4 dq = qmul(wq, r0);
    const Q4 r1u{r0.x + dq.x * 0.5f * dt, r0.y + dq.y * 0.5f * dt, r0.z + dq.z * 0.5f * dt, r0.w + dq.w * 0.5f * dt};
    const Q4 r1 = qnormalize(r1u);
    const float damp = 1.0f - damping * dt;
    // reverse
    const V3 gp{gout[0], gout[1], gout[2]}, gv{gout[7], gout[8], gout[9]}, gw{gout[10], gout[11], gout[12]};
    Q4f gr1{gout[3], gout[4], gout[5], gout[6]};
    V3 gw1a = mul(gw, damp);
    // p = x1 - qrot(r1, com), x1 = x0 + qrot(r0, com) + v1 dt
    qrot_vjp_q(r1, com, neg(gp), 1.0f, gr1);
    const Q4f gr1u = qnormalize_vjp(r1u, gr1);
    Q4f gr0 = gr1u;
    const Q4f gdq{gr1u.x * 0.5f * dt, gr1u.y * 0.5f * dt, gr1u.z * 0.5f * dt, gr1u.w * 0.5f * dt};
    Q4f gwq{0.0f, 0.0f, 0.0f, 0.0f};
    qmul_vjp(wq, r0, gdq, gwq, gr0);
    gw1a = add(gw1a, V3{gwq.x, gwq.y, gwq.z});
    qrot_vjp_q(r0, sv, gw1a, 1.0f, gr0);
    const V3 gsv = qrot_inv(r0, gw1a);
    V3 gwb = gsv;
    const V3 gtb = mul(mtv(inv_I, gsv), dt);
    // tb = qrot_inv(r0, t0) - wb x (I wb)
    qrot_vjp_q(r0, t0, gtb, -1.0f, gr0);
    const V3 gt0 = qrot(r0, gtb);
    V3 gy{0.0f, 0.0f, 0.0f};
    cross_vjp(wb, y, neg(gtb), gwb, gy);
    gwb = add(gwb, mtv(I, gy));
    qrot_vjp_q(r0, w0, gwb, -1.0f, gr0);
    const V3 gw0 = qrot(r0, gwb);
    const V3 gv1 = add(gv, mul(gp, dt));
    qrot_vjp_q(r0, com, gp, 1.0f, gr0);
    gs[0] = gp.x; gs[1] = gp.y; gs[2] = gp.z;
    gs[3] = gr0.x; gs[4] = gr0.y; gs[5] = gr0.z; gs[6] = gr0.w;
    gs[7] = gv1.x; gs[8] = gv1.y; gs[9] = gv1.z;
    gs[10] = gw0.x; gs[11] = gw0.y; gs[12] = gw0.z;
    gf[0] = gv1.x * inv_mass * dt; gf[1] = gv1.y * inv_mass * dt; gf[2] = gv1.z * inv_mass * dt;
    gf[3] = gt0.x; gf[4] = gt0.y; gf[5] = gt0.z;
    (void)x0;
}

// contact: inputs A pose (7) + A omega (3) + B pose (7) + B omega (3); outputs the four deltas (12)
__device__ __forceinline__ void vjp_contact(const ContactC& c, const float* sa, const float* sb, float relaxation, float dt,
                            const float* gout, float* ga, float* gb) {
#pragma unroll
    for (int j0 = 0; j0 < 20; j0 += kDirs) {
        BodyT<Dual<kDirs>> A, B;
        A.p = {seed<kDirs>(sa[0], 0, j0), seed<kDirs>(sa[1], 1, j0), seed<kDirs>(sa[2], 2, j0)};
        A.r = {seed<kDirs>(sa[3], 3, j0), seed<kDirs>(sa[4], 4, j0), seed<kDirs>(sa[5], 5, j0),
               seed<kDirs>(sa[6], 6, j0)};
        A.v = {Dual<kDirs>(sa[7]), Dual<kDirs>(sa[8]), Dual<kDirs>(sa[9])};
        A.w = {seed<kDirs>(sa[10], 7, j0), seed<kDirs>(sa[11], 8, j0), seed<kDirs>(sa[12], 9, j0)};
        B.p = {seed<kDirs>(sb[0], 10, j0), seed<kDirs>(sb[1], 11, j0), seed<kDirs>(sb[2], 12, j0)};
        B.r = {seed<kDirs>(sb[3], 13, j0), seed<kDirs>(sb[4], 14, j0), seed<kDirs>(sb[5], 15, j0),
               seed<kDirs>(sb[6], 16, j0)};
        B.v = {Dual<kDirs>(sb[7]), Dual<kDirs>(sb[8]), Dual<kDirs>(sb[9])};
        B.w = {seed<kDirs>(sb[10], 17, j0), seed<kDirs>(sb[11], 18, j0), seed<kDirs>(sb[12], 19, j0)};
        V3T<Dual<kDirs>> la, aa, lb, ab;
        Branches br;
        if (!contact_g(c, A, B, relaxation, dt, la, aa, lb, ab, Dual<kDirs>(c.mu), br)) return;
        const Dual<kDirs> o[12] = {la.x, la.y, la.z, aa.x, aa.y, aa.z, lb.x, lb.y, lb.z, ab.x, ab.y, ab.z};
#pragma unroll
        for (int k = 0; k < kDirs && j0 + k < 20; ++k) {
            float acc = 0.0f;
#pragma unroll
            for (int i = 0; i < 12; ++i) acc += gout[i] * o[i].d[k];
            const int j = j0 + k;
            // A: pose -> state 0..6, omega -> state 10..12; B likewise
            if (j < 7) ga[j] += acc;
            else if (j < 10) ga[j + 3] += acc;
            else if (j < 17) gb[j - 10] += acc;
            else gb[j - 7] += acc;
        }
    }
}

// contact: the derivative of the four deltas along the contact's friction coefficient, contracted with
// their cotangents (one forward-mode direction; nonzero where the friction cone clamps)
__device__ __forceinline__ float vjp_contact_mu(const ContactC& c, const float* sa, const float* sb, float relaxation,
                                                float dt, const float* gout) {
    const BodyT<Dual<1>> A = body_from<Dual<1>>(sa), B = body_from<Dual<1>>(sb);
    Dual<1> mu(c.mu);
    mu.d[0] = 1.0f;
    V3T<Dual<1>> la, aa, lb, ab;
    Branches br;
    if (!contact_g(c, A, B, relaxation, dt, la, aa, lb, ab, mu, br)) return 0.0f;
    const Dual<1> o[12] = {la.x, la.y, la.z, aa.x, aa.y, aa.z, lb.x, lb.y, lb.z, ab.x, ab.y, ab.z};
    float acc = 0.0f;
#pragma unroll
    for (int i = 0; i < 12; ++i) acc += gout[i] * o[i].d[0];
    return acc;
}

// ---------------------------------------------------------------- the per-world kernel

__device__ __forceinline__ bool kinematic(const NbModelDesc& m, int bi) {
    return (m.body_flags[bi] & NB_BODY_KINEMATIC) != 0;
}

__device__ ContactC load_contact(const NbModelDesc& m, const float4* r, int b0, const float* tape_it) {
    ContactC c;
    c.p0 = V3{r[0].x, r[0].y, r[0].z};
    c.p1 = V3{r[1].x, r[1].y, r[1].z};
    c.n = V3{r[2].x, r[2].y, r[2].z};
    c.off0 = V3{r[3].x, r[3].y, r[3].z};
    c.off1 = V3{r[4].x, r[4].y, r[4].z};
    c.thickness = r[0].w + r[1].w;
    const int tag = __float_as_int(r[2].w);
    c.la = (tag & 0xFFF) - 1;
    c.lb = ((tag >> 12) & 0xFFF) - 1;
    const int sa = __float_as_int(r[3].w), sb = __float_as_int(r[4].w);
    int nz = 0;
    c.mu = c.mut = c.mur = 0.0f;
    if (sa >= 0) { nz += 1; c.mu += m.shape_mu[sa]; c.mut += m.shape_mu_torsional[sa]; c.mur += m.shape_mu_rolling[sa]; }
    if (sb >= 0) { nz += 1; c.mu += m.shape_mu[sb]; c.mut += m.shape_mu_torsional[sb]; c.mur += m.shape_mu_rolling[sb]; }
    if (nz > 0) { c.mu /= (float)nz; c.mut /= (float)nz; c.mur /= (float)nz; }
    c.com_a = c.com_b = V3{0.0f, 0.0f, 0.0f};
    c.m_inv_a = c.m_inv_b = 0.0f;
    c.Ia = c.Ib = zero_m33();
    c.kin_a = c.kin_b = false;
    c.kv_a = c.kw_a = c.kv_b = c.kw_b = V3{0.0f, 0.0f, 0.0f};
    if (c.la >= 0) {
        const int bi = b0 + c.la;
        c.kin_a = kinematic(m, bi);
        c.com_a = load_v3(m.body_com + 3 * (size_t)bi);
        c.m_inv_a = c.kin_a ? 0.0f : m.body_inv_mass[bi];
        c.Ia = c.kin_a ? zero_m33() : load_m33(m.body_inv_inertia + 9 * (size_t)bi);
        const float* s = tape_it + 13 * (size_t)bi;
        c.kv_a = V3{s[7], s[8], s[9]};
        c.kw_a = V3{s[10], s[11], s[12]};
    }
    if (c.lb >= 0) {
        const int bi = b0 + c.lb;
        c.kin_b = kinematic(m, bi);
        c.com_b = load_v3(m.body_com + 3 * (size_t)bi);
        c.m_inv_b = c.kin_b ? 0.0f : m.body_inv_mass[bi];
        c.Ib = c.kin_b ? zero_m33() : load_m33(m.body_inv_inertia + 9 * (size_t)bi);
        const float* s = tape_it + 13 * (size_t)bi;
        c.kv_b = V3{s[7], s[8], s[9]};
        c.kw_b = V3{s[10], s[11], s[12]};
    }
    return c;
}

// state of a contact side: the body's tape row, or the identity pose at rest for the static side
__device__ __forceinline__ void side_state(const float* tape_it, int b0, int l, float* s) {
    if (l >= 0) {
        const float* t = tape_it + 13 * (size_t)(b0 + l);
#pragma unroll
        for (int k = 0; k < 13; ++k) s[k] = t[k];
    } else {
#pragma unroll
        for (int k = 0; k < 13; ++k) s[k] = 0.0f;
        s[6] = 1.0f;
    }
}

// forward recording, one CTA per world
__global__ void __launch_bounds__(kThreads) adjoint_forward_kernel(NbModelDesc m, NbXpbdParams p, NbAdjointIO io,
                                                                   NbContactSeg seg, int has_contacts, float dt) {
    const int w = blockIdx.x;
    const int t = threadIdx.x;
    const int b0 = m.world_body_start[w], b1 = m.world_body_start[w + 1];
    const int nb = b1 - b0;
    if (nb <= 0) return;
    const size_t B = (size_t)m.body_count;
    const int K = p.iterations;
    const bool weighting = p.rigid_contact_con_weighting != 0;
    const bool model_joints = m.joint_count > 0;
    // enabled non-free joints are not differentiated
    __shared__ int s_flag;
    __shared__ nb::OrderedBatch<kThreads> s_batch;
    if (t == 0) s_flag = 0;
    __syncthreads();
    for (int j = m.world_joint_start[w] + t; j < m.world_joint_start[w + 1]; j += kThreads)
        if (m.joint_enabled[j] && m.joint_type[j] != NB_JOINT_FREE) s_flag = 1;
    __syncthreads();
    if (s_flag) {
        // not differentiated: the tape holds the input state throughout and no contact is active,
        // so the reverse kernels read defined values; the status bit makes the caller discard them
        if (t == 0) atomicOr(io.status, (unsigned)NB_STATUS_ADJOINT_UNSUPPORTED);
        for (int i = t; i < nb; i += kThreads) {
            const int bi = b0 + i;
            for (int it = 0; it <= K; ++it) {
                float* o = io.tape_state + ((size_t)it * B + bi) * 13;
                for (int k = 0; k < 7; ++k) o[k] = io.body_q_in[7 * (size_t)bi + k];
                for (int k = 0; k < 6; ++k) o[7 + k] = io.body_qd_in[6 * (size_t)bi + k];
                if (it < K) {
                    for (int k = 0; k < 6; ++k) io.tape_delta[((size_t)it * B + bi) * 6 + k] = 0.0f;
                    io.tape_weight[(size_t)it * B + bi] = 1.0f;
                }
            }
        }
        return;
    }
    const int nc = has_contacts ? seg.world_count[w] : 0;
    const float4* R = has_contacts ? reinterpret_cast<const float4*>(seg.rec) + (size_t)seg.world_base[w] * 5 : nullptr;

    // ---- forward: integrate, then K iterations, recording the tape
    for (int i = t; i < nb; i += kThreads) {
        const int bi = b0 + i;
        const float* q = io.body_q_in + 7 * (size_t)bi;
        const float* qd = io.body_qd_in + 6 * (size_t)bi;
        float s[13] = {q[0], q[1], q[2], q[3], q[4], q[5], q[6], qd[0], qd[1], qd[2], qd[3], qd[4], qd[5]};
        if (!kinematic(m, bi)) {
            BodyT<float> b = body_from<float>(s);
            const float* f = io.body_f_in + 6 * (size_t)bi;
            int wi = m.body_world[bi];
            wi = wi < 0 ? 0 : wi;
            integrate_g(b, V3T<float>{f[0], f[1], f[2]}, V3T<float>{f[3], f[4], f[5]},
                        load_v3(m.body_com + 3 * (size_t)bi), load_m33(m.body_inertia + 9 * (size_t)bi),
                        m.body_inv_mass[bi], load_m33(m.body_inv_inertia + 9 * (size_t)bi),
                        load_v3(m.gravity + 3 * (size_t)wi), p.angular_damping, dt);
            body_to(b, s);
        }
        float* o = io.tape_state + 13 * (size_t)bi;
#pragma unroll
        for (int k = 0; k < 13; ++k) o[k] = s[k];
    }
    __syncthreads();
    for (int it = 0; it < K; ++it) {
        const float* S_it = io.tape_state + (size_t)it * B * 13;
        float* S_next = io.tape_state + (size_t)(it + 1) * B * 13;
        for (int i = t; i < nb; i += kThreads) {
#pragma unroll
            for (int k = 0; k < 6; ++k) io.delta_acc[6 * (size_t)(b0 + i) + k] = 0.0f;
            io.count_acc[b0 + i] = 0;
        }
        __syncthreads();
        // the solver's contact pass: each body's delta is the float sum of its active contacts'
        // deltas in record order (nb_ordered.cuh), as in nb_xpbd_step
        // branch bytes of this iteration's records (record / replay modes)
        uint8_t* BC = io.branch_mode != 0 && io.branch_contact
                          ? io.branch_contact + (size_t)it * (size_t)m.contact_capacity + (size_t)seg.world_base[w]
                          : nullptr;
        auto test = [&](int k, int& ends) -> bool {
            const float4* r = R + (size_t)k * 5;
            if (__float_as_int(r[3].w) == __float_as_int(r[4].w)) {
                if (io.branch_mode == 1 && BC) BC[k] = 0;
                return false;
            }
            const ContactC c = load_contact(m, r, b0, S_it);
            if (c.la == c.lb) {
                if (io.branch_mode == 1 && BC) BC[k] = 0;
                return false;
            }
            Branches br;
            if (io.branch_mode == 2) {
                br.replay = true;
                br.bits = BC[k];
                if (!(br.bits & 1u)) return false;
            } else {
                float sa[13], sb[13];
                side_state(S_it, b0, c.la, sa);
                side_state(S_it, b0, c.lb, sb);
                V3T<float> la, aa, lb, ab;
                const bool on = contact_g(c, body_from<float>(sa), body_from<float>(sb), p.rigid_contact_relaxation,
                                          dt, la, aa, lb, ab, c.mu, br);
                if (io.branch_mode == 1 && BC) BC[k] = (uint8_t)br.bits;
                if (!on) return false;
            }
            ends = nb::ends_pack(c.la, c.lb);
            return true;
        };
        auto solve = [&](int k, float* d12) {
            const float4* r = R + (size_t)k * 5;
            const ContactC c = load_contact(m, r, b0, S_it);
            float sa[13], sb[13];
            side_state(S_it, b0, c.la, sa);
            side_state(S_it, b0, c.lb, sb);
            V3T<float> la, aa, lb, ab;
            Branches br;
            if (io.branch_mode == 2) {
                br.replay = true;
                br.bits = BC[k];
            }
            contact_g(c, body_from<float>(sa), body_from<float>(sb), p.rigid_contact_relaxation, dt, la, aa, lb, ab,
                      c.mu, br);
            // the reverse pass differentiates this iteration's active contacts only
            const int slot = atomicAdd(io.active_count + it, 1);
            if (slot < io.active_capacity) {
                io.active[2 * ((size_t)it * io.active_capacity + slot)] = (int32_t)(seg.world_base[w] + k);
                io.active[2 * ((size_t)it * io.active_capacity + slot) + 1] = w;
            } else {
                atomicOr(io.status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);
            }
            d12[0] = la.x; d12[1] = la.y; d12[2] = la.z; d12[3] = aa.x; d12[4] = aa.y; d12[5] = aa.z;
            d12[6] = lb.x; d12[7] = lb.y; d12[8] = lb.z; d12[9] = ab.x; d12[10] = ab.y; d12[11] = ab.z;
        };
        auto add = [&](int i, int, const float* d6) {
            float* acc = io.delta_acc + 6 * (size_t)(b0 + i);
#pragma unroll
            for (int q = 0; q < 6; ++q) acc[q] = acc[q] + d6[q];
            if (weighting) io.count_acc[b0 + i] += 1;
        };
        nb::ordered_pass<kThreads, kThreads>(s_batch, nc, 0, t, test, solve, add);
        __syncthreads();
        for (int i = t; i < nb; i += kThreads) {
            const int bi = b0 + i;
            float dl[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) dl[k] = io.delta_acc[6 * (size_t)bi + k];
            const int cnt = io.count_acc[bi];
            const float weight = (weighting && cnt > 0) ? 1.0f / (float)cnt : 1.0f;
            float* D = io.tape_delta + ((size_t)it * B + bi) * 6;
#pragma unroll
            for (int k = 0; k < 6; ++k) D[k] = dl[k];
            io.tape_weight[(size_t)it * B + bi] = weight;
            BodyT<float> b = body_from<float>(S_it + 13 * (size_t)bi);
            uint8_t* BB = io.branch_mode != 0 && io.branch_body ? io.branch_body + (size_t)it * B + bi : nullptr;
            Branches br;
            if (io.branch_mode == 2) {
                br.replay = true;
                br.bits = *BB;
            }
            if (!kinematic(m, bi))
                body_update_g(b, V3T<float>{dl[0], dl[1], dl[2]}, V3T<float>{dl[3], dl[4], dl[5]}, weight,
                              has_contacts != 0, model_joints, load_v3(m.body_com + 3 * (size_t)bi),
                              load_m33(m.body_inertia + 9 * (size_t)bi), m.body_inv_mass[bi],
                              load_m33(m.body_inv_inertia + 9 * (size_t)bi), dt, br);
            if (io.branch_mode == 1 && BB) *BB = (uint8_t)br.bits;
            body_to(b, S_next + 13 * (size_t)bi);
        }
        __syncthreads();
    }
    if (io.body_q_out) {
        const float* S_K = io.tape_state + (size_t)K * B * 13;
        for (int i = t; i < nb; i += kThreads) {
            const float* s = S_K + 13 * (size_t)(b0 + i);
#pragma unroll
            for (int k = 0; k < 7; ++k) io.body_q_out[7 * (size_t)(b0 + i) + k] = s[k];
#pragma unroll
            for (int k = 0; k < 6; ++k) io.body_qd_out[6 * (size_t)(b0 + i) + k] = s[7 + k];
        }
    }

}

// ---- reverse: flat kernels over all bodies / all active contacts of one iteration

__global__ void __launch_bounds__(kThreads) adjoint_seed_kernel(NbModelDesc m, NbAdjointIO io) {
    for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < m.body_count; bi += gridDim.x * blockDim.x) {
        double* g = io.grad_acc + 13 * (size_t)bi;
        for (int k = 0; k < 7; ++k) g[k] = io.grad_q_out[7 * (size_t)bi + k];
        for (int k = 0; k < 6; ++k) g[7 + k] = io.grad_qd_out[6 * (size_t)bi + k];
    }
}

// bodies of iteration it: VJP of the body update; the cotangent of the delta replaces it on the tape
__global__ void __launch_bounds__(kThreads) adjoint_bodies_kernel(NbModelDesc m, NbAdjointIO io, int it,
                                                                  int has_contacts, float dt) {
    const size_t B = (size_t)m.body_count;
    const bool model_joints = m.joint_count > 0;
    const float* S_it = io.tape_state + (size_t)it * B * 13;
    for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < m.body_count; bi += gridDim.x * blockDim.x) {
        float* D = io.tape_delta + ((size_t)it * B + bi) * 6;
        if (kinematic(m, bi)) {
            for (int k = 0; k < 6; ++k) D[k] = 0.0f;
            continue;
        }
        double* g = io.grad_acc + 13 * (size_t)bi;
        float gout[13], gs[13], gd[6], dl[6];
        for (int k = 0; k < 13; ++k) gout[k] = (float)g[k];
        for (int k = 0; k < 6; ++k) dl[k] = D[k];
        vjp_apply(S_it + 13 * (size_t)bi, dl, io.tape_weight[(size_t)it * B + bi], has_contacts != 0, model_joints,
                  load_v3(m.body_com + 3 * (size_t)bi), load_m33(m.body_inertia + 9 * (size_t)bi), m.body_inv_mass[bi],
                  load_m33(m.body_inv_inertia + 9 * (size_t)bi), dt, gout, gs, gd);
        for (int k = 0; k < 13; ++k) g[k] = gs[k];
        for (int k = 0; k < 6; ++k) D[k] = gd[k];
    }
}

// active contacts of iteration it: VJP of the contact's deltas into its bodies' poses and angular velocities
__global__ void __launch_bounds__(kThreads) adjoint_contacts_kernel(NbModelDesc m, NbXpbdParams p, NbAdjointIO io,
                                                                    NbContactSeg seg, int it, float dt) {
    const size_t B = (size_t)m.body_count;
    const float* S_it = io.tape_state + (size_t)it * B * 13;
    int n = io.active_count[it];
    n = n < io.active_capacity ? n : io.active_capacity;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int rec = io.active[2 * ((size_t)it * io.active_capacity + e)];
        const int w = io.active[2 * ((size_t)it * io.active_capacity + e) + 1];
        const int b0 = m.world_body_start[w];
        const float4* r = reinterpret_cast<const float4*>(seg.rec) + (size_t)rec * 5;
        const ContactC c = load_contact(m, r, b0, S_it);
        const bool dyn_a = c.la >= 0 && !c.kin_a, dyn_b = c.lb >= 0 && !c.kin_b;
        if (!dyn_a && !dyn_b) continue;
        float sa[13], sb[13];
        side_state(S_it, b0, c.la, sa);
        side_state(S_it, b0, c.lb, sb);
        float gout[12];
        for (int q = 0; q < 6; ++q) {
            gout[q] = dyn_a ? io.tape_delta[((size_t)it * B + b0 + c.la) * 6 + q] : 0.0f;
            gout[6 + q] = dyn_b ? io.tape_delta[((size_t)it * B + b0 + c.lb) * 6 + q] : 0.0f;
        }
        float ga[13] = {}, gb[13] = {};
        vjp_contact(c, sa, sb, p.rigid_contact_relaxation, dt, gout, ga, gb);
        if (io.grad_shape_mu && c.mu > 0.0f) {
            // the contact's mu is the mean of its shapes' (kernels.py:2160-2178)
            const float gmu = vjp_contact_mu(c, sa, sb, p.rigid_contact_relaxation, dt, gout);
            if (gmu != 0.0f) {
                const int s0 = __float_as_int(r[3].w), s1 = __float_as_int(r[4].w);
                const int nz = (s0 >= 0) + (s1 >= 0);
                if (s0 >= 0) atomicAdd(io.grad_shape_mu + s0, (double)gmu / nz);
                if (s1 >= 0) atomicAdd(io.grad_shape_mu + s1, (double)gmu / nz);
            }
        }
        if (dyn_a)
            for (int q = 0; q < 13; ++q)
                if (ga[q] != 0.0f) atomicAdd(io.grad_acc + 13 * (size_t)(b0 + c.la) + q, (double)ga[q]);
        if (dyn_b)
            for (int q = 0; q < 13; ++q)
                if (gb[q] != 0.0f) atomicAdd(io.grad_acc + 13 * (size_t)(b0 + c.lb) + q, (double)gb[q]);
    }
}

// integration: cotangents of the step's inputs
__global__ void __launch_bounds__(kThreads) adjoint_integrate_kernel(NbModelDesc m, NbXpbdParams p, NbAdjointIO io,
                                                                     float dt) {
    for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < m.body_count; bi += gridDim.x * blockDim.x) {
        const double* g = io.grad_acc + 13 * (size_t)bi;
        float gout[13], gs[13], gf[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        for (int k = 0; k < 13; ++k) gout[k] = (float)g[k];
        if (!kinematic(m, bi)) {
            const float* q = io.body_q_in + 7 * (size_t)bi;
            const float* qd = io.body_qd_in + 6 * (size_t)bi;
            const float s[13] = {q[0], q[1], q[2], q[3], q[4], q[5], q[6], qd[0], qd[1], qd[2], qd[3], qd[4], qd[5]};
            int wi = m.body_world[bi];
            wi = wi < 0 ? 0 : wi;
            vjp_integrate(s, io.body_f_in + 6 * (size_t)bi, load_v3(m.body_com + 3 * (size_t)bi),
                          load_m33(m.body_inertia + 9 * (size_t)bi), m.body_inv_mass[bi],
                          load_m33(m.body_inv_inertia + 9 * (size_t)bi), load_v3(m.gravity + 3 * (size_t)wi),
                          p.angular_damping, dt, gout, gs, gf);
        } else {
            for (int k = 0; k < 13; ++k) gs[k] = gout[k];
        }
        for (int k = 0; k < 7; ++k) io.grad_q_in[7 * (size_t)bi + k] = gs[k];
        for (int k = 0; k < 6; ++k) io.grad_qd_in[6 * (size_t)bi + k] = gs[7 + k];
        if (io.grad_f_in)
            for (int k = 0; k < 6; ++k) io.grad_f_in[6 * (size_t)bi + k] = gf[k];
    }
}

}  // namespace

cudaError_t nb_launch_xpbd_adjoint(const NbModelDesc* m, const NbXpbdParams* p, const NbAdjointIO* io,
                                   const NbContactSeg* seg, int has_contacts, float dt, cudaStream_t s) {
    if (m->world_count <= 0 || m->body_count <= 0) return cudaSuccess;
    const int K = p->iterations;
    cudaError_t e = cudaMemsetAsync(io->active_count, 0, sizeof(int32_t) * (size_t)(K > 0 ? K : 1), s);
    if (e != cudaSuccess) return e;
    adjoint_forward_kernel<<<m->world_count, kThreads, 0, s>>>(*m, *p, *io, *seg, has_contacts, dt);
    if (io->forward_only) return cudaGetLastError();
    const int gb = nb_contact_grid(m->body_count, kThreads);
    adjoint_seed_kernel<<<gb, kThreads, 0, s>>>(*m, *io);
    const int gc = nb_contact_grid(io->active_capacity > 0 ? io->active_capacity : 1, kThreads);
    for (int it = K - 1; it >= 0; --it) {
        adjoint_bodies_kernel<<<gb, kThreads, 0, s>>>(*m, *io, it, has_contacts, dt);
        if (has_contacts && io->active_capacity > 0)
            adjoint_contacts_kernel<<<gc, kThreads, 0, s>>>(*m, *p, *io, *seg, it, dt);
    }
    adjoint_integrate_kernel<<<gb, kThreads, 0, s>>>(*m, *p, *io, dt);
    return cudaGetLastError();
}
