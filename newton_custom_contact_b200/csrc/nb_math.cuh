// Device-side fp32 vector / quaternion / transform helpers with Warp's builtin
// semantics (quat = x,y,z,w; transform = p,q; spatial_vector = top,bottom).
// Every expression keeps the reference call sites' evaluation order; the
// parity build of the library is compiled with --fmad=false, so no a*b+c is
// contracted there (the product build lets the compiler contract them).
#pragma once
#include <cstdint>

#define NB_D __device__ __forceinline__

struct V3 { float x, y, z; };
struct Q4 { float x, y, z, w; };
struct TF { V3 p; Q4 q; };
struct M33 { float m[3][3]; };

NB_D V3 mk3(float x, float y, float z) { return V3{x, y, z}; }
NB_D V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
NB_D V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
NB_D V3 mul(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
NB_D V3 smul(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
NB_D V3 divs(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
NB_D V3 neg(V3 a) { return V3{-a.x, -a.y, -a.z}; }
NB_D float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
NB_D V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
NB_D float length_sq(V3 a) { return dot(a, a); }
NB_D float length(V3 a) { return sqrtf(dot(a, a)); }
NB_D V3 normalize(V3 a) {
    float l = length(a);
    if (l > 0.0f) return divs(a, l);
    return V3{0.0f, 0.0f, 0.0f};
}
NB_D V3 vmin(V3 a, V3 b) { return V3{a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z}; }
NB_D V3 vmax(V3 a, V3 b) { return V3{a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z}; }
NB_D float fmaxw(float a, float b) { return a > b ? a : b; }
NB_D float fminw(float a, float b) { return a < b ? a : b; }
NB_D float clampw(float x, float lo, float hi) { return fminw(fmaxw(x, lo), hi); }

// asin / acos in fp32, shared bit for bit with the CPU oracle (the joint
// solve's twist and swing angles, xpbd/kernels.py:1749-1809, need the same
// rounding on both sides).  Own approximation: asin x = x + x z P(z), z = x^2,
// on |x| <= 1/2 with P a degree-5 least-squares fit of (asin x - x) / x^3
// (relative-error weighted, iteratively reweighted toward minimax); above 1/2,
// asin x = 2 (pi/4 - asin(sqrt((1 - x) / 2))) with pi/4 split in two floats.
// Max error against float64 over [-1, 1]: 1.8 ulp (asin), 1.3 ulp (acos).
NB_D float nb_asin_poly(float z) {
    float p = 0.03597569838166237f;
    p = p * z + 0.015487337484955788f;
    p = p * z + 0.03154779598116875f;
    p = p * z + 0.044545069336891174f;
    p = p * z + 0.07500383257865906f;
    p = p * z + 0.16666661202907562f;
    return p;
}
NB_D float nb_asin(float x) {
    const float a = fabsf(x);
    float r;
    if (a <= 0.5f) {
        const float z = a * a;
        r = a + (a * z) * nb_asin_poly(z);
    } else {
        const float z = (1.0f - a) * 0.5f;
        const float s = sqrtf(z);
        const float t = s + (s * z) * nb_asin_poly(z);
        r = 2.0f * ((0.7853981852531433f - t) + -2.1855694143368964e-08f);
    }
    return x < 0.0f ? -r : r;
}
NB_D float nb_acos(float x) {
    if (fabsf(x) <= 0.5f) return (1.5707963705062866f - nb_asin(x)) + -4.371139000186243e-08f;
    if (x > 0.0f) return 2.0f * nb_asin(sqrtf((1.0f - x) * 0.5f));
    return (3.1415927410125732f - 2.0f * nb_asin(sqrtf((1.0f + x) * 0.5f))) + -8.742277657347586e-08f;
}
NB_D float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
NB_D void set_comp(V3& a, int i, float v) {
    if (i == 0) a.x = v;
    else if (i == 1) a.y = v;
    else a.z = v;
}

NB_D Q4 qmul(Q4 a, Q4 b) {
    return Q4{a.w * b.x + b.w * a.x + a.y * b.z - b.y * a.z, a.w * b.y + b.w * a.y + a.z * b.x - b.z * a.x,
              a.w * b.z + b.w * a.z + a.x * b.y - b.x * a.y, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
NB_D Q4 qinv(Q4 q) { return Q4{-q.x, -q.y, -q.z, q.w}; }
NB_D Q4 qadd(Q4 a, Q4 b) { return Q4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
NB_D Q4 qscale(Q4 a, float s) { return Q4{a.x * s, a.y * s, a.z * s, a.w * s}; }
NB_D float qdot(Q4 a, Q4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
NB_D Q4 qnormalize(Q4 q) {
    float l = sqrtf(qdot(q, q));
    if (l > 0.0f) return Q4{q.x / l, q.y / l, q.z / l, q.w / l};
    return Q4{0.0f, 0.0f, 0.0f, 1.0f};
}
NB_D V3 qrot(Q4 q, V3 v) {
    float c = 2.0f * q.w * q.w - 1.0f;
    float d = 2.0f * (q.x * v.x + q.y * v.y + q.z * v.z);
    return V3{v.x * c + q.x * d + (q.y * v.z - q.z * v.y) * q.w * 2.0f,
              v.y * c + q.y * d + (q.z * v.x - q.x * v.z) * q.w * 2.0f,
              v.z * c + q.z * d + (q.x * v.y - q.y * v.x) * q.w * 2.0f};
}
NB_D V3 qrot_inv(Q4 q, V3 v) {
    float c = 2.0f * q.w * q.w - 1.0f;
    float d = 2.0f * (q.x * v.x + q.y * v.y + q.z * v.z);
    return V3{v.x * c + q.x * d - (q.y * v.z - q.z * v.y) * q.w * 2.0f,
              v.y * c + q.y * d - (q.z * v.x - q.x * v.z) * q.w * 2.0f,
              v.z * c + q.z * d - (q.x * v.y - q.y * v.x) * q.w * 2.0f};
}
NB_D M33 quat_to_matrix(Q4 q) {
    V3 c0 = qrot(q, V3{1.0f, 0.0f, 0.0f});
    V3 c1 = qrot(q, V3{0.0f, 1.0f, 0.0f});
    V3 c2 = qrot(q, V3{0.0f, 0.0f, 1.0f});
    M33 r;
    r.m[0][0] = c0.x; r.m[0][1] = c1.x; r.m[0][2] = c2.x;
    r.m[1][0] = c0.y; r.m[1][1] = c1.y; r.m[1][2] = c2.y;
    r.m[2][0] = c0.z; r.m[2][1] = c1.z; r.m[2][2] = c2.z;
    return r;
}
NB_D V3 mv(const M33& a, V3 v) {
    return V3{a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
              a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
              a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
NB_D V3 mtv(const M33& a, V3 v) {
    return V3{a.m[0][0] * v.x + a.m[1][0] * v.y + a.m[2][0] * v.z,
              a.m[0][1] * v.x + a.m[1][1] * v.y + a.m[2][1] * v.z,
              a.m[0][2] * v.x + a.m[1][2] * v.y + a.m[2][2] * v.z};
}
NB_D M33 mscale(float s, const M33& a) {
    M33 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = s * a.m[i][j];
    return r;
}
NB_D M33 zero_m33() {
    M33 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = 0.0f;
    return r;
}
NB_D M33 load_m33(const float* p) {
    M33 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = p[i * 3 + j];
    return r;
}

NB_D TF tf_identity() { return TF{V3{0.0f, 0.0f, 0.0f}, Q4{0.0f, 0.0f, 0.0f, 1.0f}}; }
NB_D TF load_tf(const float* p) { return TF{V3{p[0], p[1], p[2]}, Q4{p[3], p[4], p[5], p[6]}}; }
NB_D void store_tf(float* p, TF t) {
    p[0] = t.p.x; p[1] = t.p.y; p[2] = t.p.z;
    p[3] = t.q.x; p[4] = t.q.y; p[5] = t.q.z; p[6] = t.q.w;
}
NB_D V3 load_v3(const float* p) { return V3{p[0], p[1], p[2]}; }
NB_D V3 tf_point(TF t, V3 v) { return add(qrot(t.q, v), t.p); }
NB_D V3 tf_vector(TF t, V3 v) { return qrot(t.q, v); }
NB_D TF tf_mul(TF a, TF b) { return TF{add(qrot(a.q, b.p), a.p), qmul(a.q, b.q)}; }
NB_D TF tf_inverse(TF t) {
    Q4 qi = qinv(t.q);
    return TF{neg(qrot(qi, t.p)), qi};
}

