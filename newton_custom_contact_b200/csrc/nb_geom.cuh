// Narrow-phase geometry for one candidate pair, device side.
//
// Restates, for plane / sphere / capsule / box:
//   support maps            newton/_src/geometry/support_function.py:106-305
//   tight AABB              newton/_src/geometry/collision_core.py:396-491
//   analytic primitives     newton/_src/geometry/collision_primitive.py:48-439, 1161-1215
//   primitive routing       newton/_src/geometry/narrow_phase.py:198-603
//   plane proxy / bsphere   newton/_src/geometry/collision_core.py:508-725
//   MPR                     newton/_src/geometry/mpr.py:56-504
//   GJK                     newton/_src/geometry/simplex_solver.py:44-491
//   fused MPR+GJK           newton/_src/geometry/collision_convex.py:26-135
//   manifold                newton/_src/geometry/multicontact.py:28-954
//   write_contact           newton/_src/sim/collide.py:62-147
// Contacts are appended to the candidate's private slot range in sub-key
// order; the caller compacts the slots of all candidates in pair-key order.
#pragma once
#include "nb_math.cuh"
#include "../../include/newton_b200.h"

namespace nbg {

static constexpr float MAXVAL = 1e10f;
static constexpr float MINVAL = 0x1.203afap-50f;
static constexpr float SIN_TILT = 0x1.1de58cp-5f;
static constexpr float COS_TILT = 0x1.ffb028p-1f;
static constexpr float COS_DEEPEST = 0x1.ffffccp-1f;

NB_D float pent_c(int e) {
    return e == 0 ? 1.0f : (e == 1 ? 0x1.3c6ef4p-2f : (e == 2 ? -0x1.9e377ap-1f : (e == 3 ? -0x1.9e377ap-1f : 0x1.3c6ef4p-2f)));
}
NB_D float pent_s(int e) {
    return e == 0 ? 0.0f : (e == 1 ? 0x1.e6f0e2p-1f : (e == 2 ? 0x1.2cf230p-1f : (e == 3 ? -0x1.2cf230p-1f : -0x1.e6f0e2p-1f)));
}

struct Shape {
    int type;
    V3 scale;
};

// world-space geometry of one shape (compute_shape_aabbs output)
struct Geom {
    TF xf;
    V3 scale;
    float margin;
    V3 lo, hi;
    int type;
    float gap;
    int body;     // global body index or -1
    int sid;      // global shape index
};

NB_D V3 support(const Shape& g, V3 d) {
    if (g.type == NB_GEO_BOX) {
        float threshold = 1.0e-10f * length(d);
        float sx = d.x >= -threshold ? 1.0f : -1.0f;
        float sy = d.y >= -threshold ? 1.0f : -1.0f;
        float sz = d.z >= -threshold ? 1.0f : -1.0f;
        return V3{sx * g.scale.x, sy * g.scale.y, sz * g.scale.z};
    }
    if (g.type == NB_GEO_SPHERE || g.type == NB_GEO_CAPSULE) {
        V3 n;
        if (length_sq(d) > 1.0e-12f) n = normalize(d);
        else n = V3{1.0f, 0.0f, 0.0f};
        V3 r = mul(n, g.scale.x);
        if (g.type == NB_GEO_CAPSULE) {
            if (d.z >= 0.0f) r = add(r, V3{0.0f, 0.0f, g.scale.y});
            else r = add(r, V3{0.0f, 0.0f, -g.scale.y});
        }
        return r;
    }
    if (g.type == NB_GEO_PLANE) {
        float sx = d.x >= 0.0f ? 1.0f : -1.0f;
        float sy = d.y >= 0.0f ? 1.0f : -1.0f;
        return V3{sx * g.scale.x, sy * g.scale.y, 0.0f};
    }
    return V3{0.0f, 0.0f, 0.0f};
}

// compute_shape_aabbs for one shape given its world transform
NB_D void shape_geom(Geom& g, TF xf, int type, V3 scale, float margin, float gap, float radius, int body) {
    g.xf = xf;
    g.type = type;
    g.body = body;
    g.gap = gap;
    g.margin = margin;
    float eff = margin + gap;
    V3 mvv{eff, eff, eff};
    bool inf_plane = type == NB_GEO_PLANE && scale.x == 0.0f && scale.y == 0.0f;
    g.scale = scale;
    if (inf_plane) {
        V3 he{radius, radius, radius};
        g.lo = sub(sub(xf.p, he), mvv);
        g.hi = add(add(xf.p, he), mvv);
    } else {
        if (type == NB_GEO_PLANE) g.scale = V3{scale.x * 0.5f, scale.y * 0.5f, 0.0f};
        Shape sh{type, g.scale};
        M33 r = quat_to_matrix(xf.q);
        V3 lx{r.m[0][0], r.m[0][1], r.m[0][2]};
        V3 ly{r.m[1][0], r.m[1][1], r.m[1][2]};
        V3 lz{r.m[2][0], r.m[2][1], r.m[2][2]};
        float max_x = dot(lx, support(sh, lx));
        float max_y = dot(ly, support(sh, ly));
        float max_z = dot(lz, support(sh, lz));
        float min_x = dot(lx, support(sh, neg(lx)));
        float min_y = dot(ly, support(sh, neg(ly)));
        float min_z = dot(lz, support(sh, neg(lz)));
        g.lo = sub(add(V3{min_x, min_y, min_z}, xf.p), mvv);
        g.hi = add(add(V3{max_x, max_y, max_z}, xf.p), mvv);
    }
}

NB_D bool aabb_overlap(const Geom& a, const Geom& b) {
    float c = 0.0f + 0.0f;
    return a.lo.x <= b.hi.x + c && a.hi.x >= b.lo.x - c && a.lo.y <= b.hi.y + c && a.hi.y >= b.lo.y - c &&
           a.lo.z <= b.hi.z + c && a.hi.z >= b.lo.z - c;
}

// ------------------------------------------------------------ writer
struct ContactData {
    V3 center;
    V3 normal;
    float dist;
    float reff_a, reff_b, margin_a, margin_b;
    float gap_sum;
    int sub_key;
};

struct Writer {
    float4* slots;       // 5 contacts x 5 float4 for this candidate
    int n;
    TF inv_a, inv_b;     // inverse body transforms (identity for static shapes)
    float gap;           // gap_a + gap_b
    int shape_a, shape_b;
    int tag;             // (body_a_local+1) | (body_b_local+1)<<12
};

NB_D bool passes_gap(const ContactData& c) {
    float total = c.reff_a + c.reff_b + c.margin_a + c.margin_b;
    V3 n = normalize(c.normal);
    V3 a = sub(c.center, mul(n, 0.5f * c.dist + c.reff_a));
    V3 b = add(c.center, mul(n, 0.5f * c.dist + c.reff_b));
    float d = dot(sub(b, a), n) - total;
    return d <= c.gap_sum;
}

NB_D void write_contact(Writer& w, const ContactData& c, bool check_gap) {
    float total = c.reff_a + c.reff_b + c.margin_a + c.margin_b;
    float off_a = c.reff_a + c.margin_a;
    float off_b = c.reff_b + c.margin_b;
    V3 n = normalize(c.normal);
    V3 a_w = sub(c.center, mul(n, 0.5f * c.dist + c.reff_a));
    V3 b_w = add(c.center, mul(n, 0.5f * c.dist + c.reff_b));
    float d = dot(sub(b_w, a_w), n) - total;
    if (check_gap && d > w.gap) return;
    if (w.n >= 5) return;
    V3 p0 = tf_point(w.inv_a, a_w);
    V3 p1 = tf_point(w.inv_b, b_w);
    V3 o0 = tf_vector(w.inv_a, mul(n, off_a));
    V3 o1 = tf_vector(w.inv_b, mul(n, -off_b));
    float4* s = w.slots + 5 * w.n;
    s[0] = make_float4(p0.x, p0.y, p0.z, off_a);
    s[1] = make_float4(p1.x, p1.y, p1.z, off_b);
    s[2] = make_float4(n.x, n.y, n.z, __int_as_float(w.shape_a));
    s[3] = make_float4(o0.x, o0.y, o0.z, __int_as_float(w.shape_b));
    s[4] = make_float4(o1.x, o1.y, o1.z, __int_as_float(w.tag | ((c.sub_key & 0xFF) << 24)));
    w.n += 1;
}

// ------------------------------------------------------------ primitives
NB_D V3 closest_segment_point(V3 a, V3 b, V3 pt) {
    V3 ab = sub(b, a);
    float t = dot(sub(pt, a), ab) / (dot(ab, ab) + 1e-6f);
    return add(a, smul(clampw(t, 0.0f, 1.0f), ab));
}

NB_D void collide_plane_sphere(V3 n, V3 ppos, V3 spos, float r, float& dist, V3& pos) {
    dist = dot(sub(spos, ppos), n) - r;
    pos = sub(spos, mul(n, r + 0.5f * dist));
}

NB_D void collide_sphere_sphere(V3 p1, float r1, V3 p2, float r2, float& dist, V3& pos, V3& n) {
    V3 dir = sub(p2, p1);
    dist = length(dir);
    if (dist == 0.0f) n = V3{1.0f, 0.0f, 0.0f};
    else n = divs(dir, dist);
    dist = dist - (r1 + r2);
    pos = add(p1, mul(n, r1 + 0.5f * dist));
}

NB_D void collide_capsule_capsule(V3 p1, V3 ax1, float r1, float h1, V3 p2, V3 ax2, float r2, float h2,
                                  float* dist, V3* pos, V3& normal) {
    dist[0] = MAXVAL;
    dist[1] = MAXVAL;
    V3 axis1 = mul(ax1, h1);
    V3 axis2 = mul(ax2, h2);
    V3 dif = sub(p1, p2);
    float ma = dot(axis1, axis1);
    float mb = -dot(axis1, axis2);
    float mc = dot(axis2, axis2);
    float u = -dot(axis1, dif);
    float v = dot(axis2, dif);
    float det = ma * mc - mb * mb;
    if (fabsf(det) >= MINVAL) {
        float inv_det = 1.0f / det;
        float x1 = (mc * u - mb * v) * inv_det;
        float x2 = (ma * v - mb * u) * inv_det;
        if (x1 > 1.0f) { x1 = 1.0f; x2 = (v - mb) / mc; }
        else if (x1 < -1.0f) { x1 = -1.0f; x2 = (v + mb) / mc; }
        if (x2 > 1.0f) { x2 = 1.0f; x1 = clampw((u - mb) / ma, -1.0f, 1.0f); }
        else if (x2 < -1.0f) { x2 = -1.0f; x1 = clampw((u + mb) / ma, -1.0f, 1.0f); }
        V3 vec1 = add(p1, mul(axis1, x1));
        V3 vec2 = add(p2, mul(axis2, x2));
        collide_sphere_sphere(vec1, r1, vec2, r2, dist[0], pos[0], normal);
    } else {
        V3 vec1 = add(p1, axis1);
        float x2 = clampw((v - mb) / mc, -1.0f, 1.0f);
        V3 vec2 = add(p2, mul(axis2, x2));
        collide_sphere_sphere(vec1, r1, vec2, r2, dist[0], pos[0], normal);
        vec1 = sub(p1, axis1);
        x2 = clampw((v + mb) / mc, -1.0f, 1.0f);
        vec2 = add(p2, mul(axis2, x2));
        V3 n2;
        collide_sphere_sphere(vec1, r1, vec2, r2, dist[1], pos[1], n2);
    }
}

NB_D void collide_plane_box(V3 n, V3 ppos, V3 bpos, const M33& rot, V3 size, float margin, float* dist, V3* pos) {
    float center_dist = dot(sub(bpos, ppos), n);
    int ncontact = 0, worst = 0;
#pragma unroll 1
    for (int i = 0; i < 8; ++i) {
        V3 corner{(i & 1) ? size.x : -size.x, (i & 2) ? size.y : -size.y, (i & 4) ? size.z : -size.z};
        corner = mv(rot, corner);
        float ldist = dot(n, corner);
        float cdist = center_dist + ldist;
        if (cdist > margin) continue;
        V3 cpos = sub(add(corner, bpos), mul(smul(0.5f, n), cdist));
        if (ncontact < 4) {
            dist[ncontact] = cdist;
            pos[ncontact] = cpos;
            if (ncontact == 0 || cdist > dist[worst]) worst = ncontact;
            ncontact += 1;
        } else if (cdist < dist[worst]) {
            dist[worst] = cdist;
            pos[worst] = cpos;
            worst = 0;
            if (dist[1] > dist[worst]) worst = 1;
            if (dist[2] > dist[worst]) worst = 2;
            if (dist[3] > dist[worst]) worst = 3;
        }
    }
}

NB_D void collide_sphere_box(V3 spos, float r, V3 bpos, const M33& rot, V3 size, float& dist, V3& pos, V3& normal) {
    V3 center = mtv(rot, sub(spos, bpos));
    V3 clamped = vmax(neg(size), vmin(size, center));
    V3 cd = sub(clamped, center);
    float d = length(cd);
    V3 cdir = (d == 0.0f) ? cd : divs(cd, d);
    V3 lpos;
    if (d <= 1e-6f) {
        float closest = 2.0f * (size.x + size.y + size.z);
        int k = 0;
#pragma unroll 1
        for (int i = 0; i < 6; ++i) {
            float sgn = (i % 2) ? 1.0f : -1.0f;
            float face = fabsf(sgn * comp(size, i / 2) - comp(center, i / 2));
            if (closest > face) { closest = face; k = i; }
        }
        V3 nearest{0.0f, 0.0f, 0.0f};
        set_comp(nearest, k / 2, (k % 2) ? -1.0f : 1.0f);
        lpos = add(center, divs(mul(nearest, r - closest), 2.0f));
        normal = mv(rot, nearest);
        dist = -closest - r;
    } else {
        V3 deepest = add(center, mul(cdir, r));
        lpos = smul(0.5f, add(clamped, deepest));
        normal = mv(rot, cdir);
        dist = d - r;
    }
    pos = add(bpos, mv(rot, lpos));
}

// ------------------------------------------------------------ MPR / GJK
struct Vert { V3 B, BtoA; };
NB_D V3 vert_a(const Vert& v) { return add(v.B, v.BtoA); }

struct Pair {
    Shape a, b;
    Q4 ob;
    V3 pb;
};

NB_D V3 support_b(const Pair& p, V3 dir) {
    V3 tmp = qrot_inv(p.ob, dir);
    V3 r = support(p.b, tmp);
    r = qrot(p.ob, r);
    return add(r, p.pb);
}

NB_D Vert minkowski(const Pair& p, V3 dir, float extend) {
    Vert v;
    V3 pa = support(p.a, dir);
    v.B = support_b(p, neg(dir));
    if (extend != 0.0f) {
        V3 d = mul(mul(normalize(dir), extend), 0.5f);
        pa = add(pa, d);
        v.B = sub(v.B, d);
    }
    v.BtoA = sub(pa, v.B);
    return v;
}

NB_D Vert geometric_center(const Pair& p) {
    Vert c;
    V3 center_a{0.0f, 0.0f, 0.0f};
    V3 cbw = add(p.pb, qrot(p.ob, V3{0.0f, 0.0f, 0.0f}));
    c.B = cbw;
    c.BtoA = sub(center_a, cbw);
    return c;
}

__device__ __noinline__ bool mpr_core(const Pair& p, float extend, V3& point_a, V3& point_b, V3& normal,
                                      float& penetration) {
    const int MAX_ITER = 30;
    const float COLLIDE_EPSILON = 1e-5f;
    const float NUMERIC_EPSILON = 1e-16f;
    penetration = 0.0f;
    point_a = V3{0, 0, 0};
    point_b = V3{0, 0, 0};
    Vert v0 = geometric_center(p);
    normal = v0.BtoA;
    if (length_sq(normal) < NUMERIC_EPSILON) {
        float best_dot = -1.0e30f;
        V3 best_dir{1.0f, 0.0f, 0.0f};
        for (int ax = 0; ax < 3; ++ax) {
            V3 probe{0.0f, 0.0f, 0.0f};
            set_comp(probe, ax, 1.0f);
            Vert sv = minkowski(p, probe, extend);
            float d = dot(sv.BtoA, probe);
            if (d > best_dot) { best_dot = d; best_dir = probe; }
        }
        v0.BtoA = mul(best_dir, 1e-05f);
    }
    normal = neg(v0.BtoA);
    Vert v1 = minkowski(p, normal, extend);
    point_a = vert_a(v1);
    point_b = v1.B;
    if (dot(v1.BtoA, normal) <= 0.0f) return false;
    normal = cross(v1.BtoA, v0.BtoA);
    if (length_sq(normal) < NUMERIC_EPSILON * NUMERIC_EPSILON) {
        normal = sub(v1.BtoA, v0.BtoA);
        normal = normalize(normal);
        penetration = dot(v1.BtoA, normal);
        return true;
    }
    Vert v2 = minkowski(p, normal, extend);
    if (dot(v2.BtoA, normal) <= 0.0f) return false;
    V3 t1 = sub(v1.BtoA, v0.BtoA);
    V3 t2 = sub(v2.BtoA, v0.BtoA);
    normal = cross(t1, t2);
    float dist = dot(normal, v0.BtoA);
    if (dist > 0.0f) {
        Vert tmp = v1;
        v1 = v2;
        v2 = tmp;
        normal = neg(normal);
    }
    int phase1 = 0, phase2 = 0;
    bool hit = false;
    Vert v3;
    while (true) {
        if (phase1 > MAX_ITER) return false;
        phase1 += 1;
        v3 = minkowski(p, normal, extend);
        if (dot(v3.BtoA, normal) <= 0.0f) return false;
        V3 tt = cross(v1.BtoA, v3.BtoA);
        if (dot(tt, v0.BtoA) < 0.0f) {
            v2 = v3;
            normal = cross(sub(v1.BtoA, v0.BtoA), sub(v3.BtoA, v0.BtoA));
            continue;
        }
        tt = cross(v3.BtoA, v2.BtoA);
        if (dot(tt, v0.BtoA) < 0.0f) {
            v1 = v3;
            normal = cross(sub(v3.BtoA, v0.BtoA), sub(v2.BtoA, v0.BtoA));
            continue;
        }
        break;
    }
    while (true) {
        phase2 += 1;
        V3 a1 = sub(v2.BtoA, v1.BtoA);
        V3 a2 = sub(v3.BtoA, v1.BtoA);
        normal = cross(a1, a2);
        float normal_sq = length_sq(normal);
        if (normal_sq < NUMERIC_EPSILON * NUMERIC_EPSILON) return false;
        if (!hit) {
            float d = dot(normal, v1.BtoA);
            hit = d >= 0.0f;
        }
        Vert v4 = minkowski(p, normal, extend);
        V3 t3 = sub(v4.BtoA, v3.BtoA);
        float delta = dot(t3, normal);
        penetration = dot(v4.BtoA, normal);
        if (delta * delta <= COLLIDE_EPSILON * COLLIDE_EPSILON * normal_sq || penetration <= 0.0f ||
            phase2 > MAX_ITER) {
            if (hit) {
                float inv_normal = 1.0f / sqrtf(normal_sq);
                penetration *= inv_normal;
                normal = mul(normal, inv_normal);
                V3 t4 = cross(v1.BtoA, a1);
                float gamma = dot(t4, normal) * inv_normal;
                t4 = cross(a2, v1.BtoA);
                float beta = dot(t4, normal) * inv_normal;
                float alpha = 1.0f - gamma - beta;
                point_a = add(add(smul(alpha, vert_a(v1)), smul(beta, vert_a(v2))), smul(gamma, vert_a(v3)));
                point_b = add(add(smul(alpha, v1.B), smul(beta, v2.B)), smul(gamma, v3.B));
            }
            return hit;
        }
        V3 t5 = cross(v4.BtoA, v0.BtoA);
        float dd = dot(t5, v1.BtoA);
        if (dd >= 0.0f) {
            dd = dot(t5, v2.BtoA);
            if (dd >= 0.0f) v1 = v4;
            else v3 = v4;
        } else {
            dd = dot(t5, v3.BtoA);
            if (dd >= 0.0f) v2 = v4;
            else v1 = v4;
        }
    }
}

static constexpr float GJK_EPS = 1e-8f;

struct Simplex {
    V3 v[8];
};

NB_D void gjk_segment(const Simplex& s, int i0, int i1, V3& closest, float* bc, unsigned& mask) {
    V3 a = s.v[2 * i0 + 1];
    V3 b = s.v[2 * i1 + 1];
    V3 edge = sub(b, a);
    float vsq = length_sq(edge);
    bool degenerate = vsq < GJK_EPS;
    float denom = degenerate ? GJK_EPS : vsq;
    float t = -dot(a, edge) / denom;
    float l0 = 1.0f - t;
    float l1 = t;
    mask = (1u << i0) | (1u << i1);
    bc[0] = bc[1] = bc[2] = bc[3] = 0.0f;
    if (l0 < 0.0f || degenerate) { mask = 1u << i1; l0 = 0.0f; l1 = 1.0f; }
    else if (l1 < 0.0f) { mask = 1u << i0; l0 = 1.0f; l1 = 0.0f; }
    bc[i0] = l0;
    bc[i1] = l1;
    closest = add(smul(l0, a), smul(l1, b));
}

__device__ __noinline__ void gjk_triangle(const Simplex& s, int i0, int i1, int i2, V3& closest, float* bc,
                                          unsigned& mask) {
    V3 a = s.v[2 * i0 + 1];
    V3 b = s.v[2 * i1 + 1];
    V3 c = s.v[2 * i2 + 1];
    V3 u = sub(a, b);
    V3 w = sub(a, c);
    V3 normal = cross(u, w);
    float t = length_sq(normal);
    bool degenerate = t < GJK_EPS;
    float denom = degenerate ? GJK_EPS : t;
    float it = 1.0f / denom;
    V3 c1 = cross(u, a);
    V3 c2 = cross(a, w);
    float l2 = dot(c1, normal) * it;
    float l1 = dot(c2, normal) * it;
    float l0 = 1.0f - l2 - l1;
    float best = 1e30f;
    V3 cp{0, 0, 0};
    float bcl[4] = {0, 0, 0, 0};
    unsigned m = 0;
    V3 cl;
    float bt[4];
    unsigned mt;
    if (l0 < 0.0f || degenerate) {
        gjk_segment(s, i1, i2, cl, bt, mt);
        float d = length_sq(cl);
        if (d < best) { bcl[0] = bt[0]; bcl[1] = bt[1]; bcl[2] = bt[2]; bcl[3] = bt[3]; m = mt; best = d; cp = cl; }
    }
    if (l1 < 0.0f || degenerate) {
        gjk_segment(s, i0, i2, cl, bt, mt);
        float d = length_sq(cl);
        if (d < best) { bcl[0] = bt[0]; bcl[1] = bt[1]; bcl[2] = bt[2]; bcl[3] = bt[3]; m = mt; best = d; cp = cl; }
    }
    if (l2 < 0.0f || degenerate) {
        gjk_segment(s, i0, i1, cl, bt, mt);
        float d = length_sq(cl);
        if (d < best) { bcl[0] = bt[0]; bcl[1] = bt[1]; bcl[2] = bt[2]; bcl[3] = bt[3]; m = mt; cp = cl; }
    }
    if (m != 0) {
        closest = cp;
        bc[0] = bcl[0]; bc[1] = bcl[1]; bc[2] = bcl[2]; bc[3] = bcl[3];
        mask = m;
        return;
    }
    bc[0] = bc[1] = bc[2] = bc[3] = 0.0f;
    bc[i0] = l0;
    bc[i1] = l1;
    bc[i2] = l2;
    mask = (1u << i0) | (1u << i1) | (1u << i2);
    closest = add(add(smul(l0, a), smul(l1, b)), smul(l2, c));
}

NB_D float det4(V3 a, V3 b, V3 c, V3 d) { return dot(sub(b, a), cross(sub(c, a), sub(d, a))); }

__device__ __noinline__ void gjk_tetra(const Simplex& s, V3& closest, float* bc, unsigned& mask) {
    V3 v0 = s.v[1], v1 = s.v[3], v2 = s.v[5], v3 = s.v[7];
    float det_t = det4(v0, v1, v2, v3);
    bool degenerate = fabsf(det_t) < GJK_EPS;
    float denom = degenerate ? GJK_EPS : det_t;
    float inv = 1.0f / denom;
    V3 z{0.0f, 0.0f, 0.0f};
    float ls[4];
    ls[0] = det4(z, v1, v2, v3) * inv;
    ls[1] = det4(v0, z, v2, v3) * inv;
    ls[2] = det4(v0, v1, z, v3) * inv;
    ls[3] = 1.0f - ls[0] - ls[1] - ls[2];
    float best = 1e30f;
    V3 cp{0, 0, 0};
    float bcl[4] = {0, 0, 0, 0};
    unsigned m = 0;
    V3 cl;
    float bt[4];
    unsigned mt;
#pragma unroll 1
    for (int f = 0; f < 4; ++f) {
        if (ls[f] < 0.0f || degenerate) {
            int t0 = f == 0 ? 1 : 0;
            int t1 = f <= 1 ? 2 : 1;
            int t2 = f <= 2 ? 3 : 2;
            gjk_triangle(s, t0, t1, t2, cl, bt, mt);
            float d = length_sq(cl);
            if (d < best) {
                bcl[0] = bt[0]; bcl[1] = bt[1]; bcl[2] = bt[2]; bcl[3] = bt[3];
                m = mt;
                if (f < 3) best = d;
                cp = cl;
            }
        }
    }
    if (m != 0) {
        closest = cp;
        bc[0] = bcl[0]; bc[1] = bcl[1]; bc[2] = bcl[2]; bc[3] = bcl[3];
        mask = m;
        return;
    }
    bc[0] = ls[0]; bc[1] = ls[1]; bc[2] = ls[2]; bc[3] = ls[3];
    mask = 15u;
    closest = z;
}

NB_D void simplex_closest(const Simplex& s, const float* bc, unsigned mask, V3& pa, V3& pb) {
    pa = V3{0, 0, 0};
    pb = V3{0, 0, 0};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if ((mask & (1u << i)) == 0) continue;
        V3 B = s.v[2 * i], BtoA = s.v[2 * i + 1];
        pa = add(pa, smul(bc[i], add(B, BtoA)));
        pb = add(pb, smul(bc[i], B));
    }
}

__device__ __noinline__ bool gjk_core(const Pair& p, float extend, V3& point_a, V3& point_b, V3& normal,
                                      float& distance) {
    const int MAX_ITER = 30;
    const float CE = 1e-4f;
    distance = 0.0f;
    point_a = V3{0, 0, 0};
    point_b = V3{0, 0, 0};
    normal = V3{0, 0, 0};
    Simplex s;
#pragma unroll
    for (int i = 0; i < 8; ++i) s.v[i] = V3{0, 0, 0};
    float bc[4] = {0, 0, 0, 0};
    unsigned mask = 0;
    int iter = MAX_ITER;
    Vert center = geometric_center(p);
    V3 v = center.BtoA;
    float dist_sq = length_sq(v);
    V3 last_dir{1.0f, 0.0f, 0.0f};
    while (iter > 0) {
        iter -= 1;
        if (dist_sq < CE * CE) {
            distance = 0.0f;
            normal = V3{0, 0, 0};
            simplex_closest(s, bc, mask, point_a, point_b);
            return false;
        }
        V3 search = neg(v);
        last_dir = search;
        Vert w = minkowski(p, search, extend);
        V3 wv = w.BtoA;
        float delta = dot(v, sub(v, wv));
        if (delta < CE * sqrtf(dist_sq)) break;
        bool dup = false;
        for (int i = 0; i < 4; ++i) {
            if (mask & (1u << i)) {
                if (length_sq(sub(s.v[2 * i + 1], wv)) < CE * CE) { dup = true; break; }
            }
        }
        if (dup) break;
        int use = 0, free_slot = 0;
        int idx[4] = {0, 0, 0, 0};
        for (int i = 0; i < 4; ++i) {
            if (mask & (1u << i)) { idx[use] = i; use += 1; }
            else free_slot = i;
        }
        idx[use] = free_slot;
        use += 1;
        s.v[2 * free_slot] = w.B;
        s.v[2 * free_slot + 1] = w.BtoA;
        V3 closest{0, 0, 0};
        bool success = true;
        if (use == 1) {
            closest = s.v[2 * idx[0] + 1];
            mask = 1u << idx[0];
            bc[idx[0]] = 1.0f;
        } else if (use == 2) {
            gjk_segment(s, idx[0], idx[1], closest, bc, mask);
        } else if (use == 3) {
            gjk_triangle(s, idx[0], idx[1], idx[2], closest, bc, mask);
        } else if (use == 4) {
            gjk_tetra(s, closest, bc, mask);
            success = !(mask == 15u);
        } else {
            success = false;
        }
        if (!success) {
            distance = 0.0f;
            normal = V3{0, 0, 0};
            simplex_closest(s, bc, mask, point_a, point_b);
            return false;
        }
        v = closest;
        dist_sq = length_sq(v);
    }
    distance = sqrtf(dist_sq);
    simplex_closest(s, bc, mask, point_a, point_b);
    V3 delta = sub(point_b, point_a);
    float dl = length_sq(delta);
    if (dl > GJK_EPS * GJK_EPS) normal = mul(delta, 1.0f / sqrtf(dl));
    else if (distance > CE) normal = mul(v, -1.0f / distance);
    else {
        float nsq = length_sq(last_dir);
        if (nsq > 0.0f) normal = mul(last_dir, 1.0f / sqrtf(nsq));
        else normal = V3{1.0f, 0.0f, 0.0f};
    }
    return true;
}

// ------------------------------------------------------------ manifold
struct V2 { float x, y; };
NB_D V2 v2sub(V2 a, V2 b) { return V2{a.x - b.x, a.y - b.y}; }
NB_D float v2lensq(V2 a) { return a.x * a.x + a.y * a.y; }
NB_D float signed_area(V2 a, V2 b, V2 q) { return (b.x - a.x) * (q.y - a.y) - (b.y - a.y) * (q.x - a.x); }

NB_D V3 ray_plane(V3 o, V3 dir, float pd, V3 pn) {
    float denom = dot(dir, pn);
    if (fabsf(denom) < 1.0e-12f) return o;
    float t = -(dot(o, pn) + pd) / denom;
    return add(o, mul(dir, t));
}

struct Proj { float d; V3 n; };
struct Tracker { V3 ref, prev, normal; float area; };

NB_D void tracker_update(Tracker& t, V3 p, int id) {
    if (id == 0) { t.ref = p; t.area = 0.0f; }
    else if (id == 1) { t.prev = p; }
    else {
        V3 e1 = sub(t.prev, t.ref);
        V3 e2 = sub(p, t.ref);
        V3 c = cross(e1, e2);
        float a = dot(c, c);
        if (a > t.area) { t.area = a; t.normal = c; }
        t.prev = p;
    }
}

NB_D V3 segment_projector_normal(V3 dir, V3 ref) {
    V3 right = cross(dir, ref);
    V3 n = cross(right, dir);
    float l = length(n);
    return l > 1.0e-12f ? divs(n, l) : ref;
}

NB_D void make_projectors(const Tracker& ta, V3 anchor_a, const Tracker& tb, V3 anchor_b, V3 cn, Proj& pa,
                          Proj& pb) {
    pa = Proj{0.0f, V3{0, 0, 0}};
    pb = Proj{0.0f, V3{0, 0, 0}};
    if (ta.area == 0.0f && tb.area == 0.0f) {
        V3 da = sub(ta.prev, ta.ref);
        V3 db = sub(tb.prev, tb.ref);
        V3 ppa = smul(0.5f, add(ta.ref, ta.prev));
        pa.n = segment_projector_normal(da, cn);
        pa.d = -dot(ppa, pa.n);
        V3 ppb = smul(0.5f, add(tb.ref, tb.prev));
        pb.n = segment_projector_normal(db, cn);
        pb.d = -dot(ppb, pb.n);
        return;
    }
    if (ta.area > 0.0f) {
        float l = sqrtf(fmaxw(1.0e-12f, ta.area));
        pa.n = divs(ta.normal, l);
        pa.d = -dot(anchor_a, pa.n);
    }
    if (tb.area > 0.0f) {
        float l = sqrtf(fmaxw(1.0e-12f, tb.area));
        pb.n = divs(tb.normal, l);
        pb.d = -dot(anchor_b, pb.n);
    }
    if (ta.area == 0.0f) {
        V3 d = sub(ta.prev, ta.ref);
        V3 pp = smul(0.5f, add(ta.ref, ta.prev));
        pa.n = segment_projector_normal(d, pb.n);
        pa.d = -dot(pp, pa.n);
    }
    if (tb.area == 0.0f) {
        V3 d = sub(tb.prev, tb.ref);
        V3 pp = smul(0.5f, add(tb.ref, tb.prev));
        pb.n = segment_projector_normal(d, pa.n);
        pb.d = -dot(pp, pb.n);
    }
}

NB_D V2 intersection_point(V2 s, V2 e, V2 a, V2 b) {
    float sa = signed_area(s, e, a);
    float sb = signed_area(s, e, b);
    float t = fabsf(sa) / fabsf(sa - sb);
    return V2{(1.0f - t) * a.x + t * b.x, (1.0f - t) * a.y + t * b.y};
}

// polygon of B at buf[0..], polygon of A aliased at buf[5..9] (multicontact.py:812-813)
static constexpr int MBUF = 16;

NB_D void insert_v2(V2* arr, int count, int index, V2 e) {
    int i = count;
    while (i > index) {
        if (i < MBUF) arr[i] = arr[i - 1];
        i -= 1;
    }
    if (index < MBUF) arr[index] = e;
}

__device__ __noinline__ int trim_in_place(V2 s, V2 e, V2* loop, int loop_count) {
    if (loop_count < 3) return loop_count;
    V2 ia{0, 0}, ib{0, 0};
    int change_a = -1, change_b = -1;
    bool keep = false;
    bool prev_out = signed_area(s, e, loop[0]) <= 0.0f;
    for (int i = 0; i < loop_count; ++i) {
        int nx = (i + 1) % loop_count;
        bool out = signed_area(s, e, loop[nx]) <= 0.0f;
        if (out != prev_out) {
            V2 ip = intersection_point(s, e, loop[i], loop[nx]);
            if (change_a < 0) { change_a = i; keep = !prev_out; ia = ip; }
            else { change_b = i; ib = ip; }
        }
        prev_out = out;
    }
    int new_count;
    if (change_a >= 0 && change_b >= 0) {
        int li = -1;
        new_count = loop_count;
        int i = 0;
        while (i < loop_count && li < MBUF - 2) {
            if (keep) { li += 1; loop[li] = loop[i]; }
            if (i == change_a || i == change_b) {
                V2 pt = (i == change_a) ? ia : ib;
                if (li == i && !keep) {
                    li += 1;
                    insert_v2(loop, new_count, li, pt);
                    new_count += 1;
                    i += 1;
                    change_b += 1;
                    loop_count += 1;
                } else {
                    li += 1;
                    loop[li] = pt;
                }
                keep = !keep;
            }
            i += 1;
        }
        new_count = li + 1;
    } else if (prev_out) {
        new_count = 0;
    } else {
        new_count = loop_count;
    }
    return new_count;
}

NB_D int trim_all(V2* trim, int trim_count, V2* loop, int loop_count) {
    if (trim_count <= 1) return loop_count < 1 ? loop_count : 1;
    const float move = 1e-5f;
    if (trim_count == 2) {
        V2 p0 = trim[0], p1 = trim[1];
        float dx = p1.x - p0.x, dy = p1.y - p0.y;
        float dl = sqrtf(dx * dx + dy * dy);
        if (dl > 1e-10f) {
            float px = -dy / dl, py = dx / dl;
            float ox = px * move, oy = py * move;
            trim[0] = V2{p0.x - ox, p0.y - oy};
            trim[1] = V2{p1.x - ox, p1.y - oy};
            trim[2] = V2{p1.x + ox, p1.y + oy};
            trim[3] = V2{p0.x + ox, p0.y + oy};
            trim_count = 4;
        } else {
            return loop_count < 1 ? loop_count : 1;
        }
    }
    if (loop_count == 2) {
        V2 p0 = loop[0], p1 = loop[1];
        float dx = p1.x - p0.x, dy = p1.y - p0.y;
        float dl = sqrtf(dx * dx + dy * dy);
        if (dl > 1e-10f) {
            float px = -dy / dl, py = dx / dl;
            float ox = px * move, oy = py * move;
            loop[0] = V2{p0.x - ox, p0.y - oy};
            loop[1] = V2{p1.x - ox, p1.y - oy};
            loop[2] = V2{p1.x + ox, p1.y + oy};
            loop[3] = V2{p0.x + ox, p0.y + oy};
            loop_count = 4;
        } else {
            return loop_count < 1 ? loop_count : 1;
        }
    }
    int cur = loop_count;
    V2 t0 = trim[0];
    for (int i = 0; i < trim_count; ++i) {
        V2 s = trim[i];
        V2 e = (i == trim_count - 1) ? t0 : trim[i + 1];
        cur = trim_in_place(s, e, loop, cur);
    }
    return cur;
}

NB_D void calipers(const V2* hull, int n, int* res) {
    int p1 = 0, p3 = 1;
    V2 d0 = v2sub(hull[p1], hull[p3]);
    float max_d = d0.x * d0.x + d0.y * d0.y;
    const float tie = 1.0e-3f;
    int j = 1;
    for (int i = 0; i < n; ++i) {
        V2 hi = hull[i], hi1 = hull[(i + 1) % n];
        for (int guard = 0; guard < 64; ++guard) {
            V2 hj = hull[j], hj1 = hull[(j + 1) % n];
            float a1 = signed_area(hi, hi1, hj1);
            float a0 = signed_area(hi, hi1, hj);
            if (a1 > a0) j = (j + 1) % n;
            else break;
        }
        V2 hj = hull[j];
        V2 d1 = V2{hull[i].x - hj.x, hull[i].y - hj.y};
        float ds1 = d1.x * d1.x + d1.y * d1.y;
        if (ds1 > max_d * (1.0f + tie)) { max_d = ds1; p1 = i; p3 = j; }
        V2 hip = hull[(i + 1) % n];
        V2 d2 = V2{hip.x - hj.x, hip.y - hj.y};
        float ds2 = d2.x * d2.x + d2.y * d2.y;
        if (ds2 > max_d * (1.0f + tie)) { max_d = ds2; p1 = (i + 1) % n; p3 = j; }
    }
    int p2 = 0, p4 = 0;
    float ma1 = 0.0f, ma2 = 0.0f;
    V2 hp1 = hull[p1], hp3 = hull[p3];
    for (int i = 0; i < n; ++i) {
        float a = signed_area(hp1, hp3, hull[i]);
        if (a > ma1 * (1.0f + tie)) { ma1 = a; p2 = i; }
        else if (-a > ma2 * (1.0f + tie)) { ma2 = -a; p4 = i; }
    }
    res[0] = p1; res[1] = p2; res[2] = p3; res[3] = p4;
}

NB_D int remove_zero_edges(V2* loop, int n, float eps) {
    if (n < 2) return 0;
    int w = 0;
    for (int r = 1; r < n; ++r) {
        V2 d = v2sub(loop[r], loop[w]);
        if (v2lensq(d) > eps) { w += 1; loop[w] = loop[r]; }
    }
    int nc;
    if (w > 0) {
        V2 d = v2sub(loop[w], loop[0]);
        nc = v2lensq(d) < eps ? w : w + 1;
    } else {
        nc = w + 1;
    }
    if (nc < 2) nc = 0;
    return nc;
}

NB_D int add_unique(V2* arr, int count, V2 v, float eps, bool& added) {
    if (count > 0 && v2lensq(v2sub(arr[0], v)) < eps) { added = false; return count; }
    if (count > 1 && v2lensq(v2sub(arr[count - 1], v)) < eps) { added = false; return count; }
    arr[count] = v;
    added = true;
    return count + 1;
}

NB_D void orthonormal_basis(V3 n, V3& b1, V3& b2) {
    if (n.z < 0.0f) {
        float a = 1.0f / (1.0f - n.z);
        float b = n.x * n.y * a;
        b1 = V3{1.0f - n.x * n.x * a, -b, n.x};
        b2 = V3{b, n.y * n.y * a - 1.0f, -n.y};
    } else {
        float a = 1.0f / (1.0f + n.z);
        float b = -n.x * n.y * a;
        b1 = V3{1.0f - n.x * n.x * a, b, -n.x};
        b2 = V3{b, 1.0f - n.y * n.y * a, -n.y};
    }
}

NB_D void post_process(ContactData& c, int type_a, int type_b) {
    V3 n = c.normal;
    if (type_a == NB_GEO_SPHERE || type_a == NB_GEO_CAPSULE) {
        c.center = add(c.center, mul(n, c.reff_a * 0.5f));
        c.dist = c.dist - c.reff_a;
    }
    if (type_b == NB_GEO_SPHERE || type_b == NB_GEO_CAPSULE) {
        c.center = sub(c.center, mul(n, c.reff_b * 0.5f));
        c.dist = c.dist - c.reff_b;
    }
}

__device__ __noinline__ void build_manifold(Writer& w, const Pair& p, Q4 qa, V3 pa_w, V3 p_a, V3 p_b, V3 normal,
                                            const ContactData& tmpl) {
    const float EPS = 0.00001f;
    int a_count = 0, b_count = 0;
    V3 ta, tb;
    orthonormal_basis(normal, ta, tb);
    Tracker tra, trb;
    tra.area = 0.0f; trb.area = 0.0f;
    tra.ref = tra.prev = tra.normal = V3{0, 0, 0};
    trb.ref = trb.prev = trb.normal = V3{0, 0, 0};
    V3 center = smul(0.5f, add(p_a, p_b));
    V2 buf[MBUF];
#pragma unroll
    for (int i = 0; i < MBUF; ++i) buf[i] = V2{0.0f, 0.0f};
    V2* bbuf = buf;
    V2* abuf = buf + 5;
    V3 lnb = qrot_inv(p.ob, neg(normal));
    V3 ltab = qrot_inv(p.ob, neg(ta));
    V3 ltbb = qrot_inv(p.ob, neg(tb));
    for (int e = 0; e < 5; ++e) {
        float c = pent_c(e), s = pent_s(e);
        float c_sin = c * SIN_TILT;
        float s_sin = s * SIN_TILT;
        V3 dir_a = add(add(mul(normal, COS_TILT), smul(c_sin, ta)), smul(s_sin, tb));
        V3 pa3 = support(p.a, dir_a);
        V3 proj_a = sub(pa3, center);
        V2 pa2{dot(ta, proj_a), dot(tb, proj_a)};
        bool added;
        a_count = add_unique(abuf, a_count, pa2, EPS, added);
        if (added) tracker_update(tra, pa3, a_count - 1);
        V3 ldb = add(add(mul(lnb, COS_TILT), smul(c_sin, ltab)), smul(s_sin, ltbb));
        V3 pbl = support(p.b, ldb);
        V3 pb3 = add(qrot(p.ob, pbl), p.pb);
        V3 proj_b = sub(pb3, center);
        V2 pb2{dot(ta, proj_b), dot(tb, proj_b)};
        b_count = add_unique(bbuf, b_count, pb2, EPS, added);
        if (added) tracker_update(trb, pb3, b_count - 1);
    }
    V3 normal_world = qrot(qa, normal);
    int count_out;
    float normal_dot;
    if (a_count < 2 || b_count < 2) {
        count_out = 0;
        normal_dot = 0.0f;
    } else {
        Proj pja, pjb;
        make_projectors(tra, p_a, trb, p_b, normal, pja, pjb);
        bool dev_a = fabsf(dot(normal, pja.n)) < COS_TILT;
        bool dev_b = fabsf(dot(normal, pjb.n)) < COS_TILT;
        if (dev_a || dev_b) {
            count_out = 0;
            normal_dot = 0.0f;
        } else {
            normal_dot = fabsf(dot(pja.n, pjb.n));
            int loop_count = trim_all(abuf, a_count, bbuf, b_count);
            loop_count = remove_zero_edges(bbuf, loop_count, EPS);
            if (loop_count > 1) {
                int res[4] = {0, 1, 2, 3};
                if (loop_count > 4) {
                    calipers(bbuf, loop_count, res);
                    loop_count = 4;
                }
                for (int i = 0; i < loop_count; ++i) {
                    int ia = res[i];
                    V3 pl = add(add(smul(bbuf[ia].x, ta), smul(bbuf[ia].y, tb)), center);
                    V3 a = ray_plane(pl, normal, pja.d, pja.n);
                    V3 b = ray_plane(pl, normal, pjb.d, pjb.n);
                    V3 cpl = smul(0.5f, add(a, b));
                    float sd = dot(sub(b, a), normal);
                    V3 cpw = add(qrot(qa, cpl), pa_w);
                    ContactData cd = tmpl;
                    cd.center = cpw;
                    cd.normal = normal_world;
                    cd.dist = sd;
                    cd.sub_key = (tmpl.sub_key << 3) | i;
                    post_process(cd, p.a.type, p.b.type);
                    write_contact(w, cd, true);
                }
            } else {
                normal_dot = 0.0f;
                loop_count = 0;
            }
            count_out = loop_count < 4 ? loop_count : 4;
        }
    }
    if (normal_dot < COS_DEEPEST || count_out == 0) {
        V3 dcl = smul(0.5f, add(p_a, p_b));
        float dsd = dot(sub(p_b, p_a), normal);
        V3 dcw = add(qrot(qa, dcl), pa_w);
        ContactData cd = tmpl;
        cd.center = dcw;
        cd.normal = normal_world;
        cd.dist = dsd;
        cd.sub_key = (tmpl.sub_key << 3) | count_out;
        post_process(cd, p.a.type, p.b.type);
        write_contact(w, cd, true);
    }
}

NB_D void plane_to_cube(Q4 pq, V3 ppos, V3 other, float other_radius, Shape& out, V3& adj) {
    out.type = NB_GEO_BOX;
    float lateral = other_radius * 10.0f;
    float depth = other_radius * 10.0f;
    out.scale = V3{lateral, lateral, depth};
    V3 n = qrot(pq, V3{0.0f, 0.0f, 1.0f});
    V3 to_other = sub(other, ppos);
    float dn = dot(to_other, n);
    V3 surf = sub(other, mul(n, dn));
    adj = sub(surf, mul(n, depth));
}

// Everything of the reference's MPR/GJK pair routine (narrow_phase.py:598-720
// with multicontact.py) that precedes MPR: the infinite-plane rejection and
// plane-as-cube substitution, the small-radius stand-ins for spheres and
// capsules, the contact template, the relative frame and MPR's enlargement.
// A pure function of the two geometries, so the manifold stage recomputes it
// instead of storing it.
struct GjkSetup {
    Pair p;
    Q4 qa;
    V3 pa;
    ContactData tmpl;
    float threshold;
    float enlarge;
    bool skip_multi;
};

// false: the pair produces nothing (two infinite planes, or an infinite plane
// beyond the other shape's bounding sphere)
NB_D bool gjk_prepare(const Geom& ga, const Geom& gb, GjkSetup& s) {
    bool inf_a = ga.type == NB_GEO_PLANE && ga.scale.x == 0.0f && ga.scale.y == 0.0f;
    bool inf_b = gb.type == NB_GEO_PLANE && gb.scale.x == 0.0f && gb.scale.y == 0.0f;
    if (inf_a && inf_b) return false;
    float bra = 0.0f, brb = 0.0f;
    if (inf_a || inf_b) {
        V3 ca = smul(0.5f, add(ga.lo, ga.hi));
        bra = length(smul(0.5f, sub(ga.hi, ga.lo)));
        V3 cb = smul(0.5f, add(gb.lo, gb.hi));
        brb = length(smul(0.5f, sub(gb.hi, gb.lo)));
        V3 ppos, oc;
        Q4 pq;
        float orad;
        if (inf_a) { ppos = ga.xf.p; pq = ga.xf.q; oc = cb; orad = brb; }
        else { ppos = gb.xf.p; pq = gb.xf.q; oc = ca; orad = bra; }
        V3 pn = qrot(pq, V3{0.0f, 0.0f, 1.0f});
        float cdist = dot(sub(oc, ppos), pn);
        if (!(cdist <= orad)) return false;
    }
    float gap_sum = ga.gap + gb.gap;
    Shape A{ga.type, ga.scale}, B{gb.type, gb.scale};
    V3 pa = ga.xf.p, pb = gb.xf.p;
    Q4 qa = ga.xf.q, qb = gb.xf.q;
    if (inf_a) plane_to_cube(qa, ga.xf.p, gb.xf.p, brb + gap_sum, A, pa);
    if (inf_b) plane_to_cube(qb, gb.xf.p, ga.xf.p, bra + gap_sum, B, pb);
    float reff_a = 0.0f, reff_b = 0.0f;
    const float small_radius = 0.0001f;
    if (A.type == NB_GEO_SPHERE || A.type == NB_GEO_CAPSULE) { reff_a = A.scale.x; A.scale.x = small_radius; }
    if (B.type == NB_GEO_SPHERE || B.type == NB_GEO_CAPSULE) { reff_b = B.scale.x; B.scale.x = small_radius; }
    ContactData& tmpl = s.tmpl;
    tmpl.reff_a = reff_a;
    tmpl.reff_b = reff_b;
    tmpl.margin_a = ga.margin;
    tmpl.margin_b = gb.margin;
    tmpl.gap_sum = gap_sum;
    tmpl.sub_key = 0;
    tmpl.center = V3{0, 0, 0};
    tmpl.normal = V3{0, 0, 0};
    tmpl.dist = 0.0f;
    s.threshold = gap_sum + reff_a + reff_b + ga.margin + gb.margin;
    s.skip_multi = A.type == NB_GEO_SPHERE || B.type == NB_GEO_SPHERE;
    s.p.a = A;
    s.p.b = B;
    s.p.ob = qmul(qinv(qa), qb);
    s.p.pb = qrot_inv(qa, sub(pb, pa));
    s.qa = qa;
    s.pa = pa;
    float margin_sum = tmpl.margin_a + tmpl.margin_b;
    const float eps = 1.0e-4f;
    if (margin_sum <= 0.0f) s.enlarge = eps;
    else if (margin_sum < eps) s.enlarge = 2.0f * eps;
    else s.enlarge = 0.0f;
    return true;
}

// MPR, then GJK when MPR finds no overlap.  Returns true when the pair still
// needs its manifold (build_manifold from the returned witness points and
// normal, in the pair's relative frame); false when it is finished -- rejected
// early, or its single contact (spheres, or a distance beyond the threshold)
// already written.
__device__ __noinline__ bool gjk_stage(Writer& w, const Geom& ga, const Geom& gb, V3& point_a, V3& point_b,
                                       V3& normal) {
    GjkSetup s;
    if (!gjk_prepare(ga, gb, s)) return false;
    float pen, sd;
    bool collision = mpr_core(s.p, s.enlarge, point_a, point_b, normal, pen);
    if (collision) {
        sd = -pen + s.enlarge;
        float he = s.enlarge * 0.5f;
        point_a = sub(point_a, mul(normal, he));
        point_b = add(point_b, mul(normal, he));
    } else {
        gjk_core(s.p, 0.0f, point_a, point_b, normal, sd);
    }
    if (s.skip_multi || sd > s.threshold) {
        V3 pt = smul(0.5f, add(point_a, point_b));
        pt = add(qrot(s.qa, pt), s.pa);
        V3 nws = qrot(s.qa, normal);
        ContactData cd = s.tmpl;
        cd.center = pt;
        cd.normal = nws;
        cd.dist = sd;
        cd.sub_key = s.tmpl.sub_key << 3;
        post_process(cd, s.p.a.type, s.p.b.type);
        write_contact(w, cd, true);
        return false;
    }
    return true;
}

// the manifold of a pair gjk_stage left unfinished, from its witness points and normal
__device__ __noinline__ void gjk_manifold(Writer& w, const Geom& ga, const Geom& gb, V3 point_a, V3 point_b,
                                          V3 normal) {
    GjkSetup s;
    if (!gjk_prepare(ga, gb, s)) return;  // never: the stage passed the same test
    build_manifold(w, s.p, s.qa, s.pa, point_a, point_b, normal, s.tmpl);
}

// narrow_phase_primitive_kernel body for one pair (type_a <= type_b).
// Returns false when the pair falls through to MPR/GJK (no analytic branch
// produced a finite distance, narrow_phase.py:598-603).
__device__ __forceinline__ bool narrow_analytic(Writer& w, const Geom& ga, const Geom& gb) {
    int ta = ga.type, tb = gb.type;
    V3 sca = ga.scale, scb = gb.scale;
    V3 pos_a = ga.xf.p, pos_b = gb.xf.p;
    Q4 qa = ga.xf.q, qb = gb.xf.q;
    float gap_sum = ga.gap + gb.gap;
    bool plane_a = ta == NB_GEO_PLANE;
    bool sph_a = ta == NB_GEO_SPHERE, sph_b = tb == NB_GEO_SPHERE;
    bool cap_a = ta == NB_GEO_CAPSULE, cap_b = tb == NB_GEO_CAPSULE;
    bool box_b = tb == NB_GEO_BOX;
    float reff_a = (sph_a || cap_a) ? sca.x : 0.0f;
    float reff_b = (sph_b || cap_b) ? scb.x : 0.0f;
    float dist[4] = {MAXVAL, MAXVAL, MAXVAL, MAXVAL};
    V3 pos[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    V3 normal{0, 0, 0};
    if (plane_a && sph_b) {
        V3 pn = qrot(qa, V3{0.0f, 0.0f, 1.0f});
        collide_plane_sphere(pn, pos_a, pos_b, scb.x, dist[0], pos[0]);
        normal = pn;
    } else if (plane_a && box_b) {
        V3 pn = qrot(qa, V3{0.0f, 0.0f, 1.0f});
        M33 rot = quat_to_matrix(qb);
        collide_plane_box(pn, pos_a, pos_b, rot, scb, gap_sum, dist, pos);
        normal = pn;
    } else if (sph_a && sph_b) {
        collide_sphere_sphere(pos_a, sca.x, pos_b, scb.x, dist[0], pos[0], normal);
    } else if (plane_a && cap_b) {
        V3 pn = qrot(qa, V3{0.0f, 0.0f, 1.0f});
        V3 ax = qrot(qb, V3{0.0f, 0.0f, 1.0f});
        V3 seg = mul(ax, scb.y);
        collide_plane_sphere(pn, pos_a, add(pos_b, seg), scb.x, dist[0], pos[0]);
        collide_plane_sphere(pn, pos_a, sub(pos_b, seg), scb.x, dist[1], pos[1]);
        normal = pn;
    } else if (sph_a && cap_b) {
        V3 ax = qrot(qb, V3{0.0f, 0.0f, 1.0f});
        V3 seg = mul(ax, scb.y);
        V3 pt = closest_segment_point(sub(pos_b, seg), add(pos_b, seg), pos_a);
        collide_sphere_sphere(pos_a, sca.x, pt, scb.x, dist[0], pos[0], normal);
    } else if (cap_a && cap_b) {
        V3 ax1 = qrot(qa, V3{0.0f, 0.0f, 1.0f});
        V3 ax2 = qrot(qb, V3{0.0f, 0.0f, 1.0f});
        collide_capsule_capsule(pos_a, ax1, sca.x, sca.y, pos_b, ax2, scb.x, scb.y, dist, pos, normal);
    } else if (sph_a && box_b) {
        M33 rot = quat_to_matrix(qb);
        collide_sphere_box(pos_a, sca.x, pos_b, rot, scb, dist[0], pos[0], normal);
    }
    int num = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) num += dist[i] < MAXVAL ? 1 : 0;
    if (num > 0) {
        ContactData cd;
        cd.normal = normal;
        cd.reff_a = reff_a;
        cd.reff_b = reff_b;
        cd.margin_a = ga.margin;
        cd.margin_b = gb.margin;
        cd.gap_sum = gap_sum;
        cd.sub_key = 0;
        bool valid[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            valid[i] = false;
            if (dist[i] < MAXVAL) {
                cd.center = pos[i];
                cd.dist = dist[i];
                valid[i] = passes_gap(cd);
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (!valid[i]) continue;
            cd.center = pos[i];
            cd.dist = dist[i];
            cd.sub_key = i;
            write_contact(w, cd, false);
        }
        return true;
    }
    return false;
}

}  // namespace nbg
