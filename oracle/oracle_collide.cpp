// TEST INFRASTRUCTURE ONLY -- CPU oracle of Newton's rigid collision pipeline.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it.
//
// Sequential restatement, per world, of:
//   compute_shape_aabbs            newton/_src/sim/collide.py:150-275
//   BroadPhaseExplicit AABB test   newton/_src/geometry/broad_phase_nxn.py:28-66,
//                                  newton/_src/geometry/broad_phase_common.py:18-35
//   narrow_phase_primitive_kernel  newton/_src/geometry/narrow_phase.py:153-603
//   narrow_phase_kernel_gjk_mpr    newton/_src/geometry/narrow_phase.py:627-776
//     find_contacts / plane proxy  newton/_src/geometry/collision_core.py:508-725
//     solve_convex_multi_contact   newton/_src/geometry/collision_convex.py:26-135
//     MPR                          newton/_src/geometry/mpr.py:56-504
//     GJK                          newton/_src/geometry/simplex_solver.py:44-491
//     build_manifold               newton/_src/geometry/multicontact.py:28-954
//     support maps                 newton/_src/geometry/support_function.py:106-305
//   write_contact                  newton/_src/sim/collide.py:62-147
// Contacts of a world are emitted in the deterministic key order
// (shape_a, shape_b, sort_sub_key) of contact_data.py:59-83 because the world's
// candidate pairs are visited in key order and each pair writes its contacts
// in ascending sub-key order.
#include "oracle_math.h"
#include "../include/newton_b200.h"

#include <cstring>
#include <vector>

namespace orc {

static const float MAXVAL = 1e10f;
static const float MINVAL = 0x1.203afap-50f;  // 1e-15
static const float SIN_TILT = 0x1.1de58cp-5f;
static const float COS_TILT = 0x1.ffb028p-1f;
static const float COS_DEEPEST = 0x1.ffffccp-1f;
static const float PENT_C[5] = {1.0f, 0x1.3c6ef4p-2f, -0x1.9e377ap-1f, -0x1.9e377ap-1f, 0x1.3c6ef4p-2f};
static const float PENT_S[5] = {0.0f, 0x1.e6f0e2p-1f, 0x1.2cf230p-1f, -0x1.2cf230p-1f, -0x1.e6f0e2p-1f};

struct Shape {  // GenericShapeData (support_function.py:83-104)
    int type;
    V3 scale;
};

// ---------------------------------------------------------------- support maps
// support_function.py:106-305 (box deadband :39,:175; sphere :189; capsule :198; plane :287)
static V3 support(const Shape& g, V3 d) {
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

// collision_core.py:396-491 (generic path: 6 support evaluations)
static void tight_aabb(const Shape& g, Q4 q, V3 pos, V3& lo, V3& hi) {
    M33 r = quat_to_matrix(q);
    // rows of r == columns of transpose(r)
    V3 lx{r.m[0][0], r.m[0][1], r.m[0][2]};
    V3 ly{r.m[1][0], r.m[1][1], r.m[1][2]};
    V3 lz{r.m[2][0], r.m[2][1], r.m[2][2]};
    float max_x = dot(lx, support(g, lx));
    float max_y = dot(ly, support(g, ly));
    float max_z = dot(lz, support(g, lz));
    float min_x = dot(lx, support(g, neg(lx)));
    float min_y = dot(ly, support(g, neg(ly)));
    float min_z = dot(lz, support(g, neg(lz)));
    lo = add(V3{min_x, min_y, min_z}, pos);
    hi = add(V3{max_x, max_y, max_z}, pos);
}

// ------------------------------------------------------------ world geometry
struct GeomWS {        // per shape, output of compute_shape_aabbs
    TF xf;             // geom_xform
    V3 scale;          // geom_data.xyz
    float margin;      // geom_data.w
    V3 lo, hi;         // expanded AABB
    int type;
    float gap;
    int body;
};

static GeomWS compute_geom(const NbModelDesc* m, const float* body_q, int s) {
    GeomWS g;
    int b = m->shape_body[s];
    TF xs = load_tf(m->shape_transform + 7 * s);
    g.xf = (b == -1) ? xs : tf_mul(load_tf(body_q + 7 * b), xs);
    g.type = m->shape_type[s];
    g.body = b;
    g.gap = m->shape_gap[s];
    g.margin = m->shape_margin[s];
    float eff = g.margin + m->shape_gap[s];
    V3 mv3{eff, eff, eff};
    V3 scale = load_v3(m->shape_scale + 3 * s);
    bool inf_plane = g.type == NB_GEO_PLANE && scale.x == 0.0f && scale.y == 0.0f;
    g.scale = scale;
    if (inf_plane) {
        float rad = m->shape_radius[s];
        V3 he{rad, rad, rad};
        g.lo = sub(sub(g.xf.p, he), mv3);
        g.hi = add(add(g.xf.p, he), mv3);
    } else {
        if (g.type == NB_GEO_PLANE) g.scale = V3{scale.x * 0.5f, scale.y * 0.5f, 0.0f};
        Shape sh{g.type, g.scale};
        V3 lo, hi;
        tight_aabb(sh, g.xf.q, g.xf.p, lo, hi);
        g.lo = sub(lo, mv3);
        g.hi = add(hi, mv3);
    }
    return g;
}

// broad_phase_common.py:18-35 with zero cutoffs (AABBs are pre-expanded)
static bool aabb_overlap(const GeomWS& a, const GeomWS& b) {
    float c = 0.0f + 0.0f;
    return a.lo.x <= b.hi.x + c && a.hi.x >= b.lo.x - c && a.lo.y <= b.hi.y + c &&
           a.hi.y >= b.lo.y - c && a.lo.z <= b.hi.z + c && a.hi.z >= b.lo.z - c;
}

// ------------------------------------------------------------ contact writer
struct ContactData {   // contact_data.py:17-56
    V3 center;
    V3 normal;
    float dist;
    float reff_a, reff_b, margin_a, margin_b;
    int shape_a, shape_b;
    float gap_sum;
    int sub_key;
};

struct OutContact {
    V3 p0, p1, n, o0, o1;
    float m0, m1;
    int s0, s1, sub;
};

struct Writer {
    const NbModelDesc* m;
    const float* body_q;
    std::vector<OutContact>* out;
};

// contact_data.py:86-117
static bool passes_gap(const ContactData& c) {
    float total = c.reff_a + c.reff_b + c.margin_a + c.margin_b;
    V3 n = normalize(c.normal);
    V3 a = sub(c.center, mul(n, 0.5f * c.dist + c.reff_a));
    V3 b = add(c.center, mul(n, 0.5f * c.dist + c.reff_b));
    float d = dot(sub(b, a), n) - total;
    return d <= c.gap_sum;
}

// collide.py:62-147; check_gap == (output_index < 0)
static void write_contact(const Writer& w, const ContactData& c, bool check_gap) {
    float total = c.reff_a + c.reff_b + c.margin_a + c.margin_b;
    float off_a = c.reff_a + c.margin_a;
    float off_b = c.reff_b + c.margin_b;
    V3 n = normalize(c.normal);
    V3 a_w = sub(c.center, mul(n, 0.5f * c.dist + c.reff_a));
    V3 b_w = add(c.center, mul(n, 0.5f * c.dist + c.reff_b));
    float d = dot(sub(b_w, a_w), n) - total;
    float gap = w.m->shape_gap[c.shape_a] + w.m->shape_gap[c.shape_b];
    if (check_gap && d > gap) return;
    int b0 = w.m->shape_body[c.shape_a];
    int b1 = w.m->shape_body[c.shape_b];
    TF xa = b0 == -1 ? tf_identity() : tf_inverse(load_tf(w.body_q + 7 * b0));
    TF xb = b1 == -1 ? tf_identity() : tf_inverse(load_tf(w.body_q + 7 * b1));
    OutContact o;
    o.p0 = tf_point(xa, a_w);
    o.p1 = tf_point(xb, b_w);
    o.o0 = tf_vector(xa, mul(n, off_a));
    o.o1 = tf_vector(xb, mul(n, -off_b));
    o.n = n;
    o.m0 = off_a;
    o.m1 = off_b;
    o.s0 = c.shape_a;
    o.s1 = c.shape_b;
    o.sub = c.sub_key;
    w.out->push_back(o);
}

// ------------------------------------------------------------ primitives
// collision_primitive.py:48-439, 1161-1215
static V3 closest_segment_point(V3 a, V3 b, V3 pt) {
    V3 ab = sub(b, a);
    float t = dot(sub(pt, a), ab) / (dot(ab, ab) + 1e-6f);
    return add(a, smul(clampw(t, 0.0f, 1.0f), ab));
}

static void collide_plane_sphere(V3 n, V3 ppos, V3 spos, float r, float& dist, V3& pos) {
    dist = dot(sub(spos, ppos), n) - r;
    pos = sub(spos, mul(n, r + 0.5f * dist));
}

static void collide_sphere_sphere(V3 p1, float r1, V3 p2, float r2, float& dist, V3& pos, V3& n) {
    V3 dir = sub(p2, p1);
    dist = length(dir);
    if (dist == 0.0f) n = V3{1.0f, 0.0f, 0.0f};
    else n = divs(dir, dist);
    dist = dist - (r1 + r2);
    pos = add(p1, mul(n, r1 + 0.5f * dist));
}

static void collide_capsule_capsule(V3 p1, V3 ax1, float r1, float h1, V3 p2, V3 ax2, float r2, float h2,
                                    float dist[2], V3 pos[2], V3& normal) {
    dist[0] = MAXVAL; dist[1] = MAXVAL;
    pos[0] = V3{0, 0, 0}; pos[1] = V3{0, 0, 0};
    normal = V3{0, 0, 0};
    V3 axis1 = mul(ax1, h1);
    V3 axis2 = mul(ax2, h2);
    V3 dif = sub(p1, p2);
    float ma = dot(axis1, axis1);
    float mb = -dot(axis1, axis2);
    float mc = dot(axis2, axis2);
    float u = -dot(axis1, dif);
    float v = dot(axis2, dif);
    float det = ma * mc - mb * mb;
    if (std::fabs(det) >= MINVAL) {
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

static void collide_plane_box(V3 n, V3 ppos, V3 bpos, const M33& rot, V3 size, float margin,
                              float dist[4], V3 pos[4]) {
    float center_dist = dot(sub(bpos, ppos), n);
    for (int i = 0; i < 4; ++i) { dist[i] = MAXVAL; pos[i] = V3{0, 0, 0}; }
    int ncontact = 0, worst = 0;
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

static void collide_sphere_box(V3 spos, float r, V3 bpos, const M33& rot, V3 size, float& dist, V3& pos,
                               V3& normal) {
    V3 center = mtv(rot, sub(spos, bpos));
    V3 clamped = vmax(neg(size), vmin(size, center));
    V3 cd = sub(clamped, center);
    float d = length(cd);
    V3 cdir = (d == 0.0f) ? cd : divs(cd, d);
    V3 lpos;
    if (d <= 1e-6f) {
        float closest = 2.0f * (size.x + size.y + size.z);
        int k = 0;
        for (int i = 0; i < 6; ++i) {
            float sgn = (i % 2) ? 1.0f : -1.0f;
            float face = std::fabs(sgn * comp(size, i / 2) - comp(center, i / 2));
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
static inline V3 vert_a(const Vert& v) { return add(v.B, v.BtoA); }

struct Pair {          // geometry of a GJK/MPR pair in A's frame
    Shape a, b;
    Q4 ob;             // orientation of B relative to A
    V3 pb;             // position of B relative to A (A frame)
};

// mpr.py:60-90
static V3 support_b(const Pair& p, V3 dir) {
    V3 tmp = qrot_inv(p.ob, dir);
    V3 r = support(p.b, tmp);
    r = qrot(p.ob, r);
    return add(r, p.pb);
}

// mpr.py:92-125
static Vert minkowski(const Pair& p, V3 dir, float extend) {
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

// mpr.py:127-214 (primitive shapes: both local centres are the origin)
static Vert geometric_center(const Pair& p) {
    Vert c;
    V3 center_a{0.0f, 0.0f, 0.0f};
    V3 cbw = add(p.pb, qrot(p.ob, V3{0.0f, 0.0f, 0.0f}));
    c.B = cbw;
    c.BtoA = sub(center_a, cbw);
    return c;
}

// mpr.py:240-504
static bool mpr_core(const Pair& p, float extend, V3& point_a, V3& point_b, V3& normal, float& penetration) {
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
                float inv_normal = 1.0f / std::sqrt(normal_sq);
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

// simplex_solver.py:44-491
static const float GJK_EPS = 1e-8f;

struct Simplex {
    V3 v[8];           // v[2i] = B, v[2i+1] = BtoA
};

static void gjk_segment(const Simplex& s, int i0, int i1, V3& closest, float bc[4], uint32_t& mask) {
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
    for (int i = 0; i < 4; ++i) bc[i] = 0.0f;
    if (l0 < 0.0f || degenerate) { mask = 1u << i1; l0 = 0.0f; l1 = 1.0f; }
    else if (l1 < 0.0f) { mask = 1u << i0; l0 = 1.0f; l1 = 0.0f; }
    bc[i0] = l0;
    bc[i1] = l1;
    closest = add(smul(l0, a), smul(l1, b));
}

static void gjk_triangle(const Simplex& s, int i0, int i1, int i2, V3& closest, float bc[4], uint32_t& mask) {
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
    uint32_t m = 0;
    V3 cl; float bt[4]; uint32_t mt;
    if (l0 < 0.0f || degenerate) {
        gjk_segment(s, i1, i2, cl, bt, mt);
        float d = length_sq(cl);
        if (d < best) { for (int i = 0; i < 4; ++i) bcl[i] = bt[i]; m = mt; best = d; cp = cl; }
    }
    if (l1 < 0.0f || degenerate) {
        gjk_segment(s, i0, i2, cl, bt, mt);
        float d = length_sq(cl);
        if (d < best) { for (int i = 0; i < 4; ++i) bcl[i] = bt[i]; m = mt; best = d; cp = cl; }
    }
    if (l2 < 0.0f || degenerate) {
        gjk_segment(s, i0, i1, cl, bt, mt);
        float d = length_sq(cl);
        if (d < best) { for (int i = 0; i < 4; ++i) bcl[i] = bt[i]; m = mt; cp = cl; }
    }
    if (m != 0) {
        closest = cp;
        for (int i = 0; i < 4; ++i) bc[i] = bcl[i];
        mask = m;
        return;
    }
    for (int i = 0; i < 4; ++i) bc[i] = 0.0f;
    bc[i0] = l0; bc[i1] = l1; bc[i2] = l2;
    mask = (1u << i0) | (1u << i1) | (1u << i2);
    closest = add(add(smul(l0, a), smul(l1, b)), smul(l2, c));
}

static float det4(V3 a, V3 b, V3 c, V3 d) { return dot(sub(b, a), cross(sub(c, a), sub(d, a))); }

static void gjk_tetra(const Simplex& s, V3& closest, float bc[4], uint32_t& mask) {
    V3 v0 = s.v[1], v1 = s.v[3], v2 = s.v[5], v3 = s.v[7];
    float det_t = det4(v0, v1, v2, v3);
    bool degenerate = std::fabs(det_t) < GJK_EPS;
    float denom = degenerate ? GJK_EPS : det_t;
    float inv = 1.0f / denom;
    V3 z{0.0f, 0.0f, 0.0f};
    float l0 = det4(z, v1, v2, v3) * inv;
    float l1 = det4(v0, z, v2, v3) * inv;
    float l2 = det4(v0, v1, z, v3) * inv;
    float l3 = 1.0f - l0 - l1 - l2;
    float best = 1e30f;
    V3 cp{0, 0, 0};
    float bcl[4] = {0, 0, 0, 0};
    uint32_t m = 0;
    V3 cl; float bt[4]; uint32_t mt;
    const int tri[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    const float ls[4] = {l0, l1, l2, l3};
    for (int f = 0; f < 4; ++f) {
        if (ls[f] < 0.0f || degenerate) {
            gjk_triangle(s, tri[f][0], tri[f][1], tri[f][2], cl, bt, mt);
            float d = length_sq(cl);
            if (d < best) {
                for (int i = 0; i < 4; ++i) bcl[i] = bt[i];
                m = mt;
                if (f < 3) best = d;
                cp = cl;
            }
        }
    }
    if (m != 0) {
        closest = cp;
        for (int i = 0; i < 4; ++i) bc[i] = bcl[i];
        mask = m;
        return;
    }
    bc[0] = l0; bc[1] = l1; bc[2] = l2; bc[3] = l3;
    mask = 15u;
    closest = z;
}

static void simplex_closest(const Simplex& s, const float bc[4], uint32_t mask, V3& pa, V3& pb) {
    pa = V3{0, 0, 0};
    pb = V3{0, 0, 0};
    for (int i = 0; i < 4; ++i) {
        if ((mask & (1u << i)) == 0) continue;
        V3 B = s.v[2 * i], BtoA = s.v[2 * i + 1];
        pa = add(pa, smul(bc[i], add(B, BtoA)));
        pb = add(pb, smul(bc[i], B));
    }
}

// returns "separated"
static bool gjk_core(const Pair& p, float extend, V3& point_a, V3& point_b, V3& normal, float& distance) {
    const int MAX_ITER = 30;
    const float CE = 1e-4f;
    distance = 0.0f;
    point_a = V3{0, 0, 0};
    point_b = V3{0, 0, 0};
    normal = V3{0, 0, 0};
    Simplex s;
    for (int i = 0; i < 8; ++i) s.v[i] = V3{0, 0, 0};
    float bc[4] = {0, 0, 0, 0};
    uint32_t mask = 0;
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
        if (delta < CE * std::sqrt(dist_sq)) break;
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
    distance = std::sqrt(dist_sq);
    simplex_closest(s, bc, mask, point_a, point_b);
    V3 delta = sub(point_b, point_a);
    float dl = length_sq(delta);
    if (dl > GJK_EPS * GJK_EPS) normal = mul(delta, 1.0f / std::sqrt(dl));
    else if (distance > CE) normal = mul(v, -1.0f / distance);
    else {
        float nsq = length_sq(last_dir);
        if (nsq > 0.0f) normal = mul(last_dir, 1.0f / std::sqrt(nsq));
        else normal = V3{1.0f, 0.0f, 0.0f};
    }
    return true;
}

// ------------------------------------------------------------ manifold
// multicontact.py:28-954
struct V2 { float x, y; };
static inline V2 v2sub(V2 a, V2 b) { return V2{a.x - b.x, a.y - b.y}; }
static inline float v2lensq(V2 a) { return a.x * a.x + a.y * a.y; }

static float signed_area(V2 a, V2 b, V2 q) { return (b.x - a.x) * (q.y - a.y) - (b.y - a.y) * (q.x - a.x); }

static V3 ray_plane(V3 o, V3 dir, float pd, V3 pn) {
    float denom = dot(dir, pn);
    if (std::fabs(denom) < 1.0e-12f) return o;
    float t = -(dot(o, pn) + pd) / denom;
    return add(o, mul(dir, t));
}

struct Proj { float d; V3 n; };
struct Tracker { V3 ref, prev, normal; float area; };

static void tracker_update(Tracker& t, V3 p, int id) {
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

static V3 segment_projector_normal(V3 dir, V3 ref) {
    V3 right = cross(dir, ref);
    V3 n = cross(right, dir);
    float l = length(n);
    return l > 1.0e-12f ? divs(n, l) : ref;
}

static void make_projectors(const Tracker& ta, V3 anchor_a, const Tracker& tb, V3 anchor_b, V3 cn, Proj& pa,
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
        float l = std::sqrt(fmaxw(1.0e-12f, ta.area));
        pa.n = divs(ta.normal, l);
        pa.d = -dot(anchor_a, pa.n);
    }
    if (tb.area > 0.0f) {
        float l = std::sqrt(fmaxw(1.0e-12f, tb.area));
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

static V2 intersection_point(V2 s, V2 e, V2 a, V2 b) {
    float sa = signed_area(s, e, a);
    float sb = signed_area(s, e, b);
    float t = std::fabs(sa) / std::fabs(sa - sb);
    return V2{(1.0f - t) * a.x + t * b.x, (1.0f - t) * a.y + t * b.y};
}

// The manifold buffer: loop (polygon of B) at buf[0..], polygon of A aliased at
// buf[5..9] exactly as multicontact.py:812-813 does; sized with headroom.
static const int BUF = 16;

static void insert_v2(V2* arr, int count, int index, V2 e) {
    int i = count;
    while (i > index) {
        if (i < BUF) arr[i] = arr[i - 1];
        i -= 1;
    }
    if (index < BUF) arr[index] = e;
}

static int trim_in_place(V2 s, V2 e, V2* loop, int loop_count) {
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
        while (i < loop_count && li < BUF - 2) {
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

static int trim_all(V2* trim, int trim_count, V2* loop, int loop_count) {
    if (trim_count <= 1) return loop_count < 1 ? loop_count : 1;
    const float move = 1e-5f;
    if (trim_count == 2) {
        V2 p0 = trim[0], p1 = trim[1];
        float dx = p1.x - p0.x, dy = p1.y - p0.y;
        float dl = std::sqrt(dx * dx + dy * dy);
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
        float dl = std::sqrt(dx * dx + dy * dy);
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

static void calipers(const V2* hull, int n, int res[4]) {
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

static int remove_zero_edges(V2* loop, int n, float eps) {
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

static int add_unique(V2* arr, int count, V2 v, float eps, bool& added) {
    if (count > 0 && v2lensq(v2sub(arr[0], v)) < eps) { added = false; return count; }
    if (count > 1 && v2lensq(v2sub(arr[count - 1], v)) < eps) { added = false; return count; }
    arr[count] = v;
    added = true;
    return count + 1;
}

// math/__init__.py:236-272
static void orthonormal_basis(V3 n, V3& b1, V3& b2) {
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

// collision_core.py:144-169 (sphere/capsule Minkowski adjustment; the axial
// rolling branch of :172-275 only concerns cylinders and cones)
static void post_process(ContactData& c, int type_a, int type_b) {
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

struct GjkCtx {
    int type_a, type_b;  // original shape types (for post-processing)
    Q4 qa;               // world orientation of A
    V3 pa;               // world position of A (adjusted)
};

static int build_manifold(const Writer& w, const Pair& p, const GjkCtx& g, V3 p_a, V3 p_b, V3 normal,
                          const ContactData& tmpl) {
    const float EPS = 0.00001f;
    int a_count = 0, b_count = 0;
    V3 ta, tb;
    orthonormal_basis(normal, ta, tb);
    Tracker tra{}, trb{};
    tra.area = 0.0f; trb.area = 0.0f;
    tra.ref = tra.prev = tra.normal = V3{0, 0, 0};
    trb.ref = trb.prev = trb.normal = V3{0, 0, 0};
    V3 center = smul(0.5f, add(p_a, p_b));
    V2 buf[BUF];
    for (int i = 0; i < BUF; ++i) buf[i] = V2{0.0f, 0.0f};
    V2* bbuf = buf;
    V2* abuf = buf + 5;
    V3 lnb = qrot_inv(p.ob, neg(normal));
    V3 ltab = qrot_inv(p.ob, neg(ta));
    V3 ltbb = qrot_inv(p.ob, neg(tb));
    for (int e = 0; e < 5; ++e) {
        float c = PENT_C[e], s = PENT_S[e];
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
    V3 normal_world = qrot(g.qa, normal);
    int count_out;
    float normal_dot;
    if (a_count < 2 || b_count < 2) {
        count_out = 0;
        normal_dot = 0.0f;
    } else {
        Proj pja, pjb;
        make_projectors(tra, p_a, trb, p_b, normal, pja, pjb);
        bool dev_a = std::fabs(dot(normal, pja.n)) < COS_TILT;
        bool dev_b = std::fabs(dot(normal, pjb.n)) < COS_TILT;
        if (dev_a || dev_b) {
            count_out = 0;
            normal_dot = 0.0f;
        } else {
            // extract_4_point_contact_manifolds (multicontact.py:625-700)
            normal_dot = std::fabs(dot(pja.n, pjb.n));
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
                    V3 cpw = add(qrot(g.qa, cpl), g.pa);
                    ContactData cd = tmpl;
                    cd.center = cpw;
                    cd.normal = normal_world;
                    cd.dist = sd;
                    cd.sub_key = (tmpl.sub_key << 3) | i;
                    post_process(cd, g.type_a, g.type_b);
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
        V3 dcw = add(qrot(g.qa, dcl), g.pa);
        ContactData cd = tmpl;
        cd.center = dcw;
        cd.normal = normal_world;
        cd.dist = dsd;
        cd.sub_key = (tmpl.sub_key << 3) | count_out;
        post_process(cd, g.type_a, g.type_b);
        write_contact(w, cd, true);
        count_out += 1;
    }
    return count_out;
}

// collision_core.py:508-567
static void plane_to_cube(Q4 pq, V3 ppos, V3 other, float other_radius, Shape& out, V3& adj) {
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

// narrow_phase.py:627-776 for one pair (type_a <= type_b)
static void gjk_pair(const Writer& w, const GeomWS& ga, const GeomWS& gb, int sa, int sb) {
    bool inf_a = ga.type == NB_GEO_PLANE && ga.scale.x == 0.0f && ga.scale.y == 0.0f;
    bool inf_b = gb.type == NB_GEO_PLANE && gb.scale.x == 0.0f && gb.scale.y == 0.0f;
    if (inf_a && inf_b) return;
    float bra = 0.0f, brb = 0.0f;
    if (inf_a || inf_b) {
        V3 ca = smul(0.5f, add(ga.lo, ga.hi));
        bra = length(smul(0.5f, sub(ga.hi, ga.lo)));
        V3 cb = smul(0.5f, add(gb.lo, gb.hi));
        brb = length(smul(0.5f, sub(gb.hi, gb.lo)));
        // check_infinite_plane_bsphere_overlap (collision_core.py:570-620)
        V3 ppos, oc;
        Q4 pq;
        float orad;
        if (inf_a) { ppos = ga.xf.p; pq = ga.xf.q; oc = cb; orad = brb; }
        else { ppos = gb.xf.p; pq = gb.xf.q; oc = ca; orad = bra; }
        V3 pn = qrot(pq, V3{0.0f, 0.0f, 1.0f});
        float cdist = dot(sub(oc, ppos), pn);
        if (!(cdist <= orad)) return;
    }
    float gap_sum = ga.gap + gb.gap;
    Shape A{ga.type, ga.scale}, B{gb.type, gb.scale};
    V3 pa = ga.xf.p, pb = gb.xf.p;
    Q4 qa = ga.xf.q, qb = gb.xf.q;
    if (inf_a) plane_to_cube(qa, ga.xf.p, gb.xf.p, brb + gap_sum, A, pa);
    if (inf_b) plane_to_cube(qb, gb.xf.p, ga.xf.p, bra + gap_sum, B, pb);
    // compute_gjk_mpr_contacts (collision_core.py:298-381)
    float reff_a = 0.0f, reff_b = 0.0f;
    const float small_radius = 0.0001f;
    if (A.type == NB_GEO_SPHERE || A.type == NB_GEO_CAPSULE) { reff_a = A.scale.x; A.scale.x = small_radius; }
    if (B.type == NB_GEO_SPHERE || B.type == NB_GEO_CAPSULE) { reff_b = B.scale.x; B.scale.x = small_radius; }
    ContactData tmpl;
    tmpl.reff_a = reff_a;
    tmpl.reff_b = reff_b;
    tmpl.margin_a = ga.margin;
    tmpl.margin_b = gb.margin;
    tmpl.shape_a = sa;
    tmpl.shape_b = sb;
    tmpl.gap_sum = gap_sum;
    tmpl.sub_key = 0;
    float threshold = gap_sum + reff_a + reff_b + ga.margin + gb.margin;
    bool skip_multi = A.type == NB_GEO_SPHERE || B.type == NB_GEO_SPHERE;
    // solve_convex_multi_contact (collision_convex.py:36-132)
    Pair p;
    p.a = A;
    p.b = B;
    p.ob = qmul(qinv(qa), qb);
    p.pb = qrot_inv(qa, sub(pb, pa));
    float margin_sum = tmpl.margin_a + tmpl.margin_b;
    const float eps = 1.0e-4f;
    float enlarge;
    if (margin_sum <= 0.0f) enlarge = eps;
    else if (margin_sum < eps) enlarge = 2.0f * eps;
    else enlarge = 0.0f;
    V3 point_a, point_b, normal;
    float pen, sd;
    bool collision = mpr_core(p, enlarge, point_a, point_b, normal, pen);
    if (collision) {
        sd = -pen + enlarge;
        float he = enlarge * 0.5f;
        point_a = sub(point_a, mul(normal, he));
        point_b = add(point_b, mul(normal, he));
    } else {
        gjk_core(p, 0.0f, point_a, point_b, normal, sd);
    }
    GjkCtx g;
    g.type_a = A.type;
    g.type_b = B.type;
    g.qa = qa;
    g.pa = pa;
    if (skip_multi || sd > threshold) {
        V3 pt = smul(0.5f, add(point_a, point_b));
        pt = add(qrot(qa, pt), pa);
        V3 nws = qrot(qa, normal);
        ContactData cd = tmpl;
        cd.center = pt;
        cd.normal = nws;
        cd.dist = sd;
        cd.sub_key = tmpl.sub_key << 3;
        post_process(cd, g.type_a, g.type_b);
        write_contact(w, cd, true);
        return;
    }
    build_manifold(w, p, g, point_a, point_b, normal, tmpl);
}

// narrow_phase_primitive_kernel body for one pair (narrow_phase.py:198-603)
static void narrow_pair(const Writer& w, const GeomWS& ga, const GeomWS& gb, int sa, int sb) {
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
    for (int i = 0; i < 4; ++i) num += dist[i] < MAXVAL ? 1 : 0;
    if (num > 0) {
        ContactData cd;
        cd.normal = normal;
        cd.reff_a = reff_a;
        cd.reff_b = reff_b;
        cd.margin_a = ga.margin;
        cd.margin_b = gb.margin;
        cd.shape_a = sa;
        cd.shape_b = sb;
        cd.gap_sum = gap_sum;
        bool valid[4];
        for (int i = 0; i < 4; ++i) {
            valid[i] = false;
            if (dist[i] < MAXVAL) {
                cd.center = pos[i];
                cd.dist = dist[i];
                valid[i] = passes_gap(cd);
            }
        }
        for (int i = 0; i < 4; ++i) {
            if (!valid[i]) continue;
            cd.center = pos[i];
            cd.dist = dist[i];
            cd.sub_key = i;
            write_contact(w, cd, false);
        }
        return;
    }
    gjk_pair(w, ga, gb, sa, sb);
}

}  // namespace orc

using namespace orc;

extern "C" {

// Collide every world into host-side solver-format segments (seg->rec0..rec4 as
// float[cap*4] arrays, seg->world_count).  Pairs come from model->pair_shapes.
// Returns NB_ERR_CAPACITY if a world's segment would overflow.
int orc_collide(const NbModelDesc* m, const float* body_q, const OrcSeg* seg) {
    int rc = 0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int w = 0; w < m->world_count; ++w) {
        int s0 = m->world_shape_start[w], s1 = m->world_shape_start[w + 1];
        // geometry for the world's shapes and the global shapes, indexed by global id
        std::vector<int> ids;
        for (int s = s0; s < s1; ++s) ids.push_back(s);
        for (int g = 0; g < m->global_shape_count; ++g) ids.push_back(m->global_shapes[g]);
        std::vector<GeomWS> gws(ids.size());
        for (size_t i = 0; i < ids.size(); ++i) gws[i] = compute_geom(m, body_q, ids[i]);
        std::vector<OutContact> out;
        Writer wr{m, body_q, &out};
        for (int p = m->world_pair_start[w]; p < m->world_pair_start[w + 1]; ++p) {
            int la = (int)(m->pair_shapes[p] & 0xFFFFu), lb = (int)(m->pair_shapes[p] >> 16);
            int sa = ids[la], sb = ids[lb];
            const GeomWS& ga = gws[la];
            const GeomWS& gb = gws[lb];
            if (sa == sb || sa < 0 || sb < 0) continue;
            if (!aabb_overlap(ga, gb)) continue;
            narrow_pair(wr, ga, gb, sa, sb);
        }
        int64_t c0 = 5 * (int64_t)m->world_pair_start[w], c1 = 5 * (int64_t)m->world_pair_start[w + 1];
        if ((int64_t)out.size() > c1 - c0) {
#pragma omp atomic write
            rc = NB_ERR_CAPACITY;
            continue;
        }
        seg->world_count[w] = (int32_t)out.size();
        for (size_t i = 0; i < out.size(); ++i) {
            int64_t k = c0 + (int64_t)i;
            const OutContact& o = out[i];
            int32_t bits;
            float* r0 = seg->rec0 + 4 * k;
            r0[0] = o.p0.x; r0[1] = o.p0.y; r0[2] = o.p0.z; r0[3] = o.m0;
            float* r1 = seg->rec1 + 4 * k;
            r1[0] = o.p1.x; r1[1] = o.p1.y; r1[2] = o.p1.z; r1[3] = o.m1;
            float* r2 = seg->rec2 + 4 * k;
            r2[0] = o.n.x; r2[1] = o.n.y; r2[2] = o.n.z;
            bits = o.s0; std::memcpy(&r2[3], &bits, 4);
            float* r3 = seg->rec3 + 4 * k;
            r3[0] = o.o0.x; r3[1] = o.o0.y; r3[2] = o.o0.z;
            bits = o.s1; std::memcpy(&r3[3], &bits, 4);
            float* r4 = seg->rec4 + 4 * k;
            r4[0] = o.o1.x; r4[1] = o.o1.y; r4[2] = o.o1.z;
            int b0 = m->shape_body[o.s0], b1 = m->shape_body[o.s1];
            int l0 = b0 < 0 ? -1 : b0 - m->world_body_start[w];
            int l1 = b1 < 0 ? -1 : b1 - m->world_body_start[w];
            bits = ((l0 + 1) & 0xFFF) | (((l1 + 1) & 0xFFF) << 12) | ((o.sub & 0xFF) << 24);
            std::memcpy(&r4[3], &bits, 4);
        }
    }
    return rc;
}

// Shape AABBs (compute_shape_aabbs) for every shape: lo/hi [S,3].
int orc_shape_aabbs(const NbModelDesc* m, const float* body_q, float* lo, float* hi) {
    for (int s = 0; s < m->shape_count; ++s) {
        GeomWS g = compute_geom(m, body_q, s);
        store_v3(lo + 3 * s, g.lo);
        store_v3(hi + 3 * s, g.hi);
    }
    return 0;
}

// Single-pair narrow phase for known-answer tests: shapes given directly in
// world space.  Writes up to 5 contacts as rows of 16 floats:
//   center-free form: point0_world(3) point1_world(3) normal(3) margin0 margin1 dist sub 0 0 0
// using identity bodies (shape_body = -1), so body-frame == world-frame.
int orc_collide_pair(int type_a, const float* xf_a, const float* scale_a, float margin_a, float gap_a,
                     int type_b, const float* xf_b, const float* scale_b, float margin_b, float gap_b,
                     float* out_rows, int max_rows) {
    NbModelDesc m;
    std::memset(&m, 0, sizeof(m));
    int32_t sbody[2] = {-1, -1};
    int32_t stype[2] = {type_a, type_b};
    float sxf[14], ssc[6], smg[2] = {margin_a, margin_b}, sgp[2] = {gap_a, gap_b};
    std::memcpy(sxf, xf_a, 7 * sizeof(float));
    std::memcpy(sxf + 7, xf_b, 7 * sizeof(float));
    std::memcpy(ssc, scale_a, 3 * sizeof(float));
    std::memcpy(ssc + 3, scale_b, 3 * sizeof(float));
    float srad[2] = {1e6f, 1e6f};
    m.shape_count = 2;
    m.shape_body = sbody;
    m.shape_type = stype;
    m.shape_transform = sxf;
    m.shape_scale = ssc;
    m.shape_margin = smg;
    m.shape_gap = sgp;
    m.shape_radius = srad;
    GeomWS ga = compute_geom(&m, nullptr, 0);
    GeomWS gb = compute_geom(&m, nullptr, 1);
    std::vector<OutContact> out;
    Writer wr{&m, nullptr, &out};
    int sa = 0, sb = 1;
    const GeomWS* pa = &ga;
    const GeomWS* pb = &gb;
    if (type_a > type_b) { sa = 1; sb = 0; pa = &gb; pb = &ga; }
    narrow_pair(wr, *pa, *pb, sa, sb);
    int n = (int)out.size();
    for (int i = 0; i < n && i < max_rows; ++i) {
        float* r = out_rows + 16 * i;
        const OutContact& o = out[i];
        r[0] = o.p0.x; r[1] = o.p0.y; r[2] = o.p0.z;
        r[3] = o.p1.x; r[4] = o.p1.y; r[5] = o.p1.z;
        r[6] = o.n.x; r[7] = o.n.y; r[8] = o.n.z;
        r[9] = o.m0; r[10] = o.m1;
        r[11] = dot(sub(o.p1, o.p0), o.n) - (o.m0 + o.m1);
        r[12] = (float)o.sub;
        r[13] = (float)o.s0;
        r[14] = (float)o.s1;
        r[15] = 0.0f;
    }
    return n;
}

}  // extern "C"
