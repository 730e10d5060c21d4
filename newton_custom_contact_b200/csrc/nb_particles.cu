// XPBD particle path: soft contacts between particles and shapes, and the
// particle substep (integration, particle-shape and particle-particle
// contacts, springs, position corrections).
//
// Layout: particles are SoA float3 rows ([P,3]); every kernel runs one thread
// per particle.  Each particle GATHERS its corrections (its own soft contacts,
// its neighbours, its springs) in a fixed order and writes its delta once, in
// place of the reference's per-constraint atomic scatter: no atomics on the
// data path and the same bits on every run.
//
// Particle-particle neighbours come from two hashed cell tables, rebuilt from
// the positions each iteration reads: the apply kernel of iteration i inserts
// every particle into table (i+1)&1 as it writes its new position, and the
// constraint kernel of iteration i clears table (i+1)&1 before that.
#include <cuda_runtime.h>

#include <cstdint>

#include "nb_kernels.cuh"
#include "nb_math.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kCollideParticles = 1 << 2;  // ShapeFlags.COLLIDE_PARTICLES

NB_D bool active(const NbParticleDesc& pd, int p) { return (pd.particle_flags[p] & NB_PARTICLE_ACTIVE) != 0; }
NB_D V3 ld3(const float* a, int i) { return V3{a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
NB_D void st3(float* a, int i, V3 v) {
    a[3 * i] = v.x;
    a[3 * i + 1] = v.y;
    a[3 * i + 2] = v.z;
}
// wp.sign: -1 for negative arguments, +1 otherwise
NB_D float warp_sign(float x) { return x < 0.0f ? -1.0f : 1.0f; }

// atan2 from the library's asin (nb_math.cuh), so the CPU oracle reproduces it bit for bit: the angle
// is asin of the smaller of |x|, |y| over the radius (argument at most 1/sqrt 2, where asin is well
// conditioned), shifted into its quadrant.  atan2(0, 0) = 0.
NB_D float nb_atan2(float y, float x) {
    const float r = sqrtf(x * x + y * y);
    if (r == 0.0f) return 0.0f;
    if (fabsf(y) <= fabsf(x)) {
        const float a = nb_asin(y / r);
        if (x > 0.0f) return a;
        return y < 0.0f ? -3.1415927410125732f - a : 3.1415927410125732f - a;
    }
    const float a = 1.5707963705062866f - nb_asin(x / r);
    return y < 0.0f ? -a : a;
}

// Signed distance and outward gradient in the shape frame (newton/_src/geometry/
// kernels.py:165-330 sdf_sphere/_grad, sdf_box/_grad, sdf_capsule/_grad with the
// Z up axis, 568-590 sdf_plane).
NB_D void shape_sdf(int type, V3 p, V3 s, float& d, V3& n) {
    d = 1.0e6f;
    n = V3{0.0f, 0.0f, 0.0f};
    if (type == NB_GEO_SPHERE) {
        d = length(p) - s.x;
        const float l = length(p);
        n = l > 1.0e-8f ? divs(p, l) : V3{0.0f, 0.0f, 1.0f};
    } else if (type == NB_GEO_BOX) {
        const float qx = fabsf(p.x) - s.x, qy = fabsf(p.y) - s.y, qz = fabsf(p.z) - s.z;
        const V3 e = V3{fmaxw(qx, 0.0f), fmaxw(qy, 0.0f), fmaxw(qz, 0.0f)};
        d = length(e) + fminw(fmaxw(qx, fmaxw(qy, qz)), 0.0f);
        if (qx > 0.0f || qy > 0.0f || qz > 0.0f) {
            const V3 c = V3{clampw(p.x, -s.x, s.x), clampw(p.y, -s.y, s.y), clampw(p.z, -s.z, s.z)};
            n = normalize(sub(p, c));
        } else if ((qx > qy && qx > qz) || (qy == 0.0f && qz == 0.0f)) {
            n = V3{warp_sign(p.x), 0.0f, 0.0f};
        } else if ((qy > qx && qy > qz) || (qx == 0.0f && qz == 0.0f)) {
            n = V3{0.0f, warp_sign(p.y), 0.0f};
        } else {
            n = V3{0.0f, 0.0f, warp_sign(p.z)};
        }
    } else if (type == NB_GEO_CAPSULE) {
        const float r = s.x, hh = s.y;
        V3 v;
        V3 fallback;
        if (p.z > hh) {
            v = V3{p.x, p.y, p.z - hh};
            fallback = V3{0.0f, 0.0f, 1.0f};
        } else if (p.z < -hh) {
            v = V3{p.x, p.y, p.z + hh};
            fallback = V3{0.0f, 0.0f, -1.0f};
        } else {
            v = V3{p.x, p.y, 0.0f};
            fallback = V3{0.0f, 0.0f, 1.0f};
        }
        d = length(v) - r;
        const float l = length(v);
        n = l > 1.0e-8f ? divs(v, l) : fallback;
    } else if (type == NB_GEO_PLANE) {
        const float w = s.x * 0.5f, l = s.y * 0.5f;
        if (w > 0.0f && l > 0.0f) {
            const float dd = fmaxw(fabsf(p.x) - w, fabsf(p.y) - l);
            d = fmaxw(dd, fabsf(p.z));
        } else {
            d = p.z;
        }
        n = V3{0.0f, 0.0f, 1.0f};
    }
}

// One (particle, shape) test of create_soft_contacts (newton/_src/geometry/kernels.py:1029-1140).
// Returns true for a contact and fills its body-frame point, velocity and world normal.
NB_D bool soft_contact(const NbParticleDesc& pd, const float* body_q, int p, int s, V3 px, float radius,
                       float margin, V3& body_pos, V3& body_vel, V3& world_normal) {
    if ((pd.shape_flags[s] & kCollideParticles) == 0) return false;
    const int pw = pd.particle_world[p], sw = pd.shape_world[s];
    if (pw != -1 && sw != -1 && pw != sw) return false;
    const int rigid = pd.shape_body[s];
    const TF X_wb = rigid >= 0 ? load_tf(body_q + 7 * rigid) : tf_identity();
    const TF X_bs = load_tf(pd.shape_transform + 7 * s);
    const TF X_ws = tf_mul(X_wb, X_bs);
    const TF X_sw = tf_inverse(X_ws);
    const V3 x_local = tf_point(X_sw, px);
    float d;
    V3 n;
    shape_sdf(pd.shape_type[s], x_local, load_v3(pd.shape_scale + 3 * s), d, n);
    if (!(d < margin + radius)) return false;
    body_pos = tf_point(X_bs, sub(x_local, mul(n, d)));
    body_vel = tf_vector(X_bs, V3{0.0f, 0.0f, 0.0f});
    world_normal = tf_vector(X_ws, n);
    return true;
}

NB_D int particle_soft_count(const NbParticleDesc& pd, const float* body_q, int p, const float* q, float margin) {
    if (!active(pd, p)) return 0;
    const V3 px = ld3(q, p);
    const float radius = pd.particle_radius[p];
    int c = 0;
    for (int s = 0; s < pd.shape_count; ++s) {
        V3 a, b, n;
        c += soft_contact(pd, body_q, p, s, px, radius, margin, a, b, n) ? 1 : 0;
    }
    return c;
}

// Exclusive scan of one value per thread over a block of kScanThreads threads.
__device__ int block_exclusive_scan(int v, int& total) {
    __shared__ int warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    total = warp_sums[kScanThreads / 32 - 1];
    const int before = warp > 0 ? warp_sums[warp - 1] : 0;
    __syncthreads();
    return before + x - v;
}

// Pass 1: every particle's contact count (kept in particle_start[p]) and each block's sum.
__global__ void __launch_bounds__(kScanThreads) soft_count_kernel(NbParticleDesc pd, const float* q,
                                                                  const float* body_q, NbSoftContacts sc) {
    const int p = blockIdx.x * kScanThreads + threadIdx.x;
    const int P = pd.particle_count;
    const int c = p < P ? particle_soft_count(pd, body_q, p, q, sc.margin) : 0;
    if (p < P) sc.particle_start[p] = c;
    int total;
    block_exclusive_scan(c, total);
    if (threadIdx.x == 0) sc.particle_start[P + 1 + blockIdx.x] = total;
}

// Pass 2 (one block): exclusive scan of the block sums; the grand total is the contact count.
__global__ void __launch_bounds__(kScanThreads) soft_scan_blocks_kernel(NbParticleDesc pd, NbSoftContacts sc,
                                                                        int blocks) {
    const int P = pd.particle_count;
    int* sums = sc.particle_start + P + 1;
    int carry = 0;
    for (int base = 0; base < blocks; base += kScanThreads) {
        const int b = base + threadIdx.x;
        const int v = b < blocks ? sums[b] : 0;
        int total;
        const int ex = block_exclusive_scan(v, total);
        if (b < blocks) sums[b] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) {
        sc.particle_start[P] = carry;
        sc.count[0] = carry;
    }
}

// Pass 3: each particle's first contact, then its contacts in shape order (the first max are stored).
__global__ void __launch_bounds__(kScanThreads) soft_write_kernel(NbParticleDesc pd, const float* q,
                                                                  const float* body_q, NbSoftContacts sc) {
    const int p = blockIdx.x * kScanThreads + threadIdx.x;
    const int P = pd.particle_count;
    const int c = p < P ? sc.particle_start[p] : 0;
    int total;
    const int ex = block_exclusive_scan(c, total);
    if (p >= P) return;
    int at = sc.particle_start[P + 1 + blockIdx.x] + ex;
    sc.particle_start[p] = at;
    if (c == 0) return;
    const V3 px = ld3(q, p);
    const float radius = pd.particle_radius[p];
    for (int s = 0; s < pd.shape_count && at < sc.max; ++s) {
        V3 bp, bv, n;
        if (!soft_contact(pd, body_q, p, s, px, radius, sc.margin, bp, bv, n)) continue;
        sc.particle[at] = p;
        sc.shape[at] = s;
        st3(sc.body_pos, at, bp);
        st3(sc.body_vel, at, bv);
        st3(sc.normal, at, n);
        ++at;
    }
}

// ---------------------------------------------------------------- substep
struct Grid {
    int32_t* head;  // [2*size]
    int32_t* next;  // [P]
    uint32_t mask;
    float inv_h;
    bool on;
};

NB_D int cell_of(float x, float inv_h) { return (int)floorf(x * inv_h); }
NB_D uint32_t cell_hash(int cx, int cy, int cz, uint32_t mask) {
    return ((uint32_t)cx * 73856093u ^ (uint32_t)cy * 19349663u ^ (uint32_t)cz * 83492791u) & mask;
}
NB_D void grid_insert(const Grid& g, int table, int p, V3 x) {
    const uint32_t b = cell_hash(cell_of(x.x, g.inv_h), cell_of(x.y, g.inv_h), cell_of(x.z, g.inv_h), g.mask);
    g.next[p] = atomicExch(&g.head[(size_t)table * (g.mask + 1u) + b], p);
}

// integrate_particles (newton/_src/solvers/solver.py:11-47): semi-implicit Euler, gravity on
// particles with positive inverse mass, velocity clamp.  An inactive particle keeps its state.
__global__ void __launch_bounds__(kThreads) particle_integrate_kernel(NbParticleDesc pd, NbParticleIO io,
                                                                      float dt, Grid g) {
    const int p = blockIdx.x * kThreads + threadIdx.x;
    if (p >= pd.particle_count) return;
    const V3 x0 = ld3(io.particle_q, p);
    const V3 v0 = ld3(io.particle_qd, p);
    if (!active(pd, p)) {
        st3(io.particle_q_out, p, x0);
        st3(io.particle_qd_out, p, v0);
        return;
    }
    const V3 f0 = io.particle_f ? ld3(io.particle_f, p) : V3{0.0f, 0.0f, 0.0f};
    const float inv_mass = pd.particle_inv_mass[p];
    const int w = pd.particle_world[p];
    const V3 grav = ld3(pd.gravity, w > 0 ? w : 0);
    const float gate = -inv_mass < 0.0f ? 1.0f : 0.0f;  // wp.step(-inv_mass)
    V3 v1 = add(v0, mul(add(mul(f0, inv_mass), mul(grav, gate)), dt));
    const float v1_mag = length(v1);
    if (v1_mag > pd.particle_max_velocity) v1 = mul(v1, pd.particle_max_velocity / v1_mag);
    const V3 x1 = add(x0, mul(v1, dt));
    st3(io.particle_q_out, p, x1);
    st3(io.particle_qd_out, p, v1);
    if (g.on) grid_insert(g, 0, p, x1);
}

// The corrections of one particle in one iteration: soft contacts (kernels.py:114-222, static
// shapes), particle neighbours (kernels.py:225-289) and springs (kernels.py:292-356), summed in
// that order.  kGroup lanes serve one particle: they split its neighbour cells between them (the
// cell-list walks are chains of dependent loads) and each computes the contribution of the
// neighbours it accepts; the group's first lane sorts them by neighbour index and sums them in that
// order, then adds the soft contacts and springs.  Which lane computes a contribution does not change
// its bits, so the result equals a sequential sum in ascending neighbour index.  The kernel also
// clears the cell table the following apply fills.
#ifndef NB_PARTICLE_GROUP
#define NB_PARTICLE_GROUP 8
#endif
constexpr int kGroup = NB_PARTICLE_GROUP;  // lanes per particle: 2, 4, 8 or 16
static_assert(kGroup >= 2 && kGroup <= 16 && (kGroup & (kGroup - 1)) == 0, "lanes per particle");
constexpr int kSlots = kThreads / kGroup;  // particles per block

__global__ void __launch_bounds__(kThreads) particle_constraints_kernel(NbParticleDesc pd, NbParticleIO io,
                                                                        NbSoftContacts sc, int has_sc, float dt,
                                                                        float relaxation, Grid g, int table) {
    __shared__ int s_n[kSlots];
    __shared__ int s_j[kSlots][NB_PARTICLE_MAX_NEIGHBORS];
    __shared__ float s_c[kSlots][NB_PARTICLE_MAX_NEIGHBORS][3];
    const int tid = blockIdx.x * kThreads + threadIdx.x;
    if (g.on) {
        int32_t* other = g.head + (size_t)(table ^ 1) * (g.mask + 1u);
        for (uint32_t t = tid; t <= g.mask; t += gridDim.x * kThreads) other[t] = -1;
    }
    const int lane = threadIdx.x & (kGroup - 1);
    const int slot = threadIdx.x / kGroup;
    const unsigned gmask = ((1u << kGroup) - 1u) << (threadIdx.x & 31 & ~(kGroup - 1));
    const int i = blockIdx.x * kSlots + slot;
    const bool valid = i < pd.particle_count;
    const bool act = valid && active(pd, i);
    const float* xq = io.particle_q_out;
    const float* vq = io.particle_qd_out;
    if (lane == 0) s_n[slot] = 0;
    __syncwarp(gmask);
    V3 x = V3{0.0f, 0.0f, 0.0f}, v = x;
    float w1 = 0.0f, radius = 0.0f;
    if (valid) {
        x = ld3(xq, i);
        v = ld3(vq, i);
        w1 = pd.particle_inv_mass[i];
        radius = pd.particle_radius[i];
    }

    if (act && g.on) {
        const float reach = (radius + pd.particle_max_radius + pd.particle_cohesion) * 1.001f + 1.0e-6f;
        // the reach is at most ~1 cell (cell size 2 * max radius + cohesion), so a span of 3 cells per axis;
        // the cap keeps the loops bounded whatever the scale
        const int x0 = cell_of(x.x - reach, g.inv_h), x1 = min(cell_of(x.x + reach, g.inv_h), x0 + 4);
        const int y0 = cell_of(x.y - reach, g.inv_h), y1 = min(cell_of(x.y + reach, g.inv_h), y0 + 4);
        const int z0 = cell_of(x.z - reach, g.inv_h), z1 = min(cell_of(x.z + reach, g.inv_h), z0 + 4);
        const int nx = x1 - x0 + 1, ny = y1 - y0 + 1, ncell = nx * ny * (z1 - z0 + 1);
        const int32_t* head = g.head + (size_t)table * (g.mask + 1u);
        bool overflow = false;
        for (int c = lane; c < ncell; c += kGroup) {
            const int cx = x0 + c % nx, cy = y0 + (c / nx) % ny, cz = z0 + c / (nx * ny);
            for (int j = head[cell_hash(cx, cy, cz, g.mask)]; j >= 0; j = g.next[j]) {
                if (j == i) continue;
                const V3 xj = ld3(xq, j);
                // each particle sits in one cell: skip other cells hashed to this bucket
                if (cell_of(xj.x, g.inv_h) != cx || cell_of(xj.y, g.inv_h) != cy || cell_of(xj.z, g.inv_h) != cz)
                    continue;
                if (!active(pd, j)) continue;
                V3 n = sub(x, xj);
                const float d = length(n);
                const float err = d - radius - pd.particle_radius[j];
                const float denom = w1 + pd.particle_inv_mass[j];
                if (!(err <= pd.particle_cohesion && denom > 0.0f)) continue;
                const int at = atomicAdd(&s_n[slot], 1);
                if (at >= NB_PARTICLE_MAX_NEIGHBORS) {
                    overflow = true;
                    continue;
                }
                n = divs(n, d);
                const V3 vrel = sub(v, ld3(vq, j));
                const float lambda_n = err;
                const V3 delta_n = mul(n, lambda_n);
                const float vn = dot(n, vrel);
                const V3 vt = sub(vrel, mul(n, vn));
                const float lambda_f = fmaxw(pd.particle_mu * lambda_n, -length(vt) * dt);
                const V3 delta_f = mul(normalize(vt), lambda_f);
                const V3 contrib = divs(sub(delta_f, delta_n), denom);
                s_j[slot][at] = j;
                s_c[slot][at][0] = contrib.x;
                s_c[slot][at][1] = contrib.y;
                s_c[slot][at][2] = contrib.z;
            }
        }
        if (overflow) atomicOr(io.status, NB_STATUS_NEIGHBOR_OVERFLOW);
    }
    __syncwarp(gmask);
    if (lane != 0 || !valid) return;

    V3 delta = V3{0.0f, 0.0f, 0.0f};
    if (act && has_sc) {
        const int lim = min(sc.max, sc.count[0]);
        const int hi = min(sc.particle_start[i + 1], lim);
        for (int k = sc.particle_start[i]; k < hi; ++k) {
            const int s = sc.shape[k];
            if (pd.shape_body[s] >= 0) {
                atomicOr(io.status, NB_STATUS_PARTICLE_BODY_CONTACT);
                continue;
            }
            // static shape: identity body transform, zero body velocity
            const TF X_wb = tf_identity();
            const V3 bx = tf_point(X_wb, ld3(sc.body_pos, k));
            const V3 r = sub(bx, tf_point(X_wb, V3{0.0f, 0.0f, 0.0f}));
            const V3 n = ld3(sc.normal, k);
            const float c = dot(n, sub(x, bx)) - radius;
            if (c > pd.particle_adhesion) continue;
            const float mu = 0.5f * (pd.soft_contact_mu + pd.shape_mu[s]);
            const V3 body_w = V3{0.0f, 0.0f, 0.0f}, body_v = V3{0.0f, 0.0f, 0.0f};
            const V3 bv = add(add(body_v, cross(body_w, r)), tf_vector(X_wb, ld3(sc.body_vel, k)));
            const V3 vr = sub(v, bv);
            const float lambda_n = c;
            const V3 delta_n = mul(n, lambda_n);
            const float vn = dot(n, vr);
            const V3 vt = sub(vr, mul(n, vn));
            const float denom = w1 + 0.0f;
            if (denom == 0.0f) continue;
            const float lambda_f = fmaxw(mu * lambda_n, -length(vt) * dt);
            const V3 delta_f = mul(normalize(vt), lambda_f);
            const V3 delta_total = mul(divs(sub(delta_f, delta_n), denom), relaxation);
            delta = add(delta, smul(w1, delta_total));
        }
    }

    if (act && g.on) {
        // neighbours in ascending index (insertion sort of the group's accepted list)
        const int count = min(s_n[slot], NB_PARTICLE_MAX_NEIGHBORS);
        int* js = s_j[slot];
        float(*cs)[3] = s_c[slot];
        for (int a = 1; a < count; ++a) {
            const int j = js[a];
            const float c0 = cs[a][0], c1 = cs[a][1], c2 = cs[a][2];
            int b = a;
            while (b > 0 && js[b - 1] > j) {
                js[b] = js[b - 1];
                cs[b][0] = cs[b - 1][0];
                cs[b][1] = cs[b - 1][1];
                cs[b][2] = cs[b - 1][2];
                --b;
            }
            js[b] = j;
            cs[b][0] = c0;
            cs[b][1] = c1;
            cs[b][2] = c2;
        }
        V3 dpp = V3{0.0f, 0.0f, 0.0f};
        for (int k = 0; k < count; ++k) dpp = add(dpp, V3{cs[k][0], cs[k][1], cs[k][2]});
        delta = add(delta, mul(mul(dpp, w1), relaxation));
    }

    if (pd.spring_count > 0) {
        const int s_hi = pd.particle_spring_start[i + 1];
        for (int k = pd.particle_spring_start[i]; k < s_hi; ++k) {
            const int s = pd.particle_spring_list[k];
            const int a = pd.spring_indices[2 * s], b = pd.spring_indices[2 * s + 1];
            const float ke = pd.spring_stiffness[s], kd = pd.spring_damping[s], rest = pd.spring_rest_length[s];
            const V3 xij = sub(ld3(xq, a), ld3(xq, b));
            const V3 vij = sub(ld3(vq, a), ld3(vq, b));
            const float l = length(xij);
            if (l == 0.0f) continue;
            const V3 n = divs(xij, l);
            const float c = l - rest;
            const float wi = pd.particle_inv_mass[a], wj = pd.particle_inv_mass[b];
            const float denom = wi + wj;
            if (denom <= 0.0f || ke <= 0.0f || kd < 0.0f) continue;
            const float alpha = 1.0f / (ke * dt * dt);
            const float gamma = kd / (ke * dt);
            const float grad_c_dot_v = dt * dot(n, vij);
            const float lambda_prev = 0.0f;  // the solver zeroes the spring multipliers every iteration
            const float dlambda =
                -1.0f * (c + alpha * lambda_prev + gamma * grad_c_dot_v) / ((1.0f + gamma) * denom + alpha);
            if (i == a) delta = add(delta, mul(n, wi * dlambda));
            if (i == b) delta = add(delta, mul(smul(-1.0f, n), wj * dlambda));
        }
    }
    st3(io.delta, i, delta);
}

NB_D float det3(const M33& m) {
    return m.m[0][0] * (m.m[1][1] * m.m[2][2] - m.m[1][2] * m.m[2][1]) -
           m.m[0][1] * (m.m[1][0] * m.m[2][2] - m.m[1][2] * m.m[2][0]) +
           m.m[0][2] * (m.m[1][0] * m.m[2][1] - m.m[1][1] * m.m[2][0]);
}
NB_D M33 matmul3(const M33& a, const M33& b) {
    M33 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}
NB_D M33 from_cols(V3 a, V3 b, V3 c) {
    M33 r;
    r.m[0][0] = a.x; r.m[1][0] = a.y; r.m[2][0] = a.z;
    r.m[0][1] = b.x; r.m[1][1] = b.y; r.m[2][1] = b.z;
    r.m[0][2] = c.x; r.m[1][2] = c.y; r.m[2][2] = c.z;
    return r;
}
NB_D V3 col(const M33& m, int c) { return V3{m.m[0][c], m.m[1][c], m.m[2][c]}; }

// Tetrahedra of one particle (solve_tetrahedra, kernels.py:459-628): per element a stretch term
// (trace(F^T F) - 3) and a volume term (det F - 1), each a compliant constraint with compliance
// `relaxation` (the solver's soft_body_relaxation) scaled by the inverse rest volume.
NB_D V3 tet_terms(const NbParticleDesc& pd, const float* xq, int i, int t, float dt, V3 delta) {
    const int* ix = pd.tet_indices + 4 * t;
    const V3 x0 = ld3(xq, ix[0]), x1 = ld3(xq, ix[1]), x2 = ld3(xq, ix[2]), x3 = ld3(xq, ix[3]);
    const float w[4] = {pd.particle_inv_mass[ix[0]], pd.particle_inv_mass[ix[1]], pd.particle_inv_mass[ix[2]],
                        pd.particle_inv_mass[ix[3]]};
    const M33 Ds = from_cols(sub(x1, x0), sub(x2, x0), sub(x3, x0));
    M33 Dm, inv_QT;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Dm.m[r][c] = pd.tet_poses[9 * t + 3 * r + c];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) inv_QT.m[r][c] = Dm.m[c][r];
    const float inv_rest_volume = det3(Dm) * 6.0f;
    const M33 Fm = matmul3(Ds, Dm);
    const V3 f1 = col(Fm, 0), f2 = col(Fm, 1), f3 = col(Fm, 2);
    const float tr = dot(f1, f1) + dot(f2, f2) + dot(f3, f3);
    for (int term = 0; term < 2; ++term) {
        float C;
        M33 dC;
        if (term == 0) {
            C = tr - 3.0f;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) dC.m[r][c] = Fm.m[r][c] * 2.0f;
        } else {
            C = det3(Fm) - 1.0f;
            dC = from_cols(cross(f2, f3), cross(f3, f1), cross(f1, f2));
        }
        if (C == 0.0f) continue;
        const M33 dP = matmul3(dC, inv_QT);
        V3 grad[4];
        grad[1] = col(dP, 0);
        grad[2] = col(dP, 1);
        grad[3] = col(dP, 2);
        grad[0] = sub(sub(neg(grad[1]), grad[2]), grad[3]);
        const float wsum = dot(grad[0], grad[0]) * w[0] + dot(grad[1], grad[1]) * w[1] +
                           dot(grad[2], grad[2]) * w[2] + dot(grad[3], grad[3]) * w[3];
        if (!(wsum > 0.0f)) continue;
        float alpha = pd.soft_body_relaxation / dt / dt;
        if (inv_rest_volume > 0.0f) alpha *= inv_rest_volume;
        const float dlambda = -C / (wsum + alpha);
        for (int r = 0; r < 4; ++r)
            if (ix[r] == i) delta = add(delta, mul(grad[r], w[r] * dlambda));
    }
    return delta;
}

// Bending edges (bending_constraint, kernels.py:358-457), then tetrahedra, of one particle, added to its
// delta after the constraint kernel's terms (the same order as one sequential sum); a kernel of its own
// so that the constraint kernel keeps its register budget.  The solver zeroes the multipliers every iteration.
__global__ void __launch_bounds__(kThreads) particle_bending_kernel(NbParticleDesc pd, NbParticleIO io, float dt) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= pd.particle_count) return;
    const int e_lo = pd.edge_count > 0 ? pd.particle_edge_start[i] : 0;
    const int e_hi = pd.edge_count > 0 ? pd.particle_edge_start[i + 1] : 0;
    const int t_lo = pd.tet_count > 0 ? pd.particle_tet_start[i] : 0;
    const int t_hi = pd.tet_count > 0 ? pd.particle_tet_start[i + 1] : 0;
    if (e_lo == e_hi && t_lo == t_hi) return;
    const float* xq = io.particle_q_out;
    const float* vq = io.particle_qd_out;
    V3 delta = ld3(io.delta, i);
    {
        for (int k = e_lo; k < e_hi; ++k) {
            const int e = pd.particle_edge_list[k];
            const int* ix = pd.edge_indices + 4 * e;
            const float ke = pd.edge_bending_properties[2 * e], kd = pd.edge_bending_properties[2 * e + 1];
            const V3 x1 = ld3(xq, ix[0]), x2 = ld3(xq, ix[1]), x3 = ld3(xq, ix[2]), x4 = ld3(xq, ix[3]);
            const float w[4] = {pd.particle_inv_mass[ix[0]], pd.particle_inv_mass[ix[1]],
                                pd.particle_inv_mass[ix[2]], pd.particle_inv_mass[ix[3]]};
            const V3 n1 = cross(sub(x3, x1), sub(x4, x1));
            const V3 n2 = cross(sub(x4, x2), sub(x3, x2));
            const V3 ev = sub(x4, x3);
            const float n1_length = length(n1), n2_length = length(n2), e_length = length(ev);
            if (n1_length < 1.0e-6f || n2_length < 1.0e-6f || e_length < 1.0e-6f) continue;
            const V3 n1_hat = divs(n1, n1_length), n2_hat = divs(n2, n2_length), e_hat = divs(ev, e_length);
            const float cos_theta = dot(n1_hat, n2_hat);
            const float sin_theta = dot(cross(n1_hat, n2_hat), e_hat);
            const float c = nb_atan2(sin_theta, cos_theta) - pd.edge_rest_angle[e];
            V3 grad[4];
            grad[0] = mul(neg(n1_hat), e_length);
            grad[1] = mul(neg(n2_hat), e_length);
            grad[2] = sub(mul(neg(n1_hat), dot(sub(x1, x4), e_hat)), mul(n2_hat, dot(sub(x2, x4), e_hat)));
            grad[3] = sub(mul(neg(n1_hat), dot(sub(x3, x1), e_hat)), mul(n2_hat, dot(sub(x3, x2), e_hat)));
            const float denominator = w[0] * length_sq(grad[0]) + w[1] * length_sq(grad[1]) +
                                      w[2] * length_sq(grad[2]) + w[3] * length_sq(grad[3]);
            if (denominator <= 0.0f || ke <= 0.0f || kd < 0.0f) continue;
            const float alpha = 1.0f / (ke * dt * dt);
            const float gamma = kd / (ke * dt);
            const float grad_dot_v = dt * (dot(grad[0], ld3(vq, ix[0])) + dot(grad[1], ld3(vq, ix[1])) +
                                           dot(grad[2], ld3(vq, ix[2])) + dot(grad[3], ld3(vq, ix[3])));
            const float lambda_prev = 0.0f;
            const float dlambda =
                -1.0f * (c + alpha * lambda_prev + gamma * grad_dot_v) / ((1.0f + gamma) * denominator + alpha);
            for (int r = 0; r < 4; ++r)
                if (ix[r] == i) delta = add(delta, mul(grad[r], w[r] * dlambda));
        }
    }
    for (int k = t_lo; k < t_hi; ++k) delta = tet_terms(pd, xq, i, pd.particle_tet_list[k], dt, delta);
    st3(io.delta, i, delta);
}

// apply_particle_deltas (kernels.py:776-807), in place; then the particle enters the next cell table.
__global__ void __launch_bounds__(kThreads) particle_apply_kernel(NbParticleDesc pd, NbParticleIO io, float dt,
                                                                  Grid g, int next_table, int insert) {
    const int p = blockIdx.x * kThreads + threadIdx.x;
    if (p >= pd.particle_count || !active(pd, p)) return;
    const V3 x0 = ld3(io.particle_q, p);
    const V3 xp = ld3(io.particle_q_out, p);
    const V3 x_new = add(xp, ld3(io.delta, p));
    V3 v_new = divs(sub(x_new, x0), dt);
    const float v_mag = length(v_new);
    if (v_mag > pd.particle_max_velocity) v_new = mul(v_new, pd.particle_max_velocity / v_mag);
    st3(io.particle_q_out, p, x_new);
    st3(io.particle_qd_out, p, v_new);
    if (insert) grid_insert(g, next_table, p, x_new);
}

// apply_particle_shape_restitution (kernels.py:34-112) for static shapes: contacts tested at the
// substep's start position; each particle adds the velocity change of its contacts, in list order, to
// its velocity after the iterations (every change computed from that velocity).
__global__ void __launch_bounds__(kThreads) particle_restitution_kernel(NbParticleDesc pd, NbParticleIO io,
                                                                        NbSoftContacts sc) {
    const int p = blockIdx.x * kThreads + threadIdx.x;
    if (p >= pd.particle_count || !active(pd, p)) return;
    const int lim = min(sc.max, sc.count[0]);
    const int lo = sc.particle_start[p], hi = min(sc.particle_start[p + 1], lim);
    if (lo >= hi) return;
    const V3 v_new = ld3(io.particle_qd_out, p);
    const V3 px = ld3(io.particle_q, p);
    const V3 v_old = ld3(io.particle_qd, p);
    V3 v_out = v_new;
    for (int k = lo; k < hi; ++k) {
        if (pd.shape_body[sc.shape[k]] >= 0) continue;  // body-attached shapes: not coupled
        const TF X_wb = tf_identity(), X_wb_prev = tf_identity();
        const V3 bx = tf_point(X_wb, ld3(sc.body_pos, k));
        const V3 n = ld3(sc.normal, k);
        const float c = dot(n, sub(px, bx)) - pd.particle_radius[p];
        if (c > pd.particle_adhesion) continue;
        const V3 bv_contact = tf_vector(X_wb_prev, ld3(sc.body_vel, k));
        const float rel_vel_old = dot(n, sub(v_old, bv_contact));
        const float rel_vel_new = dot(n, sub(v_new, bv_contact));
        if (rel_vel_old < 0.0f) {
            const V3 dv = mul(n, -rel_vel_new + fmaxw(-pd.soft_contact_restitution * rel_vel_old, 0.0f));
            v_out = add(v_out, dv);
        }
    }
    st3(io.particle_qd_out, p, v_out);
}

bool check_pd(const NbParticleDesc* pd) {
    if (!pd || pd->particle_count < 0 || pd->spring_count < 0 || pd->shape_count < 0 || pd->world_count < 1)
        return false;
    if (pd->particle_count == 0) return true;
    if (!pd->particle_inv_mass || !pd->particle_radius || !pd->particle_flags || !pd->particle_world ||
        !pd->gravity)
        return false;
    if (pd->spring_count > 0 && (!pd->spring_indices || !pd->spring_rest_length || !pd->spring_stiffness ||
                                 !pd->spring_damping || !pd->particle_spring_start || !pd->particle_spring_list))
        return false;
    if (pd->tet_count < 0 || (pd->tet_count > 0 && (!pd->tet_indices || !pd->tet_poses || !pd->particle_tet_start ||
                                                     !pd->particle_tet_list)))
        return false;
    if (pd->edge_count < 0 || (pd->edge_count > 0 && (!pd->edge_indices || !pd->edge_rest_angle ||
                                                       !pd->edge_bending_properties || !pd->particle_edge_start ||
                                                       !pd->particle_edge_list)))
        return false;
    if (pd->shape_count > 0 && (!pd->shape_body || !pd->shape_type || !pd->shape_transform || !pd->shape_scale ||
                                !pd->shape_world || !pd->shape_flags || !pd->shape_mu))
        return false;
    return true;
}

}  // namespace

extern "C" {

int nb_soft_collide(const NbParticleDesc* pd, const float* particle_q, const float* body_q,
                    const NbSoftContacts* sc, void* stream) {
    if (!check_pd(pd) || !sc || !sc->count || sc->max < 0) return NB_ERR_INVALID;
    const cudaStream_t st = (cudaStream_t)stream;
    const int P = pd->particle_count;
    if (P == 0 || pd->shape_count == 0)
        return nb_cuda_rc(cudaMemsetAsync(sc->count, 0, sizeof(int32_t), st));
    if (!particle_q || !sc->particle_start) return NB_ERR_INVALID;
    if (sc->max > 0 && (!sc->particle || !sc->shape || !sc->body_pos || !sc->body_vel || !sc->normal))
        return NB_ERR_INVALID;
    const int blocks = (P + kScanThreads - 1) / kScanThreads;
    soft_count_kernel<<<blocks, kScanThreads, 0, st>>>(*pd, particle_q, body_q, *sc);
    soft_scan_blocks_kernel<<<1, kScanThreads, 0, st>>>(*pd, *sc, blocks);
    soft_write_kernel<<<blocks, kScanThreads, 0, st>>>(*pd, particle_q, body_q, *sc);
    return nb_cuda_rc(cudaGetLastError());
}

int nb_particle_step(const NbParticleDesc* pd, const NbParticleIO* io, const NbSoftContacts* sc, float dt,
                     int32_t iterations, float relaxation, void* stream) {
    if (!check_pd(pd) || !io || iterations < 0 || !(dt > 0.0f)) return NB_ERR_INVALID;
    const int P = pd->particle_count;
    if (P == 0) return NB_OK;
    if (!io->particle_q || !io->particle_qd || !io->particle_q_out || !io->particle_qd_out || !io->delta ||
        !io->status)
        return NB_ERR_INVALID;
    if (sc && (!sc->count || !sc->particle_start || sc->max < 0 ||
               (sc->max > 0 && (!sc->shape || !sc->body_pos || !sc->body_vel || !sc->normal))))
        return NB_ERR_INVALID;
    const cudaStream_t st = (cudaStream_t)stream;
    Grid g{};
    g.on = pd->particle_max_radius > 0.0f && P > 1;
    if (g.on) {
        const float h = 2.0f * pd->particle_max_radius + pd->particle_cohesion;
        const int32_t n = io->grid_size;
        if (!io->grid_head || !io->grid_next || n <= 0 || (n & (n - 1)) != 0 || !(h > 0.0f)) return NB_ERR_INVALID;
        g.head = io->grid_head;
        g.next = io->grid_next;
        g.mask = (uint32_t)n - 1u;
        g.inv_h = 1.0f / h;
        cudaError_t e = cudaMemsetAsync(g.head, 0xff, sizeof(int32_t) * (size_t)n, st);
        if (e != cudaSuccess) return nb_cuda_rc(e);
    }
    NbSoftContacts none{};
    const int has_sc = sc != nullptr && pd->shape_count > 0;
    const NbSoftContacts scv = sc ? *sc : none;
    const int blocks = (P + kThreads - 1) / kThreads;
    particle_integrate_kernel<<<blocks, kThreads, 0, st>>>(*pd, *io, dt, g);
    const int con_blocks = (P + kSlots - 1) / kSlots;
    for (int it = 0; it < iterations; ++it) {
        const int table = it & 1;
        particle_constraints_kernel<<<con_blocks, kThreads, 0, st>>>(*pd, *io, scv, has_sc, dt, relaxation, g,
                                                                     table);
        if (pd->edge_count > 0 || pd->tet_count > 0)
            particle_bending_kernel<<<blocks, kThreads, 0, st>>>(*pd, *io, dt);
        particle_apply_kernel<<<blocks, kThreads, 0, st>>>(*pd, *io, dt, g, table ^ 1,
                                                           g.on && it + 1 < iterations ? 1 : 0);
    }
    if (io->enable_restitution && has_sc)
        particle_restitution_kernel<<<blocks, kThreads, 0, st>>>(*pd, *io, scv);
    return nb_cuda_rc(cudaGetLastError());
}

}  // extern "C"
