// TEST INFRASTRUCTURE ONLY -- CPU oracle of frame-to-frame contact matching.
// Only tests/ may use it.
//
// Sequential restatement of newton/_src/geometry/contact_match.py:
//   _match_contacts_kernel   :252-331  (pair range by key without the sub-key,
//                                       closest world-space midpoint passing the
//                                       normal-dot gate, packed distance/key claim)
//   _resolve_claims_kernel   :352-391  (winner keeps the index, losers -> -2)
//   _save_sorted_state_kernel:434-510  (midpoint = 0.5 * (world p0 + world p1))
// The pair range is searched inside the contact's own world of the previous
// frame (contacts are published in (world, key) order).
#include "oracle_math.h"
#include "../include/newton_b200.h"

#include <cstdint>
#include <cstring>
#include <vector>

using namespace orc;

namespace {

V3 world_point(const NbModelDesc* m, const float* body_q, int shape, V3 p) {
    const int b = shape >= 0 ? m->shape_body[shape] : -1;
    return b < 0 ? p : tf_point(load_tf(body_q + 7 * (size_t)b), p);
}

uint32_t order_bits(float f) {
    uint32_t i;
    std::memcpy(&i, &f, 4);
    const uint32_t mask = (uint32_t)(-(int32_t)(i >> 31)) | 0x80000000u;
    return i ^ mask;
}

int64_t lower_bound(const int64_t* keys, int64_t lo, int64_t hi, int64_t target) {
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (keys[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

}  // namespace

extern "C" {

// world-space midpoints of n contacts [n,3]
int orc_contact_midpoints(const NbModelDesc* m, const float* body_q, int n, const float* p0, const float* p1,
                          const int32_t* s0, const int32_t* s1, float* mid_out) {
    for (int i = 0; i < n; ++i) {
        const V3 a = world_point(m, body_q, s0[i], load_v3(p0 + 3 * (size_t)i));
        const V3 b = world_point(m, body_q, s1[i], load_v3(p1 + 3 * (size_t)i));
        const V3 c = mul(add(a, b), 0.5f);
        mid_out[3 * (size_t)i] = c.x;
        mid_out[3 * (size_t)i + 1] = c.y;
        mid_out[3 * (size_t)i + 2] = c.z;
    }
    return 0;
}

// match + resolve; match_out[n_new], prev_matched_out[n_old] (0/1)
int orc_match_contacts(int W, int n_new, const int64_t* world_offset, const int64_t* keys, const float* mid,
                       const float* normal, int n_old, const int64_t* prev_world_offset, const int64_t* prev_keys,
                       const float* prev_mid, const float* prev_normal, float pos_thr_sq, float ndot_thr,
                       int32_t* match_out, uint8_t* prev_matched_out) {
    std::vector<int64_t> claim((size_t)(n_old > 0 ? n_old : 1), INT64_MAX);
    for (int i = 0; i < n_new; ++i) {
        if (n_old == 0) {
            match_out[i] = -1;
            continue;
        }
        int w = 0;
        while (w + 1 < W && world_offset[w + 1] <= i) ++w;
        int64_t lo = prev_world_offset[w], hi = prev_world_offset[w + 1];
        if (hi > n_old) hi = n_old;
        if (lo > hi) lo = hi;
        const int64_t prefix = keys[i] & ~(int64_t)0x7FFFFF;
        const int64_t r0 = lower_bound(prev_keys, lo, hi, prefix);
        const int64_t r1 = lower_bound(prev_keys, r0, hi, prefix + 0x800000);
        if (r0 >= r1) {
            match_out[i] = -1;
            continue;
        }
        const V3 c = load_v3(mid + 3 * (size_t)i), n = load_v3(normal + 3 * (size_t)i);
        int64_t best = -1;
        float best_d2 = pos_thr_sq;
        for (int64_t k = r0; k < r1; ++k) {
            const V3 d = sub(c, load_v3(prev_mid + 3 * (size_t)k));
            const float d2 = dot(d, d);
            const float nd = dot(n, load_v3(prev_normal + 3 * (size_t)k));
            if (d2 <= best_d2 && nd >= ndot_thr) {
                best_d2 = d2;
                best = k;
            }
        }
        if (best < 0) {
            match_out[i] = -2;
            continue;
        }
        match_out[i] = (int32_t)best;
        const int64_t packed = (int64_t)(((uint64_t)order_bits(best_d2) << 32) | ((uint64_t)keys[i] & 0xFFFFFFFFull));
        if (packed < claim[best]) claim[best] = packed;
    }
    std::memset(prev_matched_out, 0, (size_t)(n_old > 0 ? n_old : 0));
    for (int i = 0; i < n_new; ++i) {
        const int32_t cand = match_out[i];
        if (cand < 0) continue;
        if ((claim[cand] & 0xFFFFFFFFll) == (keys[i] & 0xFFFFFFFFll)) prev_matched_out[cand] = 1;
        else match_out[i] = -2;
    }
    return 0;
}

}  // extern "C"
