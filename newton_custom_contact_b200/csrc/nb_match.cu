// Frame-to-frame contact matching (CollisionPipeline contact_matching =
// "latest" / "sticky", newton/_src/geometry/contact_match.py:252-620 and
// newton/_src/sim/collide.py:1083-1182).
//
// Contacts are published in (world, key) order, so the previous frame's keys
// are sorted inside each world: a new contact binary-searches only its own
// world's previous range for its shape pair (key without the sort sub-key),
// takes the closest previous contact by world-space midpoint among those whose
// normal passes the dot threshold, and claims it with one 64-bit atomicMin of
// (orderable distance << 32 | low 32 key bits); a resolve pass demotes the
// losers to MATCH_BROKEN.  Sticky mode then replays the previous frame's
// body-frame points, offsets and normal into matched rows -- of the public
// arrays and of the solver records the step reads -- and the frame's sorted
// state is saved for the next call.
#include <cuda_runtime.h>

#include "nb_kernels.cuh"
#include "nb_math.cuh"

namespace {

constexpr int kT = 256;
constexpr int32_t kNotFound = -1;
constexpr int32_t kBroken = -2;
constexpr long long kClaimFree = 0x7FFFFFFFFFFFFFFFll;

// orderable encoding of a float (non-negative inputs: strictly monotone)
__device__ __forceinline__ unsigned order_bits(float f) {
    const unsigned i = __float_as_uint(f);
    const unsigned mask = (unsigned)(-(int)(i >> 31)) | 0x80000000u;
    return i ^ mask;
}

__device__ __forceinline__ V3 world_point(const NbModelDesc& m, const float* body_q, int shape, V3 p) {
    const int b = shape >= 0 ? m.shape_body[shape] : -1;
    return b < 0 ? p : tf_point(load_tf(body_q + 7 * (size_t)b), p);
}

__device__ __forceinline__ V3 ld3(const float* a, int64_t i) { return load_v3(a + 3 * (size_t)i); }
__device__ __forceinline__ void st3(float* a, int64_t i, V3 v) {
    a[3 * (size_t)i] = v.x;
    a[3 * (size_t)i + 1] = v.y;
    a[3 * (size_t)i + 2] = v.z;
}

// first index in [lo, hi) with keys[index] >= target
__device__ __forceinline__ int64_t lower_bound(const int64_t* keys, int64_t lo, int64_t hi, int64_t target) {
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (keys[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// world of public contact i: last w with world_offset[w] <= i
__device__ __forceinline__ int world_of(const int64_t* wo, int W, int64_t i) {
    int lo = 0, hi = W;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (wo[mid] <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The kernels below loop over live rows only (counts read on the device) with
// a grid sized from the SM count: cost follows the contacts, not the capacity.
#define FOR_ROWS(i, n) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

__device__ __forceinline__ int live_count(const NbContactsPublic& pub) {
    return pub.count[0] < pub.capacity ? pub.count[0] : pub.capacity;
}

__global__ void clear_claims_kernel(NbMatchState st) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (st.new_count) st.new_count[0] = 0;
        if (st.broken_count) st.broken_count[0] = 0;
    }
    FOR_ROWS(i, st.prev_count[0]) {
        st.prev_claim[i] = kClaimFree;
        if (st.prev_was_matched) st.prev_was_matched[i] = 0;
    }
}

__device__ void match_row(const NbModelDesc& m, const float* __restrict__ body_q, const NbContactsPublic& pub,
                          const NbMatchState& st, int n_new, int n_old, int i) {
    if (i >= n_new || n_old == 0) {
        st.match_index[i] = kNotFound;
        return;
    }
    const int w = world_of(pub.world_offset, m.world_count, i);
    int64_t lo = st.prev_world_offset[w], hi = st.prev_world_offset[w + 1];
    hi = hi < n_old ? hi : n_old;
    lo = lo < hi ? lo : hi;
    const int64_t key = pub.sort_key[i];
    const int64_t prefix = key & ~(int64_t)0x7FFFFF;  // shape pair without the sort sub-key
    const int64_t r0 = lower_bound(st.prev_keys, lo, hi, prefix);
    const int64_t r1 = lower_bound(st.prev_keys, r0, hi, prefix + 0x800000);
    if (r0 >= r1) {
        st.match_index[i] = kNotFound;
        return;
    }
    const V3 p0w = world_point(m, body_q, pub.shape0[i], ld3(pub.point0, i));
    const V3 p1w = world_point(m, body_q, pub.shape1[i], ld3(pub.point1, i));
    const V3 mid = mul(add(p0w, p1w), 0.5f);
    const V3 n = ld3(pub.normal, i);
    int64_t best = -1;
    float best_d2 = st.pos_threshold_sq;
    for (int64_t k = r0; k < r1; ++k) {
        const V3 d = sub(mid, ld3(st.prev_mid, k));
        const float d2 = dot(d, d);
        const float nd = dot(n, ld3(st.prev_normal, k));
        if (d2 <= best_d2 && nd >= st.normal_dot_threshold) {
            best_d2 = d2;
            best = k;
        }
    }
    if (best >= 0) {
        st.match_index[i] = (int32_t)best;
        const long long claim = (long long)(((unsigned long long)order_bits(best_d2) << 32) |
                                            ((unsigned long long)key & 0xFFFFFFFFull));
        atomicMin(reinterpret_cast<long long*>(st.prev_claim) + best, claim);
    } else {
        st.match_index[i] = kBroken;
    }
}

__global__ void __launch_bounds__(kT) match_kernel(NbModelDesc m, const float* __restrict__ body_q,
                                                   NbContactsPublic pub, NbMatchState st) {
    const int n_new = live_count(pub);
    const int n_old = st.prev_count[0];
    // rows past the live count that the last call wrote go back to "not found"
    const int rows = n_new > st.prev_count[1] ? n_new : st.prev_count[1];
    FOR_ROWS(i, rows) match_row(m, body_q, pub, st, n_new, n_old, i);
}

__global__ void resolve_kernel(NbContactsPublic pub, NbMatchState st) {
    FOR_ROWS(i, live_count(pub)) {
        const int32_t cand = st.match_index[i];
        if (cand < 0) continue;
        const long long winner = st.prev_claim[cand] & 0xFFFFFFFFll;
        if (winner == (pub.sort_key[i] & 0xFFFFFFFFll)) {
            if (st.prev_was_matched) st.prev_was_matched[cand] = 1;
        } else {
            st.match_index[i] = kBroken;
        }
    }
}

// sticky: matched rows take the previous frame's body-frame points, offsets
// and normal, in the public arrays and in the solver record (same index)
__device__ void replay_row(const NbContactsPublic& pub, const NbContactSeg& seg, const NbMatchState& st, int i) {
    const int32_t k = st.match_index[i];
    if (k < 0) return;
    const V3 p0 = ld3(st.prev_point0, k), p1 = ld3(st.prev_point1, k);
    const V3 o0 = ld3(st.prev_offset0, k), o1 = ld3(st.prev_offset1, k);
    const V3 n = ld3(st.prev_normal_sticky, k);
    st3(pub.point0, i, p0);
    st3(pub.point1, i, p1);
    st3(pub.offset0, i, o0);
    st3(pub.offset1, i, o1);
    st3(pub.normal, i, n);
    float4* r = reinterpret_cast<float4*>(seg.rec) + (size_t)i * 5;
    r[0] = make_float4(p0.x, p0.y, p0.z, r[0].w);
    r[1] = make_float4(p1.x, p1.y, p1.z, r[1].w);
    r[2] = make_float4(n.x, n.y, n.z, r[2].w);
    r[3] = make_float4(o0.x, o0.y, o0.z, r[3].w);
    r[4] = make_float4(o1.x, o1.y, o1.z, r[4].w);
}

__global__ void replay_kernel(NbContactsPublic pub, NbContactSeg seg, NbMatchState st) {
    FOR_ROWS(i, live_count(pub)) replay_row(pub, seg, st, i);
}

__global__ void report_kernel(NbContactsPublic pub, NbMatchState st) {
    const int n_new = live_count(pub), n_old = st.prev_count[0];
    FOR_ROWS(i, n_new > n_old ? n_new : n_old) {
        if (i < n_new && st.match_index[i] < 0) st.new_indices[atomicAdd(st.new_count, 1)] = i;
        if (i < n_old && st.prev_was_matched[i] == 0) st.broken_indices[atomicAdd(st.broken_count, 1)] = i;
    }
}

__device__ void save_row(const NbModelDesc& m, const float* __restrict__ body_q, const NbContactsPublic& pub,
                         const NbMatchState& st, int n_new, int i) {
    if (i <= m.world_count) st.prev_world_offset[i] = pub.world_offset[i];
    if (i >= n_new) return;
    st.prev_keys[i] = pub.sort_key[i];
    const V3 p0 = ld3(pub.point0, i), p1 = ld3(pub.point1, i);
    const V3 p0w = world_point(m, body_q, pub.shape0[i], p0);
    const V3 p1w = world_point(m, body_q, pub.shape1[i], p1);
    st3(st.prev_mid, i, mul(add(p0w, p1w), 0.5f));
    const V3 n = ld3(pub.normal, i);
    st3(st.prev_normal, i, n);
    if (st.sticky) {
        st3(st.prev_point0, i, p0);
        st3(st.prev_point1, i, p1);
        st3(st.prev_offset0, i, ld3(pub.offset0, i));
        st3(st.prev_offset1, i, ld3(pub.offset1, i));
        st3(st.prev_normal_sticky, i, n);
    }
}

__global__ void save_kernel(NbModelDesc m, const float* __restrict__ body_q, NbContactsPublic pub, NbMatchState st) {
    const int n_new = live_count(pub);
    FOR_ROWS(i, n_new > m.world_count + 1 ? n_new : m.world_count + 1) save_row(m, body_q, pub, st, n_new, i);
}

__global__ void save_count_kernel(NbContactsPublic pub, NbMatchState st) {
    st.prev_count[0] = live_count(pub);
    st.prev_count[1] = live_count(pub);  // match_index rows holding values other than "not found"
}

}  // namespace

cudaError_t nb_launch_match(const NbModelDesc* m, const float* body_q, const NbContactsPublic* pub,
                            const NbContactSeg* seg, const NbMatchState* st, cudaStream_t stream) {
    const int cap = st->capacity;
    const long n = cap > m->world_count + 1 ? cap : m->world_count + 1;
    const int blocks = nb_contact_grid(n, kT);
    clear_claims_kernel<<<blocks, kT, 0, stream>>>(*st);
    match_kernel<<<blocks, kT, 0, stream>>>(*m, body_q, *pub, *st);
    resolve_kernel<<<blocks, kT, 0, stream>>>(*pub, *st);
    if (st->sticky) replay_kernel<<<blocks, kT, 0, stream>>>(*pub, *seg, *st);
    if (st->new_indices) report_kernel<<<blocks, kT, 0, stream>>>(*pub, *st);
    save_kernel<<<blocks, kT, 0, stream>>>(*m, body_q, *pub, *st);
    save_count_kernel<<<1, 1, 0, stream>>>(*pub, *st);
    return cudaGetLastError();
}
