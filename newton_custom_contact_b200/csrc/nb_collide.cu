// Collision detection for many independent worlds.
//
// Kernels per substep:
//   1. broadphase_kernel -- one warp per world (worlds pulled from a device
//      counter, largest first; worlds with 2048+ candidate pairs are shared
//      by the whole CTA).  The warp computes every shape's world
//      transform and AABB (compute_shape_aabbs, newton/_src/sim/collide.py:150-275),
//      stages the AABBs in shared memory and the full geometry in global
//      memory, then tests the world's candidate pairs (explicit pair list
//      sorted by contact key; BroadPhaseExplicit,
//      newton/_src/geometry/broad_phase_nxn.py:28-66) 32 at a time.  Hits are
//      compacted *in order* with __ballot_sync / __popc into the world's
//      candidate list and pushed to one of two work queues: pairs the analytic
//      primitive path finishes and pairs that need MPR/GJK, so the narrow
//      phase runs on convergent warps.
//   2. narrow phase -- one thread per candidate of every world, with
//      write_contact semantics (narrow_phase.py:153-776, collide.py:62-147),
//      <= 5 contacts written into the candidate's own slots:
//      narrow_analytic_kernel (primitive pairs), gjk_prefilter_kernel (drops
//      pairs that are provably farther apart than the contact threshold and
//      compacts the rest), narrow_gjk_kernel (MPR / GJK) and
//      narrow_manifold_kernel (the manifolds of the pairs within the threshold).
//   3. publish (world_scan_kernel + publish_kernel) -- the reference's dense
//      Contacts arrays ordered by (world, key): walking a world's candidates
//      in order and each candidate's slots in sub-key order is exactly the key
//      order of newton/_src/geometry/contact_data.py:59-83, so no sort is needed
//      (ContactSorter, contact_sort.py:194-445).
#include <cuda_runtime.h>

#include <mutex>

#include "nb_geom.cuh"
#include "nb_kernels.cuh"

namespace {

using namespace nbg;

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBT = 256;             // broad phase: threads per CTA (8 worlds in flight)
constexpr int kNT = 128;             // narrow phase: threads per CTA
constexpr int kGjkMinBlocks = 12;     // MPR/GJK kernel: resident CTAs per SM the registers are fitted to
constexpr int kManifoldMinBlocks = 5;   // manifold kernel (96 registers: fewer, heavier threads measure faster)
constexpr int kSlotF4 = 25;          // 5 contacts x 5 float4 per candidate

__device__ __forceinline__ void store_geom(float4* g, const Geom& x) {
    g[0] = make_float4(x.xf.p.x, x.xf.p.y, x.xf.p.z, x.margin);
    g[1] = make_float4(x.xf.q.x, x.xf.q.y, x.xf.q.z, x.xf.q.w);
    g[2] = make_float4(x.scale.x, x.scale.y, x.scale.z, x.gap);
    g[3] = make_float4(x.lo.x, x.lo.y, x.lo.z, __int_as_float(x.type));
    g[4] = make_float4(x.hi.x, x.hi.y, x.hi.z, __int_as_float(x.body));
}

__device__ __forceinline__ Geom load_geom(const float4* g, int sid) {
    float4 a = g[0], b = g[1], c = g[2], d = g[3], e = g[4];
    Geom x;
    x.xf = TF{V3{a.x, a.y, a.z}, Q4{b.x, b.y, b.z, b.w}};
    x.margin = a.w;
    x.scale = V3{c.x, c.y, c.z};
    x.gap = c.w;
    x.lo = V3{d.x, d.y, d.z};
    x.type = __float_as_int(d.w);
    x.hi = V3{e.x, e.y, e.z};
    x.body = __float_as_int(e.w);
    x.sid = sid;
    return x;
}

// pairs the analytic path of narrow_phase.py:198-591 finishes without falling
// through to MPR/GJK (plane-box falls through only when no corner is within
// the gap, where the plane's bounding-sphere test rejects it at once)
__device__ __forceinline__ bool analytic_pair(int ta, int tb) {
    if (ta == NB_GEO_SPHERE || tb == NB_GEO_SPHERE) return true;
    if (ta == NB_GEO_CAPSULE && tb == NB_GEO_CAPSULE) return true;
    if (ta == NB_GEO_PLANE && (tb == NB_GEO_CAPSULE || tb == NB_GEO_BOX)) return true;
    return false;
}

constexpr int kQB = 160;  // staged queue items per warp and class (> 128 = one chunk's maximum)

// push a warp's staged items: analytic queue from the front (sign = 0), MPR/GJK
// queue from the back (index `back - k`)
__device__ __forceinline__ void flush_queue(const int2* buf, int n, int32_t* counter, int2* queue, long long back,
                                            int lane) {
    if (n == 0) return;
    int base = 0;
    if (lane == 0) base = atomicAdd(counter, n);
    base = __shfl_sync(kFull, base, 0);
    for (int i = lane; i < n; i += 32) {
        const long long k = (long long)base + i;
        queue[back ? back - k : k] = buf[i];
    }
    __syncwarp();
}

// world transform, AABB and full geometry of every shape slot of world w;
// slot i < nloc is world shape s0 + i, slot nloc + g the global shape g
__device__ __forceinline__ void stage_shapes(const NbModelDesc& m, const float* __restrict__ body_q, int w, int k,
                                             float4* lo, float4* hi, float4* geom, int first, int stride) {
    const int s0 = m.world_shape_start[w];
    const int nloc = m.world_shape_start[w + 1] - s0;
    const int ns = nloc + m.global_shape_count;
    for (int i = first; i < ns; i += stride) {
        const int s = i < nloc ? s0 + i : m.global_shapes[i - nloc];
        const int b = m.shape_body[s];
        TF xs = load_tf(m.shape_transform + 7 * (size_t)s);
        TF xf = b == -1 ? xs : tf_mul(load_tf(body_q + 7 * (size_t)b), xs);
        Geom g;
        shape_geom(g, xf, m.shape_type[s], load_v3(m.shape_scale + 3 * (size_t)s), m.shape_margin[s],
                   m.shape_gap[s], m.shape_radius[s], b);
        lo[i] = make_float4(g.lo.x, g.lo.y, g.lo.z, __int_as_float(g.type));
        hi[i] = make_float4(g.hi.x, g.hi.y, g.hi.z, 0.0f);
        // global shapes are static: the first world processed stages them
        if (i < nloc || k == 0) store_geom(geom + 5 * (size_t)s, g);
    }
}

// the lane's four pairs q + 32 r (r = 0..3) of a 128-pair chunk (q = chunk
// start + lane, so neighbouring lanes read neighbouring shape slots: no bank
// conflicts): AABB overlap bits and, among the hits, the pairs the analytic
// path finishes
__device__ __forceinline__ void test_pairs(const unsigned (&pw)[4], int q, int p1, const float4* lo, const float4* hi,
                                           int ns, uint32_t* status, unsigned& hit, unsigned& easy) {
    hit = 0u;
    easy = 0u;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int p = q + 32 * r;
        if (p >= p1) continue;
        const int la = (int)(pw[r] & 0xFFFFu), lb = (int)(pw[r] >> 16);
        // slots index shared memory: never trust them blindly
        if (la >= ns || lb >= ns) {
            atomicOr(status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);
            continue;
        }
        if (la == lb) continue;
        const float4 al = lo[la], ah = hi[la], bl = lo[lb], bh = hi[lb];
        const float c = 0.0f + 0.0f;
        if (al.x <= bh.x + c && ah.x >= bl.x - c && al.y <= bh.y + c && ah.y >= bl.y - c && al.z <= bh.z + c &&
            ah.z >= bl.z - c) {
            hit |= 1u << r;
            if (analytic_pair(__float_as_int(al.w), __float_as_int(bl.w))) easy |= 1u << r;
        }
    }
}

// per-warp staging of narrow-phase queue items (pushed with one atomic per flush;
// queue order is free: every item writes only its own candidate's slots)
struct QueueStage {
    int2* qa;
    int2* qg;
    int nqa, nqg;  // warp-uniform fill levels
};

// writes a chunk's hits (bit r of this lane = pair q + 32 r) as candidates
// cand_base + running index, in pair order, and stages their queue items
__device__ __forceinline__ void emit_chunk(const NbContactSeg& seg, int2* queue, long long gjk_back, QueueStage& st,
                                           int q, unsigned hit, unsigned easy, int w, int cand_base, int lane,
                                           int& tot_h) {
    const unsigned below = (1u << lane) - 1u;
    unsigned bh[4], ba[4];
    int tot_a = 0;
    tot_h = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        bh[r] = __ballot_sync(kFull, (hit >> r) & 1u);
        ba[r] = __ballot_sync(kFull, (easy >> r) & 1u);
        tot_h += __popc(bh[r]);
        tot_a += __popc(ba[r]);
    }
    const int tot_g = tot_h - tot_a;
    // make room in the staging buffers (warp-uniform decisions)
    if (st.nqa + tot_a > kQB) {
        flush_queue(st.qa, st.nqa, &seg.work_counter[2], queue, 0, lane);
        st.nqa = 0;
    }
    if (st.nqg + tot_g > kQB) {
        flush_queue(st.qg, st.nqg, &seg.work_counter[3], queue, gjk_back, lane);
        st.nqg = 0;
    }
    int oh = 0, oa = 0;  // hits and analytic items of the rounds before r
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        if ((hit >> r) & 1u) {
            const int c = cand_base + oh + __popc(bh[r] & below);
            seg.cand[c] = q + 32 * r;
            if ((easy >> r) & 1u) st.qa[st.nqa + oa + __popc(ba[r] & below)] = make_int2(c, w);
            else st.qg[st.nqg + (oh - oa) + __popc(bh[r] & ~ba[r] & below)] = make_int2(c, w);
        }
        oh += __popc(bh[r]);
        oa += __popc(ba[r]);
    }
    st.nqa += tot_a;
    st.nqg += tot_g;
    __syncwarp();
}

struct SapScratch;
template <bool kSap>
__device__ bool world_sap_if(const NbModelDesc& m, const NbContactSeg& seg, int w, const float4* lo, const float4* hi,
                             QueueStage& st, SapScratch* sc, int lane);

// one world by one warp: shapes, then its pair chunks in order (the next chunk's
// pairs are loaded while this chunk is tested); with kSap the sweep and prune
// path runs first and the pair test only when it cannot take the world
template <bool kSap = false>
__device__ void world_by_warp(const NbModelDesc& m, const float* __restrict__ body_q, const NbContactSeg& seg, int k,
                              float4* lo, float4* hi, QueueStage& st, int lane, SapScratch* sc = nullptr) {
    const unsigned* pairs = m.pair_shapes;
    int2* queue = reinterpret_cast<int2*>(seg.queue);
    const long long gjk_back = 2 * (long long)m.pair_count - 1;
    const int w = m.world_order[k];
    const int ns = m.world_shape_start[w + 1] - m.world_shape_start[w] + m.global_shape_count;
    stage_shapes(m, body_q, w, k, lo, hi, reinterpret_cast<float4*>(seg.geom), lane, 32);
    __syncwarp();
    if constexpr (kSap) {
        if (world_sap_if<kSap>(m, seg, w, lo, hi, st, sc, lane)) return;
    }
    const int p0 = m.world_pair_start[w], p1 = m.world_pair_start[w + 1];
    int ncand = 0;
    unsigned nxt[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) nxt[r] = p0 + lane + 32 * r < p1 ? pairs[p0 + lane + 32 * r] : 0u;
    for (int base = p0; base < p1; base += 128) {
        const int q = base + lane;
        unsigned pw[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            pw[r] = nxt[r];
            nxt[r] = q + 128 + 32 * r < p1 ? pairs[q + 128 + 32 * r] : 0u;
        }
        unsigned hit, easy;
        test_pairs(pw, q, p1, lo, hi, ns, seg.status, hit, easy);
        int tot_h;
        emit_chunk(seg, queue, gjk_back, st, q, hit, easy, w, p0 + ncand, lane, tot_h);
        ncand += tot_h;
    }
    if (lane == 0) {
        seg.cand_count[w] = ncand;
        seg.world_count[w] = 0;
    }
    __syncwarp();
}

// one large world by the whole CTA: shapes staged once, the pair chunks split
// into one contiguous run per warp; pass 1 counts each run's hits, a scan over
// the warps gives every run its first candidate index, pass 2 re-tests (a few
// comparisons per pair) and writes -- the candidates stay in pair order
__device__ void world_by_cta(const NbModelDesc& m, const float* __restrict__ body_q, const NbContactSeg& seg, int k,
                             float4* lo, float4* hi, QueueStage& st, int* s_run, int warp, int lane) {
    const unsigned* pairs = m.pair_shapes;
    int2* queue = reinterpret_cast<int2*>(seg.queue);
    const long long gjk_back = 2 * (long long)m.pair_count - 1;
    const int w = m.world_order[k];
    const int ns = m.world_shape_start[w + 1] - m.world_shape_start[w] + m.global_shape_count;
    stage_shapes(m, body_q, w, k, lo, hi, reinterpret_cast<float4*>(seg.geom), threadIdx.x, kBT);
    __syncthreads();
    const int p0 = m.world_pair_start[w], p1 = m.world_pair_start[w + 1];
    const int cbase = p0;
    const int nchunks = (p1 - cbase + 127) / 128;
    constexpr int kWarps = kBT / 32;
    const int per = (nchunks + kWarps - 1) / kWarps;
    const int c0 = warp * per, c1 = min(nchunks, c0 + per);
    int count = 0;
    for (int c = c0; c < c1; ++c) {
        const int q = cbase + 128 * c + lane;
        unsigned pw[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) pw[r] = q + 32 * r < p1 ? pairs[q + 32 * r] : 0u;
        unsigned hit, easy;
        test_pairs(pw, q, p1, lo, hi, ns, seg.status, hit, easy);
        count += __popc(hit);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(kFull, count, o);
    if (lane == 0) s_run[warp] = count;
    __syncthreads();
    int first = 0, total = 0;
#pragma unroll
    for (int i = 0; i < kWarps; ++i) {
        const int v = s_run[i];
        if (i < warp) first += v;
        total += v;
    }
    int ncand = 0;
    for (int c = c0; c < c1; ++c) {
        const int q = cbase + 128 * c + lane;
        unsigned pw[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) pw[r] = q + 32 * r < p1 ? pairs[q + 32 * r] : 0u;
        unsigned hit, easy;
        test_pairs(pw, q, p1, lo, hi, ns, seg.status, hit, easy);
        int tot_h;
        emit_chunk(seg, queue, gjk_back, st, q, hit, easy, w, p0 + first + ncand, lane, tot_h);
        ncand += tot_h;
    }
    if (threadIdx.x == 0) {
        seg.cand_count[w] = total;
        seg.world_count[w] = 0;
    }
    __syncthreads();  // shapes and run counts are reused by the next world
}

// ---- sweep and prune (broad_phase="sap"; broad_phase_sap.py:397-677)

constexpr int kSapShapes = 256;  // shape slots of a world the warp sorts in shared memory
constexpr int kSapHits = 512;    // overlapping pairs one world may collect before falling back to the pair test

struct SapScratch {
    float key[kSapShapes];  // lo.x of the sorted slots (+inf padding)
    int idx[kSapShapes];    // slot at each sorted position
    int hit[kSapHits];      // pair indices of the overlaps found
    int nhit;
};

// global shape index of world slot l
__device__ __forceinline__ int slot_shape(const NbModelDesc& m, int s0, int nloc, int l) {
    return l < nloc ? s0 + l : m.global_shapes[l - nloc];
}

// index of the pair (sa, sb) of global shapes in the world's pair list [p0, p1) (sorted by (sa, sb),
// the pair list's key order), or -1
__device__ __forceinline__ int find_pair(const NbModelDesc& m, int p0, int p1, int s0, int nloc, int sa, int sb) {
    const long long want = ((long long)sa << 32) | (unsigned)sb;
    int lo = p0, hi = p1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const unsigned pw = m.pair_shapes[mid];
        const int a = slot_shape(m, s0, nloc, (int)(pw & 0xFFFFu)), b = slot_shape(m, s0, nloc, (int)(pw >> 16));
        const long long have = ((long long)a << 32) | (unsigned)b;
        if (have < want) lo = mid + 1;
        else hi = mid;
    }
    if (lo < p1) {
        const unsigned pw = m.pair_shapes[lo];
        if (slot_shape(m, s0, nloc, (int)(pw & 0xFFFFu)) == sa && slot_shape(m, s0, nloc, (int)(pw >> 16)) == sb)
            return lo;
    }
    return -1;
}

// warp-wide bitonic sort of n (a power of two) (key, value) pairs, ascending by (key, value)
__device__ __forceinline__ void warp_bitonic(float* key, int* val, int n, int lane) {
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < n / 2; t += 32) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const bool up = (i & size) == 0;
                const float ki = key[i], kj = key[j];
                const int vi = val[i], vj = val[j];
                const bool gt = ki > kj || (ki == kj && vi > vj);
                if (gt == up) {
                    key[i] = kj;
                    key[j] = ki;
                    val[i] = vj;
                    val[j] = vi;
                }
            }
            __syncwarp();
        }
    }
}

// emits one candidate per lane (pair index p when `valid`), the warp's candidates in lane order
__device__ __forceinline__ void emit_hits(const NbContactSeg& seg, int2* queue, long long gjk_back, QueueStage& st,
                                          int p, bool valid, bool easy, int w, int cand_base, int lane, int& tot) {
    const unsigned below = (1u << lane) - 1u;
    const unsigned bh = __ballot_sync(kFull, valid);
    const unsigned ba = __ballot_sync(kFull, valid && easy);
    tot = __popc(bh);
    const int tot_a = __popc(ba), tot_g = tot - tot_a;
    if (st.nqa + tot_a > kQB) {
        flush_queue(st.qa, st.nqa, &seg.work_counter[2], queue, 0, lane);
        st.nqa = 0;
    }
    if (st.nqg + tot_g > kQB) {
        flush_queue(st.qg, st.nqg, &seg.work_counter[3], queue, gjk_back, lane);
        st.nqg = 0;
    }
    if (valid) {
        const int c = cand_base + __popc(bh & below);
        seg.cand[c] = p;
        if (easy) st.qa[st.nqa + __popc(ba & below)] = make_int2(c, w);
        else st.qg[st.nqg + __popc(bh & ~ba & below)] = make_int2(c, w);
    }
    st.nqa += tot_a;
    st.nqg += tot_g;
    __syncwarp();
}

// One world by one warp with sweep and prune: the shape slots sorted by AABB
// lower x; every slot sweeps the slots after it while their lower x is within
// its upper x (exactly the pairs that overlap along x) and tests y and z with
// the pair test's predicate; overlaps whose pair is in the world's pair list
// (the world, collision-group and filter rules the list encodes) are
// collected, sorted by pair index and emitted in that order -- the same
// candidates, in the same order, as testing every pair.  Returns false (and
// emits nothing) when the world has more slots or overlaps than the shared
// buffers hold; the caller then tests every pair.
__device__ bool world_by_warp_sap(const NbModelDesc& m, const NbContactSeg& seg, int w, const float4* lo,
                                  const float4* hi, QueueStage& st, SapScratch& sc, int lane) {
    const int s0 = m.world_shape_start[w];
    const int nloc = m.world_shape_start[w + 1] - s0;
    const int ns = nloc + m.global_shape_count;
    if (ns > kSapShapes) return false;
    int n = 32;
    while (n < ns) n <<= 1;
    for (int i = lane; i < n; i += 32) {
        float k = i < ns ? lo[i].x : INFINITY;
        if (k != k) k = INFINITY;  // a NaN box overlaps nothing (all its comparisons fail)
        sc.key[i] = k;
        sc.idx[i] = i;
    }
    if (lane == 0) sc.nhit = 0;
    __syncwarp();
    warp_bitonic(sc.key, sc.idx, n, lane);
    const int p0 = m.world_pair_start[w], p1 = m.world_pair_start[w + 1];
    const int32_t* tbl = m.pair_table ? m.pair_table + m.world_table_start[w] : nullptr;
    for (int i = lane; i < ns; i += 32) {
        const int a = sc.idx[i];
        if (a >= ns) continue;
        const float4 al = lo[a], ah = hi[a];
        const int ta = __float_as_int(al.w);
        for (int j = i + 1; j < ns; ++j) {
            if (!(sc.key[j] <= ah.x)) break;
            const int b = sc.idx[j];
            const float4 bl = lo[b], bh = hi[b];
            if (!(al.x <= bh.x && ah.x >= bl.x && al.y <= bh.y && ah.y >= bl.y && al.z <= bh.z && ah.z >= bl.z))
                continue;
            int pidx;
            if (tbl) {
                // the world's dense slot-pair table: one load
                pidx = __ldg(tbl + (size_t)a * ns + b);
            } else {
                const int tb = __float_as_int(bl.w);
                const int ga = slot_shape(m, s0, nloc, a), gb = slot_shape(m, s0, nloc, b);
                // the pair list orders each pair by shape type (narrow_phase.py:207-210); equal types keep
                // the list's own order, so both orientations are looked up
                if (ta < tb) pidx = find_pair(m, p0, p1, s0, nloc, ga, gb);
                else if (ta > tb) pidx = find_pair(m, p0, p1, s0, nloc, gb, ga);
                else {
                    pidx = find_pair(m, p0, p1, s0, nloc, ga, gb);
                    if (pidx < 0) pidx = find_pair(m, p0, p1, s0, nloc, gb, ga);
                }
            }
            if (pidx < p0 || pidx >= p1) continue;  // -1: not a listed pair
            const int h = atomicAdd(&sc.nhit, 1);
            if (h < kSapHits) sc.hit[h] = pidx;
        }
    }
    __syncwarp();
    const int nh = sc.nhit;
    if (nh > kSapHits) return false;
    // sort the overlaps by pair index (padded with INT_MAX to a power of two <= kSapHits)
    int n2 = 32;
    while (n2 < nh) n2 <<= 1;
    for (int i = nh + lane; i < n2; i += 32) sc.hit[i] = 0x7fffffff;
    __syncwarp();
    for (int size = 2; size <= n2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < n2 / 2; t += 32) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const bool up = (i & size) == 0;
                const int vi = sc.hit[i], vj = sc.hit[j];
                if ((vi > vj) == up) {
                    sc.hit[i] = vj;
                    sc.hit[j] = vi;
                }
            }
            __syncwarp();
        }
    }
    int2* queue = reinterpret_cast<int2*>(seg.queue);
    const long long gjk_back = 2 * (long long)m.pair_count - 1;
    int ncand = 0;
    for (int base = 0; base < nh; base += 32) {
        const int h = base + lane;
        const bool valid = h < nh;
        int p = 0;
        bool easy = false;
        if (valid) {
            p = sc.hit[h];
            const unsigned pw = m.pair_shapes[p];
            easy = analytic_pair(__float_as_int(lo[pw & 0xFFFFu].w), __float_as_int(lo[pw >> 16].w));
        }
        int tot;
        emit_hits(seg, queue, gjk_back, st, p, valid, easy, w, p0 + ncand, lane, tot);
        ncand += tot;
    }
    if (lane == 0) {
        seg.cand_count[w] = ncand;
        seg.world_count[w] = 0;
    }
    __syncwarp();
    return true;
}

template <bool kSap>
__device__ bool world_sap_if(const NbModelDesc& m, const NbContactSeg& seg, int w, const float4* lo, const float4* hi,
                             QueueStage& st, SapScratch* sc, int lane) {
    return world_by_warp_sap(m, seg, w, lo, hi, st, *sc, lane);
}

constexpr int kCtaWorldPairs = 2048;  // worlds with at least this many pairs are shared by a whole CTA

// Worlds are taken in decreasing cost.  While the next world is large, the CTA
// takes it together (world_by_cta); from the first small world on, every warp
// takes worlds on its own (world_by_warp).
// kSap (broad_phase="sap"): every world by one warp, sweep and prune first.
template <bool kSap>
__global__ void __launch_bounds__(kBT)
broadphase_kernel(NbModelDesc m, const float* __restrict__ body_q, NbContactSeg seg) {
    extern __shared__ __align__(16) float4 sbox[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nsh = m.max_world_shapes;
    float4* lo = sbox + (size_t)warp * 2 * nsh;   // (lo.xyz, type)
    float4* hi = lo + nsh;                         // (hi.xyz, 0)
    __shared__ int2 s_qa[kBT / 32][kQB], s_qg[kBT / 32][kQB];
    __shared__ int s_k, s_run[kBT / 32];
    QueueStage st{s_qa[warp], s_qg[warp], 0, 0};
    if constexpr (kSap) {
        // sweep-and-prune scratch of every warp after the warps' box arrays (dynamic shared memory)
        SapScratch* s_sap = reinterpret_cast<SapScratch*>(sbox + (size_t)(kBT / 32) * 2 * nsh);
        for (;;) {
            int k = 0;
            if (lane == 0) k = atomicAdd(&seg.work_counter[0], 1);
            k = __shfl_sync(kFull, k, 0);
            if (k >= m.world_count) break;
            world_by_warp<true>(m, body_q, seg, k, lo, hi, st, lane, &s_sap[warp]);
        }
        int2* queue = reinterpret_cast<int2*>(seg.queue);
        flush_queue(st.qa, st.nqa, &seg.work_counter[2], queue, 0, lane);
        flush_queue(st.qg, st.nqg, &seg.work_counter[3], queue, 2 * (long long)m.pair_count - 1, lane);
        return;
    }
    int small_k = -1;  // the first small world this CTA took: warp 0 does it
    for (;;) {
        if (threadIdx.x == 0) s_k = atomicAdd(&seg.work_counter[0], 1);
        __syncthreads();
        const int k = s_k;
        __syncthreads();
        if (k >= m.world_count) break;
        const int w = m.world_order[k];
        if (m.world_pair_start[w + 1] - m.world_pair_start[w] < kCtaWorldPairs) {
            small_k = k;
            break;
        }
        // the CTA shares warp 0's shape arrays for this world
        world_by_cta(m, body_q, seg, k, sbox, sbox + nsh, st, s_run, warp, lane);
    }
    if (small_k >= 0 && warp == 0) world_by_warp(m, body_q, seg, small_k, lo, hi, st, lane);
    if (small_k >= 0) {
        for (;;) {
            int k = 0;
            if (lane == 0) k = atomicAdd(&seg.work_counter[0], 1);
            k = __shfl_sync(kFull, k, 0);
            if (k >= m.world_count) break;
            world_by_warp(m, body_q, seg, k, lo, hi, st, lane);
        }
    }
    int2* queue = reinterpret_cast<int2*>(seg.queue);
    flush_queue(st.qa, st.nqa, &seg.work_counter[2], queue, 0, lane);
    flush_queue(st.qg, st.nqg, &seg.work_counter[3], queue, 2 * (long long)m.pair_count - 1, lane);
}

struct NarrowItem {
    int c, w;
    Geom ga, gb;
    Writer wr;
};

// false (and NB_STATUS_CONTACT_OVERFLOW) for a queue entry whose candidate or world is out of range --
// never produced by the broad phase; the check keeps a corrupted queue from indexing past the arrays
__device__ __forceinline__ bool narrow_setup(const NbModelDesc& m, const NbContactSeg& seg, const float* body_q,
                                             int2 e, NarrowItem& it) {
    const float4* geom = reinterpret_cast<const float4*>(seg.geom);
    it.c = e.x;
    it.w = e.y;
    if ((unsigned)it.c >= (unsigned)m.pair_count || (unsigned)it.w >= (unsigned)m.world_count ||
        (unsigned)seg.cand[it.c] >= (unsigned)m.pair_count) {
        atomicOr(seg.status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);
        return false;
    }
    const unsigned pw = reinterpret_cast<const unsigned*>(m.pair_shapes)[seg.cand[it.c]];
    const int la = (int)(pw & 0xFFFFu), lb = (int)(pw >> 16);
    const int s0 = m.world_shape_start[it.w];
    const int nloc = m.world_shape_start[it.w + 1] - s0;
    const int sa = la < nloc ? s0 + la : m.global_shapes[la - nloc];
    const int sb = lb < nloc ? s0 + lb : m.global_shapes[lb - nloc];
    it.ga = load_geom(geom + 5 * (size_t)sa, sa);
    it.gb = load_geom(geom + 5 * (size_t)sb, sb);
    const int b0 = m.world_body_start[it.w];
    it.wr.slots = reinterpret_cast<float4*>(seg.slots) + (size_t)it.c * kSlotF4;
    it.wr.n = 0;
    it.wr.inv_a = it.ga.body == -1 ? tf_identity() : tf_inverse(load_tf(body_q + 7 * (size_t)it.ga.body));
    it.wr.inv_b = it.gb.body == -1 ? tf_identity() : tf_inverse(load_tf(body_q + 7 * (size_t)it.gb.body));
    it.wr.gap = it.ga.gap + it.gb.gap;
    it.wr.shape_a = sa;
    it.wr.shape_b = sb;
    const int lba = it.ga.body < 0 ? -1 : it.ga.body - b0;
    const int lbb = it.gb.body < 0 ? -1 : it.gb.body - b0;
    it.wr.tag = ((lba + 1) & 0xFFF) | (((lbb + 1) & 0xFFF) << 12);
    return true;
}

__device__ __forceinline__ void narrow_finish(const NbContactSeg& seg, const NarrowItem& it) {
    seg.counts[it.c] = (uint8_t)it.wr.n;
    if (it.wr.n) atomicAdd(&seg.world_count[it.w], it.wr.n);
}

// analytic queue: sphere / capsule / plane pairs; a plane-box pair with no
// corner inside the gap is forwarded to the MPR/GJK queue (narrow_phase.py:598-603)
__global__ void __launch_bounds__(kNT)
narrow_analytic_kernel(NbModelDesc m, const float* __restrict__ body_q, NbContactSeg seg) {
    const int n0 = seg.work_counter[2];
    const int P = m.pair_count;
    int2* queue = reinterpret_cast<int2*>(seg.queue);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n0; i += gridDim.x * blockDim.x) {
        const int2 e = queue[i];
        NarrowItem it;
        if (!narrow_setup(m, seg, body_q, e, it)) continue;
        if (narrow_analytic(it.wr, it.ga, it.gb)) {
            narrow_finish(seg, it);
        } else {
            const int k = atomicAdd(&seg.work_counter[3], 1);
            queue[2 * (size_t)P - 1 - k] = e;
        }
    }
}

// ---- separation prefilter of the MPR/GJK queue

__device__ __forceinline__ V3 mat_col(const M33& r, int k) { return V3{r.m[0][k], r.m[1][k], r.m[2][k]}; }

__device__ __forceinline__ float bounding_radius(const Geom& g) {
    if (g.type == NB_GEO_BOX) return length(g.scale);
    if (g.type == NB_GEO_CAPSULE) return g.scale.x + g.scale.y;
    return g.scale.x;  // sphere
}

// extent of a box (half extents h, axes R) along unit axis L
__device__ __forceinline__ float box_extent(const M33& R, V3 h, V3 L) {
    return fabsf(dot(L, mat_col(R, 0))) * h.x + fabsf(dot(L, mat_col(R, 1))) * h.y +
           fabsf(dot(L, mat_col(R, 2))) * h.z;
}

// True only when the pair provably produces no contact: a lower bound of the
// distance between the two shapes (bounding spheres; separating axes for
// box-box and capsule-box; the signed distance of the bounding sphere for an
// infinite plane) exceeds the contact threshold gap_a + gap_b + margin_a +
// margin_b by a slack that covers fp32 rounding and MPR's 1e-4 inflation.  Such
// a pair makes MPR find no overlap and leaves the GJK distance above the
// threshold (narrow_phase.py:627-776, collision_core.py:626-725), so the
// reference path writes nothing for it either.
__device__ __noinline__ bool gjk_pair_separated(const Geom& a, const Geom& b) {
    const V3 pa = a.xf.p, pb = b.xf.p;
    const float mag = fmaxf(fmaxf(fabsf(pa.x), fmaxf(fabsf(pa.y), fabsf(pa.z))),
                            fmaxf(fabsf(pb.x), fmaxf(fabsf(pb.y), fabsf(pb.z))));
    const float thr = a.gap + b.gap + a.margin + b.margin + 2.0e-3f + 1.0e-5f * mag;
    if (a.type == NB_GEO_PLANE || b.type == NB_GEO_PLANE) {
        const Geom& pl = a.type == NB_GEO_PLANE ? a : b;
        const Geom& o = a.type == NB_GEO_PLANE ? b : a;
        if (o.type == NB_GEO_PLANE || pl.scale.x != 0.0f || pl.scale.y != 0.0f) return false;  // finite planes
        const V3 n = qrot(pl.xf.q, V3{0.0f, 0.0f, 1.0f});
        return dot(sub(o.xf.p, pl.xf.p), n) - bounding_radius(o) > thr;
    }
    const V3 d = sub(pb, pa);
    if (length(d) - bounding_radius(a) - bounding_radius(b) > thr) return true;
    const bool box_a = a.type == NB_GEO_BOX, box_b = b.type == NB_GEO_BOX;
    if (box_a && box_b) {
        const M33 Ra = quat_to_matrix(a.xf.q), Rb = quat_to_matrix(b.xf.q);
        for (int i = 0; i < 3; ++i) {
            V3 L = mat_col(Ra, i);
            if (fabsf(dot(d, L)) - box_extent(Ra, a.scale, L) - box_extent(Rb, b.scale, L) > thr) return true;
            L = mat_col(Rb, i);
            if (fabsf(dot(d, L)) - box_extent(Ra, a.scale, L) - box_extent(Rb, b.scale, L) > thr) return true;
        }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const V3 c = cross(mat_col(Ra, i), mat_col(Rb, j));
                const float len = length(c);
                if (!(len > 1.0e-3f)) continue;  // near-parallel edges: covered by the face axes
                const V3 L = smul(1.0f / len, c);
                if (fabsf(dot(d, L)) - box_extent(Ra, a.scale, L) - box_extent(Rb, b.scale, L) > thr) return true;
            }
        return false;
    }
    if ((box_a && b.type == NB_GEO_CAPSULE) || (box_b && a.type == NB_GEO_CAPSULE)) {
        const Geom& bx = box_a ? a : b;
        const Geom& cp = box_a ? b : a;
        const M33 Rb = quat_to_matrix(bx.xf.q);
        const V3 u = qrot(cp.xf.q, V3{0.0f, 0.0f, 1.0f});
        const float r = cp.scale.x, hh = cp.scale.y;
        for (int i = 0; i < 4; ++i) {
            const V3 L = i < 3 ? mat_col(Rb, i) : u;
            if (fabsf(dot(d, L)) - box_extent(Rb, bx.scale, L) - (fabsf(dot(u, L)) * hh + r) > thr) return true;
        }
        for (int i = 0; i < 3; ++i) {
            const V3 c = cross(u, mat_col(Rb, i));
            const float len = length(c);
            if (!(len > 1.0e-3f)) continue;
            const V3 L = smul(1.0f / len, c);
            if (fabsf(dot(d, L)) - box_extent(Rb, bx.scale, L) - (fabsf(dot(u, L)) * hh + r) > thr) return true;
        }
    }
    return false;
}

// One thread per MPR/GJK item: provably separated pairs get zero contacts,
// the rest are compacted (warp-aggregated) into the queue's front, which the
// analytic kernel has consumed: box-box items from index 0 up, every other
// pair type from index n1 - 1 down, so the MPR/GJK kernel's warps mostly run
// one pair type (fewer divergent branches, one code path in the instruction
// cache).  Front and back cannot overlap (the back holds n1 <= pair_count
// items of 2 * pair_count).
__global__ void __launch_bounds__(kNT)
gjk_prefilter_kernel(NbModelDesc m, NbContactSeg seg) {
    const int n1 = seg.work_counter[3];
    const int P = m.pair_count;
    int2* queue = reinterpret_cast<int2*>(seg.queue);
    const float4* geom = reinterpret_cast<const float4*>(seg.geom);
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n1; base += stride) {
        const int i = base + lane;
        bool keep = false, boxes = false;
        int2 e = make_int2(0, 0);
        if (i < n1) {
            e = queue[2 * (size_t)P - 1 - i];
            const unsigned pw = reinterpret_cast<const unsigned*>(m.pair_shapes)[seg.cand[e.x]];
            const int la = (int)(pw & 0xFFFFu), lb = (int)(pw >> 16);
            const int s0 = m.world_shape_start[e.y];
            const int nloc = m.world_shape_start[e.y + 1] - s0;
            const int sa = la < nloc ? s0 + la : m.global_shapes[la - nloc];
            const int sb = lb < nloc ? s0 + lb : m.global_shapes[lb - nloc];
            const Geom ga = load_geom(geom + 5 * (size_t)sa, sa), gb = load_geom(geom + 5 * (size_t)sb, sb);
            keep = !gjk_pair_separated(ga, gb);
            boxes = ga.type == NB_GEO_BOX && gb.type == NB_GEO_BOX;
            if (!keep) seg.counts[e.x] = 0;
        }
        const unsigned below = (1u << lane) - 1u;
        const unsigned bal0 = __ballot_sync(kFull, keep && boxes);
        const unsigned bal1 = __ballot_sync(kFull, keep && !boxes);
        int off0 = 0, off1 = 0;
        if (lane == 0 && bal0) off0 = atomicAdd(&seg.work_counter[5], __popc(bal0));
        if (lane == 0 && bal1) off1 = atomicAdd(&seg.work_counter[6], __popc(bal1));
        off0 = __shfl_sync(kFull, off0, 0);
        off1 = __shfl_sync(kFull, off1, 0);
        if (keep && boxes) queue[off0 + __popc(bal0 & below)] = e;
        if (keep && !boxes) queue[n1 - 1 - (off1 + __popc(bal1 & below))] = e;
    }
}

// MPR / GJK on the items that survived the prefilter, then the manifolds in a
// second kernel.  Almost every item runs MPR (which rarely finds an overlap),
// then GJK, and about nine in ten then build a manifold (polygon clipping in
// local arrays): split in two kernels, each warp runs one of the two code
// paths at a time and each kernel's code is half the size in the instruction
// cache.  An item that needs a manifold leaves its witness points and normal
// (relative frame) in its own last contact slot -- unused until the manifold
// writes its contacts, read before that -- and its queue entry in the
// queue's back half, which the prefilter has consumed: box-box items from
// the top down, the others from the bottom of that region up (the items
// never exceed the n1 <= pair_count entries the region held).
// Latency and divergence bound: 12 CTAs per SM (48 warps, 40 registers, a
// few bytes of spills) hide more of it than 6, 8, 10 or 16 (measured) or the
// unconstrained 122 registers at 4 CTAs.
__global__ void __launch_bounds__(kNT, kGjkMinBlocks)
narrow_gjk_kernel(NbModelDesc m, const float* __restrict__ body_q, NbContactSeg seg) {
    const int n_box = seg.work_counter[5], n_other = seg.work_counter[6], n1 = seg.work_counter[3];
    const int n = n_box + n_other;
    int2* queue = reinterpret_cast<int2*>(seg.queue);
    const long long top = 2 * (long long)m.pair_count - 1;
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int i = base + lane;
        const bool box = i < n_box;
        bool manifold = false;
        int2 e = make_int2(0, 0);
        if (i < n) {
            e = box ? queue[i] : queue[n1 - 1 - (i - n_box)];
            NarrowItem it;
            if (narrow_setup(m, seg, body_q, e, it)) {
                V3 pa, pb, nrm;
                manifold = gjk_stage(it.wr, it.ga, it.gb, pa, pb, nrm);
                if (manifold) {
                    float4* h = it.wr.slots + kSlotF4 - 3;
                    h[0] = make_float4(pa.x, pa.y, pa.z, 0.0f);
                    h[1] = make_float4(pb.x, pb.y, pb.z, 0.0f);
                    h[2] = make_float4(nrm.x, nrm.y, nrm.z, 0.0f);
                } else {
                    narrow_finish(seg, it);
                }
            }
        }
        const unsigned below = (1u << lane) - 1u;
        const unsigned bb = __ballot_sync(kFull, manifold && box);
        const unsigned bo = __ballot_sync(kFull, manifold && !box);
        int ob = 0, oo = 0;
        if (lane == 0 && bb) ob = atomicAdd(&seg.work_counter[1], __popc(bb));
        if (lane == 0 && bo) oo = atomicAdd(&seg.work_counter[7], __popc(bo));
        ob = __shfl_sync(kFull, ob, 0);
        oo = __shfl_sync(kFull, oo, 0);
        if (manifold && box) queue[top - (ob + __popc(bb & below))] = e;
        if (manifold && !box) queue[top - n1 + 1 + (oo + __popc(bo & below))] = e;
    }
}

__global__ void __launch_bounds__(kNT, kManifoldMinBlocks)
narrow_manifold_kernel(NbModelDesc m, const float* __restrict__ body_q, NbContactSeg seg) {
    const int n1 = seg.work_counter[3];
    int nb = seg.work_counter[1], no = seg.work_counter[7];
    // never more than the items the MPR/GJK kernel read; the clamps keep corrupted
    // counters inside the queue's back region
    nb = nb < 0 ? 0 : (nb > n1 ? n1 : nb);
    no = no < 0 ? 0 : (no > n1 - nb ? n1 - nb : no);
    const int2* queue = reinterpret_cast<const int2*>(seg.queue);
    const long long top = 2 * (long long)m.pair_count - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb + no; i += gridDim.x * blockDim.x) {
        const int2 e = i < nb ? queue[top - i] : queue[top - n1 + 1 + (i - nb)];
        NarrowItem it;
        if (!narrow_setup(m, seg, body_q, e, it)) continue;
        const float4* h = it.wr.slots + kSlotF4 - 3;
        const float4 h0 = h[0], h1 = h[1], h2 = h[2];
        gjk_manifold(it.wr, it.ga, it.gb, V3{h0.x, h0.y, h0.z}, V3{h1.x, h1.y, h1.z}, V3{h2.x, h2.y, h2.z});
        narrow_finish(seg, it);
    }
}

// Exclusive scan of world contact counts (single CTA) -> world_offset[W+1]
// (public arrays) and world_base[W] (solver records; same offsets), count[0]
// = total (may exceed the public capacity, as in the reference).
__global__ void __launch_bounds__(1024) world_scan_kernel(int W, int32_t* __restrict__ world_count,
                                                          int64_t* world_offset, int64_t* world_base,
                                                          int32_t* count_out, int cap, uint32_t* status,
                                                          int32_t* generation) {
    __shared__ int64_t warp_sums[32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < W; base += 1024) {
        int i = base + threadIdx.x;
        int64_t v = i < W ? world_count[i] : 0;
        int64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t run = 0;
            for (int k = 0; k < 32; ++k) {
                int64_t t = warp_sums[k];
                warp_sums[k] = run;
                run += t;
            }
        }
        __syncthreads();
        int64_t excl = carry + warp_sums[warp] + x - v;
        if (i < W) {
            world_offset[i] = excl;
            world_base[i] = excl;
            // the solver records hold the first `cap` contacts (those the public arrays hold): a world
            // past the capacity keeps only its records below it
            const int64_t room = (int64_t)cap - excl;
            if (v > room) world_count[i] = (int32_t)(room > 0 ? room : 0);
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        world_offset[W] = carry;
        count_out[0] = carry > 0x7fffffff ? 0x7fffffff : (int32_t)carry;
        if (carry > cap) atomicOr(status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);
        if (generation) {
            // Contacts.contact_generation, bumped once per collide with the wraparound of
            // compute_shape_aabbs (collide.py:211-218)
            const int32_t g = generation[0];
            generation[0] = g == 2147483647 ? 0 : g + 1;
        }
    }
}

// Dense public Contacts arrays ordered by (world, key), and the same contacts
// as solver records (rec), contiguous per world; one warp per world.  The
// warp scans the contact counts of 32 candidates at a time, then its lanes
// take the chunk's outputs in order (lane k writes output k, k + 32, ...),
// each finding its candidate among the 32 scanned counts, so consecutive
// lanes store to consecutive rows of every array.
__global__ void __launch_bounds__(256) publish_kernel(NbModelDesc m, NbContactSeg seg, NbContactsPublic pub) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const float4* slots = reinterpret_cast<const float4*>(seg.slots);
    float4* rec = reinterpret_cast<float4*>(seg.rec);
    for (int w = gw; w < m.world_count; w += nw) {
        const int c0 = m.world_pair_start[w];
        // a world's candidates never exceed its pairs, a candidate's contacts never exceed 5; the
        // clamps keep corrupted counts from indexing past the slots
        const int npair = m.world_pair_start[w + 1] - c0;
        int nc = seg.cand_count[w];
        nc = nc < 0 ? 0 : (nc > npair ? npair : nc);
        const int64_t dst0 = pub.world_offset[w];
        int64_t running = 0;
        for (int base = 0; base < nc; base += 32) {
            const int i = base + lane;
            int n = i < nc ? (int)seg.counts[c0 + i] : 0;
            n = n > 5 ? 5 : n;
            int x = n;  // inclusive scan of the chunk's counts
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(kFull, x, o);
                if (lane >= o) x += y;
            }
            const int tot = __shfl_sync(kFull, x, 31);
            for (int o0 = 0; o0 < tot; o0 += 32) {
                const int o = o0 + lane;
                // source lane: the number of lanes whose inclusive sum is <= o
                int src = 0;
#pragma unroll
                for (int k = 0; k < 32; ++k) src += __shfl_sync(kFull, x, k) <= o ? 1 : 0;
                const int src_c = src < 31 ? src : 31;
                const int x_src = __shfl_sync(kFull, x, src_c);
                const int n_src = __shfl_sync(kFull, n, src_c);
                if (o >= tot) continue;
                const int j = o - (x_src - n_src);
                const int64_t d = dst0 + running + o;
                const float4* sl = slots + ((size_t)(c0 + base + src) * 5 + j) * 5;
                const float4 a = sl[0], b = sl[1], c = sl[2], e = sl[3], f = sl[4];
                // solver record: the tag moves next to the normal so the
                // penetration test reads the first 48 bytes only
                // rec and the public rows hold the first `capacity` contacts (world_scan_kernel flagged
                // an overflow and clamped the worlds' solver counts; a negative offset is corrupt)
                if (d < 0 || d >= pub.capacity) continue;
                float4* r = rec + (size_t)d * 5;
                r[0] = a;
                r[1] = b;
                r[2] = make_float4(c.x, c.y, c.z, f.w);
                r[3] = make_float4(e.x, e.y, e.z, c.w);
                r[4] = make_float4(f.x, f.y, f.z, e.w);
                if (seg.rec_index) seg.rec_index[d] = (int32_t)d;
                const int s0 = __float_as_int(c.w), s1 = __float_as_int(e.w);
                pub.shape0[d] = s0;
                pub.shape1[d] = s1;
                pub.point0[3 * d] = a.x; pub.point0[3 * d + 1] = a.y; pub.point0[3 * d + 2] = a.z;
                pub.point1[3 * d] = b.x; pub.point1[3 * d + 1] = b.y; pub.point1[3 * d + 2] = b.z;
                pub.normal[3 * d] = c.x; pub.normal[3 * d + 1] = c.y; pub.normal[3 * d + 2] = c.z;
                pub.offset0[3 * d] = e.x; pub.offset0[3 * d + 1] = e.y; pub.offset0[3 * d + 2] = e.z;
                pub.offset1[3 * d] = f.x; pub.offset1[3 * d + 1] = f.y; pub.offset1[3 * d + 2] = f.z;
                pub.margin0[d] = a.w;
                pub.margin1[d] = b.w;
                if (pub.sort_key) {
                    const int sub = (__float_as_int(f.w) >> 24) & 0xFF;
                    pub.sort_key[d] = ((int64_t)(s0 & 0xFFFFF) << 43) | ((int64_t)(s1 & 0xFFFFF) << 23) | (int64_t)sub;
                }
            }
            running += tot;
        }
    }
}

// Custom contacts in the public arrays -> solver records, in three kernels.
// ingest_bucket_kernel finds each public contact's world and appends its
// public index to the world's bucket (world_pair_start[w]*5 + k: every world
// owns room for 5 contacts per candidate pair; the buckets live in the slots
// buffer, which collide rewrites anyway); the append order is that of the
// atomics.  ingest_scan_kernel makes the worlds' record bases (an exclusive
// scan of the bucket sizes: the records are dense, at most the public
// capacity).  ingest_place_kernel (one CTA per world) ranks every bucket
// entry by its public index and writes the record at the world's base +
// rank, so the records of a world follow the public order whatever the
// atomics did -- the order the solver sums each body's deltas in.
__global__ void ingest_bucket_kernel(NbModelDesc m, NbContactsPublic pub, NbContactSeg seg) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    int n = pub.count[0] < pub.capacity ? pub.count[0] : pub.capacity;
    if (c >= n) return;
    int s0 = pub.shape0[c], s1 = pub.shape1[c];
    if (s0 >= m.shape_count || s1 >= m.shape_count) {
        atomicOr(seg.status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);  // invalid shape index: dropped
        return;
    }
    int b0 = s0 >= 0 ? m.shape_body[s0] : -1;
    int b1 = s1 >= 0 ? m.shape_body[s1] : -1;
    int bw = b0 >= 0 ? b0 : b1;
    if (bw < 0) return;  // static-static: never moves anything
    int lo = 0, hi = m.world_count;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (m.world_body_start[mid] <= bw) lo = mid;
        else hi = mid;
    }
    const int w = lo;
    const int wb = m.world_body_start[w];
    if ((b0 >= 0 && (b0 < wb || b0 >= m.world_body_start[w + 1])) ||
        (b1 >= 0 && (b1 < wb || b1 >= m.world_body_start[w + 1]))) {
        atomicOr(seg.status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);  // cross-world contact: dropped
        return;
    }
    const int k = atomicAdd(&seg.world_count[w], 1);
    const int64_t cap = 5 * (int64_t)(m.world_pair_start[w + 1] - m.world_pair_start[w]);
    if (k >= cap) {
        atomicOr(seg.status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);
        return;
    }
    reinterpret_cast<int32_t*>(seg.slots)[(size_t)m.world_pair_start[w] * 5 + k] = c;
}

__global__ void __launch_bounds__(1024) ingest_scan_kernel(NbModelDesc m, NbContactSeg seg) {
    __shared__ int64_t warp_sums[32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int W = m.world_count;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < W; base += 1024) {
        const int i = base + threadIdx.x;
        int64_t v = 0;
        if (i < W) {
            const int room = 5 * (m.world_pair_start[i + 1] - m.world_pair_start[i]);
            const int nw = seg.world_count[i];
            v = nw < room ? nw : room;
            seg.world_count[i] = (int32_t)v;
        }
        int64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t run = 0;
            for (int k = 0; k < 32; ++k) {
                const int64_t t = warp_sums[k];
                warp_sums[k] = run;
                run += t;
            }
        }
        __syncthreads();
        const int64_t excl = carry + warp_sums[warp] + x - v;
        if (i < W) seg.world_base[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
}

constexpr int kIngestTile = 2048;  // bucket entries one CTA compares against at a time (shared memory)

__global__ void __launch_bounds__(256) ingest_place_kernel(NbModelDesc m, NbContactsPublic pub, NbContactSeg seg) {
    __shared__ int32_t s_tile[kIngestTile];
    const int w = blockIdx.x;
    const int c0 = m.world_pair_start[w];
    const int nw = seg.world_count[w];  // clamped to the world's room by ingest_scan_kernel
    const int64_t base = seg.world_base[w];
    const int32_t* bucket = reinterpret_cast<const int32_t*>(seg.slots) + 5 * (int64_t)c0;
    // rank of entry i = the number of the bucket's public indices below its own (indices are distinct)
    for (int i0 = 0; i0 < nw; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        const int32_t x = i < nw ? bucket[i] : 0;
        int rank = 0;
        for (int t0 = 0; t0 < nw; t0 += kIngestTile) {
            const int len = nw - t0 < kIngestTile ? nw - t0 : kIngestTile;
            __syncthreads();
            for (int j = threadIdx.x; j < len; j += blockDim.x) s_tile[j] = bucket[t0 + j];
            __syncthreads();
            if (i < nw)
                for (int j = 0; j < len; ++j) rank += s_tile[j] < x ? 1 : 0;
        }
        if (i >= nw) continue;
        const int c = x;
        const int s0 = pub.shape0[c], s1 = pub.shape1[c];
        const int b0 = s0 >= 0 ? m.shape_body[s0] : -1;
        const int b1 = s1 >= 0 ? m.shape_body[s1] : -1;
        const int wb = m.world_body_start[w];
        const int la = b0 < 0 ? -1 : b0 - wb, lb = b1 < 0 ? -1 : b1 - wb;
        const int tag = ((la + 1) & 0xFFF) | (((lb + 1) & 0xFFF) << 12);
        const int64_t ri = base + rank;
        if (seg.rec_index) seg.rec_index[ri] = c;
        float4* sl = reinterpret_cast<float4*>(seg.rec) + ri * 5;
        sl[0] = make_float4(pub.point0[3 * c], pub.point0[3 * c + 1], pub.point0[3 * c + 2], pub.margin0[c]);
        sl[1] = make_float4(pub.point1[3 * c], pub.point1[3 * c + 1], pub.point1[3 * c + 2], pub.margin1[c]);
        sl[2] = make_float4(pub.normal[3 * c], pub.normal[3 * c + 1], pub.normal[3 * c + 2], __int_as_float(tag));
        sl[3] = make_float4(pub.offset0[3 * c], pub.offset0[3 * c + 1], pub.offset0[3 * c + 2], __int_as_float(s0));
        sl[4] = make_float4(pub.offset1[3 * c], pub.offset1[3 * c + 1], pub.offset1[3 * c + 2], __int_as_float(s1));
    }
}

int sm_count() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace

size_t nb_collide_smem_bytes(const NbModelDesc* m) {
    return (size_t)(kBT / 32) * 2 * (size_t)m->max_world_shapes * sizeof(float4) +
           (m->broad_phase == 1 ? (kBT / 32) * sizeof(SapScratch) : 0);
}

size_t nb_collide_static_smem_bytes(const NbModelDesc*) { return (size_t)2 * (kBT / 32) * kQB * sizeof(int2); }

namespace {

// Occupancy of the narrow-phase kernels per device ordinal (a process may
// drive several GPUs; the mutex orders first calls from several host threads).
constexpr int kMaxCollideDevices = 64;
struct NarrowOccupancy {
    int analytic = 0, prefilter = 0, gjk = 0, manifold = 0;
};
std::mutex g_occ_mutex;
NarrowOccupancy g_occ[kMaxCollideDevices];

cudaError_t narrow_occupancy(NarrowOccupancy* out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxCollideDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_occ_mutex);
    NarrowOccupancy& c = g_occ[dev];
    if (!c.gjk) {
        // default grids: one wave at each kernel's occupancy (grid-stride loops)
        int a = 0, p = 0, g = 0, f = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, narrow_analytic_kernel, kNT, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, gjk_prefilter_kernel, kNT, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g, narrow_gjk_kernel, kNT, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&f, narrow_manifold_kernel, kNT, 0);
        c.analytic = a > 0 ? a : 4;
        c.prefilter = p > 0 ? p : 4;
        c.gjk = g > 0 ? g : 4;
        c.manifold = f > 0 ? f : 4;
    }
    *out = c;
    return cudaSuccess;
}

}  // namespace

cudaError_t nb_launch_collide(const NbModelDesc* m, const float* body_q, const NbContactSeg* seg, int grid,
                              cudaStream_t stream) {
    const size_t smem = nb_collide_smem_bytes(m);
    const bool sap = m->broad_phase == 1;
    cudaError_t e = nb_raise_dynamic_smem(sap ? (const void*)broadphase_kernel<true> : (const void*)broadphase_kernel<false>,
                                          smem);
    if (e != cudaSuccess) return e;
    NarrowOccupancy occ;
    e = narrow_occupancy(&occ);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(seg->work_counter, 0, 4 * sizeof(int32_t), stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(seg->work_counter + 5, 0, 3 * sizeof(int32_t), stream);
    if (e != cudaSuccess) return e;
    const int sms = sm_count();
    if (sap) broadphase_kernel<true><<<sms * 4, kBT, smem, stream>>>(*m, body_q, *seg);
    else broadphase_kernel<false><<<sms * 4, kBT, smem, stream>>>(*m, body_q, *seg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    narrow_analytic_kernel<<<grid > 0 ? grid : sms * occ.analytic, kNT, 0, stream>>>(*m, body_q, *seg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    gjk_prefilter_kernel<<<grid > 0 ? grid : sms * occ.prefilter, kNT, 0, stream>>>(*m, *seg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    narrow_gjk_kernel<<<grid > 0 ? grid : sms * occ.gjk, kNT, 0, stream>>>(*m, body_q, *seg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    narrow_manifold_kernel<<<grid > 0 ? grid : sms * occ.manifold, kNT, 0, stream>>>(*m, body_q, *seg);
    return cudaGetLastError();
}

cudaError_t nb_launch_publish(const NbModelDesc* m, const NbContactSeg* seg, const NbContactsPublic* pub,
                              cudaStream_t stream) {
    world_scan_kernel<<<1, 1024, 0, stream>>>(m->world_count, seg->world_count, pub->world_offset, seg->world_base,
                                              pub->count, pub->capacity, seg->status, pub->generation);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int blocks = (m->world_count * 32 + 255) / 256;
    publish_kernel<<<blocks < 1 ? 1 : blocks, 256, 0, stream>>>(*m, *seg, *pub);
    return cudaGetLastError();
}

cudaError_t nb_launch_ingest(const NbModelDesc* m, const NbContactsPublic* pub, const NbContactSeg* seg,
                             cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(seg->world_count, 0, sizeof(int32_t) * (size_t)m->world_count, stream);
    if (e != cudaSuccess) return e;
    if (pub->capacity > 0) {
        ingest_bucket_kernel<<<(pub->capacity + 255) / 256, 256, 0, stream>>>(*m, *pub, *seg);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    ingest_scan_kernel<<<1, 1024, 0, stream>>>(*m, *seg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ingest_place_kernel<<<m->world_count, 256, 0, stream>>>(*m, *pub, *seg);
    return cudaGetLastError();
}
