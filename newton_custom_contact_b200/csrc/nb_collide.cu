// Collision detection for many independent worlds, one world per CTA.
//
// A persistent grid pulls worlds (largest first) from a device counter.  Per
// world the CTA
//   1. computes every shape's world transform + AABB into shared memory
//      (compute_shape_aabbs, newton/_src/sim/collide.py:150-275),
//   2. tests the world's candidate pairs (explicit pair list, sorted by
//      contact key) and compacts the overlapping ones *in order* with
//      ballot/popc prefix sums (BroadPhaseExplicit,
//      newton/_src/geometry/broad_phase_nxn.py:28-66),
//   3. runs the narrow phase one candidate per thread, staging each
//      candidate's <= 5 contacts in per-CTA scratch,
//   4. block-scans the per-candidate counts and copies the contacts into the
//      world's segment, so the segment is sorted by the deterministic key
//      (shape_a, shape_b, sub_key) of newton/_src/geometry/contact_data.py:59-83
//      without a global sort (ContactSorter, contact_sort.py:194-445).
#include <cuda_runtime.h>

#include "nb_geom.cuh"
#include "nb_kernels.cuh"

namespace {

using namespace nbg;

constexpr int kCT = NB_COLLIDE_THREADS;     // threads per CTA
constexpr int kMaxCand = 2048;              // candidates buffered per pass
constexpr int kSlotF4 = 25;                 // 5 contacts x 5 float4 per candidate

__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_tmp, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tmp[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int i = 0; i < kCT / 32; ++i) {
            int t = warp_tmp[i];
            warp_tmp[i] = run;
            run += t;
        }
        warp_tmp[kCT / 32] = run;
    }
    __syncthreads();
    int excl = warp_tmp[warp] + x - v;
    total = warp_tmp[kCT / 32];
    __syncthreads();
    return excl;
}

__global__ void __launch_bounds__(kCT, 2)
collide_worlds_kernel(NbModelDesc m, const float* __restrict__ body_q, NbContactSeg seg) {
    extern __shared__ __align__(16) unsigned char smem[];
    Geom* geo = reinterpret_cast<Geom*>(smem);
    int* cand = reinterpret_cast<int*>(geo + m.max_world_shapes);
    __shared__ int s_world, s_total, s_ncand;
    __shared__ int warp_tmp[kCT / 32 + 1];

    float4* scratch = reinterpret_cast<float4*>(seg.slot_scratch) + (size_t)blockIdx.x * kCT * kSlotF4;
    float4* rec0 = reinterpret_cast<float4*>(seg.rec0);
    float4* rec1 = reinterpret_cast<float4*>(seg.rec1);
    float4* rec2 = reinterpret_cast<float4*>(seg.rec2);
    float4* rec3 = reinterpret_cast<float4*>(seg.rec3);
    float4* rec4 = reinterpret_cast<float4*>(seg.rec4);
    const int tid = threadIdx.x;

    for (;;) {
        if (tid == 0) {
            int k = atomicAdd(&seg.work_counter[0], 1);
            s_world = k < m.world_count ? m.world_order[k] : -1;
            s_total = 0;
        }
        __syncthreads();
        const int w = s_world;
        if (w < 0) break;
        const int s0 = m.world_shape_start[w];
        const int nloc = m.world_shape_start[w + 1] - s0;
        const int ns = nloc + m.global_shape_count;
        const int b0 = m.world_body_start[w];
        for (int i = tid; i < ns; i += kCT) {
            int s = i < nloc ? s0 + i : m.global_shapes[i - nloc];
            int b = m.shape_body[s];
            TF xs = load_tf(m.shape_transform + 7 * (size_t)s);
            TF xf = b == -1 ? xs : tf_mul(load_tf(body_q + 7 * (size_t)b), xs);
            Geom g;
            shape_geom(g, xf, m.shape_type[s], load_v3(m.shape_scale + 3 * (size_t)s), m.shape_margin[s],
                       m.shape_gap[s], m.shape_radius[s], b);
            g.sid = s;
            geo[i] = g;
        }
        __syncthreads();
        const int p_begin = m.world_pair_start[w], p_end = m.world_pair_start[w + 1];
        const int64_t cbase = m.contact_cap_start[w];
        const int64_t ccap = m.contact_cap_start[w + 1] - cbase;
        int pnext = p_begin;
        while (pnext < p_end) {
            // ---- broad phase: ordered compaction of overlapping pairs
            if (tid == 0) s_ncand = 0;
            __syncthreads();
            while (pnext < p_end && s_ncand + kCT <= kMaxCand) {
                int p = pnext + tid;
                bool hit = false;
                if (p < p_end) {
                    int la = m.pair_shapes[2 * (size_t)p], lb = m.pair_shapes[2 * (size_t)p + 1];
                    // slots index the shared geometry table: never trust them blindly
                    bool valid = (unsigned)la < (unsigned)ns && (unsigned)lb < (unsigned)ns;
                    if (!valid) atomicOr(seg.status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);
                    hit = valid && la != lb && aabb_overlap(geo[la], geo[lb]);
                }
                unsigned bal = __ballot_sync(0xffffffffu, hit);
                int lane = tid & 31, warp = tid >> 5;
                if (lane == 0) warp_tmp[warp] = __popc(bal);
                __syncthreads();
                if (tid == 0) {
                    int run = 0;
                    for (int i = 0; i < kCT / 32; ++i) {
                        int t = warp_tmp[i];
                        warp_tmp[i] = run;
                        run += t;
                    }
                    warp_tmp[kCT / 32] = run;
                }
                __syncthreads();
                if (hit) cand[s_ncand + warp_tmp[warp] + __popc(bal & ((1u << lane) - 1u))] = p;
                __syncthreads();
                if (tid == 0) s_ncand += warp_tmp[kCT / 32];
                pnext += kCT;
                __syncthreads();
            }
            const int ncand = s_ncand;
            // ---- narrow phase in rounds of kCT candidates
            for (int r = 0; r < ncand; r += kCT) {
                int ci = r + tid;
                int n = 0;
                float4* myslots = scratch + (size_t)tid * kSlotF4;
                if (ci < ncand) {
                    int p = cand[ci];
                    int la = m.pair_shapes[2 * (size_t)p], lb = m.pair_shapes[2 * (size_t)p + 1];
                    const Geom& ga = geo[la];
                    const Geom& gb = geo[lb];
                    Writer wr;
                    wr.slots = myslots;
                    wr.n = 0;
                    wr.inv_a = ga.body == -1 ? tf_identity() : tf_inverse(load_tf(body_q + 7 * (size_t)ga.body));
                    wr.inv_b = gb.body == -1 ? tf_identity() : tf_inverse(load_tf(body_q + 7 * (size_t)gb.body));
                    wr.gap = m.shape_gap[ga.sid] + m.shape_gap[gb.sid];
                    wr.shape_a = ga.sid;
                    wr.shape_b = gb.sid;
                    int lba = ga.body < 0 ? -1 : ga.body - b0;
                    int lbb = gb.body < 0 ? -1 : gb.body - b0;
                    wr.tag = ((lba + 1) & 0xFFF) | (((lbb + 1) & 0xFFF) << 12);
                    narrow_pair(wr, ga, gb);
                    n = wr.n;
                }
                int total;
                int off = block_exclusive_scan(n, warp_tmp, total);
                const int base = s_total;
                for (int k = 0; k < n; ++k) {
                    int64_t dst = (int64_t)base + off + k;
                    if (dst < ccap) {
                        dst += cbase;
                        const float4* sl = myslots + 5 * k;
                        rec0[dst] = sl[0];
                        rec1[dst] = sl[1];
                        rec2[dst] = sl[2];
                        rec3[dst] = sl[3];
                        rec4[dst] = sl[4];
                    }
                }
                __syncthreads();
                if (tid == 0) s_total = base + total;
                __syncthreads();
            }
        }
        if (tid == 0) {
            int t = s_total;
            if ((int64_t)t > ccap) {
                atomicOr(seg.status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);
                t = (int)ccap;
            }
            seg.world_count[w] = t;
        }
        __syncthreads();
    }
}

// Exclusive scan of world contact counts (single CTA) -> world_offset[W+1],
// count[0] = total (may exceed the public capacity, as in the reference).
__global__ void __launch_bounds__(1024) world_scan_kernel(int W, const int32_t* __restrict__ world_count,
                                                          int64_t* world_offset, int32_t* count_out, int cap,
                                                          uint32_t* status) {
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
            int64_t y = __shfl_up_sync(0xffffffffu, x, o);
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
        if (i < W) world_offset[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        world_offset[W] = carry;
        count_out[0] = carry > 0x7fffffff ? 0x7fffffff : (int32_t)carry;
        if (carry > cap) atomicOr(status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);
    }
}

// Dense public Contacts arrays ordered by (world, key).
__global__ void __launch_bounds__(256) publish_kernel(NbModelDesc m, NbContactSeg seg, NbContactsPublic pub) {
    const int w = blockIdx.x;
    if (w >= m.world_count) return;
    const int n = seg.world_count[w];
    const int64_t src0 = m.contact_cap_start[w];
    const int64_t dst0 = pub.world_offset[w];
    const float4* rec0 = reinterpret_cast<const float4*>(seg.rec0);
    const float4* rec1 = reinterpret_cast<const float4*>(seg.rec1);
    const float4* rec2 = reinterpret_cast<const float4*>(seg.rec2);
    const float4* rec3 = reinterpret_cast<const float4*>(seg.rec3);
    const float4* rec4 = reinterpret_cast<const float4*>(seg.rec4);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        int64_t d = dst0 + k;
        if (d >= pub.capacity) break;
        int64_t s = src0 + k;
        float4 a = rec0[s], b = rec1[s], c = rec2[s], e = rec3[s], f = rec4[s];
        int s0 = __float_as_int(c.w), s1 = __float_as_int(e.w);
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
            int sub = (__float_as_int(f.w) >> 24) & 0xFF;
            pub.sort_key[d] = ((int64_t)(s0 & 0xFFFFF) << 43) | ((int64_t)(s1 & 0xFFFFF) << 23) | (int64_t)sub;
        }
    }
}

// Custom contacts written into the public arrays -> per-world segments.
// Contacts of a world land in an arbitrary order; the solver's fixed-point
// accumulation makes its result independent of that order.
__global__ void ingest_kernel(NbModelDesc m, NbContactsPublic pub, NbContactSeg seg) {
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
    // world of a body: binary search in world_body_start
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
    int slot = atomicAdd(&seg.world_count[w], 1);
    const int64_t cap = m.contact_cap_start[w + 1] - m.contact_cap_start[w];
    if (slot >= cap) {
        atomicOr(seg.status, (unsigned)NB_STATUS_CONTACT_OVERFLOW);
        return;
    }
    int64_t d = m.contact_cap_start[w] + slot;
    int la = b0 < 0 ? -1 : b0 - wb, lb = b1 < 0 ? -1 : b1 - wb;
    int tag = ((la + 1) & 0xFFF) | (((lb + 1) & 0xFFF) << 12);
    reinterpret_cast<float4*>(seg.rec0)[d] = make_float4(pub.point0[3 * c], pub.point0[3 * c + 1], pub.point0[3 * c + 2], pub.margin0[c]);
    reinterpret_cast<float4*>(seg.rec1)[d] = make_float4(pub.point1[3 * c], pub.point1[3 * c + 1], pub.point1[3 * c + 2], pub.margin1[c]);
    reinterpret_cast<float4*>(seg.rec2)[d] = make_float4(pub.normal[3 * c], pub.normal[3 * c + 1], pub.normal[3 * c + 2], __int_as_float(s0));
    reinterpret_cast<float4*>(seg.rec3)[d] = make_float4(pub.offset0[3 * c], pub.offset0[3 * c + 1], pub.offset0[3 * c + 2], __int_as_float(s1));
    reinterpret_cast<float4*>(seg.rec4)[d] = make_float4(pub.offset1[3 * c], pub.offset1[3 * c + 1], pub.offset1[3 * c + 2], __int_as_float(tag));
}

}  // namespace

size_t nb_collide_smem_bytes(const NbModelDesc* m) {
    return (size_t)m->max_world_shapes * sizeof(Geom) + (size_t)kMaxCand * sizeof(int);
}

cudaError_t nb_launch_collide(const NbModelDesc* m, const float* body_q, const NbContactSeg* seg, int grid,
                              cudaStream_t stream) {
    size_t smem = nb_collide_smem_bytes(m);
    // raise the dynamic shared-memory limit only when needed, so calls made
    // during CUDA-graph capture (after a first eager call) touch no attributes
    static size_t configured = 0;
    cudaError_t e;
    if (smem > configured) {
        e = cudaFuncSetAttribute(collide_worlds_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    e = cudaMemsetAsync(seg->work_counter, 0, sizeof(int32_t), stream);
    if (e != cudaSuccess) return e;
    collide_worlds_kernel<<<grid, kCT, smem, stream>>>(*m, body_q, *seg);
    return cudaGetLastError();
}

cudaError_t nb_launch_publish(const NbModelDesc* m, const NbContactSeg* seg, const NbContactsPublic* pub,
                              cudaStream_t stream) {
    world_scan_kernel<<<1, 1024, 0, stream>>>(m->world_count, seg->world_count, pub->world_offset, pub->count,
                                              pub->capacity, seg->status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    publish_kernel<<<m->world_count, 256, 0, stream>>>(*m, *seg, *pub);
    return cudaGetLastError();
}

cudaError_t nb_launch_ingest(const NbModelDesc* m, const NbContactsPublic* pub, const NbContactSeg* seg,
                             cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(seg->world_count, 0, sizeof(int32_t) * (size_t)m->world_count, stream);
    if (e != cudaSuccess) return e;
    if (pub->capacity <= 0) return cudaSuccess;
    ingest_kernel<<<(pub->capacity + 255) / 256, 256, 0, stream>>>(*m, *pub, *seg);
    return cudaGetLastError();
}
