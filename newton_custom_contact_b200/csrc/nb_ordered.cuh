// Ordered accumulation of per-body deltas within one world, for a group of G
// threads.
//
// The reference sums the deltas its constraint kernels produce into per-body
// accumulators with float atomics (solve_body_contact_positions,
// solve_body_joints, apply_rigid_restitution in
// newton/_src/solvers/xpbd/kernels.py): run sequentially, every body's delta is
// the float sum of its contributions in item order (contact index, joint
// index), starting from zero.  ordered_pass reproduces exactly that sum, in
// parallel and deterministically:
//
//   1. test: the group tests items in rounds of G (thread t takes item
//      base + t) and appends the active ones to a shared batch in item order
//      (warp ballots; across warps a prefix of the per-warp counts);
//   2. solve: when the batch could overflow, every thread solves batch entries
//      a = t, t + G, ... into the batch's delta rows (A side, B side);
//   3. gather: body i belongs to thread i % G; every thread adds, in batch
//      order, the rows of the entries that touch its bodies.  One-warp groups
//      first mark, per owner thread, which entries touch it (a bit per entry,
//      shared-memory atomicOr, one word per 32 entries), so each thread visits
//      only its own entries; larger groups walk the whole batch.
//
// No atomics touch the accumulators, and because batches are flushed in item
// order and walked in order, each body sees its contributions in item order.
#pragma once

#include "nb_math.cuh"

namespace nb {

// per owner thread of a one-warp group: bit (a & 31) of word [a >> 5] is set
// when batch entry a touches one of the thread's bodies on side A (a) / B (b)
template <int kWords, bool kOn>
struct OwnerMasks {
    unsigned a[kWords][32];
    unsigned b[kWords][32];
};
template <int kWords>
struct OwnerMasks<kWords, false> {};

// one entry of a batch: item index and the two bodies (world-local, -1 = static)
template <int kCap>
struct OrderedBatch {
    static constexpr int kWords = (kCap + 31) / 32;
    static constexpr bool kMasks = kCap <= 64;  // the batches of one-warp groups
    float d[kCap][12];   // A side (lin 3, ang 3), B side (lin 3, ang 3)
    int item[kCap];
    int ends[kCap];      // (la + 1) | (lb + 1) << 16
    int wcnt[8];         // per-warp counts of one test round (G > 32)
    OwnerMasks<kWords, kMasks> own;
};

__device__ __forceinline__ int ends_pack(int la, int lb) { return (la + 1) | ((lb + 1) << 16); }
__device__ __forceinline__ int ends_a(int e) { return (e & 0xFFFF) - 1; }
__device__ __forceinline__ int ends_b(int e) { return ((e >> 16) & 0xFFFF) - 1; }

// barrier of a group of G threads (group g of the CTA): a warp, a named
// barrier over the group's warps, or the whole CTA
template <int G, int kCTA>
__device__ __forceinline__ void ordered_sync(int g) {
    if constexpr (G == 32) {
        __syncwarp();
    } else if constexpr (G == kCTA) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(G) : "memory");
    }
}

// Appends the active items of one test round to the batch in item order;
// n (uniform over the group) is the batch's entry count before and after.
template <int G, int kCTA, int kCap>
__device__ __forceinline__ void ordered_append(OrderedBatch<kCap>& B, bool active, int k, int ends, int g, int t,
                                               int& n) {
    const unsigned lane = (unsigned)t & 31u;
    const unsigned ball = __ballot_sync(0xffffffffu, active);
    const unsigned below = ball & ((1u << lane) - 1u);
    if constexpr (G == 32) {
        if (active) {
            const int pos = n + __popc(below);
            B.item[pos] = k;
            B.ends[pos] = ends;
        }
        n += __popc(ball);
    } else {
        const int warp = t >> 5;
        if (lane == 0) B.wcnt[warp] = __popc(ball);
        ordered_sync<G, kCTA>(g);
        int off = n, total = n;
#pragma unroll
        for (int w = 0; w < G / 32; ++w) {
            const int c = B.wcnt[w];
            if (w < warp) off += c;
            total += c;
        }
        if (active) {
            const int pos = off + __popc(below);
            B.item[pos] = k;
            B.ends[pos] = ends;
        }
        n = total;
        ordered_sync<G, kCTA>(g);  // every thread read wcnt before the next round rewrites it
    }
}

// Solves the batch's n entries and adds their rows to the owners' accumulators
// in entry (= item) order.  solve(item, d[12]) fills a row; add(i, side, d6)
// adds a 6-float row to body i (called by body i's owner thread only).
template <int G, int kCTA, int kCap, class Solve, class Add>
__device__ __forceinline__ void ordered_flush(OrderedBatch<kCap>& B, int n, int g, int t, Solve& solve, Add& add) {
    if constexpr (G == 32 && OrderedBatch<kCap>::kMasks) {
        constexpr int kW = OrderedBatch<kCap>::kWords;
#pragma unroll
        for (int w = 0; w < kW; ++w) {
            B.own.a[w][t] = 0u;
            B.own.b[w][t] = 0u;
        }
        __syncwarp();  // the entries and the cleared masks are visible
        for (int a = t; a < n; a += 32) {
            solve(B.item[a], B.d[a]);
            const int e = B.ends[a];
            const int la = ends_a(e), lb = ends_b(e);
            const unsigned bit = 1u << (a & 31);
            if (la >= 0) atomicOr(&B.own.a[a >> 5][la & 31], bit);
            if (lb >= 0) atomicOr(&B.own.b[a >> 5][lb & 31], bit);
        }
        __syncwarp();  // the rows and the masks are visible
#pragma unroll
        for (int w = 0; w < kW; ++w) {
            const unsigned ma = B.own.a[w][t], mb = B.own.b[w][t];
            unsigned rest = ma | mb;
            while (rest) {
                const int j = __ffs(rest) - 1;
                rest &= rest - 1u;
                const int a = (w << 5) + j;
                const int e = B.ends[a];
                if ((ma >> j) & 1u) add(ends_a(e), 0, &B.d[a][0]);
                if ((mb >> j) & 1u) add(ends_b(e), 1, &B.d[a][6]);
            }
        }
        __syncwarp();  // the batch may be refilled
    } else {
        ordered_sync<G, kCTA>(g);  // the entries are visible
        for (int a = t; a < n; a += G) solve(B.item[a], B.d[a]);
        ordered_sync<G, kCTA>(g);  // the rows are visible
        for (int a = 0; a < n; ++a) {
            const int e = B.ends[a];
            const int la = ends_a(e), lb = ends_b(e);
            if (la >= 0 && la % G == t) add(la, 0, &B.d[a][0]);
            if (lb >= 0 && lb % G == t) add(lb, 1, &B.d[a][6]);
        }
        ordered_sync<G, kCTA>(g);  // the batch may be refilled
    }
}

// The pass over items 0 .. n_items - 1.  test(k, ends) -> bool decides whether
// item k contributes (and to which bodies); every thread of the group must
// call this with the same n_items.
template <int G, int kCTA, int kCap, class Test, class Solve, class Add>
__device__ __forceinline__ void ordered_pass(OrderedBatch<kCap>& B, int n_items, int g, int t, Test& test,
                                             Solve& solve, Add& add) {
    static_assert(kCap >= G, "a batch must hold one full test round");
    int n = 0;
    for (int base = 0; base < n_items; base += G) {
        if (n + G > kCap) {
            ordered_flush<G, kCTA>(B, n, g, t, solve, add);
            n = 0;
        }
        const int k = base + t;
        int ends = 0;
        const bool active = k < n_items && test(k, ends);
        ordered_append<G, kCTA>(B, active, k, ends, g, t, n);
    }
    if (n > 0) ordered_flush<G, kCTA>(B, n, g, t, solve, add);
}

}  // namespace nb
