// Learned warm start of the XPBD contact solve: per-contact features, the
// BF16 MLP 24 -> 128 -> 128 -> 3 (SiLU) that predicts each contact's total
// impulse in its contact frame, and the MLP's training kernels.  The network
// works relative to a physical prior: the previous substep's correction of
// the same contact (through contact matching), else the velocity that
// removes the depth expected after the integration.  Inputs are ratios to
// the prior and inverse-mass shares; outputs y give the contact's velocity
// correction c = prior * y, and the impulse is c / w with w the contact's
// generalised inverse mass (normal / tangents), so the map the network
// learns does not depend on the bodies' scale.
//
// Inference runs on the 5th-generation tensor cores: a CTA of 128 threads
// takes 128 contacts per tile, stages the normalised features and the
// hidden activations as BF16 in shared memory in the K-major core-matrix
// layout (8 rows x 16 bytes per core matrix, no swizzle), issues one
// tcgen05.mma chain per layer from a single thread with FP32 accumulators in
// tensor memory, waits on an mbarrier signalled by tcgen05.commit, and reads
// the accumulators back with tcgen05.ld for the bias + SiLU epilogue.  Every
// wait is bounded; a timeout sets NB_STATUS_QUEUE_TIMEOUT and the CTA frees
// its tensor memory and returns.
//
// Training runs its GEMMs on the tensor cores too (tc_gemm: BF16 operands,
// FP32 accumulation, gradients split into two BF16 parts), with
// straight-through BF16 rounding of weights and activations, so the trained
// network is the one inference evaluates.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "nb_kernels.cuh"
#include "nb_math.cuh"

namespace {

constexpr int kIn = NB_WS_INPUTS;     // 24 network inputs
constexpr int kFeat = NB_WS_FEATURES; // + generalised inverse masses (normal, tangents), prior
constexpr int kMuCol = 17;            // friction coefficient column of a feature row
constexpr int kFeatBlock = 256;       // threads (rows) per block of the features kernel
static_assert((kFeatBlock * kFeat * 4) % 16 == 0, "feature blocks must start on 16-byte boundaries");
constexpr int kInPad = 32;            // K of layer 1 (two K=16 MMA steps)
constexpr int kHid = NB_WS_HIDDEN;    // 128
constexpr int kOut = NB_WS_OUTPUTS;   // 3
constexpr int kOutPad = 16;           // N of layer 3 (smallest legal N for M = 128)
constexpr int kTile = 128;            // contacts per tile = MMA M
static_assert((kTile * kFeat * 4) % 16 == 0, "inference tiles must start on 16-byte boundaries");

// ---------------------------------------------------------------- features

__device__ __forceinline__ void contact_basis(V3 n, V3& t1, V3& t2) {
    const V3 a = fabsf(n.x) < 0.9f ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 1.0f, 0.0f};
    t1 = normalize(cross(n, a));
    t2 = cross(n, t1);
}

// Contact kernels below loop over the live contacts (count read on the device)
// with a grid sized from the SM count, not from the buffer capacity.
__device__ __forceinline__ int live_count(const NbContactsPublic& pub) {
    return pub.count[0] < pub.capacity ? pub.count[0] : pub.capacity;
}

__global__ void ws_count_kernel(NbModelDesc m, NbContactsPublic pub, int32_t* body_count) {
    const int n = live_count(pub);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s0 = pub.shape0[i], s1 = pub.shape1[i];
        const int b0 = s0 >= 0 ? m.shape_body[s0] : -1, b1 = s1 >= 0 ? m.shape_body[s1] : -1;
        if (b0 >= 0) atomicAdd(body_count + b0, 1);
        if (b1 >= 0) atomicAdd(body_count + b1, 1);
    }
}

struct BodyView {
    TF x;
    V3 v, w, com_w;
    float inv_m;
    M33 iI;  // effective (body frame) inverse inertia
    int count;
};

__device__ __forceinline__ BodyView body_view(const NbModelDesc& m, const float* q, const float* qd,
                                              const int32_t* body_count, int b, V3 anchor) {
    BodyView v;
    if (b < 0) {
        v.x = tf_identity();
        v.v = v.w = V3{0.0f, 0.0f, 0.0f};
        v.com_w = anchor;
        v.inv_m = 0.0f;
        v.iI = zero_m33();
        v.count = 0;
        return v;
    }
    const bool kin = (m.body_flags[b] & NB_BODY_KINEMATIC) != 0;
    v.x = load_tf(q + 7 * (size_t)b);
    v.v = load_v3(qd + 6 * (size_t)b);
    v.w = load_v3(qd + 6 * (size_t)b + 3);
    v.com_w = tf_point(v.x, load_v3(m.body_com + 3 * (size_t)b));
    v.inv_m = kin ? 0.0f : m.body_inv_mass[b];
    v.iI = kin ? zero_m33() : load_m33(m.body_inv_inertia + 9 * (size_t)b);
    v.count = body_count[b];
    return v;
}

// effective angular inverse mass of a unit impulse along u at lever r
__device__ __forceinline__ float clip10(float x) { return fminf(10.0f, fmaxf(-10.0f, x)); }

__device__ __forceinline__ float ang_inv(const BodyView& b, V3 r, V3 u) {
    const V3 k = qrot_inv(b.x.q, cross(r, u));
    return dot(k, mv(b.iI, k));
}

__device__ void features_row(const NbModelDesc& m, const float* __restrict__ q, const float* __restrict__ qd,
                             const NbContactsPublic& pub, const float* __restrict__ prev_lambda,
                             const int32_t* __restrict__ match_index, const int32_t* __restrict__ body_count,
                             float dt, float* __restrict__ row_out, int i) {
    const int s0 = pub.shape0[i], s1 = pub.shape1[i];
    const int ba = s0 >= 0 ? m.shape_body[s0] : -1, bb = s1 >= 0 ? m.shape_body[s1] : -1;
    const V3 p0 = load_v3(pub.point0 + 3 * (size_t)i), p1 = load_v3(pub.point1 + 3 * (size_t)i);
    const TF xa = ba >= 0 ? load_tf(q + 7 * (size_t)ba) : tf_identity();
    const TF xb = bb >= 0 ? load_tf(q + 7 * (size_t)bb) : tf_identity();
    const V3 pa = tf_point(xa, p0), pb = tf_point(xb, p1);
    const BodyView A = body_view(m, q, qd, body_count, ba, pa);
    const BodyView B = body_view(m, q, qd, body_count, bb, pb);
    const V3 nrm = load_v3(pub.normal + 3 * (size_t)i);
    V3 t1, t2;
    contact_basis(nrm, t1, t2);
    const float thick = pub.margin0[i] + pub.margin1[i];
    const V3 ra = sub(pa, A.com_w), rb = sub(pb, B.com_w);
    const V3 vrel = sub(add(B.v, cross(B.w, rb)), add(A.v, cross(A.w, ra)));
    const V3 dcom = sub(B.com_w, A.com_w);
    float mu = 0.0f;
    int nz = 0;
    if (s0 >= 0) { mu += m.shape_mu[s0]; nz += 1; }
    if (s1 >= 0) { mu += m.shape_mu[s1]; nz += 1; }
    if (nz) mu /= (float)nz;
    const int bw = ba >= 0 ? ba : bb;
    int wi = bw >= 0 ? m.body_world[bw] : 0;
    wi = wi > 0 ? wi : 0;
    const V3 g = load_v3(m.gravity + 3 * (size_t)wi);
    // generalised inverse masses of a unit impulse along the normal / the tangents
    const float lin = A.inv_m + B.inv_m;
    const float wn = lin + ang_inv(A, ra, nrm) + ang_inv(B, rb, nrm);
    const float wt = lin + 0.5f * (ang_inv(A, ra, t1) + ang_inv(A, ra, t2) + ang_inv(B, rb, t1) + ang_inv(B, rb, t2));
    // features are inputs to a BF16 network: fast reciprocal / log intrinsics suffice
    const float iwn = wn > 0.0f ? __frcp_rn(wn) : 0.0f;
    const float idt = __frcp_rn(dt);
    // the previous substep's solved impulse of the same contact, as a velocity correction c = lambda * w
    float pc[3] = {0.0f, 0.0f, 0.0f};
    if (prev_lambda && match_index) {
        const int k = match_index[i];
        if (k >= 0) {
            pc[0] = prev_lambda[3 * (size_t)k] * wn;
            pc[1] = prev_lambda[3 * (size_t)k + 1] * wt;
            pc[2] = prev_lambda[3 * (size_t)k + 2] * wt;
        }
    }
    const float d = dot(nrm, sub(pb, pa)) - thick;
    const float vn = dot(vrel, nrm);
    // gravity changes a dynamic body's velocity by g dt in one substep; a static side does not move
    const float gv = dot(g, nrm) * dt;
    const float gsep = gv * ((B.inv_m > 0.0f ? 1.0f : 0.0f) - (A.inv_m > 0.0f ? 1.0f : 0.0f));
    // prior: the previous correction of a matched contact, else the velocity that removes the
    // depth expected after the integration in one substep
    const bool matched = pc[0] > 0.0f;
    const float est = fmaxf(0.0f, -(d + (vn + gsep) * dt)) * idt;
    const float prior = matched ? pc[0] : est;
    float f[kFeat];
    if (prior > 0.0f && wn > 0.0f) {
        const float ip = __frcp_rn(prior);
        const float dn = sqrtf(dot(dcom, dcom));
        f[0] = matched ? 1.0f : 0.0f;
        f[1] = clip10(est * ip);
        f[2] = clip10(pc[0] * ip);
        f[3] = clip10(pc[1] * ip);
        f[4] = clip10(pc[2] * ip);
        f[5] = clip10(dot(vrel, t1) * ip);
        f[6] = clip10(dot(vrel, t2) * ip);
        f[7] = clip10(vn * ip);
        f[8] = clip10(d * idt * ip);
        f[9] = clip10(gv * ip);
        f[10] = nrm.x;
        f[11] = nrm.y;
        f[12] = nrm.z;
        f[13] = A.inv_m * iwn;
        f[14] = B.inv_m * iwn;
        f[15] = (wn - lin) * iwn;
        f[16] = wt * iwn;
        f[17] = mu;
        f[18] = (float)A.count;
        f[19] = (float)B.count;
        f[20] = __log2f(prior);
        f[21] = clip10(thick * idt * ip);
        f[22] = dn > 0.0f ? __fdividef(dot(dcom, nrm), dn) : 0.0f;
        f[23] = (B.inv_m > 0.0f ? 1.0f : 0.0f) - (A.inv_m > 0.0f ? 1.0f : 0.0f);
        f[24] = wn;
        f[25] = wt;
        f[26] = prior;
    } else {
        // nothing to predict: lambda = 0 (mu kept for the friction bound)
        for (int j = 0; j < kFeat; ++j) f[j] = 0.0f;
        f[17] = mu;
        f[24] = wn;
        f[25] = wt;
    }
    for (int j = 0; j < kFeat; ++j) row_out[j] = f[j];
}

__global__ void ws_features_kernel(NbModelDesc m, const float* __restrict__ q, const float* __restrict__ qd,
                                   NbContactsPublic pub, const float* __restrict__ prev_lambda,
                                   const int32_t* __restrict__ match_index, const int32_t* __restrict__ body_count,
                                   float dt, float* __restrict__ feat) {
    // rows are built in shared memory and written out as one contiguous block
    // (coalesced 16-byte stores) instead of 27 strided stores per thread
    __shared__ __align__(16) float sf[kFeatBlock * kFeat];
    const int n = live_count(pub);
    const int t = threadIdx.x;
    for (int base = blockIdx.x * kFeatBlock; base < n; base += gridDim.x * kFeatBlock) {
        if (base + t < n) features_row(m, q, qd, pub, prev_lambda, match_index, body_count, dt, sf + t * kFeat, base + t);
        __syncthreads();
        const int rows = n - base < kFeatBlock ? n - base : kFeatBlock;
        float* dst = feat + (size_t)base * kFeat;
        if (rows == kFeatBlock) {
            // base is a multiple of kFeatBlock, so dst is 16-byte aligned (kFeatBlock * kFeat * 4 % 16 == 0)
            const float4* s4 = reinterpret_cast<const float4*>(sf);
            float4* d4 = reinterpret_cast<float4*>(dst);
            for (int e = t; e < kFeatBlock * kFeat / 4; e += kFeatBlock) d4[e] = s4[e];
        } else {
            for (int e = t; e < rows * kFeat; e += kFeatBlock) dst[e] = sf[e];
        }
        __syncthreads();
    }
}

// contact-frame components (n, t1, t2) of accumulated A-side impulses:
// lambda_n = -L.n (pushes the bodies apart), lambda_t = L.t; with `clear` the
// impulse rows are zeroed after reading (the step only ever writes live rows,
// so the whole buffer is zero again for the next step)
__global__ void ws_targets_kernel(NbContactsPublic pub, float* __restrict__ impulse, float* __restrict__ lam,
                                  int clear) {
    const int n = live_count(pub);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V3 nrm = load_v3(pub.normal + 3 * (size_t)i);
        V3 t1, t2;
        contact_basis(nrm, t1, t2);
        float* row = impulse + 6 * (size_t)i;
        const V3 L = load_v3(row);
        lam[3 * (size_t)i] = -dot(L, nrm);
        lam[3 * (size_t)i + 1] = dot(L, t1);
        lam[3 * (size_t)i + 2] = dot(L, t2);
        if (clear)
            for (int k = 0; k < 6; ++k) row[k] = 0.0f;
    }
}

// ---------------------------------------------------------------- tcgen05 inference

constexpr uint32_t kSmW1 = 0;                                    // [128 x 32]  bf16
constexpr uint32_t kSmW2 = kSmW1 + kHid * kInPad * 2;            // [128 x 128]
constexpr uint32_t kSmW3 = kSmW2 + kHid * kHid * 2;              // [16 x 128]
constexpr uint32_t kSmA1 = kSmW3 + kOutPad * kHid * 2;           // [128 x 32]
constexpr uint32_t kSmA2 = kSmA1 + kTile * kInPad * 2;           // [128 x 128] hidden (both layers)
constexpr uint32_t kSmF = kSmA2 + kTile * kHid * 2;              // fp32 params
constexpr uint32_t kSmB1 = kSmF;
constexpr uint32_t kSmB2 = kSmB1 + kHid * 4;
constexpr uint32_t kSmB3 = kSmB2 + kHid * 4;
constexpr uint32_t kSmMean = kSmB3 + kOutPad * 4;
constexpr uint32_t kSmIstd = kSmMean + kInPad * 4;
constexpr uint32_t kSmOsc = kSmIstd + kInPad * 4;
constexpr uint32_t kSmFeat = (kSmOsc + 16 + 15) & ~15u;          // [128 x 27] fp32 feature rows of the tile
constexpr uint32_t kSmBar = kSmFeat + kTile * kFeat * 4;          // mbarrier (8 B)
constexpr uint32_t kSmTmem = kSmBar + 8;                         // tensor-memory base address
constexpr uint32_t kSmBytes = kSmTmem + 8;
constexpr uint32_t kTmemCols = 128;                              // one accumulator, reused by the layers
constexpr long kWaitLimit = 1L << 26;                            // mbarrier polls before giving up

// byte offset of element (row r, column k) of a K-major [rows x K] bf16 tile in
// the no-swizzle core-matrix layout: 8 x 8 core matrices of 128 B, K-chunks
// 128 B apart (leading byte offset), 8-row groups K/8 * 128 B apart (stride)
__device__ __forceinline__ uint32_t cm_offset(int r, int k, int K) {
    return (uint32_t)(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    // start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46), descriptor version 1 at
    // bit 46, base offset 0, no swizzle (layout type 0 at [61,64))
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at [17,23), M >> 4 at [24,29)
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// 64 consecutive accumulator columns of this thread's lane, load and wait in one
// statement so no use of the registers can be scheduled before the wait
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int j = 0; j < 64; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float silu(float x) { return x / (1.0f + expf(-x)); }

// inference epilogue: silu(u) = u sigmoid(u) = h + h tanh(h) with h = u / 2, one
// hardware tanh (tanh.approx.f32, relative error about 2^-11) per activation --
// far below the BF16 rounding the activations get next
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float silu_fast(float u) {
    const float h = 0.5f * u;
    return __fmaf_rn(h, tanh_approx(h), h);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// copy a row-major [rows x K] bf16 matrix from global into the core-matrix layout
// (8 independent 16-byte loads in flight per thread before their stores)
__device__ void stage_matrix(unsigned char* sm, const uint16_t* __restrict__ g, int rows, int K) {
    const int chunks = rows * (K / 8);
    for (int c0 = threadIdx.x; c0 < chunks; c0 += 8 * blockDim.x) {
        uint4 v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int c = c0 + u * blockDim.x;
            if (c < chunks) {
                const int r = c / (K / 8), k = (c % (K / 8)) * 8;
                v[u] = __ldg(reinterpret_cast<const uint4*>(g + (size_t)r * K + k));
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int c = c0 + u * blockDim.x;
            if (c < chunks) {
                const int r = c / (K / 8), k = (c % (K / 8)) * 8;
                *reinterpret_cast<uint4*>(sm + cm_offset(r, k, K)) = v[u];
            }
        }
    }
}

// 256 threads per CTA: thread t owns tile row t % 128 (its tensor-memory lane)
// and half t / 128 of the 128 hidden columns in the epilogues
constexpr int kInferThreads = 256;

__global__ void __launch_bounds__(kInferThreads, 2)
ws_infer_kernel(NbWsNet net, const float* __restrict__ feat, const int32_t* __restrict__ count, int cap,
                float* __restrict__ out, uint32_t* status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int t = threadIdx.x, warp = t >> 5;
    const int r = t & (kTile - 1), half = t >> 7;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const uint32_t bar = sbase + kSmBar;
    float* fb1 = reinterpret_cast<float*>(sm + kSmB1);
    float* fb2 = reinterpret_cast<float*>(sm + kSmB2);
    float* fb3 = reinterpret_cast<float*>(sm + kSmB3);
    float* fmean = reinterpret_cast<float*>(sm + kSmMean);
    float* fistd = reinterpret_cast<float*>(sm + kSmIstd);
    float* fosc = reinterpret_cast<float*>(sm + kSmOsc);
    // ---- weights and parameters, once per CTA
    stage_matrix(sm + kSmW1, net.w1, kHid, kInPad);
    stage_matrix(sm + kSmW2, net.w2, kHid, kHid);
    stage_matrix(sm + kSmW3, net.w3, kOutPad, kHid);
    if (t < kHid) {
        fb1[t] = net.b1[t];
        fb2[t] = net.b2[t];
    }
    if (t < kOutPad) fb3[t] = net.b3[t];
    if (t < kInPad) {
        fmean[t] = t < kIn ? net.in_mean[t] : 0.0f;
        fistd[t] = t < kIn ? net.in_inv_std[t] : 0.0f;
    }
    if (t < 4) fosc[t] = t < kOut ? net.out_scale[t] : 0.0f;
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + kSmTmem),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kSmTmem);
    const int n = count[0] < cap ? count[0] : cap;
    // a warp reaches the 32 lanes 32 * (warp % 4) .. + 31: rows r of both halves
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    uint32_t phase = 0;
    bool ok = true;
    const uint32_t id_h = idesc_bf16(kTile, kHid), id_o = idesc_bf16(kTile, kOutPad);
    for (int base = blockIdx.x * kTile; base < n && ok; base += gridDim.x * kTile) {
        const int row = base + r;
        // ---- the tile's feature rows: one contiguous block, read with coalesced 16-byte loads
        float* sfeat = reinterpret_cast<float*>(sm + kSmFeat);
        {
            const int rows = n - base < kTile ? n - base : kTile;
            const float* src = feat + (size_t)base * kFeat;
            if (rows == kTile) {
                // base is a multiple of kTile: kTile * kFeat * 4 bytes keep src 16-byte aligned
                const float4* s4 = reinterpret_cast<const float4*>(src);
                float4* d4 = reinterpret_cast<float4*>(sfeat);
                for (int e = t; e < kTile * kFeat / 4; e += kInferThreads) d4[e] = s4[e];
            } else {
                for (int e = t; e < rows * kFeat; e += kInferThreads) sfeat[e] = src[e];
            }
        }
        __syncthreads();
        const float* fr = sfeat + r * kFeat;
        // ---- A1: normalised features of row r, columns 16 * half .. + 15 (zeros past n / past 24)
        {
            float x[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int col = 16 * half + j;
                const float raw = (row < n && col < kIn) ? fr[col] : 0.0f;
                x[j] = (raw - fmean[col]) * fistd[col];
            }
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                uint4 v;
                v.x = pack_bf16(x[8 * c], x[8 * c + 1]);
                v.y = pack_bf16(x[8 * c + 2], x[8 * c + 3]);
                v.z = pack_bf16(x[8 * c + 4], x[8 * c + 5]);
                v.w = pack_bf16(x[8 * c + 6], x[8 * c + 7]);
                *reinterpret_cast<uint4*>(sm + kSmA1 + cm_offset(r, 16 * half + 8 * c, kInPad)) = v;
            }
        }
        // ---- three layers: MMA chain from one thread, epilogue by every thread on its row and half
        for (int layer = 0; layer < 3 && ok; ++layer) {
            fence_async_smem();
            tc_before_sync();
            __syncthreads();
            if (t == 0) {
                tc_after_sync();
                const int K = layer == 0 ? kInPad : kHid;
                const uint32_t a_off = layer == 0 ? kSmA1 : kSmA2;
                const uint32_t b_off = layer == 0 ? kSmW1 : (layer == 1 ? kSmW2 : kSmW3);
                const uint32_t idesc = layer == 2 ? id_o : id_h;
                for (int s = 0; s < K / 16; ++s) {
                    const uint64_t da = smem_desc(sbase + a_off + s * 256, 128, (K / 8) * 128);
                    const uint64_t db = smem_desc(sbase + b_off + s * 256, 128, (K / 8) * 128);
                    umma_bf16(tmem, da, db, idesc, s > 0 ? 1u : 0u);
                }
                umma_commit(bar);
            }
            ok = __syncthreads_and(mbar_wait(bar, phase)) != 0;
            phase ^= 1u;
            tc_after_sync();
            if (!ok) break;
            if (layer < 2) {
                const float* bias = layer == 0 ? fb1 : fb2;
                const int c0 = 64 * half;
                float v[64];
                tmem_ld64(tmem + lane_base + (uint32_t)c0, v);
#pragma unroll
                for (int j = 0; j < 64; ++j) v[j] = silu_fast(v[j] + bias[c0 + j]);
#pragma unroll
                for (int h = 0; h < 8; ++h) {
                    uint4 p;
                    p.x = pack_bf16(v[8 * h], v[8 * h + 1]);
                    p.y = pack_bf16(v[8 * h + 2], v[8 * h + 3]);
                    p.z = pack_bf16(v[8 * h + 4], v[8 * h + 5]);
                    p.w = pack_bf16(v[8 * h + 6], v[8 * h + 7]);
                    *reinterpret_cast<uint4*>(sm + kSmA2 + cm_offset(r, c0 + 8 * h, kHid)) = p;
                }
            } else if (half == 0) {
                float v[16];
                tmem_ld16(tmem + lane_base, v);
                if (row < n) {
                    // c = prior * y; lambda = c / w with lambda_n >= 0 and the tangential part inside
                    // the friction cone |lambda_t| <= mu lambda_n; zero where there is no prior
                    const float wn = fr[kIn], wt = fr[kIn + 1], prior = fr[kIn + 2], mu = fr[kMuCol];
                    float ln = 0.0f, l1 = 0.0f, l2 = 0.0f;
                    if (prior > 0.0f && wn > 0.0f && wt > 0.0f) {
                        ln = fmaxf(0.0f, (v[0] + fb3[0]) * fosc[0]) * prior / wn;
                        l1 = (v[1] + fb3[1]) * fosc[1] * prior / wt;
                        l2 = (v[2] + fb3[2]) * fosc[2] * prior / wt;
                        const float lt = sqrtf(l1 * l1 + l2 * l2), cap = mu * ln;
                        if (lt > cap) {
                            const float s = lt > 0.0f ? cap / lt : 0.0f;
                            l1 *= s;
                            l2 *= s;
                        }
                    }
                    out[(size_t)row * kOut] = ln;
                    out[(size_t)row * kOut + 1] = l1;
                    out[(size_t)row * kOut + 2] = l2;
                }
            }
        }
        tc_before_sync();
        __syncthreads();  // tile done: A1 / A2 / features / tensor memory free for the next tile
    }
    if (!ok && t == 0) atomicOr(status, (unsigned)NB_STATUS_QUEUE_TIMEOUT);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// ---------------------------------------------------------------- training

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Training GEMMs on the tensor cores: C(m, n) = sum_k A(m, k) B(n, k) for FP32
// operands in global memory with arbitrary strides (so transposed operands
// need no copy), BF16 tcgen05.mma with an FP32 accumulator in tensor memory.
// A CTA of 128 threads owns a 128 x nt tile of C (nt = 16 / 32 / 64 / 128)
// and a slice of K (split-K CTAs add their partial tiles atomically into a
// zeroed C).  Per 64-wide K chunk every thread converts 8-element runs of A
// and B to BF16 into the K-major core-matrix layout; operands that are not
// exactly BF16 (the gradients) are split into hi = bf16(x) and
// lo = bf16(x - hi) and multiplied as hi.hi + hi.lo + lo.hi, which keeps the
// products at about FP32 accuracy.
struct TcGemm {
    const float* A;
    long sam, sak;
    const float* B;
    long sbn, sbk;
    float* C;
    long scm, scn;
    int M, N, K;
    int nt;        // tile width in n: 16, 32, 64 or 128
    int k_per;     // K range per split (multiple of 64)
    int split;     // > 1: atomic accumulation into C
    int exact;     // operands are BF16 values: hi only
};

constexpr int kGemmKc = 64;
constexpr uint32_t kGemmTileA = 128 * kGemmKc * 2;  // bytes of one 128 x 64 BF16 tile
constexpr uint32_t kGemmTileB = 128 * kGemmKc * 2;  // at most 128 rows
constexpr uint32_t kGemmSmem = 2 * kGemmTileA + 2 * kGemmTileB + 16;

__device__ __forceinline__ void split_bf16(const float (&x)[8], uint4& hi, uint4& lo) {
    float h[8], l[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        h[j] = __bfloat162float(__float2bfloat16_rn(x[j]));
        l[j] = x[j] - h[j];
    }
    hi = make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]), pack_bf16(h[6], h[7]));
    lo = make_uint4(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]), pack_bf16(l[4], l[5]), pack_bf16(l[6], l[7]));
}

__global__ void __launch_bounds__(128, 1) tc_gemm_kernel(TcGemm g, uint32_t* status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int t = threadIdx.x, warp = t >> 5;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const uint32_t sAh = 0, sAl = kGemmTileA, sBh = 2 * kGemmTileA, sBl = 2 * kGemmTileA + kGemmTileB;
    const uint32_t bar = sbase + 2 * kGemmTileA + 2 * kGemmTileB;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * g.nt;
    const int k_beg = blockIdx.z * g.k_per;
    const int k_end = min(g.K, k_beg + g.k_per);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __shared__ uint32_t s_tmem;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(&s_tmem)),
                     "r"(128u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = idesc_bf16(128, g.nt);
    uint32_t phase = 0;
    bool ok = true, any = false;
    for (int kc = k_beg; kc < k_end && ok; kc += kGemmKc) {
        // stage A (128 rows) and B (nt rows) of this K chunk
        for (int e = t; e < (128 + g.nt) * (kGemmKc / 8); e += 128) {
            const bool isA = e < 128 * (kGemmKc / 8);
            const int ee = isA ? e : e - 128 * (kGemmKc / 8);
            const int r = ee / (kGemmKc / 8), k8 = (ee % (kGemmKc / 8)) * 8;
            const int row = isA ? m0 + r : n0 + r;
            const bool rin = isA ? row < g.M : row < g.N;
            float x[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int k = kc + k8 + j;
                x[j] = (rin && k < k_end) ? (isA ? g.A[row * g.sam + k * g.sak] : g.B[row * g.sbn + k * g.sbk])
                                          : 0.0f;
            }
            uint4 hi, lo;
            split_bf16(x, hi, lo);
            const uint32_t off = cm_offset(r, k8, kGemmKc);
            *reinterpret_cast<uint4*>(sm + (isA ? sAh : sBh) + off) = hi;
            if (!g.exact) *reinterpret_cast<uint4*>(sm + (isA ? sAl : sBl) + off) = lo;
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        if (t == 0) {
            tc_after_sync();
            for (int s = 0; s < kGemmKc / 16; ++s) {
                const uint32_t o = s * 256;
                const uint32_t lbo = 128, sbo = (kGemmKc / 8) * 128;
                umma_bf16(tmem, smem_desc(sbase + sAh + o, lbo, sbo), smem_desc(sbase + sBh + o, lbo, sbo), idesc,
                          any ? 1u : 0u);
                any = true;
                if (!g.exact) {
                    umma_bf16(tmem, smem_desc(sbase + sAh + o, lbo, sbo), smem_desc(sbase + sBl + o, lbo, sbo),
                              idesc, 1u);
                    umma_bf16(tmem, smem_desc(sbase + sAl + o, lbo, sbo), smem_desc(sbase + sBh + o, lbo, sbo),
                              idesc, 1u);
                }
            }
            umma_commit(bar);
        }
        any = true;
        ok = __syncthreads_and(mbar_wait(bar, phase)) != 0;
        phase ^= 1u;
        tc_after_sync();
    }
    if (ok && any) {
        const int row = m0 + t;
        const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
        for (int c0 = 0; c0 < g.nt; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + (uint32_t)c0, v);
            if (row < g.M)
                for (int j = 0; j < 16; ++j) {
                    const int n = n0 + c0 + j;
                    if (n >= g.N) break;
                    float* c = g.C + row * g.scm + n * g.scn;
                    if (g.split > 1) atomicAdd(c, v[j]);
                    else *c = v[j];
                }
        }
    }
    if (!ok && t == 0) atomicOr(status, (unsigned)NB_STATUS_QUEUE_TIMEOUT);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u) : "memory");
}

cudaError_t tc_gemm(const float* A, long sam, long sak, const float* B, long sbn, long sbk, float* C, long scm,
                    long scn, int M, int N, int K, bool exact, uint32_t* status, cudaStream_t s) {
    cudaError_t e = nb_raise_dynamic_smem((const void*)tc_gemm_kernel, kGemmSmem);
    if (e != cudaSuccess) return e;
    if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
    TcGemm g;
    g.A = A; g.sam = sam; g.sak = sak;
    g.B = B; g.sbn = sbn; g.sbk = sbk;
    g.C = C; g.scm = scm; g.scn = scn;
    g.M = M; g.N = N; g.K = K;
    g.nt = N <= 16 ? 16 : (N <= 32 ? 32 : (N <= 64 ? 64 : 128));
    g.exact = exact ? 1 : 0;
    const int mt = (M + 127) / 128, ntiles = (N + g.nt - 1) / g.nt;
    // split K until the grid has about one CTA per SM, at least 8 chunks (512) per split
    const int chunks = (K + kGemmKc - 1) / kGemmKc;
    int split = 1;
    while (mt * ntiles * split * 2 <= 148 && chunks / (split * 2) >= 8) split *= 2;
    g.k_per = ((chunks + split - 1) / split) * kGemmKc;
    g.split = (K + g.k_per - 1) / g.k_per;
    if (g.split > 1) {
        // C is dense [M, N] in one of the two orders for every split GEMM here
        cudaError_t e = cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * N, s);
        if (e != cudaSuccess) return e;
    }
    dim3 grid(mt, ntiles, g.split);
    tc_gemm_kernel<<<grid, 128, kGemmSmem, s>>>(g, status);
    return cudaGetLastError();
}

// X[rows, cols]: normalise (features) or round weights, to bf16 values held in fp32
__global__ void normalise_kernel(const float* __restrict__ x, const float* __restrict__ mean,
                                 const float* __restrict__ istd, int rows, int cols, float* __restrict__ y) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= (long)rows * cols) return;
    const int c = (int)(i % cols);
    y[i] = bf16_round(mean ? (x[i] - mean[c]) * istd[c] : x[i]);
}

// Z += bias; H = bf16(silu(Z))
__global__ void bias_silu_kernel(float* __restrict__ z, const float* __restrict__ b, float* __restrict__ h, int rows,
                                 int cols) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= (long)rows * cols) return;
    const float v = z[i] + b[i % cols];
    z[i] = v;
    h[i] = bf16_round(silu(v));
}

// Y += b3; loss and dY = 2 (Y - T / scale) / rows
__global__ void out_grad_kernel(float* __restrict__ y, const float* __restrict__ b, const float* __restrict__ t,
                                const float* __restrict__ scale, int rows, float* __restrict__ dy,
                                float* __restrict__ loss) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= (long)rows * kOut) return;
    const int c = (int)(i % kOut);
    const float v = y[i] + b[c];
    y[i] = v;
    const float e = v - t[i] / scale[c];
    dy[i] = 2.0f * e / (float)rows;
    atomicAdd(loss, e * e / (float)rows);
}

// dZ = dH * silu'(Z)
__global__ void silu_grad_kernel(const float* __restrict__ z, float* __restrict__ dh, long count) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float s = 1.0f / (1.0f + expf(-z[i]));
    dh[i] = dh[i] * (s + z[i] * s * (1.0f - s));
}

// db[c] = sum_r dZ[r, c]
__global__ void col_sum_kernel(const float* __restrict__ dz, int rows, int cols, float* __restrict__ db) {
    const int c = blockIdx.x;
    float s = 0.0f;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) s += dz[(size_t)r * cols + c];
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[c] = red[0];
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, long count, float lr, float b1, float b2, float eps, float wd,
                            float c1, float c2) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    m1[i] = b1 * m1[i] + (1.0f - b1) * gi;
    m2[i] = b2 * m2[i] + (1.0f - b2) * gi * gi;
    const float mh = m1[i] / c1, vh = m2[i] / c2;
    w[i] -= lr * (mh / (sqrtf(vh) + eps) + wd * w[i]);
}

inline int blocks(long n, int t = 256) { return (int)((n + t - 1) / t); }

inline int contact_grid(long capacity) { return nb_contact_grid(capacity, 256); }

}  // namespace

cudaError_t nb_launch_ws_features(const NbModelDesc* m, const float* q, const float* qd,
                                  const NbContactsPublic* pub, const float* prev_lambda, const int32_t* match_index,
                                  int32_t* body_count, float dt, float* feat, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(body_count, 0, sizeof(int32_t) * (size_t)(m->body_count > 0 ? m->body_count : 1), s);
    if (e != cudaSuccess) return e;
    if (pub->capacity <= 0) return cudaSuccess;
    const int g = contact_grid(pub->capacity);
    ws_count_kernel<<<g, 256, 0, s>>>(*m, *pub, body_count);
    ws_features_kernel<<<g, 256, 0, s>>>(*m, q, qd, *pub, prev_lambda, match_index, body_count, dt, feat);
    return cudaGetLastError();
}

cudaError_t nb_launch_ws_targets(const NbContactsPublic* pub, float* impulse, float* lam, int clear, cudaStream_t s) {
    if (pub->capacity <= 0) return cudaSuccess;
    ws_targets_kernel<<<contact_grid(pub->capacity), 256, 0, s>>>(*pub, impulse, lam, clear);
    return cudaGetLastError();
}

cudaError_t nb_launch_ws_infer(const NbWsNet* net, const float* feat, const int32_t* count, int cap, float* out,
                               uint32_t* status, cudaStream_t s) {
    cudaError_t e = nb_raise_dynamic_smem((const void*)ws_infer_kernel, kSmBytes);
    if (e != cudaSuccess) return e;
    if (cap <= 0) return cudaSuccess;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (cap + kTile - 1) / kTile;
    const int grid = tiles < 2 * sms ? tiles : 2 * sms;  // shared memory fits 2 CTAs per SM
    ws_infer_kernel<<<grid, kInferThreads, kSmBytes, s>>>(*net, feat, count, cap, out, status);
    return cudaGetLastError();
}

cudaError_t nb_launch_ws_grads(const NbWsTrain* a, cudaStream_t s) {
    const int R = a->rows;
    float* Wq[3] = {a->scratch_wq, a->scratch_wq + kHid * kIn, a->scratch_wq + kHid * kIn + kHid * kHid};
    cudaError_t e = cudaMemsetAsync(a->loss, 0, sizeof(float), s);
    if (e != cudaSuccess) return e;
    // bf16-rounded weights and normalised inputs (what inference multiplies)
    normalise_kernel<<<blocks(kHid * kIn), 256, 0, s>>>(a->w1, nullptr, nullptr, kHid, kIn, Wq[0]);
    normalise_kernel<<<blocks(kHid * kHid), 256, 0, s>>>(a->w2, nullptr, nullptr, kHid, kHid, Wq[1]);
    normalise_kernel<<<blocks(kOut * kHid), 256, 0, s>>>(a->w3, nullptr, nullptr, kOut, kHid, Wq[2]);
    normalise_kernel<<<blocks((long)R * kIn), 256, 0, s>>>(a->x, a->in_mean, a->in_inv_std, R, kIn, a->xn);
    uint32_t* st = a->status;
    // forward: operands are BF16 values, one MMA per K step
    if ((e = tc_gemm(a->xn, kIn, 1, Wq[0], kIn, 1, a->z1, kHid, 1, R, kHid, kIn, true, st, s))) return e;
    bias_silu_kernel<<<blocks((long)R * kHid), 256, 0, s>>>(a->z1, a->b1, a->h1, R, kHid);
    if ((e = tc_gemm(a->h1, kHid, 1, Wq[1], kHid, 1, a->z2, kHid, 1, R, kHid, kHid, true, st, s))) return e;
    bias_silu_kernel<<<blocks((long)R * kHid), 256, 0, s>>>(a->z2, a->b2, a->h2, R, kHid);
    if ((e = tc_gemm(a->h2, kHid, 1, Wq[2], kHid, 1, a->y, kOut, 1, R, kOut, kHid, true, st, s))) return e;
    out_grad_kernel<<<blocks((long)R * kOut), 256, 0, s>>>(a->y, a->b3, a->t, a->out_scale, R, a->dy, a->loss);
    // backward: gradient operands split into hi + lo BF16
    // g_w3[o, h] = sum_r dy[r, o] h2[r, h]  (m = h, n = o, k = r)
    if ((e = tc_gemm(a->h2, 1, kHid, a->dy, 1, kOut, a->g_w3, 1, kHid, kHid, kOut, R, false, st, s))) return e;
    col_sum_kernel<<<kOut, 256, 0, s>>>(a->dy, R, kOut, a->g_b3);
    // dh[r, h] = sum_o dy[r, o] w3[o, h]
    if ((e = tc_gemm(a->dy, kOut, 1, Wq[2], 1, kHid, a->dh, kHid, 1, R, kHid, kOut, false, st, s))) return e;
    silu_grad_kernel<<<blocks((long)R * kHid), 256, 0, s>>>(a->z2, a->dh, (long)R * kHid);
    // g_w2[i, j] = sum_r dz2[r, i] h1[r, j]
    if ((e = tc_gemm(a->dh, 1, kHid, a->h1, 1, kHid, a->g_w2, kHid, 1, kHid, kHid, R, false, st, s))) return e;
    col_sum_kernel<<<kHid, 256, 0, s>>>(a->dh, R, kHid, a->g_b2);
    // dh2[r, j] = sum_i dz2[r, i] w2[i, j]
    if ((e = tc_gemm(a->dh, kHid, 1, Wq[1], 1, kHid, a->dh2, kHid, 1, R, kHid, kHid, false, st, s))) return e;
    silu_grad_kernel<<<blocks((long)R * kHid), 256, 0, s>>>(a->z1, a->dh2, (long)R * kHid);
    // g_w1[i, j] = sum_r dz1[r, i] xn[r, j]
    if ((e = tc_gemm(a->dh2, 1, kHid, a->xn, 1, kIn, a->g_w1, kIn, 1, kHid, kIn, R, false, st, s))) return e;
    col_sum_kernel<<<kHid, 256, 0, s>>>(a->dh2, R, kHid, a->g_b1);
    return cudaGetLastError();
}

cudaError_t nb_launch_ws_adam(float* w, const float* g, float* m1, float* m2, long count, float lr, float b1,
                              float b2, float eps, float wd, int step, cudaStream_t s) {
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    adam_kernel<<<blocks(count), 256, 0, s>>>(w, g, m1, m2, count, lr, b1, b2, eps, wd, c1, c2);
    return cudaGetLastError();
}
