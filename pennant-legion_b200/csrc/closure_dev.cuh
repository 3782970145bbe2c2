// closure_dev.cuh -- the learned QCS closure on the device: corner
// features, the network's parameter image, and its tcgen05 inference.
//
// The closure stands in for QCS::calcForce's corner forces (QCS.cc:246-327,
// setQCnForce: cqe1 = crmu (u_p - u_prev) / elen_prev and cqe2 = crmu
// (u_next - u_p) / elen, crmu = zkur * zrp * evol) on corners that compress.
// Its inputs are 14 dimensionless numbers of the corner, expressed in a
// frame whose x axis runs from the corner's point to the zone centre:
//
//   0-1   (u_p - u_prev) / D           velocity differences along the two
//   2-3   (u_next - u_p) / D           edges and to the zone centre,
//   4-5   (u_zone - u_p) / D           D = the largest of the three
//   6-7   (x_prev - x_p) / L           the two edges, L = mean edge length
//   8-9   (x_next - x_p) / L
//   10    |x_zone - x_p| / L
//   11    rho = a D / (a D + b c)      compression: a = q2 (qgamma+1) / 4,
//                                      b = q1, c = the zone sound speed
//   12-13 direction of the mean corner velocity (evol's axis choice)
//
// and its 4 outputs are cqe1 and cqe2 in that frame divided by
// zrp * D * (a D + b c), the scale of the QCS force, so the network maps
// bounded numbers to bounded numbers whatever the mesh size, energy or the
// deck's q1/q2.  Corners with D <= dead * c carry a negligible viscous force
// and get none (the dead zone); corners that are compressed beyond rho_max,
// or whose normalised inputs lie beyond ood_kappa standard deviations of
// the training data, fall back to the plain QCS.
//
// Network: 14 -> 64 -> 64 -> 4, GELU (tanh form, Hendrycks & Gimpel 2016),
// BF16 weights and activations, FP32 accumulation.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace pnt {

constexpr int kClIn = 14;       // inputs
constexpr int kClInPad = 16;    // padded to one MMA K step
constexpr int kClHid = 64;      // hidden width
constexpr int kClOut = 4;       // outputs
constexpr int kClOutPad = 16;   // layer-3 MMA N
// parameters in the order W1 [64][14], b1 [64], W2 [64][64], b2 [64],
// W3 [4][64], b3 [4] (row = output unit)
constexpr int kClW1 = 0;
constexpr int kClB1 = kClW1 + kClHid * kClIn;
constexpr int kClW2 = kClB1 + kClHid;
constexpr int kClB2 = kClW2 + kClHid * kClHid;
constexpr int kClW3 = kClB2 + kClHid;
constexpr int kClB3 = kClW3 + kClOut * kClHid;
constexpr int kClParams = kClB3 + kClOut;   // 5380

// Corner classes counted by the learned cycle.
enum { kClassZero = 0, kClassDead = 1, kClassMlp = 2, kClassFallback = 3, kClassOod = 4, kClassAcute = 5,
       kClassErr = 6, kClassZones = 7, kClassCount = 8 };

// The parameter image: byte layout of the tcgen05 inference's shared-memory
// copy (operands in the K-major canonical layout without swizzle: element
// (row r, k) of an R-row operand at byte (k/8)*R*16 + r*16 + (k%8)*2).
constexpr int kImgW1 = 0;        // N=64 x K=16 bf16
constexpr int kImgW2 = 2048;     // N=64 x K=64
constexpr int kImgW3 = 10240;    // N=16 x K=64 (rows 4..15 zero)
constexpr int kImgB1 = 12288;    // 64 f32
constexpr int kImgB2 = 12544;    // 64 f32
constexpr int kImgB3 = 12800;    // 16 f32 (4 used)
constexpr int kImgFMean = 12864; // 16 f32 (14 used)
constexpr int kImgFIstd = 12928; // 16 f32 (1/std; 0 for the pad inputs)
constexpr int kImgTMean = 12992; // 4 f32
constexpr int kImgTStd = 13008;  // 4 f32
constexpr int kImgThr = 13024;   // dead, rho_max, ood_kappa, pad (f32)
constexpr int kImgBytes = 13056;

__host__ __device__ constexpr int canon_off(int r, int k, int rows) { return (k >> 3) * rows * 16 + r * 16 + (k & 7) * 2; }

// Deferred corners of the learned cycle: pass A records every zone that has
// a compressing corner outside the dead zone (64 zones = 256 rows per
// inference batch) with the raw FP32 data of each corner, relative to the
// zone's first point: position, previous and next points, zone centre,
// velocities of the point, previous and next points and the zone centre,
// the mean corner velocity (absolute), the zone's sound speed and density,
// and a flag (1 = deferred corner).  Per zone: first side, sides.
constexpr int kRecFloats = 24;
enum { kRecX = 0, kRecXp = 2, kRecXn = 4, kRecXz = 6, kRecU = 8, kRecUp = 10, kRecUn = 12, kRecUz = 14,
       kRecUav = 16, kRecSs = 18, kRecRho = 19, kRecFlag = 20 };

// Shared memory of the 256-row inference block.
constexpr int kMlpRows = 256;
constexpr int kSmImg = 0;
constexpr int kSmA0 = 13312;                        // 2 tiles x 128 x 16 bf16
constexpr int kSmH = kSmA0 + 2 * 128 * 16 * 2;      // 2 tiles x 128 x 64 bf16
constexpr int kSmBar = kSmH + 2 * 128 * 64 * 2;     // mbarrier (8 B) + TMEM address (4 B)
constexpr int kMlpSmemBytes = kSmBar + 64;
constexpr uint32_t kTmemCols = 128;                 // two 128 x 64 f32 accumulators

// ----------------------------------------------------------------------
// Corner features (T = double for the harvest, float in the FP32 cycle)
// ----------------------------------------------------------------------
template <typename T>
struct ClV {
    T x, y;
};

__device__ __forceinline__ double cl_sqrt(double v) { return sqrt(v); }
__device__ __forceinline__ float cl_sqrt(float v) { return sqrtf(v); }

// Fills f[0..13]; returns false for a corner in the dead zone.  The frame
// (cx, cy) and force scale D * (a D + b c) are returned for the caller.
template <typename T>
__device__ __forceinline__ bool closure_features(ClV<T> xp, ClV<T> xpp, ClV<T> xpn, ClV<T> xz, ClV<T> up, ClV<T> upp,
                                                 ClV<T> upn, ClV<T> uz, ClV<T> uav, T css, T qa, T qb, T dead,
                                                 float* f, T& cx, T& cy, T& scale) {
    // the dead-zone test first, on squares: most compressing corners ahead
    // of a shock carry round-off velocities and stop here
    const T d1x = up.x - upp.x, d1y = up.y - upp.y;
    const T d2x = upn.x - up.x, d2y = upn.y - up.y;
    const T dcx = uz.x - up.x, dcy = uz.y - up.y;
    T m2 = d1x * d1x + d1y * d1y;
    const T n2 = d2x * d2x + d2y * d2y, nc = dcx * dcx + dcy * dcy;
    m2 = (n2 > m2) ? n2 : m2;
    m2 = (nc > m2) ? nc : m2;
    const T lim = dead * css;
    if (!(m2 > lim * lim)) return false;
    const T D = cl_sqrt(m2);
    const T dx = xz.x - xp.x, dy = xz.y - xp.y;
    const T il = T(1) / cl_sqrt(dx * dx + dy * dy);
    cx = dx * il;
    cy = dy * il;
    const T e1x = xpp.x - xp.x, e1y = xpp.y - xp.y;
    const T e2x = xpn.x - xp.x, e2y = xpn.y - xp.y;
    const T iL = T(2) / (cl_sqrt(e1x * e1x + e1y * e1y) + cl_sqrt(e2x * e2x + e2y * e2y));
    const T Q = qa * D + qb * css;
    scale = D * Q;
    const T iD = T(1) / D;
    f[0] = (float)((cx * d1x + cy * d1y) * iD);
    f[1] = (float)((cx * d1y - cy * d1x) * iD);
    f[2] = (float)((cx * d2x + cy * d2y) * iD);
    f[3] = (float)((cx * d2y - cy * d2x) * iD);
    f[4] = (float)((cx * dcx + cy * dcy) * iD);
    f[5] = (float)((cx * dcy - cy * dcx) * iD);
    f[6] = (float)((cx * e1x + cy * e1y) * iL);
    f[7] = (float)((cx * e1y - cy * e1x) * iL);
    f[8] = (float)((cx * e2x + cy * e2y) * iL);
    f[9] = (float)((cx * e2y - cy * e2x) * iL);
    f[10] = (float)(T(1) / il * iL);
    f[11] = (float)(qa * D / Q);
    const T am = cl_sqrt(uav.x * uav.x + uav.y * uav.y);
    const T ia = (am > T(0)) ? T(1) / am : T(0);
    f[12] = (float)((cx * uav.x + cy * uav.y) * ia);
    f[13] = (float)((cx * uav.y - cy * uav.x) * ia);
    return true;
}

// ----------------------------------------------------------------------
// GELU (tanh form)
// ----------------------------------------------------------------------
constexpr float kGeluC = 0.7978845608028654f;   // sqrt(2/pi)
constexpr float kGeluA = 0.044715f;

__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu_fast(float x) {
    const float u = kGeluC * (x + kGeluA * x * x * x);
    return 0.5f * x * (1.f + tanh_approx(u));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// ----------------------------------------------------------------------
// tcgen05 / TMEM / mbarrier primitives (PTX ISA 8.7, sm_100a)
// ----------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle.  lbo = byte distance
// between the two 8-element K halves of an MMA step, sbo = between 8-row
// groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version of sm_100
    return d;                 // base offset 0, layout type 0 (no swizzle)
}
// Instruction descriptor of kind::f16: BF16 A and B (both K-major), F32 D.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
// Bounded wait: false if the phase did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, int limit = 1 << 20) {
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float* v) {
    uint32_t r[4];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
}

// Hidden layer epilogue: this thread's row of a 128 x 64 accumulator ->
// bias, GELU, BF16 -> its row of the next layer's A operand.
__device__ __forceinline__ void mlp_hidden_epilogue(uint32_t tacc, const float* bias, uint8_t* hrow) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float v[16];
        tmem_ld16(tacc + 16 * c, v);
        uint32_t w[8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
            w[i] = pack_bf16(gelu_fast(v[2 * i] + bias[16 * c + 2 * i]), gelu_fast(v[2 * i + 1] + bias[16 * c + 2 * i + 1]));
        // k = 16c..16c+7 is K chunk 2c, k = 16c+8.. chunk 2c+1 (128 rows: 2048 B apart)
        *reinterpret_cast<uint4*>(hrow + (2 * c) * 2048) = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4*>(hrow + (2 * c + 1) * 2048) = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

// The network on the kMlpRows (256) rows of a CTA of 256 threads: thread t
// owns row t (row t % 128 of M tile t / 128, whose accumulator is TMEM lane
// t % 128).  Every thread of the CTA calls setup once, rows once per batch
// of 256 rows, and teardown once.  smem: kMlpSmemBytes of dynamic shared
// memory (16-byte aligned); gimg: the parameter image in global memory.
//
// Tensor-core waits are bounded.  Once a wait runs out on any thread, the
// CTA agrees on it at its next barrier (__syncthreads_and) and issues no
// further MMA, commit or TMEM load: the rows of that batch and of every
// later one come out as zeros, and teardown waits (bounded again) for the
// last commit issued, which covers every MMA still in flight, before it
// frees the TMEM columns.
struct MlpState {
    uint32_t tbase;   // TMEM columns of the two accumulators
    uint32_t phase;   // commits issued (each ends one mbarrier phase)
    bool ok;          // every tensor-core wait so far completed
};

__device__ __forceinline__ void closure_mlp_setup(uint8_t* smem, const uint8_t* __restrict__ gimg, MlpState& st) {
    const int t = threadIdx.x;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kSmBar + 8);
    for (int i = t; i < kImgBytes / 16; i += kMlpRows)
        reinterpret_cast<uint4*>(smem + kSmImg)[i] = __ldg(reinterpret_cast<const uint4*>(gimg) + i);
    if (t == 0) mbar_init(smem_addr(smem + kSmBar), 1);
    if ((t >> 5) == 0) {
        tmem_alloc(smem_addr(tslot), kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    st.tbase = *tslot;
    st.phase = 0;
    st.ok = true;
}

// f: this row's raw inputs; out: its 4 outputs, denormalised (zero after a
// wait ran out, in this batch or an earlier one).
__device__ __forceinline__ void closure_mlp_rows(uint8_t* smem, MlpState& st, const float* f, float* out) {
    const int t = threadIdx.x;
    const int warp = t >> 5;
    const int tile = t >> 7;
    const int row = t & 127;
    const uint32_t mbar = smem_addr(smem + kSmBar);
#pragma unroll
    for (int i = 0; i < 4; ++i) out[i] = 0.f;
    // a wait that ran out earlier on any thread: no more tensor-core work
    st.ok = __syncthreads_and(st.ok) != 0;
    if (!st.ok) return;
    // normalised inputs -> this row of the layer-1 A operand
    {
        const float* mean = reinterpret_cast<const float*>(smem + kImgFMean);
        const float* istd = reinterpret_cast<const float*>(smem + kImgFIstd);
        float z[kClInPad];
#pragma unroll
        for (int i = 0; i < kClInPad; ++i) z[i] = (i < kClIn) ? (f[i] - mean[i]) * istd[i] : 0.f;
        uint8_t* arow = smem + kSmA0 + tile * 4096 + row * 16;
        *reinterpret_cast<uint4*>(arow) =
            make_uint4(pack_bf16(z[0], z[1]), pack_bf16(z[2], z[3]), pack_bf16(z[4], z[5]), pack_bf16(z[6], z[7]));
        *reinterpret_cast<uint4*>(arow + 2048) = make_uint4(pack_bf16(z[8], z[9]), pack_bf16(z[10], z[11]),
                                                           pack_bf16(z[12], z[13]), pack_bf16(z[14], z[15]));
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = st.tbase;
    const uint32_t tacc = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(tile * 64);
    const uint32_t sb = smem_addr(smem);

    // layer 1: [128 x 16] x [16 x 64] per tile
    if (t == 0) {
        for (int j = 0; j < 2; ++j)
            umma_bf16(tbase + j * 64, umma_desc(sb + kSmA0 + j * 4096, 2048, 128), umma_desc(sb + kImgW1, 1024, 128),
                      umma_idesc_bf16(128, 64), 0u);
        umma_commit(mbar);
    }
    ++st.phase;
    bool w = mbar_wait(mbar, (st.phase - 1) & 1);
    tc_fence_after();
    uint8_t* hrow = smem + kSmH + tile * 16384 + row * 16;
    if (w) mlp_hidden_epilogue(tacc, reinterpret_cast<const float*>(smem + kImgB1), hrow);
    fence_async_smem();
    tc_fence_before();
    st.ok = __syncthreads_and(w) != 0;
    tc_fence_after();
    if (!st.ok) return;

    // layer 2: [128 x 64] x [64 x 64]
    if (t == 0) {
        for (int j = 0; j < 2; ++j)
            for (int kb = 0; kb < 4; ++kb)
                umma_bf16(tbase + j * 64, umma_desc(sb + kSmH + j * 16384 + kb * 4096, 2048, 128),
                          umma_desc(sb + kImgW2 + kb * 2048, 1024, 128), umma_idesc_bf16(128, 64), kb > 0 ? 1u : 0u);
        umma_commit(mbar);
    }
    ++st.phase;
    w = mbar_wait(mbar, (st.phase - 1) & 1);
    tc_fence_after();
    if (w) mlp_hidden_epilogue(tacc, reinterpret_cast<const float*>(smem + kImgB2), hrow);
    fence_async_smem();
    tc_fence_before();
    st.ok = __syncthreads_and(w) != 0;
    tc_fence_after();
    if (!st.ok) return;

    // layer 3: [128 x 64] x [64 x 16] (4 outputs used)
    if (t == 0) {
        for (int j = 0; j < 2; ++j)
            for (int kb = 0; kb < 4; ++kb)
                umma_bf16(tbase + j * 64, umma_desc(sb + kSmH + j * 16384 + kb * 4096, 2048, 128),
                          umma_desc(sb + kImgW3 + kb * 512, 256, 128), umma_idesc_bf16(128, 16), kb > 0 ? 1u : 0u);
        umma_commit(mbar);
    }
    ++st.phase;
    w = mbar_wait(mbar, (st.phase - 1) & 1);
    tc_fence_after();
    if (w) {
        float y[4];
        tmem_ld4(tacc, y);
        const float* b3 = reinterpret_cast<const float*>(smem + kImgB3);
        const float* tmean = reinterpret_cast<const float*>(smem + kImgTMean);
        const float* tstd = reinterpret_cast<const float*>(smem + kImgTStd);
#pragma unroll
        for (int i = 0; i < 4; ++i) out[i] = (y[i] + b3[i]) * tstd[i] + tmean[i];
    }
    // this thread's view; the next batch's (or teardown's) barrier makes it
    // the CTA's
    st.ok = w;
    // the next batch's layer-1 MMA overwrites these accumulators after the
    // barrier that follows its input writes
    tc_fence_before();
}

// Frees the TMEM columns.  After a wait that ran out, first waits (bounded)
// for the last commit issued, so no MMA still writes the columns; returns
// false on every thread if any tensor-core wait ran out.
__device__ __forceinline__ bool closure_mlp_teardown(uint8_t* smem, MlpState& st) {
    tc_fence_before();
    const bool ok = __syncthreads_and(st.ok) != 0;
    if (!ok && st.phase > 0) {
        mbar_wait(smem_addr(smem + kSmBar), (st.phase - 1) & 1);
        tc_fence_before();
        __syncthreads();
    }
    if ((threadIdx.x >> 5) == 0) {
        tc_fence_after();
        tmem_dealloc(st.tbase, kTmemCols);
    }
    return ok;
}

// One batch of 256 rows (the standalone inference).
__device__ __forceinline__ bool closure_mlp_block(uint8_t* smem, const uint8_t* __restrict__ gimg, const float* f,
                                                  float* out) {
    MlpState st;
    closure_mlp_setup(smem, gimg, st);
    closure_mlp_rows(smem, st, f, out);
    return closure_mlp_teardown(smem, st);
}

}  // namespace pnt
