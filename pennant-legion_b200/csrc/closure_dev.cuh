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
#include <cuda_fp16.h>
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
// a compressing corner outside the dead zone, kZoneRecF4 float4 (112 B) a
// zone, in FP32 relative to the zone's first point:
//   [0], [1]  positions of points 0..3 (x, y pairs)
//   [2], [3]  velocities of points 0..3 (relative to point 0's)
//   [4]       zone centre, mean velocity of the zone's points
//   [5]       velocity of point 0 (absolute), sound speed, density
//   [6]       first side, sides, deferred-corner bits (int bits), unused
// (points 3 of a 3-sided zone are zeros).
constexpr int kZoneRecF4 = 7;

// The closure pass: kCpThreads threads a CTA, kCpCtasPerSm CTAs an SM (64
// TMEM columns per 128 threads).  Its shared memory: the parameter image,
// the BF16 input rows of up to kCpRows corners (two a thread, 128-row
// operand tiles), the hidden activations of one run of kCpThreads rows, an
// mbarrier and the TMEM address.  The outputs of a run overwrite the first
// kCpThreads * 16 bytes of its own operand tiles, whose MMAs are complete
// by then.
#ifndef PNT_CLOSURE_THREADS
#define PNT_CLOSURE_THREADS 256
#endif
constexpr int kCpThreads = PNT_CLOSURE_THREADS;
static_assert(kCpThreads == 128 || kCpThreads == 256, "one or two M tiles a run");
constexpr int kCpCtasPerSm = kCpThreads == 128 ? 6 : 3;
constexpr uint32_t kCpTmemCols = kCpThreads / 2;
constexpr int kCpRows = 2 * kCpThreads;
constexpr int kCpA0 = 13312;
constexpr int kCpH = kCpA0 + kCpRows * 32;
constexpr int kCpBar = kCpH + (kCpThreads / 128) * 128 * 64 * 2;
constexpr int kCpSmemBytes = kCpBar + 64;

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

// GELU of two values: the argument u = c (x + a x^3) and the result
// 0.5 x (1 + tanh u) in packed FP32 (two lanes an instruction), tanh u in
// FP16 (tanh.approx.f16x2: two a special-function instruction, relative
// error ~2^-11, below the BF16 rounding the activation gets next; u beyond
// the FP16 range rounds to +-inf, whose tanh is +-1).  Every rounding is
// written out: the same bits in every kernel that inlines it, whatever the
// compiler's contraction flags.
__device__ __forceinline__ float2 gelu2_fast(float2 x) {
    const float2 p = __ffma2_rn(__fmul2_rn(make_float2(kGeluA, kGeluA), __fmul2_rn(x, x)), x, x);   // x + a x^3
    const float2 u = __fmul2_rn(make_float2(kGeluC, kGeluC), p);
    const float2 th = __half22float2(h2tanh_approx(__floats2half2_rn(u.x, u.y)));
    const float2 hx = __fmul2_rn(make_float2(0.5f, 0.5f), x);
    return __ffma2_rn(hx, th, hx);
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
        for (int i = 0; i < 8; ++i) {
            const float2 g = gelu2_fast(__fadd2_rn(make_float2(v[2 * i], v[2 * i + 1]),
                                                   make_float2(bias[16 * c + 2 * i], bias[16 * c + 2 * i + 1])));
            w[i] = pack_bf16(g.x, g.y);
        }
        // k = 16c..16c+7 is K chunk 2c, k = 16c+8.. chunk 2c+1 (128 rows: 2048 B apart)
        *reinterpret_cast<uint4*>(hrow + (2 * c) * 2048) = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4*>(hrow + (2 * c + 1) * 2048) = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

// Tensor-core state of a CTA running the network.  Every thread of the CTA
// calls setup once, the row functions once per batch, and teardown once.
//
// Tensor-core waits are bounded.  Once a wait runs out on any thread, the
// CTA agrees on it at its next barrier (__syncthreads_and) and issues no
// further MMA, commit or TMEM load: the rows of that batch and of every
// later one get no output, and teardown waits (bounded again) for the last
// commit issued, which covers every MMA still in flight, before it frees
// the TMEM columns.
struct MlpState {
    uint32_t tbase;   // TMEM columns of the accumulators (64 per 128-row M tile)
    uint32_t ncols;   // TMEM columns allocated
    uint32_t phase;   // commits issued (each ends one mbarrier phase)
    uint32_t bar;     // shared-memory address of the mbarrier
    bool ok;          // every tensor-core wait so far completed
};

// img: kImgBytes of shared memory (16-byte aligned) for the parameter image,
// copied from gimg; bar: an mbarrier; tslot: where tcgen05.alloc writes the
// TMEM address; ncols: TMEM columns to allocate (64 per M tile).
__device__ __forceinline__ void closure_mlp_setup(uint8_t* img, const uint8_t* __restrict__ gimg, uint64_t* bar,
                                                  uint32_t* tslot, uint32_t ncols, MlpState& st) {
    const int t = threadIdx.x;
    for (int i = t; i < kImgBytes / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(img)[i] = __ldg(reinterpret_cast<const uint4*>(gimg) + i);
    if (t == 0) mbar_init(smem_addr(bar), 1);
    if ((t >> 5) == 0) {
        tmem_alloc(smem_addr(tslot), ncols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    st.tbase = *tslot;
    st.ncols = ncols;
    st.phase = 0;
    st.bar = smem_addr(bar);
    st.ok = true;
}

// Row `slot` of a staged input operand a0 (128-row tiles of 4 KB): this
// corner's inputs, normalised, in BF16.
__device__ __forceinline__ void closure_stage_row(uint8_t* a0, int slot, const float* f, const float* mean,
                                                  const float* istd) {
    float z[kClInPad];
#pragma unroll
    for (int i = 0; i < kClInPad; ++i) z[i] = (i < kClIn) ? __fmul_rn(__fsub_rn(f[i], mean[i]), istd[i]) : 0.f;
    uint8_t* arow = a0 + (slot >> 7) * 4096 + (slot & 127) * 16;
    *reinterpret_cast<uint4*>(arow) =
        make_uint4(pack_bf16(z[0], z[1]), pack_bf16(z[2], z[3]), pack_bf16(z[4], z[5]), pack_bf16(z[6], z[7]));
    *reinterpret_cast<uint4*>(arow + 2048) = make_uint4(pack_bf16(z[8], z[9]), pack_bf16(z[10], z[11]),
                                                       pack_bf16(z[12], z[13]), pack_bf16(z[14], z[15]));
}

// The network on staged rows [base, base + 2 * 128) of the operand tiles at
// a0 (its M tiles base / 128 and base / 128 + 1, the second only when more
// than 128 of the n staged rows fall in the run; a CTA of 128 threads runs
// one M tile), hidden activations in h (16 KB per M tile).  Thread t takes
// row base + t (TMEM lane t % 128 of M tile t / 128), and warps without
// staged rows skip the epilogues.  The output of row base + t
// (denormalised) goes to float4 t of the run's first operand tile, whose
// MMAs are complete by then.  Every thread of the CTA calls it; the caller
// has staged the rows and issued fence_async_smem().  After a wait runs out
// no further MMA is issued and the run's outputs are not written.
__device__ __forceinline__ void closure_mlp_run(const uint8_t* img, uint8_t* a0, uint8_t* h, MlpState& st, int base,
                                                int n) {
    const int t = threadIdx.x;
    const int warp = t >> 5;
    const int tile = t >> 7;
    const int row = t & 127;
    const int mt = (n - base > 128 && blockDim.x > 128) ? 2 : 1;
    const bool live = base + 32 * warp < n;   // warp-uniform
    const uint32_t mbar = st.bar;
    // the previous run's TMEM loads finish before this run's MMAs overwrite
    // the accumulators; the staged rows are visible to the tensor cores
    tc_fence_before();
    st.ok = __syncthreads_and(st.ok) != 0;
    tc_fence_after();
    if (!st.ok) return;
    const uint32_t tbase = st.tbase;
    const uint32_t tacc = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(tile * 64);
    const uint32_t si = smem_addr(img);
    const uint32_t sh = smem_addr(h);
    uint8_t* out_tile = a0 + (base >> 7) * 4096;
    const uint32_t sa = smem_addr(out_tile);
    const float* fimg = reinterpret_cast<const float*>(img);

    // layer 1: [128 x 16] x [16 x 64] per M tile
    if (t == 0) {
        for (int j = 0; j < mt; ++j)
            umma_bf16(tbase + j * 64, umma_desc(sa + j * 4096, 2048, 128), umma_desc(si + kImgW1, 1024, 128),
                      umma_idesc_bf16(128, 64), 0u);
        umma_commit(mbar);
    }
    ++st.phase;
    bool w = __all_sync(0xffffffffu, mbar_wait(mbar, (st.phase - 1) & 1));
    tc_fence_after();
    uint8_t* hrow = h + tile * 16384 + row * 16;
    if (w && live) mlp_hidden_epilogue(tacc, fimg + kImgB1 / 4, hrow);
    fence_async_smem();
    tc_fence_before();
    st.ok = __syncthreads_and(w) != 0;
    tc_fence_after();
    if (!st.ok) return;

    // layer 2: [128 x 64] x [64 x 64]
    if (t == 0) {
        for (int j = 0; j < mt; ++j)
            for (int kb = 0; kb < 4; ++kb)
                umma_bf16(tbase + j * 64, umma_desc(sh + j * 16384 + kb * 4096, 2048, 128),
                          umma_desc(si + kImgW2 + kb * 2048, 1024, 128), umma_idesc_bf16(128, 64), kb > 0 ? 1u : 0u);
        umma_commit(mbar);
    }
    ++st.phase;
    w = __all_sync(0xffffffffu, mbar_wait(mbar, (st.phase - 1) & 1));
    tc_fence_after();
    if (w && live) mlp_hidden_epilogue(tacc, fimg + kImgB2 / 4, hrow);
    fence_async_smem();
    tc_fence_before();
    st.ok = __syncthreads_and(w) != 0;
    tc_fence_after();
    if (!st.ok) return;

    // layer 3: [128 x 64] x [64 x 16] (4 outputs used)
    if (t == 0) {
        for (int j = 0; j < mt; ++j)
            for (int kb = 0; kb < 4; ++kb)
                umma_bf16(tbase + j * 64, umma_desc(sh + j * 16384 + kb * 4096, 2048, 128),
                          umma_desc(si + kImgW3 + kb * 512, 256, 128), umma_idesc_bf16(128, 16), kb > 0 ? 1u : 0u);
        umma_commit(mbar);
    }
    ++st.phase;
    w = __all_sync(0xffffffffu, mbar_wait(mbar, (st.phase - 1) & 1));
    tc_fence_after();
    if (w && live) {
        float y[4];
        tmem_ld4(tacc, y);
        const float* b3 = fimg + kImgB3 / 4;
        const float* tmean = fimg + kImgTMean / 4;
        const float* tstd = fimg + kImgTStd / 4;
        if (base + t < n)
            reinterpret_cast<float4*>(out_tile)[t] = make_float4(
                __fmaf_rn(__fadd_rn(y[0], b3[0]), tstd[0], tmean[0]), __fmaf_rn(__fadd_rn(y[1], b3[1]), tstd[1], tmean[1]),
                __fmaf_rn(__fadd_rn(y[2], b3[2]), tstd[2], tmean[2]), __fmaf_rn(__fadd_rn(y[3], b3[3]), tstd[3], tmean[3]));
    }
    // this thread's view; the next run's (or teardown's) barrier makes it
    // the CTA's
    st.ok = w;
    tc_fence_before();
}

// Frees the TMEM columns.  After a wait that ran out, first waits (bounded)
// for the last commit issued, so no MMA still writes the columns; returns
// false on every thread if any tensor-core wait ran out.
__device__ __forceinline__ bool closure_mlp_teardown(MlpState& st) {
    tc_fence_before();
    const bool ok = __syncthreads_and(st.ok) != 0;
    if (!ok && st.phase > 0) {
        mbar_wait(st.bar, (st.phase - 1) & 1);
        tc_fence_before();
        __syncthreads();
    }
    if ((threadIdx.x >> 5) == 0) {
        tc_fence_after();
        tmem_dealloc(st.tbase, st.ncols);
    }
    return ok;
}

// One batch of up to 256 rows in a CTA of 256 threads (the standalone
// inference): thread t's inputs f -> its outputs (zeros for rows >= n or
// after a wait ran out).  smem: kMlpSmemBytes of dynamic shared memory
// (16-byte aligned); gimg: the parameter image in global memory.
__device__ __forceinline__ bool closure_mlp_block(uint8_t* smem, const uint8_t* __restrict__ gimg, const float* f,
                                                  int n, float* out) {
    MlpState st;
    closure_mlp_setup(smem + kSmImg, gimg, reinterpret_cast<uint64_t*>(smem + kSmBar),
                      reinterpret_cast<uint32_t*>(smem + kSmBar + 8), kTmemCols, st);
    const int t = threadIdx.x;
    if (t < n)
        closure_stage_row(smem + kSmA0, t, f, reinterpret_cast<const float*>(smem + kImgFMean),
                          reinterpret_cast<const float*>(smem + kImgFIstd));
    fence_async_smem();
    closure_mlp_run(smem + kSmImg, smem + kSmA0, smem + kSmH, st, 0, n);
    const bool ok = closure_mlp_teardown(st);   // its barrier publishes the outputs
    const float4 y = reinterpret_cast<const float4*>(smem + kSmA0)[t];
    const bool have = ok && t < n;
    out[0] = have ? y.x : 0.f;
    out[1] = have ? y.y : 0.f;
    out[2] = have ? y.z : 0.f;
    out[3] = have ? y.w : 0.f;
    return ok;
}

}  // namespace pnt
