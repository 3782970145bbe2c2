// closure_train.cuh -- the loss gradient of the closure network on the
// tensor cores (tcgen05, accumulators in TMEM), 128 training rows per CTA.
//
// Every contraction of one training step is a tcgen05.mma with BF16
// operands in shared memory (K-major canonical layout without swizzle, the
// layout of closure_dev.cuh: element (r, k) of an R-row operand at byte
// (k/8)*R*16 + r*16 + (k%8)*2) and FP32 accumulators in TMEM, M = 128 (the
// CTA's rows, one per thread and TMEM lane):
//
//   forward    D1 = X W1^T, H1 = gelu(D1 + b1);  D2 = H1 W2^T, H2 = gelu(..);
//              D3 = H2 W3^T, y = D3 + b3
//   backward   dY = 2 (y - t) / (rows * 4);  D4 = dY W3 -> dZ2 = D4 gelu'(Z2);
//              D5 = dZ2 W2 -> dZ1 = D5 gelu'(Z1)
//   weights    the contractions over the rows need the rows as K: the
//              epilogues also write transposed copies (dZ2^T and dZ1^T
//              stacked as one 128-row operand T1, H2^T as T2, H1^T, X^T,
//              dY^T), and   G1 = T1 H1^T  (rows 0-63: dW2),
//                           G2 = T1 X^T   (rows 64-127: dW1),
//                           G3 = T2 dY^T  (rows 0-63: dW3^T)
//
// The rounding points are those of the CPU oracle (closure_oracle.py
// loss_grad): inputs, hidden activations and backward deltas rounded to
// BF16 as MMA operands, products summed in FP32; bias gradients and the
// loss are FP32 sums of the unrounded values (warp shuffles in a fixed
// order, then the warps in order), so a gradient is bit-reproducible.
// Each CTA writes its partial gradient; closure_reduce_adam sums them.
//
// Every wait on an MMA commit is bounded; once one runs out no further MMA
// is issued, the partial is written as NaN, *err is set, and teardown
// waits (bounded) for the last commit before freeing the TMEM columns.
#pragma once

#include "closure_dev.cuh"

namespace pnt {
namespace train {

constexpr int kThreads = 128;
constexpr int kRows = 128;

// Training image in global memory (bf16 operands in the canonical layout;
// W1, W2, W3 at the offsets of the inference image).
constexpr int kImgW1 = 0;        // B [64 x 16]  (n = j, k = i)  W1[j][i], i < 14
constexpr int kImgW2 = 2048;     // B [64 x 64]  (n = j, k = i)  W2[j][i]
constexpr int kImgW3 = 10240;    // B [16 x 64]  (n = o, k = j)  W3[o][j], o < 4
constexpr int kImgW3T = 12288;   // B [64 x 16]  (n = j, k = o)  W3[o][j], o < 4
constexpr int kImgW2T = 14336;   // B [64 x 64]  (n = i, k = j)  W2[j][i]
constexpr int kImgB1 = 22528;    // f32 [64]
constexpr int kImgB2 = 22784;    // f32 [64]
constexpr int kImgB3 = 23040;    // f32 [16] (4 used)
constexpr int kImgBytes = 23104;

// Shared memory of the kernel.
constexpr int kSImg = 0;
constexpr int kSX = 23552;                 // A [128 x 16]   X
constexpr int kSH1 = kSX + 4096;           // A [128 x 64]   H1
constexpr int kSH2 = kSH1 + 16384;         // A [128 x 64]   H2
constexpr int kSDY = kSH2 + 16384;         // A [128 x 16]   dY (o < 4)
constexpr int kSDZ2 = kSDY + 4096;         // A [128 x 64]   dZ2
constexpr int kST1 = kSDZ2 + 16384;        // A [128 x 128]  rows 0-63 dZ2^T, 64-127 dZ1^T
constexpr int kST2 = kST1 + 32768;         // A [128 x 128]  rows 0-63 H2^T, 64-127 zero
constexpr int kSH1T = kST2 + 32768;        // B [64 x 128]   H1^T
constexpr int kSXT = kSH1T + 16384;        // B [16 x 128]   X^T
constexpr int kSDYT = kSXT + 4096;         // B [16 x 128]   dY^T (o < 4)
constexpr int kSBias = kSDYT + 4096;       // f32 [4 warps][132] bias gradient partials
constexpr int kSLoss = kSBias + 4 * 132 * 4;
constexpr int kSBar = kSLoss + 16;         // mbarrier (8 B) + TMEM address (4 B)
constexpr int kSmemBytes = kSBar + 16;
constexpr uint32_t kTmemCols = 512;
// TMEM columns of the accumulators
constexpr uint32_t kD1 = 0, kD2 = 64, kD3 = 128, kD4 = 160, kD5 = 224, kG1 = 288, kG2 = 352, kG3 = 384;

static_assert(kSX >= kImgBytes && kSX % 1024 == 0 && kSBar % 8 == 0, "layout");

struct Args {
    const uint8_t* img;
    const __nv_bfloat16* x;   // [n][16]
    const float* t;           // [n][4]
    int64_t n, first, rows;   // this step: rows (first + i) mod n, i < rows
    float inv_count;          // 1 / (rows * 4)
    float* partial;           // [gridDim.x][kClParams + 1]
    int* err;                 // set when a tensor-core wait ran out
};

// GELU and its derivative with the accurate tanh (training)
__device__ __forceinline__ void gelu_exact(float x, float& y, float& dy) {
    const float x2 = x * x;
    const float u = kGeluC * (x + kGeluA * x2 * x);
    const float th = tanhf(u);
    y = 0.5f * x * (1.f + th);
    dy = 0.5f * (1.f + th) + 0.5f * x * (1.f - th * th) * kGeluC * (1.f + 3.f * kGeluA * x2);
}

__device__ __forceinline__ uint32_t canon(int r, int k, int rows) { return (uint32_t)canon_off(r, k, rows); }
__device__ __forceinline__ void st_bf16(uint8_t* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

// This thread's row (t) of a K-major A operand [128 x K]: 8 values (one
// 16-byte chunk, k = 8c .. 8c+7).
__device__ __forceinline__ void st_row8(uint8_t* op, int t, int c, const float* v) {
    *reinterpret_cast<uint4*>(op + (c * 128 + t) * 16) =
        make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
}

// Column sums over the warp's 32 rows of 16 values, fixed xor tree; lane 0
// holds the sums.
__device__ __forceinline__ void warp_colsum16(float* v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
}

// MMA issue + bounded wait for its commit (thread 0 issues; every thread
// waits).  ok becomes false on every thread, and stays, once a wait ran out.
struct Tc {
    uint32_t sb, mbar, tbase, phase;
    bool ok;
    __device__ __forceinline__ void mma(uint32_t dcol, uint32_t a_off, int arows, uint32_t b_off, int brows,
                                        int ksteps, uint32_t acc0) const {
        for (int kb = 0; kb < ksteps; ++kb)
            umma_bf16(tbase + dcol, umma_desc(sb + a_off + kb * 32 * arows, arows * 16, 128),
                      umma_desc(sb + b_off + kb * 32 * brows, brows * 16, 128), umma_idesc_bf16(128, brows),
                      (kb > 0 || acc0) ? 1u : 0u);
    }
    // after a wait ran out nothing more is issued or committed, so the last
    // commit (phase - 1) is the one teardown drains
    __device__ __forceinline__ void commit_wait() {
        if (!ok) return;
        if (threadIdx.x == 0) umma_commit(mbar);
        ++phase;
        bool w = mbar_wait(mbar, (phase - 1) & 1);
        tc_fence_after();
        ok = __syncthreads_and(w && ok) != 0;
    }
    // barrier after the epilogue's operand writes, before the next MMA
    __device__ __forceinline__ void publish() const {
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    __device__ __forceinline__ uint32_t lane_addr(uint32_t col) const {
        return tbase + ((uint32_t)(32 * (threadIdx.x >> 5)) << 16) + col;
    }
};

__global__ void __launch_bounds__(kThreads, 1) grad_kernel(Args A) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    // ---- setup: image, this thread's row of X (and X^T), zero paddings
    for (int i = t; i < kImgBytes / 16; i += kThreads)
        reinterpret_cast<uint4*>(sm + kSImg)[i] = __ldg(reinterpret_cast<const uint4*>(A.img) + i);
    const int64_t idx = (int64_t)blockIdx.x * kRows + t;
    const bool live = idx < A.rows;
    const int64_t row = live ? (A.first + idx) % A.n : 0;
    {
        uint4 v0 = make_uint4(0u, 0u, 0u, 0u), v1 = v0;
        if (live) {
            v0 = __ldg(reinterpret_cast<const uint4*>(A.x + row * 16));
            v1 = __ldg(reinterpret_cast<const uint4*>(A.x + row * 16) + 1);
        }
        *reinterpret_cast<uint4*>(sm + kSX + (0 * 128 + t) * 16) = v0;
        *reinterpret_cast<uint4*>(sm + kSX + (1 * 128 + t) * 16) = v1;
        const __nv_bfloat16* xv0 = reinterpret_cast<const __nv_bfloat16*>(&v0);
        const __nv_bfloat16* xv1 = reinterpret_cast<const __nv_bfloat16*>(&v1);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            *reinterpret_cast<__nv_bfloat16*>(sm + kSXT + canon(i, t, 16)) = xv0[i];
            *reinterpret_cast<__nv_bfloat16*>(sm + kSXT + canon(8 + i, t, 16)) = xv1[i];
        }
    }
    for (int i = t; i < 64 * 128 * 2 / 16; i += kThreads)   // T2 rows 64-127 (k-chunks interleave rows)
        reinterpret_cast<uint4*>(sm + kST2)[(i / 64) * 128 + 64 + (i % 64)] = make_uint4(0u, 0u, 0u, 0u);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSBar + 8);
    Tc tc{(uint32_t)__cvta_generic_to_shared(sm), (uint32_t)__cvta_generic_to_shared(sm + kSBar), 0u, 0u, true};
    if (t == 0) mbar_init(tc.mbar, 1);
    if (w == 0) {
        tmem_alloc((uint32_t)__cvta_generic_to_shared(tslot), kTmemCols);
        tmem_relinquish();
    }
    tc.publish();
    tc.tbase = *tslot;
    const float* b1 = reinterpret_cast<const float*>(sm + kImgB1);
    const float* b2 = reinterpret_cast<const float*>(sm + kImgB2);
    const float* b3 = reinterpret_cast<const float*>(sm + kImgB3);
    float* bsum = reinterpret_cast<float*>(sm + kSBias) + w * 132;
    float loss = 0.f;

    // ---- layer 1
    if (t == 0) tc.mma(kD1, kSX, 128, kImgW1, 64, 1, 0);
    tc.commit_wait();
    if (tc.ok) {
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            float v[16], h[16];
            tmem_ld16(tc.lane_addr(kD1 + 16 * c), v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float d;
                gelu_exact(v[i] + b1[16 * c + i], h[i], d);
                st_bf16(sm + kSH1T, canon(16 * c + i, t, 64), h[i]);
            }
            st_row8(sm + kSH1, t, 2 * c, h);
            st_row8(sm + kSH1, t, 2 * c + 1, h + 8);
        }
    }
    tc.publish();
    // ---- layer 2
    if (t == 0 && tc.ok) tc.mma(kD2, kSH1, 128, kImgW2, 64, 4, 0);
    tc.commit_wait();
    if (tc.ok) {
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            float v[16], h[16];
            tmem_ld16(tc.lane_addr(kD2 + 16 * c), v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float d;
                gelu_exact(v[i] + b2[16 * c + i], h[i], d);
                st_bf16(sm + kST2, canon(16 * c + i, t, 128), h[i]);
            }
            st_row8(sm + kSH2, t, 2 * c, h);
            st_row8(sm + kSH2, t, 2 * c + 1, h + 8);
        }
    }
    tc.publish();
    // ---- layer 3, loss, dY
    if (t == 0 && tc.ok) tc.mma(kD3, kSH2, 128, kImgW3, 16, 4, 0);
    tc.commit_wait();
    float dy[16];
    for (int i = 0; i < 16; ++i) dy[i] = 0.f;
    if (tc.ok) {
        float v[4];
        tmem_ld4(tc.lane_addr(kD3), v);
        if (live) {
            const float4 tt = __ldg(reinterpret_cast<const float4*>(A.t + row * 4));
            const float tv[4] = {tt.x, tt.y, tt.z, tt.w};
#pragma unroll
            for (int o = 0; o < kClOut; ++o) {
                const float d = v[o] + b3[o] - tv[o];
                loss += d * d;
                dy[o] = 2.f * d * A.inv_count;
            }
        }
#pragma unroll
        for (int o = 0; o < 16; ++o) st_bf16(sm + kSDYT, canon(o, t, 16), dy[o]);
        st_row8(sm + kSDY, t, 0, dy);
        st_row8(sm + kSDY, t, 1, dy + 8);
    }
    {
        warp_colsum16(dy);   // the bias gradient of layer 3 (FP32, unrounded)
        if (lane == 0)
            for (int o = 0; o < 4; ++o) bsum[128 + o] = dy[o];
    }
    tc.publish();
    // ---- dZ2 = (dY W3) gelu'(Z2)
    if (t == 0 && tc.ok) tc.mma(kD4, kSDY, 128, kImgW3T, 64, 1, 0);
    tc.commit_wait();
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
        float dz[16];
        for (int i = 0; i < 16; ++i) dz[i] = 0.f;
        if (tc.ok) {
            float g[16], z[16];
            tmem_ld16(tc.lane_addr(kD4 + 16 * c), g);
            tmem_ld16(tc.lane_addr(kD2 + 16 * c), z);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float h, d;
                gelu_exact(z[i] + b2[16 * c + i], h, d);
                dz[i] = g[i] * d;
                st_bf16(sm + kST1, canon(16 * c + i, t, 128), dz[i]);
            }
            st_row8(sm + kSDZ2, t, 2 * c, dz);
            st_row8(sm + kSDZ2, t, 2 * c + 1, dz + 8);
        }
        warp_colsum16(dz);
        if (lane == 0)
            for (int i = 0; i < 16; ++i) bsum[64 + 16 * c + i] = dz[i];
    }
    tc.publish();
    // ---- dZ1 = (dZ2 W2) gelu'(Z1)
    if (t == 0 && tc.ok) tc.mma(kD5, kSDZ2, 128, kImgW2T, 64, 4, 0);
    tc.commit_wait();
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
        float dz[16];
        for (int i = 0; i < 16; ++i) dz[i] = 0.f;
        if (tc.ok) {
            float g[16], z[16];
            tmem_ld16(tc.lane_addr(kD5 + 16 * c), g);
            tmem_ld16(tc.lane_addr(kD1 + 16 * c), z);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float h, d;
                gelu_exact(z[i] + b1[16 * c + i], h, d);
                dz[i] = g[i] * d;
                st_bf16(sm + kST1, canon(64 + 16 * c + i, t, 128), dz[i]);
            }
        }
        warp_colsum16(dz);
        if (lane == 0)
            for (int i = 0; i < 16; ++i) bsum[16 * c + i] = dz[i];
    }
    // the loss: the warp's rows, then the warps in order below
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) reinterpret_cast<float*>(sm + kSLoss)[w] = loss;
    tc.publish();
    // ---- weight gradients: contractions over the CTA's 128 rows
    if (t == 0 && tc.ok) {
        tc.mma(kG1, kST1, 128, kSH1T, 64, 8, 0);
        tc.mma(kG2, kST1, 128, kSXT, 16, 8, 0);
        tc.mma(kG3, kST2, 128, kSDYT, 16, 8, 0);
    }
    tc.commit_wait();
    float* P = A.partial + (int64_t)blockIdx.x * (kClParams + 1);
    if (w < 2) {   // rows 0-63: dW2[j][.] and dW3[.][j], j = t
        for (int c = 0; c < 4; ++c) {
            float v[16];
            if (tc.ok) tmem_ld16(tc.lane_addr(kG1 + 16 * c), v);
            for (int i = 0; i < 16; ++i) P[kClW2 + t * 64 + 16 * c + i] = tc.ok ? v[i] : __int_as_float(0x7fc00000);
        }
        float v[4];
        if (tc.ok) tmem_ld4(tc.lane_addr(kG3), v);
        for (int o = 0; o < kClOut; ++o) P[kClW3 + o * 64 + t] = tc.ok ? v[o] : __int_as_float(0x7fc00000);
    } else {       // rows 64-127: dW1[j][.], j = t - 64
        float v[16];
        if (tc.ok) tmem_ld16(tc.lane_addr(kG2), v);
        for (int i = 0; i < kClIn; ++i) P[kClW1 + (t - 64) * kClIn + i] = tc.ok ? v[i] : __int_as_float(0x7fc00000);
    }
    // ---- biases (warps summed in order) and the loss
    const float* bs = reinterpret_cast<const float*>(sm + kSBias);
    for (int i = t; i < 132; i += kThreads) {
        if (i >= 128 + kClOut) continue;
        const float s = ((bs[i] + bs[132 + i]) + bs[264 + i]) + bs[396 + i];
        if (i < 64) P[kClB1 + i] = s;
        else if (i < 128) P[kClB2 + i - 64] = s;
        else P[kClB3 + i - 128] = s;
    }
    if (t == 0) {
        const float* ls = reinterpret_cast<const float*>(sm + kSLoss);
        P[kClParams] = tc.ok ? ((ls[0] + ls[1]) + ls[2]) + ls[3] : __int_as_float(0x7fc00000);
        if (!tc.ok) atomicOr(A.err, 1);
    }
    // ---- teardown: after a wait ran out, the last commit must land first
    tc_fence_before();
    __syncthreads();
    if (!tc.ok && tc.phase > 0) {
        mbar_wait(tc.mbar, (tc.phase - 1) & 1);
        __syncthreads();
    }
    if (w == 0) {
        tc_fence_after();
        tmem_dealloc(tc.tbase, kTmemCols);
    }
}

}  // namespace train
}  // namespace pnt
