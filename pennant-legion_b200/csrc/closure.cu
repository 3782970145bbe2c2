// closure.cu -- the learned QCS closure: training data harvested from the
// FP64 cycle, the network's training kernels, its standalone tcgen05
// inference, and the pnt_closure object (C ABI in include/pennant_b200.h).
//
// Harvest: for every corner that compresses (cdiv < 0), lies outside the
// dead zone and belongs to a zone without an acute corner, the 14 inputs
// of closure_dev.cuh and the 4 normalised outputs of the exact FP64 QCS
// (QCS.cc:116-327) on the state at the start of a cycle, sub-sampled by a
// hash of (seed, cycle, side) and compacted in a deterministic order.
//
// Training: the loss gradient of 128 rows per CTA on the tensor cores
// (closure_train.cuh: tcgen05.mma with BF16 operands in shared memory and
// FP32 accumulators in TMEM, forward, backward and the weight gradients as
// contractions over the CTA's rows); per-CTA partial gradients are summed
// in a fixed order and applied with Adam, so a run is deterministic.  The
// inference in the hydro cycle uses the tcgen05 block of closure_dev.cuh on
// the same parameters.
//
// Compiled with -fmad=false: the harvested targets repeat the FP64
// cycle's QCS arithmetic.
#include "closure_dev.cuh"
#include "closure_train.cuh"
#include "hydro_fp64_body.cuh"
#include "pnt_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

using namespace pnt;

namespace pnt {
namespace {

using namespace fp64;

// ----------------------------------------------------------------------
// Harvest (FP64, the arithmetic of pass A, four lanes per zone)
// ----------------------------------------------------------------------
struct HarvestArgs {
    double dead, qa, qb;
    uint32_t keep;      // keep a corner when its hash < keep (keep_all: every corner)
    int32_t keep_all;
    uint64_t seed;
    int32_t* counts;         // [blocks]
    const int64_t* offsets;  // [blocks] first record of each block
    float* feats;            // [capacity][14]
    float* targs;            // [capacity][4]
    int32_t* sides;          // [capacity]
    int64_t capacity;
};

__device__ __forceinline__ uint32_t corner_hash(uint64_t seed, int cycle, int64_t s) {
    uint64_t x = seed ^ ((uint64_t)(uint32_t)cycle * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)s * 0xD1B54A32D192ED03ull);
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (uint32_t)(x >> 32);
}

template <bool kWrite>
__global__ void __launch_bounds__(kZoneThreads) harvest_kernel(DevArrays a, HydroConst c, HarvestArgs h) {
    const Ctl* ctl = a.ctl;
    const bool run = !skip_cycle(ctl);
    const int cur = run ? (ctl->cycle & 1) : 0;
    const double dt = run ? ctl->dt : 0.;
    const int64_t tid = (int64_t)blockIdx.x * kZoneThreads + threadIdx.x;
    const int64_t z = tid >> 2;
    const int k = (int)(tid & 3);
    const int lane = threadIdx.x & 31;
    const int g = lane & ~3;
    const bool zok = run && z < a.numz;
    const int n = zok ? a.znump[z] : 4;
    const int64_t s = (zok ? (int64_t)a.zfirst[z] : 0) + k;
    const bool act = zok && k < n;
    const int lp = g + (k == 0 ? n - 1 : k - 1);
    const int ln = g + (k + 1 >= n ? 0 : k + 1);

    const int32_t p1 = act ? __ldg(a.mapsp1 + s) : 0;
    const double2 x0 = act ? a.px[cur][p1] : mk(0., 0.);
    const double2 u0 = act ? a.pu[cur][p1] : mk(0., 0.);
    const double zm = zok ? a.zm[z] : 1.;
    const double zr = zok ? a.zr[z] : 1.;
    const double ze = zok ? a.ze[z] : 0.;

    const double dth = 0.5 * dt;
    const double2 xp = add(x0, smul(dth, u0));
    const double2 xp2 = shfl2(xp, ln);
    const double2 xpp = shfl2(xp, lp);
    const double2 u02 = shfl2(u0, ln);
    const double rn = 1. / (double)n;
    const double2 zxp = zsum2(mk(xp.x * rn, xp.y * rn), g, n);
    const double third = 1. / 3.;
    const double sa = 0.5 * cross(sub(xp2, xp), sub(zxp, xp));
    const double sv = third * sa * (xp.x + xp2.x + zxp.x);
    const double zvolp = zsum(sv, g, n);
    const double e = dmax(ze, 0.);
    const double p = c.gm1 * zr * e;
    const double pre = c.gm1 * e;
    const double per = c.gm1 * zr;
    const double rA = ((k == 0) ? per * p : 1.) / ((k == 0) ? zr * zr : zm);
    const double q = shfl(rA, g);
    const double minv = shfl(rA, g + 1);
    const double csqd = dmax(c.ssmin2, pre + q);
    const double zss = sqrt(csqd);
    const double rB = ((k == 0) ? zm : 1.) / ((k == 0) ? zvolp : 1.);
    const double zrp = shfl(rB, g);
    (void)minv;

    // QCS corner (the FP64 cycle's arithmetic)
    const double2 zuc = zsum2(mk(u0.x * rn, u0.y * rn), g, n);
    const double2 ex = smul(0.5, add(xp, xp2));
    const double2 up0 = u0, xq0 = xp;
    const double2 upp = shfl2(u0, lp);
    const double2 up1 = smul(0.5, add(up0, u02));
    const double2 xq1 = ex;
    const double2 up2 = zuc, xq2 = zxp;
    const double2 up3 = smul(0.5, add(upp, up0));
    const double2 xq3 = shfl2(ex, lp);
    const double cvolume = 0.5 * cross(sub(xq2, xq0), sub(xq3, xq1));
    const double2 v1 = sub(xq3, xq0);
    const double2 v2 = sub(xq1, xq0);
    const double elen = length(sub(xp2, xp));
    const double rinv_el = 1. / elen;
    const double de1 = shfl(elen, lp);
    const double rinv_de1 = shfl(rinv_el, lp);
    const double de2 = elen;
    const double minelen = dmin(de1, de2);
    const double cdiv = (cross(sub(up2, up0), sub(xq3, xq1)) - cross(sub(up3, up1), sub(xq2, xq0))) /
                        (2.0 * cvolume);
    double crmu = 0.;
    if (act && cdiv < 0.0) {
        const double2 dxx1 = smul(0.5, sub(sub(add(xq1, xq2), xq0), xq3));
        const double2 dxx2 = smul(0.5, sub(sub(add(xq2, xq3), xq0), xq1));
        const double dx1 = length(dxx1);
        const double dx2 = length(dxx2);
        const double2 duav = smul(0.25, add(add(add(up0, up1), up2), up3));
        const double test1 = fabs(dot(dxx1, duav) * dx2);
        const double test2 = fabs(dot(dxx2, duav) * dx1);
        const double num = (test1 > test2 ? dx1 : dx2);
        const double den = (test1 > test2 ? dx2 : dx1);
        double evol = sqrt(4.0 * cvolume * (num / den));
        evol = dmin(evol, 2.0 * minelen);
        const double du = sqrt(dmax(length2(sub(sub(add(up1, up2), up0), up3)), length2(sub(sub(add(up2, up3), up0), up1))));
        const double ztmp2 = c.q2 * 0.25 * c.gammap1 * du;
        const double ztmp1 = c.q1 * zss;
        const double zkur = ztmp2 + sqrt(ztmp2 * ztmp2 + ztmp1 * ztmp1);
        crmu = zkur * zrp * evol;
    }
    const double2 t1 = smul(crmu, sub(up0, upp));
    const double2 cqe1 = mk(t1.x * rinv_de1, t1.y * rinv_de1);
    const double2 t2 = smul(crmu, sub(u02, up0));
    const double2 cqe2 = mk(t2.x * rinv_el, t2.y * rinv_el);
    // zones with an acute corner keep the plain QCS in the learned cycle
    const double ssin = 4. * cross(v1, v2) / (de1 * de2);
    int acute = (act && ssin * ssin < 0.25) ? 1 : 0;
    acute |= __shfl_xor_sync(kFull, acute, 1);
    acute |= __shfl_xor_sync(kFull, acute, 2);

    bool keep = false;
    float f[kClIn], tg[4];
    if (act && cdiv < 0.0 && !acute && (h.keep_all || corner_hash(h.seed, ctl->cycle, s) < h.keep)) {
        const double2 duav = smul(0.25, add(add(add(up0, up1), up2), up3));
        double cx, cy, scale;
        keep = closure_features<double>({xp.x, xp.y}, {xpp.x, xpp.y}, {xp2.x, xp2.y}, {zxp.x, zxp.y}, {up0.x, up0.y},
                                        {upp.x, upp.y}, {u02.x, u02.y}, {zuc.x, zuc.y}, {duav.x, duav.y}, zss, h.qa,
                                        h.qb, h.dead, f, cx, cy, scale);
        if (keep) {
            const double inv = 1. / (zrp * scale);
            tg[0] = (float)((cx * cqe1.x + cy * cqe1.y) * inv);
            tg[1] = (float)((cx * cqe1.y - cy * cqe1.x) * inv);
            tg[2] = (float)((cx * cqe2.x + cy * cqe2.y) * inv);
            tg[3] = (float)((cx * cqe2.y - cy * cqe2.x) * inv);
        }
    }
    if (!kWrite) {
        const int cnt = __syncthreads_count(keep);
        if (threadIdx.x == 0) h.counts[blockIdx.x] = cnt;
        return;
    }
    __shared__ int wsum[kZoneThreads / 32];
    const unsigned m = __ballot_sync(kFull, keep);
    const int warp = threadIdx.x >> 5;
    if (lane == 0) wsum[warp] = __popc(m);
    __syncthreads();
    int before = 0;
    for (int i = 0; i < warp; ++i) before += wsum[i];
    const int64_t idx = h.offsets[blockIdx.x] + before + __popc(m & ((1u << lane) - 1u));
    if (keep && idx < h.capacity) {
        for (int i = 0; i < kClIn; ++i) h.feats[idx * kClIn + i] = f[i];
        for (int i = 0; i < 4; ++i) h.targs[idx * 4 + i] = tg[i];
        h.sides[idx] = (int32_t)s;
    }
}

// Exclusive scan of the block counts (one block, contiguous segments per
// thread), starting at base; total = base + sum.
__global__ void __launch_bounds__(1024) scan_counts(const int32_t* counts, int nb, int64_t base, int64_t* offsets,
                                                    int64_t* total) {
    __shared__ int64_t ws[32];
    const int t = threadIdx.x;
    const int seg = (nb + 1023) / 1024;
    const int b0 = min(nb, t * seg), b1 = min(nb, b0 + seg);
    int64_t local = 0;
    for (int b = b0; b < b1; ++b) local += counts[b];
    // inclusive scan over the block
    int64_t v = local;
    const int lane = t & 31, w = t >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        int64_t x = ws[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        ws[lane] = x;
    }
    __syncthreads();
    int64_t run = base + v - local + (w > 0 ? ws[w - 1] : 0);
    for (int b = b0; b < b1; ++b) {
        offsets[b] = run;
        run += counts[b];
    }
    if (t == 1023) *total = run;
}

// ----------------------------------------------------------------------
// Normalisation and data preparation
// ----------------------------------------------------------------------
constexpr int kNormCols = kClIn + kClOut;   // 18

__global__ void __launch_bounds__(256) norm_partials(const float* feats, const float* targs, int64_t n, double* out) {
    __shared__ double red[256];
    double s[kNormCols], q[kNormCols];
    for (int i = 0; i < kNormCols; ++i) s[i] = q[i] = 0.;
    for (int64_t r = (int64_t)blockIdx.x * 256 + threadIdx.x; r < n; r += (int64_t)gridDim.x * 256) {
        for (int i = 0; i < kNormCols; ++i) {
            const double v = (i < kClIn) ? feats[r * kClIn + i] : targs[r * 4 + (i - kClIn)];
            s[i] += v;
            q[i] += v * v;
        }
    }
    for (int i = 0; i < 2 * kNormCols; ++i) {
        red[threadIdx.x] = (i < kNormCols) ? s[i] : q[i - kNormCols];
        __syncthreads();
        for (int o = 128; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[blockIdx.x * 2 * kNormCols + i] = red[0];
        __syncthreads();
    }
}

struct Norm {
    float fmean[16], fistd[16], tmean[4], tstd[4];
};

__global__ void prepare_kernel(const float* feats, const float* targs, int64_t n, Norm nm, __nv_bfloat16* x,
                               float* t) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    uint32_t w[8];
    for (int i = 0; i < 8; ++i) {
        const float a = (2 * i < kClIn) ? (feats[r * kClIn + 2 * i] - nm.fmean[2 * i]) * nm.fistd[2 * i] : 0.f;
        const float b = (2 * i + 1 < kClIn) ? (feats[r * kClIn + 2 * i + 1] - nm.fmean[2 * i + 1]) * nm.fistd[2 * i + 1] : 0.f;
        w[i] = pack_bf16(a, b);
    }
    uint4* xo = reinterpret_cast<uint4*>(x + r * 16);
    xo[0] = make_uint4(w[0], w[1], w[2], w[3]);
    xo[1] = make_uint4(w[4], w[5], w[6], w[7]);
    for (int i = 0; i < 4; ++i) t[r * 4 + i] = (targs[r * 4 + i] - nm.tmean[i]) / nm.tstd[i];
}

// ----------------------------------------------------------------------
// Parameter images
// ----------------------------------------------------------------------
// The training image is train::kImg* (closure_train.cuh): the inference
// operands W1, W2, W3 in the same canonical layout, the transposed W3^T and
// W2^T the backward pass multiplies by, and the biases.
__device__ __forceinline__ void put_bf16(uint8_t* img, int off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(img + off) = __float2bfloat16_rn(v);
}

__global__ void pack_images(const float* P, Norm nm, float thr0, float thr1, float thr2, uint8_t* inf, uint8_t* tr) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 8192; e += gridDim.x * blockDim.x) {
        // W1, W2 and W2^T: (j, i) over 64 x 64
        if (e < 4096) {
            const int j = e >> 6, i = e & 63;
            const float w2 = P[kClW2 + j * 64 + i];
            put_bf16(inf, kImgW2 + canon_off(j, i, 64), w2);
            put_bf16(tr, train::kImgW2 + canon_off(j, i, 64), w2);
            put_bf16(tr, train::kImgW2T + canon_off(i, j, 64), w2);
            if (i < 16) {
                const float w1 = (i < kClIn) ? P[kClW1 + j * kClIn + i] : 0.f;
                put_bf16(inf, kImgW1 + canon_off(j, i, 64), w1);
                put_bf16(tr, train::kImgW1 + canon_off(j, i, 64), w1);
            }
        } else {
            // W3 (o, j) over 16 x 64 (rows o >= 4 zero) and W3^T (j, o)
            const int r = e - 4096;
            const int o = r >> 6, j = r & 63;   // o 0..63
            if (o < 16) {
                const float w3 = (o < kClOut) ? P[kClW3 + o * 64 + j] : 0.f;
                put_bf16(inf, kImgW3 + canon_off(o, j, 16), w3);
                put_bf16(tr, train::kImgW3 + canon_off(o, j, 16), w3);
                put_bf16(tr, train::kImgW3T + canon_off(j, o, 64), w3);
            }
        }
        if (e < 64) {
            reinterpret_cast<float*>(inf + kImgB1)[e] = P[kClB1 + e];
            reinterpret_cast<float*>(inf + kImgB2)[e] = P[kClB2 + e];
            reinterpret_cast<float*>(tr + train::kImgB1)[e] = P[kClB1 + e];
            reinterpret_cast<float*>(tr + train::kImgB2)[e] = P[kClB2 + e];
        }
        if (e < 16) {
            reinterpret_cast<float*>(inf + kImgB3)[e] = (e < kClOut) ? P[kClB3 + e] : 0.f;
            reinterpret_cast<float*>(tr + train::kImgB3)[e] = (e < kClOut) ? P[kClB3 + e] : 0.f;
            reinterpret_cast<float*>(inf + kImgFMean)[e] = nm.fmean[e];
            reinterpret_cast<float*>(inf + kImgFIstd)[e] = nm.fistd[e];
        }
        if (e < 4) {
            reinterpret_cast<float*>(inf + kImgTMean)[e] = nm.tmean[e];
            reinterpret_cast<float*>(inf + kImgTStd)[e] = nm.tstd[e];
            reinterpret_cast<float*>(inf + kImgThr)[e] = (e == 0) ? thr0 : (e == 1) ? thr1 : (e == 2) ? thr2 : 0.f;
        }
    }
}

// Sum of the per-CTA partials (fixed order); Adam step when `apply`.
__global__ void closure_reduce_adam(float* params, float* m, float* v, const float* partial, int nparts, float lr,
                                    float bc1, float bc2, float inv_count, int apply, float* grad_out, float* loss_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > kClParams) return;
    float s = 0.f;
    for (int b = 0; b < nparts; ++b) s += partial[(int64_t)b * (kClParams + 1) + p];
    if (p == kClParams) {
        *loss_out = s * inv_count;
        return;
    }
    if (grad_out) grad_out[p] = s;
    if (!apply) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float mm = b1 * m[p] + (1.f - b1) * s;
    const float vv = b2 * v[p] + (1.f - b2) * s * s;
    m[p] = mm;
    v[p] = vv;
    params[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

// ----------------------------------------------------------------------
// Standalone inference (tcgen05): 256 rows per CTA.  The CTA takes more
// shared memory than the block uses (one CTA per SM either way), so every
// operand read of the tensor cores stays inside the allocation whatever the
// descriptors' strides.
// ----------------------------------------------------------------------
constexpr int kForwardSmem = 160 * 1024;
__global__ void __launch_bounds__(kMlpRows, 1) closure_forward_kernel(const uint8_t* img, const float* feats, int64_t n,
                                                                     float* out, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int64_t r = (int64_t)blockIdx.x * kMlpRows + threadIdx.x;
    float f[kClIn];
    for (int i = 0; i < kClIn; ++i) f[i] = (r < n) ? feats[r * kClIn + i] : 0.f;
    float y[4];
    const int64_t left = n - (int64_t)blockIdx.x * kMlpRows;
    const bool ok = closure_mlp_block(smem, img, f, left < kMlpRows ? (int)left : kMlpRows, y);
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    if (r < n)
        for (int i = 0; i < 4; ++i) out[r * 4 + i] = y[i];
}

// The bounded wait of the tensor-core kernels on its own: one mbarrier of
// arrival count 1 that this thread completes first (arrive = 1) or that
// nothing completes (arrive = 0).  The wait ends either way, after at most
// `limit` polls; *timed_out records which.  No tensor-core work is in
// flight, so giving up leaves nothing behind.
__global__ void __launch_bounds__(32, 1) bounded_wait_probe(int arrive, int limit, int* timed_out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    const uint32_t mbar = smem_addr(&bar);
    mbar_init(mbar, 1);
    if (arrive) mbar_arrive(mbar);
    *timed_out = mbar_wait(mbar, 0, limit) ? 0 : 1;
}

}  // namespace
}  // namespace pnt

// ----------------------------------------------------------------------
// Host side
// ----------------------------------------------------------------------
namespace {

#define CUDA_TRY(expr)                                                                                          \
    do {                                                                                                        \
        const cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess)                                                                                  \
            return fail(PNT_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__);     \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int now = -1;
        if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
    }
};

constexpr uint32_t kFileMagic = 0x31435150u;   // "PQC1"

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

struct pnt_closure {
    int device = 0;
    std::vector<float> params = std::vector<float>(kClParams, 0.f);
    float fmean[kClIn] = {}, fstd[kClIn] = {}, tmean[kClOut] = {}, tstd[kClOut] = {};
    float thr[3] = {1e-6f, 0.5f, 6.f};   // dead zone, rho_max, ood_kappa
    float* d_params = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    uint8_t* d_img = nullptr;
    uint8_t* d_trimg = nullptr;
    float* d_partial = nullptr;
    int partial_cap = 0;
    float* d_loss = nullptr;     // [2]: loss, error flag
    float* d_grad = nullptr;
    int* d_err = nullptr;        // set by a training step whose tensor-core wait ran out
    int64_t adam_t = 0;
    cudaStream_t stream = nullptr;

    ~pnt_closure() {
        DeviceGuard dg(device);
        for (void* p : {(void*)d_params, (void*)d_m, (void*)d_v, (void*)d_img, (void*)d_trimg, (void*)d_partial,
                        (void*)d_loss, (void*)d_grad, (void*)d_err})
            if (p) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }

    pnt::Norm norm() const {
        pnt::Norm n{};
        for (int i = 0; i < kClIn; ++i) {
            n.fmean[i] = fmean[i];
            n.fistd[i] = 1.f / fstd[i];
        }
        for (int i = 0; i < kClOut; ++i) {
            n.tmean[i] = tmean[i];
            n.tstd[i] = tstd[i];
        }
        return n;
    }

    pnt_status setup() {
        CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaMalloc(&d_params, kClParams * sizeof(float)));
        CUDA_TRY(cudaMalloc(&d_m, kClParams * sizeof(float)));
        CUDA_TRY(cudaMalloc(&d_v, kClParams * sizeof(float)));
        CUDA_TRY(cudaMalloc(&d_img, kImgBytes));
        CUDA_TRY(cudaMalloc(&d_trimg, train::kImgBytes));
        CUDA_TRY(cudaMalloc(&d_err, sizeof(int)));
        CUDA_TRY(cudaMemset(d_err, 0, sizeof(int)));
        CUDA_TRY(cudaMalloc(&d_loss, 16));
        CUDA_TRY(cudaMalloc(&d_grad, kClParams * sizeof(float)));
        CUDA_TRY(cudaMemset(d_img, 0, kImgBytes));
        CUDA_TRY(cudaMemset(d_trimg, 0, train::kImgBytes));
        CUDA_TRY(cudaMemset(d_m, 0, kClParams * sizeof(float)));
        CUDA_TRY(cudaMemset(d_v, 0, kClParams * sizeof(float)));
        static bool attr_done[64] = {};
        if (device < 64 && !attr_done[device]) {
            CUDA_TRY(cudaFuncSetAttribute(train::grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          train::kSmemBytes));
            CUDA_TRY(cudaFuncSetAttribute(closure_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kForwardSmem));
            attr_done[device] = true;
        }
        return upload();
    }

    // host params/normalisation -> device master copy and both images
    pnt_status upload() {
        CUDA_TRY(cudaMemcpyAsync(d_params, params.data(), kClParams * sizeof(float), cudaMemcpyHostToDevice, stream));
        return repack();
    }
    pnt_status repack() {
        pack_images<<<32, 256, 0, stream>>>(d_params, norm(), thr[0], thr[1], thr[2], d_img, d_trimg);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamSynchronize(stream));
        return PNT_OK;
    }
    // a training step's tensor-core wait that ran out (the flag is cleared)
    pnt_status check_err() {
        int e = 0;
        CUDA_TRY(cudaMemcpyAsync(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        if (!e) return PNT_OK;
        CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
        return fail(PNT_ERR_TIMEOUT, "a tensor-core wait of the training kernel ran out");
    }
    pnt_status download() {
        CUDA_TRY(cudaMemcpyAsync(params.data(), d_params, kClParams * sizeof(float), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return PNT_OK;
    }
    pnt_status ensure_partial(int nparts) {
        if (nparts <= partial_cap) return PNT_OK;
        if (d_partial) cudaFree(d_partial);
        d_partial = nullptr;
        partial_cap = 0;
        CUDA_TRY(cudaMalloc(&d_partial, (size_t)nparts * (kClParams + 1) * sizeof(float)));
        partial_cap = nparts;
        return PNT_OK;
    }
    // One gradient pass over rows (first + i) mod n, i < rows; Adam step when apply.
    pnt_status step(const void* x, const float* t, int64_t n, int64_t first, int64_t rows, float lr, bool apply,
                    float* grad_host, float* loss_host) {
        const int nparts = (int)((rows + train::kRows - 1) / train::kRows);
        pnt_status st = ensure_partial(nparts);
        if (st) return st;
        train::Args A{d_trimg, static_cast<const __nv_bfloat16*>(x), t, n, first, rows, 1.f / (float)(rows * 4),
                      d_partial, d_err};
        train::grad_kernel<<<nparts, train::kThreads, train::kSmemBytes, stream>>>(A);
        CUDA_TRY(cudaGetLastError());
        float bc1 = 1.f, bc2 = 1.f;
        if (apply) {
            ++adam_t;
            bc1 = 1.f - powf(0.9f, (float)adam_t);
            bc2 = 1.f - powf(0.999f, (float)adam_t);
        }
        closure_reduce_adam<<<(kClParams + 1 + 255) / 256, 256, 0, stream>>>(
            d_params, d_m, d_v, d_partial, nparts, lr, bc1, bc2, A.inv_count, apply ? 1 : 0,
            grad_host ? d_grad : nullptr, d_loss);
        CUDA_TRY(cudaGetLastError());
        if (apply) {
            pack_images<<<32, 256, 0, stream>>>(d_params, norm(), thr[0], thr[1], thr[2], d_img, d_trimg);
            CUDA_TRY(cudaGetLastError());
        }
        if (grad_host)
            CUDA_TRY(cudaMemcpyAsync(grad_host, d_grad, kClParams * sizeof(float), cudaMemcpyDeviceToHost, stream));
        if (loss_host) CUDA_TRY(cudaMemcpyAsync(loss_host, d_loss, sizeof(float), cudaMemcpyDeviceToHost, stream));
        if (grad_host || loss_host) CUDA_TRY(cudaStreamSynchronize(stream));
        return PNT_OK;
    }
};

namespace pnt {
const uint8_t* closure_image(const pnt_closure* c) { return c->d_img; }
int closure_device(const pnt_closure* c) { return c->device; }
}  // namespace pnt

extern "C" {

pnt_status pnt_closure_create(int32_t device, uint64_t seed, pnt_closure** out) {
    if (!out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(PNT_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(PNT_ERR_INVALID_ARG, "device %d out of range", device);
    DeviceGuard dg(device);
    pnt_closure* c = new (std::nothrow) pnt_closure();
    if (!c) return fail(PNT_ERR_NOMEM, "out of memory");
    c->device = device;
    // Glorot-uniform weights, zero biases, identity normalisation
    uint64_t s = seed;
    auto uni = [&](float lim) { return (float)(((double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0)) * 2. - 1.) * lim; };
    const float l1 = sqrtf(6.f / (kClIn + kClHid)), l2 = sqrtf(6.f / (kClHid + kClHid)), l3 = sqrtf(6.f / (kClHid + kClOut));
    for (int i = 0; i < kClHid * kClIn; ++i) c->params[kClW1 + i] = uni(l1);
    for (int i = 0; i < kClHid * kClHid; ++i) c->params[kClW2 + i] = uni(l2);
    for (int i = 0; i < kClOut * kClHid; ++i) c->params[kClW3 + i] = uni(l3);
    for (int i = 0; i < kClIn; ++i) c->fstd[i] = 1.f;
    for (int i = 0; i < kClOut; ++i) c->tstd[i] = 1.f;
    pnt_status st = c->setup();
    if (st) {
        delete c;
        return st;
    }
    *out = c;
    return PNT_OK;
}

void pnt_closure_destroy(pnt_closure* c) { delete c; }

pnt_status pnt_closure_get(const pnt_closure* c, float* params, float* norm, float* thresholds) {
    if (!c) return fail(PNT_ERR_INVALID_ARG, "null closure");
    if (params) std::memcpy(params, c->params.data(), kClParams * sizeof(float));
    if (norm) {
        std::memcpy(norm, c->fmean, sizeof(c->fmean));
        std::memcpy(norm + kClIn, c->fstd, sizeof(c->fstd));
        std::memcpy(norm + 2 * kClIn, c->tmean, sizeof(c->tmean));
        std::memcpy(norm + 2 * kClIn + kClOut, c->tstd, sizeof(c->tstd));
    }
    if (thresholds) std::memcpy(thresholds, c->thr, sizeof(c->thr));
    return PNT_OK;
}

pnt_status pnt_closure_set(pnt_closure* c, const float* params, const float* norm, const float* thresholds) {
    if (!c) return fail(PNT_ERR_INVALID_ARG, "null closure");
    if (norm) {
        for (int i = 0; i < kClIn; ++i)
            if (!(norm[kClIn + i] > 0.f)) return fail(PNT_ERR_INVALID_ARG, "input std %d must be > 0", i);
        for (int i = 0; i < kClOut; ++i)
            if (!(norm[2 * kClIn + kClOut + i] > 0.f)) return fail(PNT_ERR_INVALID_ARG, "output std %d must be > 0", i);
    }
    DeviceGuard dg(c->device);
    if (params) std::memcpy(c->params.data(), params, kClParams * sizeof(float));
    if (norm) {
        std::memcpy(c->fmean, norm, sizeof(c->fmean));
        std::memcpy(c->fstd, norm + kClIn, sizeof(c->fstd));
        std::memcpy(c->tmean, norm + 2 * kClIn, sizeof(c->tmean));
        std::memcpy(c->tstd, norm + 2 * kClIn + kClOut, sizeof(c->tstd));
    }
    if (thresholds) std::memcpy(c->thr, thresholds, sizeof(c->thr));
    if (params) {
        c->adam_t = 0;
        cudaMemsetAsync(c->d_m, 0, kClParams * sizeof(float), c->stream);
        cudaMemsetAsync(c->d_v, 0, kClParams * sizeof(float), c->stream);
    }
    return c->upload();
}

pnt_status pnt_closure_save(const pnt_closure* c, const char* path) {
    if (!c || !path) return fail(PNT_ERR_INVALID_ARG, "null argument");
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(PNT_ERR_INVALID_ARG, "cannot write %s", path);
    const uint32_t hdr[4] = {kFileMagic, (uint32_t)kClParams, (uint32_t)kClIn, (uint32_t)kClOut};
    bool ok = std::fwrite(hdr, sizeof(hdr), 1, fp) == 1;
    ok = ok && std::fwrite(c->params.data(), sizeof(float), kClParams, fp) == (size_t)kClParams;
    ok = ok && std::fwrite(c->fmean, sizeof(c->fmean), 1, fp) == 1 && std::fwrite(c->fstd, sizeof(c->fstd), 1, fp) == 1;
    ok = ok && std::fwrite(c->tmean, sizeof(c->tmean), 1, fp) == 1 && std::fwrite(c->tstd, sizeof(c->tstd), 1, fp) == 1;
    ok = ok && std::fwrite(c->thr, sizeof(c->thr), 1, fp) == 1;
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? PNT_OK : fail(PNT_ERR_INVALID_ARG, "short write to %s", path);
}

pnt_status pnt_closure_load(const char* path, int32_t device, pnt_closure** out) {
    if (!path || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return fail(PNT_ERR_INVALID_ARG, "cannot open %s", path);
    uint32_t hdr[4] = {};
    std::vector<float> p(kClParams);
    float norm[2 * kClIn + 2 * kClOut], thr[3];
    bool ok = std::fread(hdr, sizeof(hdr), 1, fp) == 1 && hdr[0] == kFileMagic && hdr[1] == (uint32_t)kClParams &&
              hdr[2] == (uint32_t)kClIn && hdr[3] == (uint32_t)kClOut;
    ok = ok && std::fread(p.data(), sizeof(float), kClParams, fp) == (size_t)kClParams;
    ok = ok && std::fread(norm, sizeof(norm), 1, fp) == 1 && std::fread(thr, sizeof(thr), 1, fp) == 1;
    std::fclose(fp);
    if (!ok) return fail(PNT_ERR_INVALID_ARG, "%s is not a closure file of this network", path);
    pnt_closure* c = nullptr;
    pnt_status st = pnt_closure_create(device, 0, &c);
    if (st) return st;
    st = pnt_closure_set(c, p.data(), norm, thr);
    if (st) {
        delete c;
        return st;
    }
    *out = c;
    return PNT_OK;
}

pnt_status pnt_closure_fit_normalization(pnt_closure* c, const float* feats, const float* targets, int64_t n) {
    if (!c || !feats || !targets || n < 2) return fail(PNT_ERR_INVALID_ARG, "need at least 2 samples");
    DeviceGuard dg(c->device);
    const int nb = 256;
    double* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, nb * 2 * kNormCols * sizeof(double)));
    norm_partials<<<nb, 256, 0, c->stream>>>(feats, targets, n, d);
    std::vector<double> h(nb * 2 * kNormCols);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "normalisation: %s", cudaGetErrorString(e));
    for (int i = 0; i < kNormCols; ++i) {
        double s = 0., q = 0.;
        for (int b = 0; b < nb; ++b) {
            s += h[b * 2 * kNormCols + i];
            q += h[b * 2 * kNormCols + kNormCols + i];
        }
        const double mean = s / (double)n;
        const double sd = std::max(std::sqrt(std::max(q / (double)n - mean * mean, 0.)), 1e-6);
        if (i < kClIn) {
            c->fmean[i] = (float)mean;
            c->fstd[i] = (float)sd;
        } else {
            c->tmean[i - kClIn] = (float)mean;
            c->tstd[i - kClIn] = (float)sd;
        }
    }
    return c->repack();
}

pnt_status pnt_closure_prepare(const pnt_closure* c, const float* feats, const float* targets, int64_t n, void* x,
                               float* t) {
    if (!c || !feats || !targets || !x || !t || n < 0) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return PNT_OK;
    DeviceGuard dg(c->device);
    prepare_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(feats, targets, n, c->norm(),
                                                                       static_cast<__nv_bfloat16*>(x), t);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PNT_OK;
}

pnt_status pnt_closure_train(pnt_closure* c, const void* x, const float* t, int64_t n, int64_t first, int32_t steps,
                             int32_t rows_per_step, float lr, float* losses) {
    if (!c || !x || !t || n <= 0 || first < 0 || steps < 0 || rows_per_step <= 0 || !(lr > 0.f))
        return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(c->device);
    for (int s = 0; s < steps; ++s) {
        const int64_t f0 = (first + (int64_t)s * rows_per_step) % n;
        pnt_status st = c->step(x, t, n, f0, rows_per_step, lr, true, nullptr, losses ? losses + s : nullptr);
        if (st) return st;
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (pnt_status st = c->check_err()) return st;
    return c->download();
}

pnt_status pnt_closure_gradient(pnt_closure* c, const void* x, const float* t, int64_t n, float* grad, float* loss) {
    if (!c || !x || !t || n <= 0 || !grad) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(c->device);
    float l = 0.f;
    pnt_status st = c->step(x, t, n, 0, n, 0.f, false, grad, &l);
    if (st) return st;
    if ((st = c->check_err())) return st;
    if (loss) *loss = l;
    return PNT_OK;
}

pnt_status pnt_closure_wait_probe(int32_t device, int32_t arrive, int32_t limit) {
    if ((arrive != 0 && arrive != 1) || limit < 1 || limit > (1 << 20))
        return fail(PNT_ERR_INVALID_ARG, "arrive must be 0 or 1 and limit in 1 .. 2^20");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(PNT_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(PNT_ERR_INVALID_ARG, "device %d out of range", device);
    DeviceGuard dg(device);
    int* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, sizeof(int)));
    cudaError_t e = cudaMemset(d, 0xff, sizeof(int));
    if (e == cudaSuccess) {
        bounded_wait_probe<<<1, 32>>>(arrive, limit, d);
        e = cudaGetLastError();
    }
    int h = -1;
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "bounded wait probe: %s", cudaGetErrorString(e));
    if (h != 0 && h != 1) return fail(PNT_ERR_CUDA, "bounded wait probe wrote %d", h);
    if (h) return fail(PNT_ERR_TIMEOUT, "the bounded wait ran out after %d polls", limit);
    return PNT_OK;
}

pnt_status pnt_closure_forward(const pnt_closure* c, const float* feats, int64_t n, float* out) {
    if (!c || !feats || !out || n < 0) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return PNT_OK;
    DeviceGuard dg(c->device);
    int* err = nullptr;
    CUDA_TRY(cudaMalloc(&err, sizeof(int)));
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), c->stream);
    if (e == cudaSuccess) {
        closure_forward_kernel<<<(unsigned)((n + kMlpRows - 1) / kMlpRows), kMlpRows, kForwardSmem, c->stream>>>(
            c->d_img, feats, n, out, err);
        e = cudaGetLastError();
    }
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(err);
    if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "closure forward: %s", cudaGetErrorString(e));
    if (herr) return fail(PNT_ERR_TIMEOUT, "tensor-core wait ran out in the closure forward");
    return PNT_OK;
}

pnt_status pnt_hydro_harvest(pnt_hydro* h, double dead, double keep, uint64_t seed, float* feats, float* targets,
                             int32_t* sides, int64_t capacity, int64_t* count) {
    if (!h || !feats || !targets || !sides || !count || capacity < 0 || *count < 0 || !(keep >= 0.) || !(dead >= 0.))
        return fail(PNT_ERR_INVALID_ARG, "bad argument");
    pnt::HydroAccess ha;
    if (!pnt::hydro_access(h, &ha)) return fail(PNT_ERR_INVALID_ARG, "bad hydro");
    DeviceGuard dg(ha.device);
    const int nb = (int)zone_blocks(ha.a.numz);
    int32_t* counts = nullptr;
    int64_t* offs = nullptr;
    CUDA_TRY(cudaMalloc(&counts, (size_t)nb * sizeof(int32_t) + 64));
    cudaError_t e = cudaMalloc(&offs, ((size_t)nb + 1) * sizeof(int64_t));
    if (e != cudaSuccess) {
        cudaFree(counts);
        return fail(PNT_ERR_CUDA, "harvest scratch: %s", cudaGetErrorString(e));
    }
    HarvestArgs args{};
    args.dead = dead;
    args.qa = ha.c.q2 * 0.25 * ha.c.gammap1;
    args.qb = ha.c.q1;
    args.keep_all = keep >= 1.0 ? 1 : 0;
    args.keep = (uint32_t)std::min(keep * 4294967296.0, 4294967295.0);
    args.seed = seed;
    args.counts = counts;
    args.offsets = offs;
    args.feats = feats;
    args.targs = targets;
    args.sides = sides;
    args.capacity = capacity;
    harvest_kernel<false><<<nb, kZoneThreads, 0, ha.stream>>>(ha.a, ha.c, args);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        scan_counts<<<1, 1024, 0, ha.stream>>>(counts, nb, *count, offs, offs + nb);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        harvest_kernel<true><<<nb, kZoneThreads, 0, ha.stream>>>(ha.a, ha.c, args);
        e = cudaGetLastError();
    }
    int64_t total = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, offs + nb, sizeof(int64_t), cudaMemcpyDeviceToHost, ha.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ha.stream);
    cudaFree(counts);
    cudaFree(offs);
    if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "harvest: %s", cudaGetErrorString(e));
    *count = std::min(total, capacity);
    return PNT_OK;
}

}  // extern "C"
