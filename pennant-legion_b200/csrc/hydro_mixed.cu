// hydro_mixed.cu -- the mixed-precision hydro cycle (precision = mixed).
//
// Same passes and data flow as the FP64 cycle (hydro_fp64.cu), with the
// per-side work of the predictor in FP32:
//
//   FP64  point positions and velocities (advPosHalf, advPosFull), the
//         zone centre, side areas and RZ volumes with their zone sums (the
//         half-step volume change zvolp - zvol0 of PolyGas::calcStateHalf
//         would cancel in FP32), the zone EOS, calcRho, the corner-mass and
//         corner-force sums at points, calcWork/calcWorkRate/calcEnergy and
//         the dt reduction;
//   FP32  edge lengths, surface vectors, characteristic lengths, the TTS
//         side force and every QCS corner quantity, formed in coordinates
//         and velocities relative to the zone's first point so that FP32
//         keeps its precision on small zones far from the origin.  Zones
//         with a corner sharper than ~30 degrees (the centre of a pie mesh)
//         form their QCS side force in FP64: there it is a small difference
//         of terms weighted by 1/sin^2 of the corner angle.
//
// The pressure force sfp is formed in FP64 (its surface vectors cancel
// around each zone, and calcWork needs that cancellation), and sfp + sfq is
// handed to calcWork in FP64; the corner mass and corner force handed to the
// point pass are stored in FP32 (4 + 8 B per side instead of 24 B).  Pass A
// runs one thread per zone (128 registers, 4 blocks of 128 per SM): with the
// divisions and square roots in FP32 it is 40% faster than four lanes per
// zone.  The learned cycle (precision learned) is this cycle with the QCS
// corner forces of compressing corners moved to the closure pass.
// Compiled with fast math; the accuracy of this path is stated as its L1
// error against the FP64 run (tests/test_gpu_mixed.py).
#include "closure_dev.cuh"
#include "hydro_fp64_body.cuh"
#include "batch_dev.h"
#include "hydro_dev.h"
#include "row_tiles.cuh"
#include "zone_tiles.cuh"

#include <cuda_runtime.h>

namespace pnt {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double2 add(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 sub(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 smul(double r, double2 v) { return mk(v.x * r, v.y * r); }
__device__ __forceinline__ double dot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ double cross(double2 a, double2 b) { return a.x * b.y - a.y * b.x; }
__device__ __forceinline__ double2 project(double2 v, double ux, double uy) {
    const double d = v.x * ux + v.y * uy;
    return mk(v.x - ux * d, v.y - uy * d);
}
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ float2 fk(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 fadd(float2 a, float2 b) { return fk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 fsub(float2 a, float2 b) { return fk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 fmul(float r, float2 v) { return fk(v.x * r, v.y * r); }
__device__ __forceinline__ float fdot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ float fcross(float2 a, float2 b) { return a.x * b.y - a.y * b.x; }
__device__ __forceinline__ float flen(float2 v) { return sqrtf(v.x * v.x + v.y * v.y); }
__device__ __forceinline__ float flen2(float2 v) { return v.x * v.x + v.y * v.y; }
__device__ __forceinline__ float2 f2(double2 v) { return fk((float)v.x, (float)v.y); }

__device__ __forceinline__ float2 shflf2(float2 v, int src) {
    return fk(__shfl_sync(kFull, v.x, src), __shfl_sync(kFull, v.y, src));
}

template <typename T>
__device__ __forceinline__ T zsum4(T v, int g, int n) {
    T s = __shfl_sync(kFull, v, g);
    s += __shfl_sync(kFull, v, g + 1);
    s += __shfl_sync(kFull, v, g + 2);
    const T d = __shfl_sync(kFull, v, g + 3);
    if (n == 4) s += d;
    return s;
}

__device__ __forceinline__ bool skip_cycle(const Ctl* ctl) {
    return ctl->done || ctl->cycle >= ctl->stop_at;
}

template <bool kMin, int kThreads>
__device__ __forceinline__ void block_fold(double v, double* out) {
    __shared__ double red[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(kFull, v, o);
        v = kMin ? dmin(v, w) : ((w > v) ? w : v);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = red[0];
        for (int i = 1; i < kThreads / 32; ++i) r = kMin ? dmin(r, red[i]) : ((red[i] > r) ? red[i] : r);
        *out = r;
    }
}

// ---------------------------------------------------------------------
// Pass A, mixed precision, one thread per zone of N sides (N = 3 or 4): the
// arithmetic of pass_a_mixed side by side in the zone's side order.
// ---------------------------------------------------------------------
// QCS side force of one zone in FP64 (QCS.cc:116-380), for zones with an
// acute corner: there sfq is a small difference of large terms (cw grows as
// 1/sin^2 of the corner angle) that FP32 cannot carry.
template <int N>
__device__ __forceinline__ void qcs_sfq_fp64_zone(const DevArrays& a, const HydroConst& c, int cur, int64_t s0,
                                                  const double2* xp, double2 zxp, double zss, double zrp,
                                                  double2* sfq) {
    double2 u0[N];
#pragma unroll
    for (int k = 0; k < N; ++k) u0[k] = a.pu[cur][__ldg(a.mapsp1 + s0 + k)];
    const double rn = 1. / (double)N;
    double zx = u0[0].x * rn, zy = u0[0].y * rn;
#pragma unroll
    for (int k = 1; k < N; ++k) {
        zx += u0[k].x * rn;
        zy += u0[k].y * rn;
    }
    const double2 zuc = mk(zx, zy);
    double2 ex[N], cqe1[N], cqe2[N];
    double elen[N], cw[N], cc[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int nk = (k + 1 == N) ? 0 : k + 1;
        ex[k] = smul(0.5, add(xp[k], xp[nk]));
        const double2 d = sub(xp[nk], xp[k]);
        elen[k] = sqrt(dot(d, d));
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int pk = (k == 0) ? N - 1 : k - 1;
        const int nk = (k + 1 == N) ? 0 : k + 1;
        const double2 up0 = u0[k], xq0 = xp[k], xq1 = ex[k], up2 = zuc, xq2 = zxp, upp = u0[pk], xq3 = ex[pk];
        const double2 up1 = smul(0.5, add(up0, u0[nk]));
        const double2 up3 = smul(0.5, add(upp, up0));
        const double de1 = elen[pk], de2 = elen[k];
        const double cvolume = 0.5 * cross(sub(xq2, xq0), sub(xq3, xq1));
        const double2 v1 = sub(xq3, xq0), v2 = sub(xq1, xq0);
        const double minelen = dmin(de1, de2);
        double ccos = (minelen < 1.e-12) ? 0. : 4. * dot(v1, v2) / (de1 * de2);
        const double cdiv = (cross(sub(up2, up0), sub(xq3, xq1)) - cross(sub(up3, up1), sub(xq2, xq0))) /
                            (2.0 * cvolume);
        double crmu = 0.;
        if (cdiv < 0.0) {
            const double2 dxx1 = smul(0.5, sub(sub(add(xq1, xq2), xq0), xq3));
            const double2 dxx2 = smul(0.5, sub(sub(add(xq2, xq3), xq0), xq1));
            const double dx1 = sqrt(dot(dxx1, dxx1)), dx2 = sqrt(dot(dxx2, dxx2));
            const double2 duav = smul(0.25, add(add(add(up0, up1), up2), up3));
            const double test1 = fabs(dot(dxx1, duav) * dx2);
            const double test2 = fabs(dot(dxx2, duav) * dx1);
            const double rr = (test1 > test2) ? dx1 / dx2 : dx2 / dx1;
            const double evol = dmin(sqrt(4.0 * cvolume * rr), 2.0 * minelen);
            const double2 w1 = sub(sub(add(up1, up2), up0), up3), w2 = sub(sub(add(up2, up3), up0), up1);
            const double du = sqrt(dmax(dot(w1, w1), dot(w2, w2)));
            const double ztmp2 = c.q2 * 0.25 * c.gammap1 * du;
            const double ztmp1 = c.q1 * zss;
            crmu = (ztmp2 + sqrt(ztmp2 * ztmp2 + ztmp1 * ztmp1)) * zrp * evol;
        }
        cqe1[k] = smul(crmu / de1, sub(up0, upp));
        cqe2[k] = smul(crmu / de2, sub(u0[nk], up0));
        const double csin2 = 1.0 - ccos * ccos;
        cw[k] = (csin2 < 1.e-4) ? 0. : cvolume / csin2;
        cc[k] = (csin2 < 1.e-4) ? 0. : ccos;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int nk = (k + 1 == N) ? 0 : k + 1;
        sfq[k] = smul(1. / elen[k], add(smul(cw[k], add(cqe2[k], smul(cc[k], cqe1[k]))),
                                        smul(cw[nk], add(cqe1[nk], smul(cc[nk], cqe2[nk])))));
    }
}

constexpr int kZoneThreadsZT = 128;   // pass A: one zone per thread

// Per-side values parked in the thread's shared-memory slots between their
// computation and their last use ([side][thread]: conflict-free).
struct SideSpill {
    double2* sfp_;
    float2* sft_;
    int t;
    int stride = kZoneThreadsZT;   // threads of the CTA
    __device__ __forceinline__ double2& sfp(int k) const { return sfp_[k * stride + t]; }
    __device__ __forceinline__ float2& sft(int k) const { return sft_[k * stride + t]; }
};

// Where the learned cycle's pass A records a zone for the closure: record
// i at base + (i & mask) * kZoneRecF4, i from an atomic counter (global or
// shared memory).
struct RecSink {
    int* count;
    float4* base;
    int mask;
};

// nbad counts the zone's inverted sides; cnt[3]: its corners without
// compression, in the dead zone, in an acute zone (learned cycle).
// in: the zone's inputs (fp64::GlobalZoneIn, or a row tile's shared-memory
// stage); sink: where a zone with deferred corners is recorded (learned).
template <int N, bool kLearned, typename In>
__device__ __forceinline__ void pass_a_mixed_zone(const DevArrays& a, const HydroConst& c, const In& in, int cur,
                                                  double dt, int64_t z, int64_t s0, double& zdthyd, int& nbad,
                                                  int* cnt, const SideSpill& sp, const RecSink& sink = RecSink{}) {
    double2 xp[N];
    float2 uf[N];
    double mf[N];
    const double dth = 0.5 * dt;
    double2 uref;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const double2 u0 = in.u0(k);
        xp[k] = add(in.x0(k), smul(dth, u0));
        if (k == 0) uref = u0;
        // velocities relative to the zone's first point: QCS works on
        // velocity differences, which absolute FP32 values would round away
        uf[k] = f2(sub(u0, uref));
        mf[k] = in.mf(k);
    }
    const double zm = in.zm(), zr = in.zr(), ze = in.ze(), zwrate = in.zwrate(), zvol0 = in.zvol();
    // FP64: positions, zone centre, side areas and volumes
    const double rn = 1. / (double)N;
    double zx = xp[0].x * rn, zy = xp[0].y * rn;
#pragma unroll
    for (int k = 1; k < N; ++k) {
        zx += xp[k].x * rn;
        zy += xp[k].y * rn;
    }
    const double2 zxp = mk(zx, zy);
    const double third = 1. / 3.;
    double sa[N];
    double zareap = 0., zvolp = 0.;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int nk = (k + 1 == N) ? 0 : k + 1;
        sa[k] = 0.5 * cross(sub(xp[nk], xp[k]), sub(zxp, xp[k]));
        const double sv = third * sa[k] * (xp[k].x + xp[nk].x + zxp.x);
        zareap = (k == 0) ? sa[k] : zareap + sa[k];
        zvolp = (k == 0) ? sv : zvolp + sv;
        nbad += (sv <= 0.) ? 1 : 0;
    }
    // Zone EOS and density (PolyGas.cc:63-109, Hydro.cc:1034-1054): the
    // half-step pressure zp in FP64 (it feeds the FP64 pressure force); the
    // sound speed and the half-step density feed only FP32 quantities (TTS,
    // QCS, the corner mass, the Courant dt), so they are formed in FP32.
    // q = per p / zr^2 is written gm1 pre (the same quantity, no division).
    const double e = dmax(ze, 0.);
    const double p = c.gm1 * zr * e;
    const double pre = c.gm1 * e;
    const double per = c.gm1 * zr;
    const double q = c.gm1 * pre;
    const double minv = 1. / zm;
    const double csqd = dmax(c.ssmin2, pre + q);
    const double dv = (zvolp - zvol0) * minv;
    const double bulk = zr * csqd;
    const double denom = 1. + 0.5 * per * dv;
    const double src = zwrate * dth * minv;
    const double zp = p + (per * src - zr * bulk * dv) / denom;
    const float zssf = sqrtf((float)csqd);
    const float zrpf = (float)zm / (float)zvolp;
    {
        const float hz = 0.5f * zrpf * (float)zareap;
#pragma unroll
        for (int k = 0; k < N; ++k)
            a.cmass_f[s0 + k] = hz * ((float)mf[k] + (float)mf[(k == 0) ? N - 1 : k - 1]);
    }
    a.zp[z] = zp;

    // FP32 from here, relative to the zone's first point
    float2 r[N], ex[N];
    float elen[N], rinv[N];
#pragma unroll
    for (int k = 0; k < N; ++k) r[k] = f2(sub(xp[k], xp[0]));
    const float2 zc = f2(sub(zxp, xp[0]));
    const float rnf = (float)rn;
    float zux = uf[0].x * rnf, zuy = uf[0].y * rnf;
#pragma unroll
    for (int k = 1; k < N; ++k) {
        zux += uf[k].x * rnf;
        zuy += uf[k].y * rnf;
    }
    const float2 zuc = fk(zux, zuy);
    const float fac = (N == 3 ? 3.f : 4.f);
    float zdl = __int_as_float(0x7f800000);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int nk = (k + 1 == N) ? 0 : k + 1;
        ex[k] = fmul(0.5f, fadd(r[k], r[nk]));
        elen[k] = flen(fsub(r[nk], r[k]));
        rinv[k] = 1.f / elen[k];
        zdl = fminf(zdl, fac * (float)sa[k] / elen[k]);
    }

    // The side forces that do not involve QCS, formed now so that the FP64
    // positions, smf and side areas are dead during the corner loop: the
    // PolyGas force in FP64 (its surface vectors cancel around the zone and
    // calcWork takes the residual) and TTS in FP32, parked in shared memory.
    {
        float sstmp = fmaxf(zssf, (float)c.tts_ssmin);
        sstmp = (float)c.alfa * sstmp * sstmp;
        const float zareapf = (float)zareap;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int nk = (k + 1 == N) ? 0 : k + 1;
            const double2 ex64 = smul(0.5, add(xp[k], xp[nk]));
            sp.sfp(k) = smul(-zp, mk(-(ex64.y - zxp.y), ex64.x - zxp.x));
            const float2 ssurf = fk(-(ex[k].y - zc.y), ex[k].x - zc.x);
            const float srho = zrpf * (float)mf[k] * (zareapf / (float)sa[k]);
            sp.sft(k) = fmul(-(sstmp * (srho - zrpf)), ssurf);
        }
    }

    // QCS corners (QCS.cc:116-380), FP32; sin^2 of the corner angle as
    // (4 cross / (de1 de2))^2 (the reference's 1 - ccos^2 loses the small
    // sines of acute corners in FP32); zones with a corner under ~30 degrees
    // take the FP64 form below
    float2 cqe1[N], cqe2[N];
    float cw[N], cc[N];
    bool acute = false;
    bool defer_any = false;
    uint32_t defer_bits = 0;
    const float dead = kLearned ? __ldg(reinterpret_cast<const float*>(a.closure_img + kImgThr)) : 0.f;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int pk = (k == 0) ? N - 1 : k - 1;
        const int nk = (k + 1 == N) ? 0 : k + 1;
        const float2 up0 = uf[k], xq0 = r[k];
        const float2 up1 = fmul(0.5f, fadd(up0, uf[nk]));
        const float2 xq1 = ex[k];
        const float2 up2 = zuc, xq2 = zc;
        const float2 up3 = fmul(0.5f, fadd(uf[pk], up0));
        const float2 xq3 = ex[pk];
        const float cvolume = 0.5f * fcross(fsub(xq2, xq0), fsub(xq3, xq1));
        const float2 v1 = fsub(xq3, xq0), v2 = fsub(xq1, xq0);
        const float de1 = elen[pk], de2 = elen[k];
        const float minelen = fminf(de1, de2);
        float ccos = (minelen < 1.e-12f) ? 0.f : 4.f * fdot(v1, v2) / (de1 * de2);
        const float cdiv = (fcross(fsub(up2, up0), fsub(xq3, xq1)) - fcross(fsub(up3, up1), fsub(xq2, xq0))) /
                           (2.f * cvolume);
        const float ssin = 4.f * fcross(v1, v2) / (de1 * de2);
        const float csin2 = (minelen < 1.e-12f) ? 1.f : ssin * ssin;
        acute = acute || (csin2 < 0.25f);
        float crmu = 0.f;
        if constexpr (kLearned) {
            // learned cycle: no QCS force here; compressing corners past the
            // dead zone are deferred to the closure pass
            if (cdiv < 0.f) {
                const float2 d1 = fsub(up0, uf[pk]), d2 = fsub(uf[nk], up0), dcz = fsub(zuc, up0);
                const float m2 = fmaxf(fmaxf(flen2(d1), flen2(d2)), flen2(dcz));
                const float lim = dead * zssf;
                if (m2 > lim * lim) defer_bits |= 1u << k;
                else ++cnt[1];
            } else {
                ++cnt[0];
            }
        } else if (cdiv < 0.f) {
            const float2 dxx1 = fmul(0.5f, fsub(fsub(fadd(xq1, xq2), xq0), xq3));
            const float2 dxx2 = fmul(0.5f, fsub(fsub(fadd(xq2, xq3), xq0), xq1));
            const float dx1 = flen(dxx1), dx2 = flen(dxx2);
            const float2 duav = fadd(fmul(0.25f, fadd(fadd(fadd(up0, up1), up2), up3)), f2(uref));
            const float test1 = fabsf(fdot(dxx1, duav) * dx2);
            const float test2 = fabsf(fdot(dxx2, duav) * dx1);
            const float rr = (test1 > test2) ? dx1 / dx2 : dx2 / dx1;
            const float evol = fminf(sqrtf(4.f * cvolume * rr), 2.f * minelen);
            const float du = sqrtf(fmaxf(flen2(fsub(fsub(fadd(up1, up2), up0), up3)),
                                         flen2(fsub(fsub(fadd(up2, up3), up0), up1))));
            const float ztmp2 = (float)(c.q2 * 0.25 * c.gammap1) * du;
            const float ztmp1 = (float)c.q1 * zssf;
            crmu = (ztmp2 + sqrtf(ztmp2 * ztmp2 + ztmp1 * ztmp1)) * zrpf * evol;
        }
        if constexpr (!kLearned) {
            cqe1[k] = fmul(crmu * rinv[pk], fsub(up0, uf[pk]));
            cqe2[k] = fmul(crmu * rinv[k], fsub(uf[nk], up0));
            cw[k] = (csin2 < 1.e-4f) ? 0.f : cvolume / csin2;
            cc[k] = (csin2 < 1.e-4f) ? 0.f : ccos;
        }
    }
    if constexpr (kLearned) {
        if (acute) {   // the zone keeps the FP64 QCS: its corners are counted as acute
            cnt[0] = cnt[1] = 0;
            cnt[2] = N;
            defer_bits = 0;
        }
        defer_any = defer_bits != 0;
        // record the zone for the closure pass (warp-aggregated slot)
        const unsigned am = __activemask();
        const unsigned m = __ballot_sync(am, defer_any);
        if (defer_any) {
            const int lane = threadIdx.x & 31;
            const int leader = __ffs(m) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(sink.count, __popc(m));
            base = __shfl_sync(m, base, leader);
            const int idx = base + __popc(m & ((1u << lane) - 1u));
            float4* rec = sink.base + (int64_t)(idx & sink.mask) * kZoneRecF4;
            const float2 r3 = (N == 4) ? r[N - 1] : fk(0.f, 0.f), u3 = (N == 4) ? uf[N - 1] : fk(0.f, 0.f);
            rec[0] = make_float4(r[0].x, r[0].y, r[1].x, r[1].y);
            rec[1] = make_float4(r[2].x, r[2].y, r3.x, r3.y);
            rec[2] = make_float4(uf[0].x, uf[0].y, uf[1].x, uf[1].y);
            rec[3] = make_float4(uf[2].x, uf[2].y, u3.x, u3.y);
            rec[4] = make_float4(zc.x, zc.y, zuc.x, zuc.y);
            rec[5] = make_float4((float)uref.x, (float)uref.y, zssf, zrpf);
            rec[6] = make_float4(__int_as_float((int)s0), __int_as_float(N), __int_as_float((int)defer_bits), 0.f);
        }
    }
    // QCS::setForce (QCS.cc:331-380); in the learned cycle no corner outside
    // an acute zone has a QCS force here (the closure pass adds the deferred
    // ones), so sfq starts at zero there
    float2 sfq[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int nk = (k + 1 == N) ? 0 : k + 1;
        if constexpr (kLearned)
            sfq[k] = fk(0.f, 0.f);
        else
            sfq[k] = fmul(rinv[k], fadd(fmul(cw[k], fadd(cqe2[k], fmul(cc[k], cqe1[k]))),
                                        fmul(cw[nk], fadd(cqe1[nk], fmul(cc[nk], cqe2[nk])))));
    }
    if (acute) {
        // the half-step positions again (advPosHalf, as above), for the
        // FP64 QCS of this rare zone
        double2 xq[N], q64[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int32_t p = __ldg(a.mapsp1 + s0 + k);
            xq[k] = add(a.px[cur][p], smul(dth, a.pu[cur][p]));
        }
        qcs_sfq_fp64_zone<N>(a, c, cur, s0, xq, zxp, (double)zssf, (double)zrpf, q64);
#pragma unroll
        for (int k = 0; k < N; ++k) sfq[k] = f2(q64[k]);
    }
    // QCS::setVelDiff, calcDtNew (FP64 reduction)
    float ztmp = 0.f;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int nk = (k + 1 == N) ? 0 : k + 1;
        const float dux = fabsf(fdot(fsub(uf[nk], uf[k]), fsub(r[nk], r[k]))) * rinv[k];
        ztmp = fmaxf(ztmp, (elen[k] > 0.f) ? dux : 0.f);
    }
    const float zdu = (float)c.q1 * zssf + 2.f * (float)c.q2 * ztmp;
    const float cdu = fmaxf(zdu, fmaxf(zssf, 1.e-30f));
    zdthyd = (double)(zdl * (float)c.cfl / cdu);

    // corner force and sfp + sfq for calcWork
    double2 ftot[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const float2 sft = sp.sft(k);
        const double2 sfpq = add(sp.sfp(k), mk((double)sfq[k].x, (double)sfq[k].y));
        ftot[k] = add(sfpq, mk((double)sft.x, (double)sft.y));
        a.sftot[s0 + k] = sfpq;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) a.cforce_f[s0 + k] = f2(sub(ftot[k], ftot[(k == 0) ? N - 1 : k - 1]));
}

#ifndef PNT_MIXED_ZT_MIN_BLOCKS
#define PNT_MIXED_ZT_MIN_BLOCKS 4
#endif

template <bool kQuads, bool kLearned>
__global__ void __launch_bounds__(kZoneThreadsZT, PNT_MIXED_ZT_MIN_BLOCKS) pass_a_mixed_zt(DevArrays a, HydroConst c) {
    pdl_wait();
    const Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const int64_t z = (int64_t)blockIdx.x * kZoneThreadsZT + threadIdx.x;
    double zdthyd = 1.e99;
    int bad = 0;
    int cnt[3] = {0, 0, 0};
    __shared__ double2 s_sfp[4 * kZoneThreadsZT];
    __shared__ float2 s_sft[4 * kZoneThreadsZT];
    const SideSpill sp{s_sfp, s_sft, (int)threadIdx.x};
    if (z < a.numz) {
        const int cur = ctl->cycle & 1;
        const double dt = ctl->dt;
        const RecSink sink{a.closure_nrec, reinterpret_cast<float4*>(a.closure_rec), 0x7fffffff};
        if (kQuads) {
            const fp64::GlobalZoneIn in{a, cur, z, 4 * z};
            pass_a_mixed_zone<4, kLearned>(a, c, in, cur, dt, z, 4 * z, zdthyd, bad, cnt, sp, sink);
        } else {
            const int n = a.znump[z];
            const int64_t s0 = a.zfirst[z];
            const fp64::GlobalZoneIn in{a, cur, z, s0};
            if (n == 4) pass_a_mixed_zone<4, kLearned>(a, c, in, cur, dt, z, s0, zdthyd, bad, cnt, sp, sink);
            else pass_a_mixed_zone<3, kLearned>(a, c, in, cur, dt, z, s0, zdthyd, bad, cnt, sp, sink);
        }
    }
    __shared__ unsigned wcount[kLearned ? kZoneThreadsZT / 32 : 1][3];
    if constexpr (kLearned) {
        for (int q = 0; q < 3; ++q) {
            const unsigned t = __reduce_add_sync(kFull, (unsigned)cnt[q]);
            if ((threadIdx.x & 31) == 0) wcount[threadIdx.x >> 5][q] = t;
        }
    }
    const int nbad = tiles::block_isum<kZoneThreadsZT>(bad);   // its barrier also orders wcount
    if constexpr (kLearned) {
        constexpr int kCounted[3] = {kClassZero, kClassDead, kClassAcute};
        if (threadIdx.x < 3) {
            unsigned t = 0;
            for (int w = 0; w < kZoneThreadsZT / 32; ++w) t += wcount[w][threadIdx.x];
            if (t) atomicAdd(a.closure_counts + kCounted[threadIdx.x] * 64 + (blockIdx.x & 63), (unsigned long long)t);
        }
    }
    fp64::block_to_cycle<true, kZoneThreadsZT>(a.cyc_red, zdthyd, nbad);
}

// ---------------------------------------------------------------------
// The learned closure's corner work.  Pass A records every zone with
// deferred corners (closure_dev.cuh: kZoneRecF4 float4 a zone).  A round
// takes up to J * blockDim.x / 4 recorded zones, thread t corner t & 3 of
// zones t / 4, t / 4 + blockDim.x / 4, ...  Each deferred corner is
// classified (compression past rho_max or inputs out of distribution: plain
// QCS, QCS.cc:116-327 in FP32 as in the mixed pass A; otherwise the
// network); the network's corners of a round are packed into consecutive
// rows of the tensor-core operand, so the network (tcgen05, closure_dev.cuh)
// runs on those corners only.  A corner's QCS forces cqe1, cqe2 enter
// QCS::setForce (QCS.cc:331-380) linearly: its side s gets
// d1 = cw (cqe2 + ccos cqe1) / elen[s] and the previous side
// d2 = cw (cqe1 + ccos cqe2) / elen[s3].  The corner force of side s,
// ftot[s] - ftot[s3] (Hydro.cc:1159-1193), and sfp + sfq of side s then
// change by
//   dcforce[s] = d1(s) - d2(s) - d1(s3) + d2(s4),  dsftot[s] = d1(s) + d2(s4),
// which only touch the recorded zone's own sides: no two records write the
// same side, so the update is deterministic without atomics.
// ---------------------------------------------------------------------

// Corner k of a zone record; deferred = k is a corner of the zone and was
// deferred by pass A.
struct RecCorner {
    float2 x, xpv, xn, xz, u, upv, un, uz, uav;
    float css, rho;
    int s0, n;
    bool deferred;
};

__device__ __forceinline__ float2 sel4(int k, float2 a, float2 b, float2 c, float2 d) {
    return k == 0 ? a : (k == 1 ? b : (k == 2 ? c : d));
}

__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// A zone record as loaded (kZoneRecF4 float4).
struct ZoneRec {
    float4 q[kZoneRecF4];
};
__device__ __forceinline__ ZoneRec load_zone_rec(const float4* __restrict__ rec) {
    ZoneRec r;
#pragma unroll
    for (int i = 0; i < kZoneRecF4; ++i) r.q[i] = rec[i];
    return r;
}

__device__ __forceinline__ RecCorner rec_corner(const ZoneRec& zr, int k) {
    const float4 q0 = zr.q[0], q1 = zr.q[1], q2 = zr.q[2], q3 = zr.q[3], q4 = zr.q[4], q5 = zr.q[5], q6 = zr.q[6];
    RecCorner o;
    o.s0 = __float_as_int(q6.x);
    o.n = __float_as_int(q6.y);
    const int n = o.n;
    o.deferred = k < n && ((__float_as_int(q6.z) >> k) & 1);
    const int pk = (k == 0) ? n - 1 : k - 1;
    const int nk = (k + 1 >= n) ? 0 : k + 1;
    const float2 r0 = fk(q0.x, q0.y), r1 = fk(q0.z, q0.w), r2 = fk(q1.x, q1.y), r3 = fk(q1.z, q1.w);
    const float2 v0 = fk(q2.x, q2.y), v1 = fk(q2.z, q2.w), v2 = fk(q3.x, q3.y), v3 = fk(q3.z, q3.w);
    o.x = sel4(k, r0, r1, r2, r3);
    o.xpv = sel4(pk, r0, r1, r2, r3);
    o.xn = sel4(nk, r0, r1, r2, r3);
    o.u = sel4(k, v0, v1, v2, v3);
    o.upv = sel4(pk, v0, v1, v2, v3);
    o.un = sel4(nk, v0, v1, v2, v3);
    o.xz = fk(q4.x, q4.y);
    o.uz = fk(q4.z, q4.w);
    // the mean corner velocity as pass A forms it (absolute)
    const float2 up1 = fmul(0.5f, fadd(o.u, o.un)), up3 = fmul(0.5f, fadd(o.upv, o.u));
    o.uav = fadd(fmul(0.25f, fadd(fadd(fadd(o.u, up1), o.uz), up3)), fk(q5.x, q5.y));
    o.css = q5.z;
    o.rho = q5.w;
    return o;
}

// Corner k of the zone record zr: its class (-1: not deferred or in the
// dead zone; kClassMlp, kClassFallback, kClassOod) and, when classified,
// its inputs f, frame (cx, cy) and force scale rho D (a D + b c) in
// frame[0..2].  img: the parameter image (shared memory).
__device__ __forceinline__ int closure_classify(const ZoneRec& zr, int k, const uint8_t* img, float qa, float qb,
                                                float* f, float* frame) {
    const RecCorner q = rec_corner(zr, k);
    float cx = 0.f, cy = 0.f, scale = 0.f;
    if (!q.deferred ||
        !closure_features<float>({q.x.x, q.x.y}, {q.xpv.x, q.xpv.y}, {q.xn.x, q.xn.y}, {q.xz.x, q.xz.y},
                                 {q.u.x, q.u.y}, {q.upv.x, q.upv.y}, {q.un.x, q.un.y}, {q.uz.x, q.uz.y},
                                 {q.uav.x, q.uav.y}, q.css, qa, qb, 0.f, f, cx, cy, scale))
        return -1;
    frame[0] = cx;
    frame[1] = cy;
    frame[2] = q.rho * scale;
    const float* thr = reinterpret_cast<const float*>(img + kImgThr);
    if (f[11] > thr[1]) return kClassFallback;   // rho_max
    const float* mean = reinterpret_cast<const float*>(img + kImgFMean);
    const float* istd = reinterpret_cast<const float*>(img + kImgFIstd);
    float zmax = 0.f;
#pragma unroll
    for (int i = 0; i < kClIn; ++i) zmax = fmaxf(zmax, fabsf((f[i] - mean[i]) * istd[i]));
    return (zmax > thr[2]) ? kClassOod : kClassMlp;   // ood_kappa
}

// The QCS forces of corner k of the record, as QCS::setForce distributes
// them: d[0..1] = d1 to side k, d[2..3] = d2 to side k - 1.  how: 1 the
// network's outputs y in the frame (cx, cy) scaled by frame[2], 2 plain
// QCS (FP32 as in the mixed pass A), 0 none.
__device__ __forceinline__ void closure_corner_forces(const ZoneRec& zr, int k, int how, float4 y, const float* frame,
                                                      float qa, float qb, float* d) {
    const RecCorner q = rec_corner(zr, k);
    // corner geometry (QCS::setCornerDiv / setForce)
    const float2 xc = q.x, xpv = q.xpv, xn = q.xn, xz = q.xz;
    const float2 ex = fmul(0.5f, fadd(xc, xn));
    const float2 xq3 = fmul(0.5f, fadd(xpv, xc));
    const float cvolume = 0.5f * fcross(fsub(xz, xc), fsub(xq3, ex));
    const float2 v1 = fsub(xq3, xc), v2 = fsub(ex, xc);
    const float de1 = flen(fsub(xc, xpv)), de2 = flen(fsub(xn, xc));
    const float rinv_de1 = 1.f / de1, rinv_el = 1.f / de2;
    const float minelen = fminf(de1, de2);
    float ccos = (minelen < 1.e-12f) ? 0.f : 4.f * fdot(v1, v2) / (de1 * de2);
    float2 q1 = fk(0.f, 0.f), q2 = fk(0.f, 0.f);
    if (how == 1) {
        const float cx = frame[0], cy = frame[1], sc = frame[2];
        q1 = fk((cx * y.x - cy * y.y) * sc, (cy * y.x + cx * y.y) * sc);
        q2 = fk((cx * y.z - cy * y.w) * sc, (cy * y.z + cx * y.w) * sc);
    } else if (how == 2) {
        const float2 u = q.u, upv = q.upv, un = q.un, uz = q.uz, uav = q.uav;
        const float2 up1 = fmul(0.5f, fadd(u, un)), up3 = fmul(0.5f, fadd(upv, u));
        const float2 dxx1 = fmul(0.5f, fsub(fsub(fadd(ex, xz), xc), xq3));
        const float2 dxx2 = fmul(0.5f, fsub(fsub(fadd(xz, xq3), xc), ex));
        const float dx1 = flen(dxx1), dx2 = flen(dxx2);
        const float test1 = fabsf(fdot(dxx1, uav) * dx2);
        const float test2 = fabsf(fdot(dxx2, uav) * dx1);
        const float rr = (test1 > test2) ? dx1 / dx2 : dx2 / dx1;
        const float evol = fminf(sqrtf(4.f * cvolume * rr), 2.f * minelen);
        const float du = sqrtf(fmaxf(flen2(fsub(fsub(fadd(up1, uz), u), up3)),
                                     flen2(fsub(fsub(fadd(uz, up3), u), up1))));
        const float ztmp2 = qa * du;
        const float ztmp1 = qb * q.css;
        const float crmu = (ztmp2 + sqrtf(ztmp2 * ztmp2 + ztmp1 * ztmp1)) * q.rho * evol;
        q1 = fmul(crmu * rinv_de1, fsub(u, upv));
        q2 = fmul(crmu * rinv_el, fsub(un, u));
    }
    const float ssin = 4.f * fcross(v1, v2) / (de1 * de2);
    const float csin2 = (minelen < 1.e-12f) ? 1.f : ssin * ssin;
    const float cw = (csin2 < 1.e-4f) ? 0.f : cvolume / csin2;
    ccos = (csin2 < 1.e-4f) ? 0.f : ccos;
    const float2 d1 = fmul(cw * rinv_el, fadd(q2, fmul(ccos, q1)));
    const float2 d2 = fmul(cw * rinv_de1, fadd(q1, fmul(ccos, q2)));
    d[0] = d1.x;
    d[1] = d1.y;
    d[2] = d2.x;
    d[3] = d2.y;
}

// A CTA's closure state: the parameter image (shared memory), the packed
// operand tiles and hidden activations (closure_mlp_run), the packed-row
// counter (zero between rounds) and the class counters (network, fallback,
// out of distribution) in shared memory.
struct ClosureCtx {
    const uint8_t* img;
    uint8_t* a0;
    uint8_t* h;
    int* nrow;
    unsigned* ncls;
};

// Zones zfirst .. zfirst + nz - 1 of the records rec_at(i); every thread of
// the CTA calls it.
template <int J, typename RecAt>
__device__ __forceinline__ void closure_round(const DevArrays& a, const HydroConst& c, const ClosureCtx& x,
                                              MlpState& st, RecAt&& rec_at, int zfirst, int nz) {
    const int t = threadIdx.x, k = t & 3, lane = t & 31, g = lane & ~3;
    const int zpj = (int)(blockDim.x >> 2);
    const int mode = (int)reinterpret_cast<const float*>(x.img + kImgThr)[3];   // 0 network, 1 no force, 2 plain QCS
    const float* mean = reinterpret_cast<const float*>(x.img + kImgFMean);
    const float* istd = reinterpret_cast<const float*>(x.img + kImgFIstd);
    const float qa = (float)(c.q2 * 0.25 * c.gammap1), qb = (float)c.q1;
    // the previous round's readers of the operand tiles are done
    __syncthreads();
    int slot[J], how[J], s0[J], nsd[J];
    float frame[J][3];
    // every record of the round in flight before the first is used (into
    // L1: no registers held)
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const int zl = j * zpj + (t >> 2);
        if (j * zpj < nz && zl < nz) {
            const float4* r = rec_at(zfirst + zl);
            prefetch_l1(r);
            prefetch_l1(r + kZoneRecF4 - 1);
        }
    }
#pragma unroll
    for (int j = 0; j < J; ++j) {
        slot[j] = -1;
        how[j] = 0;
        s0[j] = 0;
        nsd[j] = 4;
        if (j * zpj >= nz) continue;   // CTA-uniform
        const int zl = j * zpj + (t >> 2);
        int cls = -1;
        float f[kClIn];
        if (zl < nz) {
            const ZoneRec zr = load_zone_rec(rec_at(zfirst + zl));
            s0[j] = __float_as_int(zr.q[6].x);
            nsd[j] = __float_as_int(zr.q[6].y);
            cls = closure_classify(zr, k, x.img, qa, qb, f, frame[j]);
        }
        const bool net = cls == kClassMlp && mode == 0;
        how[j] = net ? 1 : ((cls == kClassFallback || cls == kClassOod || (cls == kClassMlp && mode == 2)) ? 2 : 0);
        const unsigned mnet = __ballot_sync(kFull, net);
        const unsigned nm = __popc(__ballot_sync(kFull, cls == kClassMlp));
        const unsigned nf = __popc(__ballot_sync(kFull, cls == kClassFallback));
        const unsigned no = __popc(__ballot_sync(kFull, cls == kClassOod));
        int base = 0;
        if (lane == 0) {
            if (nm) atomicAdd(x.ncls + 0, nm);
            if (nf) atomicAdd(x.ncls + 1, nf);
            if (no) atomicAdd(x.ncls + 2, no);
            if (mnet) base = atomicAdd(x.nrow, (int)__popc(mnet));
        }
        base = __shfl_sync(kFull, base, 0);
        if (net) {
            slot[j] = base + __popc(mnet & ((1u << lane) - 1u));
            closure_stage_row(x.a0, slot[j], f, mean, istd);
        }
    }
    fence_async_smem();
    __syncthreads();
    const int n = *x.nrow;
    for (int base = 0; base < n; base += (int)blockDim.x) closure_mlp_run(x.img, x.a0, x.h, st, base, n);
    // the runs' outputs are visible to every thread; after a tensor-core
    // wait ran out the network's corners get no force
    const bool mlp_ok = __syncthreads_and(st.ok) != 0;
    if (t == 0) *x.nrow = 0;
    // the records of the forced corners and the side values to update in
    // flight at once
#pragma unroll
    for (int j = 0; j < J; ++j) {
        if (j * zpj + (t >> 2) < nz && k < nsd[j]) {
            prefetch_l1(a.cforce_f + s0[j] + k);
            prefetch_l1(a.sftot + s0[j] + k);
            if (how[j]) {
                const float4* r = rec_at(zfirst + j * zpj + (t >> 2));
                prefetch_l1(r);
                prefetch_l1(r + kZoneRecF4 - 1);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < J; ++j) {
        if (j * zpj >= nz) continue;   // CTA-uniform
        const bool zok = j * zpj + (t >> 2) < nz;
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        const int hw = (how[j] == 1 && !mlp_ok) ? 0 : how[j];
        if (hw) {
            float4 y = make_float4(0.f, 0.f, 0.f, 0.f);
            if (hw == 1) {
                const int run = slot[j] / (int)blockDim.x;
                y = reinterpret_cast<const float4*>(x.a0 + run * (int)(blockDim.x >> 7) * 4096)
                    [slot[j] - run * (int)blockDim.x];
            }
            const ZoneRec zr = load_zone_rec(rec_at(zfirst + j * zpj + (t >> 2)));
            closure_corner_forces(zr, k, hw, y, frame[j], qa, qb, d);
        }
        const int n4 = nsd[j];
        const int lp = g + (k == 0 ? n4 - 1 : k - 1);
        const int ln = g + (k + 1 >= n4 ? 0 : k + 1);
        const float2 d1 = fk(d[0], d[1]), d2 = fk(d[2], d[3]);
        const float2 d1p = shflf2(d1, lp);
        const float2 d2n = shflf2(d2, ln);
        if (zok && k < n4) {
            const int64_t sd = (int64_t)s0[j] + k;
            const float2 cf = a.cforce_f[sd];
            a.cforce_f[sd] = fadd(cf, fadd(fsub(d1, d2), fsub(d2n, d1p)));
            const double2 sf = a.sftot[sd];
            const float2 ds = fadd(d1, d2n);
            a.sftot[sd] = mk(sf.x + (double)ds.x, sf.y + (double)ds.y);
        }
    }
}

// Adds a CTA's closure class counts and recorded zones to the counters.
__device__ __forceinline__ void closure_add_counts(const DevArrays& a, const unsigned* ncls, int zones) {
    if (threadIdx.x < 3 && ncls[threadIdx.x]) {
        const int q = threadIdx.x == 0 ? kClassMlp : (threadIdx.x == 1 ? kClassFallback : kClassOod);
        atomicAdd(a.closure_counts + q * 64 + (blockIdx.x & 63), (unsigned long long)ncls[threadIdx.x]);
    }
    if (threadIdx.x == 3 && zones)
        atomicAdd(a.closure_counts + kClassZones * 64 + (blockIdx.x & 63), (unsigned long long)zones);
}

// Pass A over row tiles of a rect mesh (row_tiles.cuh): the same zone body
// reading its inputs from the tile's shared-memory stage, persistent CTAs,
// two stages, 96-zone tiles and CTAs of 96 threads, 4 CTAs per SM (168
// registers).  At 1920^2 Sedov the learned pass A takes 0.231 ms, against
// 0.236 ms with 128-zone tiles (3 CTAs per SM), 0.236 ms with 64-zone tiles
// (6 CTAs), 0.247-0.254 ms with 64-zone tiles held to 144 or 128 registers
// (7 or 8 CTAs, spills) and 0.258 ms for the gathering kernel; three stages
// were slower (fewer resident CTAs).
#ifndef PNT_ROWS_A_STAGES
#define PNT_ROWS_A_STAGES 2
#endif
#ifndef PNT_ROWS_A_T
#define PNT_ROWS_A_T 96
#endif
#ifndef PNT_ROWS_A_MIN_BLOCKS
#define PNT_ROWS_A_MIN_BLOCKS 4
#endif
constexpr int kRowsAStages = PNT_ROWS_A_STAGES;
constexpr int kRowsAT = PNT_ROWS_A_T;   // zones a tile, threads a CTA
using AStage = rows::PassAStage<kRowsAT>;
constexpr int kRowsASmem = kRowsAStages * AStage::kBytes;

template <bool kLearned>
__global__ void
#ifdef PNT_ROWS_A_MAXREG
    __maxnreg__(PNT_ROWS_A_MAXREG)
#else
    __launch_bounds__(kRowsAT, PNT_ROWS_A_MIN_BLOCKS)
#endif
    pass_a_mixed_rows(DevArrays a, HydroConst c) {
    extern __shared__ __align__(128) unsigned char smem_a[];
    __shared__ __align__(8) uint64_t bars[kRowsAStages];
    __shared__ double2 s_sfp[4 * kRowsAT];
    __shared__ float2 s_sft[4 * kRowsAT];
    pdl_wait();
    const Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const int cur = ctl->cycle & 1;
    const double dt = ctl->dt;
    const int32_t nzx = a.rect_nzx;
    const int64_t npx = (int64_t)nzx + 1;
    const int64_t ntiles = rows::num_tiles<kRowsAT>(nzx, a.numz);
    const int t = threadIdx.x;
    const SideSpill sp{s_sfp, s_sft, t, kRowsAT};
    double zdthyd = 1.e99;
    int bad = 0;
    int cnt[3] = {0, 0, 0};
    const RecSink sink{a.closure_nrec, reinterpret_cast<float4*>(a.closure_rec), 0x7fffffff};
    auto bytes = [&](int64_t g) { return AStage::bytes(rows::tile_of<kRowsAT>(g, nzx)); };
    auto issue = [&](unsigned char* st, int64_t g, uint32_t bar) {
        AStage::issue(st, a, cur, rows::tile_of<kRowsAT>(g, nzx), npx, bar);
    };
    auto compute = [&](const unsigned char* st, int64_t g) {
        const rows::Tile tl = rows::tile_of<kRowsAT>(g, nzx);
        if (t >= tl.nt) return;
        const rows::RowZoneIn<kRowsAT> in{st, t, (int)(tl.z0 & 1)};
        const int64_t z = tl.z0 + t;
        double v = 1.e99;
        int zc[3] = {0, 0, 0};   // the zone's own corner classes (an acute zone overwrites them)
        pass_a_mixed_zone<4, kLearned>(a, c, in, cur, dt, z, 4 * z, v, bad, zc, sp, sink);
        zdthyd = dmin(zdthyd, v);
#pragma unroll
        for (int q = 0; q < 3; ++q) cnt[q] += zc[q];
    };
    if (!rows::for_tiles<kRowsAStages, AStage::kBytes>(ntiles, smem_a, bars, bytes, issue, compute) && t == 0)
        atomicOr(reinterpret_cast<unsigned long long*>(a.cyc_red + 4), 1ull);
    __shared__ unsigned wcount[kLearned ? kRowsAT / 32 : 1][3];
    if constexpr (kLearned) {
        for (int q = 0; q < 3; ++q) {
            const unsigned tt = __reduce_add_sync(kFull, (unsigned)cnt[q]);
            if ((threadIdx.x & 31) == 0) wcount[threadIdx.x >> 5][q] = tt;
        }
    }
    const int nbad = tiles::block_isum<kRowsAT>(bad);   // its barrier also orders wcount
    if constexpr (kLearned) {
        constexpr int kCounted[3] = {kClassZero, kClassDead, kClassAcute};
        if (threadIdx.x < 3) {
            unsigned tt = 0;
            for (int w = 0; w < kRowsAT / 32; ++w) tt += wcount[w][threadIdx.x];
            if (tt) atomicAdd(a.closure_counts + kCounted[threadIdx.x] * 64 + (blockIdx.x & 63), (unsigned long long)tt);
        }
    }
    fp64::block_to_cycle<true, kRowsAT>(a.cyc_red, zdthyd, nbad);
}

// ---------------------------------------------------------------------
// Pass B, mixed: FP32 corner inputs summed in FP64
// ---------------------------------------------------------------------
// kRect: a rect mesh, the point's corners from its index
// (fp64::rect_point_corners: the CSR's sides in the CSR's order).
template <bool kRect = false>
__device__ __forceinline__ void pass_b_mixed_point(const DevArrays& a, const HydroConst& c, int cur, double dt,
                                                   int64_t p) {
    const double2 x0 = a.px[cur][p];
    const double2 u0 = a.pu[cur][p];
    double m = 0.;
    double2 f = mk(0., 0.);
    if (kRect) {
        int64_t sc[4];
        const int n = fp64::rect_point_corners(a.rect_nzx, a.numz / a.rect_nzx, p, sc);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q < n) {
                m = __dadd_rn(m, (double)a.cmass_f[sc[q]]);
                const float2 cf = a.cforce_f[sc[q]];
                f = mk(__dadd_rn(f.x, (double)cf.x), __dadd_rn(f.y, (double)cf.y));
            }
        }
    } else {
        const int32_t o0 = a.poff[p], o1 = a.poff[p + 1];
        for (int32_t i = o0; i < o1; ++i) {
            const int32_t s = __ldg(a.pcorner + i);
            m = __dadd_rn(m, (double)a.cmass_f[s]);
            const float2 cf = a.cforce_f[s];
            f = mk(__dadd_rn(f.x, (double)cf.x), __dadd_rn(f.y, (double)cf.y));
        }
    }
    double2 x, u;
    fp64::advance_point(c, dt, a.bcmask[p], m, f, x0, u0, x, u);
    a.px[cur ^ 1][p] = x;
    a.pu[cur ^ 1][p] = u;
}

template <bool kRect>
__global__ void __launch_bounds__(kPointThreads) pass_b_mixed(DevArrays a, HydroConst c) {
    pdl_wait();
    const Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const int64_t p = (int64_t)blockIdx.x * kPointThreads + threadIdx.x;
    if (p >= a.nump) return;
    pass_b_mixed_point<kRect>(a, c, ctl->cycle & 1, ctl->dt, p);
}

// ---------------------------------------------------------------------
// The mixed cycle of a batch of meshes (batch.cu): the zone and point
// bodies above over the batch's work lists, as batch_pass_a and
// batch_point_pass run the FP64 ones.
// ---------------------------------------------------------------------
template <bool kAllQuads>
__global__ void __launch_bounds__(kBatchZT, PNT_MIXED_ZT_MIN_BLOCKS) batch_pass_a_mixed(BatchDev b) {
    const int t = blockIdx.x;
    if (t >= b.nztiles) return;   // no tiles left: the grid is one idle CTA
    const Tile tile = b.ztiles[t];
    const Ctl& ctl = b.ctls[tile.inst];
    if (inst_skip(ctl)) return;   // uniform over the CTA
    const HydroConst& c = b.consts[tile.inst];
    const int cur = ctl.cycle & 1;
    const double dt = ctl.dt;
    __shared__ double2 s_sfp[4 * kBatchZT];
    __shared__ float2 s_sft[4 * kBatchZT];
    const SideSpill sp{s_sfp, s_sft, (int)threadIdx.x};
    double fold = 1.e99;
    int nbad = 0;
    for (int zb = tile.beg; zb < tile.end; zb += kBatchZT) {
        const int64_t z = (int64_t)zb + threadIdx.x;
        if (z >= tile.end) continue;
        double v = 1.e99;
        int cnt[3] = {0, 0, 0};
        if (kAllQuads || tile.quads) {
            const fp64::GlobalZoneIn in{b.a, cur, z, 4 * z};
            pass_a_mixed_zone<4, false>(b.a, c, in, cur, dt, z, 4 * z, v, nbad, cnt, sp);
        } else {
            const int n = b.a.znump[z];
            const int64_t s0 = b.a.zfirst[z];
            const fp64::GlobalZoneIn in{b.a, cur, z, s0};
            if (n == 4) pass_a_mixed_zone<4, false>(b.a, c, in, cur, dt, z, s0, v, nbad, cnt, sp);
            else pass_a_mixed_zone<3, false>(b.a, c, in, cur, dt, z, s0, v, nbad, cnt, sp);
        }
        fold = dmin(fold, v);
    }
    nbad = tiles::block_isum<kBatchZT>(nbad);
    block_fold<true, kBatchZT>(fold, b.a.part_dtnew + t);
    if (threadIdx.x == 0) b.a.part_badA[t] = nbad;
}

__global__ void __launch_bounds__(kBatchThreads) batch_point_pass_mixed(BatchDev b) {
    for (int t = blockIdx.x; t < b.nptiles; t += gridDim.x) {
        const Tile tile = b.ptiles[t];
        const Ctl& ctl = b.ctls[tile.inst];
        if (inst_skip(ctl)) continue;
        const HydroConst& c = b.consts[tile.inst];
        const int cur = ctl.cycle & 1;
        for (int64_t p = (int64_t)tile.beg + threadIdx.x; p < tile.end; p += kBatchThreads)
            pass_b_mixed_point(b.a, c, cur, ctl.dt, p);
    }
}

// ---------------------------------------------------------------------
// Closure pass (learned cycle): the zones pass A recorded, each CTA an
// equal contiguous share, rounds of 128 zones (two corners a thread, up to
// 512 packed rows in runs of 256).
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(kCpThreads, kCpCtasPerSm) closure_pass(DevArrays a, HydroConst c) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ unsigned s_ncls[3];
    __shared__ int s_nrow;
    if (threadIdx.x < 3) s_ncls[threadIdx.x] = 0u;
    if (threadIdx.x == 0) s_nrow = 0;
    // the image and the tensor memory need nothing from pass A: set up while
    // it drains
    MlpState st;
    closure_mlp_setup(smem, a.closure_img, reinterpret_cast<uint64_t*>(smem + kCpBar),
                      reinterpret_cast<uint32_t*>(smem + kCpBar + 8), kCpTmemCols, st);   // publishes the zeros
    pdl_wait();
    const int nrec = skip_cycle(a.ctl) ? 0 : *a.closure_nrec;
    const int chunk = (nrec + (int)gridDim.x - 1) / (int)gridDim.x;
    const int zb = (int)blockIdx.x * chunk;
    const int ze = min(nrec, zb + chunk);
    const ClosureCtx cx{smem, smem + kCpA0, smem + kCpH, &s_nrow, s_ncls};
    const float4* recs = reinterpret_cast<const float4*>(a.closure_rec);
    auto rec_at = [&](int i) { return recs + (int64_t)i * kZoneRecF4; };
    for (int zr = zb; zr < ze; zr += 128) closure_round<2>(a, c, cx, st, rec_at, zr, min(128, ze - zr));
    const bool ok = closure_mlp_teardown(st);   // its barrier orders the counters
    if (threadIdx.x == 0 && !ok) atomicAdd(a.closure_counts + kClassErr * 64, 1ull);
    closure_add_counts(a, s_ncls, ze > zb ? ze - zb : 0);
}

}  // namespace

namespace {

cudaError_t launch_cycle_mixed_impl(const DevArrays& a, const HydroConst& c, cudaStream_t stream, cudaEvent_t* ev,
                                    bool learned, int phases) {
    const int pb = (int)((a.nump + kPointThreads - 1) / kPointThreads);
    const int zba = (int)((a.numz + kZoneThreadsZT - 1) / kZoneThreadsZT);
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    if (phases & kPhaseForces) {
        if (ev) cudaEventRecord(ev[0], stream);
        if (a.rect_nzx > 0) {
            chk(launch_pdl(learned ? pass_a_mixed_rows<true> : pass_a_mixed_rows<false>, a.gridA, kRowsAT, kRowsASmem,
                           stream, a, c));
        } else {
            auto k = learned ? (a.quads ? pass_a_mixed_zt<true, true> : pass_a_mixed_zt<false, true>)
                             : (a.quads ? pass_a_mixed_zt<true, false> : pass_a_mixed_zt<false, false>);
            chk(launch_pdl(k, zba, kZoneThreadsZT, 0, stream, a, c));
        }
        if (ev) cudaEventRecord(ev[1], stream);
        if (learned) chk(launch_pdl(closure_pass, a.closure_grid, kCpThreads, kCpSmemBytes, stream, a, c));
        if (ev) cudaEventRecord(ev[2], stream);
    }
    if (phases & kPhaseAdvance) {
        chk(launch_pdl(a.rect_nzx > 0 ? pass_b_mixed<true> : pass_b_mixed<false>, pb, kPointThreads, 0, stream, a,
                       c));
        if (ev) cudaEventRecord(ev[3], stream);
        launch_pass_c(a, c, true, stream);   // its last CTA ends the cycle
        if (ev) cudaEventRecord(ev[4], stream);
        if (ev) cudaEventRecord(ev[5], stream);   // no separate finalize step
    }
    return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace

cudaError_t launch_cycle_mixed(const DevArrays& a, const HydroConst& c, cudaStream_t stream, cudaEvent_t* ev,
                               int phases) {
    return launch_cycle_mixed_impl(a, c, stream, ev, false, phases);
}

cudaError_t launch_cycle_learned(const DevArrays& a, const HydroConst& c, cudaStream_t stream, cudaEvent_t* ev,
                                 int phases) {
    return launch_cycle_mixed_impl(a, c, stream, ev, true, phases);
}

cudaError_t prepare_pass_a_rows_mixed(bool learned, int32_t rect_nzx, int32_t numz, int nsm, int32_t* grid) {
    const int64_t nt = rows::num_tiles<kRowsAT>(rect_nzx, numz);
    return learned ? rows::prepare(pass_a_mixed_rows<true>, kRowsAT, kRowsASmem, nt, nsm, grid)
                   : rows::prepare(pass_a_mixed_rows<false>, kRowsAT, kRowsASmem, nt, nsm, grid);
}

void launch_batch_pass_a_mixed(const BatchDev& b, bool all_quads, cudaStream_t stream) {
    const int grid = b.nztiles > 1 ? b.nztiles : 1;
    if (all_quads) batch_pass_a_mixed<true><<<grid, kBatchZT, 0, stream>>>(b);
    else batch_pass_a_mixed<false><<<grid, kBatchZT, 0, stream>>>(b);
}

void launch_batch_point_pass_mixed(const BatchDev& b, int grid, cudaStream_t stream) {
    batch_point_pass_mixed<<<grid, kBatchThreads, 0, stream>>>(b);
}

cudaError_t prepare_learned_kernels() {
    return cudaFuncSetAttribute(closure_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, kCpSmemBytes);
}

}  // namespace pnt
