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
// point pass are stored in FP32 (4 + 8 B per side instead of 24 B).  Compiled with fast math; the accuracy of this path is stated as
// its L1 error against the FP64 run (tests/test_gpu_mixed.py).
#include "closure_dev.cuh"
#include "hydro_dev.h"

#include <cuda_runtime.h>

namespace pnt {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double2 add(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 sub(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 smul(double r, double2 v) { return mk(v.x * r, v.y * r); }
__device__ __forceinline__ double2 neg(double2 a) { return mk(-a.x, -a.y); }
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

__device__ __forceinline__ double shfl(double v, int src) { return __shfl_sync(kFull, v, src); }
__device__ __forceinline__ float shflf(float v, int src) { return __shfl_sync(kFull, v, src); }
__device__ __forceinline__ double2 shfl2(double2 v, int src) {
    return mk(__shfl_sync(kFull, v.x, src), __shfl_sync(kFull, v.y, src));
}
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

// QCS side force of one zone in FP64 (QCS.cc:116-380), for zones with an
// acute corner: there sfq is a small difference of large terms (cw grows as
// 1/sin^2 of the corner angle) that FP32 cannot carry.  All lanes of the
// warp must call it (it shuffles).
__device__ double2 qcs_sfq_fp64(double2 xp, double2 xp2, double2 zxp, double2 u0, double rn, int g, int n,
                                int lp, int ln, double zss, double zrp, const HydroConst& c) {
    const double2 u02 = shfl2(u0, ln), upp = shfl2(u0, lp);
    const double2 zuc = mk(zsum4(u0.x * rn, g, n), zsum4(u0.y * rn, g, n));
    const double2 ex = smul(0.5, add(xp, xp2));
    const double2 xq3 = shfl2(ex, lp);
    const double2 d = sub(xp2, xp);
    const double elen = sqrt(dot(d, d));
    const double de1 = shfl(elen, lp), de2 = elen;
    const double2 up0 = u0, xq0 = xp, xq1 = ex, up2 = zuc, xq2 = zxp;
    const double2 up1 = smul(0.5, add(up0, u02));
    const double2 up3 = smul(0.5, add(upp, up0));
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
    const double2 cqe1 = smul(crmu / de1, sub(up0, upp));
    const double2 cqe2 = smul(crmu / de2, sub(u02, up0));
    const double csin2 = 1.0 - ccos * ccos;
    const double cw = (csin2 < 1.e-4) ? 0. : cvolume / csin2;
    ccos = (csin2 < 1.e-4) ? 0. : ccos;
    const double cw2 = shfl(cw, ln), ccos2 = shfl(ccos, ln);
    const double2 cqe12 = shfl2(cqe1, ln), cqe22 = shfl2(cqe2, ln);
    return smul(1. / elen, add(smul(cw, add(cqe2, smul(ccos, cqe1))), smul(cw2, add(cqe12, smul(ccos2, cqe22)))));
}

// ---------------------------------------------------------------------
// Pass A, mixed precision
// ---------------------------------------------------------------------
#ifndef PNT_LEARNED_A_MIN_BLOCKS
#define PNT_LEARNED_A_MIN_BLOCKS 4
#endif
#ifndef PNT_MIXED_A_MIN_BLOCKS
#define PNT_MIXED_A_MIN_BLOCKS 4
#endif
template <bool kQuads, bool kLearned>
__global__ void __launch_bounds__(kZoneThreads, kLearned ? PNT_LEARNED_A_MIN_BLOCKS : PNT_MIXED_A_MIN_BLOCKS)
    pass_a_mixed(DevArrays a, HydroConst c) {
    const Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const int cur = ctl->cycle & 1;
    const double dt = ctl->dt;
    const double2* __restrict__ px0 = a.px[cur];
    const double2* __restrict__ pu0 = a.pu[cur];

    const int64_t tid = (int64_t)blockIdx.x * kZoneThreads + threadIdx.x;
    const int64_t z = tid >> 2;
    const int k = (int)(tid & 3);
    const int lane = threadIdx.x & 31;
    const int g = lane & ~3;
    const bool zok = z < a.numz;
    int n = 4;
    int64_t s = 4 * z + k;
    if (!kQuads) {
        n = zok ? a.znump[z] : 4;
        s = (zok ? (int64_t)a.zfirst[z] : 0) + k;
    }
    const bool act = zok && k < n;
    const int lp = g + (k == 0 ? n - 1 : k - 1);
    const int ln = g + (k + 1 >= n ? 0 : k + 1);

    const int32_t p1 = act ? __ldg(a.mapsp1 + s) : 0;
    const double2 x0 = act ? px0[p1] : mk(0., 0.);
    const double2 u0 = act ? pu0[p1] : mk(0., 0.);
    const double mf = act ? __ldg(a.smf + s) : 0.;
    const double zm = zok ? a.zm[z] : 1.;
    const double zr = zok ? a.zr[z] : 1.;
    const double ze = zok ? a.ze[z] : 0.;
    const double zwrate = zok ? a.zwrate[z] : 0.;
    const double zvol0 = zok ? a.zvol[z] : 1.;

    // FP64: positions, zone centre, side areas and volumes
    const double dth = 0.5 * dt;
    const double2 xp = add(x0, smul(dth, u0));
    const double2 xp2 = shfl2(xp, ln);
    const double rn = 1. / (double)n;
    const double2 zxp = mk(zsum4(xp.x * rn, g, n), zsum4(xp.y * rn, g, n));
    const double third = 1. / 3.;
    const double sa = 0.5 * cross(sub(xp2, xp), sub(zxp, xp));
    const double sv = third * sa * (xp.x + xp2.x + zxp.x);
    const double zareap = zsum4(sa, g, n);
    const double zvolp = zsum4(sv, g, n);
    const bool bad = act && (sv <= 0.);

    // FP64 zone EOS and density (PolyGas.cc:63-109, Hydro.cc:1034-1054),
    // quotients split over the zone's lanes
    const double e = dmax(ze, 0.);
    const double p = c.gm1 * zr * e;
    const double pre = c.gm1 * e;
    const double per = c.gm1 * zr;
    const double rA = ((k == 0) ? per * p : 1.) / ((k == 0) ? zr * zr : zm);
    const double q = shfl(rA, g);
    const double minv = shfl(rA, g + 1);
    const double csqd = dmax(c.ssmin2, pre + q);
    const double zss = sqrt(csqd);
    const double dv = (zvolp - zvol0) * minv;
    const double bulk = zr * csqd;
    const double denom = 1. + 0.5 * per * dv;
    const double src = zwrate * dth * minv;
    const double rB = ((k == 0) ? zm : per * src - zr * bulk * dv) / ((k == 0) ? zvolp : denom);
    const double zrp = shfl(rB, g);
    const double zp = p + shfl(rB, g + 1);
    const double mf3 = shfl(mf, lp);
    if (act) a.cmass_f[s] = (float)(zrp * zareap * 0.5 * (mf + mf3));
    if (zok && k == 0) a.zp[z] = zp;

    // FP32 from here, relative to the zone's first point
    const double2 xref = shfl2(xp, g);
    const float2 r = f2(sub(xp, xref));
    const float2 r2 = shflf2(r, ln);
    const float2 zc = f2(sub(zxp, xref));
    // velocities relative to the zone's first point as well: QCS works on
    // velocity differences, which absolute FP32 values would round away
    const double2 uref = shfl2(u0, g);
    const float2 uf = f2(sub(u0, uref));
    const float2 u2f = shflf2(uf, ln);
    const float2 upf = shflf2(uf, lp);
    const float rnf = (float)rn;
    const float2 zuc = fk(zsum4(uf.x * rnf, g, n), zsum4(uf.y * rnf, g, n));
    const float2 ex = fmul(0.5f, fadd(r, r2));
    const float2 ssurf = fk(-(ex.y - zc.y), ex.x - zc.x);
    const float elen = flen(fsub(r2, r));
    const float saf = (float)sa;
    const float fac = (n == 3 ? 3.f : 4.f);
    // zone minimum over the group's 4 lanes; the idle lane of a triangle
    // contributes +inf
    float zdl = act ? fac * saf / elen : __int_as_float(0x7f800000);
    zdl = fminf(zdl, __shfl_xor_sync(kFull, zdl, 1));
    zdl = fminf(zdl, __shfl_xor_sync(kFull, zdl, 2));
    const float rinv_el = 1.f / elen;

    const float zssf = (float)zss, zrpf = (float)zrp;
    // PolyGas::calcForce in FP64: the pressure forces of a zone cancel
    // around its closed boundary, and calcWork takes the small residual of
    // their work on moving points; FP32 surface vectors break that
    // cancellation
    const double2 ex64 = smul(0.5, add(xp, xp2));
    const double2 sfp = smul(-zp, mk(-(ex64.y - zxp.y), ex64.x - zxp.x));
    // TTS (TTS.cc:55-104)
    const float srho = zrpf * (float)mf * ((float)zareap / saf);
    float sstmp = fmaxf(zssf, (float)c.tts_ssmin);
    sstmp = (float)c.alfa * sstmp * sstmp;
    const float2 sft = fmul(-(sstmp * (srho - zrpf)), ssurf);

    // QCS corner (QCS.cc:116-380), FP32
    const float2 up0 = uf, xq0 = r;
    const float2 up1 = fmul(0.5f, fadd(up0, u2f));
    const float2 xq1 = ex;
    const float2 up2 = zuc, xq2 = zc;
    const float2 up3 = fmul(0.5f, fadd(upf, up0));
    const float2 xq3 = shflf2(ex, lp);
    const float cvolume = 0.5f * fcross(fsub(xq2, xq0), fsub(xq3, xq1));
    const float2 v1 = fsub(xq3, xq0), v2 = fsub(xq1, xq0);
    const float de1 = shflf(elen, lp), de2 = elen;
    const float rinv_de1 = shflf(rinv_el, lp);
    const float minelen = fminf(de1, de2);
    float ccos = (minelen < 1.e-12f) ? 0.f : 4.f * fdot(v1, v2) / (de1 * de2);
    const float cdiv = (fcross(fsub(up2, up0), fsub(xq3, xq1)) - fcross(fsub(up3, up1), fsub(xq2, xq0))) /
                       (2.f * cvolume);
    // sin^2 of the corner angle.  The reference forms 1 - ccos^2, which in
    // FP32 loses the small sines of the acute corners of thin zones (3-degree
    // corners at the centre of a pie mesh); v1 and v2 run to the edge
    // midpoints, |v_i| = de_i / 2, so (4 cross / (de1 de2))^2 is the same
    // quantity without the cancellation.  Zones with a corner under ~30
    // degrees take the FP64 form (warp-uniform branch; never taken on
    // rectangular meshes).  The learned cycle needs the flag before the
    // corner forces, the plain one after them (fewer live registers).
    float csin2 = 1.f;
    int acute = 0;
    auto corner_sin2 = [&]() {
        const float ssin = 4.f * fcross(v1, v2) / (de1 * de2);
        csin2 = (minelen < 1.e-12f) ? 1.f : ssin * ssin;
        acute = (act && csin2 < 0.25f) ? 1 : 0;
        acute |= __shfl_xor_sync(kFull, acute, 1);
        acute |= __shfl_xor_sync(kFull, acute, 2);
    };
    if constexpr (kLearned) corner_sin2();

    // The learned cycle (closure_dev.cuh) forms no QCS corner force here:
    // compressing corners outside the dead zone are deferred (their zones
    // recorded with the corners' raw data) to the closure pass, which runs
    // the network or, past its range, the plain QCS; the rest carry none.
    // Zones with an acute corner keep the FP64 QCS below.
    bool plain = cdiv < 0.f;
    int cls = kClassZero;
    if constexpr (kLearned) {
        plain = false;
        const float dead = __ldg(reinterpret_cast<const float*>(a.closure_img + kImgThr));
        // dead-zone test on squares (closure_features' first step)
        const float2 d1 = fsub(uf, upf), d2 = fsub(u2f, uf), dc = fsub(zuc, uf);
        const float m2 = fmaxf(fmaxf(flen2(d1), flen2(d2)), flen2(dc));
        const float lim = dead * zssf;
        if (act && acute) cls = kClassAcute;
        else if (act && cdiv < 0.f) cls = (m2 > lim * lim) ? kClassMlp : kClassDead;   // kClassMlp: deferred
        const bool defer = cls == kClassMlp;
        int zflag = defer ? 1 : 0;
        zflag |= __shfl_xor_sync(kFull, zflag, 1);
        zflag |= __shfl_xor_sync(kFull, zflag, 2);
        const float2 xpp = shflf2(r, lp);
        const unsigned zbits = __ballot_sync(kFull, zflag && k == 0);
        int base = 0;
        if (lane == 0 && zbits) base = atomicAdd(a.closure_nrec, __popc(zbits));
        base = __shfl_sync(kFull, base, 0);
        if (zflag) {
            const int idx = base + __popc(zbits & ((1u << g) - 1u));
            float4* rec = reinterpret_cast<float4*>(a.closure_rec + ((int64_t)idx * 4 + k) * kRecFloats);
            const float2 uav = fadd(fmul(0.25f, fadd(fadd(fadd(up0, up1), up2), up3)), f2(uref));
            rec[0] = make_float4(r.x, r.y, xpp.x, xpp.y);
            rec[1] = make_float4(r2.x, r2.y, zc.x, zc.y);
            rec[2] = make_float4(uf.x, uf.y, upf.x, upf.y);
            rec[3] = make_float4(u2f.x, u2f.y, zuc.x, zuc.y);
            rec[4] = make_float4(uav.x, uav.y, zssf, zrpf);
            rec[5] = make_float4(defer ? 1.f : 0.f, 0.f, 0.f, 0.f);
            if (k == 0) a.closure_zhdr[idx] = make_int2((int)(s - k), n);
        }
    }
    float crmu = 0.f;
    if (plain) {
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
    const float2 cqe1 = fmul(crmu * rinv_de1, fsub(up0, upf));
    const float2 cqe2 = fmul(crmu * rinv_el, fsub(u2f, up0));
    if constexpr (!kLearned) corner_sin2();
    const float cw = (csin2 < 1.e-4f) ? 0.f : cvolume / csin2;
    ccos = (csin2 < 1.e-4f) ? 0.f : ccos;
    const float cw2 = shflf(cw, ln), ccos2 = shflf(ccos, ln);
    const float2 cqe12 = shflf2(cqe1, ln), cqe22 = shflf2(cqe2, ln);
    float2 sfq = fmul(rinv_el, fadd(fmul(cw, fadd(cqe2, fmul(ccos, cqe1))),
                                    fmul(cw2, fadd(cqe12, fmul(ccos2, cqe22)))));
    if (__any_sync(kFull, acute)) {
        const double2 q = qcs_sfq_fp64(xp, xp2, zxp, u0, rn, g, n, lp, ln, zss, zrp, c);
        if (acute) sfq = f2(q);
    }

    // QCS::setVelDiff, calcDtNew (FP64 reduction)
    float dux = fabsf(fdot(fsub(u2f, uf), fsub(r2, r))) * rinv_el;
    dux = (act && elen > 0.f) ? dux : 0.f;
    float ztmp = fmaxf(dux, __shfl_xor_sync(kFull, dux, 1));
    ztmp = fmaxf(ztmp, __shfl_xor_sync(kFull, ztmp, 2));   // idle triangle lanes carry 0
    const double zdu = c.q1 * zss + 2. * c.q2 * (double)ztmp;
    const double cdu = dmax(zdu, dmax(zss, 1.e-99));
    const double zdthyd = zok ? (double)zdl * c.cfl / cdu : 1.e99;

    const double2 sfpq = add(sfp, mk((double)sfq.x, (double)sfq.y));
    const double2 ftot = add(sfpq, mk((double)sft.x, (double)sft.y));
    const double2 ftot3 = shfl2(ftot, lp);
    if (act) {
        a.cforce_f[s] = f2(sub(ftot, ftot3));
        a.sftot[s] = sfpq;
    }

    // pass A counts the corners without compression, in the dead zone and in
    // acute zones; the closure pass counts the deferred ones by class
    constexpr int kCounted[3] = {kClassZero, kClassDead, kClassAcute};
    __shared__ unsigned wcount[kLearned ? kZoneThreads / 32 : 1][3];
    if constexpr (kLearned) {
        for (int q = 0; q < 3; ++q) {
            const unsigned nq = __popc(__ballot_sync(kFull, act && cls == kCounted[q]));
            if (lane == 0) wcount[threadIdx.x >> 5][q] = nq;
        }
    }

    const int nbad = __syncthreads_count(bad);
    if constexpr (kLearned) {
        if (threadIdx.x < 3) {
            unsigned t = 0;
            for (int w = 0; w < kZoneThreads / 32; ++w) t += wcount[w][threadIdx.x];
            if (t) atomicAdd(a.closure_counts + kCounted[threadIdx.x] * 64 + (blockIdx.x & 63), (unsigned long long)t);
        }
    }
    if (blockIdx.x >= (unsigned)a.npartA) return;   // partials are sized for this grid
    block_fold<true, kZoneThreads>(zdthyd, a.part_dtnew + blockIdx.x);
    if (threadIdx.x == 0) a.part_badA[blockIdx.x] = nbad;
}

// ---------------------------------------------------------------------
// Pass B, mixed: FP32 corner inputs summed in FP64
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(kPointThreads) pass_b_mixed(DevArrays a, HydroConst c) {
    const Ctl* ctl = a.ctl;
    // the closure pass has consumed this cycle's zone records
    if (a.closure_nrec && blockIdx.x == 0 && threadIdx.x == 0) *a.closure_nrec = 0;
    if (skip_cycle(ctl)) return;
    const int64_t p = (int64_t)blockIdx.x * kPointThreads + threadIdx.x;
    if (p >= a.nump) return;
    const int cur = ctl->cycle & 1;
    const double dt = ctl->dt;
    const double2 x0 = a.px[cur][p];
    double2 u0 = a.pu[cur][p];
    const int32_t o0 = a.poff[p], o1 = a.poff[p + 1];
    double m = 0.;
    double2 f = mk(0., 0.);
    for (int32_t i = o0; i < o1; ++i) {
        const int32_t s = __ldg(a.pcorner + i);
        m += (double)a.cmass_f[s];
        const float2 cf = a.cforce_f[s];
        f = mk(f.x + (double)cf.x, f.y + (double)cf.y);
    }
    const unsigned mask = a.bcmask[p];
    if (mask) {
        for (int b = 0; b < c.nbc; ++b) {
            if (mask & (1u << b)) {
                u0 = project(u0, c.vfix[b][0], c.vfix[b][1]);
                f = project(f, c.vfix[b][0], c.vfix[b][1]);
            }
        }
    }
    const double minv = 1. / dmax(m, 1.e-99);
    const double2 pa = mk(f.x * minv, f.y * minv);
    const double2 u = add(u0, smul(dt, pa));
    const double2 x = add(x0, smul(dt * 0.5, add(u0, u)));
    a.px[cur ^ 1][p] = x;
    a.pu[cur ^ 1][p] = u;
}

// ---------------------------------------------------------------------
// Closure pass (learned cycle): the deferred corners of the zones pass A
// recorded, 64 zones (256 corners) per batch, persistent.  Each deferred
// corner is classified (compression past rho_max or inputs out of
// distribution: plain QCS, QCS.cc:116-327 in FP32 as in the mixed pass A;
// otherwise the network, tcgen05, closure_dev.cuh); a tile without network
// corners skips the network.  A corner's QCS forces cqe1, cqe2 enter
// QCS::setForce (QCS.cc:331-380) linearly: its side s gets
// d1 = cw (cqe2 + ccos cqe1) / elen[s] and the previous side
// d2 = cw (cqe1 + ccos cqe2) / elen[s3].  The corner force of side s,
// ftot[s] - ftot[s3] (Hydro.cc:1159-1193), and sfp + sfq of side s then
// change by
//   dcforce[s] = d1(s) - d2(s) - d1(s3) + d2(s4),  dsftot[s] = d1(s) + d2(s4),
// which only touch the recorded zone's own sides: no two records write the
// same side, so the update is deterministic without atomics.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(kMlpRows, 3) closure_pass(DevArrays a, HydroConst c) {
    if (skip_cycle(a.ctl)) return;
    const int nrec = *a.closure_nrec;
    if (blockIdx.x == 0 && threadIdx.x == 0 && nrec)
        atomicAdd(a.closure_counts + kClassZones * 64, (unsigned long long)nrec);
    if ((int64_t)blockIdx.x * 64 >= nrec) return;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ unsigned ccount[3];   // network, fallback, out of distribution
    if (threadIdx.x < 3) ccount[threadIdx.x] = 0u;
    MlpState st;
    closure_mlp_setup(smem, a.closure_img, st);   // its barrier publishes ccount's zeros
    const float* thr = reinterpret_cast<const float*>(smem + kImgThr);
    const float rho_max = thr[1], kappa = thr[2];
    const int mode = (int)thr[3];   // 0 network, 1 no force, 2 plain QCS
    const float* mean = reinterpret_cast<const float*>(smem + kImgFMean);
    const float* istd = reinterpret_cast<const float*>(smem + kImgFIstd);
    const float qa = (float)(c.q2 * 0.25 * c.gammap1), qb = (float)c.q1;
    const int k = threadIdx.x & 3, lane = threadIdx.x & 31, g = lane & ~3;
    for (int tile = blockIdx.x; (int64_t)tile * 64 < nrec; tile += gridDim.x) {
        const int zi = tile * 64 + (threadIdx.x >> 2);
        const bool zok = zi < nrec;
        float v[kRecFloats];
        const float4* rec = reinterpret_cast<const float4*>(a.closure_rec + ((int64_t)zi * 4 + k) * kRecFloats);
#pragma unroll
        for (int i = 0; i < kRecFloats / 4; ++i) {
            const float4 q = zok ? rec[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            v[4 * i] = q.x;
            v[4 * i + 1] = q.y;
            v[4 * i + 2] = q.z;
            v[4 * i + 3] = q.w;
        }
        const int2 hdr = zok ? a.closure_zhdr[zi] : make_int2(0, 4);
        const float2 x = fk(v[kRecX], v[kRecX + 1]), xpv = fk(v[kRecXp], v[kRecXp + 1]);
        const float2 xn = fk(v[kRecXn], v[kRecXn + 1]), xz = fk(v[kRecXz], v[kRecXz + 1]);
        const float2 u = fk(v[kRecU], v[kRecU + 1]), upv = fk(v[kRecUp], v[kRecUp + 1]);
        const float2 un = fk(v[kRecUn], v[kRecUn + 1]), uz = fk(v[kRecUz], v[kRecUz + 1]);
        const float2 uav = fk(v[kRecUav], v[kRecUav + 1]);
        const float css = v[kRecSs], rho = v[kRecRho];
        // classify the deferred corners
        int cls = -1;
        float f[kClIn];
        float cx = 0.f, cy = 0.f, scale = 0.f;
        if (v[kRecFlag] != 0.f &&
            closure_features<float>({x.x, x.y}, {xpv.x, xpv.y}, {xn.x, xn.y}, {xz.x, xz.y}, {u.x, u.y},
                                    {upv.x, upv.y}, {un.x, un.y}, {uz.x, uz.y}, {uav.x, uav.y}, css, qa, qb, 0.f,
                                    f, cx, cy, scale)) {
            if (f[11] > rho_max) cls = kClassFallback;
            else {
                float zmax = 0.f;
#pragma unroll
                for (int i = 0; i < kClIn; ++i) zmax = fmaxf(zmax, fabsf((f[i] - mean[i]) * istd[i]));
                cls = (zmax > kappa) ? kClassOod : kClassMlp;
            }
        }
        const bool net = cls == kClassMlp && mode == 0;
        const bool plain = cls == kClassFallback || cls == kClassOod || (cls == kClassMlp && mode == 2);
        {
            const unsigned nm = __popc(__ballot_sync(kFull, cls == kClassMlp));
            const unsigned nf = __popc(__ballot_sync(kFull, cls == kClassFallback));
            const unsigned no = __popc(__ballot_sync(kFull, cls == kClassOod));
            if (lane == 0) {
                if (nm) atomicAdd(&ccount[0], nm);
                if (nf) atomicAdd(&ccount[1], nf);
                if (no) atomicAdd(&ccount[2], no);
            }
        }
        if (!net) {
#pragma unroll
            for (int i = 0; i < kClIn; ++i) f[i] = 0.f;
        }
        float y[4] = {0.f, 0.f, 0.f, 0.f};
        if (__syncthreads_or(net)) closure_mlp_rows(smem, st, f, y);
        // corner geometry (QCS::setCornerDiv / setForce, FP32 as in pass A)
        const float2 ex = fmul(0.5f, fadd(x, xn));
        const float2 xq3 = fmul(0.5f, fadd(xpv, x));
        const float cvolume = 0.5f * fcross(fsub(xz, x), fsub(xq3, ex));
        const float2 v1 = fsub(xq3, x), v2 = fsub(ex, x);
        const float de1 = flen(fsub(x, xpv)), de2 = flen(fsub(xn, x));
        const float rinv_de1 = 1.f / de1, rinv_el = 1.f / de2;
        const float minelen = fminf(de1, de2);
        float ccos = (minelen < 1.e-12f) ? 0.f : 4.f * fdot(v1, v2) / (de1 * de2);
        float2 q1 = fk(0.f, 0.f), q2 = fk(0.f, 0.f);
        if (net) {
            const float sc = rho * scale;
            q1 = fk((cx * y[0] - cy * y[1]) * sc, (cy * y[0] + cx * y[1]) * sc);
            q2 = fk((cx * y[2] - cy * y[3]) * sc, (cy * y[2] + cx * y[3]) * sc);
        } else if (plain) {
            const float2 up1 = fmul(0.5f, fadd(u, un)), up3 = fmul(0.5f, fadd(upv, u));
            const float2 dxx1 = fmul(0.5f, fsub(fsub(fadd(ex, xz), x), xq3));
            const float2 dxx2 = fmul(0.5f, fsub(fsub(fadd(xz, xq3), x), ex));
            const float dx1 = flen(dxx1), dx2 = flen(dxx2);
            const float test1 = fabsf(fdot(dxx1, uav) * dx2);
            const float test2 = fabsf(fdot(dxx2, uav) * dx1);
            const float rr = (test1 > test2) ? dx1 / dx2 : dx2 / dx1;
            const float evol = fminf(sqrtf(4.f * cvolume * rr), 2.f * minelen);
            const float du = sqrtf(fmaxf(flen2(fsub(fsub(fadd(up1, uz), u), up3)),
                                         flen2(fsub(fsub(fadd(uz, up3), u), up1))));
            const float ztmp2 = qa * du;
            const float ztmp1 = qb * css;
            const float crmu = (ztmp2 + sqrtf(ztmp2 * ztmp2 + ztmp1 * ztmp1)) * rho * evol;
            q1 = fmul(crmu * rinv_de1, fsub(u, upv));
            q2 = fmul(crmu * rinv_el, fsub(un, u));
        }
        const float ssin = 4.f * fcross(v1, v2) / (de1 * de2);
        const float csin2 = (minelen < 1.e-12f) ? 1.f : ssin * ssin;
        const float cw = (csin2 < 1.e-4f) ? 0.f : cvolume / csin2;
        ccos = (csin2 < 1.e-4f) ? 0.f : ccos;
        const int n = hdr.y;
        const int lp = g + (k == 0 ? n - 1 : k - 1);
        const int ln = g + (k + 1 >= n ? 0 : k + 1);
        const float2 d1 = fmul(cw * rinv_el, fadd(q2, fmul(ccos, q1)));
        const float2 d2 = fmul(cw * rinv_de1, fadd(q1, fmul(ccos, q2)));
        const float2 d1p = shflf2(d1, lp);
        const float2 d2n = shflf2(d2, ln);
        if (zok && k < n) {
            const int64_t sd = (int64_t)hdr.x + k;
            const float2 cf = a.cforce_f[sd];
            a.cforce_f[sd] = fadd(cf, fadd(fsub(d1, d2), fsub(d2n, d1p)));
            const double2 sf = a.sftot[sd];
            const float2 ds = fadd(d1, d2n);
            a.sftot[sd] = mk(sf.x + (double)ds.x, sf.y + (double)ds.y);
        }
    }
    const bool ok = closure_mlp_teardown(st);
    if (threadIdx.x == 0 && !ok) atomicAdd(a.closure_counts + kClassErr * 64, 1ull);
    if (threadIdx.x < 3 && ccount[threadIdx.x]) {
        const int q = threadIdx.x == 0 ? kClassMlp : (threadIdx.x == 1 ? kClassFallback : kClassOod);
        atomicAdd(a.closure_counts + q * 64 + (blockIdx.x & 63), (unsigned long long)ccount[threadIdx.x]);
    }
}

// ---------------------------------------------------------------------
// Pass C, mixed: FP64 corrector with the FP32 sfp + sfq input
// ---------------------------------------------------------------------
template <bool kQuads>
__global__ void __launch_bounds__(kZoneThreadsC) pass_c_mixed(DevArrays a, HydroConst c) {
    const Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const int cur = ctl->cycle & 1;
    const double dt = ctl->dt;
    const int64_t tid = (int64_t)blockIdx.x * kZoneThreadsC + threadIdx.x;
    const int64_t z = tid >> 2;
    const int k = (int)(tid & 3);
    const int lane = threadIdx.x & 31;
    const int g = lane & ~3;
    const bool zok = z < a.numz;
    int n = 4;
    int64_t s = 4 * z + k;
    if (!kQuads) {
        n = zok ? a.znump[z] : 4;
        s = (zok ? (int64_t)a.zfirst[z] : 0) + k;
    }
    const bool act = zok && k < n;
    const int ln = g + (k + 1 >= n ? 0 : k + 1);

    const int32_t p1 = act ? __ldg(a.mapsp1 + s) : 0;
    const double2 x0 = act ? a.px[cur][p1] : mk(0., 0.);
    const double2 u0 = act ? a.pu[cur][p1] : mk(0., 0.);
    const double2 x = act ? a.px[cur ^ 1][p1] : mk(0., 0.);
    const double2 u = act ? a.pu[cur ^ 1][p1] : mk(0., 0.);
    const unsigned mask = act ? a.bcmask[p1] : 0u;
    const double2 sft = act ? a.sftot[s] : mk(0., 0.);
    const double zm = zok ? a.zm[z] : 1.;
    const double zetot0 = zok ? a.zetot[z] : 0.;
    const double zvol0 = zok ? a.zvol[z] : 1.;
    const double zp = zok ? a.zp[z] : 0.;

    const double dth = 0.5 * dt;
    const double2 xp = add(x0, smul(dth, u0));
    double2 u0b = u0;
    if (mask) {
        for (int b = 0; b < c.nbc; ++b)
            if (mask & (1u << b)) u0b = project(u0b, c.vfix[b][0], c.vfix[b][1]);
    }
    const double2 x2 = shfl2(x, ln);
    const double2 xp2 = shfl2(xp, ln);
    const double2 u0b2 = shfl2(u0b, ln);
    const double2 u2 = shfl2(u, ln);
    const double rn = 1. / (double)n;
    const double2 zx = mk(zsum4(x.x * rn, g, n), zsum4(x.y * rn, g, n));
    const double third = 1. / 3.;
    const double sa = 0.5 * cross(sub(x2, x), sub(zx, x));
    const double sv = third * sa * (x.x + x2.x + zx.x);
    const double zvol = zsum4(sv, g, n);
    const bool bad = act && (sv <= 0.);
    const double sd1 = dot(sft, add(u0b, u));
    const double sd2 = dot(neg(sft), add(u0b2, u2));
    const double dwork = -dth * (sd1 * xp.x + sd2 * xp2.x);
    const double zw = zsum4(dwork, g, n);
    const double zetot = zetot0 + zw;
    const double zwrate = (zw + zp * (zvol - zvol0)) * ctl->dtinv;
    const double qv = ((k == 0) ? zm : (k == 1 ? zetot : zvol - zvol0)) /
                      ((k == 0) ? zvol : (k == 1 ? zm + 1.e-99 : zvol0));
    const double zdvov = (zok && k == 2) ? fabs(qv) : 1.e-99;
    __syncwarp();
    if (zok) {
        if (k == 0) { a.zvol[z] = zvol; a.zr[z] = qv; }
        else if (k == 1) { a.zetot[z] = zetot; a.ze[z] = qv; }
        else if (k == 2) a.zwrate[z] = zwrate;
    }
    const int nbad = __syncthreads_count(bad);
    if (blockIdx.x >= (unsigned)a.npartC) return;   // partials are sized for this grid
    block_fold<false, kZoneThreadsC>(zdvov, a.part_dvov + blockIdx.x);
    if (threadIdx.x == 0) a.part_badC[blockIdx.x] = nbad;
}

}  // namespace

namespace {

cudaError_t launch_cycle_mixed_impl(const DevArrays& a, const HydroConst& c, cudaStream_t stream, cudaEvent_t* ev,
                                    bool learned) {
    const int zb = (int)zone_blocks(a.numz);
    const int zbc = (int)zone_blocks(a.numz, kZoneThreadsC);
    const int pb = (int)((a.nump + kPointThreads - 1) / kPointThreads);
    if (ev) cudaEventRecord(ev[0], stream);
    if (learned) {
        if (a.quads) pass_a_mixed<true, true><<<zb, kZoneThreads, 0, stream>>>(a, c);
        else pass_a_mixed<false, true><<<zb, kZoneThreads, 0, stream>>>(a, c);
        if (ev) cudaEventRecord(ev[1], stream);
        closure_pass<<<a.closure_grid, kMlpRows, kMlpSmemBytes, stream>>>(a, c);
    } else {
        if (a.quads) pass_a_mixed<true, false><<<zb, kZoneThreads, 0, stream>>>(a, c);
        else pass_a_mixed<false, false><<<zb, kZoneThreads, 0, stream>>>(a, c);
        if (ev) cudaEventRecord(ev[1], stream);
    }
    if (ev) cudaEventRecord(ev[2], stream);
    pass_b_mixed<<<pb, kPointThreads, 0, stream>>>(a, c);
    if (ev) cudaEventRecord(ev[3], stream);
    if (a.quads) pass_c_mixed<true><<<zbc, kZoneThreadsC, 0, stream>>>(a, c);
    else pass_c_mixed<false><<<zbc, kZoneThreadsC, 0, stream>>>(a, c);
    if (ev) cudaEventRecord(ev[4], stream);
    launch_finalize(a, c, zb, zbc, stream);
    if (ev) cudaEventRecord(ev[5], stream);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_cycle_mixed(const DevArrays& a, const HydroConst& c, cudaStream_t stream, cudaEvent_t* ev) {
    return launch_cycle_mixed_impl(a, c, stream, ev, false);
}

cudaError_t launch_cycle_learned(const DevArrays& a, const HydroConst& c, cudaStream_t stream, cudaEvent_t* ev) {
    return launch_cycle_mixed_impl(a, c, stream, ev, true);
}

cudaError_t prepare_learned_kernels() {
    return cudaFuncSetAttribute(closure_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, kMlpSmemBytes);
}

}  // namespace pnt
