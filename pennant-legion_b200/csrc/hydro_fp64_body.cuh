// hydro_fp64_body.cuh -- the FP64 hydro cycle's pass A zone body (one
// thread per zone), pass B point body and end-of-cycle step, shared by the
// single-mesh kernels (hydro_fp64.cu) and the batched persistent kernels
// (batch.cu) so both run exactly the same arithmetic; pass C's body is in
// pass_c_staged.cuh.  The four-lane helpers (zsum, shfl2) serve the
// closure harvest (closure.cu), whose four consecutive lanes form a zone.
//
// Every expression keeps the reference's operation order, including
// Vec2.hh's `v / r` = v * (1/r) (Vec2.hh:145-149); translation units that
// include this header are compiled with -fmad=false, so results match a
// serial CPU run of the reference bit for bit.
#pragma once

#include "hydro_dev.h"

#include <cuda_runtime.h>

namespace pnt {
namespace fp64 {

constexpr unsigned kFull = 0xffffffffu;

// ----- double2 arithmetic with the reference's semantics (Vec2.hh) ------
__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double2 add(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 sub(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 neg(double2 a) { return mk(-a.x, -a.y); }
__device__ __forceinline__ double2 smul(double r, double2 v) { return mk(v.x * r, v.y * r); }
__device__ __forceinline__ double2 sdiv(double2 v, double r) {
    const double rinv = 1. / r;
    return mk(v.x * rinv, v.y * rinv);
}
__device__ __forceinline__ double dot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ double cross(double2 a, double2 b) { return a.x * b.y - a.y * b.x; }
__device__ __forceinline__ double length(double2 v) { return sqrt(v.x * v.x + v.y * v.y); }
__device__ __forceinline__ double length2(double2 v) { return v.x * v.x + v.y * v.y; }
__device__ __forceinline__ double2 rotateCCW(double2 v) { return mk(-v.y, v.x); }
__device__ __forceinline__ double2 project(double2 v, double ux, double uy) {
    const double d = v.x * ux + v.y * uy;
    return mk(v.x - ux * d, v.y - uy * d);
}
// std::min / std::max: min(a,b) = (b < a) ? b : a, max(a,b) = (a < b) ? b : a
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

// x / y, with the division left out where IEEE 754 fixes its result without
// it: a zero dividend over a finite non-zero divisor gives a zero whose sign
// is the XOR of the operands' signs, which is exactly x * y; a divisor of 1
// gives x (NaN dividends excepted, whose payload a division may change).
// Every other case is the correctly rounded division.  In a quiescent part
// of the mesh (zero velocities, zero pressure) most of the QCS quotients
// take the first two branches.
__device__ __forceinline__ double xdiv(double x, double y) {
    if (x == 0.0 && fabs(y) < __longlong_as_double(0x7ff0000000000000LL) && y != 0.0) return x * y;
    if (y == 1.0 && x == x) return x;
    return x / y;
}
#ifndef PNT_FP64_XDIV
#define PNT_FP64_XDIV 1
#endif
#if PNT_FP64_XDIV
#define PNT_QDIV(x, y) xdiv((x), (y))
#else
#define PNT_QDIV(x, y) ((x) / (y))
#endif

__device__ __forceinline__ double shfl(double v, int src) { return __shfl_sync(kFull, v, src); }
__device__ __forceinline__ double2 shfl2(double2 v, int src) {
    return mk(__shfl_sync(kFull, v.x, src), __shfl_sync(kFull, v.y, src));
}

// Zone reductions over the group's lanes g..g+n-1 in side order, starting
// from 0.0 as the reference's zeroed accumulators do.
__device__ __forceinline__ double zsum(double v, int g, int n) {
    const double a = shfl(v, g), b = shfl(v, g + 1), c = shfl(v, g + 2), d = shfl(v, g + 3);
    double s = __dadd_rn(0.0, a);
    s = s + b;
    s = s + c;
    if (n == 4) s = s + d;
    return s;
}
__device__ __forceinline__ double2 zsum2(double2 v, int g, int n) {
    return mk(zsum(v.x, g, n), zsum(v.y, g, n));
}

__device__ __forceinline__ bool skip_cycle(const Ctl* ctl) {
    return ctl->done || ctl->cycle >= ctl->stop_at;
}

// Block-wide min (dt) / max (dvov) in the reference fold semantics; the
// result is valid in thread 0.
template <bool kMin, int kThreads>
__device__ __forceinline__ double block_fold_value(double v) {
    __shared__ double red[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(kFull, v, o);
        v = kMin ? dmin(v, w) : ((w > v) ? w : v);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double r = red[0];
    if (threadIdx.x == 0)
        for (int i = 1; i < kThreads / 32; ++i) r = kMin ? dmin(r, red[i]) : ((red[i] > r) ? red[i] : r);
    return r;
}

// The same, written to *out (one partial per block).
template <bool kMin, int kThreads>
__device__ __forceinline__ void block_fold(double v, double* out) {
    const double r = block_fold_value<kMin, kThreads>(v);
    if (threadIdx.x == 0) *out = r;
}

// Order-preserving 64-bit keys of doubles: dkey(x) < dkey(y) iff x < y for
// any two non-NaN values, so a minimum or maximum over keys with integer
// atomics is exact in any order.
__device__ __forceinline__ long long dkey(double d) {
    const long long b = __double_as_longlong(d);
    return b ^ ((b >> 63) & 0x7fffffffffffffffLL);
}
__device__ __forceinline__ double dkey_value(long long k) {
    return __longlong_as_double(k ^ ((k >> 63) & 0x7fffffffffffffffLL));
}

// A block's share of the cycle reductions (one mesh): its minimum zone dt
// (pass A) or maximum |dV/V0| (pass C) into cyc_red[0] / [1], its inverted
// sides into [2] / [3].  A NaN result is left out, as the serial fold leaves
// NaN out after its first value.
template <bool kPassA, int kThreads>
__device__ __forceinline__ void block_to_cycle(long long* cyc_red, double v, int nbad) {
    const double r = block_fold_value<kPassA, kThreads>(v);
    if (threadIdx.x == 0) {
        if (r == r) {
            if (kPassA) atomicMin(cyc_red, dkey(r));
            else atomicMax(cyc_red + 1, dkey(r));
        }
        if (nbad)
            atomicAdd(reinterpret_cast<unsigned long long*>(cyc_red + (kPassA ? 2 : 3)), (unsigned long long)nbad);
    }
}


// ---------------------------------------------------------------------
// Pass A, one corner of the QCS (QCS.cc:116-380), shared by the zone
// bodies below: corner k at point k, its side k and the previous side pk.
// Returns the two terms of setForce's side sum the corner contributes:
// A = cw (cqe2 + ccos cqe1) to side k and B = cw (cqe1 + ccos cqe2) to side
// pk, so sfq[k] = (A_k + B_nk) / elen[k] in the reference's order.
// ---------------------------------------------------------------------
__device__ __forceinline__ void qcs_corner(const HydroConst& c, double2 up0, double2 upp, double2 upn, double2 xq0,
                                           double2 xq1, double2 xq3, double2 zxp, double2 zuc, double de1,
                                           double de2, double rinv_pk, double rinv_k, double zss, double zrp,
                                           double2& A, double2& B) {
    const double2 up1 = smul(0.5, add(up0, upn));
    const double2 up2 = zuc, xq2 = zxp;
    const double2 up3 = smul(0.5, add(upp, up0));
    const double cvolume = 0.5 * cross(sub(xq2, xq0), sub(xq3, xq1));
    const double2 v1 = sub(xq3, xq0);
    const double2 v2 = sub(xq1, xq0);
    const double minelen = dmin(de1, de2);
    const double ccos = ((minelen < 1.e-12) ? 0. : PNT_QDIV(4. * dot(v1, v2), de1 * de2));
    const double cdiv = PNT_QDIV(cross(sub(up2, up0), sub(xq3, xq1)) - cross(sub(up3, up1), sub(xq2, xq0)),
                                 2.0 * cvolume);
    double evol = 0., du = 0.;
    if (cdiv < 0.0) {
        const double2 dxx1 = smul(0.5, sub(sub(add(xq1, xq2), xq0), xq3));
        const double2 dxx2 = smul(0.5, sub(sub(add(xq2, xq3), xq0), xq1));
        const double dx1 = length(dxx1);
        const double dx2 = length(dxx2);
        const double2 duav = smul(0.25, add(add(add(up0, up1), up2), up3));
        const double test1 = fabs(dot(dxx1, duav) * dx2);
        const double test2 = fabs(dot(dxx2, duav) * dx1);
        const double num = (test1 > test2 ? dx1 : dx2);
        const double den = (test1 > test2 ? dx2 : dx1);
        const double r = num / den;
        evol = sqrt(4.0 * cvolume * r);
        evol = dmin(evol, 2.0 * minelen);
        const double dv1 = length2(sub(sub(add(up1, up2), up0), up3));
        const double dv2 = length2(sub(sub(add(up2, up3), up0), up1));
        du = sqrt(dmax(dv1, dv2));
    }
    double crmu = 0.;
    if (!(cdiv > 0.0)) {
        const double ztmp2 = c.q2 * 0.25 * c.gammap1 * du;
        const double ztmp1 = c.q1 * zss;
#if PNT_FP64_XDIV
        // no compression (evol = du = 0): zkur = ztmp2 + sqrt(ztmp2^2 +
        // ztmp1^2) with ztmp2 a zero is a finite zkur >= +0 when |ztmp1| <
        // 1e150, and with |zrp| < 1e150 too, (zkur zrp) evol is a zero with
        // the sign of zrp: exactly zrp * 0
        if (!(cdiv < 0.0) && ztmp2 == 0.0 && fabs(ztmp1) < 1.e150 && fabs(zrp) < 1.e150) {
            crmu = zrp * 0.0;
        } else
#endif
        {
            const double zkur = ztmp2 + sqrt(ztmp2 * ztmp2 + ztmp1 * ztmp1);
            crmu = zkur * zrp * evol;
        }
    }
    const double2 t1 = smul(crmu, sub(up0, upp));
    const double2 cqe1 = mk(t1.x * rinv_pk, t1.y * rinv_pk);   // / elen[s]
    const double2 t2 = smul(crmu, sub(upn, up0));
    const double2 cqe2 = mk(t2.x * rinv_k, t2.y * rinv_k);     // / elen[s2]
    const double csin2 = 1.0 - ccos * ccos;
    const double cw = ((csin2 < 1.e-4) ? 0. : PNT_QDIV(cvolume, csin2));
    const double cc = ((csin2 < 1.e-4) ? 0. : ccos);
    A = smul(cw, add(cqe2, smul(cc, cqe1)));
    B = smul(cw, add(cqe1, smul(cc, cqe2)));
}

// ---------------------------------------------------------------------
// Pass A, one thread per zone of N sides (N = 3 or 4, static so the side
// arrays stay in registers): the zone's sides in its side order, so zone
// sums keep the reference's serial order and every zone-level quantity is
// formed once.  Scheduled for few live registers: the PolyGas and TTS side
// forces and setVelDiff are formed before the QCS corner loop (so smf, the
// side areas and zdl die early), the corners are taken in order and each
// side is finished as soon as its second corner is known.  nbad counts the
// zone's inverted sides (checkBadSides counts sides, Mesh.cc:1531-1550).
// ---------------------------------------------------------------------
// Pass A's inputs of one zone gathered from global memory: the position
// and velocity of each side's first point (current buffer), the side mass
// fractions and the zone fields.  The row-tile kernels read the same
// values from shared memory through an accessor of the same shape.
struct GlobalZoneIn {
    const DevArrays& a;
    int cur;
    int64_t z, s0;
    __device__ __forceinline__ int32_t p(int k) const { return __ldg(a.mapsp1 + s0 + k); }
    __device__ __forceinline__ double2 x0(int k) const { return a.px[cur][p(k)]; }
    __device__ __forceinline__ double2 u0(int k) const { return a.pu[cur][p(k)]; }
    __device__ __forceinline__ double mf(int k) const { return __ldg(a.smf + s0 + k); }
    __device__ __forceinline__ double zm() const { return a.zm[z]; }
    __device__ __forceinline__ double zr() const { return a.zr[z]; }
    __device__ __forceinline__ double ze() const { return a.ze[z]; }
    __device__ __forceinline__ double zwrate() const { return a.zwrate[z]; }
    __device__ __forceinline__ double zvol() const { return a.zvol[z]; }
};

// The same reads on a mesh numbered as the rect generator numbers it
// (zones row-major, nzx a row; side 4z + k of zone z = (i, j) starts at
// point (i, j), (i+1, j), (i+1, j+1), (i, j+1) for k = 0..3): the point
// indices follow from z, with no load of mapsp1 before the gathers.
struct RectZoneIn {
    const DevArrays& a;
    int cur;
    int64_t z, s0, p0, npx;
    // zone z (global) of a rect mesh of nzx zones a row whose zone zl and
    // point 0 are the global zone z and point po (one mesh: zl = z, po = 0)
    __device__ __forceinline__ RectZoneIn(const DevArrays& a_, int cur_, int64_t z_, int32_t nzx, int64_t zl,
                                          int64_t po)
        : a(a_), cur(cur_), z(z_), s0(4 * z_), npx((int64_t)nzx + 1) {
        const int64_t zj = zl / nzx;
        p0 = po + zj * npx + (zl - zj * nzx);
    }
    __device__ __forceinline__ RectZoneIn(const DevArrays& a_, int cur_, int64_t z_)
        : RectZoneIn(a_, cur_, z_, a_.rect_nzx, z_, 0) {}
    __device__ __forceinline__ int64_t p(int k) const {
        return p0 + (k == 1 ? 1 : (k == 2 ? npx + 1 : (k == 3 ? npx : 0)));
    }
    __device__ __forceinline__ double2 x0(int k) const { return a.px[cur][p(k)]; }
    __device__ __forceinline__ double2 u0(int k) const { return a.pu[cur][p(k)]; }
    __device__ __forceinline__ double mf(int k) const { return __ldg(a.smf + s0 + k); }
    __device__ __forceinline__ double zm() const { return a.zm[z]; }
    __device__ __forceinline__ double zr() const { return a.zr[z]; }
    __device__ __forceinline__ double ze() const { return a.ze[z]; }
    __device__ __forceinline__ double zwrate() const { return a.zwrate[z]; }
    __device__ __forceinline__ double zvol() const { return a.zvol[z]; }
};

template <int N, typename In>
__device__ __forceinline__ void pass_a_zone_thread(const DevArrays& a, const HydroConst& c, const In& in, double dt,
                                                   int64_t z, int64_t s0, double& zdthyd, int& nbad) {
    double2 xp[N], u0[N];
    double mf[N];
    const double dth = 0.5 * dt;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const double2 x0 = in.x0(k);
        u0[k] = in.u0(k);
        mf[k] = in.mf(k);
        xp[k] = add(x0, smul(dth, u0[k]));   // advPosHalf (Hydro.cc:986-1006)
    }
    const double zm = in.zm(), zr = in.zr(), ze = in.ze(), zwrate = in.zwrate(), zvol0 = in.zvol();
    const double rn = 1. / (double)N;
    // calcCtrs (Mesh.cc:797-837)
    double zx = __dadd_rn(0.0, xp[0].x * rn), zy = __dadd_rn(0.0, xp[0].y * rn);
#pragma unroll
    for (int k = 1; k < N; ++k) {
        zx = zx + xp[k].x * rn;
        zy = zy + xp[k].y * rn;
    }
    const double2 zxp = mk(zx, zy);
    // calcVols (Mesh.cc:928-989), calcEdgeLen (:1151-1179), calcCharLen (:1216-1244)
    const double third = 1. / 3.;
    const double fac = (N == 3 ? 3. : 4.);
    double sa[N], elen[N], rinv[N];
    double zareap = 0., zvolp = 0., zdl = 1.e99;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int nk = (k + 1 == N) ? 0 : k + 1;
        sa[k] = 0.5 * cross(sub(xp[nk], xp[k]), sub(zxp, xp[k]));
        const double sv = third * sa[k] * (xp[k].x + xp[nk].x + zxp.x);
        zareap = (k == 0) ? __dadd_rn(0.0, sa[k]) : zareap + sa[k];
        zvolp = (k == 0) ? __dadd_rn(0.0, sv) : zvolp + sv;
        nbad += (sv <= 0.) ? 1 : 0;
        elen[k] = length(sub(xp[nk], xp[k]));
        rinv[k] = 1. / elen[k];
    }
#pragma unroll
    for (int k = 0; k < N; ++k) zdl = dmin(zdl, fac * sa[k] / elen[k]);
    // PolyGas::calcStateHalf (PolyGas.cc:63-109) with calcRho
    const double e = dmax(ze, 0.);
    const double p = c.gm1 * zr * e;
    const double pre = c.gm1 * e;
    const double per = c.gm1 * zr;
    const double q = PNT_QDIV(per * p, zr * zr);
    const double minv = 1. / zm;
    const double csqd = dmax(c.ssmin2, pre + q);
    const double zss = sqrt(csqd);
    const double dv = (zvolp - zvol0) * minv;
    const double bulk = zr * csqd;
    const double denom = 1. + 0.5 * per * dv;
    const double src = zwrate * dth * minv;
    const double zrp = zm / zvolp;
    const double zp = p + PNT_QDIV(per * src - zr * bulk * dv, denom);
    a.zp[z] = zp;
    // calcCrnrMass (Hydro.cc:1083-1117)
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int pk = (k == 0) ? N - 1 : k - 1;
        a.cmass[s0 + k] = zrp * zareap * 0.5 * (mf[k] + mf[pk]);
    }
    // PolyGas::calcForce (PolyGas.cc:164-184) and TTS::calcForce (TTS.cc:55-104)
    double2 ex[N];
#pragma unroll
    for (int k = 0; k < N; ++k) ex[k] = smul(0.5, add(xp[k], xp[(k + 1 == N) ? 0 : k + 1]));
    double sstmp = dmax(zss, c.tts_ssmin);
    sstmp = c.alfa * sstmp * sstmp;
    double2 sfp[N], sft[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const double2 ssurf = rotateCCW(sub(ex[k], zxp));
        const double2 fp = smul(-zp, ssurf);
        const double vfacinv = zareap / sa[k];
        const double srho = zrp * mf[k] * vfacinv;
        const double sdp = sstmp * (srho - zrp);
        sfp[k] = fp;
        sft[k] = smul(-sdp, ssurf);
    }
    // QCS::setVelDiff (QCS.cc:384-448) and calcDtNew (Hydro.cc:1591-1619)
    {
        double ztmp = 0.;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int nk = (k + 1 == N) ? 0 : k + 1;
            const double2 dxs = sub(xp[nk], xp[k]);
            const double2 dus = sub(u0[nk], u0[k]);
            double dux = dot(dus, dxs);
            dux = (elen[k] > 0. ? PNT_QDIV(fabs(dux), elen[k]) : 0.);
            ztmp = dmax(ztmp, dux);
        }
        const double zdu = c.q1 * zss + 2. * c.q2 * ztmp;
        const double cdu = dmax(zdu, dmax(zss, 1.e-99));
        zdthyd = zdl * c.cfl / cdu;
    }
    // QCS::setCornerDiv / setQCnForce / setForce (QCS.cc:116-380), corner k at
    // point k; side k is finished once corner k + 1 is known
    double zux = __dadd_rn(0.0, u0[0].x * rn), zuy = __dadd_rn(0.0, u0[0].y * rn);
#pragma unroll
    for (int k = 1; k < N; ++k) {
        zux = zux + u0[k].x * rn;
        zuy = zuy + u0[k].y * rn;
    }
    const double2 zuc = mk(zux, zuy);
    double2 B0 = mk(0., 0.), Aprev = mk(0., 0.), ftot0 = mk(0., 0.), fprev = mk(0., 0.);
    // side j's sfq from fs = A_j + B_(j+1): sftot, ftot, and the corner force
    // ftot[j] - ftot[j-1] (Hydro.cc:1159-1193; side 0's after the loop)
    auto finish_side = [&](int j, double2 fs) {
        const double2 sfq = mk(fs.x * rinv[j], fs.y * rinv[j]);
        const double2 sfpq = add(sfp[j], sfq);
        const double2 ftot = add(sfpq, sft[j]);
        a.sftot[s0 + j] = sfpq;
        if (j == 0) ftot0 = ftot;
        else a.cforce[s0 + j] = sub(ftot, fprev);
        fprev = ftot;
    };
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int pk = (k == 0) ? N - 1 : k - 1;
        const int nk = (k + 1 == N) ? 0 : k + 1;
        double2 A, B;
        qcs_corner(c, u0[k], u0[pk], u0[nk], xp[k], ex[k], ex[pk], zxp, zuc, elen[pk], elen[k], rinv[pk], rinv[k],
                   zss, zrp, A, B);
        if (k == 0) B0 = B;
        else finish_side(k - 1, add(Aprev, B));
        Aprev = A;
    }
    finish_side(N - 1, add(Aprev, B0));
    a.cforce[s0] = sub(ftot0, fprev);
}

// The same zone with its inputs gathered from global memory.
template <int N>
__device__ __forceinline__ void pass_a_zone_thread(const DevArrays& a, const HydroConst& c, int cur, double dt,
                                                   int64_t z, int64_t s0, double& zdthyd, int& nbad) {
    const GlobalZoneIn in{a, cur, z, s0};
    pass_a_zone_thread<N>(a, c, in, dt, z, s0, zdthyd, nbad);
}

// ---------------------------------------------------------------------
// Pass B, one point
// ---------------------------------------------------------------------
// The point from its corner sums m (mass) and f (force): applyFixedBC per
// plane in deck order (Hydro.cc:773-798, HydroBC.cc:150-182), calcAccel
// (Hydro.cc:1235-1254, pa = f * (1 / max(m, 1e-99))) and advPosFull
// (:1281-1306).  Written with explicit round-to-nearest operations, so the
// result does not depend on the including file's contraction flags: the
// FP64 and mixed cycles, the batch and the fused row-tile pass all advance
// a point bit-identically from the same sums.
__device__ __forceinline__ double2 project_rn(double2 v, double ux, double uy) {
    const double d = __dadd_rn(__dmul_rn(v.x, ux), __dmul_rn(v.y, uy));
    return mk(__dsub_rn(v.x, __dmul_rn(ux, d)), __dsub_rn(v.y, __dmul_rn(uy, d)));
}
__device__ __forceinline__ void advance_point(const HydroConst& c, double dt, unsigned mask, double m, double2 f,
                                              double2 x0, double2 u0, double2& x, double2& u) {
    if (mask) {
        for (int b = 0; b < c.nbc; ++b) {
            if (mask & (1u << b)) {
                u0 = project_rn(u0, c.vfix[b][0], c.vfix[b][1]);
                f = project_rn(f, c.vfix[b][0], c.vfix[b][1]);
            }
        }
    }
    const double rinv = __ddiv_rn(1., dmax(m, 1.e-99));
    const double2 pa = mk(__dmul_rn(f.x, rinv), __dmul_rn(f.y, rinv));
    u = mk(__dadd_rn(u0.x, __dmul_rn(pa.x, dt)), __dadd_rn(u0.y, __dmul_rn(pa.y, dt)));
    const double dth = __dmul_rn(dt, 0.5);
    x = mk(__dadd_rn(x0.x, __dmul_rn(__dadd_rn(u0.x, u.x), dth)),
           __dadd_rn(x0.y, __dmul_rn(__dadd_rn(u0.y, u.y), dth)));
}

// The corners of point p = (i, j) of a rect mesh (nzx zones a row, nzy
// rows) in ascending side order, as the point-to-corner CSR lists them:
// side 2 of the zone below-left, 3 of the zone below, 1 of the zone to the
// left, 0 of the zone (sides 4z + k start at (i, j), (i+1, j), (i+1, j+1),
// (i, j+1)).  With Z the zone below-left these are 4Z + 2 < 4Z + 7 <
// 4(Z + nzx) + 1 < 4(Z + nzx + 1) when all four exist (nzx >= 2); a point
// on the boundary keeps the same order over fewer.  Returns their count.
__device__ __forceinline__ int rect_point_corners(int32_t nzx, int32_t nzy, int64_t p, int64_t* s) {
    const int64_t npx = (int64_t)nzx + 1;
    const int64_t j = p / npx, i = p - j * npx;
    int n = 0;
    if (j > 0) {
        if (i > 0) s[n++] = 4 * ((j - 1) * nzx + i - 1) + 2;
        if (i < nzx) s[n++] = 4 * ((j - 1) * nzx + i) + 3;
    }
    if (j < nzy) {
        if (i > 0) s[n++] = 4 * (j * nzx + i - 1) + 1;
        if (i < nzx) s[n++] = 4 * (j * nzx + i);
    }
    return n;
}

// kRect: a rect mesh (a.rect_nzx > 0), the point's corners from its index
// instead of the CSR (the same sides in the same order).
template <bool kRect = false>
__device__ __forceinline__ void pass_b_point(const DevArrays& a, const HydroConst& c, int cur, double dt,
                                             int64_t p) {
    const double2 x0 = a.px[cur][p];
    const double2 u0 = a.pu[cur][p];
    // corner mass and force, ascending side order from zero (Hydro.cc:1100-1116, :1175-1192)
    double m = 0.;
    double2 f = mk(0., 0.);
    if (kRect) {
        int64_t sc[4];
        const int n = rect_point_corners(a.rect_nzx, a.numz / a.rect_nzx, p, sc);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q < n) {
                m = __dadd_rn(m, a.cmass[sc[q]]);
                const double2 cf = a.cforce[sc[q]];
                f = mk(__dadd_rn(f.x, cf.x), __dadd_rn(f.y, cf.y));
            }
        }
    } else {
        const int32_t o0 = a.poff[p], o1 = a.poff[p + 1];
        for (int32_t i = o0; i < o1; ++i) {
            const int32_t s = __ldg(a.pcorner + i);
            m = __dadd_rn(m, a.cmass[s]);
            const double2 cf = a.cforce[s];
            f = mk(__dadd_rn(f.x, cf.x), __dadd_rn(f.y, cf.y));
        }
    }
    double2 x, u;
    advance_point(c, dt, a.bcmask[p], m, f, x0, u0, x, u);
    a.px[cur ^ 1][p] = x;
    a.pu[cur ^ 1][p] = u;
}

// ---------------------------------------------------------------------
// End of a cycle for one mesh: calcDt (Hydro.cc:1647-1667), checkBadSides
// (Mesh.cc:1531-1550), update_time/update_cycle and calcGlobalDt
// (Driver.cc:213-280), given the reduced dtnew, dvovmax and bad counts.
// ---------------------------------------------------------------------
__device__ __forceinline__ void finish_cycle(Ctl* ctl, const HydroConst& c, double dtn, double dvm, int badA,
                                             int badC) {
    const double dt = ctl->dt;
    ctl->dtnew = dtn;
    ctl->dvovmax = dvm;
    double dtrec = 1.e99;
    if (dtn < dtrec) dtrec = dtn;
    const double dtnew2 = dt * c.cflv / dvm;
    if (dtnew2 < dtrec) dtrec = dtnew2;
    ctl->dtrec = dtrec;
    if (badA > 0 || badC > 0) {   // predictor check first, as Hydro.cc:801 precedes :980
        ctl->status = 3;          // PNT_ERR_BADSIDES
        ctl->nbad = badA > 0 ? badA : badC;
        ctl->done = 1;
        return;
    }
    const double time = ctl->time + dt;
    const int cycle = ctl->cycle + 1;
    ctl->time = time;
    ctl->dtlast = dt;
    ctl->cycle = cycle;
    if (cycle >= c.cstop || !(time < c.tstop)) {
        ctl->done = 1;
        return;
    }
    double ndt = c.dtmax;
    const double dtrecover = c.dtfac * dt;
    if (dtrecover < ndt) ndt = dtrecover;
    if ((c.tstop - time) < ndt) ndt = c.tstop - time;
    if (dtrec < ndt) ndt = dtrec;
    ctl->dt = ndt;
    ctl->dtinv = 1. / ndt;
}

// Pass C's CTAs, after their block_to_cycle: the last one to finish
// (ticket) takes the cycle's reductions, resets them for the next cycle and
// ends the cycle, or, in a multi-piece run, hands this piece's values to
// the caller (piece_red).  Called by every thread of the CTA.
__device__ __forceinline__ void end_cycle_if_last(const DevArrays& a, const HydroConst& c) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(a.fin_ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    unsigned long long* r = reinterpret_cast<unsigned long long*>(a.cyc_red);
    const double dtn = dkey_value((long long)atomicExch(r, (unsigned long long)dkey(1.e99)));
    const double dvm = dkey_value((long long)atomicExch(r + 1, (unsigned long long)dkey(1.e-99)));
    const int badA = (int)atomicExch(r + 2, 0ull);
    const int badC = (int)atomicExch(r + 3, 0ull);
    *a.fin_ticket = 0u;
    if (!a.piece_red && *(volatile unsigned long long*)(r + 4)) {   // a bounded wait ran out this cycle
        a.ctl->status = 6;                                           // PNT_ERR_TIMEOUT
        a.ctl->done = 1;
        return;
    }
    if (a.piece_red) {
        a.piece_red[0] = dtn;
        a.piece_red[1] = -dvm;
        a.piece_red[2] = (double)badA;
        a.piece_red[3] = (double)badC;
    } else {
        finish_cycle(a.ctl, c, dtn, dvm, badA, badC);
    }
}

}  // namespace fp64
}  // namespace pnt
