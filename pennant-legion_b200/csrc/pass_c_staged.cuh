// pass_c_staged.cuh -- pass C (the corrector zone pass: calcCtrs, calcVols,
// calcWork, calcWorkRate, calcEnergy, calcRho, calcDvol at the end of
// Hydro::doCycle, Hydro.cc:924-983) as a persistent kernel that stages its
// gathered inputs in shared memory.
//
// Pass C reads, per side, the start-of-cycle and new position and velocity
// of the side's first point (a gather through mapsp1) and the side's sfp +
// sfq, and per zone four scalars.  Loaded straight into registers by four
// lanes per zone (a chain of two dependent memory latencies, ~36 shuffles
// per lane) it ran at 31% of peak DRAM throughput; here the zone-tile
// driver of zone_tiles.cuh stages the gathered point data and the zone
// scalars in shared memory, one thread per zone, and each thread reads its
// sides' sfp + sfq (contiguous) from global memory.  On the B200 more
// resident CTAs beat deeper pipelines (1024^2 Sedov, with sfp + sfq still
// staged: 1 stage and 10 CTAs of 64 per SM 56 us, 2 stages 59 us, 3 stages
// 72 us), so the default is one stage.
//
// The zone arithmetic is the four-lane pass C's, one zone per thread:
// kMixed = false keeps the reference's serial side order and operation
// order (zone sums start from 0.0, bit-identical to pass_c_zone when the
// including file is compiled with -fmad=false); kMixed = true is the mixed
// cycle's form (sums start from the first side, zetot = zetot0 + the zone's
// work).
#pragma once

#include "zone_tiles.cuh"

#include <cuda_runtime.h>

namespace pnt {
namespace stagedc {

#ifndef PNT_STAGED_C_TILE
#define PNT_STAGED_C_TILE 64
#endif
#ifndef PNT_STAGED_C_STAGES
#define PNT_STAGED_C_STAGES 1
#endif
constexpr int kTile = PNT_STAGED_C_TILE;       // zones (threads) per tile
constexpr int kStages = PNT_STAGED_C_STAGES;   // tiles resident per CTA
static_assert(kTile % 32 == 0 && kStages >= 1, "tile of whole warps");

// Bytes of one stage per zone: per side x0.x (8), u0 (16), x (16), u (16),
// the 32-bit bcmask word holding the point's mask (4); per zone zm, zetot,
// zvol, zp (32), the side count and mask parities (4) and the first side
// (4).  The sides' sfp + sfq (64 contiguous bytes a quad zone) are read from
// global memory where they are used: the smaller stage holds 12 CTAs an SM
// instead of 10.
constexpr int kOffX0x = 0;
constexpr int kOffU0 = kOffX0x + 4 * 8 * kTile;
constexpr int kOffX = kOffU0 + 4 * 16 * kTile;
constexpr int kOffU = kOffX + 4 * 16 * kTile;
constexpr int kOffMw = kOffU + 4 * 16 * kTile;
constexpr int kOffZs = kOffMw + 4 * 4 * kTile;
constexpr int kOffMeta = kOffZs + 4 * 8 * kTile;
constexpr int kOffS0 = kOffMeta + 4 * kTile;
constexpr int kStageBytes = kOffS0 + 4 * kTile;
constexpr int kSmemBytes = kStages * kStageBytes;

using tiles::cp16;
using tiles::cp4;
using tiles::cp8;
using tiles::ZoneIdx;
using tiles::pick;

// Issues the copies of zone z's inputs into slot t of stage st.  bcmask is
// 16-bit per point; its 32-bit word is copied (the buffer is padded to a
// whole word) and the point's parity kept in the zone's meta word.
__device__ __forceinline__ void issue(const DevArrays& a, int cur, unsigned char* st, int t, int64_t z,
                                      const ZoneIdx& ix) {
    const double2* px0 = a.px[cur];
    const double2* pu0 = a.pu[cur];
    const double2* px1 = a.px[cur ^ 1];
    const double2* pu1 = a.pu[cur ^ 1];
    const uint32_t* mw = reinterpret_cast<const uint32_t*>(a.bcmask);
    int meta = ix.n;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k < ix.n) {
            const int p = pick(ix.p, k);
            cp8(st + kOffX0x + (k * kTile + t) * 8, &px0[p].x);
            cp16(st + kOffU0 + (k * kTile + t) * 16, pu0 + p);
            cp16(st + kOffX + (k * kTile + t) * 16, px1 + p);
            cp16(st + kOffU + (k * kTile + t) * 16, pu1 + p);
            cp4(st + kOffMw + (k * kTile + t) * 4, mw + (p >> 1));
            meta |= (p & 1) << (4 + k);
        }
    }
    cp8(st + kOffZs + (0 * kTile + t) * 8, a.zm + z);
    cp8(st + kOffZs + (1 * kTile + t) * 8, a.zetot + z);
    cp8(st + kOffZs + (2 * kTile + t) * 8, a.zvol + z);
    cp8(st + kOffZs + (3 * kTile + t) * 8, a.zp + z);
    reinterpret_cast<int*>(st + kOffMeta)[t] = meta;
    reinterpret_cast<int*>(st + kOffS0)[t] = ix.s0;
}

__device__ __forceinline__ double2 mk2(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double2 proj(double2 v, double ux, double uy) {
    const double d = v.x * ux + v.y * uy;
    return mk2(v.x - ux * d, v.y - uy * d);
}

// One zone's corrector from its inputs, read through `in` where they are
// used: for side k < n, in.x(k) / in.u(k) the new position and velocity of
// the side's first point, in.u0(k) its start-of-cycle velocity (before the
// boundary projections), in.x0x(k) its start-of-cycle x, in.mask(k) its BC
// plane mask, in.sf(k) the side's sfp + sfq; in.zm() etc. the zone's
// scalars.  Writes zvol, zr, zetot, ze, zwrate; returns |dV/V0| and adds the
// zone's inverted sides to nbad.
template <bool kQuads, bool kMixed, typename In>
__device__ __forceinline__ double zone_core(const DevArrays& a, const HydroConst& c, int n, const In& in, int64_t z,
                                            double dt, double dtinv, int& nbad) {
    if (kQuads) n = 4;
    const double zm = in.zm(), zetot0 = in.zetot(), zvol0 = in.zvol(), zp = in.zp();
    const double dth = 0.5 * dt;

    double2 x[4], ub[4];
    double xpx[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k < n) {
            x[k] = in.x(k);
            const double2 u0 = in.u0(k);
            xpx[k] = in.x0x(k) + u0.x * dth;   // advPosHalf's x, from pu0 before the BCs
            // applyFixedBC on pu0 (Hydro.cc:1008-1032), planes in deck order
            const unsigned mask = in.mask(k);
            double2 u0b = u0;
            if (mask) {
                for (int b = 0; b < c.nbc; ++b)
                    if (mask & (1u << b)) u0b = proj(u0b, c.vfix[b][0], c.vfix[b][1]);
            }
            ub[k] = u0b;
        } else {
            x[k] = mk2(0., 0.);
            ub[k] = mk2(0., 0.);
            xpx[k] = 0.;
        }
    }
    // calcCtrs + calcVols at the new positions (Mesh.cc:797-837, :928-989)
    const double rn = 1. / (double)n;
    double zxx, zxy;
    if (kMixed) {
        zxx = x[0].x * rn + x[1].x * rn + x[2].x * rn;
        zxy = x[0].y * rn + x[1].y * rn + x[2].y * rn;
    } else {
        zxx = __dadd_rn(0.0, x[0].x * rn) + x[1].x * rn + x[2].x * rn;
        zxy = __dadd_rn(0.0, x[0].y * rn) + x[1].y * rn + x[2].y * rn;
    }
    if (n == 4) {
        zxx = zxx + x[3].x * rn;
        zxy = zxy + x[3].y * rn;
    }
    const double third = 1. / 3.;
    double zvol = 0., zetot = zetot0, zw = 0.;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k < n) {
            const int k2 = (k + 1 == n) ? 0 : k + 1;
            const double2 x2 = x[k2];
            const double sa = 0.5 * ((x2.x - x[k].x) * (zxy - x[k].y) - (x2.y - x[k].y) * (zxx - x[k].x));
            const double sv = third * sa * (x[k].x + x2.x + zxx);
            nbad += (sv <= 0.) ? 1 : 0;
            // calcWork (Hydro.cc:1339-1406): the side's force against the
            // average velocity of its two points, at the half-step positions
            const double2 sf = in.sf(k);
            const double2 u = in.u(k);
            const double2 u2 = in.u(k2);
            const double sd1 = sf.x * (ub[k].x + u.x) + sf.y * (ub[k].y + u.y);
            const double sd2 = (-sf.x) * (ub[k2].x + u2.x) + (-sf.y) * (ub[k2].y + u2.y);
            const double dwork = -dth * (sd1 * xpx[k] + sd2 * xpx[k2]);
            if (kMixed) {
                zvol = (k == 0) ? sv : zvol + sv;
                zw = (k == 0) ? dwork : zw + dwork;
            } else {
                zvol = (k == 0) ? __dadd_rn(0.0, sv) : zvol + sv;
                zw = (k == 0) ? __dadd_rn(0.0, dwork) : zw + dwork;
                zetot = zetot + dwork;
            }
        }
    }
    if (kMixed) zetot = zetot0 + zw;
    // calcWorkRate (Hydro.cc:1483-1510), calcEnergy (:1545-1564),
    // calcRho (:1034-1054), calcDvol (:1622-1644)
    const double dvol = zvol - zvol0;
    const double zwrate = (zw + zp * dvol) * dtinv;
    a.zvol[z] = zvol;
    a.zr[z] = zm / zvol;
    a.zetot[z] = zetot;
    a.ze[z] = zetot / (zm + 1.e-99);
    a.zwrate[z] = zwrate;
    return fabs((zvol - zvol0) / zvol0);
}

// The staged layout above, slot t of stage st; sfg: the zone's sfp + sfq
// (global memory).
struct StagedIn {
    const unsigned char* st;
    int t, meta;
    const double2* sfg;
    __device__ __forceinline__ double2 x(int k) const {
        return reinterpret_cast<const double2*>(st + kOffX)[k * kTile + t];
    }
    __device__ __forceinline__ double2 u(int k) const {
        return reinterpret_cast<const double2*>(st + kOffU)[k * kTile + t];
    }
    __device__ __forceinline__ double2 u0(int k) const {
        return reinterpret_cast<const double2*>(st + kOffU0)[k * kTile + t];
    }
    __device__ __forceinline__ double x0x(int k) const {
        return reinterpret_cast<const double*>(st + kOffX0x)[k * kTile + t];
    }
    __device__ __forceinline__ double2 sf(int k) const { return sfg[k]; }
    __device__ __forceinline__ unsigned mask(int k) const {
        const uint32_t w = reinterpret_cast<const uint32_t*>(st + kOffMw)[k * kTile + t];
        return (w >> (((meta >> (4 + k)) & 1) * 16)) & 0xffffu;
    }
    __device__ __forceinline__ double zs(int f) const { return reinterpret_cast<const double*>(st + kOffZs)[f * kTile + t]; }
    __device__ __forceinline__ double zm() const { return zs(0); }
    __device__ __forceinline__ double zetot() const { return zs(1); }
    __device__ __forceinline__ double zvol() const { return zs(2); }
    __device__ __forceinline__ double zp() const { return zs(3); }
};

// One zone's corrector from stage st, slot t.
template <bool kQuads, bool kMixed>
__device__ __forceinline__ double zone(const DevArrays& a, const HydroConst& c, const unsigned char* st, int t,
                                       int64_t z, double dt, double dtinv, int& nbad) {
    const int meta = reinterpret_cast<const int*>(st + kOffMeta)[t];
    const StagedIn in{st, t, meta, a.sftot + reinterpret_cast<const int*>(st + kOffS0)[t]};
    return zone_core<kQuads, kMixed>(a, c, meta & 15, in, z, dt, dtinv, nbad);
}

// The persistent pass C over the CTA's tiles: the maximum |dV/V0| into
// dvm, the inverted sides into nbad.
template <bool kQuads, bool kMixed>
__device__ __forceinline__ void pass_c_tiles(const DevArrays& a, const HydroConst& c, unsigned char* smem,
                                             double& dvm, int& nbad) {
    const Ctl* ctl = a.ctl;
    const int cur = ctl->cycle & 1;
    const double dt = ctl->dt, dtinv = ctl->dtinv;
    const int t = threadIdx.x;
    tiles::for_tiles<kQuads, kTile, kStages, kStageBytes>(
        a, smem, [&](unsigned char* st, int64_t z, const ZoneIdx& ix) { issue(a, cur, st, t, z, ix); },
        [&](const unsigned char* st, int64_t z) {
            if (z < a.numz) {
                const double d = zone<kQuads, kMixed>(a, c, st, t, z, dt, dtinv, nbad);
                dvm = (d > dvm) ? d : dvm;
            }
        });
}

}  // namespace stagedc
}  // namespace pnt
