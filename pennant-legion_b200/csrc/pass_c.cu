// pass_c.cu -- pass C of the single-mesh cycles: the corrector zone pass
// (calcCtrs, calcVols, calcWork, calcWorkRate, calcEnergy, calcRho,
// calcDvol; Hydro.cc:924-983) as the persistent staged kernel of
// pass_c_staged.cuh, in its FP64 form (bit-identical to a serial run of the
// reference: this file is compiled with -fmad=false) and its mixed form
// (the mixed and learned cycles).  Each CTA adds the maximum |dV/V0| and
// the count of inverted sides over its tiles to the cycle's reductions; the
// last CTA to finish ends the cycle (calcDt, checkBadSides, time/cycle, the
// next calcGlobalDt), so a cycle needs no separate finalize launch.
#include "hydro_fp64_body.cuh"
#include "pass_c_staged.cuh"
#include "row_tiles.cuh"

namespace pnt {
namespace {

// ---------------------------------------------------------------------
// Pass C over row tiles of a rect mesh (row_tiles.cuh): per tile of up to
// kRowT zones, the bottom and top point rows of px0, pu0, px, pu and four
// zone fields arrive by bulk copies; each thread reads its zone's sfp + sfq
// (64 contiguous bytes) and the BC plane masks (two bytes a point, cached)
// from global memory.  64 zones and two stages a CTA, shared memory for 10
// CTAs an SM: 1920^2 Sedov 0.149 ms, against 0.163 ms with sfp + sfq in the
// stages (7 CTAs an SM), 0.152 ms with the zone fields also from global
// memory, 0.174-0.185 ms with three stages and 0.173 ms for the staged
// gathers.
// ---------------------------------------------------------------------
#ifndef PNT_ROWS_C_T
#define PNT_ROWS_C_T 64
#endif
#ifndef PNT_ROWS_C_STAGES
#define PNT_ROWS_C_STAGES 2
#endif
constexpr int kRowT = PNT_ROWS_C_T;
constexpr int kRowStages = PNT_ROWS_C_STAGES;
constexpr int kRowRB = (kRowT + 1) * 16;               // one point row of a double2 field
constexpr int kRowOffZs = 8 * kRowRB;                  // [X0 b,t][U0 b,t][X b,t][U b,t], then zm, zetot, zvol, zp: kRowT + 2 each
constexpr int kRowZB = (kRowT + 2) * 8;
constexpr int kRowStageBytes = kRowOffZs + 4 * kRowZB;
constexpr int kRowSmemBytes = kRowStages * kRowStageBytes;
static_assert(kRowT % 2 == 0 && kRowStageBytes % 16 == 0, "16-byte aligned stages");

struct RowIn {
    const unsigned char* st;
    const uint16_t* bcmask;
    int64_t pb, npx;
    int t, shift;
    __device__ __forceinline__ int row(int k) const { return k >= 2 ? 1 : 0; }
    __device__ __forceinline__ int col(int k) const { return t + ((k == 1 || k == 2) ? 1 : 0); }
    __device__ __forceinline__ const double2* f(int field, int k) const {
        return reinterpret_cast<const double2*>(st + (2 * field + row(k)) * kRowRB) + col(k);
    }
    __device__ __forceinline__ double x0x(int k) const { return f(0, k)->x; }
    __device__ __forceinline__ double2 u0(int k) const { return *f(1, k); }
    __device__ __forceinline__ double2 x(int k) const { return *f(2, k); }
    __device__ __forceinline__ double2 u(int k) const { return *f(3, k); }
    const double2* sfg;   // the zone's sfp + sfq (global memory)
    __device__ __forceinline__ double2 sf(int k) const { return sfg[k]; }
    __device__ __forceinline__ unsigned mask(int k) const { return __ldg(bcmask + pb + row(k) * npx + col(k)); }
    __device__ __forceinline__ double zs(int fld) const {
        return reinterpret_cast<const double*>(st + kRowOffZs + fld * kRowZB)[shift + t];
    }
    __device__ __forceinline__ double zm() const { return zs(0); }
    __device__ __forceinline__ double zetot() const { return zs(1); }
    __device__ __forceinline__ double zvol() const { return zs(2); }
    __device__ __forceinline__ double zp() const { return zs(3); }
};

template <bool kMixed>
__global__ void __launch_bounds__(kRowT) pass_c_rows(DevArrays a, HydroConst c) {
    extern __shared__ __align__(128) unsigned char smem_r[];
    __shared__ __align__(8) uint64_t bars[kRowStages];
    pdl_wait();
    // the learned cycle's closure pass and pass B are done with this cycle's
    // zone records
    if (a.closure_nrec && blockIdx.x == 0 && threadIdx.x == 0) *a.closure_nrec = 0;
    const Ctl* ctl = a.ctl;
    if (fp64::skip_cycle(ctl)) return;
    const int cur = ctl->cycle & 1;
    const double dt = ctl->dt, dtinv = ctl->dtinv;
    const int32_t nzx = a.rect_nzx;
    const int64_t npx = (int64_t)nzx + 1;
    const int64_t ntiles = rows::num_tiles<kRowT>(nzx, a.numz);
    const int t = threadIdx.x;
    double dvm = 1.e-99;
    int nbad = 0;
    auto bytes = [&](int64_t g) -> uint32_t {
        const rows::Tile tl = rows::tile_of<kRowT>(g, nzx);
        const rows::ZoneRun zr = rows::zone_run(tl);
        return (uint32_t)(8 * (tl.nt + 1) * 16 + 4 * zr.count * 8);
    };
    auto issue = [&](unsigned char* st, int64_t g, uint32_t bar) {
        const rows::Tile tl = rows::tile_of<kRowT>(g, nzx);
        const rows::ZoneRun zr = rows::zone_run(tl);
        const uint32_t rb = (uint32_t)(tl.nt + 1) * 16;
        const double2* fields[4] = {a.px[cur], a.pu[cur], a.px[cur ^ 1], a.pu[cur ^ 1]};
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            rows::bulk_g2s(st + (2 * f) * kRowRB, fields[f] + tl.pb, rb, bar);
            rows::bulk_g2s(st + (2 * f + 1) * kRowRB, fields[f] + tl.pb + npx, rb, bar);
        }
        const double* zf[4] = {a.zm, a.zetot, a.zvol, a.zp};
#pragma unroll
        for (int f = 0; f < 4; ++f)
            rows::bulk_g2s(st + kRowOffZs + f * kRowZB, zf[f] + zr.zs, (uint32_t)(zr.count * 8), bar);
    };
    auto compute = [&](const unsigned char* st, int64_t g) {
        const rows::Tile tl = rows::tile_of<kRowT>(g, nzx);
        if (t >= tl.nt) return;
        const RowIn in{st, a.bcmask, tl.pb, npx, t, (int)(tl.z0 & 1), a.sftot + 4 * (tl.z0 + t)};
        const double d = stagedc::zone_core<true, kMixed>(a, c, 4, in, tl.z0 + t, dt, dtinv, nbad);
        dvm = (d > dvm) ? d : dvm;
    };
    if (!rows::for_tiles<kRowStages, kRowStageBytes>(ntiles, smem_r, bars, bytes, issue, compute) && t == 0)
        atomicOr(reinterpret_cast<unsigned long long*>(a.cyc_red + 4), 1ull);
    const int nb = tiles::block_isum<kRowT>(nbad);
    fp64::block_to_cycle<false, kRowT>(a.cyc_red, dvm, nb);
    fp64::end_cycle_if_last(a, c);
}

template <bool kQuads, bool kMixed>
__global__ void __launch_bounds__(stagedc::kTile) pass_c_staged(DevArrays a, HydroConst c) {
    extern __shared__ __align__(16) unsigned char smem_c[];
    pdl_wait();
    if (a.closure_nrec && blockIdx.x == 0 && threadIdx.x == 0) *a.closure_nrec = 0;
    if (fp64::skip_cycle(a.ctl)) return;
    double dvm = 1.e-99;
    int nbad = 0;
    stagedc::pass_c_tiles<kQuads, kMixed>(a, c, smem_c, dvm, nbad);
    const int nb = tiles::block_isum<stagedc::kTile>(nbad);
    fp64::block_to_cycle<false, stagedc::kTile>(a.cyc_red, dvm, nb);
    fp64::end_cycle_if_last(a, c);
}

using Kernel = void (*)(DevArrays, HydroConst);

Kernel pick_kernel(bool mixed, bool quads) {
    if (mixed) return quads ? pass_c_staged<true, true> : pass_c_staged<false, true>;
    return quads ? pass_c_staged<true, false> : pass_c_staged<false, false>;
}

}  // namespace

cudaError_t prepare_pass_c(bool mixed, bool quads, int32_t rect_nzx, int32_t numz, int nsm, int32_t* grid) {
    if (rect_nzx > 0) {
        const Kernel k = mixed ? pass_c_rows<true> : pass_c_rows<false>;
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowSmemBytes);
        if (e != cudaSuccess) return e;
        int occ = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, kRowT, kRowSmemBytes);
        if (e != cudaSuccess) return e;
        if (occ < 1) return cudaErrorInvalidConfiguration;
        int64_t g = (int64_t)occ * nsm;
        const int64_t nt = rows::num_tiles<kRowT>(rect_nzx, numz);
        if (g > nt) g = nt;
        *grid = (int32_t)(g < 1 ? 1 : g);
        return cudaSuccess;
    }
    return tiles::prepare(pick_kernel(mixed, quads), stagedc::kTile, stagedc::kSmemBytes, numz, nsm, grid);
}

void launch_pass_c(const DevArrays& a, const HydroConst& c, bool mixed, cudaStream_t stream) {
    if (a.rect_nzx > 0) {
        launch_pdl(mixed ? pass_c_rows<true> : pass_c_rows<false>, a.gridC, kRowT, kRowSmemBytes, stream, a, c);
        return;
    }
    launch_pdl(pick_kernel(mixed, a.quads != 0), a.gridC, stagedc::kTile, stagedc::kSmemBytes, stream, a, c);
}

}  // namespace pnt
