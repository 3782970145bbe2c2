// row_tiles.cuh -- persistent zone passes over row tiles of a rectangular
// mesh, their inputs brought into shared memory by TMA bulk copies.
//
// A mesh from the reference's rect generator (genPointsRect / genZonesRect
// / genSidesRect, GenMesh.cc:790-829, 898-930, 987-1100) numbers its zones
// row-major, nzx to a row, its points (nzx + 1) to a row, and the sides of
// zone z as 4z + k (k = bottom, right, top, left).  A tile of up to T zones
// of one row therefore needs two contiguous runs of points (the row below
// and the row above) and contiguous runs of its side and zone fields: a
// handful of `cp.async.bulk` copies issued by one thread replace the
// per-zone gathers (pass C issued 28 asynchronous copies per zone).
//
// Pipeline: each CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ...
// through kStages shared-memory stages.  Thread 0 issues the copies of the
// tile kStages - 1 ahead into the stage the previous tile released, with an
// mbarrier per stage counting the bytes (expect_tx / complete_tx); every
// thread waits for its tile's stage, computes its zone from shared memory,
// and the CTA barrier that ends the tile releases the stage.  Every wait is
// bounded: a wait that runs out sets *err, the CTA stops taking tiles, and
// thread 0 waits (bounded again) for every copy it issued before the CTA
// exits.
#pragma once

#include "hydro_dev.h"

#include <cuda_runtime.h>

namespace pnt {
namespace rows {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded: false if the phase of the given parity did not complete within
// `limit` polls (each poll may itself wait a hardware-defined time).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit = 1 << 20) {
    for (int i = 0; i < limit; ++i)
        if (mbar_try(bar, parity)) return true;
    return false;
}
// Global -> shared bulk copy completing `bytes` on the mbarrier.  Source and
// destination 16-byte aligned, bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(saddr(dst)),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tile g of a rect mesh with nzx zones a row and T zones a tile.
struct Tile {
    int64_t z0;   // first zone
    int64_t pb;   // first point of the row below (its zone row's bottom edge)
    int32_t nt;   // zones in the tile
};
template <int T>
__device__ __forceinline__ Tile tile_of(int64_t g, int32_t nzx) {
    const int32_t per_row = (nzx + T - 1) / T;
    const int64_t zj = g / per_row;
    const int32_t zi0 = (int32_t)(g - zj * per_row) * T;
    Tile t;
    t.z0 = zj * nzx + zi0;
    t.pb = zj * (int64_t)(nzx + 1) + zi0;
    t.nt = (nzx - zi0 < T) ? nzx - zi0 : T;
    return t;
}
template <int T>
__host__ __device__ inline int64_t num_tiles(int32_t nzx, int32_t numz) {
    if (nzx <= 0) return 0;
    return (int64_t)(numz / nzx) * ((nzx + T - 1) / T);
}

// Zone fields are copied from an even zone so the source is 16-byte
// aligned; the tile's zones then start at slot `shift` of the copy, which
// holds `count` (even) zones.  Zone arrays are padded by one element.
struct ZoneRun {
    int64_t zs;
    int32_t shift, count;
};
__device__ __forceinline__ ZoneRun zone_run(const Tile& t) {
    ZoneRun r;
    r.shift = (int32_t)(t.z0 & 1);
    r.zs = t.z0 - r.shift;
    r.count = (t.nt + r.shift + 1) & ~1;
    return r;
}

// The tile loop.  bytes(g) = the bytes issue() copies for tile g;
// issue(stage, g, bar) issues them (thread 0 only); compute(stage, g) is
// called by every thread for each of the CTA's tiles.  bars: kStages
// mbarriers in shared memory.  Returns false on every thread if a wait ran
// out (after the drain).
template <int kStages, int kStageBytes, typename Bytes, typename Issue, typename Compute>
__device__ __forceinline__ bool for_tiles(int64_t ntiles, unsigned char* smem, uint64_t* bars, Bytes&& bytes,
                                          Issue&& issue, Compute&& compute) {
    const int tid = threadIdx.x;
    const int64_t step = gridDim.x;
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(saddr(bars + s), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int64_t issued = 0;   // tiles whose copies thread 0 has issued (this CTA's k-th tile is k)
    if (tid == 0) {
        for (int j = 0; j < kStages - 1; ++j) {
            const int64_t g = blockIdx.x + j * step;
            if (g >= ntiles) break;
            const uint32_t bar = saddr(bars + j);
            mbar_expect_tx(bar, bytes(g));
            issue(smem + j * kStageBytes, g, bar);
            ++issued;
        }
    }
    bool ok = true;
    int64_t k = 0;
    for (int64_t g = blockIdx.x; g < ntiles; g += step, ++k) {
        if (tid == 0) {
            const int64_t kn = k + kStages - 1;
            const int64_t gn = blockIdx.x + kn * step;
            if (gn < ntiles) {
                const int sn = (int)(kn % kStages);
                const uint32_t bar = saddr(bars + sn);
                fence_proxy_async();   // the stage's last readers finished before the barrier below
                mbar_expect_tx(bar, bytes(gn));
                issue(smem + sn * kStageBytes, gn, bar);
                ++issued;
            }
        }
        const int s = (int)(k % kStages);
        const bool w = mbar_wait(saddr(bars + s), (uint32_t)((k / kStages) & 1));
        if (w) compute(smem + s * kStageBytes, g);
        if (__syncthreads_or(!w)) {
            ok = false;
            break;
        }
    }
    if (!ok && tid == 0) {
        // copies still in flight land in shared memory: wait for each issued
        // stage beyond the last completed one before the CTA may exit
        for (int64_t j = k; j < issued; ++j) mbar_wait(saddr(bars + (int)(j % kStages)), (uint32_t)((j / kStages) & 1));
    }
    if (!ok) __syncthreads();
    return ok;
}

// ---------------------------------------------------------------------
// Pass A's stage: position and velocity (current buffer) of the tile's
// bottom and top point rows, the side mass fractions of its 4T sides and
// five zone fields, T (even) zones a tile.
// ---------------------------------------------------------------------
template <int T>
struct PassAStage {
    static constexpr int kRB = (T + 1) * 16;        // one point row of a double2 field
    static constexpr int kOffMf = 4 * kRB;          // [X0 b,t][U0 b,t], then smf
    static constexpr int kOffZs = kOffMf + 32 * T;  // zm, zr, ze, zwrate, zvol: T + 2 each
    static constexpr int kZB = (T + 2) * 8;
    static constexpr int kBytes = kOffZs + 5 * kZB;
    static_assert(T % 2 == 0 && kBytes % 16 == 0, "16-byte aligned stages");

    __device__ static uint32_t bytes(const Tile& tl) {
        return (uint32_t)(4 * (tl.nt + 1) * 16 + 32 * tl.nt + 5 * zone_run(tl).count * 8);
    }
    __device__ static void issue(unsigned char* st, const DevArrays& a, int cur, const Tile& tl, int64_t npx,
                                 uint32_t bar) {
        const ZoneRun zr = zone_run(tl);
        const uint32_t rb = (uint32_t)(tl.nt + 1) * 16;
        bulk_g2s(st, a.px[cur] + tl.pb, rb, bar);
        bulk_g2s(st + kRB, a.px[cur] + tl.pb + npx, rb, bar);
        bulk_g2s(st + 2 * kRB, a.pu[cur] + tl.pb, rb, bar);
        bulk_g2s(st + 3 * kRB, a.pu[cur] + tl.pb + npx, rb, bar);
        bulk_g2s(st + kOffMf, a.smf + 4 * tl.z0, (uint32_t)(32 * tl.nt), bar);
        const double* zf[5] = {a.zm, a.zr, a.ze, a.zwrate, a.zvol};
#pragma unroll
        for (int f = 0; f < 5; ++f) bulk_g2s(st + kOffZs + f * kZB, zf[f] + zr.zs, (uint32_t)(zr.count * 8), bar);
    }
};

// Zone t of a pass A stage, read as fp64::GlobalZoneIn reads global memory:
// side k of a rect zone starts at point (i, j), (i+1, j), (i+1, j+1),
// (i, j+1) for k = 0..3.
template <int T>
struct RowZoneIn {
    const unsigned char* st;
    int t, shift;
    __device__ __forceinline__ const double2* pt(int f, int k) const {
        return reinterpret_cast<const double2*>(st + (2 * f + (k >= 2 ? 1 : 0)) * PassAStage<T>::kRB) + t +
               ((k == 1 || k == 2) ? 1 : 0);
    }
    __device__ __forceinline__ double2 x0(int k) const { return *pt(0, k); }
    __device__ __forceinline__ double2 u0(int k) const { return *pt(1, k); }
    __device__ __forceinline__ double mf(int k) const {
        return reinterpret_cast<const double*>(st + PassAStage<T>::kOffMf)[4 * t + k];
    }
    __device__ __forceinline__ double zs(int f) const {
        return reinterpret_cast<const double*>(st + PassAStage<T>::kOffZs + f * PassAStage<T>::kZB)[shift + t];
    }
    __device__ __forceinline__ double zm() const { return zs(0); }
    __device__ __forceinline__ double zr() const { return zs(1); }
    __device__ __forceinline__ double ze() const { return zs(2); }
    __device__ __forceinline__ double zwrate() const { return zs(3); }
    __device__ __forceinline__ double zvol() const { return zs(4); }
};

// Persistent grid of a row-tile kernel: resident CTAs per SM x nsm, at
// most one per tile.
template <typename K>
inline cudaError_t prepare(K k, int threads, int smem_bytes, int64_t ntiles, int nsm, int32_t* grid) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, smem_bytes);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    int64_t g = (int64_t)occ * nsm;
    if (g > ntiles) g = ntiles;
    *grid = (int32_t)(g < 1 ? 1 : g);
    return cudaSuccess;
}

}  // namespace rows
}  // namespace pnt
