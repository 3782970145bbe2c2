// zone_tiles.cuh -- a persistent zone-tile driver for zone passes that
// gather point records (pass C, pass_c_staged.cuh).
//
// A zone pass reads, per side, records of the side's first point (a gather
// through mapsp1) and per-side and per-zone arrays.  Loaded straight into
// registers, the point gathers wait on the index load and hold registers
// until used.  Here each CTA walks its tiles of kTile zones, one thread per
// zone (tiles blockIdx.x, blockIdx.x + gridDim.x, ...): the thread issues
// all the asynchronous copies (`cp.async`, global -> shared) of its zone's
// inputs at once, with the point indices already in registers (loaded one
// tile ahead), then waits for the copies of the oldest tile in flight and
// computes that zone from shared memory.  kStages - 1 further tiles stay in
// flight during the compute.  A thread copies and reads only its own
// zone's slots (structure-of-arrays across the tile's threads: conflict-free
// shared-memory accesses), so `cp.async.wait_group` alone orders them; no
// block barrier inside the loop.
//
// Pass A gains nothing from it: one thread per zone there is bound by its
// arithmetic (1024^2 Sedov: staged 91-105 us mixed, 195-216 us FP64, against
// 89 and 173 us loading straight into registers, 128 and 168 registers),
// so pass A keeps plain loads.
#pragma once

#include "hydro_dev.h"

#include <cuda_runtime.h>

namespace pnt {
namespace tiles {

__device__ __forceinline__ unsigned saddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp16(void* s, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp8(void* s, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp4(void* s, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(saddr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void wait_groups() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Where one zone's inputs live: its first side, side count and point indices.
struct ZoneIdx {
    int4 p;
    int32_t s0;
    int32_t n;
};

template <bool kQuads>
__device__ __forceinline__ ZoneIdx load_idx(const DevArrays& a, int64_t z) {
    ZoneIdx r{make_int4(0, 0, 0, 0), 0, 0};
    if (z >= a.numz) return r;
    if (kQuads) {
        r.s0 = (int32_t)(4 * z);
        r.n = 4;
        r.p = __ldg(reinterpret_cast<const int4*>(a.mapsp1) + z);
    } else {
        r.s0 = a.zfirst[z];
        r.n = a.znump[z];
        r.p.x = a.mapsp1[r.s0];
        r.p.y = a.mapsp1[r.s0 + 1];
        r.p.z = a.mapsp1[r.s0 + 2];
        r.p.w = r.n == 4 ? a.mapsp1[r.s0 + 3] : 0;
    }
    return r;
}

__device__ __forceinline__ int pick(const int4& v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

// The tile loop.  issue(stage, z, idx) copies zone z's inputs (z < numz)
// into its slot of a stage; compute(stage, z) is called by every thread
// for each of the CTA's tiles, z >= numz included (it must skip those), so
// warp-collective code in it sees whole warps.
template <bool kQuads, int kTile, int kStages, int kStageBytes, typename Issue, typename Compute>
__device__ __forceinline__ void for_tiles(const DevArrays& a, unsigned char* smem, Issue&& issue,
                                          Compute&& compute) {
    const int t = threadIdx.x;
    const int64_t ntiles = ((int64_t)a.numz + kTile - 1) / kTile;
    const int64_t step = gridDim.x;
    int64_t tile = blockIdx.x;
    constexpr int kAhead = kStages - 1;
#pragma unroll
    for (int j = 0; j < kAhead; ++j) {
        const int64_t tj = tile + j * step;
        if (tj < ntiles) {
            const int64_t z = tj * kTile + t;
            if (z < a.numz) issue(smem + j * kStageBytes, z, load_idx<kQuads>(a, z));
        }
        commit();
    }
    ZoneIdx nix{};
    if (kQuads) {
        const int64_t tn = tile + kAhead * step;
        if (tn < ntiles) nix = load_idx<kQuads>(a, tn * kTile + t);
    }
    for (int j = 0; tile < ntiles; ++j, tile += step) {
        // tile j + kAhead into the stage tile j - 1 used
        const int64_t ti = tile + kAhead * step;
        if (ti < ntiles) {
            const int64_t z = ti * kTile + t;
            if (!kQuads) nix = load_idx<kQuads>(a, z);
            if (z < a.numz) issue(smem + ((j + kAhead) % kStages) * kStageBytes, z, nix);
        }
        commit();
        if (kQuads) {
            const int64_t tn = ti + step;
            if (tn < ntiles) nix = load_idx<kQuads>(a, tn * kTile + t);
        }
        wait_groups<kAhead>();   // this thread's copies of tile j have landed
        compute(smem + (j % kStages) * kStageBytes, tile * kTile + t);
    }
    wait_groups<0>();
}

// Raises kernel k's dynamic shared-memory limit and returns its persistent
// grid: resident CTAs per SM x nsm, at most one per tile.
template <typename K>
inline cudaError_t prepare(K k, int threads, int smem_bytes, int32_t numz, int nsm, int32_t* grid) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, smem_bytes);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    const int64_t ntiles = ((int64_t)numz + threads - 1) / threads;
    int64_t g = (int64_t)occ * nsm;
    if (g > ntiles) g = ntiles;
    *grid = (int32_t)(g < 1 ? 1 : g);
    return cudaSuccess;
}

// Block sum of a per-thread count (called by every thread of the block).
template <int kThreads>
__device__ __forceinline__ int block_isum(int v) {
    __shared__ int ws[kThreads / 32];
    v = (int)__reduce_add_sync(0xffffffffu, (unsigned)v);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    int s = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s += ws[w];
    return s;
}

}  // namespace tiles
}  // namespace pnt
