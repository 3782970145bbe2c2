// batch_dev.h -- device view of a batch of meshes (pnt_batch_*, batch.cu)
// and the batch kernels of the mixed-precision cycle (hydro_mixed.cu, so
// that they are compiled as the single-mesh mixed cycle is and every
// instance matches its own mixed run bit for bit).
#pragma once

#include "hydro_dev.h"

namespace pnt {

// A work-list entry: a range of one instance's zones or points.
struct Tile {
    int32_t inst;   // instance
    int32_t beg;    // first zone (zone tiles) or point (point tiles), global
    int32_t end;    // one past the last
    int32_t quads;  // the instance's zones are all quads at sides 4z..4z+3
    int32_t nzx;    // zone tiles of a quad instance numbered as the rect generator numbers it: zones a row (else 0)
    int32_t zo;     // the instance's first zone and first point (global)
    int32_t po;
    int32_t pad;
};

struct BatchDev {
    DevArrays a;              // concatenated mesh and state; a.ctl unused
    const Tile* ztiles;       // zone tiles grouped by instance
    const Tile* ptiles;       // point tiles
    int32_t nztiles, nptiles;
    const int32_t* inst_tbeg; // [ninst+1] zone-tile range of each instance
    const HydroConst* consts; // [ninst]
    Ctl* ctls;                // [ninst]
    int32_t ninst;
};

constexpr int kBatchThreads = 256;          // points per point-pass iteration; finalize warps
constexpr int kBatchZT = 128;               // pass A: one zone per thread
constexpr int kZonesPerIter = 64;           // zone tiles are whole multiples of this

__device__ __forceinline__ bool inst_skip(const Ctl& ctl) { return ctl.done || ctl.cycle >= ctl.stop_at; }

// Mixed-precision batch cycle: pass A over the zone tiles (one CTA per
// tile, one partial per tile as the FP64 batch pass A writes) and the point
// pass over the point tiles (persistent, `grid` CTAs).
void launch_batch_pass_a_mixed(const BatchDev& b, bool all_quads, cudaStream_t stream);
void launch_batch_point_pass_mixed(const BatchDev& b, int grid, cudaStream_t stream);

}  // namespace pnt
