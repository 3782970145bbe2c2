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

namespace pnt {
namespace {

template <bool kQuads, bool kMixed>
__global__ void __launch_bounds__(stagedc::kTile) pass_c_staged(DevArrays a, HydroConst c) {
    extern __shared__ __align__(16) unsigned char smem_c[];
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

cudaError_t prepare_pass_c(bool mixed, bool quads, int32_t numz, int nsm, int32_t* grid) {
    return tiles::prepare(pick_kernel(mixed, quads), stagedc::kTile, stagedc::kSmemBytes, numz, nsm, grid);
}

void launch_pass_c(const DevArrays& a, const HydroConst& c, bool mixed, cudaStream_t stream) {
    pick_kernel(mixed, a.quads != 0)<<<a.gridC, stagedc::kTile, stagedc::kSmemBytes, stream>>>(a, c);
}

}  // namespace pnt
