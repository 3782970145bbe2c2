// hydro_fp64.cu -- the plain FP64 hydro cycle on sm_100a (one mesh).
//
// One cycle of Hydro::doCycle (Hydro.cc:342-983) runs as three kernels:
//
//   pass A  zone pass, predictor: advPosHalf, calcCtrs, calcVols,
//           calcSurfVecs, calcEdgeLen, calcCharLen, calcRho, calcCrnrMass,
//           PolyGas::calcStateHalf/calcForce, TTS::calcForce, QCS
//           setCornerDiv/setQCnForce/setForce/setVelDiff, the side part of
//           sumCrnrForce, calcDtNew (block minimum)
//   pass B  point pass: corner mass and force gathered through the
//           point->corner CSR in ascending side order (no float atomics),
//           applyFixedBC, calcAccel, advPosFull
//   pass C  zone pass, corrector: calcCtrs, calcVols, calcWork,
//           calcWorkRate, calcEnergy, calcRho, calcDvol (block maximum);
//           its last CTA then runs calcDt, checkBadSides, the time/cycle
//           update and the next cycle's calcGlobalDt (Driver.cc:213-245)
// Passes A and C add their blocks' dt minimum, dV/V maximum and inverted
// sides to the cycle's reductions with atomics (exact in any order).
//
// Pass A runs one thread per zone (pass_a_zone_thread): the zone's sides
// in the reference's side order, each zone-level quantity (centre, sums,
// EOS) formed once, no shuffles, scheduled so the side arrays die early;
// 128 registers, 4 blocks of 128 per SM.  It is bound by its ~2400
// instructions per zone, a third of them the correctly rounded FP64
// divisions and square roots; quotients whose IEEE result is fixed without
// the division (zero over a finite non-zero divisor, division by one, the
// zkur square root of a corner without compression) skip it, which a
// quiescent region (zero velocities and pressure) hits on most corners.
// Pass C is the persistent staged kernel of pass_c.cu (one
// thread per zone, inputs gathered into shared memory by asynchronous
// copies); the batched kernels run the same two bodies.  1/elen is formed
// once per side and shared with the neighbouring corner; QCS terms the
// reference computes and then discards (evol and du unless cdiv < 0, zkur
// when cdiv > 0) are not computed, which leaves every stored value
// unchanged.  The arithmetic lives in hydro_fp64_body.cuh (shared with the
// batched kernels); this file is compiled with -fmad=false, so the results
// match a serial CPU run of the reference bit for bit.
#include "hydro_fp64_body.cuh"

#include <algorithm>
#include "zone_tiles.cuh"

namespace pnt {
namespace {

using namespace fp64;

#ifndef PNT_PASS_A_ZT_MIN_BLOCKS
#define PNT_PASS_A_ZT_MIN_BLOCKS 4
#endif
constexpr int kZoneThreadsZT = 128;   // one zone per thread

// kRect: a rect mesh (a.rect_nzx > 0), point indices from the zone index.
template <bool kQuads, bool kRect = false>
__global__ void __launch_bounds__(kZoneThreadsZT, PNT_PASS_A_ZT_MIN_BLOCKS) pass_a_zt(DevArrays a, HydroConst c) {
    pdl_wait();
    const Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const int64_t z = (int64_t)blockIdx.x * kZoneThreadsZT + threadIdx.x;
    double zdthyd = 1.e99;
    int bad = 0;
    if (z < a.numz) {
        const int cur = ctl->cycle & 1;
        const double dt = ctl->dt;
        if (kRect) {
            const RectZoneIn in(a, cur, z);
            pass_a_zone_thread<4>(a, c, in, dt, z, 4 * z, zdthyd, bad);
        } else if (kQuads) {
            pass_a_zone_thread<4>(a, c, cur, dt, z, 4 * z, zdthyd, bad);
        } else {
            const int n = a.znump[z];
            const int64_t s0 = a.zfirst[z];
            if (n == 4) pass_a_zone_thread<4>(a, c, cur, dt, z, s0, zdthyd, bad);
            else pass_a_zone_thread<3>(a, c, cur, dt, z, s0, zdthyd, bad);
        }
    }
    const int nbad = tiles::block_isum<kZoneThreadsZT>(bad);
    block_to_cycle<true, kZoneThreadsZT>(a.cyc_red, zdthyd, nbad);
}

template <bool kRect>
__global__ void __launch_bounds__(kPointThreads) pass_b(DevArrays a, HydroConst c) {
    pdl_wait();
    const Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const int64_t p = (int64_t)blockIdx.x * kPointThreads + threadIdx.x;
    if (p >= a.nump) return;
    pass_b_point<kRect>(a, c, ctl->cycle & 1, ctl->dt, p);
}

// Multi-piece runs: the corner values the neighbours need, and the end of
// the cycle from the reduction over all pieces (min dtnew, max dvovmax,
// summed inverted sides: exact in any order).
__global__ void piece_pack(DevArrays a, const int32_t* __restrict__ send_side, int32_t nsend,
                           unsigned char* __restrict__ send, size_t foff, bool mixed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsend) return;
    const int32_t s = send_side[i];
    if (mixed) {
        reinterpret_cast<float*>(send)[i] = a.cmass_f[s];
        reinterpret_cast<float2*>(send + foff)[i] = a.cforce_f[s];
    } else {
        reinterpret_cast<double*>(send)[i] = a.cmass[s];
        reinterpret_cast<double2*>(send + foff)[i] = a.cforce[s];
    }
}

// The first non-finite element of a[0 .. n): its index into *first by
// atomic minimum (a thread's indices grow along its grid-stride loop, so it
// stops at its first).
__global__ void find_nonfinite(const double* __restrict__ a, int64_t n, unsigned long long* first) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (!isfinite(__ldg(a + i))) {
            atomicMin(first, (unsigned long long)i);
            return;
        }
    }
}

__global__ void piece_finish(DevArrays a, HydroConst c) {
    Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const double* r = a.piece_red;
    finish_cycle(ctl, c, r[0], -r[1], (int)r[2], (int)r[3]);
}

}  // namespace
cudaError_t launch_cycle_fp64(const DevArrays& a, const HydroConst& c, cudaStream_t stream, cudaEvent_t* ev,
                              int phases) {
    const int pb = (int)((a.nump + kPointThreads - 1) / kPointThreads);
    const int zba = (int)((a.numz + kZoneThreadsZT - 1) / kZoneThreadsZT);
    cudaError_t e = cudaSuccess;
    if (phases & kPhaseForces) {
        if (ev) cudaEventRecord(ev[0], stream);
        e = launch_pdl(a.rect_nzx > 0 ? pass_a_zt<true, true> : (a.quads ? pass_a_zt<true> : pass_a_zt<false>), zba,
                       kZoneThreadsZT, 0, stream, a, c);
        if (ev) cudaEventRecord(ev[1], stream);
        if (ev) cudaEventRecord(ev[2], stream);   // no closure pass
    }
    if (phases & kPhaseAdvance) {
        const cudaError_t eb =
            launch_pdl(a.rect_nzx > 0 ? pass_b<true> : pass_b<false>, pb, kPointThreads, 0, stream, a, c);
        if (e == cudaSuccess) e = eb;
        if (ev) cudaEventRecord(ev[3], stream);
        launch_pass_c(a, c, false, stream);   // its last CTA ends the cycle
        if (ev) cudaEventRecord(ev[4], stream);
        if (ev) cudaEventRecord(ev[5], stream);   // no separate finalize step
    }
    return e != cudaSuccess ? e : cudaGetLastError();
}

void launch_piece_pack(const DevArrays& a, const int32_t* send_side, int32_t nsend, unsigned char* send,
                       size_t foff, bool mixed, cudaStream_t stream) {
    if (nsend > 0) piece_pack<<<(nsend + 255) / 256, 256, 0, stream>>>(a, send_side, nsend, send, foff, mixed);
}

void launch_find_nonfinite(const double* a, int64_t n, unsigned long long* first, cudaStream_t stream) {
    if (n <= 0) return;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 8);
    find_nonfinite<<<(int)blocks, 256, 0, stream>>>(a, n, first);
}

void launch_piece_finish(const DevArrays& a, const HydroConst& c, cudaStream_t stream) {
    piece_finish<<<1, 1, 0, stream>>>(a, c);
}


}  // namespace pnt
