// hydro_fp64.cu -- the plain FP64 hydro cycle on sm_100a (one mesh).
//
// One cycle of Hydro::doCycle (Hydro.cc:342-983) runs as four kernels:
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
//           calcWorkRate, calcEnergy, calcRho, calcDvol (block maximum)
//   finalize  calcDt, checkBadSides, time/cycle update and the next
//           cycle's calcGlobalDt (Driver.cc:213-245), all on the device
//
// Pass A runs one thread per zone (pass_a_zone_thread): the zone's sides
// in the reference's side order, each zone-level quantity (centre, sums,
// EOS) formed once, 4-way independent corner work for latency hiding, no
// shuffles; 168 registers, 3 blocks of 128 per SM (13% faster than four
// lanes per zone at a developed 1024^2 Sedov state;
// it is bound by the ~50 correctly rounded FP64 divisions and square roots
// of a zone).  Pass C is the persistent staged kernel of pass_c.cu (one
// thread per zone, inputs gathered into shared memory by asynchronous
// copies); the batched kernels run the same two bodies.  1/elen is formed
// once per side and shared with the neighbouring corner; QCS terms the
// reference computes and then discards (evol and du unless cdiv < 0, zkur
// when cdiv > 0) are not computed, which leaves every stored value
// unchanged.  The arithmetic lives in hydro_fp64_body.cuh (shared with the
// batched kernels); this file is compiled with -fmad=false, so the results
// match a serial CPU run of the reference bit for bit.
#include "hydro_fp64_body.cuh"
#include "zone_tiles.cuh"

namespace pnt {
namespace {

using namespace fp64;

#ifndef PNT_PASS_A_ZT_MIN_BLOCKS
#define PNT_PASS_A_ZT_MIN_BLOCKS 3
#endif
constexpr int kZoneThreadsZT = 128;   // one zone per thread

template <bool kQuads>
__global__ void __launch_bounds__(kZoneThreadsZT, PNT_PASS_A_ZT_MIN_BLOCKS) pass_a_zt(DevArrays a, HydroConst c) {
    const Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const int64_t z = (int64_t)blockIdx.x * kZoneThreadsZT + threadIdx.x;
    double zdthyd = 1.e99;
    int bad = 0;
    if (z < a.numz) {
        const int cur = ctl->cycle & 1;
        const double dt = ctl->dt;
        if (kQuads) {
            pass_a_zone_thread<4>(a, c, cur, dt, z, 4 * z, zdthyd, bad);
        } else {
            const int n = a.znump[z];
            const int64_t s0 = a.zfirst[z];
            if (n == 4) pass_a_zone_thread<4>(a, c, cur, dt, z, s0, zdthyd, bad);
            else pass_a_zone_thread<3>(a, c, cur, dt, z, s0, zdthyd, bad);
        }
    }
    const int nbad = tiles::block_isum<kZoneThreadsZT>(bad);
    if (blockIdx.x >= (unsigned)a.npartA) return;   // partials are sized for this grid
    block_fold<true, kZoneThreadsZT>(zdthyd, a.part_dtnew + blockIdx.x);
    if (threadIdx.x == 0) a.part_badA[blockIdx.x] = nbad;
}

__global__ void __launch_bounds__(kPointThreads) pass_b(DevArrays a, HydroConst c) {
    const Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    const int64_t p = (int64_t)blockIdx.x * kPointThreads + threadIdx.x;
    if (p >= a.nump) return;
    pass_b_point(a, c, ctl->cycle & 1, ctl->dt, p);
}

// finalize: kFinBlocks blocks reduce slices of the pass A / pass C
// partials; the last block to finish (ticket counter) reduces the blocks'
// results and ends the cycle.  Minimum, maximum and integer sums are exact
// in any order, so the result does not depend on which block is last.
constexpr int kFinThreads = 512;

__device__ __forceinline__ void fin_block_reduce(double& dtn, double& dvm, int& badA, int& badC) {
    __shared__ double sdt[kFinThreads / 32], sdv[kFinThreads / 32];
    __shared__ int sba[kFinThreads / 32], sbc[kFinThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        dtn = dmin(dtn, __shfl_xor_sync(kFull, dtn, o));
        const double w = __shfl_xor_sync(kFull, dvm, o);
        dvm = (w > dvm) ? w : dvm;
        badA += __shfl_xor_sync(kFull, badA, o);
        badC += __shfl_xor_sync(kFull, badC, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sdt[warp] = dtn; sdv[warp] = dvm; sba[warp] = badA; sbc[warp] = badC; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < kFinThreads / 32; ++i) {
            dtn = dmin(dtn, sdt[i]);
            dvm = (sdv[i] > dvm) ? sdv[i] : dvm;
        }
        badA = 0;
        badC = 0;
        for (int i = 0; i < kFinThreads / 32; ++i) { badA += sba[i]; badC += sbc[i]; }
    }
    __syncthreads();   // the shared slots are reused by the last block
}

__global__ void __launch_bounds__(kFinThreads) finalize(DevArrays a, HydroConst c, int nblocksA, int nblocksC) {
    Ctl* ctl = a.ctl;
    if (skip_cycle(ctl)) return;
    double dtn = 1.e99, dvm = 1.e-99;
    int badA = 0, badC = 0;
    const int stride = gridDim.x * kFinThreads;
    for (int i = blockIdx.x * kFinThreads + threadIdx.x; i < nblocksA; i += stride) {
        dtn = dmin(dtn, a.part_dtnew[i]);
        badA += a.part_badA[i];
    }
    for (int i = blockIdx.x * kFinThreads + threadIdx.x; i < nblocksC; i += stride) {
        const double v = a.part_dvov[i];
        dvm = (v > dvm) ? v : dvm;
        badC += a.part_badC[i];
    }
    fin_block_reduce(dtn, dvm, badA, badC);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        a.fin_part[blockIdx.x] = dtn;
        a.fin_part[kFinBlocks + blockIdx.x] = dvm;
        a.fin_bad[blockIdx.x] = badA;
        a.fin_bad[kFinBlocks + blockIdx.x] = badC;
        __threadfence();
        last = atomicAdd(a.fin_ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    dtn = 1.e99;
    dvm = 1.e-99;
    badA = badC = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kFinThreads) {
        dtn = dmin(dtn, __ldcg(a.fin_part + i));
        const double v = __ldcg(a.fin_part + kFinBlocks + i);
        dvm = (v > dvm) ? v : dvm;
        badA += __ldcg(a.fin_bad + i);
        badC += __ldcg(a.fin_bad + kFinBlocks + i);
    }
    fin_block_reduce(dtn, dvm, badA, badC);
    if (threadIdx.x == 0) {
        *a.fin_ticket = 0u;
        if (a.piece_red) {   // a piece: the caller reduces over pieces, then piece_finish
            a.piece_red[0] = dtn;
            a.piece_red[1] = -dvm;
            a.piece_red[2] = (double)badA;
            a.piece_red[3] = (double)badC;
        } else {
            finish_cycle(ctl, c, dtn, dvm, badA, badC);
        }
    }
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
    if (phases & kPhaseForces) {
        if (ev) cudaEventRecord(ev[0], stream);
        if (a.quads) pass_a_zt<true><<<zba, kZoneThreadsZT, 0, stream>>>(a, c);
        else pass_a_zt<false><<<zba, kZoneThreadsZT, 0, stream>>>(a, c);
        if (ev) cudaEventRecord(ev[1], stream);
        if (ev) cudaEventRecord(ev[2], stream);   // no closure pass
    }
    if (phases & kPhaseAdvance) {
        pass_b<<<pb, kPointThreads, 0, stream>>>(a, c);
        if (ev) cudaEventRecord(ev[3], stream);
        launch_pass_c(a, c, false, stream);
        if (ev) cudaEventRecord(ev[4], stream);
        finalize<<<kFinBlocks, kFinThreads, 0, stream>>>(a, c, zba, a.gridC);
        if (ev) cudaEventRecord(ev[5], stream);
    }
    return cudaGetLastError();
}

void launch_piece_pack(const DevArrays& a, const int32_t* send_side, int32_t nsend, unsigned char* send,
                       size_t foff, bool mixed, cudaStream_t stream) {
    if (nsend > 0) piece_pack<<<(nsend + 255) / 256, 256, 0, stream>>>(a, send_side, nsend, send, foff, mixed);
}

void launch_piece_finish(const DevArrays& a, const HydroConst& c, cudaStream_t stream) {
    piece_finish<<<1, 1, 0, stream>>>(a, c);
}

void launch_finalize(const DevArrays& a, const HydroConst& c, int nA, int nC, cudaStream_t stream) {
    finalize<<<kFinBlocks, kFinThreads, 0, stream>>>(a, c, nA, nC);
}

}  // namespace pnt
