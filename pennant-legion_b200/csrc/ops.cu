// ops.cu -- per-task operators on caller-owned device arrays.
//
// These replace individual GPU task variants of the reference one for one,
// for callers that keep their own field storage (as the reference's Legion
// regions do) and only want the kernel.  Compiled with -fmad=false like
// the cycle kernels, so results are bit-identical to the reference's
// serial CPU tasks.
#include "pennant_b200.h"
#include "pnt_internal.h"

#include <cuda_runtime.h>

using namespace pnt;

namespace {

constexpr int kDtThreads = 256;
constexpr int kDtZonesPerThread = 8;
constexpr int kDtZonesPerBlock = kDtThreads * kDtZonesPerThread;   // 2048
constexpr int kDtFinThreads = 1024;

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double fold_max(double a, double b) { return (b > a) ? b : a; }

// calcDtNew (Hydro.cc:1591-1619) and calcDvol (Hydro.cc:1622-1644) over
// one block's zones; partial[2*block] = min zdthyd, partial[2*block+1] =
// max |dV/V0|, in the reference's fold semantics (NaN terms never win).
__global__ void __launch_bounds__(kDtThreads) dt_partials(const double* __restrict__ zdl,
                                                          const double* __restrict__ zdu,
                                                          const double* __restrict__ zss,
                                                          const double* __restrict__ zvol,
                                                          const double* __restrict__ zvol0, int64_t numz,
                                                          double cfl, double* __restrict__ partial) {
    double dtn = 1.e99, dvm = 1.e-99;
    const int64_t base = (int64_t)blockIdx.x * kDtZonesPerBlock + threadIdx.x;
#pragma unroll
    for (int j = 0; j < kDtZonesPerThread; ++j) {
        const int64_t z = base + (int64_t)j * kDtThreads;
        if (z < numz) {
            // cdu = max(zdu, max(zss, fuzz)) with std::max(a, b) = (a < b) ? b : a
            const double zssz = zss[z], zduz = zdu[z];
            const double inner = (zssz < 1.e-99) ? 1.e-99 : zssz;
            const double cdu = (zduz < inner) ? inner : zduz;
            const double zdthyd = zdl[z] * cfl / cdu;
            dtn = (zdthyd < dtn) ? zdthyd : dtn;
            const double zdvov = fabs((zvol[z] - zvol0[z]) / zvol0[z]);
            dvm = (zdvov > dvm) ? zdvov : dvm;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        dtn = dmin(dtn, __shfl_xor_sync(0xffffffffu, dtn, o));
        dvm = fold_max(dvm, __shfl_xor_sync(0xffffffffu, dvm, o));
    }
    __shared__ double sdt[kDtThreads / 32], sdv[kDtThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sdt[warp] = dtn;
        sdv[warp] = dvm;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < kDtThreads / 32; ++i) {
            dtn = dmin(dtn, sdt[i]);
            dvm = fold_max(dvm, sdv[i]);
        }
        partial[2 * blockIdx.x] = dtn;
        partial[2 * blockIdx.x + 1] = dvm;
    }
}

// Reduces the partials and applies calcDtTask (Hydro.cc:1647-1667):
// out[0] = dtrec, out[1] = dtnew, out[2] = dvovmax.
__global__ void __launch_bounds__(kDtFinThreads) dt_finish(const double* __restrict__ partial, int nblocks,
                                                           double dtlast, double cflv, double* __restrict__ out) {
    double dtn = 1.e99, dvm = 1.e-99;
    for (int i = threadIdx.x; i < nblocks; i += kDtFinThreads) {
        dtn = dmin(dtn, partial[2 * i]);
        dvm = fold_max(dvm, partial[2 * i + 1]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        dtn = dmin(dtn, __shfl_xor_sync(0xffffffffu, dtn, o));
        dvm = fold_max(dvm, __shfl_xor_sync(0xffffffffu, dvm, o));
    }
    __shared__ double sdt[kDtFinThreads / 32], sdv[kDtFinThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sdt[warp] = dtn;
        sdv[warp] = dvm;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int i = 1; i < kDtFinThreads / 32; ++i) {
        dtn = dmin(dtn, sdt[i]);
        dvm = fold_max(dvm, sdv[i]);
    }
    double dtrec = 1.e99;
    if (dtn < dtrec) dtrec = dtn;
    const double dtnew2 = dtlast * cflv / dvm;
    if (dtnew2 < dtrec) dtrec = dtnew2;
    out[0] = dtrec;
    out[1] = dtn;
    out[2] = dvm;
}

pnt_status check_dt_args(const double* zdl, const double* zdu, const double* zss, const double* zvol,
                         const double* zvol0, int64_t numz, const double* out) {
    if (!out) return fail(PNT_ERR_INVALID_ARG, "null output pointer");
    if (numz < 0) return fail(PNT_ERR_INVALID_ARG, "numz < 0");
    if (numz > 0 && (!zdl || !zdu || !zss || !zvol || !zvol0)) return fail(PNT_ERR_INVALID_ARG, "null input pointer");
    if ((numz + kDtZonesPerBlock - 1) / kDtZonesPerBlock > INT32_MAX / 2)
        return fail(PNT_ERR_INVALID_ARG, "numz too large");
    return PNT_OK;
}

}  // namespace

extern "C" pnt_status pnt_op_calc_dt(const double* zdl, const double* zdu, const double* zss, const double* zvol,
                                     const double* zvol0, int64_t numz, double cfl, double cflv, double dtlast,
                                     double* out, void* stream) {
    pnt_status st = check_dt_args(zdl, zdu, zss, zvol, zvol0, numz, out);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int nblocks = (int)((numz + kDtZonesPerBlock - 1) / kDtZonesPerBlock);
    double* partial = nullptr;
    cudaError_t e = cudaSuccess;
    if (nblocks > 0) {
        // stream-ordered scratch for the per-block partials
        e = cudaMallocAsync((void**)&partial, sizeof(double) * 2 * (size_t)nblocks, s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(PNT_ERR_NOMEM, "scratch allocation: %s", cudaGetErrorString(e));
        }
        dt_partials<<<nblocks, kDtThreads, 0, s>>>(zdl, zdu, zss, zvol, zvol0, numz, cfl, partial);
    }
    dt_finish<<<1, kDtFinThreads, 0, s>>>(partial, nblocks, dtlast, cflv, out);
    e = cudaGetLastError();
    if (partial) cudaFreeAsync(partial, s);
    if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "pnt_op_calc_dt launch: %s", cudaGetErrorString(e));
    return PNT_OK;
}
