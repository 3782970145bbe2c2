// ops.cu -- per-task operators on caller-owned device arrays.
//
// These replace individual GPU task variants of the reference one for one,
// for callers that keep their own field storage (as the reference's Legion
// regions do) and only want the kernel.  Compiled with -fmad=false like
// the cycle kernels, so results are bit-identical to the reference's
// serial CPU tasks.
#include "pennant_b200.h"
#include "pnt_internal.h"

#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

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

// ---------------------------------------------------------------------
// pnt_op_calc_dt_noalloc: the same two kernels with their per-block
// partials in a fixed device array instead of allocated scratch.
//
// Who needs it: code that must not allocate device memory itself.  A
// Legion GPU task is the reference's own case: the runtime's mapper owns
// every instance and a task body is expected to take memory only through
// the runtime.  Others are latency-critical loops where an allocation can
// stall on device synchronisation or fail under memory pressure, and
// processes whose device memory is capped by a pool they do not control.
//
// The array below exists once per GPU that loads this library and stays
// resident until the process exits (128 KiB).  Every call on a device uses
// the same array and overwrites the partials it later reads, so nothing
// needs clearing between calls; calls that overlap on the GPU (different
// streams, or different host threads on one device) race on it and must be
// serialised by the caller.  The first call on each device looks up the
// array's device address (cudaGetSymbolAddress); make that first call
// before any stream capture.  The address is kept per device together with
// the identity of the device's CUDA context: after cudaDeviceReset (or any
// other end of the context) the array lives in a new context, and the next
// call looks the address up again -- make that call before stream capture
// too.
// ---------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxBlocks = 8192;
constexpr int64_t kNoAllocMaxZones = (int64_t)kNoAllocMaxBlocks * kDtZonesPerBlock;   // 16,777,216
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_dt_scratch[2 * kNoAllocMaxBlocks];

std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

// The unique id of the calling thread's current CUDA context (cuCtxGetId,
// reached through the runtime's driver entry-point query, so the library
// needs no link to libcuda), or 0 when it cannot be had.  Called with
// g_scratch_mu held.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        looked_up = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    }
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_dt_scratch on the current device.  In host code the
// symbol name is only a host-side stand-in, never a device address.
pnt_status noalloc_scratch(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PNT_ERR_NO_DEVICE, "no current CUDA device: %s", cudaGetErrorString(e));
    }
    if (dev < 0 || dev >= kMaxDevices) return fail(PNT_ERR_UNSUPPORTED, "device ordinal %d >= %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    // the runtime makes the device's primary context current at its first
    // call; the id is taken after cudaGetSymbolAddress on a first look-up
    unsigned long long ctx = g_scratch_addr[dev] ? current_context_id() : 0;
    if (!g_scratch_addr[dev] || (ctx != 0 && ctx != g_scratch_ctx[dev])) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_dt_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return fail(PNT_ERR_CUDA, "cudaGetSymbolAddress of the no-allocation scratch: %s",
                        cudaGetErrorString(e));
        }
        g_scratch_addr[dev] = p;
        g_scratch_ctx[dev] = current_context_id();
    }
    *out = static_cast<double*>(g_scratch_addr[dev]);
    return PNT_OK;
}

}  // namespace

extern "C" pnt_status pnt_op_calc_dt_noalloc(const double* zdl, const double* zdu, const double* zss,
                                             const double* zvol, const double* zvol0, int64_t numz, double cfl,
                                             double cflv, double dtlast, double* out, void* stream) {
    pnt_status st = check_dt_args(zdl, zdu, zss, zvol, zvol0, numz, out);
    if (st) return st;
    if (numz > kNoAllocMaxZones)
        return fail(PNT_ERR_INVALID_ARG,
                    "numz %lld exceeds the no-allocation limit of %lld zones (use pnt_op_calc_dt)",
                    (long long)numz, (long long)kNoAllocMaxZones);
    double* scratch = nullptr;
    if ((st = noalloc_scratch(&scratch))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int nblocks = (int)((numz + kDtZonesPerBlock - 1) / kDtZonesPerBlock);
    if (nblocks > 0) dt_partials<<<nblocks, kDtThreads, 0, s>>>(zdl, zdu, zss, zvol, zvol0, numz, cfl, scratch);
    dt_finish<<<1, kDtFinThreads, 0, s>>>(scratch, nblocks, dtlast, cflv, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "pnt_op_calc_dt_noalloc launch: %s", cudaGetErrorString(e));
    return PNT_OK;
}
