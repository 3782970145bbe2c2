// batch.cu -- many independent meshes advanced together (pnt_batch_*).
//
// The meshes are concatenated into one set of device arrays (global point,
// side and zone numbering; every instance keeps its own run state and
// constants).  One cycle of the batch is four persistent launches: each
// CTA walks a work list of (instance, tile) entries, so meshes of very
// uneven size share the GPU without a launch per mesh, and instances that
// are done are skipped tile by tile.  The per-zone and per-point
// arithmetic is the FP64 body shared with the single-mesh kernels
// (pass A: pass_a_zone_thread of hydro_fp64_body.cuh, one thread per zone;
// pass C: the staged corrector of pass_c_staged.cuh), so every instance is
// bit-identical to its own single-mesh run; tiles only change which CTA
// does the work.  Pass A runs one CTA per zone tile; passes B and C are
// persistent.  The batch cycle is captured in a CUDA graph.  The tile size
// (passes A and C) and the point pass's CTAs per SM are picked by
// pnt_batch_tune, which times candidate shapes on the run's own cycles (the
// results do not depend on the shape).
//
// Compiled with -fmad=false (FP64 parity).
#include "batch_dev.h"
#include "hydro_fp64_body.cuh"
#include "pass_c_staged.cuh"
#include "pnt_internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

using namespace pnt;

namespace pnt {
namespace {

using namespace fp64;

// Pass A: one CTA per tile (no persistent loop: its state would cost the
// zone body registers), one thread per zone (pass_a_zone_thread), 128 zones
// per step through the tile; one partial per tile.
// kAllQuads: every instance's zones are quads at sides 4z..4z+3, so only
// the 4-sided body is compiled (fewer registers than the general form).
template <bool kAllQuads>
__global__ void __launch_bounds__(kBatchZT, 3) batch_pass_a(BatchDev b) {
    {
        const int t = blockIdx.x;
        if (t >= b.nztiles) return;   // no tiles left: the grid is one idle CTA
        const Tile tile = b.ztiles[t];
        const Ctl& ctl = b.ctls[tile.inst];
        if (inst_skip(ctl)) return;   // uniform over the CTA
        const HydroConst& c = b.consts[tile.inst];
        const int cur = ctl.cycle & 1;
        const double dt = ctl.dt;
        double fold = 1.e99;
        int nbad = 0;
        for (int zb = tile.beg; zb < tile.end; zb += kBatchZT) {
            const int64_t z = (int64_t)zb + threadIdx.x;
            if (z >= tile.end) continue;
            double v = 1.e99;
            if (tile.nzx > 0) {   // a rect instance: point indices from the zone index
                const RectZoneIn in(b.a, cur, z, tile.nzx, z - tile.zo, tile.po);
                pass_a_zone_thread<4>(b.a, c, in, dt, z, 4 * z, v, nbad);
            } else if (kAllQuads || tile.quads) {
                pass_a_zone_thread<4>(b.a, c, cur, dt, z, 4 * z, v, nbad);
            } else {
                const int n = b.a.znump[z];
                const int64_t s0 = b.a.zfirst[z];
                if (n == 4) pass_a_zone_thread<4>(b.a, c, cur, dt, z, s0, v, nbad);
                else pass_a_zone_thread<3>(b.a, c, cur, dt, z, s0, v, nbad);
            }
            fold = dmin(fold, v);
        }
        nbad = tiles::block_isum<kBatchZT>(nbad);
        block_fold<true, kBatchZT>(fold, b.a.part_dtnew + t);
        if (threadIdx.x == 0) b.a.part_badA[t] = nbad;
    }
}

// Pass C: the staged corrector of pass_c_staged.cuh, one stage, its
// kTile zones per step through the tile (copies issued, waited for,
// computed); one partial per tile.
// kAllQuads as in batch_pass_a; quad tiles load the next step's point
// indices while the current step's copies are in flight.
template <bool kAllQuads, bool kMixed>
__global__ void __launch_bounds__(stagedc::kTile) batch_pass_c(BatchDev b) {
    extern __shared__ __align__(16) unsigned char smem_c[];
    const int th = threadIdx.x;
    for (int t = blockIdx.x; t < b.nztiles; t += gridDim.x) {
        const Tile tile = b.ztiles[t];
        const Ctl& ctl = b.ctls[tile.inst];
        if (inst_skip(ctl)) continue;   // uniform over the CTA
        const HydroConst& c = b.consts[tile.inst];
        const int cur = ctl.cycle & 1;
        const double dt = ctl.dt, dtinv = ctl.dtinv;
        double dvm = 1.e-99;
        int nbad = 0;
        const bool quads = kAllQuads || tile.quads;
        tiles::ZoneIdx nix{};
        if (quads && (int64_t)tile.beg + th < tile.end) nix = tiles::load_idx<true>(b.a, (int64_t)tile.beg + th);
        for (int zb = tile.beg; zb < tile.end; zb += stagedc::kTile) {
            const int64_t z = (int64_t)zb + th;
            const bool zok = z < tile.end;
            if (zok) {
                const tiles::ZoneIdx ix = quads ? nix : tiles::load_idx<false>(b.a, z);
                stagedc::issue(b.a, cur, smem_c, th, z, ix);
            }
            tiles::commit();
            if (quads && z + stagedc::kTile < tile.end) nix = tiles::load_idx<true>(b.a, z + stagedc::kTile);
            tiles::wait_groups<0>();
            if (zok) {
                const double d = quads ? stagedc::zone<true, kMixed>(b.a, c, smem_c, th, z, dt, dtinv, nbad)
                                       : stagedc::zone<false, kMixed>(b.a, c, smem_c, th, z, dt, dtinv, nbad);
                dvm = (d > dvm) ? d : dvm;
            }
        }
        nbad = tiles::block_isum<stagedc::kTile>(nbad);
        block_fold<false, stagedc::kTile>(dvm, b.a.part_dvov + t);
        if (threadIdx.x == 0) b.a.part_badC[t] = nbad;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBatchThreads) batch_point_pass(BatchDev b) {
    for (int t = blockIdx.x; t < b.nptiles; t += gridDim.x) {
        const Tile tile = b.ptiles[t];
        const Ctl& ctl = b.ctls[tile.inst];
        if (inst_skip(ctl)) continue;
        const HydroConst& c = b.consts[tile.inst];
        const int cur = ctl.cycle & 1;
        for (int64_t p = (int64_t)tile.beg + threadIdx.x; p < tile.end; p += kBatchThreads)
            pass_b_point(b.a, c, cur, ctl.dt, p);
    }
}

// One warp per instance: reduce its tiles' partials and end its cycle.
__global__ void __launch_bounds__(kBatchThreads) batch_finalize(BatchDev b) {
    const int inst = (int)((blockIdx.x * (int64_t)kBatchThreads + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (inst >= b.ninst) return;   // whole warps leave together
    Ctl* ctl = b.ctls + inst;
    if (inst_skip(*ctl)) return;
    double dtn = 1.e99, dvm = 1.e-99;
    int badA = 0, badC = 0;
    for (int t = b.inst_tbeg[inst] + lane; t < b.inst_tbeg[inst + 1]; t += 32) {
        dtn = dmin(dtn, b.a.part_dtnew[t]);
        const double v = b.a.part_dvov[t];
        dvm = (v > dvm) ? v : dvm;
        badA += b.a.part_badA[t];
        badC += b.a.part_badC[t];
    }
    for (int o = 16; o > 0; o >>= 1) {
        dtn = dmin(dtn, __shfl_xor_sync(kFull, dtn, o));
        const double w = __shfl_xor_sync(kFull, dvm, o);
        dvm = (w > dvm) ? w : dvm;
        badA += __shfl_xor_sync(kFull, badA, o);
        badC += __shfl_xor_sync(kFull, badC, o);
    }
    if (lane == 0) finish_cycle(ctl, b.consts[inst], dtn, dvm, badA, badC);
}

// Count of instances still running, for the host's stop test.
__global__ void batch_count_running(const Ctl* ctls, int ninst, int* out) {
    int n = 0;
    for (int i = threadIdx.x; i < ninst; i += blockDim.x) n += inst_skip(ctls[i]) ? 0 : 1;
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(kFull, n, o);
    __shared__ int s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += s[i];
        *out = t;
    }
}

}  // namespace
}  // namespace pnt

// ---------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------
namespace {

#define CUDA_TRY(expr)                                                                                  \
    do {                                                                                                \
        const cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess)                                                                          \
            return fail(PNT_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

struct Shape {
    int zones_per_tile;
    int ctas_per_sm;
};

}  // namespace

struct pnt_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    BatchDev b{};
    int32_t ninst = 0;
    std::vector<int64_t> zoff, poff, soff;      // instance offsets (host)
    std::vector<int32_t> nz, np, ns;
    std::vector<int32_t> quads;
    std::vector<int32_t> rect_nzx;               // zones a row of a rect-numbered quad instance (else 0)
    bool all_quads = false;                      // every instance: quads at sides 4z..4z+3
    bool mixed = false;                          // the mixed-precision cycle (every instance)
    Ctl* ctl_host = nullptr;                     // pinned [ninst]
    int* running_dev = nullptr;
    int* running_host = nullptr;                 // pinned
    Shape shape{256, 3};
    int nsm = 148;
    int grid_c = 148;                            // resident pass C CTAs (occupancy x SMs)
    // device tile lists (rebuilt when the shape changes)
    Tile* ztiles = nullptr;
    Tile* ptiles = nullptr;
    int32_t* inst_tbeg = nullptr;
    void* parts = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_cycles = 8;
    int32_t live = 0;                            // instances in the current work lists
    std::vector<char> listed;                    // [ninst] the instance is in the current work lists

    ~pnt_batch() {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (graph) cudaGraphExecDestroy(graph);
        for (void* p : allocs) cudaFree(p);
        if (ztiles) cudaFree(ztiles);
        if (ptiles) cudaFree(ptiles);
        if (inst_tbeg) cudaFree(inst_tbeg);
        if (parts) cudaFree(parts);
        if (ctl_host) cudaFreeHost(ctl_host);
        if (running_host) cudaFreeHost(running_host);
        if (stream) cudaStreamDestroy(stream);
        if (prev >= 0) cudaSetDevice(prev);
    }

    template <typename T>
    pnt_status alloc(T** out, size_t count) {
        void* p = nullptr;
        const cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(e == cudaErrorMemoryAllocation ? PNT_ERR_NOMEM : PNT_ERR_CUDA, "cudaMalloc of %zu bytes: %s",
                        count * sizeof(T), cudaGetErrorString(e));
        }
        allocs.push_back(p);
        *out = static_cast<T*>(p);
        return PNT_OK;
    }

    // Work lists for a tile shape over the instances still running (ctl_host
    // must be current); partial arrays sized to the zone tiles.  Finished
    // instances get no tiles, so the persistent passes do not walk them.
    pnt_status build_tiles(const Shape& sh) {
        std::vector<Tile> zt, pt;
        std::vector<int32_t> tb(ninst + 1, 0);
        const int ppt = kBatchThreads * 4;   // points per point tile
        int32_t nlive = 0;
        listed.assign(ninst, 0);
        for (int i = 0; i < ninst; ++i) {
            tb[i] = (int32_t)zt.size();
            if (ctl_host[i].done) continue;
            ++nlive;
            listed[i] = 1;
            for (int64_t z = 0; z < nz[i]; z += sh.zones_per_tile)
                zt.push_back({i, (int32_t)(zoff[i] + z), (int32_t)(zoff[i] + std::min<int64_t>(nz[i], z + sh.zones_per_tile)),
                              quads[i], rect_nzx[i], (int32_t)zoff[i], (int32_t)poff[i], 0});
            for (int64_t p = 0; p < np[i]; p += ppt)
                pt.push_back({i, (int32_t)(poff[i] + p), (int32_t)(poff[i] + std::min<int64_t>(np[i], p + ppt)), quads[i]});
        }
        tb[ninst] = (int32_t)zt.size();
        live = nlive;
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
        CUDA_TRY(cudaStreamSynchronize(stream));
        if (ztiles) cudaFree(ztiles);
        if (ptiles) cudaFree(ptiles);
        if (inst_tbeg) cudaFree(inst_tbeg);
        if (parts) cudaFree(parts);
        ztiles = nullptr; ptiles = nullptr; inst_tbeg = nullptr; parts = nullptr;
        const size_t nzt = zt.size();
        CUDA_TRY(cudaMalloc(&ztiles, std::max<size_t>(nzt, 1) * sizeof(Tile)));
        CUDA_TRY(cudaMalloc(&ptiles, std::max<size_t>(pt.size(), 1) * sizeof(Tile)));
        CUDA_TRY(cudaMalloc(&inst_tbeg, tb.size() * sizeof(int32_t)));
        CUDA_TRY(cudaMalloc(&parts, std::max<size_t>(nzt, 1) * (2 * sizeof(double) + 2 * sizeof(int32_t))));
        if (nzt) CUDA_TRY(cudaMemcpy(ztiles, zt.data(), nzt * sizeof(Tile), cudaMemcpyHostToDevice));
        if (!pt.empty()) CUDA_TRY(cudaMemcpy(ptiles, pt.data(), pt.size() * sizeof(Tile), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(inst_tbeg, tb.data(), tb.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        b.ztiles = ztiles;
        b.ptiles = ptiles;
        b.nztiles = (int32_t)nzt;
        b.nptiles = (int32_t)pt.size();
        b.inst_tbeg = inst_tbeg;
        b.a.part_dtnew = static_cast<double*>(parts);
        b.a.part_dvov = b.a.part_dtnew + nzt;
        b.a.part_badA = reinterpret_cast<int32_t*>(b.a.part_dvov + nzt);
        b.a.part_badC = b.a.part_badA + nzt;
        b.a.npartA = b.a.npartC = (int32_t)nzt;
        shape = sh;
        return PNT_OK;
    }

    cudaError_t launch_cycle(cudaEvent_t* ev = nullptr) {
        const int grid_p = std::max(1, std::min(b.nptiles, nsm * shape.ctas_per_sm));
        const int grid_f = (ninst * 32 + kBatchThreads - 1) / kBatchThreads;
        if (ev) cudaEventRecord(ev[0], stream);
        if (mixed) launch_batch_pass_a_mixed(b, all_quads, stream);
        else if (all_quads) batch_pass_a<true><<<std::max(1, b.nztiles), kBatchZT, 0, stream>>>(b);
        else batch_pass_a<false><<<std::max(1, b.nztiles), kBatchZT, 0, stream>>>(b);
        if (ev) cudaEventRecord(ev[1], stream);
        if (mixed) launch_batch_point_pass_mixed(b, grid_p, stream);
        else batch_point_pass<<<grid_p, kBatchThreads, 0, stream>>>(b);
        if (ev) cudaEventRecord(ev[2], stream);
        const int gc = std::max(1, std::min(b.nztiles, grid_c));
        const size_t smc = stagedc::kSmemBytes;
        if (mixed) {
            if (all_quads) batch_pass_c<true, true><<<gc, stagedc::kTile, smc, stream>>>(b);
            else batch_pass_c<false, true><<<gc, stagedc::kTile, smc, stream>>>(b);
        } else {
            if (all_quads) batch_pass_c<true, false><<<gc, stagedc::kTile, smc, stream>>>(b);
            else batch_pass_c<false, false><<<gc, stagedc::kTile, smc, stream>>>(b);
        }
        if (ev) cudaEventRecord(ev[3], stream);
        batch_finalize<<<grid_f, kBatchThreads, 0, stream>>>(b);
        if (ev) cudaEventRecord(ev[4], stream);
        return cudaGetLastError();
    }

    pnt_status ensure_graph() {
        if (graph) return PNT_OK;
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < graph_cycles && e == cudaSuccess; ++i) e = launch_cycle();
        const cudaError_t e2 = cudaStreamEndCapture(stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return fail(PNT_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { graph = nullptr; return fail(PNT_ERR_CUDA, "batch graph: %s", cudaGetErrorString(e)); }
        return PNT_OK;
    }

    pnt_status enqueue(int n) {
        pnt_status st = ensure_graph();
        if (st) return st;
        while (n >= graph_cycles) {
            CUDA_TRY(cudaGraphLaunch(graph, stream));
            n -= graph_cycles;
        }
        for (; n > 0; --n) CUDA_TRY(launch_cycle());
        return PNT_OK;
    }

    pnt_status running(int* out) {
        batch_count_running<<<1, 1024, 0, stream>>>(b.ctls, ninst, running_dev);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(running_host, running_dev, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        *out = *running_host;
        return PNT_OK;
    }

    // Share of the listed zones that belong to finished instances (ctl_host
    // current).  Their tiles cost little (each CTA sees the instance done
    // and returns), so the lists are rebuilt only once they hold a quarter
    // of the listed zones: every rebuild drains the stream, reallocates the
    // lists and captures a new graph.
    double finished_share() const {
        int64_t all = 0, fin = 0;
        for (int i = 0; i < ninst; ++i) {
            if (i >= (int)listed.size() || !listed[i]) continue;
            all += nz[i];
            if (ctl_host[i].done) fin += nz[i];
        }
        return all > 0 ? (double)fin / (double)all : 0.;
    }

    pnt_status fetch_ctls() {
        CUDA_TRY(cudaMemcpyAsync(ctl_host, b.ctls, sizeof(Ctl) * ninst, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return PNT_OK;
    }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int now = -1;
        if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
    }
};

// Hydro::init of one instance into the concatenated host arrays (the same
// steps as the single-mesh object, hydro.cu).
void init_instance(const Mesh& m, const pnt_params& p, HydroConst& c, Ctl& ctl, double* zr, double* ze, double* zwrate,
                   double* zm, double* zetot, double* pu, uint16_t* bcmask) {
    c.cfl = p.cfl;
    c.cflv = p.cflv;
    c.gm1 = p.gamma - 1.;
    c.ssmin2 = std::max(p.pgas_ssmin * p.pgas_ssmin, 1.e-99);
    c.alfa = p.alfa;
    c.tts_ssmin = p.tts_ssmin;
    c.gammap1 = p.qgamma + 1.0;
    c.q1 = p.q1;
    c.q2 = p.q2;
    c.dtmax = p.dtmax;
    c.dtinit = p.dtinit;
    c.dtfac = p.dtfac;
    c.tstop = p.tstop;
    c.cstop = p.cstop;
    c.nbc = p.nbcx + p.nbcy;
    const double eps = 1.e-12;
    for (int bi = 0; bi < c.nbc; ++bi) {
        const bool xplane = bi < p.nbcx;
        const double bound = xplane ? p.bcx[bi] : p.bcy[bi - p.nbcx];
        c.vfix[bi][0] = xplane ? 1. : 0.;
        c.vfix[bi][1] = xplane ? 0. : 1.;
        for (int64_t q = 0; q < m.nump; ++q) {
            const double coord = xplane ? m.px[2 * q] : m.px[2 * q + 1];
            if (fabs(coord - bound) < eps) bcmask[q] |= (uint16_t)(1u << bi);
        }
    }
    for (int64_t z = 0; z < m.numz; ++z) {
        zr[z] = p.rinit;
        ze[z] = p.einit;
        zwrate[z] = 0.;
    }
    if (p.has_subregion) {
        const double* sr = p.subregion;
        for (int64_t z = 0; z < m.numz; ++z) {
            const double zxx = m.zx[2 * z], zxy = m.zx[2 * z + 1];
            if (zxx > (sr[0] - eps) && zxx < (sr[1] + eps) && zxy > (sr[2] - eps) && zxy < (sr[3] + eps)) {
                zr[z] = p.rinitsub;
                ze[z] = p.einitsub;
            }
        }
    }
    for (int64_t z = 0; z < m.numz; ++z) {
        zm[z] = zr[z] * m.zvol[z];
        zetot[z] = ze[z] * zm[z];
    }
    if (p.uinitradial != 0.) {
        for (int64_t q = 0; q < m.nump; ++q) {
            const double x = m.px[2 * q], y = m.px[2 * q + 1];
            const double pmag = sqrt(x * x + y * y);
            if (pmag > eps) {
                const double rinv = 1. / pmag;
                pu[2 * q] = (x * p.uinitradial) * rinv;
                pu[2 * q + 1] = (y * p.uinitradial) * rinv;
            }
        }
    }
    std::memset(&ctl, 0, sizeof(ctl));
    double dt = p.dtmax;
    if (p.dtinit < dt) dt = p.dtinit;
    if ((p.tstop - 0.) < dt) dt = p.tstop - 0.;
    ctl.dt = dt;
    ctl.dtinv = 1. / dt;
    ctl.done = (p.cstop <= 0 || !(0. < p.tstop)) ? 1 : 0;
    ctl.stop_at = INT_MAX;
}

}  // namespace

extern "C" {

pnt_status pnt_batch_create(const pnt_mesh* const* meshes, const pnt_params* params, int32_t n, int32_t device,
                            pnt_batch** out) {
    if (!meshes || !params || !out || n <= 0) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(PNT_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(PNT_ERR_INVALID_ARG, "device %d out of range", device);
    for (int i = 0; i < n; ++i) {
        if (!meshes[i]) return fail(PNT_ERR_INVALID_ARG, "null mesh %d", i);
        if (params[i].precision == PNT_PREC_LEARNED)
            return fail(PNT_ERR_UNSUPPORTED, "batched instances run the FP64 or the mixed cycle (instance %d)", i);
        if (params[i].precision != params[0].precision)
            return fail(PNT_ERR_UNSUPPORTED, "batched instances share one precision (instance %d)", i);
        if (params[i].nbcx + params[i].nbcy > kMaxBC) return fail(PNT_ERR_UNSUPPORTED, "too many BC planes");
    }
    DeviceGuard dg(device);
    pnt_batch* bt = new (std::nothrow) pnt_batch();
    if (!bt) return fail(PNT_ERR_NOMEM, "out of memory");
    bt->device = device;
    bt->ninst = n;
    bt->mixed = params[0].precision == PNT_PREC_MIXED;
    cudaDeviceGetAttribute(&bt->nsm, cudaDevAttrMultiProcessorCount, device);
    pnt_status st = PNT_OK;
    try {
        int64_t NZ = 0, NP = 0, NS = 0;
        for (int i = 0; i < n; ++i) {
            const Mesh& m = meshes[i]->m;
            bt->zoff.push_back(NZ);
            bt->poff.push_back(NP);
            bt->soff.push_back(NS);
            bt->nz.push_back(m.numz);
            bt->np.push_back(m.nump);
            bt->ns.push_back(m.nums);
            // the quad fast path indexes sides as 4z, which holds while every
            // earlier instance is all-quad too
            bt->quads.push_back(m.all_quads && NS == 4 * NZ ? 1 : 0);
            bt->rect_nzx.push_back(bt->quads.back() ? m.rect_nzx : 0);
            NZ += m.numz;
            NP += m.nump;
            NS += m.nums;
        }
        bt->all_quads = std::all_of(bt->quads.begin(), bt->quads.end(), [](int32_t q) { return q != 0; });
        if (NZ > INT32_MAX || NP > INT32_MAX || NS > INT32_MAX) {
            delete bt;
            return fail(PNT_ERR_UNSUPPORTED, "batch exceeds int32 indexing");
        }
        std::vector<int32_t> zfirst(NZ), znump(NZ), mapsp1(NS), poffv(NP + 1), pcorner(NS);
        std::vector<double> smf(NS), px(2 * NP), pu(2 * NP, 0.), zr(NZ), ze(NZ), zwrate(NZ), zm(NZ), zetot(NZ),
            zvol(NZ);
        std::vector<uint16_t> bcmask(NP, 0);
        std::vector<HydroConst> consts(n);
        std::vector<Ctl> ctls(n);
        for (int i = 0; i < n; ++i) {
            const Mesh& m = meshes[i]->m;
            const int64_t zo = bt->zoff[i], po = bt->poff[i], so = bt->soff[i];
            for (int64_t z = 0; z < m.numz; ++z) {
                zfirst[zo + z] = (int32_t)(so + m.zfirst[z]);
                znump[zo + z] = m.znump[z];
                zvol[zo + z] = m.zvol[z];
            }
            for (int64_t s = 0; s < m.nums; ++s) {
                mapsp1[so + s] = (int32_t)(po + m.mapsp1[s]);
                smf[so + s] = m.smf[s];
                pcorner[so + s] = (int32_t)(so + m.pcorner[s]);
            }
            for (int64_t q = 0; q < m.nump; ++q) poffv[po + q] = (int32_t)(so + m.poff[q]);
            std::copy(m.px.begin(), m.px.end(), px.begin() + 2 * po);
            init_instance(m, params[i], consts[i], ctls[i], zr.data() + zo, ze.data() + zo, zwrate.data() + zo,
                          zm.data() + zo, zetot.data() + zo, pu.data() + 2 * po, bcmask.data() + po);
        }
        poffv[NP] = (int32_t)NS;

        DevArrays& a = bt->b.a;
        a.nump = (int32_t)NP;
        a.numz = (int32_t)NZ;
        a.nums = (int32_t)NS;
        a.quads = 0;
        int32_t *d_zfirst = nullptr, *d_znump = nullptr, *d_mapsp1 = nullptr, *d_poff = nullptr, *d_pcorner = nullptr;
        double* d_smf = nullptr;
        uint16_t* d_mask = nullptr;
        HydroConst* d_consts = nullptr;
        Ctl* d_ctls = nullptr;
        if ((st = bt->alloc(&d_zfirst, NZ)) || (st = bt->alloc(&d_znump, NZ)) || (st = bt->alloc(&d_mapsp1, NS)) ||
            (st = bt->alloc(&d_smf, NS)) || (st = bt->alloc(&d_poff, NP + 1)) || (st = bt->alloc(&d_pcorner, NS)) ||
            (st = bt->alloc(&d_mask, NP + 2)) || (st = bt->alloc(&a.px[0], NP)) || (st = bt->alloc(&a.px[1], NP)) ||
            (st = bt->alloc(&a.pu[0], NP)) || (st = bt->alloc(&a.pu[1], NP)) || (st = bt->alloc(&a.zm, NZ)) ||
            (st = bt->alloc(&a.zr, NZ)) || (st = bt->alloc(&a.ze, NZ)) || (st = bt->alloc(&a.zetot, NZ)) ||
            (st = bt->alloc(&a.zwrate, NZ)) || (st = bt->alloc(&a.zvol, NZ)) || (st = bt->alloc(&a.zp, NZ)) ||
            (st = bt->alloc(&a.cmass, NS)) || (st = bt->alloc(&a.cforce, NS)) || (st = bt->alloc(&a.sftot, NS)) ||
            (st = bt->alloc(&d_consts, n)) || (st = bt->alloc(&d_ctls, n)) || (st = bt->alloc(&bt->running_dev, 1))) {
            delete bt;
            return st;
        }
        a.zfirst = d_zfirst;
        a.znump = d_znump;
        a.mapsp1 = d_mapsp1;
        a.smf = d_smf;
        a.poff = d_poff;
        a.pcorner = d_pcorner;
        a.bcmask = d_mask;
        a.cmass_f = reinterpret_cast<float*>(a.cmass);
        a.cforce_f = reinterpret_cast<float2*>(a.cforce);
        a.sftot_f = reinterpret_cast<float2*>(a.sftot);
        a.ctl = nullptr;
        bt->b.consts = d_consts;
        bt->b.ctls = d_ctls;
        bt->b.ninst = n;
        cudaError_t e = cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMallocHost((void**)&bt->ctl_host, sizeof(Ctl) * n);
        if (e == cudaSuccess) e = cudaMallocHost((void**)&bt->running_host, sizeof(int));
        auto up = [&](void* dst, const void* src, size_t bytes) { return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice); };
        if (e == cudaSuccess) {
            if ((e = up(d_zfirst, zfirst.data(), NZ * 4)) || (e = up(d_znump, znump.data(), NZ * 4)) ||
                (e = up(d_mapsp1, mapsp1.data(), NS * 4)) || (e = up(d_smf, smf.data(), NS * 8)) ||
                (e = up(d_poff, poffv.data(), (NP + 1) * 4)) || (e = up(d_pcorner, pcorner.data(), NS * 4)) ||
                (e = up(d_mask, bcmask.data(), NP * 2)) || (e = up(a.px[0], px.data(), NP * 16)) ||
                (e = up(a.pu[0], pu.data(), NP * 16)) || (e = up(a.zm, zm.data(), NZ * 8)) ||
                (e = up(a.zr, zr.data(), NZ * 8)) || (e = up(a.ze, ze.data(), NZ * 8)) ||
                (e = up(a.zetot, zetot.data(), NZ * 8)) || (e = up(a.zwrate, zwrate.data(), NZ * 8)) ||
                (e = up(a.zvol, zvol.data(), NZ * 8)) || (e = up(d_consts, consts.data(), sizeof(HydroConst) * n)) ||
                (e = up(d_ctls, ctls.data(), sizeof(Ctl) * n)))
                ;
        }
        if (e == cudaSuccess) e = cudaMemset(a.zp, 0, NZ * 8);
        if (e == cudaSuccess) e = cudaMemset(d_mask + NP, 0, 4);   // pass C copies 32-bit mask words
        if (e == cudaSuccess) {
            // the staged pass C: its shared-memory limit and resident CTAs per SM
            for (auto k : {batch_pass_c<true, false>, batch_pass_c<false, false>, batch_pass_c<true, true>,
                           batch_pass_c<false, true>})
                if (e == cudaSuccess)
                    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, stagedc::kSmemBytes);
            int occ = 0;
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &occ, bt->mixed ? batch_pass_c<false, true> : batch_pass_c<false, false>, stagedc::kTile,
                    stagedc::kSmemBytes);
            if (e == cudaSuccess && occ < 1) e = cudaErrorInvalidConfiguration;
            bt->grid_c = bt->nsm * std::max(occ, 1);
        }
        if (e != cudaSuccess) {
            delete bt;
            return fail(PNT_ERR_CUDA, "batch setup: %s", cudaGetErrorString(e));
        }
        std::memcpy(bt->ctl_host, ctls.data(), sizeof(Ctl) * n);
        if ((st = bt->build_tiles(Shape{256, 3}))) {
            delete bt;
            return st;
        }
    } catch (const std::bad_alloc&) {
        delete bt;
        return fail(PNT_ERR_NOMEM, "out of host memory building the batch");
    }
    *out = bt;
    return PNT_OK;
}

void pnt_batch_destroy(pnt_batch* bt) { delete bt; }

pnt_status pnt_batch_set_shape(pnt_batch* bt, int32_t zones_per_tile, int32_t ctas_per_sm) {
    if (!bt || zones_per_tile < kZonesPerIter || zones_per_tile % kZonesPerIter || ctas_per_sm < 1 || ctas_per_sm > 8)
        return fail(PNT_ERR_INVALID_ARG, "tile must be a positive multiple of %d zones, 1-8 CTAs per SM",
                    kZonesPerIter);
    DeviceGuard dg(bt->device);
    pnt_status st = bt->fetch_ctls();
    if (st) return st;
    return bt->build_tiles(Shape{zones_per_tile, ctas_per_sm});
}

pnt_status pnt_batch_get_shape(pnt_batch* bt, int32_t* zones_per_tile, int32_t* ctas_per_sm) {
    if (!bt || !zones_per_tile || !ctas_per_sm) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *zones_per_tile = bt->shape.zones_per_tile;
    *ctas_per_sm = bt->shape.ctas_per_sm;
    return PNT_OK;
}

pnt_status pnt_batch_enqueue(pnt_batch* bt, int32_t ncycles) {
    if (!bt || ncycles < 0) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(bt->device);
    return bt->enqueue(ncycles);
}

pnt_status pnt_batch_time_cycles(pnt_batch* bt, int32_t ncycles, double* elapsed_ms) {
    if (!bt || !elapsed_ms || ncycles < 0) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(bt->device);
    pnt_status st = bt->ensure_graph();
    if (st) return st;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    cudaEventRecord(e0, bt->stream);
    st = bt->enqueue(ncycles);
    cudaEventRecord(e1, bt->stream);
    const cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (!st && e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "batch timing: %s", cudaGetErrorString(e));
    *elapsed_ms = ms;
    return PNT_OK;
}

pnt_status pnt_batch_tune(pnt_batch* bt, int32_t trial_cycles, int32_t* zones_per_tile, int32_t* ctas_per_sm,
                          double* ms_per_cycle) {
    if (!bt || trial_cycles <= 0) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(bt->device);
    static const int kTiles[] = {64, 128, 256, 512, 1024};
    static const int kCtas[] = {2, 3, 4};
    Shape best{256, 3};
    double best_ms = 1e300;
    if (pnt_status st = bt->fetch_ctls()) return st;
    for (int tz : kTiles) {
        for (int cs : kCtas) {
            pnt_status st = bt->build_tiles(Shape{tz, cs});
            double ms = 0.;
            if (!st) st = pnt_batch_time_cycles(bt, 1, &ms);   // graph build + warm-up
            if (!st) st = pnt_batch_time_cycles(bt, trial_cycles, &ms);
            if (st) return st;
            if (ms < best_ms) {
                best_ms = ms;
                best = Shape{tz, cs};
            }
        }
    }
    pnt_status st = bt->fetch_ctls();
    if (!st) st = bt->build_tiles(best);
    if (st) return st;
    if (zones_per_tile) *zones_per_tile = best.zones_per_tile;
    if (ctas_per_sm) *ctas_per_sm = best.ctas_per_sm;
    if (ms_per_cycle) *ms_per_cycle = best_ms / trial_cycles;
    return PNT_OK;
}

pnt_status pnt_batch_run(pnt_batch* bt, int32_t max_cycles, int32_t* running_left) {
    if (!bt) return fail(PNT_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(bt->device);
    int64_t done_cycles = 0;
    int running = 0;
    pnt_status st = bt->running(&running);
    while (!st && running > 0 && (max_cycles <= 0 || done_cycles < max_cycles)) {
        // drop finished instances from the work lists once they hold a
        // quarter of the listed zones
        if (running < bt->live && (st = bt->fetch_ctls()) == PNT_OK && bt->finished_share() >= 0.25)
            st = bt->build_tiles(bt->shape);
        if (st) break;
        const int chunk = max_cycles > 0 ? (int)std::min<int64_t>(64, max_cycles - done_cycles) : 64;
        if ((st = bt->enqueue(chunk))) break;
        done_cycles += chunk;
        st = bt->running(&running);
    }
    if (st) return st;
    if (running_left) *running_left = running;
    return PNT_OK;
}

pnt_status pnt_batch_scalars(pnt_batch* bt, int32_t i, pnt_scalars* out) {
    if (!bt || !out || i < 0 || i >= bt->ninst) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(bt->device);
    pnt_status st = bt->fetch_ctls();
    if (st) return st;
    const Ctl& c = bt->ctl_host[i];
    out->cycle = c.cycle;
    out->done = c.done;
    out->status = c.status;
    out->nbad = c.nbad;
    out->time = c.time;
    out->dt = c.dtlast;
    out->dtrec = c.dtrec;
    out->dtnew = c.dtnew;
    out->dvovmax = c.dvovmax;
    return PNT_OK;
}

pnt_status pnt_batch_download(pnt_batch* bt, int32_t i, int32_t field, void* dst, size_t bytes) {
    if (!bt || !dst || i < 0 || i >= bt->ninst) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(bt->device);
    pnt_status st = bt->fetch_ctls();
    if (st) return st;
    const int cur = bt->ctl_host[i].cycle & 1;
    const DevArrays& a = bt->b.a;
    const void* src = nullptr;
    size_t n = 0;
    switch (field) {
        case PNT_FIELD_PX: src = a.px[cur] + bt->poff[i]; n = (size_t)bt->np[i] * 16; break;
        case PNT_FIELD_PU: src = a.pu[cur] + bt->poff[i]; n = (size_t)bt->np[i] * 16; break;
        case PNT_FIELD_ZR: src = a.zr + bt->zoff[i]; n = (size_t)bt->nz[i] * 8; break;
        case PNT_FIELD_ZE: src = a.ze + bt->zoff[i]; n = (size_t)bt->nz[i] * 8; break;
        case PNT_FIELD_ZP: src = a.zp + bt->zoff[i]; n = (size_t)bt->nz[i] * 8; break;
        case PNT_FIELD_ZM: src = a.zm + bt->zoff[i]; n = (size_t)bt->nz[i] * 8; break;
        case PNT_FIELD_ZETOT: src = a.zetot + bt->zoff[i]; n = (size_t)bt->nz[i] * 8; break;
        case PNT_FIELD_ZVOL: src = a.zvol + bt->zoff[i]; n = (size_t)bt->nz[i] * 8; break;
        case PNT_FIELD_ZWRATE: src = a.zwrate + bt->zoff[i]; n = (size_t)bt->nz[i] * 8; break;
        default: return fail(PNT_ERR_INVALID_ARG, "unknown field %d", field);
    }
    if (bytes != n) return fail(PNT_ERR_INVALID_ARG, "field %d of instance %d has %zu bytes, got %zu", field, i, n, bytes);
    CUDA_TRY(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, bt->stream));
    CUDA_TRY(cudaStreamSynchronize(bt->stream));
    return PNT_OK;
}

}  // extern "C"
