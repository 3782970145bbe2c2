// hydro.cu -- the pnt_hydro object: device state of one mesh on one GPU,
// Hydro::init, the cycle driver with CUDA-graph replay, field transfer and
// the output writers.  C ABI in include/pennant_b200.h.
#include "closure_dev.cuh"
#include "hydro_dev.h"
#include "pnt_internal.h"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <vector>

using namespace pnt;

namespace {

#define CUDA_TRY(expr)                                                                  \
    do {                                                                                \
        const cudaError_t e_ = (expr);                                                  \
        if (e_ != cudaSuccess)                                                          \
            return fail(PNT_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_),  \
                        __FILE__, __LINE__);                                            \
    } while (0)

// Makes `dev` current for the scope and restores the caller's device.
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

}  // namespace

struct pnt_hydro {
    int device = 0;
    cudaStream_t stream = nullptr;
    pnt_params params{};
    HydroConst hc{};
    DevArrays a{};
    Ctl* ctl_host = nullptr;   // pinned mirror of the device Ctl
    std::vector<void*> allocs;
    // host copies needed by the output writers
    std::vector<int32_t> znump, mapsp1;
    int32_t nump = 0, numz = 0, nums = 0;
    // captured CUDA graphs of graph_cycles cycles and of one cycle (the
    // single steps of pnt_hydro_cycle)
    cudaGraphExec_t graph = nullptr;
    cudaGraphExec_t graph1 = nullptr;
    int graph_cycles = 0;
    // the cycle of the selected precision
    cudaError_t (*launch)(const DevArrays&, const HydroConst&, cudaStream_t, cudaEvent_t*, int) = launch_cycle_fp64;
    // learned closure: this object's copy of the parameter image (set by
    // pnt_hydro_set_closure) and the corner class counters
    bool learned = false;
    // multi-piece runs (a hydro object over a piece mesh): the send lists,
    // the send buffer (corner masses, then corner forces at send_foff) and
    // the per-corner byte sizes of the cycle's precision
    unsigned long long* scan = nullptr;   // pnt_hydro_check_finite's results
    bool piece = false;
    int32_t nsend = 0, nhalo = 0;
    int32_t* send_side = nullptr;
    unsigned char* send = nullptr;
    size_t send_foff = 0;
    int32_t cmass_bytes = 8, cforce_bytes = 16;

    ~pnt_hydro() {
        DeviceGuard dg(device);
        if (graph) cudaGraphExecDestroy(graph);
        if (graph1) cudaGraphExecDestroy(graph1);
        for (void* p : allocs) cudaFree(p);
        if (ctl_host) cudaFreeHost(ctl_host);
        if (stream) cudaStreamDestroy(stream);
    }

    template <typename T>
    pnt_status alloc(T** out, size_t count) {
        void* p = nullptr;
        const cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(e == cudaErrorMemoryAllocation ? PNT_ERR_NOMEM : PNT_ERR_CUDA,
                        "cudaMalloc of %zu bytes: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        allocs.push_back(p);
        *out = static_cast<T*>(p);
        return PNT_OK;
    }

    pnt_status check_closure() const {
        if (learned && !a.closure_img)
            return fail(PNT_ERR_STATE, "precision learned needs a closure (pnt_hydro_set_closure)");
        return PNT_OK;
    }
    // whole cycles (a piece steps with pnt_hydro_piece_*)
    pnt_status check_ready() const {
        if (piece) return fail(PNT_ERR_STATE, "a piece object steps with pnt_hydro_piece_forces/advance/finish");
        return check_closure();
    }

    pnt_status launch_cycles(int n) {
        if (pnt_status st = check_ready()) return st;
        for (int i = 0; i < n; ++i) {
            const cudaError_t e = launch(a, hc, stream, nullptr, kPhaseAll);
            if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "cycle launch: %s", cudaGetErrorString(e));
        }
        return PNT_OK;
    }

    // One cycle as a graph: one launch per step instead of one per kernel.
    pnt_status ensure_graph1() {
        if (graph1) return PNT_OK;
        if (pnt_status st = check_ready()) return st;
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t e = launch(a, hc, stream, nullptr, kPhaseAll);
        const cudaError_t e2 = cudaStreamEndCapture(stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return fail(PNT_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        const cudaError_t e3 = cudaGraphInstantiate(&graph1, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) {
            graph1 = nullptr;
            return fail(PNT_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e3));
        }
        return PNT_OK;
    }

    pnt_status ensure_graph() {
        if (graph) return PNT_OK;
        if (pnt_status st = check_ready()) return st;
        graph_cycles = params.graph_cycles > 0 ? params.graph_cycles : 16;
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < graph_cycles; ++i) {
            const cudaError_t e = launch(a, hc, stream, nullptr, kPhaseAll);
            if (e != cudaSuccess) {
                cudaStreamEndCapture(stream, &g);
                if (g) cudaGraphDestroy(g);
                return fail(PNT_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
            }
        }
        CUDA_TRY(cudaStreamEndCapture(stream, &g));
        const cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            graph = nullptr;
            return fail(PNT_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
        }
        return PNT_OK;
    }

    // Enqueue n cycles: whole graphs, then single-cycle launches.
    pnt_status enqueue(int n) {
        pnt_status st = ensure_graph();
        if (st) return st;
        while (n >= graph_cycles) {
            CUDA_TRY(cudaGraphLaunch(graph, stream));
            n -= graph_cycles;
        }
        return launch_cycles(n);
    }

    pnt_status fetch_ctl() {
        CUDA_TRY(cudaMemcpyAsync(ctl_host, a.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return PNT_OK;
    }

    void scalars(pnt_scalars* out) const {
        if (!out) return;
        out->cycle = ctl_host->cycle;
        out->done = ctl_host->done;
        out->status = ctl_host->status;
        out->nbad = ctl_host->nbad;
        out->time = ctl_host->time;
        out->dt = ctl_host->dtlast;
        out->dtrec = ctl_host->dtrec;
        out->dtnew = ctl_host->dtnew;
        out->dvovmax = ctl_host->dvovmax;
    }

    pnt_status set_stop_at(int32_t stop_at) {
        CUDA_TRY(cudaMemcpyAsync(&a.ctl->stop_at, &stop_at, sizeof(int32_t), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        ctl_host->stop_at = stop_at;
        return PNT_OK;
    }
};

namespace {

struct FieldInfo {
    void* dev;
    size_t bytes;
};

FieldInfo field_info(pnt_hydro* h, int32_t field, int cur) {
    const size_t np = (size_t)h->nump, nz = (size_t)h->numz, ns = (size_t)h->nums;
    switch (field) {
        case PNT_FIELD_PX: return {h->a.px[cur], np * sizeof(double2)};
        case PNT_FIELD_PU: return {h->a.pu[cur], np * sizeof(double2)};
        case PNT_FIELD_ZR: return {h->a.zr, nz * sizeof(double)};
        case PNT_FIELD_ZE: return {h->a.ze, nz * sizeof(double)};
        case PNT_FIELD_ZP: return {h->a.zp, nz * sizeof(double)};
        case PNT_FIELD_ZM: return {h->a.zm, nz * sizeof(double)};
        case PNT_FIELD_ZETOT: return {h->a.zetot, nz * sizeof(double)};
        case PNT_FIELD_ZVOL: return {h->a.zvol, nz * sizeof(double)};
        case PNT_FIELD_ZWRATE: return {h->a.zwrate, nz * sizeof(double)};
        case PNT_FIELD_SMF: return {const_cast<double*>(h->a.smf), ns * sizeof(double)};
        default: return {nullptr, 0};
    }
}

// Hydro::init (Hydro.cc:241-339) and the constants of the cycle.
pnt_status init_hydro(pnt_hydro* h, const Mesh& m, const pnt_params& p) {
    const int64_t np = m.nump, nz = m.numz, ns = m.nums;
    HydroConst& c = h->hc;
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
    if (c.nbc > kMaxBC) return fail(PNT_ERR_UNSUPPORTED, "more than %d boundary planes", kMaxBC);

    // Boundary planes in deck order, bcx then bcy (Hydro.cc:220-225); a
    // point belongs to a plane when its coordinate is within 1e-12 of it
    // (HydroBC.cc:63-144, 222-326).
    std::vector<uint16_t> bcmask(np, 0);
    const double eps = 1.e-12;
    for (int b = 0; b < c.nbc; ++b) {
        const bool xplane = b < p.nbcx;
        const double bound = xplane ? p.bcx[b] : p.bcy[b - p.nbcx];
        c.vfix[b][0] = xplane ? 1. : 0.;
        c.vfix[b][1] = xplane ? 0. : 1.;
        for (int64_t q = 0; q < np; ++q) {
            const double coord = xplane ? m.px[2 * q] : m.px[2 * q + 1];
            if (fabs(coord - bound) < eps) bcmask[q] |= (uint16_t)(1u << b);
        }
    }

    std::vector<double> zr(nz, p.rinit), ze(nz, p.einit), zwrate(nz, 0.), zm(nz), zetot(nz);
    if (p.has_subregion) {   // initSubrgnTask (Hydro.cc:1738-1762)
        const double* sr = p.subregion;
        for (int64_t z = 0; z < nz; ++z) {
            const double zxx = m.zx[2 * z], zxy = m.zx[2 * z + 1];
            if (zxx > (sr[0] - eps) && zxx < (sr[1] + eps) && zxy > (sr[2] - eps) && zxy < (sr[3] + eps)) {
                zr[z] = p.rinitsub;
                ze[z] = p.einitsub;
            }
        }
    }
    for (int64_t z = 0; z < nz; ++z) {   // initHydroTask (Hydro.cc:1765-1784)
        zm[z] = zr[z] * m.zvol[z];
        zetot[z] = ze[z] * zm[z];
    }
    std::vector<double> pu(2 * np, 0.);
    if (p.uinitradial != 0.) {   // initRadialVelTask (Hydro.cc:1787-1807)
        for (int64_t q = 0; q < np; ++q) {
            const double x = m.px[2 * q], y = m.px[2 * q + 1];
            const double pmag = sqrt(x * x + y * y);
            if (pmag > eps) {
                const double rinv = 1. / pmag;
                pu[2 * q] = (x * p.uinitradial) * rinv;
                pu[2 * q + 1] = (y * p.uinitradial) * rinv;
            }
        }
    }

    DevArrays& a = h->a;
    a.nump = (int32_t)np;
    a.numz = (int32_t)nz;
    a.nums = (int32_t)ns;
    a.quads = m.all_quads ? 1 : 0;
    a.rect_nzx = m.rect_nzx;
    int32_t *zfirst = nullptr, *znump = nullptr, *mapsp1 = nullptr, *poff = nullptr, *pcorner = nullptr;
    double* smf = nullptr;
    uint16_t* mask = nullptr;
    // the persistent pass C's grid
    {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
        cudaError_t e = prepare_pass_c(p.precision != PNT_PREC_FP64, a.quads != 0, a.rect_nzx, a.numz, nsm, &a.gridC);
        if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "pass C setup: %s", cudaGetErrorString(e));
        if (a.rect_nzx > 0 && p.precision != PNT_PREC_FP64) {
            e = prepare_pass_a_rows_mixed(p.precision == PNT_PREC_LEARNED, a.rect_nzx, a.numz, nsm, &a.gridA);
            if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "pass A setup: %s", cudaGetErrorString(e));
        }
    }
    pnt_status st = PNT_OK;
    if ((st = h->alloc(&zfirst, nz)) || (st = h->alloc(&znump, nz)) || (st = h->alloc(&mapsp1, ns)) ||
        (st = h->alloc(&smf, ns)) || (st = h->alloc(&poff, np + 1)) || (st = h->alloc(&pcorner, m.pcorner.size())) ||
        (st = h->alloc(&mask, np + 2)) || (st = h->alloc(&a.px[0], np)) || (st = h->alloc(&a.px[1], np)) ||
        (st = h->alloc(&a.pu[0], np)) || (st = h->alloc(&a.pu[1], np)) || (st = h->alloc(&a.zm, nz + 2)) ||
        (st = h->alloc(&a.zr, nz + 2)) || (st = h->alloc(&a.ze, nz + 2)) || (st = h->alloc(&a.zetot, nz + 2)) ||
        (st = h->alloc(&a.zwrate, nz + 2)) || (st = h->alloc(&a.zvol, nz + 2)) || (st = h->alloc(&a.zp, nz + 2)) ||
        (st = h->alloc(&a.cmass, ns + m.nhalo)) || (st = h->alloc(&a.cforce, ns + m.nhalo)) || (st = h->alloc(&a.sftot, ns)) ||
        (st = h->alloc(&a.cyc_red, 5)) || (st = h->alloc(&a.fin_ticket, 1)) || (st = h->alloc(&a.ctl, 1)))
        return st;
    a.cmass_f = reinterpret_cast<float*>(a.cmass);
    a.cforce_f = reinterpret_cast<float2*>(a.cforce);
    a.sftot_f = reinterpret_cast<float2*>(a.sftot);
    a.zfirst = zfirst;
    a.znump = znump;
    a.mapsp1 = mapsp1;
    a.smf = smf;
    a.poff = poff;
    a.pcorner = pcorner;
    a.bcmask = mask;
    if (m.is_piece) {
        // a piece: halo corner slots follow the local sides in cmass/cforce
        h->piece = true;
        h->nhalo = m.nhalo;
        h->nsend = (int32_t)m.send_side.size();
        const bool fp64 = p.precision == PNT_PREC_FP64;
        h->cmass_bytes = fp64 ? 8 : 4;
        h->cforce_bytes = fp64 ? 16 : 8;
        h->send_foff = ((size_t)h->nsend * h->cmass_bytes + 15) / 16 * 16;
        if ((st = h->alloc(&h->send_side, (size_t)h->nsend)) ||
            (st = h->alloc(&h->send, h->send_foff + (size_t)h->nsend * h->cforce_bytes)) ||
            (st = h->alloc(&a.piece_red, 4)))
            return st;
        if (h->nsend > 0)
            CUDA_TRY(cudaMemcpy(h->send_side, m.send_side.data(), (size_t)h->nsend * 4, cudaMemcpyHostToDevice));
    }

    // Driver::run start: time 0, cycle 0 and calcGlobalDt for cycle 0
    // (Driver.cc:213-245).
    Ctl ctl{};
    double dt = p.dtmax;
    if (p.dtinit < dt) dt = p.dtinit;
    if ((p.tstop - 0.) < dt) dt = p.tstop - 0.;
    ctl.dt = dt;
    ctl.dtinv = 1. / dt;
    ctl.cycle = 0;
    ctl.time = 0.;
    ctl.done = (p.cstop <= 0 || !(0. < p.tstop)) ? 1 : 0;
    ctl.stop_at = INT_MAX;

    // the cycle reductions' starting values: minimum from 1e99, maximum
    // from 1e-99 (keys of positive doubles are their bits), no bad sides
    long long cyc_red_init[5] = {0, 0, 0, 0, 0};
    {
        const double lo = 1.e99, hi = 1.e-99;
        std::memcpy(&cyc_red_init[0], &lo, 8);
        std::memcpy(&cyc_red_init[1], &hi, 8);
    }
    cudaStream_t s = h->stream;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    };
    cudaError_t e = cudaSuccess;
    if ((e = up(zfirst, m.zfirst.data(), nz * 4)) || (e = up(znump, m.znump.data(), nz * 4)) ||
        (e = up(mapsp1, m.mapsp1.data(), ns * 4)) || (e = up(smf, m.smf.data(), ns * 8)) ||
        (e = up(poff, m.poff.data(), (np + 1) * 4)) || (e = up(pcorner, m.pcorner.data(), m.pcorner.size() * 4)) ||
        (e = up(mask, bcmask.data(), np * 2)) || (e = up(a.px[0], m.px.data(), np * 16)) ||
        (e = up(a.pu[0], pu.data(), np * 16)) || (e = up(a.zm, zm.data(), nz * 8)) ||
        (e = up(a.zr, zr.data(), nz * 8)) || (e = up(a.ze, ze.data(), nz * 8)) ||
        (e = up(a.zetot, zetot.data(), nz * 8)) || (e = up(a.zwrate, zwrate.data(), nz * 8)) ||
        (e = up(a.zvol, m.zvol.data(), nz * 8)) || (e = up(a.ctl, &ctl, sizeof(Ctl))) ||
        (e = up(a.cyc_red, cyc_red_init, sizeof(cyc_red_init))))
        return fail(PNT_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
    if ((e = cudaMemsetAsync(a.zp, 0, nz * 8, s)) || (e = cudaMemsetAsync(a.fin_ticket, 0, 4, s)) ||
        (e = cudaMemsetAsync(mask + np, 0, 4, s)) ||   // pad: pass C copies whole 32-bit mask words
        (e = cudaMemsetAsync(a.px[1], 0, np * 16, s)) ||
        (e = cudaMemsetAsync(a.pu[1], 0, np * 16, s)))
        return fail(PNT_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
    CUDA_TRY(cudaStreamSynchronize(s));
    *h->ctl_host = ctl;
    return PNT_OK;
}

pnt_status write_xy(const char* path, const std::vector<double>& zr, const std::vector<double>& ze,
                    const std::vector<double>& zp) {
    FILE* f = fopen(path, "w");
    if (!f) return fail(PNT_ERR_INVALID_ARG, "cannot open %s", path);
    const std::vector<double>* v[3] = {&zr, &ze, &zp};
    const char* nm[3] = {"zr", "ze", "zp"};
    for (int k = 0; k < 3; ++k) {
        fprintf(f, "#  %s\n", nm[k]);
        for (size_t z = 0; z < v[k]->size(); ++z) fprintf(f, "%5d%18.8e\n", (int)z + 1, (*v[k])[z]);
    }
    fclose(f);
    return PNT_OK;
}

}  // namespace

extern "C" {

pnt_status pnt_hydro_create(const pnt_mesh* mesh, const pnt_params* params, int32_t device, pnt_hydro** out) {
    if (!mesh || !params || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (params->precision != PNT_PREC_FP64 && params->precision != PNT_PREC_MIXED &&
        params->precision != PNT_PREC_LEARNED)
        return fail(PNT_ERR_INVALID_ARG, "unknown precision %d", params->precision);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(PNT_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(PNT_ERR_INVALID_ARG, "device %d out of range", device);
    DeviceGuard dg(device);
    pnt_hydro* h = new (std::nothrow) pnt_hydro();
    if (!h) return fail(PNT_ERR_NOMEM, "out of memory");
    h->device = device;
    h->params = *params;
    h->launch = (params->precision == PNT_PREC_MIXED)     ? launch_cycle_mixed
                : (params->precision == PNT_PREC_LEARNED) ? launch_cycle_learned
                                                          : launch_cycle_fp64;
    h->learned = params->precision == PNT_PREC_LEARNED;
    pnt_status st = PNT_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&h->ctl_host, sizeof(Ctl));
    if (e != cudaSuccess) {
        delete h;
        return fail(PNT_ERR_CUDA, "stream/host alloc: %s", cudaGetErrorString(e));
    }
    const Mesh& m = mesh->m;
    h->nump = m.nump;
    h->numz = m.numz;
    h->nums = m.nums;
    try {
        h->znump = m.znump;
        h->mapsp1 = m.mapsp1;
        st = init_hydro(h, m, *params);
        if (!st && h->learned) {
            unsigned long long* counts = nullptr;
            st = h->alloc(&counts, kClassCount * 64);
            if (!st && cudaMemset(counts, 0, kClassCount * 64 * sizeof(unsigned long long)) != cudaSuccess)
                st = fail(PNT_ERR_CUDA, "counter memset failed");
            h->a.closure_counts = counts;
        }
    } catch (const std::bad_alloc&) {
        st = fail(PNT_ERR_NOMEM, "out of host memory");
    }
    if (st) {
        delete h;
        return st;
    }
    *out = h;
    return PNT_OK;
}

void pnt_hydro_destroy(pnt_hydro* h) { delete h; }

namespace {
// The status of a run the device ended: inverted sides, or a bounded wait
// of a kernel that ran out.
pnt_status run_failure(const Ctl& c) {
    if (c.status == PNT_ERR_TIMEOUT)
        return fail(PNT_ERR_TIMEOUT, "a bounded device-side wait ran out on cycle %d", c.cycle);
    return fail(c.status, "%d negative side volumes on cycle %d", c.nbad, c.cycle);
}
}  // namespace

pnt_status pnt_hydro_cycle(pnt_hydro* h, pnt_scalars* out) {
    if (!h) return fail(PNT_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(h->device);
    pnt_status st = h->ensure_graph1();
    if (st) return st;
    CUDA_TRY(cudaGraphLaunch(h->graph1, h->stream));
    st = h->fetch_ctl();
    if (st) return st;
    h->scalars(out);
    if (h->ctl_host->status) return run_failure(*h->ctl_host);
    return PNT_OK;
}

pnt_status pnt_hydro_run(pnt_hydro* h, int32_t max_cycles, pnt_report_fn report, void* user, pnt_scalars* out) {
    if (!h) return fail(PNT_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(h->device);
    pnt_status st = h->fetch_ctl();
    if (st) return st;
    const int32_t start = h->ctl_host->cycle;
    const int32_t stop_at =
        (max_cycles > 0 && (int64_t)start + max_cycles < INT_MAX) ? start + max_cycles : INT_MAX;
    if ((st = h->set_stop_at(stop_at))) return st;
    if ((st = h->ensure_graph())) return st;
    const int dtreport = h->params.dtreport > 0 ? h->params.dtreport : 10;
    auto t_prev = std::chrono::steady_clock::now();
    while (!h->ctl_host->done && h->ctl_host->cycle < stop_at) {
        const int32_t cyc = h->ctl_host->cycle;
        int64_t target;
        if (report) target = (cyc < 1) ? 1 : ((int64_t)cyc / dtreport + 1) * dtreport;
        else target = (int64_t)cyc + 64LL * h->graph_cycles;   // poll the done flag now and then
        target = std::min<int64_t>(target, stop_at);
        if ((st = h->enqueue((int)(target - cyc)))) break;
        if ((st = h->fetch_ctl())) break;
        if (report && !h->ctl_host->status && h->ctl_host->cycle == target &&
            (target == 1 || target % dtreport == 0)) {
            const auto t_now = std::chrono::steady_clock::now();
            const double us = std::chrono::duration<double, std::micro>(t_now - t_prev).count();
            t_prev = t_now;
            pnt_scalars sc;
            h->scalars(&sc);
            report(&sc, us, user);
        }
    }
    if (!st) st = h->set_stop_at(INT_MAX);
    if (st) return st;
    h->scalars(out);
    if (h->ctl_host->status) return run_failure(*h->ctl_host);
    return PNT_OK;
}

pnt_status pnt_hydro_enqueue(pnt_hydro* h, int32_t ncycles) {
    if (!h || ncycles < 0) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(h->device);
    return h->enqueue(ncycles);
}

pnt_status pnt_hydro_time_kernels(pnt_hydro* h, int32_t ncycles, double* kernel_ms, int32_t nkernels) {
    if (!h || !kernel_ms || ncycles <= 0 || nkernels <= 0) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(h->device);
    if (pnt_status st0 = h->check_ready()) return st0;
    std::vector<cudaEvent_t> ev((size_t)ncycles * kNumEvents, nullptr);
    pnt_status st = PNT_OK;
    for (auto& e : ev) {
        if (cudaEventCreate(&e) != cudaSuccess) { st = fail(PNT_ERR_CUDA, "cudaEventCreate failed"); break; }
    }
    for (int32_t i = 0; i < ncycles && !st; ++i) {
        const cudaError_t e = h->launch(h->a, h->hc, h->stream, &ev[(size_t)i * kNumEvents], kPhaseAll);
        if (e != cudaSuccess) st = fail(PNT_ERR_CUDA, "cycle launch: %s", cudaGetErrorString(e));
    }
    if (!st && cudaStreamSynchronize(h->stream) != cudaSuccess) st = fail(PNT_ERR_CUDA, "synchronize failed");
    if (!st) {
        for (int k = 0; k < nkernels; ++k) kernel_ms[k] = 0.;
        // kernel k runs between events from[k] and from[k] + 1
        static const int from[kNumKernels] = {0, 2, 3, 4, 1};
        for (int32_t i = 0; i < ncycles; ++i) {
            for (int k = 0; k < kNumKernels && k < nkernels; ++k) {
                float ms = 0.f;
                const cudaEvent_t* e = &ev[(size_t)i * kNumEvents];
                cudaEventElapsedTime(&ms, e[from[k]], e[from[k] + 1]);
                kernel_ms[k] += ms / ncycles;
            }
        }
    }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (!st) st = h->fetch_ctl();
    return st;
}

pnt_status pnt_hydro_time_cycles(pnt_hydro* h, int32_t ncycles, double* elapsed_ms) {
    if (!h || !elapsed_ms || ncycles < 0) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    DeviceGuard dg(h->device);
    pnt_status st = h->ensure_graph();
    if (st) return st;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return fail(PNT_ERR_CUDA, "cudaEventCreate failed");
    }
    cudaError_t e = cudaEventRecord(e0, h->stream);
    if (e == cudaSuccess) st = h->enqueue(ncycles);
    if (e == cudaSuccess && !st) e = cudaEventRecord(e1, h->stream);
    if (e == cudaSuccess && !st) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess && !st) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    if (e != cudaSuccess) return fail(PNT_ERR_CUDA, "cycle timing: %s", cudaGetErrorString(e));
    *elapsed_ms = ms;
    return h->fetch_ctl();
}

pnt_status pnt_hydro_synchronize(pnt_hydro* h) {
    if (!h) return fail(PNT_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(h->device);
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PNT_OK;
}

pnt_status pnt_hydro_get_scalars(pnt_hydro* h, pnt_scalars* out) {
    if (!h || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(h->device);
    const pnt_status st = h->fetch_ctl();
    if (st) return st;
    h->scalars(out);
    return PNT_OK;
}

pnt_status pnt_hydro_download(pnt_hydro* h, int32_t field, void* dst, size_t bytes) {
    if (!h || !dst) return fail(PNT_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(h->device);
    pnt_status st = h->fetch_ctl();
    if (st) return st;
    const FieldInfo fi = field_info(h, field, h->ctl_host->cycle & 1);
    if (!fi.dev) return fail(PNT_ERR_INVALID_ARG, "unknown field %d", field);
    if (bytes != fi.bytes) return fail(PNT_ERR_INVALID_ARG, "field %d has %zu bytes, got %zu", field, fi.bytes, bytes);
    CUDA_TRY(cudaMemcpyAsync(dst, fi.dev, bytes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PNT_OK;
}

pnt_status pnt_hydro_upload(pnt_hydro* h, int32_t field, const void* src, size_t bytes) {
    if (!h || !src) return fail(PNT_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(h->device);
    pnt_status st = h->fetch_ctl();
    if (st) return st;
    const FieldInfo fi = field_info(h, field, h->ctl_host->cycle & 1);
    if (!fi.dev || field == PNT_FIELD_SMF) return fail(PNT_ERR_INVALID_ARG, "field %d is not writable", field);
    if (bytes != fi.bytes) return fail(PNT_ERR_INVALID_ARG, "field %d has %zu bytes, got %zu", field, fi.bytes, bytes);
    CUDA_TRY(cudaMemcpyAsync(fi.dev, src, bytes, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PNT_OK;
}

pnt_status pnt_hydro_device_ptr(pnt_hydro* h, int32_t field, void** dptr) {
    if (!h || !dptr) return fail(PNT_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(h->device);
    pnt_status st = h->fetch_ctl();
    if (st) return st;
    const FieldInfo fi = field_info(h, field, h->ctl_host->cycle & 1);
    if (!fi.dev) return fail(PNT_ERR_INVALID_ARG, "unknown field %d", field);
    *dptr = fi.dev;
    return PNT_OK;
}

pnt_status pnt_hydro_piece_buffers(pnt_hydro* h, pnt_piece_buffers* out) {
    if (!h || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    if (!h->piece) return fail(PNT_ERR_STATE, "not a piece object");
    out->send = h->send;
    out->send_cforce_offset = h->send_foff;
    out->halo_cmass = reinterpret_cast<unsigned char*>(h->a.cmass) + (size_t)h->nums * h->cmass_bytes;
    out->halo_cforce = reinterpret_cast<unsigned char*>(h->a.cforce) + (size_t)h->nums * h->cforce_bytes;
    out->cmass_bytes = h->cmass_bytes;
    out->cforce_bytes = h->cforce_bytes;
    out->red = h->a.piece_red;
    out->stream = (void*)h->stream;
    return PNT_OK;
}

pnt_status pnt_hydro_piece_forces(pnt_hydro* h) {
    if (!h) return fail(PNT_ERR_INVALID_ARG, "null argument");
    if (!h->piece) return fail(PNT_ERR_STATE, "not a piece object");
    if (pnt_status st = h->check_closure()) return st;
    DeviceGuard dg(h->device);
    CUDA_TRY(h->launch(h->a, h->hc, h->stream, nullptr, kPhaseForces));
    launch_piece_pack(h->a, h->send_side, h->nsend, h->send, h->send_foff, h->params.precision != PNT_PREC_FP64,
                      h->stream);
    CUDA_TRY(cudaGetLastError());
    return PNT_OK;
}

pnt_status pnt_hydro_piece_advance(pnt_hydro* h) {
    if (!h) return fail(PNT_ERR_INVALID_ARG, "null argument");
    if (!h->piece) return fail(PNT_ERR_STATE, "not a piece object");
    if (pnt_status st = h->check_closure()) return st;
    DeviceGuard dg(h->device);
    CUDA_TRY(h->launch(h->a, h->hc, h->stream, nullptr, kPhaseAdvance));
    return PNT_OK;
}

pnt_status pnt_hydro_piece_finish(pnt_hydro* h) {
    if (!h) return fail(PNT_ERR_INVALID_ARG, "null argument");
    if (!h->piece) return fail(PNT_ERR_STATE, "not a piece object");
    DeviceGuard dg(h->device);
    launch_piece_finish(h->a, h->hc, h->stream);
    CUDA_TRY(cudaGetLastError());
    return PNT_OK;
}

pnt_status pnt_hydro_check_finite(pnt_hydro* h, int32_t* field, int64_t* index) {
    if (!h || !field || !index) return fail(PNT_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(h->device);
    pnt_status st = h->fetch_ctl();
    if (st) return st;
    static const int32_t kFields[] = {PNT_FIELD_PX, PNT_FIELD_PU, PNT_FIELD_ZR, PNT_FIELD_ZE, PNT_FIELD_ZP,
                                      PNT_FIELD_ZM, PNT_FIELD_ZETOT, PNT_FIELD_ZVOL, PNT_FIELD_ZWRATE};
    constexpr int kN = (int)(sizeof(kFields) / sizeof(kFields[0]));
    if (!h->scan && (st = h->alloc(&h->scan, kN))) return st;
    CUDA_TRY(cudaMemsetAsync(h->scan, 0xff, kN * sizeof(unsigned long long), h->stream));
    for (int i = 0; i < kN; ++i) {
        const FieldInfo fi = field_info(h, kFields[i], h->ctl_host->cycle & 1);
        launch_find_nonfinite(static_cast<const double*>(fi.dev), (int64_t)(fi.bytes / 8), h->scan + i, h->stream);
    }
    CUDA_TRY(cudaGetLastError());
    unsigned long long first[kN];
    CUDA_TRY(cudaMemcpyAsync(first, h->scan, sizeof(first), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    *field = -1;
    *index = -1;
    for (int i = 0; i < kN; ++i) {
        if (first[i] != ~0ull) {
            *field = kFields[i];
            const bool point = kFields[i] == PNT_FIELD_PX || kFields[i] == PNT_FIELD_PU;
            *index = (int64_t)(point ? first[i] / 2 : first[i]);
            break;
        }
    }
    return PNT_OK;
}

pnt_status pnt_hydro_stream(pnt_hydro* h, void** stream) {
    if (!h || !stream) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *stream = (void*)h->stream;
    return PNT_OK;
}

pnt_status pnt_hydro_write_xy(pnt_hydro* h, const char* path) {
    if (!h || !path) return fail(PNT_ERR_INVALID_ARG, "null argument");
    std::vector<double> zr(h->numz), ze(h->numz), zp(h->numz);
    pnt_status st;
    if ((st = pnt_hydro_download(h, PNT_FIELD_ZR, zr.data(), zr.size() * 8)) ||
        (st = pnt_hydro_download(h, PNT_FIELD_ZE, ze.data(), ze.size() * 8)) ||
        (st = pnt_hydro_download(h, PNT_FIELD_ZP, zp.data(), zp.size() * 8)))
        return st;
    return write_xy(path, zr, ze, zp);
}

// ExportGold::write (ExportGold.cc:31-307): case file, geometry with the
// zones sorted into triangles / quads / others, and per-zone variables.
pnt_status pnt_hydro_write_gold(pnt_hydro* h, const char* base) {
    if (!h || !base) return fail(PNT_ERR_INVALID_ARG, "null argument");
    const int64_t nz = h->numz, np = h->nump;
    std::vector<double> zr(nz), ze(nz), zp(nz), px(2 * np);
    pnt_status st;
    if ((st = pnt_hydro_download(h, PNT_FIELD_ZR, zr.data(), nz * 8)) ||
        (st = pnt_hydro_download(h, PNT_FIELD_ZE, ze.data(), nz * 8)) ||
        (st = pnt_hydro_download(h, PNT_FIELD_ZP, zp.data(), nz * 8)) ||
        (st = pnt_hydro_download(h, PNT_FIELD_PX, px.data(), np * 16)))
        return st;
    std::vector<int64_t> mapzs(nz);
    std::vector<int64_t> tris, quads, others;
    int64_t sc = 0;
    for (int64_t z = 0; z < nz; ++z) {
        const int n = h->znump[z];
        (n == 3 ? tris : n == 4 ? quads : others).push_back(z);
        mapzs[z] = sc;
        sc += n;
    }
    const std::string b(base);
    FILE* f = fopen((b + ".case").c_str(), "w");
    if (!f) return fail(PNT_ERR_INVALID_ARG, "cannot open %s.case", base);
    fprintf(f,
            "#\n# Created by PENNANT\n#\nFORMAT\ntype: ensight gold\nGEOMETRY\nmodel: %s.geo\n"
            "VARIABLE\nscalar per element: zr %s.zr\nscalar per element: ze %s.ze\n"
            "scalar per element: zp %s.zp\n",
            base, base, base, base);
    fclose(f);
    f = fopen((b + ".geo").c_str(), "w");
    if (!f) return fail(PNT_ERR_INVALID_ARG, "cannot open %s.geo", base);
    fprintf(f, "cycle = %8d\nt = %15.8e\nnode id assign\nelement id given\npart\n%10d\nuniverse\n"
               "coordinates\n%10lld\n",
            h->ctl_host->cycle, h->ctl_host->time, 1, (long long)np);
    for (int64_t q = 0; q < np; ++q) fprintf(f, "%12.5e\n", px[2 * q]);
    for (int64_t q = 0; q < np; ++q) fprintf(f, "%12.5e\n", px[2 * q + 1]);
    for (int64_t q = 0; q < np; ++q) fprintf(f, "%12.5e\n", 0.);
    const std::vector<int64_t>* groups[2] = {&tris, &quads};
    const char* tags[2] = {"tria3", "quad4"};
    for (int k = 0; k < 2; ++k) {
        const auto& gz = *groups[k];
        if (gz.empty()) continue;
        fprintf(f, "%s\n%10lld\n", tags[k], (long long)gz.size());
        for (int64_t z : gz) fprintf(f, "%10lld\n", (long long)z + 1);
        for (int64_t z : gz) {
            for (int i = 0; i < h->znump[z]; ++i) fprintf(f, "%10d", h->mapsp1[mapzs[z] + i] + 1);
            fprintf(f, "\n");
        }
    }
    if (!others.empty()) {
        fprintf(f, "nsided\n%10lld\n", (long long)others.size());
        for (int64_t z : others) fprintf(f, "%10lld\n", (long long)z + 1);
        for (int64_t z : others) fprintf(f, "%10d\n", h->znump[z]);
        for (int64_t z : others) {
            for (int i = 0; i < h->znump[z]; ++i) fprintf(f, "%10d", h->mapsp1[mapzs[z] + i] + 1);
            fprintf(f, "\n");
        }
    }
    fclose(f);
    const std::vector<double>* vars[3] = {&zr, &ze, &zp};
    const char* vn[3] = {"zr", "ze", "zp"};
    for (int v = 0; v < 3; ++v) {
        f = fopen((b + "." + vn[v]).c_str(), "w");
        if (!f) return fail(PNT_ERR_INVALID_ARG, "cannot open %s.%s", base, vn[v]);
        fprintf(f, "%s\npart\n%10d\n", vn[v], 1);
        for (int k = 0; k < 2; ++k) {
            if (groups[k]->empty()) continue;
            fprintf(f, "%s\n", tags[k]);
            for (int64_t z : *groups[k]) fprintf(f, "%12.5e\n", (*vars[v])[z]);
        }
        if (!others.empty()) {
            fprintf(f, "nsided\n");
            for (int64_t z : others) fprintf(f, "%12.5e\n", (*vars[v])[z]);
        }
        fclose(f);
    }
    return PNT_OK;
}

pnt_status pnt_hydro_set_closure(pnt_hydro* h, const pnt_closure* c, int32_t mode) {
    if (!h || !c || mode < 0 || mode > 2) return fail(PNT_ERR_INVALID_ARG, "bad argument");
    if (!h->learned) return fail(PNT_ERR_STATE, "the hydro object was not created with precision learned");
    if (pnt::closure_device(c) != h->device) return fail(PNT_ERR_INVALID_ARG, "closure lives on another device");
    DeviceGuard dg(h->device);
    if (!h->a.closure_img) {
        uint8_t* img = nullptr;
        float* rec = nullptr;
        int32_t* nrec = nullptr;
        if (pnt_status st = h->alloc(&img, kImgBytes)) return st;
        if (pnt_status st = h->alloc(&rec, (size_t)h->numz * kZoneRecF4 * 4)) return st;
        if (pnt_status st = h->alloc(&nrec, 1)) return st;
        CUDA_TRY(cudaMemset(nrec, 0, sizeof(int32_t)));
        CUDA_TRY(prepare_learned_kernels());
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
        h->a.closure_img = img;
        h->a.closure_rec = rec;
        h->a.closure_nrec = nrec;
        h->a.closure_grid = kCpCtasPerSm * nsm;
    }
    // the image lives in this object: a copy of the closure's, with the mode
    uint8_t* img = const_cast<uint8_t*>(h->a.closure_img);
    const float fmode = (float)mode;
    CUDA_TRY(cudaMemcpyAsync(img, pnt::closure_image(c), kImgBytes, cudaMemcpyDeviceToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(img + kImgThr + 12, &fmode, sizeof(float), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (h->graph1) {   // the captured cycle holds the old DevArrays
        cudaGraphExecDestroy(h->graph1);
        h->graph1 = nullptr;
    }
    if (h->graph) {   // the captured cycles hold the old DevArrays
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    return PNT_OK;
}

pnt_status pnt_hydro_closure_counts(pnt_hydro* h, uint64_t* counts, int32_t reset) {
    if (!h || !counts) return fail(PNT_ERR_INVALID_ARG, "null argument");
    if (!h->learned) return fail(PNT_ERR_STATE, "the hydro object was not created with precision learned");
    DeviceGuard dg(h->device);
    std::vector<unsigned long long> raw(kClassCount * 64);
    CUDA_TRY(cudaMemcpyAsync(raw.data(), h->a.closure_counts, raw.size() * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, h->stream));
    if (reset)
        CUDA_TRY(cudaMemsetAsync(h->a.closure_counts, 0, raw.size() * sizeof(unsigned long long), h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int q = 0; q < PNT_CLOSURE_NCLASS; ++q) {
        uint64_t t = 0;
        for (int b = 0; b < 64; ++b) t += raw[q * 64 + b];
        counts[q] = t;
    }
    return PNT_OK;
}

pnt_status pnt_hydro_copy_state(pnt_hydro* dst, const pnt_hydro* src) {
    if (!dst || !src) return fail(PNT_ERR_INVALID_ARG, "null argument");
    if (dst->device != src->device || dst->nump != src->nump || dst->numz != src->numz || dst->nums != src->nums)
        return fail(PNT_ERR_INVALID_ARG, "objects differ in mesh or device");
    if (dst == src) return PNT_OK;
    DeviceGuard dg(dst->device);
    pnt_hydro* s = const_cast<pnt_hydro*>(src);
    if (pnt_status st = s->fetch_ctl()) return st;
    const size_t np = (size_t)src->nump * sizeof(double2), nz = (size_t)src->numz * sizeof(double);
    CUDA_TRY(cudaStreamSynchronize(dst->stream));
    for (int b = 0; b < 2; ++b) {
        CUDA_TRY(cudaMemcpyAsync(dst->a.px[b], src->a.px[b], np, cudaMemcpyDeviceToDevice, dst->stream));
        CUDA_TRY(cudaMemcpyAsync(dst->a.pu[b], src->a.pu[b], np, cudaMemcpyDeviceToDevice, dst->stream));
    }
    double* zd[] = {dst->a.zm, dst->a.zr, dst->a.ze, dst->a.zetot, dst->a.zwrate, dst->a.zvol, dst->a.zp};
    const double* zs[] = {src->a.zm, src->a.zr, src->a.ze, src->a.zetot, src->a.zwrate, src->a.zvol, src->a.zp};
    for (int i = 0; i < 7; ++i) CUDA_TRY(cudaMemcpyAsync(zd[i], zs[i], nz, cudaMemcpyDeviceToDevice, dst->stream));
    // run state: the source's, with done judged again by dst's deck
    Ctl c = *src->ctl_host;
    c.stop_at = INT_MAX;
    c.done = (c.status != 0 || c.cycle >= dst->params.cstop || !(c.time < dst->params.tstop)) ? 1 : 0;
    *dst->ctl_host = c;
    CUDA_TRY(cudaMemcpyAsync(dst->a.ctl, dst->ctl_host, sizeof(Ctl), cudaMemcpyHostToDevice, dst->stream));
    CUDA_TRY(cudaStreamSynchronize(dst->stream));
    return PNT_OK;
}

}  // extern "C"

namespace pnt {

pnt_status write_xy_file(const char* path, const std::vector<double>& zr, const std::vector<double>& ze,
                         const std::vector<double>& zp) {
    return write_xy(path, zr, ze, zp);
}

}  // namespace pnt

namespace pnt {
bool hydro_access(pnt_hydro* h, HydroAccess* out) {
    if (!h || !out) return false;
    out->a = h->a;
    out->c = h->hc;
    out->stream = h->stream;
    out->device = h->device;
    return true;
}
}  // namespace pnt
