// pieces.cpp -- numpcs pieces of one mesh stepped together by the library
// (pnt_pieces_*): the reference's Mesh(inp, numpcs) on one node
// (Mesh.cc:211-241), its halo sums of corner mass and force at shared
// points (Hydro.cc:571-574, 766-769) and its dt reductions
// (Hydro.cc:961-970), without Legion.
//
// Each piece is a pnt_hydro over a pnt_mesh_piece mesh on its own device
// and stream.  A cycle is, from one host thread:
//   1. every piece: pnt_hydro_piece_forces (pass A, closure, pack) and an
//      event after it;
//   2. every piece q, for each neighbour r: its stream waits for r's event,
//      then a peer copy (cudaMemcpyPeerAsync; over NVLink between devices,
//      a plain device copy on one device) brings r's corner masses and
//      forces for q into q's halo slots;
//   3. every piece: pnt_hydro_piece_advance (passes B, C, its reduction);
//   4. the host reads the four scalars of every piece, reduces them
//      (minimum dt and -dvovmax, summed inverted sides: exact in any order)
//      and writes the result back to every piece;
//   5. every piece: pnt_hydro_piece_finish.
// Step 4 synchronises every stream, so a piece's send buffer is not
// overwritten by the next cycle's pack before its neighbours have copied it.
// Every piece ends each cycle with exactly the single-piece values of its
// zones and points.
#include "pnt_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <new>
#include <vector>

namespace {

struct Piece {
    pnt_mesh* mesh = nullptr;
    pnt_hydro* hydro = nullptr;
    pnt_piece_desc desc{};
    pnt_piece_buffers buf{};
    int device = 0;
    int32_t numz = 0, nump = 0;
    cudaEvent_t packed = nullptr;
};

struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int d) {
        cudaGetDevice(&prev);
        cudaSetDevice(d);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

pnt_status cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    return pnt::fail(PNT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace

struct pnt_pieces {
    std::vector<Piece> p;
    pnt_params params{};
    int32_t numz = 0, nump = 0;
    double* red_host = nullptr;   // pinned [npieces][4]
    // a cycle that failed part way leaves some pieces a phase ahead of others
    bool broken = false;

    ~pnt_pieces() {
        for (Piece& q : p) {
            DeviceScope ds(q.device);
            if (q.packed) cudaEventDestroy(q.packed);
            if (q.hydro) pnt_hydro_destroy(q.hydro);
            if (q.mesh) pnt_mesh_destroy(q.mesh);
        }
        if (red_host) cudaFreeHost(red_host);
    }

    pnt_status cycle() {
        const int n = (int)p.size();
        for (Piece& q : p) {
            if (pnt_status st = pnt_hydro_piece_forces(q.hydro)) return st;
            DeviceScope ds(q.device);
            const cudaError_t e = cudaEventRecord(q.packed, (cudaStream_t)q.buf.stream);
            if (e != cudaSuccess) return cuda_fail(e, "event record");
        }
        for (int qi = 0; qi < n; ++qi) {
            Piece& q = p[qi];
            DeviceScope ds(q.device);
            cudaStream_t s = (cudaStream_t)q.buf.stream;
            for (int j = 0; j < q.desc.nnbr; ++j) {
                const Piece& r = p[q.desc.nbr[j]];
                // r's send range for q
                int k = 0;
                while (k < r.desc.nnbr && r.desc.nbr[k] != qi) ++k;
                if (k == r.desc.nnbr) return pnt::fail(PNT_ERR_STATE, "pieces %d and %d disagree on sharing", qi, q.desc.nbr[j]);
                const size_t s0 = (size_t)r.desc.send_off[k], s1 = (size_t)r.desc.send_off[k + 1];
                const size_t r0 = (size_t)q.desc.recv_off[j], r1 = (size_t)q.desc.recv_off[j + 1];
                if (s1 - s0 != r1 - r0) return pnt::fail(PNT_ERR_STATE, "halo sizes of pieces %d and %d differ", qi, q.desc.nbr[j]);
                const size_t cnt = r1 - r0;
                cudaError_t e = cudaStreamWaitEvent(s, r.packed, 0);
                const char* src = static_cast<const char*>(r.buf.send);
                char* hm = static_cast<char*>(q.buf.halo_cmass);
                char* hf = static_cast<char*>(q.buf.halo_cforce);
                if (e == cudaSuccess && cnt)
                    e = cudaMemcpyPeerAsync(hm + r0 * q.buf.cmass_bytes, q.device, src + s0 * r.buf.cmass_bytes, r.device,
                                            cnt * q.buf.cmass_bytes, s);
                if (e == cudaSuccess && cnt)
                    e = cudaMemcpyPeerAsync(hf + r0 * q.buf.cforce_bytes, q.device,
                                            src + r.buf.send_cforce_offset + s0 * r.buf.cforce_bytes, r.device,
                                            cnt * q.buf.cforce_bytes, s);
                if (e != cudaSuccess) return cuda_fail(e, "halo copy");
            }
        }
        for (int qi = 0; qi < n; ++qi) {
            Piece& q = p[qi];
            if (pnt_status st = pnt_hydro_piece_advance(q.hydro)) return st;
            DeviceScope ds(q.device);
            const cudaError_t e = cudaMemcpyAsync(red_host + 4 * qi, q.buf.red, 4 * sizeof(double),
                                                  cudaMemcpyDeviceToHost, (cudaStream_t)q.buf.stream);
            if (e != cudaSuccess) return cuda_fail(e, "reduction read");
        }
        for (Piece& q : p) {
            DeviceScope ds(q.device);
            const cudaError_t e = cudaStreamSynchronize((cudaStream_t)q.buf.stream);
            if (e != cudaSuccess) return cuda_fail(e, "piece synchronize");
        }
        // minimum of dtnew and -dvovmax, sums of the inverted sides
        double r[4] = {red_host[0], red_host[1], red_host[2], red_host[3]};
        for (int qi = 1; qi < n; ++qi) {
            const double* v = red_host + 4 * qi;
            r[0] = (v[0] < r[0]) ? v[0] : r[0];
            r[1] = (v[1] < r[1]) ? v[1] : r[1];
            r[2] += v[2];
            r[3] += v[3];
        }
        for (int qi = 0; qi < n; ++qi) std::copy(r, r + 4, red_host + 4 * qi);
        for (int qi = 0; qi < n; ++qi) {
            Piece& q = p[qi];
            DeviceScope ds(q.device);
            const cudaError_t e = cudaMemcpyAsync(q.buf.red, red_host + 4 * qi, 4 * sizeof(double),
                                                  cudaMemcpyHostToDevice, (cudaStream_t)q.buf.stream);
            if (e != cudaSuccess) return cuda_fail(e, "reduction write");
            if (pnt_status st = pnt_hydro_piece_finish(q.hydro)) return st;
        }
        return PNT_OK;
    }
};

extern "C" {

pnt_status pnt_pieces_create(const pnt_mesh* mesh, const pnt_params* params, int32_t npieces, const int32_t* devices,
                             int32_t ndevices, pnt_pieces** out) {
    if (!mesh || !params || !out || npieces < 2 || (ndevices > 0 && !devices))
        return pnt::fail(PNT_ERR_INVALID_ARG, "bad argument (at least 2 pieces)");
    *out = nullptr;
    pnt_pieces* ps = new (std::nothrow) pnt_pieces();
    if (!ps) return pnt::fail(PNT_ERR_NOMEM, "out of memory");
    pnt_status st = PNT_OK;
    try {
        ps->p.resize(npieces);
        pnt_mesh_desc gd;
        if ((st = pnt_mesh_describe(mesh, &gd))) throw st;
        ps->numz = gd.numz;
        ps->nump = gd.nump;
        ps->params = *params;
        for (int qi = 0; qi < npieces && !st; ++qi) {
            Piece& q = ps->p[qi];
            q.device = ndevices > 0 ? devices[qi % ndevices] : 0;
            if ((st = pnt_mesh_piece(mesh, npieces, qi, &q.mesh))) break;
            if ((st = pnt_mesh_piece_describe(q.mesh, &q.desc))) break;
            pnt_mesh_desc d;
            if ((st = pnt_mesh_describe(q.mesh, &d))) break;
            q.numz = d.numz;
            q.nump = d.nump;
            if ((st = pnt_hydro_create(q.mesh, params, q.device, &q.hydro))) break;
            if ((st = pnt_hydro_piece_buffers(q.hydro, &q.buf))) break;
            DeviceScope ds(q.device);
            const cudaError_t e = cudaEventCreateWithFlags(&q.packed, cudaEventDisableTiming);
            if (e != cudaSuccess) st = cuda_fail(e, "event create");
        }
        if (!st) {
            // peer access where it helps (copies work without it, through the host)
            for (Piece& q : ps->p)
                for (const Piece& r : ps->p)
                    if (q.device != r.device) {
                        int can = 0;
                        cudaDeviceCanAccessPeer(&can, q.device, r.device);
                        if (can) {
                            DeviceScope ds(q.device);
                            cudaDeviceEnablePeerAccess(r.device, 0);
                            cudaGetLastError();   // already enabled is fine
                        }
                    }
            const cudaError_t e = cudaMallocHost((void**)&ps->red_host, sizeof(double) * 4 * npieces);
            if (e != cudaSuccess) st = cuda_fail(e, "pinned reduction buffer");
        }
    } catch (pnt_status s) {
        st = s;
    } catch (const std::bad_alloc&) {
        st = pnt::fail(PNT_ERR_NOMEM, "out of host memory");
    }
    if (st) {
        delete ps;
        return st;
    }
    *out = ps;
    return PNT_OK;
}

pnt_status pnt_pieces_cycle(pnt_pieces* ps, pnt_scalars* out) {
    if (!ps) return pnt::fail(PNT_ERR_INVALID_ARG, "null argument");
    if (ps->broken) return pnt::fail(PNT_ERR_STATE, "an earlier cycle of these pieces failed part way");
    if (pnt_status st = ps->cycle()) {
        ps->broken = true;
        return st;
    }
    pnt_scalars s{};
    if (pnt_status st = pnt_hydro_get_scalars(ps->p[0].hydro, &s)) return st;
    if (out) *out = s;
    if (s.status) return pnt::fail(s.status, "%d negative side volumes on cycle %d", s.nbad, s.cycle);
    return PNT_OK;
}

pnt_status pnt_pieces_run(pnt_pieces* ps, int32_t max_cycles, pnt_report_fn report, void* user, pnt_scalars* out) {
    if (!ps) return pnt::fail(PNT_ERR_INVALID_ARG, "null argument");
    pnt_scalars s{};
    if (pnt_status st = pnt_hydro_get_scalars(ps->p[0].hydro, &s)) return st;
    // the report cadence of Driver::run (Driver.cc:147-156): cycle 1, then every dtreport
    const int dtreport = ps->params.dtreport > 0 ? ps->params.dtreport : 10;
    const auto t0 = std::chrono::steady_clock::now();
    int n = 0;
    while (!s.done && (max_cycles <= 0 || n < max_cycles)) {
        if (pnt_status st = pnt_pieces_cycle(ps, &s)) {
            if (out) *out = s;
            return st;
        }
        ++n;
        if (report && (s.cycle == 1 || s.cycle % dtreport == 0)) {
            const double us = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
            report(&s, us, user);
        }
    }
    if (out) *out = s;
    return PNT_OK;
}

pnt_status pnt_pieces_download(pnt_pieces* ps, int32_t field, void* dst, size_t bytes) {
    if (!ps || !dst) return pnt::fail(PNT_ERR_INVALID_ARG, "null argument");
    const bool point = field == PNT_FIELD_PX || field == PNT_FIELD_PU;
    const bool zone = field >= PNT_FIELD_ZR && field <= PNT_FIELD_ZWRATE;
    if (!point && !zone) return pnt::fail(PNT_ERR_UNSUPPORTED, "field %d is not gathered from pieces", field);
    const size_t need = point ? (size_t)ps->nump * 16 : (size_t)ps->numz * 8;
    if (bytes != need) return pnt::fail(PNT_ERR_INVALID_ARG, "field %d needs %zu bytes, got %zu", field, need, bytes);
    std::vector<double> tmp;
    for (const Piece& q : ps->p) {
        if (zone) {
            pnt_status st = pnt_hydro_download(q.hydro, field, static_cast<double*>(dst) + q.desc.zone0,
                                               (size_t)q.numz * 8);
            if (st) return st;
        } else {
            tmp.resize(2 * (size_t)q.nump);
            pnt_status st = pnt_hydro_download(q.hydro, field, tmp.data(), tmp.size() * 8);
            if (st) return st;
            double* d = static_cast<double*>(dst);
            for (int32_t i = 0; i < q.nump; ++i) {   // shared points hold the same values in every piece
                d[2 * (size_t)q.desc.gpoint[i]] = tmp[2 * (size_t)i];
                d[2 * (size_t)q.desc.gpoint[i] + 1] = tmp[2 * (size_t)i + 1];
            }
        }
    }
    return PNT_OK;
}

pnt_status pnt_pieces_set_closure(pnt_pieces* ps, const pnt_closure* closure, int32_t mode) {
    if (!ps) return pnt::fail(PNT_ERR_INVALID_ARG, "null argument");
    for (Piece& q : ps->p)
        if (pnt_status st = pnt_hydro_set_closure(q.hydro, closure, mode)) return st;
    return PNT_OK;
}

pnt_status pnt_pieces_write_xy(pnt_pieces* ps, const char* path) {
    if (!ps || !path) return pnt::fail(PNT_ERR_INVALID_ARG, "null argument");
    std::vector<double> zr(ps->numz), ze(ps->numz), zp(ps->numz);
    pnt_status st = pnt_pieces_download(ps, PNT_FIELD_ZR, zr.data(), zr.size() * 8);
    if (!st) st = pnt_pieces_download(ps, PNT_FIELD_ZE, ze.data(), ze.size() * 8);
    if (!st) st = pnt_pieces_download(ps, PNT_FIELD_ZP, zp.data(), zp.size() * 8);
    if (st) return st;
    return pnt::write_xy_file(path, zr, ze, zp);
}

void pnt_pieces_destroy(pnt_pieces* ps) { delete ps; }

}  // extern "C"
