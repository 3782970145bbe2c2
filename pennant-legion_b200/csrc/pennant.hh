// pennant.hh -- C++ host classes with the reference's method surface
// (InputFile, Mesh, Hydro, Driver), built on the C ABI in pennant_b200.h.
//
// These mirror InputFile.hh:21-42, Mesh.hh:424-705 (construction, sizes
// and connectivity), Hydro.hh:90-111 (coefficients, ctor, doCycle),
// PolyGas.hh:35-39, TTS.hh:34-38, QCS.hh:39-44, HydroBC.hh:50-66 (their
// coefficients and boundary point lists) and Driver.hh:60-82 (the run
// loop), so code written against the reference's classes ports by
// re-linking.  Every coefficient comes from pnt_params_from_deck, the same
// parse the GPU cycle uses.  Errors throw pnt::Error carrying the C ABI
// status instead of calling exit().
#pragma once

#include "pennant_b200.h"

#include <cmath>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace pnt {

class Error : public std::runtime_error {
public:
    Error(pnt_status st, const std::string& what) : std::runtime_error(what), status(st) {}
    pnt_status status;
};

inline void check(pnt_status st) {
    if (st) throw Error(st, std::string(pnt_status_string(st)) + ": " + pnt_last_error());
}

class InputFile {
public:
    explicit InputFile(const char* filename) { check(pnt_deck_load(filename, &deck_)); }
    ~InputFile() { pnt_deck_destroy(deck_); }
    InputFile(const InputFile&) = delete;
    InputFile& operator=(const InputFile&) = delete;

    int getInt(const std::string& key, int dflt) const { return pnt_deck_get_int(deck_, key.c_str(), dflt); }
    double getDouble(const std::string& key, double dflt) const {
        return pnt_deck_get_double(deck_, key.c_str(), dflt);
    }
    std::string getString(const std::string& key, const std::string& dflt) const {
        const int n = pnt_deck_get_string(deck_, key.c_str(), dflt.c_str(), nullptr, 0);
        std::string s(n, '\0');
        pnt_deck_get_string(deck_, key.c_str(), dflt.c_str(), &s[0], n + 1);
        return s;
    }
    std::vector<double> getDoubleList(const std::string& key, const std::vector<double>& dflt) const {
        const int n = pnt_deck_get_double_list(deck_, key.c_str(), nullptr, 0);
        if (n < 0) return dflt;
        std::vector<double> v(n);
        pnt_deck_get_double_list(deck_, key.c_str(), v.data(), n);
        return v;
    }
    const pnt_deck* handle() const { return deck_; }

private:
    pnt_deck* deck_ = nullptr;
};

inline pnt_params params_of(const InputFile* inp) {
    pnt_params p;
    check(pnt_params_from_deck(inp->handle(), &p));
    return p;
}

#ifdef __CUDACC__
using ::double2;
#else
struct double2 {   // the reference's Vec2.hh double2 (x, y)
    double x, y;
};
#endif

class Hydro;

// PolyGas (PolyGas.hh:35-39, PolyGas.cc:57-60).
class PolyGas {
public:
    PolyGas(const InputFile* inp, Hydro* h) : hydro(h) {
        const pnt_params p = params_of(inp);
        gamma = p.gamma;
        ssmin = p.pgas_ssmin;
    }
    Hydro* hydro;
    double gamma = 0., ssmin = 0.;
};

// TTS (TTS.hh:34-38, TTS.cc:45-48).
class TTS {
public:
    TTS(const InputFile* inp, Hydro* h) : hydro(h) {
        const pnt_params p = params_of(inp);
        alfa = p.alfa;
        ssmin = p.tts_ssmin;
    }
    Hydro* hydro;
    double alfa = 0., ssmin = 0.;
};

// QCS (QCS.hh:39-44, QCS.cc:83-86).
class QCS {
public:
    QCS(const InputFile* inp, Hydro* h) : hydro(h) {
        const pnt_params p = params_of(inp);
        qgamma = p.qgamma;
        q1 = p.q1;
        q2 = p.q2;
    }
    Hydro* hydro;
    double qgamma = 0., q1 = 0., q2 = 0.;
};

class Mesh {
public:
    // The whole mesh (one piece); its pieces are pnt_mesh_piece meshes, and
    // pnt_pieces steps numpcs of them together (the `pennant -n` path).
    Mesh(const InputFile* inp, int numpcs = 1) {
        if (numpcs != 1) throw Error(PNT_ERR_UNSUPPORTED, "build the pieces with pnt_mesh_piece / pnt_pieces_create");
        check(pnt_mesh_generate(inp->handle(), &mesh_));
        pnt_mesh_desc d;
        check(pnt_mesh_describe(mesh_, &d));
        nump = d.nump;
        numz = d.numz;
        nums = d.nums;
        numc = d.nums;
    }
    ~Mesh() { pnt_mesh_destroy(mesh_); }
    Mesh(const Mesh&) = delete;
    Mesh& operator=(const Mesh&) = delete;
    const pnt_mesh* handle() const { return mesh_; }

    // Initial point coordinates and side maps (reference numbering; the
    // arrays stay owned by the mesh).
    const double2* px() const { return reinterpret_cast<const double2*>(desc().px); }
    const int32_t* znump() const { return desc().znump; }
    const int32_t* mapsp1() const { return desc().mapsp1; }
    const int32_t* mapsp2() const { return desc().mapsp2; }
    const int32_t* mapsz() const { return desc().mapsz; }
    const int32_t* mapss3() const { return desc().mapss3; }
    const int32_t* mapss4() const { return desc().mapss4; }

    int nump = 0, numz = 0, nums = 0, numc = 0;

private:
    pnt_mesh_desc desc() const {
        pnt_mesh_desc d;
        check(pnt_mesh_describe(mesh_, &d));
        return d;
    }
    pnt_mesh* mesh_ = nullptr;
};

// HydroBC (HydroBC.hh:50-66, HydroBC.cc:63-144): a fixed plane x = bound
// (xplane) or y = bound with its velocity-projection vector vfix and its
// boundary points, the points within 1e-12 of the plane in ascending order.
class HydroBC {
public:
    HydroBC(Mesh* msh, const double2 v, const double bound, const bool xplane) : mesh(msh), vfix(v) {
        const double2* px = msh->px();
        for (int p = 0; p < msh->nump; ++p) {
            const double c = xplane ? px[p].x : px[p].y;
            if (std::fabs(c - bound) < 1.e-12) mapbp.push_back(p);
        }
        numb = (int)mapbp.size();
    }
    Mesh* mesh;
    int numb = 0;
    double2 vfix;
    std::vector<int> mapbp;
};

class Hydro {
public:
    // Hydro(inp, mesh) + init() (Hydro.cc:200-339): the coefficients, the
    // physics objects and the boundaries in deck order (bcx then bcy,
    // Hydro.cc:220-225), then the device state.
    Hydro(const InputFile* inp, Mesh* m, int device = 0)
        : mesh(m), params(params_of(inp)), pgas(new PolyGas(inp, this)), tts(new TTS(inp, this)),
          qcs(new QCS(inp, this)) {
        cfl = params.cfl;
        cflv = params.cflv;
        rinit = params.rinit;
        einit = params.einit;
        rinitsub = params.rinitsub;
        einitsub = params.einitsub;
        uinitradial = params.uinitradial;
        bcx.assign(params.bcx, params.bcx + params.nbcx);
        bcy.assign(params.bcy, params.bcy + params.nbcy);
        for (double b : bcx) bcs.emplace_back(new HydroBC(m, double2{1., 0.}, b, true));
        for (double b : bcy) bcs.emplace_back(new HydroBC(m, double2{0., 1.}, b, false));
        check(pnt_hydro_create(m->handle(), &params, device, &hydro_));
    }
    ~Hydro() { pnt_hydro_destroy(hydro_); }
    Hydro(const Hydro&) = delete;
    Hydro& operator=(const Hydro&) = delete;

    // One Driver::run iteration around Hydro::doCycle; returns the
    // scalars after it (dtrec is the value the reference's doCycle returns).
    pnt_scalars doCycle() {
        pnt_scalars s;
        check(pnt_hydro_cycle(hydro_, &s));
        return s;
    }
    pnt_hydro* handle() { return hydro_; }

    Mesh* mesh;
    pnt_params params;
    std::unique_ptr<PolyGas> pgas;
    std::unique_ptr<TTS> tts;
    std::unique_ptr<QCS> qcs;
    std::vector<std::unique_ptr<HydroBC>> bcs;
    double cfl = 0., cflv = 0., rinit = 0., einit = 0., rinitsub = 0., einitsub = 0., uinitradial = 0.;
    std::vector<double> bcx, bcy;

private:
    pnt_hydro* hydro_ = nullptr;
};

// Driver (Driver.hh:60-82, Driver.cc:65-187): the stop and dt keys, the
// mesh and the hydro object, and run(): cycles to tstop or cstop with the
// reference's report line (Driver.cc:344-345) at cycle 1 and every dtreport
// cycles.  run() returns the final scalars; negative side volumes throw
// pnt::Error with PNT_ERR_BADSIDES.
class Driver {
public:
    Driver(const InputFile* inp, const std::string& pname, int device = 0)
        : probname(pname), mesh(new Mesh(inp)), hydro(new Hydro(inp, mesh.get(), device)) {
        const pnt_params& p = hydro->params;
        tstop = p.tstop;
        cstop = p.cstop;
        dtmax = p.dtmax;
        dtinit = p.dtinit;
        dtfac = p.dtfac;
        dtreport = p.dtreport;
    }

    pnt_scalars run() {
        pnt_scalars s{};
        check(pnt_hydro_run(hydro->handle(), 0, &Driver::report, nullptr, &s));
        return s;
    }

    static void report(const pnt_scalars* s, double wall_us, void*) {
        std::printf("End cycle %6d, time = %11.5g, dt = %11.5g, wall = %11lld us\n", s->cycle, s->time, s->dt,
                    (long long)wall_us);
        std::fflush(stdout);
    }

    std::string probname;
    double tstop = 0., dtmax = 0., dtinit = 0., dtfac = 0.;
    int cstop = 0, dtreport = 0;
    std::unique_ptr<Mesh> mesh;
    std::unique_ptr<Hydro> hydro;
};

}  // namespace pnt
