// pennant.hh -- C++ host classes with the reference's method surface
// (InputFile, Mesh, Hydro, Driver), built on the C ABI in pennant_b200.h.
//
// These mirror InputFile.hh:21-42, Mesh.hh:424-705 (construction and
// sizes), Hydro.hh:101-111 (ctor, init, doCycle) and Driver.hh:74-82 so
// code written against the reference's classes ports by re-linking.  Errors
// throw pnt::Error carrying the C ABI status instead of calling exit().
#pragma once

#include "pennant_b200.h"

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

    int nump = 0, numz = 0, nums = 0, numc = 0;

private:
    pnt_mesh* mesh_ = nullptr;
};

class Hydro {
public:
    Hydro(const InputFile* inp, Mesh* m, int device = 0) : mesh(m) {
        check(pnt_params_from_deck(inp->handle(), &params));
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

private:
    pnt_hydro* hydro_ = nullptr;
};

}  // namespace pnt
