// pnt_internal.h -- host-side objects behind the C ABI (include/pennant_b200.h).
#pragma once

#include "pennant_b200.h"

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace pnt {

// Records the calling thread's last error message and returns `st`.
pnt_status fail(pnt_status st, const char* fmt, ...);
void clear_error();

// InputFile (InputFile.hh:21-42): ordered key -> rest-of-line text.
struct Deck {
    std::vector<std::pair<std::string, std::string>> kv;
    const std::string* find(const std::string& key) const;
};

// Parses deck text as InputFile::InputFile does (InputFile.cc:24-60).
pnt_status parse_deck(const std::string& text, Deck& out);
int get_int(const Deck& d, const char* key, int dflt);
double get_double(const Deck& d, const char* key, double dflt);
std::string get_string(const Deck& d, const char* key, const std::string& dflt);
// -1 when the key is absent.
int get_double_list(const Deck& d, const char* key, std::vector<double>& out);

// Single-piece mesh in reference numbering plus the derived structures the
// device passes use.
struct Mesh {
    int32_t nump = 0, numz = 0, nums = 0;
    std::vector<double> px;  // 2*nump
    std::vector<int32_t> znump, mapsp1, mapsp2, mapsz, mapss3, mapss4;
    // derived
    std::vector<int32_t> zfirst;       // first side of each zone
    std::vector<int32_t> poff, pcorner;  // point -> sides CSR (ascending side)
    bool all_quads = false;            // every zone has 4 sides at 4z..4z+3
    // initial geometry (Mesh::init, Mesh.cc:619-623)
    std::vector<double> zx, zarea, zvol, sarea, svol, smf;
};

// GenMesh rect/pie generation (GenMesh.cc:790-1282), single piece.
pnt_status generate_mesh(const Deck& d, Mesh& m);
// Validates connectivity, builds zfirst/CSR and the initial geometry.
pnt_status finish_mesh(Mesh& m);

// The closure's device parameter image and device (closure.cu).
const uint8_t* closure_image(const pnt_closure* c);
int closure_device(const pnt_closure* c);

}  // namespace pnt

struct pnt_deck {
    pnt::Deck d;
};

struct pnt_mesh {
    pnt::Mesh m;
};
