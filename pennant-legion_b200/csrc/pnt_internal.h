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
    int32_t rect_nzx = 0;              // > 0: the rect generator's numbering, nzx zones a row
    // initial geometry (Mesh::init, Mesh.cc:619-623)
    std::vector<double> zx, zarea, zvol, sarea, svol, smf;
    // Multi-piece runs (make_piece): this mesh is piece `piece` of
    // `npieces`, local zones are the global zones zone0.., local sides the
    // global sides side0.., gpoint maps local to global points.  The point
    // -> corner CSR also lists halo slots nums + h: corners of the piece's
    // points that belong to other pieces' sides (global side halo_side[h]),
    // grouped by owning neighbour (nbr, recv_off) in global side order.
    // send_side[send_off[j] .. send_off[j+1]) are the local sides whose
    // corner values neighbour nbr[j] needs, in global side order.
    bool is_piece = false;             // made by make_piece (1 piece included): stepped piece by piece
    int32_t piece = 0, npieces = 1;
    int32_t zone0 = 0, side0 = 0;
    std::vector<int32_t> gpoint;
    int32_t nhalo = 0;
    std::vector<int32_t> halo_side;
    std::vector<int32_t> nbr, send_off, send_side, recv_off;
};

// GenMesh rect/pie generation (GenMesh.cc:790-1282), single piece.
pnt_status generate_mesh(const Deck& d, Mesh& m);
// Validates connectivity, builds zfirst/CSR and the initial geometry.
pnt_status finish_mesh(Mesh& m);
// Piece `piece` of `npieces` (at most 64) of a finished single-piece mesh:
// the contiguous zone range [numz*piece/npieces, numz*(piece+1)/npieces).
pnt_status make_piece(const Mesh& g, int npieces, int piece, Mesh& out);

// The reference's .xy writer (WriteXY.cc:28-52) for zone fields in global
// order (hydro.cu).
pnt_status write_xy_file(const char* path, const std::vector<double>& zr, const std::vector<double>& ze,
                         const std::vector<double>& zp);
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
