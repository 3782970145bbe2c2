// host_mesh.cpp -- deck parsing (InputFile), mesh generation (GenMesh) and
// the mesh data-structure build (Mesh::init) for one piece, plus their C ABI.
//
// Compiled with -ffp-contract=off: the initial geometry (Mesh.cc:619-623)
// must carry the reference's exact IEEE operation order.
#include "pnt_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <unordered_map>

namespace pnt {

static thread_local std::string g_err;

pnt_status fail(pnt_status st, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return st;
}

void clear_error() { g_err.clear(); }

const std::string* Deck::find(const std::string& key) const {
    for (const auto& p : kv)
        if (p.first == key) return &p.second;
    return nullptr;
}

// InputFile::InputFile (InputFile.cc:24-60).  Each line: first
// whitespace-separated token is the key, the rest of the line the value;
// empty lines and keys starting with '#' are skipped; a repeated key is an
// error.  As in the reference, getline() reaching end-of-file ends the
// loop, so a final line without a trailing newline is not read.
pnt_status parse_deck(const std::string& text, Deck& out) {
    out.kv.clear();
    size_t pos = 0;
    while (pos < text.size()) {
        const size_t eol = text.find('\n', pos);
        if (eol == std::string::npos) break;
        std::istringstream iss(text.substr(pos, eol - pos));
        pos = eol + 1;
        std::string key;
        iss >> key;
        if (key.empty() || key[0] == '#') continue;
        if (out.find(key)) return fail(PNT_ERR_DECK, "Duplicate key %s in input file", key.c_str());
        std::string val;
        std::getline(iss, val);
        out.kv.emplace_back(key, val);
    }
    return PNT_OK;
}

// InputFile::get<T> (InputFile.cc:63-73): stream-extract one value.
template <typename T>
static T get_value(const Deck& d, const char* key, const T& dflt) {
    const std::string* v = d.find(key);
    if (!v) return dflt;
    std::istringstream iss(*v);
    T val{};
    iss >> val;
    return val;
}

int get_int(const Deck& d, const char* key, int dflt) { return get_value<int>(d, key, dflt); }
double get_double(const Deck& d, const char* key, double dflt) { return get_value<double>(d, key, dflt); }
std::string get_string(const Deck& d, const char* key, const std::string& dflt) {
    return get_value<std::string>(d, key, dflt);
}

// InputFile::getDoubleList (InputFile.cc:91-104).
int get_double_list(const Deck& d, const char* key, std::vector<double>& out) {
    out.clear();
    const std::string* v = d.find(key);
    if (!v) return -1;
    std::istringstream iss(*v);
    double val;
    while (iss >> val) out.push_back(val);
    return (int)out.size();
}

// ---------------------------------------------------------------------
// GenMesh, one piece (numpcx = numpcy = 1).
// ---------------------------------------------------------------------
pnt_status generate_mesh(const Deck& d, Mesh& m) {
    // GenMesh::GenMesh (GenMesh.cc:87-129)
    const std::string meshtype = get_string(d, "meshtype", "");
    if (meshtype.empty()) return fail(PNT_ERR_DECK, "must specify meshtype");
    if (meshtype != "pie" && meshtype != "rect" && meshtype != "hex")
        return fail(PNT_ERR_DECK, "invalid meshtype %s", meshtype.c_str());
    if (meshtype == "hex")
        return fail(PNT_ERR_UNSUPPORTED,
                    "meshtype hex: the reference's parallel hex generator is unimplemented");
    std::vector<double> params;
    if (get_double_list(d, "meshparams", params) <= 0)
        return fail(PNT_ERR_DECK, "must specify meshparams");
    if (params.size() > 4) return fail(PNT_ERR_DECK, "meshparams must have <= 4 values");
    const int nzx = (int)params[0];
    const int nzy = (params.size() >= 2 ? (int)params[1] : nzx);
    const bool pie = (meshtype == "pie");
    const double lenx = pie ? (params.size() >= 3 ? params[2] : 90.0) * M_PI / 180.0
                            : (params.size() >= 3 ? params[2] : 1.0);
    const double leny = (params.size() >= 4 ? params[3] : 1.0);
    if (nzx <= 0 || nzy <= 0 || lenx <= 0. || leny <= 0.)
        return fail(PNT_ERR_DECK, "meshparams values must be positive");
    if (pie && lenx >= 2. * M_PI) return fail(PNT_ERR_DECK, "meshparams theta must be < 360");

    const int64_t npx = nzx + 1, npy = nzy + 1;
    const int64_t np = pie ? npx * (npy - 1) + 1 : npx * npy;    // GenMesh.cc:485-500
    const int64_t nz = (int64_t)nzx * nzy;
    const int64_t ns = pie ? 4 * (int64_t)nzx * (nzy - 1) + 3 * (int64_t)nzx : 4 * nz;
    if (ns > INT32_MAX || np > INT32_MAX) return fail(PNT_ERR_UNSUPPORTED, "mesh exceeds int32 indexing");
    m.nump = (int32_t)np;
    m.numz = (int32_t)nz;
    m.nums = (int32_t)ns;
    m.px.assign(2 * np, 0.);
    m.znump.assign(nz, 4);
    m.mapsp1.assign(ns, 0);
    m.mapsp2.assign(ns, 0);
    m.mapsz.assign(ns, 0);
    m.mapss3.assign(ns, 0);
    m.mapss4.assign(ns, 0);

    if (!pie) {
        // genPointsRect (GenMesh.cc:790-829): p = j*(nzx+1)+i at (dx*i, dy*j)
        const double dx = lenx / (double)nzx;
        const double dy = leny / (double)nzy;
        for (int64_t p = 0; p < np; ++p) {
            const int64_t i = p % npx, j = p / npx;
            m.px[2 * p] = dx * double(i);
            m.px[2 * p + 1] = dy * double(j);
        }
        // genSidesRect (GenMesh.cc:987-1100): side k of zone z is s = 4z+k,
        // k = bottom, right, top, left; zones row-major.
        for (int64_t s = 0; s < ns; ++s) {
            const int k = (int)(s % 4);
            const int64_t z = s / 4;
            const int64_t zi = z % nzx, zj = z / nzx;
            m.mapss3[s] = (int32_t)(k == 0 ? s + 3 : s - 1);
            m.mapss4[s] = (int32_t)(k == 3 ? s - 3 : s + 1);
            m.mapsz[s] = (int32_t)z;
            static const int di1[4] = {0, 1, 1, 0}, dj1[4] = {0, 0, 1, 1};
            static const int di2[4] = {1, 1, 0, 0}, dj2[4] = {0, 1, 1, 0};
            m.mapsp1[s] = (int32_t)((zj + dj1[k]) * npx + zi + di1[k]);
            m.mapsp2[s] = (int32_t)((zj + dj2[k]) * npx + zi + di2[k]);
        }
    } else {
        // genPointsPie (GenMesh.cc:831-873): point 0 is the origin, then
        // rings j = 1..nzy of npx points at angle dth*(nzx - i).
        const double dth = lenx / (double)nzx;
        const double dr = leny / (double)nzy;
        for (int64_t p = 1; p < np; ++p) {
            const int64_t i = (p - 1) % npx, j = (p - 1) / npx + 1;
            const double th = dth * (double)(nzx - i);
            const double r = dr * (double)j;
            m.px[2 * p] = r * cos(th);
            m.px[2 * p + 1] = r * sin(th);
        }
        // genZonesPie (GenMesh.cc:932-975): 3 sides in the innermost row.
        for (int64_t z = 0; z < nz; ++z) m.znump[z] = (z < nzx) ? 3 : 4;
        // genSidesPie (GenMesh.cc:1102-1282) with one piece.
        for (int64_t s = 0; s < ns; ++s) {
            int64_t z;
            int k;
            if (s < 3 * (int64_t)nzx) {
                z = s / 3;
                k = (int)(s % 3);
            } else {
                z = nzx + (s - 3 * (int64_t)nzx) / 4;
                k = (int)((s - 3 * (int64_t)nzx) % 4);
            }
            m.mapsz[s] = (int32_t)z;
            const int64_t zi = z % nzx, zj = z / nzx;
            if (zj == 0) {
                m.mapss3[s] = (int32_t)(k == 0 ? s + 2 : s - 1);
                m.mapss4[s] = (int32_t)(k == 2 ? s - 2 : s + 1);
                const int64_t p0 = zi + 1;
                const int64_t a[3] = {0, p0 + 1, p0};
                m.mapsp1[s] = (int32_t)a[k];
                m.mapsp2[s] = (int32_t)a[(k + 1) % 3];
            } else {
                m.mapss3[s] = (int32_t)(k == 0 ? s + 3 : s - 1);
                m.mapss4[s] = (int32_t)(k == 3 ? s - 3 : s + 1);
                const int64_t p0 = (zj - 1) * npx + zi + 1;
                const int64_t a[4] = {p0, p0 + 1, p0 + npx + 1, p0 + npx};
                m.mapsp1[s] = (int32_t)a[k];
                m.mapsp2[s] = (int32_t)a[(k + 1) % 4];
            }
        }
    }
    return PNT_OK;
}

// ---------------------------------------------------------------------
// Mesh::init derived data (Mesh.cc:610-623) and validation.
// ---------------------------------------------------------------------

// The zones-per-row count nzx when the mesh is numbered as genPointsRect /
// genZonesRect / genSidesRect number a rect mesh (GenMesh.cc:790-829,
// 898-930, 987-1100: zones row-major, points nzx + 1 a row, side 4z + k of
// zone (i, j) starting at point (i, j), (i+1, j), (i+1, j+1), (i, j+1)),
// else 0.  The row-tile passes (row_tiles.cuh) rely on exactly this.
int32_t rect_columns(const Mesh& m, bool quads) {
    if (!quads || m.is_piece || m.numz < 1) return 0;
    const int64_t npx = m.mapsp1[3];   // zone 0's left side starts at point (0, 1)
    const int64_t nzx = npx - 1, nz = m.numz;
    if (nzx < 1 || nz % nzx != 0 || (int64_t)m.nump != (nz / nzx + 1) * npx) return 0;
    static const int di[4] = {0, 1, 1, 0}, dj[4] = {0, 0, 1, 1};
    for (int64_t z = 0; z < nz; ++z) {
        const int64_t zi = z % nzx, zj = z / nzx;
        for (int k = 0; k < 4; ++k)
            if (m.mapsp1[4 * z + k] != (zj + dj[k]) * npx + zi + di[k]) return 0;
    }
    return (int32_t)nzx;
}

pnt_status finish_mesh(Mesh& m) {
    const int64_t np = m.nump, nz = m.numz, ns = m.nums;
    if (np <= 0 || nz <= 0 || ns <= 0) return fail(PNT_ERR_INVALID_ARG, "empty mesh");
    if ((int64_t)m.px.size() != 2 * np || (int64_t)m.znump.size() != nz ||
        (int64_t)m.mapsp1.size() != ns || (int64_t)m.mapsp2.size() != ns ||
        (int64_t)m.mapsz.size() != ns || (int64_t)m.mapss3.size() != ns ||
        (int64_t)m.mapss4.size() != ns)
        return fail(PNT_ERR_INVALID_ARG, "mesh array sizes do not match nump/numz/nums");
    // Zones own contiguous side ranges in zone order; the device passes map
    // 4 lanes to a zone, so zones have 3 or 4 sides.
    m.zfirst.assign(nz, 0);
    int64_t s = 0;
    bool quads = true;
    for (int64_t z = 0; z < nz; ++z) {
        const int n = m.znump[z];
        if (n < 3 || n > 4)
            return fail(PNT_ERR_UNSUPPORTED, "zone %lld has %d sides; 3 or 4 supported", (long long)z, n);
        if (n != 4) quads = false;
        m.zfirst[z] = (int32_t)s;
        for (int k = 0; k < n; ++k, ++s) {
            if (s >= ns) return fail(PNT_ERR_INVALID_ARG, "znump sums past nums");
            if (m.mapsz[s] != z) return fail(PNT_ERR_INVALID_ARG, "sides of zone %lld not contiguous", (long long)z);
            const int64_t s3 = m.zfirst[z] + (k + n - 1) % n;
            const int64_t s4 = m.zfirst[z] + (k + 1) % n;
            if (m.mapss3[s] != s3 || m.mapss4[s] != s4)
                return fail(PNT_ERR_INVALID_ARG, "mapss3/mapss4 of side %lld do not circulate", (long long)s);
            if (m.mapsp1[s] < 0 || m.mapsp1[s] >= np || m.mapsp2[s] < 0 || m.mapsp2[s] >= np)
                return fail(PNT_ERR_INVALID_ARG, "side %lld point index out of range", (long long)s);
        }
    }
    if (s != ns) return fail(PNT_ERR_INVALID_ARG, "znump does not sum to nums");
    for (int64_t t = 0; t < ns; ++t)
        if (m.mapsp2[t] != m.mapsp1[m.mapss4[t]])
            return fail(PNT_ERR_INVALID_ARG, "mapsp2[%lld] != mapsp1[mapss4[%lld]]", (long long)t, (long long)t);
    m.all_quads = quads;
    m.rect_nzx = rect_columns(m, quads);

    // Point -> corner CSR, ascending side order inside each point.
    m.poff.assign(np + 1, 0);
    for (int64_t t = 0; t < ns; ++t) m.poff[m.mapsp1[t] + 1]++;
    for (int64_t p = 0; p < np; ++p) m.poff[p + 1] += m.poff[p];
    m.pcorner.assign(ns, 0);
    std::vector<int32_t> fillpos(m.poff.begin(), m.poff.end() - 1);
    for (int64_t t = 0; t < ns; ++t) m.pcorner[fillpos[m.mapsp1[t]]++] = (int32_t)t;

    // Initial geometry: calcCtrs (Mesh.cc:797-837), calcVols (:928-989),
    // calcSideFracs (:1085-1101), in the serial side order.
    m.zx.assign(2 * nz, 0.);
    m.zarea.assign(nz, 0.);
    m.zvol.assign(nz, 0.);
    m.sarea.assign(ns, 0.);
    m.svol.assign(ns, 0.);
    m.smf.assign(ns, 0.);
    const double* px = m.px.data();
    for (int64_t t = 0; t < ns; ++t) {
        const int32_t p1 = m.mapsp1[t], z = m.mapsz[t];
        const double rinv = 1. / (double)m.znump[z];
        m.zx[2 * z] += px[2 * p1] * rinv;
        m.zx[2 * z + 1] += px[2 * p1 + 1] * rinv;
    }
    const double third = 1. / 3.;
    int nbad = 0;
    for (int64_t t = 0; t < ns; ++t) {
        const int32_t p1 = m.mapsp1[t], p2 = m.mapsp2[t], z = m.mapsz[t];
        const double x1 = px[2 * p1], y1 = px[2 * p1 + 1];
        const double x2 = px[2 * p2], y2 = px[2 * p2 + 1];
        const double zxx = m.zx[2 * z], zxy = m.zx[2 * z + 1];
        const double ax = x2 - x1, ay = y2 - y1, bx = zxx - x1, by = zxy - y1;
        const double sa = 0.5 * (ax * by - ay * bx);
        const double sv = third * sa * (x1 + x2 + zxx);
        m.sarea[t] = sa;
        m.svol[t] = sv;
        m.zarea[z] += sa;
        m.zvol[z] += sv;
        if (sv <= 0.) nbad += 1;
    }
    if (nbad > 0)
        return fail(PNT_ERR_BADSIDES, "%d negative side volumes during initialization", nbad);
    for (int64_t t = 0; t < ns; ++t) m.smf[t] = m.sarea[t] / m.zarea[m.mapsz[t]];
    return PNT_OK;
}

// ---------------------------------------------------------------------
// Multi-piece decomposition: the role of Mesh(inp, numpcs) with its
// private, master and ghost points (Mesh.cc:211-241, :441-617), here as
// contiguous zone ranges in the reference's numbering.  A piece keeps its
// zones' sides and every point they touch, with local ids in global order,
// and copies the single-piece initial geometry, so each zone and point
// computes exactly what it computes in the single-piece run.  The corners
// of a shared point that other pieces own become halo slots after the
// local sides; the point -> corner CSR lists local and halo slots merged in
// global side order, so the corner-force and corner-mass sums at shared
// points keep the single-piece summation order (the reference sums shared
// points through Legion reductions instead, Hydro.cc:571-574, 766-769).
// ---------------------------------------------------------------------
pnt_status make_piece(const Mesh& g, int npieces, int piece, Mesh& m) {
    if (g.is_piece) return fail(PNT_ERR_INVALID_ARG, "the mesh is already a piece");
    if (npieces < 1 || npieces > 64 || piece < 0 || piece >= npieces)
        return fail(PNT_ERR_INVALID_ARG, "piece %d of %d: 1-64 pieces", piece, npieces);
    const int64_t np = g.nump, nz = g.numz, ns = g.nums;
    if (npieces > nz) return fail(PNT_ERR_INVALID_ARG, "%d pieces for %lld zones", npieces, (long long)nz);
    std::vector<int32_t> zbeg(npieces + 1);
    for (int q = 0; q <= npieces; ++q) zbeg[q] = (int32_t)(nz * q / npieces);
    auto piece_of = [&](int32_t z) {
        return (int)(std::upper_bound(zbeg.begin(), zbeg.end(), z) - zbeg.begin()) - 1;
    };
    // the pieces that touch each point (bit q: a zone of piece q has it)
    std::vector<uint64_t> pmask(np, 0);
    for (int q = 0; q < npieces; ++q)
        for (int64_t s = g.zfirst[zbeg[q]]; s < (zbeg[q + 1] < nz ? g.zfirst[zbeg[q + 1]] : ns); ++s)
            pmask[g.mapsp1[s]] |= 1ull << q;
    const int32_t z0 = zbeg[piece], z1 = zbeg[piece + 1];
    const int32_t s0 = g.zfirst[z0], s1 = z1 < nz ? g.zfirst[z1] : (int32_t)ns;

    m = Mesh();
    m.piece = piece;
    m.npieces = npieces;
    m.is_piece = true;
    m.zone0 = z0;
    m.side0 = s0;
    std::vector<int32_t> lp(np, -1);
    for (int64_t p = 0; p < np; ++p)
        if ((pmask[p] >> piece) & 1) {
            lp[p] = (int32_t)m.gpoint.size();
            m.gpoint.push_back((int32_t)p);
        }
    m.nump = (int32_t)m.gpoint.size();
    m.numz = z1 - z0;
    m.nums = s1 - s0;
    m.px.resize(2 * (size_t)m.nump);
    for (int32_t p = 0; p < m.nump; ++p) {
        m.px[2 * p] = g.px[2 * (size_t)m.gpoint[p]];
        m.px[2 * p + 1] = g.px[2 * (size_t)m.gpoint[p] + 1];
    }
    m.znump.assign(g.znump.begin() + z0, g.znump.begin() + z1);
    m.zfirst.resize(m.numz);
    m.all_quads = true;
    for (int32_t z = 0; z < m.numz; ++z) {
        m.zfirst[z] = g.zfirst[z0 + z] - s0;
        if (m.znump[z] != 4) m.all_quads = false;
    }
    m.mapsp1.resize(m.nums);
    m.mapsp2.resize(m.nums);
    m.mapsz.resize(m.nums);
    m.mapss3.resize(m.nums);
    m.mapss4.resize(m.nums);
    for (int32_t s = 0; s < m.nums; ++s) {
        const int32_t t = s0 + s;
        m.mapsp1[s] = lp[g.mapsp1[t]];
        m.mapsp2[s] = lp[g.mapsp2[t]];
        m.mapsz[s] = g.mapsz[t] - z0;
        m.mapss3[s] = g.mapss3[t] - s0;
        m.mapss4[s] = g.mapss4[t] - s0;
    }
    m.zx.assign(g.zx.begin() + 2 * (size_t)z0, g.zx.begin() + 2 * (size_t)z1);
    m.zarea.assign(g.zarea.begin() + z0, g.zarea.begin() + z1);
    m.zvol.assign(g.zvol.begin() + z0, g.zvol.begin() + z1);
    m.sarea.assign(g.sarea.begin() + s0, g.sarea.begin() + s1);
    m.svol.assign(g.svol.begin() + s0, g.svol.begin() + s1);
    m.smf.assign(g.smf.begin() + s0, g.smf.begin() + s1);

    // halo slots: corners at local points owned by other pieces, grouped by
    // owner, in global side order
    std::vector<std::pair<int, int32_t>> hs;
    for (int32_t p = 0; p < m.nump; ++p) {
        const int32_t gp = m.gpoint[p];
        for (int32_t c = g.poff[gp]; c < g.poff[gp + 1]; ++c) {
            const int32_t t = g.pcorner[c];
            if (t < s0 || t >= s1) hs.push_back({piece_of(g.mapsz[t]), t});
        }
    }
    std::sort(hs.begin(), hs.end());
    m.nhalo = (int32_t)hs.size();
    std::unordered_map<int32_t, int32_t> hslot;
    hslot.reserve(hs.size() * 2 + 1);
    m.recv_off.push_back(0);
    for (size_t h = 0; h < hs.size(); ++h) {
        m.halo_side.push_back(hs[h].second);
        hslot[hs[h].second] = (int32_t)h;
        if (m.nbr.empty() || m.nbr.back() != hs[h].first) {
            if (!m.nbr.empty()) m.recv_off.push_back((int32_t)h);
            m.nbr.push_back(hs[h].first);
        }
    }
    if (!m.nbr.empty()) m.recv_off.push_back(m.nhalo);
    // point -> corner CSR over local and halo slots, global side order
    m.poff.assign(m.nump + 1, 0);
    m.pcorner.clear();
    m.pcorner.reserve(m.nums + m.nhalo);
    for (int32_t p = 0; p < m.nump; ++p) {
        const int32_t gp = m.gpoint[p];
        for (int32_t c = g.poff[gp]; c < g.poff[gp + 1]; ++c) {
            const int32_t t = g.pcorner[c];
            m.pcorner.push_back((t >= s0 && t < s1) ? t - s0 : m.nums + hslot[t]);
        }
        m.poff[p + 1] = (int32_t)m.pcorner.size();
    }
    // send lists: each neighbour needs the local corners at the points it
    // shares, in global side order
    std::vector<std::vector<int32_t>> sl(m.nbr.size());
    std::vector<int> slot_of(npieces, -1);
    for (size_t j = 0; j < m.nbr.size(); ++j) slot_of[m.nbr[j]] = (int)j;
    for (int32_t s = 0; s < m.nums; ++s) {
        uint64_t bits = pmask[g.mapsp1[s0 + s]] & ~(1ull << piece);
        while (bits) {
            const int q = __builtin_ctzll(bits);
            bits &= bits - 1;
            if (slot_of[q] < 0) return fail(PNT_ERR_INVALID_ARG, "piece %d shares a point with %d but owns none of its corners", piece, q);
            sl[slot_of[q]].push_back(s);
        }
    }
    m.send_off.push_back(0);
    for (auto& v : sl) {
        m.send_side.insert(m.send_side.end(), v.begin(), v.end());
        m.send_off.push_back((int32_t)m.send_side.size());
    }
    return PNT_OK;
}

}  // namespace pnt

using namespace pnt;

// ---------------------------------------------------------------------
// C ABI: status, deck, mesh, params
// ---------------------------------------------------------------------
extern "C" {

const char* pnt_status_string(pnt_status st) {
    switch (st) {
        case PNT_OK: return "ok";
        case PNT_ERR_INVALID_ARG: return "invalid argument";
        case PNT_ERR_DECK: return "malformed input deck";
        case PNT_ERR_BADSIDES: return "negative side volumes";
        case PNT_ERR_CUDA: return "CUDA error";
        case PNT_ERR_UNSUPPORTED: return "unsupported";
        case PNT_ERR_TIMEOUT: return "device wait timed out";
        case PNT_ERR_NOMEM: return "out of memory";
        case PNT_ERR_NO_DEVICE: return "no usable CUDA device";
        case PNT_ERR_STATE: return "invalid state";
        default: return "unknown status";
    }
}

const char* pnt_last_error(void) { return g_err.c_str(); }

int32_t pnt_abi_version(void) { return PNT_ABI_VERSION; }

pnt_status pnt_deck_parse(const char* text, pnt_deck** out) {
    if (!text || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    pnt_deck* d = new (std::nothrow) pnt_deck();
    if (!d) return fail(PNT_ERR_NOMEM, "out of memory");
    const pnt_status st = parse_deck(text, d->d);
    if (st) { delete d; return st; }
    *out = d;
    return PNT_OK;
}

pnt_status pnt_deck_load(const char* path, pnt_deck** out) {
    if (!path || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    std::ifstream ifs(path, std::ios::binary);
    if (!ifs.good()) return fail(PNT_ERR_DECK, "File %s not found", path);
    std::ostringstream ss;
    ss << ifs.rdbuf();
    return pnt_deck_parse(ss.str().c_str(), out);
}

pnt_status pnt_deck_set(pnt_deck* deck, const char* key, const char* value) {
    if (!deck || !key || !value || !key[0]) return fail(PNT_ERR_INVALID_ARG, "null argument");
    std::string v = std::string(" ") + value;
    for (auto& p : deck->d.kv)
        if (p.first == key) { p.second = v; return PNT_OK; }
    deck->d.kv.emplace_back(key, v);
    return PNT_OK;
}

int32_t pnt_deck_has(const pnt_deck* deck, const char* key) {
    return (deck && key && deck->d.find(key)) ? 1 : 0;
}

int32_t pnt_deck_get_int(const pnt_deck* deck, const char* key, int32_t dflt) {
    return (deck && key) ? get_int(deck->d, key, dflt) : dflt;
}

double pnt_deck_get_double(const pnt_deck* deck, const char* key, double dflt) {
    return (deck && key) ? get_double(deck->d, key, dflt) : dflt;
}

int32_t pnt_deck_get_string(const pnt_deck* deck, const char* key, const char* dflt, char* buf,
                            size_t buflen) {
    std::string v = (deck && key) ? get_string(deck->d, key, dflt ? dflt : "") : (dflt ? dflt : "");
    if (buf && buflen) {
        const size_t n = std::min(buflen - 1, v.size());
        memcpy(buf, v.data(), n);
        buf[n] = 0;
    }
    return (int32_t)v.size();
}

int32_t pnt_deck_get_double_list(const pnt_deck* deck, const char* key, double* out, int32_t maxn) {
    if (!deck || !key) return -1;
    std::vector<double> v;
    const int n = get_double_list(deck->d, key, v);
    for (int i = 0; i < n && i < maxn && out; ++i) out[i] = v[i];
    return n;
}

void pnt_deck_destroy(pnt_deck* deck) { delete deck; }

pnt_status pnt_mesh_generate(const pnt_deck* deck, pnt_mesh** out) {
    if (!deck || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    pnt_mesh* m = new (std::nothrow) pnt_mesh();
    if (!m) return fail(PNT_ERR_NOMEM, "out of memory");
    try {
        pnt_status st = generate_mesh(deck->d, m->m);
        if (!st) st = finish_mesh(m->m);
        if (st) { delete m; return st; }
    } catch (const std::bad_alloc&) {
        delete m;
        return fail(PNT_ERR_NOMEM, "out of host memory building the mesh");
    }
    *out = m;
    return PNT_OK;
}

pnt_status pnt_mesh_create(const pnt_mesh_desc* d, pnt_mesh** out) {
    if (!d || !out || !d->px || !d->znump || !d->mapsp1 || !d->mapsp2 || !d->mapsz || !d->mapss3 ||
        !d->mapss4)
        return fail(PNT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (d->nump <= 0 || d->numz <= 0 || d->nums <= 0) return fail(PNT_ERR_INVALID_ARG, "empty mesh");
    pnt_mesh* m = new (std::nothrow) pnt_mesh();
    if (!m) return fail(PNT_ERR_NOMEM, "out of memory");
    try {
        Mesh& g = m->m;
        g.nump = d->nump;
        g.numz = d->numz;
        g.nums = d->nums;
        g.px.assign(d->px, d->px + 2 * (size_t)d->nump);
        g.znump.assign(d->znump, d->znump + d->numz);
        g.mapsp1.assign(d->mapsp1, d->mapsp1 + d->nums);
        g.mapsp2.assign(d->mapsp2, d->mapsp2 + d->nums);
        g.mapsz.assign(d->mapsz, d->mapsz + d->nums);
        g.mapss3.assign(d->mapss3, d->mapss3 + d->nums);
        g.mapss4.assign(d->mapss4, d->mapss4 + d->nums);
        const pnt_status st = finish_mesh(g);
        if (st) { delete m; return st; }
    } catch (const std::bad_alloc&) {
        delete m;
        return fail(PNT_ERR_NOMEM, "out of host memory building the mesh");
    }
    *out = m;
    return PNT_OK;
}

pnt_status pnt_mesh_describe(const pnt_mesh* mesh, pnt_mesh_desc* out) {
    if (!mesh || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    const Mesh& g = mesh->m;
    out->nump = g.nump;
    out->numz = g.numz;
    out->nums = g.nums;
    out->px = g.px.data();
    out->znump = g.znump.data();
    out->mapsp1 = g.mapsp1.data();
    out->mapsp2 = g.mapsp2.data();
    out->mapsz = g.mapsz.data();
    out->mapss3 = g.mapss3.data();
    out->mapss4 = g.mapss4.data();
    return PNT_OK;
}

pnt_status pnt_mesh_point_corners(const pnt_mesh* mesh, const int32_t** offsets, const int32_t** sides) {
    if (!mesh || !offsets || !sides) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *offsets = mesh->m.poff.data();
    *sides = mesh->m.pcorner.data();
    return PNT_OK;
}

void pnt_mesh_destroy(pnt_mesh* mesh) { delete mesh; }

pnt_status pnt_mesh_piece(const pnt_mesh* mesh, int32_t npieces, int32_t piece, pnt_mesh** out) {
    if (!mesh || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    pnt_mesh* pm = new (std::nothrow) pnt_mesh();
    if (!pm) return fail(PNT_ERR_NOMEM, "out of memory");
    pnt_status st;
    try {
        st = make_piece(mesh->m, npieces, piece, pm->m);
    } catch (const std::bad_alloc&) {
        st = fail(PNT_ERR_NOMEM, "out of host memory building piece %d", piece);
    }
    if (st) {
        delete pm;
        return st;
    }
    *out = pm;
    return PNT_OK;
}

pnt_status pnt_mesh_piece_describe(const pnt_mesh* mesh, pnt_piece_desc* out) {
    if (!mesh || !out) return fail(PNT_ERR_INVALID_ARG, "null argument");
    const Mesh& m = mesh->m;
    out->piece = m.piece;
    out->npieces = m.npieces;
    out->zone0 = m.zone0;
    out->side0 = m.side0;
    out->gpoint = m.is_piece ? m.gpoint.data() : nullptr;
    out->nhalo = m.nhalo;
    out->halo_side = m.halo_side.data();
    out->nnbr = (int32_t)m.nbr.size();
    out->nbr = m.nbr.data();
    out->send_off = m.is_piece ? m.send_off.data() : nullptr;
    out->send_side = m.send_side.data();
    out->recv_off = m.is_piece ? m.recv_off.data() : nullptr;
    return PNT_OK;
}

pnt_status pnt_params_default(pnt_params* p) {
    if (!p) return fail(PNT_ERR_INVALID_ARG, "null argument");
    memset(p, 0, sizeof(*p));
    p->cstop = 999999;        // Driver.cc:78-87
    p->tstop = 1.e99;
    p->dtmax = 1.e99;
    p->dtinit = 1.e99;
    p->dtfac = 1.2;
    p->dtreport = 10;
    p->cfl = 0.6;             // Hydro.cc:206-212
    p->cflv = 0.1;
    p->rinit = 1.;
    p->einit = 0.;
    p->rinitsub = 1.;
    p->einitsub = 0.;
    p->uinitradial = 0.;
    p->gamma = 5. / 3.;       // PolyGas.cc:58-59
    p->pgas_ssmin = 0.;
    p->alfa = 0.5;            // TTS.cc:46-47
    p->tts_ssmin = 0.;
    p->qgamma = 5. / 3.;      // QCS.cc:84-86
    p->q1 = 0.;
    p->q2 = 2.;
    p->precision = PNT_PREC_FP64;
    p->graph_cycles = 0;
    return PNT_OK;
}

pnt_status pnt_params_from_deck(const pnt_deck* deck, pnt_params* p) {
    if (!deck || !p) return fail(PNT_ERR_INVALID_ARG, "null argument");
    pnt_params_default(p);
    const Deck& d = deck->d;
    p->cstop = get_int(d, "cstop", p->cstop);
    p->tstop = get_double(d, "tstop", p->tstop);
    if (p->cstop == 999999 && p->tstop == 1.e99)
        return fail(PNT_ERR_DECK, "Must specify either cstop or tstop");
    p->dtmax = get_double(d, "dtmax", p->dtmax);
    p->dtinit = get_double(d, "dtinit", p->dtinit);
    p->dtfac = get_double(d, "dtfac", p->dtfac);
    p->dtreport = get_int(d, "dtreport", p->dtreport);
    p->cfl = get_double(d, "cfl", p->cfl);
    p->cflv = get_double(d, "cflv", p->cflv);
    p->rinit = get_double(d, "rinit", p->rinit);
    p->einit = get_double(d, "einit", p->einit);
    p->rinitsub = get_double(d, "rinitsub", p->rinitsub);
    p->einitsub = get_double(d, "einitsub", p->einitsub);
    p->uinitradial = get_double(d, "uinitradial", p->uinitradial);
    std::vector<double> v;
    const int nsub = get_double_list(d, "subregion", v);
    if (nsub > 0 && nsub != 4) return fail(PNT_ERR_DECK, "subregion must have 4 entries");  // Mesh.cc:219-223
    p->has_subregion = (nsub == 4);
    for (int i = 0; i < 4 && p->has_subregion; ++i) p->subregion[i] = v[i];
    int n = get_double_list(d, "bcx", v);
    if (n > PNT_MAX_BC) return fail(PNT_ERR_UNSUPPORTED, "more than %d bcx planes", PNT_MAX_BC);
    p->nbcx = n < 0 ? 0 : n;
    for (int i = 0; i < p->nbcx; ++i) p->bcx[i] = v[i];
    n = get_double_list(d, "bcy", v);
    if (n > PNT_MAX_BC) return fail(PNT_ERR_UNSUPPORTED, "more than %d bcy planes", PNT_MAX_BC);
    p->nbcy = n < 0 ? 0 : n;
    for (int i = 0; i < p->nbcy; ++i) p->bcy[i] = v[i];
    if (p->nbcx + p->nbcy > PNT_MAX_BC)
        return fail(PNT_ERR_UNSUPPORTED, "more than %d boundary planes", PNT_MAX_BC);
    p->gamma = get_double(d, "gamma", p->gamma);
    p->pgas_ssmin = get_double(d, "ssmin", p->pgas_ssmin);
    p->alfa = get_double(d, "alfa", p->alfa);
    p->tts_ssmin = get_double(d, "ssmin", p->tts_ssmin);
    p->qgamma = get_double(d, "qgamma", p->qgamma);
    p->q1 = get_double(d, "q1", p->q1);
    p->q2 = get_double(d, "q2", p->q2);
    const std::string prec = get_string(d, "precision", "fp64");
    if (prec == "fp64") p->precision = PNT_PREC_FP64;
    else if (prec == "mixed") p->precision = PNT_PREC_MIXED;
    else if (prec == "learned") p->precision = PNT_PREC_LEARNED;
    else return fail(PNT_ERR_DECK, "precision must be fp64, mixed or learned");
    p->graph_cycles = get_int(d, "graphcycles", 0);
    return PNT_OK;
}

}  // extern "C"
