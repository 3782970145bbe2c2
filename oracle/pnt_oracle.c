/*
 * pnt_oracle.c -- CPU oracle for PENNANT's Lagrangian staggered-grid hydro
 * cycle (Hydro::doCycle).
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path and the
 * timed CPU baseline in bench.py.  Nothing in the product library links or
 * calls this file.
 *
 * It restates, in plain C and in the reference's serial task order, the
 * CPU task bodies of StanfordLegion/pennant-legion for a single mesh piece
 * (the reference's default `-n 1`).  Citations are file:line within that
 * project.  Every arithmetic expression keeps the reference's operation
 * order, including Vec2.hh's `operator/` (multiply by the reciprocal,
 * Vec2.hh:145-149), so a build with -ffp-contract=off gives the same bits
 * as the reference's own CPU build.
 *
 * Parity pin: reproduces test/sedov/sedov.xy (8 significant digits) and
 * sedov.geo coordinates (5 digits) -- tests/test_oracle_golden.py.
 *
 * With orc_set_threads(sim, n > 1) the loops run as the reference's
 * *OMPTask variants do (one `omp parallel for` per task, atomic updates
 * for the side-to-zone and side-to-point sums); that mode is
 * order-nondeterministic and serves only as the timed CPU baseline.
 */
#define _GNU_SOURCE
#include "pnt_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------ */
/* double2 helpers (Vec2.hh:80-205)                                    */
/* ------------------------------------------------------------------ */
typedef struct { double x, y; } d2;

static inline d2 mk(double x, double y) { d2 r; r.x = x; r.y = y; return r; }
static inline d2 add(d2 a, d2 b) { return mk(a.x + b.x, a.y + b.y); }
static inline d2 sub(d2 a, d2 b) { return mk(a.x - b.x, a.y - b.y); }
static inline d2 neg(d2 a) { return mk(-a.x, -a.y); }
/* r * v and v * r both evaluate (v.x * r, v.y * r) (Vec2.hh:131-142) */
static inline d2 smul(double r, d2 v) { return mk(v.x * r, v.y * r); }
/* v / r multiplies by the reciprocal (Vec2.hh:145-149) */
static inline d2 sdiv(d2 v, double r) { double rinv = 1. / r; return mk(v.x * rinv, v.y * rinv); }
static inline double dot(d2 a, d2 b) { return a.x * b.x + a.y * b.y; }
static inline double cross(d2 a, d2 b) { return a.x * b.y - a.y * b.x; }
static inline double length(d2 v) { return sqrt(v.x * v.x + v.y * v.y); }
static inline double length2(d2 v) { return v.x * v.x + v.y * v.y; }
static inline d2 rotateCCW(d2 v) { return mk(-v.y, v.x); }
/* project v onto the subspace perpendicular to unit u (Vec2.hh:196-201) */
static inline d2 project(d2 v, d2 u) { return sub(v, smul(dot(v, u), u)); }
/* std::min / std::max semantics: min(a,b) = (b < a) ? b : a */
static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static inline double dmax(double a, double b) { return (a < b) ? b : a; }

/* Atomic helpers for the OpenMP baseline mode (restating SumOp/MinOp/MaxOp
 * apply<false>, Mesh.hh:245-327). */
static inline void atom_add(int par, double* p, double v) {
    if (par) {
#pragma omp atomic
        *p += v;
    } else {
        *p += v;
    }
}
static inline void atom_min(int par, double* p, double v) {
    if (!par) { *p = dmin(*p, v); return; }
    double old;
    __atomic_load(p, &old, __ATOMIC_RELAXED);
    for (;;) {
        double nv = dmin(old, v);
        if (nv == old) return;
        if (__atomic_compare_exchange(p, &old, &nv, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
    }
}
static inline void atom_max(int par, double* p, double v) {
    if (!par) { *p = dmax(*p, v); return; }
    double old;
    __atomic_load(p, &old, __ATOMIC_RELAXED);
    for (;;) {
        double nv = dmax(old, v);
        if (nv == old) return;
        if (__atomic_compare_exchange(p, &old, &nv, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
    }
}

/* ------------------------------------------------------------------ */
/* Deck (InputFile.cc:24-104)                                          */
/* ------------------------------------------------------------------ */
typedef struct {
    int n, cap;
    char** keys;
    char** vals;
} deck_t;

static void deck_free(deck_t* d) {
    for (int i = 0; i < d->n; ++i) { free(d->keys[i]); free(d->vals[i]); }
    free(d->keys); free(d->vals);
    memset(d, 0, sizeof(*d));
}

static void seterr(char* err, size_t len, const char* fmt, ...) {
    if (!err || !len) return;
    va_list ap; va_start(ap, fmt); vsnprintf(err, len, fmt, ap); va_end(ap);
}

/* Parse deck text.  Like InputFile::InputFile, a final line that is not
 * terminated by a newline is dropped (getline hits EOF and the loop breaks,
 * InputFile.cc:36-37). */
static int deck_parse_text(const char* text, deck_t* d, char* err, size_t errlen) {
    memset(d, 0, sizeof(*d));
    const char* p = text;
    while (*p) {
        const char* eol = strchr(p, '\n');
        if (!eol) break;                       /* unterminated last line dropped */
        const char* q = p;
        while (q < eol && (*q == ' ' || *q == '\t' || *q == '\r' || *q == '\v' || *q == '\f')) ++q;
        const char* k0 = q;
        while (q < eol && !(*q == ' ' || *q == '\t' || *q == '\r' || *q == '\v' || *q == '\f')) ++q;
        size_t klen = (size_t)(q - k0);
        if (klen == 0 || k0[0] == '#') { p = eol + 1; continue; }
        for (int i = 0; i < d->n; ++i) {
            if (strlen(d->keys[i]) == klen && !strncmp(d->keys[i], k0, klen)) {
                seterr(err, errlen, "Duplicate key %.*s in input file", (int)klen, k0);
                deck_free(d);
                return ORC_ERR_DECK;
            }
        }
        if (d->n == d->cap) {
            d->cap = d->cap ? 2 * d->cap : 32;
            d->keys = (char**)realloc(d->keys, sizeof(char*) * d->cap);
            d->vals = (char**)realloc(d->vals, sizeof(char*) * d->cap);
        }
        d->keys[d->n] = strndup(k0, klen);
        d->vals[d->n] = strndup(q, (size_t)(eol - q));
        d->n++;
        p = eol + 1;
    }
    return ORC_OK;
}

static const char* deck_find(const deck_t* d, const char* key) {
    for (int i = 0; i < d->n; ++i)
        if (!strcmp(d->keys[i], key)) return d->vals[i];
    return NULL;
}
static double deck_double(const deck_t* d, const char* key, double dflt) {
    const char* v = deck_find(d, key);
    if (!v) return dflt;
    char* end; double x = strtod(v, &end);
    return (end == v) ? 0. : x;
}
static int deck_int(const deck_t* d, const char* key, int dflt) {
    const char* v = deck_find(d, key);
    if (!v) return dflt;
    char* end; long x = strtol(v, &end, 10);
    return (end == v) ? 0 : (int)x;
}
static int deck_list(const deck_t* d, const char* key, double* out, int maxn) {
    const char* v = deck_find(d, key);
    if (!v) return -1;
    int n = 0;
    const char* p = v;
    for (;;) {
        char* end; double x = strtod(p, &end);
        if (end == p) break;
        if (n < maxn) out[n] = x;
        ++n; p = end;
    }
    return n;
}
static int deck_string(const deck_t* d, const char* key, char* out, size_t len) {
    const char* v = deck_find(d, key);
    out[0] = 0;
    if (!v) return 0;
    while (*v == ' ' || *v == '\t') ++v;
    size_t n = 0;
    while (v[n] && v[n] != ' ' && v[n] != '\t' && v[n] != '\r' && n + 1 < len) { out[n] = v[n]; ++n; }
    out[n] = 0;
    return 1;
}

/* ------------------------------------------------------------------ */
/* Simulation state                                                    */
/* ------------------------------------------------------------------ */
#define ORC_MAXBC 16

struct orc_sim {
    /* Driver (Driver.cc:78-87) */
    int cstop, dtreport;
    double tstop, dtmax, dtinit, dtfac;
    /* Hydro (Hydro.cc:206-214) */
    double cfl, cflv, rinit, einit, rinitsub, einitsub, uinitradial;
    double subregion[4]; int has_subregion;
    /* PolyGas (PolyGas.cc:57-60), TTS (TTS.cc:45-48), QCS (QCS.cc:83-86) */
    double pgamma, pssmin, alfa, tssmin, qgamma, q1, q2;
    /* mesh */
    int meshtype; /* 0 rect, 1 pie */
    int nzx, nzy; double lenx, leny;
    int nump, numz, nums;
    int *znump, *mapsp1, *mapsp2, *mapsz, *mapss3, *mapss4;
    /* point fields */
    d2 *px, *pxp, *px0, *pu, *pu0, *pf, *pap; double* pmaswt;
    /* zone fields */
    d2 *zx, *zxp, *zuc;
    double *zarea, *zvol, *zareap, *zvolp, *zvol0, *zdl, *zm, *zr, *zrp, *ze,
           *zetot, *zw, *zwrate, *zp, *zss, *zdu, *ztmp;
    /* side / corner fields */
    d2 *ex, *expp, *ssurfp, *sfp, *sfq, *sft, *cqe1, *cqe2;
    double *sarea, *svol, *sareap, *svolp, *elen, *smf, *carea, *cevol, *cdu,
           *cdiv, *ccos, *crmu, *cw;
    /* boundary conditions (Hydro.cc:220-225): bcx then bcy */
    int nbc; d2 bcvfix[ORC_MAXBC]; double bcbound[ORC_MAXBC]; int bcxplane[ORC_MAXBC];
    int* bcpts[ORC_MAXBC]; int bcn[ORC_MAXBC];
    /* driver state */
    double time, dt, dtrec, dtnew, dvovmax;
    int cycle, done, nbad_last;
    int nthreads;
};

void orc_set_threads(orc_sim* s, int n) { s->nthreads = n; }

#define PAR (sim->nthreads > 1)
#define NT (sim->nthreads > 1 ? sim->nthreads : 1)

static void* xalloc(size_t n) { void* p = calloc(n ? n : 1, 1); return p; }

/* ------------------------------------------------------------------ */
/* Mesh generation, single piece (GenMesh.cc:790-873, 898-975,          */
/* 987-1282; calcNumPoints/Zones/Sides :485-528)                        */
/* ------------------------------------------------------------------ */
static int gen_mesh(orc_sim* sim, char* err, size_t errlen) {
    const int nzx = sim->nzx, nzy = sim->nzy;
    const int npx = nzx + 1, npy = nzy + 1;
    if (sim->meshtype == 0) {
        sim->nump = npx * npy;
        sim->numz = nzx * nzy;
        sim->nums = 4 * sim->numz;
    } else {
        sim->nump = npx * (npy - 1) + 1;
        sim->numz = nzx * nzy;
        sim->nums = 4 * nzx * (nzy - 1) + 3 * nzx;
    }
    const int np = sim->nump, nz = sim->numz, ns = sim->nums;
#define AL(f, T, n) sim->f = (T*)xalloc(sizeof(T) * (size_t)(n))
    AL(znump, int, nz);
    AL(mapsp1, int, ns); AL(mapsp2, int, ns); AL(mapsz, int, ns);
    AL(mapss3, int, ns); AL(mapss4, int, ns);
    AL(px, d2, np); AL(pxp, d2, np); AL(px0, d2, np); AL(pu, d2, np);
    AL(pu0, d2, np); AL(pf, d2, np); AL(pap, d2, np); AL(pmaswt, double, np);
    AL(zx, d2, nz); AL(zxp, d2, nz); AL(zuc, d2, nz);
    AL(zarea, double, nz); AL(zvol, double, nz); AL(zareap, double, nz);
    AL(zvolp, double, nz); AL(zvol0, double, nz); AL(zdl, double, nz);
    AL(zm, double, nz); AL(zr, double, nz); AL(zrp, double, nz);
    AL(ze, double, nz); AL(zetot, double, nz); AL(zw, double, nz);
    AL(zwrate, double, nz); AL(zp, double, nz); AL(zss, double, nz);
    AL(zdu, double, nz); AL(ztmp, double, nz);
    AL(ex, d2, ns); AL(expp, d2, ns); AL(ssurfp, d2, ns); AL(sfp, d2, ns);
    AL(sfq, d2, ns); AL(sft, d2, ns); AL(cqe1, d2, ns); AL(cqe2, d2, ns);
    AL(sarea, double, ns); AL(svol, double, ns); AL(sareap, double, ns);
    AL(svolp, double, ns); AL(elen, double, ns); AL(smf, double, ns);
    AL(carea, double, ns); AL(cevol, double, ns); AL(cdu, double, ns);
    AL(cdiv, double, ns); AL(ccos, double, ns); AL(crmu, double, ns);
    AL(cw, double, ns);
#undef AL
    if (!sim->cw) { seterr(err, errlen, "out of memory"); return ORC_ERR_NOMEM; }

    if (sim->meshtype == 0) {
        /* genPointsRect GenMesh.cc:790-829 (non-precompacted numbering) */
        const double dx = sim->lenx / (double)nzx;
        const double dy = sim->leny / (double)nzy;
        for (int p = 0; p < np; ++p) {
            const int i = p % npx, j = p / npx;
            sim->px[p] = mk(dx * (double)i, dy * (double)j);
        }
        /* generateZonesParallel fills ZNUMP with 4 (GenMesh.cc:571-578) */
        for (int z = 0; z < nz; ++z) sim->znump[z] = 4;
        /* genSidesRect GenMesh.cc:987-1100 */
        for (int s = 0; s < ns; ++s) {
            const int side = s % 4;
            sim->mapss3[s] = (side == 0) ? s + 3 : s - 1;
            sim->mapss4[s] = (side == 3) ? s - 3 : s + 1;
            const int z = s / 4;
            sim->mapsz[s] = z;
            const int zidx = z % nzx, zidy = z / nzx;
            int pidx1, pidx2, pidy1, pidy2;
            switch (side) {
            case 0: pidx1 = zidx; pidx2 = zidx + 1; pidy1 = zidy; pidy2 = zidy; break;
            case 1: pidx1 = zidx + 1; pidx2 = zidx + 1; pidy1 = zidy; pidy2 = zidy + 1; break;
            case 2: pidx1 = zidx + 1; pidx2 = zidx; pidy1 = zidy + 1; pidy2 = zidy + 1; break;
            default: pidx1 = zidx; pidx2 = zidx; pidy1 = zidy + 1; pidy2 = zidy; break;
            }
            sim->mapsp1[s] = pidy1 * (nzx + 1) + pidx1;
            sim->mapsp2[s] = pidy2 * (nzx + 1) + pidx2;
        }
    } else {
        /* genPointsPie GenMesh.cc:831-873 */
        const double dth = sim->lenx / (double)nzx;
        const double dr = sim->leny / (double)nzy;
        sim->px[0] = mk(0., 0.);
        for (int p = 1; p < np; ++p) {
            const int i = (p - 1) % npx, j = (p - 1) / npx + 1;
            const double th = dth * (double)(nzx - i);
            const double r = dr * (double)j;
            sim->px[p] = mk(r * cos(th), r * sin(th));
        }
        /* genZonesPie GenMesh.cc:932-975 */
        for (int z = 0; z < nz; ++z) sim->znump[z] = (z / nzx == 0) ? 3 : 4;
        /* genSidesPie GenMesh.cc:1102-1282, single piece */
        for (int s = 0; s < ns; ++s) {
            int z, side;
            if (s < 3 * nzx) { z = s / 3; side = s % 3; }
            else { z = nzx + (s - 3 * nzx) / 4; side = (s - 3 * nzx) % 4; }
            sim->mapsz[s] = z;
            const int zidx = z % nzx, zidy = z / nzx;
            if (zidy == 0) {
                sim->mapss3[s] = (side == 0) ? s + 2 : s - 1;
                sim->mapss4[s] = (side == 2) ? s - 2 : s + 1;
                const int p0 = zidx + 1;
                switch (side) {
                case 0: sim->mapsp1[s] = 0; sim->mapsp2[s] = p0 + 1; break;
                case 1: sim->mapsp1[s] = p0 + 1; sim->mapsp2[s] = p0; break;
                default: sim->mapsp1[s] = p0; sim->mapsp2[s] = 0; break;
                }
            } else {
                sim->mapss3[s] = (side == 0) ? s + 3 : s - 1;
                sim->mapss4[s] = (side == 3) ? s - 3 : s + 1;
                const int p0 = (zidy - 1) * npx + zidx + 1;
                switch (side) {
                case 0: sim->mapsp1[s] = p0; sim->mapsp2[s] = p0 + 1; break;
                case 1: sim->mapsp1[s] = p0 + 1; sim->mapsp2[s] = p0 + npx + 1; break;
                case 2: sim->mapsp1[s] = p0 + npx + 1; sim->mapsp2[s] = p0 + npx; break;
                default: sim->mapsp1[s] = p0 + npx; sim->mapsp2[s] = p0; break;
                }
            }
        }
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* Mesh geometry tasks (Mesh.cc)                                       */
/* ------------------------------------------------------------------ */
/* calcCtrsTask Mesh.cc:797-837 */
static void calc_ctrs(orc_sim* sim, const d2* px, d2* ex, d2* zx) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) zx[z] = mk(0., 0.);
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const int p1 = sim->mapsp1[s], p2 = sim->mapsp2[s], z = sim->mapsz[s];
        const d2 px1 = px[p1], px2 = px[p2];
        ex[s] = smul(0.5, add(px1, px2));
        const int n = sim->znump[z];
        const d2 t = sdiv(px1, (double)n);
        atom_add(par, &zx[z].x, t.x);
        atom_add(par, &zx[z].y, t.y);
    }
}

/* calcVolsTask Mesh.cc:928-989; returns the count of sides with sv <= 0 */
static int calc_vols(orc_sim* sim, const d2* px, const d2* zx, double* sarea,
                     double* svol, double* zarea, double* zvol) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) { zarea[z] = 0.; zvol[z] = 0.; }
    const double third = 1. / 3.;
    int count = 0;
#pragma omp parallel for num_threads(NT) if (par) schedule(static) reduction(+ : count)
    for (int s = 0; s < sim->nums; ++s) {
        const int p1 = sim->mapsp1[s], p2 = sim->mapsp2[s], z = sim->mapsz[s];
        const d2 px1 = px[p1], px2 = px[p2], zxz = zx[z];
        const double sa = 0.5 * cross(sub(px2, px1), sub(zxz, px1));
        const double sv = third * sa * (px1.x + px2.x + zxz.x);
        sarea[s] = sa;
        svol[s] = sv;
        atom_add(par, &zarea[z], sa);
        atom_add(par, &zvol[z], sv);
        if (sv <= 0.) count += 1;
    }
    return count;
}

/* calcSideFracsTask Mesh.cc:1085-1101 */
static void calc_side_fracs(orc_sim* sim) {
    for (int s = 0; s < sim->nums; ++s) sim->smf[s] = sim->sarea[s] / sim->zarea[sim->mapsz[s]];
}

/* calcSurfVecsTask Mesh.cc:1104-1123 */
static void calc_surf_vecs(orc_sim* sim) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s)
        sim->ssurfp[s] = rotateCCW(sub(sim->expp[s], sim->zxp[sim->mapsz[s]]));
}

/* calcEdgeLenTask Mesh.cc:1151-1179 */
static void calc_edge_len(orc_sim* sim) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s)
        sim->elen[s] = length(sub(sim->pxp[sim->mapsp2[s]], sim->pxp[sim->mapsp1[s]]));
}

/* calcCharLenTask Mesh.cc:1216-1244 */
static void calc_char_len(orc_sim* sim) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) sim->zdl[z] = 1.e99;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const int z = sim->mapsz[s];
        const double area = sim->sareap[s];
        const double base = sim->elen[s];
        const int np = sim->znump[z];
        const double fac = (np == 3 ? 3. : 4.);
        const double sdl = fac * area / base;
        atom_min(par, &sim->zdl[z], sdl);
    }
}

/* ------------------------------------------------------------------ */
/* Hydro tasks (Hydro.cc:986-1807)                                     */
/* ------------------------------------------------------------------ */
/* calcRhoTask Hydro.cc:1034-1054 */
static void calc_rho(orc_sim* sim, const double* zvol, double* zr) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) zr[z] = sim->zm[z] / zvol[z];
}

/* calcCrnrMassTask Hydro.cc:1083-1117 */
static void calc_crnr_mass(orc_sim* sim) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const int s3 = sim->mapss3[s], z = sim->mapsz[s], p = sim->mapsp1[s];
        const double r = sim->zrp[z];
        const double area = sim->zareap[z];
        const double mf = sim->smf[s];
        const double mf3 = sim->smf[s3];
        const double mwt = r * area * 0.5 * (mf + mf3);
        atom_add(par, &sim->pmaswt[p], mwt);
    }
}

/* PolyGas::calcStateHalfTask PolyGas.cc:63-109 */
static void calc_state_half(orc_sim* sim, double dt) {
    const int par = PAR;
    const double gamma = sim->pgamma, ssmin = sim->pssmin;
    const double dth = 0.5 * dt;
    const double gm1 = gamma - 1.;
    const double ssmin2 = dmax(ssmin * ssmin, 1.e-99);
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) {
        const double r = sim->zr[z];
        const double e = dmax(sim->ze[z], 0.);
        const double p = gm1 * r * e;
        const double pre = gm1 * e;
        const double per = gm1 * r;
        const double csqd = dmax(ssmin2, pre + per * p / (r * r));
        const double ss = sqrt(csqd);
        const double minv = 1. / sim->zm[z];
        const double volp = sim->zvolp[z];
        const double vol0 = sim->zvol0[z];
        const double wrate = sim->zwrate[z];
        const double dv = (volp - vol0) * minv;
        const double bulk = r * csqd;
        const double denom = 1. + 0.5 * per * dv;
        const double src = wrate * dth * minv;
        sim->zp[z] = p + (per * src - r * bulk * dv) / denom;
        sim->zss[z] = ss;
    }
}

/* PolyGas::calcForceTask PolyGas.cc:164-184 */
static void calc_force_pgas(orc_sim* sim) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const double p = sim->zp[sim->mapsz[s]];
        sim->sfp[s] = smul(-p, sim->ssurfp[s]);
    }
}

/* TTS::calcForceTask TTS.cc:55-104 */
static void calc_force_tts(orc_sim* sim) {
    const int par = PAR;
    const double alfa = sim->alfa, ssmin = sim->tssmin;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const int z = sim->mapsz[s];
        const double sarea = sim->sareap[s];
        const double zarea = sim->zareap[z];
        const double vfacinv = zarea / sarea;
        const double r = sim->zrp[z];
        const double mf = sim->smf[s];
        const double srho = r * mf * vfacinv;
        const double ss = sim->zss[z];
        double sstmp = dmax(ss, ssmin);
        sstmp = alfa * sstmp * sstmp;
        const double sdp = sstmp * (srho - r);
        sim->sft[s] = smul(-sdp, sim->ssurfp[s]);
    }
}

/* QCS::setCornerDivTask QCS.cc:116-242 */
static void qcs_set_corner_div(orc_sim* sim) {
    const int par = PAR;
    const d2* pu = sim->pu0;
    const d2* px = sim->pxp;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) sim->zuc[z] = mk(0., 0.);
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const int p = sim->mapsp1[s], z = sim->mapsz[s];
        const int n = sim->znump[z];
        const d2 t = sdiv(pu[p], (double)n);
        if (par) {
            atom_add(par, &sim->zuc[z].x, t.x);
            atom_add(par, &sim->zuc[z].y, t.y);
        } else {
            sim->zuc[z] = add(sim->zuc[z], t);
        }
    }
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int c = 0; c < sim->nums; ++c) {
        const int s2 = c;
        const int s = sim->mapss3[s2];
        const int z = sim->mapsz[s];
        const int p = sim->mapsp2[s];
        const int p1 = sim->mapsp1[s];
        const int p2 = sim->mapsp2[s2];
        const d2 up0 = pu[p];
        const d2 xp0 = px[p];
        const d2 up1 = smul(0.5, add(up0, pu[p2]));
        const d2 xp1 = sim->expp[s2];
        const d2 up2 = sim->zuc[z];
        const d2 xp2 = sim->zxp[z];
        const d2 up3 = smul(0.5, add(pu[p1], up0));
        const d2 xp3 = sim->expp[s];
        double cvolume = 0.5 * cross(sub(xp2, xp0), sub(xp3, xp1));
        sim->carea[c] = cvolume;
        const d2 v1 = sub(xp3, xp0);
        const d2 v2 = sub(xp1, xp0);
        const double de1 = sim->elen[s];
        const double de2 = sim->elen[s2];
        const double minelen = dmin(de1, de2);
        const double ccos = ((minelen < 1.e-12) ? 0. : 4. * dot(v1, v2) / (de1 * de2));
        sim->ccos[c] = ccos;
        const double cdiv = (cross(sub(up2, up0), sub(xp3, xp1)) -
                             cross(sub(up3, up1), sub(xp2, xp0))) / (2.0 * cvolume);
        sim->cdiv[c] = cdiv;
        const d2 dxx1 = smul(0.5, sub(sub(add(xp1, xp2), xp0), xp3));
        const d2 dxx2 = smul(0.5, sub(sub(add(xp2, xp3), xp0), xp1));
        const double dx1 = length(dxx1);
        const double dx2 = length(dxx2);
        const d2 duav = smul(0.25, add(add(add(up0, up1), up2), up3));
        const double test1 = fabs(dot(dxx1, duav) * dx2);
        const double test2 = fabs(dot(dxx2, duav) * dx1);
        const double num = (test1 > test2 ? dx1 : dx2);
        const double den = (test1 > test2 ? dx2 : dx1);
        const double r = num / den;
        double evol = sqrt(4.0 * cvolume * r);
        evol = dmin(evol, 2.0 * minelen);
        const double dv1 = length2(sub(sub(add(up1, up2), up0), up3));
        const double dv2 = length2(sub(sub(add(up2, up3), up0), up1));
        double du = sqrt(dmax(dv1, dv2));
        evol = (cdiv < 0.0 ? evol : 0.);
        du = (cdiv < 0.0 ? du : 0.);
        sim->cevol[c] = evol;
        sim->cdu[c] = du;
    }
}

/* QCS::setQCnForceTask QCS.cc:246-327 */
static void qcs_set_qcn_force(orc_sim* sim) {
    const int par = PAR;
    const double gammap1 = sim->qgamma + 1.0;
    const double q1 = sim->q1, q2 = sim->q2;
    const d2* pu = sim->pu0;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int c = 0; c < sim->nums; ++c) {
        const int z = sim->mapsz[c];
        const double cdu = sim->cdu[c];
        const double ztmp2 = q2 * 0.25 * gammap1 * cdu;
        const double zss = sim->zss[z];
        const double ztmp1 = q1 * zss;
        const double zkur = ztmp2 + sqrt(ztmp2 * ztmp2 + ztmp1 * ztmp1);
        const double zrp = sim->zrp[z];
        const double cevol = sim->cevol[c];
        const double crmu = zkur * zrp * cevol;
        const double cdiv = sim->cdiv[c];
        sim->crmu[c] = ((cdiv > 0.0) ? 0. : crmu);
    }
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int c = 0; c < sim->nums; ++c) {
        const int s2 = c;
        const int s = sim->mapss3[s2];
        const int p = sim->mapsp2[s];
        const int p1 = sim->mapsp1[s];
        const int p2 = sim->mapsp2[s2];
        const double crmu = sim->crmu[c];
        const d2 pc = pu[p];
        const d2 pu1 = pu[p1];
        const double elen = sim->elen[s];
        sim->cqe1[c] = sdiv(smul(crmu, sub(pc, pu1)), elen);
        const d2 pu2 = pu[p2];
        const double elen2 = sim->elen[s2];
        sim->cqe2[c] = sdiv(smul(crmu, sub(pu2, pc)), elen2);
    }
}

/* QCS::setForceTask QCS.cc:331-380 */
static void qcs_set_force(orc_sim* sim) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int c = 0; c < sim->nums; ++c) {
        const double ccos = sim->ccos[c];
        const double csin2 = 1.0 - ccos * ccos;
        const double carea = sim->carea[c];
        const double cw = ((csin2 < 1.e-4) ? 0. : carea / csin2);
        sim->cw[c] = cw;
        sim->ccos[c] = ((csin2 < 1.e-4) ? 0. : ccos);
    }
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const int c1 = s;
        const int c2 = sim->mapss4[s];
        const double el = sim->elen[s];
        const double cw1 = sim->cw[c1], cw2 = sim->cw[c2];
        const double ccos1 = sim->ccos[c1], ccos2 = sim->ccos[c2];
        const d2 cqe11 = sim->cqe1[c1], cqe12 = sim->cqe1[c2];
        const d2 cqe21 = sim->cqe2[c1], cqe22 = sim->cqe2[c2];
        const d2 t1 = smul(cw1, add(cqe21, smul(ccos1, cqe11)));
        const d2 t2 = smul(cw2, add(cqe12, smul(ccos2, cqe22)));
        sim->sfq[s] = sdiv(add(t1, t2), el);
    }
}

/* QCS::setVelDiffTask QCS.cc:384-448 */
static void qcs_set_vel_diff(orc_sim* sim) {
    const int par = PAR;
    const double q1 = sim->q1, q2 = sim->q2;
    const d2* pu = sim->pu0;
    const d2* px = sim->pxp;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) sim->ztmp[z] = 0.;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const int p1 = sim->mapsp1[s], p2 = sim->mapsp2[s], z = sim->mapsz[s];
        const d2 dx = sub(px[p2], px[p1]);
        const d2 du = sub(pu[p2], pu[p1]);
        const double lenx = sim->elen[s];
        double dux = dot(du, dx);
        dux = (lenx > 0. ? fabs(dux) / lenx : 0.);
        atom_max(par, &sim->ztmp[z], dux);
    }
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z)
        sim->zdu[z] = q1 * sim->zss[z] + 2. * q2 * sim->ztmp[z];
}

/* sumCrnrForceTask Hydro.cc:1159-1193 */
static void sum_crnr_force(orc_sim* sim) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const int s3 = sim->mapss3[s], p = sim->mapsp1[s];
        const d2 cf = sub(add(add(sim->sfp[s], sim->sfq[s]), sim->sft[s]),
                          add(add(sim->sfp[s3], sim->sfq[s3]), sim->sft[s3]));
        atom_add(par, &sim->pf[p].x, cf.x);
        atom_add(par, &sim->pf[p].y, cf.y);
    }
}

/* HydroBC::applyFixedBCTask HydroBC.cc:150-182 */
static void apply_fixed_bc(orc_sim* sim, int b) {
    const int par = PAR;
    const d2 vfix = sim->bcvfix[b];
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int i = 0; i < sim->bcn[b]; ++i) {
        const int p = sim->bcpts[b][i];
        sim->pu0[p] = project(sim->pu0[p], vfix);
        sim->pf[p] = project(sim->pf[p], vfix);
    }
}

/* calcAccelTask Hydro.cc:1235-1254 */
static void calc_accel(orc_sim* sim) {
    const int par = PAR;
    const double fuzz = 1.e-99;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int p = 0; p < sim->nump; ++p)
        sim->pap[p] = sdiv(sim->pf[p], dmax(sim->pmaswt[p], fuzz));
}

/* advPosFullTask Hydro.cc:1281-1306 */
static void adv_pos_full(orc_sim* sim, double dt) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int p = 0; p < sim->nump; ++p) {
        const d2 x0 = sim->px0[p], u0 = sim->pu0[p], a = sim->pap[p];
        const d2 u = add(u0, smul(dt, a));
        sim->pu[p] = u;
        sim->px[p] = add(x0, smul(dt * 0.5, add(u0, u)));
    }
}

/* calcWorkTask Hydro.cc:1339-1406 */
static void calc_work(orc_sim* sim, double dt) {
    const int par = PAR;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) sim->zw[z] = 0.;
    const double dth = 0.5 * dt;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int s = 0; s < sim->nums; ++s) {
        const int p1 = sim->mapsp1[s], p2 = sim->mapsp2[s], z = sim->mapsz[s];
        const d2 sftot = add(sim->sfp[s], sim->sfq[s]);
        const double sd1 = dot(sftot, add(sim->pu0[p1], sim->pu[p1]));
        const double sd2 = dot(neg(sftot), add(sim->pu0[p2], sim->pu[p2]));
        const d2 px1 = sim->pxp[p1], px2 = sim->pxp[p2];
        const double dwork = -dth * (sd1 * px1.x + sd2 * px2.x);
        atom_add(par, &sim->zetot[z], dwork);
        atom_add(par, &sim->zw[z], dwork);
    }
}

/* calcWorkRateTask Hydro.cc:1483-1510 */
static void calc_work_rate(orc_sim* sim, double dt) {
    const int par = PAR;
    const double dtinv = 1. / dt;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) {
        const double dvol = sim->zvol[z] - sim->zvol0[z];
        sim->zwrate[z] = (sim->zw[z] + sim->zp[z] * dvol) * dtinv;
    }
}

/* calcEnergyTask Hydro.cc:1545-1564 */
static void calc_energy(orc_sim* sim) {
    const int par = PAR;
    const double fuzz = 1.e-99;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int z = 0; z < sim->numz; ++z) sim->ze[z] = sim->zetot[z] / (sim->zm[z] + fuzz);
}

/* calcDtNewTask Hydro.cc:1591-1619 (OMP: :1670-1704) */
static double calc_dt_new(orc_sim* sim) {
    const int par = PAR;
    const double fuzz = 1.e-99, cfl = sim->cfl;
    double dtnew = 1.e99;
#pragma omp parallel num_threads(NT) if (par)
    {
        double local = 1.e99;
#pragma omp for schedule(static)
        for (int z = 0; z < sim->numz; ++z) {
            const double cdu = dmax(sim->zdu[z], dmax(sim->zss[z], fuzz));
            const double zdthyd = sim->zdl[z] * cfl / cdu;
            local = (zdthyd < local ? zdthyd : local);
        }
#pragma omp critical
        dtnew = (local < dtnew ? local : dtnew);
    }
    return dtnew;
}

/* calcDvolTask Hydro.cc:1622-1644 (OMP: :1707-1735) */
static double calc_dvol(orc_sim* sim) {
    const int par = PAR;
    double dvovmax = 1.e-99;
#pragma omp parallel num_threads(NT) if (par)
    {
        double local = 1.e-99;
#pragma omp for schedule(static)
        for (int z = 0; z < sim->numz; ++z) {
            const double zdvov = fabs((sim->zvol[z] - sim->zvol0[z]) / sim->zvol0[z]);
            local = (zdvov > local ? zdvov : local);
        }
#pragma omp critical
        dvovmax = (local > dvovmax ? local : dvovmax);
    }
    return dvovmax;
}

/* calcDtTask Hydro.cc:1647-1667 */
static double calc_dt(double dtlast, double dtnew, double dvovmax, double cflv) {
    double dtrec = 1.e99;
    if (dtnew < dtrec) dtrec = dtnew;
    const double dtnew2 = dtlast * cflv / dvovmax;
    if (dtnew2 < dtrec) dtrec = dtnew2;
    return dtrec;
}

/* Hydro::doCycle Hydro.cc:342-983.  Returns the bad-side count of the
 * first check that fails (predictor :801, corrector :980), else 0. */
static int do_cycle(orc_sim* sim, double dt) {
    const int par = PAR;
    const int np = sim->nump, nz = sim->numz;
    /* copies and fills :361-418; advPosHalf :986-1006 */
    memcpy(sim->zvol0, sim->zvol, sizeof(double) * (size_t)nz);
    const double dth = 0.5 * dt;
#pragma omp parallel for num_threads(NT) if (par) schedule(static)
    for (int p = 0; p < np; ++p) {
        sim->px0[p] = sim->px[p];
        sim->pu0[p] = sim->pu[p];
        sim->pmaswt[p] = 0.;
        sim->pf[p] = mk(0., 0.);
        sim->pxp[p] = add(sim->px0[p], smul(dth, sim->pu0[p]));
    }
    /* predictor geometry :439-542 */
    calc_ctrs(sim, sim->pxp, sim->expp, sim->zxp);
    const int nbadp = calc_vols(sim, sim->pxp, sim->zxp, sim->sareap, sim->svolp,
                                sim->zareap, sim->zvolp);
    calc_surf_vecs(sim);
    calc_edge_len(sim);
    calc_char_len(sim);
    calc_rho(sim, sim->zvolp, sim->zrp);        /* :544-554 */
    calc_crnr_mass(sim);                        /* :556-576 */
    calc_state_half(sim, dt);                   /* :578-596 */
    calc_force_pgas(sim);                       /* :598-611 */
    calc_force_tts(sim);                        /* :613-632 */
    qcs_set_corner_div(sim);                    /* :634-669 */
    qcs_set_qcn_force(sim);                     /* :671-703 */
    qcs_set_force(sim);                         /* :705-722 */
    qcs_set_vel_diff(sim);                      /* :724-752 */
    sum_crnr_force(sim);                        /* :754-771 */
    for (int b = 0; b < sim->nbc; ++b) apply_fixed_bc(sim, b);  /* :773-798 */
    if (nbadp > 0) { sim->nbad_last = nbadp; return nbadp; }     /* :801 */
    calc_accel(sim);                            /* :803-833 */
    adv_pos_full(sim, dt);                      /* :835-858 */
    /* corrector geometry :860-883 */
    calc_ctrs(sim, sim->px, sim->ex, sim->zx);
    const int nbadc = calc_vols(sim, sim->px, sim->zx, sim->sarea, sim->svol,
                                sim->zarea, sim->zvol);
    calc_work(sim, dt);                         /* :885-914 */
    calc_work_rate(sim, dt);                    /* :916-928 */
    calc_energy(sim);                           /* :930-940 */
    calc_rho(sim, sim->zvol, sim->zr);          /* :942-950 */
    sim->dtnew = calc_dt_new(sim);              /* :952-961 */
    sim->dvovmax = calc_dvol(sim);              /* :963-970 */
    sim->dtrec = calc_dt(dt, sim->dtnew, sim->dvovmax, sim->cflv);  /* :972-977 */
    if (nbadc > 0) { sim->nbad_last = nbadc; return nbadc; }     /* :980 */
    return 0;
}

/* Driver::calcGlobalDtTask Driver.cc:213-245 */
static double calc_global_dt(const orc_sim* sim) {
    double dt = sim->dtmax;
    if (sim->cycle == 0) {
        if (sim->dtinit < dt) dt = sim->dtinit;
    } else {
        const double dtrecover = sim->dtfac * sim->dt;
        if (dtrecover < dt) dt = dtrecover;
    }
    if ((sim->tstop - sim->time) < dt) dt = sim->tstop - sim->time;
    if (sim->cycle > 0) {
        if (sim->dtrec < dt) dt = sim->dtrec;
    }
    return dt;
}

/* One iteration of Driver::run (Driver.cc:127-145), stopping as the
 * predicated build does (Driver.cc:140-144, :300-307): no further cycle
 * once cycle >= cstop or time >= tstop. */
int orc_cycle(orc_sim* sim) {
    if (sim->done) return ORC_OK;
    sim->dt = calc_global_dt(sim);
    const int nbad = do_cycle(sim, sim->dt);
    if (nbad > 0) { sim->done = 1; return ORC_ERR_BADSIDES; }
    sim->time = sim->time + sim->dt;
    sim->cycle += 1;
    if (sim->cycle >= sim->cstop || !(sim->time < sim->tstop)) sim->done = 1;
    return ORC_OK;
}

int orc_run(orc_sim* sim, int max_cycles) {
    int n = 0;
    while (!sim->done && (max_cycles <= 0 || n < max_cycles)) {
        const int st = orc_cycle(sim);
        if (st) return st;
        ++n;
    }
    return ORC_OK;
}

int orc_done(const orc_sim* sim) { return sim->done; }

/* ------------------------------------------------------------------ */
/* Construction: Driver ctor (Driver.cc:65-93), Mesh::init              */
/* (Mesh.cc:249-652), Hydro ctor + init (Hydro.cc:200-339), HydroBC     */
/* point lists (HydroBC.cc:63-144, 222-326)                             */
/* ------------------------------------------------------------------ */
static int build(orc_sim* sim, const deck_t* d, char* err, size_t errlen) {
    sim->cstop = deck_int(d, "cstop", 999999);
    sim->tstop = deck_double(d, "tstop", 1.e99);
    if (sim->cstop == 999999 && sim->tstop == 1.e99) {
        seterr(err, errlen, "Must specify either cstop or tstop");
        return ORC_ERR_DECK;
    }
    sim->dtmax = deck_double(d, "dtmax", 1.e99);
    sim->dtinit = deck_double(d, "dtinit", 1.e99);
    sim->dtfac = deck_double(d, "dtfac", 1.2);
    sim->dtreport = deck_int(d, "dtreport", 10);

    double sub[8];
    const int nsub = deck_list(d, "subregion", sub, 8);
    if (nsub > 0 && nsub != 4) {
        seterr(err, errlen, "subregion must have 4 entries");
        return ORC_ERR_DECK;
    }
    sim->has_subregion = (nsub == 4);
    for (int i = 0; i < 4 && sim->has_subregion; ++i) sim->subregion[i] = sub[i];

    /* GenMesh ctor GenMesh.cc:87-129 */
    char mt[64];
    deck_string(d, "meshtype", mt, sizeof(mt));
    if (!mt[0]) { seterr(err, errlen, "must specify meshtype"); return ORC_ERR_DECK; }
    if (!strcmp(mt, "rect")) sim->meshtype = 0;
    else if (!strcmp(mt, "pie")) sim->meshtype = 1;
    else if (!strcmp(mt, "hex")) {
        seterr(err, errlen, "meshtype hex is not generated by the reference's parallel mesh generator");
        return ORC_ERR_UNSUPPORTED;
    } else { seterr(err, errlen, "invalid meshtype %s", mt); return ORC_ERR_DECK; }
    double mp[8];
    const int nmp = deck_list(d, "meshparams", mp, 8);
    if (nmp <= 0) { seterr(err, errlen, "must specify meshparams"); return ORC_ERR_DECK; }
    if (nmp > 4) { seterr(err, errlen, "meshparams must have <= 4 values"); return ORC_ERR_DECK; }
    sim->nzx = (int)mp[0];
    sim->nzy = (nmp >= 2 ? (int)mp[1] : sim->nzx);
    if (sim->meshtype != 1) sim->lenx = (nmp >= 3 ? mp[2] : 1.0);
    else sim->lenx = (nmp >= 3 ? mp[2] : 90.0) * M_PI / 180.0;
    sim->leny = (nmp >= 4 ? mp[3] : 1.0);
    if (sim->nzx <= 0 || sim->nzy <= 0 || sim->lenx <= 0. || sim->leny <= 0.) {
        seterr(err, errlen, "meshparams values must be positive");
        return ORC_ERR_DECK;
    }
    if (sim->meshtype == 1 && sim->lenx >= 2. * M_PI) {
        seterr(err, errlen, "meshparams theta must be < 360");
        return ORC_ERR_DECK;
    }
    int st = gen_mesh(sim, err, errlen);
    if (st) return st;

    /* Mesh::init initial geometry Mesh.cc:619-623 */
    calc_ctrs(sim, sim->px, sim->ex, sim->zx);
    const int nbad = calc_vols(sim, sim->px, sim->zx, sim->sarea, sim->svol, sim->zarea, sim->zvol);
    if (nbad > 0) {
        seterr(err, errlen, "%d negative side volumes during initialization", nbad);
        return ORC_ERR_BADSIDES;
    }
    calc_side_fracs(sim);

    /* Hydro ctor Hydro.cc:206-225 */
    sim->cfl = deck_double(d, "cfl", 0.6);
    sim->cflv = deck_double(d, "cflv", 0.1);
    sim->rinit = deck_double(d, "rinit", 1.);
    sim->einit = deck_double(d, "einit", 0.);
    sim->rinitsub = deck_double(d, "rinitsub", 1.);
    sim->einitsub = deck_double(d, "einitsub", 0.);
    sim->uinitradial = deck_double(d, "uinitradial", 0.);
    sim->pgamma = deck_double(d, "gamma", 5. / 3.);
    sim->pssmin = deck_double(d, "ssmin", 0.);
    sim->alfa = deck_double(d, "alfa", 0.5);
    sim->tssmin = deck_double(d, "ssmin", 0.);
    sim->qgamma = deck_double(d, "qgamma", 5. / 3.);
    sim->q1 = deck_double(d, "q1", 0.);
    sim->q2 = deck_double(d, "q2", 2.);
    double bcx[ORC_MAXBC], bcy[ORC_MAXBC];
    int nbcx = deck_list(d, "bcx", bcx, ORC_MAXBC);
    int nbcy = deck_list(d, "bcy", bcy, ORC_MAXBC);
    if (nbcx < 0) nbcx = 0;
    if (nbcy < 0) nbcy = 0;
    if (nbcx + nbcy > ORC_MAXBC) { seterr(err, errlen, "too many boundary planes"); return ORC_ERR_UNSUPPORTED; }
    sim->nbc = 0;
    for (int i = 0; i < nbcx; ++i) {
        sim->bcvfix[sim->nbc] = mk(1., 0.); sim->bcbound[sim->nbc] = bcx[i];
        sim->bcxplane[sim->nbc] = 1; sim->nbc++;
    }
    for (int i = 0; i < nbcy; ++i) {
        sim->bcvfix[sim->nbc] = mk(0., 1.); sim->bcbound[sim->nbc] = bcy[i];
        sim->bcxplane[sim->nbc] = 0; sim->nbc++;
    }
    /* HydroBC point lists: private points in ascending order whose
     * coordinate is within 1e-12 of the plane (HydroBC.cc:222-326) */
    const double eps = 1.e-12;
    for (int b = 0; b < sim->nbc; ++b) {
        int cnt = 0;
        for (int p = 0; p < sim->nump; ++p) {
            const double c = sim->bcxplane[b] ? sim->px[p].x : sim->px[p].y;
            if (fabs(c - sim->bcbound[b]) < eps) ++cnt;
        }
        sim->bcpts[b] = (int*)xalloc(sizeof(int) * (size_t)cnt);
        sim->bcn[b] = 0;
        for (int p = 0; p < sim->nump; ++p) {
            const double c = sim->bcxplane[b] ? sim->px[p].x : sim->px[p].y;
            if (fabs(c - sim->bcbound[b]) < eps) sim->bcpts[b][sim->bcn[b]++] = p;
        }
    }

    /* Hydro::init Hydro.cc:241-339 */
    for (int z = 0; z < sim->numz; ++z) {
        sim->zr[z] = sim->rinit;
        sim->ze[z] = sim->einit;
        sim->zwrate[z] = 0.;
    }
    if (sim->has_subregion) {   /* initSubrgnTask Hydro.cc:1738-1762 */
        const double* sr = sim->subregion;
        for (int z = 0; z < sim->numz; ++z) {
            const d2 zx = sim->zx[z];
            if (zx.x > (sr[0] - eps) && zx.x < (sr[1] + eps) &&
                zx.y > (sr[2] - eps) && zx.y < (sr[3] + eps)) {
                sim->zr[z] = sim->rinitsub;
                sim->ze[z] = sim->einitsub;
            }
        }
    }
    for (int z = 0; z < sim->numz; ++z) {   /* initHydroTask Hydro.cc:1765-1784 */
        const double zm = sim->zr[z] * sim->zvol[z];
        sim->zm[z] = zm;
        sim->zetot[z] = sim->ze[z] * zm;
    }
    if (sim->uinitradial != 0.) {   /* initRadialVelTask Hydro.cc:1787-1807 */
        for (int p = 0; p < sim->nump; ++p) {
            const d2 x = sim->px[p];
            const double pmag = length(x);
            if (pmag > eps) sim->pu[p] = sdiv(smul(sim->uinitradial, x), pmag);
            else sim->pu[p] = mk(0., 0.);
        }
    } else {
        for (int p = 0; p < sim->nump; ++p) sim->pu[p] = mk(0., 0.);
    }
    sim->time = 0.; sim->cycle = 0; sim->dt = 0.; sim->dtrec = 0.;
    sim->done = (sim->cstop <= 0) || !(sim->time < sim->tstop);
    return ORC_OK;
}

static char* read_file(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char* buf = (char*)malloc((size_t)n + 1);
    if (!buf) { fclose(f); return NULL; }
    size_t got = fread(buf, 1, (size_t)n, f);
    buf[got] = 0;
    fclose(f);
    return buf;
}

int orc_create(const char* path, const char* text, orc_sim** out, char* err, size_t errlen) {
    if (!out || (!path && !text)) return ORC_ERR_ARG;
    *out = NULL;
    char* owned = NULL;
    if (!text) {
        owned = read_file(path);
        if (!owned) { seterr(err, errlen, "File %s not found", path); return ORC_ERR_DECK; }
        text = owned;
    }
    deck_t d;
    int st = deck_parse_text(text, &d, err, errlen);
    free(owned);
    if (st) return st;
    orc_sim* sim = (orc_sim*)xalloc(sizeof(orc_sim));
    sim->nthreads = 1;
    st = build(sim, &d, err, errlen);
    deck_free(&d);
    if (st) { orc_destroy(sim); return st; }
    *out = sim;
    return ORC_OK;
}

void orc_destroy(orc_sim* sim) {
    if (!sim) return;
    void* arrs[] = {
        sim->znump, sim->mapsp1, sim->mapsp2, sim->mapsz, sim->mapss3, sim->mapss4,
        sim->px, sim->pxp, sim->px0, sim->pu, sim->pu0, sim->pf, sim->pap, sim->pmaswt,
        sim->zx, sim->zxp, sim->zuc, sim->zarea, sim->zvol, sim->zareap, sim->zvolp,
        sim->zvol0, sim->zdl, sim->zm, sim->zr, sim->zrp, sim->ze, sim->zetot, sim->zw,
        sim->zwrate, sim->zp, sim->zss, sim->zdu, sim->ztmp,
        sim->ex, sim->expp, sim->ssurfp, sim->sfp, sim->sfq, sim->sft, sim->cqe1, sim->cqe2,
        sim->sarea, sim->svol, sim->sareap, sim->svolp, sim->elen, sim->smf, sim->carea,
        sim->cevol, sim->cdu, sim->cdiv, sim->ccos, sim->crmu, sim->cw};
    for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); ++i) free(arrs[i]);
    for (int b = 0; b < sim->nbc; ++b) free(sim->bcpts[b]);
    free(sim);
}

/* ------------------------------------------------------------------ */
/* Accessors                                                           */
/* ------------------------------------------------------------------ */
int64_t orc_num(const orc_sim* sim, const char* w) {
    if (!strcmp(w, "nump")) return sim->nump;
    if (!strcmp(w, "numz")) return sim->numz;
    if (!strcmp(w, "nums")) return sim->nums;
    if (!strcmp(w, "cycle")) return sim->cycle;
    if (!strcmp(w, "nbc")) return sim->nbc;
    if (!strcmp(w, "cstop")) return sim->cstop;
    if (!strcmp(w, "dtreport")) return sim->dtreport;
    if (!strcmp(w, "done")) return sim->done;
    if (!strcmp(w, "nbad")) return sim->nbad_last;
    if (!strcmp(w, "nzx")) return sim->nzx;
    if (!strcmp(w, "nzy")) return sim->nzy;
    return -1;
}

double orc_scalar(const orc_sim* sim, const char* w) {
    if (!strcmp(w, "time")) return sim->time;
    if (!strcmp(w, "dt")) return sim->dt;
    if (!strcmp(w, "dtrec")) return sim->dtrec;
    if (!strcmp(w, "dtnew")) return sim->dtnew;
    if (!strcmp(w, "dvovmax")) return sim->dvovmax;
    if (!strcmp(w, "tstop")) return sim->tstop;
    /* the deck parameters (Driver.cc:78-87, Hydro.cc:206-214,
     * PolyGas.cc:58-59, TTS.cc:46-47, QCS.cc:84-86) */
    if (!strcmp(w, "dtmax")) return sim->dtmax;
    if (!strcmp(w, "dtinit")) return sim->dtinit;
    if (!strcmp(w, "dtfac")) return sim->dtfac;
    if (!strcmp(w, "cfl")) return sim->cfl;
    if (!strcmp(w, "cflv")) return sim->cflv;
    if (!strcmp(w, "rinit")) return sim->rinit;
    if (!strcmp(w, "einit")) return sim->einit;
    if (!strcmp(w, "rinitsub")) return sim->rinitsub;
    if (!strcmp(w, "einitsub")) return sim->einitsub;
    if (!strcmp(w, "uinitradial")) return sim->uinitradial;
    if (!strcmp(w, "gamma")) return sim->pgamma;
    if (!strcmp(w, "pgas_ssmin")) return sim->pssmin;
    if (!strcmp(w, "alfa")) return sim->alfa;
    if (!strcmp(w, "tts_ssmin")) return sim->tssmin;
    if (!strcmp(w, "qgamma")) return sim->qgamma;
    if (!strcmp(w, "q1")) return sim->q1;
    if (!strcmp(w, "q2")) return sim->q2;
    return NAN;
}

int orc_bc_count(const orc_sim* sim, int i) {
    return (i >= 0 && i < sim->nbc) ? sim->bcn[i] : -1;
}

void* orc_field(orc_sim* sim, const char* n) {
#define F(name, ptr) if (!strcmp(n, name)) return (void*)(ptr)
    F("znump", sim->znump); F("mapsp1", sim->mapsp1); F("mapsp2", sim->mapsp2);
    F("mapsz", sim->mapsz); F("mapss3", sim->mapss3); F("mapss4", sim->mapss4);
    F("px", sim->px); F("pxp", sim->pxp); F("px0", sim->px0); F("pu", sim->pu);
    F("pu0", sim->pu0); F("pf", sim->pf); F("pap", sim->pap); F("pmaswt", sim->pmaswt);
    F("zx", sim->zx); F("zxp", sim->zxp); F("zuc", sim->zuc); F("zarea", sim->zarea);
    F("zvol", sim->zvol); F("zareap", sim->zareap); F("zvolp", sim->zvolp);
    F("zvol0", sim->zvol0); F("zdl", sim->zdl); F("zm", sim->zm); F("zr", sim->zr);
    F("zrp", sim->zrp); F("ze", sim->ze); F("zetot", sim->zetot); F("zw", sim->zw);
    F("zwrate", sim->zwrate); F("zp", sim->zp); F("zss", sim->zss); F("zdu", sim->zdu);
    F("ztmp", sim->ztmp); F("ex", sim->ex); F("exp", sim->expp); F("ssurfp", sim->ssurfp);
    F("sfp", sim->sfp); F("sfq", sim->sfq); F("sft", sim->sft); F("cqe1", sim->cqe1);
    F("cqe2", sim->cqe2); F("sarea", sim->sarea); F("svol", sim->svol);
    F("sareap", sim->sareap); F("svolp", sim->svolp); F("elen", sim->elen);
    F("smf", sim->smf); F("carea", sim->carea); F("cevol", sim->cevol); F("cdu", sim->cdu);
    F("cdiv", sim->cdiv); F("ccos", sim->ccos); F("crmu", sim->crmu); F("cw", sim->cw);
#undef F
    if (!strncmp(n, "bcpts", 5)) {
        const int b = atoi(n + 5);
        if (b >= 0 && b < sim->nbc) return sim->bcpts[b];
    }
    return NULL;
}

/* ------------------------------------------------------------------ */
/* Output (WriteXY.cc:28-52, ExportGold.cc:31-307)                      */
/* ------------------------------------------------------------------ */
int orc_write_xy(const orc_sim* sim, const char* path) {
    FILE* f = fopen(path, "w");
    if (!f) return ORC_ERR_ARG;
    const double* v[3] = {sim->zr, sim->ze, sim->zp};
    const char* nm[3] = {"zr", "ze", "zp"};
    for (int k = 0; k < 3; ++k) {
        fprintf(f, "#  %s\n", nm[k]);
        for (int z = 0; z < sim->numz; ++z) fprintf(f, "%5d%18.8e\n", z + 1, v[k][z]);
    }
    fclose(f);
    return ORC_OK;
}

int orc_write_gold(const orc_sim* sim, const char* base) {
    char fn[4096];
    const int nz = sim->numz, np = sim->nump;
    int* mapzs = (int*)xalloc(sizeof(int) * (size_t)nz);
    int nt = 0, nq = 0, no = 0, sc = 0;
    for (int z = 0; z < nz; ++z) {
        if (sim->znump[z] == 3) ++nt; else if (sim->znump[z] == 4) ++nq; else ++no;
        mapzs[z] = sc; sc += sim->znump[z];
    }
    snprintf(fn, sizeof(fn), "%s.case", base);
    FILE* f = fopen(fn, "w");
    if (!f) { free(mapzs); return ORC_ERR_ARG; }
    fprintf(f, "#\n# Created by PENNANT\n#\nFORMAT\ntype: ensight gold\nGEOMETRY\nmodel: %s.geo\n"
               "VARIABLE\nscalar per element: zr %s.zr\nscalar per element: ze %s.ze\n"
               "scalar per element: zp %s.zp\n", base, base, base, base);
    fclose(f);
    snprintf(fn, sizeof(fn), "%s.geo", base);
    f = fopen(fn, "w");
    if (!f) { free(mapzs); return ORC_ERR_ARG; }
    fprintf(f, "cycle = %8d\nt = %15.8e\nnode id assign\nelement id given\npart\n%10d\nuniverse\n"
               "coordinates\n%10d\n", sim->cycle, sim->time, 1, np);
    for (int p = 0; p < np; ++p) fprintf(f, "%12.5e\n", sim->px[p].x);
    for (int p = 0; p < np; ++p) fprintf(f, "%12.5e\n", sim->px[p].y);
    for (int p = 0; p < np; ++p) fprintf(f, "%12.5e\n", 0.);
    const int sizes[2] = {3, 4};
    const char* tags[2] = {"tria3", "quad4"};
    const int counts[2] = {nt, nq};
    for (int k = 0; k < 2; ++k) {
        if (!counts[k]) continue;
        fprintf(f, "%s\n%10d\n", tags[k], counts[k]);
        for (int z = 0; z < nz; ++z) if (sim->znump[z] == sizes[k]) fprintf(f, "%10d\n", z + 1);
        for (int z = 0; z < nz; ++z) {
            if (sim->znump[z] != sizes[k]) continue;
            for (int i = 0; i < sizes[k]; ++i) fprintf(f, "%10d", sim->mapsp1[mapzs[z] + i] + 1);
            fprintf(f, "\n");
        }
    }
    if (no) {
        fprintf(f, "nsided\n%10d\n", no);
        for (int z = 0; z < nz; ++z) if (sim->znump[z] > 4) fprintf(f, "%10d\n", z + 1);
        for (int z = 0; z < nz; ++z) if (sim->znump[z] > 4) fprintf(f, "%10d\n", sim->znump[z]);
        for (int z = 0; z < nz; ++z) {
            if (sim->znump[z] <= 4) continue;
            for (int i = 0; i < sim->znump[z]; ++i) fprintf(f, "%10d", sim->mapsp1[mapzs[z] + i] + 1);
            fprintf(f, "\n");
        }
    }
    fclose(f);
    const double* vars[3] = {sim->zr, sim->ze, sim->zp};
    const char* vn[3] = {"zr", "ze", "zp"};
    for (int v = 0; v < 3; ++v) {
        snprintf(fn, sizeof(fn), "%s.%s", base, vn[v]);
        f = fopen(fn, "w");
        if (!f) { free(mapzs); return ORC_ERR_ARG; }
        fprintf(f, "%s\npart\n%10d\n", vn[v], 1);
        for (int k = 0; k < 2; ++k) {
            if (!counts[k]) continue;
            fprintf(f, "%s\n", tags[k]);
            for (int z = 0; z < nz; ++z) if (sim->znump[z] == sizes[k]) fprintf(f, "%12.5e\n", vars[v][z]);
        }
        if (no) {
            fprintf(f, "nsided\n");
            for (int z = 0; z < nz; ++z) if (sim->znump[z] > 4) fprintf(f, "%12.5e\n", vars[v][z]);
        }
        fclose(f);
    }
    free(mapzs);
    return ORC_OK;
}
