/*
 * pnt_oracle.h -- CPU oracle for PENNANT's Lagrangian hydro cycle.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a serial (optionally OpenMP) C
 * restatement of the reference's CPU task bodies, used by the test suite
 * as the parity checker and by bench.py as the timed CPU baseline.  The
 * product library (libpennant_b200.so) never links, loads or calls it.
 *
 * Parity pin: with the reference deck test/sedov/sedov.pnt the oracle
 * reproduces the reference's own golden output test/sedov/sedov.xy (zr, ze,
 * zp of 2025 zones, 8 significant digits) and sedov.geo (point coordinates,
 * 5 significant digits) after 10 cycles; see tests/test_oracle_golden.py.
 */
#ifndef PNT_ORACLE_H
#define PNT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

enum {
    ORC_OK = 0,
    ORC_ERR_ARG = 1,
    ORC_ERR_DECK = 2,
    ORC_ERR_BADSIDES = 3,
    ORC_ERR_NOMEM = 7,
    ORC_ERR_UNSUPPORTED = 5
};

/* Build a simulation from a .pnt deck file (Driver ctor + Mesh + Hydro).
 * `text` may be given instead of `path` (deck contents in memory). */
int orc_create(const char* path, const char* text, orc_sim** out,
               char* err, size_t errlen);
void orc_destroy(orc_sim* sim);

/* One Driver::run iteration: calcGlobalDt, Hydro::doCycle, time/cycle
 * update.  Returns ORC_ERR_BADSIDES on negative side volumes.  A call after
 * the run is done (cycle >= cstop or time >= tstop) does nothing. */
int orc_cycle(orc_sim* sim);
/* Run cycles until done or max_cycles (<=0: no limit) more cycles ran. */
int orc_run(orc_sim* sim, int max_cycles);
int orc_done(const orc_sim* sim);

/* Threads for the OpenMP variant (restating the reference's *OMPTask loops
 * with atomic reductions; order-nondeterministic, timing only).  0 or 1
 * selects the serial, bit-reproducible task order. */
void orc_set_threads(orc_sim* sim, int nthreads);

/* Sizes: "nump", "numz", "nums", "cycle", "nbc". */
int64_t orc_num(const orc_sim* sim, const char* what);
/* Scalars: "time", "dt", "dtrec", "dtnew", "dvovmax" ... */
double orc_scalar(const orc_sim* sim, const char* what);
/* Pointer to a field array by reference field name (e.g. "zr", "px",
 * "mapsp1", "bcpts0").  Points/sides/zones in reference numbering.
 * double2 fields are interleaved (x, y). */
void* orc_field(orc_sim* sim, const char* name);
/* Element count of the BC point list `i` (deck order: bcx..., bcy...). */
int orc_bc_count(const orc_sim* sim, int i);

/* Output writers restating WriteXY::write and ExportGold::write. */
int orc_write_xy(const orc_sim* sim, const char* path);
int orc_write_gold(const orc_sim* sim, const char* basename);

#ifdef __cplusplus
}
#endif
#endif
