/*
 * pennant_b200.h -- C ABI of the B200-native PENNANT hydro cycle.
 *
 * This is the drop-in boundary for the reference's Hydro::doCycle path
 * (StanfordLegion/pennant-legion).  Each entry point names the reference
 * interface it replaces (file:line within that project).  All signatures
 * use plain C types: pointers, sizes, POD structs.  Every call returns a
 * pnt_status (0 = success) and never exits the process; pnt_last_error()
 * gives the message of the last failure on the calling thread.
 *
 * Ownership: host buffers passed in are owned by the caller and only read
 * (or written, for downloads) during the call.  Device memory is owned by
 * the library object that allocated it.  One CUDA stream per pnt_hydro;
 * calls on one object are not thread-safe, distinct objects may be driven
 * concurrently from different threads.
 */
#ifndef PENNANT_B200_H
#define PENNANT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PNT_ABI_VERSION 1

typedef int32_t pnt_status;
enum {
    PNT_OK = 0,
    PNT_ERR_INVALID_ARG = 1,  /* bad pointer, size or value */
    PNT_ERR_DECK = 2,         /* malformed .pnt deck (InputFile.cc:28-50, GenMesh.cc:89-127) */
    PNT_ERR_BADSIDES = 3,     /* negative side volumes (Mesh.cc:1531-1550) */
    PNT_ERR_CUDA = 4,         /* CUDA runtime failure */
    PNT_ERR_UNSUPPORTED = 5,  /* feature outside this build (e.g. hex meshes) */
    PNT_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up */
    PNT_ERR_NOMEM = 7,        /* host or device allocation failed */
    PNT_ERR_NO_DEVICE = 8,    /* no CUDA device, or the kernels are not loadable */
    PNT_ERR_STATE = 9         /* call not valid in the object's current state */
};

const char* pnt_status_string(pnt_status st);
/* Message of the last failing call on this thread ("" if none). */
const char* pnt_last_error(void);
int32_t pnt_abi_version(void);

/* ------------------------------------------------------------------ */
/* Input deck: replaces InputFile (InputFile.hh:21-42, InputFile.cc:24-104) */
/* ------------------------------------------------------------------ */
typedef struct pnt_deck pnt_deck;

/* InputFile::InputFile(filename): `key value...` lines, '#' comments,
 * duplicate key is an error (PNT_ERR_DECK). */
pnt_status pnt_deck_load(const char* path, pnt_deck** out);
/* Same, from the deck's text in memory. */
pnt_status pnt_deck_parse(const char* text, pnt_deck** out);
/* Set or replace one key (the value is the text after the key). */
pnt_status pnt_deck_set(pnt_deck* deck, const char* key, const char* value);
int32_t pnt_deck_has(const pnt_deck* deck, const char* key);
/* InputFile::getInt / getDouble / getString / getDoubleList (InputFile.cc:63-104) */
int32_t pnt_deck_get_int(const pnt_deck* deck, const char* key, int32_t dflt);
double pnt_deck_get_double(const pnt_deck* deck, const char* key, double dflt);
/* Copies the first token (or dflt) into buf; returns its length. */
int32_t pnt_deck_get_string(const pnt_deck* deck, const char* key, const char* dflt,
                            char* buf, size_t buflen);
/* Returns the number of values (written up to maxn), or -1 if absent. */
int32_t pnt_deck_get_double_list(const pnt_deck* deck, const char* key, double* out,
                                 int32_t maxn);
void pnt_deck_destroy(pnt_deck* deck);

/* ------------------------------------------------------------------ */
/* Mesh: replaces Mesh(inp, numpcs) + GenMesh (Mesh.cc:211-652,        */
/* GenMesh.cc:87-129, 790-1282) for a single piece, reference numbering */
/* ------------------------------------------------------------------ */
typedef struct pnt_mesh pnt_mesh;

/* Connectivity in the reference's numbering: zones, sides 4z+k (rect),
 * points j*(nzx+1)+i (rect).  Sides of a zone are contiguous and circulate
 * (mapsp2[s] == mapsp1[mapss4[s]]).  px is double2 interleaved (x, y). */
typedef struct {
    int32_t nump, numz, nums;
    const double* px;        /* [2*nump] initial point coordinates */
    const int32_t* znump;    /* [numz]   sides (= points) per zone, 3 or 4 */
    const int32_t* mapsp1;   /* [nums]   side -> first point  (FID_MAPSP1) */
    const int32_t* mapsp2;   /* [nums]   side -> second point (FID_MAPSP2) */
    const int32_t* mapsz;    /* [nums]   side -> zone         (FID_MAPSZ)  */
    const int32_t* mapss3;   /* [nums]   previous side in zone (FID_MAPSS3) */
    const int32_t* mapss4;   /* [nums]   next side in zone     (FID_MAPSS4) */
} pnt_mesh_desc;

/* GenMesh::generate{Points,Zones,Sides}Parallel for meshtype rect or pie
 * (GenMesh.cc:528-665) with one piece.  meshtype hex: PNT_ERR_UNSUPPORTED
 * (the reference's parallel hex generator asserts, GenMesh.cc:875-896). */
pnt_status pnt_mesh_generate(const pnt_deck* deck, pnt_mesh** out);
/* Mesh from caller-provided connectivity (validated; copied). */
pnt_status pnt_mesh_create(const pnt_mesh_desc* desc, pnt_mesh** out);
/* Pointers stay owned by the mesh and valid until pnt_mesh_destroy. */
pnt_status pnt_mesh_describe(const pnt_mesh* mesh, pnt_mesh_desc* out);
/* Point -> corner CSR used by the deterministic force/mass gather:
 * sides[offsets[p] .. offsets[p+1]) are the sides s with mapsp1[s] == p in
 * ascending order (the serial summation order of Hydro.cc:1100-1116,
 * :1175-1192). offsets has nump+1 entries. */
pnt_status pnt_mesh_point_corners(const pnt_mesh* mesh, const int32_t** offsets,
                                  const int32_t** sides);
void pnt_mesh_destroy(pnt_mesh* mesh);

/* Multi-piece runs: replaces the numpcs decomposition of Mesh(inp, numpcs)
 * with its private, master and ghost points (Mesh.cc:211-241, :441-617).
 * Piece `piece` of `npieces` (1-64) of a single-piece mesh is the zone range
 * [numz*piece/npieces, numz*(piece+1)/npieces): its zones, their sides and
 * every point they touch, numbered in global order, with the single-piece
 * initial geometry.  For a piece mesh pnt_mesh_describe gives the local
 * connectivity, and pnt_mesh_point_corners lists, per local point, local
 * sides s < nums and halo slots nums + h merged in global side order: the
 * halo slots hold corners of that point that other pieces own, so the
 * corner sums at shared points keep the single-piece order.  A hydro object
 * created from a piece steps with pnt_hydro_piece_* and exchanges halo
 * corners with its neighbours every cycle. */
pnt_status pnt_mesh_piece(const pnt_mesh* mesh, int32_t npieces, int32_t piece, pnt_mesh** out);

typedef struct {
    int32_t piece, npieces;
    int32_t zone0;               /* global id of local zone 0 (local zones are contiguous) */
    int32_t side0;               /* global id of local side 0 (local sides are contiguous) */
    const int32_t* gpoint;       /* [nump] global id of each local point (NULL for one piece) */
    int32_t nhalo;               /* halo corner slots after the nums local sides */
    const int32_t* halo_side;    /* [nhalo] global side of each halo slot */
    int32_t nnbr;                /* neighbour pieces (sharing points), ascending */
    const int32_t* nbr;          /* [nnbr] */
    /* recv_off[j] .. recv_off[j+1]: halo slots neighbour nbr[j] fills, in
     * global side order; send_side[send_off[j] .. send_off[j+1]): local
     * sides whose corner mass and force neighbour nbr[j] needs, in global
     * side order (the same sides as its halo slots from this piece). */
    const int32_t* recv_off;     /* [nnbr+1] */
    const int32_t* send_off;     /* [nnbr+1] */
    const int32_t* send_side;    /* [send_off[nnbr]] */
} pnt_piece_desc;

/* Pointers stay owned by the mesh. */
pnt_status pnt_mesh_piece_describe(const pnt_mesh* mesh, pnt_piece_desc* out);

/* ------------------------------------------------------------------ */
/* Parameters: deck keys and defaults of Driver (Driver.cc:78-87),       */
/* Hydro (Hydro.cc:206-214), PolyGas (PolyGas.cc:57-60), TTS             */
/* (TTS.cc:45-48), QCS (QCS.cc:83-86), HydroBC planes (Hydro.cc:220-225) */
/* ------------------------------------------------------------------ */
#define PNT_MAX_BC 16

enum { PNT_PREC_FP64 = 0, PNT_PREC_MIXED = 1, PNT_PREC_LEARNED = 2 };

typedef struct {
    /* Driver */
    int32_t cstop, dtreport;
    double tstop, dtmax, dtinit, dtfac;
    /* Hydro */
    double cfl, cflv, rinit, einit, rinitsub, einitsub, uinitradial;
    int32_t has_subregion;
    double subregion[4];
    int32_t nbcx, nbcy;
    double bcx[PNT_MAX_BC], bcy[PNT_MAX_BC];
    /* PolyGas */
    double gamma, pgas_ssmin;
    /* TTS */
    double alfa, tts_ssmin;
    /* QCS */
    double qgamma, q1, q2;
    /* Project-only keys (ignored by the reference): arithmetic of the
     * side pass, cycles per captured CUDA graph in pnt_hydro_run. */
    int32_t precision;
    int32_t graph_cycles;
    int32_t reserved[14];
} pnt_params;

pnt_status pnt_params_default(pnt_params* out);
/* Reads every key above from the deck (missing keys keep defaults);
 * "precision fp64|mixed|learned" and "graphcycles N" are the project-only
 * keys. */
pnt_status pnt_params_from_deck(const pnt_deck* deck, pnt_params* out);

/* ------------------------------------------------------------------ */
/* Hydro on one GPU: replaces Hydro(inp, mesh) + Hydro::init()           */
/* (Hydro.cc:200-339) and the Driver loop around Hydro::doCycle          */
/* (Driver.cc:102-187, Hydro.cc:342-983)                                 */
/* ------------------------------------------------------------------ */
typedef struct pnt_hydro pnt_hydro;

typedef struct {
    int32_t cycle;      /* completed cycles */
    int32_t done;       /* 1 once cycle >= cstop, time >= tstop, or error */
    pnt_status status;  /* PNT_ERR_BADSIDES after negative side volumes */
    int32_t nbad;       /* negative side count behind that error */
    double time;        /* simulation time after the last completed cycle */
    double dt;          /* dt used by the last completed cycle */
    double dtrec;       /* hydro-recommended dt (Hydro::calcDtTask) */
    double dtnew;       /* Courant limit (calcDtNewTask) of the last cycle */
    double dvovmax;     /* max |dV/V| (calcDvolTask) of the last cycle */
} pnt_scalars;

/* Allocates device state on `device`, uploads the mesh and runs
 * Hydro::init (subregion, zm, zetot, radial velocity). */
pnt_status pnt_hydro_create(const pnt_mesh* mesh, const pnt_params* params, int32_t device,
                            pnt_hydro** out);
void pnt_hydro_destroy(pnt_hydro* hydro);

/* One iteration of Driver::run: calcGlobalDt (Driver.cc:213-245),
 * Hydro::doCycle, time/cycle update; blocks until done.  Stops (no-op)
 * once done, as the predicated reference does (Driver.cc:140-144). */
pnt_status pnt_hydro_cycle(pnt_hydro* hydro, pnt_scalars* out);

/* Report callback, called at cycle 1 and every dtreport cycles with the
 * state of Driver::reportMeasurementTask (Driver.cc:329-347). */
typedef void (*pnt_report_fn)(const pnt_scalars* s, double wall_us, void* user);

/* Runs up to max_cycles more cycles (<= 0: until cstop/tstop) as replays
 * of a captured CUDA graph; the host only synchronises at report points. */
pnt_status pnt_hydro_run(pnt_hydro* hydro, int32_t max_cycles, pnt_report_fn report,
                         void* user, pnt_scalars* out);
/* Enqueues `ncycles` cycles on the object's stream without waiting
 * (graph replay); read the result with pnt_hydro_get_scalars. */
pnt_status pnt_hydro_enqueue(pnt_hydro* hydro, int32_t ncycles);
pnt_status pnt_hydro_synchronize(pnt_hydro* hydro);
pnt_status pnt_hydro_get_scalars(pnt_hydro* hydro, pnt_scalars* out);

/* Instrumentation (the role of the reference's TimingLauncher,
 * Driver.cc:117-168): runs `ncycles` cycles launching each pass separately
 * with CUDA events around it and writes the mean milliseconds of pass i to
 * kernel_ms[i] for i < nkernels (0 pass A zone predictor, 1 pass B point
 * update, 2 pass C zone corrector, which also ends the cycle, 3 a separate
 * end-of-cycle step (none any more: about 0), 4 the learned cycle's closure
 * pass, 0 for the other cycles). */
pnt_status pnt_hydro_time_kernels(pnt_hydro* hydro, int32_t ncycles, double* kernel_ms,
                                  int32_t nkernels);
/* Copies the run state (point positions and velocities, zone fields, time,
 * dt, cycle) of `src` into `dst`: two objects of the same mesh on the same
 * device, whatever their precision (a restart of dst from src's state; no
 * counterpart in the reference). */
pnt_status pnt_hydro_copy_state(pnt_hydro* dst, const pnt_hydro* src);
/* Enqueues `ncycles` cycles (graph replay) between two CUDA events on the
 * object's stream, waits, and returns the elapsed device milliseconds. */
pnt_status pnt_hydro_time_cycles(pnt_hydro* hydro, int32_t ncycles, double* elapsed_ms);

/* Field ids for upload/download, reference numbering and field names
 * (Mesh.cc:258-423).  double2 fields are interleaved (x, y). */
enum {
    PNT_FIELD_PX = 0,     /* double2 [nump] point position */
    PNT_FIELD_PU = 1,     /* double2 [nump] point velocity */
    PNT_FIELD_ZR = 2,     /* double  [numz] density */
    PNT_FIELD_ZE = 3,     /* double  [numz] specific internal energy */
    PNT_FIELD_ZP = 4,     /* double  [numz] half-step pressure of the last cycle */
    PNT_FIELD_ZM = 5,     /* double  [numz] zone mass */
    PNT_FIELD_ZETOT = 6,  /* double  [numz] zone total internal energy */
    PNT_FIELD_ZVOL = 7,   /* double  [numz] zone volume (RZ, per radian) */
    PNT_FIELD_ZWRATE = 8, /* double  [numz] work rate */
    PNT_FIELD_SMF = 9,    /* double  [nums] side mass fraction (constant) */
    PNT_FIELD_COUNT = 10
};
/* bytes must equal the field's size (element count x element size). */
pnt_status pnt_hydro_download(pnt_hydro* hydro, int32_t field, void* host_dst, size_t bytes);
pnt_status pnt_hydro_upload(pnt_hydro* hydro, int32_t field, const void* host_src, size_t bytes);
/* Multi-piece cycle (a hydro object created from a pnt_mesh_piece mesh;
 * pnt_hydro_cycle/run/enqueue/time_* refuse it).  One cycle on the
 * object's stream, every piece in step:
 *   pnt_hydro_piece_forces   pass A (and the learned closure pass) on the
 *                            local zones, then the corner mass and force of
 *                            the send lists into the send buffer;
 *   (caller)                 for each neighbour nbr[j]: send its send range
 *                            and receive its halo range (byte offsets below);
 *   pnt_hydro_piece_advance  passes B and C on the local points and zones
 *                            and this piece's reduction into red[4] =
 *                            {dtnew, -dvovmax, inverted sides in pass A, in
 *                            pass C};
 *   (caller)                 red[0:2] <- minimum over pieces, red[2:4] <-
 *                            sum over pieces;
 *   pnt_hydro_piece_finish   calcDt, the bad-side status, time/cycle and the
 *                            next dt from the reduced red (Hydro.cc:961-970,
 *                            Driver.cc:213-245).
 * Every piece then holds exactly the single-piece values of its zones and
 * points (shared points are advanced by each piece that holds them, from
 * the same corner sums in the same order). */
typedef struct {
    void* send;                   /* device: corner masses of send_side[] ... */
    size_t send_cforce_offset;    /* ... and their corner forces from this byte offset */
    void* halo_cmass;             /* device: halo slot h's corner mass at h*cmass_bytes */
    void* halo_cforce;            /* device: halo slot h's corner force at h*cforce_bytes */
    int32_t cmass_bytes;          /* 8 and 16 (fp64) or 4 and 8 (mixed, learned) */
    int32_t cforce_bytes;
    double* red;                  /* device [4] */
    void* stream;                 /* the object's cudaStream_t */
} pnt_piece_buffers;
pnt_status pnt_hydro_piece_buffers(pnt_hydro* hydro, pnt_piece_buffers* out);
pnt_status pnt_hydro_piece_forces(pnt_hydro* hydro);
pnt_status pnt_hydro_piece_advance(pnt_hydro* hydro);
pnt_status pnt_hydro_piece_finish(pnt_hydro* hydro);

/* Device address of the current copy of a field (valid until the next
 * cycle swaps the point buffers) and the object's cudaStream_t. */
pnt_status pnt_hydro_device_ptr(pnt_hydro* hydro, int32_t field, void** dptr);
pnt_status pnt_hydro_stream(pnt_hydro* hydro, void** cuda_stream);

/* ------------------------------------------------------------------ */
/* Batches of independent meshes on one GPU (project extension: the       */
/* reference advances one mesh per Driver).  Every instance runs the FP64 */
/* (or, for a batch of precision-mixed decks, the mixed) cycle            */
/* bit-identically to its own pnt_hydro; the batch advances all running   */
/* instances by one of their own cycles per batch cycle.                  */
/* ------------------------------------------------------------------ */
typedef struct pnt_batch pnt_batch;

/* n meshes with their own parameters (params[i]; one precision for all,
 * FP64 or mixed, else PNT_ERR_UNSUPPORTED); the meshes are copied.  Each
 * instance starts as pnt_hydro_create would. */
pnt_status pnt_batch_create(const pnt_mesh* const* meshes, const pnt_params* params, int32_t n,
                            int32_t device, pnt_batch** out);
void pnt_batch_destroy(pnt_batch* batch);
/* Work-list shape: zones per tile of the zone passes (multiple of 64) and
 * CTAs per SM of the persistent point pass.  Results do not depend on it. */
pnt_status pnt_batch_set_shape(pnt_batch* batch, int32_t zones_per_tile, int32_t ctas_per_sm);
pnt_status pnt_batch_get_shape(pnt_batch* batch, int32_t* zones_per_tile, int32_t* ctas_per_sm);
/* Autotuner: times each candidate shape on `trial_cycles` cycles of this
 * run (the cycles count: the run advances) and keeps the fastest. */
pnt_status pnt_batch_tune(pnt_batch* batch, int32_t trial_cycles, int32_t* zones_per_tile,
                          int32_t* ctas_per_sm, double* ms_per_cycle);
/* Runs batch cycles until every instance is done or max_cycles (<= 0: no
 * limit) have been enqueued; *running_left = instances still running. */
pnt_status pnt_batch_run(pnt_batch* batch, int32_t max_cycles, int32_t* running_left);
pnt_status pnt_batch_enqueue(pnt_batch* batch, int32_t ncycles);
pnt_status pnt_batch_time_cycles(pnt_batch* batch, int32_t ncycles, double* elapsed_ms);
pnt_status pnt_batch_scalars(pnt_batch* batch, int32_t instance, pnt_scalars* out);
pnt_status pnt_batch_download(pnt_batch* batch, int32_t instance, int32_t field, void* host_dst,
                              size_t bytes);

/* ------------------------------------------------------------------ */
/* Per-task operators on caller-owned device arrays                     */
/* ------------------------------------------------------------------ */

/* Hydro::calcDtNewTask + calcDvolTask + calcDtTask (Hydro.cc:1591-1667;
 * GPU variants gpu_calc_dt_new / gpu_calc_dvol, Hydro.cu:563-681) over
 * numz zones of caller device arrays: out[0] = dtrec, out[1] = dtnew
 * (Courant minimum), out[2] = dvovmax, written to device memory on
 * `stream` (a cudaStream_t; NULL = default stream).  Asynchronous; per-block
 * partial results go to stream-ordered scratch (cudaMallocAsync /
 * cudaFreeAsync on `stream`).  numz may be 0 (dtnew = 1e99, dvovmax = 1e-99). */
pnt_status pnt_op_calc_dt(const double* zdl, const double* zdu, const double* zss,
                          const double* zvol, const double* zvol0, int64_t numz, double cfl,
                          double cflv, double dtlast, double* out, void* stream);

/* pnt_op_calc_dt for callers that must not allocate device memory (no
 * counterpart in the reference).  Same arguments and results; it calls no
 * allocator.  Its scratch is a fixed 128 KiB device array that each GPU
 * holds from library load until process exit, which limits numz to
 * PNT_OP_CALC_DT_NOALLOC_MAX_ZONES (larger numz: PNT_ERR_INVALID_ARG).
 * Runs on the calling thread's current device.  The first call on a
 * device looks up the array's address: make it before any stream capture.
 * A device reset (cudaDeviceReset, or the end of the device's context)
 * moves the array; the next call after it looks the address up again, so
 * make that call before stream capture as well.  All calls on a device
 * share the array, so calls that overlap on the GPU race; serialise them. */
#define PNT_OP_CALC_DT_NOALLOC_MAX_ZONES 16777216
pnt_status pnt_op_calc_dt_noalloc(const double* zdl, const double* zdu, const double* zss,
                                  const double* zvol, const double* zvol0, int64_t numz,
                                  double cfl, double cflv, double dtlast, double* out,
                                  void* stream);

/* ------------------------------------------------------------------ */
/* Learned QCS closure (no counterpart in the reference): a 14-64-64-4   */
/* network that stands in for the corner forces of QCS::calcForce        */
/* (QCS.cc:246-327) on compressing corners in the precision-learned      */
/* cycle (the mixed cycle otherwise).  Corners past the compression      */
/* threshold, out of the training distribution, or in zones with an      */
/* acute corner keep the plain QCS; corners in the dead zone (velocity   */
/* jump <= dead * sound speed) get no viscous force.                     */
/* ------------------------------------------------------------------ */
typedef struct pnt_closure pnt_closure;

#define PNT_CLOSURE_PARAMS 5380  /* W1[64][14] b1[64] W2[64][64] b2[64] W3[4][64] b3[4] */
#define PNT_CLOSURE_NORM 36      /* input mean[14], std[14], output mean[4], std[4] */
/* corner classes counted by the learned cycle */
enum {
    PNT_CLOSURE_ZERO = 0,     /* no compression: no force, as in QCS */
    PNT_CLOSURE_DEAD = 1,     /* dead zone: no force */
    PNT_CLOSURE_MLP = 2,      /* the network */
    PNT_CLOSURE_FALLBACK = 3, /* compression past rho_max: plain QCS */
    PNT_CLOSURE_OOD = 4,      /* out of distribution: plain QCS */
    PNT_CLOSURE_ACUTE = 5,    /* zone with an acute corner: plain FP64 QCS */
    PNT_CLOSURE_ERROR = 6,    /* blocks whose tensor-core wait ran out */
    PNT_CLOSURE_ZONES = 7,    /* zones evaluated by the closure pass */
    PNT_CLOSURE_NCLASS = 8
};

/* Random (Glorot-uniform, seeded) network with identity normalisation. */
pnt_status pnt_closure_create(int32_t device, uint64_t seed, pnt_closure** out);
pnt_status pnt_closure_load(const char* path, int32_t device, pnt_closure** out);
pnt_status pnt_closure_save(const pnt_closure* closure, const char* path);
void pnt_closure_destroy(pnt_closure* closure);
/* Host copies of the parameters (PNT_CLOSURE_PARAMS floats), the
 * normalisation (PNT_CLOSURE_NORM) and the thresholds {dead, rho_max,
 * ood_kappa}; any pointer may be NULL.  Setting parameters resets Adam. */
pnt_status pnt_closure_get(const pnt_closure* closure, float* params, float* norm, float* thresholds);
pnt_status pnt_closure_set(pnt_closure* closure, const float* params, const float* norm,
                           const float* thresholds);
/* Training data from the FP64 state at the start of the next cycle of
 * `hydro` (which must be FP64): every eligible corner, kept with
 * probability `keep` by a hash of (seed, cycle, side), appended at *count
 * (in/out) to device arrays feats [capacity][14], targets [capacity][4]
 * (QCS corner forces in the closure's frame and scale) and sides
 * [capacity].  Deterministic order. */
pnt_status pnt_hydro_harvest(pnt_hydro* hydro, double dead, double keep, uint64_t seed, float* feats,
                             float* targets, int32_t* sides, int64_t capacity, int64_t* count);
/* Mean and standard deviation of n harvested samples (device arrays). */
pnt_status pnt_closure_fit_normalization(pnt_closure* closure, const float* feats,
                                         const float* targets, int64_t n);
/* Normalised BF16 inputs x [n][16] and FP32 targets t [n][4] (device). */
pnt_status pnt_closure_prepare(const pnt_closure* closure, const float* feats, const float* targets,
                               int64_t n, void* x, float* t);
/* `steps` Adam steps (BF16 tensor-core forward and backward, FP32
 * accumulation) of mean squared error; step s uses rows (first +
 * s*rows_per_step + i) mod n, i < rows_per_step.  losses[s] (host, may be
 * NULL) receives each step's loss. */
pnt_status pnt_closure_train(pnt_closure* closure, const void* x, const float* t, int64_t n,
                             int64_t first, int32_t steps, int32_t rows_per_step, float lr,
                             float* losses);
/* Loss gradient over all n rows (host grad[PNT_CLOSURE_PARAMS]). */
pnt_status pnt_closure_gradient(pnt_closure* closure, const void* x, const float* t, int64_t n,
                                float* grad, float* loss);
/* The network on n raw input rows (device feats [n][14] -> out [n][4]),
 * the tcgen05 inference of the learned cycle. */
pnt_status pnt_closure_forward(const pnt_closure* closure, const float* feats, int64_t n, float* out);
/* The bounded device-side wait the tensor-core kernels use for their MMA
 * completions, run on its own on `device`: one mbarrier polled at most
 * `limit` (1 .. 2^20) times, completed first by the waiting thread
 * (arrive = 1) or by nothing (arrive = 0).  PNT_OK when the wait completed,
 * PNT_ERR_TIMEOUT when it ran out; the device stays usable either way.  It
 * exercises the timeout path of those kernels without a fault. */
pnt_status pnt_closure_wait_probe(int32_t device, int32_t arrive, int32_t limit);
/* Gives a precision-learned hydro object its copy of the closure.  mode 0:
 * the network; 1: no force on the network's corners (ablation); 2: plain
 * QCS on them (isolates the classification). */
pnt_status pnt_hydro_set_closure(pnt_hydro* hydro, const pnt_closure* closure, int32_t mode);
/* Corner counts per class (PNT_CLOSURE_NCLASS entries) summed over the
 * cycles run since the last reset. */
pnt_status pnt_hydro_closure_counts(pnt_hydro* hydro, uint64_t* counts, int32_t reset);

/* Output writers: WriteXY::write (WriteXY.cc:28-52) and ExportGold::write
 * (ExportGold.cc:31-307) of the current state. */
pnt_status pnt_hydro_write_xy(pnt_hydro* hydro, const char* path);
pnt_status pnt_hydro_write_gold(pnt_hydro* hydro, const char* basename);

/* The analogue of the reference's NAN_CHECK accessors (MyLegion.hh:29-206):
 * scans the current point positions and velocities and the zone fields
 * (PNT_FIELD_PX .. PNT_FIELD_ZWRATE) on the device for NaN or Inf.  *field
 * = the first such field in that order and *index = the smallest point or
 * zone index holding one, or -1 and -1 when every value is finite. */
pnt_status pnt_hydro_check_finite(pnt_hydro* hydro, int32_t* field, int64_t* index);

/* numpcs pieces of one mesh stepped together by the library: the
 * reference's Mesh(inp, numpcs) on one node (Mesh.cc:211-241), without
 * Legion.  Piece q (pnt_mesh_piece) runs on devices[q % ndevices] (device 0
 * when ndevices is 0).  Every cycle the halo corners move by peer copies on
 * the receiving piece's stream after the sending piece's pack, and the four
 * per-piece scalars are reduced on the host; results are bit-identical to
 * the single-piece run.  A cycle that fails part way (a CUDA error) leaves
 * the pieces out of step: later cycles return PNT_ERR_STATE.
 * pnt_pieces_download gathers a point or zone field of the whole mesh in
 * reference order; pnt_pieces_write_xy writes the reference's .xy file
 * (WriteXY.cc:28-52). */
typedef struct pnt_pieces pnt_pieces;
pnt_status pnt_pieces_create(const pnt_mesh* mesh, const pnt_params* params, int32_t npieces,
                             const int32_t* devices, int32_t ndevices, pnt_pieces** out);
pnt_status pnt_pieces_set_closure(pnt_pieces* pieces, const pnt_closure* closure, int32_t mode);
pnt_status pnt_pieces_cycle(pnt_pieces* pieces, pnt_scalars* out);
pnt_status pnt_pieces_run(pnt_pieces* pieces, int32_t max_cycles, pnt_report_fn report, void* user,
                          pnt_scalars* out);
pnt_status pnt_pieces_download(pnt_pieces* pieces, int32_t field, void* dst, size_t bytes);
pnt_status pnt_pieces_write_xy(pnt_pieces* pieces, const char* path);
void pnt_pieces_destroy(pnt_pieces* pieces);

#ifdef __cplusplus
}
#endif
#endif /* PENNANT_B200_H */
