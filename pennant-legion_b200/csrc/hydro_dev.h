// hydro_dev.h -- device-side data of one hydro instance and the launch
// entry points of the cycle kernels.
#pragma once

#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

struct pnt_hydro;

namespace pnt {

constexpr int kMaxBC = 16;

// Run state the kernels read and the finalize step updates; it lives in
// device memory so the whole cycle can be replayed from a CUDA graph.
struct Ctl {
    double dt;       // dt of the next cycle to run
    double dtinv;    // 1/dt, as calcWorkRate forms it (Hydro.cc:1496)
    double dtlast;   // dt of the last completed cycle
    double time;     // simulation time after the last completed cycle
    double dtrec;    // Hydro::calcDtTask result of the last cycle
    double dtnew;    // calcDtNew of the last cycle
    double dvovmax;  // calcDvol of the last cycle
    int32_t cycle;   // completed cycles; the current point buffer is cycle & 1
    int32_t done;    // cstop/tstop reached or an error
    int32_t status;  // pnt_status of a failure
    int32_t nbad;    // negative side count of a failure
    int32_t stop_at; // kernels skip once cycle >= stop_at
    int32_t pad;
};

// Per-run constants (deck values and the quantities the reference
// computes once per task from them).
struct HydroConst {
    double cfl, cflv;
    double gm1, ssmin2;           // PolyGas: gamma - 1, max(ssmin^2, 1e-99)
    double alfa, tts_ssmin;       // TTS
    double gammap1, q1, q2;       // QCS: qgamma + 1
    double dtmax, dtinit, dtfac, tstop;
    int32_t cstop;
    int32_t nbc;
    double vfix[kMaxBC][2];
};

// Device arrays of one mesh + state, reference numbering.
struct DevArrays {
    int32_t nump, numz, nums;
    int32_t quads;               // all zones are quads at sides 4z..4z+3
    int32_t rect_nzx;            // > 0: numbered as the rect generator does, nzx zones a row (row_tiles.cuh)
    const int32_t* zfirst;       // [numz]
    const int32_t* znump;        // [numz]
    const int32_t* mapsp1;       // [nums]
    const double* smf;           // [nums]
    const int32_t* poff;         // [nump+1]
    const int32_t* pcorner;      // [nums]
    const uint16_t* bcmask;      // [nump] bit b: point on BC plane b
    double2* px[2];              // point position, double buffered by cycle parity
    double2* pu[2];              // point velocity
    double* zm;
    double* zr;
    double* ze;
    double* zetot;
    double* zwrate;
    double* zvol;
    double* zp;
    // per-side intermediates written by pass A
    double* cmass;               // corner mass of side s at point mapsp1[s]
    double2* cforce;             // corner force of side s at point mapsp1[s]
    double2* sftot;              // sfp + sfq of side s (calcWork)
    // the same buffers in FP32 for the mixed-precision cycle
    float* cmass_f;
    float2* cforce_f;
    float2* sftot_f;
    // batched meshes: per-tile partial reductions (npartA entries for pass
    // A, npartC for C)
    int32_t npartA, npartC;
    double* part_dtnew;
    int32_t* part_badA;
    double* part_dvov;
    int32_t* part_badC;
    // one mesh: the cycle's reductions, combined by every CTA of passes A
    // and C with atomics ([0] minimum zone dt and [1] maximum |dV/V0| as
    // order-preserving keys (dkey), [2] / [3] inverted sides in A / C), and
    // the ticket that picks pass C's last CTA, which ends the cycle and
    // resets them; [4] is set when a bounded wait of a kernel ran out
    long long* cyc_red;
    uint32_t* fin_ticket;
    Ctl* ctl;
    // learned closure (precision = learned): parameter image and the corner
    // class counters [class][64] (closure_dev.cuh)
    const uint8_t* closure_img;
    unsigned long long* closure_counts;
    // zones whose corners the closure pass evaluates: records
    // [numz][kZoneRecF4] float4 (closure_dev.cuh) and this cycle's count
    float* closure_rec;
    int32_t* closure_nrec;
    int32_t closure_grid;   // CTAs of the persistent closure pass
    int32_t gridC;          // CTAs of the persistent pass C (pass_c_staged.cuh)
    int32_t gridA;          // CTAs of the persistent row-tile mixed/learned pass A (rect meshes)
    // multi-piece runs: pass C's last CTA writes this piece's [dtnew,
    // -dvovmax, inverted sides in A, in C] here instead of ending the cycle
    // (nullptr for a single piece)
    double* piece_red;
};

constexpr int kZoneThreads = 256;   // pass A: 64 zones x 4 side lanes per block
constexpr int kPointThreads = 256;

inline int64_t zone_blocks(int32_t numz, int threads = kZoneThreads) {
    return (4 * (int64_t)numz + threads - 1) / threads;
}

// Events a cycle records when timed: before pass A, after A, after the
// closure pass (right after A when there is none), after B, C, finalize.
constexpr int kNumEvents = 6;
constexpr int kNumKernels = 5;   // A, B, C, finalize, closure pass

// Phases of a cycle: the corner forces (pass A and the learned closure
// pass) and the advance (passes B, C and the finalize step).
// Programmatic dependent launch: the cycle's kernels are launched with
// launch_pdl, so that each is launched while the kernel before it drains
// rather than after it has completed.  Every such kernel calls pdl_wait()
// before it reads anything an earlier kernel wrote or writes anything an
// earlier kernel reads; the wait returns once the previous grid has
// completed and its memory is visible.  No kernel signals its dependents
// early (griddepcontrol.launch_dependents): dependent CTAs waiting on the
// SMs while the previous kernel still ran made the 1920^2 cycles 5-17%
// slower, against 0.1-0.7% faster without that signal.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
#endif

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                              Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

constexpr int kPhaseForces = 1;
constexpr int kPhaseAdvance = 2;
constexpr int kPhaseAll = kPhaseForces | kPhaseAdvance;

// One hydro cycle (passes A, B, C and the finalize step) on `stream`, or
// the given phases of it.  With `ev` non-null (whole cycles only), the
// kNumEvents events above are recorded.
cudaError_t launch_cycle_fp64(const DevArrays& a, const HydroConst& c, cudaStream_t stream,
                              cudaEvent_t* ev = nullptr, int phases = kPhaseAll);
// The mixed-precision cycle (hydro_mixed.cu).
cudaError_t launch_cycle_mixed(const DevArrays& a, const HydroConst& c, cudaStream_t stream,
                               cudaEvent_t* ev = nullptr, int phases = kPhaseAll);
// The learned-closure cycle: the mixed cycle with the closure pass after
// pass A.
cudaError_t launch_cycle_learned(const DevArrays& a, const HydroConst& c, cudaStream_t stream,
                                 cudaEvent_t* ev = nullptr, int phases = kPhaseAll);
// Multi-piece runs (hydro_fp64.cu): gathers the corner mass and force of
// the nsend local sides send_side[] into send (corner masses, then the
// corner forces at byte offset foff; FP32 when mixed), and ends the cycle
// from the globally reduced piece_red.
void launch_piece_pack(const DevArrays& a, const int32_t* send_side, int32_t nsend, unsigned char* send,
                       size_t foff, bool mixed, cudaStream_t stream);
void launch_piece_finish(const DevArrays& a, const HydroConst& c, cudaStream_t stream);
// The index of the first non-finite value of a[0 .. n) into *first (an
// atomic minimum; *first must start at ULLONG_MAX).
void launch_find_nonfinite(const double* a, int64_t n, unsigned long long* first, cudaStream_t stream);
// Raises the closure pass's dynamic shared-memory limit on the current device.
cudaError_t prepare_learned_kernels();
// Pass C of the FP64 (mixed = false) or mixed/learned cycle (pass_c.cu):
// prepare_pass_c raises the kernel's shared-memory limit on the current
// device and returns its persistent grid (resident CTAs per SM x nsm, at
// most one per tile); launch_pass_c launches it with a.gridC CTAs, which
// write a.gridC partials.
cudaError_t prepare_pass_c(bool mixed, bool quads, int32_t rect_nzx, int32_t numz, int nsm, int32_t* grid);
void launch_pass_c(const DevArrays& a, const HydroConst& c, bool mixed, cudaStream_t stream);
// The row-tile pass A of the mixed or learned cycle (hydro_mixed.cu): raises
// the kernel's shared-memory limit on the current device and returns its
// persistent grid.
cudaError_t prepare_pass_a_rows_mixed(bool learned, int32_t rect_nzx, int32_t numz, int nsm, int32_t* grid);

// Device state of a pnt_hydro for the closure harvest (closure.cu).
struct HydroAccess {
    DevArrays a;
    HydroConst c;
    cudaStream_t stream;
    int device;
};
bool hydro_access(pnt_hydro* h, HydroAccess* out);

}  // namespace pnt
