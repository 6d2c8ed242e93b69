// plan.hpp - host-side objects behind the C ABI (opaque to callers).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/gp5cu.h"
#include "ops.cuh"

namespace gp5 {

// Optional per-launch timing: when a plan has a recorder, every kernel launch is followed by
// an event on the plan stream, and kinds[i] labels launch i (axis*10 + mode, or 90 for a
// point-wise kernel).
struct ProfRec {
    std::vector<cudaEvent_t> ev;
    std::vector<int> kinds;
    size_t idx = 0;
    void record(cudaStream_t s, int kind);
};

struct AxisPlan {
    int n = 0;
    bool reg = false;     // register engine (power of two in [32, 512])
    int reg_threads = 0;  // register engine: threads per line (radix schedule 0)
    int reg_threads1 = 0; // the same for radix schedule 1
    LineSchedule sched{};  // mixed-radix schedule for the shared-memory engine
    void *tw = nullptr;    // device twiddle table, plan precision, forward sign
    int smem_lines = 0;    // lines per tile of the shared-memory engine
};

// The autotuned passes, in the order of gp5cu_plan_get_tiles: (axis, mode) of the strided
// register-engine launches (y fwd, y inv, z fwd, z inv, z fwd*K^2*inv).
constexpr int kTunedPasses = 5;
constexpr int kTunedAxis[kTunedPasses] = {1, 1, 2, 2, 2};
constexpr int kTunedMode[kTunedPasses] = {MODE_FWD, MODE_INV, MODE_FWD, MODE_INV, MODE_FWD_MID_INV};

// Thrown inside the library, caught at the C boundary and turned into a status code.
struct Gp5Error {
    int status;
    std::string msg;
};

void set_last_error(const std::string &msg);
[[noreturn]] void fail(int status, const std::string &msg);
void check_cuda(cudaError_t e, const char *what);

}  // namespace gp5

gp5cu_plan *create_plan(const int shape[3], const double *const *lefts, const double *const *rights, int nsolve,
                        int ncomp, int precision, int device);

struct gp5cu_plan {
    int dev = 0;
    int shape[3] = {0, 0, 0};
    double left[3] = {0, 0, 0}, right[3] = {0, 0, 0};
    int ncomp = 1;
    int prec = GP5_C128;
    long long nsites = 0;  // nx*ny*nz
    int nsolve = 1;              // independent solves of this grid carried by every launch
    long long solve_stride = 0;  // elements between consecutive solves' fields (nsites*ncomp)
    size_t elem_bytes = 16;
    size_t field_bytes = 0;
    double dV = 1.0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    gp5::AxisPlan ax[3];
    void *work = nullptr;                         // one field of FFT workspace
    double *partials = nullptr;
    unsigned *counter = nullptr;
    long long max_blocks = 0;
    gp5::DevScalars *ds = nullptr;         // [nsolve]
    gp5::SolveParams *sp_lap = nullptr;    // [nsolve]: geometry, kinetic factor -1/N^3
    std::vector<gp5::SolveParams> sp_host; // [nsolve]: geometry of every solve
    unsigned long long *dmax = nullptr;
    int pw_blocks = 0;  // grid of the single-solve point-wise kernels
    int pw_bps = 0;     // point-wise blocks per solve
    int sms = 148;      // multiprocessors of the device
    gp5::ProfRec *prof = nullptr;
    bool dry = false;  // launch helpers only configure kernels (before a stream capture)
    // threads per CTA of the register-engine passes along y/z, by [axis][mode] (0: the
    // default rule); chosen by the autotuner when the plan is created
    int tile_threads[3][4] = {};
    // radix schedule (0 or 1, RegCfg) of the register-engine passes along y/z by [axis][mode],
    // and of the stage boundary; chosen by the autotuner, the same for every plan of one
    // (device, grid, components, precision)
    int radix[3][4] = {};
    int radix_boundary = 0;
    // launches of the stepper path use programmatic dependent launch (GP5_PDL=0 turns it off)
    bool pdl = true;
    // the stage boundary takes its tiles in reverse order (GP5_L2ORDER): it then starts on the
    // planes the y inverse pass wrote last, which are still in L2, and the next y forward pass
    // starts on the planes the boundary wrote last (default on)
    bool l2_order = true;
    // the stage boundary reads and writes psi and the k buffers with evict-first cache hints
    // (GP5_STREAM_AUX), so that they do not push the transform buffer out of L2 (default: on
    // for complex64 plans)
    bool stream_aux = false;
    // the merged RK step runs its y/z passes on this many slabs of consecutive x values
    // (GP5_YZ_SLABS; 1: one launch per pass over the whole field)
    int yz_slabs = 1;
    // x range of the strided (y/z) launches being queued: [xr0, xr0 + xr_n), or all when 0
    int xr0 = 0, xr_n = 0;
    // bound of the bulk-copy ring's waits (gp5cu_plan_set_wait_bound)
    unsigned long long ring_wait_ns = GP5_RING_WAIT_DEFAULT_NS;
    // kinetic term of the merged RK step: 0 = 3D transform (y fwd, z fwd*K^2*inv, y inv, x
    // boundary inverse/forward); 1 = per-axis spectral second derivatives (y pass, z pass
    // accumulating, x term inside the boundary; Launch::step_axes).  GP5_KIN_SCHEME.
    int kin_scheme = 0;
};

struct gp5cu_functional {
    gp5cu_plan *plan = nullptr;
    gp5cu_functional_desc desc{};
    std::vector<gp5::SolveParams> sp_host;  // [nsolve]
    gp5::SolveParams *sp = nullptr;         // device copy
};

struct gp5cu_stepper {
    gp5cu_functional *func = nullptr;
    int kind = GP5_STEP_RK4;
    double dt = 0;
    int imaginary = 1;
    double tre = 0, tim = 0;  // complex time step
    bool renorm = false;
    double N[2] = {0, 0};
    void *phase_exp = nullptr;  // e^{i phi}, plan precision, owned
    void *Ka = nullptr, *Kb = nullptr;
    void *dstate = nullptr;  // resident state of the host-buffer entry point
    void *T = nullptr;       // per-axis scheme: the y + z kinetic terms of the stage input
    // compensated complex64 state (gp5cu_stepper_set_compensation): BF16 pairs per element, valid
    // for the state at comp_field; active only without renormalisation and phase constraint
    bool compensate = false;
    // complex64: stochastic rounding of the state update (gp5cu_stepper_set_stochastic_rounding;
    // on by default for complex64 plans)
    bool sround = false;
    void *comp = nullptr;
    void *comp_field = nullptr;
    gp5::DevScalars *ds = nullptr;          // [nsolve]
    std::vector<gp5::SolveParams> sp_host;  // [nsolve]: functional + time step + targets
    gp5::SolveParams *sp = nullptr;
    cudaGraphExec_t exec = nullptr;
    void *graph_field = nullptr;
    bool graph_merged = false;
    int graph_steps = 0;
    // the graphs of the previously stepped fields, most recent first (the device states of
    // the pipelined host-buffer entry point rotate without re-capturing)
    static constexpr int kAltGraphs = 2;
    cudaGraphExec_t exec_alt[kAltGraphs] = {};
    void *graph_field_alt[kAltGraphs] = {};
    bool graph_merged_alt[kAltGraphs] = {};
    int graph_steps_alt[kAltGraphs] = {};
    // pipelined host-buffer entry point: kHostStates device states in rotation (dstate is the
    // first), upload / download streams and their events (created on first use).  A state's
    // buffer is busy for its upload, its steps and its download; with three of them the
    // uploads and downloads run back to back on the copy engines.
    static constexpr int kHostStates = 3;
    void *dstate_more[kHostStates - 1] = {};
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t ev_up[kHostStates] = {}, ev_done[kHostStates] = {}, ev_down[kHostStates] = {};
    double t = 0;
    int launches_per_step = 0;
};

// the compensated update runs for complex64 plans without renormalisation or phase constraint
inline bool compensation_active(const gp5cu_stepper *st) {
    return st->compensate && st->comp && !st->renorm && !st->phase_exp && st->func->plan->prec == GP5_C64;
}

namespace gp5 {

// precision-specific launchers (gp5cu_kernels_f64.cu / gp5cu_kernels_f32.cu)
template <typename Real> struct Launch {
    static void fft(gp5cu_plan *p, const void *src, void *dst, int dir);
    static void laplacian(gp5cu_plan *p, const void *src, void *dst);
    static void apply_h(gp5cu_functional *f, const void *src, void *dst, bool obs);
    static void residual(gp5cu_plan *p, const void *psi, const void *hpsi, DevScalars *ds, const SolveParams *sp);
    static void norm(gp5cu_plan *p, const void *field, int comp, double Ntarget, DevScalars *ds);
    static void scale(gp5cu_plan *p, void *field, int comp, DevScalars *ds, bool from_sigma);
    static void max_density(gp5cu_plan *p, const void *field);
    static void convert(gp5cu_plan *p, const double *in128, void *out, const void *in, double *out128, long long n);
    static int step(gp5cu_stepper *st, void *field);  // queue one step; returns launches
    static int step_merged(gp5cu_stepper *st, void *field, bool prologue);
    static int step_axes(gp5cu_stepper *st, void *field);  // step_merged's per-axis scheme
    static void prologue(gp5cu_stepper *st, void *field);  // forward x transform of psi
    static void phase_exp(gp5cu_plan *p, const void *phase, void *out);
    static void init_gaussian(gp5cu_plan *p, void *field, int comp, const double sigma[3]);
    // one preconditioned gradient iteration of every solve (ground states, single component)
    static void precond_iter(gp5cu_functional *f, const SolveParams *sp_norm, void *psi, void *hbuf, double theta);
    static constexpr int kPrecondLaunches = 11;
    // times every tile shape (and, with radix, both radix schedules) of the strided y/z passes
    // on the zeroed work field, and with radix both schedules of the stage boundary; keeps the
    // fastest in p->tile_threads, p->radix and p->radix_boundary
    static void autotune(gp5cu_plan *p, int nrep, bool radix);
};

void set_scalars(cudaStream_t s, DevScalars *ds, int n = 1);

void build_axis_plan(gp5cu_plan *p, int d);

}  // namespace gp5

// host helpers shared by the single-solve and batched entry points (gp5cu_host.cu)
void fill_functional_params(const gp5cu_plan *p, const gp5cu_functional_desc &d, gp5::SolveParams &S);
void upload_params(const std::vector<gp5::SolveParams> &h, gp5::SolveParams **dptr);
bool merged_path(const gp5cu_plan *p);
void autotune_plan(gp5cu_plan *p, bool force);
int queue_step(gp5cu_stepper *st, void *field, bool merged, bool prologue);
void build_graph(gp5cu_stepper *st, void *field, bool merged, int ksteps);
void capture_graph(gp5cu_stepper *st, void *field, bool merged, int ksteps);
void drop_graph(gp5cu_stepper *st);
