/*
 * gp5cu.h - C ABI of the B200 (sm_100a) pseudo-spectral Gross-Pitaevskii stepper.
 *
 * Plain C: opaque handles, raw pointers and sizes, int status codes.  Every field is a
 * complex array of shape (nx, ny, nz, ncomp) in ColMajor order (x fastest, component
 * slowest), interleaved (re, im): the layout of the reference's
 * tensor_t = Eigen::Tensor<std::complex<double>,4> (src/traits.h:20) and of the numpy
 * F-order view that gpCpp hands to Python (src/pyTools.h:93-104).  Precision GP5_C128
 * stores complex128 (double2), GP5_C64 stores complex64 (float2); reductions are FP64 in
 * both.
 *
 * Device pointers ("d" prefix) must come from cudaMalloc (or gp5cu_field_alloc, or a torch
 * tensor) on the plan's device and be 16-byte aligned.  All work is queued on the plan's
 * stream; calls that return host scalars synchronise that stream.  Calls on one plan (and
 * on its functionals/steppers) are not thread-safe; distinct plans are independent.
 *
 * Each entry point names the reference interface it replaces (file:line in
 * lucaparisi91/GP5).
 */
#ifndef GP5CU_H
#define GP5CU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference throws std::runtime_error; gpCpp rethrows these) ---- */
#define GP5_OK 0
#define GP5_ERR_ARG 1         /* invalid argument (shape, pointer, kind, size) */
#define GP5_ERR_CUDA 2        /* a CUDA runtime call failed; see gp5cu_last_error */
#define GP5_ERR_NONFINITE 3   /* a reduction met NaN/Inf (norm blow-up) */
#define GP5_ERR_TIMEOUT 4     /* a bounded device wait ran out */
#define GP5_ERR_UNSUPPORTED 5 /* size/radix/feature not supported */
#define GP5_ERR_STATE 6       /* object used in the wrong state */
#define GP5_ERR_NOMEM 7       /* device allocation failed */
#define GP5_ERR_IO 8          /* a file could not be read or written, or is malformed */

/* ---- enums ---- */
#define GP5_C128 0 /* complex128 bulk arithmetic */
#define GP5_C64 1  /* complex64 bulk arithmetic, FP64 reductions */

#define GP5_FORWARD (-1) /* e^{-2 pi i jk/n}, FFTW_FORWARD */
#define GP5_BACKWARD 1   /* e^{+2 pi i jk/n}, FFTW_BACKWARD, unnormalised */

#define GP5_FUNC_GP 0           /* gpFunctional (src/functional.cpp:13-102) */
#define GP5_FUNC_LHY 1          /* LHYDropletFunctional (src/functional.cpp:105-122) */
#define GP5_FUNC_LHY_UNLOCKED 2 /* LHYDropletUnlockedFunctional (src/functional.cpp:125-150) */

#define GP5_POT_NONE 0
#define GP5_POT_HARMONIC 1 /* harmonicPotential (src/externalPotential.cpp:11-32) */
#define GP5_POT_ARRAY 2    /* potentialFromFile / sumPotential: caller's real array */

#define GP5_STEP_EULER 0 /* euleroStepper (src/stepper.cpp:30-44) */
#define GP5_STEP_RK4 1   /* RK4Stepper (src/stepper.cpp:46-82) */

typedef struct gp5cu_plan gp5cu_plan;
typedef struct gp5cu_functional gp5cu_functional;
typedef struct gp5cu_stepper gp5cu_stepper;

/* Library version (major*10000 + minor*100 + patch) and a message for a status code. */
int gp5cu_version(void);
const char *gp5cu_status_string(int status);
/* Last error message recorded on this thread (empty when none). */
const char *gp5cu_last_error(void);

/* ---- discretisation + FFT plan ----------------------------------------------------------
 * Replaces fourierTransformCreator::create (src/fourierTransform.cpp:227-249), the
 * fftwFourierTransform constructor/plan (src/fourierTransform.cpp:129-181) and
 * createUniformDiscretization for one rank (src/geometry.cpp:56-105).  shape = {nx,ny,nz};
 * left/right = domain corners (gp::domain, src/geometry.h:41-65).  Any axis length in
 * [2, 4096] whose prime factors are <= 61 is accepted.  device = CUDA ordinal. */
int gp5cu_plan_create(gp5cu_plan **out, const int shape[3], const double left[3],
                      const double right[3], int ncomp, int precision, int device);
int gp5cu_plan_destroy(gp5cu_plan *plan);
/* Queue all subsequent work of this plan on a caller stream (cudaStream_t); NULL = the
 * plan's own stream. */
int gp5cu_plan_set_stream(gp5cu_plan *plan, void *cuda_stream);
int gp5cu_plan_synchronize(gp5cu_plan *plan);
/* Bytes of one field (nx*ny*nz*ncomp complex elements of the plan's precision). */
size_t gp5cu_field_bytes(const gp5cu_plan *plan);
int gp5cu_field_alloc(gp5cu_plan *plan, void **dfield);
int gp5cu_field_free(gp5cu_plan *plan, void *dfield);
/* Host <-> device copies of one field in the plan precision (field::setTensor /
 * field::getTensor, src/gpCpp.cpp:97-102; pyTools.h:12-56,68-105). */
int gp5cu_upload(gp5cu_plan *plan, void *dfield, const void *host);
int gp5cu_download(gp5cu_plan *plan, const void *dfield, void *host);
/* Complex128 host data into a plan of either precision (converts on the device). */
int gp5cu_upload_c128(gp5cu_plan *plan, void *dfield, const double *host_c128);
int gp5cu_download_c128(gp5cu_plan *plan, const void *dfield, double *host_c128);

/* ---- transforms and operators -------------------------------------------------------- */
/* fourierTransform::apply(src, dst, FORWARD|BACKWARD) (src/fourierTransform.h:23;
 * fftwFourierTransform::apply src/fourierTransform.cpp:184-214): unnormalised 3D C2C of
 * every component, k-space in natural order.  src == dst is allowed. */
int gp5cu_fft(gp5cu_plan *plan, const void *dsrc, void *ddst, int direction);
/* operators::laplacian::apply (src/operators.cpp:28-36): dst = IFFT(-K^2 FFT(src)) / N^3. */
int gp5cu_laplacian(gp5cu_plan *plan, const void *dsrc, void *ddst);
/* gp::norm (src/geometry.cpp:190-214): dV * sum |psi_c|^2, FP64. */
int gp5cu_norm(gp5cu_plan *plan, const void *dfield, int comp, double *out);
/* gp::normalize (src/geometry.cpp:217-229): psi_c *= sqrt(N / norm_c). */
int gp5cu_normalize(gp5cu_plan *plan, void *dfield, int comp, double N);
/* gp::initGaussian (src/geometry.cpp:251-276): psi_comp = exp(-sum_d x_d^2 / (2 sigma_d^2)) + 0i
 * at the cell centres; the other components are left as they are.  Single-solve plans. */
int gp5cu_init_gaussian(gp5cu_plan *plan, void *dfield, int comp, const double sigma[3]);
/* gp.maxDensity (python/gp/gp.py:210-222): max |psi|^2 over all sites and components. */
int gp5cu_max_density(gp5cu_plan *plan, const void *dfield, double *out);

/* ---- functionals ---------------------------------------------------------------------- */
typedef struct gp5cu_functional_desc {
    int kind;              /* GP5_FUNC_* */
    int has_couplings;     /* gpFunctional::setCouplings was called (functional.h:59) */
    double couplings[4];   /* g(i,j) at [i*2+j]; 1 component uses [0] */
    double masses[2];      /* gpFunctional::setMasses (default 1) */
    double c3, c4;         /* LHY: H = -1/2 lap + (c3 n + c4 n^{3/2}); reference -3, 5/2 */
    double alpha, beta, eta; /* unlocked LHY constants */
    int potential;         /* GP5_POT_* */
    double omegas[2][3];   /* harmonic trap frequencies per component */
    const void *dpotential; /* GP5_POT_ARRAY: real array (nx,ny,nz,ncomp), double for
                               GP5_C128 / float for GP5_C64, device memory, not copied */
} gp5cu_functional_desc;

/* Fills the reference defaults: LHY, c3 = -3, c4 = 5/2, masses 1, no potential. */
void gp5cu_functional_desc_init(gp5cu_functional_desc *desc);
/* functionalConstructor::create (src/functional.cpp:154-258) and the gpCpp LHY model
 * (src/gpCpp.cpp:151-199). */
int gp5cu_functional_create(gp5cu_plan *plan, const gp5cu_functional_desc *desc,
                            gp5cu_functional **out);
int gp5cu_functional_destroy(gp5cu_functional *func);
/* functional::apply(old, new, t) (src/functional.h:15; model::apply src/gpCpp.cpp:167-171):
 * dst = H src.  src != dst. */
int gp5cu_apply_H(gp5cu_functional *func, const void *dsrc, void *ddst);

typedef struct gp5cu_observables_t {
    double norm;     /* dV sum |psi|^2 (all components) */
    double energy;   /* E = ekin + epot + eint */
    double ekin;     /* dV Re sum conj(psi) T psi, T = -1/2 (1/m) lap */
    double epot;     /* dV sum V |psi|^2 */
    double eint;     /* dV sum e_int(n); GP (g/2) n^2, LHY (c3/2) n^2 + (2 c4/5) n^{5/2} */
    double mu;       /* Re <psi|H psi> / <psi|psi> */
    double residual; /* ||H psi - mu psi|| / ||psi|| */
} gp5cu_observables_t;
/* Energy, chemical potential and residual (no reference counterpart: the reference only
 * estimates mu from the norm decay, python/test/regressionTests/LHY_imaginary.py:48). */
int gp5cu_observables(gp5cu_functional *func, const void *dfield, gp5cu_observables_t *out);

/* ---- steppers ------------------------------------------------------------------------
 * timeStepper (src/gpCpp.cpp:202-287) over euleroStepper / RK4Stepper
 * (src/stepper.cpp:30-82).  imaginary != 0: time step (dt, 0); else (0, dt)
 * (src/gpCpp.cpp:217-224). */
int gp5cu_stepper_create(gp5cu_functional *func, int kind, double dt, int imaginary,
                         gp5cu_stepper **out);
int gp5cu_stepper_destroy(gp5cu_stepper *st);
/* timeStepper::setRenormalization / unsetRenormalization (src/gpCpp.cpp:243-253); n = 0
 * disables.  N[c] = target norm of component c. */
int gp5cu_stepper_set_renormalization(gp5cu_stepper *st, int n, const double *N);
/* phaseConstraint (src/constraint.cpp:6-17): psi <- |psi| e^{i phi} after each step;
 * dphase = real array (nx,ny,nz,ncomp) in the plan precision, device memory; NULL = the
 * nullConstraint (src/constraint.h:15-21). */
int gp5cu_stepper_set_phase_constraint(gp5cu_stepper *st, const void *dphase);
/* No reference counterpart.  Compensated state update for complex64 plans: the stepper keeps
 * the part of psi below FP32 resolution in a BF16 pair per element and folds it into every
 * step's update (two-sum), so increments far below the state's last bit are not lost (the
 * source of complex64's norm and energy drift at small time steps).  Costs 8 bytes per site per
 * step.  Active only without renormalisation and phase constraint; the correction restarts from
 * zero when advance is given another state buffer (or a new host state).  on = 0 frees it. */
int gp5cu_stepper_set_compensation(gp5cu_stepper *st, int on);
/* No reference counterpart.  Stochastic rounding of the complex64 state update: the new state
 * p - d sum of the last RK4 stage (or of Euler) is rounded to one of its two neighbouring
 * floats with probabilities that make the rounding unbiased (the exact rounding error, from a
 * two-sum, against a reproducible hash of the element index and the element's values), so
 * the sub-resolution part of small increments is kept on average instead of being lost with a
 * consistent sign.  No extra memory traffic (about 2% more time); results are deterministic,
 * and a batched solve rounds as it does alone.  On by default for complex64 steppers; where
 * the compensated update is active it takes precedence.  on = 1 needs a complex64 plan; on = 0
 * restores round-to-nearest. */
int gp5cu_stepper_set_stochastic_rounding(gp5cu_stepper *st, int on);
/* timeStepper::advance(field, nSteps) (src/gpCpp.cpp:255-269): nsteps steps in place on a
 * device field; t += dt per step.  The step sequence is replayed from a CUDA graph. */
int gp5cu_stepper_advance(gp5cu_stepper *st, void *dfield, int nsteps);
/* timeStepper::getTime (src/gpCpp.cpp:273). */
int gp5cu_stepper_get_time(const gp5cu_stepper *st, double *t);
int gp5cu_stepper_set_time(gp5cu_stepper *st, double t);
/* Host-buffer form of advance for callers that keep the field in host memory (the
 * reference's Eigen tensor): upload, nsteps steps, download, on the plan stream.
 * host_in and host_out may alias. */
int gp5cu_stepper_advance_host(gp5cu_stepper *st, const void *host_in, void *host_out,
                               int nsteps);
/* The same for nstates independent host states (an ensemble, or states a caller streams
 * through the GPU): state i is uploaded from host_in[i], advanced nsteps steps and downloaded
 * to host_out[i].  Three device states rotate, with uploads and downloads on their own
 * streams, so the upload of state i+1 and the download of state i-1 overlap the steps of
 * state i and each other (pinned host buffers are needed for the copies to overlap).  host_in[i] and
 * host_out[i] may alias; states that share an output buffer overwrite it in order.  The stepper's time
 * advances by nsteps steps once.  Single-solve plans only.  No reference counterpart (the
 * reference keeps one state per process). */
int gp5cu_stepper_advance_host_many(gp5cu_stepper *st, int nstates, const void *const *host_in,
                                    void *const *host_out, int nsteps);
/* Kernel launches one step issues (for launch accounting). */
int gp5cu_stepper_launches_per_step(const gp5cu_stepper *st);
/* Diagnostics (no reference counterpart; the reference's "step"/"FFT" timers,
 * src/timers.h:112-113, are its nearest analogue): runs nrep eager steps with a CUDA event
 * after every kernel launch and returns the mean duration of each launch of one step in
 * ms[i] (milliseconds) with its kind in kinds[i] (axis*10 + mode: mode 0 forward, 1 inverse,
 * 2 forward*K^2*inverse; 90 = point-wise kernel).  *nlaunch = launches per step; at most cap
 * entries are written. */
int gp5cu_stepper_profile(gp5cu_stepper *st, void *dfield, int nrep, double *ms, int *kinds, int cap,
                          int *nlaunch);

/* ---- batched independent ground-state solves ---------------------------------------------
 * No reference counterpart (the reference runs one solve per process; its imaginary-time
 * protocol is python/test/regressionTests/LHY_imaginary.py).  Many LHY droplet solves, each
 * on its own cubic grid, box, atom number, coefficients and time step, advance together:
 * solves of the same grid size share every kernel launch (one launch per pass covers all of
 * them), the steps between convergence checks replay from CUDA graphs, and solves that reach
 * the residual tolerance stop: at the next check the solves still running are packed into
 * the first slots of their group and the launches shrink to them, so a long tail of slow
 * solves does not pay for the finished ones.
 * precision GP5_C64: every solve first runs with complex64 transforms and state (FP64
 * reductions) until its residual is at most GP5_BATCH_SWITCH_RESIDUAL or stops falling near
 * the complex64 floor (rounding of the FP32 state, amplified by the kinetic operator, keeps
 * the residual above about 1e-6); the state is then converted to complex128 and the solve
 * continues in complex128 to `tol`. */
#define GP5_BATCH_SWITCH_RESIDUAL 1e-5
typedef struct gp5cu_batch gp5cu_batch;

typedef struct gp5cu_solve_desc {
    int n;          /* grid points per axis (n^3 grid); power of two in [32, 512] */
    double L;       /* box [-L/2, L/2]^3 */
    double N;       /* atom number: the state is renormalised to it every step */
    double c3, c4;  /* H = -1/2 lap + (c3 n + c4 n^{3/2}) + V */
    double omega;   /* isotropic harmonic trap V = omega^2 r^2 / 2 (0: none) */
    double dt;      /* imaginary time step */
} gp5cu_solve_desc;

typedef struct gp5cu_solve_result {
    int steps;        /* RK4 steps taken (0 if the initial state already met tol) */
    int converged;    /* residual <= tol */
    double residual;  /* ||H psi - mu psi|| / ||psi|| at the last check */
    double energy, mu, norm;
    int steps_c64;    /* of `steps`, those taken in complex64 (GP5_C64 batches; 0 otherwise) */
} gp5cu_solve_result;

int gp5cu_batch_create(gp5cu_batch **out, int nsolves, const gp5cu_solve_desc *solves, int precision,
                       int device);
/* The same over several GPUs of one process: the solves are split by index over `devices`
 * (gp5cu_batch_assign_devices) and every device runs its own groups; the solves are
 * independent, so nothing moves between devices (no collective, no peer access).  One host
 * thread drives all devices: their launches are asynchronous, so the devices work at once
 * and the host waits for each at the convergence checks. */
int gp5cu_batch_create_devices(gp5cu_batch **out, int nsolves, const gp5cu_solve_desc *solves, int precision,
                               int ndevices, const int *devices);
/* The split used by gp5cu_batch_create_devices, computed on the host only: solves in order of
 * decreasing grid sites (ties by index), each to the device position with the fewest sites so
 * far (ties to the lower position).  device_index[i] receives a position in [0, ndevices). */
int gp5cu_batch_assign_devices(int nsolves, const gp5cu_solve_desc *solves, int ndevices, int *device_index);
/* Device ordinal of one solve (-1 for a bad argument). */
int gp5cu_batch_device(const gp5cu_batch *b, int solve);
int gp5cu_batch_destroy(gp5cu_batch *b);
/* Initial / current state of one solve, complex128 host data of n^3 elements. */
int gp5cu_batch_set_state(gp5cu_batch *b, int solve, const double *host_c128);
int gp5cu_batch_get_state(gp5cu_batch *b, int solve, double *host_c128);
/* Imaginary-time RK4 of every solve until residual <= tol (checked every check_every steps)
 * or max_steps; results[i] per solve.  Returns GP5_OK even if some solves did not converge. */
int gp5cu_batch_solve(gp5cu_batch *b, double tol, int check_every, int max_steps,
                      gp5cu_solve_result *results);
/* Method of the following gp5cu_batch_solve calls.  No reference counterpart (the reference
 * reaches ground states only by imaginary-time stepping).
 * GP5_BATCH_RK4 (the default): renormalised imaginary-time RK4 with each solve's dt.
 * GP5_BATCH_PRECOND: preconditioned gradient iteration towards the same ground state,
 *   psi <- normalise_N(psi - theta (alpha - 1/2 lap)^{-1} (H psi - mu psi)),
 * mu = <psi|H psi>/<psi|psi> and alpha = max(|mu|, 0.05, Vmax/2) per solve (Vmax: the trap's
 * potential at the farthest cell centre, 0 without a trap), the shifted inverse kinetic
 * operator applied in k-space; its fixed point (zero residual at norm N) is the one imaginary
 * time converges to, and it takes tens of iterations where imaginary time takes thousands of
 * steps (each iteration costs about half an RK4 step: eleven launches).  The dt of the solve
 * descriptors is not used; gp5cu_solve_result.steps counts iterations.  theta in (0, 1]; 0.5
 * converges on the droplets of N in [20, 2000], c3 in [-3.2, -2.8]. */
#define GP5_BATCH_RK4 0
#define GP5_BATCH_PRECOND 1
int gp5cu_batch_set_method(gp5cu_batch *b, int method, double theta);
/* Kernel launches of the last gp5cu_batch_solve call. */
long long gp5cu_batch_launches(const gp5cu_batch *b);

/* ---- droplet decomposition --------------------------------------------------------------
 * gp::decompose::decompose (src/cluster.cpp:17-83) behind the gpCpp `decomposition` class
 * (src/gpCpp.cpp:289-313): labels (int32, the field's layout (nx, ny, nz, ncomp)) of the
 * connected components of the sites of component `comp` with |psi|^2 > cutoff, 26-connected,
 * periodic; sites at or below the cutoff get -1, the other components 0; clusters are numbered
 * from 1 in the order in which a scan over (i, j, k), i slowest, meets their first site.
 * *nclusters receives their number.  Plans of one solve only.  dlabels: device memory;
 * gp5cu_decompose_host writes host memory (and allocates a device label buffer for the call). */
int gp5cu_decompose(gp5cu_plan *plan, const void *dfield, int comp, double cutoff, int *dlabels, int *nclusters);
int gp5cu_decompose_host(gp5cu_plan *plan, const void *dfield, int comp, double cutoff, int *labels,
                         int *nclusters);

/* ---- learned warm start ------------------------------------------------------------------
 * No counterpart in the reference, which starts every solve from a Gaussian
 * (python/test/regressionTests/LHY_imaginary.py:14).  A 3 -> 256 -> 256 -> 256 -> 64 MLP with
 * GELU hidden layers maps solve parameters to radial samples of the ground state.  Its GEMMs
 * are tcgen05 tensor-core kernels with BF16 operands and FP32 accumulation; parameters are
 * kept in FP32 (Adam's master copy) and used as BF16.
 * Parameter vector layout (gp5cu_mlp_num_params floats): for each layer l, W_l row-major
 * [fan_out][fan_in], then b_l [fan_out].  Inputs x are [B][3] and outputs/targets [B][64],
 * row-major FP32 host arrays. */
typedef struct gp5cu_mlp gp5cu_mlp;
int gp5cu_mlp_create(gp5cu_mlp **out, int device, unsigned long long seed);
int gp5cu_mlp_destroy(gp5cu_mlp *net);
long long gp5cu_mlp_num_params(const gp5cu_mlp *net);
int gp5cu_mlp_get_params(gp5cu_mlp *net, float *host);
int gp5cu_mlp_set_params(gp5cu_mlp *net, const float *host);
/* inference of B samples: y[B][64] */
int gp5cu_mlp_forward(gp5cu_mlp *net, const float *x, int B, float *y);
/* gradient of the loss sum((y - t)^2) / (B * 64) with respect to every parameter (same layout
 * as the parameter vector) and the loss itself */
int gp5cu_mlp_gradients(gp5cu_mlp *net, const float *x, const float *t, int B, float *grad, double *loss);
/* Adam (beta1 0.9, beta2 0.999, eps 1e-8) over `epochs` seeded shuffles of the `count`
 * samples in mini-batches of `batch` (a trailing partial batch is skipped);
 * loss_history[epoch] (may be NULL) receives each epoch's mean loss. */
int gp5cu_mlp_train(gp5cu_mlp *net, const float *x, const float *t, int count, int epochs, int batch, float lr,
                    unsigned long long seed, float *loss_history);
/* C[m*ldc + n] = sum_k A(m,k) B(n,k), A(m,k) = A[m*sam + k*sak], B(n,k) = B[n*sbn + k*sbk]:
 * BF16 device operands, FP32 device result, on `stream` (cudaStream_t or NULL; synchronised) */
int gp5cu_gemm_bf16(const void *A, long long sam, long long sak, const void *B, long long sbn, long long sbk,
                    float *C, long long ldc, int M, int N, int K, void *stream);
/* Bound of the tensor-core GEMMs' device-side wait for each K chunk's MMAs, for the net's
 * later calls (default GP5_GEMM_WAIT_DEFAULT_NS = 2 s).  When a wait runs out, the CTA stops,
 * waits (with the fixed 2 s bound) for the MMAs it issued, frees its tensor memory and flags
 * the error; the call then returns GP5_ERR_TIMEOUT and the net stays usable.  A bound of 0
 * fails every wait whose MMAs have not completed at the first probe (used to test the path). */
#define GP5_GEMM_WAIT_DEFAULT_NS 2000000000ULL
int gp5cu_mlp_set_wait_bound(gp5cu_mlp *net, unsigned long long ns);

/* ---- tile-shape and radix autotuner -------------------------------------------------------
 * No reference counterpart (FFTW plans its own transforms).  The strided y/z passes of the
 * register engine (axis lengths 32..512, powers of two) come in tile shapes of 128, 256 or 512
 * threads per CTA (more threads = more consecutive x values per tile = wider coalesced rows),
 * and every register-engine pass along y/z, and the stage boundary along x, in two radix
 * schedules (0: e.g. radix 16 x 16 at 256 with 16 elements per thread; 1: e.g. 8 x 8 x 4 with 8
 * elements per thread, fewer registers, more resident CTAs).  gp5cu_plan_create times both
 * schedules and every shape of the five passes below, and both schedules of the boundary, on
 * the plan's zeroed work field and keeps the fastest.  The schedules round differently (at the
 * level of the last bit), so they are chosen once per (device, grid, components, precision)
 * and every later plan of that grid uses them whatever its number of solves; the thread
 * counts change no result bit and are tuned per number of solves.  Choices are remembered for
 * the life of the process and in a JSON file (GP5_AUTOTUNE_CACHE).  GP5_AUTOTUNE=0 keeps the
 * default shapes and schedule 0; GP5_RADIX=0|1 fixes the schedules.
 * threads[5]: y forward, y inverse, z forward, z inverse, z forward*K^2*inverse; 0 = the
 * default shape (or an axis that uses the shared-memory engine).  radix[6]: the schedules of
 * the same five passes, then the stage boundary's choice: bit 0 its schedule, bit 1 its operand
 * feed (0: register loads, one tile per CTA; 1: the bulk-copy ring, one persistent CTA per SM
 * whose tiles' streams arrive by cp.async.bulk into a ring of shared-memory stages while the
 * previous tile transforms; where the ring has no tile shape for the schedule, or for the
 * compensated complex64 update, the register-load kernel runs).  The autotuner times all four
 * boundary choices.  Steppers capture these choices in their CUDA graphs when they first
 * advance: set them before creating steppers. */
int gp5cu_plan_autotune(gp5cu_plan *plan);
int gp5cu_plan_get_tiles(const gp5cu_plan *plan, int threads[5]);
int gp5cu_plan_set_tiles(gp5cu_plan *plan, const int threads[5]);
int gp5cu_plan_get_radix(const gp5cu_plan *plan, int radix[6]);
int gp5cu_plan_set_radix(gp5cu_plan *plan, const int radix[6]);
/* Bound of the bulk-copy ring's device-side wait for a stage's copies (default
 * GP5_RING_WAIT_DEFAULT_NS = 2 s), for launches queued or captured afterwards.  When a wait
 * runs out, the CTA stops taking tiles, waits (with the fixed 2 s bound) for the copies it
 * issued and flags DS_TIMEOUT: the stepper call then returns GP5_ERR_TIMEOUT and the plan
 * stays usable.  A bound of 0 fails every wait whose copies have not landed at the first probe
 * (used to test the path). */
#define GP5_RING_WAIT_DEFAULT_NS 2000000000ULL
int gp5cu_plan_set_wait_bound(gp5cu_plan *plan, unsigned long long ns);

/* ---- HDF5 field files ----------------------------------------------------------------------
 * The reference's on-disk format, read and written without libhdf5 (host only, no GPU):
 * gp::save / gp::load (src/io.cpp:56-152, 154-256), bound as field.save / field.load
 * (src/gpCpp.cpp:105-118, 343-344).  One dataset "field" in the root group, element
 * H5Tarray(double, [2]) (src/io.cpp:45), dims [nComp][Nz][Ny][Nx], contiguous; its raw data is
 * the field's memory order (x fastest, components slowest), so host_c128 is the same buffer
 * gp5cu_upload / gp5cu_download use.  save writes superblock 0, version-1 object headers and a
 * symbol-table root group; load also reads superblocks 0-3 (with a user block), version-2
 * object headers, link-message groups and complex elements stored as a compound of two
 * doubles, from contiguous or compact storage.  Errors: GP5_ERR_IO (file), GP5_ERR_ARG (no
 * "field" dataset, or a shape other than the one requested), GP5_ERR_UNSUPPORTED (chunked,
 * filtered or dense-link storage). */
int gp5cu_h5_save_field(const char *path, const double *host_c128, const int shape[3], int ncomp);
int gp5cu_h5_field_shape(const char *path, int shape[3], int *ncomp);
int gp5cu_h5_load_field(const char *path, double *host_c128, const int shape[3], int ncomp);
/* Any float64 dataset of the root group: its rank, dims (slowest first, at most 8) and whether
 * its element is complex (two doubles); then its values as doubles (count = product of dims,
 * times 2 when complex). */
int gp5cu_h5_dataset_info(const char *path, const char *name, int *rank, long long dims[8], int *complex_elems);
int gp5cu_h5_read_dataset(const char *path, const char *name, double *out, long long count);

/* ---- allocation-free norm ---------------------------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc when they need
 * a norm (their device memory belongs to another allocator, or the device is full): the same
 * value as gp5cu_norm, dV * sum |psi_comp|^2, computed without a plan and without allocating.
 * Its scratch (block partial sums, a ticket, the result slot) is a file-scope static device
 * array of 33,024 bytes that every GPU loading the library keeps until the process exits.
 * Limit: at most GP5_NOALLOC_MAX_SITES sites (256^3); larger fields return GP5_ERR_ARG.
 * dfield: device field (shape[0]*shape[1]*shape[2] sites, ncomp components, `precision`) on
 * the current device, 16-byte aligned for GP5_C128 and 8-byte aligned for GP5_C64; stream:
 * cudaStream_t or NULL; *out receives the norm (host): the call reads it back and
 * synchronises `stream` before it returns.  The first call on a device (and the first after
 * its CUDA context is re-created) looks up the scratch address (cudaGetSymbolAddress): make
 * it before any stream capture.  Calls share the scratch, so calls that overlap on the GPU
 * race. */
#define GP5_NOALLOC_MAX_SITES 16777216LL
int gp5cu_norm_noalloc(const void *dfield, int precision, const int shape[3], int ncomp, int comp,
                       double dV, void *stream, double *out);

#ifdef __cplusplus
}
#endif

#endif /* GP5CU_H */
