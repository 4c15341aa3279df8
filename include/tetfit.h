/*
 * tetfit.h -- C ABI of the B200-native TetFIT leapfrog time-stepping path.
 *
 * The entry points replace the two calls a TetFIT driver makes
 * (src/DGA/main/dga_main.cpp:52-62):
 *   Discretization(std::string inputfile)            Discretization.hpp:45-211
 *   RunSimulation(const Simulation&, const uint32_t&) Discretization.hpp:289-2303
 * and expose the hot loop stepwise so that a caller can drive it, sample it and
 * read the state back.  All buffers passed in are host memory owned by the
 * caller; device memory is owned by the context.  Every function returns 0 on
 * success or a negative TF_E* code; tf_last_error() gives the message (for
 * script errors the reference's own text, "Input file error at line N: ...",
 * Utilities.hpp:371-375).  One context per host thread; a context is not
 * re-entrant.  Nothing throws across this boundary.
 */
#ifndef TETFIT_H
#define TETFIT_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TF_API __attribute__((visibility("default")))
#else
#define TF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tf_ctx tf_ctx;

enum {
  TF_OK = 0,
  TF_E_SCRIPT = -1,      /* script / mesh / solids file error (MyThrow text)        */
  TF_E_ARG = -2,         /* bad argument, unknown simulation label, buffer too small */
  TF_E_CUDA = -3,        /* CUDA runtime error or no usable sm_100 device           */
  TF_E_UNSUPPORTED = -4, /* feature outside the time-stepping path (e.g. PML)         */
  TF_E_STATE = -5,       /* call out of order (e.g. tf_step before tf_prepare)       */
  TF_E_SOLVER = -6       /* iterative solve hit its iteration limit                 */
};

enum { TF_FP64 = 0, TF_FP32 = 1 };

typedef struct tf_opts {
  int32_t precision;    /* TF_FP64 (default) or TF_FP32 field state                     */
  int32_t device;       /* CUDA device ordinal                                          */
  int32_t write_files;  /* tf_run: write <name><label>_probe_E/H.dat (probepoint) or one
                           <name><label>_<dump>.tfd per print time (silo, tets), and
                           poynting.dat                                            */
  int32_t verbose;      /* print the reference's parameter banner and stats            */
  int32_t graph_steps;  /* steps per captured CUDA graph (0: automatic)                */
  int32_t mass_model;   /* gfdtd eps-mass: 0 as the reference builds it, 1 consistent  */
  int32_t warm_start;   /* gfdtd CG guess: 0 previous solution (reference), 1 zero,
                           2 polynomial extrapolation, 3 learned per-edge MLP        */
  int32_t cg_criterion; /* 0 ||r||/||r0|| <= tol (reference), 1 ||r|| <= tol ||b||   */
  int32_t cg_maxiter;   /* 0: 100, the reference's limit                             */
  int32_t batch_mode;   /* tf_batch_open: 0 all members advance together in one
                           group, 1 each member alone (one after another)       */
  int32_t host_threads; /* host threads of the set-up (tf_prepare, tf_batch_open), 0 all */
  int32_t learn_steps;  /* warm_start 3: steps whose solutions train the network
                           (0: 500); the extrapolation is used meanwhile         */
  int32_t fit_variant;  /* fdtd: 0 automatic (first steps time the variants on grids
                           of 2 M cells or more), k > 0 forces variant k - 1 for
                           both halves (all give bitwise identical results)     */
  int32_t file_digits;  /* tf_run: significant digits of the probe files (0: 6, the
                           reference's default stream precision; 17 round-trips) */
  int32_t reserved[2];
} tf_opts;

typedef struct tf_info {
  uint64_t n_edges, n_faces, n_cells;  /* dofs: edges (U) and faces (B)           */
  uint64_t n_probes, n_steps;          /* probes inside the mesh; loop length     */
  uint64_t step_index;                 /* steps already taken                     */
  uint32_t nx, ny, nz;                 /* Cartesian cells per axis (0 for tets)   */
  int32_t method;                      /* 0 fdtd, 1 dga, 2 gfdtd, 3 fem           */
  double dt, dt_estimate;              /* step used; courant x stability estimate */
  int32_t possibly_unstable;           /* SET step exceeded the estimate          */
  int32_t precision;
  uint64_t device_bytes;               /* device memory held by the context       */
  uint32_t kernels_per_step;           /* kernel launches one leapfrog step makes */
  uint32_t n_sources;                  /* sources of the simulation (label order) */
  uint64_t n_free, nnz_system;         /* gfdtd: CG unknowns and nonzeros of A    */
  uint64_t nnz_operators;              /* nonzeros of H (dga) or of E (gfdtd)     */
  uint32_t cg_blocks;                  /* gfdtd: blocks of the persistent CG kernel */
  int32_t cg_variant;                  /* gfdtd: CG variant the autotuner picked;
                                          fdtd: E variant + 8 x H variant (0 one
                                          thread per node, 1/2 z-march over 4/16
                                          planes, 3 per-dof coefficient arrays,
                                          4 z-march with TMA-staged planes,
                                          5 coefficient classes)               */
  uint64_t reserved[3];
} tf_info;

/* Parse a .fdtd script (Discretization(std::string), Discretization.hpp:45-211). */
TF_API int tf_open(const char* fdtd_path, tf_ctx** out);
/* The parsed script as canonical JSON (no reference counterpart: the parsed
 * primitives of Discretization.hpp:45-211 made visible): materials, bcs,
 * meshes, sources, simulations and outputs by ascending label with doubles to
 * 17 significant digits, the 100-slot surface-to-bc table, and the solids of
 * each cartesian mesh file.  *len receives the size needed including the
 * terminating 0; a smaller non-zero cap returns TF_E_ARG with the text cut. */
TF_API int tf_script_dump(tf_ctx* ctx, char* buf, size_t cap, size_t* len);
/* Simulation labels in ascending order (the order dga_main.cpp:52-62 runs them). */
TF_API int tf_simulations(tf_ctx* ctx, uint32_t* labels, uint32_t cap, uint32_t* n);
/* Build mesh, operators and device state for one simulation
 * (RunSimulation up to the time loop, Discretization.hpp:289-428, 4347-5690). */
TF_API int tf_prepare(tf_ctx* ctx, uint32_t sim_label, const tf_opts* opts);
TF_API int tf_get_info(tf_ctx* ctx, tf_info* info);
/* Advance up to nsteps leapfrog steps (Discretization.hpp:1840-1933). */
TF_API int tf_step(tf_ctx* ctx, uint64_t nsteps, uint64_t* done);
/* Probe series so far: times[n], values[n][n_probes][6] = Ex Ey Ez Hx Hy Hz
 * (ExportFitFields, Discretization.hpp:3096-3158).  *n_samples is always set.
 * In silo mode on tets every tet is a probe, at its barycentre, in tet order
 * (the per-tet E and H of the reference's Silo export, :2601-2677). */
TF_API int tf_get_probes(tf_ctx* ctx, double* times, double* values, size_t cap_samples, size_t* n_samples);
/* Probe coordinates [n_probes][3] and containing cell index (reference numbering). */
TF_API int tf_get_probe_points(tf_ctx* ctx, double* xyz, uint64_t* cells, size_t cap);
/* Field state in the reference's numbering: U[n_edges], B[n_faces], F[n_faces]
 * (any pointer may be NULL).  Values are converted to double. */
TF_API int tf_get_state(tf_ctx* ctx, double* U, size_t nU, double* B, size_t nB, double* F, size_t nF);
/* Overwrite U and F (reference numbering); B is derived as F / M_nu on the H grid. */
TF_API int tf_set_state(tf_ctx* ctx, const double* U, size_t nU, const double* F, size_t nF);
/* Per-step boundary flux 0.5 (U_old + U) . curl_fb (Discretization.hpp:1901). */
TF_API int tf_get_flux(tf_ctx* ctx, double* flux, size_t cap, size_t* n);
/* Per-step Joule loss, the third column of poynting.dat: 0.25 (U_old + U)^T
 * Si (U_old + U) (fdtd, Discretization.hpp:1902; dga :895; gfdtd :1519).  As
 * in the reference, the fdtd conductance vector Si is filled only for l2norm
 * outputs (:5368, :5594-5597), so the loss is zero for other outputs; gfdtd
 * and fem give the reference's list (:1518-1546, :1733-1757) with
 * conducting materials; dga never fills its SigMat, so its loss is zero.
 * FP64 accumulation on the GPU. */
TF_API int tf_get_losses(tf_ctx* ctx, double* losses, size_t cap, size_t* n);
/* Discrete leapfrog energy of the current state (U^n, F^{n+1/2}) in FP64
 * accumulation: fdtd 0.5 U^n.Me.U^n + 0.5 F^{n+1/2}.Mmu.F^{n-1/2} (F^{n-1/2}
 * recomputed from U^n); gfdtd 0.5 U^n.E.U^n + 0.5 B^{n-1/2}.N.B^{n+1/2} over the
 * free edges (B^{n+1/2} recomputed); dga 0.5 U^n.H^-1.U^{n+1} +
 * 0.5 B^{n+1/2}.N.B^{n+1/2} over the class-1 edges (U^{n+1} - U^n = dt H cf
 * from the current F; H^-1 U^n by a GPU PCG solve to 1e-15).  All are
 * invariants of the lossless leapfrog once the sources are off.  fem, and dga
 * with conducting or magnetically lossy materials, return TF_E_UNSUPPORTED. */
TF_API int tf_energy(tf_ctx* ctx, double* energy);
/* One step driven from host memory: carrier_in[n_sources] replaces the script
 * waveform's value for this step (NULL keeps it); probe_out[n_probes*6]
 * receives the sample this step exports, if it exports one (NULL skips). */
TF_API int tf_step_io(tf_ctx* ctx, const double* carrier_in, double* probe_out, uint64_t* done);
/* Runs up to nsteps steps with CUDA events between kernels and returns the
 * device milliseconds spent per phase: ms[0] sources/BC edges, ms[1] E update,
 * ms[2] source scatter + boundary flux, ms[3] probe export, ms[4] H update
 * (the reference's per-phase averages, Discretization.hpp:2286-2302). */
TF_API int tf_phase_times(tf_ctx* ctx, uint64_t nsteps, double* ms5, uint64_t* done);
/* Whole simulation as RunSimulation does it: prepare, every step, output files. */
TF_API int tf_run(tf_ctx* ctx, uint32_t sim_label, const tf_opts* opts);
/* gfdtd: CG iterations and final relative residual of every step taken so far
 * (the reference's "mean solver iterations", Discretization.hpp:2286-2302). */
TF_API int tf_solver_stats(tf_ctx* ctx, int32_t* iters, double* resid, size_t cap, size_t* n);
/* warm_start 3: per step taken, 1 when the CG kept the network's guess and 0
 * when the polynomial extrapolation had the smaller initial residual (or the
 * network was still training). */
TF_API int tf_guess_stats(tf_ctx* ctx, int8_t* kept, size_t cap, size_t* n);
/* warm_start 3: training loss of every Adam step so far. */
TF_API int tf_training_loss(tf_ctx* ctx, float* loss, size_t cap, size_t* n);
/* Standalone Jacobi-PCG solve of a symmetric positive definite CSR system held
 * in device memory, with the persistent kernel of the gfdtd path
 * (ConjugateGradientSolver.hpp:52-129: Jacobi preconditioner 1/diag, stop on
 * ||r||/||r0|| <= tol (criterion 0) or ||r|| <= tol ||b|| (criterion 1), at
 * most maxiter iterations, 0 meaning 100).  x holds the initial guess and
 * receives the solution.  Returns TF_E_SOLVER when the iteration limit is hit
 * first (x then holds the last iterate).  Allocates its work space (4 n + a
 * few hundred doubles) on the device for the duration of the call.  Errors are
 * reported through tf_last_error(NULL). */
typedef struct tf_pcg_args {
  int32_t n;                 /* rows = columns                                  */
  int32_t device;
  const int64_t* row_ptr;    /* device, n + 1 entries                           */
  const int32_t* col;        /* device                                          */
  const double* val;         /* device                                          */
  const double* b;           /* device, n                                       */
  double* x;                 /* device, n: initial guess in, solution out       */
  double tol;
  int32_t maxiter;
  int32_t criterion;
  void* stream;              /* cudaStream_t, or NULL for the default stream    */
} tf_pcg_args;
TF_API int tf_pcg_solve(const tf_pcg_args* args, int32_t* iters, double* rel_resid);
/* tf_pcg_solve without any device allocation.  This entry point has no
 * counterpart in the reference; it serves callers that cannot allocate device
 * memory while they solve: a host whose own pool allocator already holds the
 * GPU's memory (a cudaMalloc there fails or fragments the pool), or a loop that
 * must not stall other streams, since cudaMalloc and cudaFree can synchronize
 * the device.  The work space is a file-scope device array sized for at most
 * 262,144 unknowns (about 8 MiB); every GPU that loads the library holds it
 * until the process exits, and larger n is rejected with TF_E_ARG.  The first
 * call on a device looks up the array's device address (once per device, that
 * device current); make that first call before any stream capture.  All calls
 * share the one array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.  The address lookup is
 * kept for the life of the process, so cudaDeviceReset (which reloads the
 * module) is not supported while the library is loaded.  Same arguments,
 * results and status codes as tf_pcg_solve. */
TF_API int tf_pcg_solve_noalloc(const tf_pcg_args* args, int32_t* iters, double* rel_resid);
/* Self-check of the bounded grid barrier that the persistent CG kernels (the
 * batch/gfdtd solve and tf_pcg_solve) use; no reference counterpart.  `blocks`
 * co-resident blocks (one cooperative launch, blocks <= the SM count) pass
 * `rounds` barriers that each wait for `expected` arrivals, every wait bounded
 * by timeout_us.  With expected == blocks every barrier completes and *status
 * is 0; with expected > blocks the first wait can never complete, it runs out,
 * the launch still ends and *status is 2 -- the flag on which the CG kernels'
 * callers return TF_E_CUDA.  *ms (optional) is the launch's duration.
 * Arguments: 1 <= blocks, 1 <= expected <= 2 blocks, 1 <= rounds <= 100000,
 * 1 <= timeout_us <= 1000000; otherwise TF_E_ARG (checked before the GPU is
 * touched).  Errors through tf_last_error(NULL). */
TF_API int tf_barrier_check(int32_t device, uint32_t blocks, uint32_t expected, uint32_t rounds,
                            uint32_t timeout_us, int32_t* status, double* ms);
/* ---- Batches: many gfdtd simulations advanced together ---------------------
 * The reference runs the simulations of a script one after another
 * (dga_main.cpp:52-62), each with its own mesh, materials, sources and time
 * step.  A batch holds n such simulations (scripts[i], simulation label
 * labels[i], method gfdtd) built on the host in parallel and laid out in one
 * device image: one launch sequence and one persistent CG kernel per step
 * advance every member (batch_mode 0), each member keeping its own time step,
 * tolerance, stopping test, probes and statistics.  batch_mode 1 keeps every
 * member in its own device image and steps them one after another (the
 * reference's order).  Members are numbered 0..n-1 in argument order.  Errors
 * are reported through tf_batch_last_error. */
typedef struct tf_batch tf_batch;
TF_API int tf_batch_open(const char* const* scripts, const uint32_t* labels, uint32_t n, const tf_opts* opts,
                         tf_batch** out);
TF_API int tf_batch_info(tf_batch* b, uint32_t member, tf_info* info);
/* Advance every unfinished member by up to nsteps steps; *done = the most any member took. */
TF_API int tf_batch_step(tf_batch* b, uint64_t nsteps, uint64_t* done);
/* tf_phase_times over the batch: ms5 = H update + probes, sources + rhs, CG, scatter, step end. */
TF_API int tf_batch_phase_times(tf_batch* b, uint64_t nsteps, double* ms5, uint64_t* done);
/* One step of every member from host memory: carriers_in holds n_sources values
 * per member in member order (NULL keeps the scripts' waveforms); probes_out
 * receives n_probes * 6 values per member in member order for the members that
 * export a sample this step (others' slots are left untouched). */
TF_API int tf_batch_step_io(tf_batch* b, const double* carriers_in, double* probes_out, uint64_t* done);
TF_API int tf_batch_get_probes(tf_batch* b, uint32_t member, double* times, double* values, size_t cap_samples,
                               size_t* n_samples);
TF_API int tf_batch_get_probe_points(tf_batch* b, uint32_t member, double* xyz, uint64_t* cells, size_t cap);
TF_API int tf_batch_get_state(tf_batch* b, uint32_t member, double* U, size_t nU, double* B, size_t nB, double* F,
                              size_t nF);
TF_API int tf_batch_get_flux(tf_batch* b, uint32_t member, double* flux, size_t cap, size_t* n);
/* tf_energy of one member (gfdtd: 0.5 U^n.E.U^n + 0.5 B^{n-1/2}.N.B^{n+1/2}, GPU FP64 reduction). */
TF_API int tf_batch_energy(tf_batch* b, uint32_t member, double* energy);
TF_API int tf_batch_solver_stats(tf_batch* b, uint32_t member, int32_t* iters, double* resid, size_t cap,
                                 size_t* n);
TF_API int tf_batch_guess_stats(tf_batch* b, uint32_t member, int8_t* kept, size_t cap, size_t* n);
/* Training loss of the network that member's group learns (one network per group). */
TF_API int tf_batch_training_loss(tf_batch* b, uint32_t member, float* loss, size_t cap, size_t* n);
/* Current parameters of that network (tf_mlp_param_count() floats). */
TF_API int tf_batch_mlp_params(tf_batch* b, uint32_t member, float* params);
/* Device time of the last tf_batch_step (summed over members in batch_mode 1). */
TF_API int tf_batch_last_step_ms(tf_batch* b, double* ms);
TF_API const char* tf_batch_last_error(tf_batch* b);
TF_API void tf_batch_close(tf_batch* b);
/* ---- Learned CG warm start network ------------------------------------------
 * The per-edge network of warm_start 3 (no counterpart in the reference, whose
 * CG starts from the previous solution, Discretization.hpp:1536): 6 inputs ->
 * 64 -> 64 -> 1 with SiLU, BF16 weights and activations on the tensor cores,
 * FP32 accumulation and FP32 master parameters.  The parameter vector holds
 * tf_mlp_param_count() floats: W1[64][16] (inputs 6..15 zero), b1[64],
 * W2[64][64], b2[64], W3[64], b3, W[n][k] the weight from input k to output n.
 * These calls run the group engine's own kernels on host buffers (current
 * device); errors through tf_last_error(NULL). */
TF_API int tf_mlp_param_count(void);
/* He-uniform initial parameters (output layer scaled by 0.1) from a seed. */
TF_API int tf_mlp_init(uint64_t seed, float* params);
/* outputs[n] of inputs[n][6]. */
TF_API int tf_mlp_forward(const float* params, int64_t n, const float* inputs, float* outputs);
/* Gradient of sum_i w_i (y_i - t_i)^2 / n with respect to the parameters
 * (weights NULL: all 1), and that loss; n <= 2^24. */
TF_API int tf_mlp_gradient(const float* params, int64_t n, const float* inputs, const float* targets,
                           const float* weights, float* grad, float* loss);
/* Device time of the last tf_step call, from CUDA events on the context stream. */
TF_API int tf_last_step_ms(tf_ctx* ctx, double* ms);
/* Message of the last failure on ctx; with ctx == NULL, of the last
 * context-free call (tf_pcg_solve) on this host thread. */
TF_API const char* tf_last_error(tf_ctx* ctx);
TF_API void tf_close(tf_ctx* ctx);
/* Fills *opts with defaults (FP64, device 0, no files, quiet, automatic graphs). */
TF_API void tf_default_opts(tf_opts* opts);

#ifdef __cplusplus
}
#endif
#endif /* TETFIT_H */
