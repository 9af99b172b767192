/*
 * qgn_gpu.h -- C-ABI of the B200 (sm_100a) QGN spectral right-hand side and time steppers.
 *
 * This is the drop-in boundary for the reference's TimeStep path
 * (iangrooms/QGN_Fortran).  A Fortran host binds these entry points through
 * iso_c_binding from an include file selected exactly like the reference's
 * schemes (QGN_Module.f90:306).  Every entry point returns an int status
 * (QGN_OK == 0); qgn_last_error() gives the message of the last failure.
 *
 * Array conventions (identical to the reference's Fortran storage):
 *   spectral  complex(dp) q_hat(nx/2+1, ny, nz)  -> interleaved (re,im) doubles,
 *             element (i,j,k) (1-based) at offset 2*((i-1) + (nx/2+1)*((j-1) + ny*(k-1))).
 *   physical  real(dp) q(nx, ny, nz), column-major.
 *   Modes     real(dp) Modes(nz, nz), column-major: Modes(kk,k) = layer kk of mode k.
 *
 * Threading: one host thread per context; a context is not re-entrant (as the
 * reference's module state is not).  Distinct contexts are independent.
 */
#ifndef QGN_GPU_H
#define QGN_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define QGN_OK                0
#define QGN_ERR_CONFIG        1   /* bad or unsupported parameters / inputs          */
#define QGN_ERR_CUDA          2   /* a CUDA runtime call failed                       */
#define QGN_ERR_NONFINITE     3   /* NaN/Inf found in the error norm or the state     */
#define QGN_ERR_REJECT_LIMIT  4   /* adaptive step rejected max_rejects times in a row*/
#define QGN_ERR_ARG           5   /* null pointer / invalid argument                  */
#define QGN_ERR_NO_DEVICE     6   /* no CUDA device, or not an sm_100 device          */
#define QGN_ERR_TOO_LARGE     7   /* grid does not fit QGN_STATIC_SCRATCH_BYTES (qgn_rhs_static) */

/* ---- time integrators: the include files of QGN_Module.f90:306 ---------- */
#define QGN_SCHEME_ARK43_QGLEITH 0  /* ARK43_QGLeith.f90 (reference default) */
#define QGN_SCHEME_ARK43         1  /* ARK43.f90  (fixed A8)                 */
#define QGN_SCHEME_BSRK3         2  /* BSRK3.f90  (Bogacki-Shampine 3(2))    */
#define QGN_SCHEME_RK4           3  /* RK4.f90                               */
#define QGN_SCHEME_AB3           4  /* AB3.f90                               */

/* ---- arithmetic of the spectral path ------------------------------------ */
#define QGN_PREC_FP64   0   /* everything in FP64 (parity mode)                       */
#define QGN_PREC_MIXED  1   /* FP32 transforms/products/stages, FP64 modes/norm/control */

/* Runtime copy of the compile-time constants of parameters.f90:1-31. */
typedef struct qgn_params {
    int    nx, ny, nz;       /* grid; nx, ny powers of two in [16, 2048]; 2 <= nz <= 32 */
    int    is_explicit;      /* parameters.f90:28 (0 = .FALSE.)                          */
    double Lx, Ly, Htot;
    double f0, beta;
    double A2, A8, r0, C_d;
    double TOL;              /* absolute error tolerance of the adaptive schemes         */
    double dt_max;           /* parameters.f90:31                                        */
    int    max_rejects;      /* consecutive rejected attempts before QGN_ERR_REJECT_LIMIT; 0 -> 64 */
    int    reserved;
} qgn_params;

typedef struct qgn_ctx qgn_ctx;

/*
 * Create a device context.  Replaces the device-relevant half of Initialize
 * (QGN_Module.f90:53-188): the host keeps reading H/S/UBar, building L and running
 * DGEEV; it passes the results here.
 *   H      nz layer thicknesses AFTER the rescale H=Htot*H/sum(H) (QGN_Module.f90:87)
 *   S      nz+1 stratification values S(0:nz) (validated, not otherwise used); may be NULL
 *   uBar   nz mean zonal velocities (QGN_Module.f90:145-147)
 *   qyBar  nz mean PV gradients L*(-uBar) (QGN_Module.f90:148)
 *   Modes  nz*nz normalised right eigenvectors, column-major (QGN_Module.f90:121-127)
 *   EVals  nz eigenvalues (QGN_Module.f90:121)
 * scheme: QGN_SCHEME_*; precision: QGN_PREC_*.
 */
int qgn_create(const qgn_params* p, const double* H, const double* S,
               const double* uBar, const double* qyBar,
               const double* Modes, const double* EVals,
               int scheme, int precision, qgn_ctx** out);

/*
 * One call of TimeStep(q_hat,t,dt) (QGN_Module.f90:302-309) with the scheme chosen
 * at qgn_create.  q_hat is the host spectral array (interleaved complex, Fortran
 * order).  Only the modes that DeAlias keeps are read: the entries DeAlias zeroes
 * (QGN_Module.f90:194-204) are treated as zero on input.  On output only the kept modes
 * are written (QGN_OUTPUT_KEPT, the default): the reference's TimeStep ends with
 * `call DeAlias(q_hat)` (QGN_Module.f90:307), which zeroes the others on the host, and in a
 * dealiased input -- every TimeStep output and Initialize's q_hat -- they are zero already.
 * A caller that passes an array with data in the dealiased band and wants it cleared selects
 * QGN_OUTPUT_FULL with qgn_set_output.  t and dt are updated exactly as by the reference
 * scheme.
 * Stepper memory (FSAL stage, AB history, err0) persists in the context like the
 * reference's `save` variables.
 */
int qgn_step(qgn_ctx* ctx, double* q_hat, double* t, double* dt);

/* nsteps consecutive TimeStep calls with one host<->device transfer of q_hat. */
int qgn_advance(qgn_ctx* ctx, double* q_hat, double* t, double* dt, int nsteps);

/*
 * What qgn_step and qgn_advance write back to the host q_hat.  No counterpart in the
 * reference (its TimeStep works on the host array in place).
 *   QGN_OUTPUT_KEPT  the modes DeAlias keeps (two pitched copies, 44 % of the array bytes)
 *   QGN_OUTPUT_FULL  the whole array, zeros where DeAlias zeroes
 */
#define QGN_OUTPUT_KEPT 0
#define QGN_OUTPUT_FULL 1
int qgn_set_output(qgn_ctx* ctx, int mode);

/* Device-resident variants: the state lives on the GPU between calls. */
int qgn_set_state(qgn_ctx* ctx, const double* q_hat, double t, double dt);
int qgn_get_state(qgn_ctx* ctx, double* q_hat, double* t, double* dt);  /* writes all of q_hat */
int qgn_advance_resident(qgn_ctx* ctx, int nsteps);
int qgn_get_time(qgn_ctx* ctx, double* t, double* dt);

/*
 * One GetRHS(q_hat, RHS) evaluation (QGN_Module.f90:258-296), the parity hook.
 * q_hat is dealiased on input (GetRHS assumes dealiased input, QGN_Module.f90:211);
 * rhs receives the full dealiased right-hand side (zeros included).
 */
int qgn_rhs(qgn_ctx* ctx, const double* q_hat, double* rhs);

/* psi_hat of GetPsi (QGN_Module.f90:315-341) for a host q_hat; writes all of psi_hat. */
int qgn_psi(qgn_ctx* ctx, const double* q_hat, double* psi_hat);

/* QG-Leith coefficients A8L(1:nz) of ARK43_QGLeith.f90:62-73 for the resident state. */
int qgn_leith(qgn_ctx* ctx, double* A8L);

/*
 * FP64 diagnostics of the resident state (the reference has none, QGN_Driver.f90:52-55):
 *   ke_layer[nz]       0.5*mean(u^2+v^2)*H_k/Htot per layer
 *   spectrum[nbins*nz] isotropic KE spectrum per layer in integer shells
 *                      round(sqrt((i)^2+(jj)^2)) (wavenumber index units), may be NULL
 */
int qgn_diagnostics(qgn_ctx* ctx, double* ke_layer, double* spectrum, int nbins);

/*
 * FP64 energetics of the resident state per layer k (no counterpart in the reference), each
 * weighted by H_k/Htot like ke_layer of qgn_diagnostics; any output may be NULL:
 *   ke_layer[nz]         0.5*mean(u^2+v^2)
 *   ape_layer[nz]        -0.5*mean(psi_k (L psi)_k) with L the stretching matrix of
 *                        [Del+L]psi = q (QGN_Module.f90:100-112); the layers sum to the total
 *                        available potential energy (>= 0), and KE + APE = -0.5 sum_k
 *                        H_k/Htot mean(psi_k q_k)
 *   enstrophy_layer[nz]  0.5*mean(q^2)
 */
int qgn_energetics(qgn_ctx* ctx, double* ke_layer, double* ape_layer, double* enstrophy_layer);

/*
 * WriteQP's fields (QGN_Module.f90:348-377) in physical space: q_phys = c2r(q_hat)/(nx*ny)
 * and psi_phys = c2r(psi_hat)/(nx*ny) as real(dp)(nx,ny,nz) column-major.  q_hat is a host
 * spectral array, or NULL for the resident state.  Either output pointer may be NULL.
 */
int qgn_physical(qgn_ctx* ctx, const double* q_hat, double* q_phys, double* psi_phys);

/*
 * The fields WriteQPmodal writes (QGN_Module.f90:381-440): q_mode, p_mode (psi_mode) and
 * J_mode -- the vertical-mode projections of q_hat, of psi_hat and of the full (undealiased)
 * Jacobian spectrum -- in physical space, real(dp)(nx,ny,nz) column-major each.  q_hat is a
 * host spectral array (the reference's q_hat(nx/2+1,ny,nz), dealiased), or NULL for the
 * resident state; the resident state and the stepper's history are left unchanged.
 */
int qgn_physical_modal(qgn_ctx* ctx, const double* q_hat, double* q_mode, double* p_mode, double* J_mode);

/*
 * Set the resident state from a physical PV field real(dp) q(nx,ny,nz): the forward
 * transform and DeAlias of Initialize (QGN_Module.f90:179-183), as used for the IC and
 * for restarts from q.%09d.dat (QGN_Driver.f90:21-30).
 */
int qgn_set_state_physical(qgn_ctx* ctx, const double* q_phys, double t, double dt);

/* Number of rejected attempts since creation (the reference prints 'Rejected step'). */
int qgn_rejects(qgn_ctx* ctx, long long* count);

/*
 * Kernel accounting (no counterpart in the reference, which prints only t and dt).
 * Every kernel launch is counted per kernel family; with profiling enabled each launch is
 * also bracketed by CUDA events on the context's stream.  qgn_profile_enable resets the
 * counters.  qgn_profile_read returns, for one family id in [0, QGN_KERNEL_FAMILIES),
 * the summed device time (ms), the summed algorithmic bytes of the timed launches, the
 * number of timed launches and the number of launches.
 */
#define QGN_KERNEL_FAMILIES 14
int qgn_profile_enable(qgn_ctx* ctx, int enable);
int qgn_profile_read(qgn_ctx* ctx, int kernel, double* total_ms, double* bytes,
                     long long* timed_launches, long long* launches);
const char* qgn_kernel_name(int kernel);

/* The cudaStream_t (as void*) all of this context's work is issued on. */
int qgn_stream(qgn_ctx* ctx, void** stream);

/*
 * One GetRHS (QGN_Module.f90:258-296) that allocates no device memory.  No counterpart in
 * the reference: it exists for hosts that cannot call cudaMalloc where the model is
 * evaluated -- a component coupled into a larger application that owns all device memory
 * (an OpenACC or OpenMP-offload data region, or a pool carved up at start-up), or a time
 * loop that must not take cudaMalloc's implicit device synchronisation.
 *
 * q_hat_dev and rhs_dev are DEVICE arrays in the reference's layout
 * complex(dp)(nx/2+1,ny,nz) (interleaved doubles, Fortran order); rhs_dev receives the
 * dealiased right-hand side with zeros in the dealiased band.  The other arguments are the
 * host arrays of qgn_create.  Work is enqueued on `stream` (a cudaStream_t, NULL for the
 * default stream) and is not waited for.
 *
 * Intermediates live in one file-scope device array of QGN_STATIC_SCRATCH_BYTES that the
 * library's module reserves on every GPU where it is used, until process exit.  A grid
 * needs 16*(5*nz*ny*nkxp + 2*ny*nkxp + 3*nz*nkx*nky + nx + ny) bytes plus about 18 KB of
 * constants (nkx = nx/3, nkxp = nkx rounded up to 4, nky = ny - ny/3 - 1); larger grids
 * return QGN_ERR_TOO_LARGE (256^2 x 8 and 512^2 x 2 fit).  All calls share the array and
 * it keeps the last call's contents, so calls whose GPU work overlaps (other streams,
 * other host threads on the same device) race.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and loads the module if it is not loaded
 * yet; make that first call before any stream capture on that device.
 */
#define QGN_STATIC_SCRATCH_BYTES (32u * 1024u * 1024u)
int qgn_rhs_static(const qgn_params* p, const double* H, const double* uBar, const double* qyBar,
                   const double* Modes, const double* EVals, const double* q_hat_dev, double* rhs_dev,
                   void* stream);

/*
 * ---- Ensembles ------------------------------------------------------------------------
 * No counterpart in the reference (one model per process there): independent members --
 * contexts made by qgn_create with scheme QGN_SCHEME_BSRK3 and precision QGN_PREC_FP64 --
 * advanced together with BSRK3.f90's scheme.  Grid sizes nx, ny in {128, 256, 512} and
 * layer counts 2..8 or 16 may differ between members; C_d must be 0.  Each pass of an
 * attempt is one launch for all members, the attempts run as a device-conditioned CUDA
 * graph loop, and the first advance autotunes the tile widths and grid sizes.
 *
 * The ensemble borrows the contexts (they must outlive it) and works on their buffers:
 * load states with qgn_set_state (which also restarts a member's FSAL RHS0) and read them
 * with qgn_get_state.  `precision` QGN_PREC_MIXED runs the transforms, stage right-hand
 * sides and stage inputs in FP32, with FP64 state, stage sums, GetPsi arithmetic, error
 * norm and controller.
 */
typedef struct qgn_ens qgn_ens;
int qgn_ens_create(qgn_ctx* const* members, int nmembers, int precision, qgn_ens** out);
/* every member takes nsteps accepted steps (TimeStep nsteps times); members in lockstep */
int qgn_ens_advance(qgn_ens* ens, int nsteps);
/* autotuner's choice for pass 0 (y-inverse), 1 (x pass), 2 (y-forward): CTA threads,
 * CTAs per SM of the persistent grid (0 = one CTA per tile) and the timed ms per launch */
int qgn_ens_tuning(qgn_ens* ens, int pass, int* threads, int* ctas_per_sm, float* ms);
/* the autotuner's FFT radix for the pass: elements per thread of its transforms (8, 16 or 32;
 * a transform of n points runs on n / that many threads, in radix passes of that size) */
int qgn_ens_fft_radix(qgn_ens* ens, int pass, int* elements_per_thread);
/* pin a pass to one tile variant instead of tuning it: CTA threads (as qgn_ens_tuning reports
 * them), elements per thread and CTAs per SM (0 = one CTA per tile).  Variants: y-inverse
 * 64/128/256 threads at 16 or 8 elements, x pass 96/192/384 at 16 and 192/384 at 8, y-forward
 * 64/128/256 at 16 and 128/256 at 8; QGN_PREC_MIXED adds 32 elements (y-inverse 64/128/256,
 * x pass 96/192/384, y-forward 64/128).  QGN_ERR_CONFIG for any other combination. */
int qgn_ens_set_tiles(qgn_ens* ens, int pass, int threads, int elements_per_thread, int ctas_per_sm);
int qgn_ens_profile_enable(qgn_ens* ens, int enable);
int qgn_ens_profile_read(qgn_ens* ens, int kernel, double* total_ms, double* bytes,
                         long long* timed_launches, long long* launches);
/* the ensemble's CUDA stream (cudaStream_t): its launches run there */
int qgn_ens_stream(qgn_ens* ens, void** stream);
const char* qgn_ens_last_error(qgn_ens* ens);
int qgn_ens_destroy(qgn_ens* ens);

/*
 * ---- Learned subgrid closure ------------------------------------------------------------
 * No counterpart in the reference.  A network of `layers` periodic 3x3 convolutions (GELU
 * between them) maps `cin` input channels to `cout` output channels on an H x W grid (W a
 * multiple of 128, width 64 channels), on the BF16 tensor cores with FP32 accumulation.
 * Tensors are NHWC in device memory: inputs BF16 with cin padded to a multiple of 16
 * (qgn_cnn_padded_channels), outputs and targets FP32 with cout padded the same way.
 * Weights (get/set, gradients): per layer FP32 [9][cout_p][cin_p] (tap = 3*(dy+1)+(dx+1))
 * followed by the bias [cout_p]; qgn_cnn_num_params floats in all.
 */
typedef struct qgn_cnn qgn_cnn;
int qgn_cnn_create(int cin, int width, int cout, int layers, int H, int W, int max_batch,
                   unsigned long long seed, qgn_cnn** out);
int qgn_cnn_padded_channels(const qgn_cnn* net, int* cin_padded, int* cout_padded);
long long qgn_cnn_num_params(const qgn_cnn* net);
int qgn_cnn_get_weights(qgn_cnn* net, float* host);
int qgn_cnn_set_weights(qgn_cnn* net, const float* host);   /* also resets the Adam moments */
int qgn_cnn_forward(qgn_cnn* net, const void* x, float* y, int batch, void* stream);
/* MSE loss over the real output channels and its gradient at the current weights */
int qgn_cnn_gradients(qgn_cnn* net, const void* x, const float* y, int batch, float* grads_host,
                      double* loss);
/* one Adam step (lr; beta 0.9/0.999, eps 1e-8) on samples idx[0..batch) (device int32) of a
 * dataset x_all [n][H][W][cin_p] BF16, y_all [n][H][W][cout_p] FP32; loss before the update */
int qgn_cnn_train_step(qgn_cnn* net, const void* x_all, const float* y_all, const int* idx, int batch,
                       float lr, double* loss);
/* tensor-core path of the convolutions: 0 = tcgen05 with TMEM accumulators (default; an
 * inference whose image rows fit one CTA each runs all layers in one cooperative launch),
 * 1 = warp-level mma.sync, 2 = tcgen05 with one launch per layer; 0 and 2 give identical
 * results, 1 the same up to FP32 summation order */
int qgn_cnn_set_engine(qgn_cnn* net, int engine);
/* waits for the network's stream; QGN_ERR_CUDA if a tensor-core kernel reported a timeout */
int qgn_cnn_check(qgn_cnn* net);
int qgn_cnn_stream(qgn_cnn* net, void** stream);
const char* qgn_cnn_last_error(const qgn_cnn* net);
int qgn_cnn_destroy(qgn_cnn* net);

/* coarse <- sharp spectral cutoff of fine's state (same nz, Lx, Ly; coarse grid not finer) */
int qgn_coarse_grain(qgn_ctx* fine, qgn_ctx* coarse);
/* one training sample on coarse's grid: x = scaled (q, psi) of the coarse-grained state,
 * y = scaled subgrid tendency trunc(GetRHS_fine(q)) - GetRHS_coarse(trunc(q)); in_scale [2 nz],
 * out_scale [nz] host; x_dev [ny][nx][cin_p] BF16, y_dev [ny][nx][cout_p] FP32 (device).
 * Sets coarse's state to the coarse-grained one. */
int qgn_closure_snapshot(qgn_ctx* fine, qgn_ctx* coarse, const float* in_scale, const float* out_scale,
                         void* x_dev, float* y_dev, int cin_p, int cout_p);
/* attach (net != NULL) or detach the closure of an ARK43_QGLeith FP64 context whose grid is the
 * network's: each step adds the network's tendency to every stage RHS while the energy-budget
 * check passes (then with A8 = A8_background), else runs plain QG-Leith.  The network must not
 * be used elsewhere while this context steps. */
int qgn_closure_attach(qgn_ctx* ctx, qgn_cnn* net, const float* in_scale, const float* out_scale,
                       double A8_background, double energy_limit);
/* closure evaluations and fallbacks so far; last_budget[3] = {dE/dt, dZ/dt, E} of the last one */
int qgn_closure_stats(qgn_ctx* ctx, long long* evaluations, long long* fallbacks, double* last_budget);

/* Message of the last failing call on this context (never NULL). */
const char* qgn_last_error(const qgn_ctx* ctx);

/* Release all device memory (replaces the DFTI frees of Cleanup, QGN_Module.f90:448-458). */
int qgn_destroy(qgn_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* QGN_GPU_H */
