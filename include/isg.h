/* isg.h - C ABI of the B200 MLFMA inverse-scattering solver (libisg.so).
 *
 * The library is a drop-in for the reference's MLFMA forward/adjoint solve
 * path (merthidayetoglu/inverse-solver-GPU): setup_mlfma / setup_gpu /
 * setup_bicgs, matvec, bicgs, mlfma / mlfmah and aggregate / aggregateh.
 * The reference exposes these as C++ free functions over globals
 * (vars.h:14-38, kernels.h:42); each entry point below names the routine it
 * replaces.  A C++ shim with the reference's exact names and signatures is
 * declared in isg_refapi.h.
 *
 * Conventions
 *  - Complex vectors are complex64 (interleaved float re, im) in device memory,
 *    batched right-hand side (RHS) major: RHS j of a vector of U unknowns starts
 *    at element j*U.  The library never copies caller data to or from the host.
 *  - `order` selects the unknown ordering of the caller's vectors:
 *    ISG_ORDER_TREE is the reference's tree order (leaf-major, box*box pixels
 *    per leaf, row-major inside the leaf; setup_mlfma.cpp:124-175),
 *    ISG_ORDER_RASTER is the image raster (row 0 at the top; mom.cpp's
 *    unkmap), ISG_ORDER_BLOCKED is the library's internal layout (leaves in
 *    raster order, row-major pixels inside a leaf) and costs no reordering.
 *  - `g` is the scaled contrast k0^2 (eps_r - 1) per pixel (mom.cpp:288-289);
 *    g_stride is the element distance between the contrasts of consecutive RHS:
 *    0 shares one contrast across the batch, U gives each RHS its own.
 *  - Every call is ordered on `stream` (0 = CUDA's legacy default stream).  A
 *    context is not thread-safe; use one per host thread.
 *  - Every call returns an isg_status.
 */
#ifndef ISG_H
#define ISG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct isg_ctx isg_ctx;
typedef void *isg_stream; /* a cudaStream_t */

typedef enum isg_status {
  ISG_OK = 0,
  ISG_NOT_CONVERGED = 1, /* iteration cap reached above the tolerance */
  ISG_BREAKDOWN = 2,     /* BiCGSTAB rho or omega vanished (bicgs.cpp:128,165) */
  ISG_NONFINITE = 3,     /* a NaN or Inf appeared in a residual */
  ISG_CUDA_ERROR = 4,
  ISG_BAD_ARG = 5,
  ISG_TIMEOUT = 6,
  ISG_NO_DEVICE = 7,
  ISG_UNSUPPORTED = 8
} isg_status;

typedef enum isg_order { ISG_ORDER_TREE = 0, ISG_ORDER_RASTER = 1, ISG_ORDER_BLOCKED = 2 } isg_order;

typedef struct isg_opts {
  int level;    /* tree levels; the grid is box*2^(level-1) pixels per side (mom.cpp:6,137-138) */
  int box;      /* leaf side in pixels (mom.cpp:5); 8 */
  double res;   /* pixel size in wavelengths (mom.cpp:4) */
  double k0;    /* background wavenumber (mom.cpp:136) */
  int beta;     /* excess-bandwidth parameter of the sample rule (setup_mlfma.cpp:3) */
  int ninter;   /* Lagrange interpolation taps (setup_mlfma.cpp:4) */
  int numrx;    /* far-field receiver angles (mom.cpp:90-91,149-154) */
  int max_rhs;  /* widest batch one call may pass */
  int device;   /* CUDA device ordinal */
} isg_opts;

/* Engines for the dense leaf stages (near field, P2M, L2P). */
typedef enum isg_engine {
  ISG_ENGINE_SIMT = 0,  /* complex FP32 CUDA cores: the plain solver */
  ISG_ENGINE_TENSOR = 1 /* 3xFP16 split products (hi*hi + hi*lo + lo*hi) on the tcgen05 tensor cores, FP32 accumulate */
} isg_engine;

typedef enum isg_guess {
  ISG_GUESS_ZERO = 0,   /* x0 = 0, as every reference call site (mom.cpp:254,286,324) */
  ISG_GUESS_CALLER = 1, /* x0 = the caller's x on entry (bicgs.cpp:115) */
  ISG_GUESS_LEARNED = 2 /* x0 from the context's neural-operator warm start (isg_fno_create).  isg_bicgs:
                           forward solves (adjoint solves start from zero).  isg_dbim: the forward
                           solves and the adjoint solves, the latter through the same network
                           (x0 = conj(g N(g, conj(y))), y the back-projected data residual) */
} isg_guess;

typedef struct isg_solve_opts {
  double tol;          /* relative residual target (mom.cpp:21 toli) */
  int maxit;           /* iteration cap per RHS (mom.cpp:22 iti) */
  int guess;           /* isg_guess */
  int check_every;     /* iterations between host convergence polls (>= 1) */
  int true_residual;   /* 1: after convergence recompute b - A x and restart any RHS above tol */
  int max_restarts;    /* restarts allowed by the true-residual check; each restart halves the
                          recursive-residual target of that RHS */
  int engine;          /* isg_engine */
  int graph;           /* 1: replay the check_every-iteration block as a CUDA graph captured on the
                          first poll (streams other than the legacy default stream); 0: launch directly */
} isg_solve_opts;

typedef struct isg_solve_info {
  int iterations;      /* BiCGSTAB iterations (bicgs.cpp:125) */
  int matvecs;         /* operator applications */
  int status;          /* isg_status of this RHS */
  int restarts;
  double residual;     /* final recursive ||r|| / ||b|| (bicgs.cpp:160-161) */
  double true_residual;/* ||b - A x|| / ||b|| recomputed with the operator, or -1 */
} isg_solve_info;

/* ---- lifecycle: setup_mlfma (setup_mlfma.cpp:50-640) + setup_gpu (gpu.cu:69-260)
 *      + setup_bicgs (bicgs_gpu.cu:89-113) ---- */
void isg_default_opts(isg_opts *o);
void isg_default_solve_opts(isg_solve_opts *o);
/* Builds the host tables (tree, plane-wave, interpolation, shift and receiver
 * tables).  Touches no GPU.  The near-field blocks and translation operators
 * (setup_mlfma.cpp:492-543, the tables that evaluate Bessel functions) are
 * computed on the device by isg_setup_gpu, or on the host if isg_host_table
 * asks for them first. */
isg_status isg_create(const isg_opts *opts, isg_ctx **out);
/* Uploads the tables and allocates the device workspaces for max_rhs RHS. */
isg_status isg_setup_gpu(isg_ctx *ctx);
void isg_destroy(isg_ctx *ctx);
const char *isg_status_string(isg_status s);
const char *isg_last_error(const isg_ctx *ctx);

int isg_numunk(const isg_ctx *ctx);
int isg_side(const isg_ctx *ctx);
int isg_numsamp(const isg_ctx *ctx, int lvl);
int isg_levels(const isg_ctx *ctx);
/* Host copy of a setup table, for inspection and tests.  Names follow the
 * reference's globals (setup_mlfma.cpp:6-46): "numsamp", "near", "coeff_multi",
 * "basis_local", "interp", "anterp", "shiftmul", "shiftloc", "trans", "interph",
 * "anterph", "pos", "unkmap".  Returns ISG_BAD_ARG for unknown names. */
isg_status isg_host_table(const isg_ctx *ctx, const char *name, int lvl, const void **data, int64_t *count);

/* Reorders nrhs complex64 vectors between isg_order layouts on the device. */
isg_status isg_reorder(isg_ctx *ctx, const void *in, void *out, int nrhs, int from, int to, isg_stream stream);

/* ---- operator ---- */
/* r = G x: mlfma (matvec_gpu.cu:65-79, solve.cpp:25-248); conj != 0 gives
 * mlfmah, r = conj(G conj(x)) (matvec_gpu.cu:80-101, solve.cpp:8-24). */
isg_status isg_mlfma(isg_ctx *ctx, const void *x, void *r, int nrhs, int conj, int order, int engine,
                     isg_stream stream);
/* y = x - G(g x), or y = x - conj(g G(conj x)) when hermitian (matvec,
 * bicgs_gpu.cu:61-76; bicgs.cpp:62-87). */
isg_status isg_matvec(isg_ctx *ctx, const void *x, const void *g, int64_t g_stride, void *y, int nrhs, int hermitian,
                      int order, int engine, isg_stream stream);

/* ---- solver ---- */
/* BiCGSTAB on (I - G diag(g)) x = b or its adjoint for nrhs right-hand sides at
 * once, each with its own convergence mask (bicgs, bicgs_gpu.cu:116-224;
 * bicgs.cpp:88-179).  x is the solution (and the initial guess with
 * ISG_GUESS_CALLER).  info receives nrhs records (may be NULL).  Returns
 * ISG_OK when every RHS reached tol, else the worst per-RHS status. */
isg_status isg_bicgs(isg_ctx *ctx, void *x, const void *g, int64_t g_stride, const void *b, int nrhs, int hermitian,
                     int order, const isg_solve_opts *opts, isg_solve_info *info, isg_stream stream);

/* One member of a group solve: a context and its own batch, with the meaning
 * of the isg_bicgs arguments of the same names. */
typedef struct isg_group_member {
  isg_ctx *ctx;
  void *x;
  const void *g;
  int64_t g_stride;
  const void *b;
  int nrhs;
  isg_solve_info *info; /* nrhs records, or NULL */
} isg_group_member;
/* isg_bicgs for several independent problems at once, e.g. grids of different
 * sizes (one context each): members are distinct contexts on one device and
 * share hermitian, order and opts.  Every block of check_every iterations of
 * all members is one CUDA graph whose branches are the members' iteration
 * blocks (captured on the first poll, on streams other than the legacy
 * default stream), launched once per host poll; one poll reads every
 * member's active count.  Returns ISG_OK when every RHS of every member
 * reached tol, else the worst per-RHS status.  No counterpart in the
 * reference, which solves one problem at a time (mom.cpp:250-350). */
isg_status isg_bicgs_group(int nmembers, const isg_group_member *members, int hermitian, int order,
                           const isg_solve_opts *opts, isg_stream stream);

/* ---- receivers ---- */
/* rx[numrx] = far-field pattern of x (aggregate, matvec_gpu.cu:266-368;
 * solve.cpp:249-355), all levels on the device. */
isg_status isg_aggregate(isg_ctx *ctx, const void *x, void *rx, int nrhs, int order, isg_stream stream);
/* x[U] = back-projection of rx (aggregateh, matvec_gpu.cu:369-470;
 * solve.cpp:356-456), all levels on the device. */
isg_status isg_aggregateh(isg_ctx *ctx, void *x, const void *rx, int nrhs, int order, isg_stream stream);

/* ---- near-field receivers (the reference's commented dense form, setup_born.cpp:52-60) ----
 * numrx receivers at radius * (cos 2 pi m / numrx, sin 2 pi m / numrx) wavelengths (the
 * directions of mom.cpp:149-154 at a finite radius, outside the domain).  Builds on the device
 * the dense operator go[m][n] = integrate(rx_m, pos_n) (integrate.cpp:15-41) as FP16 hi/lo
 * tables for tcgen05 GEMMs (8 bytes per receiver and pixel, twice: forward and adjoint order);
 * radius 0 removes it.  While it is set, isg_measure and isg_dbim use it in place of the
 * far-field aggregate / aggregateh. */
isg_status isg_set_nearfield_receivers(isg_ctx *ctx, double radius);
/* rx[numrx] = go x per RHS (the near-field form of aggregate; the far-field aggregate when no
 * near-field receivers are set). */
isg_status isg_receive(isg_ctx *ctx, const void *x, void *rx, int nrhs, int order, isg_stream stream);
/* x[U] = gh rx per RHS, gh = conj(go)^T (setup_born.cpp:57-59; aggregateh when none are set). */
isg_status isg_receiveh(isg_ctx *ctx, void *x, const void *rx, int nrhs, int order, isg_stream stream);

/* Size of the device array isg_aggregate_noalloc works in (one per device). */
#define ISG_STATIC_SCRATCH_BYTES (64u << 20)
/* Same result as isg_aggregate, but allocates nothing: no cudaMalloc (which
 * can synchronise the whole device), no use of the context's workspaces.  For
 * callers that must not allocate at that point, e.g. a driver whose HBM is
 * fully committed to solve workspaces, or a loop that cannot afford an
 * allocator's device-wide synchronisation.  No counterpart in the reference.
 *  - isg_setup_gpu(ctx) must have run (ISG_BAD_ARG otherwise).  Set-up looks
 *    the array's device address up (cudaGetSymbolAddress) and loads the
 *    kernels this call launches; with CUDA's lazy module loading that is when
 *    the array's ISG_STATIC_SCRATCH_BYTES of device memory are taken, so
 *    every device with a set-up context holds them until the process exits,
 *    and the calls themselves need no free device memory.
 *  - Works in a fixed array of ISG_STATIC_SCRATCH_BYTES inside libisg.so:
 *    nrhs * (multipole samples per RHS, plus numunk unless order is
 *    ISG_ORDER_BLOCKED) * 8 bytes must fit, else ISG_BAD_ARG with the limit in
 *    isg_last_error (level 8: 2 RHS in tree/raster order, 4 in blocked order);
 *    nrhs is also capped at 65535 (one grid row per RHS).
 *  - The address belongs to the context's CUDA context: after a device reset
 *    the isg context (like all its workspaces) is invalid; create a new one.
 *  - One array per device per process: calls that overlap in time on the same
 *    device (other streams, threads or contexts) race on it. */
isg_status isg_aggregate_noalloc(isg_ctx *ctx, const void *x, void *rx, int nrhs, int order, isg_stream stream);

/* ---- inversion (distorted-Born / Polak-Ribiere nonlinear CG, mom.cpp:222-399) ---- */
typedef struct isg_dbim_opts {
  int iterations;        /* Polak-Ribiere iterations (mom.cpp:277 runs 3) */
  double regular;        /* Tikhonov weight; adds regular^2 chi per transmitter (mom.cpp:32,268-269) */
  int start_from_chi;    /* 0: chi = 0 and total field = incident (mom.cpp:225-229);
                            1: start from the caller's chi (the reference's commented restart, mom.cpp:230-245) */
  isg_solve_opts solve;  /* inner BiCGSTAB options (tol: mom.cpp:21); ISG_GUESS_LEARNED seeds the
                            forward solves of the total fields from the context's network */
  int warm_start;        /* 0: every solve starts from zero, as the reference; 1: each transmitter's
                            total-field and adjoint solves start from its fields of the previous
                            iteration (same tolerance; not in the reference) */
  const char *checkpoint;  /* directory, or NULL: writes the reference's outputs there, cg_<i>.bin
                            (contrast, raster order, complex128) and hist.txt (misfit, object error,
                            regularisation cost, gradient norm, object norm per line;
                            setup_born.cpp:171-242) after the first gradient and each iteration */
} isg_dbim_opts;

typedef struct isg_dbim_record {
  double misfit;         /* sum |mesd|^2 / sum |mes|^2            (setup_born.cpp:239-240) */
  double object_error;   /* sum |chi - chi_true|^2 / sum |chi_true|^2, or -1 without chi_true */
  double reg_cost;       /* sum |regular chi|^2 / sum |mes|^2 */
  double grad_norm;      /* sum |gradient|^2 */
  double object_norm;    /* sum |chi|^2 */
  double alpha;          /* step length of the iteration (mom.cpp:315); 0 in record 0 */
  double beta_re, beta_im; /* Polak-Ribiere coefficient (mom.cpp:394) */
  int64_t solves;        /* BiCGSTAB solves so far */
  int64_t iterations;    /* BiCGSTAB iterations so far */
} isg_dbim_record;

void isg_default_dbim_opts(isg_dbim_opts *o);
/* Synthetic measurements (setup_born.cpp:139-149): per transmitter a forward
 * solve with g = k0^2 chi, then the far-field pattern of g u.  inc: ntx
 * complex64 fields in `order`; chi: complex128 contrast eps_r - 1 in `order`;
 * mes: ntx x numrx complex64.  noise > 0 adds complex Gaussian noise of
 * standard deviation noise * ||mes|| / sqrt(2 ntx numrx) per real component. */
isg_status isg_measure(isg_ctx *ctx, int ntx, const void *inc, const double *chi, int order, double noise,
                       uint64_t seed, const isg_solve_opts *solve, void *mes, isg_stream stream);
/* The inversion loop: gradient by adjoint solves, Born-linearised step
 * length, contrast update, total-field re-solve, Polak-Ribiere direction, all
 * transmitters batched (chunks of max_rhs).  chi (complex128, in/out) and
 * chi_true (optional) are in `order`; hist receives iterations + 1 records. */
isg_status isg_dbim(isg_ctx *ctx, int ntx, const void *inc, const void *mes, const double *chi_true, double *chi,
                    int order, const isg_dbim_opts *opts, isg_dbim_record *hist, isg_stream stream);

/* ---- measurement ---- */
/* Number of CUDA kernels this library has launched in the process so far. */
int64_t isg_kernel_launches(void);
/* Runs the forward matvec `reps` times on nrhs internal test vectors and writes
 * the mean device time in ms of each stage: [0] P2M, [1] M2M (all levels),
 * [2] M2L+L2L (all levels), [3] L2P+near field, [4] whole matvec. */
isg_status isg_time_stages(isg_ctx *ctx, int nrhs, int engine, int reps, double *ms_out);

/* ---- seeded synthetic inputs (the reference reads a phantom file instead,
 *      setup_born.cpp:103-113) ---- */
typedef struct isg_phantom {
  int kind;            /* 0: random ellipses, 1: Gaussian random field */
  int count;           /* ellipses */
  double axis_min;     /* semi-axis range in wavelengths */
  double axis_max;
  double eps_min;      /* relative permittivity range (real part) */
  double eps_max;
  double tand_max;     /* loss tangent drawn from [0, tand_max] per ellipse */
  double corr_len;     /* Gaussian random field correlation length (wavelengths) */
  uint64_t seed;
} isg_phantom;
/* Writes the contrast chi = eps_r - 1 (complex128, raster order, side*side). */
isg_status isg_make_phantom(const isg_ctx *ctx, const isg_phantom *ph, double *chi_raster);
/* Plane waves exp(i k0 d.r) of transmitters first .. first+count-1 out of ntx
 * directions at angle 2 pi j / ntx (setup_born.cpp:62-65, mom.cpp:141-147),
 * count rows of complex128 in the given order. */
isg_status isg_make_plane_waves(const isg_ctx *ctx, int ntx, int first, int count, int order, double *inc);
/* Line sources integrate(r_tx, r)/res^2 at ntx points on a circle of the given
 * radius (the reference's near-field form, setup_born.cpp:66-72); rows as above. */
isg_status isg_make_line_sources(const isg_ctx *ctx, int ntx, int first, int count, double radius, int order,
                                 double *inc);

/* ---- launch-shape autotuner (no counterpart in the reference) ----
 * Times the candidate launch shapes of the level-dependent kernels (M2L rows
 * per thread, L2L and M2M columns per block, near-field tiles per tensor-core
 * CTA) on the context's buffers with nrhs right-hand sides and keeps the
 * fastest per level; later calls with at least nrhs / 4 RHS use them.  The
 * outputs do not depend on the shapes.  Overwrites the context's multipole and
 * local workspaces (no caller data). */
isg_status isg_autotune(isg_ctx *ctx, int nrhs, int engine, isg_stream stream);
/* The chosen shape: what 0 = M2L rows per thread, 1 = L2L columns, 2 = M2M
 * columns (per level), 3 = near-field tiles per CTA; 0 = built-in choice. */
isg_status isg_tuned(const isg_ctx *ctx, int what, int level, int *value);

/* ---- learned warm start (no counterpart in the reference) ----
 * A Fourier neural operator on the pixel grid maps the contrast g and the
 * incident field b of a forward solve to an estimate of its total field; with
 * ISG_GUESS_LEARNED, isg_bicgs starts from it and still iterates to tol.
 * Architecture: per-pixel lift of (chi, b, chi b) (chi = g / k0^2) to `width`
 * channels, `layers` spectral layers (GELU(W v + b + Re iDFT(R(k) DFT v)) over
 * the lowest `modes` x 2 `modes` frequencies; no GELU after the last), and a
 * per-pixel projection to a correction added to b.  FP32 parameters, trained
 * by the library's own forward/backward kernels and Adam. */
typedef struct isg_fno_opts {
  int width;     /* channels (default 32) */
  int modes;     /* retained kx modes; ky keeps 2 x modes (default 12) */
  int layers;    /* spectral layers (default 4) */
  int batch;     /* samples per device pass; sizes the activation buffers (default 4) */
  uint64_t seed; /* parameter initialisation */
  int tensor;    /* 1 (default): every GEMM of the network (lift, channel mixes, x transforms,
                    projection, and their backward products) runs on the tcgen05 tensor cores with
                    BF16 operands and FP32 accumulation, and the spectral weights are rounded to
                    BF16 where they multiply; the FP32 master parameters take the Adam updates.
                    0: the same network in FP32 on the CUDA cores. */
} isg_fno_opts;
void isg_default_fno_opts(isg_fno_opts *o);
/* Attach a freshly initialised network to the context (replaces any). */
isg_status isg_fno_create(isg_ctx *ctx, const isg_fno_opts *o);
int64_t isg_fno_param_count(const isg_ctx *ctx);
/* Copy the flat FP32 parameter vector (which 0) or the last gradient (which 1)
 * to host[n]; with set = 1, load parameters from host (which must be 0). */
isg_status isg_fno_params(isg_ctx *ctx, float *host, int64_t n, int which, int set);
/* x = b + N(g, b) for nrhs RHS (device complex64, caller order); g_stride 0 or numunk. */
isg_status isg_fno_apply(isg_ctx *ctx, const void *g, int64_t g_stride, const void *b, void *x, int nrhs, int order,
                         isg_stream stream);
/* Gradient of a loss over nrhs samples; *loss receives the loss.  With u (the
 * solver's total fields): mean_s ||x0_s - u_s||^2 / ||u_s||^2, x0 = b + N(g, b).
 * With u NULL: the initial residual of the forward solves it would seed,
 * mean_s ||b_s - A_s x0_s||^2 / ||b_s||^2 with A = I - G diag(g) (one forward
 * and one adjoint matvec per sample; needs no solved fields). */
isg_status isg_fno_grad(isg_ctx *ctx, const void *g, int64_t g_stride, const void *b, const void *u, int nrhs,
                        int order, double *loss, isg_stream stream);
/* isg_fno_grad followed by one Adam step (beta 0.9, 0.999) with learning rate lr. */
isg_status isg_fno_train_step(isg_ctx *ctx, const void *g, int64_t g_stride, const void *b, const void *u, int nrhs,
                              int order, float lr, double *loss, isg_stream stream);

#ifdef __cplusplus
}
#endif
#endif
