/*
 * f3r_b200.h -- C ABI of the B200-native nested mixed-precision F3R solver.
 *
 * The reference (suzuki-hpc/F3R) has no C interface: its plugin surface is the
 * type-erased C++ concepts in library/umineko-sparse/models.hpp
 * (Operator / CoefficientMatrix / Solver, solve(b, x, cond) -> solve_res_t),
 * and the F3R method itself is assembled in the experiment drivers
 * (work/src/f3r-gpu.cpp:210-265, work/src/f3r.cpp:195-248).  Each entry point
 * below names the reference interface it replaces.  A C++ adapter with the
 * reference's names lives in f3r_b200.hpp.
 *
 * Conventions
 *  - Every function returns an f3r_status; nothing calls exit().  The reference
 *    prints and exits on bad input (matrix/io.hpp:255-256, csr.hpp:111-114).
 *  - f3r_last_error_string() gives a message for the last failure on the
 *    calling thread.
 *  - Matrices cross the boundary as host CSR (f3r_csr, borrowed for the call).
 *    idx_t is int32 as in the reference (core/interface.hpp:8).
 *  - Device objects belong to an f3r_context (one device, one CUDA stream).
 *    Objects are not thread-safe; different contexts may run concurrently.
 *  - Vectors passed to f3r_sell_* / f3r_dot are device pointers.  The solve
 *    call accepts host or device pointers for b and x.
 */
#ifndef F3R_B200_H
#define F3R_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define F3R_B200_VERSION_MAJOR 0
#define F3R_B200_VERSION_MINOR 1

typedef enum f3r_status {
  F3R_SUCCESS = 0,
  F3R_ERROR_INVALID_VALUE = 1,  /* bad argument, shape or parameter */
  F3R_ERROR_CUDA = 2,           /* a CUDA runtime call failed */
  F3R_ERROR_OUT_OF_MEMORY = 3,
  F3R_ERROR_BREAKDOWN = 5,      /* zero or non-finite norm in an Arnoldi step */
  F3R_ERROR_TIMEOUT = 7,        /* a bounded device wait gave up */
  F3R_ERROR_UNSUPPORTED = 8,
  F3R_ERROR_NO_DEVICE = 9
} f3r_status;

typedef enum f3r_dtype { F3R_F64 = 0, F3R_F32 = 1, F3R_F16 = 2 } f3r_dtype;

typedef enum f3r_precond {
  F3R_PRECOND_SDAINV = 0,      /* SDAINV Z*(W^T r), as work/src/f3r-gpu.cpp:74,215-216 */
  F3R_PRECOND_ILU0_BJ = 1,     /* block-Jacobi ILU(0), exact triangular solves, as
                                  work/src/f3r.cpp:57-58,200-201 */
  F3R_PRECOND_ILU0_JACOBI = 2, /* the same ILU(0) factors, triangular solves by trsv_iters
                                  Jacobi sweeps (trsv/jacobi.hpp:290-505) */
  F3R_PRECOND_ILU0_BAJ = 3,    /* ... by trsv_iters in-place BAJ sweeps (trsv/baj.hpp:95-190);
                                  results depend on scheduling before convergence */
  F3R_PRECOND_ILU0_LEVEL = 4   /* one global ILU(0) (ilu_blocks ignored: ilu.hpp:128-164 with
                                  one block), exact triangular solves level-scheduled over the
                                  whole GPU; the same values as ILU0_BJ with ilu_blocks = 1 */
} f3r_precond;

/* Host CSR matrix, borrowed for the duration of a call.  Rows sorted by
 * column.  Replaces kmm::CSR<double, host> (matrix/csr.hpp:12-30). */
typedef struct f3r_csr {
  int32_t nrows, ncols, nnz;
  const int32_t *rptr; /* nrows + 1 */
  const int32_t *idx;  /* nnz */
  const double *val;   /* nnz */
} f3r_csr;

/* Solver parameters; defaults as the F3R drivers (f3r_params_default). */
typedef struct f3r_params {
  int32_t m_outer;         /* outer fp64 FGMRES restart length: 100 (f3r-gpu.cpp:264) */
  int32_t max_restarts;    /* Restarted cap: 20 (f3r-gpu.cpp:265) */
  int32_t m2, m3, m4;      /* fp32 level, fp16-matrix level, Richardson steps: 8, 4, 2.
                              m3 = 0 drops the fp16-matrix level: the fp32 level then applies
                              R directly (the depth-2 "F2" ablation, work/src/depth.cpp:157-162,
                              with m4 = 1 and static_weight = 1) */
  int32_t c;               /* adaptive-weight period: 64 (suite-gpu.py:49) */
  int32_t precond;         /* f3r_precond */
  int32_t ilu_blocks;      /* block-Jacobi blocks: 112 (f3r.cpp:57) */
  double sdainv_tol;       /* drop tolerance: 0.1 (f3r-gpu.cpp:74) */
  double acc;              /* diagonal shift for SDAINV / ILU: 1.0 */
  int32_t sell_c;          /* SELL slice height: 32, or 64 (64-row offset-aligned slices, every
                              64 rows sharing their column offsets, sigma 1: each lane of the
                              product works two rows with one set of slot bases; the same sums) */
  int32_t sell_sigma;      /* SELL sorting window: 1 = no sorting */
  double rel_tol;          /* stop when |implicit residual| / ||b|| < rel_tol and no
                              cond callback is given: 1e-8 (f3r-gpu.cpp:18) */
  int32_t half_scale_log2; /* 0: plain fp32->fp16 cast of the Richardson input, as the
                              reference (f3r-gpu.cpp:231); k>0: scale it by 2^k and
                              back (a linear operator, so the result is unchanged in
                              exact arithmetic) */
  int32_t use_graphs;      /* 1: replay the fixed inner levels as CUDA graphs */
  int32_t sell_index16;    /* 0: 32-bit column indices; 1: 16-bit offsets from a per-slice-column
                              base when every slice column fits a 65536 window (32-bit otherwise).
                              Fewer bytes, but on B200 the 32-bit form streams faster (the SpMV
                              is bound by copies in flight, not by bytes) */
  double static_weight;    /* 0: adaptive weights (F3R).  w > 0: fixed weight w for every
                              Richardson step, never updated ("F3R-Static",
                              work/src/static.cpp:99-114) */
  int32_t trsv_iters;      /* ILU0_JACOBI: sweeps per triangular solve (Jacobi max_ier, 2);
                              ILU0_BAJ: BAJ max_iter (the first is the diagonal scaling) */
  int32_t format;          /* f3r_format: F3R_FORMAT_SELL (0, SELL-C-sigma as the GPU drivers,
                              f3r-gpu.cpp:66) or F3R_FORMAT_CSR (CSR as the CPU driver, f3r.cpp:50;
                              sigma 1, no SELL options).  Both give the same sums */
  double trsv_omega;       /* ILU0_JACOBI: damping omega in (0, 2], 1.0 */
  int32_t inner_sstep;     /* bit 0: level 2, bit 1: level 3 run as sFGMRES (solver/gmres2.hpp:
                              137-221): all m preconditioner + matrix applications first, on the
                              raw vectors W(j+1) = A M W(j), then the Gram-Schmidt steps.  0 */
  int32_t sell_align;      /* 1: offset-aligned SELL slices where the rows of a slice share their
                              column offsets (stencil, banded structure): no column index is
                              stored there, so an fp16 entry streams 2 bytes instead of 6.  With
                              sell_sigma = 1 a stencil aligns every slice.  Same sums in the same
                              order as the packed layout.  0 */
  int32_t sell_autotune;   /* 1: at set-up, build the fp16 copy of the matrix in each candidate
                              layout (offset-aligned SELL sigma 1 with 32- and 64-row slices; packed
                              SELL sigma 1 with 32- and 16-bit indices; packed and aligned SELL
                              sigma 256; CSR), time the fp16
                              product on it, and solve in the fastest; the layout fields above are
                              then ignored (f3r_solver_info reports the choice).  All give the same
                              sums at sigma 1; sigma 256 permutes the rows.  0 */
  int32_t half_m;          /* > 0: an FGMRES level whose basis vectors V and Z are stored in fp16
                              (FGMRES<_Float16> of work/src/depth.cpp:122-167), half_m Arnoldi steps,
                              directly above R: called by level 3, by level 2 when m3 = 0, or by the
                              outer level when m2 = 0 (m2 = 0 is allowed only with half_m > 0).  Its
                              products are fp16 x fp16 with fp32 accumulation, its dots, norms,
                              Hessenberg and Givens rotations fp32 (the reference computes them in
                              fp16), R's input and output its fp16 vectors.  The paper's F4 is m2 8,
                              m3 4, half_m 2; F3H m2 8, m3 0, half_m 8; F2H m2 0, half_m 64; each with
                              m4 1, static_weight 1 and block-Jacobi ILU(0).  0 */
  int32_t diag_load;       /* diagonal SDAINV factors (W^T and Z both diagonal): where every fp16
                              value of both is exactly 1 (what tol 0.1 leaves of a diagonally
                              scaled stencil), the Richardson kernels multiply by the constant 1
                              instead of loading it -- the same arithmetic, 4 bytes a row fewer.
                              1: load the factors always.  0 */
  int32_t reserved[5];
} f3r_params;

/* Solve outcome.  The first three fields are solve_res_t
 * (umineko-sparse/models.hpp:191-200). */
typedef struct f3r_result {
  int32_t is_solved;
  int32_t res_iter;          /* outer FGMRES steps over all restarts */
  double res_nrm2;           /* |e| of the last Givens estimate (absolute) */
  double impl_rel_res;       /* res_nrm2 / ||b|| */
  double expl_rel_res;       /* ||b - A x|| / ||b|| recomputed in fp64 */
  int32_t restarts;          /* outer FGMRES calls */
  int32_t reserved0;
  int64_t inner_applications;/* Richardson applications; the drivers' CSV Iter is this times m4
                                (res_iter * m2 * m3 * m4, f3r-gpu.cpp:94-98,280-282) */
  double solve_seconds;      /* device time of the solve (CUDA events) */
  int64_t kernel_launches;   /* kernels of this library the solve ran (graph nodes included) */
} f3r_result;

/* cond(i, |e|): nonzero stops the solve; the reference's
 * std::function<bool(int, double)> (models.hpp:208-211). */
typedef int (*f3r_cond_fn)(int32_t iter, double res_nrm2, void *user);

typedef struct f3r_host_matrix f3r_host_matrix;
typedef struct f3r_context f3r_context;
typedef struct f3r_sell f3r_sell;
typedef struct f3r_solver f3r_solver;

typedef struct f3r_sell_info {
  int32_t nrows, ncols, nnz;
  int32_t slice_height, sigma, nslices;
  int64_t nnz_padded;       /* stored entries including slice padding */
  int32_t max_width;        /* widest slice (entries per row) */
  int32_t dtypes;           /* bit (1 << f3r_dtype) set for each value copy held */
  int32_t index_bits;       /* 32, 16 (offsets from per-slice-column bases) or 0 (offset-aligned
                               slices, with or without explicit 32-bit slices among them) */
} f3r_sell_info;

/* f3r_sell_create dtype_mask flag: store the column indices as 16-bit offsets
 * when they fit (see f3r_params.sell_index16). */
#define F3R_SELL_INDEX16 (1 << 8)
/* f3r_sell_create dtype_mask flag: offset-aligned slices where they fit (see
 * f3r_params.sell_align). */
#define F3R_SELL_ALIGNED (1 << 9)
/* f3r_sell_create dtype_mask flag: keep the matrix in CSR (sigma must be 1;
 * f3r_sell_info reports slice_height 0).  The kernels sum each row in column
 * order as the packed SELL kernel does, so the results are the same. */
#define F3R_SELL_CSR (1 << 10)

/* f3r_params.format */
typedef enum f3r_format { F3R_FORMAT_SELL = 0, F3R_FORMAT_CSR = 1 } f3r_format;

/* ---------------------------------------------------------------- errors */
const char *f3r_last_error_string(void);
const char *f3r_status_string(f3r_status s);

/* ------------------------------------------------------- host matrices
 * Host-side set-up, native C++.  The reference does all of this on the host
 * too (matrix/algorithm.hpp, preconditioner/ainv.hpp, preconditioner/ilu.hpp). */
f3r_status f3r_host_matrix_from_csr(const f3r_csr *a, f3r_host_matrix **out);
f3r_status f3r_host_matrix_view(const f3r_host_matrix *m, f3r_csr *view);
void f3r_host_matrix_destroy(f3r_host_matrix *m);

/* 27-point stencil on an nx*ny*nz grid (diagonal 26, neighbours -1).
 * variant 0: matrix/hpcg.cpp:13-57.  1: matrix/hpgmp.cpp:13-57 (pure +-z
 * neighbours -1-beta / -1+beta).  2: half-space nonsymmetric form (neighbours
 * at a positive linear offset -1+beta, negative -1-beta).  Any grid size. */
f3r_status f3r_problem_stencil27(int32_t nx, int32_t ny, int32_t nz, int32_t variant,
                                 double beta, f3r_host_matrix **out);

/* 7-point variable-coefficient diffusion: face coefficient = harmonic mean of
 * exp(g) of the two cells, g a seeded stationary Gaussian random field (std
 * sigma, periodic Gaussian filter of correlation length corr_len cells),
 * Dirichlet boundary folded into the diagonal.  No reference counterpart (a
 * synthetic stress matrix). */
f3r_status f3r_problem_diffusion7(int32_t nx, int32_t ny, int32_t nz, double sigma,
                                  double corr_len, uint64_t seed, f3r_host_matrix **out);

/* D^{-1/2} A D^{-1/2} with D = |diag(A)|, in place.  Replaces
 * kmm::algorithm::scaling (matrix/algorithm.hpp:45-59). */
f3r_status f3r_host_scaling(f3r_host_matrix *m);

/* y = A x on the host in fp64 (set-up of right-hand sides b = A x*). */
f3r_status f3r_host_spmv(const f3r_csr *a, const double *x, double *y);

/* n values uniform in [lo, hi) from std::mt19937_64(seed), the generator
 * the reference uses for right-hand sides (matrix/io.hpp:112-118,
 * core/tensor.hpp:253-265). */
f3r_status f3r_random_uniform(uint64_t seed, double lo, double hi, int64_t n, double *out);

/* SDAINV factors: returns Z and W^T so that M r = Z (W^T r).  Replaces
 * kmm::algorithm::sdainv (preconditioner/ainv.hpp:27-65, 268-329). */
f3r_status f3r_host_sdainv(const f3r_csr *a, double tol, double acc, f3r_host_matrix **z,
                           f3r_host_matrix **wt);

/* Block-Jacobi ILU(0): L (unit diagonal stored last in each row) and U
 * (diagonal first).  Replaces CSR::duplicate_block_diagonal + algorithm::ilup
 * + algorithm::split (csr.hpp:109-155, ilu.hpp:128-164, algorithm.hpp:9-43).
 * Rejects block counts for which the reference's block pointers overrun
 * ((blocks-1) * ceil(n/blocks) > n). */
f3r_status f3r_host_ilu0_bj(const f3r_csr *a, int32_t blocks, double acc, f3r_host_matrix **l,
                            f3r_host_matrix **u);

/* ---------------------------------------------------------- Matrix Market
 * The on-disk formats either side of the solve (umineko-sparse/matrix/io.hpp).
 *
 * f3r_mm_read: a "matrix coordinate" file (real or integer; general or
 * symmetric) as host CSR.  Replaces io::mm::read_matrix + io::CSR(COO)
 * (io.hpp:91-96, 44-60, 129-192): explicit off-diagonal zeros are dropped,
 * symmetric files expanded, rows sorted by column, duplicates kept.
 * Pattern, complex, skew-symmetric and hermitian files are refused
 * (F3R_ERROR_UNSUPPORTED) where the reference would misread them. */
f3r_status f3r_mm_read(const char *path, f3r_host_matrix **out);
/* An n x 1 "matrix array real general" file into x[0..n) (io.hpp:196-216). */
f3r_status f3r_mm_read_vector(const char *path, int64_t n, double *x);
/* The right-hand side io::mm::read_system pairs with a matrix file
 * (io.hpp:104-126): "<stem>_b.mtx" ("_b" inserted before the last four
 * characters of matrix_path) when it exists, else n values U(0, 1) from
 * std::mt19937_64(0), the drivers' init (f3r-gpu.cpp:60).  *from_file (may be
 * NULL) is 1 when the file was read. */
f3r_status f3r_mm_read_rhs(const char *matrix_path, int64_t n, double *b, int32_t *from_file);
/* Writes a general coordinate file (1-based, %.17g values: exact round trip). */
f3r_status f3r_mm_write(const char *path, const f3r_csr *a);
/* Writes an n x 1 array file (%.17g). */
f3r_status f3r_mm_write_vector(const char *path, int64_t n, const double *x);

/* ------------------------------------------------- Jacobi triangular solves
 * trsv::{l,ld,du}::Jacobi<SELL<32, __half>> and BAJ<SELL<32, __half>>
 * (trsv/jacobi.hpp:290-505, trsv/baj.hpp:95-190) on the device: `iters`
 * parallel sweeps instead of a sequential triangular solve.  The factor is
 * given in its stored form (host CSR); vectors are fp16 device pointers. */
typedef struct f3r_trsv f3r_trsv;
typedef enum f3r_trsv_form {
  F3R_TRSV_LOWER = 0,   /* lower, unit diagonal stored last in each row (not read) */
  F3R_TRSV_LOWER_D = 1, /* lower, diagonal stored last */
  F3R_TRSV_D_UPPER = 2  /* upper, diagonal stored first */
} f3r_trsv_form;
typedef enum f3r_trsv_kind {
  F3R_TRSV_JACOBI = 0, /* y0 = w D^-1 in; iters sweeps y = w D^-1 (in - N y) + (1 - w) y */
  F3R_TRSV_BAJ = 1     /* y = D^-1 in; iters - 1 in-place sweeps y = D^-1 (in - N y) */
} f3r_trsv_kind;
f3r_status f3r_trsv_create(f3r_context *ctx, const f3r_csr *m, int32_t form, int32_t kind, int32_t iters,
                           double omega, f3r_trsv **out);
/* out = the approximate M^-1 in, on the context's stream; in must not be out. */
f3r_status f3r_trsv_solve(f3r_trsv *t, const void *in, void *out);
void f3r_trsv_destroy(f3r_trsv *t);

/* ---------------------------------------------------------------- context */
f3r_status f3r_context_create(int32_t device, f3r_context **out);
void f3r_context_destroy(f3r_context *ctx);
/* Use an external CUDA stream (cudaStream_t) instead of the context's own;
 * NULL restores the context's stream.  The context's own stream is a
 * blocking stream: it orders with work on the legacy default stream, so a
 * caller that fills inputs on the default stream needs no extra sync. */
f3r_status f3r_context_set_stream(f3r_context *ctx, void *stream);
f3r_status f3r_context_synchronize(f3r_context *ctx);

/* -------------------------------------------------------- SELL-C-sigma
 * Device sparse matrix.  Replaces kmm::SELL<32, T, device> (matrix/sell.hpp:
 * 37-97) and SELLsig<32, sigma, T, device> (sell.hpp:99-166).  One column
 * index array is shared by the fp64 / fp32 / fp16 value copies selected by
 * dtype_mask (bit 1 << f3r_dtype); with F3R_SELL_INDEX16 the indices are
 * stored as 16-bit offsets when they fit. */
f3r_status f3r_sell_create(f3r_context *ctx, const f3r_csr *a, int32_t slice_height,
                           int32_t sigma, int32_t dtype_mask, f3r_sell **out);
f3r_status f3r_sell_info_get(const f3r_sell *m, f3r_sell_info *info);
void f3r_sell_destroy(f3r_sell *m);

/* out = A in, values at val_t, accumulation in fp64 for fp64 values and fp32
 * otherwise.  Replaces SELL::operate (sell.hpp:56-71) / CoefficientMatrix::
 * operate (models.hpp:133-136).  Supported (val_t, in_t, out_t): (F64, F64,
 * F64), (F32, F32, F32), (F16, F32, F32), (F16, F16, F16), (F16, F16, F32). */
f3r_status f3r_sell_operate(f3r_sell *m, f3r_dtype val_t, f3r_dtype in_t, const void *in,
                            f3r_dtype out_t, void *out);

/* res = rhs - A in.  Replaces SELL::compute_residual (sell.hpp:72-89) /
 * CoefficientMatrix::compute_residual (models.hpp:137-141).  Supported:
 * all three types equal to val_t's vector type (F64/F64, F32/F32, F16/F16). */
f3r_status f3r_sell_compute_residual(f3r_sell *m, f3r_dtype val_t, f3r_dtype rhs_t,
                                     const void *rhs, f3r_dtype in_t, const void *in,
                                     f3r_dtype res_t, void *res);

/* One launch shape of the SELL SpMV and its measured time (f3r_sell_tune). */
typedef struct f3r_tune_entry {
  int32_t warps, stages, kc;  /* warps per CTA, bulk-copy stages per warp, columns per copy */
  int32_t index_bits;         /* 32 or 16 (the matrix's index form) */
  int32_t is_default;         /* 1 for the shape the library launches */
  int32_t reserved;
  double microseconds;        /* mean time of one product out = A x */
  double gbs_algorithmic;     /* (nnz*(s_val+4) + 4(n+1) + n*s_x + n*s_y) / time */
} f3r_tune_entry;

/* Launch-shape autotuner: times out = A x (fp16 values with fp32 vectors,
 * fp32, or fp64) on this matrix at every launch shape the library carries,
 * reps launches each, and returns up to cap entries, fastest first.  No
 * reference counterpart (the reference has one kernel shape). */
f3r_status f3r_sell_tune(f3r_sell *m, f3r_dtype val_t, int32_t reps, f3r_tune_entry *out, int32_t cap,
                         int32_t *count);

/* Runs the level-scheduled ILU solve's bounded dependency wait on one device
 * flag that is already set (set != 0) or that nothing sets (set = 0), with a
 * limit of limit_ms (1..10000) instead of the kernels' 2 s.  Returns
 * F3R_SUCCESS, or F3R_ERROR_TIMEOUT once the limit has passed; either way the
 * context's device error word is clear again and the context stays usable.
 * A check of the failure path for callers and tests; no reference
 * counterpart (the reference never waits on the device). */
f3r_status f3r_context_wait_probe(f3r_context *ctx, int32_t set, int32_t limit_ms);

/* *result = <x, y> over n entries (fp64 for F64, fp32 accumulation otherwise;
 * F16 inputs are widened to fp32 as the reference's wildcard(., tof32),
 * f3r-gpu.cpp:236).  Replaces kmm::dot (core/tensor.hpp:509-537, 686-688).
 * Synchronises the context's stream. */
f3r_status f3r_dot(f3r_context *ctx, f3r_dtype t, int64_t n, const void *x, const void *y,
                   double *result);

/* *result (a DEVICE pointer, written by the kernel) = <x, y> over n entries,
 * like f3r_dot but without a context and without allocating anything: for
 * callers that cannot call cudaMalloc (code running inside an allocator's own
 * bookkeeping, or a device whose memory is all held by a pool the caller
 * does not control).  No counterpart in the reference.  Its reduction scratch
 * is a fixed 64 KB (+256 B) device array inside the library, held on every
 * GPU that loads the library until exit; n is limited to 33,554,432 elements
 * (larger n returns F3R_ERROR_INVALID_VALUE).  Asynchronous on `stream`
 * (cudaStream_t; NULL = the default stream).  The first call on a device
 * looks up the array's device address, so make it before any stream
 * capture.  Calls that overlap on the GPU share the array and race. */
f3r_status f3r_dot_noalloc(f3r_dtype t, int64_t n, const void *x, const void *y, double *result,
                           void *stream);

/* ----------------------------------------------------------------- solver
 * The nested F3R solver: Restarted<double>( FGMRES<double>(A, FGMRES<float>(
 * A32, FGMRES<float>(A16, R, m3), m2), m_outer), max_restarts ), with R the
 * adaptive-weight fp16 Richardson over the preconditioner (f3r-gpu.cpp:
 * 229-265).  `a` is the system matrix as solved (apply f3r_host_scaling first
 * to match the drivers, f3r-gpu.cpp:65).  The preconditioner is built here. */
void f3r_params_default(f3r_params *p);
f3r_status f3r_solver_create(f3r_context *ctx, const f3r_csr *a, const f3r_params *p,
                             f3r_solver **out);
/* Solve A x = b.  x holds the initial guess on entry.  b and x may be host
 * or device pointers.  cond may be NULL (then rel_tol applies).  Replaces
 * Restarted::solve / Solver::solve (solver/restart.hpp:26-36,
 * models.hpp:207-211). */
f3r_status f3r_solver_solve(f3r_solver *s, const double *b, double *x, f3r_cond_fn cond,
                            void *user, f3r_result *result);
/* a_info: the stored matrix; precond_diagonal: 0 for general factors, 1 when
 * W^T and Z are both diagonal, 2 when moreover every fp16 value of both is
 * exactly 1 and the Richardson kernels take the constant (diag_load = 0) */
f3r_status f3r_solver_info(const f3r_solver *s, f3r_sell_info *a_info, int32_t *precond_diagonal);
/* Several right-hand sides: column k of B (b + k * ldb) is solved into
 * column k of X (x + k * ldx), x holding the initial guesses; ldb, ldx >= n;
 * host or device pointers; results (may be NULL) gets one entry per column.
 * With SDAINV and SELL storage (packed or offset-aligned, 32- or 64-row
 * slices) the columns run in lockstep blocks of up to 16 (8 from 2^20 rows;
 * a single column left over is solved alone): every product streams the matrix once
 * for the block, each column keeps its own Hessenberg matrix, rotations and
 * Richardson weights, and its result is its single solve's bit for bit.  cond
 * is then called once per outer step for each column still running, in
 * column order; a column stops when its cond (or rel_tol) says so, and the
 * block restarts until every column has stopped.  Other configurations solve
 * the columns one after another on this solver's device objects.  The nrhs
 * argument of the planned boundary's solve call. */
f3r_status f3r_solver_solve_multi(f3r_solver *s, int32_t nrhs, const double *b, int64_t ldb, double *x, int64_t ldx,
                                  f3r_cond_fn cond, void *user, f3r_result *results);
/* Independent systems at once: system i is f3r_solver_solve_multi(solvers[i],
 * nrhs[i], b[i], ldb[i], x[i], ldx[i], ...).  Solvers on different contexts
 * (streams) run concurrently, one host thread per context (at most 128),
 * solvers sharing a context one after another; so cond may be called from
 * several threads at once.  results holds sum(nrhs) entries, system by
 * system.  Every system is attempted; the first failing one (in index order)
 * gives the status.  The batched solve of the planned boundary
 * (f3r_solve_batch(handles[], ...)); the reference has no counterpart. */
f3r_status f3r_solve_batch(int32_t count, f3r_solver *const *solvers, const int32_t *nrhs, const double *const *b,
                           const int64_t *ldb, double *const *x, const int64_t *ldx, f3r_cond_fn cond, void *user,
                           f3r_result *results);

/* out = A in with the solver's own device copy of A (the matrix its levels
 * use: SELL-C-sigma, rows and columns in the solver's storage order P A P^T,
 * so with sigma > 1 `in` and `out` are in that order too).  Same type
 * combinations as f3r_sell_operate.  The kernel-level view of
 * CoefficientMatrix::operate (models.hpp:133-136) on the solved system. */
f3r_status f3r_solver_operate(f3r_solver *s, f3r_dtype val_t, f3r_dtype in_t, const void *in, f3r_dtype out_t,
                              void *out);
void f3r_solver_destroy(f3r_solver *s);

/* As f3r_solver_create with precond F3R_PRECOND_SDAINV, but the SDAINV
 * factors are given instead of computed: M r = Z (W^T r), Z and W^T square
 * CSR of a's size (for example f3r_host_sdainv's factors with their values
 * corrected by f3r_learned_correct).  The reference builds them itself
 * (work/src/f3r-gpu.cpp:74). */
f3r_status f3r_solver_create_factors(f3r_context *ctx, const f3r_csr *a, const f3r_params *p, const f3r_csr *z,
                                     const f3r_csr *wt, f3r_solver **out);

/* ---- batches of systems of one sparsity pattern --------------------------
 * Up to 16 systems that share one pattern (one grid and stencil with
 * different coefficients, for example) solved together: one lockstep solve
 * K columns wide (K = 2, 4, 8 or 16, the systems padded with inactive
 * columns), each column its own system with its own matrix values and its
 * own SDAINV factors, every product streaming the shared pattern once and
 * the systems' values interleaved.  Each system's result is that of
 * f3r_solver_solve on it with the same parameters, up to the layout: the
 * batch stores the matrices in packed SELL (sell_align, sell_index16 and
 * sell_autotune are ignored).  Takes F3R_PRECOND_SDAINV, FGMRES levels (no
 * inner_sstep, no half_m) and format SELL.  The reference solves one
 * system per run (work/src/f3r-gpu.cpp:88); it has no counterpart. */
typedef struct f3r_batch f3r_batch;
/* a[i]: system i (count of them, one pattern); z, wt: NULL (SDAINV computed
 * per system) or count given factor pairs as f3r_solver_create_factors */
f3r_status f3r_batch_create(f3r_context *ctx, int32_t count, const f3r_csr *const *a, const f3r_params *p,
                            const f3r_csr *const *z, const f3r_csr *const *wt, f3r_batch **out);
/* b[i], x[i]: system i's right-hand side and initial guess / solution, host
 * or device vectors; results: one per system (may be NULL).  cond(i, |e|)
 * is called for every unfinished system after every outer step, in order. */
f3r_status f3r_batch_solve(f3r_batch *b, const double *const *bv, double *const *x, f3r_cond_fn cond, void *user,
                           f3r_result *results);
/* count: systems; width: the block's K; precond_diagonal: 1 when every
 * system's SDAINV factors are diagonal, 2 when moreover all their fp16 values
 * (padding columns of a partial block included) are exactly 1 */
f3r_status f3r_batch_info(const f3r_batch *b, int32_t *count, int32_t *width, int32_t *precond_diagonal);
void f3r_batch_destroy(f3r_batch *b);

/* ---- learned correction of the SDAINV values ---------------------------
 * No reference counterpart.  A network 7 -> 64 -> 64 -> 8 (ReLU) maps the
 * seven coefficients of row i of a 7-point matrix in natural order (column
 * offsets 0, -1, +1, -nx, +nx, -nx*ny, +nx*ny) to corrections delta of that
 * row's SDAINV entries on their fixed pattern: Z entries at offsets
 * {0, +1, +nx, +nx*ny} and W^T entries at {0, -1, -nx, -nx*ny} become
 * v (1 + delta); entries at other offsets keep their values.  The output
 * layer starts at zero (an untrained network is plain SDAINV).  Training
 * (fp32 weights, hand-written forward / backward kernels, Adam) minimises
 * 1/P sum_p ||Z' W'^T r_p - e_p||^2 / ||e_p||^2 over residual / error pairs;
 * inference runs in BF16 on tensor cores with fp32 accumulation.
 * Parameters, flat fp32: W1 (64 x 7), b1 (64), W2 (64 x 64), b2 (64),
 * W3 (8 x 64), b3 (8); W row-major (outputs x inputs); 5192 in all. */
typedef struct f3r_learned f3r_learned;
/* hidden must be 64; seed draws the He-normal hidden layers */
f3r_status f3r_learned_create(f3r_context *ctx, int32_t hidden, uint64_t seed, f3r_learned **out);
void f3r_learned_destroy(f3r_learned *l);
/* count (may be NULL) receives the parameter count; params (may be NULL)
 * is read from the network (set = 0) or written to it (set != 0) */
f3r_status f3r_learned_params(f3r_learned *l, float *params, int32_t set, int64_t *count);
/* The training data: a 7-point matrix (several systems of one grid shape
 * may be stacked block-diagonally), its grid strides nx and nx*ny, its
 * SDAINV factors, and npairs (1..1024) pairs, r and e each npairs x n
 * (pair-major, host memory), A e_p = r_p up to the solver's error. */
f3r_status f3r_learned_set_data(f3r_learned *l, const f3r_csr *a, int32_t nx, int32_t ny, const f3r_csr *z,
                                const f3r_csr *wt, int32_t npairs, const double *r, const double *e);
/* loss at the current parameters; grad (may be NULL; 5192 floats) its gradient */
f3r_status f3r_learned_evaluate(f3r_learned *l, double *loss, float *grad);
/* steps full-batch Adam steps (beta 0.9 / 0.999); losses (may be NULL)
 * receives the loss before each step */
f3r_status f3r_learned_train(f3r_learned *l, int32_t steps, double lr, double *losses);
/* Corrected factor values of a system: z_val / wt_val (nnz of z / wt) and,
 * when delta is not NULL, the raw network outputs (n x 8).  bf16 selects the
 * forward pass: 0 the fp32 training forward pass, 1 BF16 inference on the
 * tcgen05 tensor cores (TMEM accumulators), 2 BF16 inference on mma.sync
 * (the warp-level tensor-core path, kept for comparison); 1 and 2 share their
 * arithmetic (bf16 operands, fp32 accumulation and bias). */
f3r_status f3r_learned_correct(f3r_learned *l, const f3r_csr *a, int32_t nx, int32_t ny, const f3r_csr *z,
                               const f3r_csr *wt, int32_t bf16, double *z_val, double *wt_val, float *delta);
/* Device time of the network alone on a system's features (mode as bf16
 * above): one warm-up launch, then reps launches timed with CUDA events on
 * the context's stream; *us = microseconds per launch. */
f3r_status f3r_learned_time_inference(f3r_learned *l, const f3r_csr *a, int32_t nx, int32_t ny, const f3r_csr *z,
                                      const f3r_csr *wt, int32_t mode, int32_t reps, double *us);

#ifdef __cplusplus
}
#endif

#endif /* F3R_B200_H */
