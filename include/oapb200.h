/*
 * oapb200 - B200-native (sm_100a) Arnoldi eigensolver hot path of oap.
 *
 * C ABI.  Plain pointers, sizes and status codes; no C++ or torch types.
 *
 * Matrix convention (the reference's math::Matrix, oapMatrix/Matrix.h:31-44,
 * oapMatrix/MatrixAPI.h:33-40): split real / imaginary planes, row-major,
 * element (column c, row r) at index c + r * columns.  A NULL plane is absent
 * (a real matrix has im == NULL).  A vector is 1 column x n rows.  Every
 * operator-surface call takes FP64 planes, like the reference's
 * floatt = double (project_generic.mk:34).
 *
 * Unlike the reference, the matrix handle lives on the HOST (no device
 * struct dereference, no global registry lookup): its re / im pointers are
 * device pointers.
 *
 * Errors never abort the process (the reference aborts on every CUDA error,
 * oapCuda/KernelExecutor.h:34-41); each call returns an oapb_status.
 * `stream` is a cudaStream_t (NULL = the legacy default stream).  Calls that
 * return a host scalar synchronise that stream; the others are asynchronous.
 */
#ifndef OAPB200_H
#define OAPB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define OAPB_EXPORT __attribute__((visibility("default")))
#else
#define OAPB_EXPORT
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define OAPB_API_VERSION 1

typedef enum oapb_status {
  OAPB_OK = 0,
  OAPB_ERR_ARG = 1,          /* invalid argument (dims, NULL planes, sizes) */
  OAPB_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  OAPB_NOT_CONVERGED = 3,    /* restart budget spent before the residual goal */
  OAPB_ERR_TIMEOUT = 4,      /* a bounded device-side loop gave up */
  OAPB_ERR_BOUNDS = 5,       /* a device-side bounds check fired */
  OAPB_ERR_CALLBACK = 6,     /* the user matvec callback returned non-zero */
  OAPB_ERR_NOMEM = 7,        /* device allocation failed */
  OAPB_ERR_BREAKDOWN = 8,    /* the Krylov space became invariant before hdim */
  OAPB_ERR_NONFINITE = 9     /* a NaN or infinity reached the Krylov vectors
                                (operator or callback output) or a residual */
} oapb_status;

/* Element type of a plane. */
typedef enum oapb_dtype { OAPB_F64 = 0, OAPB_F32 = 1 } oapb_dtype;

/* Host-side matrix handle over device planes (math::Matrix). */
typedef struct oapb_mat {
  uint32_t columns;
  uint32_t rows;
  void* re;        /* device pointer or NULL */
  void* im;        /* device pointer or NULL */
  int32_t dtype;   /* oapb_dtype */
} oapb_mat;

OAPB_EXPORT const char* oapb_status_string(int status);
OAPB_EXPORT int oapb_api_version(void);

/* ------------------------------------------------------------------------ */
/* Operator surface: oap::CuProceduresApi (oapMatrixCuda/CuProceduresApi.h)  */
/* ------------------------------------------------------------------------ */

/* output = params0 * params1 (CuProceduresApi.h:74, CuProceduresApi.cpp:91-105).
 * output: c x r, params0: k x r, params1: c x k.  A matrix-vector product
 * (params1 a 1-column vector) takes the coalesced GEMV path. */
OAPB_EXPORT int oapb_dot_product(const oapb_mat* output, const oapb_mat* params0,
                     const oapb_mat* params1, void* stream);

/* output = params0^T / params0^H (CuProceduresApi.h:171-173, .cpp:268-307). */
OAPB_EXPORT int oapb_transpose(const oapb_mat* output, const oapb_mat* params0, void* stream);
OAPB_EXPORT int oapb_conjugate_transpose(const oapb_mat* output, const oapb_mat* params0,
                             void* stream);

/* output = sqrt(sum |x|^2) (CuProceduresApi.h:199, .cpp:342-345). */
OAPB_EXPORT int oapb_magnitude(double* output, const oapb_mat* params0, void* stream);

/* (reoutput, imoutput) = (sum re, sum im) (CuProceduresApi.h:201-202, .cpp:358-389). */
OAPB_EXPORT int oapb_sum(double* reoutput, double* imoutput, const oapb_mat* matrix,
             void* stream);

/* Kronecker product (CuProceduresApi.h:57, .cpp:136-156): output is
 * (c0 * c1) x (r0 * r1), output[y][x] = p0[y / r1][x / c1] * p1[y % r1][x % c1]. */
OAPB_EXPORT int oapb_tensor_product(const oapb_mat* output, const oapb_mat* params0,
                        const oapb_mat* params1, void* stream);

/* element-wise output = params0 +/- params1 (CuProceduresApi.h:175-189). */
OAPB_EXPORT int oapb_add(const oapb_mat* output, const oapb_mat* params0,
             const oapb_mat* params1, void* stream);
OAPB_EXPORT int oapb_substract(const oapb_mat* output, const oapb_mat* params0,
                   const oapb_mat* params1, void* stream);

/* v = f * re (CuProceduresApi.h:215) and v = f * (re + i im), a complex scale
 * (CuProceduresApi.h:217). */
OAPB_EXPORT int oapb_multiply_re_constant(const oapb_mat* v, const oapb_mat* f, double re,
                              void* stream);
OAPB_EXPORT int oapb_multiply_constant(const oapb_mat* v, const oapb_mat* f, double re,
                           double im, void* stream);

/* output[r][column] = params0[r] for r < length (CuProceduresApi.h:191-197,
 * CuVectorUtils.h:27-69) and the inverse copy. */
OAPB_EXPORT int oapb_set_vector(const oapb_mat* output, uint32_t column,
                    const oapb_mat* params0, uint32_t length, void* stream);
OAPB_EXPORT int oapb_get_vector(const oapb_mat* vector, uint32_t length,
                    const oapb_mat* matrix, uint32_t column, void* stream);

/* I, diag(re + i im), 0 (CuProceduresApi.h:219-223). */
OAPB_EXPORT int oapb_set_identity(const oapb_mat* matrix, void* stream);
OAPB_EXPORT int oapb_set_diagonal(const oapb_mat* matrix, double re, double im, void* stream);
OAPB_EXPORT int oapb_set_zero_matrix(const oapb_mat* matrix, void* stream);

/* Givens QR A = Q R of a square matrix in one CTA (CuProceduresApi.h:303-304,
 * CuQRProcedures_GR.h:38-150).  Rotation order and sign convention of the
 * reference (c = x / r, s = y / r), FP64 throughout. */
OAPB_EXPORT int oapb_qr_givens(const oapb_mat* Q, const oapb_mat* R, const oapb_mat* A,
                   void* stream);

/* Givens QR that allocates no device memory.  No counterpart in the
 * reference: it exists for callers that cannot allocate (a stream capture
 * that forbids allocations, allocator hooks, fixed memory budgets).  Same
 * results as oapb_qr_givens; the workspace is a static 512 KiB device array
 * of the library, so n <= 128 (OAPB_ERR_ARG beyond).  The first call in a
 * context loads the array's module and should precede any stream capture;
 * calls that overlap on the GPU share the array and race. */
OAPB_EXPORT int oapb_qr_givens_noalloc(const oapb_mat* Q, const oapb_mat* R,
                                       const oapb_mat* A, void* stream);

/* Householder QR of a real square matrix (CuProceduresApi.h:306,
 * CuQRProcedures_HT.h:63-131). */
OAPB_EXPORT int oapb_qr_householder(const oapb_mat* Q, const oapb_mat* R, const oapb_mat* A,
                        void* stream);

/* 1 if every first-subdiagonal entry is within (-tolerance, tolerance) in each
 * present plane (CuProceduresApi.h:308, CuIsUpperTriangularProcedures.h:29-89;
 * the reference's fixed tolerance is 1e-3). */
OAPB_EXPORT int oapb_is_upper_triangular(int* output, const oapb_mat* matrix,
                             double tolerance, void* stream);

/* Unshifted QR iteration H <- R Q until oapb_is_upper_triangular(H, 1e-3) or
 * max_iterations, Q accumulating the rotations, entirely on the device
 * (CuProceduresApi.h:310-312, oapGenericArnoldiApi.h:268-296).  *iterations
 * (host, may be NULL) receives the count. */
OAPB_EXPORT int oapb_calc_triangular_h(const oapb_mat* H, const oapb_mat* Q,
                           uint32_t max_iterations, uint32_t* iterations,
                           void* stream);

/* Self-test of the bounded device-side wait used by every tensor-core kernel
 * (no counterpart in the reference, whose host aborts on CUDA errors,
 * oapCuda/KernelExecutor.h:34-41).  One CTA waits on a shared-memory
 * mbarrier for at most limit_us microseconds (1 .. 1000000); with arrive = 0
 * nothing arrives, the wait runs out, the kernel returns and the call
 * returns OAPB_ERR_TIMEOUT with *timed_out = 1; with arrive = 1 the wait
 * completes (OAPB_OK, *timed_out = 0).  The context stays usable either
 * way.  Synchronises `stream`; allocates nothing. */
OAPB_EXPORT int oapb_selftest_bounded_wait(uint32_t limit_us, int32_t arrive, int32_t* timed_out,
                                           void* stream);

/* ------------------------------------------------------------------------ */
/* Solver: CuHArnoldi / CuHArnoldiCallback (ArnoldiPackage)                  */
/* ------------------------------------------------------------------------ */

/* Wanted-set ordering, ArnUtils::Sort* (ArnoldiPackage/ArnoldiUtils.cpp:24-50). */
typedef enum oapb_sort {
  OAPB_SORT_LARGEST_VALUES = 0,     /* |lambda| descending (LM) */
  OAPB_SORT_LARGEST_RE = 1,
  OAPB_SORT_LARGEST_IM = 2,
  OAPB_SORT_SMALLEST_VALUES = 3,
  OAPB_SORT_SMALLEST_RE = 4,
  OAPB_SORT_SMALLEST_IM = 5
} oapb_sort;

/* Arithmetic of the solve. */
typedef enum oapb_precision {
  /* FP64 everywhere: the plain GPU Arnoldi. */
  OAPB_PREC_FP64 = 0,
  /* The chosen form (dense operators, n >= 8192; from 2048 to 8192 the
   * FP64 restart loop runs, below that - with hdim <= 32 and a random start -
   * the FP64 restart loop of one problem on one CTA, no launch per step):
   * block subspace iteration on an FP32-class copy of
   * the operator (split-BF16 tensor-core passes, or FP32 CUDA-core passes
   * with tensor_cores = 0), then FP64-anchored refinement (FP64 residual
   * passes, FP32-class Sylvester corrections) until the residual goal holds
   * against the FP64 operator; FP64 subspace iteration, FP32 IRAM and the
   * plain FP64 IRAM as fall-backs. */
  OAPB_PREC_MIXED = 1
} oapb_precision;

/* Start vector, oap::InitVVectorType (oapGenericArnoldiApi.h:38-42). */
typedef enum oapb_init {
  OAPB_INIT_RANDOM = 0,            /* seeded U[-1, 1] (reference: unseeded) */
  OAPB_INIT_FIRST_VALUE_IS_ONE = 1,
  OAPB_INIT_USER = 2               /* oapb_arnoldi_set_start_vector */
} oapb_init;

/* oap::VecMultiplicationType (oapGenericArnoldiApi.h:32-36). */
typedef enum oapb_vec_mult { OAPB_TYPE_EIGENVECTOR = 0, OAPB_TYPE_WV = 1 } oapb_vec_mult;

typedef struct oapb_arnoldi_config {
  uint32_t n;              /* operator dimension (MatrixInfo rows) */
  uint32_t hdim;           /* Krylov dimension m (CuHArnoldi::execute hdim) */
  uint32_t wanted;         /* k wanted eigenpairs */
  int32_t is_complex;      /* operator / basis complex (MatrixInfo isIm) */
  int32_t sort;            /* oapb_sort */
  int32_t precision;       /* oapb_precision */
  int32_t init;            /* oapb_init */
  uint32_t max_restarts;   /* restart budget (reference: CHECK_* rules) */
  double tolerance;        /* ||A x - l x|| / (|l_1| ||x||) goal, e.g. 1e-10 */
  double rho;              /* DGKS threshold (CuHArnoldi::setRho, default 1/3.14) */
  uint64_t seed;           /* start-vector seed for OAPB_INIT_RANDOM */
  int32_t profile;         /* 1: time every dense matvec with CUDA events
                              (oapb_arnoldi_stats.matvec_seconds) */
  int32_t fallback_random; /* 1: when a solve from a user start vector does
                              not reach the goal within max_restarts, solve
                              again from the seeded random start */
  int32_t tensor_cores;    /* 1 (default): block operator passes on the
                              tensor cores (FP32-class passes as split BF16
                              tcgen05, FP64 passes as DMMA); 0: CUDA cores */
  int32_t refine;          /* mixed form, complex LM problems: 1 (default)
                              refines the FP32-phase subspace by FP64
                              residual + FP32-class Sylvester corrections;
                              0 runs FP64 subspace iteration instead */
  int32_t autotune;        /* 1 (default): when a dense operator is set, time
                              the launch variants of the single-vector
                              operator pass and keep the fastest (cached per
                              device, n, type); 0: the default variant;
                              2 + v: variant v (0..5, diagnostics) */
} oapb_arnoldi_config;

/* Fill defaults: rho = 1/3.14, tolerance = 1e-10, LM, FP64, random start,
 * max_restarts = 300, tensor_cores = 1. */
OAPB_EXPORT void oapb_arnoldi_config_default(oapb_arnoldi_config* cfg);

typedef struct oapb_arnoldi_stats {
  uint32_t restarts;         /* implicit restarts performed */
  uint32_t matvecs;          /* single-vector operator applications */
  uint32_t block_matvecs;    /* block (multi-vector) FP64 operator passes */
  uint32_t dgks_passes;      /* reorthogonalisation passes taken */
  uint32_t refine_iterations;
  int32_t converged;
  double max_residual;       /* largest relative residual of the wanted pairs */
  double seconds;            /* host wall time of the last solve */
  double matvec_seconds;     /* device time of the timed dense matvecs (profile) */
  uint32_t matvec_timed;     /* number of dense matvec launches timed */
  uint32_t matvec_fp32;      /* of which on the FP32 operator copy */
  uint64_t kernel_launches;  /* library kernel launches over the handle's life */
  double block_seconds;      /* device time of the timed FP64 block matvecs (profile) */
  uint32_t block_timed;
  uint32_t block_fp32_timed; /* FP32-class block matvecs timed (profile; BF16 passes apart) */
  double block_fp32_seconds;
  uint32_t block_fp32_width; /* right-hand sides of the FP32 block matvec */
  uint32_t fallbacks;        /* solves restarted from the random start */
  uint32_t matvec_variant;   /* launch variant of the FP64 operator pass */
  uint32_t block_bf16;       /* block passes on the BF16 hi planes alone */
  uint32_t block_bf16_timed; /* of which timed (profile) */
  double block_bf16_seconds; /* their device time (profile) */
  uint32_t eig_fast;         /* FP64 Rayleigh-Ritz eigensolves of the refinement
                                delivered by inverse iteration on the nearly
                                triangular projected matrix (the rest: Schur) */
  uint32_t block_i8;         /* FP64-class block passes on the integer tensor
                                cores (int8 slices of the mixed form's operator) */
  uint32_t onchip;           /* 1: the last solve ran on one CTA (the chosen
                                form for dense operators with n <= 2048 and
                                hdim <= 32, random start) */
  /* device time of the tensor-core pass kernels alone (profile), between
   * events recorded right before and after each launch: [0] FP64-class
   * (int8-slice) pass, [1] split-BF16 pass, [2] BF16 hi-plane pass; the
   * block_*_seconds fields above also cover the vector split and the
   * stream-K reduction around each pass */
  double pass_kernel_seconds[3];
  uint32_t pass_kernel_timed[3];
  uint32_t symtri;           /* restart-loop eigensolves of the last plain solve
                                that took the Hermitian tridiagonal path
                                (Hermitian or real symmetric operators) */
} oapb_arnoldi_stats;

typedef struct oapb_arnoldi oapb_arnoldi;   /* opaque solver handle */

/* User operator, CuHArnoldiCallbackBase::MultiplyFunc
 * (ArnoldiProceduresImpl.h:51-56): w = A v.  v and w are n-row, 1-column FP64
 * device vectors, valid only during the call.  Return 0 on success. */
typedef int (*oapb_matvec_fn)(const oapb_mat* w, const oapb_mat* v, void* user,
                              int vec_mult_type, void* stream);

OAPB_EXPORT int oapb_arnoldi_create(oapb_arnoldi** handle, const oapb_arnoldi_config* cfg,
                        void* stream);
OAPB_EXPORT int oapb_arnoldi_destroy(oapb_arnoldi* handle);

/* Dense operator A (n x n, FP64 device planes, reference layout); im must be
 * NULL iff cfg.is_complex == 0.  With OAPB_PREC_MIXED the solver keeps an
 * FP32 copy (library-owned). */
OAPB_EXPORT int oapb_arnoldi_set_dense_operator(oapb_arnoldi* handle, const oapb_mat* A);

/* User callback operator (CuHArnoldiCallback::setCallback).  Runs FP64. */
OAPB_EXPORT int oapb_arnoldi_set_callback(oapb_arnoldi* handle, oapb_matvec_fn fn,
                              void* user);

/* Implicit Gram operator A = X X^T for FP32 images X (rows = n samples x
 * cols pixels, row-major, device; 16-byte aligned when cols % 4 == 0):
 * every operator application runs w = X (X^T v) in two HBM-bound passes
 * over X, FP64 accumulation, without forming A (the reference application
 * rebuilds the Gram on every multiplication, oap2dt3dDevice/
 * MainAPExecutor.cpp:42-127, SquareMatrixApi.cpp:143-181).  Real solves
 * only; runs the FP64 path.  X must stay valid during solves. */
OAPB_EXPORT int oapb_arnoldi_set_gram_operator(oapb_arnoldi* handle, const float* X, uint32_t rows,
                                               uint32_t cols);

/* The implicit Gram operator with X (rows = n samples x cols pixels, FP32,
 * row-major) in HOST memory, for image sets larger than HBM, as the
 * reference's application reads its images block by block
 * (oap2dt3dDevice/MainAPExecutor.cpp:59-100, oapMatrixCuda/RecToSquareApi.cpp:
 * 71-141): A v = sum_c X_c (X_c^T v) over column blocks X_c of block_cols
 * pixels (rounded up to a multiple of 4), so one application reads X once.
 * The first blocks that fit resident_bytes are copied to the device here and
 * stay; the others are copied host-to-device on every application through
 * two device buffers, the copy of the next block (on a second stream)
 * overlapping the passes over the current one; pinned host memory gives the
 * full copy rate.  X must stay valid while the operator is set.  Real solves,
 * FP64 path, like oapb_arnoldi_set_gram_operator. */
OAPB_EXPORT int oapb_arnoldi_set_gram_operator_host(oapb_arnoldi* handle, const float* X, uint32_t rows,
                                                    uint32_t cols, uint32_t block_cols,
                                                    uint64_t resident_bytes);
/* Column blocks of the host-X Gram operator, how many stay resident, and the
 * host-to-device bytes its applications streamed so far (outputs may be
 * NULL; OAPB_ERR_ARG when no such operator is set). */
OAPB_EXPORT int oapb_arnoldi_gram_stream_info(const oapb_arnoldi* handle, uint32_t* blocks,
                                              uint32_t* resident_blocks, uint64_t* streamed_bytes);

/* Start vector (device planes, n values each; im ignored for real solves). */
OAPB_EXPORT int oapb_arnoldi_set_start_vector(oapb_arnoldi* handle, const double* re,
                                  const double* im);

/* Shift filter for the user start vector: before the first Arnoldi step
 * the start vector becomes prod_i (A - shifts[i] I) v0 (host array, up to
 * 64 shifts; count 0 clears).  With shifts near the unwanted eigenvalues
 * closest to the wanted set this damps exactly the directions a restart
 * would damp (the learned shift set of a warm start). */
OAPB_EXPORT int oapb_arnoldi_set_start_shifts(oapb_arnoldi* handle,
                                              const double* shifts,
                                              uint32_t count);

/* Solve (CuHArnoldi::execute, ArnoldiProcedures.cpp:129-140).
 * Host outputs (each may be NULL): eigenvalues re / im (wanted values in
 * sort order), relative residuals.  Device output (may be NULL): eigenvectors,
 * an n x wanted matrix in the reference layout (column q = eigenvector q),
 * unit 2-norm.  Returns OAPB_OK or OAPB_NOT_CONVERGED (outputs still hold
 * the best pairs). */
OAPB_EXPORT int oapb_arnoldi_solve(oapb_arnoldi* handle, double* eig_re, double* eig_im,
                       double* residuals, const oapb_mat* eigenvectors);

/* Same as a dense solve, but the operator comes from HOST memory (FP64 planes
 * in the reference layout); the copy to the device is part of the call. */
OAPB_EXPORT int oapb_arnoldi_solve_host(oapb_arnoldi* handle, const double* a_re,
                            const double* a_im, double* eig_re, double* eig_im,
                            double* residuals, double* eigvec_re,
                            double* eigvec_im);

OAPB_EXPORT int oapb_arnoldi_get_stats(const oapb_arnoldi* handle, oapb_arnoldi_stats* out);

/* Switch the per-launch CUDA-event timing of the operator passes (config
 * field profile) on or off for the following solves; the device-side
 * counterpart of the reference's host clock macros (oapUtils/oapClock.h:74-78). */
OAPB_EXPORT int oapb_arnoldi_set_profile(oapb_arnoldi* handle, int32_t on);

/* One convergence check of the mixed form's block phases. */
typedef struct oapb_trace_rec {
  int32_t phase;        /* 1: FP32-class subspace iteration, 2: FP64 subspace
                           iteration, 3: FP64-anchored refinement */
  int32_t iteration;    /* iteration (outer step) of that phase */
  uint32_t passes;      /* block operator passes of the solve so far */
  uint32_t bf16_passes; /* of which on the BF16 hi planes alone */
  double residual;      /* largest relative residual of the wanted pairs */
} oapb_trace_rec;

/* Convergence trace of the last solve: copies up to cap records, *count =
 * the number recorded (the plain IRAM path records none).  The data behind
 * the reference's per-step logInfo printouts
 * (ArnoldiPackage/ArnoldiProcedures.cpp:391-395, 539). */
OAPB_EXPORT int oapb_arnoldi_get_trace(const oapb_arnoldi* handle, oapb_trace_rec* out, uint32_t cap,
                                       uint32_t* count);

/* Pass precision of oapb_arnoldi_apply_block only (not a solve precision):
 * the BF16 hi planes of the mixed form's operator copy on the tensor cores
 * (products within about 2^-8 |A| |X|; FP32 CUDA-core pass when
 * cfg.tensor_cores = 0). */
#define OAPB_PASS_BF16 2
/* Pass precision of oapb_arnoldi_apply_block only: the BF16 hi planes with X
 * rounded to BF16 as well (the coarse pass of the mixed form's leading
 * powers and early sweeps; products within about 2^-7 |A| |X|). */
#define OAPB_PASS_BF16_COARSE 3

/* W = A X for b <= 32 vectors (device FP64 planes, vector q at offset q n)
 * with the handle's dense operator: precision OAPB_PREC_FP64 reads the FP64
 * operator (on a mixed-form handle with cfg.tensor_cores, cfg.tolerance
 * >= 1e-12 and b <= 16 complex / 32 real vectors: its int8 slices on the
 * integer tensor cores, within 2^-42 of each row's maximum times |x|_1); OAPB_PREC_MIXED the
 * FP32-class copy of the mixed form (tensor cores when cfg.tensor_cores,
 * else CUDA-core FP32); OAPB_PASS_BF16 its BF16 hi planes;
 * OAPB_PASS_BF16_COARSE those with X rounded to BF16 too.  The block pass
 * of the solver, exposed for multiple right-hand sides and for
 * verification. */
OAPB_EXPORT int oapb_arnoldi_apply_block(oapb_arnoldi* handle, const double* x_re,
                                         const double* x_im, uint32_t b,
                                         double* w_re, double* w_im,
                                         int32_t precision);

/* Relative residual ||A x - lambda x|| / (|lambda_1| ||x||) of pair `index`
 * of the last solve (CuHArnoldi::testOutcome, ArnoldiProcedures.cpp:521-542,
 * 642-649), recomputed in FP64 on the device. */
OAPB_EXPORT int oapb_arnoldi_test_outcome(oapb_arnoldi* handle, uint32_t index, double* out);

/* Checkpoint of the plain FP64 restart loop: the complete m-step Arnoldi
 * factorization A V = V H + f e_m^T left on the device by the last solve
 * that ran the plain path (OAPB_PREC_FP64, or the mixed form's last
 * fall-back), written as one file in the reference's matrix format (the
 * utils::ByteBuffer of oap::host::SaveMatrix, oapMatrixCpu/oapHostMatrixUtils.cpp:
 * 1054-1113): a header (1 x 8: format 1, n, m, k, complex, restarts,
 * matvecs, sort), V (m columns x n rows), H (m x m) and f (1 x n).  This
 * fills the save / load / stop contract that CuHArnoldiCallbackThread
 * declares and leaves empty (ArnoldiPackage/ArnoldiProceduresImpl.cpp:59-69).
 * save: OAPB_ERR_ARG when the handle holds no such factorization.
 * load: into a handle created with the same n, hdim, wanted and is_complex
 * (OAPB_ERR_ARG otherwise). */
OAPB_EXPORT int oapb_arnoldi_save(oapb_arnoldi* handle, const char* path);
OAPB_EXPORT int oapb_arnoldi_load(oapb_arnoldi* handle, const char* path);

/* Continue the restart loop from the loaded (or last) factorization with a
 * fresh restart budget, then finish like oapb_arnoldi_solve (same outputs;
 * the operator must be set).  Interrupting a solve (max_restarts), saving,
 * loading into a new handle and resuming gives the result of the
 * uninterrupted solve. */
OAPB_EXPORT int oapb_arnoldi_resume(oapb_arnoldi* handle, double* eig_re, double* eig_im,
                                    double* residuals, const oapb_mat* eigenvectors);

/* ------------------------------------------------------------------------ */
/* Matrix files in the reference's format (oap::host::WriteMatrix /           */
/* ReadMatrix, oapMatrixCpu/oapHostMatrixUtils.cpp:974-988, 1054-1113)       */
/* ------------------------------------------------------------------------ */

/* Write device FP64 planes (im may be NULL) as one matrix file. */
OAPB_EXPORT int oapb_mat_write(const char* path, const oapb_mat* m, void* stream);
/* Dimensions and planes of the first matrix of a file (outputs may be NULL). */
OAPB_EXPORT int oapb_mat_read_info(const char* path, uint32_t* columns, uint32_t* rows,
                                   int32_t* has_re, int32_t* has_im);
/* Read the first matrix of a file into device FP64 planes of the same
 * dimensions (a plane absent from the file is zeroed; an imaginary plane
 * in the file needs dst->im). */
OAPB_EXPORT int oapb_mat_read(const char* path, const oapb_mat* dst, void* stream);

/* ------------------------------------------------------------------------ */
/* Gram operator build                                                      */
/* ------------------------------------------------------------------------ */

/* A = X X^T for X (rows x cols, FP32, row-major: rows = samples, cols =
 * pixels), replacing SquareMatrixApi::getDeviceMatrix's dotProduct(out, X,
 * X^T) (oapMatrixCuda/SquareMatrixApi.cpp:143-156, RecToSquareApi.cpp:57-69).
 * Split-BF16 on the tensor cores (tcgen05): x = hi + lo, A = hi hi^T +
 * hi lo^T + lo hi^T accumulated in FP32.  A: device rows x rows FP32; A64:
 * optional device FP64 copy (NULL to skip).  Synchronises `stream`. */
OAPB_EXPORT int oapb_gram_build(const float* X, uint32_t rows, uint32_t cols,
                                float* A, double* A64, void* stream);
/* The build's workspace (BF16 hi / lo planes of X, 4 bytes per element of X,
 * plus the tile partials) comes from a library-owned stream-ordered pool
 * that keeps the memory for the next build; this returns it to the driver
 * (current device; no counterpart in the reference). */
OAPB_EXPORT int oapb_gram_trim(void);

/* Image ingestion: `count` decoded RGB8 images of `pixels` pixels each
 * (rgb: count x pixels x 3 bytes, on the host when rgb_on_host, else on the
 * device) -> X (device FP32, count x pixels, row-major), each pixel
 * (r << 16 | g << 8 | b) / 0xFFFFFF as the reference's
 * Image::convertRgbToFloatt (oapAppUtils/Image.cpp:155-180); X is the
 * reference's DataLoader matrix (image i = column i,
 * oapAppUtils/DataLoader.cpp:47-66) transposed, the layout of
 * oapb_gram_build and oapb_arnoldi_set_gram_operator.  Synchronises
 * `stream`. */
OAPB_EXPORT int oapb_images_to_matrix(const uint8_t* rgb, int32_t rgb_on_host, uint32_t count,
                                      uint32_t pixels, float* X, void* stream);

/* ------------------------------------------------------------------------ */
/* Batched solver: many independent small problems in one persistent launch */
/* ------------------------------------------------------------------------ */

/* One problem of a batch (device planes in the reference layout). */
typedef struct oapb_batch_problem {
  uint32_t n;            /* 2 <= n <= 2048, n > wanted */
  const double* re;      /* device, n x n */
  const double* im;      /* device, or NULL for a real problem */
  double* eigvec_re;     /* device, n x wanted (column q = eigenvector q), or NULL */
  double* eigvec_im;     /* device, or NULL */
} oapb_batch_problem;

typedef struct oapb_batch_stats {
  uint32_t problems;
  uint32_t converged;
  uint64_t matvecs;      /* over all problems, including the residual checks */
  uint64_t restarts;
  uint32_t ctas;         /* resident CTAs of the persistent launch */
  double seconds;        /* host wall time of the call */
  uint32_t variant;      /* launch variant (cfg.autotune: 1 tunes, 2 + v forces v) */
  uint32_t threads;      /* threads per CTA of that variant */
  uint64_t operator_bytes; /* operator bytes read by all matvecs (8 n^2 real,
                              16 n^2 complex each): the launch's algorithmic
                              HBM traffic */
} oapb_batch_stats;

/* Solve `count` independent eigenproblems (IEigenCalculator::calculate,
 * oap2dt3dDevice/IEigenCalculator.cpp:56-70, called once per problem in the
 * reference) with one persistent kernel: each CTA takes the next problem
 * from a queue ordered by decreasing n and runs the full restart loop on the
 * device.  cfg: hdim caps the Krylov dimension (m_i = min(n_i, hdim),
 * hdim <= 32), wanted, sort, tolerance, max_restarts, rho, seed, autotune
 * (0: the default launch variant, 256 threads per CTA; 1: the variant
 * (threads per CTA x CTAs per SM the registers are budgeted for: 256 x 1,
 * 128 x 2, 256 x 2, 128 x 4, 64 x 8) that ran fastest on a sample of the
 * first batch of a given largest n, hdim, wanted and complexity, cached per
 * device; 2 + v: variant v, 0..4); n, is_complex, precision and init are
 * ignored (complex iff im != NULL, FP64, seeded random start).  `problems` is a HOST array.  Host outputs:
 * eig_re / eig_im / residuals (count x wanted, row i = problem i in sort
 * order), status (count, oapb_status per problem).  Synchronises `stream`.
 * Returns OAPB_OK when every problem converged, OAPB_NOT_CONVERGED when some
 * did not (see status), or an error. */
OAPB_EXPORT int oapb_arnoldi_solve_batched(const oapb_arnoldi_config* cfg,
                                           const oapb_batch_problem* problems,
                                           uint32_t count, double* eig_re,
                                           double* eig_im, double* residuals,
                                           int32_t* status,
                                           oapb_batch_stats* stats, void* stream);

/* ------------------------------------------------------------------------ */
/* Learned warm start: parametric operators and the BF16 network            */
/* ------------------------------------------------------------------------ */

/* out[p] = A0 + sum_i theta[p * nparams + i] B[i] for p < count (all device
 * FP64, n x n; B is a HOST array of nparams device pointers, nparams <= 32). */
OAPB_EXPORT int oapb_param_operators(const double* A0, const double* const* B,
                                     uint32_t nparams, const double* theta,
                                     uint32_t count, uint32_t n, double* out,
                                     void* stream);

/* Dense network sizes[0] -> ... -> sizes[nlayers]; by default tanh hidden
 * layers and a linear output (oapb_mlp_set_activations chooses per layer);
 * BF16 weights / activations, FP32 accumulation, FP32 master weights with
 * Adam.  Nearest reference analogue: oapNeuralDevice/oapNetwork.h:27-124
 * and the generic propagation of oapNeuralHost/oapGenericNeuralApi.h:195-360. */
typedef struct oapb_mlp oapb_mlp;

/* Activation of a layer's outputs: the reference's Activation
 * (oapNeuralHost/oapLayerStructure.h:32-38, same order), applied with its
 * derivative as activateFunc / derivativeFunc do
 * (oapNeuralHost/oapGenericNeuralApi.h:43-120). */
typedef enum oapb_activation {
  OAPB_ACT_LINEAR = 0,
  OAPB_ACT_SIGMOID = 1,   /* 1 / (1 + exp(-z)) */
  OAPB_ACT_TANH = 2,
  OAPB_ACT_SIN = 3
} oapb_activation;
OAPB_EXPORT int oapb_mlp_create(oapb_mlp** handle, const uint32_t* sizes,
                                uint32_t nlayers, uint64_t seed);
OAPB_EXPORT int oapb_mlp_destroy(oapb_mlp* handle);
OAPB_EXPORT uint64_t oapb_mlp_num_params(const oapb_mlp* handle);
/* y (device FP32, batch x out) = net(x) (device FP32, batch x in) */
OAPB_EXPORT int oapb_mlp_forward(oapb_mlp* handle, const float* x, uint32_t batch,
                                 float* y, void* stream);
/* Forward + backward of 1/(2 batch) sum (y - target)^2; gradients stay in
 * the handle (packing: all weight matrices [out x in] in layer order, then
 * all biases); *loss (host, may be NULL) receives the loss. */
OAPB_EXPORT int oapb_mlp_backward(oapb_mlp* handle, const float* x,
                                  const float* target, uint32_t batch,
                                  double* loss, void* stream);
OAPB_EXPORT int oapb_mlp_adam_step(oapb_mlp* handle, float lr, void* stream);
/* which 0: parameters, 1: gradients -> dst (host or device FP32) */
OAPB_EXPORT int oapb_mlp_copy(oapb_mlp* handle, int which, float* dst, void* stream);
OAPB_EXPORT int oapb_mlp_set_params(oapb_mlp* handle, const float* src, void* stream);
/* Activations of the nlayers layers' outputs (acts[l] for layer l, count ==
 * nlayers; the Layer activation of Network::createLayer,
 * oapNeuralDevice/oapNetwork.h:53-54); OAPB_ERR_ARG for another count or an
 * unknown value. */
OAPB_EXPORT int oapb_mlp_set_activations(oapb_mlp* handle, const int32_t* acts, uint32_t count);
OAPB_EXPORT int oapb_mlp_get_activations(const oapb_mlp* handle, int32_t* acts, uint32_t count);
/* Layer count; sizes (may be NULL) receives the nlayers + 1 sizes. */
OAPB_EXPORT uint32_t oapb_mlp_num_layers(const oapb_mlp* handle, uint32_t* sizes);
/* Network::save / Network::load (oapNeuralDevice/oapNetwork.h:109-111) in
 * the reference's matrix file format: the sizes (1 x nlayers+1), then per
 * layer its weights (in columns x out rows) and biases (1 x out), then the
 * activations (1 x nlayers; absent: the defaults).  load
 * creates a new handle (Adam state fresh; `seed` only fills it before the
 * weights are set). */
OAPB_EXPORT int oapb_mlp_save(oapb_mlp* handle, const char* path);
OAPB_EXPORT int oapb_mlp_load(oapb_mlp** handle, const char* path, uint64_t seed);

#ifdef __cplusplus
}
#endif

#endif /* OAPB200_H */
