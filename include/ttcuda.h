/*
 * libttcuda -- C ABI of the B200 (sm_100a) tensor-train rounding engine.
 *
 * Every entry point replaces one method of the Julia package TensorTrains
 * (rodrigofj99/Tensor-Train-Julia); the comment above each declaration names the
 * reference method (file:line) whose meaning, argument order and error behaviour
 * it keeps.  Host-side tensors use the reference's memory layout unchanged:
 *   TTvector core k : column-major (n_k, r_{k-1}, r_k)            (src/tt_tools.jl:24-34)
 *   TToperator core : column-major (n_k, n_k, R_{k-1}, R_k)       (src/tt_tools.jl:61-71)
 * so a Julia `ccall` passes `pointer.(x.ttv_vec)` directly, with no host transposes.
 * Ranks, dims and orthogonality flags are int64 like Julia's `Vector{Int64}`.
 *
 * All functions return a ttc_status; on failure ttc_last_error() holds a message.
 * Output tensors are written into caller-allocated buffers whose capacities
 * (rks_cap) the caller states; output ranks never exceed the capacities documented
 * per function, and the written ranks are returned in `rks`.
 */
#ifndef TTCUDA_H
#define TTCUDA_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TTC_OK = 0,
  TTC_EARG = 1,       /* invalid argument        -> Julia ArgumentError            */
  TTC_EDIM = 2,       /* dimension mismatch      -> DimensionMismatch / @assert    */
  TTC_ENOCONV = 3,    /* Jacobi SVD sweep cap    -> LAPACKException retry path      */
  TTC_ENOTPD = 4,     /* Cholesky breakdown (reserved for the CholeskyQR path)     */
  TTC_ECUDA = 5,      /* CUDA runtime error                                         */
  TTC_ENOMEM = 6,     /* device allocation failed                                   */
  TTC_EINTERNAL = 7,
  TTC_ENONFINITE = 8  /* NaN or Inf in an input                                     */
} ttc_status;

enum { TTC_DIR_LEFT = 0, TTC_DIR_RIGHT = 1 };         /* direction=:left / :right      */
enum { TTC_PREC_FP64 = 0, TTC_PREC_BF16 = 1, TTC_PREC_TF32 = 2,   /* sketch-contraction precision */
       TTC_PREC_FP32 = 3 };                                         /* FP32 with FP32 accumulation (gradient) */

typedef struct ttc_context ttc_context;
typedef struct ttc_batch ttc_batch;

/* A TTvector in host memory (read-only input). */
typedef struct {
  int32_t N;
  const int64_t* dims;          /* N     */
  const int64_t* rks;           /* N + 1 */
  const int64_t* ot;            /* N; may be NULL (= all 0) */
  const double* const* cores;   /* N host pointers, core k holds dims[k]*rks[k]*rks[k+1] doubles */
} ttc_ttv;

/* A TTvector result in host memory: the caller allocates core k with room for
 * dims[k]*rks_cap[k]*rks_cap[k+1] doubles; the library writes the actual core
 * (dims[k], rks[k], rks[k+1]) packed column-major at the start of the buffer. */
typedef struct {
  int32_t N;
  const int64_t* rks_cap;       /* N + 1, capacities the caller allocated      */
  int64_t* rks;                 /* N + 1, written                              */
  int64_t* ot;                  /* N, written                                  */
  double* const* cores;         /* N host pointers                             */
} ttc_ttv_out;

/* A TToperator in host memory. */
typedef struct {
  int32_t N;
  const int64_t* dims;          /* N     */
  const int64_t* rks;           /* N + 1 */
  const double* const* cores;   /* N host pointers, (n, n, R_{k-1}, R_k) column-major */
} ttc_tto;

/* Keywords of tt_rounding (src/tt_rounding.jl:146): tol, rmax, direction. */
typedef struct {
  double tol;
  int64_t rmax;
  int32_t direction;            /* TTC_DIR_LEFT or TTC_DIR_RIGHT */
} ttc_round_opts;

/* Keywords of ttrand_rounding / tt_recursive_sketch (src/tt_randtools.jl:112,
 * src/sketches.jl:175): orthogonal, seed, block_rks, plus the arithmetic of the
 * sketch contractions.  sketch_blocks, when not NULL, supplies the N raw sketch
 * blocks (b_{k+1}, n_k, b_k, p_k) in Julia layout (already orthogonalised and
 * scaled as generate_sketch_blocks returns them, src/sketches.jl:44-84), so that
 * host and device use identical sketches; when NULL the device draws them with
 * Philox4x32-10 keyed by `seed` (stream = site index). */
typedef struct {
  int32_t orthogonal;
  uint64_t seed;
  int64_t block_rks;            /* <= 0 means N (the reference default)  */
  int32_t precision;            /* TTC_PREC_FP64, _BF16 or _TF32 (FP32 operands read as TF32 by the tensor cores) */
  const double* const* sketch_blocks;
} ttc_sketch_opts;

/* Kernel families reported by the per-kernel profile (ttc_set_profiling). */
enum {
  TTC_KERN_GEMM_F64 = 0,   /* grouped FP64 GEMM (contractions)              */
  TTC_KERN_QR = 1,         /* batched Householder QR                        */
  TTC_KERN_JACOBI = 2,     /* batched one-sided Jacobi SVD                  */
  TTC_KERN_GEMM_BF16 = 3,  /* tcgen05 BF16 GEMM (sketch contractions)       */
  TTC_KERN_APPLY = 4,      /* MPO x TT apply                                */
  TTC_KERN_OTHER = 5,      /* copies, truncation rule, sketch generation... */
  TTC_KERN_KINDS = 8
};

/* Per-stage device times of the last call (CUDA events on the context stream), ms.
 * With profiling on, kind_ms / kind_launches hold per-kernel-family device times of the
 * last call, measured with an event pair around every launch (no graph replay). */
typedef struct {
  double total_ms;
  double sketch_ms;
  double orth_ms;     /* QR sweep (deterministic) or orthogonalise-and-project sweep */
  double svd_ms;      /* truncated-SVD sweep */
  double h2d_ms;
  double d2h_ms;
  int64_t kernel_launches;
  double kind_ms[8];
  int64_t kind_launches[8];
  /* algorithmic FLOPs of each kernel family in the last profiled call (fixed conventions:
     GEMM 2mnk; Householder QR 2mn^2-2n^3/3, doubled when Q is formed; one-sided Jacobi SVD
     of an m x n block 4mn^2+8n^3) */
  double kind_flops[8];
  /* one-sided Jacobi SVDs of the last profiled call: problems, total and largest sweep count */
  int64_t jacobi_problems, jacobi_sweeps_sum, jacobi_sweeps_max;
  /* execution plans built since the context was created (a repeated call with the same
   * shapes reuses its plan and replays it as a CUDA graph) */
  int64_t plans_built;
  /* roundings run a second time because the Jacobi SVD hit its sweep cap (TTC_ENOCONV): the
   * synchronous entry points then retry once with four times the cap, as the reference retries a
   * failed gesdd with QR iteration (src/tt_rounding.jl:191-195); counted since the context was
   * created.  The asynchronous entry points report TTC_ENOCONV from ttc_synchronize instead. */
  int64_t svd_retries;
} ttc_stats;

/* Per-kernel-family timing of subsequent calls (0 = off, the default). */
int ttc_set_profiling(ttc_context* ctx, int on);

/* ---- context (no reference counterpart: the reference runs in one Julia process) ---- */
int ttc_create(ttc_context** ctx, int device);
int ttc_destroy(ttc_context* ctx);
int ttc_set_stream(ttc_context* ctx, void* cuda_stream);
const char* ttc_last_error(const ttc_context* ctx);
int ttc_get_stats(const ttc_context* ctx, ttc_stats* out);
int ttc_synchronize(ttc_context* ctx);
/* Library build string, e.g. "libttcuda sm_100a". */
const char* ttc_version(void);

/* ---- device batches of TTvectors (same N and dims; per-TT capacities) ----
 * Replaces the Vector{TTvector} the Krylov callers hold (src/tt_solvers.jl:216-218). */
int ttc_batch_create(ttc_context* ctx, int32_t count, int32_t N, const int64_t* dims,
                     const int64_t* rks_cap /* count*(N+1) */, ttc_batch** out);
int ttc_batch_destroy(ttc_batch* b);
/* TTvector(N, vec, dims, rks, ot) constructor, src/tt_tools.jl:24-34: uploads one TT. */
int ttc_batch_upload(ttc_batch* b, int32_t index, const ttc_ttv* x);
int ttc_batch_download(ttc_batch* b, int32_t index, ttc_ttv_out* y);
/* Page-locked host memory mapped into the device address space (no counterpart in the
 * reference; a Julia caller would pass pinned CUDA.jl host arrays).  TT cores in such memory
 * skip the copy through the library's pinned staging buffer: uploads are DMA copies straight
 * to the device (one per run of cores adjacent in memory), downloads are written by the layout
 * kernel over the host link.  Pageable cores are staged. */
int ttc_host_alloc(size_t bytes, void** out);
int ttc_host_free(void* p);
/* Upload/download all `count` TTs of the batch in one transfer each. */
int ttc_batch_upload_all(ttc_batch* b, const ttc_ttv* xs);
int ttc_batch_download_all(ttc_batch* b, ttc_ttv_out* ys);
int ttc_batch_ranks(ttc_batch* b, int32_t index, int64_t* rks /* N+1 */);
/* Bytes of device memory held by the batch (cores + rank arrays). */
size_t ttc_batch_bytes(const ttc_batch* b);

/* tt_rounding(x; tol, rmax, direction) on every TT of a device batch,
 * src/tt_rounding.jl:146-154 and _tt_rounding :174-269.  `y` must have the same
 * count/N/dims and capacities >= those of x.  Left-orthogonality of x is taken
 * from the ot flags uploaded with it (is_leftorthogonal, src/tt_tools.jl:364-367). */
int ttc_batch_round_det(ttc_context* ctx, ttc_batch* x, const ttc_round_opts* opts, ttc_batch* y);
/* Same, enqueued on the context stream without the final synchronisation (device-resident
 * pipelines and timing); errors raised on the device are reported by ttc_synchronize. */
int ttc_batch_round_det_async(ttc_context* ctx, ttc_batch* x, const ttc_round_opts* opts, ttc_batch* y);

/* ttrand_rounding(y, rks; orthogonal, seed, block_rks) on every TT of a batch,
 * src/tt_randtools.jl:112-154, followed (when opts_after != NULL) by the
 * tt_rounding(.; tol) SVD sweep its callers run (src/tt_randtools.jl:476-480).
 * rks: N+1 target sketch ranks shared by the batch (default_rank_heuristic of the
 * batch, src/tt_randtools.jl:40-50, is computed by the caller). */
int ttc_batch_round_rand(ttc_context* ctx, ttc_batch* x, const int64_t* rks,
                         const ttc_sketch_opts* sk, const ttc_round_opts* opts_after,
                         ttc_batch* y);
int ttc_batch_round_rand_async(ttc_context* ctx, ttc_batch* x, const int64_t* rks,
                               const ttc_sketch_opts* sk, const ttc_round_opts* opts_after,
                               ttc_batch* y);

/* ---- one-shot entry points on host tensors (a Julia ccall binds these) ---- */

/* tt_rounding(x; tol, rmax, direction), src/tt_rounding.jl:146.  Output ranks are at
 * most r_and_d_to_rks(x.rks) (src/tt_rounding.jl:6-24); capacity x.rks suffices. */
int ttc_tt_rounding(ttc_context* ctx, const ttc_ttv* x, const ttc_round_opts* opts, ttc_ttv_out* y);

/* orthogonalize(x; i), src/tt_rounding.jl:65-97 (1-based root i). */
int ttc_orthogonalize(ttc_context* ctx, const ttc_ttv* x, int32_t i, ttc_ttv_out* y);

/* norm(x), src/tt_rounding.jl:107-114. */
int ttc_norm(ttc_context* ctx, const ttc_ttv* x, double* out);

/* tt_recursive_sketch(T, A, rks; orthogonal, reverse=true, seed, block_rks),
 * src/sketches.jl:175-305.  W[k] (k = 0..N) is written column-major
 * (rks_A[k], sketch_rks[k]) into W_out[k]; sketch_rks (N+1) is returned. */
int ttc_recursive_sketch(ttc_context* ctx, const ttc_ttv* A, const int64_t* rks,
                         const ttc_sketch_opts* sk, double* const* W_out, int64_t* sketch_rks);

/* tt_recursive_sketch(T, H, A, rks; ...), src/sketches.jl:317-461: W[k] written as
 * (rks_A[k], rks_H[k], sketch_rks[k]) column-major. */
int ttc_recursive_sketch_op(ttc_context* ctx, const ttc_tto* H, const ttc_ttv* A, const int64_t* rks,
                            const ttc_sketch_opts* sk, double* const* W_out, int64_t* sketch_rks);

/* ttrand_rounding(y, rks; ...), src/tt_randtools.jl:112-154.  Output ranks are
 * min(n*rho_k, sketch_rks[k+1]) (capacity: the sketch ranks). */
int ttc_ttrand_rounding(ttc_context* ctx, const ttc_ttv* x, const int64_t* rks,
                        const ttc_sketch_opts* sk, ttc_ttv_out* y);

/* ttrand_rounding(alpha, ys, rks; ...), src/tt_randtools.jl:223-276. */
int ttc_ttrand_rounding_lincomb(ttc_context* ctx, int32_t m, const double* alpha, const ttc_ttv* ys,
                                const int64_t* rks, const ttc_sketch_opts* sk, ttc_ttv_out* y);

/* ttrand_rounding(alpha, A, ys, rks; ...), src/tt_randtools.jl:285-354:
 * rounding of alpha_1 A ys[0] + sum_{j>0} alpha_j ys[j] without forming A ys[0]. */
int ttc_ttrand_rounding_op(ttc_context* ctx, int32_t m, const double* alpha, const ttc_tto* A,
                           const ttc_ttv* ys, const int64_t* rks, const ttc_sketch_opts* sk,
                           ttc_ttv_out* y);

/* ttrand_rounding(Atto, y, b, rks; ...), src/tt_randtools.jl:169-214: rounding of A y - b. */
int ttc_ttrand_rounding_residual(ttc_context* ctx, const ttc_tto* A, const ttc_ttv* x, const ttc_ttv* b,
                                 const int64_t* rks, const ttc_sketch_opts* sk, ttc_ttv_out* y);

/* ttrand_rounding(y::NTuple{M,TTvector}, rks; orthogonal, seed, block_rks), src/tt_randtools.jl:364-473:
 * randomized rounding of the Hadamard product ys[0] .* ... .* ys[m-1] (m == 1: ttrand_rounding
 * of ys[0]).  The last factor is never multiplied out: its sketch and projection contractions are
 * the structured (Kronecker) ones of src/sketches.jl:1735-1881; the first m-1 are multiplied out
 * on the device.  FP64 sketch only.  Output ranks as ttc_ttrand_rounding. */
int ttc_ttrand_rounding_hadamard(ttc_context* ctx, int32_t m, const ttc_ttv* ys, const int64_t* rks,
                                 const ttc_sketch_opts* sk, ttc_ttv_out* y);

/* stta(alpha, ys, rks; seed_left, seed_right, orthogonal, block_rks), src/tt_randtools.jl:551-641
 * (m == 1, alpha[0] == 1: stta(y, rks; ...)): streaming TT approximation of sum_j alpha_j ys[j]
 * from a forward sketch (block counts oversampled 1.5x, src/sketches.jl:1126-1160) and a reverse
 * one.  rks: N+1 target ranks, boundary ranks 1.  Output rank k is the smaller of the two sketch
 * ranks of bond k; ot = 0. */
int ttc_stta(ttc_context* ctx, int32_t m, const double* alpha, const ttc_ttv* ys, const int64_t* rks,
             uint64_t seed_left, uint64_t seed_right, int32_t orthogonal, int64_t block_rks, ttc_ttv_out* y);

/* *(A::TToperator, v::TTvector), src/tt_operations.jl:170-194.  Output ranks
 * R_k * r_k with the operator index fastest; ot = 0. */
int ttc_mpo_apply(ttc_context* ctx, const ttc_tto* A, const ttc_ttv* x, ttc_ttv_out* y);

/* dot(A, B), src/tt_operations.jl:302-323. */
int ttc_dot(ttc_context* ctx, const ttc_ttv* A, const ttc_ttv* B, double* out);

/* partial_contraction(A, B; reverse), src/sketches.jl:1047-1070: W[k] (r^A_k x r^B_k). */
int ttc_partial_contraction(ttc_context* ctx, const ttc_ttv* A, const ttc_ttv* B, int32_t reverse,
                            double* const* W_out);

/* dot_operator(psi, H, phi) = <psi|H|phi>, src/tt_operations.jl:390-421. */
int ttc_dot_operator(ttc_context* ctx, const ttc_ttv* psi, const ttc_tto* H, const ttc_ttv* phi,
                     double* out);

/* +(x::TTvector, y::TTvector), src/tt_operations.jl:81-112 (direct sum). */
int ttc_tt_add(ttc_context* ctx, const ttc_ttv* x, const ttc_ttv* y, ttc_ttv_out* out);

/* *(a::Number, A::TTvector), src/tt_operations.jl:428-441 (scales the first ot==0 core). */
int ttc_tt_scale(ttc_context* ctx, double a, const ttc_ttv* x, ttc_ttv_out* out);

/* Gradient of R(x) = <x|H|x>/<x|x> with respect to every core (H symmetric).
 * No reference method: it is assembled from the environment contractions of
 * src/als.jl:9-25 and dot_operator.  grads[k] has the layout of core k.
 * ckpt_every > 0 stores only every ckpt_every-th left environment and recomputes
 * the others (memory O(d/ckpt) environments instead of O(d)). */
int ttc_rayleigh_grad(ttc_context* ctx, const ttc_tto* H, const ttc_ttv* x, int32_t ckpt_every,
                      double* value, double* const* grads);
/* The same gradient with every contraction in a chosen precision: TTC_PREC_FP64, or TTC_PREC_FP32
 * (FP32 cores and environments, FP32 accumulation; value and gradient are returned widened to
 * double).  No reference method either. */
int ttc_rayleigh_grad_prec(ttc_context* ctx, const ttc_tto* H, const ttc_ttv* x, int32_t ckpt_every,
                           int32_t precision, double* value, double* const* grads);

/* Householder QR of one m x n matrix in device memory that allocates nothing.
 * No counterpart in the reference (the Julia package calls LAPACK qr on host arrays).  It
 * is for callers that cannot allocate device memory when they need the factorisation, such
 * as code running inside a memory pool or arena that owns the device's memory budget: its
 * scratch (working copy of A, reflector factors, descriptor, status word) is a fixed device
 * array of about 4.1 MiB inside the library, held by every GPU that loads it until exit.
 * A (lda >= m), Q (m x min(m,n), ldq >= m, may be NULL) and R (min(m,n) x n upper
 * triangular, ldr >= min(m,n), may be NULL) are device pointers on the current device; A
 * is not modified.  Limits: m <= 1536, m*n <= 524288, min(m,n) <= 512, else TTC_EDIM and
 * nothing runs; leading dimensions above 2^31 - 1 are refused with TTC_EARG.  Work is queued on `stream` (NULL = default stream) and the call returns
 * without waiting.  `status` (device int32, may be NULL) is zeroed and then receives the
 * kernel flags (2: non-finite value in A).  All calls on a device share the scratch: calls
 * that overlap on the GPU race and must be serialised by the caller.  The first call on a
 * device resolves the scratch address and should come before any stream capture.
 * Errors are reported by ttc_last_error(NULL). */
int ttc_qr_noalloc(int32_t m, int32_t n, const double* A, int64_t lda, double* Q, int64_t ldq, double* R,
                   int64_t ldr, int32_t* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TTCUDA_H */
