// Launchers of the device kernels of libttcuda (all FP64 unless stated).
#pragma once
#include "common.cuh"

namespace ttc {

// ---- grouped FP64 GEMM (gemm_f64.cu)
void launch_gemm_f64(const GemmDesc* d_descs, int nd, long long total_tiles, cudaStream_t s);
// ---- the same problems with float data in A, B and C, FP32 accumulation (gemm_f32.cu)
void launch_gemm_f32(const GemmDesc* d_descs, int nd, long long total_tiles, cudaStream_t s);
long long gemm_tiles(const GemmDesc& d);
// Split-K count for one FP64 problem of a launch of launch_tiles output tiles on nsm SMs (1: no
// split), and the partial-tile workspace (doubles) a split problem needs.
int gemm_pick_ksplit(const GemmDesc& d, long long launch_tiles, int nsm);
long long gemm_split_ws_doubles(const GemmDesc& d);

// Device-side size bound: min(cap, mult * *p) when p is given (a rank that an earlier kernel of
// the same plan wrote), else cap.  Rows or columns beyond the bound are exactly zero in the
// operand, so the kernels leave them out.
__device__ __forceinline__ int dev_bound(int cap, const int* p, int mult) {
  return p ? min(cap, max(0, mult * *p)) : cap;
}

// ---- batched Householder QR (qr_householder.cu)
// A (m x n, col-major, lda) is overwritten.  Q (m x K, ldq) and R (K x n, ldr),
// K = min(m, n), like LAPACK geqrf + orgqr (Julia `qr`, `Matrix(F.Q)`, `F.R`).
// Q == nullptr skips the Q formation, R == nullptr skips R.
struct QRDesc {
  int m, n;
  double* A; int lda;
  double* Q; int ldq;
  double* R; int ldr;
  double* Tws;      // >= ceil(K/16)*16*16 doubles of workspace for the block reflectors
  int r_trans;      // 1: R is written transposed, R^T[j][i] at R[i*ldr + j]
  // optional device bounds: rows >= m_mult * *m_dev and columns >= n_mult * *n_dev of A are
  // zero; the factorization runs on the bounded block (Q and R keep their full shapes)
  const int* m_dev; int m_mult;
  const int* n_dev; int n_mult;
  double* Rt; int ldrt;   // optional second copy of R, transposed: R^T[j][i] at Rt[i*ldrt + j]
};
constexpr int QR_MAX_M = 1536;
void launch_qr(const QRDesc* d_descs, int count, int max_m, cudaStream_t s, int* d_flags);

// B <- Q B with Q = H_1 ... H_K the Householder factor a QR launch left in A (reflectors below
// the diagonal, T factors in Tws): B is m x nb (ld ldb); columns >= *n_dev (when given) are
// zero and stay zero, so they are not touched.
struct QApplyDesc {
  int m, K;
  const double* A; int lda;
  const double* Tws;
  double* B; int ldb; int nb;
  const int* n_dev;
  const int* m_dev; int m_mult;   // the row bound the QR launch was given (Q acts on those rows)
};
void launch_qr_apply(const QApplyDesc* d_descs, int count, int max_m, cudaStream_t s);

// ---- batched one-sided Jacobi SVD (svd_jacobi.cu)
// X (m x n, col-major, ldx, m >= n) is overwritten by X*W whose columns are
// orthogonal; W (n x n, ldw) accumulates the rotations when not null.
// sigma[i] = ||column i||; perm lists columns by decreasing sigma.
struct JacobiDesc {
  int m, n;
  double* X; int ldx;
  double* W; int ldw;
  double* sigma;    // n
  int* perm;        // n
  int* info;        // optional: sweeps used (negative if the sweep cap was hit)
  const int* m_dev; int m_mult;   // optional: rows >= m_mult * *m_dev of X are zero
};
// `order` (count ints of device workspace, or nullptr): the launch first ranks the problems by
// their size (rows after the device bound x columns^2, largest first) so that the clusters,
// which the hardware starts in index order, take the longest problems first.
constexpr int kJacobiOrderMax = 4096;
// max_sweeps: sweep cap; a problem still rotating after it sets DFLAG_JACOBI_NOCONV.
constexpr int kJacobiDefaultSweeps = 40;
void launch_jacobi(const JacobiDesc* d_descs, int count, int max_m, int max_n, bool accw, cudaStream_t s,
                   int* d_flags, int* order = nullptr, int max_sweeps = kJacobiDefaultSweeps);

// ---- truncation rule (tt_kernels.cu): floor(s, tol) then min(k, rmax, #(s>0))
struct TruncDesc {
  const double* sigma;  // unsorted singular values
  const int* perm;      // order by decreasing sigma
  int n;                // number of singular values
  int* rank_out;        // where k is written (device rank array slot)
};
void launch_truncate(const TruncDesc* d, int count, double tol, long long rmax, cudaStream_t s);

// Build Ut (rows x cols, ld) with Ut[:, i] = X[:, perm[i]] / sigma[perm[i]] for i < k and
// 0 for i >= k (k read from *rank); with `unit_w` the columns are taken from W unscaled.
struct SelectDesc {
  const double* X; int ldx;  // source columns
  const double* sigma; const int* perm; const int* rank;
  int rows, cols;            // output rows and column capacity
  int src_cols;              // columns of X (perm entries are < src_cols)
  double* U; int ldu;
  int scale;                 // 1: divide by sigma; 0: copy; 2: multiply by sigma
  int zrows;                 // when above rows: rows [rows, zrows) of every output column are zeroed
};
void launch_select(const SelectDesc* d, int count, int max_rows, int max_cols, cudaStream_t s);

// ---- general strided copy / permute of up to 4-D tensors (tt_kernels.cu)
// dst[i0*ds0 + i1*ds1 + i2*ds2 + i3*ds3] = alpha * src[i0*ss0 + ...] for i < ext.
struct CopyDesc {
  const double* src; double* dst;
  long long ext[4];
  long long ss[4];
  long long ds[4];
  double alpha;
};
void launch_copy(const CopyDesc* d, int count, long long max_elems, cudaStream_t s);

// Zero a set of flat ranges.
struct ZeroDesc { double* p; long long n; };
void launch_zero(const ZeroDesc* d, int count, long long max_n, cudaStream_t s);

// Sum of squares of `n` doubles per problem, written to out[i] (FP64, deterministic order).
struct NormDesc { const double* p; long long n; double* out; };
void launch_sumsq(const NormDesc* d, int count, cudaStream_t s);

// ---- MPO x TT apply (tt_kernels.cu), src/tt_operations.jl:170-194, internal layouts.
struct ApplyDesc {
  const double* H;   // internal MPO core (R, n_out, n_in, R')  col-major
  const double* V;   // internal TT core  (r, n_in, r')         col-major
  double* Y;         // internal TT core  ((R r), n_out, (R' r')) col-major, R index fastest
  int R, Rn, r, rn, n;
};
// one CTA per right rank index nu' of each problem: grid (max rn, count).  Staged in shared memory:
// V[:, :, nu'] and, one a' at a time, H[:, :, :, a'].
__host__ __device__ inline long long apply_smem_doubles(const ApplyDesc& d) {
  return (long long)d.n * d.r + (long long)d.n * d.n * d.R;
}
void launch_apply(const ApplyDesc* d, int count, int max_rn, int max_smem_doubles, cudaStream_t s);

// ---- Philox sketch generation (tt_kernels.cu): Gaussian block entries
// dst (Julia layout of the block, flat index e) = scale * N(0,1)_{seed, stream, e}.
struct PhiloxDesc { double* dst; long long count; unsigned long long seed; unsigned stream; double scale; };
void launch_philox(const PhiloxDesc* d, int count, long long max_count, cudaStream_t s);

// ---- FP64 -> BF16 conversion and the tcgen05 BF16 GEMM (gemm_bf16_tc.cu)
// Operands are BF16, or FP32 read as TF32 in a launch with tf32 = true.
struct Bf16GemmDesc {
  int m, n, k, m0;                // m0: row split (row i = i0 + m0*i1) of the outputs
  const void* A; long long lda;   // operand type, K-major: A(i, kk) at A[i*lda + kk]
  const void* B; long long ldb;   // operand type, K-major: B(j, kk) at B[j*ldb + kk]
  double* C64; float* C32;        // outputs sharing strides: (i0*c_i0 + i1*c_i1 + j0*c_j + j1*c_j1)
  void* C16;                      // output in the operand type (BF16 or FP32), strides (h_i0, h_i1, h_j, h_j1)
  long long c_i0, c_i1, c_j, h_i0, h_i1, h_j;
  double alpha;
  long long tile_start;
  int n0;                         // column split j = j0 + n0*j1 of the outputs (0: no split)
  long long c_j1, h_j1;
};
void launch_gemm_bf16_tc(const Bf16GemmDesc* d, int nd, long long total_tiles, cudaStream_t s, int* d_flags,
                         bool tf32 = false);
long long bf16_gemm_tiles(const Bf16GemmDesc& d);
// Poll limit of the tensor-core GEMM's mbarrier waits on the current device (default 2^24); tests
// set 0 to make the waits give up on purpose.
void set_tc_wait_limit(long long polls);

}  // namespace ttc
