// Host runtime of libttcuda: context, device TT batches, execution plans.
//
// A plan is the complete list of kernel launches of one operation (for example the
// whole deterministic rounding of a batch), with every launch's descriptors packed in
// one host blob and uploaded once.  TT ranks that the algorithm fixes on the host
// (orthogonalisation, randomized rounding) give static shapes; ranks decided on the
// device (SVD truncation) are handled by zero padding inside capacity-sized cores, so a
// plan never needs a host round trip and can be replayed, or captured in a CUDA graph.
#pragma once
#include <cuda_runtime.h>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "kernels.cuh"

namespace ttc {
// context events 6 and 7 bracket every plan run (its total device time)
constexpr int kEvRunBegin = 6, kEvRunEnd = 7;

enum OpKind {
  OP_GEMM, OP_QR, OP_JACOBI, OP_TRUNC, OP_SELECT, OP_COPY, OP_ZERO, OP_SUMSQ, OP_APPLY,
  OP_PHILOX, OP_BF16GEMM, OP_ZEROCHK, OP_FINAL, OP_STAGE, OP_CVT_BF16, OP_SETRANK, OP_QAPPLY, OP_GEMM32, OP_CVT32,
  OP_WIDEN, OP_PINV_SCALE
};

struct Op {
  OpKind kind;
  size_t off = 0;      // byte offset of the descriptors in the plan blob
  int count = 0;       // number of descriptors
  long long total = 0; // tiles (GEMM) or max elements (streaming kernels)
  int a = 0, b = 0;    // kernel-specific (max_m, max_n, stage id ...)
  double tol = 0.0;
  long long rmax = 0;
  double flops = 0.0;  // algorithmic FLOPs of the launch (profiling only)
  int* iw = nullptr;   // kernel-specific device int workspace (the Jacobi problem order)
};

// "Finalize" descriptor: if *flag != 0, zero the TT's cores and restore its ranks.
struct FinalDesc {
  const int* flag;
  double* cores; long long n;
  int* rks; const int* rks_restore; int nrks;
};
// Zero check: flag = (sqrt(sumsq) < tol).
struct ZeroChkDesc { const double* sumsq; int* flag; double tol; };
// Set device rank slots from a constant table.
struct SetRankDesc { int* dst; const int* src; int n; };
// FP64 -> BF16 conversion with a 2-level index map: dst[i*ds_i + j*ds_j] = bf16(src[i*ss_i + j*ss_j]).
struct CvtDesc { const double* src; void* dst; long long rows, cols, ss_i, ss_j, ds_i, ds_j; double alpha; };

// Column scaling of a pseudo-inverse from a one-sided Jacobi SVD: X (m x n, ldx) holds A V
// (orthogonal columns, norms sigma); column i becomes X[:, i] / sigma_i^2 when
// sigma_i > eps * max(sigma), else zero (the kept set of src/tt_randtools.jl:485-489).
struct PinvScaleDesc { double* X; int ldx; int m, n; const double* sigma; double eps; };
void launch_pinv_scale(const PinvScaleDesc* d, int count, cudaStream_t s);
void launch_zerochk(const ZeroChkDesc* d, int count, cudaStream_t s);
void launch_final(const FinalDesc* d, int count, long long max_n, cudaStream_t s);
void launch_setrank(const SetRankDesc* d, int count, cudaStream_t s);
// FP64 -> BF16 (f32 = false) or FP64 -> FP32 rounded to TF32 (f32 = true), same index map.
void launch_cvt_bf16(const CvtDesc* d, int count, long long max_elems, cudaStream_t s, bool f32 = false);
// FP64 -> FP32 (round to nearest), same index map.
void launch_cvt_f32(const CvtDesc* d, int count, long long max_elems, cudaStream_t s);
// FP32 -> FP64: dst (double) from src holding floats, same index map (CvtDesc with the roles of the
// pointers swapped: `src` points to floats, `dst` to doubles).
void launch_widen(const CvtDesc* d, int count, long long max_elems, cudaStream_t s);

struct Plan {
  std::vector<unsigned char> blob;
  std::vector<Op> ops;
  size_t ws_needed = 0;
  unsigned char* d_blob = nullptr;
  size_t d_blob_cap = 0;
  void* ws_base = nullptr;           // workspace base the descriptors point into
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t graph_stream = nullptr;
  long long launches = 0;
  std::vector<std::pair<size_t, int>> diag;   // (blob offset, count) of Jacobi sweep counters
  ~Plan();
  template <class T>
  size_t push(const std::vector<T>& v) {
    size_t o = (blob.size() + 255) & ~size_t(255);
    blob.resize(o + v.size() * sizeof(T));
    if (!v.empty()) std::memcpy(blob.data() + o, v.data(), v.size() * sizeof(T));
    return o;
  }
};

}  // namespace ttc

struct ttc_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  int* d_flags = nullptr;
  double* d_one = nullptr;          // a device constant 1.0
  char* ws = nullptr;
  size_t ws_bytes = 0;
  ttc_stats stats{};
  cudaEvent_t ev[8]{};              // stage events 0..3 of a plan run; kEvRunBegin/kEvRunEnd
  bool last_run_graph = false;      // the last plan ran as a CUDA graph (no stage events)
  std::unordered_map<std::string, std::unique_ptr<ttc::Plan>> plans;
  bool use_graphs = true;
  void* d_stage = nullptr;          // device staging for uploads/downloads
  void* h_stage = nullptr;          // pinned host staging
  size_t stage_bytes = 0;
  double* d_sk = nullptr;           // host-provided sketch blocks
  size_t sk_cap = 0;
  bool profiling = false;           // per-kernel-family event timing (ttc_set_profiling)
  int jacobi_max_sweeps = ttc::kJacobiDefaultSweeps;   // sweep cap of the one-sided Jacobi SVD
  // device batches of the one-shot entry points (ttc_tt_rounding ...), reused by later calls of
  // the same shape, most recently used last; reuse also lets the plan cache, which is keyed on
  // batch identity, replay the captured plan
  std::vector<std::pair<std::string, ttc_batch*>> oneshot;
};

struct ttc_batch {
  ttc_context* ctx = nullptr;
  int count = 0, N = 0;
  std::vector<long long> dims;       // N
  std::vector<int> cap;              // count*(N+1)
  std::vector<long long> off;        // count*N, in doubles
  std::vector<long long> tt_off;     // count+1
  double* d_cores = nullptr;
  long long total = 0;               // doubles
  int* d_rks = nullptr;              // count*(N+1)
  int* d_zero = nullptr;             // count
  std::vector<int> h_rks;            // host ranks (valid unless rks_dirty)
  std::vector<int> h_ot;             // count*N
  bool rks_dirty = false;
  unsigned long long version = 0;    // bumped on every upload (plan cache key)
  double* core(int b, int k) const { return d_cores + off[(size_t)b * N + k]; }
  int capr(int b, int k) const { return cap[(size_t)b * (N + 1) + k]; }
  int rk(int b, int k) const { return h_rks[(size_t)b * (N + 1) + k]; }
  int* drk(int b, int k) const { return d_rks + (size_t)b * (N + 1) + k; }
};
