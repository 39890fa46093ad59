// Plan builder: collects kernel launches with their descriptors and hands out
// workspace regions from a bump allocator (mark/release per sweep step).
#pragma once
#include <functional>
#include <string>
#include <vector>

#include "runtime.cuh"

namespace ttc {

struct Builder {
  ttc_context* ctx = nullptr;
  Plan* plan = nullptr;
  char* wsbase = nullptr;                 // null in the measuring pass
  unsigned char* blob_base = nullptr;     // device address of the plan blob (null when measuring)
  size_t wsoff = 0, wshw = 0;

  double* wd(size_t n);
  int* wi(size_t n);
  size_t mark() const { return wsoff; }
  void release(size_t m) { wsoff = m; }
  void stage(int id);
  const int* const_ints(const std::vector<int>& v);
  // n ints in the plan's device blob that kernels may write (diagnostics such as Jacobi
  // sweep counts); read back by the profiled run.
  int* diag_ints(int n);

  void gemm(std::vector<GemmDesc> v);
  // the same problems with float data (FP32 accumulation)
  void gemm32(std::vector<GemmDesc> v);
  // FP64 -> FP32 (nearest) and FP32 -> FP64 conversions with the CvtDesc index map
  void cvt_f32(const std::vector<CvtDesc>& v);
  void widen(const std::vector<CvtDesc>& v);
  void qr(const std::vector<QRDesc>& v);
  void qapply(const std::vector<QApplyDesc>& v);
  void jacobi(const std::vector<JacobiDesc>& v);
  void trunc(const std::vector<TruncDesc>& v, double tol, long long rmax);
  void select(const std::vector<SelectDesc>& v);
  void copy(const std::vector<CopyDesc>& v);
  void zero(const std::vector<ZeroDesc>& v);
  void sumsq(const std::vector<NormDesc>& v);
  void apply(const std::vector<ApplyDesc>& v);
  void philox(const std::vector<PhiloxDesc>& v);
  // tcgen05 GEMM of BF16 operands, or FP32 operands read as TF32 (tf32 = true)
  void bf16gemm(std::vector<Bf16GemmDesc> v, bool tf32 = false);
  // FP64 -> BF16, or FP64 -> FP32 rounded to TF32 (f32 = true)
  void cvt_bf16(const std::vector<CvtDesc>& v, bool f32 = false);
  void zerochk(const std::vector<ZeroChkDesc>& v);
  void pinv_scale(const std::vector<PinvScaleDesc>& v);
  void finalize(const std::vector<FinalDesc>& v);
  void setrank(const std::vector<SetRankDesc>& v);
};

// Plain (unsplit) GEMM descriptor: A(i,k) at A[i*a_i + k*a_k], B(k,j) at B[k*b_k + j*b_j],
// C(i,j) at C[i*c_i + j*c_j].
GemmDesc gd(int m, int n, int k, const double* A, long long a_i, long long a_k, const double* B, long long b_k,
            long long b_j, double* C, long long c_i, long long c_j, double alpha = 1.0, double beta = 0.0);
CopyDesc cd2(const double* src, double* dst, long long e0, long long e1, long long s0, long long s1, long long d0,
             long long d1, double alpha = 1.0);
CopyDesc cd3(const double* src, double* dst, long long e0, long long e1, long long e2, long long s0, long long s1,
             long long s2, long long d0, long long d1, long long d2, double alpha = 1.0);

Plan* get_plan(ttc_context* c, const std::string& key, const std::function<void(Builder&)>& fn);
void run_plan(ttc_context* c, Plan& p);
void ensure_workspace(ttc_context* c, size_t bytes);
void check_device_flags(ttc_context* c);

ttc_batch* batch_create(ttc_context* c, int count, int N, const long long* dims, const int* cap);
void batch_destroy(ttc_batch* b);
void batch_sync_ranks(ttc_batch* b);
std::string batch_key(const ttc_batch* b);
// Key of a batch that a plan only writes (zeroed and given its ranks by the plan itself): its
// identity, whatever its current rank state.
std::string batch_out_key(const ttc_batch* b);
// version = hash of the host ranks and orthogonality flags (after an upload or a rank sync).
void batch_rehash(ttc_batch* b);

}  // namespace ttc
