// Shared definitions of libttcuda: status codes, error capture, device helpers
// and the grouped GEMM descriptor used by every contraction in the library.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <stdexcept>

#include "../../include/ttcuda.h"

namespace ttc {

// Error raised inside the host drivers; the C-ABI layer converts it into a status
// code and stores the message in the context.
struct Error : public std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define TTC_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e__ = (call);                                                       \
    if (e__ != cudaSuccess)                                                         \
      throw ::ttc::Error(TTC_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
  } while (0)

#define TTC_CHECK_LAUNCH() TTC_CUDA(cudaGetLastError())

#define TTC_REQUIRE(cond, code, msg)                                                \
  do {                                                                              \
    if (!(cond)) throw ::ttc::Error((code), (msg));                                 \
  } while (0)

// Device-side error flags (one int per context).  Kernels set bits with atomicOr;
// the host reads them at synchronisation points.
enum DeviceFlag : int {
  DFLAG_JACOBI_NOCONV = 1,   // one-sided Jacobi hit its sweep cap
  DFLAG_NONFINITE = 2,       // NaN/Inf met in a factorisation input
  DFLAG_BAD_DESC = 4,        // a kernel met an inconsistent descriptor and skipped it
  DFLAG_TIMEOUT = 8,         // a bounded mbarrier wait gave up
};

// One GEMM problem: C = alpha * op(A) * op(B) + beta * C over `batch` strided instances.
// Each of the three GEMM indices may be split in two levels so that permuted tensor
// unfoldings need no copy:  row i = i0 + m0*i1,  column j = j0 + n0*j1,  reduction
// k = k0 + k0e*k1 (an extent >= the index range means "no split").  Element offsets:
//   A(i, k) = i0*a_i0 + i1*a_i1 + k0*a_k0 + k1*a_k1 + b*a_b
//   B(k, j) = k0*b_k0 + k1*b_k1 + j0*b_j0 + j1*b_j1 + b*b_b
//   C(i, j) = i0*c_i0 + i1*c_i1 + j0*c_j0 + j1*c_j1 + b*c_b
struct GemmDesc {
  int m, n, k, batch;
  int m0, n0, k0e;
  const double* A;
  long long a_i0, a_i1, a_k0, a_k1, a_b;
  const double* B;
  long long b_k0, b_k1, b_j0, b_j1, b_b;
  double* C;
  long long c_i0, c_i1, c_j0, c_j1, c_b;
  double alpha, beta;
  long long tile_start;   // first flat tile index of this problem (prefix sum, filled by the planner)
  // Optional device-side bound on the columns that can be nonzero (for example a truncation
  // rank written by an earlier kernel): output columns >= *n_dev are B columns known to be zero,
  // so their tiles store zeros (beta == 0) or are skipped (beta != 0) without the product.
  const int* n_dev;
  // Split-K (FP64 kernel only; set by the planner): ksplit > 1 CTAs share each output tile, each
  // over a contiguous range of K; they leave their partial tiles in ws, and the last to finish
  // (counted in cnt, one zeroed counter per output tile, reset by that CTA) adds them up in split
  // order, so the result does not depend on which CTA finishes last.
  int ksplit;
  double* ws;
  unsigned* cnt;
};

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

// One-time set-up per device (kernel attributes such as the dynamic shared-memory limit) for
// launchers that host threads driving different devices may call at the same time: `fn` runs
// once for each device, under a mutex, before any launch on that device returns from here.
constexpr int kMaxDevices = 64;
struct PerDeviceOnce {
  std::mutex mu;
  bool done[kMaxDevices] = {};
  template <class F>
  void run(int dev, F&& fn) {
    if (dev < 0 || dev >= kMaxDevices) throw Error(TTC_EARG, "device index out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (!done[dev]) {
      fn();
      done[dev] = true;
    }
  }
};
// Streaming multiprocessors of the current device (queried once per device, thread-safe).
int current_sm_count();

// FP32 value rounded to the nearest TF32 (10-bit mantissa, PTX cvt.rna.tf32.f32).  The tensor
// cores read a kind::tf32 operand by dropping its low 13 mantissa bits (toward zero); operands
// rounded here first carry an unbiased error instead, which does not accumulate coherently
// through the levels of a recursive sketch.
__device__ __forceinline__ float round_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

}  // namespace ttc
