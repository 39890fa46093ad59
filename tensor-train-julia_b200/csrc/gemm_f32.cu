// Grouped, strided-batched FP32 GEMM (FP32 operands, FP32 accumulation, CUDA-core FMA) for the
// FP32 variant of the Rayleigh-quotient gradient: the same GemmDesc problems as the FP64 grouped
// GEMM (split row/column/K indices, batches, alpha/beta, the device column bound), with A, B
// and C holding float data.  64x64x16 tiles, 256 threads, a 4x4 register block per thread; CTA t
// finds its problem by binary search over the descriptors' tile prefix sums.
#include "common.cuh"
#include "kernels.cuh"

namespace ttc {

namespace {
constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

__device__ __forceinline__ int find_desc32(const GemmDesc* __restrict__ d, int nd, long long tile) {
  int lo = 0, hi = nd - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (d[mid].tile_start <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}
}  // namespace

__global__ void __launch_bounds__(NT) gemm_f32_grouped_kernel(const GemmDesc* __restrict__ descs, int nd) {
  __shared__ float As[BK][BM + 4];
  __shared__ float Bs[BK][BN + 4];
  const int tid = threadIdx.x;
  const long long tile = blockIdx.x;
  const GemmDesc D = descs[find_desc32(descs, nd, tile)];
  const int tm = ceil_div(D.m, BM), tn = ceil_div(D.n, BN);
  const int per = tm * tn;
  const long long local = tile - D.tile_start;
  if (per == 0 || local < 0 || local >= (long long)per * D.batch) return;
  const int b = (int)(local / per);
  const int rem = (int)(local - (long long)b * per);
  const int row0 = (rem % tm) * BM, col0 = (rem / tm) * BN;
  float* __restrict__ C = reinterpret_cast<float*>(D.C) + (long long)b * D.c_b;
  auto coff = [&](int gi, int gj) {
    return (long long)(gi % D.m0) * D.c_i0 + (long long)(gi / D.m0) * D.c_i1 + (long long)(gj % D.n0) * D.c_j0 +
           (long long)(gj / D.n0) * D.c_j1;
  };
  if (D.n_dev && col0 >= *D.n_dev) {          // every column of this tile is known to be zero
    if (D.beta != 0.0) return;
    for (int e = tid; e < BM * BN; e += NT) {
      const int gi = row0 + (e & 63), gj = col0 + (e >> 6);
      if (gi < D.m && gj < D.n) C[coff(gi, gj)] = 0.f;
    }
    return;
  }
  const float* __restrict__ A = reinterpret_cast<const float*>(D.A) + (long long)b * D.a_b;
  const float* __restrict__ Bm = reinterpret_cast<const float*>(D.B) + (long long)b * D.b_b;
  const int tx = tid & 15, ty = tid >> 4;     // 16 x 16 threads, each a 4 x 4 block
  float acc[4][4] = {};
  for (int k0 = 0; k0 < D.k; k0 += BK) {
#pragma unroll
    for (int t = 0; t < (BM * BK) / NT; ++t) {
      const int e = tid + NT * t;
      const int li = e & 63, lk = e >> 6;
      const int gi = row0 + li, gk = k0 + lk;
      float v = 0.f;
      if (gi < D.m && gk < D.k)
        v = A[(long long)(gi % D.m0) * D.a_i0 + (long long)(gi / D.m0) * D.a_i1 + (long long)(gk % D.k0e) * D.a_k0 +
              (long long)(gk / D.k0e) * D.a_k1];
      As[lk][li] = v;
    }
#pragma unroll
    for (int t = 0; t < (BN * BK) / NT; ++t) {
      const int e = tid + NT * t;
      const int lk = e & 15, lj = e >> 4;
      const int gj = col0 + lj, gk = k0 + lk;
      float v = 0.f;
      if (gj < D.n && gk < D.k)
        v = Bm[(long long)(gk % D.k0e) * D.b_k0 + (long long)(gk / D.k0e) * D.b_k1 + (long long)(gj % D.n0) * D.b_j0 +
               (long long)(gj / D.n0) * D.b_j1];
      Bs[lk][lj] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float a[4], bb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bb[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], bb[j], acc[i][j]);
    }
    __syncthreads();
  }
  const float alpha = (float)D.alpha, beta = (float)D.beta;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gi = row0 + ty * 4 + i, gj = col0 + tx * 4 + j;
      if (gi < D.m && gj < D.n) {
        const long long o = coff(gi, gj);
        C[o] = (beta != 0.f) ? fmaf(alpha, acc[i][j], beta * C[o]) : alpha * acc[i][j];
      }
    }
}

void launch_gemm_f32(const GemmDesc* d_descs, int nd, long long total_tiles, cudaStream_t s) {
  if (nd <= 0 || total_tiles <= 0) return;
  TTC_REQUIRE(total_tiles < (1LL << 31), TTC_EINTERNAL, "gemm: too many tiles in one launch");
  gemm_f32_grouped_kernel<<<(unsigned)total_tiles, NT, 0, s>>>(d_descs, nd);
  TTC_CHECK_LAUNCH();
}

}  // namespace ttc
