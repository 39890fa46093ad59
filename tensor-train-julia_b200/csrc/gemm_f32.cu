// Grouped, strided-batched FP32 GEMM (FP32 operands, FP32 accumulation, CUDA-core FMA) for the
// FP32 variant of the Rayleigh-quotient gradient: the same GemmDesc problems as the FP64 grouped
// GEMM (split row/column/K indices, batches, alpha/beta, the device column bound), with A, B
// and C holding float data.  64x64x16 tiles (the FP64 kernel's tile grid, so the planner's tile
// prefix sums serve both), 256 threads, a 4x4 register block per thread fed by float4 shared-memory
// loads, register-prefetch double buffering, the split K index advanced without a division, and the
// C tile staged in shared memory for stores along C's unit stride; CTA t finds its problem by
// binary search over the descriptors' tile prefix sums.
#include "common.cuh"
#include "kernels.cuh"

namespace ttc {

namespace {
// PAD = 68 floats: the float4 fragment loads of a row are contiguous, the loader's column writes
// spread over the banks; PADC = 65 for the staged C tile.
constexpr int BM = 64, BN = 64, BK = 16, NT = 256, PAD = 68, PADC = 65;

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
  __shared__ __align__(16) float smem[2 * 2 * BK * PAD];   // As[2][BK][PAD], Bs[2][BK][PAD]; then the C tile
  float (*As)[BK][PAD] = reinterpret_cast<float (*)[BK][PAD]>(smem);
  float (*Bs)[BK][PAD] = reinterpret_cast<float (*)[BK][PAD]>(smem + 2 * BK * PAD);
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

  // Loader mappings as in the FP64 kernel: contiguous along the unit-stride index when there is
  // one; each thread loads 4 elements of A at one K index (4 rows) and 4 of B (4 columns), with
  // the row/column offsets computed once and the split K coordinate advanced without a division.
  const bool a_rowfast = (D.a_i0 == 1), b_colfast = (D.b_j0 == 1);
  const int a_k = a_rowfast ? (tid >> 4) : (tid & 15);
  const int b_k = b_colfast ? (tid >> 4) : (tid & 15);
  const int ar0 = a_rowfast ? (tid & 15) : (tid >> 4), bc0 = b_colfast ? (tid & 15) : (tid >> 4);
  unsigned a_ok = 0, b_ok = 0;
  long long a_roff[4], b_coff[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int gi = row0 + ar0 + 16 * t, gj = col0 + bc0 + 16 * t;
    a_ok |= (gi < D.m ? 1u : 0u) << t;
    b_ok |= (gj < D.n ? 1u : 0u) << t;
    a_roff[t] = (long long)(gi % D.m0) * D.a_i0 + (long long)(gi / D.m0) * D.a_i1;
    b_coff[t] = (long long)(gj % D.n0) * D.b_j0 + (long long)(gj / D.n0) * D.b_j1;
  }
  const int k0e = D.k0e;
  const long long a_wrap = D.a_k1 - (long long)k0e * D.a_k0, b_wrap = D.b_k1 - (long long)k0e * D.b_k0;
  int a_kr = a_k % k0e, b_kr = b_k % k0e;
  long long a_ko = (long long)a_kr * D.a_k0 + (long long)(a_k / k0e) * D.a_k1;
  long long b_ko = (long long)b_kr * D.b_k0 + (long long)(b_k / k0e) * D.b_k1;
  float ra[4], rb[4];
  auto load_tile = [&](int k0) {
    const bool ka = k0 + a_k < D.k, kb = k0 + b_k < D.k;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      ra[t] = (ka && ((a_ok >> t) & 1u)) ? A[a_roff[t] + a_ko] : 0.f;
      rb[t] = (kb && ((b_ok >> t) & 1u)) ? Bm[b_coff[t] + b_ko] : 0.f;
    }
    a_kr += BK; a_ko += BK * D.a_k0;
    while (a_kr >= k0e) { a_kr -= k0e; a_ko += a_wrap; }
    b_kr += BK; b_ko += BK * D.b_k0;
    while (b_kr >= k0e) { b_kr -= k0e; b_ko += b_wrap; }
  };
  auto store_tile = [&](int buf) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      As[buf][a_k][ar0 + 16 * t] = ra[t];
      Bs[buf][b_k][bc0 + 16 * t] = rb[t];
    }
  };

  const int tx = tid & 15, ty = tid >> 4;     // 16 x 16 threads, each a 4 x 4 block
  float acc[4][4] = {};
  const int nk = ceil_div(D.k, BK);
  if (nk > 0) {
    load_tile(0);
    store_tile(0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
      const int cur = kt & 1;
      if (kt + 1 < nk) load_tile((kt + 1) * BK);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        const float4 a = *reinterpret_cast<const float4*>(&As[cur][kk][ty * 4]);
        const float4 bb = *reinterpret_cast<const float4*>(&Bs[cur][kk][tx * 4]);
        const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {bb.x, bb.y, bb.z, bb.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
      }
      if (kt + 1 < nk) store_tile(cur ^ 1);
      __syncthreads();
    }
  }
  // stage the C tile (64 x 65 floats, column-major), then store along C's unit stride
  float* Cs = smem;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) Cs[(tx * 4 + j) * PADC + ty * 4 + i] = acc[i][j];
  __syncthreads();
  const bool c_colfast = (D.c_j0 == 1 && D.c_i0 != 1);
  const float alpha = (float)D.alpha, beta = (float)D.beta;
  for (int e = tid; e < BM * BN; e += NT) {
    int li, lj;
    if (c_colfast) { lj = e & 63; li = e >> 6; } else { li = e & 63; lj = e >> 6; }
    const int gi = row0 + li, gj = col0 + lj;
    if (gi < D.m && gj < D.n) {
      float* p = C + coff(gi, gj);
      const float v = alpha * Cs[lj * PADC + li];
      *p = (beta == 0.f) ? v : fmaf(beta, *p, v);
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
