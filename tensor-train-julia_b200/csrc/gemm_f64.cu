// Grouped, strided-batched FP64 GEMM for the FP64 contractions of the rounding sweeps
// (FR*core, absorb U*S, Z = y_k W, Q^T y_k, environment updates).  One launch runs a
// list of GemmDesc problems; CTA t finds its problem by binary search over the
// descriptors' tile prefix sums, so ranks that differ per TT and per site share one
// launch.  64x64x16 tiles, 256 threads, register-prefetch double buffering of the shared
// A/B tiles; the products run on the FP64 tensor cores (mma.sync m8n8k4), each warp owning a
// 32 x 16 sub-tile (4 x 2 fragments of 8 x 8).  The C tile is staged through shared memory so
// that the store is coalesced along whichever C stride is 1 (plain or transposed output).
#include "common.cuh"
#include "kernels.cuh"

namespace ttc {

namespace {
// PAD = 4 mod 16 doubles: the fragment loads (4 k x 4 rows per half warp) hit distinct banks.
constexpr int BM = 64, BN = 64, BK = 16, NT = 256, PAD = 68, PADC = 65;

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ int find_desc(const GemmDesc* __restrict__ d, int nd, long long tile) {
  int lo = 0, hi = nd - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (d[mid].tile_start <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}
}  // namespace

__global__ void __launch_bounds__(NT, 2) gemm_f64_grouped_kernel(const GemmDesc* __restrict__ descs, int nd) {
  __shared__ double smem[2 * BK * PAD * 2];   // As[2][BK][PAD], Bs[2][BK][PAD]; reused for the C tile
  double (*As)[BK][PAD] = reinterpret_cast<double (*)[BK][PAD]>(smem);
  double (*Bs)[BK][PAD] = reinterpret_cast<double (*)[BK][PAD]>(smem + 2 * BK * PAD);

  const int tid = threadIdx.x;
  const long long tile = blockIdx.x;
  const int di = find_desc(descs, nd, tile);
  const GemmDesc D = descs[di];
  const int tm = ceil_div(D.m, BM), tn = ceil_div(D.n, BN);
  const long long local = tile - D.tile_start;
  const int per = tm * tn;
  if (per == 0 || local >= (long long)per * D.batch) return;
  const int b = (int)(local / per);
  const int rem = (int)(local - (long long)b * per);
  const int bm = rem % tm, bn = rem / tm;
  const int row0 = bm * BM, col0 = bn * BN;
  if (D.n_dev && col0 >= *D.n_dev) {          // every column of this tile is known to be zero
    if (D.beta != 0.0) return;
    double* __restrict__ Cz = D.C + (long long)b * D.c_b;
    for (int e = threadIdx.x; e < BM * BN; e += NT) {
      const int li = e & 63, lj = e >> 6;
      const int gi = row0 + li, gj = col0 + lj;
      if (gi < D.m && gj < D.n)
        Cz[(long long)(gi % D.m0) * D.c_i0 + (long long)(gi / D.m0) * D.c_i1 + (long long)(gj % D.n0) * D.c_j0 +
           (long long)(gj / D.n0) * D.c_j1] = 0.0;
    }
    return;
  }

  const double* __restrict__ A = D.A + (long long)b * D.a_b;
  const double* __restrict__ B = D.B + (long long)b * D.b_b;
  double* __restrict__ C = D.C + (long long)b * D.c_b;

  // Loader mappings: contiguous along the unit-stride index when there is one.
  const bool a_rowfast = (D.a_i0 == 1);          // consecutive rows contiguous
  const bool b_colfast = (D.b_j0 == 1);          // consecutive cols contiguous
  int a_i[4], a_k[4], b_k[4], b_j[4];
  long long a_roff[4], b_coff[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    if (a_rowfast) { a_i[t] = tid & 63; a_k[t] = (tid >> 6) + 4 * t; }
    else           { a_k[t] = tid & 15; a_i[t] = (tid >> 4) + 16 * t; }
    if (b_colfast) { b_j[t] = tid & 63; b_k[t] = (tid >> 6) + 4 * t; }
    else           { b_k[t] = tid & 15; b_j[t] = (tid >> 4) + 16 * t; }
    const int gi = row0 + a_i[t], gj = col0 + b_j[t];
    a_roff[t] = (long long)(gi % D.m0) * D.a_i0 + (long long)(gi / D.m0) * D.a_i1;
    b_coff[t] = (long long)(gj % D.n0) * D.b_j0 + (long long)(gj / D.n0) * D.b_j1;
  }
  const int k0e = D.k0e;

  double ra[4], rb[4];
  auto load_tile = [&](int k0) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int gi = row0 + a_i[t], gk = k0 + a_k[t];
      ra[t] = (gi < D.m && gk < D.k) ? A[a_roff[t] + (long long)(gk % k0e) * D.a_k0 + (long long)(gk / k0e) * D.a_k1] : 0.0;
      const int gj = col0 + b_j[t], gk2 = k0 + b_k[t];
      rb[t] = (gj < D.n && gk2 < D.k) ? B[b_coff[t] + (long long)(gk2 % k0e) * D.b_k0 + (long long)(gk2 / k0e) * D.b_k1] : 0.0;
    }
  };
  auto store_tile = [&](int buf) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      As[buf][a_k[t]][a_i[t]] = ra[t];
      Bs[buf][b_k[t]][b_j[t]] = rb[t];
    }
  };

  // Warp w owns rows wm*32 .. +31 and cols wn*16 .. +15 of the tile; fragment coordinates:
  // A[qr][qc] = As[k + qc][i + qr], B[qc][qr] = Bs[k + qc][j + qr], D[qr][2qc + {0,1}].
  const int warp = tid >> 5, lane = tid & 31, qr = lane >> 2, qc = lane & 3;
  const int wm = warp & 1, wn = warp >> 1;
  double acc[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }

  const int nk = ceil_div(D.k, BK);
  if (nk > 0) {
    load_tile(0);
    store_tile(0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
      const int cur = kt & 1;
      if (kt + 1 < nk) load_tile((kt + 1) * BK);
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        double a[4], bv[2];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[cur][kk + qc][wm * 32 + 8 * i + qr];
#pragma unroll
        for (int j = 0; j < 2; ++j) bv[j] = Bs[cur][kk + qc][wn * 16 + 8 * j + qr];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], bv[j]);
      }
      if (kt + 1 < nk) store_tile(cur ^ 1);
      __syncthreads();
    }
  }

  // Stage the C tile in shared memory (64 x 65 doubles, column-major), then store coalesced.
  double* Cs = smem;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e)
        Cs[(wn * 16 + 8 * j + 2 * qc + e) * PADC + (wm * 32 + 8 * i + qr)] = acc[i][j][e];
  __syncthreads();
  const bool c_colfast = (D.c_j0 == 1 && D.c_i0 != 1);
  const double alpha = D.alpha, beta = D.beta;
  for (int e = tid; e < BM * BN; e += NT) {
    int li, lj;
    if (c_colfast) { lj = e & 63; li = e >> 6; } else { li = e & 63; lj = e >> 6; }
    const int gi = row0 + li, gj = col0 + lj;
    if (gi < D.m && gj < D.n) {
      double* p = C + (long long)(gi % D.m0) * D.c_i0 + (long long)(gi / D.m0) * D.c_i1 +
                  (long long)(gj % D.n0) * D.c_j0 + (long long)(gj / D.n0) * D.c_j1;
      const double v = alpha * Cs[lj * PADC + li];
      *p = (beta == 0.0) ? v : fma(beta, *p, v);
    }
  }
}

// Host launcher: descs already resident on the device (tile_start filled).
void launch_gemm_f64(const GemmDesc* d_descs, int nd, long long total_tiles, cudaStream_t s) {
  if (nd <= 0 || total_tiles <= 0) return;
  TTC_REQUIRE(total_tiles < (1LL << 31), TTC_EINTERNAL, "gemm: too many tiles in one launch");
  gemm_f64_grouped_kernel<<<(unsigned)total_tiles, NT, 0, s>>>(d_descs, nd);
  TTC_CHECK_LAUNCH();
}

long long gemm_tiles(const GemmDesc& d) {
  if (d.m <= 0 || d.n <= 0 || d.batch <= 0) return 0;
  return (long long)ceil_div(d.m, BM) * ceil_div(d.n, BN) * d.batch;
}

}  // namespace ttc
