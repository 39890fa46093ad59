// Grouped, strided-batched FP64 GEMM for the FP64 contractions of the rounding sweeps
// (FR*core, absorb U*S, Z = y_k W, Q^T y_k, environment updates).  One launch runs a
// list of GemmDesc problems; CTA t finds its problem by binary search over the
// descriptors' tile prefix sums, so ranks that differ per TT and per site share one
// launch.  64x64x16 tiles, 256 threads, register-prefetch double buffering of the shared
// A/B tiles; the products run on the FP64 tensor cores (mma.sync m8n8k4), each warp owning a
// 32 x 16 sub-tile (4 x 2 fragments of 8 x 8).  The C tile is staged through shared memory so
// that the store is coalesced along whichever C stride is 1 (plain or transposed output).
// The split K index (k0 + k0e k1) of every loaded element advances incrementally, with no
// division in the K loop.  Launches of few output tiles and long K (the range finder and
// projections of the operator rounding, K = r R) split K over several CTAs per tile.
#include <algorithm>

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
  __shared__ int s_last;
  double (*As)[BK][PAD] = reinterpret_cast<double (*)[BK][PAD]>(smem);
  double (*Bs)[BK][PAD] = reinterpret_cast<double (*)[BK][PAD]>(smem + 2 * BK * PAD);

  const int tid = threadIdx.x;
  const long long tile = blockIdx.x;
  const int di = find_desc(descs, nd, tile);
  const GemmDesc D = descs[di];
  const int tm = ceil_div(D.m, BM), tn = ceil_div(D.n, BN);
  const long long local = tile - D.tile_start;
  const int per = tm * tn;
  const int ks = D.ksplit > 1 ? D.ksplit : 1;
  const long long tiles_out = (long long)per * D.batch;          // output tiles of this problem
  if (per == 0 || local >= tiles_out * ks) return;
  const int split = (int)(local / tiles_out);
  const long long lt = local - (long long)split * tiles_out;     // output tile
  const int b = (int)(lt / per);
  const int rem = (int)(lt - (long long)b * per);
  const int bm = rem % tm, bn = rem / tm;
  const int row0 = bm * BM, col0 = bn * BN;
  if (D.n_dev && col0 >= *D.n_dev) {          // every column of this tile is known to be zero
    if (D.beta != 0.0 || split != 0) return;  // (the same decision in every split: no counting)
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

  // Loader mappings: contiguous along the unit-stride index when there is one.  Each thread
  // loads 4 elements of A at one K index (4 rows) and 4 of B at one K index (4 columns).
  const bool a_rowfast = (D.a_i0 == 1);          // consecutive rows contiguous
  const bool b_colfast = (D.b_j0 == 1);          // consecutive cols contiguous
  const int a_k = a_rowfast ? (tid >> 4) : (tid & 15);
  const int b_k = b_colfast ? (tid >> 4) : (tid & 15);
  // rows ar0 + 16 t of A and columns bc0 + 16 t of B; a_ok / b_ok: bit t set when in range
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
  // this CTA's K range, in BK-wide steps
  const int nk_all = ceil_div(D.k, BK);
  const int chunk = ceil_div(nk_all, ks);
  const int kt_beg = min(nk_all, split * chunk), kt_end = min(nk_all, kt_beg + chunk);
  // running split K coordinate of this thread's A and B elements: kr = gk mod k0e and the
  // element offset kr k_0 + (gk / k0e) k_1, advanced by BK per step without a division
  const long long a_wrap = D.a_k1 - (long long)k0e * D.a_k0, b_wrap = D.b_k1 - (long long)k0e * D.b_k0;
  int a_kr, b_kr;
  long long a_ko, b_ko;
  {
    const int ga = kt_beg * BK + a_k, gb = kt_beg * BK + b_k;
    a_kr = ga % k0e; a_ko = (long long)a_kr * D.a_k0 + (long long)(ga / k0e) * D.a_k1;
    b_kr = gb % k0e; b_ko = (long long)b_kr * D.b_k0 + (long long)(gb / k0e) * D.b_k1;
  }

  double ra[4], rb[4];
  // loads the step at k0 and advances the running coordinates to k0 + BK
  auto load_tile = [&](int k0) {
    const bool ka = k0 + a_k < D.k, kb = k0 + b_k < D.k;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      ra[t] = (ka && ((a_ok >> t) & 1u)) ? A[a_roff[t] + a_ko] : 0.0;
      rb[t] = (kb && ((b_ok >> t) & 1u)) ? B[b_coff[t] + b_ko] : 0.0;
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

  // Warp w owns rows wm*32 .. +31 and cols wn*16 .. +15 of the tile; fragment coordinates:
  // A[qr][qc] = As[k + qc][i + qr], B[qc][qr] = Bs[k + qc][j + qr], D[qr][2qc + {0,1}].
  const int warp = tid >> 5, lane = tid & 31, qr = lane >> 2, qc = lane & 3;
  const int wm = warp & 1, wn = warp >> 1;
  double acc[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }

  if (kt_end > kt_beg) {
    load_tile(kt_beg * BK);
    store_tile(0);
    __syncthreads();
    for (int kt = kt_beg; kt < kt_end; ++kt) {
      const int cur = (kt - kt_beg) & 1;
      if (kt + 1 < kt_end) load_tile((kt + 1) * BK);
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
      if (kt + 1 < kt_end) store_tile(cur ^ 1);
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
  if (ks > 1) {
    // this split's partial tile into its slot, then the last CTA of the tile to arrive sums
    // the ks slots in split order into the staged tile
    double* slots = D.ws + lt * ks * (long long)(BM * BN);
    double* mine = slots + (long long)split * (BM * BN);
    for (int e = tid; e < BM * BN; e += NT) mine[e] = Cs[(e >> 6) * PADC + (e & 63)];
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(D.cnt + lt, 1u) == (unsigned)(ks - 1));
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int e = tid; e < BM * BN; e += NT) {
      const int ci = (e >> 6) * PADC + (e & 63);
      double v = 0.0;
      for (int s2 = 0; s2 < ks; ++s2) v += (s2 == split) ? Cs[ci] : __ldcg(slots + (long long)s2 * (BM * BN) + e);
      Cs[ci] = v;
    }
    if (tid == 0) D.cnt[lt] = 0u;   // zero again for the next launch of the plan
    __syncthreads();
  }
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
  return (long long)ceil_div(d.m, BM) * ceil_div(d.n, BN) * d.batch * (d.ksplit > 1 ? d.ksplit : 1);
}

int gemm_pick_ksplit(const GemmDesc& d, long long launch_tiles, int nsm) {
  // enough CTAs for two per SM over the whole launch, each split at least 32 K steps deep
  const long long want = 2LL * nsm;
  if (launch_tiles <= 0 || launch_tiles >= want) return 1;
  const int nk = ceil_div(d.k, BK);
  const long long by_fill = (want + launch_tiles - 1) / launch_tiles;
  const long long by_depth = nk / 32;
  return (int)std::max(1LL, std::min({by_fill, by_depth, 16LL}));
}

long long gemm_split_ws_doubles(const GemmDesc& d) {
  if (d.ksplit <= 1) return 0;
  return (long long)ceil_div(d.m, BM) * ceil_div(d.n, BN) * d.batch * d.ksplit * (BM * BN);
}

}  // namespace ttc
