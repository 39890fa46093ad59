// Batched blocked Householder QR, one CTA per problem.
//
// Replaces Julia `qr(A)` / `qr!(Z)` + `Matrix(F.Q)` (LAPACK geqrf + orgqr) on the
// tall-skinny unfoldings of the orthogonalisation sweep (src/tt_rounding.jl:75-78) and of
// the randomized range finder (src/tt_randtools.jl:134-135).  Householder is used (not
// CholeskyQR) because the range-finder matrices are rank deficient by construction when
// the sketch rank exceeds the TT rank, and zero-padded cores give exactly zero columns;
// Householder returns an orthonormal Q for any input, like LAPACK.
//
// Layout: panels of NB = 16 columns are factored in shared memory (reflectors with the
// LAPACK dlarfg convention beta = -sign(alpha)*||x||), the block reflector
// I - V T V^T (dlarft) is applied to the trailing columns by warps that own two
// columns each (V is read from shared memory once per pair of columns), and Q is formed
// backwards from the stored panels (dorgqr).
//
// One thread-block cluster of C CTAs per problem.  Every CTA factors each panel itself
// (same data, same arithmetic: identical reflectors, no broadcast needed); the column pairs
// (2p, 2p+1) of the trailing update and of Q are owned by CTA p mod C, so a column is always
// updated by the same CTA.  A cluster barrier (release/acquire at cluster scope) after each
// panel's trailing update makes the next panel visible to every CTA.  CTA 0 writes the
// factored panels and the T factors, which the Q formation reads after one more barrier.
#include <cooperative_groups.h>

#include <algorithm>

#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace ttc {
namespace {
constexpr int NB = 16;
constexpr int NT = 256;
constexpr int NW = NT / 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; `red` holds NW doubles.  All threads get the result.
__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < NW; ++i) s += red[i];
  return s;
}

// Copy `cols` columns of `rows` doubles (one warp per column, lanes over rows, four loads in
// flight per lane); returns whether a non-finite value was copied.
__device__ __forceinline__ bool copy_cols(double* __restrict__ dst, long long dld, const double* __restrict__ src,
                                          long long sld, int rows, int cols) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool bad = false;
  for (int c = warp; c < cols; c += NW) {
    const double* sc = src + (long long)c * sld;
    double* dc = dst + (long long)c * dld;
    for (int r0 = lane; r0 < rows; r0 += 128) {
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = (r0 + 32 * u < rows) ? sc[r0 + 32 * u] : 0.0;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (r0 + 32 * u < rows) { dc[r0 + 32 * u] = v[u]; bad |= !isfinite(v[u]); }
    }
  }
  return bad;
}

// Apply (I - V T^T V^T) [trans=1] or (I - V T V^T) [trans=0] to columns [c_begin, c_end) of
// the global matrix M (rows r0..m-1, ld), with V (mp x jb) in shared memory (column-major,
// stride mp_ld, unit diagonal implied, zeros above) and T (jb x jb) in shared memory.
// Column pairs (2p, 2p+1) with p mod csize == crank belong to this CTA.
__device__ void apply_block_reflector(double* M, int ld, int r0, int m, int c_begin, int c_end,
                                      const double* V, int mp_ld, int jb, const double* T, bool trans,
                                      int crank, int csize) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mp = m - r0;
  const int p_begin = c_begin >> 1, p_end = (c_end + 1) >> 1;
  const int p_first = p_begin + ((crank - p_begin) % csize + csize) % csize;
  for (int p = p_first + warp * csize; p < p_end; p += NW * csize) {
    const int c = 2 * p;
    if (c + 1 < c_begin) continue;
    // a pair may straddle c_begin (odd start) or c_end: update only the columns inside
    const bool has0 = (c >= c_begin), two = has0 ? (c + 1 < c_end) : false;
    double* col0 = M + (long long)(has0 ? c : c + 1) * ld + r0;
    double* col1 = M + (long long)(c + 1) * ld + r0;
    double w0[NB], w1[NB];
#pragma unroll
    for (int l = 0; l < NB; ++l) { w0[l] = 0.0; w1[l] = 0.0; }
#pragma unroll 4
    for (int r = lane; r < mp; r += 32) {
      const double x0 = col0[r];
      const double x1 = two ? col1[r] : 0.0;
#pragma unroll
      for (int l = 0; l < NB; ++l) {
        if (l < jb) {
          const double v = (r > l) ? V[l * mp_ld + r] : (r == l ? 1.0 : 0.0);
          w0[l] = fma(v, x0, w0[l]);
          w1[l] = fma(v, x1, w1[l]);
        }
      }
    }
#pragma unroll
    for (int l = 0; l < NB; ++l) {
      if (l < jb) { w0[l] = warp_sum(w0[l]); w1[l] = warp_sum(w1[l]); }
    }
    // u = T^T w (trans) or T w, T upper triangular, computed in place: u_l = sum_{i<=l}
    // T[i,l] w_i needs only w_0..w_l (descending l); u_l = sum_{i>=l} T[l,i] w_i needs only
    // w_l..w_{jb-1} (ascending l).
    if (trans) {
#pragma unroll
      for (int l = NB - 1; l >= 0; --l) {
        double a0 = 0.0, a1 = 0.0;
        if (l < jb) {
#pragma unroll
          for (int i = 0; i < NB; ++i)
            if (i <= l) { a0 = fma(T[l * NB + i], w0[i], a0); a1 = fma(T[l * NB + i], w1[i], a1); }
        }
        w0[l] = a0; w1[l] = a1;
      }
    } else {
#pragma unroll
      for (int l = 0; l < NB; ++l) {
        double a0 = 0.0, a1 = 0.0;
        if (l < jb) {
#pragma unroll
          for (int i = 0; i < NB; ++i)
            if (i >= l && i < jb) { a0 = fma(T[i * NB + l], w0[i], a0); a1 = fma(T[i * NB + l], w1[i], a1); }
        }
        w0[l] = a0; w1[l] = a1;
      }
    }
#pragma unroll 4
    for (int r = lane; r < mp; r += 32) {
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int l = 0; l < NB; ++l) {
        if (l < jb) {
          const double v = (r > l) ? V[l * mp_ld + r] : (r == l ? 1.0 : 0.0);
          d0 = fma(v, w0[l], d0);
          d1 = fma(v, w1[l], d1);
        }
      }
      col0[r] -= d0;
      if (two) col1[r] -= d1;
    }
  }
}
}  // namespace

// T layout in shared memory: T[col * NB + row] (upper triangular).
__global__ void __launch_bounds__(NT, 2) householder_qr_kernel(const QRDesc* __restrict__ descs, int csize, int* flags) {
  extern __shared__ double sm[];
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  const QRDesc D = descs[blockIdx.x / csize];
  const int m = D.m, n = D.n;
  if (m <= 0 || n <= 0) return;
  const int K = min(m, n);
  double* T = sm;                    // NB*NB
  double* tau = T + NB * NB;         // NB
  double* red = tau + NB;            // NW
  double* G = red + NW;              // NB*NB  (V^T V)
  double* P = G + NB * NB;           // panel, (mp_ld x NB)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double* A = D.A;
  const int lda = D.lda;
  bool nonfinite = false;

  for (int j0 = 0; j0 < K; j0 += NB) {
    const int jb = min(NB, K - j0);
    const int mp = m - j0;
    const int mp_ld = mp;
    // 1. load panel
    nonfinite |= copy_cols(P, mp_ld, A + (long long)j0 * lda + j0, lda, mp, jb);
    __syncthreads();
    // 2. factor panel
    for (int jj = 0; jj < jb; ++jj) {
      double s = 0.0;
      for (int r = jj + 1 + tid; r < mp; r += NT) { const double x = P[jj * mp_ld + r]; s = fma(x, x, s); }
      s = block_sum(s, red);
      const double alpha = P[jj * mp_ld + jj];
      double beta, t, scal;
      if (s == 0.0) { t = 0.0; beta = alpha; scal = 0.0; }
      else {
        beta = -copysign(sqrt(fma(alpha, alpha, s)), alpha);
        t = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      __syncthreads();
      if (s != 0.0)
        for (int r = jj + 1 + tid; r < mp; r += NT) P[jj * mp_ld + r] *= scal;
      if (tid == 0) { P[jj * mp_ld + jj] = beta; tau[jj] = t; }
      __syncthreads();
      // apply H_jj to the remaining panel columns (one warp per column)
      for (int c = jj + 1 + warp; c < jb; c += NW) {
        double w = 0.0;
        for (int r = jj + lane; r < mp; r += 32) {
          const double v = (r == jj) ? 1.0 : P[jj * mp_ld + r];
          w = fma(v, P[c * mp_ld + r], w);
        }
        w = warp_sum(w) * t;
        for (int r = jj + lane; r < mp; r += 32) {
          const double v = (r == jj) ? 1.0 : P[jj * mp_ld + r];
          P[c * mp_ld + r] -= w * v;
        }
      }
      __syncthreads();
    }
    // 3. T factor (dlarft, forward columnwise): G = V^T V, then T
    for (int pidx = warp; pidx < jb * jb; pidx += NW) {
      const int i = pidx / jb, l = pidx - i * jb;     // G[l][i] for l < i
      if (l < i) {
        double g = 0.0;
        for (int r = i + lane; r < mp; r += 32) {
          const double vi = (r == i) ? 1.0 : P[i * mp_ld + r];
          const double vl = P[l * mp_ld + r];          // r >= i > l
          g = fma(vl, vi, g);
        }
        g = warp_sum(g);
        if (lane == 0) G[i * NB + l] = g;
      }
    }
    __syncthreads();
    if (tid == 0) {
      for (int i = 0; i < NB; ++i)
        for (int l = 0; l < NB; ++l) T[i * NB + l] = 0.0;
      for (int i = 0; i < jb; ++i) {
        T[i * NB + i] = tau[i];
        // T[0:i, i] = -tau_i * T[0:i, 0:i] * G[0:i, i]
        for (int r = 0; r < i; ++r) {
          double a = 0.0;
          for (int l = r; l < i; ++l) a = fma(T[l * NB + r], G[i * NB + l], a);
          T[i * NB + r] = -tau[i] * a;
        }
      }
    }
    __syncthreads();
    // 4. trailing update with H^T = I - V T^T V^T (this CTA's column pairs)
    if (j0 + jb < n) apply_block_reflector(A, lda, j0, m, j0 + jb, n, P, mp_ld, jb, T, true, crank, csize);
    // 5. CTA 0 writes back the panel and keeps T
    if (crank == 0) {
      copy_cols(A + (long long)j0 * lda + j0, lda, P, mp_ld, mp, jb);
      if (D.Tws)
        for (int e = tid; e < NB * NB; e += NT) D.Tws[(j0 / NB) * NB * NB + e] = T[e];
    }
    cluster.sync();   // trailing columns and the panel visible to every CTA
  }
  if (nonfinite && crank == 0 && threadIdx.x == 0) atomicOr(flags, DFLAG_NONFINITE);

  // R = upper triangle of A[0:K, 0:n]
  if (D.R) {
    for (int j = (int)(threadIdx.x >> 5) + NW * crank; j < n; j += NW * csize)
      for (int i = (int)(threadIdx.x & 31); i < K; i += 32)
        D.R[(long long)j * D.ldr + i] = (i <= j) ? A[(long long)j * lda + i] : 0.0;
  }
  if (!D.Q) return;
  // Q = H_1 ... H_K [I; 0], accumulated backwards panel by panel.  Each CTA initialises
  // and updates only its own column pairs, so the panels need no barrier between them.
  for (int c = 0; c < K; ++c) {
    if (((c >> 1) % csize) != crank) continue;
    for (int i = tid; i < m; i += NT) D.Q[(long long)c * D.ldq + i] = (i == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int npan = (K + NB - 1) / NB;
  for (int p = npan - 1; p >= 0; --p) {
    const int j0 = p * NB, jb = min(NB, K - j0), mp = m - j0, mp_ld = mp;
    copy_cols(P, mp_ld, A + (long long)j0 * lda + j0, lda, mp, jb);
    for (int e = tid; e < NB * NB; e += NT) T[e] = D.Tws[p * NB * NB + e];
    __syncthreads();
    apply_block_reflector(D.Q, D.ldq, j0, m, j0, K, P, mp_ld, jb, T, false, crank, csize);
    __syncthreads();
  }
}

void launch_qr(const QRDesc* d_descs, int count, int max_m, cudaStream_t s, int* d_flags) {
  if (count <= 0) return;
  TTC_REQUIRE(max_m <= QR_MAX_M, TTC_EDIM, "qr: row count exceeds the supported maximum (1536)");
  const size_t smem = sizeof(double) * (NB * NB * 2 + NB + NW + (size_t)max_m * NB);
  static int attr_dev = -1;
  static int nsm = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    TTC_CUDA(cudaFuncSetAttribute(householder_qr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * (NB * NB * 2 + NB + NW + (size_t)QR_MAX_M * NB))));
    TTC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    attr_dev = dev;
  }
  // CTAs per problem: fill the resident-CTA slots of the GPU, at most 8 (portable cluster)
  int per_sm = 1;
  TTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, householder_qr_kernel, NT, smem));
  const int slots = nsm * std::max(1, per_sm);
  int c = std::min(8, std::max(1, slots / count));
  int csize = 1;
  while (csize * 2 <= c) csize *= 2;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(count * csize));
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)csize;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  TTC_CUDA(cudaLaunchKernelEx(&cfg, householder_qr_kernel, d_descs, csize, d_flags));
  TTC_CHECK_LAUNCH();
}

}  // namespace ttc
