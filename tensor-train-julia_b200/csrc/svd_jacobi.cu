// Batched one-sided (Hestenes) Jacobi SVD, one CTA per problem, FP64.
//
// Replaces the LAPACK gesdd/gesvd call of the truncated-SVD sweep
// (src/tt_rounding.jl:191-195, :235-239).  The sweep driver first QR-factors the
// unfolding, so the Jacobi input is the small triangular factor R (one-sided Jacobi
// preconditioned by QR converges in few sweeps and keeps singular values accurate to
// O(eps * ||R||), the same backward-error level as LAPACK).
//
// Data movement: columns are split into blocks of bw (<= 32) columns.  A sweep keeps
// block I in shared memory, rotates all pairs inside it, then streams every later block
// J through a second shared-memory slot and rotates all (i in I, j in J) pairs.  During
// that cross phase each warp keeps its own columns of block I in registers and only the
// partner column of J moves through shared memory.  Every pair is visited once per sweep.
// A sweep without any rotation above tol * sqrt(alpha*beta) ends the iteration.
#include "kernels.cuh"

namespace ttc {
namespace {
constexpr int NT = 256;
constexpr int NW = NT / 32;
constexpr int BWMAX = 32;
constexpr int OWN = BWMAX / NW;     // columns of block I owned per warp (<= 4)
constexpr int RPL = 16;             // register rows per lane in the cross phase (m <= 512)
constexpr int MAX_SWEEPS = 40;
// Rotation threshold |a_i.a_j| > tol * ||a_i|| ||a_j|| with tol = max(m, 16) eps, the worst-case
// rounding error of an m-term FP64 dot product.  A threshold nearer the typical error
// (sqrt(m) eps) is crossed by noise alone on a few of the ~m^2/2 pairs of every sweep when m is
// a few hundred, and the iteration would never stop.
__device__ __forceinline__ double jac_tol(int m) { return (double)(m > 16 ? m : 16) * 2.220446049250313e-16; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

struct Rot { double c, s; bool apply; bool big; };

// Columns whose squared norm is <= zthr (= (tol * ||A||_F)^2) are numerically zero: they are
// left alone, as in LAPACK's dgesvj.  Without this rule a rank-deficient matrix (more columns
// than the dimension of its column space) keeps rotating noise columns that cannot all be
// mutually orthogonal, and the iteration never stops.
__device__ __forceinline__ Rot make_rot(double alpha, double beta, double gamma, double tol, double zthr) {
  Rot r{1.0, 0.0, false, false};
  if (alpha <= zthr || beta <= zthr) return r;
  const double ag = fabs(gamma);
  const double lim = tol * sqrt(alpha) * sqrt(beta);
  if (!(ag > lim)) return r;
  r.big = true;
  const double zeta = (beta - alpha) / (2.0 * gamma);
  double t;
  if (fabs(zeta) > 1e150) t = 0.5 / zeta;
  else t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(fma(zeta, zeta, 1.0)));
  r.c = 1.0 / sqrt(fma(t, t, 1.0));
  r.s = r.c * t;
  r.apply = true;
  return r;
}

// Rotate columns x, y (both in shared memory, m rows) with one warp.  Returns whether a
// rotation above the tolerance was applied.  W columns (n rows, shared) follow along.
__device__ bool rotate_smem(double* x, double* y, int m, double* wx, double* wy, int n, double zthr) {
  const int lane = threadIdx.x & 31;
  double a = 0.0, b = 0.0, g = 0.0;
  for (int r = lane; r < m; r += 32) {
    const double u = x[r], v = y[r];
    a = fma(u, u, a); b = fma(v, v, b); g = fma(u, v, g);
  }
  a = warp_sum(a); b = warp_sum(b); g = warp_sum(g);
  const Rot R = make_rot(a, b, g, jac_tol(m), zthr);
  if (!R.apply) return false;
  for (int r = lane; r < m; r += 32) {
    const double u = x[r], v = y[r];
    x[r] = R.c * u - R.s * v;
    y[r] = fma(R.s, u, R.c * v);
  }
  if (wx)
    for (int r = lane; r < n; r += 32) {
      const double u = wx[r], v = wy[r];
      wx[r] = R.c * u - R.s * v;
      wy[r] = fma(R.s, u, R.c * v);
    }
  return R.big;
}

// Cross rotations between block I (in S0, cI columns) and block J (in S1, cJ columns).
// Warp w owns the OWNT columns a = w + NW*o of block I in registers; in round s it rotates
// a against b = (a + s) mod bw of block J.  The OWNT rotations of a warp are independent, so
// their loads, dot products, shuffle reductions and updates are interleaved to hide the
// latency chains (one rotation alone is latency bound).  Requires bw == NW*OWNT and
// m <= 32*RPLT.  Returns whether a rotation above the threshold happened.
template <int OWNT, int RPLT>
__device__ __forceinline__ int cross_regs(double* S0, double* S1, int m, int bw, int cI, int cJ, int warp, int lane,
                                          double zthr) {
  const int rpl = (m + 31) / 32;
  const double tol = jac_tol(m);
  double xr[OWNT][RPLT];
#pragma unroll
  for (int o = 0; o < OWNT; ++o) {
    const int a = warp + NW * o;
#pragma unroll
    for (int t = 0; t < RPLT; ++t) {
      const int r = lane + 32 * t;
      xr[o][t] = (a < cI && t < rpl && r < m) ? S0[a * m + r] : 0.0;
    }
  }
  int any = 0;
  for (int s = 0; s < bw; ++s) {
    double yr[OWNT][RPLT];
    double al[OWNT], be[OWNT], ga[OWNT];
    bool act[OWNT];
#pragma unroll
    for (int o = 0; o < OWNT; ++o) {
      const int a = warp + NW * o;
      const int b = (a + s) % bw;
      act[o] = (a < cI) && (b < cJ);
      const double* y = S1 + b * m;
      al[o] = 0.0; be[o] = 0.0; ga[o] = 0.0;
#pragma unroll
      for (int t = 0; t < RPLT; ++t) {
        const int r = lane + 32 * t;
        yr[o][t] = (act[o] && t < rpl && r < m) ? y[r] : 0.0;
      }
    }
#pragma unroll
    for (int t = 0; t < RPLT; ++t)
#pragma unroll
      for (int o = 0; o < OWNT; ++o) {
        al[o] = fma(xr[o][t], xr[o][t], al[o]);
        be[o] = fma(yr[o][t], yr[o][t], be[o]);
        ga[o] = fma(xr[o][t], yr[o][t], ga[o]);
      }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
      for (int o = 0; o < OWNT; ++o) {
        al[o] += __shfl_xor_sync(0xffffffffu, al[o], off);
        be[o] += __shfl_xor_sync(0xffffffffu, be[o], off);
        ga[o] += __shfl_xor_sync(0xffffffffu, ga[o], off);
      }
#pragma unroll
    for (int o = 0; o < OWNT; ++o) {
      const Rot R = act[o] ? make_rot(al[o], be[o], ga[o], tol, zthr) : Rot{1.0, 0.0, false, false};
      if (R.apply) {
        any |= R.big;
        const int a = warp + NW * o;
        double* y = S1 + ((a + s) % bw) * m;
#pragma unroll
        for (int t = 0; t < RPLT; ++t) {
          const int r = lane + 32 * t;
          const double u = xr[o][t], v = yr[o][t];
          xr[o][t] = R.c * u - R.s * v;
          if (t < rpl && r < m) y[r] = fma(R.s, u, R.c * v);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int o = 0; o < OWNT; ++o) {
    const int a = warp + NW * o;
#pragma unroll
    for (int t = 0; t < RPLT; ++t) {
      const int r = lane + 32 * t;
      if (a < cI && t < rpl && r < m) S0[a * m + r] = xr[o][t];
    }
  }
  return any;
}

// Column position in the circle-method round robin over an even count `ne` of players.
__device__ __forceinline__ int rr_player(int pos, int round, int ne) {
  if (pos == 0) return 0;
  return ((pos - 1 + round) % (ne - 1)) + 1;
}
}  // namespace

__global__ void __launch_bounds__(NT, 1) jacobi_svd_kernel(const JacobiDesc* __restrict__ descs, int smem_doubles,
                                                           int* flags) {
  extern __shared__ double sm[];
  __shared__ int s_rot;
  const JacobiDesc D = descs[blockIdx.x];
  const int m = D.m, n = D.n;
  if (m <= 0 || n <= 0) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool accw = (D.W != nullptr);
  // block width: largest power of two <= 32 whose two slots fit
  int bw = BWMAX;
  if (!accw && m > 256) bw = 16;     // register cross phase: 2 own columns x 16 rows per lane
  while (bw > 1 && 2LL * bw * (m + (accw ? n : 0)) > smem_doubles) bw >>= 1;
  const int nblk = (n + bw - 1) / bw;
  double* S0 = sm;
  double* S1 = sm + (size_t)bw * m;
  double* W0 = S1 + (size_t)bw * m;
  double* W1 = W0 + (accw ? (size_t)bw * n : 0);
  const bool use_regs = !accw && ((bw == 32 && m <= 256) || (bw == 16 && m <= 512));

  if (accw) {  // W = I
    for (long long e = tid; e < (long long)n * n; e += NT) {
      const int j = (int)(e / n), i = (int)(e - (long long)j * n);
      D.W[(long long)j * D.ldw + i] = (i == j) ? 1.0 : 0.0;
    }
  }
  // ||X||_F^2 (invariant under the rotations) -> numerical-zero threshold for columns
  __shared__ double s_red[NW];
  {
    double a = 0.0;
    for (long long e = tid; e < (long long)m * n; e += NT) {
      const int j = (int)(e / m), i = (int)(e - (long long)j * m);
      const double v = D.X[(long long)j * D.ldx + i];
      a = fma(v, v, a);
    }
    a = warp_sum(a);
    if (lane == 0) s_red[warp] = a;
  }
  __syncthreads();
  double fro2 = 0.0;
#pragma unroll
  for (int i = 0; i < NW; ++i) fro2 += s_red[i];
  const double zt = jac_tol(m);
  const double zthr = zt * zt * fro2;
  __syncthreads();

  auto load_block = [&](int blk, double* S, double* Wd) {
    const int c0 = blk * bw, cn = min(bw, n - c0);
    for (int e = tid; e < cn * m; e += NT) {
      const int c = e / m, r = e - c * m;
      S[c * m + r] = D.X[(long long)(c0 + c) * D.ldx + r];
    }
    if (accw)
      for (int e = tid; e < cn * n; e += NT) {
        const int c = e / n, r = e - c * n;
        Wd[c * n + r] = D.W[(long long)(c0 + c) * D.ldw + r];
      }
  };
  auto store_block = [&](int blk, const double* S, const double* Wd) {
    const int c0 = blk * bw, cn = min(bw, n - c0);
    for (int e = tid; e < cn * m; e += NT) {
      const int c = e / m, r = e - c * m;
      D.X[(long long)(c0 + c) * D.ldx + r] = S[c * m + r];
    }
    if (accw)
      for (int e = tid; e < cn * n; e += NT) {
        const int c = e / n, r = e - c * n;
        D.W[(long long)(c0 + c) * D.ldw + r] = Wd[c * n + r];
      }
  };

  bool converged = false;
  int sweep = 0;
  for (; sweep < MAX_SWEEPS && !converged; ++sweep) {
    if (tid == 0) s_rot = 0;
    __syncthreads();
    int any = 0;
    for (int I = 0; I < nblk; ++I) {
      const int cI = min(bw, n - I * bw);
      if (nblk > 1 || sweep == 0) { load_block(I, S0, W0); }
      __syncthreads();
      // intra-block pairs: circle method over an even number of players
      {
        const int ne = cI + (cI & 1);
        for (int rd = 0; rd < ne - 1; ++rd) {
          for (int p = warp; p < ne / 2; p += NW) {
            const int i = rr_player(p, rd, ne), j = rr_player(ne - 1 - p, rd, ne);
            if (i < cI && j < cI)
              any |= rotate_smem(S0 + i * m, S0 + j * m, m, accw ? W0 + i * n : nullptr,
                                 accw ? W0 + j * n : nullptr, n, zthr);
          }
          __syncthreads();
        }
      }
      // cross pairs with every later block
      for (int J = I + 1; J < nblk; ++J) {
        const int cJ = min(bw, n - J * bw);
        load_block(J, S1, W1);
        __syncthreads();
        if (use_regs) {
          if (bw == 32) any |= cross_regs<4, 8>(S0, S1, m, bw, cI, cJ, warp, lane, zthr);
          else any |= cross_regs<2, 16>(S0, S1, m, bw, cI, cJ, warp, lane, zthr);
        } else {
          for (int s = 0; s < bw; ++s) {
            for (int a = warp; a < cI; a += NW) {
              const int b = (a + s) % bw;
              if (b < cJ)
                any |= rotate_smem(S0 + a * m, S1 + b * m, m, accw ? W0 + a * n : nullptr,
                                   accw ? W1 + b * n : nullptr, n, zthr);
            }
            __syncthreads();
          }
        }
        __syncthreads();
        store_block(J, S1, W1);
        __syncthreads();
      }
      if (nblk > 1) store_block(I, S0, W0);
      __syncthreads();
    }
    if (any && lane == 0) atomicOr(&s_rot, 1);
    __syncthreads();
    converged = (s_rot == 0);
    __syncthreads();
  }
  if (nblk == 1) { store_block(0, S0, W0); __syncthreads(); }
  if (!converged && tid == 0) atomicOr(flags, DFLAG_JACOBI_NOCONV);
  if (D.info && tid == 0) *D.info = converged ? sweep : -sweep;

  // singular values = column norms; order by decreasing value (ties by index)
  double* sig = sm;   // reuse shared memory
  for (int c = warp; c < n; c += NW) {
    double a = 0.0;
    for (int r = lane; r < m; r += 32) { const double u = D.X[(long long)c * D.ldx + r]; a = fma(u, u, a); }
    a = warp_sum(a);
    if (lane == 0) { sig[c] = sqrt(a); D.sigma[c] = sqrt(a); }
  }
  __syncthreads();
  for (int c = tid; c < n; c += NT) {
    const double v = sig[c];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double w = sig[j];
      rank += (w > v) || (w == v && j < c);
    }
    D.perm[rank] = c;
  }
}

void launch_jacobi(const JacobiDesc* d_descs, int count, int max_m, int max_n, cudaStream_t s, int* d_flags) {
  if (count <= 0) return;
  (void)max_m; (void)max_n;
  const int smem_bytes = 200 * 1024;
  static bool attr_set = false;
  if (!attr_set) {
    TTC_CUDA(cudaFuncSetAttribute(jacobi_svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes));
    attr_set = true;
  }
  jacobi_svd_kernel<<<count, NT, smem_bytes, s>>>(d_descs, smem_bytes / (int)sizeof(double), d_flags);
  TTC_CHECK_LAUNCH();
}

}  // namespace ttc
