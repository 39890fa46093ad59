// Batched one-sided (Hestenes) Jacobi SVD, FP64, one thread-block cluster per problem.
//
// Replaces the LAPACK gesdd/gesvd call of the truncated-SVD sweep
// (src/tt_rounding.jl:191-195, :235-239).  The sweep driver first QR-factors the
// unfolding, so the Jacobi input is a small square factor (one-sided Jacobi preconditioned
// by QR converges in few sweeps and keeps singular values accurate to O(eps * ||X||), the
// backward-error level of LAPACK).
//
// Parallel block ordering.  Columns are split into nblk blocks of bw columns.  One sweep =
// (a) the pairs inside every block, then (b) nblk'-1 rounds of the circle method over the
// blocks (nblk' = nblk rounded up to even): in a round the block pairs are disjoint, so the
// C CTAs of the cluster take them in turn, each streaming its two blocks from global memory
// (L2-resident) into shared memory, rotating all b x b cross pairs and writing them back.
// Rounds are separated by cluster barriers (barrier.cluster with release/acquire semantics,
// which orders the global-memory writes of one CTA before the reads of the next round);
// the "any rotation" flag of a sweep is OR-reduced into CTA 0's shared memory through
// distributed shared memory.  Control flow is identical in every CTA of a cluster, so
// every CTA reaches every barrier.
//
// Cross phase: each warp keeps its OWNT columns of the first block in registers, and only
// the partner column of the second block moves through shared memory; the OWNT rotations
// of a warp are independent and interleaved for instruction-level parallelism.
//
// Rotation: with alpha = ||x||^2, beta = ||y||^2, gamma = x.y, rotate when
// gamma^2 > tol^2 alpha beta; with d = beta - alpha and h = sqrt(d^2 + 4 gamma^2) the angle of
// modulus <= pi/4 has cos 2theta = |d|/h, sin 2theta = sign(d) 2 gamma / h, so
// c = sqrt((1 + cos 2theta)/2), s = sin 2theta / (2c) -- the rotation of Rutishauser's
// t = sign(d) 2 gamma / (|d| + h), computed with two reciprocal square roots and no division.
//
// Inert columns: a column whose squared norm is at most the numerical-zero threshold is never
// rotated (see make_rot), so its norm never changes.  Such columns (for example the
// (rank-deficient) trailing columns of an oversampled randomized-rounding factor) are left
// out of the sweeps: every CTA builds the same list of active columns and the blocks are
// gathered from it.
// alpha, beta, gamma are scaled by a power of two that brings ||X||_F^2 into [1/4, 1], so
// the squares cannot overflow or underflow (the rotation is scale invariant).
#include <cooperative_groups.h>

#include <algorithm>

#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace ttc {
namespace {
constexpr int NT = 256;
constexpr int NW = NT / 32;

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

struct Rot { double c, s; bool apply; };

// Parameters shared by all rotations of one problem.
struct RotCfg {
  double sc;     // power-of-two scale applied to alpha, beta, gamma
  double tol2;   // tol^2
  double zthr;   // scaled squared norm below which a column is numerically zero
};

// Columns whose squared norm is <= zthr (= (tol * ||A||_F)^2) are numerically zero: they are
// left alone, as in LAPACK's dgesvj.  Without this rule a rank-deficient matrix (more columns
// than the dimension of its column space) keeps rotating noise columns that cannot all be
// mutually orthogonal, and the iteration never stops.
__device__ __forceinline__ Rot make_rot(double alpha, double beta, double gamma, const RotCfg& q) {
  Rot r{1.0, 0.0, false};
  alpha *= q.sc; beta *= q.sc; gamma *= q.sc;
  if (alpha <= q.zthr || beta <= q.zthr) return r;
  const double g2 = gamma * gamma;
  if (!(g2 > q.tol2 * alpha * beta)) return r;
  const double d = beta - alpha;
  const double rh = rsqrt(fma(d, d, 4.0 * g2));
  const double c2 = fma(0.5 * fabs(d), rh, 0.5);
  const double rc = rsqrt(c2);
  r.c = c2 * rc;
  r.s = copysign(1.0, d) * gamma * rh * rc;
  r.apply = true;
  return r;
}

// Rotate columns x, y (both in shared memory, m rows) with one warp.  W columns (n rows,
// shared) follow along.  Returns whether a rotation was applied.
__device__ bool rotate_smem(double* x, double* y, int m, double* wx, double* wy, int n, const RotCfg& q) {
  const int lane = threadIdx.x & 31;
  double a = 0.0, b = 0.0, g = 0.0;
  for (int r = lane; r < m; r += 32) {
    const double u = x[r], v = y[r];
    a = fma(u, u, a); b = fma(v, v, b); g = fma(u, v, g);
  }
  a = warp_sum(a); b = warp_sum(b); g = warp_sum(g);
  const Rot R = make_rot(a, b, g, q);
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
  return true;
}

// Cross rotations between block I (in S0, cI columns) and block J (in S1, cJ columns), both
// of width bw = NW * OWNT.  Warp w owns the columns a = w + NW*o of block I in registers; in
// step s it rotates a against b = (a + s) mod bw of block J.  Requires m <= 32 * RPLT.
template <int OWNT, int RPLT>
__device__ __forceinline__ bool cross_regs(double* S0, double* S1, int m, int ms, int cI, int cJ, const RotCfg& q) {
  constexpr int bw = NW * OWNT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double xr[OWNT][RPLT];
#pragma unroll
  for (int o = 0; o < OWNT; ++o) {
    const int a = warp + NW * o;
#pragma unroll
    for (int t = 0; t < RPLT; ++t) {
      const int r = lane + 32 * t;
      xr[o][t] = (a < cI && r < m) ? S0[a * ms + r] : 0.0;
    }
  }
  bool any = false;
  for (int s = 0; s < bw; ++s) {
    double yr[OWNT][RPLT];
    double al[OWNT], be[OWNT], ga[OWNT];
    bool act[OWNT];
#pragma unroll
    for (int o = 0; o < OWNT; ++o) {
      const int a = warp + NW * o;
      const int b = (a + s) % bw;
      act[o] = (a < cI) && (b < cJ);
      const double* y = S1 + b * ms;
      al[o] = 0.0; be[o] = 0.0; ga[o] = 0.0;
#pragma unroll
      for (int t = 0; t < RPLT; ++t) {
        const int r = lane + 32 * t;
        yr[o][t] = (act[o] && r < m) ? y[r] : 0.0;
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
      const Rot R = act[o] ? make_rot(al[o], be[o], ga[o], q) : Rot{1.0, 0.0, false};
      if (R.apply) {
        any = true;
        const int a = warp + NW * o;
        double* y = S1 + ((a + s) % bw) * ms;
#pragma unroll
        for (int t = 0; t < RPLT; ++t) {
          const int r = lane + 32 * t;
          const double u = xr[o][t], v = yr[o][t];
          xr[o][t] = R.c * u - R.s * v;
          if (r < m) y[r] = fma(R.s, u, R.c * v);
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
      if (a < cI && r < m) S0[a * ms + r] = xr[o][t];
    }
  }
  return any;
}

// Cross rotations through shared memory only (W accumulation, or m beyond the register path).
__device__ bool cross_smem(double* S0, double* S1, double* W0, double* W1, int m, int ms, int n, int bw, int cI,
                           int cJ, const RotCfg& q) {
  const int warp = threadIdx.x >> 5;
  bool any = false;
  for (int s = 0; s < bw; ++s) {
    for (int a = warp; a < cI; a += NW) {
      const int b = (a + s) % bw;
      if (b < cJ)
        any |= rotate_smem(S0 + a * ms, S1 + b * ms, m, W0 ? W0 + a * n : nullptr, W1 ? W1 + b * n : nullptr, n, q);
    }
    __syncthreads();
  }
  return any;
}

// Copy `cols` columns of `rows` doubles between global memory and shared memory (or back):
// one warp per column, lanes over rows, four independent loads in flight per lane.
__device__ __forceinline__ void copy_cols(double* __restrict__ dst, long long dld, const double* __restrict__ src,
                                          long long sld, int rows, int cols) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c = warp; c < cols; c += NW) {
    const double* sc = src + (long long)c * sld;
    double* dc = dst + (long long)c * dld;
    for (int r0 = lane; r0 < rows; r0 += 128) {
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = (r0 + 32 * u < rows) ? sc[r0 + 32 * u] : 0.0;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (r0 + 32 * u < rows) dc[r0 + 32 * u] = v[u];
    }
  }
}

// One column of `rows` doubles copied by one warp (four loads in flight per lane).
__device__ __forceinline__ void copy_col_warp(double* __restrict__ dc, const double* __restrict__ sc, int rows) {
  const int lane = threadIdx.x & 31;
  for (int r0 = lane; r0 < rows; r0 += 128) {
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = (r0 + 32 * u < rows) ? sc[r0 + 32 * u] : 0.0;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (r0 + 32 * u < rows) dc[r0 + 32 * u] = v[u];
  }
}

// Gather the columns idx[0..cols) of a global matrix into packed shared-memory columns, or
// scatter them back; one warp per column.
__device__ __forceinline__ void gather_cols(double* __restrict__ dst, int dld, const double* __restrict__ src,
                                            long long ld, const int* idx, int rows, int cols) {
  for (int c = threadIdx.x >> 5; c < cols; c += NW) copy_col_warp(dst + (long long)c * dld, src + (long long)idx[c] * ld, rows);
}
__device__ __forceinline__ void scatter_cols(double* __restrict__ dst, long long ld, const double* __restrict__ src,
                                             int sld, const int* idx, int rows, int cols) {
  for (int c = threadIdx.x >> 5; c < cols; c += NW) copy_col_warp(dst + (long long)idx[c] * ld, src + (long long)c * sld, rows);
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Screening of a block pair in the later sweeps: whether any column pair (a of block I, b of
// block J; a < b inside one block) would be rotated.  The 16 x 16 Gram block S0^T S1 is formed
// on the FP64 tensor cores (mma.sync m8n8k4; warp w: tile w mod 4, half w / 4 of the rows) and
// tested with the column norms exactly as make_rot tests a pair.  A pair that passes needs no
// rotation, so its blocks are left as they are.  bw == 16; every thread gets the same answer.
__device__ bool screen_pair(const double* S0, const double* S1, int m, int ms, int cI, int cJ, bool same,
                            const RotCfg& q, double* scr) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, qr = lane >> 2, qc = lane & 3;
  double* nrm = scr;            // 32 column norms^2
  double* part = scr + 32;      // 4 tiles x 64 partial sums of the upper row half
  for (int c = warp; c < 32; c += NW) {
    const bool ok = (c < 16) ? (c < cI) : (c - 16 < cJ);
    const double* col = (c < 16) ? S0 + c * ms : S1 + (c - 16) * ms;
    double a = 0.0;
    if (ok)
      for (int r = lane; r < m; r += 32) a = fma(col[r], col[r], a);
    a = warp_sum(a);
    if (lane == 0) nrm[c] = a;
  }
  const int t = warp & 3, ti = t >> 1, tj = t & 1, h = warp >> 2;
  const int kh = ((m + 7) >> 3) << 2;
  const int kbeg = h ? kh : 0, kend = h ? m : (kh < m ? kh : m);
  const int ca = 8 * ti + qr, cb = 8 * tj + qr;
  double ga0 = 0.0, ga1 = 0.0, gb0 = 0.0, gb1 = 0.0;   // two accumulator chains
  for (int k0 = kbeg; k0 < kend; k0 += 8) {
    const int k = k0 + qc, k2 = k0 + 4 + qc;
    const double a = (k < kend && ca < cI) ? S0[ca * ms + k] : 0.0;
    const double b = (k < kend && cb < cJ) ? S1[cb * ms + k] : 0.0;
    const double a2 = (k2 < kend && ca < cI) ? S0[ca * ms + k2] : 0.0;
    const double b2 = (k2 < kend && cb < cJ) ? S1[cb * ms + k2] : 0.0;
    dmma(ga0, ga1, a, b);
    dmma(gb0, gb1, a2, b2);
  }
  double g0 = ga0 + gb0, g1 = ga1 + gb1;
  if (h == 1) { part[t * 64 + 2 * lane] = g0; part[t * 64 + 2 * lane + 1] = g1; }
  __syncthreads();
  int need = 0;
  if (h == 0) {
    g0 += part[t * 64 + 2 * lane];
    g1 += part[t * 64 + 2 * lane + 1];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int a = 8 * ti + qr, b = 8 * tj + 2 * qc + e;
      if (a < cI && b < cJ && (!same || a < b)) {
        const double al = nrm[a] * q.sc, be = nrm[16 + b] * q.sc, ga = (e ? g1 : g0) * q.sc;
        if (al > q.zthr && be > q.zthr && ga * ga > q.tol2 * al * be) need = 1;
      }
    }
  }
  return __syncthreads_or(need) != 0;
}

// Column position in the circle-method round robin over an even count `ne` of players.
__device__ __forceinline__ int rr_player(int pos, int round, int ne) {
  if (pos == 0) return 0;
  return ((pos - 1 + round) % (ne - 1)) + 1;
}

// Register-path dispatch on the rows per lane (bw = 16: two own columns per warp), up to
// RMAX rows per lane.
template <int RMAX>
__device__ bool cross_dispatch(double* S0, double* S1, int m, int ms, int cI, int cJ, const RotCfg& q) {
  const int rpl = (m + 31) / 32;
  if (rpl <= 2) return cross_regs<2, 2>(S0, S1, m, ms, cI, cJ, q);
  if (rpl <= 4) return cross_regs<2, 4>(S0, S1, m, ms, cI, cJ, q);
  if (RMAX <= 8 || rpl <= 8) return cross_regs<2, (RMAX < 8 ? RMAX : 8)>(S0, S1, m, ms, cI, cJ, q);
  return cross_regs<2, RMAX>(S0, S1, m, ms, cI, cJ, q);
}
}  // namespace

// Column stride of the shared blocks: rows rounded up to 4 mod 16 doubles, so the tensor-core
// fragment loads of the screening Gram (4 columns x 4 rows per half warp) hit distinct banks.
__host__ __device__ __forceinline__ int smem_stride(int m) { return m + ((4 - m) & 15); }

// Doubles of the dynamic shared memory before the active-column list: two blocks of bw
// columns of stride ms (and their W columns), at least n doubles (column norms, singular values).
__host__ __device__ __forceinline__ size_t dyn_doubles(int bw, int ms, int n, bool accw) {
  const size_t blocks = 2 * (size_t)bw * (size_t)(ms + (accw ? n : 0));
  return blocks > (size_t)n ? blocks : (size_t)n;
}

// grid = count * csize CTAs, clusters of csize CTAs (one cluster per problem).  RMAX bounds
// the register rows per lane of the cross phase (m <= 32 RMAX); RMAX = 8 keeps the kernel
// within 128 registers so that two CTAs share an SM.
template <int RMAX>
__global__ void __launch_bounds__(NT, RMAX <= 8 ? 2 : 1)
    jacobi_svd_kernel(const JacobiDesc* __restrict__ descs, const int* __restrict__ order, int bw, int csize,
                      int* flags, int max_sweeps) {
  extern __shared__ double sm[];
  __shared__ int s_any, s_nact;
  __shared__ double s_red[NW];
  __shared__ double s_scr[32 + 4 * 64];
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  const int prob = (int)(blockIdx.x / csize);
  const JacobiDesc D = descs[order ? order[prob] : prob];
  if (D.m <= 0 || D.n <= 0) return;             // uniform across the cluster
  // rows beyond the device bound are zero and stay zero under the rotations (at least one row
  // is kept so that an all-zero problem still reports its zero singular values)
  const int m = max(1, dev_bound(D.m, D.m_dev, D.m_mult)), n = D.n;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool accw = (D.W != nullptr);
  const int ms = smem_stride(m);                 // column stride of the shared blocks
  double* S0 = sm;
  double* S1 = sm + (size_t)bw * ms;
  double* W0 = S1 + (size_t)bw * ms;
  double* W1 = W0 + (accw ? (size_t)bw * n : 0);
  const bool use_regs = !accw && bw == 16 && m <= 32 * RMAX;

  if (accw) {  // W = I (columns split over the cluster)
    for (long long e = tid + (long long)crank * NT; e < (long long)n * n; e += (long long)NT * csize) {
      const int j = (int)(e / n), i = (int)(e - (long long)j * n);
      D.W[(long long)j * D.ldw + i] = (i == j) ? 1.0 : 0.0;
    }
  }
  // column norms (into sm, free until the first block load) and ||X||_F^2, which the
  // rotations leave invariant: scale and numerical-zero threshold
  int* act = reinterpret_cast<int*>(sm + dyn_doubles(bw, ms, n, accw));   // active columns
  {
    double a = 0.0;
    for (int j = warp; j < n; j += NW) {
      const double* xc = D.X + (long long)j * D.ldx;
      double cj = 0.0;
      for (int i = lane; i < m; i += 32) cj = fma(xc[i], xc[i], cj);
      cj = warp_sum(cj);
      if (lane == 0) sm[j] = cj;
      a += cj;
    }
    if (lane == 0) s_red[warp] = a;
  }
  if (tid == 0) s_any = 0;
  __syncthreads();
  double fro2 = 0.0;
#pragma unroll
  for (int i = 0; i < NW; ++i) fro2 += s_red[i];
  RotCfg q;
  {
    const double tol = jac_tol(D.m);   // the stored row count, whatever the device bound
    int e2 = 0;
    if (fro2 > 0.0 && isfinite(fro2)) { frexp(fro2, &e2); e2 = (e2 + 1) & ~1; }   // even exponent
    q.sc = (fro2 > 0.0 && isfinite(fro2)) ? ldexp(1.0, -e2) : 1.0;
    q.tol2 = tol * tol;
    q.zthr = q.tol2 * fro2 * q.sc;
  }
  if (warp == 0) {   // the same list in every CTA of the cluster
    int cnt = 0;
    for (int c0 = 0; c0 < n; c0 += 32) {
      const int c = c0 + lane;
      const bool on = (c < n) && (sm[c] * q.sc > q.zthr);
      const unsigned b = __ballot_sync(0xffffffffu, on);
      if (on) act[cnt + __popc(b & ((1u << lane) - 1u))] = c;
      cnt += __popc(b);
    }
    if (lane == 0) s_nact = cnt;
  }
  __syncthreads();
  const int na = s_nact;
  const int nblk = (na + bw - 1) / bw;
  const int ne = nblk + (nblk & 1);

  auto load_block = [&](int blk, double* S, double* Wd) {
    const int c0 = blk * bw, cn = min(bw, na - c0);
    gather_cols(S, ms, D.X, D.ldx, act + c0, m, cn);
    if (accw) gather_cols(Wd, n, D.W, D.ldw, act + c0, n, cn);
  };
  auto store_block = [&](int blk, const double* S, const double* Wd) {
    const int c0 = blk * bw, cn = min(bw, na - c0);
    scatter_cols(D.X, D.ldx, S, ms, act + c0, m, cn);
    if (accw) scatter_cols(D.W, D.ldw, Wd, n, act + c0, n, cn);
  };
  cluster.sync();   // W = I visible to every CTA

  int* any0 = cluster.map_shared_rank(&s_any, 0);
  bool converged = false;
  int sweep = 0;
  for (; sweep < max_sweeps && !converged; ++sweep) {
    bool any = false;
    const bool screen = (sweep >= 3) && (bw == 16);   // late sweeps: skip block pairs that need no rotation
    // (a) pairs inside each block; blocks dealt to the CTAs of the cluster
    for (int blk = crank; blk < nblk; blk += csize) {
      const int cI = min(bw, na - blk * bw);
      load_block(blk, S0, W0);
      __syncthreads();
      if (screen && !screen_pair(S0, S0, m, ms, cI, cI, true, q, s_scr)) continue;   // block unchanged
      const int nee = cI + (cI & 1);
      for (int rd = 0; rd < nee - 1; ++rd) {
        for (int p = warp; p < nee / 2; p += NW) {
          const int i = rr_player(p, rd, nee), j = rr_player(nee - 1 - p, rd, nee);
          if (i < cI && j < cI)
            any |= rotate_smem(S0 + i * ms, S0 + j * ms, m, accw ? W0 + i * n : nullptr, accw ? W0 + j * n : nullptr,
                               n, q);
        }
        __syncthreads();
      }
      store_block(blk, S0, W0);
      __syncthreads();
    }
    cluster.sync();
    // (b) cross pairs: circle method over the blocks, disjoint pairs per round
    for (int rd = 0; rd < ne - 1; ++rd) {
      for (int p = crank; p < ne / 2; p += csize) {
        const int bi = rr_player(p, rd, ne), bj = rr_player(ne - 1 - p, rd, ne);
        if (bi >= nblk || bj >= nblk) continue;
        const int cI = min(bw, na - bi * bw), cJ = min(bw, na - bj * bw);
        load_block(bi, S0, W0);
        load_block(bj, S1, W1);
        __syncthreads();
        if (screen && !screen_pair(S0, S1, m, ms, cI, cJ, false, q, s_scr)) continue;   // blocks unchanged
        if (use_regs) any |= cross_dispatch<RMAX>(S0, S1, m, ms, cI, cJ, q);
        else any |= cross_smem(S0, S1, accw ? W0 : nullptr, accw ? W1 : nullptr, m, ms, n, bw, cI, cJ, q);
        __syncthreads();
        store_block(bi, S0, W0);
        store_block(bj, S1, W1);
        __syncthreads();
      }
      cluster.sync();
    }
    // OR of the per-CTA flags into CTA 0; every CTA reads it; CTA 0 clears it for the next sweep
    if (any && lane == 0) atomicOr(any0, 1);
    cluster.sync();
    converged = (*any0 == 0);
    cluster.sync();
    if (crank == 0 && tid == 0) s_any = 0;
  }
  if (crank != 0) return;   // no distributed-shared-memory access follows
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
  // the keys order NaN (a non-finite input, flagged by the QR) below every singular value, so
  // that the ranks form a permutation whatever the values and perm stays a valid index list
  for (int c = tid; c < n; c += NT) {
    const double v = (sig[c] == sig[c]) ? sig[c] : -1.0;
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double w = (sig[j] == sig[j]) ? sig[j] : -1.0;
      rank += (w > v) || (w == v && j < c);
    }
    D.perm[rank] = c;
  }
}

// Small problems (m, n <= 32, no W): one warp per problem, lane j holding column j in
// registers.  A round of the circle method pairs the columns; the two lanes of a pair exchange
// their columns by shuffles and both compute alpha, beta, gamma with the same operations in the
// same order (so both find the same rotation bit for bit), each updating its own column.  No
// barrier is needed, which is what bounds the cluster kernel on these sizes.  Same rotation, zero
// threshold and convergence rule (a sweep without rotations) as the cluster kernel.
__global__ void __launch_bounds__(128) jacobi_small_kernel(const JacobiDesc* __restrict__ descs, int count, int* flags,
                                                          int max_sweeps) {
  const int lane = threadIdx.x & 31;
  const int prob = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (prob >= count) return;                        // uniform within the warp
  const JacobiDesc D = descs[prob];
  if (D.m <= 0 || D.n <= 0) return;
  const int m = max(1, dev_bound(D.m, D.m_dev, D.m_mult)), n = D.n;
  double x[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) x[i] = (lane < n && i < m) ? D.X[(long long)lane * D.ldx + i] : 0.0;
  double nrm = 0.0;
#pragma unroll
  for (int i = 0; i < 32; ++i) nrm = fma(x[i], x[i], nrm);
  const double fro2 = warp_sum(nrm);
  RotCfg q;
  {
    const double tol = jac_tol(D.m);
    int e2 = 0;
    if (fro2 > 0.0 && isfinite(fro2)) { frexp(fro2, &e2); e2 = (e2 + 1) & ~1; }
    q.sc = (fro2 > 0.0 && isfinite(fro2)) ? ldexp(1.0, -e2) : 1.0;
    q.tol2 = tol * tol;
    q.zthr = q.tol2 * fro2 * q.sc;
  }
  const int ne = n + (n & 1);
  bool converged = false;
  int sweep = 0;
  for (; sweep < max_sweeps && !converged; ++sweep) {
    bool any = false;
    for (int rd = 0; rd < ne - 1; ++rd) {
      // this lane's position in the round, and its partner column
      int pos = 0;
      if (lane != 0) pos = ((lane - 1 - rd) % (ne - 1) + (ne - 1)) % (ne - 1) + 1;
      const int partner = rr_player(ne - 1 - pos, rd, ne);
      const bool act = lane < n && partner < n;
      const int src = act ? partner : lane;
      const bool low = lane < partner;
      double a = 0.0, b = 0.0, g = 0.0;            // alpha (low column), beta (high), gamma
      double y[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        y[i] = __shfl_sync(0xffffffffu, x[i], src);
        const double lo = low ? x[i] : y[i], hi = low ? y[i] : x[i];
        a = fma(lo, lo, a);
        b = fma(hi, hi, b);
        g = fma(lo, hi, g);
      }
      const Rot R = act ? make_rot(a, b, g, q) : Rot{1.0, 0.0, false};
      if (R.apply) {
        any = true;
#pragma unroll
        for (int i = 0; i < 32; ++i)
          x[i] = low ? (R.c * x[i] - R.s * y[i]) : fma(R.s, y[i], R.c * x[i]);
      }
    }
    converged = !__any_sync(0xffffffffu, any);
  }
  if (!converged && lane == 0) atomicOr(flags, DFLAG_JACOBI_NOCONV);
  if (D.info && lane == 0) *D.info = converged ? sweep : -sweep;
  double c2 = 0.0;
#pragma unroll
  for (int i = 0; i < 32; ++i) c2 = fma(x[i], x[i], c2);
  const double sg = sqrt(c2);
  if (lane < n) {
#pragma unroll
    for (int i = 0; i < 32; ++i)
      if (i < m) D.X[(long long)lane * D.ldx + i] = x[i];
    D.sigma[lane] = sg;
  }
  // ranking by decreasing value (NaN last, ties by index), as in the cluster kernel
  const double key = (lane < n) ? ((sg == sg) ? sg : -1.0) : -2.0;
  int rank = 0;
  for (int j = 0; j < n; ++j) {
    const double w = __shfl_sync(0xffffffffu, key, j);
    rank += (w > key) || (w == key && j < lane);
  }
  if (lane < n) D.perm[rank] = lane;
}

// Problem order of a launch: by decreasing size m x n^2, m the rows left by the device bound and
// n the columns (at most m when bounded: the bounded factor is square), ties by index.
__global__ void jacobi_order_kernel(const JacobiDesc* __restrict__ descs, int count, int* __restrict__ order) {
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    auto key = [&](int j) {
      const JacobiDesc& d = descs[j];
      const double m = dev_bound(d.m, d.m_dev, d.m_mult);
      const double n = d.m_dev ? fmin((double)d.n, m) : (double)d.n;
      return m * n * n;
    };
    const double ki = key(i);
    int rank = 0;
    for (int j = 0; j < count; ++j) {
      const double kj = key(j);
      rank += (kj > ki) || (kj == ki && j < i);
    }
    order[rank] = i;
  }
}


// Block width and dynamic shared memory of a launch: dyn_doubles(bw, ...) doubles and the
// active-column list (max_n ints).
static int jacobi_bw(int max_m, int max_n, bool accw, size_t* smem_out) {
  int bw = 16;
  auto need = [&](int b) {
    return sizeof(double) * dyn_doubles(b, smem_stride(max_m), max_n, accw) + sizeof(int) * (size_t)max_n;
  };
  while (bw > 1 && need(bw) > 200 * 1024) bw >>= 1;
  *smem_out = need(bw);
  return bw;
}

// Cluster size of an ordered launch (measured on the 64-TT rounding: 8 for the two-CTA-per-SM
// instance, 4 for the one-CTA-per-SM instance; 8 there runs 3.5 waves and loses).
template <int RMAX>
constexpr int kOrderedCsize = RMAX <= 8 ? 8 : 4;
template <int RMAX>
static int jacobi_cluster_size(int count, int max_n, int bw, size_t smem, bool ordered) {
  // CTAs per problem: fill the SMs (resident CTAs per SM from registers and shared memory),
  // at most 8 (portable cluster size) and at most the disjoint block pairs of a round.  With
  // the problems ordered largest first the grid may exceed the resident slots (the clusters
  // that start later take the smaller problems): then at least kOrderedCsize<RMAX>.
  int per_sm = 1;
  TTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_svd_kernel<RMAX>, NT, smem));
  per_sm = std::max(1, per_sm);
  const int slots = current_sm_count() * per_sm;
  const int pairs = std::max(1, ((max_n + bw - 1) / bw + 1) / 2);
  int c = std::max(1, slots / std::max(1, count));
  if (ordered) c = std::max(c, kOrderedCsize<RMAX>);
  c = std::min(c, std::min(8, pairs));
  int p2 = 1;
  while (p2 * 2 <= c) p2 *= 2;
  return p2;
}

template <int RMAX>
static void launch_jacobi_t(const JacobiDesc* d_descs, int count, int max_n, int bw, size_t smem, cudaStream_t s,
                            int* d_flags, int* order, int max_sweeps) {
  static PerDeviceOnce attr_once;
  int dev = 0;
  TTC_CUDA(cudaGetDevice(&dev));
  attr_once.run(dev, [] {
    TTC_CUDA(cudaFuncSetAttribute(jacobi_svd_kernel<RMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  });
  if (order) {
    jacobi_order_kernel<<<1, 512, 0, s>>>(d_descs, count, order);
    TTC_CHECK_LAUNCH();
  }
  const int csize = jacobi_cluster_size<RMAX>(count, max_n, bw, smem, order != nullptr);
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
  TTC_CUDA(cudaLaunchKernelEx(&cfg, jacobi_svd_kernel<RMAX>, d_descs, (const int*)order, bw, csize, d_flags,
                              max_sweeps));
  TTC_CHECK_LAUNCH();
}

void launch_jacobi(const JacobiDesc* d_descs, int count, int max_m, int max_n, bool accw, cudaStream_t s,
                   int* d_flags, int* order, int max_sweeps) {
  if (count <= 0) return;
  TTC_REQUIRE(max_sweeps >= 1, TTC_EARG, "jacobi: the sweep cap must be at least 1");
  size_t smem = 0;
  const int bw = jacobi_bw(max_m, max_n, accw, &smem);
  TTC_REQUIRE(smem <= 200 * 1024, TTC_EDIM, "jacobi: matrix too large for the shared-memory blocks");
  if (count > kJacobiOrderMax) order = nullptr;
  if (!accw && max_m <= 32 && max_n <= 32) {       // every problem fits one warp's registers
    jacobi_small_kernel<<<(unsigned)((count + 3) / 4), 128, 0, s>>>(d_descs, count, d_flags, max_sweeps);
    TTC_CHECK_LAUNCH();
    return;
  }
  if (max_m <= 256) launch_jacobi_t<8>(d_descs, count, max_n, bw, smem, s, d_flags, order, max_sweeps);
  else launch_jacobi_t<16>(d_descs, count, max_n, bw, smem, s, d_flags, order, max_sweeps);
}

}  // namespace ttc
