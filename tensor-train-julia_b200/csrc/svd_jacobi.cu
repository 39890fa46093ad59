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

struct Rot { double c, s, t; bool apply; };   // t = s / c (= s rsqrt(c^2): no division)

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
  Rot r{1.0, 0.0, 0.0, false};
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
  r.t = r.s * rc;
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

// Block variant for problems without W and with m <= 512 rows (the truncated-SVD sweeps).
//
// The cross steps of jacobi_svd_kernel rotate 256-row columns one pair at a time: every step
// streams a block through shared memory, reduces three dot products across the warp and waits at a
// barrier, and measured per step that is several thousand cycles, 70 % of the kernel.  Here a CTA
// takes its block pair (32 column slots: block I in slots 0-15, block J in 16-31) and
//   1. forms the 32 x 32 Gram matrix G = S^T S on the FP64 tensor cores (mma.sync m8n8k4);
//   2. runs the Jacobi rotations on G instead of on the columns (two-sided: G <- J^T G J, with the
//      rotations accumulated in V, V <- V J), 16 disjoint pairs per inner round and two barriers
//      per round, on 32-element rows instead of m-row columns;
//   3. applies V to the columns with the tensor cores again (S V, m x 32 x 32), writing the result
//      straight back to the problem's columns in global memory.
// Each rotation is the one jacobi_svd_kernel would take for the same three numbers (make_rot: the
// same threshold, zero rule and formulas), computed from G's entries: alpha = G_ii, beta = G_jj,
// gamma = G_ij.  The diagonal of a rotated pair is updated as alpha - t gamma and beta + t gamma
// (t = s / c) and gamma set to zero, as in the scalar recurrences; the other entries take the rotation
// on both sides.  An entry updated this way keeps an error of the order of eps sqrt(G_ii G_kk) (the
// rotation angle of a large and a small column is small in proportion), so the decisions have the
// relative accuracy of the column-based ones (Demmel and Veselic, SIAM J. Matrix Anal. Appl. 13,
// 1992).  A block pair is left untouched (not stored) when no pair of its Gram matrix passes the
// rotation test.
// Sweep structure: the circle method over the blocks as in jacobi_svd_kernel.  In round 0 every block
// meets its partner with all 496 slot pairs (a full inner sweep, which covers the pairs inside the
// blocks); in the later rounds only the 256 cross pairs (inner round s pairs slot p with
// 16 + (p + s) mod 16).  A sweep thus visits every column pair once, and it converges when no CTA of
// the cluster rotated anything during a whole sweep.
namespace {
constexpr int GLD = 36;          // leading dimension of G and V in shared memory (= 4 mod 16: no bank conflicts)

// Rotation of one pair in an inner round, split by who reads it: RotA (slots, cosine, sine; read by
// every role) and RotB (t = s / c and the pair's entries of G before the round; read by the threads
// that update the diagonal or compute the next round's rotations).
struct __align__(16) RotA {
  double c, s;
  int i, j, on, pad;
};
struct __align__(16) RotB {
  double t, gii, gjj, gij;
};

// Shared-memory doubles of a launch of jacobi_block_kernel: S (32 slots of stride ms), G, V and the
// column norms (n); the active-column list (n ints) follows.
__host__ __device__ __forceinline__ size_t block_dyn_doubles(int ms, int n) {
  return (size_t)32 * ms + 2 * 32 * GLD + (size_t)n;
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

// Pairing of inner round r: the circle method over the 32 slots (full) or the cross pairs
// (p, 16 + (p + r) mod 16).  Partner of slot x and the index of its pair.
__device__ __forceinline__ void inner_partner(int x, int r, bool full, int& y, int& pidx) {
  if (full) {
    const int pos = (x == 0) ? 0 : ((x - 1 - r) % 31 + 31) % 31 + 1;
    y = rr_player(31 - pos, r, 32);
    pidx = min(pos, 31 - pos);
  } else if (x < 16) {
    y = 16 + ((x + r) & 15);
    pidx = x;
  } else {
    pidx = (x - 16 - r) & 15;
    y = pidx;
  }
}

// make_rot without branches (the same operations; a pair that does not rotate gets c = 1, s = t = 0),
// for the inner rounds' critical path.
__device__ __forceinline__ Rot make_rot_nb(double alpha, double beta, double gamma, const RotCfg& q) {
  alpha *= q.sc; beta *= q.sc; gamma *= q.sc;
  const double g2 = gamma * gamma;
  const bool ap = (alpha > q.zthr) && (beta > q.zthr) && (g2 > q.tol2 * alpha * beta);
  const double d = beta - alpha;
  const double rh = rsqrt(fma(d, d, 4.0 * g2));
  const double c2 = fma(0.5 * fabs(d), rh, 0.5);
  const double rc = rsqrt(c2);
  const double s = copysign(1.0, d) * gamma * rh * rc;
  Rot r;
  r.c = ap ? c2 * rc : 1.0;
  r.s = ap ? s : 0.0;
  r.t = ap ? s * rc : 0.0;
  r.apply = ap;
  return r;
}

// Rotation of slots x, y from their entries of G, written with i = min(x, y), j = max(x, y); returns
// whether it rotates.
__device__ __forceinline__ bool set_pair(RotA& PA, RotB& PB, int x, int y, double gxx, double gyy, double gxy,
                                         const RotCfg& q) {
  const int i = min(x, y), j = max(x, y);
  const double gii = (x < y) ? gxx : gyy, gjj = (x < y) ? gyy : gxx;
  const Rot R = make_rot_nb(gii, gjj, gxy, q);
  PA.c = R.c; PA.s = R.s; PA.i = i; PA.j = j; PA.on = R.apply ? 1 : 0;
  PB.t = R.t; PB.gii = gii; PB.gjj = gjj; PB.gij = gxy;
  return R.apply;
}

// The 2 x 2 block of G in rows (A.i, A.j) and columns (B.i, B.j) after the round's rotations:
// rows i' = c i - s j, j' = s i + c j by A, then the same on the columns by B.
__device__ __forceinline__ void rotate_block(const RotA& A, const RotA& B, double& b00, double& b01, double& b10,
                                             double& b11) {
  if (A.on) {
    const double u0 = A.c * b00 - A.s * b10, v0 = fma(A.s, b00, A.c * b10);
    const double u1 = A.c * b01 - A.s * b11, v1 = fma(A.s, b01, A.c * b11);
    b00 = u0; b10 = v0; b01 = u1; b11 = v1;
  }
  if (B.on) {
    const double u0 = B.c * b00 - B.s * b01, v0 = fma(B.s, b00, B.c * b01);
    const double u1 = B.c * b10 - B.s * b11, v1 = fma(B.s, b10, B.c * b11);
    b00 = u0; b01 = v0; b10 = u1; b11 = v1;
  }
}

// rotate_block without branches: a pair that does not rotate has c = 1, s = 0 exactly, which leaves
// finite entries unchanged bit for bit.
__device__ __forceinline__ void rotate_block_nb(const RotA& A, const RotA& B, double& b00, double& b01, double& b10,
                                                double& b11) {
  const double u0 = A.c * b00 - A.s * b10, v0 = fma(A.s, b00, A.c * b10);
  const double u1 = A.c * b01 - A.s * b11, v1 = fma(A.s, b01, A.c * b11);
  b00 = B.c * u0 - B.s * u1; b01 = fma(B.s, u0, B.c * u1);
  b10 = B.c * v0 - B.s * v1; b11 = fma(B.s, v0, B.c * v1);
}

// V's rows in registers (thread = row): the rotations of inner round R, whose slots are known at
// compile time, applied to the row.
__host__ __device__ constexpr int rr_slot(int pos, int round) { return pos == 0 ? 0 : ((pos - 1 + round) % 31) + 1; }
template <int R, bool FULL>
__device__ __forceinline__ void v_apply(double (&v)[32], const RotA* P) {
  // a pair that does not rotate has c = 1, s = 0 exactly (make_rot), so every pair is applied
  // without a branch and all sixteen loads are issued first
  double c[16], s[16];
#pragma unroll
  for (int p = 0; p < 16; ++p) {   // (c, s) are the first 16 bytes of a 16-byte aligned RotA
    const double2 cs = *reinterpret_cast<const double2*>(&P[p].c);
    c[p] = cs.x; s[p] = cs.y;
  }
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    const int x = FULL ? rr_slot(p, R) : p, y = FULL ? rr_slot(31 - p, R) : 16 + ((p + R) & 15);
    const int i = x < y ? x : y, j = x < y ? y : x;
    const double a = v[i], b = v[j];
    v[i] = c[p] * a - s[p] * b;
    v[j] = fma(s[p], a, c[p] * b);
  }
}
#define TTC_VCASE(R) \
  case R: v_apply<R, FULL>(v, P); break;
template <bool FULL>
__device__ __forceinline__ void v_round(double (&v)[32], const RotA* P, int r) {
  switch (r) {
    TTC_VCASE(0) TTC_VCASE(1) TTC_VCASE(2) TTC_VCASE(3) TTC_VCASE(4) TTC_VCASE(5) TTC_VCASE(6) TTC_VCASE(7)
    TTC_VCASE(8) TTC_VCASE(9) TTC_VCASE(10) TTC_VCASE(11) TTC_VCASE(12) TTC_VCASE(13) TTC_VCASE(14) TTC_VCASE(15)
    default:
      if constexpr (FULL) {
        switch (r) {
          TTC_VCASE(16) TTC_VCASE(17) TTC_VCASE(18) TTC_VCASE(19) TTC_VCASE(20) TTC_VCASE(21) TTC_VCASE(22)
          TTC_VCASE(23) TTC_VCASE(24) TTC_VCASE(25) TTC_VCASE(26) TTC_VCASE(27) TTC_VCASE(28) TTC_VCASE(29)
          TTC_VCASE(30)
          default: break;
        }
      }
      break;
  }
}
#undef TTC_VCASE

// One inner round r on G with the rotations (cA, cB) computed from G before the round, in one
// barrier interval, the roles dealt by warps (a warp whose lanes take different roles runs the roles
// one after another, and warps w and w + 4 share a scheduler):
//  * warps 0-2 and lanes 0-23 of warp 4 apply the rotations to the 120 off-diagonal 2 x 2 blocks
//    (pair p rows, pair q columns, p < q; table blk) of G <- J^T G J, and lanes 0-15 of warp 5 to
//    the 16 diagonal blocks;
//  * warp 6 applies them to V, whose rows it holds in registers (thread = row);
//  * lanes 0-15 of warp 3, the round's critical path, with its scheduler to itself (warp 7 idles),
//    compute the rotations of round r + 1 into (nA, nB), one pair each:
//    the pair's two slots lie in two different pairs of round r (a round robin never repeats a pair
//    in consecutive rounds), so its three entries after this round follow from the pre-round block
//    of those pairs and their rotations, evaluated with the same operations as the block update.
template <bool FULL>
__device__ __forceinline__ void gram_round(double* G, double (&vrow)[32], const RotA* cA, const RotB* cB, RotA* nA,
                                           RotB* nB, const unsigned char* blk, const unsigned long long* sched, int r, int nr,
                                           const RotCfg& q, int* s_rot, unsigned long long& pre) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp < 3 || (warp == 4 && lane < 24)) {
    const int bk = warp < 3 ? tid : 96 + lane;
    const RotA A = cA[blk[2 * bk]], B = cA[blk[2 * bk + 1]];
    if (A.on || B.on) {
      double b00 = G[A.i + B.i * GLD], b01 = G[A.i + B.j * GLD];
      double b10 = G[A.j + B.i * GLD], b11 = G[A.j + B.j * GLD];
      rotate_block(A, B, b00, b01, b10, b11);
      G[A.i + B.i * GLD] = b00; G[B.i + A.i * GLD] = b00;
      G[A.i + B.j * GLD] = b01; G[B.j + A.i * GLD] = b01;
      G[A.j + B.i * GLD] = b10; G[B.i + A.j * GLD] = b10;
      G[A.j + B.j * GLD] = b11; G[B.j + A.j * GLD] = b11;
    }
  } else if (warp == 5 && lane < 16) {
    const RotA A = cA[lane];
    if (A.on) {
      const RotB Bd = cB[lane];
      G[A.i * (GLD + 1)] = Bd.gii - Bd.t * Bd.gij;
      G[A.j * (GLD + 1)] = Bd.gjj + Bd.t * Bd.gij;
      G[A.i + A.j * GLD] = 0.0;
      G[A.j + A.i * GLD] = 0.0;
    }
  } else if (warp == 6) {
    v_round<FULL>(vrow, cA, r);
  } else if (warp == 3 && lane < 16) {
    if (r + 1 < nr) {
      const int p = lane;
      // pair p of round r + 1 = (u, v); u lies in pair ia, v in pair ib of round r (ia < ib, the
      // block update's orientation), whose slots (Ai, Aj), (Bi, Bj) the schedule fixes
      int ia, ib, Ai, Aj, Bi, Bj, u, v;
      if (FULL) {
        const unsigned long long e = pre;   // schedule entry of round r + 1, loaded a round earlier
        if (r + 2 < nr) pre = sched[(r + 2) * 16 + p];
        ia = e & 15; ib = (e >> 4) & 15; Ai = (e >> 8) & 31; Aj = (e >> 13) & 31;
        Bi = (e >> 18) & 31; Bj = (e >> 23) & 31; u = (e >> 28) & 31; v = (e >> 33) & 31;
      } else {
        // (p, 16 + (p + r + 1) mod 16): p lies in pair p, the other slot in pair p + 1 (mod 16)
        const int a = p, b = (p + 1) & 15, ya = 16 + ((p + r) & 15), yb = 16 + ((p + 1 + r) & 15);
        const bool sw = a > b;
        ia = sw ? b : a; ib = sw ? a : b;
        Ai = ia; Aj = sw ? yb : ya; Bi = ib; Bj = sw ? ya : yb;
        u = sw ? yb : p; v = sw ? p : yb;
      }
      double b00 = G[Ai + Bi * GLD], b01 = G[Ai + Bj * GLD];
      double b10 = G[Aj + Bi * GLD], b11 = G[Aj + Bj * GLD];
      const RotA A = cA[ia], B = cA[ib];
      const RotB AB = cB[ia], BB = cB[ib];
      rotate_block_nb(A, B, b00, b01, b10, b11);
      // a pair that does not rotate has t = 0: its diagonal stays as it is
      const double guv = (u == Ai) ? ((v == Bi) ? b00 : b01) : ((v == Bi) ? b10 : b11);
      const double guu = (u == Ai) ? AB.gii - AB.t * AB.gij : AB.gjj + AB.t * AB.gij;
      const double gvv = (v == Bi) ? BB.gii - BB.t * BB.gij : BB.gjj + BB.t * BB.gij;
      if (set_pair(nA[p], nB[p], u, v, guu, gvv, guv, q)) *s_rot = 1;
    }
  }
  __syncthreads();
}
}  // namespace

__global__ void __launch_bounds__(NT, 2)
    jacobi_block_kernel(const JacobiDesc* __restrict__ descs, const int* __restrict__ order, int csize, int* flags,
                        int max_sweeps) {
  extern __shared__ double sm[];
  __shared__ int s_any, s_nact;
  __shared__ double s_red[NW];
  __shared__ RotA s_ra[2][16];
  __shared__ RotB s_rb[2][16];
  __shared__ unsigned char s_blk[2 * 120];
  __shared__ unsigned long long s_sched[31 * 16];   // full inner sweep: pair p of round r, see gram_round
  __shared__ int s_rot;
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  const int prob = (int)(blockIdx.x / csize);
  const JacobiDesc D = descs[order ? order[prob] : prob];
  if (D.m <= 0 || D.n <= 0) return;             // uniform across the cluster
  const int m = max(1, dev_bound(D.m, D.m_dev, D.m_mult)), n = D.n;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, qr = lane >> 2, qc = lane & 3;
  const int ms = smem_stride(m);
  double* S = sm;
  double* G = S + (size_t)32 * ms;
  double* V = G + 32 * GLD;
  double* nrm = V + 32 * GLD;
  int* act = reinterpret_cast<int*>(sm + block_dyn_doubles(ms, n));

  // column norms and ||X||_F^2: scale and numerical-zero threshold, as in jacobi_svd_kernel
  {
    double a = 0.0;
    for (int j = warp; j < n; j += NW) {
      const double* xc = D.X + (long long)j * D.ldx;
      double cj = 0.0;
      for (int i = lane; i < m; i += 32) cj = fma(xc[i], xc[i], cj);
      cj = warp_sum(cj);
      if (lane == 0) nrm[j] = cj;
      a += cj;
    }
    if (lane == 0) s_red[warp] = a;
  }
  if (tid == 0) s_any = 0;
  if (tid < 120) {   // the off-diagonal 2 x 2 blocks (p, q), p < q, of an inner round
    int p = 0, rem = tid;
    while (rem >= 15 - p) { rem -= 15 - p; ++p; }
    s_blk[2 * tid] = (unsigned char)p;
    s_blk[2 * tid + 1] = (unsigned char)(p + 1 + rem);
  }
  for (int e = tid; e < 31 * 16; e += NT) {
    const int r = e >> 4, p = e & 15;
    unsigned long long w = 0;
    if (r > 0) {
      const int x = rr_player(p, r, 32), y = rr_player(31 - p, r, 32);
      int xp, a, yp, b;
      inner_partner(x, r - 1, true, xp, a);
      inner_partner(y, r - 1, true, yp, b);
      const bool sw = a > b;
      const int ia = sw ? b : a, ib = sw ? a : b;
      const int u = sw ? y : x, up = sw ? yp : xp, v = sw ? x : y, vp = sw ? xp : yp;
      w = (unsigned long long)ia | ((unsigned long long)ib << 4) | ((unsigned long long)min(u, up) << 8) |
          ((unsigned long long)max(u, up) << 13) | ((unsigned long long)min(v, vp) << 18) |
          ((unsigned long long)max(v, vp) << 23) | ((unsigned long long)u << 28) | ((unsigned long long)v << 33);
    }
    s_sched[e] = w;
  }

  __syncthreads();
  double fro2 = 0.0;
#pragma unroll
  for (int i = 0; i < NW; ++i) fro2 += s_red[i];
  RotCfg q;
  {
    const double tol = jac_tol(D.m);
    int e2 = 0;
    if (fro2 > 0.0 && isfinite(fro2)) { frexp(fro2, &e2); e2 = (e2 + 1) & ~1; }
    q.sc = (fro2 > 0.0 && isfinite(fro2)) ? ldexp(1.0, -e2) : 1.0;
    q.tol2 = tol * tol;
    q.zthr = q.tol2 * fro2 * q.sc;
  }
  if (warp == 0) {   // the same list in every CTA of the cluster
    int cnt = 0;
    for (int c0 = 0; c0 < n; c0 += 32) {
      const int c = c0 + lane;
      const bool on = (c < n) && (nrm[c] * q.sc > q.zthr);
      const unsigned b = __ballot_sync(0xffffffffu, on);
      if (on) act[cnt + __popc(b & ((1u << lane) - 1u))] = c;
      cnt += __popc(b);
    }
    if (lane == 0) s_nact = cnt;
  }
  __syncthreads();
  const int na = s_nact;
  const int nblk = (na + 15) / 16;
  const int ne = nblk + (nblk & 1);
  cluster.sync();   // every CTA of the cluster runs before the first distributed-shared-memory access

  int* any0 = cluster.map_shared_rank(&s_any, 0);
  bool converged = false;
  int sweep = 0;
  for (; sweep < max_sweeps && !converged; ++sweep) {
    bool any = false;
    for (int rd = 0; rd < ne - 1; ++rd) {
      const bool full = (rd == 0);
      for (int p = crank; p < ne / 2; p += csize) {
        int bi = rr_player(p, rd, ne), bj = rr_player(ne - 1 - p, rd, ne);
        if (bi >= nblk || bj >= nblk) {       // partner is the phantom of an odd block count
          if (!full) continue;
          bi = min(bi, bj);
          bj = -1;
        }
        const int cI = min(16, na - bi * 16), cJ = bj >= 0 ? min(16, na - bj * 16) : 0;
        // load the valid slots: a warp per slot, lanes over rows, every copy in flight at once
        for (int slot = warp; slot < 32; slot += NW) {
          const bool inI = slot < 16;
          const int k = inI ? slot : slot - 16;
          if (k >= (inI ? cI : cJ)) continue;
          const double* src = D.X + (long long)act[(inI ? bi : bj) * 16 + k] * D.ldx;
          double* dst = S + (size_t)slot * ms;
          for (int r = lane; r < m; r += 32) cp_async8(dst + r, src + r);
        }
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();
        auto valid = [&](int slot) { return slot < 16 ? slot < cI : slot - 16 < cJ; };
        // G = S^T S: 16 tiles of 8 x 8, tiles warp and warp + 8 of each warp in one K loop, two
        // accumulator chains per tile
        {
          const int t0 = warp, t1 = warp + NW;
          const int ca0 = 8 * (t0 >> 2) + qr, cb0 = 8 * (t0 & 3) + qr;
          const int ca1 = 8 * (t1 >> 2) + qr, cb1 = 8 * (t1 & 3) + qr;
          const bool va0 = valid(ca0), vb0 = valid(cb0), va1 = valid(ca1), vb1 = valid(cb1);
          const double* Sa0 = S + (size_t)ca0 * ms;
          const double* Sb0 = S + (size_t)cb0 * ms;
          const double* Sa1 = S + (size_t)ca1 * ms;
          const double* Sb1 = S + (size_t)cb1 * ms;
          double g[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
          for (int k0 = 0; k0 < m; k0 += 8) {
            const int k = k0 + qc, k2 = k0 + 4 + qc;
            const bool in1 = k < m, in2 = k2 < m;
            dmma(g[0][0], g[0][1], (va0 && in1) ? Sa0[k] : 0.0, (vb0 && in1) ? Sb0[k] : 0.0);
            dmma(g[1][0], g[1][1], (va0 && in2) ? Sa0[k2] : 0.0, (vb0 && in2) ? Sb0[k2] : 0.0);
            dmma(g[2][0], g[2][1], (va1 && in1) ? Sa1[k] : 0.0, (vb1 && in1) ? Sb1[k] : 0.0);
            dmma(g[3][0], g[3][1], (va1 && in2) ? Sa1[k2] : 0.0, (vb1 && in2) ? Sb1[k2] : 0.0);
          }
          G[ca0 + (8 * (t0 & 3) + 2 * qc) * GLD] = g[0][0] + g[1][0];
          G[ca0 + (8 * (t0 & 3) + 2 * qc + 1) * GLD] = g[0][1] + g[1][1];
          G[ca1 + (8 * (t1 & 3) + 2 * qc) * GLD] = g[2][0] + g[3][0];
          G[ca1 + (8 * (t1 & 3) + 2 * qc + 1) * GLD] = g[2][1] + g[3][1];
        }
        __syncthreads();
        // does any pair of this visit (all slot pairs in round 0, the cross pairs later) need a rotation?
        int need = 0;
        for (int e = tid; e < 32 * 32; e += NT) {
          const int i = e & 31, j = e >> 5;
          if (i < j && (full || (i < 16 && j >= 16)) && valid(i) && valid(j)) {
            const double al = G[i * (GLD + 1)] * q.sc, be = G[j * (GLD + 1)] * q.sc, ga = G[i + j * GLD] * q.sc;
            if (al > q.zthr && be > q.zthr && ga * ga > q.tol2 * al * be) need = 1;
          }
        }
        if (!__syncthreads_or(need)) continue;   // block pair unchanged
        if (tid < 16) {   // the rotations of inner round 0 (pair index = tid)
          const int x = full ? rr_player(tid, 0, 32) : tid, y = full ? rr_player(31 - tid, 0, 32) : 16 + tid;
          set_pair(s_ra[0][tid], s_rb[0][tid], x, y, G[x * (GLD + 1)], G[y * (GLD + 1)], G[x + y * GLD], q);
        }
        if (tid == 0) s_rot = 0;
        __syncthreads();
        if (tid < 16 && s_ra[0][tid].on) s_rot = 1;
        {
          // V = I, its rows in the registers of warp 6 during the inner rounds
          double vrow[32];
#pragma unroll
          for (int c = 0; c < 32; ++c) vrow[c] = (c == lane) ? 1.0 : 0.0;
          unsigned long long pre = (warp == 3 && lane < 16) ? s_sched[16 + lane] : 0ull;
          if (full) {
            for (int r = 0; r < 31; ++r)
              gram_round<true>(G, vrow, s_ra[r & 1], s_rb[r & 1], s_ra[(r + 1) & 1], s_rb[(r + 1) & 1], s_blk, s_sched,
                               r, 31, q, &s_rot, pre);
          } else {
            for (int r = 0; r < 16; ++r)
              gram_round<false>(G, vrow, s_ra[r & 1], s_rb[r & 1], s_ra[(r + 1) & 1], s_rb[(r + 1) & 1], s_blk,
                                s_sched, r, 16, q, &s_rot, pre);
          }
          if (warp == 6) {
#pragma unroll
            for (int c = 0; c < 32; ++c) V[lane + c * GLD] = vrow[c];
          }
        }
        any |= (s_rot != 0);
        __syncthreads();   // V complete
        // columns <- S V, written to the problem's columns: 8-row tiles dealt to the warps
        for (int rt = warp; rt * 8 < m; rt += 2 * NW) {   // row tiles rt and rt + NW
          const int r0 = rt * 8 + qr, r1 = (rt + NW) * 8 + qr;   // A rows (lane / 4) = C rows
          double c[2][4][2] = {};
#pragma unroll
          for (int k0 = 0; k0 < 32; k0 += 4) {
            const int k = k0 + qc;
            const bool vk = valid(k);
            const double a0 = (vk && r0 < m) ? S[(size_t)k * ms + r0] : 0.0;
            const double a1 = (vk && r1 < m) ? S[(size_t)k * ms + r1] : 0.0;
#pragma unroll
            for (int tn = 0; tn < 4; ++tn) {
              const double b = V[k + (8 * tn + qr) * GLD];
              dmma(c[0][tn][0], c[0][tn][1], a0, b);
              dmma(c[1][tn][0], c[1][tn][1], a1, b);
            }
          }
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int rw = u ? r1 : r0;
            if (rw >= m) continue;
#pragma unroll
            for (int tn = 0; tn < 4; ++tn)
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int slot = 8 * tn + 2 * qc + e;
                if (valid(slot)) {
                  const int col = slot < 16 ? act[bi * 16 + slot] : act[bj * 16 + slot - 16];
                  D.X[(long long)col * D.ldx + rw] = c[u][tn][e];
                }
              }
          }
        }
        __syncthreads();   // S and V are read before the next visit loads
      }
      cluster.sync();      // the round's columns are in global memory for the next round's loads
    }
    if (any && lane == 0) atomicOr(any0, 1);
    cluster.sync();
    converged = (*any0 == 0);
    cluster.sync();
    if (crank == 0 && tid == 0) s_any = 0;
  }
  if (crank != 0) return;   // no distributed-shared-memory access follows
  if (!converged && tid == 0) atomicOr(flags, DFLAG_JACOBI_NOCONV);
  if (D.info && tid == 0) *D.info = converged ? sweep : -sweep;
  double* sig = nrm;
  for (int c = warp; c < n; c += NW) {
    double a = 0.0;
    for (int r = lane; r < m; r += 32) { const double u = D.X[(long long)c * D.ldx + r]; a = fma(u, u, a); }
    a = warp_sum(a);
    if (lane == 0) { sig[c] = sqrt(a); D.sigma[c] = sqrt(a); }
  }
  __syncthreads();
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

// Cluster size of a jacobi_block_kernel launch: as jacobi_cluster_size, for the block kernel's
// occupancy (two CTAs per SM up to 256 rows, one beyond).
static int jacobi_block_csize(int count, int max_n, size_t smem, bool ordered) {
  int per_sm = 1;
  TTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_block_kernel, NT, smem));
  per_sm = std::max(1, per_sm);
  const int slots = current_sm_count() * per_sm;
  const int pairs = std::max(1, ((max_n + 15) / 16 + 1) / 2);
  int c = std::max(1, slots / std::max(1, count));
  if (ordered) c = std::max(c, per_sm >= 2 ? 8 : 4);
  c = std::min(c, std::min(8, pairs));
  // a power of two, rounded up when the launch is ordered: a problem whose block pairs outnumber
  // its CTAs takes two visits per round, which doubles its latency
  int p2 = 1;
  if (ordered) while (p2 < c) p2 *= 2;
  else while (p2 * 2 <= c) p2 *= 2;
  return p2;
}

static void launch_jacobi_block(const JacobiDesc* d_descs, int count, int max_m, int max_n, cudaStream_t s,
                                int* d_flags, int* order, int max_sweeps) {
  static PerDeviceOnce attr_once;
  int dev = 0;
  TTC_CUDA(cudaGetDevice(&dev));
  attr_once.run(dev, [] {
    TTC_CUDA(cudaFuncSetAttribute(jacobi_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  });
  const size_t smem = sizeof(double) * block_dyn_doubles(smem_stride(max_m), max_n) + sizeof(int) * (size_t)max_n;
  TTC_REQUIRE(smem <= 200 * 1024, TTC_EDIM, "jacobi: matrix too large for the shared-memory blocks");
  if (order) {
    jacobi_order_kernel<<<1, 512, 0, s>>>(d_descs, count, order);
    TTC_CHECK_LAUNCH();
  }
  const int csize = jacobi_block_csize(count, max_n, smem, order != nullptr);
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
  TTC_CUDA(cudaLaunchKernelEx(&cfg, jacobi_block_kernel, d_descs, (const int*)order, csize, d_flags, max_sweeps));
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
  if (!accw && max_m <= 512) {
    launch_jacobi_block(d_descs, count, max_m, max_n, s, d_flags, order, max_sweeps);
    return;
  }
  if (max_m <= 256) launch_jacobi_t<8>(d_descs, count, max_n, bw, smem, s, d_flags, order, max_sweeps);
  else launch_jacobi_t<16>(d_descs, count, max_n, bw, smem, s, d_flags, order, max_sweeps);
}

}  // namespace ttc
