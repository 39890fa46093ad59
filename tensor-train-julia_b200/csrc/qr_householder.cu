// Batched blocked Householder QR, one thread-block cluster per problem.
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
// (same data, same arithmetic: identical reflectors, no broadcast needed); the column octets
// (8o .. 8o+7) of the trailing update and of Q are owned by CTA o mod C, so a column is always
// updated by the same CTA.  The block reflectors are applied on the FP64 tensor cores
// (mma.sync m8n8k4).  A cluster barrier (release/acquire at cluster scope) after each
// panel's trailing update makes the next panel visible to every CTA.  CTA 0 writes the
// factored panels and the T factors, which the Q formation reads after one more barrier.
#include <cooperative_groups.h>

#include <algorithm>

#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace ttc {
namespace {
constexpr int NB = 16;
constexpr int NT = 512;
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

// D += A B on the FP64 tensor-core path (mma.sync m8n8k4): per lane a = A[lane>>2][lane&3],
// b = B[lane&3][lane>>2], d = D[lane>>2][2(lane&3) + {0,1}].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Reflector entry V[l][r] of the panel (unit diagonal and zeros above it implied).
__device__ __forceinline__ double vref(const double* V, int mp_ld, int jb, int mp, int l, int r) {
  if (l >= jb || r >= mp || r < l) return 0.0;
  return (r == l) ? 1.0 : V[l * mp_ld + r];
}

// Apply (I - V T^T V^T) [trans=1] or (I - V T V^T) [trans=0] to columns [c_begin, c_end) of
// the global matrix M (rows r0..m-1, ld), with V (mp x jb) in shared memory (column-major,
// stride mp_ld = 4 mod 16 for conflict-free fragment loads) and T (jb x jb) in shared memory.
// One warp per octet of 8 columns; octet o belongs to CTA o mod csize.  Both products run on
// the FP64 tensor cores: W (16 x 8) = V^T C accumulated over 4-row steps, U = T^T W (or T W)
// through a per-warp scratch Ws (16 x 8), then C -= V U per 8-row tile.
__device__ void apply_block_reflector(double* M, int ld, int r0, int m, int c_begin, int c_end,
                                      const double* V, int mp_ld, int jb, const double* T, bool trans,
                                      int crank, int csize, double* Wscr) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int qr = lane >> 2, qc = lane & 3;
  const int mp = m - r0;
  double* Ws = Wscr + warp * 128;
  const int o_begin = c_begin >> 3, o_end = (c_end + 7) >> 3;
  const int o_first = o_begin + ((crank - o_begin) % csize + csize) % csize;
  for (int o = o_first + warp * csize; o < o_end; o += NW * csize) {
    const int c0 = 8 * o;
    // pass 1: W = V^T C; B fragment = C[r][c0 + qr]
    const int cb = c0 + qr;
    const bool cb_ok = (cb >= c_begin && cb < c_end);
    const double* colb = M + (long long)(cb_ok ? cb : c_begin) * ld + r0;
    // 32-row chunks, the next chunk's loads in flight while the current one is multiplied;
    // even and odd k-steps accumulate into separate tiles (four independent MMA chains)
    double w00 = 0.0, w01 = 0.0, w10 = 0.0, w11 = 0.0, x00 = 0.0, x01 = 0.0, x10 = 0.0, x11 = 0.0;
    double ba[8], bn[8];
    auto load8 = [&](double (&bb)[8], int k0) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int r = k0 + 4 * u + qc;
        bb[u] = (cb_ok && r < mp) ? colb[r] : 0.0;
      }
    };
    auto mma8 = [&](const double (&bb)[8], int k0) {
#pragma unroll
      for (int u = 0; u < 8; u += 2) {
        const int r = k0 + 4 * u + qc;
        dmma(w00, w01, vref(V, mp_ld, jb, mp, qr, r), bb[u]);
        dmma(w10, w11, vref(V, mp_ld, jb, mp, 8 + qr, r), bb[u]);
        dmma(x00, x01, vref(V, mp_ld, jb, mp, qr, r + 4), bb[u + 1]);
        dmma(x10, x11, vref(V, mp_ld, jb, mp, 8 + qr, r + 4), bb[u + 1]);
      }
    };
    load8(ba, 0);
    for (int k0 = 0;; k0 += 64) {
      const bool more1 = k0 + 32 < mp;
      if (more1) load8(bn, k0 + 32);
      mma8(ba, k0);
      if (!more1) break;
      const bool more2 = k0 + 64 < mp;
      if (more2) load8(ba, k0 + 64);
      mma8(bn, k0 + 32);
      if (!more2) break;
    }
    w00 += x00; w01 += x01; w10 += x10; w11 += x11;
    Ws[qr * 8 + 2 * qc] = w00;
    Ws[qr * 8 + 2 * qc + 1] = w01;
    Ws[(8 + qr) * 8 + 2 * qc] = w10;
    Ws[(8 + qr) * 8 + 2 * qc + 1] = w11;
    __syncwarp();
    // U = T^T W or T W (T upper triangular); this lane needs -U[4s + qc][qr], s = 0..3
    double ub[4];
#pragma unroll
    for (int sidx = 0; sidx < 4; ++sidx) {
      const int l = 4 * sidx + qc;
      double u = 0.0;
      if (l < jb) {
        if (trans) {
          for (int i = 0; i <= l; ++i) u = fma(T[l * NB + i], Ws[i * 8 + qr], u);
        } else {
          for (int i = l; i < jb; ++i) u = fma(T[i * NB + l], Ws[i * 8 + qr], u);
        }
      }
      ub[sidx] = -u;
    }
    __syncwarp();   // Ws is rewritten for the next octet
    // pass 2: C[rt..rt+7][c0..c0+7] -= V[rt.., 0..15] U
    const int ca = c0 + 2 * qc;
    const bool ok0 = (ca >= c_begin && ca < c_end), ok1 = (ca + 1 >= c_begin && ca + 1 < c_end);
    double* col0 = M + (long long)(ok0 ? ca : c_begin) * ld + r0;
    double* col1 = M + (long long)(ok1 ? ca + 1 : c_begin) * ld + r0;
    // 32-row sets of four 8-row tiles, the next set's loads in flight while the current one is
    // multiplied and stored
    double da0[4], da1[4], dn0[4], dn1[4];
    auto load4 = [&](double (&d0)[4], double (&d1)[4], int rt0) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int r = rt0 + 8 * u + qr;
        const bool rok = r < mp;
        d0[u] = (ok0 && rok) ? col0[r] : 0.0;
        d1[u] = (ok1 && rok) ? col1[r] : 0.0;
      }
    };
    auto upd4 = [&](double (&d0)[4], double (&d1)[4], int rt0) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int r = rt0 + 8 * u + qr;
#pragma unroll
        for (int sidx = 0; sidx < 4; ++sidx) dmma(d0[u], d1[u], vref(V, mp_ld, jb, mp, 4 * sidx + qc, r), ub[sidx]);
        if (ok0 && r < mp) col0[r] = d0[u];
        if (ok1 && r < mp) col1[r] = d1[u];
      }
    };
    load4(da0, da1, 0);
    for (int rt0 = 0;; rt0 += 64) {
      const bool more1 = rt0 + 32 < mp;
      if (more1) load4(dn0, dn1, rt0 + 32);
      upd4(da0, da1, rt0);
      if (!more1) break;
      const bool more2 = rt0 + 64 < mp;
      if (more2) load4(da0, da1, rt0 + 64);
      upd4(dn0, dn1, rt0 + 32);
      if (!more2) break;
    }
  }
}
}  // namespace

// Column steps of a panel held in registers (panel rows mp <= 32 * RMAX): warp w keeps panel
// column (w + 1) mod NW, lane l its rows l + 32 i, for the whole panel.  Step jj reads only the
// reflector column x = P[:, jj] and its diagonal from shared memory: the warps of the columns
// c > jj apply reflector jj to their column (x unscaled, as in the shared-memory loop below),
// the warps of the finished columns c < jj form x_c . x_jj below row jj for V^T V, and the warp
// of column jj + 1 returns its squared norm below the diagonal and publishes the column to P,
// where it is the next step's reflector.  Every column reaches P at the step that finishes it.
template <int RMAX>
__device__ __forceinline__ void panel_steps_regs(double* P, int mp, int mp_ld, int jb, double* nrm2, double* tau,
                                                 double* sv, double* bet, double* gs) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int c = (warp + 1) % NW;
  const bool own = c < jb;
  double* pc = P + c * mp_ld;
  double cr[RMAX];
#pragma unroll
  for (int i = 0; i < RMAX; ++i) {
    const int r = lane + 32 * i;
    cr[i] = (own && r < mp) ? pc[r] : 0.0;
  }
  for (int jj = 0; jj < jb; ++jj) {
    const double s = nrm2[jj & 1];
    const double alpha = P[jj * mp_ld + jj];
    double beta, t, scal;
    if (s == 0.0) { t = 0.0; beta = alpha; scal = 0.0; }
    else {
      beta = -copysign(sqrt(fma(alpha, alpha, s)), alpha);
      t = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    const double* x = P + jj * mp_ld;
    if (own && c != jj) {
      double dd[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int i = 0; i < RMAX; ++i) {
        const int r = lane + 32 * i;
        const double xv = (r > jj && r < mp) ? x[r] : 0.0;
        dd[i & 3] = fma(xv, cr[i], dd[i & 3]);
      }
      const double d = warp_sum((dd[0] + dd[1]) + (dd[2] + dd[3]));
      if (c < jj) {
        if (lane == 0) gs[c * NB + jj] = d;
      } else {
        const double cj = __shfl_sync(0xffffffffu, cr[0], jj);   // row jj < 32: lane jj, i = 0
        const double w = fma(scal, d, cj) * t;                   // tau v^T c
        const double ws = w * scal;
        double qq[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < RMAX; ++i) {
          const int r = lane + 32 * i;
          if (r > jj && r < mp) {
            cr[i] = fma(-ws, x[r], cr[i]);
            if (r > jj + 1) qq[i & 3] = fma(cr[i], cr[i], qq[i & 3]);
          }
        }
        if (lane == jj) cr[0] = cj - w;
        if (c == jj + 1) {
          const double q = warp_sum((qq[0] + qq[1]) + (qq[2] + qq[3]));
          if (lane == 0) nrm2[(jj + 1) & 1] = q;
#pragma unroll
          for (int i = 0; i < RMAX; ++i) {
            const int r = lane + 32 * i;
            if (r < mp) pc[r] = cr[i];
          }
        }
      }
    }
    if (tid == 0) { tau[jj] = t; sv[jj] = scal; bet[jj] = beta; }
    __syncthreads();
  }
}

// T layout in shared memory: T[col * NB + row] (upper triangular).
__global__ void __launch_bounds__(NT, 1) householder_qr_kernel(const QRDesc* __restrict__ descs, int csize, int* flags) {
  extern __shared__ double sm[];
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  const QRDesc D = descs[blockIdx.x / csize];
  if (D.m <= 0 || D.n <= 0) return;
  // the factored block (rows and columns beyond the device bounds are zero) and the shapes of
  // R (Kc x D.n) and Q (D.m x Kc)
  const int m = dev_bound(D.m, D.m_dev, D.m_mult), n = dev_bound(D.n, D.n_dev, D.n_mult);
  const int K = min(m, n), Kc = min(D.m, D.n);
  double* T = sm;                    // NB*NB
  double* tau = T + NB * NB;         // NB
  double* red = tau + NB;            // NW
  double* sv = red + NW;             // NB   reflector scales 1/(alpha - beta)
  double* bet = sv + NB;             // NB   betas (diagonal of R)
  double* nrm2 = bet + NB;           // 2    squared norm below the diagonal of the next column
  double* gs = nrm2 + 2;             // NB*NB  x_l . x_i below row i (l < i), unscaled
  double* xl_i = gs + NB * NB;       // NB*NB  x_l[i] (l < i), unscaled
  double* G = xl_i + NB * NB;        // NB*NB  (V^T V)
  double* Wscr = G + NB * NB;        // NW*128  per-warp 16 x 8 scratch of the reflector products
  double* P = Wscr + NW * 128;       // panel, (mp_ld x NB), mp_ld = 4 mod 16
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double* A = D.A;
  const int lda = D.lda;
  bool nonfinite = false;

  for (int j0 = 0; j0 < K; j0 += NB) {
    const int jb = min(NB, K - j0);
    const int mp = m - j0;
    const int mp_ld = mp + ((4 - mp) & 15);
    // 1. load panel
    nonfinite |= copy_cols(P, mp_ld, A + (long long)j0 * lda + j0, lda, mp, jb);
    __syncthreads();
    // 2. factor panel, one CTA barrier per column: reflector jj (dlarfg: beta =
    //    -sign(alpha) ||(alpha, x)||, tau = (beta - alpha)/beta, v = [1; x/(alpha - beta)]) is
    //    applied to columns c > jj with x unscaled; the warp that updates column jj+1 also
    //    returns its squared norm below the diagonal for the next reflector.  The reflector
    //    columns are scaled, and the betas stored, after the loop.
    {
      double s0 = 0.0;
      for (int r = 1 + tid; r < mp; r += NT) { const double x = P[r]; s0 = fma(x, x, s0); }
      s0 = block_sum(s0, red);
      if (tid == 0) nrm2[0] = s0;
      __syncthreads();
    }
    // the panel's own row count picks the column-step routine (uniform across the cluster):
    // registers up to 512 rows, else the shared-memory loop below (the register column and the
    // loads in flight no longer fit 128 registers at 24 rows per lane)
    if (mp <= 256) panel_steps_regs<8>(P, mp, mp_ld, jb, nrm2, tau, sv, bet, gs);
    else if (mp <= 512) panel_steps_regs<16>(P, mp, mp_ld, jb, nrm2, tau, sv, bet, gs);
    else for (int jj = 0; jj < jb; ++jj) {
      const double s = nrm2[jj & 1];
      const double alpha = P[jj * mp_ld + jj];
      double beta, t, scal;
      if (s == 0.0) { t = 0.0; beta = alpha; scal = 0.0; }
      else {
        beta = -copysign(sqrt(fma(alpha, alpha, s)), alpha);
        t = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      const double* x = P + jj * mp_ld;
      // slot k of warp k mod NW: column k < jj gives x_k . x_jj below row jj (for V^T V),
      // column k + 1 > jj gets the reflector
      for (int k = warp; k < jb - 1; k += NW) {
        if (k < jj) {
          const double* pl = P + k * mp_ld;
          double g = 0.0, g2 = 0.0;
          for (int r = jj + 1 + lane; r < mp; r += 64) {
            g = fma(pl[r], x[r], g);
            if (r + 32 < mp) g2 = fma(pl[r + 32], x[r + 32], g2);
          }
          g = warp_sum(g + g2);
          if (lane == 0) gs[k * NB + jj] = g;
          continue;
        }
        const int c = k + 1;
        double* pc = P + c * mp_ld;
        const double cj = pc[jj];
        double d = 0.0, d2 = 0.0;       // two chains
        for (int r = jj + 1 + lane; r < mp; r += 64) {
          d = fma(x[r], pc[r], d);
          if (r + 32 < mp) d2 = fma(x[r + 32], pc[r + 32], d2);
        }
        d = warp_sum(d + d2);
        const double w = fma(scal, d, cj) * t;     // tau v^T c
        const double ws = w * scal;
        double q = 0.0, q2 = 0.0;
        for (int r = jj + 1 + lane; r < mp; r += 64) {
          const double u = fma(-ws, x[r], pc[r]);
          pc[r] = u;
          if (r > jj + 1) q = fma(u, u, q);
          if (r + 32 < mp) {
            const double u2 = fma(-ws, x[r + 32], pc[r + 32]);
            pc[r + 32] = u2;
            q2 = fma(u2, u2, q2);
          }
        }
        q += q2;
        if (c == jj + 1) {
          q = warp_sum(q);
          if (lane == 0) nrm2[(jj + 1) & 1] = q;
        }
        if (lane == 0) pc[jj] = cj - w;
      }
      if (tid == 0) { tau[jj] = t; sv[jj] = scal; bet[jj] = beta; }
      __syncthreads();
    }
    for (int e = tid; e < NB * NB; e += NT) {        // unscaled x_l[i] for V^T V
      const int i = e / NB, l = e - i * NB;
      if (l < i && i < jb) xl_i[l * NB + i] = P[l * mp_ld + i];
    }
    __syncthreads();
    for (int c = warp; c < jb; c += NW) {
      double* pc = P + c * mp_ld;
      const double sc = sv[c];
      for (int r = c + 1 + lane; r < mp; r += 32) pc[r] *= sc;
      if (lane == 0) pc[c] = bet[c];
    }
    __syncthreads();
    // 3. T factor.  G = V^T V (l < i) from the dot products of the panel loop:
    //    v_l[i] = scal_l x_l[i], v_i[i] = 1, rows below i scaled by both (x unscaled there);
    //    then T from T^{-1} + T^{-T} = V^T V (compact WY): T^{-1} = striu(G) + diag(1/tau), so
    //    T[r][j] = -tau_r sum_{r < l <= j} G[r][l] T[l][j], T[j][j] = tau_j; lane j of warp 0
    //    back-substitutes column j in registers (a zero tau gives a zero row, as in dlarft).
    for (int e = tid; e < NB * NB; e += NT) {
      const int i = e / NB, l = e - i * NB;
      if (l < i) G[i * NB + l] = (i < jb) ? sv[l] * fma(sv[i], gs[l * NB + i], xl_i[l * NB + i]) : 0.0;
    }
    __syncthreads();
    if (warp == 0 && lane < NB) {
      const int j = lane;
      double tc[NB];
#pragma unroll
      for (int k = 0; k < NB; ++k) tc[k] = (k == j && j < jb) ? tau[k] : 0.0;
#pragma unroll
      for (int r = NB - 2; r >= 0; --r) {
        double a2 = 0.0;
#pragma unroll
        for (int l = r + 1; l < NB; ++l) a2 = fma(G[l * NB + r], tc[l], a2);
        if (r < j && j < jb) tc[r] = -tau[r] * a2;
      }
#pragma unroll
      for (int k = 0; k < NB; ++k) T[j * NB + k] = tc[k];
    }
    __syncthreads();
    // 4. trailing update with H^T = I - V T^T V^T (this CTA's column octets)
    if (j0 + jb < n) apply_block_reflector(A, lda, j0, m, j0 + jb, n, P, mp_ld, jb, T, true, crank, csize, Wscr);
    // 5. CTA 0 writes back the panel and keeps T
    if (crank == 0) {
      copy_cols(A + (long long)j0 * lda + j0, lda, P, mp_ld, mp, jb);
      if (D.Tws)
        for (int e = tid; e < NB * NB; e += NT) D.Tws[(j0 / NB) * NB * NB + e] = T[e];
    }
    cluster.sync();   // trailing columns and the panel visible to every CTA
  }
  if (nonfinite && crank == 0 && threadIdx.x == 0) atomicOr(flags, DFLAG_NONFINITE);

  // R = upper triangle of A[0:Kc, 0:D.n] (zero outside the factored block)
  if (D.R) {
    for (int j = (int)(threadIdx.x >> 5) + NW * crank; j < D.n; j += NW * csize)
      for (int i = (int)(threadIdx.x & 31); i < Kc; i += 32) {
        const double v = (i <= j) ? A[(long long)j * lda + i] : 0.0;
        if (D.r_trans) D.R[(long long)i * D.ldr + j] = v;
        else D.R[(long long)j * D.ldr + i] = v;
        if (D.Rt) D.Rt[(long long)i * D.ldrt + j] = v;
      }
  }
  if (!D.Q) return;
  // Q = H_1 ... H_K [I; 0], accumulated backwards panel by panel.  Each CTA initialises
  // and updates only its own column octets, so the panels need no barrier between them.
  // The reflectors act on rows < m; identity columns c >= K are untouched unless a column
  // bound leaves some of them with c < m.
  for (int c = 0; c < Kc; ++c) {
    if (((c >> 3) % csize) != crank) continue;
    for (int i = tid; i < D.m; i += NT) D.Q[(long long)c * D.ldq + i] = (i == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int qc_end = (n < D.n) ? Kc : K;
  const int npan = (K + NB - 1) / NB;
  for (int p = npan - 1; p >= 0; --p) {
    const int j0 = p * NB, jb = min(NB, K - j0), mp = m - j0, mp_ld = mp + ((4 - mp) & 15);
    copy_cols(P, mp_ld, A + (long long)j0 * lda + j0, lda, mp, jb);
    for (int e = tid; e < NB * NB; e += NT) T[e] = D.Tws[p * NB * NB + e];
    __syncthreads();
    apply_block_reflector(D.Q, D.ldq, j0, m, j0, qc_end, P, mp_ld, jb, T, false, crank, csize, Wscr);
    __syncthreads();
  }
}

// B <- Q B from the stored panels, backwards (as the Q formation, but from B instead of the
// identity and over all its columns).  CTA problem / csize owns the column octets o with
// o mod csize == CTA rank; the panels are only read, so no CTA waits for another.
__global__ void __launch_bounds__(NT, 1) householder_apply_q_kernel(const QApplyDesc* __restrict__ descs, int csize) {
  extern __shared__ double sm[];
  const int crank = (int)(blockIdx.x % csize);
  const QApplyDesc D = descs[blockIdx.x / csize];
  const int m = dev_bound(D.m, D.m_dev, D.m_mult), K = min(D.K, m);   // H_k = I for k >= m
  if (m <= 0 || K <= 0 || D.nb <= 0) return;
  const int nb = D.n_dev ? min(D.nb, *D.n_dev) : D.nb;
  if (nb <= 0) return;
  double* T = sm;                    // NB*NB
  double* Wscr = T + NB * NB;        // NW*128
  double* P = Wscr + NW * 128;       // panel, (mp_ld x NB)
  const int tid = threadIdx.x;
  const int npan = (K + NB - 1) / NB;
  for (int p = npan - 1; p >= 0; --p) {
    const int j0 = p * NB, jb = min(NB, K - j0), mp = m - j0, mp_ld = mp + ((4 - mp) & 15);
    copy_cols(P, mp_ld, D.A + (long long)j0 * D.lda + j0, D.lda, mp, jb);
    for (int e = tid; e < NB * NB; e += NT) T[e] = D.Tws[p * NB * NB + e];
    __syncthreads();
    apply_block_reflector(D.B, D.ldb, j0, m, 0, nb, P, mp_ld, jb, T, false, crank, csize, Wscr);
    __syncthreads();
  }
}

void launch_qr_apply(const QApplyDesc* d_descs, int count, int max_m, cudaStream_t s) {
  if (count <= 0) return;
  TTC_REQUIRE(max_m <= QR_MAX_M, TTC_EDIM, "qr apply: row count exceeds the supported maximum (1536)");
  const size_t smem = sizeof(double) * (NB * NB + NW * 128 + (size_t)(max_m + 15) * NB);
  static PerDeviceOnce attr_once;
  int dev = 0;
  TTC_CUDA(cudaGetDevice(&dev));
  attr_once.run(dev, [] {
    TTC_CUDA(cudaFuncSetAttribute(householder_apply_q_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * (NB * NB + NW * 128 + (size_t)(QR_MAX_M + 15) * NB))));
  });
  const int nsm = current_sm_count();
  int per_sm = 1;
  TTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, householder_apply_q_kernel, NT, smem));
  const int csize = std::min(8, std::max(1, nsm * std::max(1, per_sm) / count));
  householder_apply_q_kernel<<<(unsigned)(count * csize), NT, smem, s>>>(d_descs, csize);
  TTC_CHECK_LAUNCH();
}

namespace {
size_t qr_smem(int max_m) {
  return sizeof(double) * (NB * NB * 4 + 3 * NB + NW + 2 + NW * 128 + (size_t)(max_m + 15) * NB);
}

constexpr int kQrWaves = 2;
void launch_qr_cfg(const QRDesc* d_descs, int count, int max_m, cudaStream_t s, int* d_flags) {
  const size_t smem = qr_smem(max_m);
  static PerDeviceOnce attr_once;
  int dev = 0;
  TTC_CUDA(cudaGetDevice(&dev));
  attr_once.run(dev, [] {
    TTC_CUDA(cudaFuncSetAttribute(householder_qr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)qr_smem(QR_MAX_M)));
  });
  const int nsm = current_sm_count();
  // CTAs per problem: up to two waves of the resident-CTA slots of the GPU (the planner puts the
  // largest problems first, so the second wave holds the short ones), at most 8 (portable cluster)
  int per_sm = 1;
  TTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, householder_qr_kernel, NT, smem));
  const int slots = nsm * std::max(1, per_sm);
  int c = std::min(8, std::max(1, kQrWaves * slots / count));
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
}  // namespace

void launch_qr(const QRDesc* d_descs, int count, int max_m, cudaStream_t s, int* d_flags) {
  if (count <= 0) return;
  TTC_REQUIRE(max_m <= QR_MAX_M, TTC_EDIM, "qr: row count exceeds the supported maximum (1536)");
  launch_qr_cfg(d_descs, count, max_m, s, d_flags);
}

}  // namespace ttc
