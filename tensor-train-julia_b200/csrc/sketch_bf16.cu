// Mixed-precision reverse recursive sketch (src/sketches.jl:221-239, kernel
// contract_sketch_core_backwards!, :1602-1638): both contractions of every site run on
// the tcgen05 BF16 GEMM with FP32 accumulation.  Per site k and block j:
//   T[(a,z), be]   = sum_al A_k[a, z, al] W_{k+1}[al, be, j]        (GEMM 1)
//   W_k[a, b, j]   = sum_{z,be} T[a, z, be] S_k[z, be, b, j]          (GEMM 2)
// GEMM 1 writes T directly as the K-major BF16 operand of GEMM 2; GEMM 2 writes W_k in
// FP64 (for the FP64 range finder Z = y_k W_{k+1}) and as the K-major BF16 operand of the
// next site's GEMM 1.  Cores and sketch blocks are converted to BF16 once per call.
//
// Precision policy.  The range finder Z = y_{k-1} W_k recovers the TT exactly (s_k >= r_k)
// when range(y_{k-1} W_k) contains range(y_{k-1} R_k), R_k the right interface of bond k.
// That holds for ANY perturbed W_k of full row rank when R_k has full row rank, so BF16
// rounding is harmless there.  When R_k is rank deficient (a non-minimal TT: r_k larger
// than n_k times the rank of R_{k+1}, e.g. sums of TTs or independently drawn ranks), W_k
// must stay of the form R_k X, which rounding A_k or W_{k+1} to BF16 breaks (the captured
// subspace then moves by ~1e-3).  Levels whose right interface is structurally rank
// deficient, rho_k = min(r_k, n_k rho_{k+1}) < r_k, are therefore contracted in FP64 from
// the FP64 W_{k+1}; their BF16 copy of W_k is made afterwards for the next BF16 level.
// Numerically (not structurally) deficient interfaces are not detected.
#include <algorithm>

#include "drivers.cuh"

namespace ttc {

static inline long long pad8(long long v) { return (v + 7) & ~7LL; }

void emit_sketch_bf16(Builder& B, ttc_batch* x, const std::vector<int>& tts, const SketchPlan& sp,
                      const std::vector<double*>& S, std::vector<std::vector<double*>>& W, bool tf32) {
  const int N = x->N;
  const size_t T = tts.size();
  W.assign(T, std::vector<double*>(N + 1, nullptr));
  const long long esz = tf32 ? 4 : 2;   // operand bytes: BF16, or FP32 read as TF32
  auto at = [&](const void* p, long long elems) -> void* { return (void*)((const char*)p + elems * esz); };
  // Operand buffers are carved from double-sized workspace blocks (zeroed: padding must be 0).
  std::vector<ZeroDesc> zr;
  auto bf = [&](long long elems) -> void* {
    const long long nd = (elems * esz + 7) / 8;
    double* p = B.wd((size_t)nd);
    zr.push_back({p, nd});
    return (void*)p;
  };
  std::vector<std::vector<void*>> A16(T, std::vector<void*>(N)), W16(T, std::vector<void*>(N + 1));
  std::vector<void*> S16(N);
  std::vector<CvtDesc> cv;
  // f64lvl[i][k]: the right interface of bond k of TT i is structurally rank deficient
  std::vector<std::vector<char>> f64lvl(T, std::vector<char>(N + 1, 0));
  for (size_t i = 0; i < T; ++i) {
    long long rho = 1;
    for (int k = N - 1; k >= 0; --k) {
      rho = std::min<long long>(x->rk(tts[i], k), x->dims[k] * rho);
      f64lvl[i][k] = rho < x->rk(tts[i], k);
    }
  }
  for (size_t i = 0; i < T; ++i) {
    const int t = tts[i];
    for (int k = 0; k < N; ++k) {
      const long long n = x->dims[k], r0 = x->rk(t, k), r1 = x->rk(t, k + 1), xc = x->capr(t, k);
      const long long lda = pad8(r1);
      W[i][k] = B.wd((size_t)r0 * sp.b[k] * sp.p[k]);
      W16[i][k] = (k > 0) ? bf(pad8(r0) * sp.b[k] * sp.p[k]) : nullptr;
      if (f64lvl[i][k]) continue;
      A16[i][k] = bf(r0 * n * lda);
      for (long long z = 0; z < n; ++z) {
        CvtDesc c{};
        c.src = x->core(t, k) + z * xc;
        c.dst = at(A16[i][k], r0 * z * lda);
        c.rows = r0; c.cols = r1;
        c.ss_i = 1; c.ss_j = xc * n;
        c.ds_i = lda; c.ds_j = 1;
        c.alpha = 1.0;
        cv.push_back(c);
      }
    }
    W[i][N] = B.ctx->d_one;
    W16[i][N] = bf(8);
    CvtDesc one{};
    one.src = B.ctx->d_one; one.dst = W16[i][N];
    one.rows = 1; one.cols = 1; one.ss_i = 0; one.ss_j = 0; one.ds_i = 1; one.ds_j = 1; one.alpha = 1.0;
    cv.push_back(one);
  }
  for (int k = 0; k < N; ++k) {
    const long long n = x->dims[k], bl = sp.b[k + 1], br = sp.b[k], pk = sp.p[k];
    const long long lds = pad8(n * bl);
    S16[k] = bf(lds * br * pk);
    for (long long j = 0; j < pk; ++j) {
      CvtDesc c{};
      c.src = S[k] + j * n * bl * br;
      c.dst = at(S16[k], j * lds * br);
      c.rows = n * bl; c.cols = br;
      c.ss_i = 1; c.ss_j = n * bl;
      c.ds_i = 1; c.ds_j = lds;
      c.alpha = 1.0;
      cv.push_back(c);
    }
  }
  B.zero(zr);
  B.cvt_bf16(cv, tf32);
  for (int k = N - 1; k >= 0; --k) {
    const size_t mk = B.mark();
    std::vector<ZeroDesc> zt;
    std::vector<Bf16GemmDesc> g1, g2;
    std::vector<GemmDesc> f1, f2;
    std::vector<CvtDesc> cw;
    const long long n = x->dims[k], bl = sp.b[k + 1], br = sp.b[k], pk = sp.p[k];
    const long long ldt = pad8(n * bl), lds = pad8(n * bl);
    for (size_t i = 0; i < T; ++i) {
      const int t = tts[i];
      const long long r0 = x->rk(t, k), r1 = x->rk(t, k + 1);
      const long long ldw1 = pad8(r1), ldw0 = pad8(r0);
      if (f64lvl[i][k]) {
        // FP64 level: T[(a,z), be] = sum_al A_k[a,z,al] W_{k+1}[al,be,j]; W_k = T S_k
        const long long xc = x->capr(t, k);
        double* Tm = B.wd((size_t)(r0 * n * bl * pk));
        GemmDesc d = gd((int)(r0 * n), (int)bl, (int)r1, x->core(t, k), 1, xc * n, W[i][k + 1], 1, r1, Tm, 1, r0 * n);
        d.m0 = (int)r0; d.a_i0 = 1; d.a_i1 = xc;
        d.c_i0 = 1; d.c_i1 = r0;
        d.batch = (int)pk;
        d.a_b = 0;
        d.b_b = (k < N - 1) ? r1 * bl : 0;
        d.c_b = r0 * n * bl;
        f1.push_back(d);
        GemmDesc e = gd((int)r0, (int)br, (int)(n * bl), Tm, 1, r0, S[k], 1, n * bl, W[i][k], 1, r0);
        e.batch = (int)pk;
        e.a_b = r0 * n * bl;
        e.b_b = n * bl * br;
        e.c_b = r0 * br;
        f2.push_back(e);
        if (k > 0) {   // BF16 copy of W_k (a, (b, j)) at a + ldw0 (b + br j)
          CvtDesc c{};
          c.src = W[i][k]; c.dst = W16[i][k];
          c.rows = r0; c.cols = br * pk;
          c.ss_i = 1; c.ss_j = r0;
          c.ds_i = 1; c.ds_j = ldw0;
          c.alpha = 1.0;
          cw.push_back(c);
        }
        continue;
      }
      const long long tnd = (r0 * ldt * pk * esz + 7) / 8;
      double* Tbuf = B.wd((size_t)tnd);
      zt.push_back({Tbuf, tnd});
      for (long long j = 0; j < pk; ++j) {
        void* T16 = at(Tbuf, j * r0 * ldt);
        Bf16GemmDesc d{};
        d.m = (int)(r0 * n); d.n = (int)bl; d.k = (int)r1; d.m0 = (int)r0;
        d.A = A16[i][k]; d.lda = ldw1;
        const long long jn = (k < N - 1) ? j : 0;
        d.B = at(W16[i][k + 1], jn * ldw1 * bl); d.ldb = ldw1;
        d.C16 = T16; d.h_i0 = ldt; d.h_i1 = 1; d.h_j = n;
        d.alpha = 1.0;
        g1.push_back(d);
        Bf16GemmDesc e{};
        e.m = (int)r0; e.n = (int)br; e.k = (int)(n * bl); e.m0 = (int)std::max<long long>(r0, 1);
        e.A = T16; e.lda = ldt;
        e.B = at(S16[k], j * lds * br); e.ldb = lds;
        e.C64 = W[i][k] + j * r0 * br; e.c_i0 = 1; e.c_i1 = 0; e.c_j = r0;
        if (k > 0) { e.C16 = at(W16[i][k], j * ldw0 * br); e.h_i0 = 1; e.h_i1 = 0; e.h_j = ldw0; }
        e.alpha = 1.0;
        g2.push_back(e);
      }
    }
    B.zero(zt);
    B.bf16gemm(g1, tf32);
    B.bf16gemm(g2, tf32);
    B.gemm(f1);
    B.gemm(f2);
    B.cvt_bf16(cw, tf32);
    B.release(mk);
  }
}

}  // namespace ttc
