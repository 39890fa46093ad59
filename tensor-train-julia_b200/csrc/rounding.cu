// Sweep drivers: deterministic TT rounding (src/tt_rounding.jl:146-269) and randomized
// TT rounding (src/tt_randtools.jl:112-154 with src/sketches.jl:175-305) on device
// batches.  Internal core layout: column-major (r_{k-1}, n_k, r_k) inside a capacity
// (cap_{k-1}, n_k, cap_k) slab whose padding is zero, so that
//   left unfolding  (cap_{k-1} n_k) x cap_k   has ld cap_{k-1} n_k, and
//   right unfolding  cap_{k-1} x (n_k cap_k)  has ld cap_{k-1}.
// Every step of a sweep handles all TTs of the batch in one launch per kernel kind.
#include <algorithm>
#include <cmath>

#include "builder.cuh"
#include "drivers.cuh"

namespace ttc {

static inline int qr_tws(int m, int n) { return ((std::min(m, n) + 15) / 16) * 256 + 256; }

// ---------------------------------------------------------------- helpers
void emit_zero_tts(Builder& B, ttc_batch* y, const std::vector<int>& tts) {
  std::vector<ZeroDesc> z;
  for (int t : tts) z.push_back({y->core(t, 0), y->tt_off[t + 1] - y->tt_off[t]});
  B.zero(z);
}

void emit_set_ranks(Builder& B, ttc_batch* y, const std::vector<int>& tts, const std::vector<std::vector<int>>& r) {
  std::vector<SetRankDesc> v;
  for (size_t i = 0; i < tts.size(); ++i) v.push_back({y->drk(tts[i], 0), B.const_ints(r[i]), y->N + 1});
  B.setrank(v);
}

// Copy the TTs of x into y (ranks r), changing only the capacity padding.
void emit_copy_tts(Builder& B, ttc_batch* x, ttc_batch* y, const std::vector<int>& tts,
                   const std::vector<std::vector<int>>& r) {
  std::vector<CopyDesc> v;
  for (size_t i = 0; i < tts.size(); ++i) {
    const int t = tts[i];
    for (int k = 0; k < x->N; ++k) {
      const long long n = x->dims[k], xc = x->capr(t, k), yc = y->capr(t, k);
      v.push_back(cd3(x->core(t, k), y->core(t, k), r[i][k], n, r[i][k + 1], 1, xc, xc * n, 1, yc, yc * n));
    }
  }
  B.copy(v);
}

// L->R Householder QR sweep, orthogonalize(x; i=N) (src/tt_rounding.jl:72-79, :92-95).
// rp[i] are the output ranks (min(n r'_k, r_{k+1}) recursion).
void emit_orth_left(Builder& B, ttc_batch* x, ttc_batch* y, const std::vector<int>& tts,
                    const std::vector<std::vector<int>>& rp) {
  const int N = x->N;
  const size_t T = tts.size();
  if (T == 0) return;
  const size_t mark0 = B.mark();
  std::vector<double*> FR(T), FRn(T);
  for (size_t i = 0; i < T; ++i) {
    const int t = tts[i];
    size_t mx = 1;
    for (int k = 1; k < N; ++k) mx = std::max(mx, (size_t)rp[i][k] * x->rk(t, k));
    FR[i] = B.wd(mx);
    FRn[i] = B.wd(mx);
  }
  for (int j = 0; j + 1 < N; ++j) {
    const size_t m = B.mark();
    std::vector<GemmDesc> g;
    std::vector<QRDesc> q;
    std::vector<CopyDesc> cp;
    const int n = (int)x->dims[j];
    for (size_t i = 0; i < T; ++i) {
      const int t = tts[i];
      const int a = rp[i][j], an = rp[i][j + 1];
      const int xr0 = x->rk(t, j), xr1 = x->rk(t, j + 1), xc = x->capr(t, j), yc = y->capr(t, j);
      double* C = B.wd((size_t)a * n * xr1);
      double* Tws = B.wd(qr_tws(a * n, xr1));
      const double* A = (j == 0) ? B.ctx->d_one : FR[i];
      g.push_back(gd(a, n * xr1, xr0, A, 1, a, x->core(t, j), 1, xc, C, 1, a));
      if (yc == a) {   // core j of y has Q's layout (a n rows, column stride a n): Q is written there
        q.push_back({a * n, xr1, C, a * n, y->core(t, j), a * n, FRn[i], an, Tws});
      } else {
        double* Q = B.wd((size_t)a * n * an);
        q.push_back({a * n, xr1, C, a * n, Q, a * n, FRn[i], an, Tws});
        cp.push_back(cd3(Q, y->core(t, j), a, n, an, 1, a, (long long)a * n, 1, yc, (long long)yc * n));
      }
    }
    B.gemm(g);
    B.qr(q);
    B.copy(cp);
    std::swap(FR, FRn);
    B.release(m);
  }
  std::vector<GemmDesc> g;
  const int n = (int)x->dims[N - 1];
  for (size_t i = 0; i < T; ++i) {
    const int t = tts[i];
    const int a = rp[i][N - 1];
    const double* A = (N == 1) ? B.ctx->d_one : FR[i];
    g.push_back(gd(a, n, x->rk(t, N - 1), A, 1, a, x->core(t, N - 1), 1, x->capr(t, N - 1), y->core(t, N - 1), 1,
                   y->capr(t, N - 1)));
  }
  B.gemm(g);
  B.release(mark0);
}

// R->L truncated-SVD sweep of _tt_rounding, direction=:left (src/tt_rounding.jl:179-217),
// on y (left-orthogonal, ranks rp).  The truncation rank of bond j is written to y's
// device rank array; cores keep their capacity and are zero beyond the kept rank.
void emit_svd_left(Builder& B, ttc_batch* y, const std::vector<int>& tts, const std::vector<std::vector<int>>& rp,
                   double tol, long long rmax) {
  const int N = y->N;
  const size_t T = tts.size();
  if (T == 0) return;
  // The product T2 = core(j-1) T1 of bond j has core j-1's layout (ld n_{j-1} capr(j-1)) and is
  // zero beyond the kept rank, so bond j-1 reads it in place of core j-1, which it rewrites
  // anyway; only the last bond's product is copied into core 0.  Two buffers per TT alternate.
  const size_t mark0 = B.mark();
  std::vector<double*> T2buf[2] = {std::vector<double*>(T), std::vector<double*>(T)};
  for (size_t i = 0; i < T; ++i) {
    size_t mx = 1;
    for (int j = N - 1; j >= 1; --j)
      mx = std::max(mx, (size_t)y->capr(tts[i], j - 1) * (size_t)y->dims[j - 1] * (size_t)rp[i][j]);
    T2buf[0][i] = B.wd(mx);
    T2buf[1][i] = B.wd(mx);
  }
  for (int j = N - 1; j >= 1; --j) {
    const size_t mk = B.mark();
    std::vector<CopyDesc> cpX, cpW, cpT2;
    std::vector<QRDesc> qr, qr2;
    std::vector<JacobiDesc> jac;
    std::vector<TruncDesc> tr;
    std::vector<SelectDesc> sel;
    std::vector<GemmDesc> g2, g3;
    std::vector<QApplyDesc> qa;
    int* infos = B.diag_ints((int)T);
    const int n = (int)y->dims[j], nl = (int)y->dims[j - 1];
    for (size_t i = 0; i < T; ++i) {
      const int t = tts[i];
      const int q = rp[i][j], p = n * rp[i][j + 1];
      const int yc = y->capr(t, j), ycl = y->capr(t, j - 1);
      const int ml = ycl * nl;
      int* rank = y->drk(t, j);
      // core j is zero beyond the kept rank r' of bond j+1 (truncated at step j+1, or the
      // boundary rank 1), so its unfolding has n r' nonzero (n, r_{j+1}) combinations, the last
      // ones in the device layout: the factorizations below run on that block
      const int* rk1 = y->drk(t, j + 1);
      int* info = infos + i;
      double* X = B.wd((size_t)p * q);
      double* T1 = B.wd((size_t)q * q);
      double* T2 = T2buf[j & 1][i];
      // core j as this bond reads it: the previous bond's product (core j is rewritten below)
      const double* Cj = (j == N - 1) ? y->core(t, j) : T2buf[(j + 1) & 1][i];
      if (p >= q) {
        // M^T = Q R1 (Householder), R1^T = Q2 R2, one-sided Jacobi on R2^T = R1 Q2: same left
        // singular vectors as R1 in about half the sweeps (QR-LQ preconditioning); the factor
        // absorbed into core j-1 stays R1^T U.  Q is not formed: its stored reflectors are
        // applied to [U; 0] (columns up to the kept rank) to give core j = (Q U)^T.
        double* R = B.wd((size_t)q * q);
        double* Y = B.wd((size_t)q * q);
        double* Rc = B.wd((size_t)q * q);
        double* sig = B.wd(q);
        int* perm = B.wi(q);
        double* Tws = B.wd(qr_tws(p, q));
        double* Tws2 = B.wd(qr_tws(q, q));
        double* Bq = B.wd((size_t)p * q);           // [U; 0], then Q [U; 0]
        cpX.push_back(cd2(Cj, X, q, p, 1, yc, p, 1));
        qr.push_back({p, q, X, p, nullptr, 0, R, q, Tws, 0, rk1, n, nullptr, 0, Y, q});   // and Y = R1^T
        // R1 has rows >= n r' zero, so R1^T has those columns zero and R2^T those rows
        qr2.push_back({q, q, Y, q, nullptr, 0, Rc, q, Tws2, 1, nullptr, 0, rk1, n});   // R2^T into Rc
        jac.push_back({q, q, Rc, q, nullptr, 0, sig, perm, info, rk1, n});
        tr.push_back({sig, perm, q, rank});
        sel.push_back({Rc, q, sig, perm, rank, q, q, q, Bq, p, 1, p});   // [U; 0]: rows q .. p-1 zeroed
        g2.push_back(gd(q, q, q, R, q, 1, Bq, 1, p, T1, 1, q));
        g2.back().n_dev = rank;                       // U is zero beyond the kept rank
        qa.push_back({p, q, X, p, Tws, Bq, p, q, rank, rk1, n});
        cpW.push_back(cd2(Bq, y->core(t, j), p, q, 1, p, yc, 1));
      } else {
        // M = Q1 R1 (q > p, Q1 not formed); one-sided Jacobi on R1^T (p x p) gives V Sigma
        // in its columns: core j <- V^T (normalised columns, exactly orthonormal up to the
        // rotation threshold), and the factor absorbed into core j-1 is M V = U Sigma.
        double* Rc = B.wd((size_t)p * p);
        double* sig = B.wd(p);
        int* perm = B.wi(p);
        double* Tws = B.wd(qr_tws(q, p));
        double* Vt = B.wd((size_t)p * q);
        cpX.push_back(cd2(Cj, X, q, p, 1, yc, 1, q));
        // columns >= n r' zero; R1 written transposed: Rc = R1^T
        qr.push_back({q, p, X, q, nullptr, 0, Rc, p, Tws, 1, nullptr, 0, rk1, n});
        jac.push_back({p, p, Rc, p, nullptr, 0, sig, perm, info, rk1, n});   // rows >= n r' zero
        tr.push_back({sig, perm, p, rank});
        sel.push_back({Rc, p, sig, perm, rank, p, q, p, Vt, p, 1});
        cpW.push_back(cd2(Vt, y->core(t, j), p, q, 1, p, yc, 1));
        g2.push_back(gd(q, q, p, Cj, 1, yc, Vt, 1, p, T1, 1, q));   // M V
        g2.back().n_dev = rank;                       // Vt is zero beyond the kept rank
      }
      g3.push_back(gd(ml, q, q, y->core(t, j - 1), 1, ml, T1, 1, q, T2, 1, ml));
      g3.back().n_dev = rank;                         // T1 is zero beyond the kept rank
      if (j == 1) cpT2.push_back(cd2(T2, y->core(t, j - 1), ml, q, 1, ml, 1, ml));
    }
    B.copy(cpX);
    B.qr(qr);
    B.qr(qr2);
    B.jacobi(jac);
    B.trunc(tr, tol, rmax);
    B.select(sel);
    B.gemm(g2);      // reads U (p >= q) or Cj (p < q; core j itself at the first bond) before
                     // qapply / cpW overwrite them
    B.qapply(qa);
    B.copy(cpW);
    B.gemm(g3);
    B.copy(cpT2);
    B.release(mk);
  }
  B.release(mark0);
}

// Early exit of _tt_rounding (src/tt_rounding.jl:179-181): norm(core N) < tol.
void emit_zero_check(Builder& B, ttc_batch* y, const std::vector<int>& tts, int core, double tol) {
  std::vector<NormDesc> nd;
  std::vector<ZeroChkDesc> zc;
  for (int t : tts) {
    double* s = B.wd(1);
    const int k = core;
    nd.push_back({y->core(t, k), (long long)y->capr(t, k) * y->dims[k] * y->capr(t, k + 1), s});
    zc.push_back({s, y->d_zero + t, tol});
  }
  B.sumsq(nd);
  B.zerochk(zc);
}

void emit_finalize(Builder& B, ttc_batch* y, const std::vector<int>& tts, const std::vector<std::vector<int>>& rp) {
  std::vector<FinalDesc> v;
  for (size_t i = 0; i < tts.size(); ++i) {
    const int t = tts[i];
    v.push_back({y->d_zero + t, y->core(t, 0), y->tt_off[t + 1] - y->tt_off[t], y->drk(t, 0), B.const_ints(rp[i]),
                 y->N + 1});
  }
  B.finalize(v);
}

std::vector<int> orth_left_ranks(const ttc_batch* x, int t) {
  const int N = x->N;
  std::vector<int> r(N + 1, 1);
  for (int k = 0; k + 1 < N; ++k) r[k + 1] = (int)std::min<long long>((long long)x->dims[k] * r[k], x->rk(t, k + 1));
  r[N] = 1;
  return r;
}

bool is_left_orth(const ttc_batch* x, int t) {
  for (int k = 0; k + 1 < x->N; ++k)
    if (x->h_ot[(size_t)t * x->N + k] != 1) return false;
  return true;
}

// ---------------------------------------------------------------- deterministic rounding
void round_det(ttc_context* c, ttc_batch* x, const ttc_round_opts& o, ttc_batch* y) {
  TTC_REQUIRE(o.direction == TTC_DIR_LEFT || o.direction == TTC_DIR_RIGHT, TTC_EARG,
              "Invalid direction. Use direction=:right or direction=:left");
  TTC_REQUIRE(o.direction == TTC_DIR_LEFT, TTC_EARG, "direction=:right is served by the host wrapper (reversal)");
  TTC_REQUIRE(x != y, TTC_EARG, "round: input and output batches must differ");
  TTC_REQUIRE(y->count == x->count && y->N == x->N && y->dims == x->dims, TTC_EDIM, "round: output batch shape differs");
  batch_sync_ranks(x);
  const int N = x->N;
  std::vector<int> all, orth, keep;
  std::vector<std::vector<int>> rp_all, rp_orth, rp_keep;
  for (int t = 0; t < x->count; ++t) {
    all.push_back(t);
    std::vector<int> r;
    if (is_left_orth(x, t)) {
      r.assign(x->h_rks.begin() + (size_t)t * (N + 1), x->h_rks.begin() + (size_t)(t + 1) * (N + 1));
      keep.push_back(t);
      rp_keep.push_back(r);
    } else {
      r = orth_left_ranks(x, t);
      orth.push_back(t);
      rp_orth.push_back(r);
    }
    for (int k = 0; k <= N; ++k)
      TTC_REQUIRE(y->capr(t, k) >= r[k], TTC_EDIM, "round: output capacity below the orthogonalised ranks");
    rp_all.push_back(r);
  }
  char kb[128];
  snprintf(kb, sizeof kb, "det:%.17g:%lld:", o.tol, (long long)o.rmax);
  const std::string key = std::string(kb) + batch_key(x) + batch_out_key(y);
  Plan* p = get_plan(c, key, [&](Builder& B) {
    B.stage(0);
    emit_zero_tts(B, y, all);
    emit_set_ranks(B, y, all, rp_all);
    emit_copy_tts(B, x, y, keep, rp_keep);
    emit_orth_left(B, x, y, orth, rp_orth);
    B.stage(1);
    emit_zero_check(B, y, all, N - 1, o.tol);
    emit_svd_left(B, y, all, rp_all, o.tol, o.rmax);
    emit_finalize(B, y, all, rp_all);
    B.stage(2);
  });
  run_plan(c, *p);
  for (int t = 0; t < y->count; ++t)
    for (int k = 0; k < N; ++k) y->h_ot[(size_t)t * N + k] = (k == 0) ? 0 : -1;
  for (int t = 0; t < y->count; ++t)
    for (int k = 0; k <= N; ++k) y->h_rks[(size_t)t * (N + 1) + k] = rp_all[t][k];
  y->rks_dirty = true;
  y->version++;
}

// ---------------------------------------------------------------- reverse sketch
// Sketch blocks of the reverse recursive sketch (src/sketches.jl:44-84, :186-198).
SketchPlan sketch_plan(const std::vector<long long>& dims, const std::vector<long long>& rks, long long block_rks) {
  const int N = (int)dims.size();
  SketchPlan sp;
  sp.b.assign(N + 1, 1);
  for (int k = 0; k < N; ++k) sp.b[k] = block_rks <= 0 ? N : (int)block_rks;
  sp.b[N] = 1;
  for (int k = N - 1; k >= 0; --k) sp.b[k] = (int)std::min<long long>(sp.b[k], dims[k] * sp.b[k + 1]);
  sp.p.assign(N + 1, 1);
  for (int k = 0; k <= N; ++k) sp.p[k] = (int)((rks[k] + sp.b[k] - 1) / sp.b[k]);
  for (int i = 1; i < N; ++i) sp.p[i] = std::max(sp.p[i], sp.p[i - 1]);
  sp.p[N] = 1;
  sp.s.resize(N + 1);
  for (int k = 0; k <= N; ++k) sp.s[k] = sp.b[k] * sp.p[k];
  return sp;
}

// Emit the draws of sketch blocks (src/sketches.jl:44-84): for site k, p blocks of shape
// (left, n, right) in the Julia layout, from the Philox stream (seed, k); orthogonal blocks are
// the Q factors of the (left n x right) Gaussian blocks scaled by sqrt(left n / right), or the
// identity when right == left n; Gaussian blocks are scaled by 1/sqrt(right).
void emit_block_draws(Builder& B, const std::vector<BlockShape>& sh, const ttc_sketch_opts& o, std::vector<double*>& raw) {
  const int N = (int)sh.size();
  raw.assign(N, nullptr);
  std::vector<PhiloxDesc> ph;
  std::vector<QRDesc> qr;
  std::vector<CopyDesc> cpQ;
  std::vector<ZeroDesc> zr;
  for (int k = 0; k < N; ++k) {
    const long long bl = sh[k].left, n = sh[k].n, br = sh[k].right, pk = sh[k].p;
    const long long cnt = bl * n * br * pk;
    raw[k] = B.wd(cnt);
    const bool orth = o.orthogonal != 0;
    const bool ident = orth && (br == bl * n);
    if (ident) {
      // identity 'sketch' (src/sketches.jl:58-65): block[i,i,j] = 1
      zr.push_back({raw[k], cnt});
      CopyDesc c{};   // write ones on the diagonal: src = the device constant 1.0 with zero strides
      c.src = B.ctx->d_one; c.dst = raw[k];
      c.ext[0] = br; c.ext[1] = pk; c.ext[2] = 1; c.ext[3] = 1;
      c.ss[0] = 0; c.ss[1] = 0;
      c.ds[0] = bl * n + 1; c.ds[1] = bl * n * br;
      c.alpha = 1.0;
      cpQ.push_back(c);
      continue;
    }
    const double scale = orth ? 1.0 : 1.0 / std::sqrt((double)br);
    ph.push_back({raw[k], cnt, (unsigned long long)o.seed, (unsigned)k, scale});
    if (orth) {
      // QR of each (bl*n x br) block, Q scaled by sqrt(bl*n/br) (src/sketches.jl:71-78)
      for (long long j = 0; j < pk; ++j) {
        double* A = raw[k] + j * bl * n * br;
        double* Qd = B.wd(bl * n * br);
        double* Tws = B.wd(qr_tws((int)(bl * n), (int)br));
        qr.push_back({(int)(bl * n), (int)br, A, (int)(bl * n), Qd, (int)(bl * n), nullptr, 0, Tws});
        cpQ.push_back(cd2(Qd, A, bl * n, br, 1, bl * n, 1, bl * n, std::sqrt((double)(bl * n) / (double)br)));
      }
    }
  }
  B.philox(ph);
  B.zero(zr);
  B.qr(qr);
  B.copy(cpQ);
}

// Emit generation of the raw sketch blocks of the reverse sketch (Julia layout
// (b_{k+1}, n, b_k, p_k)) into raw[k] and their permutation into the GEMM layout
// (n, b_{k+1}, b_k, p_k) in S[k].
void emit_sketch_blocks(Builder& B, const std::vector<long long>& dims, const SketchPlan& sp, const ttc_sketch_opts& o,
                        const std::vector<const double*>& host_raw, std::vector<double*>& S) {
  const int N = (int)dims.size();
  S.assign(N, nullptr);
  std::vector<double*> raw(N, nullptr);
  std::vector<CopyDesc> cpS;
  for (int k = 0; k < N; ++k) S[k] = B.wd((size_t)sp.b[k + 1] * dims[k] * sp.b[k] * sp.p[k]);
  if (!host_raw.empty()) {
    for (int k = 0; k < N; ++k) raw[k] = const_cast<double*>(host_raw[k]);
  } else {
    std::vector<BlockShape> sh(N);
    for (int k = 0; k < N; ++k) sh[k] = {sp.b[k + 1], (int)dims[k], sp.b[k], sp.p[k]};
    emit_block_draws(B, sh, o, raw);
  }
  for (int k = 0; k < N; ++k) {
    const long long bl = sp.b[k + 1], n = dims[k], br = sp.b[k], pk = sp.p[k];
    // raw (be, z, b, j) at be + bl*(z + n*(b + br*j))  ->  S (z, be, (b, j)) at z + n*be + n*bl*(b + br*j)
    cpS.push_back(cd3(raw[k], S[k], bl, n, br * pk, 1, bl, bl * n, n, 1, n * bl));
  }
  B.copy(cpS);
}

// Reverse recursive sketch of every TT of x (src/sketches.jl:221-239) in FP64.  W[t][k] is
// the unscaled (r_k, b_k, p_k) array; the 1/sqrt(p_k) factor (src/sketches.jl:300-302) is
// applied by the consumers.  W[t][N] is the constant 1.
void emit_sketch_f64(Builder& B, ttc_batch* x, const std::vector<int>& tts, const SketchPlan& sp,
                     const std::vector<double*>& S, std::vector<std::vector<double*>>& W) {
  const int N = x->N;
  W.assign(tts.size(), std::vector<double*>(N + 1, nullptr));
  for (size_t i = 0; i < tts.size(); ++i) {
    const int t = tts[i];
    for (int k = 0; k < N; ++k) W[i][k] = B.wd((size_t)x->rk(t, k) * sp.b[k] * sp.p[k]);
    W[i][N] = B.ctx->d_one;
  }
  for (int k = N - 1; k >= 0; --k) {
    const size_t mk = B.mark();
    std::vector<GemmDesc> g1, g2;
    const int n = (int)x->dims[k];
    const int bl = sp.b[k + 1], br = sp.b[k], pk = sp.p[k];
    for (size_t i = 0; i < tts.size(); ++i) {
      const int t = tts[i];
      const int r0 = x->rk(t, k), r1 = x->rk(t, k + 1), xc = x->capr(t, k);
      double* Tm = B.wd((size_t)r0 * n * bl * pk);
      // T[(a,z), be] = sum_al A_k[a, z, al] W_{k+1}[al, be, j]
      GemmDesc d = gd(r0 * n, bl, r1, x->core(t, k), 1, (long long)xc * n, W[i][k + 1], 1, r1, Tm, 1,
                      (long long)r0 * n);
      d.m0 = r0; d.a_i0 = 1; d.a_i1 = xc;                       // rows a + r0*z inside the capacity slab
      d.c_i0 = 1; d.c_i1 = r0;                                  // packed rows of T
      d.batch = pk;
      d.a_b = 0;
      d.b_b = (k < N - 1) ? (long long)r1 * bl : 0;
      d.c_b = (long long)r0 * n * bl;
      g1.push_back(d);
      // W_k[a, b, j] = sum_{z, be} T[a, z, be] S[z, be, b, j]
      GemmDesc e = gd(r0, br, n * bl, Tm, 1, r0, S[k], 1, (long long)n * bl, W[i][k], 1, r0);
      e.batch = pk;
      e.a_b = (long long)r0 * n * bl;
      e.b_b = (long long)n * bl * br;
      e.c_b = (long long)r0 * br;
      g2.push_back(e);
    }
    B.gemm(g1);
    B.gemm(g2);
    B.release(mk);
  }
}

// Left-to-right orthogonalise-and-project sweep of ttrand_rounding (src/tt_randtools.jl:123-151):
// Z = y_k W_{k+1}, Q = qr(Z) (thin Householder Q), core k = Q, y_{k+1} = Q^T y_k A_{k+1}.
//
// y_k is kept compact: only its first e_k left indices can be nonzero (e_0 = 1), stored as
// (e_k, n, r_{k+1}), so its unfolding Y is m x c with m = n e_k and c = r_{k+1}.  Z = Y W has
// rank q <= min(m, c, s) (s = sketch rank of bond k+1), and the Householder QR of Z is formed
// three ways, all giving the same first q columns (up to the reflectors' sign convention, which
// is LAPACK's in each QR):
//  * F (q = s: Z has full column rank, the randomized compression case): Z is formed and
//    factored as the reference does.
//  * T (q = c < m, s: more sketch columns than Y has columns): Z = Y W = Q1 (R1 W).  Householder
//    QR of Z factors its columns left to right, so its first c columns are the QR of
//    Z[:, :c] = Q1 M1 with M1 = R1 W[:, :c]: Q1 Q_M, Q_M the Q of the c x c matrix M1.  The
//    columns beyond c (Z's numerical null space: there LAPACK orthonormalises rounding noise)
//    are completed deterministically: the reflectors of Y applied to unit vectors, then unit
//    vectors in y_k's zero rows.
//  * W (q = m <= c, m < s): Q1 = I, M1 = Y W[:, :m], and core k's first m columns are Q_M.
// Then Q^T y_k = [Q_M^T R1; 0] (T) or [Q_M^T Y; 0] (W): y_{k+1} has e_{k+1} = q nonzero rows.
// The represented tensor is the reference's: range(Q) contains range(y_k), and the completion
// columns meet zero rows of y_{k+1}.  When the truncated-SVD sweep follows in the same plan
// (`complete` false) the completion columns are not written: the sweep reads cores only up to
// the effective ranks e, which `eff` returns, and the cores must stay zero beyond their ranks.
// The sweep then also needs only range(Q), not the reference's basis of it, and the T and W
// levels take their reduced forms: core k = Q1 with Q^T y_k = R1 (T), core k = I_m with
// Q^T y_k = Y (W).  range(Q1 Q_M) = range(Q1) and range(Q_M) = R^m, so the represented tensor
// and every singular value the SVD sweep sees are unchanged; the sketch is not read there.
void emit_rand_sweep(Builder& B, ttc_batch* x, ttc_batch* y, const std::vector<int>& tts, const SketchPlan& sp,
                     const std::vector<std::vector<double*>>& W, const std::vector<std::vector<int>>& rho,
                     bool complete, std::vector<std::vector<int>>* eff) {
  const int N = x->N;
  const size_t T = tts.size();
  std::vector<double*> Y(T), Yn(T);
  std::vector<int> e(T, 1);
  if (eff) eff->assign(T, std::vector<int>(N + 1, 1));
  const size_t mark0 = B.mark();
  for (size_t i = 0; i < T; ++i) {
    const int t = tts[i];
    size_t mx = 1;
    for (int k = 0; k < N; ++k)
      mx = std::max(mx, (size_t)((long long)rho[i][k] * x->dims[k] * x->rk(t, k + 1)));
    Y[i] = B.wd(mx);
    Yn[i] = B.wd(mx);
  }
  // unit vectors of core k's completion in the rows of y_k that are zero (left index >= e):
  // columns col0 .. col0 + cnt - 1, rows taken left index fastest
  auto outside_units = [&](std::vector<CopyDesc>& v, double* core, int e_, int rh, int n, int yc, long long col0,
                           long long cnt) {
    const long long per = rh - e_;
    if (cnt <= 0 || per <= 0) return;
    const long long full = cnt / per, rem = cnt % per;
    const long long cs = (long long)yc * n;          // column stride of the core's left unfolding
    CopyDesc c{};
    c.src = B.ctx->d_one;
    c.alpha = 1.0;
    c.ext[2] = c.ext[3] = 1;
    if (full > 0) {
      c.dst = core + e_ + cs * col0;
      c.ext[0] = per; c.ext[1] = full;
      c.ds[0] = 1 + cs; c.ds[1] = yc + cs * per;
      v.push_back(c);
    }
    if (rem > 0) {
      c.dst = core + e_ + (long long)yc * full + cs * (col0 + full * per);
      c.ext[0] = rem; c.ext[1] = 1;
      c.ds[0] = 1 + cs; c.ds[1] = 0;
      v.push_back(c);
    }
  };
  for (int k = 0; k + 1 < N; ++k) {
    const size_t mk = B.mark();
    std::vector<CopyDesc> cp0, cpQ, cpC;
    std::vector<QRDesc> qrY, qrZ;
    std::vector<GemmDesc> gz, gp, gy;
    std::vector<ZeroDesc> zb;
    std::vector<QApplyDesc> qa;
    const int n = (int)x->dims[k], nn = (int)x->dims[k + 1];
    const int s = sp.s[k + 1];
    const double wscale = 1.0 / std::sqrt((double)sp.p[k + 1]);
    for (size_t i = 0; i < T; ++i) {
      const int t = tts[i];
      const int rh = rho[i][k], rhn = rho[i][k + 1], c = x->rk(t, k + 1), r2 = x->rk(t, k + 2);
      const int m = n * e[i];
      const int q = std::min(std::min(m, c), s);
      const int yc = y->capr(t, k);
      double* core = y->core(t, k);
      // Y: m x c with leading dimension m (k = 0: core 0 of x, whose left capacity is 1)
      const double* Yk = (k == 0) ? x->core(t, 0) : Y[i];
      const long long yld = (k == 0) ? (long long)x->capr(t, 0) * n : m;
      const double* Wk = W[i][k + 1];                 // r_{k+1} x s, leading dimension r_{k+1}
      double* P = nullptr;                             // Q^T y_k, its q nonzero rows (leading dimension pld)
      long long pld = q;
      // core k has the layout of an m-row factor with column stride m when its left capacity is
      // e: a Q is then written there by its QR, not copied
      const bool in_core = (yc == e[i]);
      if (q == s) {                                    // F
        P = B.wd((size_t)q * c);
        double* Z = B.wd((size_t)m * s);
        double* Q = in_core ? core : B.wd((size_t)m * s);
        double* Tws = B.wd(qr_tws(m, s));
        gz.push_back(gd(m, s, c, Yk, 1, yld, Wk, 1, c, Z, 1, m, wscale));
        qrZ.push_back({m, s, Z, m, Q, m, nullptr, 0, Tws});
        if (!in_core) cpC.push_back(cd3(Q, core, e[i], n, s, 1, e[i], (long long)e[i] * n, 1, yc, (long long)yc * n));
        gp.push_back(gd(s, c, m, Q, m, 1, Yk, 1, yld, P, 1, s));
      } else if (q == c && !complete) {                // T, reduced: core k = Q1, Q^T y_k = R1
        double* Yw = const_cast<double*>(Yk);
        if (k == 0) {
          Yw = B.wd((size_t)m * c);
          cp0.push_back(cd2(Yk, Yw, m, c, 1, yld, 1, m));
        }
        double* Q1 = in_core ? core : B.wd((size_t)m * c);
        P = B.wd((size_t)c * c);
        qrY.push_back({m, c, Yw, m, Q1, m, P, c, B.wd(qr_tws(m, c))});
        if (!in_core) cpC.push_back(cd3(Q1, core, e[i], n, c, 1, e[i], (long long)e[i] * n, 1, yc, (long long)yc * n));
      } else if (q == c) {                             // T: c < m, c < s
        double* Yw = const_cast<double*>(Yk);
        if (k == 0) {                                  // the QR overwrites its input: not x's core
          Yw = B.wd((size_t)m * c);
          cp0.push_back(cd2(Yk, Yw, m, c, 1, yld, 1, m));
        }
        P = B.wd((size_t)q * c);
        double* R1 = B.wd((size_t)c * c);
        double* M1 = B.wd((size_t)c * c);
        double* QM = B.wd((size_t)c * c);
        double* TwsY = B.wd(qr_tws(m, c));
        double* TwsM = B.wd(qr_tws(c, c));
        const int ncols = complete ? std::min(m, rhn) : c;
        double* Bq = B.wd((size_t)m * ncols);
        qrY.push_back({m, c, Yw, m, nullptr, 0, R1, c, TwsY});
        gz.push_back(gd(c, c, c, R1, 1, c, Wk, 1, c, M1, 1, c, wscale));
        qrZ.push_back({c, c, M1, c, QM, c, nullptr, 0, TwsM});
        zb.push_back({Bq, (long long)m * ncols});
        cpQ.push_back(cd2(QM, Bq, c, c, 1, c, 1, m));
        if (ncols > c) {                               // unit vectors e_c .. e_{ncols-1}
          CopyDesc u{};
          u.src = B.ctx->d_one; u.dst = Bq + c + (long long)m * c; u.alpha = 1.0;
          u.ext[0] = ncols - c; u.ext[1] = u.ext[2] = u.ext[3] = 1;
          u.ds[0] = (long long)m + 1;
          cpQ.push_back(u);
        }
        qa.push_back({m, c, Yw, m, TwsY, Bq, m, ncols, nullptr, nullptr, 0});
        cpC.push_back(cd3(Bq, core, e[i], n, ncols, 1, e[i], (long long)e[i] * n, 1, yc, (long long)yc * n));
        if (complete) outside_units(cpC, core, e[i], rh, n, yc, ncols, (long long)rhn - ncols);
        gp.push_back(gd(c, c, c, QM, c, 1, R1, 1, c, P, 1, c));
      } else if (!complete) {                          // W, reduced: core k = I_m, Q^T y_k = Y
        CopyDesc u{};
        const long long cs = (long long)yc * n;        // column stride of the core's left unfolding
        u.src = B.ctx->d_one; u.dst = core; u.alpha = 1.0;
        u.ext[0] = e[i]; u.ext[1] = n; u.ext[2] = u.ext[3] = 1;
        u.ds[0] = 1 + cs; u.ds[1] = yc + cs * e[i];    // row (a, z) -> column a + e z
        cpC.push_back(u);
        P = const_cast<double*>(Yk);
        pld = yld;
      } else {                                         // W: q = m <= c, m < s
        P = B.wd((size_t)q * c);
        double* M1 = B.wd((size_t)m * m);
        double* QM = in_core ? core : B.wd((size_t)m * m);
        double* TwsM = B.wd(qr_tws(m, m));
        gz.push_back(gd(m, m, c, Yk, 1, yld, Wk, 1, c, M1, 1, m, wscale));
        qrZ.push_back({m, m, M1, m, QM, m, nullptr, 0, TwsM});
        if (!in_core) cpC.push_back(cd3(QM, core, e[i], n, m, 1, e[i], (long long)e[i] * n, 1, yc, (long long)yc * n));
        if (complete) outside_units(cpC, core, e[i], rh, n, yc, m, (long long)rhn - m);
        gp.push_back(gd(m, c, m, QM, m, 1, Yk, 1, yld, P, 1, m));
      }
      // y_{k+1} = P A_{k+1}: (q, nn, r_{k+2}) compact
      gy.push_back(gd(q, nn * r2, c, P, 1, pld, x->core(t, k + 1), 1, x->capr(t, k + 1), Yn[i], 1, q));
      e[i] = q;
      if (eff) (*eff)[i][k + 1] = q;
    }
    B.copy(cp0);
    B.qr(qrY);
    B.gemm(gz);
    B.qr(qrZ);
    B.zero(zb);
    B.copy(cpQ);
    B.qapply(qa);
    B.copy(cpC);
    B.gemm(gp);
    B.gemm(gy);
    std::swap(Y, Yn);
    B.release(mk);
  }
  std::vector<CopyDesc> cp;
  for (size_t i = 0; i < T; ++i) {
    const int t = tts[i];
    const int n = (int)x->dims[N - 1], yc = y->capr(t, N - 1);
    const double* src = (N == 1) ? x->core(t, 0) : Y[i];
    cp.push_back(cd2(src, y->core(t, N - 1), e[i], n, 1, e[i], 1, yc));
  }
  B.copy(cp);
  B.release(mark0);
}

// Whether any level of emit_rand_sweep over the TTs `tts` of x takes the F form (q = s: the
// sketch rank is below both of Y's dimensions, so the range finder compresses).  Follows the
// sweep's effective ranks e on the host: e_0 = 1, e_{k+1} = min(n_k e_k, r_{k+1}, s_{k+1}).
bool sketch_compresses(const ttc_batch* x, const std::vector<int>& tts, const SketchPlan& sp) {
  const int N = x->N;
  for (int t : tts) {
    long long e = 1;
    for (int k = 0; k + 1 < N; ++k) {
      const long long m = x->dims[k] * e, c = x->rk(t, k + 1), s = sp.s[k + 1];
      const long long q = std::min(std::min(m, c), s);
      if (q == s) return true;
      e = q;
    }
  }
  return false;
}

std::vector<int> rand_out_ranks(const std::vector<long long>& dims, const SketchPlan& sp) {
  const int N = (int)dims.size();
  std::vector<int> r(N + 1, 1);
  for (int k = 0; k + 1 < N; ++k) r[k + 1] = (int)std::min<long long>(dims[k] * r[k], sp.s[k + 1]);
  r[N] = 1;
  return r;
}

void round_rand(ttc_context* c, ttc_batch* x, const std::vector<long long>& rks, const ttc_sketch_opts& o,
                const ttc_round_opts* after, ttc_batch* y, const std::vector<const double*>& host_raw,
                const std::string& raw_key) {
  TTC_REQUIRE(x != y, TTC_EARG, "round: input and output batches must differ");
  TTC_REQUIRE(y->count == x->count && y->N == x->N && y->dims == x->dims, TTC_EDIM, "round: output batch shape differs");
  check_precision(o.precision);
  const int N = x->N;
  TTC_REQUIRE((int)rks.size() == N + 1, TTC_EDIM, "ttrand_rounding: rks must have length N+1");
  TTC_REQUIRE(rks[N] == 1, TTC_EDIM, "ttrand_rounding: rks[N+1] must be 1");
  batch_sync_ranks(x);
  for (int t = 0; t < x->count; ++t)
    TTC_REQUIRE(x->rk(t, N) == 1, TTC_EDIM, "ttrand_rounding: the last TT rank must be 1");
  const SketchPlan sp = sketch_plan(x->dims, rks, o.block_rks);
  if (o.orthogonal)
    for (int k = 0; k < N; ++k)
      TTC_REQUIRE(sp.b[k] <= (long long)x->dims[k] * sp.b[k + 1], TTC_EARG, "generate_sketch_blocks: right_rank > dim*left_rank");
  const std::vector<int> rho = rand_out_ranks(x->dims, sp);
  std::vector<int> all;
  std::vector<std::vector<int>> rho_all;
  for (int t = 0; t < x->count; ++t) {
    all.push_back(t);
    rho_all.push_back(rho);
    for (int k = 0; k <= N; ++k)
      TTC_REQUIRE(y->capr(t, k) >= rho[k], TTC_EDIM, "ttrand_rounding: output capacity below the sketch ranks");
  }
  char kb[256];
  snprintf(kb, sizeof kb, "rand:%d:%llu:%lld:%d:%d:%.17g:%lld:", o.orthogonal, (unsigned long long)o.seed,
           (long long)o.block_rks, o.precision, after ? 1 : 0, after ? after->tol : 0.0, after ? (long long)after->rmax : 0LL);
  std::string key = std::string(kb) + raw_key + batch_key(x) + batch_out_key(y);
  for (long long r : rks) key += std::to_string(r) + ",";
  // With the SVD sweep following, only F levels read the sketch (the reduced T and W forms of
  // emit_rand_sweep do not): without one, the sketch is not computed.
  const bool need_sketch = !after || sketch_compresses(x, all, sp);
  Plan* p = get_plan(c, key, [&](Builder& B) {
    B.stage(0);
    emit_zero_tts(B, y, all);
    emit_set_ranks(B, y, all, rho_all);
    std::vector<std::vector<double*>> W(all.size(), std::vector<double*>(N + 1, nullptr));
    if (need_sketch) {
      std::vector<double*> S;
      emit_sketch_blocks(B, x->dims, sp, o, host_raw, S);
      if (tensor_core_sketch(o.precision)) emit_sketch_bf16(B, x, all, sp, S, W, o.precision == TTC_PREC_TF32);
      else emit_sketch_f64(B, x, all, sp, S, W);
    }
    B.stage(1);
    std::vector<std::vector<int>> eff;
    emit_rand_sweep(B, x, y, all, sp, W, rho_all, after == nullptr, &eff);
    B.stage(2);
    if (after) {
      emit_zero_check(B, y, all, N - 1, after->tol);
      emit_svd_left(B, y, all, eff, after->tol, after->rmax);
      emit_finalize(B, y, all, rho_all);
    }
    B.stage(3);
  });
  run_plan(c, *p);
  for (int t = 0; t < y->count; ++t) {
    for (int k = 0; k < N; ++k) {
      int ot;
      if (after) ot = (k == 0) ? 0 : -1;
      else ot = (k < N - 1) ? 1 : 0;
      y->h_ot[(size_t)t * N + k] = ot;
    }
    for (int k = 0; k <= N; ++k) y->h_rks[(size_t)t * (N + 1) + k] = rho[k];
  }
  y->rks_dirty = after != nullptr;
  if (after) for (int t = 0; t < y->count; ++t) {}
  y->version++;
}

}  // namespace ttc
