// Streaming tensor-train approximation (STTA) of a TT or of a linear combination of TTs
// (src/tt_randtools.jl:551-641, src/sketches.jl:1126-1160; Kressner, Vandereycken and Voorhaar,
// SIAM J. Sci. Comput. 45(5), 2023).
//
// A forward recursive sketch W_L (left to right, block counts oversampled 1.5x) and a reverse one
// W_R of each term give, per bond k, the overlap Omega_k = W_L[k+1]^T W_R[k+1] (sl x sr) and,
// per core, Psi_k = x_k x_left W_L[k] x_right W_R[k+1] (sl_k, n, sr_{k+1}); the approximation
// joins the Psi cores through the pseudo-inverse of Omega_k on the side of the smaller sketch
// rank.  Everything runs in one plan on the device:
//   * forward and reverse sketch blocks (Philox streams seed_left / seed_right, one per core);
//   * forward sketch: per core two grouped GEMMs, T = W_L[k]^T x_k, W_L[k+1] = T S_k;
//   * Omega and Psi: grouped GEMMs, accumulated over the terms of a combination;
//   * pinv(Omega_k) (src/tt_randtools.jl:485-489): one-sided Jacobi SVD with the right singular
//     vectors accumulated, columns A V scaled by 1/sigma^2 (zero below 1e-12 sigma_max), one GEMM;
//   * the joins: left multiplications, then right ones (they act on different sides of a core,
//     so every bond's join is one launch).
// The internal core layout is the device batch's (left rank, n, right rank).
#include <algorithm>
#include <cmath>

#include "api_impl.cuh"

namespace ttc {

namespace {
void run_plan_once(ttc_context* c, const std::function<void(Builder&)>& fn) {
  static unsigned long long serial = 0;
  const std::string key = "stta:" + std::to_string(++serial);
  Plan* p = get_plan(c, key, fn);
  run_plan(c, *p);
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  c->plans.erase(key);
  check_device_flags(c);
}
}  // namespace

// Block structure of the forward recursive sketch (src/sketches.jl:243-258): b_0 = 1,
// b_{k+1} = min(block_rks, n_k b_k); p = ceil(rks ./ b), made non-increasing left to right,
// p_0 = 1, then p_{1..N} scaled by `oversampling` (rounded up).
SketchPlan sketch_plan_fwd(const std::vector<long long>& dims, const std::vector<long long>& rks, long long block_rks,
                           double oversampling) {
  const int N = (int)dims.size();
  SketchPlan sp;
  sp.b.assign(N + 1, 1);
  for (int k = 1; k <= N; ++k) sp.b[k] = block_rks <= 0 ? N : (int)block_rks;
  for (int k = 0; k < N; ++k) sp.b[k + 1] = (int)std::min<long long>(sp.b[k + 1], dims[k] * sp.b[k]);
  sp.p.assign(N + 1, 1);
  for (int k = 0; k <= N; ++k) sp.p[k] = (int)((rks[k] + sp.b[k] - 1) / sp.b[k]);
  for (int i = N - 1; i >= 1; --i) sp.p[i] = std::max(sp.p[i], sp.p[i + 1]);
  sp.p[0] = 1;
  if (oversampling != 1.0)
    for (int k = 1; k <= N; ++k) sp.p[k] = (int)std::ceil(oversampling * sp.p[k]);
  sp.s.resize(N + 1);
  for (int k = 0; k <= N; ++k) sp.s[k] = sp.b[k] * sp.p[k];
  return sp;
}

// Forward recursive sketch (src/sketches.jl:260-297) of the TTs `tts` of x in FP64: W[i][k+1] =
// sum over the blocks j of W[i][k][:, :, j]^T-contracted core k and block j of site k, as the
// unscaled (r_{k+1}, b_{k+1}, p_{k+1}) array (the 1/sqrt(p) factors are the consumers').  W[i][0]
// is the constant 1.  raw[k] holds site k's blocks in the Julia layout (b_k, n, b_{k+1}, p_{k+1}).
void emit_sketch_fwd_f64(Builder& B, ttc_batch* x, const std::vector<int>& tts, const SketchPlan& sp,
                         const std::vector<double*>& raw, std::vector<std::vector<double*>>& W) {
  const int N = x->N;
  W.assign(tts.size(), std::vector<double*>(N + 1, nullptr));
  for (size_t i = 0; i < tts.size(); ++i) {
    W[i][0] = B.ctx->d_one;
    for (int k = 0; k < N; ++k) W[i][k + 1] = B.wd((size_t)x->rk(tts[i], k + 1) * sp.b[k + 1] * sp.p[k + 1]);
  }
  for (int k = 0; k < N; ++k) {
    const size_t mk = B.mark();
    std::vector<GemmDesc> g1, g2;
    const int n = (int)x->dims[k];
    const int bl = sp.b[k], br = sp.b[k + 1], pk = sp.p[k + 1];
    for (size_t i = 0; i < tts.size(); ++i) {
      const int t = tts[i];
      const int r0 = x->rk(t, k), r1 = x->rk(t, k + 1), xc = x->capr(t, k);
      double* Tm = B.wd((size_t)bl * n * r1 * pk);
      // T[be, (z, a), j] = sum_al W_k[al, be, j] A_k[al, z, a]
      GemmDesc d = gd(bl, n * r1, r0, W[i][k], r0, 1, x->core(t, k), 1, xc, Tm, 1, bl);
      d.batch = pk;
      d.a_b = (k > 0) ? (long long)r0 * bl : 0;
      d.b_b = 0;
      d.c_b = (long long)bl * n * r1;
      g1.push_back(d);
      // W_{k+1}[a, b, j] = sum_{be, z} T[be, z, a, j] S[be, z, b, j]
      GemmDesc e = gd(r1, br, bl * n, Tm, (long long)bl * n, 1, raw[k], 1, (long long)bl * n, W[i][k + 1], 1, r1);
      e.batch = pk;
      e.a_b = (long long)bl * n * r1;
      e.b_b = (long long)bl * n * br;
      e.c_b = (long long)r1 * br;
      g2.push_back(e);
    }
    B.gemm(g1);
    B.gemm(g2);
    B.release(mk);
  }
}

void stta_host(ttc_context* c, int m, const double* alpha, const ttc_ttv* ys, const int64_t* rks, uint64_t seed_left,
               uint64_t seed_right, int orthogonal, int64_t block_rks, ttc_ttv_out* y) {
  TTC_REQUIRE(m >= 1, TTC_EARG, "stta: empty combination");
  const int N = ys[0].N;
  for (int j = 0; j < m; ++j) {
    validate_ttv(&ys[j]);
    TTC_REQUIRE(ys[j].N == N, TTC_EDIM, "stta: terms differ in N");
    for (int k = 0; k < N; ++k) TTC_REQUIRE(ys[j].dims[k] == ys[0].dims[k], TTC_EDIM, "stta: terms differ in dims");
  }
  const auto r = rks_vec(rks, N);
  TTC_REQUIRE(r[0] == 1 && r[N] == 1, TTC_EDIM, "stta: boundary ranks must be 1");
  std::vector<long long> dims(ys[0].dims, ys[0].dims + N);
  const SketchPlan spR = sketch_plan(dims, r, block_rks);
  const SketchPlan spL = sketch_plan_fwd(dims, r, block_rks, 1.5);
  if (orthogonal)
    for (int k = 0; k < N; ++k) {
      TTC_REQUIRE(spR.b[k] <= dims[k] * spR.b[k + 1], TTC_EARG, "generate_sketch_blocks: right_rank > dim*left_rank");
      TTC_REQUIRE(spL.b[k + 1] <= dims[k] * spL.b[k], TTC_EARG, "generate_sketch_blocks: right_rank > dim*left_rank");
    }
  const std::vector<int>& sl = spL.s;
  const std::vector<int>& sr = spR.s;
  // ranks of the result: the smaller sketch rank of every bond
  std::vector<int> res(N + 1, 1);
  for (int k = 1; k < N; ++k) res[k] = std::min(sl[k], sr[k]);
  std::vector<int> cap;
  for (int j = 0; j < m; ++j)
    for (int k = 0; k <= N; ++k) cap.push_back((int)ys[j].rks[k]);
  BatchHolder BH;
  ttc_batch* X = BH.add(batch_create(c, m, N, dims.data(), cap.data()));
  batch_upload_many(X, 0, m, ys, false);
  ttc_batch* Y = BH.add(batch_create(c, 1, N, dims.data(), res.data()));
  ttc_sketch_opts skL{}, skR{};
  skL.orthogonal = skR.orthogonal = orthogonal;
  skL.block_rks = skR.block_rks = block_rks;
  skL.seed = seed_left;
  skR.seed = seed_right;
  std::vector<int> terms(m);
  for (int j = 0; j < m; ++j) terms[j] = j;

  run_plan_once(c, [&](Builder& B) {
    B.stage(0);
    emit_zero_tts(B, Y, {0});
    emit_set_ranks(B, Y, {0}, {res});
    std::vector<double*> SR, SLraw;
    emit_sketch_blocks(B, dims, spR, skR, {}, SR);
    std::vector<BlockShape> sh(N);
    for (int k = 0; k < N; ++k) sh[k] = {spL.b[k], (int)dims[k], spL.b[k + 1], spL.p[k + 1]};
    emit_block_draws(B, sh, skL, SLraw);
    std::vector<std::vector<double*>> WR, WL;
    emit_sketch_f64(B, X, terms, spR, SR, WR);
    emit_sketch_fwd_f64(B, X, terms, spL, SLraw, WL);
    B.stage(1);
    // Psi_k (sl_k, n, sr_{k+1}) and Omega_k (sl_{k+1} x sr_{k+1}), summed over the terms
    std::vector<double*> Psi(N), Om(N > 1 ? N - 1 : 0), U(N);
    for (int k = 0; k < N; ++k) {
      Psi[k] = B.wd((size_t)sl[k] * dims[k] * sr[k + 1]);
      size_t mx = 1;
      for (int j = 0; j < m; ++j) mx = std::max(mx, (size_t)X->rk(j, k) * (size_t)dims[k] * (size_t)sr[k + 1]);
      U[k] = B.wd(mx);
    }
    for (int k = 0; k + 1 < N; ++k) Om[k] = B.wd((size_t)sl[k + 1] * sr[k + 1]);
    for (int j = 0; j < m; ++j) {
      std::vector<GemmDesc> gu, gp, go;
      for (int k = 0; k < N; ++k) {
        const int n = (int)dims[k], r0 = X->rk(j, k), r1 = X->rk(j, k + 1), xc = X->capr(j, k);
        const double wsc = alpha[j] / std::sqrt((double)spL.p[k] * (double)spR.p[k + 1]);
        // U[(al, z), b] = sum_be A_k[al, z, be] W_R[k+1][be, b]
        GemmDesc d = gd(r0 * n, sr[k + 1], r1, X->core(j, k), 1, (long long)xc * n, WR[j][k + 1], 1, r1, U[k], 1,
                        (long long)r0 * n);
        d.m0 = r0; d.a_i0 = 1; d.a_i1 = xc; d.c_i0 = 1; d.c_i1 = r0;
        gu.push_back(d);
        // Psi[a, (z, b)] += sum_al W_L[k][al, a] U[al, (z, b)]
        gp.push_back(gd(sl[k], n * sr[k + 1], r0, WL[j][k], r0, 1, U[k], 1, r0, Psi[k], 1, sl[k], wsc,
                        j == 0 ? 0.0 : 1.0));
        if (k + 1 < N) {
          const double osc = alpha[j] / std::sqrt((double)spL.p[k + 1] * (double)spR.p[k + 1]);
          // Omega[a, b] += sum_be W_L[k+1][be, a] W_R[k+1][be, b]
          go.push_back(gd(sl[k + 1], sr[k + 1], r1, WL[j][k + 1], r1, 1, WR[j][k + 1], 1, r1, Om[k], 1, sl[k + 1],
                          osc, j == 0 ? 0.0 : 1.0));
        }
      }
      B.gemm(gu);
      B.gemm(gp);
      B.gemm(go);
    }
    B.stage(2);
    // pinv(Omega_k) (sr x sl): Jacobi on Omega (sl >= sr) or Omega^T, V accumulated
    std::vector<double*> P(N > 1 ? N - 1 : 0);
    std::vector<CopyDesc> cpx;
    std::vector<JacobiDesc> jac;
    std::vector<PinvScaleDesc> psc;
    std::vector<GemmDesc> gpi;
    int max_m = 1, max_n = 1;
    int* infos = B.diag_ints(std::max(N - 1, 1));
    for (int k = 0; k + 1 < N; ++k) {
      const int rl = sl[k + 1], rr = sr[k + 1];
      const bool tall = rl >= rr;
      const int mm = tall ? rl : rr, nn = tall ? rr : rl;
      double* Xk = B.wd((size_t)mm * nn);
      double* Vk = B.wd((size_t)nn * nn);
      double* sig = B.wd(nn);
      int* perm = B.wi(nn);
      P[k] = B.wd((size_t)rr * rl);
      if (tall) cpx.push_back(cd2(Om[k], Xk, rl, rr, 1, rl, 1, rl));
      else cpx.push_back(cd2(Om[k], Xk, rl, rr, 1, rl, rr, 1));           // Omega^T
      jac.push_back({mm, nn, Xk, mm, Vk, nn, sig, perm, infos + k, nullptr, 0});
      psc.push_back({Xk, mm, mm, nn, sig, 1e-12});
      // tall: P = V Xs^T (rr x rl); wide: P = Xs V^T (rr x rl)
      if (tall) gpi.push_back(gd(rr, rl, nn, Vk, 1, nn, Xk, rl, 1, P[k], 1, rr));
      else gpi.push_back(gd(rr, rl, nn, Xk, 1, rr, Vk, rl, 1, P[k], 1, rr));
      max_m = std::max(max_m, mm);
      max_n = std::max(max_n, nn);
    }
    B.copy(cpx);
    B.jacobi(jac);
    B.pinv_scale(psc);
    B.gemm(gpi);
    B.stage(3);
    // joins: core k takes P[k-1] on the left when bond k's sl >= sr, P[k] on the right when
    // bond k+1's sl < sr
    std::vector<double*> T(N);
    std::vector<GemmDesc> gl, gr;
    std::vector<CopyDesc> cpo;
    for (int k = 0; k < N; ++k) {
      const int n = (int)dims[k];
      const bool left = (k >= 1) && !(sl[k] < sr[k]);
      const bool right = (k + 1 < N) && (sl[k + 1] < sr[k + 1]);
      T[k] = Psi[k];
      if (left) {
        T[k] = B.wd((size_t)res[k] * n * sr[k + 1]);
        // T[a', (z, b)] = sum_a P[k-1][a', a] Psi[a, (z, b)]
        gl.push_back(gd(res[k], n * sr[k + 1], sl[k], P[k - 1], 1, res[k], Psi[k], 1, sl[k], T[k], 1, res[k]));
      }
      const int yc = Y->capr(0, k);
      if (right) {
        // Y_k[(a, z), b'] = sum_b T[(a, z), b] P[k][b, b']
        GemmDesc d = gd(res[k] * n, res[k + 1], sr[k + 1], T[k], 1, (long long)res[k] * n, P[k], 1, sr[k + 1],
                        Y->core(0, k), 1, (long long)yc * n);
        d.m0 = res[k]; d.a_i0 = 1; d.a_i1 = res[k]; d.c_i0 = 1; d.c_i1 = yc;
        gr.push_back(d);
      } else {
        cpo.push_back(cd3(T[k], Y->core(0, k), res[k], n, res[k + 1], 1, res[k], (long long)res[k] * n, 1, yc,
                          (long long)yc * n));
      }
    }
    B.gemm(gl);
    B.gemm(gr);
    B.copy(cpo);
    B.stage(4);
  });
  for (int k = 0; k < N; ++k) Y->h_ot[k] = 0;
  for (int k = 0; k <= N; ++k) Y->h_rks[k] = res[k];
  Y->rks_dirty = false;
  batch_download_many(Y, 0, 1, y, false);
}

}  // namespace ttc
