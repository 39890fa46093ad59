// Randomized rounding of a Hadamard (element-wise) product of TTs, ttrand_rounding(y::NTuple, rks)
// (src/tt_randtools.jl:364-473), without forming the product for its last factor.
//
// For M factors, the first M-1 are multiplied out on the device into P (slice-wise Kronecker cores,
// rank prod r_i, src/tt_operations.jl:273-287); the last factor B stays separate, and P (x) B is
// sketched and projected through structured contractions (the GEMM form of the Kronecker kernels,
// src/sketches.jl:1735-1881):
//   reverse sketch, site k, block j:  T1[(al, be), (z, c)] = W_{k+1}[(al, be), ga] S[ga, z, c]
//                                     T2[a, be, z, c]      = sum_al P_k[a, z, al] T1[al, be, z, c]
//                                     W_k[(a, b), c]       = sum_{be, z} T2[a, be, z, c] B_k[b, z, be]
//   projection: Qy = y_k^T Q, then   V[L, l2, rho]         = sum_l1 P_{k+1}[l1, z, L] Qy[(l1, l2), rho]
//                                     y_{k+1}[rho, z, (L, L2)] = sum_l2 V[L, l2, rho] B_{k+1}[l2, z, L2]
// with the range finder of the reference (Z = y_k W_{k+1}, Householder QR, core k = Q).  The
// combined rank index puts the first factor's index fastest.  Every step is a grouped GEMM.
#include <algorithm>
#include <cmath>

#include "api_impl.cuh"

namespace ttc {

namespace {
inline int qr_tws_h(int m, int n) { return ((std::min(m, n) + 15) / 16) * 256 + 256; }

void run_plan_once(ttc_context* c, const std::function<void(Builder&)>& fn) {
  static unsigned long long serial = 0;
  const std::string key = "hadamard:" + std::to_string(++serial);
  Plan* p = get_plan(c, key, fn);
  run_plan(c, *p);
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  c->plans.erase(key);
  check_device_flags(c);
}

// Outer products C[(a, b), z, (al, be)] = A[a, z, al] B[b, z, be] per z as K = 1 GEMMs: row index
// (a, al), column index (b, be), both split; A, B in the batch layout (left capacity ca / cb).
GemmDesc kron_core(const double* A, int ra, int ra1, int ca, const double* Bm, int rb, int rb1, int cb, int n,
                   double* C, long long ldc_left, long long ldc_right) {
  GemmDesc d{};
  d.m = ra * ra1; d.n = rb * rb1; d.k = 1; d.batch = n;
  d.m0 = ra; d.n0 = rb; d.k0e = 1;
  d.A = A; d.a_i0 = 1; d.a_i1 = (long long)ca * n; d.a_k0 = 0; d.a_b = ca;
  d.B = Bm; d.b_j0 = 1; d.b_j1 = (long long)cb * n; d.b_k0 = 0; d.b_b = cb;
  // C[(a + ra b) + ldc_left z + ldc_right (al + ra1 be)]
  d.C = C; d.c_i0 = 1; d.c_i1 = ldc_right; d.c_j0 = ra; d.c_j1 = ldc_right * ra1; d.c_b = ldc_left;
  d.alpha = 1.0; d.beta = 0.0;
  return d;
}
}  // namespace

void hadamard_rounding_host(ttc_context* c, int m, const ttc_ttv* ys, const int64_t* rks, const ttc_sketch_opts& sk,
                            ttc_ttv_out* y) {
  TTC_REQUIRE(m >= 2, TTC_EARG, "hadamard rounding: needs two or more factors");
  check_precision(sk.precision);
  TTC_REQUIRE(sk.precision == TTC_PREC_FP64, TTC_EARG, "hadamard rounding: FP64 sketch only");
  const int N = ys[0].N;
  for (int j = 0; j < m; ++j) {
    validate_ttv(&ys[j]);
    TTC_REQUIRE(ys[j].N == N, TTC_EDIM, "hadamard rounding: factors differ in N");
    for (int k = 0; k < N; ++k)
      TTC_REQUIRE(ys[j].dims[k] == ys[0].dims[k], TTC_EDIM, "hadamard rounding: factors differ in dims");
  }
  const auto r = rks_vec(rks, N);
  TTC_REQUIRE(r[N] == 1, TTC_EDIM, "ttrand_rounding: rks[N+1] must be 1");
  std::vector<long long> dims(ys[0].dims, ys[0].dims + N);
  const SketchPlan sp = sketch_plan(dims, r, sk.block_rks);
  if (sk.orthogonal)
    for (int k = 0; k < N; ++k)
      TTC_REQUIRE(sp.b[k] <= dims[k] * sp.b[k + 1], TTC_EARG, "generate_sketch_blocks: right_rank > dim*left_rank");
  // ranks of the formed product P of the first m-1 factors, and of the last factor
  std::vector<long long> rp(N + 1, 1);
  for (int j = 0; j + 1 < m; ++j)
    for (int k = 0; k <= N; ++k) rp[k] *= ys[j].rks[k];
  for (int k = 0; k <= N; ++k)
    TTC_REQUIRE(rp[k] * ys[m - 1].rks[k] < (1LL << 24), TTC_EDIM, "hadamard rounding: product rank too large");
  std::vector<int> cap;
  for (int j = 0; j < m; ++j)
    for (int k = 0; k <= N; ++k) cap.push_back((int)ys[j].rks[k]);
  BatchHolder BH;
  ttc_batch* X = BH.add(batch_create(c, m, N, dims.data(), cap.data()));
  batch_upload_many(X, 0, m, ys, false);
  const std::vector<int> rho = rand_out_ranks(dims, sp);
  ttc_batch* Y = BH.add(batch_create(c, 1, N, dims.data(), rho.data()));
  std::string rawkey;
  const auto host_raw = upload_host_blocks(c, dims, sp, sk.sketch_blocks, rawkey);
  const int bt = m - 1;                       // the factor kept separate
  auto rB = [&](int k) { return X->rk(bt, k); };
  auto rP = [&](int k) { return (int)rp[k]; };

  run_plan_once(c, [&](Builder& B) {
    B.stage(0);
    emit_zero_tts(B, Y, {0});
    emit_set_ranks(B, Y, {0}, {rho});
    // P = factor 0 (m == 2), or the multiplied-out product of factors 0..m-2, packed (rP_k, n, rP_{k+1})
    std::vector<const double*> Pc(N);
    std::vector<int> pcap(N);
    if (m == 2) {
      for (int k = 0; k < N; ++k) { Pc[k] = X->core(0, k); pcap[k] = X->capr(0, k); }
    } else {
      std::vector<const double*> cur(N);
      std::vector<long long> rc(N + 1);
      std::vector<int> ccap(N);
      for (int k = 0; k < N; ++k) { cur[k] = X->core(0, k); ccap[k] = X->capr(0, k); }
      for (int k = 0; k <= N; ++k) rc[k] = X->rk(0, k);
      for (int j = 1; j + 1 < m; ++j) {
        std::vector<GemmDesc> g;
        std::vector<const double*> nxt(N);
        for (int k = 0; k < N; ++k) {
          const int n = (int)dims[k];
          const long long L = rc[k] * X->rk(j, k), R = rc[k + 1] * X->rk(j, k + 1);
          double* C = B.wd((size_t)(L * n * R));
          g.push_back(kron_core(cur[k], (int)rc[k], (int)rc[k + 1], ccap[k], X->core(j, k), X->rk(j, k),
                                X->rk(j, k + 1), X->capr(j, k), n, C, L, L * n));
          nxt[k] = C;
        }
        B.gemm(g);
        for (int k = 0; k < N; ++k) { cur[k] = nxt[k]; ccap[k] = (int)(rc[k] * X->rk(j, k)); }
        for (int k = 0; k <= N; ++k) rc[k] *= X->rk(j, k);
      }
      for (int k = 0; k < N; ++k) { Pc[k] = cur[k]; pcap[k] = ccap[k]; }
    }
    // sketch blocks in the Julia layout (b_{k+1}, n, b_k, p_k)
    std::vector<double*> raw(N);
    if (!host_raw.empty()) {
      for (int k = 0; k < N; ++k) raw[k] = const_cast<double*>(host_raw[k]);
    } else {
      std::vector<BlockShape> sh(N);
      for (int k = 0; k < N; ++k) sh[k] = {sp.b[k + 1], (int)dims[k], sp.b[k], sp.p[k]};
      emit_block_draws(B, sh, sk, raw);
    }
    B.stage(1);
    // reverse Kronecker sketch: W[k] ((rP_k rB_k), b_k, p_k), unscaled; W[N] = 1
    std::vector<double*> W(N + 1);
    W[N] = B.ctx->d_one;
    for (int k = 0; k < N; ++k) W[k] = B.wd((size_t)rP(k) * rB(k) * sp.b[k] * sp.p[k]);
    for (int k = N - 1; k >= 0; --k) {
      const size_t mk = B.mark();
      const int n = (int)dims[k], bl = sp.b[k + 1], br = sp.b[k], pk = sp.p[k];
      const int a0 = rP(k), a1 = rP(k + 1), b0 = rB(k), b1 = rB(k + 1);
      const int cb = X->capr(bt, k);
      const long long R1 = (long long)a1 * b1;
      double* T1 = B.wd((size_t)(R1 * n * br * pk));
      double* T2 = B.wd((size_t)((long long)a0 * b1 * n * br * pk));
      // T1[(al, be), (z, c), j] = sum_ga W_{k+1}[(al, be), ga, j'] S[ga, (z, c), j]
      GemmDesc d1 = gd((int)R1, n * br, bl, W[k + 1], 1, R1, raw[k], 1, bl, T1, 1, R1);
      d1.batch = pk;
      d1.a_b = (k < N - 1) ? R1 * bl : 0;
      d1.b_b = (long long)bl * n * br;
      d1.c_b = R1 * n * br;
      B.gemm({d1});
      // T2[a, be, z, (c, j)] = sum_al P_k[a, z, al] T1[al, be, z, (c, j)]   (one problem per z)
      GemmDesc d2{};
      d2.m = a0; d2.n = b1 * br * pk; d2.k = a1; d2.batch = n;
      d2.m0 = a0; d2.n0 = b1; d2.k0e = a1;
      d2.A = Pc[k]; d2.a_i0 = 1; d2.a_k0 = (long long)pcap[k] * n; d2.a_b = pcap[k];
      d2.B = T1; d2.b_k0 = 1; d2.b_j0 = a1; d2.b_j1 = R1 * n; d2.b_b = R1;
      d2.C = T2; d2.c_i0 = 1; d2.c_j0 = a0; d2.c_j1 = (long long)a0 * b1 * n; d2.c_b = (long long)a0 * b1;
      d2.alpha = 1.0; d2.beta = 0.0;
      B.gemm({d2});
      // W_k[(a, b), (c, j)] = sum_{be, z} T2[a, be, z, (c, j)] B_k[b, z, be]   (one problem per (c, j))
      GemmDesc d3{};
      d3.m = a0; d3.n = b0; d3.k = b1 * n; d3.batch = br * pk;
      d3.m0 = a0; d3.n0 = b0; d3.k0e = b1;
      d3.A = T2; d3.a_i0 = 1; d3.a_k0 = a0; d3.a_k1 = (long long)a0 * b1; d3.a_b = (long long)a0 * b1 * n;
      d3.B = X->core(bt, k); d3.b_k0 = (long long)cb * n; d3.b_k1 = cb; d3.b_j0 = 1;
      d3.b_b = 0;
      d3.C = W[k]; d3.c_i0 = 1; d3.c_j0 = a0; d3.c_b = (long long)a0 * b0;
      d3.alpha = 1.0; d3.beta = 0.0;
      B.gemm({d3});
      B.release(mk);
    }
    B.stage(2);
    // range finder and projection sweep; y_k is (rho_k, n, (a, b)) packed
    size_t ymax = 1;
    for (int k = 0; k < N; ++k) ymax = std::max(ymax, (size_t)rho[k] * (size_t)dims[k] * (size_t)rP(k + 1) * (size_t)rB(k + 1));
    double* Yc = B.wd(ymax);
    double* Yn = B.wd(ymax);
    {  // y_0[0, z, (al, be)] = P_0[0, z, al] B_0[0, z, be]
      const int n = (int)dims[0];
      B.gemm({kron_core(Pc[0], 1, rP(1), pcap[0], X->core(bt, 0), 1, rB(1), X->capr(bt, 0), n, Yc, 1, n)});
    }
    for (int k = 0; k + 1 < N; ++k) {
      const size_t mk = B.mark();
      const int n = (int)dims[k], nn = (int)dims[k + 1];
      const int rh = rho[k], rhn = rho[k + 1], s = sp.s[k + 1];
      const long long R = (long long)rP(k + 1) * rB(k + 1);
      const double ws = 1.0 / std::sqrt((double)sp.p[k + 1]);
      double* Z = B.wd((size_t)rh * n * s);
      double* Q = B.wd((size_t)rh * n * rhn);
      double* Tws = B.wd(qr_tws_h(rh * n, s));
      B.gemm({gd(rh * n, s, (int)R, Yc, 1, (long long)rh * n, W[k + 1], 1, R, Z, 1, (long long)rh * n, ws)});
      B.qr({{rh * n, s, Z, rh * n, Q, rh * n, nullptr, 0, Tws}});
      const int yc = Y->capr(0, k);
      B.copy({cd3(Q, Y->core(0, k), rh, n, rhn, 1, rh, (long long)rh * n, 1, yc, (long long)yc * n)});
      // Qy[(l1, l2), rho'] = sum_{rho, z} y_k[rho, z, (l1, l2)] Q[rho, z, rho']
      double* Qy = B.wd((size_t)(R * rhn));
      B.gemm({gd((int)R, rhn, rh * n, Yc, (long long)rh * n, 1, Q, 1, (long long)rh * n, Qy, 1, R)});
      const int p0 = rP(k + 1), p1 = rP(k + 2), q0 = rB(k + 1), q1 = rB(k + 2);
      const int pc = pcap[k + 1], bc = X->capr(bt, k + 1);
      // V[L, (l2, rho'), z] = sum_l1 P_{k+1}[l1, z, L] Qy[l1, (l2, rho')]   (one problem per z)
      double* V = B.wd((size_t)p1 * q0 * rhn * nn);
      GemmDesc va = gd(p1, q0 * rhn, p0, Pc[k + 1], (long long)pc * nn, 1, Qy, 1, p0, V, 1, p1);
      va.batch = nn; va.a_b = pc; va.b_b = 0; va.c_b = (long long)p1 * q0 * rhn;
      // y_{k+1}[rho', z, (L, L2)] = sum_l2 V[L, l2, rho', z] B_{k+1}[l2, z, L2]   (one problem per z;
      // rows (L, rho') with L fastest)
      GemmDesc vb{};
      vb.m = p1 * rhn; vb.n = q1; vb.k = q0; vb.batch = nn;
      vb.m0 = p1; vb.n0 = q1; vb.k0e = q0;
      vb.A = V; vb.a_i0 = 1; vb.a_i1 = (long long)p1 * q0; vb.a_k0 = p1; vb.a_b = (long long)p1 * q0 * rhn;
      vb.B = X->core(bt, k + 1); vb.b_k0 = 1; vb.b_j0 = (long long)bc * nn; vb.b_b = bc;
      vb.C = Yn; vb.c_i0 = (long long)rhn * nn; vb.c_i1 = 1; vb.c_j0 = (long long)rhn * nn * p1; vb.c_b = rhn;
      vb.alpha = 1.0; vb.beta = 0.0;
      B.gemm({va});
      B.gemm({vb});
      std::swap(Yc, Yn);
      B.release(mk);
    }
    {  // last core: y_{N-1} (rho, n, 1)
      const int rh = rho[N - 1], n = (int)dims[N - 1], yc = Y->capr(0, N - 1);
      B.copy({cd3(Yc, Y->core(0, N - 1), rh, n, 1, 1, rh, (long long)rh * n, 1, yc, (long long)yc * n)});
    }
    B.stage(3);
  });
  for (int k = 0; k < N; ++k) Y->h_ot[k] = (k < N - 1) ? 1 : 0;
  for (int k = 0; k <= N; ++k) Y->h_rks[k] = rho[k];
  Y->rks_dirty = false;
  batch_download_many(Y, 0, 1, y, false);
}

}  // namespace ttc
